import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def _ensure_built():
    lib = os.path.join(ROOT, "bml_b200", "libbml_b200.so")
    if not os.path.exists(lib):
        # load build.py on its own: importing the package needs the library
        import importlib.util
        spec = importlib.util.spec_from_file_location("bml_b200_build",
                                                      os.path.join(ROOT, "bml_b200", "build.py"))
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
        mod.build()
    ora = os.path.join(ROOT, "oracle", "_ref", "libbml_oracle.so")
    if not os.path.exists(ora):
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "oracle"], check=True,
                       capture_output=True)


_ensure_built()


@pytest.fixture(scope="session")
def oracle_mod():
    from oracle import oracle
    if not oracle.available():
        pytest.skip("oracle/_ref not built (make -C oracle needs the reference sources)")
    return oracle

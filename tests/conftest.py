import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    config.addinivalue_line("markers", "unordered: runs the ELLPACK products in the unordered form "
                                       "(GPU tests default to the ordered, bit-identical form)")


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


@pytest.fixture(autouse=True)
def _ellpack_product_form(request):
    """GPU tests that compare bit for bit run the ordered products; tests
    marked `unordered` run the unordered (default) form."""
    if request.node.get_closest_marker("gpu") is None:
        yield
        return
    import bml_b200 as B
    old = B.lib.bml_b200_set_x2_exact(0 if request.node.get_closest_marker("unordered") else 1)
    yield
    B.lib.bml_b200_set_x2_exact(old)

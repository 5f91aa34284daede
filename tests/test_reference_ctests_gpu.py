"""The reference's own C test driver (tests/C-tests/bml_test.c with the
test sources of the operations on this library's path), compiled with gcc
against the reference's headers and linked to libbml_b200.so in place of
libbml by oracle/Makefile (target ctest).  A C caller built against bml.h,
struct layouts and enums included, runs unchanged: each test must exit 0,
as it does under the reference's CTest (tests/C-tests/CMakeLists.txt,
bml-test -n TEST -t TYPE -p PRECISION, default N = 13, M = N)."""
import os
import subprocess

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "oracle", "_ref", "bml-test-b200")

TESTS = ["add", "allocate", "convert", "copy", "get_element", "get_set_diagonal", "get_sparsity",
         "import_export", "introspection", "io_matrix", "multiply", "multiply_banded", "multiply_x2",
         "normalize", "print", "scale", "set_element", "set_row", "threshold", "trace", "trace_mult",
         "transpose"]


@pytest.fixture(scope="module")
def exe():
    if not os.path.exists(EXE):
        pytest.skip("oracle/_ref/bml-test-b200 is not built (make -C oracle ctest needs the reference's tests)")
    return EXE


@pytest.mark.parametrize("prec", ["single_real", "double_real"])
@pytest.mark.parametrize("mtype", ["ellpack", "ellblock"])
@pytest.mark.parametrize("test", TESTS)
def test_reference_c_test(exe, test, mtype, prec, tmp_path):
    r = subprocess.run([exe, "-n", test, "-t", mtype, "-p", prec], cwd=tmp_path, capture_output=True,
                       text=True, timeout=120)
    assert r.returncode == 0, "%s %s %s exited %d:\n%s\n%s" % (test, mtype, prec, r.returncode,
                                                                r.stdout[-2000:], r.stderr[-2000:])


@pytest.mark.parametrize("test", ["multiply_x2", "multiply", "add", "threshold", "trace", "transpose"])
@pytest.mark.parametrize("mtype", ["ellpack", "ellblock"])
def test_reference_c_test_larger_N(exe, test, mtype, tmp_path):
    """The same tests on 301 x 301 matrices (the driver's -N)."""
    r = subprocess.run([exe, "-n", test, "-t", mtype, "-p", "double_real", "-N", "301"], cwd=tmp_path,
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, "%s %s exited %d:\n%s" % (test, mtype, r.returncode, r.stderr[-2000:])

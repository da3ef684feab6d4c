"""Step hooks compile without a device (NVRTC for sm_100a), and compiler
errors come back as PS_ERR_COMPILE with the compiler's log naming the file,
as PyCUDA's SourceModule reports them when the reference builds its kernels
(pysweep/core/io.py:146-155)."""
import os

import pytest

HOOKS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "hooks")


@pytest.mark.parametrize("name,nv,ops,its", [
    ("heat_numpy_order.cu", 1, 1, 2), ("half_numpy_order.cu", 1, 1, 2),
    ("example_numpy_order.cu", 3, 2, 1), ("checker_numpy_order.cu", 1, 2, 2),
    ("wave4.cu", 2, 2, 2)])
def test_hook_files_compile(name, nv, ops, its):
    from pysweep_b200 import check_hook
    check_hook(os.path.join(HOOKS, name), nv, ops, its)


def test_compile_error_reports_the_log():
    from pysweep_b200 import PySweepError, check_hook
    src = "__device__ void step(double* s, int idx, int g)\n{\n  s[idx + TIMES] = missing(s);\n}\n"
    with pytest.raises(PySweepError) as err:
        check_hook(src, name="mine.cu")
    assert err.value.code == -6
    assert "mine.cu(3)" in str(err.value) and "missing" in str(err.value)


REF = os.environ.get("PYSWEEP_REFERENCE_HOOKS", "")


@pytest.mark.skipif(not os.path.isdir(REF), reason="PYSWEEP_REFERENCE_HOOKS not set")
@pytest.mark.parametrize("name,nv,ops,its", [
    ("heat.cu", 1, 1, 1), ("euler.cu", 4, 2, 2), ("example.cu", 1, 1, 2),
    ("checker.cu", 1, 1, 1), ("half.cu", 1, 1, 2)])
def test_reference_plugin_hooks_compile_unmodified(name, nv, ops, its):
    """The reference's own plugin .cu files (given by PYSWEEP_REFERENCE_HOOKS;
    they are not part of this repository), as they are."""
    from pysweep_b200 import check_hook
    check_hook(os.path.join(REF, name), nv, ops, its)

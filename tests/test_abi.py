"""CPU-side checks of the drop-in boundary: the library builds, loads, exports
exactly what include/linompss_b200.h declares, and rejects bad arguments
before touching a device."""
import ctypes as C
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "linompss_b200.h")


def declared_symbols():
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"LNB_EXPORT\s+[\w\s\*]+?\b(\w+)\s*\(", txt)))


@pytest.fixture(scope="module")
def lnb():
    import linompss_b200
    if not os.path.exists(linompss_b200.LIB_PATH):
        subprocess.check_call(["make", "-s", "-C", os.path.join(ROOT, "linompss_b200", "csrc")])
    return linompss_b200


def test_header_declares_reference_entry_points():
    syms = declared_symbols()
    for name in ["ompss_dchol_rl", "ompss_dchol_ll", "ompss_dchol_hrl", "ompss_dchol_hll",
                 "ompss_dchol_nhrl", "ompss_dchol_nhll", "ompss_schol_rl", "dspdsolv_main",
                 "ompss_dtrsm", "task_dpotrf", "task_dtrsm", "task_dsyrk", "task_dgemm",
                 "ompss_dcg", "ompss_ditref"]:
        assert name in syms


def test_library_exports_every_declared_symbol(lnb):
    lib = C.CDLL(lnb.LIB_PATH)
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing


def test_library_exports_nothing_else(lnb):
    out = subprocess.check_output(["nm", "-D", "--defined-only", lnb.LIB_PATH]).decode()
    exported = {line.split()[-1] for line in out.splitlines() if " T " in line}
    assert exported == set(declared_symbols())


def test_build_targets_sm100a_only():
    mk = open(os.path.join(ROOT, "linompss_b200", "csrc", "Makefile")).read()
    assert re.findall(r"arch=compute_\w+,code=\w+", mk) == ["arch=compute_100a,code=sm_100a"]


def test_version_and_error_string(lnb):
    assert "sm_100a" in lnb.version()
    assert isinstance(lnb.last_error(), str)


def test_argument_errors_are_reported_without_a_device(lnb):
    import numpy as np
    A = np.zeros((4, 4), order="F")
    with pytest.raises(lnb.LinompssError) as e:
        lnb.ompss_dchol_rl(4, 0, 0, A, 4)  # tile size 0
    assert e.value.code == lnb.LNB_EINVAL
    with pytest.raises(lnb.LinompssError) as e:
        lnb.ompss_dchol_rl(4, 2, 0, A, 3)  # lda < n
    assert e.value.code == lnb.LNB_EINVAL
    with pytest.raises(lnb.LinompssError) as e:
        lnb.ompss_dtrsm("R", "L", "N", "N", 4, 4, 2, 1.0, A, 4, A, 4)  # right side: not in the reference
    assert e.value.code == lnb.LNB_EINVAL
    # n = 0 is a no-op returning 0, as in the reference
    assert lnb.ompss_dchol_rl(0, 2, 0, A, 1) == 0


def test_no_device_is_loud(lnb):
    """Without a GPU the entry points fail with LNB_ENODEV; nothing computes on the CPU."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    import numpy as np
    A = np.asfortranarray(np.eye(8))
    with pytest.raises(lnb.LinompssError) as e:
        lnb.ompss_dchol_rl(8, 4, 4, A, 8)
    assert e.value.code == lnb.LNB_ENODEV
    np.testing.assert_array_equal(A, np.eye(8))

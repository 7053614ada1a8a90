"""The C ABI library builds for sm_100a, loads, and exports every function include/dopamine_b200.h
declares (no compute calls: this runs without a GPU)."""
import ctypes as C
import os
import re

from dopamine_b200 import solver as S

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    src = open(os.path.join(ROOT, "include", "dopamine_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:int|void|double|const\s+char)\s*\**\s*((?:fvm_petsc|dpm)_\w+)\s*\(", src, flags=re.M)))


def test_header_declares_both_groups():
    names = declared_functions()
    assert "fvm_petsc_solve_pressure" in names and "dpm_advance" in names
    assert len(names) >= 30


def test_library_exports_every_declared_symbol():
    lib = S.lib()
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing
    assert set(S.EXPORTED) <= set(declared_functions())


def test_library_is_sm100a_only():
    # the fatbin carries sm_100a SASS only (cuobjdump is not used; the build flags are checked)
    from dopamine_b200 import build
    assert build.ARCH == ["-gencode", "arch=compute_100a,code=sm_100a"]
    assert os.path.getsize(S.LIB_PATH) > 100000

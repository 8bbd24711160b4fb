"""The CUDA library loads without a GPU and exports every function include/gbght.h declares."""
import ctypes
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    text = open(os.path.join(ROOT, "include", "gbght.h")).read()
    return sorted(set(re.findall(r"^\s*(?:const\s+)?(?:int|void|char\s*\*|const char\s*\*)\s*\*?\s*(gbght_\w+)\s*\(",
                                  text, re.M)))


def test_header_declares_the_boundary():
    names = declared_functions()
    for must in ("gbght_create", "gbght_step", "gbght_deposit", "gbght_advect", "gbght_advance",
                 "gbght_state_import", "gbght_state_export", "gbght_observables", "gbght_spectrum"):
        assert must in names


def test_library_exports_every_declared_symbol(cuda_library):
    lib = ctypes.CDLL(cuda_library)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_library_reports_its_version(cuda_library):
    lib = ctypes.CDLL(cuda_library)
    lib.gbght_version.restype = ctypes.c_char_p
    assert lib.gbght_version().startswith(b"gbght-b200")

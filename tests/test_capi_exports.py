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


def test_config_layout_matches_the_header(cuda_library):
    # gbght_config_default fills the ctypes mirror of gbght_config: every default lands in its
    # own field, so the mirror's offsets agree with the C struct, the forcing blocks included.
    import math
    import gbght
    lib = gbght.load_library(cuda_library)
    cfg = gbght.Config()
    lib.gbght_config_default(ctypes.byref(cfg))
    assert (cfg.grid_points_per_axis, cfg.precision, cfg.scheme, cfg.scalar) == (64, 0, 0, 1)
    assert cfg.side_length == 2 * math.pi and cfg.viscosity == 0.01 and cfg.schmidt == 1.0
    for f in (cfg.velocity_forcing, cfg.scalar_forcing):
        assert (f.kind, f.rate, f.target, f.gain, f.turnover_time, f.over) == (0, 0.0, 0.0, 1.0, 0.0, 0)
        assert (f.lowest_shell, f.highest_shell) == (1, 2.0)
    assert tuple(cfg.mean_gradient) == (0.0, 0.0, 0.0) and cfg.tracers == 0
    assert cfg.cfl == 0.5 and cfg.max_dt == math.inf and cfg.device == 0

"""The allocation-free velocity recovery against the regular deposit, through the C ABI.

gbght_velocity_physical_noalloc serves callers that cannot allocate device memory: one whose
memory is owned by another allocator (a framework's caching pool that holds the GPU), or a loop
that keeps the rule of no field-scale allocation inside a step. It keeps every intermediate in
one static device array. Here the caller's buffers are torch tensors (the caller's allocator, not
the library's). Two calls in a row, on different spectra, must each match what gbght_deposit +
gbght_velocity_physical_export give for the same spectrum: a stale scratch array would show up
on the second call. Every grid the array admits is covered (their radix plans 8, 2·3·2, 4·4,
2·3·2·2, 4·8, 4·3·4 and 8·8; N = 64 fills most of the array), and a sequence that changes the grid
back and forth checks that the per-grid set-up kept between calls (tensor maps, twiddles) follows
the grid.
"""
import ctypes

import numpy as np
import pytest

import gbght
from gbght import seed as S

pytestmark = pytest.mark.gpu

TOL = 1e-12
SIZES = (8, 12, 16, 24, 32, 48, 64)


def _regular(lib_path, N, uh):
    run = gbght.Run(gbght.Setup(grid_points_per_axis=N, scalar=False), library=lib_path)
    run.import_state(uh)
    run.deposit()
    u, m = run.velocity_physical(), run.max_speed()
    run.close()
    return u, m


def _entry(lib_path):
    lib = ctypes.CDLL(lib_path)
    fn = lib.gbght_velocity_physical_noalloc
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_void_p, ctypes.c_void_p,
                   ctypes.POINTER(ctypes.c_double), ctypes.c_void_p]
    lib.gbght_global_error.restype = ctypes.c_char_p
    return lib, fn


def _call_and_check(lib, fn, lib_path, N, seed, energy):
    import torch

    uh = S.seed_velocity(N, energy, seed=seed)
    u_ref, m_ref = _regular(lib_path, N, uh)
    d_uh = torch.from_numpy(uh.view(np.float64).copy()).cuda()
    d_u = torch.full((3, N, N, N), float("nan"), dtype=torch.float64, device="cuda")
    m = ctypes.c_double(-1.0)
    stream = torch.cuda.current_stream()
    torch.cuda.synchronize()
    rc = fn(N, 2 * np.pi, d_uh.data_ptr(), d_u.data_ptr(), ctypes.byref(m), stream.cuda_stream)
    assert rc == 0, lib.gbght_global_error().decode()
    torch.cuda.synchronize()
    u = d_u.cpu().numpy()
    err = np.linalg.norm(u - u_ref) / np.linalg.norm(u_ref)
    assert err <= TOL, (N, seed, err)
    assert m.value == pytest.approx(m_ref, rel=TOL)


@pytest.mark.parametrize("N", SIZES)
def test_noalloc_velocity_matches_the_regular_deposit(cuda_library, N):
    lib, fn = _entry(cuda_library)
    for call, seed in enumerate((11, 12)):
        _call_and_check(lib, fn, cuda_library, N, seed, 0.5 + 0.25 * call)


def test_noalloc_follows_grid_changes(cuda_library):
    lib, fn = _entry(cuda_library)
    for k, N in enumerate((64, 32, 64, 12, 12, 48, 8, 64)):
        _call_and_check(lib, fn, cuda_library, N, 20 + k, 0.5)


def test_noalloc_refuses_grids_beyond_its_array(cuda_library):
    lib, fn = _entry(cuda_library)
    rc = fn(128, 2 * np.pi, ctypes.c_void_p(16), ctypes.c_void_p(16), None, None)
    assert rc == gbght.ERR_ARGUMENT
    assert b"at most 64" in lib.gbght_global_error()

"""Host-side seeding of spectral states and tracer positions.

The reference draws its seeds on the host so that one seed gives the same field on every backend
(src/State.jl:164-172; src/Particles.jl:152-158). This module follows that rule with NumPy's PCG64
stream. The reference's Julia MersenneTwister streams cannot be reproduced here.

The spectrum is the k⁴ form the benchmark configurations name:
E(k) ∝ k⁴ exp(−2(k/4)²), with uniform random phases. The reference's own seeder uses a Gaussian
envelope instead (src/State.jl:206-234). Every retained mode gets amplitude
√(E(|κ|)/(4π|κ|²)) and a phase drawn from the seed. The kx = 0 plane is completed Hermitian
(f̂(0,−ky,−kz) = conj f̂(0,ky,kz)). The velocity is then Leray-projected, and both fields are cut
to the 2/3 closed ball and rescaled, to kinetic energy ½⟨|u|²⟩ or to variance ⟨φ²⟩. The arrays
are in the reference's spectral layout [comp][kz][ky][kx], complex128, kx ∈ [0, N/2].
"""
from __future__ import annotations

import math

import numpy as np


def _axis_integers(N):
    return np.fft.fftfreq(N, d=1.0 / N).round().astype(np.int64)


def wavenumbers(N: int, L: float = 2 * math.pi):
    s = 2 * math.pi / L
    kx = (s * np.arange(N // 2 + 1, dtype=np.float64))[None, None, :]
    ky = (s * _axis_integers(N).astype(np.float64))[None, :, None]
    kz = (s * _axis_integers(N).astype(np.float64))[:, None, None]
    k2 = (kx * kx + ky * ky) + kz * kz
    return kx, ky, kz, k2


def retained_mask(N: int, L: float = 2 * math.pi):
    """The 2/3 closed ball: |κ|² ≤ (T(2/3)·T(N/2)·T(2π/L))² (src/SimulationDomain.jl:342-363)."""
    _, _, _, k2 = wavenumbers(N, L)
    cutoff = (2 / 3) * (N / 2) * (2 * math.pi / L)
    return k2 <= cutoff * cutoff


def _hermitian_complete(fh: np.ndarray) -> np.ndarray:
    """Complete the kx = 0 plane (and kx = N/2 for even N) so f̂(−ky,−kz) = conj f̂(ky,kz). Of
    each pair the member with the smaller flat index (kz·N + ky) keeps its draw. Self-conjugate
    modes keep their real part."""
    N = fh.shape[-2]
    out = fh.copy()
    neg = (-np.arange(N)) % N
    q = np.arange(N)[:, None] * N + np.arange(N)[None, :]           # flat index [kz][ky]
    qp = neg[:, None] * N + neg[None, :]
    keep = q <= qp
    for p in [0] + ([N // 2] if N % 2 == 0 else []):
        plane = out[..., p]
        flipped = np.conj(plane[..., neg, :][..., :, neg])
        plane = np.where(keep, plane, flipped)
        selfc = q == qp
        plane = np.where(selfc, plane.real + 0j, plane)
        out[..., p] = plane
    return out


def _inner(fh, gh, N):
    w = np.full(N // 2 + 1, 2.0)
    w[0] = 1.0
    if N % 2 == 0:
        w[N // 2] = 1.0
    return float(((np.conj(fh) * gh).real * w).sum()) / float(N) ** 6


def _amplitude(N, L):
    _, _, _, k2 = wavenumbers(N, L)
    k = np.sqrt(k2)
    E = k2 * k2 * np.exp(-2.0 * (k / 4.0) ** 2)
    with np.errstate(divide="ignore", invalid="ignore"):
        amp = np.sqrt(np.where(k2 > 0, E / (4 * math.pi * k2), 0.0))
    return amp


def seed_velocity(N: int, kinetic_energy: float = 0.5, seed: int = 0, L: float = 2 * math.pi):
    """A random solenoidal, band-limited velocity with the k⁴ seed spectrum, rescaled to
    ½⟨|u|²⟩ = kinetic_energy. Returns (3, N, N, N/2+1) complex128."""
    rng = np.random.default_rng(seed)
    theta = rng.random((3, N, N, N // 2 + 1)) * (2 * math.pi)
    amp = _amplitude(N, L)
    uh = amp[None] * np.exp(1j * theta)
    uh = _hermitian_complete(uh)
    kx, ky, kz, k2 = wavenumbers(N, L)
    safe = np.where(k2 > 0, k2, 1.0)
    kdotu = (kx * uh[0] + ky * uh[1]) + kz * uh[2]
    coef = np.where(k2 > 0, kdotu / safe, 0.0)
    uh = np.stack([uh[0] - kx * coef, uh[1] - ky * coef, uh[2] - kz * coef])
    uh = uh * retained_mask(N, L)[None]
    uh[:, 0, 0, 0] = 0.0
    energy = _inner(uh, uh, N) / 2
    if not energy > 0:
        raise ValueError("the seeded velocity has no energy to rescale")
    return uh * math.sqrt(kinetic_energy / energy)


def seed_scalar(N: int, variance: float = 0.5, seed: int = 1, L: float = 2 * math.pi):
    """A random mean-zero band-limited scalar with the k⁴ seed spectrum, rescaled to
    ⟨φ²⟩ = variance. Returns (N, N, N/2+1) complex128."""
    rng = np.random.default_rng(seed)
    theta = rng.random((N, N, N // 2 + 1)) * (2 * math.pi)
    ph = _amplitude(N, L) * np.exp(1j * theta)
    ph = _hermitian_complete(ph)
    ph = ph * retained_mask(N, L)
    ph[0, 0, 0] = 0.0
    var = _inner(ph, ph, N)
    if not var > 0:
        raise ValueError("the seeded scalar has no variance to rescale")
    return ph * math.sqrt(variance / var)


def seed_tracers(M: int, seed: int = 2, L: float = 2 * math.pi):
    """M uniform-random positions in [0, L)³, as (3, M) float64 (the SoA form of the reference's
    column-major (M, 3) array)."""
    rng = np.random.default_rng(seed)
    return rng.random((3, M)) * L

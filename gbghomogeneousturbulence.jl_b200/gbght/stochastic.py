"""The Ornstein–Uhlenbeck process of a StochasticOU forcing, on the host.

The reference (`StochasticOU`, src/Forcing.jl:1224-1415) keeps the force as a field on a coarse
companion grid of Nc = 2·(highest_shell + 1) points per axis over the same box, and advances it
once per step (`prepare_forcing!`, :1401-1411) by one exact OU transition
a ← α a + scale·√(σ²(1 − α²))·ξ̂, α = exp(−Δt/T_L), with ξ a real Gaussian field drawn on the host
(`_advance_process!`, :1362-1375): transformed, cut to the band, projected transverse to κ for the
velocity, and scaled so that its expected box mean square is 1 (scale = 1/√(retained/Nc³), retained
= 2M for the velocity and M for the scalar, M the band's lattice modes counted over the whole
spectrum, :1283-1294). The first draw (α = 0) starts the process stationary (:1378-1382). The
force is added to the field's right-hand side at every stage of the step
(`add_forcing_source!`, :1415), where the run's modes and the companion's coincide.

Here the amplitudes are physical: a_k is the coefficient of e^{iκ·x} (the companion's rfft divided
by Nc³), in the companion's reference layout (complex128, [comp][kz][ky][kx], kx ≤ Nc/2); the
library adds N³·a_k, the run's unnormalised coefficient, to N̂ on the band. The draws come from
NumPy's PCG64 seeded with (seed, draw count, field order), so the stream is a pure function of the
three, as the reference's key (`_draw_key`, :1356-1358) makes it; the reference's Julia Xoshiro
stream itself cannot be reproduced here, so a realisation matches the reference's in law, not
draw for draw.
"""
from __future__ import annotations

import math

import numpy as np


def companion_size(highest_shell: int) -> int:
    """Nc = 2·(highest_shell + 1): even, with the band strictly below its Nyquist wavenumber."""
    return 2 * (int(highest_shell) + 1)


def _wavenumbers(n: int, L: float):
    k0 = 2 * math.pi / L
    m = np.fft.fftfreq(n, d=1.0 / n).round()
    kx = (k0 * np.arange(n // 2 + 1))[None, None, :]
    ky = (k0 * m)[None, :, None]
    kz = (k0 * m)[:, None, None]
    return kx, ky, kz


def band_mask(n: int, L: float, lowest_shell: int, highest_shell: int) -> np.ndarray:
    """The shells lowest..highest on the companion's half spectrum, [(h − ½)k0, (h + ½)k0] on the
    squares, edges included."""
    kx, ky, kz = _wavenumbers(n, L)
    k0 = 2 * math.pi / L
    lo, hi = (lowest_shell - 0.5) * k0, (highest_shell + 0.5) * k0
    k2 = (kx * kx + ky * ky) + kz * kz
    return ((k2 >= lo * lo) & (k2 <= hi * hi)).astype(np.float64)


def band_modes(n: int, L: float, lowest_shell: int, highest_shell: int) -> int:
    """M: the band's lattice wavevectors over the whole companion spectrum, both members of every
    pair (`_count_band_modes`, src/Forcing.jl:1287-1294)."""
    k0 = 2 * math.pi / L
    lo, hi = (lowest_shell - 0.5) * k0, (highest_shell + 0.5) * k0
    r = np.arange(-(n // 2), n // 2)
    i, j, k = np.meshgrid(r, r, r, indexing="ij")
    mod = k0 * np.sqrt(i * i + j * j + k * k)
    return int(np.count_nonzero((mod >= lo) & (mod <= hi)))


class OUProcess:
    """The force of one field: `vector` for the velocity (3 components, transverse), else the
    scalar's."""

    def __init__(self, forcing_variance: float, correlation_time: float, lowest_shell: int, highest_shell: int,
                 seed: int, vector: bool, L: float = 2 * math.pi):
        if not (math.isfinite(forcing_variance) and forcing_variance >= 0):
            raise ValueError(f"`forcing_variance` must be finite and non-negative, got {forcing_variance}")
        if not (math.isfinite(correlation_time) and correlation_time > 0):
            raise ValueError(f"`correlation_time` must be finite and positive, got {correlation_time}")
        if not math.isfinite(highest_shell):
            raise ValueError("StochasticOU needs a finite `highest_shell`, got Inf: it adds its process "
                             "rather than multiplying the field")
        self.sigma2, self.tl = float(forcing_variance), float(correlation_time)
        self.lo, self.hi, self.seed, self.vector, self.L = int(lowest_shell), int(highest_shell), int(seed), vector, L
        self.n = companion_size(highest_shell)
        self.band = band_mask(self.n, L, self.lo, self.hi)
        M = band_modes(self.n, L, self.lo, self.hi)
        if M == 0:
            raise ValueError("the band holds no lattice wavevector, so the forcing would drive nothing")
        retained = 2 * M if vector else M
        self.scale = 1.0 / math.sqrt(retained / float(self.n) ** 3)
        shape = (3, self.n, self.n, self.n // 2 + 1) if vector else (self.n, self.n, self.n // 2 + 1)
        self.amplitudes = np.zeros(shape, np.complex128)
        self.draws = 0
        self.advance(None)   # the stationary start

    def _draw(self) -> np.ndarray:
        order = 1 if self.vector else 0
        rng = np.random.Generator(np.random.PCG64([self.seed & 0xFFFFFFFFFFFFFFFF, self.draws, order]))
        n = self.n
        xi = rng.standard_normal((3, n, n, n) if self.vector else (n, n, n))
        xh = np.fft.rfftn(xi, axes=(-3, -2, -1)) / float(n) ** 3 * self.band
        if self.vector:   # transverse to κ
            kx, ky, kz = _wavenumbers(n, self.L)
            k2 = (kx * kx + ky * ky) + kz * kz
            kd = np.where(k2 > 0, (kx * xh[0] + ky * xh[1] + kz * xh[2]) / np.where(k2 > 0, k2, 1.0), 0.0)
            xh = np.stack([xh[0] - kx * kd, xh[1] - ky * kd, xh[2] - kz * kd])
        return xh

    def advance(self, dt: float | None):
        """One exact OU transition over dt (None: the stationary start, α = 0)."""
        alpha = 0.0 if dt is None else math.exp(-float(dt) / self.tl)
        xh = self._draw()
        self.amplitudes = alpha * self.amplitudes + (self.scale * math.sqrt(self.sigma2 * (1.0 - alpha * alpha))) * xh
        self.draws += 1
        return self.amplitudes

    def mean_square(self) -> float:
        """The force's box mean square Σ w|a_k|² (w the Hermitian weights), which the process keeps at
        σ² in expectation."""
        w = np.full(self.n // 2 + 1, 2.0)
        w[0] = 1.0
        w[-1] = 1.0
        return float(np.sum(np.abs(self.amplitudes) ** 2 * w))

"""CPU oracle for the GBGHomogeneousTurbulence.jl IF-RK time step.

TEST INFRASTRUCTURE ONLY. This module is the checker that the CUDA library is compared against.
Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` may import it.
No product path calls it, and nothing in the library falls back to it.

It restates, in FP64 NumPy with ``scipy.fft``, the algorithm of the reference's hot path: the
coupled velocity + passive-scalar integrating-factor low-storage Runge–Kutta step with 2/3-rule
dealiasing, Leray projection, the band forcings (ConstantPower, Linear, VarianceController,
VarianceRescaling) on either field, and Heun (ABM(1)) tracer advection with
Catmull–Rom interpolation. Every array is kept in the reference's own layout. That layout is the
column-major ``(kx, ky, kz, comp)`` array of the rfft, held here row-major as ``[comp][kz][ky][kx]``
with ``kx`` in ``[0, N/2]``. It is full-size and unpruned, so the oracle shares no layout or pruning
decision with the CUDA kernels.

Field arithmetic lives in the reference's unvendored dependency ``GBGPeriodicFields`` (uuid
``f1da9c2b-0ac1-4736-96f9-af1c25aedab1``, compat ``0.1.0``; ``Project.toml:7,17``). Its call sites in
the reference fix what each operation must compute. Where PF's own convention is not visible, this
file adopts one and says so at the function.

Parity pinning: the reference ships no golden fields. This restatement is pinned against the
reference's own known-answer tests, re-expressed in ``tests/test_oracle_known_answers.py``:
- the closed-form observables;
- exact diffusion;
- the RK3 and RK4 self-convergence ratios, and the order under ConstantPower;
- the Linear rate's exact growth of a single mode, and the Linear scalar's variance growth;
- VarianceController's amplitude, its scalar dissipation, the marginal law at gain 0 and the
  order kept; VarianceRescaling's uniform rescale on an unbounded band and its first order;
- the box-mean definition behind the energy below scale, and the skewness identities.

The tangent-linear model and discrete adjoint of the step (``step_tangent``, ``step_adjoint``)
have no counterpart in the reference, which has no AD. They are pinned by central
finite differences and by the dot-product identity ⟨Jv, w⟩ = ⟨v, Jᵀw⟩.
- injected power equal to ε, and a solenoidal state;
- the 2/3 closed ball against a 2N zero-padded product;
- PhaseShift's displaced-grid average against a 2N zero-padded product, both nonlinear terms
  (test/dealiasing.jl:69-114);
- Parseval, and the planted reality violation;
- tracer uniform flow, wrap, constant field and Heun order;
- the classical Adams weights.

The two config extensions are parity-unpinned: the k⁴ seed spectrum, defined in the package's
seeder, and the uniform mean scalar gradient G, defined here in ``scalar_rhs``.
"""
from __future__ import annotations

import math
import os
from dataclasses import dataclass, field
from fractions import Fraction

import numpy as np
import scipy.fft as sfft

WORKERS = os.cpu_count() or 1


# ---------------------------------------------------------------------------------------------
# Domain: grid, wavenumbers, the 2/3 closed-ball mask.  (src/SimulationDomain.jl:295-363)
# ---------------------------------------------------------------------------------------------

def _axis_integers(N: int) -> np.ndarray:
    """FFT-order integer wavenumbers of a full axis: 0..N/2-1, then -N/2..-1."""
    return np.fft.fftfreq(N, d=1.0 / N).round().astype(np.int64)


class Domain:
    """The fixed cubic box: `FixedDomain` (src/SimulationDomain.jl:275-328), TwoThirds dealiasing, or
    HouLi's filter, or PhaseShift's displaced-grid average on the (2√2/3)·κ_Ny ball.

    ``cutoff`` is ``T(2/3) * T(N/2) * T(2π/L)`` evaluated left to right in FP64, as
    `_cutoff_wavenumber` does (src/SimulationDomain.jl:342-343). The mask keeps the closed ball
    ``|κ|² ≤ cutoff²`` with ``|κ|² = κx² + κy² + κz²`` summed in that order
    (src/SimulationDomain.jl:349-363; closed-ball test on the squares).
    """

    def __init__(self, N: int, L: float = 2 * math.pi, dealiasing: str = "TwoThirds", houli_order: int = 36,
                 houli_strength: float | None = None):
        self.N = int(N)
        self.L = float(L)
        self.dealiasing = dealiasing
        N = self.N
        s = 2 * math.pi / self.L
        self.k0 = s
        self.cutoff = (2 / 3) * (N / 2) * s
        mx = np.arange(N // 2 + 1, dtype=np.int64)
        my = _axis_integers(N)
        mz = _axis_integers(N)
        self.kx = (s * mx.astype(np.float64))[None, None, :]
        self.ky = (s * my.astype(np.float64))[None, :, None]
        self.kz = (s * mz.astype(np.float64))[:, None, None]
        # squared wavenumber per mode, x + y + z in that order
        self.k2 = (self.kx * self.kx + self.ky * self.ky) + self.kz * self.kz
        # derivative multipliers: the Nyquist mode's derivative is zero (convention; masked anyway)
        dx = self.kx.copy()
        dy = self.ky.copy()
        dz = self.kz.copy()
        if N % 2 == 0:
            dx[..., N // 2] = 0.0
            dy[:, N // 2, :] = 0.0
            dz[N // 2, :, :] = 0.0
        self.dkx, self.dky, self.dkz = dx, dy, dz
        self.mask = (self.k2 <= self.cutoff * self.cutoff).astype(np.float64)
        if dealiasing == "HouLi":
            # Hou & Li's smooth filter in place of the 0/1 mask (`_build_dealias(::HouLi)`,
            # src/SimulationDomain.jl:365-376): exp(−strength·(|κ|/κ_Ny)^order), strength −log(eps)
            kny = (N / 2) * s
            strength = -math.log(np.finfo(np.float64).eps) if not houli_strength else float(houli_strength)
            self.cutoff = kny
            self.mask = np.exp(-strength * (np.sqrt(self.k2) / kny) ** houli_order)
        elif dealiasing == "PhaseShift":
            # the closed ball at (2√2/3)·κ_Ny = √2·N/3·κ₀ (src/SimulationDomain.jl:177-184,362), and
            # the translation to the grid displaced by half a cell along every axis: the mode of
            # integer wavenumbers (mx, my, mz) times e^{iπ(mx+my+mz)/N} (κ·δ with δ = L/(2N) per axis;
            # `to_shifted`, src/Generator.jl:169-175); `shift_back` is its conjugate
            self.cutoff = (2 * math.sqrt(2) / 3) * (N / 2) * s
            self.mask = (self.k2 <= self.cutoff * self.cutoff).astype(np.float64)
            msum = mx[None, None, :] + my[None, :, None] + mz[:, None, None]
            self.shift_to = np.exp(1j * math.pi * msum / N)
            self.shift_back = np.conj(self.shift_to)
        elif dealiasing != "TwoThirds":
            raise ValueError(f"unknown dealiasing strategy {dealiasing!r}")
        # Hermitian weights of the half spectrum: modes with 0 < kx < N/2 stand for a conjugate pair
        w = np.full(N // 2 + 1, 2.0)
        w[0] = 1.0
        if N % 2 == 0:
            w[N // 2] = 1.0
        self.hweight = w[None, None, :]
        self.dx = self.L / N
        self.shape_spectral = (N, N, N // 2 + 1)

    # transforms: unnormalised forward, 1/N³ inverse (docs/src/validation.md:72-74)
    def to_spectral(self, f: np.ndarray) -> np.ndarray:
        return sfft.rfftn(f, axes=(-3, -2, -1), workers=WORKERS)

    def to_physical(self, fh: np.ndarray) -> np.ndarray:
        N = self.N
        return sfft.irfftn(fh, s=(N, N, N), axes=(-3, -2, -1), workers=WORKERS)

    # normalised inner product: box average, via Parseval (docs/src/notation.md:19)
    def inner(self, a: np.ndarray, b: np.ndarray, weight=None) -> float:
        prod = (np.conj(a) * b).real * self.hweight
        if weight is not None:
            prod = prod * weight
        return float(prod.sum()) / float(self.N) ** 6


# ---------------------------------------------------------------------------------------------
# Spectral operators (the GBGPeriodicFields call sites listed in the module docstring).
# ---------------------------------------------------------------------------------------------

def curl(dom: Domain, uh: np.ndarray) -> np.ndarray:
    """ω̂ = iκ × û (`curl!`, src/Observables.jl:330)."""
    ux, uy, uz = uh
    return np.stack([
        1j * (dom.dky * uz - dom.dkz * uy),
        1j * (dom.dkz * ux - dom.dkx * uz),
        1j * (dom.dkx * uy - dom.dky * ux),
    ])


def leray(dom: Domain, vh: np.ndarray, mask=None) -> np.ndarray:
    """ℙ(κ) = I − κκᵀ/|κ|², optionally with the dealias mask folded in
    (`helmholtz_projection!`, src/Generator.jl:531-532; src/Propagator.jl:401). ℙ(0) = I."""
    k2 = dom.k2
    safe = np.where(k2 > 0, k2, 1.0)
    kdotv = (dom.kx * vh[0] + dom.ky * vh[1]) + dom.kz * vh[2]
    coef = np.where(k2 > 0, kdotv / safe, 0.0)
    out = np.stack([vh[0] - dom.kx * coef, vh[1] - dom.ky * coef, vh[2] - dom.kz * coef])
    if mask is not None:
        out = out * mask
    return out


def reality_projection(dom: Domain, fh: np.ndarray) -> np.ndarray:
    """`reality_projection!` (src/Propagator.jl:411-412): on the kx = 0 and kx = N/2 planes,
    replace each conjugate pair (ky, kz) ↔ (−ky, −kz) by its Hermitian part, so that
    f̂(−k) = conj f̂(k); self-conjugate modes keep their real part (adopted convention)."""
    N = dom.N
    out = fh.copy()
    planes = [0] + ([N // 2] if N % 2 == 0 else [])
    neg = (-np.arange(N)) % N
    for p in planes:
        plane = out[..., p]                      # [comp?][kz][ky]
        # the partner of (kz, ky) is (−kz, −ky)
        flipped = plane[..., neg, :][..., :, neg]
        out[..., p] = 0.5 * (plane + np.conj(flipped))
    return out


# ---------------------------------------------------------------------------------------------
# Flow conditions, forcing, generator.  (src/Generator.jl:81-140,484-581,648-730;
# src/Forcing.jl:110-111,435-456,1069-1117)
# ---------------------------------------------------------------------------------------------

@dataclass
class ConstantPower:
    """`ConstantPower(domain; injection_rate, lowest_shell, highest_shell)` (src/Forcing.jl:1069)."""
    injection_rate: float
    lowest_shell: int = 1
    highest_shell: float = 2


@dataclass
class Linear:
    """`Linear(domain; rate, lowest_shell = 1, highest_shell = 2)` (src/Forcing.jl:636-643): a steady
    rate A on the band, folded into the integrating factor (`steady_linear_rate`, :648-653)."""
    rate: float
    lowest_shell: int = 1
    highest_shell: float = 2


@dataclass
class VarianceController:
    """`VarianceController(domain; target, gain = 1, turnover_time, lowest_shell, highest_shell)`
    (src/Forcing.jl:828-875), with tℓ given explicitly; the amplitude is re-solved at every stage
    (`add_forcing_source!(::VarianceController)` :1041-1067)."""
    target: float
    turnover_time: float
    gain: float = 1.0
    lowest_shell: int = 1
    highest_shell: float = 2


@dataclass
class VarianceRescaling:
    """`VarianceRescaling(domain; target, over, lowest_shell, highest_shell)` (src/Forcing.jl:558-572):
    a post-step rescale of the band (`project_forcing!` :575-596)."""
    target: float
    over: str                                # "band" or "total"
    lowest_shell: int = 1
    highest_shell: float = 2


@dataclass
class StochasticOU:
    """`StochasticOU(domain; forcing_variance, correlation_time, lowest_shell, highest_shell, seed)`
    (src/Forcing.jl:1224-1415): an additive force held on a companion grid and advanced once per
    step on the host. Here `process` is the force for the current step, the companion's physical
    amplitudes a_k in its reference layout (set from outside before each step, the same arrays the
    library is given); `add_forcing_source!` (:1415) becomes N̂ += N³·a_k where the run's modes and
    the companion's coincide (`embed_modes!`)."""
    forcing_variance: float
    correlation_time: float
    lowest_shell: int = 1
    highest_shell: int = 2
    process: np.ndarray | None = None


def embed_modes(dom: Domain, a: np.ndarray) -> np.ndarray:
    """The companion's modes m (|m_a| < Nc/2, kx < Nc/2) carried into the run's half spectrum,
    zero elsewhere."""
    n = a.shape[-2]
    N = dom.N
    out = np.zeros(a.shape[:-3] + dom.shape_spectral, np.complex128)
    for mz in range(-(n // 2) + 1, n // 2):
        for my in range(-(n // 2) + 1, n // 2):
            for mx in range(0, n // 2):
                out[..., mz % N, my % N, mx] = a[..., mz % n, my % n, mx]
    return out


@dataclass
class Conditions:
    viscosity: float
    schmidt: float = 1.0
    velocity_forcing: object = None          # None (NoForcing), or one of the forcing classes above
    scalar: bool = True
    mean_gradient: tuple = (0.0, 0.0, 0.0)   # extension G1: uniform mean scalar gradient G
    scalar_forcing: object = None            # likewise, for the scalar

    def __post_init__(self):
        if not self.viscosity > 0:
            raise ValueError(f"`viscosity` must be positive, got {self.viscosity}")
        if not self.schmidt > 0:
            raise ValueError(f"`schmidt` must be positive, got {self.schmidt}")
        if self.scalar_forcing is not None and not self.scalar:
            # src/Generator.jl:312-316
            raise ValueError("a scalar forcing was given, but the run carries no scalar")

    @property
    def diffusivity(self) -> float:
        return self.viscosity / self.schmidt


def band_indicator(dom: Domain, forcing) -> np.ndarray:
    """Shells lowest..highest, shell h covering [h − ½, h + ½)·2π/L (`_shell_edges`,
    src/Forcing.jl:435-439); the band test is on the squares, both edges included."""
    k0 = 2 * math.pi / dom.L
    lo = (forcing.lowest_shell - 0.5) * k0
    top = forcing.highest_shell if math.isfinite(forcing.highest_shell) else math.ceil(math.sqrt(3) * dom.N / 2)
    hi = (top + 0.5) * k0
    return ((dom.k2 >= lo * lo) & (dom.k2 <= hi * hi)).astype(np.float64)


def target_factor(field: np.ndarray) -> float:
    """½ for the velocity (kinetic energy), 1 for the scalar (variance) (`_target_factor`,
    src/Forcing.jl:456)."""
    return 0.5 if field.ndim == 4 else 1.0


def band_is_empty(band_value: float, whole_value: float, eps_T: float) -> bool:
    """`_band_is_empty` (src/Forcing.jl:110-111)."""
    return not (math.isfinite(band_value) and band_value > 10 * eps_T * whole_value)


def constant_power_amplitude(dom: Domain, forcing, fh: np.ndarray, eps_T: float, diffusivity: float = 0.0):
    """The per-stage amplitude A of a band source A·𝟙_band·f at the stage field f, with the band.
    ConstantPower: A = ε/(2 k_band) (`add_forcing_source!(::ConstantPower)` src/Forcing.jl:1104-1117,
    `_injection_amplitude` :1091-1101). VarianceController: A = (ε_f − G(k − k∞)/tℓ)/(2 k_band), with
    k the whole field's variance and ε_f = 2·c·D·⟨f, |κ|²f⟩ its dissipation (:1041-1067). c is the
    target factor; an empty band gives A = 0."""
    c = target_factor(fh)
    band = band_indicator(dom, forcing)
    band_obs = c * dom.inner(fh, fh, band)
    whole_obs = c * dom.inner(fh, fh)
    if band_is_empty(band_obs, whole_obs, eps_T):
        return 0.0, band
    if isinstance(forcing, VarianceController):
        dissipation = 2 * c * diffusivity * dom.inner(fh, fh, dom.k2)
        restoring = forcing.gain * (whole_obs - forcing.target) / forcing.turnover_time
        return (dissipation - restoring) / (2 * band_obs), band
    return forcing.injection_rate / (2 * band_obs), band


def stage_source(dom: Domain, forcing, fh: np.ndarray, eps_T: float, diffusivity: float):
    """The additive source of a per-stage forcing (ConstantPower, VarianceController,
    StochasticOU), else None."""
    if isinstance(forcing, (ConstantPower, VarianceController)):
        A, band = constant_power_amplitude(dom, forcing, fh, eps_T, diffusivity)
        return A * band * fh
    if isinstance(forcing, StochasticOU):
        return float(dom.N) ** 3 * embed_modes(dom, forcing.process)
    return None


def project_forcing(dom: Domain, forcing, fh: np.ndarray, eps_T: float) -> np.ndarray:
    """VarianceRescaling's post-step rescale (`project_forcing!` src/Forcing.jl:575-596): the band
    takes one factor √(target_band/k_band) so the band (:band) or the whole field (:total) holds
    the target; an empty band is left alone. Other forcings project nothing."""
    if not isinstance(forcing, VarianceRescaling):
        return fh
    c = target_factor(fh)
    band = band_indicator(dom, forcing)
    band_raw = dom.inner(fh, fh, band)
    whole_raw = dom.inner(fh, fh)
    band_value = c * band_raw
    if band_is_empty(band_raw, whole_raw, eps_T):
        return fh
    if forcing.over == "total":
        target_band = max(0.0, forcing.target - c * whole_raw + band_value)
    else:
        target_band = forcing.target
    scale = math.sqrt(target_band / band_value)
    return fh + (scale - 1) * band * fh


def velocity_rhs(dom: Domain, cond: Conditions, uh, u, w, eps_T):
    """N̂_u = 𝔻ℙ FFT(u × ω) (negated Lamb vector, operands u, ω), mean mode zeroed, plus the
    ConstantPower source on the stage û (`velocity_rhs!` src/Generator.jl:484-488,
    `_velocity_advective_term!` :528-534, `mean_free_projection!` :486)."""
    nh = dom.to_spectral(_cross(u, w))
    if dom.dealiasing == "PhaseShift":
        # the average with the same term on the displaced grid, shifted back
        # (`_velocity_nonlinear!(::PhaseShift)`, src/Generator.jl:502-519)
        us = dom.to_physical(dom.shift_to * uh)
        ws = dom.to_physical(dom.shift_to * curl(dom, uh))
        nh = 0.5 * (nh + dom.shift_back * dom.to_spectral(_cross(us, ws)))
    nh = leray(dom, nh, dom.mask)
    nh[:, 0, 0, 0] = 0.0
    src = stage_source(dom, cond.velocity_forcing, uh, eps_T, cond.viscosity)
    if src is not None:
        nh = nh + src
    return nh


def scalar_rhs(dom: Domain, cond: Conditions, uh, u, phi, ph=None, eps_T: float = np.finfo(np.float64).eps):
    """N̂_φ = −𝔻 iκ·FFT(uφ) (`_scalar_flux_divergence!`, src/Generator.jl:708-720, divergence
    with α = −1), plus the mean-gradient source −G·û (extension G1: φ_total = G·x + φ, so
    ∂tφ + u·∇φ = −u·G + ϰ∇²φ)."""
    flux = u * phi[None]
    fh = dom.to_spectral(flux)
    if dom.dealiasing == "PhaseShift":
        # the flux on the displaced grid, shifted back and averaged before the divergence
        # (`_scalar_nonlinear!(::PhaseShift)`, src/Generator.jl:668-704; the shift commutes with iκ·)
        phs = dom.to_spectral(phi) if ph is None else ph
        us = dom.to_physical(dom.shift_to * uh)
        phis = dom.to_physical(dom.shift_to * phs)
        fh = 0.5 * (fh + dom.shift_back * dom.to_spectral(us * phis[None]))
    div = 1j * ((dom.dkx * fh[0] + dom.dky * fh[1]) + dom.dkz * fh[2])
    nh = -(dom.mask * div)
    G = cond.mean_gradient
    if any(g != 0.0 for g in G):
        nh = nh - ((G[0] * uh[0] + G[1] * uh[1]) + G[2] * uh[2])
    if ph is not None:
        # the scalar forcing's source at the stage φ̂ (`scalar_rhs!` src/Generator.jl:650-653)
        src = stage_source(dom, cond.scalar_forcing, ph, eps_T, cond.diffusivity)
        if src is not None:
            nh = nh + src
    return nh


# ---------------------------------------------------------------------------------------------
# The low-storage IF-RK step.  (src/Propagator.jl:140-150,267-274,304-419)
# ---------------------------------------------------------------------------------------------

def _rk4_tableau():
    a = (Fraction(0), Fraction(-567301805773, 1357537059087), Fraction(-2404267990393, 2016746695238),
         Fraction(-3550918686646, 2091501179385), Fraction(-1275806237668, 842570457699))
    b = (Fraction(1432997174477, 9575080441755), Fraction(5161836677717, 13612068292357),
         Fraction(1720146321549, 2090206949498), Fraction(3134564353537, 4481467310338),
         Fraction(2277821191437, 14882151754819))
    c = (Fraction(1432997174477, 9575080441755), Fraction(2526269341429, 6820363962896),
         Fraction(2006345519317, 3224310063776), Fraction(2802321613138, 2924317926251))
    af = tuple(float(x) for x in a)
    bf = tuple(float(x) for x in b)
    cf = tuple(float(x) for x in c)
    # d = (c₂, c₃ − c₂, c₄ − c₃, c₅ − c₄, 1 − c₅), subtracted in T after rounding (Propagator.jl:314-319)
    d = (cf[0], cf[1] - cf[0], cf[2] - cf[1], cf[3] - cf[2], 1.0 - cf[3])
    return af, bf, d


def _rk3_tableau():
    a = (0.0, float(Fraction(-5, 9)), float(Fraction(-153, 128)))
    b = (float(Fraction(1, 3)), float(Fraction(15, 16)), float(Fraction(8, 15)))
    d = (float(Fraction(1, 3)), float(Fraction(5, 12)), float(Fraction(1, 4)))
    return a, b, d


TABLEAUX = {"rk4": _rk4_tableau(), "rk3": _rk3_tableau()}


@dataclass
class State:
    uh: np.ndarray                  # (3, N, N, N/2+1) complex128
    phih: np.ndarray | None = None  # (N, N, N/2+1) complex128


def steady_rate(dom: Domain, forcing) -> np.ndarray:
    """The per-mode steady linear rate: A on the band for Linear, zero otherwise
    (`steady_linear_rate` src/Forcing.jl:281,648-653)."""
    if isinstance(forcing, Linear):
        return forcing.rate * band_indicator(dom, forcing)
    return np.zeros_like(dom.k2)


def integrating_factor(dom: Domain, diffusivity: float, rate: np.ndarray, delta: float) -> np.ndarray:
    """exp((A(κ) − D|κ|²)·δ) with δ = d_i·Δt: coefficient −D·δ on |κ|², offset A scaled by δ
    (`velocity_integrating_factor` / `scalar_integrating_factor` src/Generator.jl:565-581)."""
    return np.exp((-(diffusivity * delta)) * dom.k2 + delta * rate)


def _rhs(dom: Domain, cond: Conditions, uh, ph, eps_T):
    """Both fields' right-hand sides at a stage state (ph None without a scalar)."""
    u = dom.to_physical(uh)
    w = dom.to_physical(curl(dom, uh))
    nu_ = velocity_rhs(dom, cond, uh, u, w, eps_T)
    np_ = None
    if ph is not None:
        np_ = scalar_rhs(dom, cond, uh, u, dom.to_physical(ph), ph, eps_T)
    return nu_, np_


def _close(dom: Domain, cond: Conditions, uh, ph, eps_T) -> State:
    """The end of every scheme's step: the forcings' post-step projections, velocity first
    (`finalize!` src/Generator.jl:396-400), then the Leray and reality projections of the state
    (src/Propagator.jl:394-412)."""
    uh = project_forcing(dom, cond.velocity_forcing, uh, eps_T)
    if ph is not None:
        ph = project_forcing(dom, cond.scalar_forcing, ph, eps_T)
    uh = leray(dom, uh)
    uh = reality_projection(dom, uh)
    if ph is not None:
        ph = reality_projection(dom, ph)
    return State(uh, ph)


def _step_low_storage(dom: Domain, cond: Conditions, st: State, dt: float, scheme: str) -> State:
    """One step of `_low_storage_2n_step!` (src/Propagator.jl:326-419) with scheme "rk4"
    (`IFLowStorageRK4`, :304-320) or "rk3" (`IFLowStorageRK3`, :267-274)."""
    a, b, d = TABLEAUX[scheme]
    eps_T = np.finfo(np.float64).eps
    uh = st.uh.copy()
    ph = None if st.phih is None else st.phih.copy()
    has_scalar = ph is not None
    hu = None
    hp = None
    rate_u = steady_rate(dom, cond.velocity_forcing)
    rate_p = steady_rate(dom, cond.scalar_forcing) if has_scalar else None
    for i in range(len(a)):
        nu_, np_ = _rhs(dom, cond, uh, ph, eps_T)
        hu = dt * nu_ if i == 0 else a[i] * hu + dt * nu_
        E = integrating_factor(dom, cond.viscosity, rate_u, d[i] * dt)
        uh = E * (uh + b[i] * hu)
        if i < len(a) - 1:
            hu = E * hu
        if has_scalar:
            hp = dt * np_ if i == 0 else a[i] * hp + dt * np_
            Ep = integrating_factor(dom, cond.diffusivity, rate_p, d[i] * dt)
            ph = Ep * (ph + b[i] * hp)
            if i < len(a) - 1:
                hp = Ep * hp
    return _close(dom, cond, uh, ph, eps_T)


# ---------------------------------------------------------------------------------------------
# Tangent-linear model and discrete adjoint of the low-storage step, velocity only: the checker
# for a GPU adjoint of the step (all four schemes, every band forcing on either field). The
# reference has no AD; these are derived here from the step's
# own operations, and pinned by central finite differences and the dot-product identity.
# Inner products: physical ⟨a, b⟩ = Σ_x a·b; spectral ⟨x, y⟩ = Σ w·Re(conj(x)·y), w the Hermitian
# weights. Then irfft* = rfft/N³ and rfft* = N³·irfft; ℙ (with the mask), the curl iκ×, the
# integrating factor and the reality projection are self-adjoint; for m = u×ω the adjoint sends
# m̄ to ū = ω×m̄ and ω̄ = m̄×u.
# ---------------------------------------------------------------------------------------------

def spectral_dot(dom: Domain, x: np.ndarray, y: np.ndarray) -> float:
    return float(np.sum((np.conj(x) * y).real * dom.hweight))


def _cross(a, b):
    return np.stack([a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]])


def _tangent_supported(cond: Conditions, scheme: str, dom: Domain | None = None):
    if scheme not in SCHEMES:
        raise ValueError(f"unknown scheme {scheme!r}")
    if dom is not None and dom.dealiasing == "PhaseShift":
        raise ValueError("the tangent and adjoint are restated for the mask strategies, not PhaseShift")


def _amplitude_gradient(dom: Domain, f, x, A, band, D):
    """g with δA = ⟨g, δx⟩ (normalised inner product) for a per-stage amplitude A(x):
    ConstantPower A = ε/(2c⟨x, 𝟙x⟩); VarianceController A = (2cD⟨x, κ²x⟩ − G(c⟨x, x⟩ − k∞)/tℓ)/(2c⟨x, 𝟙x⟩)."""
    Ib = dom.inner(x, x, band)
    g = -2.0 * A * band * x / Ib
    if isinstance(f, VarianceController):
        c = target_factor(x)
        g = g + (4.0 * c * D * dom.k2 * x - 2.0 * f.gain * c * x / f.turnover_time) / (2.0 * c * Ib)
    return g


def _stage_source(dom: Domain, f, x, D, dx=None):
    """A per-stage band source s = A(x)·𝟙x (ConstantPower, VarianceController) and its tangent
    ds = δA·𝟙x + A·𝟙δx (an empty band's clamp to 0 has no tangent)."""
    if not isinstance(f, (ConstantPower, VarianceController)):
        return (0.0, 0.0) if dx is not None else 0.0
    A, band = constant_power_amplitude(dom, f, x, np.finfo(np.float64).eps, D)
    s = A * band * x
    if dx is None:
        return s
    if A == 0.0:
        return s, 0.0
    dA = dom.inner(_amplitude_gradient(dom, f, x, A, band, D), dx)
    return s, dA * band * x + A * band * dx


def _stage_source_adjoint(dom: Domain, f, x, D, lam):
    """The adjoint of x ↦ A(x)·𝟙x at x, applied to λ: A·𝟙λ + ⟨𝟙x, λ⟩·g."""
    if not isinstance(f, (ConstantPower, VarianceController)):
        return 0.0
    A, band = constant_power_amplitude(dom, f, x, np.finfo(np.float64).eps, D)
    if A == 0.0:
        return 0.0
    return A * band * lam + dom.inner(band * x, lam) * _amplitude_gradient(dom, f, x, A, band, D)


def _rescale_parts(dom: Domain, f, x):
    """VarianceRescaling's factor s at x and g with δs = ⟨g, δx⟩, or None when it leaves x alone."""
    if not isinstance(f, VarianceRescaling):
        return None
    c = target_factor(x)
    band = band_indicator(dom, f)
    Ib, Iw = dom.inner(x, x, band), dom.inner(x, x)
    if band_is_empty(Ib, Iw, np.finfo(np.float64).eps):
        return None
    bv = c * Ib
    if f.over == "total":
        Tb = f.target - c * Iw + bv
        if Tb <= 0.0:
            return 0.0, np.zeros_like(x), band
        dTb = -2.0 * c * x + 2.0 * c * band * x
    else:
        Tb, dTb = f.target, np.zeros_like(x)
    s = math.sqrt(Tb / bv)
    return s, (s / 2.0) * (dTb / Tb - 2.0 * c * band * x / bv), band


def _rescale_tangent(dom: Domain, f, x, dx):
    parts = _rescale_parts(dom, f, x)
    if parts is None:
        return dx
    s, g, band = parts
    return dx + (s - 1.0) * band * dx + dom.inner(g, dx) * band * x


def _rescale_adjoint(dom: Domain, f, x, lam):
    parts = _rescale_parts(dom, f, x)
    if parts is None:
        return lam
    s, g, band = parts
    return lam + (s - 1.0) * band * lam + dom.inner(band * x, lam) * g


def _nonlinear(dom: Domain, u, w):
    """N̂ = 𝔻ℙ FFT(u×ω), κ = 0 zeroed (the unforced part of `velocity_rhs`)."""
    nh = leray(dom, dom.to_spectral(_cross(u, w)), dom.mask)
    nh[:, 0, 0, 0] = 0.0
    return nh


def _flux_divergence(dom: Domain, f):
    """−𝔻 iκ·FFT(f) (the advective part of `scalar_rhs`)."""
    fh = dom.to_spectral(f)
    return -(dom.mask * (1j * ((dom.dkx * fh[0] + dom.dky * fh[1]) + dom.dkz * fh[2])))


def _gradient_source(cond: Conditions, uh):
    G = cond.mean_gradient
    return -((G[0] * uh[0] + G[1] * uh[1]) + G[2] * uh[2])


def step_tangent(dom: Domain, cond: Conditions, uh: np.ndarray, duh: np.ndarray, dt: float,
                 scheme: str = "rk4", ph: np.ndarray | None = None, dph: np.ndarray | None = None):
    """One step F of `scheme` and its tangent J·δ in the same pass, for the velocity alone (ph None)
    or the coupled velocity + scalar. Returns (F_u, J_u) or (F_u, F_φ, J_u, J_φ)."""
    _tangent_supported(cond, scheme, dom)
    if scheme == "heun":
        return heun_tangent(dom, cond, uh, duh, float(dt), ph, dph)
    if scheme == "ssprk3":
        return ssprk3_tangent(dom, cond, uh, duh, float(dt), ph, dph)
    a, b, d = TABLEAUX[scheme]
    scalar = ph is not None
    rate_u = steady_rate(dom, cond.velocity_forcing)
    rate_p = steady_rate(dom, cond.scalar_forcing) if scalar else None
    q, dq = uh.copy(), duh.copy()
    if scalar:
        p, dp = ph.copy(), dph.copy()
    h = dh = hp = dhp = None
    for i in range(len(a)):
        u, w = dom.to_physical(q), dom.to_physical(curl(dom, q))
        du, dw = dom.to_physical(dq), dom.to_physical(curl(dom, dq))
        n = _nonlinear(dom, u, w)
        dn = _nonlinear(dom, du, w) + _nonlinear(dom, u, dw)
        su, dsu = _stage_source(dom, cond.velocity_forcing, q, cond.viscosity, dq)
        n, dn = n + su, dn + dsu
        if scalar:
            phi, dphi = dom.to_physical(p), dom.to_physical(dp)
            npp = _flux_divergence(dom, u * phi[None]) + _gradient_source(cond, q)
            dnp = _flux_divergence(dom, du * phi[None] + u * dphi[None]) + _gradient_source(cond, dq)
            sp, dsp = _stage_source(dom, cond.scalar_forcing, p, cond.diffusivity, dp)
            npp, dnp = npp + sp, dnp + dsp
        h = dt * n if i == 0 else a[i] * h + dt * n
        dh = dt * dn if i == 0 else a[i] * dh + dt * dn
        E = integrating_factor(dom, cond.viscosity, rate_u, d[i] * dt)
        q, dq = E * (q + b[i] * h), E * (dq + b[i] * dh)
        if i < len(a) - 1:
            h, dh = E * h, E * dh
        if scalar:
            hp = dt * npp if i == 0 else a[i] * hp + dt * npp
            dhp = dt * dnp if i == 0 else a[i] * dhp + dt * dnp
            Ep = integrating_factor(dom, cond.diffusivity, rate_p, d[i] * dt)
            p, dp = Ep * (p + b[i] * hp), Ep * (dp + b[i] * dhp)
            if i < len(a) - 1:
                hp, dhp = Ep * hp, Ep * dhp
    # the forcings' post-step projections (VarianceRescaling), then the Leray and reality projections
    dq = _rescale_tangent(dom, cond.velocity_forcing, q, dq)
    q = project_forcing(dom, cond.velocity_forcing, q, np.finfo(np.float64).eps)
    q, dq = reality_projection(dom, leray(dom, q)), reality_projection(dom, leray(dom, dq))
    if not scalar:
        return q, dq
    dp = _rescale_tangent(dom, cond.scalar_forcing, p, dp)
    p = project_forcing(dom, cond.scalar_forcing, p, np.finfo(np.float64).eps)
    return q, reality_projection(dom, p), dq, reality_projection(dom, dp)


def step_adjoint(dom: Domain, cond: Conditions, uh: np.ndarray, lam: np.ndarray, dt: float,
                 scheme: str = "rk4", ph: np.ndarray | None = None, lam_p: np.ndarray | None = None):
    """Jᵀ·λ for the step at (û, φ̂): a forward pass that keeps each stage's fields, then the stages
    in reverse, each operation replaced by its adjoint. Returns λ_u, or (λ_u, λ_φ) with a scalar."""
    _tangent_supported(cond, scheme, dom)
    if scheme == "heun":
        return heun_adjoint(dom, cond, uh, lam, float(dt), ph, lam_p)
    if scheme == "ssprk3":
        return ssprk3_adjoint(dom, cond, uh, lam, float(dt), ph, lam_p)
    a, b, d = TABLEAUX[scheme]
    S = len(a)
    scalar = ph is not None
    rate_u = steady_rate(dom, cond.velocity_forcing)
    rate_p = steady_rate(dom, cond.scalar_forcing) if scalar else None
    N3 = float(dom.N) ** 3
    q = uh.copy()
    p = ph.copy() if scalar else None
    h = hp = None
    saved = []
    for i in range(S):
        u, w = dom.to_physical(q), dom.to_physical(curl(dom, q))
        phi = dom.to_physical(p) if scalar else None
        saved.append((u, w, phi, q, p))
        n = _nonlinear(dom, u, w) + _stage_source(dom, cond.velocity_forcing, q, cond.viscosity)
        h = dt * n if i == 0 else a[i] * h + dt * n
        E = integrating_factor(dom, cond.viscosity, rate_u, d[i] * dt)
        if scalar:
            npp = _flux_divergence(dom, u * phi[None]) + _gradient_source(cond, q)
            npp = npp + _stage_source(dom, cond.scalar_forcing, p, cond.diffusivity)
            hp = dt * npp if i == 0 else a[i] * hp + dt * npp
            Ep = integrating_factor(dom, cond.diffusivity, rate_p, d[i] * dt)
        q = E * (q + b[i] * h)
        if i < S - 1:
            h = E * h
        if scalar:
            p = Ep * (p + b[i] * hp)
            if i < S - 1:
                hp = Ep * hp
    # the end-of-step projections: reality and Leray, then the post-step rescale, in reverse
    lq = _rescale_adjoint(dom, cond.velocity_forcing, q, leray(dom, reality_projection(dom, lam)))
    lp = _rescale_adjoint(dom, cond.scalar_forcing, p, reality_projection(dom, lam_p)) if scalar else None
    lh_next = np.zeros_like(lq)                     # adjoints of the registers carried out of stage i
    lhp_next = np.zeros_like(lp) if scalar else None
    G = cond.mean_gradient
    for i in range(S - 1, -1, -1):
        E = integrating_factor(dom, cond.viscosity, rate_u, d[i] * dt)
        lv = E * lq                                 # q' = E·v, v = q + b h'
        lh = b[i] * lv + (E * lh_next if i < S - 1 else 0.0)
        ln = dt * lh
        lh_next = a[i] * lh if i > 0 else np.zeros_like(lh)
        u, w, phi, qi, pi_ = saved[i]
        lF = leray(dom, ln, dom.mask)
        lF[:, 0, 0, 0] = 0.0
        lm = N3 * dom.to_physical(lF)
        lu, lw = _cross(w, lm), _cross(lm, u)
        lq_new = lv + _stage_source_adjoint(dom, cond.velocity_forcing, qi, cond.viscosity, ln)
        if scalar:
            Ep = integrating_factor(dom, cond.diffusivity, rate_p, d[i] * dt)
            lvp = Ep * lp
            lhp = b[i] * lvp + (Ep * lhp_next if i < S - 1 else 0.0)
            lnp = dt * lhp
            lhp_next = a[i] * lhp if i > 0 else np.zeros_like(lhp)
            # ψ = Σ_c (−i 𝔻 κ_c) f̂_c − G·q with f = uφ
            lfh = np.stack([1j * dom.mask * dk * lnp for dk in (dom.dkx, dom.dky, dom.dkz)])
            lf = N3 * dom.to_physical(lfh)
            lu = lu + lf * phi[None]
            lphi = (lf[0] * u[0] + lf[1] * u[1]) + lf[2] * u[2]
            lq_new = lq_new - np.stack([G[0] * lnp, G[1] * lnp, G[2] * lnp])
            lp = lvp + dom.to_spectral(lphi) / N3 + _stage_source_adjoint(dom, cond.scalar_forcing, pi_, cond.diffusivity, lnp)
        lq = lq_new + dom.to_spectral(lu) / N3 + curl(dom, dom.to_spectral(lw)) / N3
    return lq if not scalar else (lq, lp)


def _rhs_pair(dom: Domain, cond: Conditions, q, p, dq=None, dp=None):
    """Both fields' right-hand sides at (q, p) with their sources, and, given (dq, dp), their
    tangents. Returns (n, np, dn, dnp, saved) with `saved` what the adjoint needs."""
    u, w = dom.to_physical(q), dom.to_physical(curl(dom, q))
    phi = dom.to_physical(p) if p is not None else None
    n = _nonlinear(dom, u, w) + _stage_source(dom, cond.velocity_forcing, q, cond.viscosity)
    npp = None
    if p is not None:
        npp = _flux_divergence(dom, u * phi[None]) + _gradient_source(cond, q) \
            + _stage_source(dom, cond.scalar_forcing, p, cond.diffusivity)
    dn = dnp = None
    if dq is not None:
        du, dw = dom.to_physical(dq), dom.to_physical(curl(dom, dq))
        dn = _nonlinear(dom, du, w) + _nonlinear(dom, u, dw) \
            + _stage_source(dom, cond.velocity_forcing, q, cond.viscosity, dq)[1]
        if p is not None:
            dphi = dom.to_physical(dp)
            dnp = _flux_divergence(dom, du * phi[None] + u * dphi[None]) + _gradient_source(cond, dq) \
                + _stage_source(dom, cond.scalar_forcing, p, cond.diffusivity, dp)[1]
    return n, npp, dn, dnp, (q, p, u, w, phi)


def _rhs_pair_adjoint(dom: Domain, cond: Conditions, saved, ln, lnp):
    """The adjoint of (q, p) ↦ (N̂_u, N̂_φ) at the saved stage, applied to (λ_n, λ_nφ)."""
    q, p, u, w, phi = saved
    N3 = float(dom.N) ** 3
    lF = leray(dom, ln, dom.mask)
    lF[:, 0, 0, 0] = 0.0
    lm = N3 * dom.to_physical(lF)
    lu, lw = _cross(w, lm), _cross(lm, u)
    lq = _stage_source_adjoint(dom, cond.velocity_forcing, q, cond.viscosity, ln)
    lp = None
    if p is not None:
        G = cond.mean_gradient
        lfh = np.stack([1j * dom.mask * dk * lnp for dk in (dom.dkx, dom.dky, dom.dkz)])
        lf = N3 * dom.to_physical(lfh)
        lu = lu + lf * phi[None]
        lphi = (lf[0] * u[0] + lf[1] * u[1]) + lf[2] * u[2]
        lq = lq - np.stack([G[0] * lnp, G[1] * lnp, G[2] * lnp])
        lp = dom.to_spectral(lphi) / N3 + _stage_source_adjoint(dom, cond.scalar_forcing, p, cond.diffusivity, lnp)
    lq = lq + dom.to_spectral(lu) / N3 + curl(dom, dom.to_spectral(lw)) / N3
    return lq, lp


def _factors(dom: Domain, cond: Conditions, delta: float, scalar: bool):
    Eu = integrating_factor(dom, cond.viscosity, steady_rate(dom, cond.velocity_forcing), delta)
    Ep = integrating_factor(dom, cond.diffusivity, steady_rate(dom, cond.scalar_forcing), delta) if scalar else None
    return Eu, Ep


def _add(a, b):
    return None if a is None else a + b


def _finish_tangent(dom, cond, q, p, dq, dp):
    dq = _rescale_tangent(dom, cond.velocity_forcing, q, dq)
    q = project_forcing(dom, cond.velocity_forcing, q, np.finfo(np.float64).eps)
    q, dq = reality_projection(dom, leray(dom, q)), reality_projection(dom, leray(dom, dq))
    if p is None:
        return q, dq
    dp = _rescale_tangent(dom, cond.scalar_forcing, p, dp)
    p = project_forcing(dom, cond.scalar_forcing, p, np.finfo(np.float64).eps)
    return q, reality_projection(dom, p), dq, reality_projection(dom, dp)


def _finish_adjoint(dom, cond, q, p, lam, lam_p):
    lq = _rescale_adjoint(dom, cond.velocity_forcing, q, leray(dom, reality_projection(dom, lam)))
    lp = _rescale_adjoint(dom, cond.scalar_forcing, p, reality_projection(dom, lam_p)) if p is not None else None
    return lq, lp


def heun_tangent(dom, cond, uh, duh, dt, ph=None, dph=None):
    """IFHeun's step (`_step_heun`) and its tangent, velocity alone or coupled."""
    half = dt / 2
    Eu, Ep = _factors(dom, cond, dt, ph is not None)
    n1, np1, dn1, dnp1, _ = _rhs_pair(dom, cond, uh, ph, duh, dph)
    qs, dqs = Eu * (uh + dt * n1), Eu * (duh + dt * dn1)
    bq, dbq = (Eu * uh) + half * (Eu * n1), (Eu * duh) + half * (Eu * dn1)
    ps = dps = bp = dbp = None
    if ph is not None:
        ps, dps = Ep * (ph + dt * np1), Ep * (dph + dt * dnp1)
        bp, dbp = (Ep * ph) + half * (Ep * np1), (Ep * dph) + half * (Ep * dnp1)
    n2, np2, dn2, dnp2, _ = _rhs_pair(dom, cond, qs, ps, dqs, dps)
    q, dq = bq + half * n2, dbq + half * dn2
    p = bp + half * np2 if ph is not None else None
    dp = dbp + half * dnp2 if ph is not None else None
    return _finish_tangent(dom, cond, q, p, dq, dp)


def heun_adjoint(dom, cond, uh, lam, dt, ph=None, lam_p=None):
    half = dt / 2
    scalar = ph is not None
    Eu, Ep = _factors(dom, cond, dt, scalar)
    n1, np1, _, _, s1 = _rhs_pair(dom, cond, uh, ph)
    qs = Eu * (uh + dt * n1)
    ps = Ep * (ph + dt * np1) if scalar else None
    n2, np2, _, _, s2 = _rhs_pair(dom, cond, qs, ps)
    q = (Eu * uh) + half * (Eu * n1) + half * n2
    p = (Ep * ph) + half * (Ep * np1) + half * np2 if scalar else None
    lq, lp = _finish_adjoint(dom, cond, q, p, lam, lam_p)
    # q = E q0 + ½Δt E N1 + ½Δt N2(q*), q* = E(q0 + Δt N1)
    lqs, lps = _rhs_pair_adjoint(dom, cond, s2, half * lq, half * lp if scalar else None)
    ln1 = half * (Eu * lq) + dt * (Eu * lqs)
    lnp1 = half * (Ep * lp) + dt * (Ep * lps) if scalar else None
    a1, b1 = _rhs_pair_adjoint(dom, cond, s1, ln1, lnp1)
    out_q = Eu * lq + Eu * lqs + a1
    out_p = Ep * lp + Ep * lps + b1 if scalar else None
    return out_q if not scalar else (out_q, out_p)


def ssprk3_tangent(dom, cond, uh, duh, dt, ph=None, dph=None):
    """IFSSPRK3's step (`_step_ssprk3`) and its tangent, velocity alone or coupled."""
    scalar = ph is not None
    Ef, Efp = _factors(dom, cond, dt, scalar)
    Eb, Ebp = _factors(dom, cond, -dt / 2, scalar)
    Eh, Ehp = _factors(dom, cond, dt / 2, scalar)
    n, npp, dn, dnp, _ = _rhs_pair(dom, cond, uh, ph, duh, dph)
    s1, ds1 = Ef * (uh + dt * n), Ef * (duh + dt * dn)
    p1 = Efp * (ph + dt * npp) if scalar else None
    dp1 = Efp * (dph + dt * dnp) if scalar else None
    n, npp, dn, dnp, _ = _rhs_pair(dom, cond, s1, p1, ds1, dp1)
    s2 = 0.25 * (Eb * (s1 + dt * n)) + Eh * (0.75 * uh)
    ds2 = 0.25 * (Eb * (ds1 + dt * dn)) + Eh * (0.75 * duh)
    p2 = 0.25 * (Ebp * (p1 + dt * npp)) + Ehp * (0.75 * ph) if scalar else None
    dp2 = 0.25 * (Ebp * (dp1 + dt * dnp)) + Ehp * (0.75 * dph) if scalar else None
    n, npp, dn, dnp, _ = _rhs_pair(dom, cond, s2, p2, ds2, dp2)
    q = Ef * ((1 / 3) * uh) + (2 / 3) * (Eh * (s2 + dt * n))
    dq = Ef * ((1 / 3) * duh) + (2 / 3) * (Eh * (ds2 + dt * dn))
    p = Efp * ((1 / 3) * ph) + (2 / 3) * (Ehp * (p2 + dt * npp)) if scalar else None
    dp = Efp * ((1 / 3) * dph) + (2 / 3) * (Ehp * (dp2 + dt * dnp)) if scalar else None
    return _finish_tangent(dom, cond, q, p, dq, dp)


def ssprk3_adjoint(dom, cond, uh, lam, dt, ph=None, lam_p=None):
    scalar = ph is not None
    Ef, Efp = _factors(dom, cond, dt, scalar)
    Eb, Ebp = _factors(dom, cond, -dt / 2, scalar)
    Eh, Ehp = _factors(dom, cond, dt / 2, scalar)
    n, npp, _, _, sv0 = _rhs_pair(dom, cond, uh, ph)
    s1 = Ef * (uh + dt * n)
    p1 = Efp * (ph + dt * npp) if scalar else None
    n, npp, _, _, sv1 = _rhs_pair(dom, cond, s1, p1)
    s2 = 0.25 * (Eb * (s1 + dt * n)) + Eh * (0.75 * uh)
    p2 = 0.25 * (Ebp * (p1 + dt * npp)) + Ehp * (0.75 * ph) if scalar else None
    n, npp, _, _, sv2 = _rhs_pair(dom, cond, s2, p2)
    q = Ef * ((1 / 3) * uh) + (2 / 3) * (Eh * (s2 + dt * n))
    p = Efp * ((1 / 3) * ph) + (2 / 3) * (Ehp * (p2 + dt * npp)) if scalar else None
    lq, lp = _finish_adjoint(dom, cond, q, p, lam, lam_p)
    # q = Ef(⅓q0) + ⅔Eh(s2 + Δt N(s2))
    lx2 = (2 / 3) * (Eh * lq)
    lxp2 = (2 / 3) * (Ehp * lp) if scalar else None
    a, b = _rhs_pair_adjoint(dom, cond, sv2, dt * lx2, dt * lxp2 if scalar else None)
    l_s2, l_p2 = lx2 + a, (lxp2 + b if scalar else None)
    l_q0 = (1 / 3) * (Ef * lq)
    l_pp0 = (1 / 3) * (Efp * lp) if scalar else None
    # s2 = ¼Eb(s1 + Δt N(s1)) + Eh(¾q0)
    lx1 = 0.25 * (Eb * l_s2)
    lxp1 = 0.25 * (Ebp * l_p2) if scalar else None
    a, b = _rhs_pair_adjoint(dom, cond, sv1, dt * lx1, dt * lxp1 if scalar else None)
    l_s1, l_p1 = lx1 + a, (lxp1 + b if scalar else None)
    l_q0 = l_q0 + 0.75 * (Eh * l_s2)
    l_pp0 = l_pp0 + 0.75 * (Ehp * l_p2) if scalar else None
    # s1 = Ef(q0 + Δt N(q0))
    lx0 = Ef * l_s1
    lxp0 = Efp * l_p1 if scalar else None
    a, b = _rhs_pair_adjoint(dom, cond, sv0, dt * lx0, dt * lxp0 if scalar else None)
    l_q0 = l_q0 + lx0 + a
    l_pp0 = l_pp0 + lxp0 + b if scalar else None
    return l_q0 if not scalar else (l_q0, l_pp0)


def _step_heun(dom: Domain, cond: Conditions, st: State, dt: float) -> State:
    """One step of `step!(::IFHeun, …)` (src/Propagator.jl:456-544): the predictor
    q* = E(q + Δt N₁), then q ← (E q + (Δt/2)(E N₁)) + (Δt/2) N₂ with N₂ at q*, in the reference's
    order of rotations and accumulations."""
    eps_T = np.finfo(np.float64).eps
    half = dt / 2
    fields = [(st.uh.copy(), cond.viscosity, steady_rate(dom, cond.velocity_forcing))]
    if st.phih is not None:
        fields.append((st.phih.copy(), cond.diffusivity, steady_rate(dom, cond.scalar_forcing)))
    n1 = _rhs(dom, cond, fields[0][0], fields[1][0] if len(fields) > 1 else None, eps_T)
    pred, banked = [], []
    for (q, D, rate), n in zip(fields, n1):
        E = integrating_factor(dom, D, rate, dt)
        pred.append(E * (q + dt * n))                    # q* = E(q + Δt N₁)
        banked.append((E * q) + half * (E * n))          # E q + (Δt/2)(E N₁)
    n2 = _rhs(dom, cond, pred[0], pred[1] if len(pred) > 1 else None, eps_T)
    out = [b + half * n for b, n in zip(banked, n2)]
    return _close(dom, cond, out[0], out[1] if len(out) > 1 else None, eps_T)


def _step_ssprk3(dom: Domain, cond: Conditions, st: State, dt: float) -> State:
    """One step of `step!(::IFSSPRK3, …)` (src/Propagator.jl:599-691), Shu–Osher form with each
    term carried to its stage's time:
    q⁽¹⁾ = E(Δt)(q + Δt N), q⁽²⁾ = ¼·E(−Δt/2)(q⁽¹⁾ + Δt N) + E(Δt/2)(¾ q),
    q ← E(Δt)(⅓ q) + ⅔·E(Δt/2)(q⁽²⁾ + Δt N)."""
    eps_T = np.finfo(np.float64).eps
    fields = [(st.uh.copy(), cond.viscosity, steady_rate(dom, cond.velocity_forcing))]
    if st.phih is not None:
        fields.append((st.phih.copy(), cond.diffusivity, steady_rate(dom, cond.scalar_forcing)))

    def rhs(stages):
        return _rhs(dom, cond, stages[0], stages[1] if len(stages) > 1 else None, eps_T)

    def E(D, rate, delta):
        return integrating_factor(dom, D, rate, delta)

    n = rhs([q for q, _, _ in fields])
    s1 = [E(D, r, dt) * (q + dt * nn) for (q, D, r), nn in zip(fields, n)]
    n = rhs(s1)
    s2 = [0.25 * (E(D, r, -dt / 2) * (s + dt * nn)) + E(D, r, dt / 2) * (0.75 * q)
          for (q, D, r), s, nn in zip(fields, s1, n)]
    n = rhs(s2)
    out = [E(D, r, dt) * ((1 / 3) * q) + (2 / 3) * (E(D, r, dt / 2) * (s + dt * nn))
           for (q, D, r), s, nn in zip(fields, s2, n)]
    return _close(dom, cond, out[0], out[1] if len(out) > 1 else None, eps_T)


SCHEMES = ("rk4", "rk3", "heun", "ssprk3")


def step(dom: Domain, cond: Conditions, st: State, dt: float, scheme: str = "rk4") -> State:
    """One field step of `scheme`: "rk4" (IFLowStorageRK4), "rk3" (IFLowStorageRK3), "heun"
    (IFHeun) or "ssprk3" (IFSSPRK3)."""
    dt = float(dt)
    if scheme == "heun":
        return _step_heun(dom, cond, st, dt)
    if scheme == "ssprk3":
        return _step_ssprk3(dom, cond, st, dt)
    return _step_low_storage(dom, cond, st, dt, scheme)


def recommended_cfl(scheme: str) -> float:
    """A scheme's advective-CFL ceiling under TwoThirds dealiasing (`recommended_cfl`,
    src/Propagator.jl:906-919; the 2/3 band leaves the base ceiling unchanged)."""
    return {"heun": 0.25, "rk3": 0.5, "ssprk3": 0.5, "rk4": 0.96}[scheme]


# ---------------------------------------------------------------------------------------------
# Deposit, max speed, CFL.  (src/Propagator.jl:808-842; src/Observables.jl:304-305;
# src/SimulationRun.jl:1051-1096)
# ---------------------------------------------------------------------------------------------

def deposit(dom: Domain, st: State):
    """u, ω (and φ) in physical representation, and max|u| = √max(|u|²)."""
    u = dom.to_physical(st.uh)
    w = dom.to_physical(curl(dom, st.uh))
    phi = None if st.phih is None else dom.to_physical(st.phih)
    speed = math.sqrt(float(np.max((u[0] * u[0] + u[1] * u[1]) + u[2] * u[2])))
    return u, w, phi, speed


def cfl_timestep(dom: Domain, cond: Conditions, speed: float, cfl: float, max_dt: float = math.inf):
    """Δt = min(C·Δx/max|u|, 1/(D·κ_min²), max_dt) (src/SimulationRun.jl:1051-1096)."""
    if not math.isfinite(speed):
        raise FloatingPointError("non-finite velocity: the run appears to have blown up")
    dx = dom.L / dom.N
    advective = cfl * dx / speed if speed > 0 else cfl * dx
    D = max(cond.viscosity, cond.diffusivity) if cond.scalar else cond.viscosity
    kmin = 2 * math.pi / dom.L
    resolution = 1 / (D * kmin ** 2)
    return min(advective, resolution, max_dt)


# ---------------------------------------------------------------------------------------------
# Tracers.  (src/Particles.jl:135-176,290-293; src/ParticlePropagator.jl:263-386)
# ---------------------------------------------------------------------------------------------

GAUSS_NODES = (-0.8611363115940526, -0.3399810435848563, 0.3399810435848563, 0.8611363115940526)
GAUSS_WEIGHTS = (0.3478548451374538, 0.6521451548625461, 0.6521451548625461, 0.3478548451374538)


def adams_weights(nodes, h):
    """Integral over [0, h] of each Lagrange basis polynomial through `nodes`, by 4-point
    Gauss–Legendre (`_adams_weights`, src/ParticlePropagator.jl:263-280)."""
    n = len(nodes)
    out = []
    for j in range(n):
        weight = 0.0
        for xi, w in zip(GAUSS_NODES, GAUSS_WEIGHTS):
            t = h * (xi + 1) / 2
            basis = 1.0
            for m in range(n):
                if m == j:
                    continue
                basis *= (t - nodes[m]) / (nodes[j] - nodes[m])
            weight += w * h / 2 * basis
        out.append(weight)
    return tuple(out)


def wrap(x: np.ndarray, L: float) -> np.ndarray:
    """Periodic reduction into [0, L): x − L·floor(x/L), a tiny negative result lifted by L, and
    a result equal to L mapped to 0 (adopted convention for PF's `displace!` wrap)."""
    y = x - L * np.floor(x / L)
    y = np.where(y < 0.0, y + L, y)
    return np.where(y >= L, 0.0, y)


def catmull_rom_weights(t: np.ndarray):
    """Catmull–Rom (Catmull & Rom 1974; Lalescu's 4-point C¹ kernel) weights for taps
    i−1, i, i+1, i+2 at fraction t ∈ [0, 1)."""
    wm1 = t * (t * (2.0 - t) - 1.0) * 0.5
    w0 = (t * t * (3.0 * t - 5.0) + 2.0) * 0.5
    w1 = t * (t * (4.0 - 3.0 * t) + 1.0) * 0.5
    w2 = t * t * (t - 1.0) * 0.5
    return (wm1, w0, w1, w2)


def cell_and_fraction(x: np.ndarray, dx: float):
    q = x / dx
    i = np.floor(q)
    return i.astype(np.int64), q - i


def stencil_polynomials(scheme) -> np.ndarray:
    """The weight polynomials of a wider interpolation scheme (src/Particles.jl:61-70, schemes of
    the unvendored GBGPeriodicFields, restated from their published definitions), as a (n, degree+1)
    array of coefficients in increasing degree for taps i − n/2 + 1 + j at fraction t:
    ("LagrangeSpline", n, _): the Lagrange basis through the taps; ("LalescuSpline", n, m) (Lalescu,
    Teaca & Carati 2010): the degree 2m + 1 Hermite interpolant on the cell, its derivatives 1..m at
    each end taken from the (n − 1)-point polynomial centred there (fitted exactly with polyfit)."""
    kind, n, m = scheme
    off = n // 2 - 1
    taps = np.arange(n) - off
    if kind == "LagrangeSpline":
        out = np.zeros((n, n))
        for j in range(n):
            others = np.delete(taps, j).astype(float)
            poly = np.polynomial.polynomial.polyfromroots(others) / np.prod(taps[j] - others)
            out[j] = poly
        return out
    if kind != "LalescuSpline":
        raise ValueError(f"unknown interpolation scheme {kind!r}")
    D = 2 * m + 1
    # derivative estimates: for each end e and order k, weights on the taps
    deriv = np.zeros((2, m + 1, n))
    for e in (0, 1):
        pts = np.arange(-(n // 2 - 1), n // 2)   # n − 1 points centred on the end
        for i, si in enumerate(pts):
            y = np.zeros(len(pts))
            y[i] = 1.0
            c = np.polynomial.polynomial.polyfit(pts.astype(float), y, len(pts) - 1)
            for k in range(m + 1):
                deriv[e, k, e + si + off] += math.factorial(k) * (c[k] if k < len(c) else 0.0)
    # Hermite basis on [0, 1]
    rows = []
    for e in (0, 1):
        for ell in range(m + 1):
            rows.append([(math.factorial(d) / math.factorial(d - ell) if d >= ell else 0.0) * (float(e) ** (d - ell) if d > ell else 1.0)
                         if (e == 1 or d == ell) else 0.0 for d in range(D + 1)])
    V = np.array(rows)
    out = np.zeros((n, D + 1))
    for e in (0, 1):
        for k in range(m + 1):
            rhs = np.zeros(D + 1)
            rhs[e * (m + 1) + k] = 1.0
            H = np.linalg.solve(V, rhs)
            out += np.outer(deriv[e, k], H)
    return out


def interpolate(dom: Domain, f: np.ndarray, X: np.ndarray, scheme=None) -> np.ndarray:
    """The gather of the physical field f ([comp][z][y][x] or [z][y][x]) at positions X (3, M)
    (`interpolate!`, src/Particles.jl:290-293): CatmullRom (= LalescuSpline(4)) by default, or a
    wider scheme (see `stencil_polynomials`). The sum runs x innermost, then y, then z."""
    if scheme is not None and tuple(scheme) != ("CatmullRom", 4, 1):
        return _interpolate_stencil(dom, f, X, stencil_polynomials(scheme))
    N = dom.N
    scalar = f.ndim == 3
    comps = f[None] if scalar else f
    ix, tx = cell_and_fraction(X[0], dom.dx)
    iy, ty = cell_and_fraction(X[1], dom.dx)
    iz, tz = cell_and_fraction(X[2], dom.dx)
    wx, wy, wz = catmull_rom_weights(tx), catmull_rom_weights(ty), catmull_rom_weights(tz)
    out = np.zeros((comps.shape[0], X.shape[1]))
    for c in range(comps.shape[0]):
        fc = comps[c]
        acc_z = np.zeros(X.shape[1])
        for cz in range(4):
            zz = (iz + cz - 1) % N
            acc_y = np.zeros(X.shape[1])
            for cy in range(4):
                yy = (iy + cy - 1) % N
                acc_x = np.zeros(X.shape[1])
                for cx in range(4):
                    xx = (ix + cx - 1) % N
                    acc_x = acc_x + wx[cx] * fc[zz, yy, xx]
                acc_y = acc_y + wy[cy] * acc_x
            acc_z = acc_z + wz[cz] * acc_y
        out[c] = acc_z
    return out[0] if scalar else out


def _interpolate_stencil(dom: Domain, f: np.ndarray, X: np.ndarray, polys: np.ndarray) -> np.ndarray:
    N, n = dom.N, polys.shape[0]
    off = n // 2 - 1
    scalar = f.ndim == 3
    comps = f[None] if scalar else f
    cells, weights = [], []
    for a in range(3):
        i, t = cell_and_fraction(X[a], dom.dx)
        cells.append(i)
        weights.append([np.polynomial.polynomial.polyval(t, polys[j]) for j in range(n)])
    (ix, iy, iz), (wx, wy, wz) = cells, weights
    out = np.zeros((comps.shape[0], X.shape[1]))
    for c in range(comps.shape[0]):
        acc_z = np.zeros(X.shape[1])
        for cz in range(n):
            zz = (iz + cz - off) % N
            acc_y = np.zeros(X.shape[1])
            for cy in range(n):
                yy = (iy + cy - off) % N
                acc_x = np.zeros(X.shape[1])
                for cx in range(n):
                    acc_x = acc_x + wx[cx] * comps[c][zz, yy, (ix + cx - off) % N]
                acc_y = acc_y + wy[cy] * acc_x
            acc_z = acc_z + wz[cz] * acc_y
        out[c] = acc_z
    return out[0] if scalar else out


def advect_adams(dom: Domain, X: np.ndarray, samples, times, u_new: np.ndarray, h: float, corrected: bool,
                 scheme=None):
    """One step of the Adams family (`_advance_positions!`, src/ParticlePropagator.jl:282-307) over
    the J samples f_{n−j} (newest first) taken at `times` (newest first): the predictor
    X* = wrap(X + Σ_j b_j f_{n−j}) with b the weights through the nodes t_{n−j} − t_n, and, when
    corrected, X ← wrap(X* + (β* f* + Σ_j (β_{j+1} − b_j) f_{n−j})) with f* = u(X*) and β the
    weights through (h, nodes…). Each displacement is summed term by term, then added.
    Returns the new positions and f* (None when not corrected)."""
    J = len(samples)
    nodes = tuple(times[j] - times[0] for j in range(J))
    b = adams_weights(nodes, h)
    disp = b[0] * samples[0]
    for j in range(1, J):
        disp = disp + b[j] * samples[j]
    Xs = wrap(X + disp, dom.L)
    if not corrected:
        return Xs, None
    fstar = interpolate(dom, u_new, Xs, scheme)
    beta = adams_weights((h,) + nodes, h)
    disp = beta[0] * fstar
    for j in range(J):
        disp = disp + (beta[j + 1] - b[j]) * samples[j]
    return wrap(Xs + disp, dom.L), fstar


TRACER_STEPS_MAX = {"abm": 7, "ab": 8}


def tracer_order(scheme: str, k: int) -> int:
    """`_order_of_accuracy` (src/ParticlePropagator.jl:255-256): k + 1 for ABM(k), k for AB(k)."""
    return k + 1 if scheme == "abm" else k


def startup_growth(order: int) -> float:
    """`_startup_growth` (src/SimulationRun.jl:1117)."""
    return 2.0 if order <= 5 else 1.5 if order <= 7 else 1.25


def binomial_repetitions(n: int, snaps: int) -> int:
    """The fewest repetitions r with C(snaps + r, snaps) ≥ n: a binomial schedule reverses n steps
    with `snaps` snapshots in at most r·n forward steps (Griewank & Walther 2000). With no snapshot
    every state is recomputed from the start, n(n − 1)/2 steps, so r = n bounds it."""
    if snaps == 0:
        return n
    r = 1
    while math.comb(snaps + r, snaps) < n:
        r += 1
    return r


def _binomial_split(n: int, snaps: int) -> int:
    """Where a binomial (revolve-style) schedule places its next snapshot in a span of n steps
    with `snaps` snapshots free: the left part keeps the steps that C(snaps + r − 1, snaps) leaves
    to the recursion."""
    r = binomial_repetitions(n, snaps)
    m = math.comb(snaps + r - 1, snaps)
    return min(max(1, n - m), n - 1)


def gradient_checkpointed(dom: Domain, cond: Conditions, st: State, dt: float, n: int, loss_grad, snaps: int,
                          scheme: str = "rk4"):
    """The gradient of a loss of the state after n steps, by the step's adjoint applied backwards
    over recomputed states, keeping at most `snaps` stored states besides the start (binomial
    checkpointing). `loss_grad(state)` gives (λ_u, λ_φ) at the end. Returns the gradient at the
    start, and the counts of recomputed forward steps and of the most states held at once."""
    stats = {"forward_steps": 0, "held": 0, "peak": 0}

    def advance(x, k):
        for _ in range(k):
            x = step(dom, cond, x, dt, scheme)
            stats["forward_steps"] += 1
        return x

    def back(x, k, free, lam):
        if k == 1:
            if x.phih is None:
                return step_adjoint(dom, cond, x.uh, lam[0], dt, scheme), None
            return step_adjoint(dom, cond, x.uh, lam[0], dt, scheme, ph=x.phih, lam_p=lam[1])
        if free == 0:   # no snapshot left: recompute every state from x
            for i in range(k - 1, -1, -1):
                lam = back(advance(x, i), 1, 0, lam)
            return lam
        m = _binomial_split(k, free)
        y = advance(x, m)
        stats["held"] += 1
        stats["peak"] = max(stats["peak"], stats["held"])
        lam = back(y, k - m, free - 1, lam)
        stats["held"] -= 1
        return back(x, m, free, lam)

    end = advance(st, n)
    lam = loss_grad(end)
    stats["forward_steps"] = 0
    grad = back(st, n, snaps, lam)
    return grad, stats


def catmull_rom_slopes(t: np.ndarray):
    """d/dt of the Catmull–Rom weights (the tangent of the gather through the positions)."""
    return ((-3.0 * t + 4.0) * t - 1.0) * 0.5, (9.0 * t - 10.0) * t * 0.5, \
        ((-9.0 * t + 8.0) * t + 1.0) * 0.5, (3.0 * t - 2.0) * t * 0.5


def _gather_taps(dom: Domain, X: np.ndarray):
    cells, weights, slopes = [], [], []
    for a in range(3):
        i, t = cell_and_fraction(X[a], dom.dx)
        cells.append(i)
        weights.append(catmull_rom_weights(t))
        slopes.append(catmull_rom_slopes(t))
    return cells, weights, slopes


def interpolate_tangent(dom: Domain, f: np.ndarray, X: np.ndarray, df: np.ndarray, dX: np.ndarray):
    """The tangent of the gather f(X) (`interpolate`): Σ w·δf at the taps plus the weights' slopes
    (per Δx) times δX. The cell index is locally constant, so it has no tangent."""
    N = dom.N
    (ix, iy, iz), (wx, wy, wz), (sx, sy, sz) = _gather_taps(dom, X)
    out = np.zeros((f.shape[0], X.shape[1]))
    for cz in range(4):
        zz = (iz + cz - 1) % N
        for cy in range(4):
            yy = (iy + cy - 1) % N
            for cx in range(4):
                xx = (ix + cx - 1) % N
                w = wz[cz] * wy[cy] * wx[cx]
                dw = (sx[cx] * wy[cy] * wz[cz] * dX[0] + wx[cx] * sy[cy] * wz[cz] * dX[1]
                      + wx[cx] * wy[cy] * sz[cz] * dX[2]) / dom.dx
                for c in range(f.shape[0]):
                    out[c] += w * df[c, zz, yy, xx] + dw * f[c, zz, yy, xx]
    return out


def interpolate_adjoint(dom: Domain, f: np.ndarray, X: np.ndarray, lam: np.ndarray):
    """The adjoint of (f, X) ↦ f(X) at (f, X), applied to λ (values at the points): the field part
    scatters w·λ onto the taps, the position part sums the slopes against f·λ."""
    N = dom.N
    (ix, iy, iz), (wx, wy, wz), (sx, sy, sz) = _gather_taps(dom, X)
    lf = np.zeros_like(f)
    lX = np.zeros_like(X)
    for cz in range(4):
        zz = (iz + cz - 1) % N
        for cy in range(4):
            yy = (iy + cy - 1) % N
            for cx in range(4):
                xx = (ix + cx - 1) % N
                w = wz[cz] * wy[cy] * wx[cx]
                fl = sum(f[c, zz, yy, xx] * lam[c] for c in range(f.shape[0]))
                lX[0] += sx[cx] * wy[cy] * wz[cz] * fl / dom.dx
                lX[1] += wx[cx] * sy[cy] * wz[cz] * fl / dom.dx
                lX[2] += wx[cx] * wy[cy] * sz[cz] * fl / dom.dx
                for c in range(f.shape[0]):
                    np.add.at(lf[c], (zz, yy, xx), w * lam[c])
    return lf, lX


def heun_push_tangent(dom: Domain, uh_new: np.ndarray, X: np.ndarray, f0: np.ndarray, h: float,
                      duh: np.ndarray, dX: np.ndarray, df0: np.ndarray):
    """The Heun push and closing deposit (X, f0; û at the end of the step) ↦ (X_new, f_new) and its
    tangent. The wrap is locally the identity."""
    u = dom.to_physical(uh_new)
    du = dom.to_physical(duh)
    (b0,) = adams_weights((0.0,), h)
    beta = adams_weights((h, 0.0), h)
    Xs = wrap(X + b0 * f0, dom.L)
    dXs = dX + b0 * df0
    fs = interpolate(dom, u, Xs)
    dfs = interpolate_tangent(dom, u, Xs, du, dXs)
    Xn = wrap(Xs + (beta[0] * fs + (beta[1] - b0) * f0), dom.L)
    dXn = dXs + beta[0] * dfs + (beta[1] - b0) * df0
    fn = interpolate(dom, u, Xn)
    dfn = interpolate_tangent(dom, u, Xn, du, dXn)
    return Xn, fn, dXn, dfn


def heun_push_adjoint(dom: Domain, uh_new: np.ndarray, X: np.ndarray, f0: np.ndarray, h: float,
                      lXn: np.ndarray, lfn: np.ndarray):
    """The adjoint of the Heun push and closing deposit: (λ_X_new, λ_f_new) ↦ (λ_û, λ_X, λ_f0)."""
    u = dom.to_physical(uh_new)
    N3 = float(dom.N) ** 3
    (b0,) = adams_weights((0.0,), h)
    beta = adams_weights((h, 0.0), h)
    Xs = wrap(X + b0 * f0, dom.L)
    fs = interpolate(dom, u, Xs)
    Xn = wrap(Xs + (beta[0] * fs + (beta[1] - b0) * f0), dom.L)
    lu, lX_n2 = interpolate_adjoint(dom, u, Xn, lfn)
    lXn_total = lXn + lX_n2
    lXs = lXn_total.copy()
    lfs = beta[0] * lXn_total
    lf0 = (beta[1] - b0) * lXn_total
    lu2, lXs2 = interpolate_adjoint(dom, u, Xs, lfs)
    lu = lu + lu2
    lXs = lXs + lXs2
    lX = lXs.copy()
    lf0 = lf0 + b0 * lXs
    return dom.to_spectral(lu) / N3, lX, lf0


def advect_heun(dom: Domain, X: np.ndarray, f0: np.ndarray, u_new: np.ndarray, h: float):
    """Heun = ABM(1) (src/ParticlePropagator.jl:165,288-315): X* = wrap(X + b₀f₀); f* = u(X*);
    X ← wrap(X* + (β₀f* + (β₁ − b₀)f₀)). Each displacement is summed term by term, then added."""
    (b0,) = adams_weights((0.0,), h)
    Xs = wrap(X + b0 * f0, dom.L)
    fstar = interpolate(dom, u_new, Xs)
    beta = adams_weights((h, 0.0), h)
    disp = beta[0] * fstar + (beta[1] - b0) * f0
    return wrap(Xs + disp, dom.L), fstar


# ---------------------------------------------------------------------------------------------
# Observables and spectra.  (src/Observables.jl:84-173,345-370,502-514)
# ---------------------------------------------------------------------------------------------

def kinetic_energy(dom, uh):
    return dom.inner(uh, uh) / 2


def dissipation(dom, uh, nu):
    return nu * dom.inner(uh, uh, dom.k2)


def scalar_variance(dom, ph):
    return dom.inner(ph, ph)


def scalar_dissipation(dom, ph, kappa):
    return 2 * kappa * dom.inner(ph, ph, dom.k2)


def energy_below_scale(dom: Domain, uh: np.ndarray, nu: float):
    """`kinetic_energy_and_dissipation_below_scale` (src/Observables.jl:253-263): for every side
    l = nL/N, k(l) = (Σ|û|² − ΣW_l²|û|²)/2 and ε(l) = ν(Σκ²|û|² − Σκ²W_l²|û|²), normalised sums with
    the Hermitian weights, W_l(κ) = ∏_a sinc(κ_a l/2) the transfer function of the box mean."""
    N, L = dom.N, dom.L
    p = (np.abs(uh) ** 2).sum(axis=0) * dom.hweight
    whole = float(p.sum()) / float(N) ** 6
    dirichlet = float((p * dom.k2).sum()) / float(N) ** 6
    scales = np.array([n * L / N for n in range(1, N + 1)])
    k = np.zeros(N)
    eps = np.zeros(N)
    for i, l in enumerate(scales):
        W = np.sinc(dom.kx * l / (2 * math.pi)) * np.sinc(dom.ky * l / (2 * math.pi)) * np.sinc(dom.kz * l / (2 * math.pi))
        W2 = W * W
        k[i] = (whole - float((p * W2).sum()) / float(N) ** 6) / 2
        eps[i] = nu * (dirichlet - float((p * dom.k2 * W2).sum()) / float(N) ** 6)
    return scales, k, eps


SKEWNESS_ISOTROPY_CONSTANT = (4 / 7) * math.sqrt(15 / 2)   # src/Observables.jl:403-406


def strain_physical(dom: Domain, uh: np.ndarray) -> np.ndarray:
    """S_ij = ½(∂_j u_i + ∂_i u_j) in physical space, as (S11, S22, S33, S12, S13, S23)."""
    d = (dom.dkx, dom.dky, dom.dkz)
    pairs = ((0, 0), (1, 1), (2, 2), (0, 1), (0, 2), (1, 2))
    return np.stack([dom.to_physical(0.5j * (d[j] * uh[i] + d[i] * uh[j])) for i, j in pairs])


def derivative_skewness(dom: Domain, uh: np.ndarray) -> float:
    """`derivative_skewness` (src/Observables.jl:466-478): C·3⟨det S⟩/⟨S:S⟩^{3/2}, with
    ⟨S:S⟩ = ½Σ|κ|²|û|² read from û and ⟨det S⟩ the grid mean of the strain's determinant."""
    ss = dom.inner(uh, uh, dom.k2) / 2
    if ss <= 0:
        return 0.0
    s11, s22, s33, s12, s13, s23 = strain_physical(dom, uh)
    det = s11 * (s22 * s33 - s23 * s23) - s12 * (s12 * s33 - s23 * s13) + s13 * (s12 * s23 - s22 * s13)
    return 3 * SKEWNESS_ISOTROPY_CONSTANT * float(det.mean()) / ss ** 1.5


def n_shells(N: int) -> int:
    return int(math.floor(math.sqrt(3) * N / 2 + 0.5)) + 1


def radial_spectrum(dom: Domain, fh: np.ndarray) -> np.ndarray:
    """Shell sums of the Hermitian-weighted |f̂|²/N⁶, shell n = floor(|κ|/Δκ + ½) (shells
    [n − ½, n + ½) as in `_shell_edges`, src/Forcing.jl:435-439)."""
    dk = 2 * math.pi / dom.L
    shell = np.floor(np.sqrt(dom.k2) / dk + 0.5).astype(np.int64)
    p = (np.abs(fh) ** 2) * dom.hweight
    if p.ndim == 4:
        p = p.sum(axis=0)
    out = np.zeros(n_shells(dom.N))
    np.add.at(out, np.broadcast_to(shell, p.shape).ravel(), p.ravel())
    return out / float(dom.N) ** 6


def energy_spectrum(dom, uh):
    """E(κ) = radial_spectrum/(2Δκ) (src/Observables.jl:502-514)."""
    dk = 2 * math.pi / dom.L
    return radial_spectrum(dom, uh) / (2 * dk)


def scalar_spectrum(dom, ph):
    """E_φ(κ) = radial_spectrum/Δκ (no reference function; the variance convention, no ½)."""
    dk = 2 * math.pi / dom.L
    return radial_spectrum(dom, ph) / dk


# ---------------------------------------------------------------------------------------------
# Run layer: one iteration of `advance!` (src/SimulationRun.jl:1155-1229).
# ---------------------------------------------------------------------------------------------

@dataclass
class Run:
    dom: Domain
    cond: Conditions
    state: State
    X: np.ndarray | None = None       # (3, M) tracer positions
    scheme: str = "rk4"
    cfl: float = 0.5
    max_dt: float = math.inf
    time: float = 0.0
    nstep: int = 0
    u: np.ndarray = field(default=None, repr=False)
    speed: float = 0.0
    tracer_scheme: tuple = ("abm", 1)  # ("abm", k) = ABM(k), Heun = ABM(1); ("ab", k) = AB(k)
    shortened_first_steps: bool = False
    interpolation: tuple = None        # the tracers' scheme (None: CatmullRom), see `interpolate`
    trail: list = field(default_factory=list, repr=False)   # (time, value), newest first

    def __post_init__(self):
        self.u, _, _, self.speed = deposit(self.dom, self.state)
        if self.X is not None:
            self.trail = [(self.time, interpolate(self.dom, self.u, self.X, self.interpolation))]

    @property
    def f0(self):
        return self.trail[0][1]

    @property
    def trail_time(self):
        return self.trail[0][0]

    def startup_bound(self, dt: float) -> float:
        """`_startup_bound` (src/SimulationRun.jl:1119-1132)."""
        kind, k = self.tracer_scheme
        if not (self.shortened_first_steps and self.X is not None and k > 1):
            return math.inf
        order = tracer_order(kind, k)
        if len(self.trail) > 1:
            return startup_growth(order) * (self.trail[0][0] - self.trail[1][0])
        nu = self.cond.viscosity
        eps = dissipation(self.dom, self.state.uh, nu)
        tau = math.sqrt(nu / eps) if eps > 0 else math.inf
        return tau * (dt / tau) ** (order / 3) if (math.isfinite(tau) and tau > 0) else math.inf

    def timestep(self) -> float:
        base = cfl_timestep(self.dom, self.cond, self.speed, self.cfl, self.max_dt)
        return min(self.startup_bound(base), base)

    def advance(self, dt: float | None = None):
        D = self.timestep() if dt is None else float(dt)
        if not (math.isfinite(D) and D > 0):
            raise ValueError(f"the timestep must be positive and finite, got {D}")
        t_new = self.time + D
        if not t_new > self.time:
            raise ValueError(f"the timestep {D} is too small to advance the clock")
        self.state = step(self.dom, self.cond, self.state, D, self.scheme)
        self.u, _, _, self.speed = deposit(self.dom, self.state)
        if self.X is not None:
            kind, k = self.tracer_scheme
            capacity = k
            if len(self.trail) >= k:
                J, corrected = k, kind == "abm"
            else:
                J, corrected = len(self.trail), True
            samples = [v for _, v in self.trail[:J]]
            times = [t for t, _ in self.trail[:J]]
            self.X, _ = advect_adams(self.dom, self.X, samples, times, self.u, D, corrected, self.interpolation)
            self.trail = [(t_new, interpolate(self.dom, self.u, self.X, self.interpolation))] + self.trail[:capacity - 1]
        if not math.isfinite(self.speed):
            raise FloatingPointError(f"non-finite velocity at step {self.nstep + 1}")
        if self.state.phih is not None and not math.isfinite(scalar_variance(self.dom, self.state.phih)):
            raise FloatingPointError(f"non-finite scalar at step {self.nstep + 1}")
        self.time = t_new
        self.nstep += 1
        return D

"""Python host side of the B200 IF-RK time step: a ctypes binding of the C ABI (include/gbght.h).

It mirrors the reference's run API (src/SimulationRun.jl, src/Propagator.jl,
src/ParticlePropagator.jl) with the same names, argument meanings and refusals. An ArgumentError
of the reference raises ``ValueError``; an ErrorException (a schedule refusal or a blow-up) raises
``ScheduleError``.

The compute runs in ``libgbght.so``, the CUDA library built in-tree by ``gbght_build.py``. There is no
host fallback: if the library is missing, `load_library` raises.
"""
from __future__ import annotations

import ctypes as C
import math
import os
from dataclasses import dataclass, field

import numpy as np

from . import seed  # noqa: F401  (host-side seeding, re-exported)
from . import stochastic as _stochastic

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(_HERE), "libgbght.so")

FP64, FP32_MIXED = 0, 1
IFRK4, IFRK3, IFHEUN, IFSSPRK3 = 0, 1, 2, 3
SCHEMES = {"IFLowStorageRK4": IFRK4, "IFLowStorageRK3": IFRK3, "IFHeun": IFHEUN, "IFSSPRK3": IFSSPRK3}
FORCING_NONE, FORCING_CONSTANT_POWER, FORCING_LINEAR, FORCING_VARIANCE_CONTROLLER, FORCING_VARIANCE_RESCALING = 0, 1, 2, 3, 4
FORCING_STOCHASTIC_OU = 5
OVER = {"band": 0, "total": 1}
TRACER_SCHEMES = {"Heun": 0, "ABM": 1, "AB": 2}
OK, ERR_ARGUMENT, ERR_SCHEDULE, ERR_CUDA, ERR_DEVICE = 0, 1, 2, 3, 4


class ScheduleError(RuntimeError):
    """The reference's ErrorException: a refused schedule or a blow-up."""


class DeviceError(RuntimeError):
    """A CUDA runtime error or a raised device status bit."""


class ForcingParams(C.Structure):
    _fields_ = [
        ("kind", C.c_int),
        ("rate", C.c_double),
        ("target", C.c_double),
        ("gain", C.c_double),
        ("turnover_time", C.c_double),
        ("over", C.c_int),
        ("lowest_shell", C.c_int),
        ("highest_shell", C.c_double),
    ]


class Config(C.Structure):
    _fields_ = [
        ("grid_points_per_axis", C.c_int),
        ("side_length", C.c_double),
        ("precision", C.c_int),
        ("scheme", C.c_int),
        ("viscosity", C.c_double),
        ("schmidt", C.c_double),
        ("scalar", C.c_int),
        ("velocity_forcing", ForcingParams),
        ("scalar_forcing", ForcingParams),
        ("mean_gradient", C.c_double * 3),
        ("tracers", C.c_int64),
        ("cfl", C.c_double),
        ("max_dt", C.c_double),
        ("device", C.c_int),
        ("tracer_scheme", C.c_int),
        ("tracer_steps", C.c_int),
        ("shortened_first_steps", C.c_int),
        ("interpolation", C.c_int),
        ("interpolation_points", C.c_int),
        ("interpolation_smoothness", C.c_int),
        ("dealiasing", C.c_int),
        ("houli_order", C.c_int),
        ("houli_strength", C.c_double),
        ("tracer_gather", C.c_int),
    ]


_DP = C.POINTER(C.c_double)
_SIGNATURES = {
    "gbght_config_default": (None, [C.POINTER(Config)]),
    "gbght_create": (C.c_int, [C.POINTER(C.c_void_p), C.POINTER(Config)]),
    "gbght_destroy": (None, [C.c_void_p]),
    "gbght_last_error": (C.c_char_p, [C.c_void_p]),
    "gbght_global_error": (C.c_char_p, []),
    "gbght_version": (C.c_char_p, []),
    "gbght_geometry": (C.c_int, [C.c_void_p, C.POINTER(C.c_int), _DP]),
    "gbght_state_import": (C.c_int, [C.c_void_p, _DP, _DP]),
    "gbght_state_export": (C.c_int, [C.c_void_p, _DP, _DP]),
    "gbght_step": (C.c_int, [C.c_void_p, C.c_double]),
    "gbght_forcing_source_set": (C.c_int, [C.c_void_p, C.c_int, _DP, C.c_int]),
    "gbght_recommended_cfl": (C.c_int, [C.c_int, _DP]),
    "gbght_recommended_cfl_dealiased": (C.c_int, [C.c_int, C.c_int, _DP]),
    "gbght_ensemble_create": (C.c_int, [C.POINTER(C.c_void_p), C.POINTER(C.c_void_p), C.c_int]),
    "gbght_ensemble_destroy": (None, [C.c_void_p]),
    "gbght_ensemble_step": (C.c_int, [C.c_void_p, C.c_double]),
    "gbght_ensemble_last_error": (C.c_char_p, [C.c_void_p]),
    "gbght_ensemble_set_batching": (C.c_int, [C.c_void_p, C.c_int]),
    "gbght_ensemble_units": (C.c_int, [C.c_void_p, C.POINTER(C.c_int)]),
    "gbght_ensemble_autotune": (C.c_int, [C.c_void_p]),
    "gbght_ensemble_tuning": (C.c_int, [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_float),
                                        C.c_int]),
    "gbght_deposit": (C.c_int, [C.c_void_p]),
    "gbght_max_speed": (C.c_int, [C.c_void_p, _DP]),
    "gbght_cfl_timestep": (C.c_int, [C.c_void_p, _DP]),
    "gbght_velocity_physical_export": (C.c_int, [C.c_void_p, _DP]),
    "gbght_velocity_physical_import": (C.c_int, [C.c_void_p, _DP]),
    "gbght_observables": (C.c_int, [C.c_void_p, _DP]),
    "gbght_spectrum_length": (C.c_int, [C.c_void_p, C.POINTER(C.c_int)]),
    "gbght_spectrum": (C.c_int, [C.c_void_p, C.c_int, _DP, C.c_int]),
    "gbght_energy_below_scale": (C.c_int, [C.c_void_p, _DP, _DP, _DP, C.c_int]),
    "gbght_derivative_skewness": (C.c_int, [C.c_void_p, _DP]),
    "gbght_tracers_import": (C.c_int, [C.c_void_p, _DP]),
    "gbght_tracers_export": (C.c_int, [C.c_void_p, _DP]),
    "gbght_tracer_sample_export": (C.c_int, [C.c_void_p, _DP, _DP]),
    "gbght_tracer_trail_reset": (C.c_int, [C.c_void_p]),
    "gbght_tracer_trail_export": (C.c_int, [C.c_void_p, C.c_int, _DP, _DP]),
    "gbght_selftest_wait_timeout": (C.c_int, [C.c_void_p, C.c_int64]),
    "gbght_tracer_sample_restore": (C.c_int, [C.c_void_p, _DP, C.c_double]),
    "gbght_advect": (C.c_int, [C.c_void_p, C.c_double]),
    "gbght_deposit_tracers": (C.c_int, [C.c_void_p, C.c_double]),
    "gbght_interpolate_velocity": (C.c_int, [C.c_void_p, _DP, C.c_int64, _DP]),
    "gbght_advance": (C.c_int, [C.c_void_p, C.c_double, _DP]),
    "gbght_clock": (C.c_int, [C.c_void_p, _DP, C.POINTER(C.c_int64)]),
    "gbght_set_clock": (C.c_int, [C.c_void_p, C.c_double, C.c_int64]),
    "gbght_status_word": (C.c_int, [C.c_void_p, C.POINTER(C.c_uint32)]),
    "gbght_synchronize": (C.c_int, [C.c_void_p]),
    "gbght_profile": (C.c_int, [C.c_void_p, C.c_int]),
    "gbght_profile_read": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_int64), _DP]),
    "gbght_timer": (C.c_int, [C.c_void_p, C.c_int, _DP]),
    "gbght_adjoint_create": (C.c_int, [C.c_void_p, C.c_int]),
    "gbght_adjoint_import": (C.c_int, [C.c_void_p, _DP, _DP]),
    "gbght_adjoint_export": (C.c_int, [C.c_void_p, _DP, _DP]),
    "gbght_adjoint_step": (C.c_int, [C.c_void_p, C.c_double]),
    "gbght_adjoint_add_observable": (C.c_int, [C.c_void_p, C.c_int, C.c_double]),
    "gbght_adjoint_forcing_gradient": (C.c_int, [C.c_void_p, _DP, C.c_int]),
    "gbght_adjoint_clear": (C.c_int, [C.c_void_p]),
    "gbght_snapshot_save": (C.c_int, [C.c_void_p, C.c_int]),
    "gbght_snapshot_load": (C.c_int, [C.c_void_p, C.c_int]),
    "gbght_adjoint_advance": (C.c_int, [C.c_void_p, C.c_double]),
    "gbght_adjoint_deposit_tracers": (C.c_int, [C.c_void_p]),
    "gbght_adjoint_tracers_import": (C.c_int, [C.c_void_p, _DP, _DP]),
    "gbght_adjoint_tracers_export": (C.c_int, [C.c_void_p, _DP, _DP]),
}

KERNELS = ("y_inverse", "x_products", "y_forward", "z_epilogue", "x_velocity", "force_amp", "reality",
           "tracers", "observables", "traversal", "x_adjoint", "z_adjoint", "z_shift")
DEALIASING = {"TwoThirds": 0, "HouLi": 1, "PhaseShift": 2}
OBSERVABLES = {"kinetic_energy": 0, "scalar_variance": 1}

_loaded: dict = {}


def load_library(path: str | None = None):
    """Load and type the C ABI from `path` (default: the in-tree CUDA library)."""
    path = os.path.abspath(path or LIB_PATH)
    if path in _loaded:
        return _loaded[path]
    if not os.path.exists(path):
        raise OSError(f"the CUDA library {path} is missing: build it with "
                      f"`python gbghomogeneousturbulence.jl_b200/gbght_build.py`")
    lib = C.CDLL(path)
    for name, (res, args) in _SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _loaded[path] = lib
    return lib


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(_DP)


def _is_device(a) -> bool:
    """Whether `a` is a CUDA tensor (device memory the library reads or writes in place)."""
    return getattr(a, "is_cuda", False)


def _dev_ptr(t, shape, what, real=False):
    """The address of a contiguous CUDA tensor: complex128 of `shape`, or float64 of `shape` + (2,)
    (interleaved re, im); with `real`, float64 of `shape`."""
    import torch
    if not t.is_contiguous():
        raise ValueError(f"{what} must be contiguous")
    if real:
        ok = t.dtype == torch.float64 and tuple(t.shape) == tuple(shape)
    else:
        ok = (t.dtype == torch.complex128 and tuple(t.shape) == tuple(shape)) or \
             (t.dtype == torch.float64 and tuple(t.shape) == tuple(shape) + (2,))
    if not ok:
        kind = "float64" if real else "complex128"
        raise ValueError(f"{what} must be a contiguous {kind} CUDA tensor of shape {shape}")
    return C.cast(C.c_void_p(t.data_ptr()), _DP)


@dataclass
class ConstantPower:
    """`ConstantPower(domain; injection_rate, lowest_shell = 1, highest_shell = 2)`
    (src/Forcing.jl:1069)."""
    injection_rate: float
    lowest_shell: int = 1
    highest_shell: float = 2


@dataclass
class Linear:
    """`Linear(domain; rate, lowest_shell = 1, highest_shell = 2)` (src/Forcing.jl:636-643): the
    steady rate A on the band, folded into the integrating factor. Either field may take it."""
    rate: float
    lowest_shell: int = 1
    highest_shell: float = 2


@dataclass
class VarianceController:
    """`VarianceController(domain; target, gain = 1, turnover_time, lowest_shell = 1,
    highest_shell = 2)` (src/Forcing.jl:828-875). The turnover time tℓ is given explicitly: the
    reference derives a default from its stationary-state model, which this backend does not carry."""
    target: float
    turnover_time: float
    gain: float = 1.0
    lowest_shell: int = 1
    highest_shell: float = 2


@dataclass
class VarianceRescaling:
    """`VarianceRescaling(domain; target, over, lowest_shell = 1, highest_shell = 2)`
    (src/Forcing.jl:558-572), `over` "band" or "total"."""
    target: float
    over: str
    lowest_shell: int = 1
    highest_shell: float = 2


@dataclass
class StochasticOU:
    """`StochasticOU(domain; forcing_variance, correlation_time, lowest_shell = 1, highest_shell = 2,
    seed)` (src/Forcing.jl:1224-1415): an additive Ornstein–Uhlenbeck force on the band, advanced
    once per step on the host (`gbght.stochastic.OUProcess`) and handed to the library before the
    step."""
    forcing_variance: float
    correlation_time: float
    lowest_shell: int = 1
    highest_shell: int = 2
    seed: int = 0


@dataclass
class NoForcing:
    """`NoForcing()` (src/Forcing.jl): a freely decaying field."""


def _fill_forcing(p: ForcingParams, f, who: str) -> None:
    """Write one field's forcing object into its gbght_forcing_params block (defaults already set)."""
    if f is None or isinstance(f, NoForcing):
        p.kind = FORCING_NONE
        return
    if isinstance(f, ConstantPower):
        p.kind, p.rate = FORCING_CONSTANT_POWER, float(f.injection_rate)
    elif isinstance(f, Linear):
        p.kind, p.rate = FORCING_LINEAR, float(f.rate)
    elif isinstance(f, VarianceController):
        p.kind, p.target, p.gain, p.turnover_time = (FORCING_VARIANCE_CONTROLLER, float(f.target), float(f.gain),
                                                      float(f.turnover_time))
    elif isinstance(f, StochasticOU):
        p.kind, p.target, p.turnover_time = FORCING_STOCHASTIC_OU, float(f.forcing_variance), float(f.correlation_time)
    elif isinstance(f, VarianceRescaling):
        if f.over not in OVER:
            raise ValueError(f"VarianceRescaling `over` must be :band or :total; got :{f.over}")
        p.kind, p.target, p.over = FORCING_VARIANCE_RESCALING, float(f.target), OVER[f.over]
    else:
        raise ValueError(f"unsupported {who} forcing {f!r}")
    p.lowest_shell = int(f.lowest_shell)
    p.highest_shell = float(f.highest_shell)


@dataclass
class Setup:
    """The run's defining parameters (`FixedDomain` + `FlowConditions` + run options)."""
    grid_points_per_axis: int
    side_length: float = 2 * math.pi
    viscosity: float = 0.01
    schmidt: float = 1.0
    scalar: bool = True
    velocity_forcing: object = field(default_factory=NoForcing)
    scalar_forcing: object = field(default_factory=NoForcing)
    mean_gradient: tuple = (0.0, 0.0, 0.0)
    precision: str = "fp64"          # "fp64" or "fp32_mixed"
    scheme: str = "IFLowStorageRK4"  # or "IFLowStorageRK3", "IFHeun", "IFSSPRK3"
    tracers: int = 0
    tracer_scheme: str = "Heun"      # "Heun" (= ABM(1)), "ABM" or "AB" (src/ParticlePropagator.jl)
    tracer_steps: int = 1            # k of ABM(k) / AB(k)
    shortened_first_steps: bool = False
    interpolation: tuple = ("CatmullRom", 4, 1)   # ("LalescuSpline", n, smoothness) or ("LagrangeSpline", n, 0)
    dealiasing: str = "TwoThirds"    # or "HouLi", "PhaseShift" (src/SimulationDomain.jl:73-177)
    houli_order: int = 36
    houli_strength: float = 0.0      # ≤ 0: −log(eps) of the precision
    tracer_gather: str = "auto"      # or "per_tracer", "warp" (16 lanes per tracer); bit-identical results
    cfl: float = 0.5
    max_dt: float = math.inf
    device: int = 0


class Run:
    """One run: `Simulation` (src/SimulationRun.jl:500-974) with its state, generator, registers,
    cache and tracers, backed by a `gbght_run` handle."""

    def __init__(self, setup: Setup, library: str | None = None):
        self.setup = setup
        self.lib = load_library(library)
        cfg = Config()
        self.lib.gbght_config_default(C.byref(cfg))
        cfg.grid_points_per_axis = int(setup.grid_points_per_axis)
        cfg.side_length = float(setup.side_length)
        cfg.precision = {"fp64": FP64, "fp32_mixed": FP32_MIXED}[setup.precision]
        if setup.scheme not in SCHEMES:
            raise ValueError(f"unknown field integration scheme {setup.scheme!r}")
        cfg.scheme = SCHEMES[setup.scheme]
        cfg.viscosity = float(setup.viscosity)
        cfg.schmidt = float(setup.schmidt)
        cfg.scalar = 1 if setup.scalar else 0
        _fill_forcing(cfg.velocity_forcing, setup.velocity_forcing, "velocity")
        _fill_forcing(cfg.scalar_forcing, setup.scalar_forcing, "scalar")
        for i in range(3):
            cfg.mean_gradient[i] = float(setup.mean_gradient[i])
        cfg.tracers = int(setup.tracers)
        if setup.tracer_scheme not in TRACER_SCHEMES:
            raise ValueError(f"unknown particle integration scheme {setup.tracer_scheme!r}")
        cfg.tracer_scheme = TRACER_SCHEMES[setup.tracer_scheme]
        cfg.tracer_steps = int(setup.tracer_steps)
        cfg.shortened_first_steps = 1 if setup.shortened_first_steps else 0
        kinds = {"CatmullRom": 0, "LalescuSpline": 1, "LagrangeSpline": 2}
        if setup.interpolation[0] not in kinds:
            raise ValueError(f"unknown interpolation scheme {setup.interpolation[0]!r}")
        cfg.interpolation = kinds[setup.interpolation[0]]
        cfg.interpolation_points = int(setup.interpolation[1])
        cfg.interpolation_smoothness = int(setup.interpolation[2])
        if setup.dealiasing not in DEALIASING:
            raise ValueError(f"unknown dealiasing strategy {setup.dealiasing!r} "
                             "(TwoThirds, HouLi and PhaseShift are built)")
        cfg.dealiasing = DEALIASING[setup.dealiasing]
        cfg.houli_order = int(setup.houli_order)
        cfg.houli_strength = float(setup.houli_strength)
        gathers = {"auto": 0, "per_tracer": 1, "warp": 2}
        if setup.tracer_gather not in gathers:
            raise ValueError(f"unknown tracer gather {setup.tracer_gather!r}")
        cfg.tracer_gather = gathers[setup.tracer_gather]
        cfg.cfl = float(setup.cfl)
        cfg.max_dt = float(setup.max_dt)
        cfg.device = int(setup.device)
        h = C.c_void_p()
        rc = self.lib.gbght_create(C.byref(h), C.byref(cfg))
        if rc != OK:
            msg = self.lib.gbght_global_error().decode()
            raise (ValueError if rc == ERR_ARGUMENT else DeviceError)(msg)
        self.h = h
        self.N = setup.grid_points_per_axis
        K = C.c_int()
        cut = C.c_double()
        self.lib.gbght_geometry(self.h, C.byref(K), C.byref(cut))
        self.K, self.cutoff = K.value, cut.value
        # StochasticOU fields: the host processes (the stationary start is drawn here)
        self.processes = {}
        for field, f in ((0, setup.velocity_forcing), (1, setup.scalar_forcing)):
            if isinstance(f, StochasticOU):
                self.processes[field] = _stochastic.OUProcess(f.forcing_variance, f.correlation_time, f.lowest_shell,
                                                              f.highest_shell, f.seed, vector=field == 0,
                                                              L=setup.side_length)

    def close(self):
        if getattr(self, "h", None):
            self.lib.gbght_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- errors -----------------------------------------------------------------------------------
    def _check(self, rc: int):
        if rc == OK:
            return
        msg = self.lib.gbght_last_error(self.h).decode()
        if rc == ERR_ARGUMENT:
            raise ValueError(msg)
        if rc == ERR_SCHEDULE:
            raise ScheduleError(msg)
        raise DeviceError(msg)

    # -- state ------------------------------------------------------------------------------------
    @property
    def spectral_shape(self):
        return (self.N, self.N, self.N // 2 + 1)

    def import_state(self, uh, phih=None):
        """ResolvedFields(û, φ̂): NumPy arrays (host memory) or CUDA tensors (device memory of the run's
        device, converted in place by the library), complex128 in the reference layout."""
        if _is_device(uh):
            if self.setup.scalar and phih is None:
                raise ValueError("this run carries a passive scalar, so phi_hat must be given")
            pu = _dev_ptr(uh, (3,) + self.spectral_shape, "u_hat")
            pp = _dev_ptr(phih, self.spectral_shape, "phi_hat") if self.setup.scalar else None
            self._check(self.lib.gbght_state_import(self.h, pu, pp))
            return
        u = np.ascontiguousarray(uh, dtype=np.complex128)
        if u.shape != (3,) + self.spectral_shape:
            raise ValueError(f"u_hat must have shape {(3,) + self.spectral_shape}")
        p = None
        if self.setup.scalar:
            if phih is None:
                raise ValueError("this run carries a passive scalar, so phi_hat must be given")
            p = np.ascontiguousarray(phih, dtype=np.complex128)
            if p.shape != self.spectral_shape:
                raise ValueError(f"phi_hat must have shape {self.spectral_shape}")
        self._check(self.lib.gbght_state_import(self.h, u.view(np.float64).ctypes.data_as(_DP),
                                                None if p is None else p.view(np.float64).ctypes.data_as(_DP)))

    def export_state(self, out=None):
        """û (and φ̂) in the reference layout. `out = (u, p)` receives them in place (contiguous
        complex128 arrays of the right shapes, e.g. in pinned memory); by default new arrays."""
        if out is not None and _is_device(out[0]):
            u, p = out
            pu = _dev_ptr(u, (3,) + self.spectral_shape, "out u")
            pp = _dev_ptr(p, self.spectral_shape, "out p") if self.setup.scalar else None
            self._check(self.lib.gbght_state_export(self.h, pu, pp))
            return u, (p if self.setup.scalar else None)
        if out is None:
            u = np.zeros((3,) + self.spectral_shape, np.complex128)
            p = np.zeros(self.spectral_shape, np.complex128) if self.setup.scalar else None
        else:
            u, p = out
            if u.dtype != np.complex128 or u.shape != (3,) + self.spectral_shape or not u.flags.c_contiguous:
                raise ValueError(f"out u must be a contiguous complex128 array of shape {(3,) + self.spectral_shape}")
            if self.setup.scalar and (p is None or p.dtype != np.complex128 or p.shape != self.spectral_shape
                                      or not p.flags.c_contiguous):
                raise ValueError(f"out p must be a contiguous complex128 array of shape {self.spectral_shape}")
            if not self.setup.scalar:
                p = None
        self._check(self.lib.gbght_state_export(self.h, u.view(np.float64).ctypes.data_as(_DP),
                                                None if p is None else p.view(np.float64).ctypes.data_as(_DP)))
        return u, p

    # -- the field step (step!, deposit!) ----------------------------------------------------------
    def set_forcing_source(self, field: int, amplitudes: np.ndarray):
        """A StochasticOU field's force for the next step (companion amplitudes, reference layout)."""
        a = np.ascontiguousarray(amplitudes, dtype=np.complex128)
        self._check(self.lib.gbght_forcing_source_set(self.h, int(field), a.view(np.float64).ctypes.data_as(_DP),
                                                      a.shape[-2]))

    def _prepare_forcing(self, dt: float):
        """`prepare_forcing!` (src/Forcing.jl:1401-1411): one OU transition of each StochasticOU
        field's process over dt, handed to the library."""
        for field, proc in self.processes.items():
            self.set_forcing_source(field, proc.advance(dt))

    def step(self, dt: float):
        self._prepare_forcing(dt)
        self._check(self.lib.gbght_step(self.h, float(dt)))

    def deposit(self):
        self._check(self.lib.gbght_deposit(self.h))

    def max_speed(self) -> float:
        v = C.c_double()
        self._check(self.lib.gbght_max_speed(self.h, C.byref(v)))
        return v.value

    def cfl_timestep(self) -> float:
        v = C.c_double()
        self._check(self.lib.gbght_cfl_timestep(self.h, C.byref(v)))
        return v.value

    def velocity_physical(self) -> np.ndarray:
        u = np.zeros((3, self.N, self.N, self.N))
        self._check(self.lib.gbght_velocity_physical_export(self.h, _ptr(u)))
        return u

    def deposit_prescribed_velocity(self, u: np.ndarray):
        a = np.ascontiguousarray(u, dtype=np.float64)
        self._check(self.lib.gbght_velocity_physical_import(self.h, _ptr(a)))

    # -- observables --------------------------------------------------------------------------------
    def observables(self) -> dict:
        out = np.zeros(4)
        self._check(self.lib.gbght_observables(self.h, _ptr(out)))
        return {"kinetic_energy": out[0], "dissipation": out[1], "scalar_variance": out[2],
                "scalar_dissipation": out[3]}

    def _spectrum(self, which: int) -> np.ndarray:
        n = C.c_int()
        self.lib.gbght_spectrum_length(self.h, C.byref(n))
        out = np.zeros(n.value)
        self._check(self.lib.gbght_spectrum(self.h, which, _ptr(out), n.value))
        return out

    def derivative_skewness(self) -> float:
        """`derivative_skewness(û, domain)` (src/Observables.jl:466-478)."""
        v = C.c_double()
        self._check(self.lib.gbght_derivative_skewness(self.h, C.byref(v)))
        return v.value

    def energy_below_scale(self):
        """`kinetic_energy_and_dissipation_below_scale(û, domain, ν)` (src/Observables.jl:253-263):
        (scales, k(l), ε(l)) for l = nL/N, n = 1..N."""
        N = self.N
        scales, k, eps = np.zeros(N), np.zeros(N), np.zeros(N)
        self._check(self.lib.gbght_energy_below_scale(self.h, _ptr(scales), _ptr(k), _ptr(eps), N))
        return scales, k, eps

    def energy_spectrum(self) -> np.ndarray:
        return self._spectrum(0)

    def scalar_spectrum(self) -> np.ndarray:
        return self._spectrum(1)

    # -- tracers (advect!, particle deposit!) -------------------------------------------------------
    def import_tracers(self, X):
        """Tracer positions (3, M): a NumPy array, or a float64 CUDA tensor read in place."""
        if _is_device(X):
            self._check(self.lib.gbght_tracers_import(self.h, _dev_ptr(X, (3, self.setup.tracers), "X", real=True)))
            return
        a = np.ascontiguousarray(X, dtype=np.float64)
        if a.shape != (3, self.setup.tracers):
            raise ValueError(f"positions must have shape (3, {self.setup.tracers})")
        self._check(self.lib.gbght_tracers_import(self.h, _ptr(a)))

    def tracers(self, out=None):
        """Tracer positions (3, M), into `out` (a float64 CUDA tensor) when given, else a new array."""
        if out is not None and _is_device(out):
            self._check(self.lib.gbght_tracers_export(self.h, _dev_ptr(out, (3, self.setup.tracers), "out", real=True)))
            return out
        X = np.zeros((3, self.setup.tracers))
        self._check(self.lib.gbght_tracers_export(self.h, _ptr(X)))
        return X

    def tracer_sample(self):
        F = np.zeros((3, self.setup.tracers))
        t = C.c_double()
        self._check(self.lib.gbght_tracer_sample_export(self.h, _ptr(F), C.byref(t)))
        return F, t.value

    def tracer_trail(self):
        """Every sample of the trail as held, oldest first: [(t, values (3, M)), ...] (what a
        checkpoint stores to restore a multistep scheme)."""
        out = []
        j = 0
        while True:
            F = np.zeros((3, self.setup.tracers))
            t = C.c_double()
            rc = self.lib.gbght_tracer_trail_export(self.h, j, _ptr(F), C.byref(t))
            if rc == ERR_ARGUMENT and j > 0:
                break
            self._check(rc)
            out.append((t.value, F))
            j += 1
        return out[::-1]

    def reset_tracer_trail(self):
        """`reset_velocity_at_particles!` (src/Cache.jl:382-386)."""
        self._check(self.lib.gbght_tracer_trail_reset(self.h))

    def restore_tracer_sample(self, values: np.ndarray, t: float):
        """`restore_velocity_at_particles!` (src/Cache.jl:388-389): push an earlier sample."""
        a = np.ascontiguousarray(values, dtype=np.float64)
        if a.shape != (3, self.setup.tracers):
            raise ValueError(f"a sample must have shape (3, {self.setup.tracers})")
        self._check(self.lib.gbght_tracer_sample_restore(self.h, _ptr(a), float(t)))

    def advect(self, dt: float):
        self._check(self.lib.gbght_advect(self.h, float(dt)))

    def deposit_tracers(self, t: float):
        self._check(self.lib.gbght_deposit_tracers(self.h, float(t)))

    def interpolate_velocity(self, X: np.ndarray) -> np.ndarray:
        a = np.ascontiguousarray(X, dtype=np.float64)
        out = np.zeros_like(a)
        self._check(self.lib.gbght_interpolate_velocity(self.h, _ptr(a), a.shape[1], _ptr(out)))
        return out

    # -- run layer (advance!) ------------------------------------------------------------------------
    def advance(self, dt: float | None = None) -> float:
        if self.processes:   # the process needs the step's Δt before the step
            dt = self.cfl_timestep() if dt is None else dt
            self._prepare_forcing(dt)
        taken = C.c_double()
        self._check(self.lib.gbght_advance(self.h, 0.0 if dt is None else float(dt), C.byref(taken)))
        return taken.value

    def clock(self):
        t = C.c_double()
        s = C.c_int64()
        self.lib.gbght_clock(self.h, C.byref(t), C.byref(s))
        return t.value, s.value

    def status_word(self) -> int:
        w = C.c_uint32()
        self._check(self.lib.gbght_status_word(self.h, C.byref(w)))
        return w.value

    def synchronize(self):
        self._check(self.lib.gbght_synchronize(self.h))

    # -- the discrete adjoint of the step (gbght_adjoint_*) ------------------------------------------
    def adjoint_create(self, snapshots: int = 0):
        """Allocate the adjoint registers and `snapshots` device state slots."""
        self._check(self.lib.gbght_adjoint_create(self.h, int(snapshots)))

    def adjoint_import(self, lam_u, lam_phi=None):
        """The cotangent λ of the state, in the state's layout (NumPy arrays or CUDA tensors)."""
        if _is_device(lam_u):
            pu = _dev_ptr(lam_u, (3,) + self.spectral_shape, "lam_u")
            pp = _dev_ptr(lam_phi, self.spectral_shape, "lam_phi") if self.setup.scalar else None
            self._check(self.lib.gbght_adjoint_import(self.h, pu, pp))
            return
        u = np.ascontiguousarray(lam_u, dtype=np.complex128)
        p = np.ascontiguousarray(lam_phi, dtype=np.complex128) if self.setup.scalar else None
        self._check(self.lib.gbght_adjoint_import(self.h, u.view(np.float64).ctypes.data_as(_DP),
                                                  None if p is None else p.view(np.float64).ctypes.data_as(_DP)))

    def adjoint_export(self):
        u = np.zeros((3,) + self.spectral_shape, np.complex128)
        p = np.zeros(self.spectral_shape, np.complex128) if self.setup.scalar else None
        self._check(self.lib.gbght_adjoint_export(self.h, u.view(np.float64).ctypes.data_as(_DP),
                                                  None if p is None else p.view(np.float64).ctypes.data_as(_DP)))
        return u, p

    def adjoint_step(self, dt: float):
        """λ ← J(q)ᵀλ for one step of size dt at the current state q (left unchanged)."""
        self._check(self.lib.gbght_adjoint_step(self.h, float(dt)))

    def adjoint_add_observable(self, which: str, weight: float):
        """λ += weight · ∂(observable)/∂state, for "kinetic_energy" or "scalar_variance"."""
        if which not in OBSERVABLES:
            raise ValueError(f"unknown observable {which!r}")
        self._check(self.lib.gbght_adjoint_add_observable(self.h, OBSERVABLES[which], float(weight)))

    def forcing_gradient(self, reset: bool = False):
        """The accumulated dL/dε of the velocity's and the scalar's ConstantPower rates."""
        out = np.zeros(2)
        self._check(self.lib.gbght_adjoint_forcing_gradient(self.h, _ptr(out), 1 if reset else 0))
        return float(out[0]), float(out[1])

    def adjoint_clear(self):
        self._check(self.lib.gbght_adjoint_clear(self.h))

    def adjoint_advance(self, dt: float):
        """The reverse of one advance! iteration (field step, Heun push, particle deposit) at the
        current state, for λ and the tracer cotangents."""
        self._check(self.lib.gbght_adjoint_advance(self.h, float(dt)))

    def adjoint_deposit_tracers(self):
        """The reverse of the particle deposit f = u(X) at the current state."""
        self._check(self.lib.gbght_adjoint_deposit_tracers(self.h))

    def adjoint_tracers_import(self, lam_X, lam_f):
        a = np.ascontiguousarray(lam_X, dtype=np.float64)
        b = np.ascontiguousarray(lam_f, dtype=np.float64)
        self._check(self.lib.gbght_adjoint_tracers_import(self.h, _ptr(a), _ptr(b)))

    def adjoint_tracers_export(self):
        a = np.zeros((3, self.setup.tracers))
        b = np.zeros((3, self.setup.tracers))
        self._check(self.lib.gbght_adjoint_tracers_export(self.h, _ptr(a), _ptr(b)))
        return a, b

    def snapshot_save(self, slot: int):
        self._check(self.lib.gbght_snapshot_save(self.h, int(slot)))

    def snapshot_load(self, slot: int):
        self._check(self.lib.gbght_snapshot_load(self.h, int(slot)))

    def selftest_wait_timeout(self, cycles: int):
        """Expire a bounded device wait on purpose (`gbght_selftest_wait_timeout`); raises the
        DeviceError a lost copy raises."""
        self._check(self.lib.gbght_selftest_wait_timeout(self.h, int(cycles)))

    def set_clock(self, time: float, step: int):
        self._check(self.lib.gbght_set_clock(self.h, float(time), int(step)))

    # -- CUDA-event timing on the run's stream ------------------------------------------------------
    def profile(self, enable: bool):
        self._check(self.lib.gbght_profile(self.h, 1 if enable else 0))

    def profile_read(self) -> dict:
        out = {}
        for k, name in enumerate(KERNELS):
            n = C.c_int64()
            ms = C.c_double()
            self._check(self.lib.gbght_profile_read(self.h, k, C.byref(n), C.byref(ms)))
            out[name] = (n.value, ms.value)
        return out

    def timer_start(self):
        self._check(self.lib.gbght_timer(self.h, 0, None))

    def timer_stop(self) -> float:
        ms = C.c_double()
        self._check(self.lib.gbght_timer(self.h, 1, C.byref(ms)))
        return ms.value


class Ensemble:
    """Runs stepped together (`gbght_ensemble_*`): `step(dt)` is `step(dt)` then `deposit()` of
    every member, one captured CUDA graph per dt on the GPU. The members stay usable runs."""

    def __init__(self, runs):
        self.runs = list(runs)
        if not self.runs:
            raise ValueError("an ensemble needs at least one member")
        self.lib = self.runs[0].lib
        arr = (C.c_void_p * len(self.runs))(*[r.h.value for r in self.runs])
        h = C.c_void_p()
        rc = self.lib.gbght_ensemble_create(C.byref(h), arr, len(self.runs))
        if rc != OK:
            raise (ValueError if rc == ERR_ARGUMENT else DeviceError)(self.lib.gbght_global_error().decode())
        self.h = h

    def step(self, dt: float):
        rc = self.lib.gbght_ensemble_step(self.h, float(dt))
        if rc != OK:
            msg = self.lib.gbght_ensemble_last_error(self.h).decode()
            raise {ERR_ARGUMENT: ValueError, ERR_SCHEDULE: ScheduleError}.get(rc, DeviceError)(msg)

    def set_batching(self, max_group):
        """Member batching: one launch per pass for each group of at most `max_group` members with
        the same kernels (True: every such member in one group), or one launch per member and pass
        (False, 0 or 1; the default)."""
        n = len(self.runs) if max_group is True else int(max_group or 0)
        if self.lib.gbght_ensemble_set_batching(self.h, n) != OK:
            raise ValueError("bad ensemble")

    def autotune(self):
        """Let the next steps time the group sizes 1, 2, 4, … (two steps each) and keep the fastest."""
        if self.lib.gbght_ensemble_autotune(self.h) != OK:
            raise DeviceError(self.lib.gbght_ensemble_last_error(self.h).decode())

    def tuning(self):
        """(group size in use, tuning done, replay milliseconds of the candidates tried so far)."""
        b, d = C.c_int(), C.c_int()
        ms = (C.c_float * 32)()
        if self.lib.gbght_ensemble_tuning(self.h, C.byref(b), C.byref(d), ms, 32) != OK:
            raise ValueError("bad ensemble")
        return b.value, bool(d.value), [v for v in ms if v > 0]

    def units(self) -> int:
        """The launching units (groups and lone members) of the last captured graph."""
        v = C.c_int()
        if self.lib.gbght_ensemble_units(self.h, C.byref(v)) != OK:
            raise ValueError("bad ensemble")
        return v.value

    def close(self):
        if getattr(self, "h", None):
            self.lib.gbght_ensemble_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def recommended_cfl(scheme: str, dealiasing: str = "TwoThirds", library: str | None = None) -> float:
    """`recommended_cfl(scheme, domain)` (src/Propagator.jl:906-919): the scheme's ceiling under the
    2/3 rule, scaled by (2/3)/f for a strategy that retains the fraction f of the Nyquist wavenumber."""
    lib = load_library(library)
    v = C.c_double()
    if scheme not in SCHEMES:
        raise ValueError(f"unknown field integration scheme {scheme!r}")
    if dealiasing not in DEALIASING:
        raise ValueError(f"unknown dealiasing strategy {dealiasing!r}")
    if lib.gbght_recommended_cfl_dealiased(SCHEMES[scheme], DEALIASING[dealiasing], C.byref(v)) != OK:
        raise ValueError(f"no CFL ceiling for {scheme!r} under {dealiasing!r}")
    return v.value


def simulation(setup: Setup, uh: np.ndarray, phih: np.ndarray | None = None, X: np.ndarray | None = None,
               library: str | None = None) -> Run:
    """Build a run and make its first deposits, as `Simulation(...)` does
    (src/SimulationRun.jl:750-931): import the state, deposit the fields, then place the tracers
    and take their first sample at t = 0."""
    run = Run(setup, library=library)
    run.import_state(uh, phih)
    run.deposit()
    if setup.tracers:
        if X is None:
            raise ValueError("a run with tracers needs their positions")
        run.import_tracers(X)
        run.deposit_tracers(0.0)
    return run

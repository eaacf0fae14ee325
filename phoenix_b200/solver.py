"""Host-side mirror of the reference's solver interface over the C ABI.

Names follow the reference:
  SystemParameters      include/system/system_parameters.hpp:22-131
  SolverFactory         include/solver/solver_factory.hpp:31-84 (keys "RK4", "DP45")
  Solver.iterate        source/cuda_solver/solver/solver.cu:22-70 (returns False once t >= t_max)
so that a caller of the reference's solver finds the same entry points.
All work happens in phoenix_b200/libphx.so on the GPU; this module only
marshals arguments and numpy arrays.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Tuple

import numpy as np

from . import _lib as L


@dataclass
class Temporal:
    """Temporal envelope of one group (envelope.hpp:63-69, envelope.cpp:466-500)."""
    kind: str = "constant"  # constant | iexp | cos | gauss
    t0: float = 0.0
    sigma: float = 0.0
    freq: float = 0.0


@dataclass
class SystemParameters:
    """The iteration's share of SystemParameters (defaults of system.cpp:18-72)."""
    N_c: int = 400
    N_r: int = 400
    L_x: float = 100.0
    L_y: float = 100.0
    h_bar_s: float = 6.582119514e-4  # hbar / e * 1e12 (calculateAuto)
    m_eff: float = 9.10938356e-31 / 1.60217662e-19 * 1e8
    gamma_c: float = 0.15
    gamma_r: float = 0.225
    g_c: float = 3e-6
    g_r: float = 6e-6
    R: float = 0.01
    g_pm: float = -6e-7
    delta_LT: float = 0.025e-3
    periodic_boundary_x: bool = False
    periodic_boundary_y: bool = False
    use_twin_mode: bool = False
    use_reservoir: bool = True
    dtype: str = "f64"  # the reference's build precision (FP64 default, FP32 with USE_32_BIT_PRECISION)
    iterator: str = "RK4"
    use_adaptive_timestep: bool = False
    tolerance: float = 0.1
    dt_min: float = 1e-4
    dt_max: float = 3.0
    fft_every: float = 1.0
    t0: float = 0.0
    t_max: float = 1000.0
    dt: float = 0.0  # 0 -> magic time step 0.5*dx*dy/scaling (calculateAuto)
    pump_temporal: List[Temporal] = field(default_factory=list)
    potential_temporal: List[Temporal] = field(default_factory=list)
    pulse_temporal: List[Temporal] = field(default_factory=list)
    norm_mode: str = "reference"  # adaptive error / imaginary-time norm: "reference" (halo-padded sums) or "interior"
    stochastic_amplitude: float = 0.0  # --dw; noise is on when > 0
    random_seed: int = 0  # key of the counter-based noise generator
    device: int = 0
    imag_time_amplitude: float = 0.0  # --imagTime A; imaginary-time propagation when != 0
    fma: bool = False  # FP32 one-kernel RK4 with fused multiply-adds (faster, not bit-identical to the reference)

    def magic_timestep(self) -> float:
        dx = self.L_x / (self.N_c - 1)
        dy = self.L_y / (self.N_r - 1)
        scaling = 9.10938356e-31 / 1.60217662e-19 * 1e8 / self.m_eff
        return 0.5 * dx * dy / scaling

    def to_abi(self) -> L.Params:
        p = L.Params()
        p.abi_version = L.ABI_VERSION
        p.N_c, p.N_r = int(self.N_c), int(self.N_r)
        p.L_x, p.L_y = float(self.L_x), float(self.L_y)
        p.h_bar_s, p.m_eff = float(self.h_bar_s), float(self.m_eff)
        p.gamma_c, p.gamma_r, p.g_c, p.g_r, p.R = (float(self.gamma_c), float(self.gamma_r), float(self.g_c),
                                                   float(self.g_r), float(self.R))
        p.g_pm, p.delta_LT = float(self.g_pm), float(self.delta_LT)
        p.periodic_x, p.periodic_y = int(bool(self.periodic_boundary_x)), int(bool(self.periodic_boundary_y))
        p.tetm, p.use_reservoir = int(bool(self.use_twin_mode)), int(bool(self.use_reservoir))
        p.dtype = L.F64 if self.dtype in ("f64", "fp64", "double") else L.F32
        key = self.iterator.upper()
        if key not in L.ITER:
            raise KeyError(f"iterator '{self.iterator}' is not registered (available: {sorted(L.ITER)})")
        p.iterator = L.ITER[key]
        p.adaptive = int(bool(self.use_adaptive_timestep))
        p.norm_mode = L.NORM_REFERENCE if self.norm_mode == "reference" else L.NORM_INTERIOR
        p.dt = float(self.dt) if self.dt > 0 else self.magic_timestep()
        p.t0, p.t_max = float(self.t0), float(self.t_max)
        p.tol, p.dt_min, p.dt_max = float(self.tolerance), float(self.dt_min), float(self.dt_max)
        p.fft_every = float(self.fft_every)
        p.stochastic_amplitude = float(self.stochastic_amplitude)
        p.seed = int(self.random_seed) & 0xFFFFFFFFFFFFFFFF
        p.imag_time_amplitude = float(self.imag_time_amplitude)
        p.n_pump_groups = len(self.pump_temporal)
        p.n_potential_groups = len(self.potential_temporal)
        p.n_pulse_groups = len(self.pulse_temporal)
        p.device = int(self.device)
        p.fma = int(bool(self.fma))
        return p


class Solver:
    """One simulation on one GPU (the reference's Solver for one subgrid layout)."""

    def __init__(self, system: SystemParameters):
        self.system = system
        self._lib = L.load()
        self._h = C.c_void_p()
        p = system.to_abi()
        L.check(self._lib.phx_create(C.byref(p), C.byref(self._h)), None)
        for fam, specs in (("pump", system.pump_temporal), ("potential", system.potential_temporal),
                           ("pulse", system.pulse_temporal)):
            for g, s in enumerate(specs):
                L.check(self._lib.phx_set_temporal(self._h, L.ENVELOPE[fam], g, L.TEMPORAL[s.kind], float(s.t0),
                                                   float(s.sigma), float(s.freq)), self._h)
        self.iteration = 0
        self.last_info = L.StepInfo()

    # -- lifetime
    def close(self):
        if self._h:
            self._lib.phx_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- fields
    def _shape(self):
        return int(self.system.N_r), int(self.system.N_c)

    def _host_types(self):
        f32 = self.system.dtype not in ("f64", "fp64", "double")
        return (np.complex64, np.float32, L.F32) if f32 else (np.complex128, np.float64, L.F64)

    def set_field(self, name: str, values, group: int = 0):
        """Upload a full N_r x N_c field.  Arrays already in the build precision
        (complex64 / float32 for FP32) are copied without conversion; pinned
        host memory then goes straight to the device by DMA."""
        fid = L.FIELDS[name]
        a = np.asarray(values)
        if a.shape != self._shape():
            raise ValueError(f"{name}: expected shape {self._shape()}, got {a.shape}")
        ctype, rtype, code = self._host_types()
        if name in L.COMPLEX_FIELDS:
            buf = np.ascontiguousarray(a, dtype=ctype).view(rtype)
        else:
            buf = np.ascontiguousarray(np.real(a), dtype=rtype)
        L.check(self._lib.phx_set_field(self._h, fid, group, buf.ctypes.data_as(C.c_void_p), buf.size, code), self._h)

    def get_field(self, name: str, group: int = 0, out=None):
        """Download a field (complex64 / float32 for FP32 builds, complex128 /
        float64 for FP64); `out` may be a preallocated array of that type."""
        fid = L.FIELDS[name]
        cplx = name in L.COMPLEX_FIELDS
        ctype, rtype, code = self._host_types()
        want = ctype if cplx else rtype
        if out is None:
            out = np.empty(self._shape(), dtype=want)
        if out.shape != self._shape() or out.dtype != want or not out.flags.c_contiguous:
            raise ValueError(f"{name}: out must be a C-contiguous {np.dtype(want).name} array of shape {self._shape()}")
        view = out.view(rtype)
        L.check(self._lib.phx_get_field(self._h, fid, group, view.ctypes.data_as(C.c_void_p), view.size, code), self._h)
        return out

    # -- device tensors (torch), no host round trip
    def _check_tensor(self, name, t):
        import torch

        cplx = name in L.COMPLEX_FIELDS
        f32 = self.system.dtype not in ("f64", "fp64", "double")
        want = (torch.complex64 if f32 else torch.complex128) if cplx else (torch.float32 if f32 else torch.float64)
        if t.dtype != want or tuple(t.shape) != self._shape() or not t.is_contiguous() or not t.is_cuda:
            raise ValueError(f"{name}: expected a contiguous CUDA {want} tensor of shape {self._shape()}")
        return (2 if cplx else 1) * t.numel()

    def _order_after_torch(self):
        import torch

        s = torch.cuda.ExternalStream(self.stream)
        s.wait_stream(torch.cuda.current_stream())

    def _order_torch_after(self):
        import torch

        torch.cuda.current_stream().wait_stream(torch.cuda.ExternalStream(self.stream))

    def set_field_tensor(self, name: str, tensor, group: int = 0):
        """Upload from a torch CUDA tensor (build precision, C-contiguous)."""
        n = self._check_tensor(name, tensor)
        self._order_after_torch()
        L.check(self._lib.phx_set_field_device(self._h, L.FIELDS[name], group, C.c_void_p(tensor.data_ptr()), n),
                self._h)

    def get_field_tensor(self, name: str, group: int = 0, out=None):
        """Download into a torch CUDA tensor (allocated when `out` is None)."""
        import torch

        cplx = name in L.COMPLEX_FIELDS
        f32 = self.system.dtype not in ("f64", "fp64", "double")
        dt = (torch.complex64 if f32 else torch.complex128) if cplx else (torch.float32 if f32 else torch.float64)
        if out is None:
            out = torch.empty(self._shape(), dtype=dt, device=f"cuda:{self.system.device}")
        n = self._check_tensor(name, out)
        self._order_after_torch()
        L.check(self._lib.phx_get_field_device(self._h, L.FIELDS[name], group, C.c_void_p(out.data_ptr()), n),
                self._h)
        self._order_torch_after()
        return out

    # -- adjoint
    def adjoint_forward(self, iterations: int, checkpoint_every: int = 0):
        """Run `iterations` RK4 iterations keeping checkpoints (default every ceil(sqrt(iterations)))."""
        self._order_after_torch()
        L.check(self._lib.phx_adjoint_forward(self._h, C.c_int64(iterations), C.c_int64(checkpoint_every)), self._h)
        self._order_torch_after()

    def adjoint_backward(self, dpsi_T, dn_T=None, want_psi0=True, want_n0=True, want_pump=True, want_potential=False):
        """dL/d(final state) -> (dL/dpsi_0, dL/dn_0, dL/dP, dL/dV) as torch CUDA
        tensors (None where not wanted; dL/dV needs a potential group)."""
        import torch

        f32 = self.system.dtype not in ("f64", "fp64", "double")
        cdt, rdt = (torch.complex64, torch.float32) if f32 else (torch.complex128, torch.float64)
        dev = dpsi_T.device
        self._check_tensor("psi_plus", dpsi_T)
        if dn_T is not None:
            self._check_tensor("n_plus", dn_T)
        g_psi = torch.empty(self._shape(), dtype=cdt, device=dev) if want_psi0 else None
        g_n = torch.empty(self._shape(), dtype=rdt, device=dev) if want_n0 and self.system.use_reservoir else None
        g_p = torch.empty(self._shape(), dtype=rdt, device=dev) if want_pump else None
        g_v = torch.empty(self._shape(), dtype=rdt, device=dev) if want_potential else None
        ptr = lambda t: C.c_void_p(t.data_ptr()) if t is not None else None  # noqa: E731
        self._order_after_torch()
        L.check(self._lib.phx_adjoint_backward(self._h, ptr(dpsi_T), ptr(dn_T), ptr(g_psi), ptr(g_n), ptr(g_p),
                                               ptr(g_v)), self._h)
        self._order_torch_after()
        return g_psi, g_n, g_p, g_v

    # -- time
    @property
    def t(self) -> float:
        t, dt = C.c_double(), C.c_double()
        L.check(self._lib.phx_get_time(self._h, C.byref(t), C.byref(dt)), self._h)
        return t.value

    @property
    def dt(self) -> float:
        t, dt = C.c_double(), C.c_double()
        L.check(self._lib.phx_get_time(self._h, C.byref(t), C.byref(dt)), self._h)
        return dt.value

    def set_time(self, t: float, dt: float):
        L.check(self._lib.phx_set_time(self._h, float(t), float(dt)), self._h)

    # -- iteration
    def run(self, max_iterations: int = 1 << 62) -> L.StepInfo:
        """iterate() until t >= t_max or max_iterations calls; returns the step record."""
        info = L.StepInfo()
        L.check(self._lib.phx_step(self._h, C.c_int64(max_iterations), C.byref(info)), self._h)
        self.iteration += info.iterations
        self.last_info = info
        return info

    def iterate(self) -> bool:
        """One Solver::iterate call; False when t >= t_max (solver.cu:30-33)."""
        return self.run(1).iterations == 1

    def sum_abs2(self, name: str = "psi_plus") -> float:
        out = C.c_double()
        L.check(self._lib.phx_sum_abs2(self._h, L.FIELDS[name], C.byref(out)), self._h)
        return out.value

    def profile(self, enable: bool = True):
        """Bracket every kernel launch with CUDA events (resets the totals)."""
        L.check(self._lib.phx_profile_enable(self._h, int(bool(enable))), self._h)

    def profile_read(self) -> Dict[str, dict]:
        """Per kernel family: device ms, launches and algorithmic HBM bytes since profile()."""
        out = {}
        for name, k in L.KERNEL_KINDS.items():
            ms, n, b = C.c_double(), C.c_int64(), C.c_double()
            L.check(self._lib.phx_profile_read(self._h, k, C.byref(ms), C.byref(n), C.byref(b)), self._h)
            if n.value:
                out[name] = {"ms": ms.value, "launches": n.value, "bytes": b.value}
        return out

    def request_abort(self):
        """Ask a phx_step running in another thread to stop before its next
        iteration (it then raises PhxError with PHX_ERR_ABORTED)."""
        L.check(self._lib.phx_request_abort(self._h), self._h)

    def set_wait_limit(self, polls: int):
        """Bound of the one-kernel iteration's wait for a tile's data, in polls
        (< 0: the default; 0: every such wait gives up at once)."""
        L.check(self._lib.phx_set_wait_limit(self._h, int(polls)), self._h)

    def tune_report(self) -> Dict[int, float]:
        """Launch shape -> median device microseconds per iteration, as timed
        by the autotuner (empty before tuning has ended)."""
        cap = 32
        shapes, meds, n = (C.c_int32 * cap)(), (C.c_double * cap)(), C.c_int32()
        L.check(self._lib.phx_tune_read(self._h, cap, shapes, meds, C.byref(n)), self._h)
        return {int(shapes[i]): float(meds[i]) for i in range(min(cap, n.value))}

    @property
    def stream(self) -> int:
        s = C.c_void_p()
        L.check(self._lib.phx_get_stream(self._h, C.byref(s)), self._h)
        return s.value or 0

    def device_ptr(self, name: str, group: int = 0) -> Tuple[int, int]:
        ptr, pitch = C.c_void_p(), C.c_int64()
        L.check(self._lib.phx_field_device_ptr(self._h, L.FIELDS[name], group, C.byref(ptr), C.byref(pitch)), self._h)
        return ptr.value, pitch.value


class SolverFactory:
    """REGISTER_SOLVER keys of the reference (source/cuda_solver/solver/iterator/*.cu), matched
    case-insensitively like the CLI's --iterator."""
    registry: Dict[str, Tuple[bool, str]] = {
        "RK4": (False, "Runge-Kutta 4"),
        "DP45": (True, "Dormand-Prince 5(4) method for time integration."),
        "RK3": (False, "Runge-Kutta 3"),
        "SSPRK3": (False, "Strong Stability Preserving Runge Kutta 3"),
        "MP": (False, "MidPoint"),
        "HEUN2": (False, "Heun2"),
        "HEUN3": (False, "Heun3"),
        "HW": (False, "Houwen-Wray"),
        "NEWTON": (False, "Newton"),
        "NYSTROEM": (False, "Nystroem's fifth-order method"),
        "RALSTON": (False, "Ralston 2nd order method for time integration."),
        "RALSTON3": (False, "Ralston 3rd order method for time integration."),
        "RALSTON4": (False, "Ralston 4th order method for time integration."),
        "RULE38": (False, "Third-order Runge-Kutta method (3/8 rule)"),
        "BOSHA": (True, "Bogacki-Shampine 3(2)"),
        "CASHKARP": (True, "Cash-Karp 5(4)"),
        "FEHLBERG2": (True, "Fehlberg 2(1) order method for time integration."),
        "FEHLBERG5": (True, "Fehlberg 5(4) order method for time integration."),
        "DP85": (True, "Dormand–Prince 8(5) method for time integration."),
        "NSRK78": (True, "Nullspace RK 13-stage 8th order"),
        "SSFM": (False, "Split Step Fourier Method"),
    }

    @classmethod
    def available(cls):
        return sorted(cls.registry)

    @classmethod
    def create(cls, system: SystemParameters) -> Solver:
        key = system.iterator.upper()
        if key not in cls.registry:
            raise KeyError(f"Solver '{system.iterator}' not registered")
        is_adaptive = cls.registry[key][0]
        if system.use_adaptive_timestep and not is_adaptive:
            # solver.cu:23-26: adaptive stepping silently falls back to fixed
            system.use_adaptive_timestep = False
        return Solver(system)


def system_from_case(case: dict, **overrides) -> SystemParameters:
    """SystemParameters for a golden-fixture case dictionary (tests/golden/make_golden.py)."""
    def temporal(specs, n):
        out = []
        for g in range(n):
            s = specs[g] if specs and g < len(specs) else None
            out.append(Temporal() if s is None else Temporal(s[0], float(s[1]), float(s[2]), float(s[3])))
        return out

    npump = len(case.get("pumps", []))
    sp = SystemParameters(
        N_c=case["N_c"], N_r=case["N_r"], L_x=case["L_x"], L_y=case["L_y"], h_bar_s=case["h_bar_s"],
        m_eff=case["m_eff"], gamma_c=case["gamma_c"], gamma_r=case["gamma_r"], g_c=case["g_c"], g_r=case["g_r"],
        R=case["R"], g_pm=case["g_pm"], delta_LT=case["delta_LT"], periodic_boundary_x=bool(case["periodic_x"]),
        periodic_boundary_y=bool(case["periodic_y"]), use_twin_mode=bool(case.get("tetm", 0)),
        use_reservoir=bool(npump > 0 or case.get("n0_amp", 0.0)), dtype=case["dtype"], iterator=case["iterator"],
        use_adaptive_timestep=bool(case.get("adaptive", 0)), tolerance=case.get("tol", 0.1),
        dt_min=case.get("dt_min", 1e-4), dt_max=case.get("dt_max", 3.0), fft_every=case.get("fft_every", 1e9),
        t0=case.get("t0", 0.0), t_max=case["t_max"], dt=case["dt"],
        stochastic_amplitude=case.get("dw", 0.0), random_seed=case.get("seed", 0),
        imag_time_amplitude=case.get("imag_time", 0.0),
        pump_temporal=temporal(case.get("pump_t"), npump),
        potential_temporal=temporal(case.get("potential_t"), len(case.get("potentials", []))),
        pulse_temporal=temporal(case.get("pulse_t"), len(case.get("pulses", []))))
    for k, v in overrides.items():
        setattr(sp, k, v)
    return sp


def load_case_fields(solver: Solver, case: dict, fields: dict):
    """Upload the input fields of a golden case into a solver."""
    comps = ["plus", "minus"] if case.get("tetm") else ["plus"]
    for comp in comps:
        solver.set_field(f"psi_{comp}", fields[f"psi_{comp}"])
        if solver.system.use_reservoir:
            solver.set_field(f"n_{comp}", np.real(fields.get(f"n_{comp}", np.zeros(solver._shape()))))
    for g in range(len(case.get("pumps", []))):
        for comp in comps:
            solver.set_field(f"pump_{comp}", np.real(fields[f"pump_{g}"]), g)
    for g in range(len(case.get("potentials", []))):
        for comp in comps:
            solver.set_field(f"potential_{comp}", np.real(fields[f"potential_{g}"]), g)
    for g in range(len(case.get("pulses", []))):
        for comp in comps:
            solver.set_field(f"pulse_{comp}", fields[f"pulse_{g}"], g)
    if "fft_mask" in fields:
        for comp in comps:
            solver.set_field(f"fft_mask_{comp}", np.real(fields["fft_mask"]))

"""Batches of independent RK4 simulations (pump-power sweeps, disorder
realisations) advanced together on one GPU.

The reference runs one simulation per process (source/main.cu:80-117); a
sweep over n parameter sets is n runs of that main loop.  `BatchSolver`
holds n instances -- each with its own grid size, physical parameters,
boundary conditions, pump, potential and initial state -- and advances all
of them by one RK4 iteration per batch iteration, in one launch of a
persistent kernel over the tiles of every instance.  Every instance's
result is bit-identical to a single-simulation `Solver` of the same
instance.

Instances are scalar, fixed-step RK4, with at most one pump and one
potential group (constant in time), no pulse, no k-space filter and no
noise; all share one dtype, one device and the use_reservoir flag.
"""
from __future__ import annotations

import ctypes as C
from typing import List, Sequence

import numpy as np

from . import _lib as L
from .solver import SystemParameters


class BatchSolver:
    def __init__(self, systems: Sequence[SystemParameters]):
        if not systems:
            raise ValueError("a batch needs at least one instance")
        self.systems: List[SystemParameters] = list(systems)
        self._lib = L.load()
        self._b = C.c_void_p()
        arr = (L.Params * len(self.systems))(*[s.to_abi() for s in self.systems])
        L.check_batch(self._lib.phx_batch_create(arr, len(self.systems), C.byref(self._b)), None)
        self.iteration = 0
        self.last_info = L.StepInfo()

    def __len__(self):
        return len(self.systems)

    # -- lifetime
    def close(self):
        if self._b:
            self._lib.phx_batch_destroy(self._b)
            self._b = C.c_void_p()

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
    def _types(self, i):
        self._shape(i)
        f32 = self.systems[i].dtype not in ("f64", "fp64", "double")
        return (np.complex64, np.float32, L.F32) if f32 else (np.complex128, np.float64, L.F64)

    def _shape(self, i):
        if not 0 <= i < len(self.systems):
            raise IndexError(f"instance {i} out of range (batch of {len(self.systems)})")
        return int(self.systems[i].N_r), int(self.systems[i].N_c)

    def set_field(self, i: int, name: str, values, group: int = 0):
        """Upload a full N_r x N_c field of instance i (see Solver.set_field)."""
        a = np.asarray(values)
        if a.shape != self._shape(i):
            raise ValueError(f"instance {i} {name}: expected shape {self._shape(i)}, got {a.shape}")
        ctype, rtype, code = self._types(i)
        if name in L.COMPLEX_FIELDS:
            buf = np.ascontiguousarray(a, dtype=ctype).view(rtype)
        else:
            buf = np.ascontiguousarray(np.real(a), dtype=rtype)
        L.check_batch(self._lib.phx_batch_set_field(self._b, i, L.FIELDS[name], group, buf.ctypes.data_as(C.c_void_p),
                                                    buf.size, code), self._b)

    def get_field(self, i: int, name: str, group: int = 0):
        ctype, rtype, code = self._types(i)
        out = np.empty(self._shape(i), dtype=ctype if name in L.COMPLEX_FIELDS else rtype)
        view = out.view(rtype)
        L.check_batch(self._lib.phx_batch_get_field(self._b, i, L.FIELDS[name], group, view.ctypes.data_as(C.c_void_p),
                                                    view.size, code), self._b)
        return out

    # -- iteration
    def run(self, iterations: int) -> L.StepInfo:
        """Advance every instance by `iterations` RK4 iterations (t_max is not consulted)."""
        info = L.StepInfo()
        L.check_batch(self._lib.phx_batch_step(self._b, C.c_int64(iterations), C.byref(info)), self._b)
        self.iteration += info.iterations
        self.last_info = info
        return info

    def time(self, i: int):
        t, dt = C.c_double(), C.c_double()
        L.check_batch(self._lib.phx_batch_get_time(self._b, i, C.byref(t), C.byref(dt)), self._b)
        return t.value, dt.value

    @property
    def stream(self) -> int:
        s = C.c_void_p()
        L.check_batch(self._lib.phx_batch_get_stream(self._b, C.byref(s)), self._b)
        return s.value or 0

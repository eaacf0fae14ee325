"""Benchmark: microseconds per RK4 iteration of the scalar polariton GP equation
with reservoir on a 1024 x 1024 grid (FP32 by default), one replica per GPU.

Workload (synthetic, seeded): 1024^2 periodic box of 100 um, hbar = 0.6582 meV ps,
m_eff = 5.6e-4 m_e (3.1840 meV ps^2/um^2), gamma_c 0.15/ps, gamma_r 0.225/ps,
g_c 6e-6, g_r 1.2e-5 meV um^2, R 0.01 ps^-1 um^2, dt 0.02 ps; Gaussian pump of
width 10 um at 1.5x threshold; disorder potential (white noise smoothed to
1 um correlation, 0.1 meV rms); k-space super-Gaussian mask (order 4, cutoff
0.8 k_max) applied every 100 iterations; psi0 complex white noise of
amplitude 1e-2, n0 = 0.

Legs of the JSON line:
  value      device time per iteration (CUDA events on the solver's stream),
             L2 flushed (256 MiB write, then read) between timed iterations, max
             over ranks; the library's own per-launch events are off in this pass
  e2e        the same workload through the public API with host buffers:
             upload psi0/n0 from pinned host memory, run in chunks of 100
             iterations reading the FP64 norm back after each chunk, download
             psi and n into pinned host memory at the end (after one untimed
             pass of the same sequence on the same handle and buffers)
  roofline   the dominant kernel (the one-kernel RK4 iteration) from per-launch
             CUDA events the library records on its stream during a second,
             identical timed pass: algorithmic bytes / average duration vs the
             measured HBM peak
  fma        the same workload and timing with phx_params.fma = 1 (FP32)
  autotune   the launch shape the library's tuner kept and its per-shape medians
  cpu_baseline  the reference's CPU build (PHOENIX compiled from its sources,
             oracle/_ref) on a bounded sample of the same workload, all host cores
  sweep      the batched sweep: 256 independent 128^2..1024^2 FP32 instances
             (pump 0.8-3.0x threshold, own disorder each) advanced by one
             batch launch per iteration, against the same instances run one
             after another through single-simulation handles
  adjoint    the inverse-design gradient: 512^2 FP32, 500 RK4 iterations, device
             time of the plain forward, the checkpointed forward and the backward
  configs    the other configurations: 256^2 FP64 RK4, 1024^2 FP64 RK4 and DP45
             adaptive (FP32, FP64), 4096^2 TE/TM FP32 with noise and without, each
             beside the reference's own CUDA build (marginal time per iteration),
             and the FP32-vs-FP64 error of every configuration at its own size
`--impl reference` runs that reference CPU build alone (rank 0 of any launch).
"""
from __future__ import annotations

import argparse
import json
import os
import re
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_DEFAULT = 1024
L_BOX = 100.0
PHYS = dict(h_bar_s=0.6582, m_eff=3.1840, gamma_c=0.15, gamma_r=0.225, g_c=6e-6, g_r=1.2e-5, R=0.01)
DT_1024 = 0.02  # ps; RK4 stability at 1024^2 with m_eff = 5.6e-4 m_e needs dt < 0.033


def dt_for(n):
    """0.02 ps at 1024^2, scaled with dx^2 for other grids (0.00125 ps at 4096^2)."""
    return min(0.04, DT_1024 * (1024.0 / n) ** 2)


DT = DT_1024
MASK_EVERY = 100
P_TH = 0.15 * 0.225 / 0.01
METRIC = "us_per_rk4_iteration_1024x1024"


def rk4_alg_bytes_per_point(esz, has_pot=True):
    """Algorithmic HBM bytes of one RK4 iteration per grid point when each
    stage is one fused kernel: stage 1 reads y0 and the coefficient fields and
    writes y1 and the accumulator A; stages 2 and 3 read y_s, y0, A and the
    coefficients and write y_{s+1} and A; stage 4 reads y3, y0, A and the
    coefficients and writes y_new (psi complex, n real, pump and potential
    real).  FP32 with a potential: 236 B (220 without); FP64: 472 (440)."""
    state = 3 * esz
    coef = esz * (2 if has_pot else 1)
    first = state + coef + 2 * state
    mid = 3 * state + coef + 2 * state
    last = 3 * state + coef + state
    return first + 2 * mid + last
REF_BIN = os.path.join(ROOT, "oracle", "_ref")
KERNEL_NAMES = {"rk4_fused": "rk4_fused_kernel / rk4_tma_kernel (whole RK4 iteration)",
                "rk4_mid": "stage_scalar_kernel<kRk4Mid>", "rk4_first": "stage_scalar_kernel<kRk4First>",
                "rk4_last": "stage_scalar_kernel<kRk4Last>"}


def workload(n, seed=2):
    rng = np.random.default_rng(seed)
    x = -L_BOX / 2 + L_BOX / (n - 1) * np.arange(n)
    X, Y = np.meshgrid(x, x)
    psi0 = 1e-2 * (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n)))
    pump = 1.5 * P_TH * np.exp(-(X ** 2 + Y ** 2) / (2 * 10.0 ** 2))
    noise = np.random.default_rng(3).standard_normal((n, n))
    k = 2 * np.pi * np.fft.fftfreq(n, d=L_BOX / (n - 1))
    KX, KY = np.meshgrid(k, k)
    pot = np.real(np.fft.ifft2(np.fft.fft2(noise) * np.exp(-(KX ** 2 + KY ** 2) * 1.0 ** 2 / 2)))
    pot *= 0.1 / np.sqrt(np.mean(pot ** 2))
    loc = -1.0 + 2.0 * np.arange(n) / (n - 1)
    LX, LY = np.meshgrid(loc, loc)
    mask = np.exp(-((0.5 * ((LX / 0.8) ** 2 + (LY / 0.8) ** 2)) ** 4))
    return dict(psi0=psi0, pump=pump, potential=pot, mask=mask)


def system(pb, n, dtype, device):
    dt = dt_for(n)
    return pb.SystemParameters(N_c=n, N_r=n, L_x=L_BOX, L_y=L_BOX, **PHYS, periodic_boundary_x=True,
                               periodic_boundary_y=True, dtype=dtype, iterator="RK4", dt=dt, t0=0.0, t_max=1e12,
                               fft_every=MASK_EVERY * dt * (1 - 1e-6), pump_temporal=[pb.Temporal()],
                               potential_temporal=[pb.Temporal()], device=device)


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    def __init__(self, index):
        self.index = index
        self.rows = []
        self.proc = None

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={q}", "--format=csv,noheader,nounits", "-lms",
                                          "100", "-i", str(self.index)], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([c.strip() for c in line.split(",")])

    def __exit__(self, *exc):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if len(r) > 2 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) > 2 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows if len(r) >= 9 for i in range(4) if "Active" in r[5 + i]
                          and "Not" not in r[5 + i]})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def write_txt(path, arr, digits=9):
    arr = np.asarray(arr)
    n_r, n_c = arr.shape
    with open(path, "w") as f:
        f.write(f"# SIZE {n_c} {n_r} {L_BOX} {L_BOX} {L_BOX / (n_c - 1)} {L_BOX / (n_r - 1)} :: PHOENIX_ MATRIX\n")
        np.savetxt(f, np.real(arr), fmt=f"%.{digits}g")
        if np.iscomplexobj(arr):
            np.savetxt(f, np.imag(arr), fmt=f"%.{digits}g")


def reference_binary(dtype, gpu):
    """The reference build for a precision: its CUDA build for sm_100 (gpu), else
    its CPU build (-march=x86-64-v3 when present)."""
    variant = "fp32" if dtype == "f32" else "fp64"
    if gpu:
        cand = [os.path.join(REF_BIN, f"phoenix_gpu_{variant}")]
    else:
        cand = [os.path.join(REF_BIN, f"phoenix_cpu_{variant}_v3"), os.path.join(REF_BIN, f"phoenix_cpu_{variant}")]
    return next((b for b in cand if os.path.exists(b)), None)


_RUNTIME = re.compile(r"Total Runtime:\s*([0-9.eE+-]+)\s*s\s*-->.*?-->.*?-->\s*([0-9.eE+-]+)\s*mus/it")


def reference_marginal(dtype, n, dt, t_lo, t_hi, loads=(), extra=(), gpu=False, fft_every=1e9, subgrids=None,
                       phys=None):
    """Marginal cost per iteration of the reference's main loop: the same run to
    t_lo and to t_hi, (runtime_hi - runtime_lo) / (iterations_hi - iterations_lo)
    from its `Total Runtime ... mus/it` line, so that set-up, the first
    iterations and exit cancel.  An untimed run to t_lo goes first, so that
    neither timed run is the first on a cold device or page cache.  loads: (flag, array, component) inputs written
    as PHOENIX text matrices.  CPU build: every host core.  Returns a dict or
    None when the build is missing or a run fails."""
    binary = reference_binary(dtype, gpu)
    if binary is None:
        return None
    cores = os.cpu_count() or 1
    ph = dict(PHYS, **(phys or {}))
    runs = []
    with tempfile.TemporaryDirectory() as tmp:
        largs = []
        for k, (flag, arr, comp) in enumerate(loads):
            path = os.path.join(tmp, f"in{k}.txt")
            write_txt(path, arr)
            largs += [flag, "load", path, "1", "add", comp]
        for t_max in (t_lo, t_lo, t_hi):
            args = [binary, "--N", str(n), str(n), "--L", str(L_BOX), str(L_BOX), "--dt", repr(dt),
                    "--tmax", repr(t_max), "--outEvery", "1e9", "--output", "none", "--path",
                    os.path.join(tmp, "out"), "--threads", str(cores), "--boundary", "periodic", "periodic",
                    "--hbarscaled", str(ph["h_bar_s"]), "--meff", str(ph["m_eff"]), "--gammaC", str(ph["gamma_c"]),
                    "--gammaR", str(ph["gamma_r"]), "--gc", str(ph["g_c"]), "--gr", str(ph["g_r"]), "--R",
                    str(ph["R"]), "--fftEvery", repr(fft_every)] + largs + list(extra)
            if subgrids:
                args += ["--subgrids", str(subgrids), str(subgrids)]
            proc = subprocess.run(args, capture_output=True, text=True, timeout=1800)
            m = _RUNTIME.search(proc.stdout)
            if proc.returncode != 0 or not m or float(m.group(2)) <= 0:
                return None
            total = float(m.group(1))
            runs.append((total, round(total / float(m.group(2)) * 1e6)))
    (s_lo, k_lo), (s_hi, k_hi) = runs[1], runs[2]
    if k_hi <= k_lo:
        return None
    return {"us_per_iteration": (s_hi - s_lo) / (k_hi - k_lo) * 1e6, "iterations": [k_lo, k_hi],
            "whole_run_us_per_iteration": s_hi / k_hi * 1e6, "cores": cores, "binary": os.path.basename(binary)}


def scalar_loads(wl, mask=True, potential=True):
    loads = [("--initState", wl["psi0"], "both"), ("--pump", wl["pump"], "both")]
    if potential:
        loads.append(("--potential", wl["potential"], "both"))
    if mask:
        loads.append(("--fftMask", wl["mask"], "both"))
    return loads


def reference_cpu_run(n, dtype, iters, wl):
    """The reference CPU build on the 1024^2 workload (mask every 100
    iterations): marginal microseconds per RK4 iteration over `iters`
    iterations beyond the first 100, all host cores; (us, cores, what) or None."""
    dt = dt_for(n)
    r = reference_marginal(dtype, n, dt, 100 * dt * (1 - 1e-9), (100 + iters) * dt * (1 - 1e-9), scalar_loads(wl),
                           fft_every=MASK_EVERY * dt * (1 - 1e-6))
    if r is None:
        return None
    return r["us_per_iteration"], r["cores"], f"{r['binary']} (iterations {r['iterations'][0]} and " \
                                              f"{r['iterations'][1]}, difference of the two runs)"


def oracle_port_run(n, dtype, iters, wl):
    """Fallback CPU baseline: the C restatement (single thread)."""
    from oracle import phx_oracle as O

    case = dict(N_c=n, N_r=n, L_x=L_BOX, L_y=L_BOX, **PHYS, g_pm=0.0, delta_LT=0.0, dtype=dtype, iterator="RK4",
                dt=dt_for(n), t_max=1e12, periodic_x=1, periodic_y=1, pumps=[(0, 0, 0)], potentials=[0.0],
                mask_cut=0.8, fft_every=MASK_EVERY * dt_for(n) * (1 - 1e-6))
    fields = {"psi_plus": wl["psi0"], "pump_0": wl["pump"], "potential_0": wl["potential"], "fft_mask": wl["mask"]}
    t0 = time.perf_counter()
    O.run(case, fields, max_steps=iters)
    return (time.perf_counter() - t0) / iters * 1e6, 1, "oracle/phx_oracle.c"


def run_reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    n = args.n
    wl = workload(n)
    iters = max(100, min(args.steps + args.warmup, args.ref_iters))
    res = reference_cpu_run(n, args.dtype, iters, wl)
    kind = "reference"
    if res is None:
        res = oracle_port_run(n, args.dtype, max(2, iters // 20), wl)
        kind = "port"
    us, cores, what = res
    line = {"metric": METRIC, "value": us, "unit": "us/iter", "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": us / 1e3, "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": args.dtype, "data": "synthetic",
            "config": config_dict(args),
            "cpu_baseline": {"value": us, "unit": "us/iter", "cores": cores, "kind": kind,
                             "sample": f"{iters} RK4 iterations of the {n}^2 workload beyond its first 100 "
                                       f"with {what}"},
            "e2e": {"value": us, "unit": "us/iter", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


SWEEP_SIZES = (128, 256, 512, 1024)


def sweep_instances(count, seed=4):
    """Config of the batched sweep: `count` independent instances, grid sizes
    uniform over {128, 256, 512, 1024}^2, pump uniform in 0.8-3.0x threshold,
    own disorder realisation of 0.05-0.2 meV rms (1 um correlation) each."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(count):
        n = int(rng.choice(SWEEP_SIZES))
        p = float(rng.uniform(0.8, 3.0)) * P_TH
        rms = float(rng.uniform(0.05, 0.2))
        r = np.random.default_rng([seed, k])
        x = -L_BOX / 2 + L_BOX / (n - 1) * np.arange(n)
        X, Y = np.meshgrid(x, x)
        kk = 2 * np.pi * np.fft.fftfreq(n, d=L_BOX / (n - 1))
        KX, KY = np.meshgrid(kk, kk)
        pot = np.real(np.fft.ifft2(np.fft.fft2(r.standard_normal((n, n))) * np.exp(-(KX ** 2 + KY ** 2) / 2)))
        pot *= rms / np.sqrt(np.mean(pot ** 2))
        psi0 = 1e-2 * (r.standard_normal((n, n)) + 1j * r.standard_normal((n, n)))
        out.append(dict(n=n, pump_factor=p / P_TH, rms=rms, psi0=psi0.astype(np.complex64),
                        pump=(p * np.exp(-(X ** 2 + Y ** 2) / (2 * 10.0 ** 2))).astype(np.float32),
                        potential=pot.astype(np.float32)))
    return out


def sweep_system(pb, n, device):
    return pb.SystemParameters(N_c=n, N_r=n, L_x=L_BOX, L_y=L_BOX, **PHYS, periodic_boundary_x=True,
                               periodic_boundary_y=True, dtype="f32", iterator="RK4", dt=dt_for(n), t0=0.0,
                               t_max=1e12, pump_temporal=[pb.Temporal()], potential_temporal=[pb.Temporal()],
                               device=device)


def run_sweep(pb, torch, count, steps, device):
    """Batched sweep vs the same instances run one after another through
    single-simulation handles.  Both advance WARM + steps iterations from the
    same inputs (WARM covers the batch's launch-shape autotuning; the single
    handles start tuned); the timed part is `steps` iterations, CUDA events
    on the solvers' streams.
    Every instance's final psi and n are compared bit for bit."""
    warm = 36  # batch: 20 tuning iterations + one 16-iteration graph
    inst = sweep_instances(count)
    zeros = {n: np.zeros((n, n), np.float32) for n in SWEEP_SIZES}
    # single handles: one throwaway handle per grid size runs the launch-shape
    # tuning (11 shapes x 6 rounds x 3 iterations), which the library then
    # remembers for every later handle of that configuration
    for n in sorted({d["n"] for d in inst}):
        d = next(x for x in inst if x["n"] == n)
        s = pb.Solver(sweep_system(pb, n, device))
        s.set_field("psi_plus", d["psi0"])
        s.set_field("n_plus", zeros[n])
        s.set_field("pump_plus", d["pump"], 0)
        s.set_field("potential_plus", d["potential"], 0)
        s.run(11 * 6 * 3 + 2)
        s.close()
    b = pb.BatchSolver([sweep_system(pb, d["n"], device) for d in inst])
    for i, d in enumerate(inst):
        b.set_field(i, "psi_plus", d["psi0"])
        b.set_field(i, "n_plus", zeros[d["n"]])
        b.set_field(i, "pump_plus", d["pump"])
        b.set_field(i, "potential_plus", d["potential"])
    bs = torch.cuda.ExternalStream(b.stream, device=device)
    b.run(warm)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(bs):
        e0.record(bs)
    info = b.run(steps)
    with torch.cuda.stream(bs):
        e1.record(bs)
    torch.cuda.synchronize()
    batch_ms = e0.elapsed_time(e1)
    got = [(b.get_field(i, "psi_plus"), b.get_field(i, "n_plus")) for i in range(count)]
    shape = info.launch_shape
    b.close()
    seq_ms = 0.0
    seq_wall = time.perf_counter()
    equal = 0
    for i, d in enumerate(inst):
        s = pb.Solver(sweep_system(pb, d["n"], device))
        s.set_field("psi_plus", d["psi0"])
        s.set_field("n_plus", zeros[d["n"]])
        s.set_field("pump_plus", d["pump"], 0)
        s.set_field("potential_plus", d["potential"], 0)
        s.run(warm)
        st = torch.cuda.ExternalStream(s.stream, device=device)
        a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(st):
            a0.record(st)
        s.run(steps)
        with torch.cuda.stream(st):
            a1.record(st)
        torch.cuda.synchronize()
        seq_ms += a0.elapsed_time(a1)
        equal += int(np.array_equal(got[i][0], s.get_field("psi_plus")) and
                     np.array_equal(got[i][1], s.get_field("n_plus")))
        s.close()
    seq_wall = time.perf_counter() - seq_wall
    points = sum(d["n"] ** 2 for d in inst)
    return {"instances": count, "grid_points": points, "steps_timed": steps, "dtype": "f32",
            "sizes": {str(n): sum(1 for d in inst if d["n"] == n) for n in SWEEP_SIZES},
            "batch_ms": batch_ms, "batch_us_per_iteration": batch_ms * 1e3 / steps,
            "batch_grid_point_updates_per_s": points * steps / (batch_ms * 1e-3),
            "batch_tile_shape": shape,
            "sequential_ms": seq_ms, "sequential_us_per_iteration": seq_ms * 1e3 / steps,
            "sequential_wall_s_incl_setup": seq_wall,
            "speedup_vs_sequential": seq_ms / batch_ms,
            "bit_identical_instances": equal,
            "note": f"one batch launch per iteration (captured graphs of 16) vs {count} single-simulation "
                    "handles run one after another, each grid size's launch shape tuned beforehand; both "
                    "device-timed over the same iterations"}


def run_adjoint(pb, torch, device, iters=500, n=512):
    """Inverse-design configuration: 512^2 FP32 RK4, T = 500, dt = 0.04 ps,
    pump disc of 1.2x threshold (radius 30 um), loss sum (|psi_T|^2 - rho)^2 dV
    against seven Gaussian spots on a hexagonal lattice.  Device time of the
    plain forward (phx_step), of the checkpointed forward and of the backward
    (recompute + vector-Jacobian kernels), CUDA events on the solver stream."""
    from phoenix_b200.adjoint import evolve

    sp = pb.SystemParameters(N_c=n, N_r=n, L_x=L_BOX, L_y=L_BOX, **PHYS, g_pm=0.0, delta_LT=0.0,
                             periodic_boundary_x=True, periodic_boundary_y=True, dtype="f32", iterator="RK4",
                             dt=0.04, t_max=1e12, fft_every=1e12, pump_temporal=[pb.Temporal()], device=device)
    x = -L_BOX / 2 + L_BOX / (n - 1) * np.arange(n)
    X, Y = np.meshgrid(x, x)
    pump = np.where(X ** 2 + Y ** 2 <= 30.0 ** 2, 1.2 * P_TH, 0.0).astype(np.float32)
    rho = np.zeros((n, n))
    for x0, y0 in [(0.0, 0.0)] + [(15 * np.cos(a), 15 * np.sin(a)) for a in np.arange(6) * np.pi / 3]:
        rho += 5.0 * np.exp(-((X - x0) ** 2 + (Y - y0) ** 2) / (2 * 4.0 ** 2))
    rng = np.random.default_rng(6)
    psi0 = (1e-2 * (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n)))).astype(np.complex64)
    dev = f"cuda:{device}"
    s = pb.Solver(sp)
    st = torch.cuda.ExternalStream(s.stream, device=device)
    ev = lambda: torch.cuda.Event(enable_timing=True)  # noqa: E731
    # plain forward (after autotuning)
    s.set_field("psi_plus", psi0)
    s.set_field("pump_plus", pump, 0)
    s.run(40)
    a, b = ev(), ev()
    with torch.cuda.stream(st):
        a.record(st)
    s.run(iters)
    with torch.cuda.stream(st):
        b.record(st)
    torch.cuda.synchronize()
    plain_ms = a.elapsed_time(b)
    P = torch.tensor(pump, device=dev, requires_grad=True)
    z0 = torch.tensor(psi0, device=dev)
    m0 = torch.zeros((n, n), dtype=torch.float32, device=dev)
    rho_t = torch.tensor(rho, dtype=torch.float32, device=dev)
    dV = (L_BOX / (n - 1)) ** 2
    times = []
    for _ in range(4):  # the first pass allocates the segment planes
        P.grad = None
        e0, e1, e2 = ev(), ev(), ev()
        torch.cuda.synchronize()
        with torch.cuda.stream(st):
            e0.record(st)
        psi_T, _ = evolve(s, P, z0, m0, iters)
        with torch.cuda.stream(st):
            e1.record(st)
        L = (((psi_T.real ** 2 + psi_T.imag ** 2) - rho_t) ** 2).sum() * dV
        L.backward()
        with torch.cuda.stream(st):
            e2.record(st)
        torch.cuda.synchronize()
        times.append((e0.elapsed_time(e1), e1.elapsed_time(e2)))
    # per-kernel device time of one more forward + backward (library events)
    s.profile(True)
    P.grad = None
    psi_T, _ = evolve(s, P, z0, m0, iters)
    (((psi_T.real ** 2 + psi_T.imag ** 2) - rho_t) ** 2).sum().backward()
    torch.cuda.synchronize()
    kernels = {k: {"ms": v["ms"], "launches": v["launches"]} for k, v in s.profile_read().items()}
    s.close()
    # the median of three timed passes: the backward issues about a thousand
    # launches on two streams, and a busy host stretches the gaps between them
    timed = sorted(times[1:], key=lambda t: t[1])
    fwd, bwd = timed[len(timed) // 2]
    return {"grid": [n, n], "iterations": iters, "dtype": "f32", "checkpoint_every": int(np.ceil(np.sqrt(iters))),
            "kernels_forward_and_backward": kernels,
            "plain_forward_ms": plain_ms, "checkpointed_forward_ms": fwd, "backward_ms": bwd,
            "backward_ms_passes": [t[1] for t in times[1:]],
            "backward_over_plain_forward": bwd / plain_ms,
            "note": "backward = per iteration one fused recompute launch (stage values stored, on a second "
                    "stream, one segment ahead) + one fused vector-Jacobian launch; loss evaluation by torch "
                    "between the two"}


def flush_l2(buf):
    """Evict L2 before a timed iteration: write a buffer twice the size of L2,
    then read it, so that L2 holds clean lines of the buffer (the write-back of
    the flush's own dirty lines is not charged to the timed iteration)."""
    buf.zero_()
    buf.view(-1, 4096).amax(dim=1)


def max_over_ranks(torch, dist, value, device):
    """The largest of every rank's value (all ranks call it; dist None: one process)."""
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    if dist:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def tune(solver, cap=600):
    """Run single iterations until the library's launch-shape autotuning has
    ended (launch_shape >= 0); returns the iterations run."""
    for k in range(1, cap + 1):
        if solver.run(1).launch_shape >= 0:
            return k
    raise RuntimeError("autotuning did not end")


def _device_us(torch, solver, device, iters):
    """Device time per iteration of `iters` iterations (CUDA events on the solver stream)."""
    st = torch.cuda.ExternalStream(solver.stream, device=device)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    with torch.cuda.stream(st):
        a.record(st)
    info = solver.run(iters)
    with torch.cuda.stream(st):
        b.record(st)
    torch.cuda.synchronize()
    return a.elapsed_time(b) * 1e3 / max(info.iterations, 1), info


def run_tetm(pb, torch, dev, n):
    """Config 3 at n x n: TE/TM FP32 RK4, ring pump (radius 20 um, width 3 um) at 1.5x threshold on both
    polarisations, delta_LT 0.05 meV, g_pm = -0.2 g_c, dt 0.0015 ps at 4096^2 (scaled with dx^2),
    with noise (dw 1e-3) and without."""
    out = {}
    x = -L_BOX / 2 + L_BOX / (n - 1) * np.arange(n, dtype=np.float64)
    X, Y = np.meshgrid(x, x)
    ring = (1.5 * P_TH * np.exp(-(np.sqrt(X ** 2 + Y ** 2) - 20.0) ** 2 / (2 * 3.0 ** 2))).astype(np.float32)
    del X, Y
    rng = np.random.default_rng(4)
    dt = 0.0015 * (4096.0 / n) ** 2
    for dw in (1e-3, 0.0):
        sp = pb.SystemParameters(N_c=n, N_r=n, L_x=L_BOX, L_y=L_BOX, **PHYS, periodic_boundary_x=True,
                                 periodic_boundary_y=True, dtype="f32", iterator="RK4", dt=dt, t0=0.0, t_max=1e12,
                                 fft_every=1e12, pump_temporal=[pb.Temporal()], device=dev, use_twin_mode=True,
                                 stochastic_amplitude=dw, random_seed=4)
        sp.g_pm, sp.delta_LT = -0.2 * PHYS["g_c"], 0.05
        with pb.Solver(sp) as s:
            for comp in ("plus", "minus"):
                psi0 = (1e-2 * (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n)))).astype(np.complex64)
                s.set_field(f"psi_{comp}", psi0)
                s.set_field(f"pump_{comp}", ring, 0)
            tune(s)
            us, info = _device_us(torch, s, dev, 20)
            key = f"tetm_{n}_f32_noise" if dw else f"tetm_{n}_f32_deterministic"
            out[key] = {"us_per_iteration": us, "grid_point_updates_per_s": 2 * n * n / (us * 1e-6),
                        "launch_shape": info.launch_shape}
    return out


def run_dp45(pb, torch, dev, n, dtype, steps):
    """Dormand-Prince 5(4) adaptive (tol 1e-6) on the n^2 workload: tuning, then
    `steps` accepted steps timed on the device, with the library's per-kernel
    times (the leg profiles run alone: `bench.py --only dp45 --steps 3`)."""
    wl = workload(n)
    sp = pb.SystemParameters(N_c=n, N_r=n, L_x=L_BOX, L_y=L_BOX, **PHYS, periodic_boundary_x=True,
                             periodic_boundary_y=True, dtype=dtype, iterator="DP45", dt=dt_for(n), t0=0.0, t_max=1e12,
                             fft_every=1e12, pump_temporal=[pb.Temporal()], potential_temporal=[pb.Temporal()],
                             use_adaptive_timestep=True, tolerance=1e-6, dt_min=1e-5, dt_max=0.05, device=dev)
    with pb.Solver(sp) as s:
        s.set_field("psi_plus", wl["psi0"])
        s.set_field("pump_plus", wl["pump"], 0)
        s.set_field("potential_plus", wl["potential"], 0)
        tune(s)
        us, info = _device_us(torch, s, dev, steps)  # without the library's own events
        s.profile(True)
        _device_us(torch, s, dev, steps)
        kernels = {k: {"ms_per_launch": v["ms"] / v["launches"], "launches": v["launches"]}
                   for k, v in s.profile_read().items()}
    return {"grid": n, "dtype": dtype, "us_per_accepted_step": us * info.iterations / max(info.accepted, 1),
            "accepted": info.accepted, "rejected": info.rejected, "kernels": kernels}


def _ref_gpu(res):
    return None if res is None else round(res["us_per_iteration"], 2)


def run_configs(pb, torch, device, ref_gpu=True):
    """The other configurations: 256^2 FP64 RK4 (1000 steps); 1024^2 FP64 RK4,
    DP45 adaptive (rtol 1e-6) in FP32 and FP64; 4096^2 TE/TM FP32 RK4 with a
    ring pump and noise (dw 1e-3) and its deterministic twin.  Device time per
    iteration after the launch-shape autotuning, each beside the reference's
    own CUDA build on the same GPU with the same flags (reference_gpu_us,
    marginal per iteration), and the FP32-vs-FP64 error of each configuration
    at its own size and length (fp32_error)."""
    out = {}
    dev = device

    def sysp(n, dtype, it="RK4", **kw):
        dt = kw.pop("dt", dt_for(n))
        return pb.SystemParameters(N_c=n, N_r=n, L_x=L_BOX, L_y=L_BOX, **PHYS, periodic_boundary_x=True,
                                   periodic_boundary_y=True, dtype=dtype, iterator=it, dt=dt, t0=0.0, t_max=1e12,
                                   fft_every=1e12, pump_temporal=[pb.Temporal()], device=dev, **kw)

    def rgpu(*a, **k):
        if not ref_gpu:
            return None
        torch.cuda.synchronize()
        return _ref_gpu(reference_marginal(*a, gpu=True, **k))

    # config 1: 256^2 FP64 RK4, dt 0.04, 1000 steps
    n = 256
    wl = workload(n, seed=1)
    with pb.Solver(sysp(n, "f64", dt=0.04)) as s:
        s.set_field("psi_plus", wl["psi0"])
        s.set_field("pump_plus", wl["pump"], 0)
        tune(s)
        us, info = _device_us(torch, s, dev, 1000)
        out["rk4_256_f64"] = {"us_per_iteration": us, "iterations": info.iterations, "launch_shape": info.launch_shape,
                              "reference_gpu_us": rgpu("f64", n, 0.04, 200 * 0.04 * (1 - 1e-9), 5200 * 0.04 * (1 - 1e-9),
                                                       scalar_loads(wl, mask=False, potential=False), subgrids=1)}
    # config 2: 1024^2 -- FP64 RK4, DP45 adaptive
    n = 1024
    wl = workload(n)
    dt = dt_for(n)
    for dtype in ("f32", "f64"):
        with pb.Solver(sysp(n, dtype, potential_temporal=[pb.Temporal()])) as s:
            s.set_field("psi_plus", wl["psi0"])
            s.set_field("pump_plus", wl["pump"], 0)
            s.set_field("potential_plus", wl["potential"], 0)
            tune(s)
            us, info = _device_us(torch, s, dev, 460)
            out[f"rk4_1024_{dtype}"] = {
                "us_per_iteration": us, "launch_shape": info.launch_shape,
                "reference_gpu_us": rgpu(dtype, n, dt, 100 * dt * (1 - 1e-9), 2100 * dt * (1 - 1e-9),
                                         scalar_loads(wl, mask=False), subgrids=1)}
    dp = ["-adaptive", "--iterator", "DP45", "--tol", "1e-06", "--rkvdt", "1e-05", "0.05"]
    for dtype in ("f32", "f64"):
        sp = sysp(n, dtype, it="DP45", potential_temporal=[pb.Temporal()], use_adaptive_timestep=True,
                  tolerance=1e-6, dt_min=1e-5, dt_max=0.05)
        with pb.Solver(sp) as s:
            s.set_field("psi_plus", wl["psi0"])
            s.set_field("pump_plus", wl["pump"], 0)
            s.set_field("potential_plus", wl["potential"], 0)
            tune(s)
            us, info = _device_us(torch, s, dev, 100)
            out[f"dp45_adaptive_1024_{dtype}"] = {
                "us_per_accepted_step": us * info.iterations / max(info.accepted, 1),
                "accepted": info.accepted, "rejected": info.rejected, "dt": info.dt,
                "reference_gpu_us": rgpu(dtype, n, dt, 0.2, 2.2, scalar_loads(wl, mask=False), extra=dp, subgrids=1)}
    # config 3: 4096^2 TE/TM FP32
    out.update(run_tetm(pb, torch, dev, 4096))
    if ref_gpu:
        dt3 = 0.0015
        tetm = ["-tetm", "--gpm", repr(-0.2 * PHYS["g_c"]), "--deltaLT", "0.05", "--initRandom", "0.01", "4",
                "--pump", repr(1.5 * P_TH), "add", "10", "10", "0", "0", "both", "1", "none", "gauss+noDivide"]
        for key, dw in (("tetm_4096_f32_deterministic", "0"), ("tetm_4096_f32_noise", "0.001")):
            out[key]["reference_gpu_us"] = rgpu("f32", 4096, dt3, 20 * dt3 * (1 - 1e-9), 170 * dt3 * (1 - 1e-9),
                                                extra=tetm + ["--dw", dw], subgrids=16)
    for k, v in out.items():
        mine = v.get("us_per_iteration", v.get("us_per_accepted_step"))
        if v.get("reference_gpu_us"):
            v["speedup_vs_reference_gpu"] = v["reference_gpu_us"] / mine
    out["fp32_error"] = fp32_errors(pb, dev)
    return out


def _rel(a, b):
    a, b = np.asarray(a, dtype=np.complex128), np.asarray(b, dtype=np.complex128)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def fp32_errors(pb, dev):
    """FP32 against FP64 from identical inputs, rel-L2 of psi and n, per
    configuration at its own size and length: config 1 (256^2, 1000 RK4
    iterations), config 2 (1024^2 with disorder and the mask every 100
    iterations: 5000 RK4 iterations, bit-exact and fused multiply-add FP32;
    Dormand-Prince adaptive at tol 1e-6 to t = 20 ps), config 3 (4096^2 TE/TM, 2000 RK4 iterations, deterministic),
    config 5 (512^2, 500 RK4 iterations, the inverse-design pump disc)."""
    out = {}

    def run(sp, loads, iters=None, fma=False):
        res = {}
        for dtype in ("f32", "f64"):
            sp.dtype = dtype
            sp.fma = fma and dtype == "f32"
            with pb.Solver(sp) as s:
                for name, arr, g in loads:
                    s.set_field(name, arr, g)
                info = s.run(iters) if iters else s.run()
                res[dtype] = ({k: s.get_field(k) for k in ("psi_plus", "n_plus", "psi_minus", "n_minus")
                               if k.endswith("plus") or sp.use_twin_mode}, info)
        return {k: _rel(res["f32"][0][k], res["f64"][0][k]) for k in res["f64"][0]}, res

    def base(n, dt, iterator="RK4", **kw):
        return pb.SystemParameters(N_c=n, N_r=n, L_x=L_BOX, L_y=L_BOX, **PHYS, periodic_boundary_x=True,
                                   periodic_boundary_y=True, dtype="f64", iterator=iterator, dt=dt, t0=0.0,
                                   t_max=1e12, fft_every=1e12, pump_temporal=[pb.Temporal()], device=dev, **kw)

    wl = workload(256, seed=1)
    out["cfg1_rk4_256_1000"], _ = run(base(256, 0.04), [("psi_plus", wl["psi0"], 0), ("pump_plus", wl["pump"], 0)],
                                      1000)
    wl = workload(1024)
    dt = dt_for(1024)
    loads = [("psi_plus", wl["psi0"], 0), ("pump_plus", wl["pump"], 0), ("potential_plus", wl["potential"], 0),
             ("fft_mask_plus", wl["mask"], 0)]
    sp = base(1024, dt, potential_temporal=[pb.Temporal()])
    sp.fft_every = MASK_EVERY * dt * (1 - 1e-6)
    out["cfg2_rk4_1024_5000_mask"], _ = run(sp, loads, 5000)
    out["cfg2_rk4_1024_5000_mask_fma"], _ = run(sp, loads, 5000, fma=True)
    sp = base(1024, dt, potential_temporal=[pb.Temporal()], iterator="DP45", use_adaptive_timestep=True,
              tolerance=1e-6, dt_min=1e-5, dt_max=0.05)
    sp.fft_every, sp.t_max = MASK_EVERY * dt * (1 - 1e-6), 20.0
    err, res = run(sp, loads)
    err["accepted_f32_f64"] = [res["f32"][1].accepted, res["f64"][1].accepted]
    out["cfg2_dp45_1024_t20ps_mask"] = err
    n = 4096
    x = -L_BOX / 2 + L_BOX / (n - 1) * np.arange(n, dtype=np.float64)
    X, Y = np.meshgrid(x, x)
    ring = 1.5 * P_TH * np.exp(-(np.sqrt(X ** 2 + Y ** 2) - 20.0) ** 2 / (2 * 3.0 ** 2))
    del X, Y
    rng = np.random.default_rng(4)
    psi = {c: 1e-2 * (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))) for c in ("plus", "minus")}
    sp = base(n, 0.0015, use_twin_mode=True)
    sp.g_pm, sp.delta_LT = -0.2 * PHYS["g_c"], 0.05
    out["cfg3_tetm_4096_2000"], _ = run(sp, [("psi_plus", psi["plus"], 0), ("psi_minus", psi["minus"], 0),
                                             ("pump_plus", ring, 0), ("pump_minus", ring, 0)], 2000)
    del psi, ring
    n = 512
    x = -L_BOX / 2 + L_BOX / (n - 1) * np.arange(n)
    X, Y = np.meshgrid(x, x)
    disc = np.where(X ** 2 + Y ** 2 <= 30.0 ** 2, 1.2 * P_TH, 0.0)
    psi0 = 1e-2 * (np.random.default_rng(6).standard_normal((n, n)) + 1j * np.random.default_rng(7).standard_normal((n, n)))
    out["cfg5_rk4_512_500"], _ = run(base(n, 0.04), [("psi_plus", psi0, 0), ("pump_plus", disc, 0)], 500)
    return out


def config_dict(args):
    return {"workload": f"rk4_scalar_reservoir_pump_potential_mask_{args.n}x{args.n}_{args.dtype}",
            "grid": [args.n, args.n], "iterator": "RK4", "boundary": "periodic", "dt_ps": dt_for(args.n),
            "mask_every_iterations": MASK_EVERY, "physics": "polariton GP + reservoir, meV/ps/um, hbar 0.6582, "
            "m_eff 5.6e-4 m_e", "replicas": "one independent simulation per GPU",
            "l2": "256 MiB write then read between timed iterations (value); e2e runs back to back",
            "arithmetic": "every operation rounded separately in the reference's order (bit-identical to its FP32 "
                          "/ FP64 build)" if args.arith == "exact" else
                          "fused multiply-adds (phx_params.fma; FP32 error vs FP64 in configs.fp32_error)"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=400)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="phx", choices=["phx", "reference"])
    ap.add_argument("--dtype", default="f32", choices=["f32", "f64"])
    ap.add_argument("--n", type=int, default=N_DEFAULT)
    ap.add_argument("--arith", default="exact", choices=["exact", "fma"],
                    help="arithmetic of the timed solver: exact (every operation rounded as the reference does) or "
                         "fma (phx_params.fma, FP32)")
    ap.add_argument("--ref-iters", type=int, default=400, help="cap on reference CPU iterations")
    ap.add_argument("--cpu-iters", type=int, default=1500, help="CPU-baseline sample in the phx arm (about 10 s)")
    ap.add_argument("--ref-gpu-iters", type=int, default=2000,
                    help="iterations of the reference GPU build beyond its first 100")
    ap.add_argument("--no-cpu-baseline", action="store_true", help="skip the reference CPU and GPU builds")
    ap.add_argument("--sweep-instances", type=int, default=256, help="instances of the batched sweep (0: skip)")
    ap.add_argument("--sweep-steps", type=int, default=200, help="timed iterations of the batched sweep")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the adjoint (inverse-design) leg")
    ap.add_argument("--no-configs", action="store_true", help="skip the other configurations' timings")
    ap.add_argument("--only", choices=["configs", "adjoint", "sweep", "tetm", "dp45"],
                    help="run one leg alone and print its JSON")
    ap.add_argument("--tetm-n", type=int, default=4096, help="grid of the --only tetm leg")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.impl == "reference":
        return run_reference_arm(args)

    import torch

    import phoenix_b200 as pb

    if args.only:
        import torch

        import phoenix_b200 as pb

        torch.cuda.set_device(0)
        leg = {"configs": lambda: run_configs(pb, torch, 0), "adjoint": lambda: run_adjoint(pb, torch, 0),
               "sweep": lambda: run_sweep(pb, torch, args.sweep_instances, args.sweep_steps, 0),
               "tetm": lambda: run_tetm(pb, torch, 0, args.tetm_n),
               "dp45": lambda: run_dp45(pb, torch, 0, args.n, args.dtype, args.steps)}[args.only]
        print(json.dumps({args.only: leg()}))
        return 0
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    torch.cuda.set_device(local)
    n = args.n
    wl = workload(n)
    sp = system(pb, n, args.dtype, local)
    sp.fma = args.arith == "fma"
    solver = pb.Solver(sp)
    solver.set_field("psi_plus", wl["psi0"])
    solver.set_field("n_plus", np.zeros((n, n)))
    solver.set_field("pump_plus", wl["pump"], 0)
    solver.set_field("potential_plus", wl["potential"], 0)
    solver.set_field("fft_mask_plus", wl["mask"])
    stream = torch.cuda.ExternalStream(solver.stream, device=local)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{local}")

    def barrier():
        if dist:
            dist.barrier()

    # launch-shape autotuning (untimed, before the warm-up): the library times
    # every candidate launch shape over its first iterations (six rounds of
    # three iterations each, medians, incumbent kept within 3 %)
    tune_iters = tune(solver)
    autotune = {"chosen": solver.run(0).launch_shape,
                "median_us_per_iteration": {str(k): round(v, 3) for k, v in solver.tune_report().items()}}

    # warm-up
    for _ in range(args.warmup):
        with torch.cuda.stream(stream):
            flush_l2(flush)
        solver.run(1)
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()

    # timed region: per iteration, flush L2 (untimed) then time the iteration
    idx = os.environ.get("CUDA_VISIBLE_DEVICES", "").split(",")
    smi_index = idx[local] if len(idx) > local and idx[local].strip().isdigit() else str(local)
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]

    def timed_pass(profile):
        """args.steps iterations, L2 flushed before each, each bracketed by an
        event pair; with profile the library also brackets each of its own
        launches (the per-kernel times of the roofline)"""
        launches = filters = 0
        shape = -1
        if profile:
            solver.profile(True)
        with torch.cuda.stream(stream):
            # an untimed ~25 ms device sleep lets the host queue the timed
            # iterations ahead of the GPU, so that no event pair spans host time
            torch.cuda._sleep(50_000_000)
            for i in range(args.steps):
                flush_l2(flush)
                starts[i].record(stream)
                info = solver.run(1)
                ends[i].record(stream)
                shape = info.launch_shape
                launches += info.kernel_launches
                filters += info.fft_filters
            torch.cuda.synchronize()
        prof = None
        if profile:
            prof = solver.profile_read()
            solver.profile(False)
        return sum(s.elapsed_time(e) for s, e in zip(starts, ends)) / args.steps, prof, launches, filters, shape

    # the timed region of `value` runs without the library's own events; a
    # second pass of the same loop with them gives the per-kernel times
    with ClockSampler(smi_index) as clocks:
        step_ms, _, launches, filters, shape = timed_pass(False)
    prof_step_ms, prof, _, _, _ = timed_pass(True)
    step_ms = max_over_ranks(torch, dist, step_ms, f"cuda:{local}")

    # back-to-back (L2-warm) iterations, one event pair
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        e0.record(stream)
    solver.run(args.steps)
    with torch.cuda.stream(stream):
        e1.record(stream)
    torch.cuda.synchronize()
    warm_ms = e0.elapsed_time(e1) / args.steps
    solver.close()

    # the same workload with the fused multiply-add arithmetic (phx_params.fma),
    # timed the same way (L2 flushed before every iteration)
    sp_fma = system(pb, n, args.dtype, local)
    sp_fma.fma = args.dtype == "f32" and args.arith == "exact"
    fma_leg = None
    if sp_fma.fma:
        sf = pb.Solver(sp_fma)
        sf.set_field("psi_plus", wl["psi0"])
        sf.set_field("n_plus", np.zeros((n, n)))
        sf.set_field("pump_plus", wl["pump"], 0)
        sf.set_field("potential_plus", wl["potential"], 0)
        sf.set_field("fft_mask_plus", wl["mask"])
        tune(sf)
        fstream = torch.cuda.ExternalStream(sf.stream, device=local)
        for _ in range(args.warmup):
            with torch.cuda.stream(fstream):
                flush_l2(flush)
            sf.run(1)
        torch.cuda.synchronize()
        fs = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
        fe = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]

        def fma_pass(profile):
            if profile:
                sf.profile(True)
            with torch.cuda.stream(fstream):
                torch.cuda._sleep(50_000_000)
                for i in range(args.steps):
                    flush_l2(flush)
                    fs[i].record(fstream)
                    info_ = sf.run(1)
                    fe[i].record(fstream)
                torch.cuda.synchronize()
            pr = None
            if profile:
                pr = sf.profile_read()
                sf.profile(False)
            return sum(a.elapsed_time(b) for a, b in zip(fs, fe)) / args.steps, pr, info_

        # timed without the library's own events, as the headline; then profiled
        f_ms, _, finfo = fma_pass(False)
        _, fprof, _ = fma_pass(True)
        sf.close()
        fk = fprof.get("rk4_fused")
        fma_leg = {"value": f_ms * 1e3, "unit": "us/iter", "launch_shape": finfo.launch_shape,
                   "kernel_avg_ms": fk["ms"] / fk["launches"] if fk else None,
                   "note": "phx_params.fma = 1: the one-kernel iteration with fused multiply-adds (FP32), same "
                           "workload and timing; its FP32-vs-FP64 error is in configs.fp32_error"}

    # end to end through the public API, host buffers in and out
    e2e_iters = args.steps
    chunk = 100
    cdt = torch.complex64 if args.dtype == "f32" else torch.complex128
    rdt = torch.float32 if args.dtype == "f32" else torch.float64
    pinned_psi = torch.from_numpy(np.ascontiguousarray(wl["psi0"])).to(cdt).pin_memory().numpy()
    pinned_n = torch.zeros((n, n), dtype=rdt).pin_memory().numpy()
    pinned_psi_out = torch.empty((n, n), dtype=cdt).pin_memory().numpy()
    pinned_n_out = torch.empty((n, n), dtype=rdt).pin_memory().numpy()
    barrier()
    torch.cuda.synchronize()
    s2 = pb.Solver(sp)
    s2.set_field("pump_plus", wl["pump"], 0)
    s2.set_field("potential_plus", wl["potential"], 0)
    s2.set_field("fft_mask_plus", wl["mask"])
    torch.cuda.synchronize()
    st2 = torch.cuda.ExternalStream(s2.stream, device=local)

    def end_to_end(iters):
        """upload the inputs from pinned host memory, iterate with an FP64 norm
        read back every `chunk` iterations, download the state"""
        s2.set_field("psi_plus", pinned_psi)
        s2.set_field("n_plus", pinned_n)
        done, norms = 0, []
        while done < iters:
            k = min(chunk, iters - done)
            s2.run(k)
            norms.append(s2.sum_abs2("psi_plus"))
            done += k
        return s2.get_field("psi_plus", out=pinned_psi_out), s2.get_field("n_plus", out=pinned_n_out), norms

    # untimed pass: first use of the pinned buffers and of the handle's planes
    end_to_end(min(chunk, e2e_iters))
    torch.cuda.synchronize()
    a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(st2):
        a0.record(st2)
    psi_out, n_out, norms = end_to_end(e2e_iters)
    with torch.cuda.stream(st2):
        a1.record(st2)
    torch.cuda.synchronize()
    e2e_ms = a0.elapsed_time(a1) / e2e_iters
    s2.close()
    t_e2e = torch.tensor([e2e_ms], dtype=torch.float64, device=f"cuda:{local}")
    if dist:
        dist.all_reduce(t_e2e, op=dist.ReduceOp.MAX)
    e2e_ms = float(t_e2e.item())
    esz = 4 if args.dtype == "f32" else 8
    h2d = n * n * 3 * esz  # psi0 (complex) and n0, pinned, in the build precision
    d2h = n * n * 3 * esz + 8 * ((e2e_iters + chunk - 1) // chunk)  # psi, n and one FP64 norm per chunk
    assert np.isfinite(psi_out).all() and np.isfinite(n_out).all() and all(np.isfinite(norms))

    # roofline of the dominant kernel (fused RK4 middle stage)
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    peak, peak_src = 6650.0, "fallback"
    if os.path.exists(peaks_path):
        with open(peaks_path) as f:
            peak = float(json.load(f)["hbm_gbs"])
        peak_src = "measured"
    # dominant kernel: the family with the largest device time in the timed region
    dom_name = max((k for k in prof if k != "other"), key=lambda k: prof[k]["ms"])
    dom = prof[dom_name]
    per_launch_bytes = dom["bytes"] / dom["launches"]
    per_launch_ms = dom["ms"] / dom["launches"]
    # algorithmic bytes: a whole-iteration launch is charged the state
    # round-trips of four one-kernel-per-stage launches (rk4_alg_bytes_per_point);
    # the fused kernel's own compulsory bytes are reported beside them
    esz = 4 if args.dtype == "f32" else 8
    alg_pp = rk4_alg_bytes_per_point(esz, has_pot=True) if dom_name == "rk4_fused" else per_launch_bytes / (n * n)
    alg_launch_bytes = alg_pp * n * n
    achieved = alg_launch_bytes / (per_launch_ms * 1e-3) / 1e9
    traffic = None
    # DRAM traffic per launch from the committed ncu summary of that kernel at
    # 4096^2 (the largest case ncu captures here), scaled to this grid by points
    tfile = os.path.join(ROOT, "profiles", "traffic_per_point.json")
    if os.path.exists(tfile):
        with open(tfile) as f:
            tj = json.load(f)
        key = f"{dom_name}_{args.dtype}"
        if key in tj:
            traffic = tj[key]["bytes_per_point"] * n * n
    step_bytes = sum(v["bytes"] for k, v in prof.items() if k.startswith("rk4")) / args.steps
    kernels_ms = {k: v["ms"] / v["launches"] for k, v in prof.items()}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        res = reference_cpu_run(n, args.dtype, args.cpu_iters, wl)
        kind = "reference"
        if res is None:
            res = oracle_port_run(n, args.dtype, 3, wl)
            kind = "port"
        us, cores, what = res
        cpu = {"value": us, "unit": "us/iter", "cores": cores, "kind": kind,
               "sample": f"{args.cpu_iters if kind == 'reference' else 3} RK4 iterations of the {n}^2 workload "
                         f"(beyond its first 100 for the reference) with {what}"}

    ref_gpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        torch.cuda.synchronize()
        dt = dt_for(n)
        res = reference_marginal(args.dtype, n, dt, 100 * dt * (1 - 1e-9), (100 + args.ref_gpu_iters) * dt * (1 - 1e-9),
                                 scalar_loads(wl), gpu=True, fft_every=MASK_EVERY * dt * (1 - 1e-6), subgrids=1)
        if res is not None:
            ref_gpu = {"value": res["us_per_iteration"], "unit": "us/iter", "binary": res["binary"],
                       "iterations": res["iterations"],
                       "note": "the reference's own CUDA build for sm_100 on this GPU, --subgrids 1 1: marginal wall "
                               "clock of its main loop per iteration between the two runs (its Total Runtime / "
                               "mus/it lines)"}

    # the single-GPU legs run at N = 1 only (with N > 1 the other ranks would
    # wait for them at the closing barrier)
    sweep = None
    if rank == 0 and world == 1 and args.sweep_instances > 0:
        sweep = run_sweep(pb, torch, args.sweep_instances, args.sweep_steps, local)
    adjoint = None
    if rank == 0 and world == 1 and not args.no_adjoint:
        adjoint = run_adjoint(pb, torch, local)
    configs = None
    if rank == 0 and world == 1 and not args.no_configs:
        configs = run_configs(pb, torch, local)

    if rank == 0:
        us = step_ms * 1e3
        line = {"metric": METRIC, "value": us, "unit": "us/iter", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": False, "scaling": "weak",
                "vs_baseline": None, "dtype": args.dtype, "data": "synthetic", "config": config_dict(args),
                "grid_point_updates_per_s": world * n * n / (step_ms * 1e-3),
                "warm_l2_us_per_iter": warm_ms * 1e3,
                "us_per_iter_with_library_events": prof_step_ms * 1e3,
                "e2e": {"value": e2e_ms * 1e3, "unit": "us/iter", "h2d_bytes_per_step": h2d / e2e_iters,
                        "d2h_bytes_per_step": d2h / e2e_iters},
                "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                             "frac": achieved / peak, "traffic": traffic, "kernel": KERNEL_NAMES.get(dom_name, dom_name),
                             "peak_source": peak_src, "alg_bytes_per_point": alg_pp,
                             "alg_bytes_per_launch": alg_launch_bytes,
                             "compulsory_bytes_per_launch": per_launch_bytes,
                             "compulsory_frac": per_launch_bytes / (per_launch_ms * 1e-3) / 1e9 / peak,
                             "step_alg_bytes": alg_pp * n * n,
                             "step_frac": alg_pp * n * n / (step_ms * 1e-3) / 1e9 / peak},
                "kernel_avg_ms": kernels_ms, "launch_shape": shape, "autotune_iterations": tune_iters,
                "autotune": autotune, "fma": fma_leg,
                "gpu_launches": launches, "fft_filters_in_timed_region": filters,
                "clocks": clocks.summary(), "cpu_baseline": cpu, "reference_gpu": ref_gpu, "sweep": sweep,
                "adjoint": adjoint, "configs": configs}
        print(json.dumps(line))
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())

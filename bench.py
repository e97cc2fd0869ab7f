#!/usr/bin/env python
"""Benchmark of the per-k-mode perturbation solve (one JSON line on stdout, rank 0).

Workload (default): flat LCDM + one 0.06 eV neutrino (5 momentum bins, l_max 12/12/17/17,
143 state variables per mode), 512 log-spaced k-modes in [1e-4, 10] /Mpc, outputs at
z = 2, 1, 0.5, 0, rtol 1e-5 / atol 1e-8.  One "step" = one cosmology: P(k) of all 512 modes
and its Jacobian with respect to theta = (omega_c, omega_b, h, n_s, ln 10^10 A_s, w0, wa,
m_nu) at the four redshifts (``--mode fwd+grad``, one discoeb_jvp launch: 6 tangent
directions through the solver, n_s and A_s analytic), or the forward solve alone
(``--mode forward``, one discoeb_fwd launch).  Under torchrun every rank solves its own
replica of the cosmology (weak scaling, no collective on the data path).

  value : k-modes/s (forward + gradient of each mode), inputs resident in HBM, CUDA events
          around each launch
  e2e   : the same metric through the public API (gradients.power_spectrum_jacobian: native
          background + Recfast with forward-mode tangents, one host thread per direction; or
          evolve_perturbations: host prologue + H2D + kernel + D2H inside the timed region)
  --impl reference : the oracle's CPU restatement of the reference algorithm (dense LU Rodas5)
          timed on all host cores on a bounded sample of the same workload; for fwd+grad the
          Jacobian of the sample comes from central differences (1 + 2 x 6 solves per mode).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time
import warnings

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "disco-eb_b200"))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

METRIC = "fwd+adjoint k-mode solves/s at ≤1e-4 rel err vs FP64 oracle; ms per cosmology"
# DRAM bytes of one launch per mode, from an ncu capture of a 48-mode case of the same kernel
# (dram__bytes_read.sum + dram__bytes_write.sum: jvp_block_kernel 1.566 MB, fwd_structured_kernel
# 0.304 MB), scaled by the number of modes: the initial states, their tangents and the outputs grow
# with it, the tables are shared (so this slightly overstates a full launch)
DRAM_BYTES_PER_MODE = {"fwd+grad": 1.566e6 / 48, "forward": 0.304e6 / 48}
# FP64 work per step attempt, counted by ncu on a 48-mode launch of the same kernel (thread-level
# smsp__sass_thread_inst_executed_op_{dadd,dmul,dfma}_pred_on.sum, a DFMA counted as two flops,
# over the launch's step attempts): jvp_block_kernel 5.526e9 + 14.086e9 + 2 x 15.101e9 = 4.982e10
# flops over 19187 attempts; fwd_structured_kernel 0.4558e9 + 0.9701e9 + 2 x 1.4198e9 = 4.2655e9 flops over
# 19187 attempts.  Scaled by the measured attempts of the timed launch.
FP64_FLOPS_PER_ATTEMPT = {"fwd+grad": 4.9815e10 / 19187, "forward": 4.2655e9 / 19187}
UNIT = "k-mode solves/s"


def _env_int(name, default):
    try:
        return int(os.environ.get(name, default))
    except ValueError:
        return default


def _background(w, backend="native"):
    from discoeb_b200.background import evolve_background
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        return evolve_background(param=w["param"], backend=backend)


def _sample_modes(w, count):
    k = np.geomspace(w["kmin"], w["kmax"], w["num_k"])
    idx = np.unique(np.linspace(0, len(k) - 1, count).round().astype(int))
    return k[idx]


def _shifted_backgrounds(w, backend="native", replay=None):
    """Backgrounds at theta +- 1e-4 |theta_i| along the 6 solver directions (central differences);
    ``replay``: a base point's Recfast trace, repeated (its step sequence held fixed)."""
    from discoeb_b200.background import evolve_background
    from discoeb_b200.gradients import ODE_DIRECTIONS, theta_to_params
    out = []
    for name in ODE_DIRECTIONS:
        for sgn in (1, -1):
            th = dict(w["theta"])
            th[name] += sgn * _fd_step(th, name)
            with warnings.catch_warnings():
                warnings.simplefilter("ignore")
                out.append(evolve_background(param=theta_to_params(th), backend=backend, replay=replay))
    return out


def _fd_step(theta, name):
    """1e-4 |theta_i|, at least 3e-7: at the workloads' w0 = -1 + 1e-6, wa = 0, w(a) crosses -1
    (where the fluid equations are singular) once wa < -1e-6, so the quotient in wa must stay well
    inside that distance."""
    return 1e-4 * max(abs(theta[name]), 3e-3)


# the oracle's tolerances for a quotient of step below 1e-5: its noise is the solve's error over
# the step (at rtol 1e-10 and step 3e-7, ~1e-4 of dP/dwa; ~1.5e-5 at rtol 1e-12)
_FINE_FD = dict(rtol=1e-12, atol=1e-15)


def oracle_accuracy(w, bg, kmodes, P, J, n_p=16, n_j=8, rtol=1e-10, atol=1e-13, J_rows=None, P_other=None):
    """Max relative error of the GPU's P(k) and dP/dtheta against the oracle (the CPU restatement,
    converged: rtol 1e-10), on modes spread over the workload's k range.

    P: |P_gpu / P_oracle - 1| over n_p modes at every output.  J: for each solver direction and
    output, max_k |J_gpu - J_fd| / max_k |J_fd| over n_j modes, J_fd the oracle's central
    difference of step _fd_step (1e-4 |theta_i|, at least 3e-7) with the start times, the
    approximation switch times and the Recfast step sequence held at the base point (the
    derivative forward-mode AD through the reference defines).  n_s and ln10As are analytic and
    not checked here."""
    from discoeb_b200.background import evolve_background
    from discoeb_b200.gradients import ODE_DIRECTIONS, THETA_NAMES, theta_to_params
    from discoeb_b200.perturbations import approximation_switch_times, determine_starting_time, get_power
    from oracle import pyoracle as O
    L = {k: w[k] for k in ("lmaxg", "lmaxgp", "lmaxr", "lmaxnu", "nqmax")}
    aout = np.asarray(w["aexp_out"], dtype=np.float64)
    t_start = time.perf_counter()

    def fixed_times(b, ks):
        tout = b["tau_of_a_spline"].evaluate(aout)
        return 0.99 * np.minimum(tout.min(), determine_starting_time(param=b, k=ks)), approximation_switch_times(b, ks)

    def power(b, ks, ts, sw, tol=None):
        tol = tol or dict(rtol=rtol, atol=atol)
        y, st = O.output_fields_fixed(b, ks, aout, ts, sw, **tol, **L)
        if (st != 0).any():
            raise RuntimeError("oracle solve failed in the accuracy check")
        return get_power(k=ks[:, None], y=y, idx=4, param=b)

    ip = np.unique(np.linspace(0, len(kmodes) - 1, n_p).round().astype(int))
    ts, sw = fixed_times(bg, kmodes[ip])
    Po = power(bg, kmodes[ip], ts, sw)
    err_p = float(np.max(np.abs(P[ip] / Po - 1)))
    # other solves of the same modes (the mixed-precision forward) against the same oracle values
    other = {name: float(np.max(np.abs(Px[ip] / Po - 1))) for name, Px in (P_other or {}).items()}
    if n_j == 0:
        out = {"P": err_p, "modes_P": int(ip.size), "oracle": f"CPU restatement, clip mode, rtol {rtol:g}, atol "
               f"{atol:g}", "seconds": time.perf_counter() - t_start}
        if other:
            out["P_other"] = other
        return out
    ij = np.unique(np.linspace(0, len(kmodes) - 1, n_j).round().astype(int))
    trace = {}
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        evolve_background(param=theta_to_params(w["theta"]), backend="numpy", trace=trace)
    shifted = _shifted_backgrounds(w, backend="numpy", replay=trace)
    ts, sw = fixed_times(bg, kmodes[ij])
    err_j, per_dir, err_r = 0.0, {}, 0.0
    for d, name in enumerate(ODE_DIRECTIONS):
        h = _fd_step(w["theta"], name)
        tol = _FINE_FD if h < 1e-5 else None
        fd = (power(shifted[2 * d], kmodes[ij], ts, sw, tol) - power(shifted[2 * d + 1], kmodes[ij], ts, sw, tol)) \
            / (2 * h)
        e = np.abs(J[THETA_NAMES.index(name)][ij] - fd).max(axis=0) / np.abs(fd).max(axis=0)
        per_dir[name] = float(e.max())
        err_j = max(err_j, per_dir[name])
        if J_rows is not None:  # the adjoint's rows of dP(k, z=0)/dtheta at the last output
            r = np.abs(J_rows[THETA_NAMES.index(name)][ij] - fd[:, -1]).max() / np.abs(fd[:, -1]).max()
            err_r = max(err_r, float(r))
    out = {"P": err_p, "J": err_j, "J_per_direction": per_dir, "modes_P": int(ip.size), "modes_J": int(ij.size),
            "oracle": f"CPU restatement, clip mode, rtol {rtol:g}, atol {atol:g}; J: central differences, step 1e-4 "
                      "max(|theta_i|, 3e-3) (rtol 1e-12 / atol 1e-15 where the step is below 1e-5), start / switch "
                      "times and Recfast steps held; max_k |dJ| / max_k |J| per direction and output",
            "seconds": time.perf_counter() - t_start}
    if J_rows is not None:
        out["J_adjoint_z0"] = err_r
    if other:
        out["P_other"] = other
    return out


def run_reference(args, rank, world):
    """CPU restatement of the reference algorithm (oracle port) on all host threads."""
    if rank != 0:
        return
    from discoeb_b200.workloads import workload
    from oracle import pyoracle as O
    w = workload(args.workload)
    # the numpy restatement of the background (no native library in this process)
    bg = _background(w, backend="numpy")
    L = {k: w[k] for k in ("lmaxg", "lmaxgp", "lmaxr", "lmaxnu", "nqmax")}
    ks = _sample_modes(w, args.ref_sample)
    threads = os.cpu_count() or 1

    grad = args.mode == "fwd+grad"
    bgs = [bg] + (_shifted_backgrounds(w, backend="numpy") if grad else [])

    def one():
        t = time.perf_counter()
        for b in bgs:
            O.evolve_perturbations(param=b, aexp_out=w["aexp_out"], kmin=0, kmax=0, num_k=0, rtol=w["rtol"],
                                   atol=w["atol"], kmodes=ks, mode="reference", de_guard_eps=1e-9,
                                   max_steps=100000, threads=threads, **L)
        return time.perf_counter() - t

    for _ in range(args.warmup):
        one()
    times = [one() for _ in range(args.steps)]
    ms = 1e3 * statistics.mean(times)
    value = len(ks) / (ms / 1e3)
    sample = (f"{len(ks)} of the {w['num_k']} modes (k evenly spread in log over [{w['kmin']:g}, {w['kmax']:g}]), "
              f"dense-LU Rodas5 with diffrax controller semantics, {threads} threads"
              + (", forward + central-difference Jacobian (13 solves per mode)" if grad else ""))
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded cosmology, no dataset)",
            "config": {"workload": args.workload, "mode": args.mode, "modes_per_step": len(ks)},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled every 200 ms during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.tmp = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.tmp,
                                         stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        self.tmp.flush()
        try:
            rows = [r.split(",") for r in open(self.tmp.name).read().strip().splitlines() if r.strip()]
        except OSError:
            rows = []
        os.unlink(self.tmp.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"], "samples": 0}
        sm = [float(r[1]) for r in rows if r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if len(r) > 5 + i and "Active" in r[5 + i]
                          and "Not" not in r[5 + i]})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def fp64_fma_tflops(torch, device):
    """Measured FP64 FMA throughput on this GPU (discoeb_fma_rate: 8 independent FMA chains per
    thread, 4 x 256 threads per SM, 65536 iterations), best of 5 launches."""
    import ctypes
    from discoeb_b200 import _abi
    lib = _abi.lib()
    n = int(lib.discoeb_fma_rate_threads())
    if n <= 0:
        raise RuntimeError(f"discoeb_fma_rate_threads failed with code {n}")
    out = torch.empty(n, dtype=torch.float64, device=device)
    stream = torch.cuda.current_stream(device)
    flops = ctypes.c_double(0.0)
    best = 0.0
    for i in range(6):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        rc = lib.discoeb_fma_rate(65536, out.data_ptr(), n, ctypes.byref(flops), stream.cuda_stream)
        e1.record(stream)
        e1.synchronize()
        if rc != 0:
            raise RuntimeError(f"discoeb_fma_rate failed with code {rc}")
        if i > 0:
            best = max(best, flops.value / (e0.elapsed_time(e1) * 1e-3) / 1e12)
    if not bool(torch.isfinite(out).all()):
        raise RuntimeError("discoeb_fma_rate produced non-finite values")
    return best


def fp64_peak_tflops(torch, device):
    """Measured FP64 peak on this GPU: cuBLAS DGEMM 8192^3, best of 5."""
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device=device)
    b = torch.randn(n, n, dtype=torch.float64, device=device)
    torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 0.0
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        e1.synchronize()
        best = max(best, 2 * n**3 / (e0.elapsed_time(e1) * 1e-3) / 1e12)
    del a, b
    torch.cuda.empty_cache()
    return best


def run_batch(args, rank, world, local):
    """Many cosmologies in one forward launch: --n-cosmo cosmologies drawn from the uneven-batch box
    (seed 0), 256 log-spaced modes each over [1e-4, 5] /Mpc, P(k) at z = 0, l_max 12/12/17/17/5,
    rtol 1e-5 / atol 1e-8.  value = k-mode solves/s of the whole launch (inputs resident)."""
    import torch

    from discoeb_b200.gradients import theta_to_params
    from discoeb_b200.perturbations import CosmologyBatch, backgrounds
    from discoeb_b200.workloads import crosses_phantom_divide, sample_thetas

    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    thetas = sample_thetas(args.n_cosmo, seed=0)
    t0 = time.perf_counter()
    bgs = [] if args.grad else backgrounds([theta_to_params(t) for t in thetas],
                                           device=device if args.host_backend == "device" else None)
    host_s = time.perf_counter() - t0
    L = dict(lmaxg=12, lmaxgp=12, lmaxr=17, lmaxnu=17, nqmax=5)
    ks = np.geomspace(1e-4, 5.0, 256)
    if args.grad:
        from discoeb_b200.gradients import JacobianBatch
        t0 = time.perf_counter()
        batch = JacobianBatch(thetas, kmodes=ks, aexp_out=np.array([1.0]), rtol=1e-5, atol=1e-8, device=device,
                              host_backend=args.host_backend, **L)
        host_s = time.perf_counter() - t0
    else:
        batch = CosmologyBatch(params=bgs, kmodes=ks, aexp_out=np.array([1.0]), rtol=1e-5, atol=1e-8, device=device,
                               **L)
    stream = torch.cuda.current_stream(device)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=device)
    for _ in range(args.warmup):
        batch.launch()
    torch.cuda.synchronize()
    times = []
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            batch.launch()
            e1.record(stream)
            e1.synchronize()
            times.append(e0.elapsed_time(e1))
    status, nsteps = batch.result(on_failure="ignore")[-2:]
    ms = statistics.mean(times)
    cross = np.array([crosses_phantom_divide(t) for t in thetas])
    ok = status == 0
    if rank == 0:
        print(json.dumps({
            "metric": ("fwd+grad (forward-mode tangents)" if args.grad else "forward") +
                      " k-mode solves/s, many cosmologies per launch",
            "value": world * ok.size / (ms / 1e3),
            "unit": "k-mode solves/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "dtype": "f64",
            "data": "synthetic (seeded uniform box of cosmologies)",
            "config": {"workload": f"box_{args.n_cosmo}x256", "n_cosmo": args.n_cosmo, "num_k": 256,
                       "mode": "fwd+grad" if args.grad else "forward",
                       "ms_per_cosmology": ms / args.n_cosmo, "host_background_s": host_s,
                       "host_backend": args.host_backend,
                       "modes_ok": int(ok.sum()), "modes_failed": int((~ok).sum()),
                       "cosmologies_crossing_w_minus_1": int(cross.sum()),
                       "failed_in_crossing_cosmologies": int((~ok[cross]).sum()) if cross.any() else 0,
                       "step_attempts_sum": int(nsteps.sum())},
            "clocks": clk.summary()}), flush=True)


def run_cmb(args, rank, world, local):
    """C_l^TT of one cosmology at the reference's compute_Cell_spectrum_from_cosmo_params defaults
    (128 camb-sampled modes, lmax 11/11/11/8/3, 320 output times, rtol = atol = 1e-4, 8192 dense k,
    16384 FFTLog points, l <= 2500), DISCO-Notebook cosmology.  Device stages timed with CUDA events
    (full solve, sources, line of sight, C_l); e2e = the public call with the host background."""
    import torch

    from discoeb_b200 import cmb
    from discoeb_b200.perturbations import solve_modes, k_sampling

    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    cmb.set_los_contraction(args.los_contraction, 7)
    p = {"Omegam": 0.3099, "Omegab": 0.0488911, "H0": 67.742, "n_s": 0.96822, "A_s": 2.1064e-09, "mnu": 0.06,
         "Tcmb": 2.7255, "YHe": 0.248, "Neff": 2.046, "Nmnu": 1, "w_DE_0": -0.99, "w_DE_a": 0.0, "cs2_DE": 1.0,
         "Omegak": 0.0, "k_p": 0.05}
    from discoeb_b200.background import evolve_background
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        bg = evolve_background(param=dict(p), num_thermo=1024)
    L = dict(lmaxg=11, lmaxgp=11, lmaxr=11, lmaxnu=8, nqmax=3)
    a = cmb.cmb_aexp_out()
    ks = k_sampling(bg, 1e-4, 1.0, 128, "camb")
    tau = bg["tau_of_a_spline"].evaluate(a)
    tau0 = float(bg["tau_of_a_spline"].evaluate(1.0))
    stream = torch.cuda.current_stream(device)
    ev = lambda: torch.cuda.Event(enable_timing=True)  # noqa: E731

    def stages():
        e = [ev() for _ in range(5)]
        e[0].record(stream)
        y = solve_modes(param=bg, kmodes=ks, tau_out=tau, rtol=1e-4, atol=1e-4, pcoeff=0.25, icoeff=0.8,
                        dcoeff=0.0, factormax=20.0, factormin=0.3, max_steps=2048, return_full=True, as_tensor=True,
                        device=device, **L)
        e[1].record(stream)
        src = cmb.compute_sources(param=bg, yout=y, kmodes=ks, aexp_out=a, device=device, **L)
        e[2].record(stream)
        th, kk = cmb.compute_theta_ell(2500, ks, tau, src["S"], tau0, n_fftlog=16384, n_k_dense=8192, device=device)
        e[3].record(stream)
        cmb.compute_Cell(th, kk, bg["n_s"], bg["k_p"], device=device)
        e[4].record(stream)
        e[4].synchronize()
        return [e[i].elapsed_time(e[i + 1]) for i in range(4)]

    def fused():  # the solve with the source assembly in its output stage (discoeb_fwd_sources)
        e = [ev() for _ in range(2)]
        e[0].record(stream)
        cmb.solve_sources(param=bg, kmodes=ks, aexp_out=a, rtol=1e-4, atol=1e-4, max_steps=2048, device=device, **L)
        e[1].record(stream)
        e[1].synchronize()
        return e[0].elapsed_time(e[1])

    for _ in range(args.warmup):
        stages()
        fused()
    with ClockSampler(local) as clk:
        times = [stages() for _ in range(args.steps)]
    per = np.mean(np.array(times), axis=0)
    fused_ms = statistics.mean([fused() for _ in range(args.steps)])
    # the line of sight alone with its frequency sum on the int8 tensor cores (the default) and as
    # an FP64 DGEMM, on the same sources, and the largest relative difference of their C_l^TT
    y = solve_modes(param=bg, kmodes=ks, tau_out=tau, rtol=1e-4, atol=1e-4, pcoeff=0.25, icoeff=0.8, dcoeff=0.0,
                    factormax=20.0, factormin=0.3, max_steps=2048, return_full=True, as_tensor=True, device=device,
                    **L)
    src_S = cmb.compute_sources(param=bg, yout=y, kmodes=ks, aexp_out=a, device=device, **L)["S"]
    before = cmb.get_los_contraction()

    def los(kind):
        cmb.set_los_contraction(kind, 7)
        e = [ev() for _ in range(2)]
        e[0].record(stream)
        th, kk = cmb.compute_theta_ell(2500, ks, tau, src_S, tau0, n_fftlog=16384, n_k_dense=8192, device=device)
        e[1].record(stream)
        e[1].synchronize()
        return e[0].elapsed_time(e[1]), cmb.compute_Cell(th, kk, bg["n_s"], bg["k_p"], device=device).cpu().numpy()

    los("fp64"), los("int8")
    los_t = {kind: [los(kind) for _ in range(args.steps)] for kind in ("fp64", "int8")}
    cmb.set_los_contraction(*before)
    cl64, cl8 = los_t["fp64"][0][1], los_t["int8"][0][1]
    los_cmp = {"int8_slices7_ms": statistics.mean(t for t, _ in los_t["int8"]),
               "fp64_dgemm_ms": statistics.mean(t for t, _ in los_t["fp64"]),
               "cl_tt_max_rel_diff": float(np.max(np.abs(cl8[2:] / cl64[2:] - 1.0)))}
    e2e = []
    for i in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        with warnings.catch_warnings():
            warnings.simplefilter("ignore")
            cmb.compute_Cell_spectrum_from_cosmo_params(dict(p), device=device)
        if i >= args.warmup:
            e2e.append(time.perf_counter() - t0)
    if rank == 0:
        ms = float(per.sum())
        print(json.dumps({
            "metric": "C_l^TT pipeline of one cosmology (compute_Cell_spectrum_from_cosmo_params defaults)",
            "value": 1e3 / ms, "unit": "spectra/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms, "higher_is_better": True, "dtype": "f64", "data": "synthetic (DISCO-Notebook cosmology)",
            "config": {"workload": "cmb_tt_disco_notebook_k128_l2500", "num_k": 128, "n_tau": 320, "n_k_dense": 8192,
                       "n_fftlog": 16384, "ellmax": 2500},
            "stages_ms": {"full_solve": per[0], "sources": per[1], "line_of_sight": per[2], "cell": per[3]},
            "fused_solve_and_sources_ms": fused_ms,
            "line_of_sight_contraction": los_cmp,
            "e2e": {"value": 1.0 / statistics.mean(e2e), "unit": "spectra/s", "ms_per_cosmology":
                    1e3 * statistics.mean(e2e)},
            "clocks": clk.summary(),
        }), flush=True)


def run_los_gemm(args, rank, world, local):
    """The line of sight's frequency sum alone: theta = A B^T with A [m, k] the FFTLog coefficient
    rows, B [n, k] the M_l(p) table (default sizes: 8192 dense modes, l <= 2500, 16384 FFTLog points,
    so k = 2 x 8193 interleaved (re, im) pairs), synthetic operands with the same decay over the
    frequencies.  Times discoeb_dgemm_i8 (the whole call: splitting, tensor-core product,
    reduction), the cuBLAS DGEMM it replaces, and cuBLASLt's int8 GEMM (torch._int_mm) as the
    measured int8 tensor rate of this GPU."""
    import torch

    from discoeb_b200 import _abi

    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    lib = _abi.lib()
    m, n, k, sl = args.gemm_m, args.gemm_n, args.gemm_k, args.slices
    g = torch.Generator(device=device)
    g.manual_seed(1234)
    q = torch.arange(k, device=device, dtype=torch.float64)
    A = torch.randn(m, k, dtype=torch.float64, device=device, generator=g) * torch.exp(-q / 3000.0)
    B = torch.randn(n, k, dtype=torch.float64, device=device, generator=g) * (1.0 + q) ** -0.8
    C = torch.empty(m, n, dtype=torch.float64, device=device)
    nb = lib.discoeb_dgemm_i8_workspace_bytes(m, n, k, sl, 0)
    ws = torch.empty(nb // 8 + 32, dtype=torch.float64, device=device)
    al = (ws.data_ptr() + 255) // 256 * 256
    stream = torch.cuda.current_stream(device)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=device)  # 256 MB > L2

    def timed(fn):
        flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fn()
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1)

    i8 = lambda: lib.discoeb_dgemm_i8(m, n, k, A.data_ptr(), k, 0, B.data_ptr(), k, 0, C.data_ptr(), n, sl, 0, al,  # noqa
                                      nb, stream.cuda_stream)
    f64 = lambda: torch.mm(A, B.T)  # noqa: E731
    ai = torch.randint(-127, 128, (8192, 16384), dtype=torch.int8, device=device)
    bi = torch.randint(-127, 128, (16384, 8192), dtype=torch.int8, device=device)
    imm = lambda: torch._int_mm(ai, bi)  # noqa: E731
    for _ in range(args.warmup):
        i8(), f64(), imm()
    with ClockSampler(local) as clk:
        t8 = [timed(i8) for _ in range(args.steps)]
    t64 = [timed(f64) for _ in range(args.steps)]
    tim = [timed(imm) for _ in range(args.steps)]
    ref = torch.mm(A, B.T)
    i8()
    torch.cuda.synchronize()
    rowmax = ref.abs().max(dim=1).values
    err = float(((C - ref).abs().max(dim=1).values / rowmax).max())
    # what the tensor cores execute: slices (slices + 1) / 2 digit-plane products over the padded tiles
    pad = lambda x, t: (x + t - 1) // t * t  # noqa: E731
    ops = 2.0 * sl * (sl + 1) / 2 * pad(m, 256) * pad(n, 256) * pad(k, 128)
    peak = 2.0 * 8192 * 16384 * 8192 / (min(tim) * 1e-3) / 1e12
    ms = statistics.mean(t8)
    if rank == 0:
        print(json.dumps({
            "metric": "line-of-sight frequency sum theta = A B^T (FP64 result)", "value": 1e3 / ms,
            "unit": "contractions/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "dtype": "f64 result from int8 digit planes", "data": "synthetic",
            "config": {"workload": f"los_contraction_m{m}_n{n}_k{k}", "slices": sl, "l2": "flushed (256 MB write)"},
            "dgemm_i8_ms": ms, "cublas_dgemm_ms": statistics.mean(t64), "speedup_vs_dgemm": statistics.mean(t64) / ms,
            "max_err_over_rowmax": err,
            "roofline": {"bound": "tensor", "achieved": ops / (ms * 1e-3) / 1e12, "peak": peak, "unit": "TOPS (int8)",
                         "frac": ops / (ms * 1e-3) / 1e12 / peak,
                         "peak_source": "cuBLASLt int8 GEMM 8192 x 16384 x 8192 (torch._int_mm), best of the run",
                         "achieved_source": "whole dgemm_i8 call (splitting and reduction included)"},
            "clocks": clk.summary(),
        }), flush=True)


def run_cmb_grad(args, rank, world, local):
    """C_l^TT and dC_l/dtheta (8 parameters) of one cosmology through cmb.compute_Cell_jacobian:
    background with six forward-mode tangents, one discoeb_jvp_full launch (states and their
    tangents at every output time), then the sources, line of sight and C_l at the base point and
    at four points along each tangent.  DISCO-Notebook cosmology; the reference's
    compute_Cell_spectrum_from_cosmo_params defaults, or with ``--cmb-large`` photon and
    polarisation l_max 50, 2000 modes over [5e-5, 0.5] and 2000 source times.  Wall-clock per
    call (host and device, results back on the host), next to the forward chain's."""
    import torch

    from discoeb_b200 import cmb

    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    cmb.set_los_contraction(args.los_contraction, 7)
    h = 0.67742
    theta = {"omega_c": (0.3099 - 0.0488911) * h * h, "omega_b": 0.0488911 * h * h, "h": h, "n_s": 0.96822,
             "ln10As": math.log(2.1064e-9 * 1e10), "w0": -0.99, "wa": 0.0, "m_nu": 0.06}
    if args.cmb_large:
        opts = dict(nmodes=2000, kmin=5e-5, kmax=0.5, lmaxg=50, lmaxgp=50, lmaxr=17, lmaxnu=17, nqmax=5,
                    aexp_out=cmb.cmb_aexp_out(200, 400, 800, 600))
        name = "cmb_tt_grad_disco_notebook_lmax50_k2000_tau2000_l2500"
    else:
        opts = {}
        name = "cmb_tt_grad_disco_notebook_k128_l2500"
    from discoeb_b200.gradients import theta_to_params

    def timed(fn):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        out = fn()
        torch.cuda.synchronize()
        return time.perf_counter() - t0, out

    fwd = lambda: cmb.compute_Cell_spectrum_from_cosmo_params(theta_to_params(theta), device=device, **opts)  # noqa
    grad = lambda: cmb.compute_Cell_jacobian(theta, device=device, **opts)  # noqa
    for _ in range(args.warmup):
        with warnings.catch_warnings():
            warnings.simplefilter("ignore")
            fwd()
            grad()
    tf, tg = [], []
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            with warnings.catch_warnings():
                warnings.simplefilter("ignore")
                tf.append(timed(fwd)[0])
                dt, (C, J, _) = timed(grad)
                tg.append(dt)
    if rank == 0:
        ms = 1e3 * statistics.mean(tg)
        print(json.dumps({
            "metric": "C_l^TT and dC_l/dtheta (8 parameters) of one cosmology", "value": 1e3 / ms,
            "unit": "spectra+gradients/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms, "higher_is_better": True, "dtype": "f64", "data": "synthetic (DISCO-Notebook cosmology)",
            "config": {"workload": name, "gradient_of": "C_l w.r.t. omega_c, omega_b, h, n_s, ln10As, w0, wa, m_nu",
                       "los_contraction": args.los_contraction,
                       **{k: (v if not isinstance(v, np.ndarray) else int(v.shape[0])) for k, v in opts.items()}},
            "e2e": {"value": 1e3 / ms, "unit": "spectra+gradients/s", "ms_per_cosmology": ms},
            "forward_only_ms": 1e3 * statistics.mean(tf),
            "finite": bool(np.isfinite(C).all() and np.isfinite(J).all()),
            "clocks": clk.summary(),
        }), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="pk_lcdm_mnu_k512_z4")
    ap.add_argument("--mode", default="fwd+grad", choices=["fwd+grad", "forward", "cmb", "cmb-grad", "batch",
                                                          "los-gemm"])
    ap.add_argument("--gemm-m", type=int, default=8192, help="--mode los-gemm: rows of A (dense modes)")
    ap.add_argument("--gemm-n", type=int, default=2501, help="--mode los-gemm: rows of B (multipoles)")
    ap.add_argument("--gemm-k", type=int, default=16386, help="--mode los-gemm: contraction length")
    ap.add_argument("--slices", type=int, default=7, help="--mode los-gemm: digit planes per operand")
    ap.add_argument("--jvp-records", default="auto", choices=["auto", "always", "never"],
                    help="fwd+grad: where the gradient kernel keeps its step records (auto: the split record "
                         "only where it lets more directions share a block)")
    ap.add_argument("--los-contraction", default="int8", choices=["int8", "fp64"],
                    help="--mode cmb / cmb-grad: the line of sight's frequency sum on the int8 tensor cores "
                         "(7 digit planes) or as an FP64 DGEMM")
    ap.add_argument("--cmb-large", action="store_true", help="cmb-grad: l_max 50, 2000 modes, 2000 source times")
    ap.add_argument("--n-cosmo", type=int, default=64, help="cosmologies per launch in --mode batch")
    ap.add_argument("--grad", action="store_true", help="--mode batch: forward + gradient (discoeb_jvp)")
    ap.add_argument("--host-backend", default="native", choices=["native", "device"],
                    help="--mode batch: backgrounds on the host (native C++) or in one GPU launch")
    ap.add_argument("--wpb", type=int, default=0, help="warps (modes) per block; 0 = the library default")
    ap.add_argument("--method", default="structured", choices=["structured", "structured-mixed"],
                    help="--mode forward: FP64 chain factors, or FP32 factors with an FP64 refinement")
    ap.add_argument("--ref-sample", type=int, default=16)
    ap.add_argument("--no-adjoint", action="store_true", help="fwd+grad: skip the reverse-mode timing")
    ap.add_argument("--checkpoint-every", type=int, default=16, help="adjoint: steps between stored states")
    ap.add_argument("--no-accuracy", action="store_true", help="skip the oracle accuracy check")
    ap.add_argument("--cpu-sample", type=int, default=16)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--kernel-only", action="store_true", help="skip the e2e loop and the FP64 peak (profiling)")
    ap.add_argument("--num-k", type=int, default=0, help="override the workload's mode count (small profiling case)")
    args = ap.parse_args()
    rank = _env_int("RANK", 0)
    world = _env_int("WORLD_SIZE", 1)
    local = _env_int("LOCAL_RANK", 0)
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if args.mode == "cmb":
        run_cmb(args, rank, world, local)
        return
    if args.mode == "cmb-grad":
        run_cmb_grad(args, rank, world, local)
        return
    if args.mode == "los-gemm":
        run_los_gemm(args, rank, world, local)
        return
    if args.mode == "batch":
        run_batch(args, rank, world, local)
        return

    import ctypes

    import torch

    from discoeb_b200 import _abi
    from discoeb_b200 import perturbations as pert
    from discoeb_b200.workloads import workload

    from discoeb_b200 import replicas

    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    rank, world, dist = replicas.init("nccl", device=device)
    w = workload(args.workload)
    if args.num_k > 0:
        w["num_k"] = args.num_k
    bg = _background(w)
    L = {k: w[k] for k in ("lmaxg", "lmaxgp", "lmaxr", "lmaxnu", "nqmax")}
    n = pert.nvar_of(**L)
    kmodes = np.geomspace(w["kmin"], w["kmax"], w["num_k"])
    K = kmodes.shape[0]
    aout = np.asarray(w["aexp_out"], dtype=np.float64)
    tau_out = bg["tau_of_a_spline"].evaluate(aout)
    nout = tau_out.shape[0]

    # ---- device-resident inputs for the kernel-only measurement ----
    tau_s = pert.determine_starting_time(param=bg, k=kmodes)
    tau_start = 0.99 * np.minimum(tau_out.min(), tau_s)
    y0 = pert.adiabatic_ics(tau=tau_start, param=bg, kmode=kmodes, **L)
    sw = pert.approximation_switch_times(bg, kmodes)
    order = np.argsort(-kmodes, kind="stable")
    dc = pert.DeviceCosmo(bg, de_guard_eps=1e-9, device=device, **L)
    f64 = dict(dtype=torch.float64, device=device)
    d_k = torch.tensor(kmodes[order], **f64)
    d_ts = torch.tensor(tau_start[order], **f64)
    d_y0 = torch.tensor(y0[order], **f64).contiguous()
    d_sw = torch.tensor(sw[order], **f64).contiguous()
    d_tout = torch.tensor(tau_out, **f64)
    d_out = torch.empty((K, nout, 20), **f64)
    d_stat = torch.empty((2, K), dtype=torch.int32, device=device)
    methods = {"structured": _abi.METHOD_RODAS5_STRUCTURED, "structured-mixed": _abi.METHOD_RODAS5_STRUCTURED_MIXED}
    ctrl = _abi.DiscoebControl(w["rtol"], w["atol"], 0.25, 0.80, 0.0, 20.0, 0.3, 100000, methods[args.method],
                               args.wpb, 0)
    lib = _abi.lib()
    stream = torch.cuda.current_stream(device)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=device)  # > 126 MB L2

    def forward(c=ctrl, out=d_out):
        rc = lib.discoeb_fwd(dc.struct.data_ptr(), ctypes.byref(dc.host), 1, ctypes.byref(c), K, None,
                             d_k.data_ptr(), d_ts.data_ptr(), d_y0.data_ptr(), d_sw.data_ptr(), nout,
                             d_tout.data_ptr(), None, out.data_ptr(), d_stat[0].data_ptr(), d_stat[1].data_ptr(),
                             stream.cuda_stream)
        if rc != 0:
            raise RuntimeError(f"discoeb_fwd returned {rc}")

    grad = args.mode == "fwd+grad"
    if grad:
        from discoeb_b200.gradients import JacobianProblem, power_spectrum_jacobian
        prob = JacobianProblem(w["theta"], aexp_out=aout, kmodes=kmodes, rtol=w["rtol"], atol=w["atol"],
                               max_steps=100000, device=device, warps_per_block=args.wpb, **L)
        n_dir = len(prob.dirs)
        rec_opt = {"auto": True, "always": "always", "never": False}[args.jvp_records]
        solve, stat_of = (lambda: prob.launch(records=rec_opt)), (lambda: prob.d_stat)
    else:
        n_dir = 0
        solve, stat_of = forward, (lambda: d_stat)

    for _ in range(args.warmup):
        solve()
    torch.cuda.synchronize()
    stat = stat_of().cpu().numpy()
    if (stat[0] != 0).any():
        raise RuntimeError(f"{int((stat[0] != 0).sum())} modes failed")
    step_attempts = int(stat[1].sum())  # per mode (every direction of a mode takes the same steps)

    def barrier():
        replicas.barrier(dist)
        torch.cuda.synchronize()

    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    with ClockSampler(local) as clk:
        barrier()
        for i in range(args.steps):
            flush.zero_()  # evict L2 between timed solves (outside the events)
            starts[i].record(stream)
            solve()
            ends[i].record(stream)
        barrier()
    times_ms = [s.elapsed_time(e) for s, e in zip(starts, ends)]
    clocks = clk.summary()
    ms = replicas.max_over_ranks(statistics.mean(times_ms), dist, device)
    value = world * K / (ms / 1e3)

    fwd_ms = mixed_ms = None
    d_out_mixed = None
    if grad:  # the forward solve alone, for comparison (same events and L2 flush), in FP64 and in the
        # mixed-precision form (FP32 chain factors, one FP64 refinement per chain solve)
        ctrl_mixed = _abi.DiscoebControl(w["rtol"], w["atol"], 0.25, 0.80, 0.0, 20.0, 0.3, 100000,
                                         _abi.METHOD_RODAS5_STRUCTURED_MIXED, args.wpb, 0)
        d_out_mixed = torch.empty_like(d_out)

        def timed_forward(fn):
            for _ in range(args.warmup):
                fn()
            times = []
            for i in range(args.steps):
                flush.zero_()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                fn()
                e1.record(stream)
                e1.synchronize()
                times.append(e0.elapsed_time(e1))
            return replicas.max_over_ranks(statistics.mean(times), dist, device)

        fwd_ms = timed_forward(forward)
        mixed_ms = timed_forward(lambda: forward(ctrl_mixed, d_out_mixed))
        if (d_stat[0] != 0).any():
            raise RuntimeError("the mixed-precision forward solve failed")

    # ---- reverse mode (discrete adjoint) on the same modes: the recorded forward plus one reverse
    # sweep per mode whose cotangent is that mode's P(k, z = 0) (every row of dP(k, z=0)/dtheta),
    # and the gradient of a scalar loss (one reverse sweep per mode, cotangent on every output)
    adj = None
    if grad and not args.no_adjoint:
        from discoeb_b200.gradients import AdjointProblem
        ap = AdjointProblem(w["theta"], aexp_out=aout, kmodes=kmodes, rtol=w["rtol"], atol=w["atol"],
                            max_steps=100000, device=device, checkpoint_every=args.checkpoint_every, **L)
        wts = torch.ones((K, nout), dtype=torch.float64, device=device)

        def timed(fn):
            ts = []
            for i in range(args.warmup + args.steps):
                flush.zero_()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                fn()
                e1.record(stream)
                e1.synchronize()
                if i >= args.warmup:
                    ts.append(e0.elapsed_time(e1))
            return replicas.max_over_ranks(statistics.mean(ts), dist, device)

        ap.launch_forward()
        torch.cuda.synchronize()
        if (ap.forward_power(on_failure="ignore")[1] != 0).any():
            raise RuntimeError("the recorded forward solve failed")
        rec_ms = timed(ap.launch_forward)
        rows_ms = timed(lambda: ap.launch_jacobian_rows(out_index=-1))
        loss_ms = timed(lambda: ap.launch_backward(wts))
        J_rows = ap.jacobian_rows()[0]
        adj = {"jacobian_rows_z0": {"value": world * K / ((rec_ms + rows_ms) / 1e3), "unit": UNIT,
                                    "ms_per_cosmology": rec_ms + rows_ms, "forward_record_ms": rec_ms,
                                    "reverse_ms": rows_ms},
               "scalar_loss_gradient": {"ms_per_cosmology": rec_ms + loss_ms, "reverse_ms": loss_ms},
               "checkpoint_every": args.checkpoint_every}

    # ---- end to end through the public API (host arrays in, host arrays out) ----
    e2e_ms = []
    for i in range(0 if args.kernel_only else args.warmup + args.steps):
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        if grad:
            power_spectrum_jacobian(w["theta"], aexp_out=aout, kmin=w["kmin"], kmax=w["kmax"], num_k=w["num_k"],
                                    rtol=w["rtol"], atol=w["atol"], max_steps=100000, k_sampling_method="log",
                                    host_threads=0, **L)
        else:
            pert.evolve_perturbations(param=dict(bg), aexp_out=aout, kmin=w["kmin"], kmax=w["kmax"],
                                      num_k=w["num_k"], rtol=w["rtol"], atol=w["atol"], max_steps=100000,
                                      k_sampling_method="log", **L)
        e1.record(stream)
        e1.synchronize()
        if i >= args.warmup:
            e2e_ms.append(e0.elapsed_time(e1))
    e2e = replicas.max_over_ranks(statistics.mean(e2e_ms) if e2e_ms else float("nan"), dist, device)
    h2d = 8 * (2 * K + K * n + 3 * K + nout) + sum(t.numel() * 8 for t in dc.tensors) + ctypes.sizeof(dc.host)
    d2h = 8 * K * nout * 20 + 8 * K
    if grad:  # + tangent tables, tangent structs, initial-state and output-time tangents; + output tangents
        h2d += sum(t.numel() * 8 for t in prob._keep) + prob.d_tan.numel() + 8 * n_dir * (K * n + nout)
        d2h += 8 * n_dir * K * nout * 20

    # ---- roofline: FP64 work of the structured Rodas5 step against a measured FP64 peak ----
    # (counted by ncu where a capture exists, FP64_FLOPS_PER_ATTEMPT; else estimated from the code)
    flops_per_step = 850.0 * n + 1650.0  # forward structured step, counted from stepper.cuh
    # one tangent direction's work per step, estimated from the operation mix of tangent_step
    # (stepper.cuh): 8 stages x (two dual RHS passes ~ 4 real RHS passes of ~10 n + 300 flops, one
    # W solve ~30 n, stage sums and the column-0 term ~16 n) + once per step a hyper-dual RHS pass
    # (~4 real passes) and the stage-state rebuild (~24 n)
    tangent_per_step = 8.0 * (4.0 * (10.0 * n + 300.0) + 46.0 * n) + 4.0 * (10.0 * n + 300.0) + 24.0 * n
    dense_per_step = (2.0 / 3.0) * n**3 + 16.0 * n**2 + 45.0 * n * n  # reference algorithm: LU + 8 solves + jacfwd
    # forward once per mode, each direction's tangent on every step (counted on every attempt:
    # an upper bound, the tangent runs on accepted steps only)
    work = step_attempts * (flops_per_step + tangent_per_step * n_dir) if grad else step_attempts * flops_per_step
    flops_source = "estimated from the operation mix of the step code (upper bound: every attempt)"
    if args.mode in FP64_FLOPS_PER_ATTEMPT and args.workload == "pk_lcdm_mnu_k512_z4" and args.method == "structured":
        work = step_attempts * FP64_FLOPS_PER_ATTEMPT[args.mode]
        flops_source = ("ncu FP64 thread instructions (dadd + dmul + 2 dfma) per step attempt of a 48-mode launch "
                        "of the same kernel, times this launch's step attempts")
    dense_work = step_attempts * dense_per_step * (1 + n_dir)
    achieved = work / (ms / 1e3) / 1e12
    peak = fp64_fma_tflops(torch, device) if rank == 0 and not args.kernel_only else None
    dgemm = fp64_peak_tflops(torch, device) if rank == 0 and not args.kernel_only else None

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline and not args.kernel_only:
        from oracle import pyoracle as O
        ks = _sample_modes(w, args.cpu_sample)
        th = os.cpu_count() or 1
        bgs = [bg] + (_shifted_backgrounds(w) if grad else [])
        t0 = time.perf_counter()
        for b in bgs:
            O.evolve_perturbations(param=b, aexp_out=aout, kmin=0, kmax=0, num_k=0, rtol=w["rtol"], atol=w["atol"],
                                   kmodes=ks, mode="reference", de_guard_eps=1e-9, max_steps=100000, threads=th, **L)
        dt = time.perf_counter() - t0
        how = ", forward + central-difference Jacobian (13 solves per mode)" if grad else ""
        cpu = {"value": len(ks) / dt, "unit": UNIT, "cores": th, "kind": "port",
               "sample": f"{len(ks)} modes spread over the workload's k range, oracle dense-LU Rodas5{how}, "
                         f"{dt:.1f} s"}

    accuracy = None
    if rank == 0 and world == 1 and not args.no_accuracy and not args.kernel_only:
        # the checker: the GPU's results of the timed launches against the converged oracle
        P_other = None
        if grad:
            P_gpu, J_gpu = prob.result()[:2]
            inv = np.empty_like(order)
            inv[order] = np.arange(K)
            P_other = {"forward_only_mixed": pert.get_power(k=kmodes[:, None], y=d_out_mixed.cpu().numpy()[inv],
                                                            idx=4, param=bg)}
        else:
            inv = np.empty_like(order)
            inv[order] = np.arange(K)
            P_gpu = pert.get_power(k=kmodes[:, None], y=d_out.cpu().numpy()[inv], idx=4, param=bg)
            J_gpu = None
        accuracy = oracle_accuracy(w, bg, kmodes, P_gpu, J_gpu, n_j=8 if grad else 0,
                                   J_rows=J_rows if adj is not None else None, P_other=P_other)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded cosmology, no dataset)",
            "config": {"workload": args.workload, "mode": args.mode, "num_k": K, "nvar": n, "n_out": nout,
                       "tangent_directions": n_dir, "gradient_of": "P(k) at every output w.r.t. omega_c, omega_b, h, "
                       "n_s, ln10As, w0, wa, m_nu" if grad else None,
                       "gradient_method": "forward-mode tangents (discoeb_jvp: 6 directions through the solver, "
                       "n_s and ln10As analytic)" if grad else None,
                       "jvp_records": args.jvp_records if grad else None,
                       "rtol": w["rtol"], "atol": w["atol"],
                       "method": "rodas5-structured" + ("-mixed" if args.method == "structured-mixed" and not grad
                                                        else ""),
                       "l2": "flushed between steps (256 MiB write outside the timed events)",
                       "ms_per_cosmology": ms, "step_attempts_per_mode_sum": step_attempts,
                       "warps_per_block": args.wpb or "default"},
            "e2e": {"value": world * K / (e2e / 1e3), "unit": UNIT, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "ms_per_cosmology": e2e},
            "gpu_launches": args.steps,
            "roofline": {"bound": "fp64", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                         "frac": (achieved / peak) if peak else None,
                         "traffic": DRAM_BYTES_PER_MODE.get(args.mode, 0.0) * K or None,
                         "traffic_source": "ncu capture of 48 modes of the same kernel, scaled by the mode count",
                         "peak_source": "FP64 FMA throughput measured in this run (discoeb_fma_rate)",
                         "flops_source": flops_source,
                         "fp64_dgemm_tflops": dgemm,
                         "dense_equivalent_tflops": dense_work / (ms / 1e3) / 1e12},
            "clocks": clocks,
        }
        if fwd_ms is not None:
            line["forward_only"] = {"value": world * K / (fwd_ms / 1e3), "unit": UNIT, "ms_per_cosmology": fwd_ms}
            line["forward_only_mixed"] = {"value": world * K / (mixed_ms / 1e3), "unit": UNIT,
                                          "ms_per_cosmology": mixed_ms,
                                          "method": "FP32 chain factors + one FP64 refinement per chain solve"}
        if cpu is not None:
            line["cpu_baseline"] = cpu
        if accuracy is not None:
            line["max_rel_err"] = accuracy
        if adj is not None:
            line["adjoint"] = adj
        print(json.dumps(line), flush=True)
    replicas.finish(dist)


if __name__ == "__main__":
    main()

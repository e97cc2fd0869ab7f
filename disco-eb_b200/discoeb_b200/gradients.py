"""Derivatives of P(k) with respect to cosmological parameters.

The reference obtains them with ``jax.jacfwd`` through ``evolve_background`` and the diffrax
solve (``DirectAdjoint``, perturbations.py:919; the gradient notebooks
``notebooks/nb_minimal_example.ipynb``, ``paper_scripts/nb_discoeb_fisher_forecast.ipynb``).
Here the same forward-mode derivative is assembled from two exact pieces:

* the background tables, scalar parameters, initial states and output times are
  differentiated on the host: ``discoeb_background`` carries one forward-mode derivative per
  parameter direction through the background and Recfast (C++, one host thread per direction;
  the derivative of the discrete background with Recfast's branches and step sequence held, as
  forward-mode AD gives), and the initial states by complex-step differentiation of
  ``adiabatic_ics``.  ``host_backend="numpy"`` takes the complex-step derivative of the numpy
  restatement with its Recfast steps replayed instead (same quantity, ~100x slower);
* the perturbation solve is differentiated on the GPU by ``discoeb_jvp``: the tangent of the
  discrete Rodas5 solution with the accepted step sequence held fixed (the step-size
  controller is not differentiated, exactly as diffrax's stop-gradient on the step factor).

The start times of the modes (a numerical choice) and the approximation switch times are held
fixed.  n_s and A_s enter P(k) only through the primordial spectrum and are differentiated
analytically.  A ``full_state`` JacobianProblem (``discoeb_jvp_full``) gives the whole states and
their tangents at every output time instead, the input of ``cmb.compute_Cell_jacobian``.
"""
from __future__ import annotations

import ctypes
import threading

import numpy as np

from . import _abi
from .background import _DIFF_FIELDS, background_from_buffer, evolve_background, native_background
from .spline import spline_interpolation
from .perturbations import (DeviceCosmo, adiabatic_ics, approximation_switch_times, determine_starting_time, k_sampling,
                            nvar_of, _check_status)
from .workloads import cosmo_params

THETA_NAMES = ("omega_c", "omega_b", "h", "n_s", "ln10As", "w0", "wa", "m_nu")
ODE_DIRECTIONS = ("omega_c", "omega_b", "h", "w0", "wa", "m_nu")
_TABLES = (("xe_of_loga_spline", "xe"), ("cs2a_of_loga_spline", "cs2a"), ("logrhonu_of_loga_spline", "logrhonu"),
           ("logpnu_of_loga_spline", "logpnu"))
_CSTEP = 1e-30


def theta_to_params(theta, **extra):
    """Reference param dict of theta = (omega_c, omega_b, h, n_s, ln10As, w0, wa, m_nu)."""
    t = dict(theta)
    return cosmo_params(h=t["h"], omega_b=t["omega_b"], omega_c=t["omega_c"], A_s=np.exp(t["ln10As"]) / 1e10,
                        n_s=t["n_s"], m_nu=t["m_nu"], w0=t["w0"], wa=t["wa"], **extra)


def _tangent_one(theta, name, trace, aexp_out, tau_start, kmodes, L, num_thermo=256):
    """Complex-step tangent of the background along one direction (Recfast steps replayed)."""
    import warnings
    tc = dict(theta)
    tc[name] = tc[name] + 1j * _CSTEP
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        bgc = evolve_background(param=theta_to_params(tc), replay=trace, num_thermo=num_thermo)
    d = {"scalars": {}, "tables": {}}
    for key, field in (("grhom", "grhom"), ("Omegam", "Omegam"), ("Omegab", "Omegab"), ("OmegaDE", "OmegaDE"),
                       ("amnu", "amnu"), ("w_DE_0", "w0"), ("w_DE_a", "wa"), ("H0", "H0")):
        d["scalars"][field] = float(np.imag(bgc[key]) / _CSTEP)
    for key, short in _TABLES:
        s = bgc[key]
        d["tables"][short] = (np.ascontiguousarray(np.imag(s.y) / _CSTEP), np.ascontiguousarray(np.imag(s.S) / _CSTEP))
    d["tau_out"] = np.imag(bgc["tau_of_a_spline"].evaluate(aexp_out)) / _CSTEP
    y0c = adiabatic_ics(tau=tau_start, param=bgc, kmode=kmodes, **L)
    d["y0"] = np.ascontiguousarray(np.imag(y0c) / _CSTEP)
    return d


def _tangent_task(args):
    return _tangent_one(*args)


_POOL = None


def _pool(nproc):
    """A persistent pool of spawned host processes (safe after CUDA is initialised), reused by
    every gradient call so that its start-up is paid once."""
    global _POOL
    if _POOL is None or _POOL[1] < nproc:
        import atexit
        import multiprocessing as mp
        if _POOL is not None:
            _POOL[0].terminate()
        _POOL = (mp.get_context("spawn").Pool(nproc), nproc)
        atexit.register(_POOL[0].terminate)
    return _POOL[0]


def background_tangents(theta, bg, trace, directions, *, aexp_out, tau_start, kmodes, L, processes=1, num_thermo=256):
    """Host-side tangents along each direction: scalars, tables, output times, initial states.

    The directions are independent: with ``processes`` > 1 (0: one per direction, up to the
    host's cores) they run in a persistent pool of spawned host processes (the calling script
    must guard its top level with ``if __name__ == "__main__":``, as spawned processes import
    it)."""
    import os
    directions = list(directions)
    nproc = min(len(directions), os.cpu_count() or 1) if not processes else processes
    args = [(dict(theta), name, trace, aexp_out, tau_start, kmodes, L, num_thermo) for name in directions]
    if nproc <= 1 or len(directions) <= 1:
        return [_tangent_task(a) for a in args]
    return _pool(nproc).map(_tangent_task, args)


def param_dots(theta, directions):
    """d(H0, Omegab, Omegam, mnu, w_DE_0, w_DE_a)/d(theta_d) for each direction (complex step of
    theta_to_params: exact for these rational maps)."""
    out = []
    for name in directions:
        tc = dict(theta)
        tc[name] = tc[name] + 1j * _CSTEP
        pc = theta_to_params(tc)
        out.append({f: float(np.imag(pc[f]) / _CSTEP) for f in _DIFF_FIELDS})
    return out


def _tangent_from_buffers(bg, buf, dot, num_thermo, aexp_out, tau_start, kmodes, L):
    """One direction's tangent record (as _tangent_one) from discoeb_background buffers."""
    lay, _ = _abi.background_layout(num_thermo)
    s = lambda nm: float(dot[lay["s:" + nm]])  # noqa: E731
    d = {"scalars": {"grhom": s("grhom"), "Omegam": s("Omegam"), "Omegab": s("Omegab"), "OmegaDE": s("OmegaDE"),
                     "amnu": s("amnu"), "w0": s("w_DE_0"), "wa": s("w_DE_a"), "H0": s("H0")}}
    c = lambda key: np.ascontiguousarray(dot[lay[key]])  # noqa: E731
    d["tables"] = {"xe": (c("t:xe"), c("t:xe_of_loga_S")), "cs2a": (c("t:cs2a"), c("t:cs2a_of_loga_S")),
                   "logrhonu": (c("n:logrhonu_y"), c("n:logrhonu_S")), "logpnu": (c("n:logpnu_y"), c("n:logpnu_S"))}
    # tau(a_out): the spline is linear in (y, S) at fixed knots
    aexp = buf[lay["t:aexp"]]
    d["tau_out"] = spline_interpolation.from_table(aexp, dot[lay["t:tau"]], dot[lay["t:tau_of_a_S"]]).evaluate(aexp_out)
    # initial states at fixed start times: complex step of adiabatic_ics through the tables it reads
    h = _CSTEP
    cx = lambda key: buf[lay[key]] + 1j * h * dot[lay[key]]  # noqa: E731
    bgc = {k: bg[k] for k in ("grhog", "grhor", "Neff", "Nmnu", "cs2_DE")}
    for key, nm in (("grhom", "grhom"), ("Omegam", "Omegam"), ("Omegab", "Omegab"), ("amnu", "amnu"),
                    ("w_DE_0", "w_DE_0"), ("w_DE_a", "w_DE_a")):
        bgc[key] = bg[key] + 1j * h * dot[lay["s:" + nm]]
    bgc["a_of_tau_spline"] = spline_interpolation.from_table(cx("t:tau"), aexp, cx("t:a_of_tau_S"))
    bgc["logrhonu_of_loga_spline"] = spline_interpolation.from_table(buf[lay["n:loga"]], cx("n:logrhonu_y"),
                                                                      cx("n:logrhonu_S"), uniform=True)
    y0c = adiabatic_ics(tau=tau_start, param=bgc, kmode=kmodes, **L)
    d["y0"] = np.ascontiguousarray(np.imag(y0c) / h)
    return d


def _native_tangents_in_background(param, num_thermo, dots, n_threads):
    """Start discoeb_background's tangent passes on a helper thread (the C++ passes hold no GIL);
    the returned function waits for them and returns the tangent buffers."""
    box = {}

    def run():
        try:
            box["dots"] = native_background(param, num_thermo, dots, n_threads)[1]
        except BaseException as e:  # re-raised in the caller's thread
            box["error"] = e

    t = threading.Thread(target=run, daemon=True)
    t.start()

    def wait():
        t.join()
        if "error" in box:
            raise box["error"]
        return box["dots"]
    return wait


def cosmology_prologue(theta, aexp_out, kmodes, L, num_thermo=256, host_backend="native", host_threads=0,
                       buffers=None):
    """Host prologue of one cosmology's P(k) Jacobian: background, output and start times,
    initial states, switch times and the per-direction tangents (ODE_DIRECTIONS).

    ``host_backend``: "native" (discoeb_background with ``host_threads`` threads, 0: one per
    direction) or "numpy" (complex step through the numpy restatement, Recfast steps replayed,
    ``host_threads`` spawned processes).  ``buffers``: the (values, tangents) buffers of this
    cosmology's background when they were computed already (discoeb_background_batch)."""
    import warnings
    aexp_out = np.atleast_1d(np.asarray(aexp_out, dtype=np.float64))
    kmodes = np.ascontiguousarray(kmodes, dtype=np.float64)
    if buffers is not None:
        host_backend = "native"
        p = theta_to_params(theta)
        buf, dots = buffers
        bg = background_from_buffer(p, buf, num_thermo)
    elif host_backend == "native":
        # the tangent passes run while this thread takes the values alone (the same bits as the
        # value part of the tangent passes) and the start times, initial states and switch times
        p = theta_to_params(theta)
        wait_dots = _native_tangents_in_background(p, num_thermo, param_dots(theta, ODE_DIRECTIONS), host_threads)
        buf = native_background(p, num_thermo)[0]
        bg = background_from_buffer(p, buf, num_thermo)
    elif host_backend == "numpy":
        trace = {}
        with warnings.catch_warnings():
            warnings.simplefilter("ignore")
            bg = evolve_background(param=theta_to_params(theta), trace=trace, num_thermo=num_thermo, backend="numpy")
    else:
        raise ValueError(f"unknown host_backend {host_backend!r}")
    tau_out = bg["tau_of_a_spline"].evaluate(aexp_out)
    if np.any(np.diff(tau_out) <= 0):
        raise ValueError("aexp_out must map to strictly increasing output times")
    tau_start = 0.99 * np.minimum(tau_out.min(), determine_starting_time(param=bg, k=kmodes))
    y0 = adiabatic_ics(tau=tau_start, param=bg, kmode=kmodes, **L)
    sw = approximation_switch_times(bg, kmodes)
    if host_backend == "native":
        if buffers is None:
            dots = wait_dots()
        tans = [_tangent_from_buffers(bg, buf, d, num_thermo, aexp_out, tau_start, kmodes, L) for d in dots]
    else:
        tans = background_tangents(theta, bg, trace, ODE_DIRECTIONS, aexp_out=aexp_out, tau_start=tau_start,
                                   kmodes=kmodes, L=L, processes=max(host_threads, 1), num_thermo=num_thermo)
    return {"bg": bg, "tau_out": tau_out, "tau_start": tau_start, "y0": y0, "sw": sw, "tans": tans}


class JacobianProblem:
    """Everything one discoeb_jvp launch needs for P(k) and dP/dtheta of one cosmology.

    The host prologue (background, its tangents, start times, initial states and their
    tangents) runs in the constructor and leaves the inputs resident on the device;
    ``launch`` enqueues the kernel on the current stream and ``result`` reads it back.
    ``host_backend`` / ``host_threads`` / ``buffers``: see cosmology_prologue (``host_processes``
    is the older name of ``host_threads``).  ``full_state``: launch discoeb_jvp_full, whose
    states and state tangents ``states`` returns, instead of the P(k) fields.
    """

    def __init__(self, theta, *, aexp_out=(1.0,), kmin=1e-4, kmax=1.0, num_k=64, kmodes=None, lmaxg=12, lmaxgp=12,
                 lmaxr=17, lmaxnu=17, nqmax=5, rtol=1e-5, atol=1e-8, pcoeff=0.25, icoeff=0.80, dcoeff=0.0,
                 factormax=20.0, factormin=0.3, max_steps=100000, k_sampling_method="log", idx=4, num_thermo=256,
                 de_guard_eps=1e-9, device=None, warps_per_block=0, host_backend="native", host_threads=0,
                 host_processes=None, full_state=False, buffers=None):
        import torch
        if device is None:
            if not torch.cuda.is_available():
                raise RuntimeError("discoeb_b200 needs a CUDA device (there is no CPU path)")
            device = torch.device("cuda", torch.cuda.current_device())
        self.torch, self.device, self.idx = torch, device, idx
        self.lib = _abi.lib()
        L = dict(lmaxg=lmaxg, lmaxgp=lmaxgp, lmaxr=lmaxr, lmaxnu=lmaxnu, nqmax=nqmax)
        if kmodes is None:
            kp = theta_to_params(theta)
            if k_sampling_method == "camb":  # needs tau_maxvis of the background
                kp = evolve_background(param=kp, num_thermo=num_thermo)
            kmodes = k_sampling(kp, kmin, kmax, num_k, k_sampling_method)
        kmodes = np.ascontiguousarray(kmodes, dtype=np.float64)
        aexp_out = np.atleast_1d(np.asarray(aexp_out, dtype=np.float64))
        if host_processes is not None:
            host_threads = host_processes
        pro = cosmology_prologue(theta, aexp_out, kmodes, L, num_thermo, host_backend, host_threads, buffers)
        bg, tau_out, tau_start, y0, sw, tans = (pro[k] for k in ("bg", "tau_out", "tau_start", "y0", "sw", "tans"))
        self.bg = bg
        K, nout = kmodes.shape[0], tau_out.shape[0]
        self.kmodes, self.K, self.nout, self.n = kmodes, K, nout, nvar_of(**L)
        self.dirs = ODE_DIRECTIONS
        # longest modes (largest k) first so that the tail of the launch is short
        order = np.argsort(-kmodes, kind="stable")
        self.order = order
        self.inv = np.empty_like(order)
        self.inv[order] = np.arange(K)
        self.dc = DeviceCosmo(bg, de_guard_eps=de_guard_eps, device=device, **L)
        f64 = dict(dtype=torch.float64, device=device)
        # every input array in one pinned host buffer and one copy (256-byte aligned slices)
        host_arrays = [kmodes[order], tau_start[order], y0[order], np.stack([d["y0"][order] for d in tans]), sw[order],
                       tau_out, np.stack([d["tau_out"] for d in tans])]
        host_arrays += [a for d in tans for (yy, SS) in d["tables"].values() for a in (yy, SS)]
        offs, o = [], 0
        for a in host_arrays:
            offs.append(o)
            o += (np.asarray(a).size + 31) // 32 * 32
        self._pinned = torch.empty(o, dtype=torch.float64, pin_memory=True)
        hp = self._pinned.numpy()
        for a, at in zip(host_arrays, offs):
            a = np.ascontiguousarray(a, dtype=np.float64)
            hp[at:at + a.size] = a.ravel()
        dev = self._pinned.to(device, non_blocking=True)
        views = [dev[at:at + np.asarray(a).size].view(np.asarray(a).shape) for a, at in zip(host_arrays, offs)]
        self.d_k, self.d_ts, self.d_y0, self.d_y0d, self.d_sw, self.d_tout, self.d_toutd = views[:7]
        self._keep = views[7:]  # the tangents' tables, in the order of the DiscoebTangent fields below
        tstructs = []
        tables = iter(self._keep)
        for d in tans:
            t = _abi.DiscoebTangent()
            for f, v in d["scalars"].items():
                setattr(t, f, v)
            for short in d["tables"]:
                setattr(t, short + "_y", next(tables).data_ptr())
                setattr(t, short + "_S", next(tables).data_ptr())
            tstructs.append(t)
        tan_arr = (_abi.DiscoebTangent * len(tstructs))(*tstructs)
        self.d_tan = torch.frombuffer(bytearray(bytes(tan_arr)), dtype=torch.uint8).to(device)
        self.full_state = bool(full_state)
        width = self.n if self.full_state else 20
        self.d_out = torch.empty((K, nout, width), **f64)
        self.d_outd = torch.empty((len(self.dirs), K, nout, width), **f64)
        self.d_stat = torch.empty((2, K), dtype=torch.int32, device=device)
        self.ctrl = _abi.DiscoebControl(rtol, atol, pcoeff, icoeff, dcoeff, factormax, factormin, int(max_steps),
                                        _abi.METHOD_RODAS5_STRUCTURED, int(warps_per_block), 0)

    def launch(self, records=True):
        """Run the launch.  ``records=False`` keeps the step records in shared memory even where a
        global workspace would let more directions share a block; ``records="always"`` uses the
        split record (factorisation in shared memory, state and stages in a global workspace) also
        where every direction already shares the block."""
        stream = self.torch.cuda.current_stream(self.device).cuda_stream
        args = (self.dc.struct.data_ptr(), ctypes.byref(self.dc.host), 1, None, self.d_tan.data_ptr(), len(self.dirs),
                ctypes.byref(self.ctrl), self.K, self.d_k.data_ptr(), self.d_ts.data_ptr(), self.d_y0.data_ptr(),
                self.d_y0d.data_ptr(), self.d_sw.data_ptr(), self.nout, self.d_tout.data_ptr(),
                self.d_toutd.data_ptr(), self.d_out.data_ptr(), self.d_outd.data_ptr(), self.d_stat[0].data_ptr(),
                self.d_stat[1].data_ptr())
        # large states (l_max 50): the step records in a global workspace let all directions share a
        # block (discoeb_jvp_records); otherwise they stay in shared memory
        size_fn = (self.lib.discoeb_jvp_split_records_bytes if records == "always" else
                   self.lib.discoeb_jvp_records_bytes)
        nb = size_fn(ctypes.byref(self.dc.host), len(self.dirs), self.K)
        if nb < 0:
            raise RuntimeError(f"discoeb_jvp_records_bytes failed with code {nb}")
        if nb > 0 and records:
            if getattr(self, "_records", None) is None or self._records.numel() * 8 < nb:
                self._records = self.torch.empty(int(nb) // 8 + 1, dtype=self.torch.float64, device=self.device)
            rc = self.lib.discoeb_jvp_records(*args, int(self.full_state), self._records.data_ptr(), int(nb), stream)
        else:
            entry = self.lib.discoeb_jvp_full if self.full_state else self.lib.discoeb_jvp
            rc = entry(*args, stream)
        if rc != 0:
            raise RuntimeError(f"discoeb_jvp failed with code {rc}")

    def state(self, on_failure="raise"):
        """y[K, nout, n]: the RSA-projected states at the output times, a device tensor in the
        caller's k order (a ``full_state`` problem)."""
        if not self.full_state:
            raise ValueError("state() needs a JacobianProblem made with full_state=True")
        stat = self.d_stat.cpu().numpy()[:, self.inv]
        _check_status(stat[0], stat[1], self.kmodes, on_failure)
        return self.d_out[self.torch.as_tensor(self.inv, device=self.device)]

    def launch_states(self, on_failure="raise"):
        """(y [K, nout, n], kmodes [K], inv): the states as the launch holds them (modes by
        descending k), without state()'s reordering copy, the launch's k of each row, and the row
        of each of the caller's modes (a device index tensor).  launch_state_tangent() gives the
        tangents in the same row order (views, no copy)."""
        if not self.full_state:
            raise ValueError("launch_states() needs a JacobianProblem made with full_state=True")
        stat = self.d_stat.cpu().numpy()[:, self.inv]
        _check_status(stat[0], stat[1], self.kmodes, on_failure)
        return self.d_out, self.kmodes[self.order], self.torch.as_tensor(self.inv, device=self.device)

    def launch_state_tangent(self, direction):
        """d y / d theta_d [K, nout, n] in the launch's row order (a view of the launch's output)."""
        if not self.full_state:
            raise ValueError("launch_state_tangent() needs a JacobianProblem made with full_state=True")
        return self.d_outd[direction]

    def state_tangent(self, direction):
        """d y / d theta_d [K, nout, n] along ODE_DIRECTIONS[direction] (output times moving
        with the parameters), a device tensor in the caller's k order; one direction at a time,
        so that a caller of large problems holds one reordered copy."""
        if not self.full_state:
            raise ValueError("state_tangent() needs a JacobianProblem made with full_state=True")
        return self.d_outd[direction][self.torch.as_tensor(self.inv, device=self.device)]

    def states(self, on_failure="raise"):
        """(y[K, nout, n], y_dot[6, K, nout, n]): state() and every state_tangent()."""
        y = self.state(on_failure)
        return y, self.torch.stack([self.state_tangent(d) for d in range(len(self.dirs))])

    def result(self, on_failure="raise"):
        """(P[K, nout], J[8, K, nout], status[K], nsteps[K]) in the caller's k order."""
        if self.full_state:
            raise ValueError("a full_state problem returns its states (states()), not P(k)")
        inv, bg, kmodes, idx = self.inv, self.bg, self.kmodes, self.idx
        y = self.d_out.cpu().numpy()[inv]
        yd = self.d_outd.cpu().numpy()[:, inv]
        stat = self.d_stat.cpu().numpy()[:, inv]
        status, nsteps = stat[0], stat[1]
        _check_status(status, nsteps, kmodes, on_failure)
        delta = y[..., idx]
        P = 2 * np.pi**2 * bg["A_s"] * (kmodes[:, None] / bg["k_p"]) ** (bg["n_s"] - 1) * kmodes[:, None] ** -3 \
            * delta**2
        J = np.zeros((len(THETA_NAMES), self.K, self.nout))
        for di, name in enumerate(self.dirs):
            J[THETA_NAMES.index(name)] = 2.0 * P * yd[di, ..., idx] / delta
        J[THETA_NAMES.index("n_s")] = P * np.log(kmodes[:, None] / bg["k_p"])
        J[THETA_NAMES.index("ln10As")] = P
        return P, J, status, nsteps


def power_spectrum_jacobian(theta, *, on_failure="raise", return_stats=False, **options):
    """P(k, a_out) of field ``idx`` (4: total matter) and its Jacobian with respect to theta.

    theta: dict with keys THETA_NAMES.  Options as JacobianProblem.  Returns
    (k, P[K, nout], J[8, K, nout]) with the rows of J in THETA_NAMES order (with
    ``return_stats`` also the per-mode status and step-attempt counts).
    """
    prob = JacobianProblem(theta, **options)
    prob.launch()
    P, J, status, nsteps = prob.result(on_failure)
    if return_stats:
        return prob.kmodes, P, J, status, nsteps
    return prob.kmodes, P, J


def power_spectrum_jacobian_sharded(theta, *, dist=None, device=None, on_failure="raise", **options):
    """power_spectrum_jacobian with one cosmology's modes spread over the ranks of ``dist`` (a
    torch.distributed process group, one process per GPU; ``replicas.init``): each rank solves its
    share (``replicas.shard``: longest-first, dealt round-robin) and every rank returns the whole
    (k, P [K, nout], J [8, K, nout]), gathered with ``replicas.gather_rows`` (``device``: where
    the collective's tensors live, the rank's GPU with NCCL, None with gloo).  One process (dist
    None): power_spectrum_jacobian.  Options as power_spectrum_jacobian."""
    from . import replicas
    rank, world = (dist.get_rank(), dist.get_world_size()) if dist is not None else (0, 1)
    k = options.pop("kmodes", None)
    if k is None:
        kp = theta_to_params(theta)
        method = options.pop("k_sampling_method", "log")
        if method == "camb":  # needs tau_maxvis of the background
            kp = evolve_background(param=kp, num_thermo=options.get("num_thermo", 256))
        k = k_sampling(kp, options.pop("kmin", 1e-4), options.pop("kmax", 1.0), options.pop("num_k", 64), method)
    k = np.ascontiguousarray(k, dtype=np.float64)
    idx = replicas.shard(k, rank, world)
    _, P, J = power_spectrum_jacobian(theta, kmodes=k[idx], on_failure=on_failure, **options)
    P_all = replicas.gather_rows(P, idx, k.shape[0], dist, device)
    J_all = replicas.gather_rows(np.moveaxis(J, 1, 0), idx, k.shape[0], dist, device)
    return k, P_all, np.moveaxis(J_all, 0, 1)


def power_spectrum_function(gradient="forward", **options):
    """A ``torch.autograd.Function`` mapping theta (float64[8], THETA_NAMES order) to
    P(k, a_out) (float64[K, nout]).

    gradient="forward": the forward pass runs ``discoeb_jvp`` (P and its full Jacobian in one
    launch) and keeps the Jacobian; the backward pass contracts it with the incoming gradient.
    gradient="adjoint": the forward pass records the solve (``discoeb_fwd_record``), the backward
    pass runs the discrete adjoint (``discoeb_bwd``): one reverse sweep per mode for any incoming
    gradient.  Either way ``torch.autograd`` sees the exact derivative of the discrete solution.
    ``options`` are those of JacobianProblem (k range, output scale factors, l_max, tolerances).
    """
    import torch

    if gradient == "adjoint":
        class PowerSpectrumAdjoint(torch.autograd.Function):
            @staticmethod
            def forward(ctx, theta):
                if theta.shape != (len(THETA_NAMES),):
                    raise ValueError(f"theta must have shape ({len(THETA_NAMES)},) in the order {THETA_NAMES}")
                th = dict(zip(THETA_NAMES, theta.detach().to("cpu", torch.float64).tolist()))
                prob = AdjointProblem(th, **options)
                prob.launch_forward()
                ctx.prob = prob
                return torch.from_numpy(prob.forward_power()[0][0]).to(theta.device)

            @staticmethod
            def backward(ctx, grad_P):
                prob = ctx.prob
                prob.launch_backward(grad_P)
                g = prob.gradient(grad_P.detach().to("cpu", torch.float64).numpy())[0]
                return torch.from_numpy(g).to(grad_P.device)

        return PowerSpectrumAdjoint
    if gradient != "forward":
        raise ValueError(f"gradient must be 'forward' or 'adjoint', not {gradient!r}")

    class PowerSpectrum(torch.autograd.Function):
        @staticmethod
        def forward(ctx, theta):
            if theta.shape != (len(THETA_NAMES),):
                raise ValueError(f"theta must have shape ({len(THETA_NAMES)},) in the order {THETA_NAMES}")
            th = dict(zip(THETA_NAMES, theta.detach().to("cpu", torch.float64).tolist()))
            _, P, J = power_spectrum_jacobian(th, **options)
            ctx.save_for_backward(torch.from_numpy(J).to(theta.device))
            return torch.from_numpy(P).to(theta.device)

        @staticmethod
        def backward(ctx, grad_P):
            (J,) = ctx.saved_tensors
            return torch.einsum("dkn,kn->d", J, grad_P.to(J.dtype))

    return PowerSpectrum


def _prologue_task(args):
    return cosmology_prologue(*args)


class JacobianBatch:
    """P(k) and dP/dtheta of many cosmologies in ONE discoeb_jvp launch (what ``jax.vmap`` of
    ``jax.jacfwd`` over cosmologies computes in the reference).

    ``thetas``: list of C theta dicts; ``kmodes``: ``[K]`` shared by all cosmologies.  The host
    prologue (cosmology_prologue) runs per cosmology: in the calling process when
    ``host_processes`` is 1 (each with ``host_threads`` threads), else in a persistent pool of
    spawned processes (0: up to the host's cores).  ``host_backend="device"`` computes all the
    backgrounds and their tangents in one GPU launch (discoeb_background_batch) first.
    ``launch`` / ``result`` as JacobianProblem; result returns
    ``(P [C, K, nout], J [C, 8, K, nout], status [C, K], nsteps [C, K])``.
    """

    def __init__(self, thetas, *, kmodes, aexp_out=(1.0,), lmaxg=12, lmaxgp=12, lmaxr=17, lmaxnu=17, nqmax=5,
                 rtol=1e-5, atol=1e-8, pcoeff=0.25, icoeff=0.80, dcoeff=0.0, factormax=20.0, factormin=0.3,
                 max_steps=100000, idx=4, num_thermo=256, de_guard_eps=1e-9, device=None, host_backend="native",
                 host_threads=0, host_processes=1):
        import os

        import torch
        if device is None:
            if not torch.cuda.is_available():
                raise RuntimeError("discoeb_b200 needs a CUDA device (there is no CPU path)")
            device = torch.device("cuda", torch.cuda.current_device())
        self.torch, self.device, self.idx, self.lib = torch, device, idx, _abi.lib()
        L = dict(lmaxg=lmaxg, lmaxgp=lmaxgp, lmaxr=lmaxr, lmaxnu=lmaxnu, nqmax=nqmax)
        kmodes = np.ascontiguousarray(kmodes, dtype=np.float64)
        aexp_out = np.atleast_1d(np.asarray(aexp_out, dtype=np.float64))
        nproc = (os.cpu_count() or 1) if not host_processes else host_processes
        nproc = min(nproc, len(thetas))
        threads = host_threads if nproc <= 1 else max(host_threads, 1)
        bufs = [None] * len(thetas)
        if host_backend == "device":
            from .background import native_backgrounds_device
            out, out_dot = native_backgrounds_device([theta_to_params(t) for t in thetas], num_thermo,
                                                     [param_dots(t, ODE_DIRECTIONS) for t in thetas], device=device)
            out, out_dot = out.cpu().numpy(), out_dot.cpu().numpy()
            bufs = [(out[c], out_dot[c]) for c in range(len(thetas))]
        args = [(dict(t), aexp_out, kmodes, L, num_thermo, host_backend, threads, b) for t, b in zip(thetas, bufs)]
        pro = [_prologue_task(a) for a in args] if nproc <= 1 else _pool(nproc).map(_prologue_task, args)
        C, K, nout, n = len(pro), kmodes.shape[0], aexp_out.shape[0], nvar_of(**L)
        nd = len(ODE_DIRECTIONS)
        self.C, self.K, self.nout, self.nd, self.kmodes = C, K, nout, nd, kmodes
        self.bgs = [p["bg"] for p in pro]
        flat_k = np.tile(kmodes, C)
        cidx = np.repeat(np.arange(C, dtype=np.int32), K)
        order = np.argsort(-flat_k, kind="stable")  # longest modes first across all cosmologies
        self.inv = np.empty_like(order)
        self.inv[order] = np.arange(C * K)
        self.dcs = [DeviceCosmo(p["bg"], de_guard_eps=de_guard_eps, device=device, **L) for p in pro]
        raw = b"".join(bytes(ctypes.string_at(ctypes.addressof(d.host), ctypes.sizeof(d.host))) for d in self.dcs)
        t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(device)  # noqa: E731
        self.d_cosmos = torch.frombuffer(bytearray(raw), dtype=torch.uint8).to(device)
        self._keep, tstructs = [], []
        for p in pro:
            for d in p["tans"]:
                ts = _abi.DiscoebTangent()
                for f, v in d["scalars"].items():
                    setattr(ts, f, v)
                for short, (yy, SS) in d["tables"].items():
                    ty, tS = t(yy), t(SS)
                    self._keep += [ty, tS]
                    setattr(ts, short + "_y", ty.data_ptr())
                    setattr(ts, short + "_S", tS.data_ptr())
                tstructs.append(ts)
        arr = (_abi.DiscoebTangent * len(tstructs))(*tstructs)
        self.d_tan = torch.frombuffer(bytearray(bytes(arr)), dtype=torch.uint8).to(device)
        self.d_k, self.d_mc = t(flat_k[order]), t(cidx[order])
        self.d_ts = t(np.concatenate([p["tau_start"] for p in pro])[order])
        self.d_y0 = t(np.concatenate([p["y0"] for p in pro])[order])
        y0d = np.stack([np.concatenate([p["tans"][di]["y0"] for p in pro])[order] for di in range(nd)])
        self.d_y0d = t(y0d)
        self.d_sw = t(np.concatenate([p["sw"] for p in pro])[order])
        self.d_tout = t(np.stack([p["tau_out"] for p in pro]))
        self.d_toutd = t(np.stack([np.stack([d["tau_out"] for d in p["tans"]]) for p in pro]))
        f64 = dict(dtype=torch.float64, device=device)
        self.d_out = torch.empty((C * K, nout, 20), **f64)
        self.d_outd = torch.empty((nd, C * K, nout, 20), **f64)
        self.d_stat = torch.empty((2, C * K), dtype=torch.int32, device=device)
        self.ctrl = _abi.DiscoebControl(rtol, atol, pcoeff, icoeff, dcoeff, factormax, factormin, int(max_steps),
                                        _abi.METHOD_RODAS5_STRUCTURED, 0, 0)

    def launch(self):
        stream = self.torch.cuda.current_stream(self.device).cuda_stream
        rc = self.lib.discoeb_jvp(self.d_cosmos.data_ptr(), ctypes.byref(self.dcs[0].host), self.C,
                                  self.d_mc.data_ptr(), self.d_tan.data_ptr(), self.nd, ctypes.byref(self.ctrl),
                                  self.C * self.K, self.d_k.data_ptr(), self.d_ts.data_ptr(), self.d_y0.data_ptr(),
                                  self.d_y0d.data_ptr(), self.d_sw.data_ptr(), self.nout, self.d_tout.data_ptr(),
                                  self.d_toutd.data_ptr(), self.d_out.data_ptr(), self.d_outd.data_ptr(),
                                  self.d_stat[0].data_ptr(), self.d_stat[1].data_ptr(), stream)
        if rc != 0:
            raise RuntimeError(f"discoeb_jvp failed with code {rc}")

    def result(self, on_failure="raise"):
        C, K, nout, inv = self.C, self.K, self.nout, self.inv
        y = self.d_out.cpu().numpy()[inv].reshape(C, K, nout, 20)
        yd = self.d_outd.cpu().numpy()[:, inv].reshape(self.nd, C, K, nout, 20)
        stat = self.d_stat.cpu().numpy()[:, inv]
        _check_status(stat[0], stat[1], np.tile(self.kmodes, C), on_failure)
        P = np.empty((C, K, nout))
        J = np.zeros((C, len(THETA_NAMES), K, nout))
        k = self.kmodes[:, None]
        for c, bg in enumerate(self.bgs):
            delta = y[c, ..., self.idx]
            P[c] = 2 * np.pi**2 * bg["A_s"] * (k / bg["k_p"]) ** (bg["n_s"] - 1) * k**-3 * delta**2
            for di, name in enumerate(ODE_DIRECTIONS):
                J[c, THETA_NAMES.index(name)] = 2.0 * P[c] * yd[di, c, ..., self.idx] / delta
            J[c, THETA_NAMES.index("n_s")] = P[c] * np.log(k / bg["k_p"])
            J[c, THETA_NAMES.index("ln10As")] = P[c]
        return P, J, stat[0].reshape(C, K), stat[1].reshape(C, K)


class _ReverseMode:
    """Reverse-mode gradients (discrete adjoint) for the modes of a JacobianProblem or a
    JacobianBatch: ``launch_forward`` solves and records the accepted steps (discoeb_fwd_record),
    ``launch_backward(grad_P)`` runs the reverse sweep from the cotangent of P(k) (discoeb_bwd)
    and contracts the cotangents with the parameter tangents the prologue computed
    (discoeb_bwd_contract); ``gradient`` returns dL/dtheta [C, 8] for L = sum grad_P * P.  One
    reverse sweep per mode whatever the number of parameters (the reference's jax.grad through
    diffeqsolve with DirectAdjoint, perturbations.py:904-925).

    ``step_capacity``: accepted steps a mode's record holds (a mode that needs more stops with
    DISCOEB_RECORD_FULL); ``checkpoint_every``: the record keeps every n-th step's start state
    (the reverse sweep recomputes the steps in between: memory against a second forward pass).
    """

    def _reverse_init(self, step_capacity, checkpoint_every):
        torch, dev = self.torch, self.device
        M = self._C * self.K
        rec = int(self.lib.discoeb_step_record_doubles(self.n, int(step_capacity), int(checkpoint_every)))
        if rec <= 0:
            raise ValueError("invalid step_capacity / checkpoint_every")
        self.step_capacity, self.checkpoint_every = int(step_capacity), int(checkpoint_every)
        f64 = dict(dtype=torch.float64, device=dev)
        self.d_rec = torch.empty((M, rec), **f64)
        self.d_nacc = torch.empty(M, dtype=torch.int32, device=dev)
        self.d_fstat = torch.empty((2, M), dtype=torch.int32, device=dev)
        self.d_bstat = torch.empty(M, dtype=torch.int32, device=dev)
        self.d_ybar = torch.zeros((M, self.nout, 20), **f64)
        self.d_y0bar = torch.empty((M, self.n), **f64)
        self.d_toutbar = torch.empty((M, self.nout), **f64)
        self.d_pbar = torch.empty((M, 8), **f64)
        self.tstride = max(bg[key].n for bg in self._bgs for key, _ in _TABLES)
        self.d_tbar = torch.zeros((self._C, 8, self.tstride), **f64)
        ws = int(self.lib.discoeb_bwd_workspace_bytes(ctypes.byref(self._host), M, self.checkpoint_every))
        self.d_ws = torch.empty(max(ws // 8, 1), **f64)
        self.d_thbar = torch.empty((self._C, len(ODE_DIRECTIONS)), **f64)
        # primordial amplitude of every mode in launch order: P = amp * delta^2
        k = np.tile(self.kmodes, self._C)
        amp = np.concatenate([2 * np.pi**2 * bg["A_s"] * (self.kmodes / bg["k_p"]) ** (bg["n_s"] - 1)
                              * self.kmodes**-3 for bg in self._bgs])
        order = np.empty_like(self.inv)
        order[self.inv] = np.arange(k.size)
        self.d_amp = torch.from_numpy(np.ascontiguousarray(amp[order])).to(dev)

    def launch_forward(self):
        stream = self.torch.cuda.current_stream(self.device).cuda_stream
        M = self._C * self.K
        rc = self.lib.discoeb_fwd_record(self._cosmos_ptr, ctypes.byref(self._host), self._C, ctypes.byref(self.ctrl),
                                         M, self._mc_ptr, self.d_k.data_ptr(), self.d_ts.data_ptr(),
                                         self.d_y0.data_ptr(), self.d_sw.data_ptr(), self.nout,
                                         self.d_tout.data_ptr(), self.d_out.data_ptr(), self.d_fstat[0].data_ptr(),
                                         self.d_fstat[1].data_ptr(), self.step_capacity, self.checkpoint_every,
                                         self.d_rec.data_ptr(), self.d_nacc.data_ptr(), stream)
        if rc != 0:
            raise RuntimeError(f"discoeb_fwd_record failed with code {rc}")

    def forward_power(self, on_failure="raise"):
        """(P [C, K, nout], status [C, K], nsteps [C, K]) of the recorded forward, caller order."""
        C, K, nout, inv = self._C, self.K, self.nout, self.inv
        y = self.d_out.cpu().numpy()[inv].reshape(C, K, nout, 20)
        stat = self.d_fstat.cpu().numpy()[:, inv]
        _check_status(stat[0], stat[1], np.tile(self.kmodes, C), on_failure)
        amp = np.stack([2 * np.pi**2 * bg["A_s"] * (self.kmodes / bg["k_p"]) ** (bg["n_s"] - 1) * self.kmodes**-3
                        for bg in self._bgs])
        P = amp[:, :, None] * y[..., self.idx] ** 2
        return P, stat[0].reshape(C, K), stat[1].reshape(C, K)

    def launch_backward(self, grad_P):
        """Reverse sweep from grad_P [C, K, nout] (or [K, nout] for one cosmology; numpy or a
        device tensor, the caller's k order)."""
        torch = self.torch
        g = torch.as_tensor(grad_P, dtype=torch.float64).to(self.device).reshape(self._C * self.K, self.nout)
        g = g[torch.as_tensor(np.argsort(self.inv), device=self.device)]  # launch order
        delta = self.d_out[:, :, self.idx]
        self.d_ybar.zero_()
        self.d_ybar[:, :, self.idx] = 2.0 * g * self.d_amp[:, None] * delta  # dL/d delta of L = sum g * amp delta^2
        self.d_tbar.zero_()
        stream = torch.cuda.current_stream(self.device).cuda_stream
        M = self._C * self.K
        rc = self.lib.discoeb_bwd(self._cosmos_ptr, ctypes.byref(self._host), self._C, self._mc_ptr, M,
                                  self.d_k.data_ptr(), self.d_ts.data_ptr(), self.d_sw.data_ptr(), self.nout,
                                  self.d_tout.data_ptr(), self.step_capacity, self.checkpoint_every,
                                  self.d_rec.data_ptr(), self.d_nacc.data_ptr(), self.d_fstat[0].data_ptr(),
                                  self.d_ybar.data_ptr(), self.d_y0bar.data_ptr(), self.d_toutbar.data_ptr(),
                                  self.d_pbar.data_ptr(), self.d_tbar.data_ptr(), self.tstride, 0,
                                  self.d_ws.data_ptr(), self.d_ws.numel() * 8, self.d_bstat.data_ptr(), stream)
        if rc != 0:
            raise RuntimeError(f"discoeb_bwd failed with code {rc}")
        rc = self.lib.discoeb_bwd_contract(self._cosmos_ptr, self._C, self._mc_ptr, M, self.n, self.nout,
                                           self.d_tan.data_ptr(), len(ODE_DIRECTIONS), self.d_y0d.data_ptr(),
                                           self.d_toutd.data_ptr(), self.d_y0bar.data_ptr(), self.d_toutbar.data_ptr(),
                                           self.d_pbar.data_ptr(), self.d_tbar.data_ptr(), self.tstride, 0,
                                           self.d_thbar.data_ptr(), stream)
        if rc != 0:
            raise RuntimeError(f"discoeb_bwd_contract failed with code {rc}")

    def launch_jacobian_rows(self, out_index=-1):
        """Reverse sweeps whose cotangent is each mode's own P at output out_index: every mode's
        row of dP(k, z)/dtheta in one launch (the per-mode table cotangents are kept apart)."""
        torch = self.torch
        M = self._C * self.K
        if getattr(self, "d_tbar_mode", None) is None:
            f64 = dict(dtype=torch.float64, device=self.device)
            self.d_tbar_mode = torch.zeros((M, 8, self.tstride), **f64)
            self.d_thbar_mode = torch.empty((M, len(ODE_DIRECTIONS)), **f64)
        j = out_index % self.nout
        self.d_ybar.zero_()
        self.d_ybar[:, j, self.idx] = 2.0 * self.d_amp * self.d_out[:, j, self.idx]
        self.d_tbar_mode.zero_()
        stream = torch.cuda.current_stream(self.device).cuda_stream
        rc = self.lib.discoeb_bwd(self._cosmos_ptr, ctypes.byref(self._host), self._C, self._mc_ptr, M,
                                  self.d_k.data_ptr(), self.d_ts.data_ptr(), self.d_sw.data_ptr(), self.nout,
                                  self.d_tout.data_ptr(), self.step_capacity, self.checkpoint_every,
                                  self.d_rec.data_ptr(), self.d_nacc.data_ptr(), self.d_fstat[0].data_ptr(),
                                  self.d_ybar.data_ptr(), self.d_y0bar.data_ptr(), self.d_toutbar.data_ptr(),
                                  self.d_pbar.data_ptr(), self.d_tbar_mode.data_ptr(), self.tstride, 1,
                                  self.d_ws.data_ptr(), self.d_ws.numel() * 8, self.d_bstat.data_ptr(), stream)
        if rc != 0:
            raise RuntimeError(f"discoeb_bwd failed with code {rc}")
        rc = self.lib.discoeb_bwd_contract(self._cosmos_ptr, self._C, self._mc_ptr, M, self.n, self.nout,
                                           self.d_tan.data_ptr(), len(ODE_DIRECTIONS), self.d_y0d.data_ptr(),
                                           self.d_toutd.data_ptr(), self.d_y0bar.data_ptr(), self.d_toutbar.data_ptr(),
                                           self.d_pbar.data_ptr(), self.d_tbar_mode.data_ptr(), self.tstride, 1,
                                           self.d_thbar_mode.data_ptr(), stream)
        if rc != 0:
            raise RuntimeError(f"discoeb_bwd_contract failed with code {rc}")
        self._rows_out = j

    def jacobian_rows(self, on_failure="raise"):
        """J [C, 8, K]: dP(k, z)/dtheta at the output of the last launch_jacobian_rows (THETA_NAMES
        order, caller's k order; n_s and ln10As in closed form)."""
        st = self.d_bstat.cpu().numpy()[self.inv]
        _check_status(st, np.zeros_like(st), np.tile(self.kmodes, self._C), on_failure)
        rows = self.d_thbar_mode.cpu().numpy()[self.inv].reshape(self._C, self.K, len(ODE_DIRECTIONS))
        P = self.forward_power(on_failure="ignore")[0][:, :, self._rows_out]
        J = np.zeros((self._C, len(THETA_NAMES), self.K))
        for di, name in enumerate(ODE_DIRECTIONS):
            J[:, THETA_NAMES.index(name)] = rows[:, :, di]
        for c, bg in enumerate(self._bgs):
            J[c, THETA_NAMES.index("n_s")] = P[c] * np.log(self.kmodes / bg["k_p"])
            J[c, THETA_NAMES.index("ln10As")] = P[c]
        return J

    def gradient(self, grad_P, on_failure="raise"):
        """dL/dtheta [C, 8] (THETA_NAMES order) of L = sum grad_P * P after launch_backward(grad_P):
        the six solver directions from the reverse sweep, n_s and ln10As in closed form."""
        st = self.d_bstat.cpu().numpy()[self.inv]
        _check_status(st, np.zeros_like(st), np.tile(self.kmodes, self._C), on_failure)
        th = self.d_thbar.cpu().numpy()
        P = self.forward_power(on_failure="ignore")[0]
        g = np.asarray(grad_P, dtype=np.float64).reshape(P.shape)
        out = np.zeros((self._C, len(THETA_NAMES)))
        for di, name in enumerate(ODE_DIRECTIONS):
            out[:, THETA_NAMES.index(name)] = th[:, di]
        for c, bg in enumerate(self._bgs):
            out[c, THETA_NAMES.index("n_s")] = np.sum(g[c] * P[c] * np.log(self.kmodes / bg["k_p"])[:, None])
            out[c, THETA_NAMES.index("ln10As")] = np.sum(g[c] * P[c])
        return out


class AdjointProblem(JacobianProblem, _ReverseMode):
    """P(k) of one cosmology with reverse-mode gradients of scalar losses (the discrete adjoint):
    the prologue and options of JacobianProblem, plus ``step_capacity`` and ``checkpoint_every``
    (see _ReverseMode)."""

    def __init__(self, theta, *, step_capacity=8192, checkpoint_every=16, **options):
        JacobianProblem.__init__(self, theta, **options)
        self._C, self._bgs, self._host, self._mc_ptr = 1, [self.bg], self.dc.host, None
        self._cosmos_ptr = self.dc.struct.data_ptr()
        self._reverse_init(step_capacity, checkpoint_every)


class AdjointBatch(JacobianBatch, _ReverseMode):
    """AdjointProblem for many cosmologies in one forward and one reverse launch (the options of
    JacobianBatch, plus ``step_capacity`` and ``checkpoint_every``)."""

    def __init__(self, thetas, *, step_capacity=8192, checkpoint_every=16, **options):
        JacobianBatch.__init__(self, thetas, **options)
        self.n = nvar_of(**{k: options.get(k, d) for k, d in (("lmaxg", 12), ("lmaxgp", 12), ("lmaxr", 17),
                                                              ("lmaxnu", 17), ("nqmax", 5))})
        self._C, self._bgs, self._host = self.C, self.bgs, self.dcs[0].host
        self._mc_ptr, self._cosmos_ptr = self.d_mc.data_ptr(), self.d_cosmos.data_ptr()
        self._reverse_init(step_capacity, checkpoint_every)


def power_spectrum_gradient(theta, grad_P, **options):
    """(k, P [K, nout], dL/dtheta [8]) for the scalar loss L = sum grad_P * P(k, a_out) by one
    forward and one reverse sweep (AdjointProblem; options as JacobianProblem)."""
    prob = AdjointProblem(theta, **options)
    prob.launch_forward()
    P = prob.forward_power()[0][0]
    prob.launch_backward(np.asarray(grad_P, dtype=np.float64).reshape(P.shape))
    return prob.kmodes, P, prob.gradient(grad_P)[0]

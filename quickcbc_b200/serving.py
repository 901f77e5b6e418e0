"""Continuous-batching PT-MCMC service (include/qcbc_serve.h) from Python, and
a driver that feeds it a Poisson stream of analyses in real time.

The time-to-posterior of a run is the time from its submission (arrival) to
the end of its last step, on the service's clock.
"""
from __future__ import annotations

import ctypes as C
import time

import numpy as np

from . import _lib
from ._lib import MIXED, QcbcError, check

_PD = C.POINTER(C.c_double)
_PI = C.POINTER(C.c_int)

RUN_QUEUED, RUN_LIVE, RUN_DONE, RUN_FAILED, RUN_CANCELLED = range(5)


class RunSpec(C.Structure):
    _fields_ = [("nifo", C.c_int), ("labels", _PI), ("Tobs", C.c_double), ("GMST", C.c_double), ("N", C.c_int),
                ("D", _PD), ("SN", _PD), ("sn_stride", C.c_int), ("fmin", C.c_double), ("fmax", C.c_double),
                ("start", _PD), ("scales", _PD), ("prior_min", _PD), ("prior_max", _PD), ("n_temps", C.c_int),
                ("n_chains", C.c_int), ("n_steps", C.c_int), ("burn_in", C.c_int), ("thin", C.c_int),
                ("ladder", C.c_double), ("seed", C.c_ulonglong), ("likelihood", C.c_int), ("proposal", C.c_int)]

LNL_FULL, LNL_HET = 0, 1
PROPOSE_GAUSS, PROPOSE_REFERENCE = 0, 1


class RunInfo(C.Structure):
    _fields_ = [("state", C.c_int), ("steps_done", C.c_int), ("t_arrival", C.c_double), ("t_admit", C.c_double),
                ("t_done", C.c_double), ("accept_cold", C.c_double), ("swap_rate", C.c_double),
                ("device_bytes", C.c_longlong), ("lnl_evals", C.c_longlong), ("n_samples", C.c_int)]


def _bind():
    L = _lib.lib()
    if getattr(L, "_serve_bound", False):
        return L
    vp, i, ll, d = C.c_void_p, C.c_int, C.c_longlong, C.c_double
    L.qcbc_server_create.restype = vp
    L.qcbc_server_create.argtypes = [ll, i, i, i]
    L.qcbc_server_destroy.argtypes = [vp]
    L.qcbc_server_clock.restype = d
    L.qcbc_server_clock.argtypes = [vp]
    L.qcbc_server_submit.restype = ll
    L.qcbc_server_submit.argtypes = [vp, C.POINTER(RunSpec)]
    L.qcbc_server_cancel.argtypes = [vp, ll]
    L.qcbc_server_step.argtypes = [vp, _PI, _PI, _PI]
    L.qcbc_server_run_info.argtypes = [vp, ll, C.POINTER(RunInfo)]
    L.qcbc_server_run_samples.argtypes = [vp, ll, _PD, i, _PI]
    L.qcbc_server_stats.argtypes = [vp, C.POINTER(ll), C.POINTER(ll), C.POINTER(ll)]
    L.qcbc_server_set_tiling.argtypes = [vp, i, i]
    L.qcbc_server_timing.argtypes = [vp, C.POINTER(d), C.POINTER(d), C.POINTER(d)]
    L.qcbc_server_set_device_steps.argtypes = [vp, i]
    L._serve_bound = True
    return L


class Server:
    """device_steps > 0 keeps the chains on the device and advances every live run by up to that
    many steps per step() call (qcbc_server_set_device_steps); 0 steps the chains on the host."""

    def __init__(self, hbm_budget_bytes=150 * 10**9, max_live=256, max_bins=1 << 17, precision=MIXED,
                 device_steps=0):
        L = _bind()
        check(L.qcbc_init(0))
        self._h = L.qcbc_server_create(int(hbm_budget_bytes), int(max_live), int(max_bins), int(precision))
        if not self._h:
            raise QcbcError(-1, _lib.last_error())
        if device_steps:
            self.set_device_steps(device_steps)

    def set_device_steps(self, steps):
        check(_bind().qcbc_server_set_device_steps(self._h, int(steps)))

    def close(self):
        if getattr(self, "_h", None):
            _bind().qcbc_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def clock(self):
        return _bind().qcbc_server_clock(self._h)

    def set_tiling(self, tile_bins, threads=0):
        check(_bind().qcbc_server_set_tiling(self._h, int(tile_bins), int(threads)))

    def submit(self, ev, start=None, n_temps=16, n_chains=8, n_steps=20000, burn_in=None, thin=10, ladder=1.15,
               seed=0, scales=None, likelihood="full", proposal="gauss"):
        """Submit a synthetic event (synth.Event); returns the run id.  likelihood "het" builds the
        heterodyne grid and tables about `start` at admission and samples the heterodyned lnL.
        proposal "reference" (device-resident stepping only) uses the reference's mixture of
        Fisher eigen-jumps, differential evolution and jiggles."""
        if likelihood not in ("full", "het"):
            raise ValueError("likelihood is 'full' or 'het'")
        if proposal not in ("gauss", "reference"):
            raise ValueError("proposal is 'gauss' or 'reference'")
        keep = dict(labels=np.ascontiguousarray(ev.labels, dtype=np.int32), D=np.ascontiguousarray(ev.D),
                    SN=np.ascontiguousarray(ev.SN),
                    start=np.ascontiguousarray(ev.inj if start is None else start, dtype=np.float64))
        if scales is not None:
            keep["scales"] = np.ascontiguousarray(scales, dtype=np.float64)
        spec = RunSpec(nifo=len(keep["labels"]), labels=keep["labels"].ctypes.data_as(_PI), Tobs=ev.Tobs,
                       GMST=ev.GMST, N=ev.N, D=keep["D"].ctypes.data_as(_PD), SN=keep["SN"].ctypes.data_as(_PD),
                       sn_stride=keep["SN"].shape[1], fmin=ev.fmin, fmax=1024.0,
                       start=keep["start"].ctypes.data_as(_PD),
                       scales=keep["scales"].ctypes.data_as(_PD) if scales is not None else None,
                       prior_min=None, prior_max=None, n_temps=n_temps, n_chains=n_chains, n_steps=n_steps,
                       burn_in=n_steps // 4 if burn_in is None else burn_in, thin=thin, ladder=ladder,
                       seed=int(seed), likelihood=LNL_HET if likelihood == "het" else LNL_FULL,
                       proposal=PROPOSE_REFERENCE if proposal == "reference" else PROPOSE_GAUSS)
        rid = _bind().qcbc_server_submit(self._h, C.byref(spec))
        if rid < 0:
            raise QcbcError(int(rid), _lib.last_error())
        return int(rid)

    def step(self):
        nl, nq, nd = C.c_int(), C.c_int(), C.c_int()
        check(_bind().qcbc_server_step(self._h, C.byref(nl), C.byref(nq), C.byref(nd)))
        return nl.value, nq.value, nd.value

    def info(self, rid):
        o = RunInfo()
        check(_bind().qcbc_server_run_info(self._h, int(rid), C.byref(o)))
        return {k: getattr(o, k) for k, _ in RunInfo._fields_}

    def samples(self, rid):
        n = self.info(rid)["n_samples"]
        out = np.zeros((max(n, 1), 12))
        got = C.c_int()
        check(_bind().qcbc_server_run_samples(self._h, int(rid), out.ctypes.data_as(_PD), n, C.byref(got)))
        return out[:got.value]

    def cancel(self, rid):
        check(_bind().qcbc_server_cancel(self._h, int(rid)))

    def stats(self):
        e, l, b = C.c_longlong(), C.c_longlong(), C.c_longlong()
        check(_bind().qcbc_server_stats(self._h, C.byref(e), C.byref(l), C.byref(b)))
        return dict(lnl_evals=e.value, launches=l.value, device_bytes_live=b.value)

    def timing(self):
        a, b, c = C.c_double(), C.c_double(), C.c_double()
        check(_bind().qcbc_server_timing(self._h, C.byref(a), C.byref(b), C.byref(c)))
        return dict(propose_s=a.value, lnl_s=b.value, update_s=c.value)

    def run_until_idle(self, max_steps=10**9):
        for _ in range(max_steps):
            nl, nq, _ = self.step()
            if nl == 0 and nq == 0:
                return


def serve_stream(server, events, rate_hz, seed=0, sampler=None, log=None):
    """Submit `events` as a Poisson stream (mean rate_hz arrivals per second, in
    real time; rate_hz=None submits every event at once, which saturates the
    service) and step the service until every run has finished.

    Returns per-run times-to-posterior, their p50/p99, and the aggregate lnL
    evaluations per second over the whole session."""
    sampler = dict(sampler or {})
    rng = np.random.default_rng(seed)
    if rate_hz is None:
        arrivals = np.zeros(len(events))
    else:
        arrivals = np.cumsum(rng.exponential(1.0 / rate_hz, size=len(events)))
        arrivals -= arrivals[0]
    t0 = server.clock()
    ids, nxt = [], 0
    e0 = server.stats()["lnl_evals"]
    while True:
        now = server.clock() - t0
        while nxt < len(events) and arrivals[nxt] <= now:
            ids.append(server.submit(events[nxt], seed=seed * 100003 + nxt, **sampler))
            nxt += 1
        nl, nq, _ = server.step()
        if nl == 0 and nq == 0:
            if nxt >= len(events):
                break
            time.sleep(max(0.0, min(0.05, arrivals[nxt] - (server.clock() - t0))))
    wall = server.clock() - t0
    infos = [server.info(r) for r in ids]
    ttp = np.array([i["t_done"] - i["t_arrival"] for i in infos if i["state"] == RUN_DONE])
    evals = server.stats()["lnl_evals"] - e0
    phases = server.timing()
    return dict(phase_s=phases, n_runs=len(ids), n_done=int(len(ttp)), ttp_s=ttp.tolist(),
                p50_s=float(np.percentile(ttp, 50)) if len(ttp) else None,
                p99_s=float(np.percentile(ttp, 99)) if len(ttp) else None,
                wall_s=wall, lnl_evals=int(evals), evals_per_s=evals / wall if wall > 0 else None,
                accept_cold=float(np.mean([i["accept_cold"] for i in infos])) if infos else None)

"""Benchmark of the QuickCBC likelihood hot path on B200.

Workload (one "step"): the batched full likelihood of the 3-detector network
(H1/L1/V1), Tobs = 16 s, fs = 4096 Hz (N = 65536, band 20-1024 Hz, 16064 bins
per detector), 2048 parameter sets per launch (64 chains x 32 proposals) drawn
around an injected IMRPhenomD signal; synthetic coloured Gaussian noise.

value  = lnL evaluations per second of the mixed-precision batched kernel
         sequence (setup + fused waveform/projection/inner product + finalise),
         inputs resident in HBM, CUDA-event timed per step with an L2 flush
         (512 MiB write) between steps outside the timed span.
e2e    = the same metric through the public C ABI call qcbc_lnl_full with host
         parameter arrays: the 2048 x 11 parameter doubles cross to the device
         and the 2048 lnL doubles back inside the timed region (the kernels
         read and write the pinned staging buffers directly).

python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
Under torchrun each rank runs its own replica (parameter sets shard with no
exchange; scaling is weak) and rank 0 prints the max-over-ranks time.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "lnL evals/sec mixed vs FP64 on 1 B200 (|dlnL|<=1e-3); p50/p99 time-to-posterior"
CONFIG = dict(workload="batched full likelihood, 3 det H1/L1/V1, Tobs 16 s, fs 4096 Hz, N 65536, "
                       "band 20-1024 Hz, 2048 parameter sets per launch (64 chains x 32 proposals)",
              B=2048, nifo=3, Tobs=16.0, fs=4096.0, fmin=20.0, l2="flushed between steps (512 MiB write)")


def env_rank():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("LOCAL_RANK", "0"))


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index, self.rows, self.proc = index, [], None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in self.rows for k in range(4) if len(r) > 5 + k and r[5 + k] == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def ncu_capture(name):
    """Per-launch figures of one kernel from a committed ncu capture: profiles/<name>.csv holds the
    `ncu -i <rep> --page raw --csv` rows of that capture (kernel name, grid, block and the DRAM
    byte counters; the command is in its first line).  Returns the mean per launch, or None."""
    import csv
    p = os.path.join(ROOT, "profiles", name + ".csv")
    if not os.path.exists(p):
        return None
    with open(p) as f:
        lines = [ln for ln in f if not ln.startswith("#")]
    rows = list(csv.DictReader(lines))
    units = rows[0] if rows and not rows[0].get("ID", "0").strip().isdigit() else None
    rows = [r for r in rows if r.get("ID", "").strip().isdigit()]
    if not rows:
        return None

    def num(r, k):
        v = float(r[k].replace(",", ""))
        u = (units or {}).get(k, "").strip().lower()
        return v * {"kbyte": 1e3, "mbyte": 1e6, "gbyte": 1e9, "us": 1e-6, "usecond": 1e-6, "ms": 1e-3,
                    "msecond": 1e-3, "ns": 1e-9, "nsecond": 1e-9}.get(u, 1.0)
    rd = [num(r, "dram__bytes_read.sum") for r in rows]
    wr = [num(r, "dram__bytes_write.sum") for r in rows]
    out = {"kernel": rows[0]["Kernel Name"], "grid": rows[0].get("Grid Size"), "block": rows[0].get("Block Size"),
           "launches": len(rows), "dram_bytes": float(np.mean(np.add(rd, wr))), "file": f"profiles/{name}.csv"}
    if "gpu__time_duration.sum" in rows[0]:
        out["duration_s"] = float(np.mean([num(r, "gpu__time_duration.sum") for r in rows]))
    return out


def capture_traffic(name, kernel, grid, block, kernel_ms):
    """roofline.traffic from the committed capture of this kernel, used only when the capture is of
    the same kernel at the same launch shape (grid, block) as the timed launches; else null."""
    cap = ncu_capture(name)
    if cap is None:
        return None, {"traffic_source": f"no capture profiles/{name}.csv"}
    same = kernel in cap["kernel"] and (grid is None or str(cap["grid"]).replace(" ", "") == grid) and \
        (block is None or str(cap["block"]).replace(" ", "") == block)
    info = {"traffic_source": cap["file"], "traffic_capture_launches": cap["launches"],
            "traffic_capture_matches_launch": bool(same)}
    if "duration_s" in cap:
        info["capture_ms_cold"] = cap["duration_s"] * 1e3
    return (cap["dram_bytes"] if same else None), info


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def fp32_peak_tflops(sm_mhz):
    """FP32 FMA peak of a B200 at the given SM clock: 148 SMs x 128 FP32 lanes x 2 flops per FMA.
    MEASURED_PEAKS.json carries only HBM and bf16 figures, so this one is derived from the spec at
    the clock sampled during the run."""
    return 148 * 128 * 2 * (sm_mhz or 1965.0) * 1e6 / 1e12


# Algorithmic FP32 work of one full-likelihood evaluation per in-band bin (the per-unit figures of
# the path): one IMRPhenomD point (~60 flops: the piecewise amplitude and phase polynomials) plus,
# per detector, the projection and the two multiply-accumulates of <d|h> and <h|h> (~14 flops).
WF_FLOPS_PER_BIN = 60
PROJ_FLOPS_PER_DET_BIN = 14


def make_workload(seed_offset=0):
    import quickcbc_b200 as q
    from quickcbc_b200 import synth

    def tmpl(info, p):
        return q.fulltemplates(info["labels"], info["GMST"], info["freq"], p, info["N"])

    ev = synth.config_event(2, tmpl)
    rng = np.random.default_rng(2000 + 500000 + seed_offset)
    P = synth.draw_params(rng, CONFIG["B"], ev.inj)
    return ev, P


def cpu_baseline_reference(ev, P, budget_s=12.0, impl_note=""):
    """The reference's log_likelihood_full (oracle/_ref, compiled from the
    reference sources) under OpenMP on all host cores, on a bounded sample."""
    try:
        from oracle import ref
        if not ref.available():
            raise FileNotFoundError
        net = ref.RefNet(ev.labels, ev.Tobs, ev.GMST, L=ref.native_lib())
        S = ev.SN.copy()
        S[:, int(16.0 * ev.Tobs):int(ev.fmin * ev.Tobs)] = np.inf   # reference built with fmin = 16 Hz
        kind, cores = "reference", ref.max_threads(net.L)
        impl_note += f", build {ref.native_variant()}"
        run = lambda X, nt=cores: ref.lnl_full_batch(net, ev.D, X, ev.freq, S, ev.N, ev.Tobs, nthreads=nt)  # noqa: E731
    except Exception:
        from oracle import ora
        kind, cores = "port", os.cpu_count()
        run = lambda X, nt=cores: ora.lnl_full_batch(ev, X)  # noqa: E731

    def sample(seconds, nt, chunk):
        n, secs, k = 0, 0.0, 0
        t_end = time.perf_counter() + seconds
        while time.perf_counter() < t_end:
            X = P[(k * chunk) % len(P):(k * chunk) % len(P) + chunk]
            _, s = run(X, nt)
            n += len(X)
            secs += s
            k += 1
        return n, secs

    chunk = 64
    n, secs = sample(budget_s, cores, chunk)
    out = {"value": n / secs, "unit": "lnL evals/s", "cores": int(cores), "kind": kind,
           "sample": f"{n} parameter sets of the benchmark batch in chunks of {chunk}, OpenMP over sets, "
                     f"{secs:.1f} s wall{impl_note}"}
    if kind == "reference":
        n1, s1 = sample(3.0, 1, 4)
        run(P[:1], cores)                 # restore the thread count
        out["single_thread"] = {"value": n1 / s1, "unit": "lnL evals/s", "sample": f"{n1} sets, 1 thread, {s1:.1f} s"}
    return out


def run_reference_arm(args):
    rank, world, _ = env_rank()
    if rank != 0:
        return
    from quickcbc_b200 import synth
    from oracle import ora

    def tmpl(info, p):
        return ora.fulltemplates(info["labels"], info["GMST"], info["freq"], p, info["N"])

    ev = synth.config_event(2, tmpl)
    P = synth.draw_params(np.random.default_rng(2000 + 500000), CONFIG["B"], ev.inj)
    sample = 128   # parameter sets per timed step (bounded sample of the 2048-set step)
    try:
        from oracle import ref
        net = ref.RefNet(ev.labels, ev.Tobs, ev.GMST, L=ref.native_lib())
        S = ev.SN.copy()
        S[:, int(16.0 * ev.Tobs):int(ev.fmin * ev.Tobs)] = np.inf
        run = lambda X: ref.lnl_full_batch(net, ev.D, X, ev.freq, S, ev.N, ev.Tobs)  # noqa: E731
        kind, cores = "reference", ref.max_threads(net.L)
        build = ref.native_variant()
    except Exception:
        run = lambda X: ora.lnl_full_batch(ev, X)  # noqa: E731
        kind, cores, build = "port", os.cpu_count(), "oracle/_build"
    for w in range(args.warmup):
        run(P[:sample])
    secs = 0.0
    for k in range(args.steps):
        X = P[(k * sample) % CONFIG["B"]:(k * sample) % CONFIG["B"] + sample]
        _, s = run(X)
        secs += s
    v = args.steps * sample / secs
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "lnL evals/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * secs / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic coloured Gaussian noise + IMRPhenomD injection", "config": dict(CONFIG),
            "cpu_baseline": {"value": v, "unit": "lnL evals/s", "cores": int(cores), "kind": kind,
                             "sample": f"{sample} of the 2048 parameter sets per step, OpenMP over sets",
                             "build": build},
            "e2e": {"value": v, "unit": "lnL evals/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def bench_cfg1_percall(q, eng, _lib):
    """Config 1: plain FP64 drop-in, one log_likelihood_full call per chain (16 temperatures)."""
    import ctypes as C
    from quickcbc_b200 import synth

    def tmpl(info, p):
        return q.fulltemplates(info["labels"], info["GMST"], info["freq"], p, info["N"])
    ev = synth.config_event(1, tmpl)
    P = synth.jitter_params(np.random.default_rng(1000 + 500000), 16, ev.inj)
    q.set_band(ev.fmin, 1024.0)
    nh = eng._NetHolder(ev.labels, ev.Tobs, ev.GMST)
    Dr, Sr = eng._rows(ev.D), eng._rows(ev.SN)
    fr, rv = eng._rv(ev.freq)
    _lib.check(_lib.lib().qcbc_bind_data(nh.ref, Dr, Sr, ev.N, ev.Tobs))
    rho = np.zeros(4)
    fn = _lib.lib().log_likelihood_full
    Pc = [np.ascontiguousarray(p) for p in P]
    for p in Pc:
        fn(nh.ref, Dr, eng._ptr(p), C.byref(rv), Sr, eng._ptr(rho), ev.N, ev.Tobs)
    steps = 64
    t0 = time.perf_counter()
    for _ in range(steps):
        for p in Pc:
            fn(nh.ref, Dr, eng._ptr(p), C.byref(rv), Sr, eng._ptr(rho), ev.N, ev.Tobs)
    dt = time.perf_counter() - t0
    _lib.lib().qcbc_unbind_all()
    q.set_band(16.0, 1024.0)
    return {"workload": "config 1: H1/L1, 4 s, 2048 Hz, 16 temperatures x 1 call, FP64 drop-in",
            "value": steps * 16 / dt, "unit": "lnL evals/s", "us_per_call": 1e6 * dt / (steps * 16)}


def _native_rate(which, net, het, D, rv, SN, N, Tobs, P, calls, nthreads):
    """Reference-signature calls per second from `nthreads` native host threads started together
    (qcbc_time_dropin: C++ threads, no interpreter between calls)."""
    import ctypes as C
    from quickcbc_b200 import _lib, engine as eng
    Pc = np.ascontiguousarray(P, dtype=np.float64)
    secs, last = C.c_double(0.0), np.zeros(nthreads)
    _lib.check(_lib.lib().qcbc_time_dropin(which, net, het, D, rv, SN, N, Tobs, eng._ptr(Pc), len(Pc), calls,
                                           nthreads, C.byref(secs), eng._ptr(last)))
    return {"value": nthreads * calls / secs.value, "us_per_call_per_thread": secs.value / calls * 1e6}


def dropin_per_call_rates(q, ev, P, calls=400):
    """log_likelihood_full under the reference's signature, one parameter set per call, from one host
    thread and from 12 at once (the reference's NC = 12 OpenMP chains, QuickCBC.c:118, 2063-2067;
    native threads), with the data registered by qcbc_bind_data and without (the unchanged
    program's path: each call checks that the cached device copy still holds the caller's D and
    SN).  Concurrent calls on one event are merged into shared launches."""
    import ctypes as C
    from quickcbc_b200 import _lib, engine as eng
    L = _lib.lib()
    nh = eng._NetHolder(ev.labels, ev.Tobs, ev.GMST)
    D, SN = eng._f64(ev.D), eng._f64(ev.SN)
    Dr, Sr = eng._rows(D), eng._rows(SN)
    fr, rv = eng._rv(ev.freq)
    Pc = np.ascontiguousarray(P[:96])

    def rate(nthreads):
        return _native_rate(0, nh.ref, None, Dr, C.byref(rv), Sr, ev.N, ev.Tobs, Pc, calls, nthreads)

    out = {"unit": "lnL evals/s", "note": "FP64, log_likelihood_full reference signature, one set per call, "
                                          "native host threads"}
    L.qcbc_unbind_all()
    out["one_thread_unbound"] = rate(1)
    out["12_threads_unbound"] = rate(12)
    _lib.check(L.qcbc_bind_data(nh.ref, Dr, Sr, ev.N, ev.Tobs))
    out["one_thread_bound"] = rate(1)
    out["12_threads_bound"] = rate(12)
    L.qcbc_unbind_all()
    out["value"] = out["one_thread_bound"]["value"]
    return out


def dropin_het_per_call_rates(q, ev, het_grid, P, calls=1000):
    """log_likelihood_het under the reference's signature (its sampler's hot call, QuickCBC.c:2372),
    one set per call, from one native host thread and from 12 at once: the rate an unchanged
    QuickCBC linked against the library sees.  The tables come from the drop-in heterodyne on the
    same grid."""
    import ctypes as C
    from quickcbc_b200 import engine as eng
    H = eng.LegacyHet(ev.labels, ev.GMST, ev.Tobs, het_grid["fgrid"], int(het_grid["MN"]), int(het_grid["MM"]),
                      int(het_grid["J"]))
    H.heterodyne(ev.D, ev.inj, ev.freq, ev.SN, ev.N)
    Pc = np.ascontiguousarray(P[:200])

    def rate(nthreads):
        return _native_rate(1, H.nh.ref, C.byref(H.het), None, None, None, ev.N, ev.Tobs, Pc, calls, nthreads)

    return {"unit": "lnL evals/s", "note": "FP64, log_likelihood_het reference signature, one set per call, "
                                          "native host threads", "one_thread": rate(1), "12_threads": rate(12)}


def cpu_baseline_het(ev, het_grid, P, budget_s=10.0):
    """The reference's log_likelihood_het (QuickCBC.c:5303, its production hot loop) on its own
    heterodyne tables for the same grid, under OpenMP over the sets on all host cores, on a bounded
    sample of the config-3 sets; plus one thread."""
    from oracle import ref
    L = ref.native_lib()
    net = ref.RefNet(ev.labels, ev.Tobs, ev.GMST, L=L)
    S = ev.SN.copy()
    S[:, int(16.0 * ev.Tobs):int(ev.fmin * ev.Tobs)] = np.inf   # reference built with fmin = 16 Hz
    het = ref.RefHet(net)
    het.set_grid(het_grid["fgrid"], int(het_grid["MN"]), int(het_grid["MM"]), int(het_grid["J"]), ev.Tobs)
    with _QuietCStdout():
        het.heterodyne(ev.D, ev.inj, ev.freq, S, ev.N, ev.Tobs)
    cores = ref.max_threads(L)

    def sample(seconds, nt, chunk):
        n, secs, k = 0, 0.0, 0
        t_end = time.perf_counter() + seconds
        while time.perf_counter() < t_end:
            X = P[(k * chunk) % len(P):(k * chunk) % len(P) + chunk]
            _, sec = het.lnl_batch(X, ev.Tobs, nthreads=nt)
            n += len(X)
            secs += sec
            k += 1
        return n, secs

    n, secs = sample(budget_s, cores, 1024)
    n1, s1 = sample(2.0, 1, 64)
    het.lnl_batch(P[:1], ev.Tobs, nthreads=cores)          # restore the thread count
    Lr, _ = het.lnl_batch(P[:256], ev.Tobs)
    return {"value": n / secs, "unit": "lnL evals/s", "cores": int(cores), "kind": "reference",
            "build": ref.native_variant(),
            "sample": f"{n} of the config-3 sets in chunks of 1024, OpenMP over sets, {secs:.1f} s wall",
            "single_thread": {"value": n1 / s1, "unit": "lnL evals/s", "sample": f"{n1} sets, 1 thread"},
            "lnl_first256": Lr}


def prior_box(Tobs):
    """MCMC_all's prior box (QuickCBC.c:1871-1896, ConstCBC.h:48-57)."""
    from quickcbc_b200 import synth
    M, PC = synth.MSUN_SI, synth.PC_SI
    pmin = np.array([np.log(0.5 * M), np.log(0.5 * M), -0.85, -0.85, 0.0, max(Tobs - 3.5, 1.5),
                     np.log(1e6 * PC), 0.0, -1.0, 0.0, -1.0])
    pmax = np.array([np.log(160 * M), np.log(300 * M), 0.85, 0.85, 2 * np.pi, Tobs - 0.5,
                     np.log(1e10 * PC), 2 * np.pi, 1.0, np.pi, 1.0])
    return pmin, pmax


def reference_het_space_child():
    """Child process: the reference's het_space + heterodyne (oracle/_ref) on config 3; prints
    the wall seconds as JSON.  Runs apart from the GPU process because the reference's
    het_space reads its grid after freeing it (QuickCBC.c:4866-4893)."""
    import tempfile
    from oracle import ora, ref
    from quickcbc_b200 import synth

    def tmpl(info, p):
        return ora.fulltemplates(info["labels"], info["GMST"], info["freq"], p, info["N"])
    ev = synth.config_event(3, tmpl)
    pmin, pmax = prior_box(ev.Tobs)
    net = ref.RefNet(ev.labels, ev.Tobs, ev.GMST)
    S = ev.SN.copy()
    S[:, int(16.0 * ev.Tobs):int(ev.fmin * ev.Tobs)] = np.inf   # reference built with fmin = 16 Hz
    het = ref.RefHet(net)
    with tempfile.TemporaryDirectory() as d:
        t0 = time.perf_counter()
        het.space(ev.inj, pmin, pmax, ev.freq, S, ev.N, ev.Tobs, d)
        het.heterodyne(ev.D, ev.inj, ev.freq, S, ev.N, ev.Tobs)
        dt = time.perf_counter() - t0
    print(json.dumps({"seconds": dt, "M": het.sizes()["M"]}))


def reference_het_space_seconds():
    """Wall time of the reference's het_space + heterodyne on this host (child process), or the
    reason it is missing.  glibc's mmap threshold is raised in the child so that the grid the
    reference frees stays mapped when it reads it back."""
    try:
        from oracle import ref
        if not ref.available():
            return {"unavailable": "oracle/_ref not built"}
        env = dict(os.environ, MALLOC_MMAP_THRESHOLD_=str(1 << 30))
        r = subprocess.run([sys.executable, os.path.abspath(__file__), "--ref-het-space-child"], env=env,
                           capture_output=True, text=True, timeout=300)
        lines = [x for x in r.stdout.splitlines() if x.startswith("{")]
        if r.returncode != 0 or not lines:
            return {"unavailable": f"reference het_space exited with {r.returncode}"}
        return json.loads(lines[-1])
    except Exception as exc:
        return {"unavailable": f"{type(exc).__name__}: {exc}"}


def bench_cfg3_het(q):
    """Config 3: 3 det, 128 s, 4096 Hz BNS; heterodyne grid search and tables on the GPU
    (het_space + heterodyne, the analysis-admission latency), then the heterodyned lnL for
    4096 sets and the full lnL for 512 sets."""
    from quickcbc_b200 import synth

    def tmpl(info, p):
        return q.fulltemplates(info["labels"], info["GMST"], info["freq"], p, info["N"])
    g3 = np.load(os.path.join(ROOT, "tests", "golden", "grid3.npz"))
    ev = synth.config_event(3, tmpl)
    e = q.Event.from_synthetic(ev)
    pmin, pmax = prior_box(ev.Tobs)
    e.het_space(ev.inj, pmin, pmax)                       # warm-up
    t0 = time.perf_counter()
    fgrid, MN, MM = e.het_space(ev.inj, pmin, pmax)
    t1 = time.perf_counter()
    e.het_setup(ev.inj, fgrid, MN, MM, 2)
    t2 = time.perf_counter()
    # sets where sampler chains sit: Fisher steps (the device Fisher_Het at the injection) whose
    # length is searched so that lnL falls by U[0.5, 10] (half the sets: posterior width),
    # U[10, 60] and U[100, 400] (burn-in) below the injection
    rng = np.random.default_rng(3000 + 500000)
    F = e.het_fisher(ev.inj[None, :])[0]
    ranges = ((0.5, 10.0, 2048), (10.0, 60.0, 1024), (100.0, 400.0, 1024))
    drops = np.concatenate([rng.uniform(lo, hi, n) for lo, hi, n in ranges])
    P = synth.cloud_at_drops(rng, ev.inj, F, drops, lambda X: e.lnl_het(X, q.FP64, allow_invalid=True))
    group = np.repeat(np.arange(len(ranges)), [n for _, _, n in ranges])
    dP = q.DeviceBuffer(P.nbytes)
    dP.upload(P)
    out = {"workload": "config 3: 3 det, 128 s, 4096 Hz, BNS 1.45+1.30, het grid M=%d; 4096 sets whose "
                       "lnL lies 0.5-10 (2048), 10-60 (1024) and 100-400 (1024) below the injection's"
                       % len(fgrid),
           "het_space_s": t1 - t0, "heterodyne_s": t2 - t1,
           "grid_equals_reference": bool(np.array_equal(fgrid, g3["fgrid"])),
           "reference_het_space_heterodyne": reference_het_space_seconds()}
    Lh64 = e.lnl_het(P, q.FP64)
    Lhm = e.lnl_het(P, q.MIXED)
    L0 = e.lnl_het(ev.inj[None, :], q.FP64)[0]
    out["het_lnl_drop_range"] = [float(np.min(L0 - Lh64)), float(np.max(L0 - Lh64))]
    out["het_max_abs_dlnL_mixed_vs_fp64_by_drop"] = {
        "%g-%g" % (lo, hi): float(np.max(np.abs(Lh64 - Lhm)[group == k])) for k, (lo, hi, _) in enumerate(ranges)}
    # the reference's own values on the fixture's 48 sets at the same three spreads
    z3 = np.load(os.path.join(ROOT, "tests", "golden", "spread3.npz"))
    if np.array_equal(fgrid, g3["fgrid"]) and ev.GMST == float(z3["GMST"]):
        Pz = z3["params"]
        out["vs_reference_spread_fixture"] = {
            "sets": int(len(Pz)),
            "het_mixed_max_abs": float(np.max(np.abs(e.lnl_het(Pz, q.MIXED) - z3["lnl_het"]))),
            "het_fp64_max_abs": float(np.max(np.abs(e.lnl_het(Pz, q.FP64) - z3["lnl_het"]))),
            "full_mixed_max_abs": float(np.max(np.abs(e.lnl_full(Pz, q.MIXED) - z3["lnl_full"]))),
            "full_fp64_max_abs": float(np.max(np.abs(e.lnl_full(Pz, q.FP64) - z3["lnl_full"]))),
        }
    for prec, name in ((q.MIXED, "het_mixed"), (q.FP64, "het_fp64")):
        q.time_lnl_het(e, dP, len(P), prec, 3, flush_l2=True)
        ms = q.time_lnl_het(e, dP, len(P), prec, 10, flush_l2=True)
        out[name] = {"value": len(P) / (np.median(ms) * 1e-3), "unit": "lnL evals/s", "ms": float(np.median(ms))}
    out["het_max_abs_dlnL_mixed_vs_fp64"] = float(np.max(np.abs(Lh64 - Lhm)))
    try:
        out["het_per_call_dropin"] = dropin_het_per_call_rates(q, ev, g3, P)
    except Exception as exc:
        out["het_per_call_dropin"] = {"unavailable": f"{type(exc).__name__}: {exc}"}
    try:
        cb = cpu_baseline_het(ev, g3, P)
        cb["max_abs_dlnL_gpu_fp64_vs_reference"] = float(np.max(np.abs(np.asarray(cb.pop("lnl_first256")) -
                                                                       Lh64[:256])))
        out["cpu_baseline_het"] = cb
    except Exception as exc:
        out["cpu_baseline_het"] = {"unavailable": f"{type(exc).__name__}: {exc}"}
    Pf = P[::8]                                          # 512 sets across the three spreads
    dPf = q.DeviceBuffer(Pf.nbytes)
    dPf.upload(Pf)
    Lf64 = e.lnl_full(Pf, q.FP64)
    Lfm = e.lnl_full(Pf, q.MIXED)
    for prec, name in ((q.MIXED, "full_mixed"), (q.FP64, "full_fp64")):
        q.time_lnl_full(e, dPf, len(Pf), prec, 2, flush_l2=True, kernel_times=False)
        ms, _ = q.time_lnl_full(e, dPf, len(Pf), prec, 5, flush_l2=True, kernel_times=False)
        out[name] = {"value": len(Pf) / (np.median(ms) * 1e-3), "unit": "lnL evals/s", "ms": float(np.median(ms))}
    out["full_max_abs_dlnL_mixed_vs_fp64"] = float(np.max(np.abs(Lf64 - Lfm)))
    out["het_vs_full_fp64_max_abs"] = float(np.max(np.abs(Lh64[::8] - Lf64)))
    e.close()
    return out


class _QuietCStdout:
    """fd 1 to /dev/null while the reference's C code runs in this process (its heterodyne prints
    "ref logL = ..."), with the C library's buffer flushed before fd 1 comes back, so that the
    bench's only stdout line stays its JSON line."""

    def __enter__(self):
        import ctypes
        self._libc = ctypes.CDLL(None)
        sys.stdout.flush()
        self._libc.fflush(None)
        self._saved = os.dup(1)
        self._null = os.open(os.devnull, os.O_WRONLY)
        os.dup2(self._null, 1)
        return self

    def __exit__(self, *exc):
        self._libc.fflush(None)
        os.dup2(self._saved, 1)
        os.close(self._saved)
        os.close(self._null)
        return False


def bench_input_stage(q):
    """Input stage at config 3 sizes (3 det, 128 s, 4096 Hz, N = 2^19): data conditioning
    (Tukey window, FFT, sqrt(Tobs)/N) and the noisemarg PSD redraw of an event holding heterodyne
    tables (makespec of every detector, weighted data, heterodyne tables rebuilt), on the GPU and
    with the reference's CPU code (tukey + GSL-layout FFT; makespec + heterodyne, one thread)."""
    from quickcbc_b200 import ingest, synth

    def tmpl(info, p):
        return q.fulltemplates(info["labels"], info["GMST"], info["freq"], p, info["N"])
    ev = synth.config_event(3, tmpl)
    g3 = np.load(os.path.join(ROOT, "tests", "golden", "grid3.npz"))
    x = synth.time_series(ev)
    ingest.condition_data(x, ev.Tobs)
    ts = []
    for _ in range(3):
        t0 = time.perf_counter()
        D = ingest.condition_data(x, ev.Tobs)
        ts.append(time.perf_counter() - t0)
    ns, nl, ffit, xs, L = synth.psd_model_arrays(np.random.default_rng(3800), 3, ev.Tobs, ev.N, nsample=4,
                                                 nknots=(64, 64, 64), nlines=(6, 6, 6))
    m = ingest.PsdModel(ffit, xs, L, ns, nl)
    e = q.Event(ev.labels, ev.Tobs, ev.GMST, ev.N, D, m.draw(0, ev.Tobs, ev.N), fmin=ev.fmin)
    e.het_setup(ev.inj, g3["fgrid"], int(g3["MN"]), int(g3["MM"]), 2)
    e.set_psd_sample(m, 1)
    tr = []
    for k in range(6):
        t0 = time.perf_counter()
        e.set_psd_sample(m, k % 4)
        tr.append(time.perf_counter() - t0)
    out = {"workload": "config 3 input stage: 3 det x N = 2^19; PSD model 64 knots + 6 lines x 4 samples, "
                       "het grid M=%d" % len(g3["fgrid"]),
           "condition_data_s": float(np.median(ts)), "noisemarg_redraw_s": float(np.median(tr))}
    try:
        from oracle import ref
        if ref.available():
            t0 = time.perf_counter()
            Dr = np.array([ref.condition(xi, ev.Tobs) for xi in x])
            out["reference_condition_s"] = time.perf_counter() - t0
            out["condition_max_rel_diff"] = float(np.max(np.abs(D - Dr)) / np.max(np.abs(Dr)))
            net = ref.RefNet(ev.labels, ev.Tobs, ev.GMST)
            het = ref.RefHet(net)
            het.set_grid(g3["fgrid"], int(g3["MN"]), int(g3["MM"]), 2, ev.Tobs)
            with _QuietCStdout():
                t0 = time.perf_counter()
                S = np.zeros((3, ev.N // 2 + 1))
                for i in range(3):
                    S[i, :ev.N // 2] = ref.makespec(ffit[i], xs[i, 1], *L[i, 1].T, ev.Tobs, ev.N)
                het.heterodyne(Dr, ev.inj, ev.freq, S, ev.N, ev.Tobs)
                out["reference_redraw_s"] = time.perf_counter() - t0
            out["reference_cores"] = 1
    except Exception as exc:
        out["reference"] = f"unavailable: {type(exc).__name__}: {exc}"
    e.close()
    m.close()
    return out


def interleaved_stream(q, b, evs, eo, P, Lm):
    """The config-4 sets in round-robin event order (set k of every event, then set k + 1, ...):
    the blocks in flight read the data of all 256 events at once, about 16 B per detector-bin
    of each set (the FP32 weighted data), far more than L2 holds, so the launch streams its
    event data from HBM.  Achieved bandwidth counts each set's in-band bins once."""
    order = np.lexsort((eo, np.arange(len(eo)) - np.searchsorted(eo, eo)))
    eo_i, P_i = eo[order], P[order]
    L_i = b.lnl(eo_i, P_i, q.MIXED)
    ms = b.time(len(P_i), q.MIXED, iters=5, flush_l2=True)
    nbytes = 0
    for e, ev in enumerate(evs):
        bins = min(int(ev.Tobs * 1024.0), ev.N // 2) - int(ev.Tobs * ev.fmin)
        # useful bytes: FP32 (wr, wi, ws) per detector-bin and one FP32 bin factor per bin
        nbytes += int(np.sum(eo == e)) * bins * 12 * len(ev.labels)
    t = float(np.median(ms)) * 1e-3
    peak, kind = load_peaks()
    return {"value": len(P_i) / t, "unit": "lnL evals/s", "ms": t * 1e3, "stream_bytes": nbytes,
            "achieved_GBs": nbytes / t / 1e9, "frac_hbm": nbytes / t / 1e9 / peak, "peak_kind": kind,
            "bytes_note": "12 B per detector-bin of every set (each set reads its event's band; the bin factor "
                          "i^-7/6 is folded into the weighted data)",
            "same_lnl_as_grouped_order": bool(np.array_equal(L_i, Lm[order]))}


def bench_cfg4_uneven(q):
    """Config 4: 256 uneven events x (32 chains x 8 proposals) in one graph-captured
    persistent launch, autotuned tiling, mixed and FP64."""
    from quickcbc_b200 import synth

    def tmpl(info, p):
        return q.fulltemplates(info["labels"], info["GMST"], info["freq"], p, info["N"])
    evs = [synth.make_event(tmpl, **s) for s in synth.uneven_event_specs(256)]
    hs = [q.Event.from_synthetic(x) for x in evs]
    b = q.Batch(hs)
    eo, P = synth.uneven_params(evs)
    tiling = b.autotune(eo, P, q.MIXED)
    Lm = b.lnl(eo, P, q.MIXED)
    L64 = b.lnl(eo, P, q.FP64)
    out = {"workload": "config 4: 256 events (Tobs 4-64 s, fs 2048/4096 Hz, 1-3 det), 65536 sets per launch",
           "tiling": list(tiling), "device_bytes": int(sum(h.device_bytes() for h in hs)),
           "max_abs_dlnL_mixed_vs_fp64": float(np.max(np.abs(Lm - L64)))}
    for prec, name, it in ((q.MIXED, "mixed", 8), (q.FP64, "fp64", 3)):
        ms = b.time(len(P), prec, iters=it, flush_l2=True)
        out[name] = {"value": len(P) / (np.median(ms) * 1e-3), "unit": "lnL evals/s", "ms": float(np.median(ms))}
    t0 = time.perf_counter()
    for _ in range(3):
        b.lnl(eo, P, q.MIXED)
    out["e2e_mixed"] = {"value": 3 * len(P) / (time.perf_counter() - t0), "unit": "lnL evals/s",
                        "h2d_bytes_per_step": int(P.nbytes + eo.nbytes), "d2h_bytes_per_step": int(len(P) * 44)}
    out["mixed_interleaved"] = interleaved_stream(q, b, evs, eo, P, Lm)
    b.close()
    for h in hs:
        h.close()
    return out


def bench_cfg5_serving(q, n_runs=32, n_steps=20000, precisions=("mixed", "fp64", "mixed-het", "mixed-dev",
                                                                 "mixed-het-dev"), rate_hz=2.0, device_steps=16):
    """Config 5: Poisson arrivals (mean rate_hz) of PT-MCMC analyses of config-4-like events
    (16 temperatures x 8 chains x n_steps), device-resident runs admitted by a 150 GB budget,
    every step of every live run merged into one multi-event launch."""
    from quickcbc_b200 import serving, synth

    def tmpl(info, p):
        return q.fulltemplates(info["labels"], info["GMST"], info["freq"], p, info["N"])
    evs = [synth.make_event(tmpl, **s) for s in synth.uneven_event_specs(n_runs, seed=5000)]
    arrivals = "all submitted at t = 0" if rate_hz is None else "Poisson %.1f/s" % rate_hz
    out = {"workload": "config 5: %d runs, %s, 16 temps x 8 chains x %d steps, config-4 events, "
                       "HBM budget 150 GB" % (n_runs, arrivals, n_steps)}
    for name in precisions:
        # "<precision>" samples the full lnL; "<precision>-het" builds each run's heterodyne grid and
        # tables on the GPU at admission and samples the heterodyned lnL, as the reference does;
        # "-dev" keeps the chains on the device, up to device_steps steps per host call; "-ref" uses
        # the reference's proposal mixture (Fisher jumps, differential evolution, jiggles)
        parts = name.split("-")
        prec = q.MIXED if parts[0] == "mixed" else q.FP64
        lik = "het" if "het" in parts else "full"
        srv = serving.Server(hbm_budget_bytes=150 * 10**9, max_live=256, max_bins=1 << 17, precision=prec,
                             device_steps=device_steps if "dev" in parts else 0)
        srv.set_tiling(8192, 256)
        res = serving.serve_stream(srv, evs, rate_hz=rate_hz, seed=5,
                                   sampler=dict(n_temps=16, n_chains=8, n_steps=n_steps, burn_in=n_steps // 4,
                                                thin=max(1, n_steps // 200), likelihood=lik,
                                                proposal="reference" if "ref" in parts else "gauss"))
        st = srv.stats()
        res.pop("ttp_s")
        res["launches"] = st["launches"]
        out[name] = res
        srv.close()
    return out


def run_profile(args):
    """Warm-up then timed steps of the benchmark workload in one precision: k_setup and the lnL
    kernel per step (and k_finalize_full when a set spans several tiles)."""
    import quickcbc_b200 as q
    from quickcbc_b200 import _lib
    _lib.check(_lib.lib().qcbc_init(0))
    ev, P = make_workload()
    e = q.Event.from_synthetic(ev)
    dbuf = q.DeviceBuffer(P.nbytes)
    dbuf.upload(P)
    prec = q.MIXED if args.prec == "mixed" else q.FP64
    q.time_lnl_full(e, dbuf, len(P), prec, args.warmup, flush_l2=False)
    ms, kms = q.time_lnl_full(e, dbuf, len(P), prec, args.steps, flush_l2=True)
    print(json.dumps({"profile": args.prec, "B": len(P), "step_ms": [float(x) for x in ms],
                      "kernel_ms": [float(x) for x in kms], "tiles_threads": e.get_launch(len(P), prec)}))
    e.close()


def run_percall(args):
    """The reference-signature drop-ins called one parameter set at a time, as QuickCBC's sampler
    calls them: device time of a B = 1 and a B = 12 step (the sizes of a lone call and of twelve
    merged ones), the host-buffer call's time, and the native-thread call rates from 1 and 12
    threads.  Config 2 for the full likelihood (FP64), config 3 for the heterodyned one (FP64)."""
    import quickcbc_b200 as q
    from quickcbc_b200 import _lib, synth
    _lib.check(_lib.lib().qcbc_init(0))

    def step_times(timer, call, P, B):
        d = q.DeviceBuffer(P[:B].nbytes)
        d.upload(P[:B])
        timer(d, B, 20)
        ms = timer(d, B, 200)
        for _ in range(20):
            call(P[:B])
        t0 = time.perf_counter()
        for _ in range(300):
            call(P[:B])
        return {"device_us_median": float(np.median(ms) * 1e3), "host_call_us": (time.perf_counter() - t0) / 300 * 1e6}

    out = {"metric": "reference-signature calls, one parameter set per call (FP64)"}
    ev, P = make_workload()
    q.set_band(ev.fmin, 1024.0)
    e = q.Event.from_synthetic(ev)
    full = {"workload": "config 2: 3 det, 16 s, 4096 Hz"}
    for B in (1, 12):
        full[f"B{B}"] = step_times(lambda d, b, n: q.time_lnl_full(e, d, b, q.FP64, n, flush_l2=False,
                                                                    kernel_times=False)[0],
                                   lambda X: e.lnl_full(X, q.FP64), P, B)
        full[f"B{B}"]["tiles_threads"] = e.get_launch(B, q.FP64)
    full["per_call"] = dropin_per_call_rates(q, ev, P)
    out["full"] = full

    def tmpl(info, p):
        return q.fulltemplates(info["labels"], info["GMST"], info["freq"], p, info["N"])
    g3 = np.load(os.path.join(ROOT, "tests", "golden", "grid3.npz"))
    ev3 = synth.config_event(3, tmpl)
    e3 = q.Event.from_synthetic(ev3)
    e3.het_setup(ev3.inj, g3["fgrid"], int(g3["MN"]), int(g3["MM"]), 2)
    P3 = synth.jitter_params(np.random.default_rng(3100), 256, ev3.inj, 1e-4)
    het = {"workload": "config 3: 3 det, 128 s, BNS, het grid M = %d" % len(g3["fgrid"])}
    for B in (1, 12):
        het[f"B{B}"] = step_times(lambda d, b, n: q.time_lnl_het(e3, d, b, q.FP64, n, flush_l2=False),
                                  lambda X: e3.lnl_het(X, q.FP64), P3, B)
    het["per_call"] = dropin_het_per_call_rates(q, ev3, g3, P3)
    out["het"] = het
    print(json.dumps(out))


def run_profile_cfg3(args):
    """Profiling run of the config-3 heterodyned step (k_setup then k_lnl_het) on 4096 sets spread
    as in the bench: grid and tables built on the GPU, `warmup` untimed steps, then `steps`."""
    import quickcbc_b200 as q
    from quickcbc_b200 import _lib, synth
    _lib.check(_lib.lib().qcbc_init(0))

    def tmpl(info, p):
        return q.fulltemplates(info["labels"], info["GMST"], info["freq"], p, info["N"])
    g3 = np.load(os.path.join(ROOT, "tests", "golden", "grid3.npz"))
    ev = synth.config_event(3, tmpl)
    e = q.Event.from_synthetic(ev)
    e.het_setup(ev.inj, g3["fgrid"], int(g3["MN"]), int(g3["MM"]), int(g3["J"]))
    rng = np.random.default_rng(3000 + 500000)
    F = e.het_fisher(ev.inj[None, :])[0]
    drops = np.concatenate([rng.uniform(0.5, 10.0, 2048), rng.uniform(10.0, 60.0, 1024), rng.uniform(100.0, 400.0, 1024)])
    P = synth.cloud_at_drops(rng, ev.inj, F, drops, lambda X: e.lnl_het(X, q.FP64, allow_invalid=True))
    d = q.DeviceBuffer(P.nbytes)
    d.upload(P)
    prec = q.MIXED if args.prec == "mixed" else q.FP64
    q.time_lnl_het(e, d, len(P), prec, args.warmup, flush_l2=True)
    ms = q.time_lnl_het(e, d, len(P), prec, args.steps, flush_l2=True)
    print(json.dumps({"profile": "config3 heterodyned " + args.prec, "B": len(P), "ms": [float(x) for x in ms]}))
    e.close()


def run_profile_cfg4(args):
    """Profiling run of the config-4 interleaved launch (the HBM-streaming case): the 256 events and
    65536 sets in round-robin event order, `warmup` untimed launches, then `steps` launches."""
    import quickcbc_b200 as q
    from quickcbc_b200 import _lib, synth
    _lib.check(_lib.lib().qcbc_init(0))

    def tmpl(info, p):
        return q.fulltemplates(info["labels"], info["GMST"], info["freq"], p, info["N"])
    evs = [synth.make_event(tmpl, **sp) for sp in synth.uneven_event_specs(256)]
    hs = [q.Event.from_synthetic(x) for x in evs]
    b = q.Batch(hs)
    eo, P = synth.uneven_params(evs)
    order = np.lexsort((eo, np.arange(len(eo)) - np.searchsorted(eo, eo)))
    b.set_tiling(8192, 256)     # fixed, so that the launch count before the captured one is known
    b.lnl(eo[order], P[order], q.MIXED)
    b.time(len(P), q.MIXED, iters=args.warmup, flush_l2=True)
    ms = b.time(len(P), q.MIXED, iters=args.steps, flush_l2=True)
    print(json.dumps({"profile": "config4 interleaved mixed", "B": len(P), "ms": [float(x) for x in ms],
                      "tiling": list(b.tiling())}))
    b.close()
    for h in hs:
        h.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extra", action="store_true", help="skip configs 1, 3, 4 and the reduced config 5")
    ap.add_argument("--serve", action="store_true", help="config 5 serving stream only")
    ap.add_argument("--input-stage", action="store_true", help="config 3 input stage only")
    ap.add_argument("--cfg3", action="store_true", help="config 3 (heterodyned, 128 s BNS) only")
    ap.add_argument("--cfg4", action="store_true", help="config 4 (256 uneven events) only")
    ap.add_argument("--serve-runs", type=int, default=32)
    ap.add_argument("--serve-steps", type=int, default=20000)
    ap.add_argument("--serve-prec", default="mixed,fp64,mixed-het,mixed-dev,mixed-het-dev")
    ap.add_argument("--serve-dev-steps", type=int, default=16)
    ap.add_argument("--profile", action="store_true",
                    help="profiling run: warm-up and timed steps of one precision only (for ncu)")
    ap.add_argument("--prec", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--profile-cfg3", action="store_true",
                    help="profiling run of the config-3 heterodyned step (for ncu)")
    ap.add_argument("--profile-cfg4", action="store_true",
                    help="profiling run of the config-4 interleaved launch (for ncu)")
    ap.add_argument("--percall", action="store_true",
                    help="reference-signature drop-ins, one set per call: step latencies and 1/12-thread rates")
    ap.add_argument("--ref-het-space-child", action="store_true", help=argparse.SUPPRESS)
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.ref_het_space_child:
        return reference_het_space_child()
    if args.impl == "reference":
        return run_reference_arm(args)
    if args.profile:
        return run_profile(args)
    if args.profile_cfg3:
        return run_profile_cfg3(args)
    if args.percall:
        return run_percall(args)
    if args.profile_cfg4:
        return run_profile_cfg4(args)
    if args.serve:
        import quickcbc_b200 as q
        from quickcbc_b200 import _lib
        _lib.check(_lib.lib().qcbc_init(0))
        res = bench_cfg5_serving(q, n_runs=args.serve_runs, n_steps=args.serve_steps,
                                 precisions=tuple(args.serve_prec.split(",")), device_steps=args.serve_dev_steps)
        print(json.dumps({"metric": "time-to-posterior p50/p99 and aggregate lnL evals/s (config 5)", **res}))
        return
    if args.cfg3:
        import quickcbc_b200 as q
        from quickcbc_b200 import _lib
        _lib.check(_lib.lib().qcbc_init(0))
        print(json.dumps({"metric": "lnL evals/s (config 3)", **bench_cfg3_het(q)}))
        return
    if args.cfg4:
        import quickcbc_b200 as q
        from quickcbc_b200 import _lib
        _lib.check(_lib.lib().qcbc_init(0))
        print(json.dumps({"metric": "lnL evals/s (config 4)", **bench_cfg4_uneven(q)}))
        return
    if args.input_stage:
        import quickcbc_b200 as q
        from quickcbc_b200 import _lib
        _lib.check(_lib.lib().qcbc_init(0))
        print(json.dumps({"metric": "input-stage seconds (config 3)", **bench_input_stage(q)}))
        return

    from quickcbc_b200.replicas import Replicas
    rep = Replicas()
    rank, world, local = rep.rank, rep.world, rep.local_rank
    import quickcbc_b200 as q
    from quickcbc_b200 import _lib
    _lib.check(_lib.lib().qcbc_init(local))

    ev, P = make_workload(seed_offset=rank)
    e = q.Event.from_synthetic(ev)
    B = len(P)
    dbuf = q.DeviceBuffer(P.nbytes)
    dbuf.upload(P)

    # parity spot check on the benchmark batch itself
    L64 = e.lnl_full(P, q.FP64)
    Lmx = e.lnl_full(P, q.MIXED)
    dmax = float(np.max(np.abs(L64 - Lmx)))

    q.time_lnl_full(e, dbuf, B, q.MIXED, args.warmup, flush_l2=True)
    rep.barrier()
    with ClockSampler(local) as clk:
        # the same workload keeps the GPU loaded around the timed steps so the
        # 200 ms clock samples are taken under this load
        t_load = time.perf_counter() + 1.0
        while time.perf_counter() < t_load:
            q.time_lnl_full(e, dbuf, B, q.MIXED, 20, flush_l2=False)
        n0 = q.launch_count()
        # the timed steps run as a plain call does (no event between the setup and the lnL
        # kernel, which would end their programmatic overlap) ...
        ms, _ = q.time_lnl_full(e, dbuf, B, q.MIXED, args.steps, flush_l2=True, kernel_times=False)
        launches = q.launch_count() - n0
        # ... and the same steps again with events around the lnL kernel give its launch duration
        # for the roofline
        _, kms = q.time_lnl_full(e, dbuf, B, q.MIXED, args.steps, flush_l2=True)
        t_load = time.perf_counter() + 0.6
        while time.perf_counter() < t_load:
            q.time_lnl_full(e, dbuf, B, q.MIXED, 20, flush_l2=False)
    t_ms = rep.max_over_ranks(float(np.sum(ms)))      # device time of the timed steps, max over ranks
    rep.barrier()
    value = world * B * args.steps / (t_ms * 1e-3)

    # FP64 batched on the same inputs (the plain form, batched)
    q.time_lnl_full(e, dbuf, B, q.FP64, 3, flush_l2=True)
    ms64, _ = q.time_lnl_full(e, dbuf, B, q.FP64, max(3, args.steps // 2), flush_l2=True, kernel_times=False)
    fp64_rate = B * len(ms64) / (np.sum(ms64) * 1e-3)

    # e2e through the public API with host buffers
    for _ in range(2):
        e.lnl_full(P, q.MIXED)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        e.lnl_full(P, q.MIXED)
    e2e_s = time.perf_counter() - t0
    e2e = {"value": world * B * args.steps / e2e_s if world == 1 else B * args.steps / e2e_s * world,
           "unit": "lnL evals/s", "h2d_bytes_per_step": int(P.nbytes),
           "d2h_bytes_per_step": int(B * 8)}

    # plain FP64 one-call-per-parameter-set drop-in (reference signature): one host thread with the
    # data bound once, and 12 host threads at once (the reference's NC = 12 OpenMP chains,
    # QuickCBC.c:118, 2063-2067) bound and unbound
    q.set_band(ev.fmin, 1024.0)
    percall = dropin_per_call_rates(q, ev, P)
    percall_rate = percall["one_thread_bound"]["value"]

    # roofline of the fused kernel: FP32 work per launch over its device time; the HBM view of the
    # same launch (the path's algorithmic 24 B per detector-bin) for context
    bins = ev.imax - ev.imin
    kmean = float(np.mean(kms)) * 1e-3
    clocks = clk.summary()
    fp32_peak = fp32_peak_tflops(clocks.get("sm_max_mhz"))
    flops_bin = WF_FLOPS_PER_BIN + PROJ_FLOPS_PER_DET_BIN * ev.nifo
    flops = B * bins * flops_bin
    tiles, threads = e.get_launch(B, q.MIXED)
    traffic, tinfo = capture_traffic("k_lnl_full_mixed_cfg2", "k_lnl_full_mixed", f"({B * tiles},1,1)",
                                     f"({threads},1,1)", kmean * 1e3)
    hbm_peak, peak_kind = load_peaks()
    alg_bytes = B * ev.nifo * bins * 24
    out = {
        "metric": METRIC, "value": value, "unit": "lnL evals/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64/f32 mixed", "data": "synthetic coloured Gaussian noise + IMRPhenomD injection",
        "config": dict(CONFIG, parallelism=f"replicas x{world}"),
        "e2e": e2e, "gpu_launches": int(launches),
        "roofline": {
            "bound": "issue", "achieved": flops / kmean / 1e12, "peak": fp32_peak, "unit": "TFLOP/s",
            "frac": flops / kmean / 1e12 / fp32_peak, "traffic": traffic, "kernel": "k_lnl_full_mixed<3>",
            "kernel_ms": kmean * 1e3, "flops_per_launch": flops, "flops_per_set_bin": flops_bin,
            "peak_kind": "FP32 FMA peak derived from the spec at the sampled max SM clock (148 SMs x 128 lanes x 2)",
            **tinfo,
            "hbm": {"algorithmic_bytes_per_launch": alg_bytes, "achieved_GBs": alg_bytes / kmean / 1e9,
                    "peak": hbm_peak, "peak_kind": peak_kind,
                    "note": "the path's 24 B per detector-bin (FP64 D re, im, S); one event's 0.6 MB of "
                            "weighted data serves all 2048 sets from L2, so DRAM carries only the "
                            "records and one pass of the data (traffic); HBM does not bind"},
            "note": "achieved = (%d + %d x %d) FP32 flops per set-bin x %d sets x %d bins / kernel time; the "
                    "kernel is bound by instruction issue (ncu: profiles/k_lnl_full_mixed_cfg2.md)"
                    % (WF_FLOPS_PER_BIN, PROJ_FLOPS_PER_DET_BIN, ev.nifo, B, bins)},
        "clocks": clocks,
        "fp64_batched": {"value": fp64_rate, "unit": "lnL evals/s", "ms_per_step": float(np.mean(ms64))},
        "fp64_per_call_dropin": percall,
        "mixed_vs_fp64_per_call": value / percall_rate / world,
        "mixed_vs_fp64_batched": value / fp64_rate / world,
        "max_abs_dlnL_mixed_vs_fp64": dmax,
    }
    if rank == 0 and world == 1 and not args.no_extra:
        from quickcbc_b200 import engine as eng
        out["config1_per_call"] = bench_cfg1_percall(q, eng, _lib)
        out["config3"] = bench_cfg3_het(q)
        out["config4_uneven"] = bench_cfg4_uneven(q)
        # the HBM-streaming case: the config-4 launch with the sets interleaved across all 256 events
        st = out["config4_uneven"]["mixed_interleaved"]
        tr, ti = capture_traffic("k_lnl_multi_cfg4", "k_lnl_multi", None, None, st["ms"])
        out["roofline_stream"] = {
            "bound": "hbm", "achieved": st["achieved_GBs"], "peak": hbm_peak, "unit": "GB/s",
            "frac": st["frac_hbm"], "traffic": tr, "peak_kind": peak_kind, "kernel": "k_lnl_multi (mixed)",
            "kernel_ms": st["ms"], "bytes_per_launch": st["stream_bytes"], **ti,
            "note": "config 4, 65536 sets interleaved across 256 events (1-3 detectors): useful bytes = "
                    "12 B (FP32 wr, wi, ws) per detector-bin of every set's band; the waveform's bin factor "
                    "is folded into those values, so no per-bin table is streamed"}
        out["input_stage"] = bench_input_stage(q)
        # config 5 as specified (32 runs of 16 x 8 chains x 20000 steps, Poisson 2/s): mixed against
        # plain FP64, heterodyned and full likelihood, chains stepped on the device
        out["config5_serving"] = bench_cfg5_serving(q, n_runs=32, n_steps=20000, rate_hz=2.0,
                                                    precisions=("mixed-het-dev", "fp64-het-dev", "mixed-dev",
                                                                "fp64-dev"))
        # the same service saturated (every run submitted at t = 0), so that the GPU, not the
        # arrival stream, sets the pace: host-stepped and device-stepped, mixed and FP64
        out["config5_serving_saturated"] = bench_cfg5_serving(q, n_runs=16, n_steps=1000, rate_hz=None,
                                                              precisions=("mixed", "fp64", "mixed-dev", "fp64-dev",
                                                                          "mixed-het-dev", "fp64-het-dev"))
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline_reference(ev, P)
    if rank == 0:
        print(json.dumps(out), flush=True)
    e.close()
    rep.close()


if __name__ == "__main__":
    main()

"""Generate the golden fixtures in tests/golden/ by running the QuickCBC
reference itself (oracle/_ref/libqcbc_ref.so: the reference C compiled
unmodified from its sources) on seeded synthetic inputs.

The reference ships no golden vectors or known-answer tests, so these
fixtures pin the CPU oracle and the CUDA kernels on machines where the
reference tree is absent.  Regenerate with:

    make -C oracle ref && python tests/golden/make_golden.py [wave cfg1 het1 grid3 spread3 secondary1 ingest1]

Contents (float64 unless noted):
  wave.npz     amp/phase of IMRPhenomDGenerateh22FDAmpPhase for 6 systems on a
               log-spaced frequency list; fbegin; F+/Fx and delays per detector
  cfg1.npz     config-1 event (H1/L1, 4 s, 2048 Hz): D, SN, GMST, injection,
               16 parameter sets, reference lnL and rho, two full templates
  het1.npz     reference heterodyne grid (het_space) and tables for config 1,
               reference het lnL at 16 nearby parameter sets
  grid3.npz    reference heterodyne grid for config 3 (3 det, 128 s, 4096 Hz)
  spread3.npz  config 3 away from the peak: 48 sets about the injection whose lnL lies
               0.5-10, 10-60 and 100-400 below it (posterior width to burn-in), with the
               reference's heterodyned, full and exact (log_likelihood_test) lnL of each
  secondary1.npz  config 1: templates and log_likelihood_intrinsic on intrinsic-layout
               parameter sets, AmpPhase, and het_diff / Fisher_Het on the reference's
               heterodyne tables of het1.npz's grid
  ingest1.npz  config-1 input stage: time series x whose conditioned data (the reference's
               tukey + real FFT + sqrt(Tobs)/N) are D; the spec-file PSD SN as read back from
               its %.15e text; a 3-sample spline-plus-lines PSD model and the reference's
               makespec of every sample and detector; reference lnL on (D, SN) and on
               (D, makespec sample 1)
"""
from __future__ import annotations

import os
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import ref  # noqa: E402
from quickcbc_b200 import synth  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))
MSUN, PC = synth.MSUN_SI, synth.PC_SI


def ref_template_factory():
    nets = {}

    def t(info, p):
        key = (tuple(int(x) for x in info["labels"]), info["Tobs"], info["GMST"])
        if key not in nets:
            nets[key] = ref.RefNet(info["labels"], info["Tobs"], info["GMST"])
        return ref.fulltemplates(nets[key], info["freq"], p, info["N"])
    return t


def prior_bounds(Tobs):
    # MCMC_all's prior box (QuickCBC.c:1871-1896, ConstCBC.h:48-57)
    pmin = np.array([np.log(0.5 * MSUN), np.log(0.5 * MSUN), -0.85, -0.85, 0.0, max(Tobs - 3.5, 1.5),
                     np.log(1e6 * PC), 0.0, -1.0, 0.0, -1.0])
    pmax = np.array([np.log(160 * MSUN), np.log(300 * MSUN), 0.85, 0.85, 2 * np.pi, Tobs - 0.5,
                     np.log(1e10 * PC), 2 * np.pi, 1.0, np.pi, 1.0])
    return pmin, pmax


def band_psd(ev):
    """PSD rows for the reference compiled with fmin = 16 Hz: bins below the
    event's fmin get an infinite PSD, so they add exactly 0 to every sum."""
    S = ev.SN.copy()
    S[:, int(16.0 * ev.Tobs):int(ev.fmin * ev.Tobs)] = np.inf
    return S


def make_wave():
    rng = np.random.default_rng(11)
    freq = np.geomspace(8.0, 2048.0, 700)
    systems = [(36.0, 29.0, 0.3, -0.1), (1.45, 1.30, 0.03, -0.02), (80.0, 10.0, 0.8, -0.5),
               (10.0, 8.0, -0.9, 0.9), (150.0, 120.0, 0.5, 0.5), (5.0, 1.4, 0.0, 0.0)]
    amps, phases, meta = [], [], []
    for (m1, m2, c1, c2) in systems:
        phi0 = rng.uniform(0, np.pi)
        dist = 400e6 * PC
        a, p = ref.amp_phase(freq, phi0, 100.0, m1 * MSUN, m2 * MSUN, c1, c2, dist)
        amps.append(a)
        phases.append(p)
        meta.append([phi0, 100.0, m1 * MSUN, m2 * MSUN, c1, c2, dist])
    P = synth.draw_params(rng, 8, np.array([0, 0, 0, 0, 0, 14.0, np.log(400e6 * PC), 0, 0, 0, 0]))
    fb = np.array([ref.fbegin(p) for p in P])
    ang = rng.uniform(size=(12, 4)) * np.array([np.pi, 2 * np.pi, 2.0, 2 * np.pi]) - np.array([0, 0, 1.0, 0])
    ant = np.array([[ref.F_ant(a[0], a[1], a[2], a[3], k) for k in range(3)] for a in ang])
    dts = np.array([ref.Times(a[1], a[2], a[3]) for a in ang])
    np.savez_compressed(os.path.join(OUT, "wave.npz"), freq=freq, amp=np.array(amps), phase=np.array(phases),
                        meta=np.array(meta), fb_params=P, fbegin=fb, ant_angles=ang, antenna=ant, delays=dts)


def make_cfg1():
    ev = synth.config_event(1, ref_template_factory())
    net = ref.RefNet(ev.labels, ev.Tobs, ev.GMST)
    rng = np.random.default_rng(1500)
    P = np.vstack([synth.jitter_params(rng, 8, ev.inj), synth.draw_params(rng, 8, ev.inj)])
    L, _ = ref.lnl_full_batch(net, ev.D, P, ev.freq, ev.SN, ev.N, ev.Tobs)
    rho = np.array([ref.lnl_full(net, ev.D, p, ev.freq, ev.SN, ev.N, ev.Tobs)[1] for p in P])
    H = np.array([ref.fulltemplates(net, ev.freq, P[k], ev.N) for k in (0, 9)])
    A, PH = ref.fullphaseamp(net, ev.freq, P[0], ev.N)
    np.savez_compressed(os.path.join(OUT, "cfg1.npz"), labels=ev.labels, Tobs=ev.Tobs, fs=ev.fs, N=ev.N,
                        fmin=ev.fmin, GMST=ev.GMST, D=ev.D, SN=ev.SN, inj=ev.inj, params=P, lnl=L, rho=rho,
                        h=H, h_idx=np.array([0, 9]), pa_amp=A, pa_phase=PH)
    return ev, net


def make_het1(ev, net):
    pmin, pmax = prior_bounds(ev.Tobs)
    het = ref.RefHet(net)
    with tempfile.TemporaryDirectory() as d:
        het.space(ev.inj, pmin, pmax, ev.freq, ev.SN, ev.N, ev.Tobs, d)
    het.heterodyne(ev.D, ev.inj, ev.freq, ev.SN, ev.N, ev.Tobs)
    t = het.export()
    rng = np.random.default_rng(1600)
    P = synth.jitter_params(rng, 16, ev.inj, scale=1e-4)
    L, _ = het.lnl_batch(P, ev.Tobs)
    Lt = np.array([het.lnl_test(ev.D, p, ev.freq, ev.SN, ev.N, ev.Tobs) for p in P])
    np.savez_compressed(os.path.join(OUT, "het1.npz"), params=P, lnl=L, lnl_exact=Lt, pref=ev.inj,
                        **{k: v for k, v in t.items()})


def make_grid3():
    ev = synth.config_event(3, ref_template_factory())
    net = ref.RefNet(ev.labels, ev.Tobs, ev.GMST)
    S = band_psd(ev)
    pmin, pmax = prior_bounds(ev.Tobs)
    het = ref.RefHet(net)
    with tempfile.TemporaryDirectory() as d:
        het.space(ev.inj, pmin, pmax, ev.freq, S, ev.N, ev.Tobs, d)
    z = het.sizes()
    het.heterodyne(ev.D, ev.inj, ev.freq, S, ev.N, ev.Tobs)
    t = het.export()
    rng = np.random.default_rng(3600)
    P = synth.jitter_params(rng, 8, ev.inj, scale=1e-6)
    L, _ = het.lnl_batch(P, ev.Tobs)
    np.savez_compressed(os.path.join(OUT, "grid3.npz"), fgrid=t["fgrid"], MN=z["MN"], MM=z["MM"], J=z["J"],
                        logLb=t["logLb"], params=P, lnl=L, inj=ev.inj, GMST=ev.GMST)


def make_spread3():
    """Config 3 away from the peak.  Reference heterodyne tables on grid3's grid about the
    injection, the reference's Fisher_Het there, and 48 sets from synth.cloud_at_drops (Fisher
    steps, distance along each searched on the reference's heterodyned lnL) at lnL drops drawn
    from U[0.5, 10] (chains at the posterior's width), U[10, 60] and U[100, 400] (burn-in), 16
    each.  For each set the reference's log_likelihood_het, log_likelihood_full and
    log_likelihood_test (the heterodyned lnL evaluated exactly from differenced full templates,
    QuickCBC.c:5621-5667)."""
    g = np.load(os.path.join(OUT, "grid3.npz"))
    ev = synth.config_event(3, ref_template_factory())
    net = ref.RefNet(ev.labels, ev.Tobs, ev.GMST)
    S = band_psd(ev)
    het = ref.RefHet(net)
    het.set_grid(g["fgrid"], int(g["MN"]), int(g["MM"]), int(g["J"]), ev.Tobs)
    het.heterodyne(ev.D, ev.inj, ev.freq, S, ev.N, ev.Tobs)
    F = het.fisher(ev.inj, ev.Tobs)
    rng = np.random.default_rng(3700)
    ranges = np.array([[0.5, 10.0], [10.0, 60.0], [100.0, 400.0]])
    drops = np.concatenate([rng.uniform(lo, hi, 16) for lo, hi in ranges])
    group = np.repeat(np.arange(len(ranges)), 16).astype(np.int32)
    P = synth.cloud_at_drops(rng, ev.inj, F, drops, lambda X: het.lnl_batch(X, ev.Tobs)[0])
    Lh, _ = het.lnl_batch(P, ev.Tobs)
    Lf, _ = ref.lnl_full_batch(net, ev.D, P, ev.freq, S, ev.N, ev.Tobs)
    Lt = np.array([het.lnl_test(ev.D, p, ev.freq, S, ev.N, ev.Tobs) for p in P])
    L0, _ = ref.lnl_full_batch(net, ev.D, ev.inj[None, :], ev.freq, S, ev.N, ev.Tobs)
    np.savez_compressed(os.path.join(OUT, "spread3.npz"), params=P, group=group, drop_ranges=ranges,
                        target_drops=drops, fisher=F, lnl_het=Lh, lnl_full=Lf, lnl_exact=Lt,
                        lnl_inj_full=float(L0[0]), inj=ev.inj, GMST=ev.GMST, logLb=het.export()["logLb"])
    for k, (lo, hi) in enumerate(ranges):
        m = group == k
        print("spread3 drops %g-%g: full lnL %.2f..%.2f (injection %.2f), |het-full| max %.3g, "
              "|het-exact| max %.3g" % (lo, hi, Lf[m].min(), Lf[m].max(), L0[0], np.abs(Lh[m] - Lf[m]).max(),
                                        np.abs(Lh[m] - Lt[m]).max()))


def intrinsic_equivalent(p, labels, GMST):
    """Intrinsic-layout parameters (QuickCBC.c:3570-3582) of the template that equals the full
    template of p (QuickCBC.c:3722-3760) in every detector: detector 0's response |F0|,
    polarisation phase lambda0 and delay td0 go into the distance, phase and merger time;
    detectors j > 0 get lambda_j - lambda0, td_j - td0 and |F_j| / |F0|."""
    alpha, sind, psi, ci = p[7], p[8], p[9], p[10]
    Ap, Ac = (1.0 + ci * ci) / 2.0, -ci
    dt = ref.Times(alpha, sind, GMST)
    Fs, lam, td = [], [], []
    for l in labels:
        fp, fx = ref.F_ant(psi, alpha, sind, GMST, int(l))
        Fs.append(np.sqrt(Ap * Ap * fp * fp + Ac * Ac * fx * fx))
        lam.append(np.mod(np.arctan2(Ac * fx, Ap * fp), 2 * np.pi))
        td.append(dt[int(l)])
    q = [p[0], p[1], p[2], p[3], (p[4] + lam[0]) / 2.0, p[5] + td[0], p[6] - np.log(Fs[0])]
    for j in range(1, len(labels)):
        q += [lam[j] - lam[0], td[j] - td[0], Fs[j] / Fs[0]]
    return np.array(q)


def intrinsic_sets(rng, n, inj, labels, GMST):
    """Intrinsic-layout sets about the intrinsic equivalent of the injection; the last two are
    far away (fewer than two detectors with SNR^2 > 25, so the reference returns 0)."""
    c = intrinsic_equivalent(inj, labels, GMST)
    P = np.tile(c, (n, 1))
    P[:, 0] += 1e-4 * rng.normal(size=n)
    P[:, 1] += 1e-3 * rng.normal(size=n)
    P[:, 2:4] = np.clip(P[:, 2:4] + 1e-2 * rng.normal(size=(n, 2)), -0.95, 0.95)
    P[:, 4] += 0.05 * rng.normal(size=n)
    P[:, 5] += 1e-4 * rng.normal(size=n)
    P[:, 6] += 0.05 * rng.normal(size=n)
    P[:, 7:] += np.array([0.05, 1e-4, 0.05]) * rng.normal(size=(n, 3))
    P[n - 2:, 6] += np.log(50.0)
    return P


def make_secondary1():
    ev = synth.config_event(1, ref_template_factory())
    net = ref.RefNet(ev.labels, ev.Tobs, ev.GMST)
    rng = np.random.default_rng(1700)
    PI = intrinsic_sets(rng, 8, ev.inj, ev.labels, ev.GMST)
    L = np.array([ref.lnl_intrinsic(net, ev.D, p, ev.freq, ev.SN, ev.N, ev.Tobs) for p in PI])
    H = np.array([ref.templates(net, ev.freq, PI[k], ev.N) for k in (0, 5)])
    PA = synth.jitter_params(rng, 2, ev.inj, scale=1e-2)
    AP = [ref.AmpPhase(ev.freq, p, ev.N) for p in PA]
    h1 = np.load(os.path.join(OUT, "het1.npz"))
    het = ref.RefHet(net)
    het.set_grid(h1["fgrid"], int(h1["MN"]), int(h1["MM"]), int(h1["J"]), ev.Tobs)
    het.heterodyne(ev.D, h1["pref"], ev.freq, ev.SN, ev.N, ev.Tobs)
    DA = synth.jitter_params(rng, 4, h1["pref"], scale=1e-4)
    DB = synth.jitter_params(rng, 4, h1["pref"], scale=1e-4)
    dif = np.array([het.het_diff(a, b) for a, b in zip(DA, DB)])
    FP = np.vstack([h1["pref"], synth.jitter_params(rng, 1, h1["pref"], scale=1e-4)])
    fish = np.array([het.fisher(p, ev.Tobs) for p in FP])
    np.savez_compressed(os.path.join(OUT, "secondary1.npz"), int_params=PI, int_lnl=L, int_h=H,
                        int_h_idx=np.array([0, 5]), ap_params=PA, ap_amp=np.array([a for a, _ in AP]),
                        ap_phase=np.array([p for _, p in AP]), diff_a=DA, diff_b=DB, diff=dif, fisher_params=FP,
                        fisher=fish)


def make_ingest1():
    ev = synth.config_event(1, ref_template_factory())
    net = ref.RefNet(ev.labels, ev.Tobs, ev.GMST)
    x = synth.time_series(ev)
    D = np.array([ref.condition(xi, ev.Tobs) for xi in x])
    nh = ev.N // 2
    # the spec file's PSD column as the reference reads it back (%.15e text)
    SN = np.array([[float("%.15e" % v) for v in row[:nh]] for row in ev.SN])
    ns, nl, ffit, xs, L = synth.psd_model_arrays(np.random.default_rng(1800), len(ev.labels), ev.Tobs, ev.N)
    S = np.zeros((xs.shape[1], len(ev.labels), nh))
    for k in range(xs.shape[1]):
        for i in range(len(ev.labels)):
            n, m = ns[i], nl[i]
            S[k, i] = ref.makespec(ffit[i, :n], xs[i, k, :n], L[i, k, :m, 0], L[i, k, :m, 1], L[i, k, :m, 2],
                                   L[i, k, :m, 3], L[i, k, :m, 4], ev.Tobs, ev.N)
    P = synth.jitter_params(np.random.default_rng(1801), 6, ev.inj)
    lnl = np.array([ref.lnl_full(net, D, p, ev.freq, SN, ev.N, ev.Tobs)[0] for p in P])
    lnl_s1 = np.array([ref.lnl_full(net, D, p, ev.freq, S[1], ev.N, ev.Tobs)[0] for p in P])
    np.savez_compressed(os.path.join(OUT, "ingest1.npz"), labels=ev.labels, Tobs=ev.Tobs, N=ev.N, fmin=ev.fmin,
                        GMST=ev.GMST, inj=ev.inj, x=x, D=D, SN=SN, nspline=ns, nlines=nl, ffit=ffit, xspline=xs,
                        lines=L, makespec=S, params=P, lnl=lnl, lnl_sample1=lnl_s1)


if __name__ == "__main__":
    which = set(sys.argv[1:]) or {"wave", "cfg1", "het1", "grid3", "spread3", "secondary1", "ingest1"}
    if "wave" in which:
        make_wave()
    if which & {"cfg1", "het1"}:
        ev, net = make_cfg1()
        if "het1" in which:
            make_het1(ev, net)
    if "grid3" in which:
        make_grid3()
    if "spread3" in which:
        make_spread3()
    if "secondary1" in which:
        make_secondary1()
    if "ingest1" in which:
        make_ingest1()
    for f in sorted(os.listdir(OUT)):
        if f.endswith(".npz"):
            print(f, os.path.getsize(os.path.join(OUT, f)))

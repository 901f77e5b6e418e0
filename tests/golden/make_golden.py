"""Generate the golden fixtures in tests/golden/ by running the QuickCBC
reference itself (oracle/_ref/libqcbc_ref.so: the reference C compiled
unmodified from its sources) on seeded synthetic inputs.

The reference ships no golden vectors or known-answer tests, so these
fixtures pin the CPU oracle and the CUDA kernels on machines where the
reference tree is absent.  Regenerate with:

    make -C oracle ref && python tests/golden/make_golden.py

Contents (float64 unless noted):
  wave.npz     amp/phase of IMRPhenomDGenerateh22FDAmpPhase for 6 systems on a
               log-spaced frequency list; fbegin; F+/Fx and delays per detector
  cfg1.npz     config-1 event (H1/L1, 4 s, 2048 Hz): D, SN, GMST, injection,
               16 parameter sets, reference lnL and rho, two full templates
  het1.npz     reference heterodyne grid (het_space) and tables for config 1,
               reference het lnL at 16 nearby parameter sets
  grid3.npz    reference heterodyne grid for config 3 (3 det, 128 s, 4096 Hz)
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


if __name__ == "__main__":
    make_wave()
    ev, net = make_cfg1()
    make_het1(ev, net)
    make_grid3()
    for f in sorted(os.listdir(OUT)):
        if f.endswith(".npz"):
            print(f, os.path.getsize(os.path.join(OUT, f)))

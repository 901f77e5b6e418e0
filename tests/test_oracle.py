"""CPU oracle (oracle/qcbc_oracle.c) pinned against the reference's outputs:
the committed golden fixtures (made by running the reference, see
tests/golden/make_golden.py) and, where it is built, the reference library
itself on fresh seeded inputs."""
import numpy as np
import pytest

from quickcbc_b200 import synth
from conftest import GoldenEvent, oracle_template


def test_amp_phase_vs_golden(ora, golden):
    z = golden("wave.npz")
    for k, m in enumerate(z["meta"]):
        a, p = ora.amp_phase(z["freq"], *m)
        ar, pr = z["amp"][k], z["phase"][k]
        nz = ar != 0
        assert np.array_equal(nz, a != 0), "fCut cut-off must match bin for bin"
        np.testing.assert_allclose(a[nz], ar[nz], rtol=1e-12)
        np.testing.assert_allclose(p, pr, rtol=0, atol=1e-9 * max(1.0, np.abs(pr).max()))


def test_fbegin_antenna_delays_vs_golden(ora, golden):
    z = golden("wave.npz")
    fb = np.array([ora.fbegin(p) for p in z["fb_params"]])
    np.testing.assert_allclose(fb, z["fbegin"], rtol=1e-14)
    for a, ant, dt in zip(z["ant_angles"], z["antenna"], z["delays"]):
        for k in range(3):
            np.testing.assert_allclose(ora.antenna(a[0], a[1], a[2], a[3], k), ant[k], rtol=1e-13, atol=1e-15)
        np.testing.assert_allclose(ora.delays(a[1], a[2], a[3]), dt, rtol=1e-14, atol=1e-18)


def test_lnl_full_vs_golden(ora, cfg1_event):
    ev, z = cfg1_event
    L, _ = ora.lnl_full_batch(ev, z["params"])
    np.testing.assert_allclose(L, z["lnl"], rtol=0, atol=1e-8)
    for k, p in enumerate(z["params"]):
        Lk, rho = ora.lnl_full(ev, p)
        np.testing.assert_allclose(rho, z["rho"][k], rtol=1e-10)


def test_templates_vs_golden(ora, cfg1_event):
    ev, z = cfg1_event
    for H, k in zip(z["h"], z["h_idx"]):
        h = ora.fulltemplates(ev.labels, ev.GMST, ev.freq, z["params"][k], ev.N)
        np.testing.assert_allclose(h, H, rtol=0, atol=1e-11 * np.abs(H).max())
    a, p = ora.fullphaseamp(ev.labels, ev.GMST, ev.Tobs, ev.freq, z["params"][0], ev.N)
    np.testing.assert_allclose(a, z["pa_amp"], rtol=1e-12, atol=1e-40)
    np.testing.assert_allclose(p, z["pa_phase"], rtol=0, atol=1e-9 * np.abs(z["pa_phase"]).max())


def test_heterodyne_vs_golden(ora, cfg1_event, golden):
    ev, _ = cfg1_event
    h = golden("het1.npz")
    t = ora.heterodyne(ev, h["pref"], h["fgrid"], int(h["MN"]), int(h["MM"]), int(h["J"]))
    assert abs(t["logLb"] - float(h["logLb"])) < 1e-9
    for k in ("amp", "phase", "IP", "SL", "lc", "ls", "aa", "rc", "rs"):
        scale = np.abs(h[k]).max()
        np.testing.assert_allclose(t[k], h[k], rtol=0, atol=1e-11 * scale, err_msg=k)
    L, _ = ora.lnl_het_batch(ev, t, h["params"])
    np.testing.assert_allclose(L, h["lnl"], rtol=0, atol=1e-8)


def test_het_consistency_with_exact(golden):
    """The reference's own self-check (log_likelihood_test, QuickCBC.c:5621):
    near the reference point the heterodyned lnL tracks the exact one."""
    h = golden("het1.npz")
    assert np.max(np.abs(h["lnl"] - h["lnl_exact"])) < 0.05


def test_oracle_vs_reference_fresh_inputs(ora, refo):
    """Fresh seeds (not in the fixtures) through both the oracle and the reference."""
    ev = synth.make_event(oracle_template(ora), labels=[2, 0], Tobs=8.0, fs=2048.0, fmin=16.0, m1=12.0, m2=7.0,
                          chi1=-0.4, chi2=0.6, snr=15.0, seed=77)
    net = refo.RefNet(ev.labels, ev.Tobs, ev.GMST)
    rng = np.random.default_rng(78)
    P = np.vstack([synth.jitter_params(rng, 6, ev.inj), synth.draw_params(rng, 10, ev.inj, mc=(4.0, 40.0))])
    Lr, _ = refo.lnl_full_batch(net, ev.D, P, ev.freq, ev.SN, ev.N, ev.Tobs)
    Lo, _ = ora.lnl_full_batch(ev, P)
    np.testing.assert_allclose(Lo, Lr, rtol=0, atol=1e-8)
    for p in P[:4]:
        ar, pr = refo.fullphaseamp(net, ev.freq, p, ev.N)
        ao, po = ora.fullphaseamp(ev.labels, ev.GMST, ev.Tobs, ev.freq, p, ev.N)
        np.testing.assert_allclose(ao, ar, rtol=1e-12, atol=1e-40)
        np.testing.assert_allclose(po, pr, rtol=0, atol=1e-9 * np.abs(pr).max())


def test_oracle_band_emulation(ora, refo):
    """The reference is compiled with fmin = 16 Hz; an infinite PSD below the
    configured fmin gives the reference the oracle's fmin = 20 Hz band."""
    ev = synth.make_event(oracle_template(ora), labels=[0, 1, 2], Tobs=4.0, fs=2048.0, fmin=20.0, m1=30.0,
                          m2=20.0, chi1=0.1, chi2=0.2, snr=12.0, seed=91)
    net = refo.RefNet(ev.labels, ev.Tobs, ev.GMST)
    S = ev.SN.copy()
    S[:, int(16 * ev.Tobs):int(20 * ev.Tobs)] = np.inf
    P = synth.draw_params(np.random.default_rng(92), 8, ev.inj)
    Lr, _ = refo.lnl_full_batch(net, ev.D, P, ev.freq, S, ev.N, ev.Tobs)
    Lo, _ = ora.lnl_full_batch(ev, P)
    np.testing.assert_allclose(Lo, Lr, rtol=0, atol=1e-8)


def test_golden_event_rebuilds(cfg1_event):
    ev, z = cfg1_event
    assert isinstance(ev, GoldenEvent)
    assert ev.D.shape == (2, 8192) and ev.SN.shape == (2, 4097)
    # noise normalisation: <n|n>/bins ~ 2 away from the signal band edges
    i = np.arange(ev.N // 4, ev.N // 2 - 1)
    r = 4 * (ev.D[0, i] ** 2 + ev.D[0, ev.N - i] ** 2) / ev.SN[0, i]
    assert 1.8 < r.mean() < 2.2

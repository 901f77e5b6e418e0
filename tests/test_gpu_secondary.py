"""Secondary reference-signature entry points (QuickCBC.h:95-151) against the
reference's own outputs (tests/golden/secondary1.npz, made by running the
reference): templates, log_likelihood_intrinsic, AmpPhase, het_diff and
Fisher_Het, plus their batched C-ABI forms.

Tolerances:
  FP64 waveform outputs   1e-11 of the largest |h| (templates), 1e-12 relative (AmpPhase amp),
                          1e-9 of the largest |phase| (AmpPhase phase)
  FP64 likelihoods        1e-8 absolute (intrinsic lnL), 1e-9 relative (het_diff)
  mixed likelihoods       1e-3 absolute
  Fisher_Het              1e-6 of sqrt(F_ii F_jj) per entry (central differences with step 1e-5)
"""
import numpy as np
import pytest

import quickcbc_b200 as q

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def sec(golden):
    return golden("secondary1.npz")


@pytest.fixture(scope="module")
def ev1(cfg1_event):
    ev, z = cfg1_event
    e = q.Event.from_synthetic(ev)
    yield ev, e
    e.close()


def test_templates_vs_reference(ev1, sec):
    ev, _ = ev1
    for H, k in zip(sec["int_h"], sec["int_h_idx"]):
        h = q.templates(ev.labels, ev.GMST, ev.freq, sec["int_params"][k], ev.N)
        np.testing.assert_allclose(h, H, rtol=0, atol=1e-11 * np.abs(H).max())


def test_lnl_intrinsic_vs_reference(ev1, sec):
    ev, e = ev1
    Lref = sec["int_lnl"]
    assert np.count_nonzero(Lref == 0.0) == 2 and np.all(Lref[:6] > 200), "fixture covers both branches of the rule"
    L = np.array([q.log_likelihood_intrinsic(ev.labels, ev.GMST, ev.D, p, ev.freq, ev.SN, ev.N, ev.Tobs)
                  for p in sec["int_params"]])
    np.testing.assert_allclose(L, Lref, rtol=0, atol=1e-8)
    Lb, snr2 = e.lnl_intrinsic(sec["int_params"], q.FP64, snrsq=True)
    np.testing.assert_allclose(Lb, Lref, rtol=0, atol=1e-8)
    loud = (snr2 > 25.0).sum(axis=1)
    assert np.array_equal(Lref == 0.0, loud < 2)
    Lm = e.lnl_intrinsic(sec["int_params"], q.MIXED)
    np.testing.assert_allclose(Lm, Lref, rtol=0, atol=1e-3)


def test_lnl_intrinsic_large_batch_ordered_launch(ev1, sec):
    """At one tile per set (B >= 1184) the intrinsic model runs in the length-ordered launch, with
    the two-detector rule applied in the lnL kernel: lnL and SNR^2 equal the multi-tile launch's
    and the fixture's for the sets it holds."""
    _, e = ev1
    base = sec["int_params"]
    P = np.tile(base, (1500 // len(base) + 1, 1))[:1500].copy()
    P[:, 6] += np.linspace(-0.01, 0.01, len(P))          # spread the sets' time offsets
    assert e.get_launch(len(P), q.FP64)[0] == 1
    L, S = e.lnl_intrinsic(P, q.FP64, snrsq=True)
    e.set_launch(4, 256)
    Lu, Su = e.lnl_intrinsic(P, q.FP64, snrsq=True)
    e.set_launch(0, 0)
    np.testing.assert_allclose(L, Lu, rtol=0, atol=1e-9)
    np.testing.assert_allclose(S, Su, rtol=1e-9, atol=1e-9)
    Lf = e.lnl_intrinsic(base, q.FP64)
    np.testing.assert_allclose(e.lnl_intrinsic(np.vstack([base, P]), q.FP64)[:len(base)], Lf, rtol=0, atol=1e-9)


def test_lnl_intrinsic_rejects_wrong_layout(ev1, sec):
    _, e = ev1
    with pytest.raises(ValueError):
        e.lnl_intrinsic(sec["int_params"][:, :9])


def test_ampphase_vs_reference(ev1, sec):
    ev, _ = ev1
    for p, Ar, Pr in zip(sec["ap_params"], sec["ap_amp"], sec["ap_phase"]):
        Af, Pf = q.ampphase(ev.freq, p, ev.N)
        np.testing.assert_allclose(Af[1:], Ar[1:], rtol=1e-12, atol=1e-40)
        np.testing.assert_allclose(Pf[1:], Pr[1:], rtol=0, atol=1e-9 * np.abs(Pr).max())


@pytest.fixture(scope="module")
def het1(ev1, golden):
    ev, _ = ev1
    h = golden("het1.npz")
    H = q.LegacyHet(ev.labels, ev.GMST, ev.Tobs, h["fgrid"], int(h["MN"]), int(h["MM"]), int(h["J"]))
    H.heterodyne(ev.D, h["pref"], ev.freq, ev.SN, ev.N)
    return H


def test_het_diff_vs_reference(het1, sec):
    d = np.array([het1.het_diff(a, b) for a, b in zip(sec["diff_a"], sec["diff_b"])])
    np.testing.assert_allclose(d, sec["diff"], rtol=1e-9, atol=0)
    assert het1.het_diff(sec["diff_a"][0], sec["diff_a"][0]) == 0.0


def fisher_close(F, G):
    s = np.sqrt(np.outer(np.diag(G), np.diag(G)))
    assert np.all(np.abs(F - G) <= 1e-6 * s), np.max(np.abs(F - G) / s)


def test_fisher_het_vs_reference(het1, sec):
    for p, G in zip(sec["fisher_params"], sec["fisher"]):
        F = het1.fisher(p)
        assert np.array_equal(F, F.T)
        fisher_close(F, G)


def test_batched_het_forms_match_drop_ins(ev1, het1, sec):
    _, e = ev1
    e.het_set(het1.tables())
    F = e.het_fisher(sec["fisher_params"])
    for k, G in enumerate(sec["fisher"]):
        fisher_close(F[k], G)
    d = e.het_diff(sec["diff_a"], sec["diff_b"])
    np.testing.assert_allclose(d, sec["diff"], rtol=1e-9, atol=0)
    # near-extremal spins: the reference's fallback matrix
    p = sec["fisher_params"][0].copy()
    p[2] = 0.99995
    F1 = e.het_fisher(p)[0]
    assert np.array_equal(F1, np.diag(np.full(11, 1.0e4)))


def test_sky_ring_map_vs_reference(ev1):
    """The sky-ring proposal map (update, QuickCBC.c:2299-2331) against the reference's skymap_all and
    skydensity_all at the sky position the GPU ring rotation gives: extrinsic parameters 1e-8;
    log Jacobian 1e-4 (one-sided differences of step 1e-6 turn last-bit differences of the map into
    ~1e-10 per entry, which cancellation in a small determinant amplifies); the rotation keeps the
    two detectors' time delay."""
    ref = pytest.importorskip("oracle.ref")
    ev, _ = ev1
    rng = np.random.default_rng(2299)
    for l1, l2 in [(0, 1), (1, 0), (0, 2), (2, 1)]:
        for _ in range(6):
            x = ev.inj.copy()
            x[4], x[9] = rng.uniform(0, 2 * np.pi), rng.uniform(0, np.pi)
            x[7], x[8], x[10] = rng.uniform(0, 2 * np.pi), rng.uniform(-0.9, 0.9), rng.uniform(-0.9, 0.9)
            y, lj = q.sky_ring_map(x, ev.GMST, l1, l2, rng.uniform(0, 2 * np.pi))
            tx, ty = ref.Times(x[7], x[8], ev.GMST), ref.Times(y[7], y[8], ev.GMST)
            assert abs((tx[l1] - tx[l2]) - (ty[l1] - ty[l2])) < 1e-12
            yr = x.copy()
            yr[7], yr[8] = y[7], y[8]
            yr = ref.skymap_all(x, yr, ev.GMST, l1, l2)
            np.testing.assert_allclose(y[[4, 5, 6, 9, 10]], yr[[4, 5, 6, 9, 10]], rtol=0, atol=1e-8)
            J = ref.skydensity_all(x, yr, ev.GMST, l1, l2)
            assert abs(lj - np.log(J)) < 1e-4


def test_sky_ring_keeps_two_detector_likelihood(ev1):
    """On an H1/L1 event the moved point gives both detectors the same signal, so the same lnL: within
    1e-4, since the map carries ~1e-8 of FP64 rounding in ln D (cancellations in the inclination
    solve) and lnL moves by about SNR^2 times that; a wrong map moves lnL by units."""
    ev, e = ev1
    assert list(ev.labels) == [0, 1]
    rng = np.random.default_rng(2300)
    X, Y = [], []
    for _ in range(8):
        x = ev.inj.copy()
        x[7] = (x[7] + rng.uniform(-0.3, 0.3)) % (2 * np.pi)
        y, _ = q.sky_ring_map(x, ev.GMST, 0, 1, rng.uniform(0, 2 * np.pi))
        y[4] %= 2 * np.pi
        y[7] %= 2 * np.pi
        y[9] %= np.pi
        X.append(x)
        Y.append(y)
    Lx = e.lnl_full(np.array(X), q.FP64)
    Ly = e.lnl_full(np.array(Y), q.FP64, allow_invalid=True)
    ok = Ly > -1e19
    assert ok.sum() >= 6
    np.testing.assert_allclose(Ly[ok], Lx[ok], rtol=0, atol=1e-4)

"""Config 3 (3 det, 128 s, 4096 Hz, BNS 1.45 + 1.30, SNR 30) away from the peak, where
sampler chains actually sit.  The 48 sets of tests/golden/spread3.npz lie 0.5-10, 10-60 and
100-400 below the injection's lnL (posterior width to burn-in); the fixture holds the
reference's log_likelihood_het, log_likelihood_full and log_likelihood_test for each.

The mixed-precision heterodyned lnL forms hc, hs from a phase difference reduced in FP64 and
an FP32 sine (QuickCBC.c:5335-5425 in FP64): these sets exercise that difference across the
posterior's width and beyond, not only at the reference point.

Tolerances (written per test): FP64 within 1e-6 absolute of the reference (lnL ~ 60-440; libm
and CUDA transcendentals round differently), mixed within 1e-3 (the stated target).
"""
import numpy as np
import pytest

import quickcbc_b200 as q
from quickcbc_b200 import synth
from conftest import load_golden, oracle_template

pytestmark = pytest.mark.gpu

ATOL_FP64 = 1e-6
ATOL_MIXED = 1e-3


@pytest.fixture(scope="module")
def cfg3(ora):
    z = load_golden("spread3.npz")
    g = load_golden("grid3.npz")
    ev = synth.config_event(3, oracle_template(ora))
    assert ev.GMST == float(z["GMST"]) and np.array_equal(ev.inj, z["inj"])
    e = q.Event.from_synthetic(ev)
    e.het_setup(ev.inj, g["fgrid"], int(g["MN"]), int(g["MM"]), int(g["J"]))
    yield ev, z, g, e
    e.close()


def _per_group(z, d):
    return {int(k): float(np.abs(d[z["group"] == k]).max()) for k in np.unique(z["group"])}


def test_spread3_heterodyned_vs_reference(cfg3):
    ev, z, g, e = cfg3
    P = z["params"]
    L64 = e.lnl_het(P, q.FP64)
    np.testing.assert_allclose(L64, z["lnl_het"], rtol=0, atol=ATOL_FP64)
    Lm = e.lnl_het(P, q.MIXED)
    worst = _per_group(z, Lm - z["lnl_het"])
    assert max(worst.values()) <= ATOL_MIXED, worst


def test_spread3_full_vs_reference(cfg3):
    ev, z, g, e = cfg3
    P = z["params"]
    L64 = e.lnl_full(P, q.FP64)
    np.testing.assert_allclose(L64, z["lnl_full"], rtol=0, atol=ATOL_FP64)
    Lm = e.lnl_full(P, q.MIXED)
    worst = _per_group(z, Lm - z["lnl_full"])
    assert max(worst.values()) <= ATOL_MIXED, worst


def test_spread3_heterodyne_vs_exact(cfg3):
    """The counterpart of the reference's log_likelihood_test (QuickCBC.c:5621-5667): the
    heterodyned lnL against the same quantity evaluated exactly.  That exact value is
    logLb - sum_ifo [<D - r|r - h> + <r - h|r - h>/2] over bins [MN, MM) with r the reference
    template; since logLb = sum_ifo <D|r> - <r|r>/2 over the same bins (QuickCBC.c:5169-5179) it
    equals the full lnL of h on the band [MN, MM), which the GPU computes on an event opened with
    that band.  Both the exact values and the heterodyne's error against them must be the
    reference's."""
    ev, z, g, e = cfg3
    MN, MM = int(g["MN"]), int(g["MM"])
    eb = q.Event(ev.labels, ev.Tobs, ev.GMST, ev.N, ev.D, ev.SN, fmin=(MN + 0.5) / ev.Tobs,
                 fmax=(MM + 0.5) / ev.Tobs)
    P = z["params"]
    X64 = eb.lnl_full(P, q.FP64)
    np.testing.assert_allclose(X64, z["lnl_exact"], rtol=0, atol=ATOL_FP64)
    Xm = eb.lnl_full(P, q.MIXED)
    assert np.max(np.abs(Xm - z["lnl_exact"])) <= ATOL_MIXED
    # the exact form at the reference point is logLb itself
    assert abs(eb.lnl_full(ev.inj, q.FP64)[0] - float(z["logLb"])) <= ATOL_FP64
    H64 = e.lnl_het(P, q.FP64)
    np.testing.assert_allclose(H64 - X64, z["lnl_het"] - z["lnl_exact"], rtol=0, atol=2 * ATOL_FP64)
    Hm = e.lnl_het(P, q.MIXED)
    assert np.max(np.abs((Hm - Xm) - (z["lnl_het"] - z["lnl_exact"]))) <= 2 * ATOL_MIXED
    eb.close()


def test_spread3_cloud_search_on_device(cfg3):
    """The bench's config-3 sets come from synth.cloud_at_drops driven by the GPU's heterodyned
    lnL and its batched Fisher_Het: the sets it returns lie at the requested drops, and their
    mixed lnL (heterodyned and full) stays within the target of FP64."""
    ev, z, g, e = cfg3
    F = e.het_fisher(ev.inj[None, :])[0]
    G = z["fisher"]                     # the reference's Fisher_Het on its own tables
    assert np.all(np.abs(F - G) <= 1e-4 * np.sqrt(np.outer(np.diag(G), np.diag(G))))
    rng = np.random.default_rng(3701)
    drops = np.concatenate([rng.uniform(0.5, 10.0, 64), rng.uniform(10.0, 60.0, 32), rng.uniform(100.0, 400.0, 32)])
    P = synth.cloud_at_drops(rng, ev.inj, F, drops, lambda X: e.lnl_het(X, q.FP64, allow_invalid=True))
    L64 = e.lnl_het(P, q.FP64)
    L0 = e.lnl_het(ev.inj[None, :], q.FP64)[0]
    np.testing.assert_allclose(L0 - L64, drops, rtol=1e-3, atol=1e-3)
    assert np.max(np.abs(e.lnl_het(P, q.MIXED) - L64)) <= ATOL_MIXED
    Pf = P[::4]
    assert np.max(np.abs(e.lnl_full(Pf, q.MIXED) - e.lnl_full(Pf, q.FP64))) <= ATOL_MIXED

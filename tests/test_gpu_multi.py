"""Many events in one launch (qcbc_lnl_multi): uneven networks, durations and
sample rates; parity with the single-event path and the CPU oracle, and each
set's result identical alone and in the mix."""
import numpy as np
import pytest

import quickcbc_b200 as q
from quickcbc_b200 import synth
from conftest import oracle_template, prior_bounds

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def uneven(ora):
    specs = synth.uneven_event_specs(n_events=10, seed=4100)
    evs = [synth.make_event(oracle_template(ora), **s) for s in specs]
    handles = [q.Event.from_synthetic(ev) for ev in evs]
    batch = q.Batch(handles)
    yield evs, handles, batch
    batch.close()
    for h in handles:
        h.close()


def test_specs_cover_the_uneven_space():
    specs = synth.uneven_event_specs(n_events=256)
    assert {s["Tobs"] for s in specs} >= {4.0, 8.0, 16.0, 32.0, 64.0} - {64.0}
    assert {len(s["labels"]) for s in specs} == {1, 2, 3}
    assert {s["fs"] for s in specs} == {2048.0, 4096.0}


def test_multi_matches_oracle_and_single_event(uneven, ora):
    evs, handles, batch = uneven
    eo, P = synth.uneven_params(evs, chains=4, proposals=3, seed=4200)
    for prec, tol in ((q.FP64, 1e-8), (q.MIXED, 1e-3)):
        L = batch.lnl(eo, P, prec)
        for e, ev in enumerate(evs):
            sel = eo == e
            Lo, _ = ora.lnl_full_batch(ev, P[sel])
            np.testing.assert_allclose(L[sel], Lo, rtol=0, atol=tol, err_msg=f"event {e} prec {prec}")
            Ls = handles[e].lnl_full(P[sel], prec)
            np.testing.assert_allclose(L[sel], Ls, rtol=0, atol=1e-9 if prec == q.FP64 else 2e-4)


def test_alone_equals_in_mix(uneven):
    evs, handles, batch = uneven
    eo, P = synth.uneven_params(evs, chains=4, proposals=4, seed=4300)
    full = batch.lnl(eo, P, q.MIXED)
    for e in (0, 3, 7):
        sel = eo == e
        alone = batch.lnl(eo[sel], P[sel], q.MIXED)
        assert np.array_equal(alone, full[sel]), "a set's lnL must not depend on the other sets in the call"
    perm = np.random.default_rng(1).permutation(len(P))
    shuffled = batch.lnl(eo[perm], P[perm], q.MIXED)
    assert np.array_equal(shuffled, full[perm])


def test_tilings_agree(uneven):
    evs, handles, batch = uneven
    eo, P = synth.uneven_params(evs, chains=2, proposals=2, seed=4400)
    ref = batch.lnl(eo, P, q.FP64)
    for tb, th in ((1024, 128), (8192, 256), (700, 64)):
        batch.set_tiling(tb, th)
        np.testing.assert_allclose(batch.lnl(eo, P, q.FP64), ref, rtol=0, atol=1e-9)
    batch.set_tiling(2048, 256)


def test_invalid_event_index_and_params(uneven):
    evs, handles, batch = uneven
    eo, P = synth.uneven_params(evs, chains=1, proposals=2, seed=4500)
    eo = eo.copy()
    eo[1] = 99
    P = P.copy()
    P[2, 2] = 2.0
    L = batch.lnl(eo, P, q.MIXED, allow_invalid=True)
    assert L[1] == -1e20 and L[2] == -1e20
    assert np.all(L[3:] > -1e19)
    with pytest.raises(q.QcbcError):
        batch.lnl(eo, P, q.MIXED)


def test_autotune_keeps_results(uneven):
    evs, handles, batch = uneven
    eo, P = synth.uneven_params(evs, chains=8, proposals=8, seed=4600)
    before = batch.lnl(eo, P, q.FP64)
    tb, th = batch.autotune(eo, P, q.MIXED)
    assert tb > 0 and th in (64, 128, 256)
    np.testing.assert_allclose(batch.lnl(eo, P, q.FP64), before, rtol=0, atol=1e-9)
    assert np.all(batch.time(len(P), q.MIXED, iters=3) > 0)


def test_multi_het_matches_single_event(uneven):
    """qcbc_lnl_multi_het: each set uses its own event's heterodyne tables (grid search and tables
    built on the GPU about each injection); equal to the single-event heterodyned lnL."""
    evs, handles, _ = uneven
    sel_events = [0, 1, 2, 3]
    for e in sel_events:
        pmin, pmax = prior_bounds(evs[e].Tobs)
        g, MN, MM = handles[e].het_space(evs[e].inj, pmin, pmax)
        handles[e].het_setup(evs[e].inj, g, MN, MM, 2)
    batch = q.Batch([handles[e] for e in sel_events] + [handles[5]])     # the last one has no tables
    rng = np.random.default_rng(4400)
    eo, P = [], []
    for k, e in enumerate(sel_events):
        P.append(synth.jitter_params(rng, 6, evs[e].inj, scale=1e-5))
        eo += [k] * 6
    eo, P = np.array(eo, dtype=np.int32), np.vstack(P)
    for prec, tol in ((q.FP64, 1e-9), (q.MIXED, 1e-9)):
        L = batch.lnl_het(eo, P, prec)
        for k, e in enumerate(sel_events):
            Ls = handles[e].lnl_het(P[eo == k], prec)
            np.testing.assert_allclose(L[eo == k], Ls, rtol=0, atol=tol)
    alone = batch.lnl_het(eo[eo == 2], P[eo == 2], q.MIXED)
    assert np.array_equal(alone, batch.lnl_het(eo, P, q.MIXED)[eo == 2])
    Lx = batch.lnl_het(np.array([4, 0], dtype=np.int32), P[:2], q.FP64, allow_invalid=True)
    assert Lx[0] == -1e20 and Lx[1] > -1e19
    batch.close()

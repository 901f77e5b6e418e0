"""Continuous-batching service: a run evolves identically alone and in a mix,
admission respects the device-memory budget, over-budget and cancelled runs
are reported, and the sampler concentrates on the injection."""
import numpy as np
import pytest

import quickcbc_b200 as q
from quickcbc_b200 import serving, synth
from conftest import oracle_template

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def events(ora):
    specs = synth.uneven_event_specs(n_events=4, seed=5100)
    for s in specs:
        s["Tobs"] = min(s["Tobs"], 8.0)
    return [synth.make_event(oracle_template(ora), **s) for s in specs]


SAMPLER = dict(n_temps=4, n_chains=2, n_steps=60, burn_in=20, thin=5)


def test_run_same_alone_and_in_mix(events):
    for prec in (q.MIXED, q.FP64):
        alone = serving.Server(max_live=8, max_bins=1 << 15, precision=prec)
        r = alone.submit(events[0], seed=11, **SAMPLER)
        alone.run_until_idle()
        s_alone = alone.samples(r)
        mix = serving.Server(max_live=8, max_bins=1 << 15, precision=prec)
        ids = [mix.submit(ev, seed=11 + k, **SAMPLER) for k, ev in enumerate(events)]
        mix.run_until_idle()
        s_mix = mix.samples(ids[0])
        assert s_alone.shape == (SAMPLER["n_chains"] * 8, 12)
        assert np.array_equal(s_alone, s_mix), "a run must evolve identically alone and in the mix"
        assert all(mix.info(i)["state"] == serving.RUN_DONE for i in ids)
        alone.close()
        mix.close()


def test_admission_by_budget_and_refusal(events):
    probe = serving.Server(max_live=1, max_bins=1 << 15)
    sizes = [probe.info(probe.submit(ev, seed=9, **SAMPLER))["device_bytes"] for ev in events[:2]]
    probe.close()
    one = max(sizes) + min(sizes) // 2          # room for either run, not for both
    srv = serving.Server(hbm_budget_bytes=one, max_live=8, max_bins=1 << 15)
    a = srv.submit(events[0], seed=1, **SAMPLER)
    b = srv.submit(events[1], seed=2, **SAMPLER)
    nl, nq, _ = srv.step()
    assert (nl, nq) == (1, 1), "only one run fits the budget"
    srv.run_until_idle()
    ia, ib = srv.info(a), srv.info(b)
    assert ia["state"] == ib["state"] == serving.RUN_DONE
    assert ib["t_admit"] >= ia["t_done"], "the queued run is admitted when memory is released"
    tiny = serving.Server(hbm_budget_bytes=1 << 10, max_live=8, max_bins=1 << 15)
    with pytest.raises(q.QcbcError) as ei:
        tiny.submit(events[0], **SAMPLER)
    assert ei.value.code == -4
    srv.close()
    tiny.close()


def test_cancel_queued_and_live(events):
    srv = serving.Server(max_live=1, max_bins=1 << 15)
    a = srv.submit(events[0], seed=1, **SAMPLER)
    b = srv.submit(events[1], seed=2, **SAMPLER)
    srv.step()
    srv.cancel(b)
    assert srv.info(b)["state"] == serving.RUN_CANCELLED
    srv.cancel(a)
    assert srv.info(a)["state"] == serving.RUN_CANCELLED
    nl, nq, _ = srv.step()
    assert nl == 0 and nq == 0
    assert srv.stats()["device_bytes_live"] == 0
    srv.close()


def test_chains_concentrate_on_injection(ora):
    ev = synth.config_event(1, oracle_template(ora), snr=40.0)
    srv = serving.Server(max_live=4, max_bins=1 << 13)
    start = ev.inj.copy()
    r = srv.submit(ev, start=start, n_temps=4, n_chains=4, n_steps=400, burn_in=200, thin=4, seed=3)
    srv.run_until_idle()
    s = srv.samples(r)
    info = srv.info(r)
    assert 0.02 < info["accept_cold"] < 0.9
    Linj, _ = ora.lnl_full(ev, ev.inj)
    assert np.max(s[:, 11]) > Linj - 5.0
    assert abs(np.median(s[:, 0]) - ev.inj[0]) < 0.05      # ln chirp mass stays near the injection
    srv.close()


def test_stream_driver_reports_latency(events):
    srv = serving.Server(max_live=8, max_bins=1 << 15)
    res = serving.serve_stream(srv, events, rate_hz=20.0, seed=4, sampler=dict(n_temps=2, n_chains=2, n_steps=40,
                                                                                 burn_in=10, thin=5))
    assert res["n_done"] == len(events)
    assert res["p50_s"] > 0 and res["p99_s"] >= res["p50_s"]
    assert res["lnl_evals"] == sum(2 * 2 * 41 for _ in events)
    srv.close()


def test_het_runs_same_alone_and_in_mix(events):
    """Heterodyned runs: grid search and tables at admission; a run evolves identically alone and
    in a mix that also holds full-likelihood runs."""
    alone = serving.Server(max_live=8, max_bins=1 << 15)
    r = alone.submit(events[0], seed=21, likelihood="het", **SAMPLER)
    alone.run_until_idle()
    s_alone = alone.samples(r)
    mix = serving.Server(max_live=8, max_bins=1 << 15)
    ids = [mix.submit(ev, seed=21 + k, likelihood="het" if k % 2 == 0 else "full", **SAMPLER)
           for k, ev in enumerate(events)]
    mix.run_until_idle()
    assert all(mix.info(i)["state"] == serving.RUN_DONE for i in ids)
    assert s_alone.shape == (SAMPLER["n_chains"] * 8, 12)
    assert np.array_equal(s_alone, mix.samples(ids[0]))
    alone.close()
    mix.close()


def test_het_chains_concentrate_on_injection(ora):
    ev = synth.config_event(1, oracle_template(ora), snr=40.0)
    srv = serving.Server(max_live=4, max_bins=1 << 13)
    r = srv.submit(ev, start=ev.inj.copy(), n_temps=4, n_chains=4, n_steps=400, burn_in=200, thin=4, seed=3,
                   likelihood="het")
    srv.run_until_idle()
    s = srv.samples(r)
    assert srv.info(r)["state"] == serving.RUN_DONE
    Linj, _ = ora.lnl_full(ev, ev.inj)
    assert np.max(s[:, 11]) > Linj - 5.0
    assert abs(np.median(s[:, 0]) - ev.inj[0]) < 0.05
    srv.close()

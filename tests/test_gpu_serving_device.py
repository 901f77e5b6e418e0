"""Continuous-batching service with device-resident stepping (qcbc_server_set_device_steps):
a run evolves identically alone and in a mix, for any number of steps per host call, with
full and heterodyned likelihoods side by side; cancelled and live runs report their samples;
the sampler concentrates on the injection."""
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


def run_alone(ev, K, prec=q.MIXED, **kw):
    srv = serving.Server(max_live=8, max_bins=1 << 15, precision=prec, device_steps=K)
    r = srv.submit(ev, **kw)
    srv.run_until_idle()
    s, info = srv.samples(r), srv.info(r)
    srv.close()
    return s, info


def test_device_run_same_alone_and_in_mix(events):
    for prec in (q.MIXED, q.FP64):
        s_alone, _ = run_alone(events[0], 4, prec, seed=11, **SAMPLER)
        mix = serving.Server(max_live=8, max_bins=1 << 15, precision=prec, device_steps=4)
        ids = [mix.submit(ev, seed=11 + k, **SAMPLER) for k, ev in enumerate(events)]
        mix.run_until_idle()
        assert all(mix.info(i)["state"] == serving.RUN_DONE for i in ids)
        assert s_alone.shape == (SAMPLER["n_chains"] * 8, 12)
        assert np.array_equal(s_alone, mix.samples(ids[0])), "a run must evolve identically alone and in the mix"
        mix.close()


def test_device_steps_per_call_do_not_change_the_chain(events):
    """K = 1, 7 and 16 steps per call give the same samples and counters: steps are the same kernels
    whatever the number queued, and a call stops early when a run finishes."""
    res = [run_alone(events[1], K, seed=5, **SAMPLER) for K in (1, 7, 16)]
    for s, info in res[1:]:
        assert np.array_equal(s, res[0][0])
        for k in ("steps_done", "accept_cold", "swap_rate", "lnl_evals", "n_samples"):
            assert info[k] == res[0][1][k], k
    assert res[0][1]["steps_done"] == SAMPLER["n_steps"]
    assert res[0][1]["lnl_evals"] == 4 * 2 * (SAMPLER["n_steps"] + 1)


def test_device_het_and_full_mix(events):
    s_alone, _ = run_alone(events[0], 8, seed=21, likelihood="het", **SAMPLER)
    mix = serving.Server(max_live=8, max_bins=1 << 15, device_steps=3)
    ids = [mix.submit(ev, seed=21 + k, likelihood="het" if k % 2 == 0 else "full", **SAMPLER)
           for k, ev in enumerate(events)]
    mix.run_until_idle()
    assert all(mix.info(i)["state"] == serving.RUN_DONE for i in ids)
    assert np.array_equal(s_alone, mix.samples(ids[0]))
    s_full, _ = run_alone(events[1], 5, seed=22, **SAMPLER)
    assert np.array_equal(s_full, mix.samples(ids[1]))
    mix.close()


def test_device_live_info_cancel_and_staggered_admission(events):
    srv = serving.Server(max_live=2, max_bins=1 << 15, device_steps=10)
    a = srv.submit(events[0], seed=1, **SAMPLER)
    b = srv.submit(events[1], seed=2, **SAMPLER)
    c = srv.submit(events[2], seed=3, **SAMPLER)
    for _ in range(4):
        srv.step()                      # 1 + 39 steps: past burn-in, some samples
    ia = srv.info(a)
    assert ia["state"] == serving.RUN_LIVE and ia["steps_done"] == 39
    assert ia["n_samples"] == SAMPLER["n_chains"] * ((39 - 20) // 5)
    part = srv.samples(a)
    assert part.shape == (ia["n_samples"], 12)
    srv.cancel(a)
    assert srv.info(a)["state"] == serving.RUN_CANCELLED
    assert np.array_equal(srv.samples(a), part)
    srv.run_until_idle()                # c is admitted into a's slot while b runs on
    assert srv.info(b)["state"] == srv.info(c)["state"] == serving.RUN_DONE
    s_c, _ = run_alone(events[2], 10, seed=3, **SAMPLER)
    assert np.array_equal(srv.samples(c), s_c)
    assert srv.stats()["device_bytes_live"] == 0
    srv.close()


def test_device_mode_settings_are_checked(events):
    srv = serving.Server(max_live=2, max_bins=1 << 15)
    srv.submit(events[0], seed=1, **SAMPLER)
    with pytest.raises(q.QcbcError):
        srv.set_device_steps(4)        # runs already submitted
    srv.close()
    srv = serving.Server(max_live=2, max_bins=1 << 15, device_steps=4)
    with pytest.raises(q.QcbcError):
        srv.submit(events[0], n_temps=65, n_chains=1, n_steps=10, burn_in=0, thin=1)
    srv.close()


@pytest.mark.parametrize("likelihood", ["full", "het"])
def test_device_chains_concentrate_on_injection(ora, likelihood):
    ev = synth.config_event(1, oracle_template(ora), snr=40.0)
    srv = serving.Server(max_live=4, max_bins=1 << 13, device_steps=32)
    r = srv.submit(ev, start=ev.inj.copy(), n_temps=4, n_chains=4, n_steps=400, burn_in=200, thin=4, seed=3,
                   likelihood=likelihood)
    srv.run_until_idle()
    s, info = srv.samples(r), srv.info(r)
    assert info["state"] == serving.RUN_DONE and s.shape == (4 * 50, 12)
    assert 0.02 < info["accept_cold"] < 0.9 and info["swap_rate"] > 0.0
    Linj, _ = ora.lnl_full(ev, ev.inj)
    assert np.max(s[:, 11]) > Linj - 5.0
    assert abs(np.median(s[:, 0]) - ev.inj[0]) < 0.05
    srv.close()


def test_device_stream_driver(events):
    srv = serving.Server(max_live=8, max_bins=1 << 15, device_steps=8)
    res = serving.serve_stream(srv, events, rate_hz=20.0, seed=4, sampler=dict(n_temps=2, n_chains=2, n_steps=40,
                                                                                 burn_in=10, thin=5))
    assert res["n_done"] == len(events)
    assert res["lnl_evals"] == sum(2 * 2 * 41 for _ in events)
    srv.close()


def reference_sampler(n_steps=400):
    return dict(n_temps=4, n_chains=4, n_steps=n_steps, burn_in=n_steps // 2, thin=4)


@pytest.mark.parametrize("likelihood", ["full", "het"])
def test_reference_proposal_concentrates_on_injection(ora, likelihood):
    """The reference's proposal mixture (Fisher eigen-jumps from Fisher_Het + FisherEvec + efix at
    the start point, differential evolution, jiggles) samples the injection's neighbourhood."""
    ev = synth.config_event(1, oracle_template(ora), snr=40.0)
    srv = serving.Server(max_live=4, max_bins=1 << 13, device_steps=32)
    r = srv.submit(ev, start=ev.inj.copy(), seed=3, likelihood=likelihood, proposal="reference",
                   **reference_sampler())
    srv.run_until_idle()
    s, info = srv.samples(r), srv.info(r)
    assert info["state"] == serving.RUN_DONE and s.shape == (4 * 50, 12)
    assert 0.02 < info["accept_cold"] < 0.9 and info["swap_rate"] > 0.0
    Linj, _ = ora.lnl_full(ev, ev.inj)
    assert np.max(s[:, 11]) > Linj - 5.0
    assert abs(np.median(s[:, 0]) - ev.inj[0]) < 0.05
    assert np.std(s[:, 5]) > 0.0 and np.std(s[:, 7]) > 0.0
    srv.close()


def test_reference_proposal_same_alone_mix_and_K(events):
    kw = dict(SAMPLER, proposal="reference")
    s1, _ = run_alone(events[0], 1, seed=31, **kw)
    s16, _ = run_alone(events[0], 16, seed=31, **kw)
    assert np.array_equal(s1, s16)
    mix = serving.Server(max_live=8, max_bins=1 << 15, device_steps=5)
    ids = [mix.submit(ev, seed=31 + k, likelihood="het" if k % 2 else "full", **kw) for k, ev in enumerate(events)]
    mix.run_until_idle()
    assert all(mix.info(i)["state"] == serving.RUN_DONE for i in ids)
    assert np.array_equal(mix.samples(ids[0]), s1)
    mix.close()


def test_reference_proposal_needs_device_steps(events):
    srv = serving.Server(max_live=2, max_bins=1 << 15)
    with pytest.raises(q.QcbcError):
        srv.submit(events[0], proposal="reference", **SAMPLER)
    srv.close()


@pytest.mark.parametrize("device_steps", [0, 16])
def test_prior_density_uniform_in_volume(events, device_steps):
    """With a likelihood that is zero everywhere (no data, PSD 1e30 times the curve) the chains
    sample the prior of update (QuickCBC.c:2352-2381).  Its distance part is uniform in volume,
    p(ln D) ~ exp(3 ln D) on [ln 1e6 pc, ln 1e10 pc]: mean b - 1/3 at the upper edge b, where a flat
    prior in ln D would give the box's middle."""
    ev = events[0]
    quiet = synth.Event(**{**ev.__dict__, "D": np.zeros_like(ev.D), "SN": ev.SN * 1e30})
    b = np.log(1e10 * synth.PC_SI)
    start = ev.inj.copy()
    start[6] = b - 0.3
    scales = np.array([1e-4, 1e-3, 0.02, 0.02, 0.1, 1e-4, 0.3, 0.01, 0.01, 0.02, 0.02])
    srv = serving.Server(max_live=2, max_bins=1 << 15, device_steps=device_steps)
    r = srv.submit(quiet, start=start, scales=scales, n_temps=1, n_chains=64, n_steps=3000, burn_in=500, thin=10,
                   seed=5)
    srv.run_until_idle()
    s = srv.samples(r)
    assert np.max(np.abs(s[:, 11])) < 1e-6, "the likelihood is flat"
    m = np.mean(s[:, 6])
    assert abs(m - (b - 1.0 / 3.0)) < 0.06, (m, b - 1.0 / 3.0)
    srv.close()

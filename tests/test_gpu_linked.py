"""An unchanged QuickCBC on the GPU library: the drop-in boundary proved end to end.

oracle/_ref/libquickcbc_linked.so (`make -C oracle linked`) is the reference's own sources compiled
unmodified, their definitions of the thirteen replaced functions weakened with objcopy, linked with
the forwarding stub include/qcbc_forward.c against libqcbc_gpu.so -- the recipe INTEGRATION.md
gives maintainers.  These tests check that

* every replaced name is defined once, strongly, by the stub (nm);
* the reference's own callers -- log_likelihood_full at chain start, het_space and heterodyne,
  Fisher_Het -> FisherEvec -> efix with het_diff, and update() with its log_likelihood_het call
  (QuickCBC.c:1898-2067, 2238-2405) -- reach the GPU: the stub's call counters and the library's
  launch counter move, and the values equal the library's batched API and the reference's CPU
  values;
* the same run from 12 OpenMP threads, as MCMC_all runs its chains (QuickCBC.c:118, 2063-2067),
  equals the serial run bit for bit;
* the unbound log_likelihood_full follows SN rewritten in place (the noisemarg redraw,
  QuickCBC.c:1994-2010) and refuses a frequency grid other than the reference's.

Tolerances: GPU against the reference's CPU values 1e-8 absolute in lnL (FP64 on both sides; libm
and CUDA transcendentals round differently); GPU against GPU bit for bit.
"""
import os
import re
import subprocess
import tempfile

import numpy as np
import pytest

import quickcbc_b200 as q
from quickcbc_b200 import synth
from conftest import prior_bounds, GoldenEvent, load_golden

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _linked():
    from oracle import ref
    if not ref.linked_available():
        pytest.skip("oracle/_ref/libquickcbc_linked.so not built (make -C oracle linked)")
    return ref


def test_replaced_names_are_the_forwarding_stubs():
    ref = _linked()
    out = subprocess.run(["nm", "-l", "--defined-only", ref.LINKED_PATH], capture_output=True, text=True,
                         check=True).stdout
    for name in ref.FORWARD_NAMES:
        lines = [ln for ln in out.splitlines() if re.search(r"\s[A-Za-z]\s%s(\s|$)" % name, ln)]
        assert len(lines) == 1, (name, lines)
        assert re.search(r"\sT\s%s\s.*qcbc_forward\.c:\d+$" % name, lines[0]), lines[0]
    # the reference's own callers are there, from its own sources
    for name in ("update", "efix", "FisherEvec", "MCMC_all", "log_likelihood_test", "Fisher_All"):
        assert re.search(r"\sT\s%s(\s|$)" % name, out), name


@pytest.fixture(scope="module")
def linked_cfg1():
    ref = _linked()
    ev = GoldenEvent(load_golden("cfg1.npz"))
    q.set_band(16.0, 1024.0)                    # ConstCBC.h:33-34, the reference's compiled band
    L = ref.linked()
    net = ref.RefNet(ev.labels, ev.Tobs, ev.GMST, L=L)
    data = ref.LinkedData(net, ev.D, ev.SN, ev.freq, ev.N, ev.Tobs)
    het = ref.RefHet(net)
    pmin, pmax = prior_bounds(ev.Tobs)
    with tempfile.TemporaryDirectory() as d:
        het.space(ev.inj, pmin, pmax, ev.freq, ev.SN, ev.N, ev.Tobs, d)      # forwarded: GPU het_space
    het.heterodyne(ev.D, ev.inj, ev.freq, ev.SN, ev.N, ev.Tobs)               # forwarded: GPU heterodyne
    yield ref, ev, net, data, het, pmin, pmax
    L.lk_unbind()


def _mcmc(ref, net, het, data, P0, pmin, pmax, steps, nthreads):
    import ctypes as C
    nc = len(P0)
    p_out, logL, logL0, ej = np.zeros((nc, 11)), np.zeros(nc), np.zeros(nc), np.zeros((nc, 11))
    acc = np.zeros(nc, dtype=np.int32)
    launches = C.c_longlong(0)
    secs = net.L.lk_mcmc(net.ptr, het.ptr, data.ptr, np.ascontiguousarray(P0), pmin.copy(), pmax.copy(), steps,
                         nthreads, 7, p_out, logL, logL0, ej, acc, C.byref(launches))
    return dict(p=p_out, logL=logL, logL0=logL0, ejump=ej, accepted=acc, launches=launches.value, secs=secs)


@pytest.mark.gpu
def test_reference_sampler_runs_on_gpu_and_threads_agree(linked_cfg1):
    ref, ev, net, data, het, pmin, pmax = linked_cfg1
    h1 = load_golden("het1.npz")
    t = het.export()
    assert np.array_equal(t["fgrid"], h1["fgrid"])           # het_space on the GPU: the reference's grid
    assert abs(t["logLb"] - float(h1["logLb"])) < 1e-8
    P0 = synth.jitter_params(np.random.default_rng(77), 12, ev.inj, scale=1e-4)
    c0 = ref.forward_calls()
    serial = _mcmc(ref, net, het, data, P0, pmin, pmax, 150, 1)
    c1 = ref.forward_calls()
    threaded = _mcmc(ref, net, het, data, P0, pmin, pmax, 150, 12)
    c2 = ref.forward_calls()
    for k in ("p", "logL", "logL0", "ejump", "accepted"):
        assert np.array_equal(serial[k], threaded[k]), k
    d1 = {n: c1[n] - c0[n] for n in c0}
    d2 = {n: c2[n] - c1[n] for n in c0}
    assert d1 == d2
    assert d1["log_likelihood_full"] == 12 and d1["Fisher_Het"] == 12
    assert d1["het_diff"] > 12 and d1["log_likelihood_het"] > 12 + 150 * 12 // 2
    assert serial["accepted"].sum() > 0
    # every forwarded likelihood call launched GPU kernels
    assert serial["launches"] >= d1["log_likelihood_full"] + d1["log_likelihood_het"] + d1["Fisher_Het"]
    # the chains' lnL are the GPU's: the batched API on the same tables gives the same numbers
    e = q.Event(ev.labels, ev.Tobs, ev.GMST, ev.N, ev.D, ev.SN, fmin=16.0)
    e.het_set(t)
    np.testing.assert_allclose(serial["logL"], e.lnl_het(serial["p"], q.FP64), rtol=0, atol=1e-12)
    L0 = np.array([e.lnl_full(p, q.FP64)[0] for p in P0])
    np.testing.assert_allclose(serial["logL0"], L0, rtol=0, atol=1e-12)
    e.close()
    # ... and the reference's own CPU values, within the FP64 tolerance
    rnet = ref.RefNet(ev.labels, ev.Tobs, ev.GMST)
    rhet = ref.RefHet(rnet)
    rhet.set_grid(t["fgrid"], int(t["MN"]), int(t["MM"]), int(t["J"]), ev.Tobs)
    rhet.heterodyne(ev.D, ev.inj, ev.freq, ev.SN, ev.N, ev.Tobs)
    np.testing.assert_allclose(serial["logL"], rhet.lnl_batch(serial["p"], ev.Tobs)[0], rtol=0, atol=1e-8)
    np.testing.assert_allclose(serial["logL0"], ref.lnl_full_batch(rnet, ev.D, P0, ev.freq, ev.SN, ev.N,
                                                                   ev.Tobs)[0], rtol=0, atol=1e-8)


@pytest.mark.gpu
def test_reference_timing_loop_from_12_threads(linked_cfg1):
    """QuickCBC.c:1931-1941's 1000-call loops, run by 12 threads at once, unbound and bound: every
    thread gets the value one thread gets, bit for bit."""
    ref, ev, net, data, het, pmin, pmax = linked_cfg1
    L = net.L
    p = ev.inj.copy()
    for which in (0, 1):
        for bind in ((False, True) if which == 0 else (False,)):
            if bind:
                assert L.lk_bind(net.ptr, data.ptr) == 0
            one, many = np.zeros(1), np.zeros(12)
            L.lk_time_calls(net.ptr, het.ptr, data.ptr, p, which, 20, 1, one)
            L.lk_time_calls(net.ptr, het.ptr, data.ptr, p, which, 20, 12, many)
            assert np.all(many == one[0]), (which, bind, many, one)
            if bind:
                L.lk_unbind()


@pytest.mark.gpu
def test_unbound_full_likelihood_follows_data_and_grid(linked_cfg1):
    ref, ev, net, data, het, pmin, pmax = linked_cfg1
    L = net.L
    p = ev.inj.copy()
    rho = np.zeros(4)
    a = L.lk_lnl_full(net.ptr, data.ptr, p, rho)
    assert L.lk_lnl_full(net.ptr, data.ptr, p, rho) == a          # the cached event, same data
    data.SN[1] *= 2.0                                              # a PSD redraw written in place
    b = L.lk_lnl_full(net.ptr, data.ptr, p, rho)
    e = q.Event(ev.labels, ev.Tobs, ev.GMST, ev.N, ev.D, data.SN, fmin=16.0)
    assert b == e.lnl_full(p, q.FP64)[0] and b != a
    e.close()
    data.SN[1] /= 2.0
    assert L.lk_lnl_full(net.ptr, data.ptr, p, rho) == a
    f = data.freq.copy()
    data.freq[:] = f * 1.5                                         # not the reference's grid
    assert L.lk_lnl_full(net.ptr, data.ptr, p, rho) == -1e20
    from quickcbc_b200 import _lib
    assert "reference grid" in _lib.last_error()
    data.freq[:] = f
    assert L.lk_lnl_full(net.ptr, data.ptr, p, rho) == a

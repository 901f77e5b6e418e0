"""Parity of the CUDA path (called through the C ABI) with the reference's
outputs (golden fixtures) and with the CPU oracle on the same seeded inputs.

Tolerances:
  FP64 plain form   lnL within 1e-8 absolute (reference arithmetic is FP64;
                    differences come from libm vs CUDA transcendental rounding)
  mixed precision   |lnL - lnL_FP64 oracle| <= 1e-3 (the stated target)
"""
import numpy as np
import pytest

import quickcbc_b200 as q
from quickcbc_b200 import synth
from conftest import GoldenEvent, oracle_template, load_golden

pytestmark = pytest.mark.gpu

LNL_ATOL_FP64 = 1e-8
LNL_ATOL_MIXED = 1e-3


@pytest.fixture(scope="module")
def ev1(cfg1_event):
    ev, z = cfg1_event
    e = q.Event.from_synthetic(ev)
    yield ev, z, e
    e.close()


@pytest.fixture(scope="module")
def cfg2(ora):
    ev = synth.config_event(2, oracle_template(ora))
    e = q.Event.from_synthetic(ev)
    yield ev, e
    e.close()


def test_amp_phase_vs_reference(golden, ora):
    z = golden("wave.npz")
    for k, m in enumerate(z["meta"]):
        st, a, p = q.amp_phase(z["freq"], *m)
        assert st == 0
        ar, pr = z["amp"][k], z["phase"][k]
        assert np.array_equal(ar != 0, a != 0)
        nz = ar != 0
        np.testing.assert_allclose(a[nz], ar[nz], rtol=1e-12)
        np.testing.assert_allclose(p, pr, rtol=0, atol=1e-9 * max(1.0, np.abs(pr).max()))


def test_amp_phase_domain_errors():
    f = np.geomspace(10, 1000, 50)
    st, _, _ = q.amp_phase(f, 0.0, 100.0, 30 * synth.MSUN_SI, 20 * synth.MSUN_SI, 1.2, 0.0, 1e25)
    assert st == 33
    st, _, _ = q.amp_phase(f, 0.0, 100.0, -1.0, 20 * synth.MSUN_SI, 0.1, 0.0, 1e25)
    assert st == 33
    # fCut below the first frequency (IMRPhenomD.c:228-233)
    st, _, _ = q.amp_phase(np.array([500.0, 600.0]), 0.0, 100.0, 2e3 * synth.MSUN_SI, 1e3 * synth.MSUN_SI, 0, 0, 1e25)
    assert st == 33


def test_fulltemplates_vs_reference(ev1):
    ev, z, _ = ev1
    for H, k in zip(z["h"], z["h_idx"]):
        h = q.fulltemplates(ev.labels, ev.GMST, ev.freq, z["params"][k], ev.N)
        np.testing.assert_allclose(h, H, rtol=0, atol=1e-11 * np.abs(H).max())


def test_fullphaseamp_vs_reference(ev1):
    ev, z, _ = ev1
    a, p = q.fullphaseamp(ev.labels, ev.GMST, ev.Tobs, ev.freq, z["params"][0], ev.N)
    np.testing.assert_allclose(a, z["pa_amp"], rtol=1e-12, atol=1e-40)
    np.testing.assert_allclose(p, z["pa_phase"], rtol=0, atol=1e-9 * np.abs(z["pa_phase"]).max())


def test_lnl_full_fp64_vs_reference(ev1):
    ev, z, e = ev1
    L, rho = e.lnl_full(z["params"], q.FP64, rho=True)
    np.testing.assert_allclose(L, z["lnl"], rtol=0, atol=LNL_ATOL_FP64)
    np.testing.assert_allclose(rho, z["rho"], rtol=1e-9)


def test_lnl_full_mixed_vs_fp64_oracle(ev1, ora):
    ev, z, e = ev1
    L = e.lnl_full(z["params"], q.MIXED)
    Lo, _ = ora.lnl_full_batch(ev, z["params"])
    assert np.max(np.abs(L - Lo)) <= LNL_ATOL_MIXED


def test_lnl_full_cfg2_fp64_and_mixed(cfg2, ora):
    ev, e = cfg2
    rng = np.random.default_rng(2501)
    P = np.vstack([synth.jitter_params(rng, 16, ev.inj), synth.draw_params(rng, 48, ev.inj)])
    Lo, _ = ora.lnl_full_batch(ev, P)
    L64 = e.lnl_full(P, q.FP64)
    np.testing.assert_allclose(L64, Lo, rtol=0, atol=LNL_ATOL_FP64 * max(1.0, np.abs(Lo).max() / 100))
    Lm = e.lnl_full(P, q.MIXED)
    assert np.max(np.abs(Lm - Lo)) <= LNL_ATOL_MIXED


def test_batch_equals_single_and_deterministic(cfg2):
    ev, e = cfg2
    rng = np.random.default_rng(2502)
    P = synth.draw_params(rng, 24, ev.inj)
    for prec in (q.FP64, q.MIXED):
        Lb = e.lnl_full(P, prec)
        Ls = np.array([e.lnl_full(p, prec)[0] for p in P[:6]])
        # a single set gets more blocks per set than a batch, so the block sums differ in order
        np.testing.assert_allclose(Ls, Lb[:6], rtol=0, atol=1e-9 if prec == q.FP64 else 2e-4)
        assert np.array_equal(Lb, e.lnl_full(P, prec)), "repeat calls must be bit-identical"


def test_launch_shapes_agree(cfg2):
    """Tile count and block size are tuning knobs only: results agree across them."""
    ev, e = cfg2
    P = synth.draw_params(np.random.default_rng(2503), 8, ev.inj)
    ref_L = e.lnl_full(P, q.FP64)
    for tiles, threads in ((1, 256), (3, 128), (17, 64), (64, 256)):
        e.set_launch(tiles, threads)
        np.testing.assert_allclose(e.lnl_full(P, q.FP64), ref_L, rtol=0, atol=1e-9)
        np.testing.assert_allclose(e.lnl_full(P, q.MIXED), ref_L, rtol=0, atol=LNL_ATOL_MIXED)
    e.set_launch(0, 0)


def test_multi_tile_sets_finalised_in_their_last_tile(cfg2):
    """At several tiles per set, the last tile of each set to finish sums the set's partials in tile
    order and finalises it (no finaliser launch).  The result equals, bit for bit, the allocation-free
    entry point's separate finaliser over the same partials; repeat calls agree (each set's tile count
    is back at zero after a launch); an invalid set among them gets -1e20 and rho 0."""
    from quickcbc_b200 import _lib
    ev, e = cfg2
    P = synth.draw_params(np.random.default_rng(2506), 40, ev.inj)
    P[3, 2] = 1.5                      # spin outside [-1, 1]
    B = len(P)
    dP = q.DeviceBuffer(P.nbytes)
    dP.upload(P)
    dL, dR = q.DeviceBuffer(B * 8), q.DeviceBuffer(B * 8 * e.nifo)
    L = _lib.lib()

    def run(fn, prec):
        rc = fn(e.handle, dP.ptr, B, dL.ptr, dR.ptr, prec, None)
        assert rc == 0, _lib.last_error()
        assert L.qcbc_synchronize() == 0
        return dL.download((B,)), dR.download((B, e.nifo))
    try:
        for tiles in (2, 7, 63):
            e.set_launch(tiles, 256)
            for prec in (q.FP64, q.MIXED):
                a = run(L.qcbc_lnl_full_dev, prec)
                assert a[0][3] == -1e20 and np.all(a[1][3] == 0.0)
                for x in (run(L.qcbc_lnl_full_dev, prec), run(L.qcbc_lnl_full_noalloc, prec)):
                    assert np.array_equal(a[0], x[0]) and np.array_equal(a[1], x[1]), (tiles, prec)
    finally:
        e.set_launch(0, 0)


def test_length_ordered_batch_matches_unordered(cfg2, ora):
    """At one tile per set (B >= 1184) the sets run in order of their bin count: every set's lnL
    equals the same set in a multi-tile launch (which runs in index order), invalid sets at
    scattered positions included, and repeat calls are bit-identical."""
    ev, e = cfg2
    rng = np.random.default_rng(2504)
    P = synth.draw_params(rng, 2048, ev.inj)
    bad = [5, 700, 2047]
    P[bad, 2] = 1.5                    # spin outside [-1, 1]
    assert e.get_launch(len(P), q.FP64)[0] == 1
    for prec, tol in ((q.FP64, 1e-9), (q.MIXED, 2e-4)):
        L = e.lnl_full(P, prec, allow_invalid=True)
        assert np.array_equal(L, e.lnl_full(P, prec, allow_invalid=True)), "repeat calls must be bit-identical"
        e.set_launch(4, 256)
        Lu = e.lnl_full(P, prec, allow_invalid=True)
        e.set_launch(0, 0)
        assert np.all(L[bad] == -1e20) and np.all(Lu[bad] == -1e20)
        np.testing.assert_allclose(L, Lu, rtol=0, atol=tol)
    # rho from the one-tile kernel (written straight into the host staging buffer) against the
    # multi-tile launch's
    L1, R1 = e.lnl_full(P, q.FP64, rho=True, allow_invalid=True)
    e.set_launch(4, 256)
    _, R1u = e.lnl_full(P, q.FP64, rho=True, allow_invalid=True)
    e.set_launch(0, 0)
    assert np.all(R1[bad] == 0.0)
    np.testing.assert_allclose(R1, R1u, rtol=1e-9, atol=1e-9)
    idx = np.array([0, 1, 511, 1024, 1500, 2046])
    Lo, _ = ora.lnl_full_batch(ev, P[idx])
    np.testing.assert_allclose(e.lnl_full(P, q.FP64, allow_invalid=True)[idx], Lo, rtol=0,
                               atol=LNL_ATOL_FP64 * max(1.0, np.abs(Lo).max() / 100))
    # more sets than the ordering kernel reads in one pass (1024 threads x 4)
    P2 = synth.draw_params(rng, 4500, ev.inj)
    L2 = e.lnl_full(P2, q.FP64)
    e.set_launch(2, 256)
    L2u = e.lnl_full(P2, q.FP64)
    e.set_launch(0, 0)
    np.testing.assert_allclose(L2, L2u, rtol=0, atol=1e-9)


def test_device_call_captured_in_graph_and_on_two_streams(cfg2):
    """qcbc_lnl_full_dev on a caller's stream, at one tile per set (2048 sets) and at several tiles
    per set (40 sets, each finalised by its last tile): captured into a CUDA graph and replayed three
    times, and alternated between two streams, it gives the uncaptured result bit for bit (each call
    clears its own launch-order counts on its stream; the per-set tile counts are left at zero by
    every launch)."""
    import ctypes as C
    import torch
    from quickcbc_b200 import _lib
    ev, e = cfg2
    L = _lib.lib()
    s1, s2 = torch.cuda.Stream(), torch.cuda.Stream()
    for B, one_tile in ((2048, True), (40, False)):
        P = synth.draw_params(np.random.default_rng(2505), B, ev.inj)
        assert (e.get_launch(B, q.MIXED)[0] == 1) == one_tile
        dP, dL = q.DeviceBuffer(P.nbytes), q.DeviceBuffer(B * 8)
        dP.upload(P)

        def clear():                         # pageable uploads may finish after cudaMemcpy returns
            dL.upload(np.full(B, np.nan))
            assert L.qcbc_synchronize() == 0

        def call(prec, s):
            rc = L.qcbc_lnl_full_dev(e.handle, dP.ptr, B, dL.ptr, None, prec, C.c_void_p(s.cuda_stream))
            assert rc == 0, _lib.last_error()

        for prec in (q.FP64, q.MIXED):
            call(prec, s1)                   # grows the thread's scratch before capture
            s1.synchronize()
            want = dL.download((B,))
            np.testing.assert_allclose(want, e.lnl_full(P, prec), rtol=0, atol=0)
            for s in (s2, s1, s2):           # alternate streams, each call ordered after the last
                clear()
                call(prec, s)
                s.synchronize()
                assert np.array_equal(dL.download((B,)), want)
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g, stream=s1, capture_error_mode="thread_local"):
                call(prec, s1)
            for rep in range(3):
                clear()
                g.replay()
                torch.cuda.synchronize()
                assert np.array_equal(dL.download((B,)), want), f"B {B} replay {rep}"
            del g
        dP.free()
        dL.free()


def test_invalid_parameter_sets_flagged(ev1):
    ev, z, e = ev1
    P = z["params"][:4].copy()
    P[1, 2] = 1.5                      # spin outside [-1, 1]
    P[3, 6] = -np.inf                  # zero distance
    L = e.lnl_full(P, q.FP64, allow_invalid=True)
    assert L[1] == -1e20 and L[3] == -1e20
    np.testing.assert_allclose(L[[0, 2]], z["lnl"][[0, 2]], rtol=0, atol=LNL_ATOL_FP64)
    with pytest.raises(q.QcbcError) as ei:
        e.lnl_full(P, q.FP64)
    assert ei.value.code == 33


def test_empty_batch_and_empty_band(ev1, ora):
    ev, z, e = ev1
    assert e.lnl_full(np.zeros((0, 11)), q.FP64).shape == (0,)
    # very heavy system: fCut = 0.2/(M Msun_s) below fmin, template is zero everywhere
    p = z["params"][0].copy()
    p[0], p[1] = synth.masses_to_params(1500.0, 1400.0)
    Lo, _ = ora.lnl_full(ev, p)
    assert Lo == 0.0
    assert e.lnl_full(p, q.FP64)[0] == 0.0 and e.lnl_full(p, q.MIXED)[0] == 0.0
    # merger time 0: fbegin is NaN in the reference, every bin is zeroed
    p = z["params"][0].copy()
    p[5] = -1.0
    Lo, _ = ora.lnl_full(ev, p)
    assert e.lnl_full(p, q.FP64)[0] == Lo


@pytest.mark.parametrize("labels,Tobs,fs", [([1], 6.0, 2048.0), ([2, 1, 0], 5.0, 1024.0), ([0, 2], 4.0, 4096.0)])
def test_networks_and_non_power_of_two_durations(ora, labels, Tobs, fs):
    ev = synth.make_event(oracle_template(ora), labels=labels, Tobs=Tobs, fs=fs, fmin=16.0, m1=20.0, m2=15.0,
                          chi1=0.2, chi2=-0.3, snr=14.0, seed=int(Tobs * 100 + fs))
    e = q.Event.from_synthetic(ev)
    P = synth.draw_params(np.random.default_rng(7), 12, ev.inj, mc=(6.0, 30.0))
    Lo, _ = ora.lnl_full_batch(ev, P)
    np.testing.assert_allclose(e.lnl_full(P, q.FP64), Lo, rtol=0, atol=1e-8)
    assert np.max(np.abs(e.lnl_full(P, q.MIXED) - Lo)) <= LNL_ATOL_MIXED
    e.close()


def test_reference_signature_full_likelihood(ev1):
    ev, z, _ = ev1
    q.set_band(16.0, 1024.0)
    for bind in (False, True):
        for k in (0, 5, 12):
            L, rho = q.log_likelihood_full(ev.labels, ev.GMST, ev.D, z["params"][k], ev.freq, ev.SN, ev.N, ev.Tobs,
                                           bind=bind)
            assert abs(L - z["lnl"][k]) < LNL_ATOL_FP64
            np.testing.assert_allclose(rho, z["rho"][k], rtol=1e-9)


def test_fourier_nwip(ev1):
    ev, z, _ = ev1
    a, b, S = ev.D[0], z["h"][0][0], ev.SN[0]
    i = np.arange(64, 4096)
    want = 4.0 * np.sum((a[i] * b[i] + a[ev.N - i] * b[ev.N - i]) / S[i])
    got = q.fourier_nwip(a, b, S, 64, 4096, ev.N)
    assert abs(got - want) <= 1e-12 * max(1.0, abs(want))


# ---------------------------------------------------------------- heterodyne
def test_het_setup_tables_vs_reference(ev1, golden):
    ev, _, e = ev1
    h = golden("het1.npz")
    e.het_setup(h["pref"], h["fgrid"], int(h["MN"]), int(h["MM"]), int(h["J"]))
    t = e.het_export()
    assert abs(t["logLb"] - float(h["logLb"])) < 1e-8
    for k in ("amp", "phase", "IP", "SL", "lc", "ls", "aa", "rc", "rs"):
        np.testing.assert_allclose(t[k], h[k], rtol=0, atol=1e-10 * np.abs(h[k]).max(), err_msg=k)


def test_lnl_het_vs_reference(ev1, golden):
    ev, _, e = ev1
    h = golden("het1.npz")
    e.het_set(h)
    L = e.lnl_het(h["params"], q.FP64)
    np.testing.assert_allclose(L, h["lnl"], rtol=0, atol=LNL_ATOL_FP64)
    Lm = e.lnl_het(h["params"], q.MIXED)
    assert np.max(np.abs(Lm - h["lnl"])) <= LNL_ATOL_MIXED


def test_het_small_batches_match_large_bit_for_bit(ev1, golden):
    """Up to 128 sets the heterodyned lnL takes a block per set (the grid points spread over the
    block), above that a warp per set: a set gets the same bits either way, invalid sets -1e20."""
    ev, _, e = ev1
    h = golden("het1.npz")
    e.het_set(h)
    P = synth.jitter_params(np.random.default_rng(2507), 300, h["pref"], 1e-3)
    P[[4, 250], 2] = 1.5               # spin outside [-1, 1]
    for prec in (q.FP64, q.MIXED):
        big = e.lnl_het(P, prec, allow_invalid=True)                 # 300 sets: a warp per set
        assert big[4] == -1e20 and big[250] == -1e20
        small = np.concatenate([e.lnl_het(P[k:k + 100], prec, allow_invalid=True) for k in (0, 100, 200)])
        assert np.array_equal(big, small), prec
        assert np.array_equal(big[:3], [e.lnl_het(P[k:k + 1], prec)[0] for k in range(3)])


def test_reference_signature_heterodyne(ev1, golden):
    ev, _, _ = ev1
    h = golden("het1.npz")
    H = q.LegacyHet(ev.labels, ev.GMST, ev.Tobs, h["fgrid"], int(h["MN"]), int(h["MM"]), int(h["J"]))
    H.heterodyne(ev.D, h["pref"], ev.freq, ev.SN, ev.N)
    t = H.tables()
    assert abs(t["logLb"] - float(h["logLb"])) < 1e-8
    np.testing.assert_allclose(t["SL"], h["SL"], rtol=0, atol=1e-10 * np.abs(h["SL"]).max())
    for k in range(len(h["params"])):
        assert abs(H.lnl(h["params"][k]) - h["lnl"][k]) < LNL_ATOL_FP64


def _from_threads(nthreads, calls, fn):
    """fn(k) from `nthreads` host threads at once (ctypes releases the GIL in the call), thread t
    starting at call 5t: (results [thread][call], launches made by each thread)."""
    import threading
    from quickcbc_b200 import _lib
    out, launches = np.zeros((nthreads, calls)), np.zeros(nthreads, dtype=np.int64)
    go = threading.Barrier(nthreads)

    def work(t):
        go.wait()
        n0 = _lib.launch_count()
        for j in range(calls):
            k = (j + 5 * t) % calls
            out[t, k] = fn(k)
        launches[t] = _lib.launch_count() - n0
    ts = [threading.Thread(target=work, args=(t,)) for t in range(nthreads)]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    return out, launches


def test_concurrent_reference_calls_merge_bit_exact(ev1, golden):
    """12 threads calling log_likelihood_het and log_likelihood_full at once, as the reference's
    OpenMP chains do: their calls share launches (fewer launches than a lone caller makes) and each
    returns the bits of the same call made alone."""
    import ctypes as C
    from quickcbc_b200 import _lib, engine as eng
    ev, z, _ = ev1
    h = golden("het1.npz")
    H = q.LegacyHet(ev.labels, ev.GMST, ev.Tobs, h["fgrid"], int(h["MN"]), int(h["MM"]), int(h["J"]))
    H.heterodyne(ev.D, h["pref"], ev.freq, ev.SN, ev.N)
    P = [np.ascontiguousarray(p) for p in synth.jitter_params(np.random.default_rng(5), 40, h["pref"], 1e-3)]
    P[7][2] = 1.5                                  # spin outside [-1, 1]: -1e20 alone and merged
    lone = np.array([H.lnl(p) for p in P])
    assert lone[7] == -1e20 and np.all(lone[np.arange(40) != 7] > -1e20)
    out, launches = _from_threads(12, len(P), lambda k: H.lnl(P[k]))
    assert np.array_equal(out, np.broadcast_to(lone, out.shape))
    assert launches.sum() < 2 * out.size           # two launches per lone call: some calls merged

    q.set_band(16.0, 1024.0)
    nh = eng._NetHolder(ev.labels, ev.Tobs, ev.GMST)
    D, SN = eng._f64(ev.D), eng._f64(ev.SN)
    Dr, Sr = eng._rows(D), eng._rows(SN)
    f, rv = eng._rv(ev.freq)
    L = _lib.lib()

    def full(k):
        rho = np.zeros(4)
        return L.log_likelihood_full(nh.ref, Dr, eng._ptr(P[k]), C.byref(rv), Sr, eng._ptr(rho), ev.N, ev.Tobs)
    lone = np.array([full(k) for k in range(len(P))])
    assert lone[7] == -1e20
    np.testing.assert_allclose(lone[:5], [q.log_likelihood_full(ev.labels, ev.GMST, ev.D, P[k], ev.freq, ev.SN,
                                                                ev.N, ev.Tobs)[0] for k in range(5)], rtol=0, atol=0)
    out, launches = _from_threads(12, len(P), full)
    assert np.array_equal(out, np.broadcast_to(lone, out.shape))
    assert launches.sum() < 2 * out.size


def test_native_thread_timer(ev1, golden):
    """qcbc_time_dropin (the bench's per-call rates): 3 native threads x 5 merged calls each end on
    the lone call's lnL; a bad `which` is refused."""
    import ctypes as C
    from quickcbc_b200 import _lib, engine as eng
    ev, _, _ = ev1
    h = golden("het1.npz")
    H = q.LegacyHet(ev.labels, ev.GMST, ev.Tobs, h["fgrid"], int(h["MN"]), int(h["MM"]), int(h["J"]))
    H.heterodyne(ev.D, h["pref"], ev.freq, ev.SN, ev.N)
    P = np.ascontiguousarray(h["params"][:1])
    L = _lib.lib()
    secs, last = C.c_double(0.0), np.zeros(3)
    rc = L.qcbc_time_dropin(1, H.nh.ref, C.byref(H.het), None, None, None, ev.N, ev.Tobs, eng._ptr(P), 1, 5, 3,
                            C.byref(secs), eng._ptr(last))
    assert rc == 0, _lib.last_error()
    assert secs.value > 0 and np.all(last == H.lnl(P[0]))
    rc = L.qcbc_time_dropin(2, H.nh.ref, C.byref(H.het), None, None, None, ev.N, ev.Tobs, eng._ptr(P), 1, 5, 3,
                            C.byref(secs), None)
    assert rc == -1 and "which" in _lib.last_error()


def test_cfg3_heterodyne_long_signal(ora):
    """Config 3 (3 det, 128 s, 4096 Hz, BNS): reference het grid, tables set up on
    the GPU in FP64, het lnL against the reference's value and the oracle."""
    g = load_golden("grid3.npz")
    ev = synth.config_event(3, oracle_template(ora))
    assert abs(ev.GMST - float(g["GMST"])) == 0.0
    e = q.Event.from_synthetic(ev)
    e.het_setup(ev.inj, g["fgrid"], int(g["MN"]), int(g["MM"]), int(g["J"]))
    t = e.het_export()
    assert abs(t["logLb"] - float(g["logLb"])) < 1e-6
    L = e.lnl_het(g["params"], q.FP64)
    np.testing.assert_allclose(L, g["lnl"], rtol=0, atol=1e-6)
    Lm = e.lnl_het(g["params"], q.MIXED)
    assert np.max(np.abs(Lm - g["lnl"])) <= LNL_ATOL_MIXED
    to = ora.heterodyne(ev, ev.inj, g["fgrid"], int(g["MN"]), int(g["MM"]), int(g["J"]))
    Lo, _ = ora.lnl_het_batch(ev, to, g["params"])
    np.testing.assert_allclose(L, Lo, rtol=0, atol=1e-7)
    e.close()


def test_cfg3_full_lnl_largest_size(ora):
    """Config 3 at full size (3 det, 128 s, 4096 Hz: 3 x 128512 bins per set), the largest
    workload of the suite: FP64 against the oracle on 6 sets, mixed against FP64 on 256 sets."""
    ev = synth.config_event(3, oracle_template(ora))
    e = q.Event.from_synthetic(ev)
    P = synth.jitter_params(np.random.default_rng(3303), 256, ev.inj, scale=1e-5)
    L64 = e.lnl_full(P, q.FP64)
    Lo, _ = ora.lnl_full_batch(ev, P[:6])
    np.testing.assert_allclose(L64[:6], Lo, rtol=0, atol=1e-6)
    assert np.max(np.abs(e.lnl_full(P, q.MIXED) - L64)) <= LNL_ATOL_MIXED
    e.close()

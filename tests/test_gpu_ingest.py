"""Input stage on the GPU (include/qcbc_ingest.h) against the reference's outputs in
tests/golden/ingest1.npz (made by running the reference) and the oracle build:

* conditioning (Tukey window, real FFT, sqrt(Tobs)/N; QuickCBC.c:244-258, 309-313):
  |D - D_ref| <= 1e-13 of max |D_ref| per detector, and the lnL on the conditioned data
  within 1e-8 of the reference's;
* the whole input stage from framed_/spec_ files: the same D as conditioning the read series,
  SN equal to the file's values, lnL within 1e-8 of the reference's;
* makespec (Utilities.c:1908) through the drop-in symbol and the PSD model: relative 1e-12
  of the reference's, per bin, ragged knot and line counts across detectors;
* the noisemarg redraw on an event (QuickCBC.c:1994-2010): lnL bit-identical to an event opened
  with the drawn PSD, full and heterodyned, FP64 and mixed; lnL within 1e-8 of the reference's.
"""
import numpy as np
import pytest

import quickcbc_b200 as q
from quickcbc_b200 import ingest, synth
from quickcbc_b200._lib import QcbcError

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def g(golden):
    return golden("ingest1.npz")


def open_event(g, D, SN):
    return q.Event(g["labels"], float(g["Tobs"]), float(g["GMST"]), int(g["N"]), D, SN, fmin=float(g["fmin"]))


def close_rows(A, B, rel):
    for a, b in zip(np.atleast_2d(A), np.atleast_2d(B)):
        assert np.max(np.abs(a - b)) <= rel * np.max(np.abs(b)), np.max(np.abs(a - b)) / np.max(np.abs(b))


def test_condition_data_vs_reference(g):
    D = ingest.condition_data(g["x"], float(g["Tobs"]))
    close_rows(D, g["D"], 1e-13)
    e = open_event(g, D, g["SN"])
    np.testing.assert_allclose(e.lnl_full(g["params"], q.FP64), g["lnl"], rtol=0, atol=1e-8)
    e.close()


def test_condition_data_larger_sizes_vs_oracle():
    ref = pytest.importorskip("oracle.ref")
    rng = np.random.default_rng(31)
    for N, Tobs in ((1 << 13, 2.0), (1 << 19, 128.0)):
        x = rng.normal(size=(1, N)) * 1e-21
        D = ingest.condition_data(x, Tobs)
        close_rows(D, ref.condition(x[0], Tobs), 1e-13)


def test_condition_data_rejects_bad_lengths():
    for N in (6, 12, 1000):
        with pytest.raises(QcbcError):
            ingest.condition_data(np.zeros((1, N)), 4.0)


def test_load_analysis_from_files(g, tmp_path):
    labels, Tobs, ttrig = [int(v) for v in g["labels"]], float(g["Tobs"]), 1187008882.43
    synth.write_analysis_files(str(tmp_path), labels, Tobs, ttrig, g["x"], g["SN"])
    D, SN, SM = ingest.load_analysis(str(tmp_path), Tobs, ttrig, labels)
    assert np.array_equal(SN, g["SN"]) and np.array_equal(SM, g["SN"])
    assert np.array_equal(D, ingest.condition_data(g["x"], Tobs))
    e = open_event(g, D, SN)
    np.testing.assert_allclose(e.lnl_full(g["params"], q.FP64), g["lnl"], rtol=0, atol=1e-8)
    e.close()


def model_from(g):
    return ingest.PsdModel(g["ffit"], g["xspline"], g["lines"], g["nspline"], g["nlines"])


def test_makespec_drop_in_vs_reference(g):
    Tobs, N = float(g["Tobs"]), int(g["N"])
    for k in range(g["xspline"].shape[1]):
        for i in range(len(g["labels"])):
            n, m = g["nspline"][i], g["nlines"][i]
            L = g["lines"][i, k, :m]
            S = ingest.makespec(g["ffit"][i, :n], g["xspline"][i, k, :n], *L.T, Tobs, N)
            np.testing.assert_allclose(S, g["makespec"][k, i], rtol=1e-12, atol=0)


def test_psd_model_vs_reference_and_files(g, tmp_path):
    Tobs, N = float(g["Tobs"]), int(g["N"])
    m = model_from(g)
    assert (m.nifo, m.nsample) == (2, 3)
    for k in range(3):
        np.testing.assert_allclose(m.draw(k, Tobs, N), g["makespec"][k], rtol=1e-12, atol=0)
    labels = [int(v) for v in g["labels"]]
    synth.write_psd_model_files(str(tmp_path), labels, g["nspline"], g["nlines"], g["ffit"], g["xspline"], g["lines"])
    mf = ingest.PsdModel.open(str(tmp_path), labels)
    for k in range(3):
        assert np.array_equal(mf.draw(k, Tobs, N), m.draw(k, Tobs, N))
    with pytest.raises(QcbcError):
        m.draw(3, Tobs, N)
    with pytest.raises(QcbcError) as ei:
        m.draw(0, Tobs, 4 * N)                # bins above the last knot: the reference's spline has no extrapolation
    assert ei.value.code == 33
    m.close()
    mf.close()


def test_psd_model_larger_size_vs_oracle(g):
    """Config-3 sized spectrum (Tobs 128 s, N = 2^19) against the oracle build's makespec."""
    ref = pytest.importorskip("oracle.ref")
    rng = np.random.default_rng(32)
    Tobs, N = 128.0, 1 << 19
    ns, nl, ffit, xs, L = synth.psd_model_arrays(rng, 3, Tobs, N, nsample=2)
    m = ingest.PsdModel(ffit, xs, L, ns, nl)
    S = m.draw(1, Tobs, N)
    for i in range(3):
        n, k = ns[i], nl[i]
        R = ref.makespec(ffit[i, :n], xs[i, 1, :n], *L[i, 1, :k].T, Tobs, N)
        np.testing.assert_allclose(S[i], R, rtol=1e-12, atol=0)
    m.close()


def test_psd_model_rejects_bad_knots(g):
    ffit = g["ffit"].copy()
    ffit[0, 3] = ffit[0, 2]
    with pytest.raises(QcbcError):
        ingest.PsdModel(ffit, g["xspline"], g["lines"], g["nspline"], g["nlines"])


def test_noisemarg_redraw_on_event(g, golden):
    """set_psd_sample equals opening the event with the drawn PSD, bit for bit, for the full and
    the heterodyned likelihood (tables rebuilt about the same point and grid)."""
    Tobs, N = float(g["Tobs"]), int(g["N"])
    h = golden("het1.npz")
    m = model_from(g)
    e = open_event(g, g["D"], g["SN"])
    e.het_setup(h["pref"], h["fgrid"], int(h["MN"]), int(h["MM"]), 2)
    P = g["params"]
    L0 = e.lnl_het(P, q.FP64)
    e.set_psd_sample(m, 1)
    S1 = m.draw(1, Tobs, N)
    fresh = open_event(g, g["D"], S1)
    fresh.het_setup(h["pref"], h["fgrid"], int(h["MN"]), int(h["MM"]), 2)
    for prec in (q.FP64, q.MIXED):
        assert np.array_equal(e.lnl_full(P, prec), fresh.lnl_full(P, prec))
        assert np.array_equal(e.lnl_het(P, prec), fresh.lnl_het(P, prec))
    np.testing.assert_allclose(e.lnl_full(P, q.FP64), g["lnl_sample1"], rtol=0, atol=1e-8)
    assert not np.allclose(e.lnl_het(P, q.FP64), L0), "the heterodyne tables follow the new PSD"
    # back to the file PSD through the host form
    e.set_psd(g["SN"])
    back = open_event(g, g["D"], g["SN"])
    assert np.array_equal(e.lnl_full(P, q.MIXED), back.lnl_full(P, q.MIXED))
    np.testing.assert_allclose(e.lnl_full(P, q.FP64), g["lnl"], rtol=0, atol=1e-8)
    for x in (e, fresh, back):
        x.close()
    m.close()


def test_redraw_in_a_batch_slot(g):
    """An event in a multi-event batch is set into its slot again after a PSD change."""
    m = model_from(g)
    e = open_event(g, g["D"], g["SN"])
    b = q.Batch([e])
    P = g["params"]
    e.set_psd_sample(m, 2)
    b.set_slot(0, e)
    Lb = b.lnl(np.zeros(len(P), dtype=np.int32), P, q.FP64)
    np.testing.assert_allclose(Lb, e.lnl_full(P, q.FP64), rtol=0, atol=1e-9)
    b.close()
    e.close()
    m.close()

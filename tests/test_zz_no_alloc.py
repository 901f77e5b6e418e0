"""The allocation-free entry point qcbc_lnl_full_noalloc, for callers that
cannot allocate device memory at call time (code inside another framework's
runtime, which owns the device memory; services with a fixed memory budget).

It is called through the C ABI on device buffers owned by the caller, twice in
a row, and must give what the existing entry point qcbc_lnl_full_dev gives for
the same inputs, within the tolerances of the other parity tests.  This file is
collected last, and it also passes on its own in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

import quickcbc_b200 as q
from quickcbc_b200 import _lib, synth

pytestmark = pytest.mark.gpu

TOL = {q.FP64: 1e-8, q.MIXED: 1e-3}


def _dev_lnl(fn, e, dP, B, prec, dL, dR):
    rc = fn(e.handle, dP.ptr, B, dL.ptr, dR.ptr, prec, None)
    assert rc == 0, _lib.last_error()
    assert _lib.lib().qcbc_synchronize() == 0
    return dL.download((B,)), dR.download((B, e.nifo))


def test_noalloc_matches_existing_entry_point_on_two_calls(cfg1_event):
    ev, z = cfg1_event
    e = q.Event.from_synthetic(ev)
    P = np.vstack([z["params"], synth.jitter_params(np.random.default_rng(41), 48, ev.inj)])
    B = len(P)
    dP = q.DeviceBuffer(P.nbytes)
    dP.upload(P)
    dL, dR = q.DeviceBuffer(B * 8), q.DeviceBuffer(B * 8 * e.nifo)
    L = _lib.lib()
    for prec in (q.FP64, q.MIXED):
        want, want_rho = _dev_lnl(L.qcbc_lnl_full_dev, e, dP, B, prec, dL, dR)
        for call in range(2):
            dL.upload(np.full(B, np.nan))
            got, got_rho = _dev_lnl(L.qcbc_lnl_full_noalloc, e, dP, B, prec, dL, dR)
            assert np.all(np.isfinite(got)), f"call {call}"
            np.testing.assert_allclose(got, want, rtol=0, atol=TOL[prec], err_msg=f"call {call}")
            np.testing.assert_allclose(got_rho, want_rho, rtol=1e-6, atol=1e-9)
    # against the reference's own values on the golden parameter sets
    np.testing.assert_allclose(_dev_lnl(L.qcbc_lnl_full_noalloc, e, dP, B, q.FP64, dL, dR)[0][:16], z["lnl"],
                               rtol=0, atol=TOL[q.FP64])
    for buf in (dP, dL, dR):
        buf.free()
    e.close()


def test_noalloc_rejects_oversized_batch(cfg1_event):
    ev, _ = cfg1_event
    e = q.Event.from_synthetic(ev)
    B = 4097                                   # QCBC_NOALLOC_MAX_SETS + 1
    dP = q.DeviceBuffer(B * 11 * 8)
    dL = q.DeviceBuffer(B * 8)
    rc = _lib.lib().qcbc_lnl_full_noalloc(e.handle, dP.ptr, B, dL.ptr, None, q.FP64, None)
    assert rc == -1
    assert "QCBC_NOALLOC_MAX_SETS" in _lib.last_error()
    dP.free()
    dL.free()
    e.close()

"""Host-side interface of the GPU likelihood engine.

Two layers, both thin wrappers over the C ABI:

* ``Event``: one analysis (network, data, PSD) resident on the device, with
  batched full and heterodyned likelihoods in FP64 or mixed precision;
* the QuickCBC reference's own entry points under their own names
  (``fulltemplates``, ``fullphaseamp``, ``log_likelihood_full``, ...), called
  through the drop-in symbols of the library with the reference's struct
  layouts, so tests read like calls into the reference.
"""
from __future__ import annotations

import ctypes as C
import numpy as np

from . import _lib
from ._lib import FP64, MIXED, QcbcError, check, lib

_PD = C.POINTER(C.c_double)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _ptr(a):
    return a.ctypes.data_as(_PD)


def precision_code(p) -> int:
    if p in (FP64, "fp64", "FP64", "double"):
        return FP64
    if p in (MIXED, "mixed", "MIXED"):
        return MIXED
    raise ValueError(f"unknown precision {p!r}")


class Event:
    """An analysis resident on the GPU (qcbc_event_open).

    D: [nifo, N] half-complex rows; SN: [nifo, >= N/2] PSD rows.
    """

    def __init__(self, labels, Tobs, GMST, N, D, SN, fmin=16.0, fmax=1024.0):
        self.labels = np.ascontiguousarray(labels, dtype=np.int32)
        self.nifo = len(self.labels)
        self.Tobs, self.GMST, self.N = float(Tobs), float(GMST), int(N)
        self.fmin, self.fmax = float(fmin), float(fmax)
        D = _f64(D)
        SN = _f64(SN)
        check(lib().qcbc_init(0))
        self._h = lib().qcbc_event_open(self.nifo, self.labels.ctypes.data_as(C.POINTER(C.c_int)), self.Tobs,
                                        self.GMST, self.N, _ptr(D), D.shape[1], _ptr(SN), SN.shape[1], self.fmin,
                                        self.fmax)
        if not self._h:
            raise QcbcError(-1, _lib.last_error())

    @classmethod
    def from_synthetic(cls, ev):
        return cls(ev.labels, ev.Tobs, ev.GMST, ev.N, ev.D, ev.SN, fmin=ev.fmin)

    @property
    def handle(self):
        return self._h

    def close(self):
        if getattr(self, "_h", None):
            lib().qcbc_event_close(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def device_bytes(self) -> int:
        return int(lib().qcbc_event_device_bytes(self._h))

    # ---- full likelihood
    def lnl_full(self, params, precision=FP64, rho=False, allow_invalid=False):
        P = _f64(np.atleast_2d(params))
        B = P.shape[0]
        out = np.empty(B)
        r = np.empty((B, self.nifo)) if rho else None
        rc = lib().qcbc_lnl_full(self._h, P.ctypes.data, B, out.ctypes.data, r.ctypes.data if rho else None,
                                 precision_code(precision))
        if rc != 0 and not (allow_invalid and rc == _lib.QCBC_EDOM):
            check(rc)
        return (out, r) if rho else out

    def lnl_intrinsic(self, params, precision=FP64, snrsq=False, allow_invalid=False):
        """Batched log_likelihood_intrinsic: params [B][7 + 3 (nifo - 1)] (templates' layout)."""
        P = _f64(np.atleast_2d(params))
        if P.shape[1] != 7 + 3 * (self.nifo - 1):
            raise ValueError(f"intrinsic parameter sets have {7 + 3 * (self.nifo - 1)} entries for {self.nifo} detectors")
        B = P.shape[0]
        out = np.zeros(B)
        r = np.zeros((B, self.nifo)) if snrsq else None
        rc = lib().qcbc_lnl_intrinsic(self._h, _ptr(P), B, _ptr(out), _ptr(r) if snrsq else None,
                                      precision_code(precision))
        if rc != 0 and not (allow_invalid and rc == _lib.QCBC_EDOM):
            check(rc)
        return (out, r) if snrsq else out

    def set_launch(self, tiles=0, threads=0):
        check(lib().qcbc_set_full_launch(self._h, tiles, threads))

    def get_launch(self, B, precision=FP64):
        t, th = C.c_int(), C.c_int()
        check(lib().qcbc_get_full_launch(self._h, B, precision_code(precision), C.byref(t), C.byref(th)))
        return t.value, th.value

    # ---- heterodyne
    def het_setup(self, pref, fgrid, MN, MM, J=2):
        g = np.ascontiguousarray(fgrid, dtype=np.int32)
        check(lib().qcbc_het_setup(self._h, _ptr(_f64(pref)), g.ctypes.data_as(C.POINTER(C.c_int)), len(g),
                                   int(MN), int(MM), int(J)))

    def het_set(self, t):
        keep = {k: _f64(t[k]) for k in ("freq", "amp", "phase", "IP", "SL", "lc", "ls", "aa", "rc", "rs")}
        g = np.ascontiguousarray(t["fgrid"], dtype=np.int32)
        M, J = len(g), int(t["J"])
        T = _lib.HetTables(M=M, MN=int(t["MN"]), MM=int(t["MM"]), J=J, NR=(M - 1) // J, logLb=float(t["logLb"]),
                           fgrid=g.ctypes.data_as(C.POINTER(C.c_int)), **{k: _ptr(v) for k, v in keep.items()})
        check(lib().qcbc_het_set(self._h, C.byref(T)))

    def het_export(self):
        M, J, NR, MN, MM = (C.c_int() for _ in range(5))
        check(lib().qcbc_het_sizes(self._h, C.byref(M), C.byref(J), C.byref(NR), C.byref(MN), C.byref(MM)))
        M, J, NR, MN, MM = M.value, J.value, NR.value, MN.value, MM.value
        nI = self.nifo
        t = dict(fgrid=np.zeros(M, dtype=np.int32), freq=np.zeros(M), amp=np.zeros((nI, M)),
                 phase=np.zeros((nI, M)), IP=np.zeros((NR, J + 1, J + 1)), SL=np.zeros((NR, nI, J + 1)),
                 lc=np.zeros((NR, nI, J + 1)), ls=np.zeros((NR, nI, J + 1)), aa=np.zeros((nI, NR)),
                 rc=np.zeros((nI, NR)), rs=np.zeros((nI, NR)))
        L = C.c_double()
        check(lib().qcbc_het_export(self._h, t["fgrid"].ctypes.data_as(C.POINTER(C.c_int)),
                                    *[_ptr(t[k]) for k in ("freq", "amp", "phase", "IP", "SL", "lc", "ls", "aa",
                                                           "rc", "rs")], C.byref(L)))
        t.update(logLb=L.value, M=M, J=J, NR=NR, MN=MN, MM=MM, Nifo=nI)
        return t

    def lnl_het(self, params, precision=FP64, allow_invalid=False):
        P = _f64(np.atleast_2d(params))
        out = np.empty(P.shape[0])
        rc = lib().qcbc_lnl_het(self._h, P.ctypes.data, P.shape[0], out.ctypes.data, precision_code(precision))
        if rc != 0 and not (allow_invalid and rc == _lib.QCBC_EDOM):
            check(rc)
        return out

    def het_space(self, params, pmin, pmax):
        """Heterodyne grid search about params (het_space): returns (fgrid, MN, MM) for het_setup."""
        M, MN, MM = C.c_int(), C.c_int(), C.c_int()
        check(lib().qcbc_het_space(self._h, _ptr(_f64(params)), _ptr(_f64(pmin)), _ptr(_f64(pmax)), C.byref(M),
                                   C.byref(MN), C.byref(MM)))
        g = np.zeros(M.value, dtype=np.int32)
        check(lib().qcbc_het_space_grid(self._h, g.ctypes.data_as(C.POINTER(C.c_int))))
        return g, MN.value, MM.value

    def het_diff(self, params_a, params_b):
        """Heterodyned squared distance between the templates of paired rows (het_diff)."""
        A, Bp = _f64(np.atleast_2d(params_a)), _f64(np.atleast_2d(params_b))
        out = np.zeros(A.shape[0])
        check(lib().qcbc_het_diff(self._h, _ptr(A), _ptr(Bp), A.shape[0], _ptr(out)))
        return out

    def set_psd(self, SN):
        """A new PSD, SN [nifo, >= N/2] (qcbc_event_set_psd): weighted data and heterodyne tables
        built by het_setup are rebuilt on the device."""
        SN = _f64(np.atleast_2d(SN))
        if SN.shape[0] != self.nifo or SN.shape[1] < self.N // 2:
            raise ValueError("SN must be [nifo, >= N/2]")
        check(lib().qcbc_event_set_psd(self._h, _ptr(SN), SN.shape[1]))

    def set_psd_sample(self, model, k):
        """noisemarg redraw (qcbc_event_set_psd_sample): PSD sample k of `model` (ingest.PsdModel)
        evaluated on the device into this event, then the same rebuilds as set_psd."""
        check(lib().qcbc_event_set_psd_sample(self._h, model.handle, int(k)))

    def het_fisher(self, params):
        """Fisher matrices [B][11][11] from the heterodyne tables (Fisher_Het), one launch for all sets."""
        P = _f64(np.atleast_2d(params))
        F = np.zeros((P.shape[0], 11, 11))
        check(lib().qcbc_het_fisher(self._h, _ptr(P), P.shape[0], _ptr(F)))
        return F


class Batch:
    """Several open events evaluated together (qcbc_batch_create / qcbc_lnl_multi).

    Parameter set b belongs to events[event_of[b]]; networks, durations, sample
    rates and bands may differ between events.  One persistent kernel serves all
    sets, launched as one captured CUDA graph per call.
    """

    def __init__(self, events):
        self.events = list(events)
        arr = (C.c_void_p * len(self.events))(*[e.handle for e in self.events])
        self._h = lib().qcbc_batch_create(arr, len(self.events))
        if not self._h:
            raise QcbcError(-1, _lib.last_error())

    def set_slot(self, slot, event):
        """(Re)fill slot `slot` with `event` (qcbc_batch_set_slot), e.g. after its PSD or heterodyne
        tables changed; None empties it."""
        check(lib().qcbc_batch_set_slot(self._h, int(slot), event.handle if event is not None else None))
        self.events[slot] = event

    def close(self):
        if getattr(self, "_h", None):
            lib().qcbc_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_tiling(self, tile_bins=0, threads=0):
        check(lib().qcbc_batch_set_tiling(self._h, int(tile_bins), int(threads)))

    def tiling(self):
        t, th = C.c_int(), C.c_int()
        check(lib().qcbc_batch_get_tiling(self._h, C.byref(t), C.byref(th)))
        return t.value, th.value

    def autotune(self, event_of, params, precision=MIXED):
        eo = np.ascontiguousarray(event_of, dtype=np.int32)
        P = _f64(np.atleast_2d(params))
        check(lib().qcbc_batch_autotune(self._h, eo.ctypes.data_as(C.POINTER(C.c_int)), _ptr(P), P.shape[0],
                                        precision_code(precision)))
        return self.tiling()

    def lnl(self, event_of, params, precision=MIXED, rho=False, allow_invalid=False):
        eo = np.ascontiguousarray(event_of, dtype=np.int32)
        P = _f64(np.atleast_2d(params))
        B = P.shape[0]
        assert eo.shape == (B,)
        out = np.zeros(B)
        r = np.zeros((B, 3)) if rho else None
        rc = lib().qcbc_lnl_multi(self._h, eo.ctypes.data_as(C.POINTER(C.c_int)), _ptr(P), B, _ptr(out),
                                  _ptr(r) if rho else None, precision_code(precision))
        if rc != 0 and not (allow_invalid and rc == _lib.QCBC_EDOM):
            check(rc)
        return (out, r) if rho else out

    def lnl_het(self, event_of, params, precision=MIXED, allow_invalid=False):
        """Heterodyned lnL of sets of many events (each event's tables as of when the batch
        took it; events without tables give -1e20)."""
        eo = np.ascontiguousarray(event_of, dtype=np.int32)
        P = _f64(np.atleast_2d(params))
        B = P.shape[0]
        assert eo.shape == (B,)
        out = np.zeros(B)
        rc = lib().qcbc_lnl_multi_het(self._h, eo.ctypes.data_as(C.POINTER(C.c_int)), _ptr(P), B, _ptr(out),
                                      precision_code(precision))
        if rc != 0 and not (allow_invalid and rc == _lib.QCBC_EDOM):
            check(rc)
        return out

    def time(self, B, precision=MIXED, iters=10, flush_l2=True):
        ms = (C.c_float * iters)()
        check(lib().qcbc_time_lnl_multi(self._h, int(B), precision_code(precision), iters, int(flush_l2), ms))
        return np.array(ms[:])


class DeviceBuffer:
    """Raw device allocation owned by the engine (for device-resident inputs)."""

    def __init__(self, nbytes):
        check(lib().qcbc_init(0))
        self.nbytes = int(nbytes)
        self.ptr = lib().qcbc_device_alloc(self.nbytes)
        if not self.ptr:
            raise QcbcError(-3, _lib.last_error())

    def upload(self, arr):
        a = np.ascontiguousarray(arr)
        assert a.nbytes <= self.nbytes
        check(lib().qcbc_memcpy_h2d(self.ptr, a.ctypes.data, a.nbytes))

    def download(self, shape, dtype=np.float64):
        out = np.empty(shape, dtype=dtype)
        check(lib().qcbc_memcpy_d2h(out.ctypes.data, self.ptr, out.nbytes))
        return out

    def free(self):
        if self.ptr:
            lib().qcbc_device_free(self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def time_lnl_full(event: Event, dbuf: DeviceBuffer, B, precision, iters, flush_l2=True, kernel_times=True):
    """Device times (ms) of `iters` full-likelihood steps, and of their lnL kernels when
    kernel_times (events recorded around the kernel; without them the step runs as a plain call
    does, the lnL kernel overlapping the setup's tail)."""
    ms = (C.c_float * iters)()
    kms = (C.c_float * iters)()
    check(lib().qcbc_time_lnl_full(event.handle, dbuf.ptr, B, precision_code(precision), iters, int(flush_l2), ms,
                                   kms if kernel_times else None))
    return np.array(ms[:]), (np.array(kms[:]) if kernel_times else None)


def time_lnl_het(event: Event, dbuf: DeviceBuffer, B, precision, iters, flush_l2=True):
    ms = (C.c_float * iters)()
    check(lib().qcbc_time_lnl_het(event.handle, dbuf.ptr, B, precision_code(precision), iters, int(flush_l2), ms))
    return np.array(ms[:])


# ============================================================ reference-signature calls
class _NetHolder:
    """struct Net with the arrays it points to kept alive."""

    def __init__(self, labels, Tobs, GMST):
        self.labels = np.ascontiguousarray(labels, dtype=np.int32)
        self.tds = np.zeros(len(self.labels) + 1)
        self.net = _lib.Net(Nifo=len(self.labels), Tobs=float(Tobs), tmax=float(Tobs) - 0.5,
                            tmin=max(float(Tobs) - 3.5, 1.5), GMST=float(GMST),
                            labels=self.labels.ctypes.data_as(C.POINTER(C.c_int)), tds=_ptr(self.tds))

    @property
    def ref(self):
        return C.byref(self.net)


def _rows(arr2d):
    """double** over the rows of a C-contiguous 2-D array."""
    R = (_PD * (arr2d.shape[0] + 1))()
    for i in range(arr2d.shape[0]):
        R[i] = C.cast(arr2d.ctypes.data + i * arr2d.strides[0], _PD)
    return R


def _rv(freq):
    f = _f64(freq)
    return f, _lib.RealVector(data=_ptr(f), length=len(f))


def fulltemplates(labels, GMST, freq, params, N):
    nh = _NetHolder(labels, 1.0 / freq[1], GMST)
    h = np.zeros((len(nh.labels), N))
    f, rv = _rv(freq)
    p = _f64(params).copy()
    lib().fulltemplates(nh.ref, _rows(h), C.byref(rv), _ptr(p), N)
    return h


def fullphaseamp(labels, GMST, Tobs, freq, params, N):
    nh = _NetHolder(labels, Tobs, GMST)
    n = N // 2
    a = np.zeros((len(nh.labels), n))
    ph = np.zeros((len(nh.labels), n))
    f, rv = _rv(freq)
    p = _f64(params).copy()
    lib().fullphaseamp(nh.ref, _rows(a), _rows(ph), C.byref(rv), _ptr(p), N)
    return a, ph


def amp_phase(freq, phi0, fRef, m1_SI, m2_SI, chi1, chi2, dist):
    """IMRPhenomDGenerateh22FDAmpPhase through the drop-in symbol; returns (status, amp, phase)."""
    f, rv = _rv(freq)
    out = C.POINTER(_lib.AmpPhaseFDWaveform)()
    st = lib().IMRPhenomDGenerateh22FDAmpPhase(C.byref(out), C.byref(rv), phi0, fRef, m1_SI, m2_SI, chi1, chi2,
                                               dist)
    if st != 0:
        return st, None, None
    n = out.contents.length
    amp = np.ctypeslib.as_array(out.contents.amp, shape=(n,)).copy()
    ph = np.ctypeslib.as_array(out.contents.phase, shape=(n,)).copy()
    libc = C.CDLL(None)
    libc.free.argtypes = [C.c_void_p]
    for p in (out.contents.freq, out.contents.amp, out.contents.phase):
        libc.free(C.cast(p, C.c_void_p))
    libc.free(C.cast(out, C.c_void_p))
    return st, amp, ph


def templates(labels, GMST, freq, params, N):
    """templates (QuickCBC.c:3527) through the drop-in symbol; intrinsic parameters."""
    nh = _NetHolder(labels, 1.0 / freq[1], GMST)
    h = np.zeros((len(nh.labels), N))
    f, rv = _rv(freq)
    p = _f64(params).copy()
    lib().templates(nh.ref, _rows(h), C.byref(rv), _ptr(p), N)
    return h


def ampphase(freq, params, N):
    """AmpPhase (QuickCBC.c:3395) through the drop-in symbol: (Af, Pf) over N/2 bins, entry 0 zero."""
    f, rv = _rv(freq)
    Af, Pf = np.zeros(N // 2), np.zeros(N // 2)
    p = _f64(params).copy()
    lib().AmpPhase(_ptr(Af), _ptr(Pf), C.byref(rv), _ptr(p), N)
    return Af, Pf


def log_likelihood_intrinsic(labels, GMST, D, params, freq, SN, N, Tobs):
    nh = _NetHolder(labels, Tobs, GMST)
    D, SN = _f64(D), _f64(SN)
    f, rv = _rv(freq)
    p = _f64(params).copy()
    return lib().log_likelihood_intrinsic(nh.ref, _rows(D), _ptr(p), C.byref(rv), _rows(SN), N, Tobs)


def fourier_nwip(a, b, S, imin, imax, N):
    a, b, S = _f64(a), _f64(b), _f64(S)
    return lib().fourier_nwip(_ptr(a), _ptr(b), _ptr(S), imin, imax, N)


def set_band(fmin, fmax):
    check(lib().qcbc_set_band(float(fmin), float(fmax)))


def log_likelihood_full(labels, GMST, D, params, freq, SN, N, Tobs, bind=False):
    nh = _NetHolder(labels, Tobs, GMST)
    D, SN = _f64(D), _f64(SN)
    Dr, Sr = _rows(D), _rows(SN)
    f, rv = _rv(freq)
    rho = np.zeros(len(nh.labels) + 1)
    if bind:
        check(lib().qcbc_bind_data(nh.ref, Dr, Sr, N, Tobs))
    p = _f64(params).copy()
    L = lib().log_likelihood_full(nh.ref, Dr, _ptr(p), C.byref(rv), Sr, _ptr(rho), N, Tobs)
    return L, rho[: len(nh.labels)]


def het_space(labels, GMST, Tobs, params, pmin, pmax, freq, SN, N):
    """het_space (QuickCBC.c:4570) through the drop-in symbol: (fgrid, MN, MM, J, NR)."""
    nh = _NetHolder(labels, Tobs, GMST)
    SN = _f64(SN)
    f, rv = _rv(freq)
    het = _lib.Het()
    lib().het_space(nh.ref, C.byref(het), _ptr(_f64(params).copy()), _ptr(_f64(pmin).copy()),
                    _ptr(_f64(pmax).copy()), C.byref(rv), _rows(SN), N, Tobs)
    if not het.fgrid:
        raise QcbcError(-1, _lib.last_error())
    g = np.array([het.fgrid[i] for i in range(het.M)], dtype=np.int32)
    libc = C.CDLL(None)
    libc.free.argtypes = [C.c_void_p]
    libc.free(C.cast(het.freq.contents.data, C.c_void_p))
    libc.free(C.cast(het.freq, C.c_void_p))
    libc.free(C.cast(het.fgrid, C.c_void_p))
    return g, het.MN, het.MM, het.J, het.NR


class LegacyHet:
    """struct Het filled by the drop-in heterodyne() (QuickCBC.c:5112)."""

    def __init__(self, labels, GMST, Tobs, fgrid, MN, MM, J=2):
        self.nh = _NetHolder(labels, Tobs, GMST)
        self.fgrid = np.ascontiguousarray(fgrid, dtype=np.int32)
        M = len(self.fgrid)
        self.freq = self.fgrid.astype(np.float64) / Tobs
        self.rv = _lib.RealVector(data=_ptr(self.freq), length=M)
        self.het = _lib.Het(M=M, MM=int(MM), MN=int(MN), J=J, NR=(M - 1) // J,
                            fgrid=self.fgrid.ctypes.data_as(C.POINTER(C.c_int)), freq=C.pointer(self.rv))
        self.Tobs = Tobs

    def heterodyne(self, D, params, freq, SN, N):
        D, SN = _f64(D), _f64(SN)
        f, rv = _rv(freq)
        p = _f64(params).copy()
        lib().heterodyne(self.nh.ref, C.byref(self.het), _rows(D), _ptr(p), C.byref(rv), _rows(SN), N, self.Tobs)
        if not self.het.IP:
            raise QcbcError(-1, _lib.last_error())

    def lnl(self, params):
        p = _f64(params).copy()
        return lib().log_likelihood_het(self.nh.ref, C.byref(self.het), _ptr(p), self.Tobs)

    def het_diff(self, params, dparams):
        p, q = _f64(params).copy(), _f64(dparams).copy()
        return lib().het_diff(self.nh.ref, C.byref(self.het), _ptr(p), _ptr(q))

    def fisher(self, params):
        F = np.zeros((11, 11))
        p = _f64(params).copy()
        lib().Fisher_Het(self.nh.ref, C.byref(self.het), _rows(F), _ptr(p), self.Tobs)
        return F

    def tables(self):
        h, nI, M, J, NR = self.het, self.nh.net.Nifo, self.het.M, self.het.J, self.het.NR
        t = dict(logLb=h.logLb, fgrid=self.fgrid.copy(), freq=self.freq.copy(), M=M, J=J, NR=NR, MN=h.MN, MM=h.MM)
        t["amp"] = np.array([[h.amp[i][j] for j in range(M)] for i in range(nI)])
        t["phase"] = np.array([[h.phase[i][j] for j in range(M)] for i in range(nI)])
        t["IP"] = np.array([[[h.IP[r][a][b] for b in range(J + 1)] for a in range(J + 1)] for r in range(NR)])
        for k in ("SL", "lc", "ls"):
            arr = getattr(h, k)
            t[k] = np.array([[[arr[r][i][a] for a in range(J + 1)] for i in range(nI)] for r in range(NR)])
        for k in ("aa", "rc", "rs"):
            arr = getattr(h, k)
            t[k] = np.array([[arr[i][r] for r in range(NR)] for i in range(nI)])
        return t


def sky_ring_map(x, GMST, label1, label2, rot):
    """The reference sampler's sky-ring map on the GPU (qcbc_sky_ring_map): x's sky position turned
    by `rot` about the line between two detectors, the extrinsic parameters that keep their signal,
    and the log Jacobian of the map.  Returns (y [11], log_jacobian)."""
    x = _f64(x).copy()
    y = np.zeros(11)
    lj = C.c_double()
    check(lib().qcbc_sky_ring_map(_ptr(x), _ptr(y), float(GMST), int(label1), int(label2), float(rot), C.byref(lj)))
    return y, lj.value

"""Input stage of an analysis (include/qcbc_ingest.h) from Python.

* QuickCBC's files: ``framed_<T>_<trig>_<ifo>.dat`` (time, strain) and
  ``spec_<T>_<trig>_<ifo>.dat`` (f, SN, SM, -), read as QuickCBC.c:198-242 reads them;
* data conditioning on the GPU: Tukey window, real FFT in GSL half-complex layout,
  times sqrt(Tobs)/N (QuickCBC.c:244-258, 309-313);
* the PSD-sample model of noise marginalisation (``summary_``, ``sfile_``, ``ffile_``,
  ``lfile_`` files, QuickCBC.c:322-378) with ``makespec`` (Utilities.c:1908) on the GPU.

File readers are host code; conditioning and makespec need the GPU.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import _lib
from ._lib import QcbcError, check, lib

_PD = C.POINTER(C.c_double)
_PI = C.POINTER(C.c_int)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _ptr(a):
    return a.ctypes.data_as(_PD)


def _path(p):
    return os.fspath(p).encode()


def framed_length(path) -> int:
    """Samples N of a framed file, counted as QuickCBC.c:205-211 counts them."""
    n = C.c_int()
    check(lib().qcbc_framed_length(_path(path), C.byref(n)))
    return n.value


def read_framed(path, N):
    """(t, x): the first N rows of a framed file."""
    t, x = np.zeros(N), np.zeros(N)
    check(lib().qcbc_read_framed(_path(path), int(N), _ptr(t), _ptr(x)))
    return t, x


def read_spec(path, nh):
    """(SN, SM): columns 2 and 3 of the first nh rows of a spec file."""
    SN, SM = np.zeros(nh), np.zeros(nh)
    check(lib().qcbc_read_spec(_path(path), int(nh), _ptr(SN), _ptr(SM)))
    return SN, SM


def analysis_paths(directory, Tobs, ttrig, label):
    """(framed, spec) file names of one detector, as QuickCBC.c builds them."""
    a, b = C.create_string_buffer(4096), C.create_string_buffer(4096)
    check(lib().qcbc_analysis_paths(_path(directory), float(Tobs), float(ttrig), int(label), a, b, 4096))
    return a.value.decode(), b.value.decode()


def condition_data(x, Tobs):
    """D [nifo, N] from time series x [nifo, N] on the GPU."""
    x = _f64(np.atleast_2d(x))
    nifo, N = x.shape
    D = np.zeros((nifo, N))
    check(lib().qcbc_condition_data(nifo, N, float(Tobs), _ptr(x), N, _ptr(D), N))
    return D


def load_analysis(directory, Tobs, ttrig, labels):
    """(D [nifo, N], SN [nifo, N/2], SM [nifo, N/2]) of one analysis from its files."""
    labels = np.ascontiguousarray(labels, dtype=np.int32)
    framed, _ = analysis_paths(directory, Tobs, ttrig, int(labels[0]))
    N = framed_length(framed)
    nifo = len(labels)
    D, SN, SM = np.zeros((nifo, N)), np.zeros((nifo, N // 2)), np.zeros((nifo, N // 2))
    check(lib().qcbc_load_analysis(_path(directory), float(Tobs), float(ttrig), nifo, labels.ctypes.data_as(_PI), N,
                                   _ptr(D), N, _ptr(SN), _ptr(SM), N // 2))
    return D, SN, SM


class PsdModel:
    """PSD samples of a spline-plus-lines noise model on the GPU (qcbc_psd_model_*).

    From arrays: nspline [nifo], nlines [nifo], ffit [nifo, nspline_max],
    xspline [nifo, nsample, nspline_max] (log PSD at the knots),
    lines [nifo, nsample, nlines_max, 5] (f, h, Q, w, deltafmax)."""

    def __init__(self, ffit, xspline, lines, nspline=None, nlines=None):
        ffit = _f64(np.atleast_2d(ffit))
        xspline = _f64(xspline)
        lines = _f64(lines)
        nifo, nsp = ffit.shape
        nsample = xspline.shape[1]
        nlm = lines.shape[2]
        if xspline.shape != (nifo, nsample, nsp) or lines.shape != (nifo, nsample, nlm, 5):
            raise ValueError("xspline must be [nifo, nsample, nspline_max], lines [nifo, nsample, nlines_max, 5]")
        ns = np.ascontiguousarray(nspline if nspline is not None else [nsp] * nifo, dtype=np.int32)
        nl = np.ascontiguousarray(nlines if nlines is not None else [nlm] * nifo, dtype=np.int32)
        if lines.size == 0:
            lines = np.zeros(5)
        self._h = lib().qcbc_psd_model_create(nifo, ns.ctypes.data_as(_PI), nl.ctypes.data_as(_PI), nsample, nsp, nlm,
                                              _ptr(ffit), _ptr(xspline), _ptr(lines))
        if not self._h:
            raise QcbcError(-1, _lib.last_error())
        self._info()

    @classmethod
    def open(cls, directory, labels):
        """From the summary_/sfile_/ffile_/lfile_ files of each detector in `directory`."""
        self = cls.__new__(cls)
        labels = np.ascontiguousarray(labels, dtype=np.int32)
        self._h = lib().qcbc_psd_model_open(_path(directory), len(labels), labels.ctypes.data_as(_PI))
        if not self._h:
            raise QcbcError(-1, _lib.last_error())
        self._info()
        return self

    def _info(self):
        a, b, c, d = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        check(lib().qcbc_psd_model_info(self._h, C.byref(a), C.byref(b), C.byref(c), C.byref(d)))
        self.nifo, self.nsample, self.nspline_max, self.nlines_max = a.value, b.value, c.value, d.value

    @property
    def handle(self):
        return self._h

    def draw(self, k, Tobs, N):
        """makespec of sample k for every detector: SN [nifo, N/2]."""
        SN = np.zeros((self.nifo, N // 2))
        check(lib().qcbc_psd_draw(self._h, int(k), float(Tobs), int(N), _ptr(SN), N // 2))
        return SN

    def close(self):
        if getattr(self, "_h", None):
            lib().qcbc_psd_model_close(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def makespec(ffit, Sspline, linef, lineh, lineQ, linew, deltafmax, Tobs, N):
    """The reference signature (Utilities.c:1908) through the library's drop-in symbol: SN [N/2]."""
    a = [_f64(v).copy() for v in (ffit, Sspline, linef, lineh, lineQ, linew, deltafmax)]
    SN = np.full(N // 2, np.nan)
    lib().makespec(len(a[0]), len(a[2]), *[_ptr(v) for v in a], _ptr(SN), float(Tobs), int(N))
    if np.isnan(SN).any():
        raise QcbcError(-1, _lib.last_error())
    return SN

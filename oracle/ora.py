"""ctypes bindings for oracle/_build/liboracle.so, the CPU restatement of the
likelihood hot path (qcbc_oracle.c).

TEST INFRASTRUCTURE ONLY: the checker for the CUDA kernels.  Imported by
tests/, ``__graft_entry__.smoke()`` and the CPU-baseline leg of bench.py.
Layouts as in oracle/ref.py.
"""
from __future__ import annotations

import ctypes as C
import os
import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
FMAX = 1024.0

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_lib = None


def available() -> bool:
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise FileNotFoundError(f"oracle not built: {LIB_PATH} (make -C oracle oracle)")
        L = C.CDLL(LIB_PATH)
        i, d = C.c_int, C.c_double
        L.ora_set_qnm.argtypes = [_dp, _dp, _dp, i]
        L.ora_amp_phase.argtypes = [_dp, i] + [d] * 7 + [_dp, _dp]
        L.ora_fbegin.restype = d
        L.ora_fbegin.argtypes = [_dp]
        L.ora_antenna.argtypes = [d, d, d, d, i, _dp]
        L.ora_delays.argtypes = [d, d, d, _dp]
        L.ora_fulltemplates.argtypes = [_ip, i, d, _dp, _dp, i, _dp]
        L.ora_fullphaseamp.argtypes = [_ip, i, d, d, _dp, _dp, i, _dp, _dp]
        L.ora_fourier_nwip.restype = d
        L.ora_fourier_nwip.argtypes = [_dp, _dp, _dp, i, i, i]
        L.ora_lnl_full.restype = d
        L.ora_lnl_full.argtypes = [_ip, i, d, _dp, _dp, i, _dp, _dp, i, d, d, d, _dp]
        L.ora_lnl_full_batch.restype = d
        L.ora_lnl_full_batch.argtypes = [_ip, i, d, _dp, _dp, i, _dp, _dp, i, i, d, d, d, _dp, i]
        L.ora_heterodyne.restype = i
        L.ora_heterodyne.argtypes = [_ip, i, d, _dp, _dp, i, _dp, _dp, i, d, _ip, i, i, i, i] + [_dp] * 10
        L.ora_lnl_het.restype = d
        L.ora_lnl_het.argtypes = [_ip, i, d, d, _dp, i, i] + [_dp] * 9 + [d, _dp]
        L.ora_lnl_het_batch.restype = d
        L.ora_lnl_het_batch.argtypes = [_ip, i, d, d, _dp, i, i] + [_dp] * 9 + [d, _dp, i, _dp, i]
        _lib = L
    return _lib


def _f(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _lab(labels):
    return np.ascontiguousarray(labels, dtype=np.int32)


def amp_phase(freq, phi0, fRef, m1_SI, m2_SI, chi1, chi2, dist):
    f = _f(freq)
    a, p = np.zeros_like(f), np.zeros_like(f)
    lib().ora_amp_phase(f, len(f), phi0, fRef, m1_SI, m2_SI, chi1, chi2, dist, a, p)
    return a, p


def fbegin(params):
    return lib().ora_fbegin(_f(params))


def antenna(psi, alpha, sindelta, GMST, ifo):
    out = np.zeros(2)
    lib().ora_antenna(psi, alpha, sindelta, GMST, ifo, out)
    return out


def delays(alpha, sindelta, GMST):
    out = np.zeros(3)
    lib().ora_delays(alpha, sindelta, GMST, out)
    return out


def fulltemplates(labels, GMST, freq, params, N):
    lab = _lab(labels)
    h = np.zeros((len(lab), N))
    lib().ora_fulltemplates(lab, len(lab), GMST, _f(freq), _f(params), N, h)
    return h


def fullphaseamp(labels, GMST, Tobs, freq, params, N):
    lab = _lab(labels)
    a = np.zeros((len(lab), N // 2))
    p = np.zeros((len(lab), N // 2))
    lib().ora_fullphaseamp(lab, len(lab), GMST, Tobs, _f(freq), _f(params), N, a, p)
    return a, p


def lnl_full(ev, params, fmax=FMAX):
    lab = _lab(ev.labels)
    rho = np.zeros(len(lab))
    L = lib().ora_lnl_full(lab, len(lab), ev.GMST, _f(ev.D), _f(ev.SN), ev.SN.shape[1], _f(ev.freq), _f(params),
                           ev.N, ev.Tobs, ev.fmin, fmax, rho)
    return L, rho


def lnl_full_batch(ev, params, nthreads=0, fmax=FMAX):
    lab = _lab(ev.labels)
    P = _f(params)
    out = np.zeros(P.shape[0])
    secs = lib().ora_lnl_full_batch(lab, len(lab), ev.GMST, _f(ev.D), _f(ev.SN), ev.SN.shape[1], _f(ev.freq), P,
                                    P.shape[0], ev.N, ev.Tobs, ev.fmin, fmax, out, nthreads)
    return out, secs


def heterodyne(ev, params, fgrid, MN, MM, J=2):
    lab = _lab(ev.labels)
    nI = len(lab)
    g = np.ascontiguousarray(fgrid, dtype=np.int32)
    M = len(g)
    NR = (M - 1) // J
    t = dict(amp=np.zeros((nI, M)), phase=np.zeros((nI, M)), IP=np.zeros((NR, J + 1, J + 1)),
             SL=np.zeros((NR, nI, J + 1)), lc=np.zeros((NR, nI, J + 1)), ls=np.zeros((NR, nI, J + 1)),
             aa=np.zeros((nI, NR)), rc=np.zeros((nI, NR)), rs=np.zeros((nI, NR)), logLb=np.zeros(1))
    lib().ora_heterodyne(lab, nI, ev.GMST, _f(ev.D), _f(ev.SN), ev.SN.shape[1], _f(ev.freq), _f(params), ev.N,
                         ev.Tobs, g, M, MN, MM, J, t["amp"], t["phase"], t["IP"], t["SL"], t["lc"], t["ls"],
                         t["aa"], t["rc"], t["rs"], t["logLb"])
    t["logLb"] = float(t["logLb"][0])
    t.update(fgrid=g, freq=g.astype(np.float64) / ev.Tobs, M=M, J=J, NR=NR, MN=MN, MM=MM, Nifo=nI)
    return t


def _het_args(ev, t):
    return (_lab(ev.labels), len(ev.labels), ev.GMST, ev.Tobs, _f(t["freq"]), t["M"], t["J"], _f(t["amp"]),
            _f(t["phase"]), _f(t["IP"]), _f(t["SL"]), _f(t["lc"]), _f(t["ls"]), _f(t["aa"]), _f(t["rc"]),
            _f(t["rs"]), float(t["logLb"]))


def lnl_het(ev, t, params):
    return lib().ora_lnl_het(*_het_args(ev, t), _f(params))


def lnl_het_batch(ev, t, params, nthreads=0):
    P = _f(params)
    out = np.zeros(P.shape[0])
    secs = lib().ora_lnl_het_batch(*_het_args(ev, t), P, P.shape[0], out, nthreads)
    return out, secs

"""ctypes bindings for oracle/_ref/libqcbc_ref.so -- the QuickCBC reference C,
compiled unmodified from its own sources against the GSL-API shim.

TEST INFRASTRUCTURE ONLY: imported by tests/, by ``__graft_entry__.smoke()``
and by the CPU-baseline leg of bench.py.  The product never imports this.

Flat layouts used here (all float64, C order):
  D      [Nifo, N]            half-complex rows (GSL layout, Utilities.c:716-736)
  SN     [Nifo, N//2 + 1]     one-sided PSD per bin (row length N/2+1 like the
                              reference's double_matrix(Nifo, N/2), Utilities.c:2981)
  params [B, 11]              the reference's `pall` layout (QuickCBC.c:1867)
"""
from __future__ import annotations

import ctypes as C
import os
import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_ref", "libqcbc_ref.so")

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_lib = None


def available() -> bool:
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise FileNotFoundError(f"reference oracle not built: {LIB_PATH} (make -C oracle ref)")
        L = C.CDLL(LIB_PATH)
        vp = C.c_void_p
        L.ref_net_new.restype = vp
        L.ref_net_new.argtypes = [C.c_int, _ip, C.c_double, C.c_double]
        L.ref_net_free.argtypes = [vp]
        L.ref_amp_phase.restype = C.c_int
        L.ref_amp_phase.argtypes = [_dp, C.c_int] + [C.c_double] * 7 + [_dp, _dp]
        L.ref_fbegin.restype = C.c_double
        L.ref_fbegin.argtypes = [_dp]
        L.ref_F_ant.argtypes = [C.c_double] * 4 + [C.c_int, _dp]
        L.ref_Times.argtypes = [C.c_double] * 3 + [_dp]
        L.ref_fulltemplates.argtypes = [vp, _dp, _dp, C.c_int, _dp, C.c_int]
        L.ref_fullphaseamp.argtypes = [vp, _dp, _dp, _dp, C.c_int, _dp, C.c_int]
        L.ref_fourier_nwip.restype = C.c_double
        L.ref_fourier_nwip.argtypes = [_dp, _dp, _dp, C.c_int, C.c_int, C.c_int]
        L.ref_lnl_full.restype = C.c_double
        L.ref_lnl_full.argtypes = [vp, _dp, _dp, _dp, _dp, C.c_int, _dp, C.c_int, C.c_double]
        L.ref_lnl_full_batch.restype = C.c_double
        L.ref_lnl_full_batch.argtypes = [vp, _dp, _dp, C.c_int, _dp, _dp, C.c_int, C.c_int,
                                         C.c_double, _dp, C.c_int]
        L.ref_max_threads.restype = C.c_int
        L.ref_het_new.restype = vp
        L.ref_het_space.restype = C.c_int
        L.ref_het_space.argtypes = [vp, vp, _dp, _dp, _dp, _dp, _dp, C.c_int, C.c_int, C.c_double]
        L.ref_het_set_grid.argtypes = [vp, _ip, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double]
        L.ref_heterodyne.argtypes = [vp, vp, _dp, _dp, _dp, _dp, C.c_int, C.c_int, C.c_double]
        L.ref_het_sizes.argtypes = [vp, vp, _ip]
        L.ref_het_export.argtypes = [vp, vp, _ip] + [_dp] * 11
        L.ref_lnl_het.restype = C.c_double
        L.ref_lnl_het.argtypes = [vp, vp, _dp, C.c_double]
        L.ref_lnl_het_batch.restype = C.c_double
        L.ref_lnl_het_batch.argtypes = [vp, vp, _dp, C.c_int, C.c_double, _dp, C.c_int]
        L.ref_lnl_test.restype = C.c_double
        L.ref_lnl_test.argtypes = [vp, vp, _dp, _dp, _dp, _dp, C.c_int, C.c_int, C.c_double]
        L.ref_het_free.argtypes = [vp, vp]
        L.ref_templates.argtypes = [vp, _dp, _dp, C.c_int, _dp, C.c_int]
        L.ref_lnl_intrinsic.restype = C.c_double
        L.ref_lnl_intrinsic.argtypes = [vp, _dp, _dp, _dp, _dp, C.c_int, C.c_int, C.c_double]
        L.ref_AmpPhase.argtypes = [_dp, _dp, _dp, C.c_int, _dp, C.c_int]
        L.ref_het_diff.restype = C.c_double
        L.ref_het_diff.argtypes = [vp, vp, _dp, _dp]
        L.ref_Fisher_Het.argtypes = [vp, vp, _dp, _dp, C.c_double]
        L.ref_framed_count.argtypes = [C.c_char_p]
        L.ref_framed_count.restype = C.c_int
        L.ref_condition.argtypes = [_dp, C.c_int, C.c_double, _dp]
        L.makespec.argtypes = [C.c_int, C.c_int] + [_dp] * 8 + [C.c_double, C.c_int]
        L.makespec.restype = None
        L.skymap_all.argtypes = [_dp, _dp, C.c_double, C.c_int, C.c_int]
        L.skymap_all.restype = None
        L.skydensity_all.argtypes = [_dp, _dp, C.c_double, C.c_int, C.c_int]
        L.skydensity_all.restype = C.c_double
        _lib = L
    return _lib


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


class RefNet:
    """struct Net (QuickCBC.h:13-25) owned by the reference library."""

    def __init__(self, labels, Tobs, GMST):
        self.labels = np.ascontiguousarray(labels, dtype=np.int32)
        self.nifo = len(self.labels)
        self.Tobs = float(Tobs)
        self.GMST = float(GMST)
        self.ptr = lib().ref_net_new(self.nifo, self.labels, self.Tobs, self.GMST)

    def __del__(self):
        try:
            lib().ref_net_free(self.ptr)
        except Exception:
            pass


def amp_phase(freq, phi0, fRef, m1_SI, m2_SI, chi1, chi2, dist):
    f = _f64(freq)
    a = np.zeros_like(f)
    p = np.zeros_like(f)
    lib().ref_amp_phase(f, len(f), phi0, fRef, m1_SI, m2_SI, chi1, chi2, dist, a, p)
    return a, p


def fbegin(params):
    return lib().ref_fbegin(_f64(params).copy())


def F_ant(psi, alpha, sindelta, GMST, ifo):
    out = np.zeros(2)
    lib().ref_F_ant(psi, alpha, sindelta, GMST, ifo, out)
    return out


def Times(alpha, sindelta, GMST):
    out = np.zeros(3)
    lib().ref_Times(alpha, sindelta, GMST, out)
    return out


def fulltemplates(net: RefNet, freq, params, N):
    h = np.zeros((net.nifo, N))
    f = _f64(freq)
    lib().ref_fulltemplates(net.ptr, h, f, len(f), _f64(params).copy(), N)
    return h


def fullphaseamp(net: RefNet, freq, params, N):
    a = np.zeros((net.nifo, N // 2))
    p = np.zeros((net.nifo, N // 2))
    f = _f64(freq)
    lib().ref_fullphaseamp(net.ptr, a, p, f, len(f), _f64(params).copy(), N)
    return a, p


def fourier_nwip(a, b, S, imin, imax, N):
    return lib().ref_fourier_nwip(_f64(a), _f64(b), _f64(S), imin, imax, N)


def lnl_full(net: RefNet, D, params, freq, SN, N, Tobs):
    rho = np.zeros(net.nifo + 1)
    SN = _f64(SN)
    L = lib().ref_lnl_full(net.ptr, _f64(D), _f64(params).copy(), _f64(freq), SN, SN.shape[1], rho, N, Tobs)
    return L, rho[: net.nifo]


def templates(net: RefNet, freq, params, N):
    """templates (QuickCBC.c:3527): intrinsic parameters, 7 + 3 (Nifo - 1) entries."""
    h = np.zeros((net.nifo, N))
    f = _f64(freq)
    lib().ref_templates(net.ptr, h, f, len(f), _f64(params).copy(), N)
    return h


def lnl_intrinsic(net: RefNet, D, params, freq, SN, N, Tobs):
    SN = _f64(SN)
    return lib().ref_lnl_intrinsic(net.ptr, _f64(D), _f64(params).copy(), _f64(freq), SN, SN.shape[1], N, Tobs)


def AmpPhase(freq, params, N):
    """AmpPhase (QuickCBC.c:3395): (Af, Pf) over N/2 bins, entry 0 left at zero."""
    Af = np.zeros(N // 2)
    Pf = np.zeros(N // 2)
    f = _f64(freq)
    lib().ref_AmpPhase(Af, Pf, f, len(f), _f64(params).copy(), N)
    return Af, Pf


def lnl_full_batch(net: RefNet, D, params, freq, SN, N, Tobs, nthreads=0):
    P = _f64(params)
    out = np.zeros(P.shape[0])
    SN = _f64(SN)
    secs = lib().ref_lnl_full_batch(net.ptr, _f64(D), P, P.shape[0], _f64(freq), SN, SN.shape[1], N,
                                    Tobs, out, nthreads)
    return out, secs


def max_threads():
    return lib().ref_max_threads()


class RefHet:
    """struct Het (QuickCBC.h:27-51) built by the reference's het_space/heterodyne."""

    def __init__(self, net: RefNet):
        self.net = net
        self.ptr = lib().ref_het_new()

    def space(self, params, pmin, pmax, freq, SN, N, Tobs, workdir):
        cwd = os.getcwd()
        os.makedirs(workdir, exist_ok=True)
        os.chdir(workdir)        # het_space writes diagnostic .dat files into the cwd
        try:
            SN = _f64(SN)
            return lib().ref_het_space(self.net.ptr, self.ptr, _f64(params).copy(), _f64(pmin).copy(),
                                       _f64(pmax).copy(), _f64(freq), SN, SN.shape[1], N, Tobs)
        finally:
            os.chdir(cwd)

    def set_grid(self, fgrid, MN, MM, J, Tobs):
        g = np.ascontiguousarray(fgrid, dtype=np.int32)
        lib().ref_het_set_grid(self.ptr, g, len(g), MN, MM, J, Tobs)

    def heterodyne(self, D, params, freq, SN, N, Tobs):
        SN = _f64(SN)
        lib().ref_heterodyne(self.net.ptr, self.ptr, _f64(D), _f64(params).copy(), _f64(freq), SN,
                             SN.shape[1], N, Tobs)

    def sizes(self):
        s = np.zeros(6, dtype=np.int32)
        lib().ref_het_sizes(self.net.ptr, self.ptr, s)
        return dict(M=int(s[0]), MN=int(s[1]), MM=int(s[2]), J=int(s[3]), NR=int(s[4]), Nifo=int(s[5]))

    def export(self):
        z = self.sizes()
        M, J, NR, nI = z["M"], z["J"], z["NR"], z["Nifo"]
        t = dict(
            fgrid=np.zeros(M, dtype=np.int32), freq=np.zeros(M), amp=np.zeros((nI, M)),
            phase=np.zeros((nI, M)), IP=np.zeros((NR, J + 1, J + 1)), SL=np.zeros((NR, nI, J + 1)),
            lc=np.zeros((NR, nI, J + 1)), ls=np.zeros((NR, nI, J + 1)), aa=np.zeros((nI, NR)),
            rc=np.zeros((nI, NR)), rs=np.zeros((nI, NR)), logLb=np.zeros(1),
        )
        lib().ref_het_export(self.net.ptr, self.ptr, t["fgrid"], t["freq"], t["amp"], t["phase"], t["IP"],
                             t["SL"], t["lc"], t["ls"], t["aa"], t["rc"], t["rs"], t["logLb"])
        t["logLb"] = float(t["logLb"][0])
        t.update(z)
        return t

    def lnl(self, params, Tobs):
        return lib().ref_lnl_het(self.net.ptr, self.ptr, _f64(params).copy(), Tobs)

    def lnl_batch(self, params, Tobs, nthreads=0):
        P = _f64(params)
        out = np.zeros(P.shape[0])
        secs = lib().ref_lnl_het_batch(self.net.ptr, self.ptr, P, P.shape[0], Tobs, out, nthreads)
        return out, secs

    def het_diff(self, params, dparams):
        return lib().ref_het_diff(self.net.ptr, self.ptr, _f64(params).copy(), _f64(dparams).copy())

    def fisher(self, params, Tobs):
        F = np.zeros((11, 11))
        lib().ref_Fisher_Het(self.net.ptr, self.ptr, F, _f64(params).copy(), Tobs)
        return F

    def lnl_test(self, D, params, freq, SN, N, Tobs):
        SN = _f64(SN)
        return lib().ref_lnl_test(self.net.ptr, self.ptr, _f64(D), _f64(params).copy(), _f64(freq), SN,
                                  SN.shape[1], N, Tobs)


def framed_count(path):
    """Row count of a framed file as QuickCBC.c:205-211 computes it (-2: unreadable content)."""
    return lib().ref_framed_count(str(path).encode())


def condition(x, Tobs):
    """QuickCBC.c:244-258 + 309-313 on one time series: tukey, GSL real FFT, sqrt(Tobs)/N."""
    x = _f64(x)
    D = np.zeros(len(x))
    lib().ref_condition(x, len(x), float(Tobs), D)
    return D


def makespec(ffit, Sspline, linef, lineh, lineQ, linew, deltafmax, Tobs, N):
    """The reference's makespec (Utilities.c:1908): SN[N/2]."""
    a = [_f64(v).copy() for v in (ffit, Sspline, linef, lineh, lineQ, linew, deltafmax)]
    SN = np.zeros(N // 2)
    lib().makespec(len(a[0]), len(a[2]), *a, SN, float(Tobs), int(N))
    return SN


def skymap_all(x, y, GMST, ifo1, ifo2):
    """The reference's skymap_all (QuickCBC.c:7085): fills y's [4, 5, 6, 9, 10] for y's sky position."""
    x = _f64(x).copy()
    y = _f64(y).copy()
    lib().skymap_all(x, y, float(GMST), int(ifo1), int(ifo2))
    return y


def skydensity_all(x, y, GMST, ifo1, ifo2):
    """The reference's skydensity_all (QuickCBC.c:7411): |det| of the map's 4 x 4 Jacobian."""
    x = _f64(x).copy()
    y = _f64(y).copy()
    return lib().skydensity_all(x, y, float(GMST), int(ifo1), int(ifo2))

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
        _lib = _declare(C.CDLL(LIB_PATH))
    return _lib


_native = None


def _cpu_flags():
    try:
        with open("/proc/cpuinfo") as f:
            for ln in f:
                if ln.startswith("flags"):
                    return set(ln.split(":", 1)[1].split())
    except OSError:
        pass
    return set()


def native_variant():
    """The build of the reference library matched to this host's CPU: oracle/_ref/x86-64-v4 (AVX-512)
    or x86-64-v3 (AVX2, FMA), both -O3 (make -C oracle ref-native), else the portable oracle/_ref."""
    f = _cpu_flags()
    for name, need in (("x86-64-v4", {"avx512f", "avx512bw", "avx512cd", "avx512dq", "avx512vl"}),
                       ("x86-64-v3", {"avx2", "fma", "bmi2", "movbe"})):
        if need <= f and os.path.exists(os.path.join(_HERE, "_ref", name, "libqcbc_ref.so")):
            return name
    return "portable"


def native_lib():
    """The reference library built for this host's instruction set (native_variant); used by the
    CPU baselines.  Tests use lib(), the portable build."""
    global _native
    if _native is None:
        v = native_variant()
        _native = lib() if v == "portable" else _declare(C.CDLL(os.path.join(_HERE, "_ref", v, "libqcbc_ref.so")))
    return _native


LINKED_PATH = os.path.join(_HERE, "_ref", "libquickcbc_linked.so")
_linked = None


def linked_available() -> bool:
    return os.path.exists(LINKED_PATH)


def linked():
    """oracle/_ref/libquickcbc_linked.so: the reference's sources unmodified, their thirteen
    replaced functions weakened and forwarded to libqcbc_gpu.so by include/qcbc_forward.c
    (make -C oracle linked).  Same ref_* harness as lib(), plus lk_mcmc / lk_time_calls
    (link_harness.c) and the stub's call counters qcbc_forward_calls[13]."""
    global _linked
    if _linked is None:
        if not linked_available():
            raise FileNotFoundError(f"linked reference not built: {LINKED_PATH} (make -C oracle linked)")
        L = _declare(C.CDLL(LINKED_PATH))
        vp, d, i = C.c_void_p, C.c_double, C.c_int
        L.lk_data_new.restype = vp
        L.lk_data_new.argtypes = [i, _dp, _dp, i, _dp, i, d]
        L.lk_data_free.argtypes = [vp]
        L.lk_lnl_full.restype = d
        L.lk_lnl_full.argtypes = [vp, vp, _dp, _dp]
        L.lk_bind.argtypes = [vp, vp]
        L.lk_unbind.argtypes = []
        L.lk_mcmc.restype = d
        L.lk_mcmc.argtypes = [vp, vp, vp, _dp, _dp, _dp, i, i, C.c_ulong, _dp, _dp, _dp, _dp, _ip,
                              C.POINTER(C.c_longlong)]
        L.lk_time_calls.restype = d
        L.lk_time_calls.argtypes = [vp, vp, vp, _dp, i, i, i, _dp]
        _linked = L
    return _linked


FORWARD_NAMES = ("log_likelihood_full", "log_likelihood_het", "heterodyne", "fulltemplates", "fullphaseamp",
                 "IMRPhenomDGenerateh22FDAmpPhase", "fourier_nwip", "log_likelihood_intrinsic", "templates",
                 "AmpPhase", "het_diff", "Fisher_Het", "het_space")


def forward_calls():
    """The forwarding stub's call counts, by name (FORWARD_NAMES order)."""
    arr = (C.c_longlong * len(FORWARD_NAMES)).in_dll(linked(), "qcbc_forward_calls")
    return {n: int(arr[k]) for k, n in enumerate(FORWARD_NAMES)}


class LinkedData:
    """D, SN and freq held by the linked reference as QuickCBC holds them for a run: row-pointer
    arrays made once over these numpy buffers (writes into SN are seen by the next call)."""

    def __init__(self, net: RefNet, D, SN, freq, N, Tobs):
        self.L = net.L
        self.D, self.SN, self.freq = _f64(D).copy(), _f64(SN).copy(), _f64(freq).copy()
        self.N, self.Tobs = int(N), float(Tobs)
        self.ptr = self.L.lk_data_new(net.nifo, self.D, self.SN, self.SN.shape[1], self.freq, self.N, self.Tobs)

    def __del__(self):
        try:
            self.L.lk_data_free(self.ptr)
        except Exception:
            pass


def _declare(L):
    if True:
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
    return L


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


class RefNet:
    """struct Net (QuickCBC.h:13-25) owned by the reference library."""

    def __init__(self, labels, Tobs, GMST, L=None):
        self.L = L if L is not None else lib()
        self.labels = np.ascontiguousarray(labels, dtype=np.int32)
        self.nifo = len(self.labels)
        self.Tobs = float(Tobs)
        self.GMST = float(GMST)
        self.ptr = self.L.ref_net_new(self.nifo, self.labels, self.Tobs, self.GMST)

    def __del__(self):
        try:
            self.L.ref_net_free(self.ptr)
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
    net.L.ref_fulltemplates(net.ptr, h, f, len(f), _f64(params).copy(), N)
    return h


def fullphaseamp(net: RefNet, freq, params, N):
    a = np.zeros((net.nifo, N // 2))
    p = np.zeros((net.nifo, N // 2))
    f = _f64(freq)
    net.L.ref_fullphaseamp(net.ptr, a, p, f, len(f), _f64(params).copy(), N)
    return a, p


def fourier_nwip(a, b, S, imin, imax, N):
    return lib().ref_fourier_nwip(_f64(a), _f64(b), _f64(S), imin, imax, N)


def lnl_full(net: RefNet, D, params, freq, SN, N, Tobs):
    rho = np.zeros(net.nifo + 1)
    SN = _f64(SN)
    L = net.L.ref_lnl_full(net.ptr, _f64(D), _f64(params).copy(), _f64(freq), SN, SN.shape[1], rho, N, Tobs)
    return L, rho[: net.nifo]


def templates(net: RefNet, freq, params, N):
    """templates (QuickCBC.c:3527): intrinsic parameters, 7 + 3 (Nifo - 1) entries."""
    h = np.zeros((net.nifo, N))
    f = _f64(freq)
    net.L.ref_templates(net.ptr, h, f, len(f), _f64(params).copy(), N)
    return h


def lnl_intrinsic(net: RefNet, D, params, freq, SN, N, Tobs):
    SN = _f64(SN)
    return net.L.ref_lnl_intrinsic(net.ptr, _f64(D), _f64(params).copy(), _f64(freq), SN, SN.shape[1], N, Tobs)


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
    secs = net.L.ref_lnl_full_batch(net.ptr, _f64(D), P, P.shape[0], _f64(freq), SN, SN.shape[1], N,
                                    Tobs, out, nthreads)
    return out, secs


def max_threads(L=None):
    return (L if L is not None else lib()).ref_max_threads()


class RefHet:
    """struct Het (QuickCBC.h:27-51) built by the reference's het_space/heterodyne."""

    def __init__(self, net: RefNet):
        self.net = net
        self.L = net.L
        self.ptr = self.L.ref_het_new()

    def space(self, params, pmin, pmax, freq, SN, N, Tobs, workdir):
        cwd = os.getcwd()
        os.makedirs(workdir, exist_ok=True)
        os.chdir(workdir)        # het_space writes diagnostic .dat files into the cwd
        try:
            SN = _f64(SN)
            return self.L.ref_het_space(self.net.ptr, self.ptr, _f64(params).copy(), _f64(pmin).copy(),
                                       _f64(pmax).copy(), _f64(freq), SN, SN.shape[1], N, Tobs)
        finally:
            os.chdir(cwd)

    def set_grid(self, fgrid, MN, MM, J, Tobs):
        g = np.ascontiguousarray(fgrid, dtype=np.int32)
        self.L.ref_het_set_grid(self.ptr, g, len(g), MN, MM, J, Tobs)

    def heterodyne(self, D, params, freq, SN, N, Tobs):
        SN = _f64(SN)
        self.L.ref_heterodyne(self.net.ptr, self.ptr, _f64(D), _f64(params).copy(), _f64(freq), SN,
                             SN.shape[1], N, Tobs)

    def sizes(self):
        s = np.zeros(6, dtype=np.int32)
        self.L.ref_het_sizes(self.net.ptr, self.ptr, s)
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
        self.L.ref_het_export(self.net.ptr, self.ptr, t["fgrid"], t["freq"], t["amp"], t["phase"], t["IP"],
                             t["SL"], t["lc"], t["ls"], t["aa"], t["rc"], t["rs"], t["logLb"])
        t["logLb"] = float(t["logLb"][0])
        t.update(z)
        return t

    def lnl(self, params, Tobs):
        return self.L.ref_lnl_het(self.net.ptr, self.ptr, _f64(params).copy(), Tobs)

    def lnl_batch(self, params, Tobs, nthreads=0):
        P = _f64(params)
        out = np.zeros(P.shape[0])
        secs = self.L.ref_lnl_het_batch(self.net.ptr, self.ptr, P, P.shape[0], Tobs, out, nthreads)
        return out, secs

    def het_diff(self, params, dparams):
        return self.L.ref_het_diff(self.net.ptr, self.ptr, _f64(params).copy(), _f64(dparams).copy())

    def fisher(self, params, Tobs):
        F = np.zeros((11, 11))
        self.L.ref_Fisher_Het(self.net.ptr, self.ptr, F, _f64(params).copy(), Tobs)
        return F

    def lnl_test(self, D, params, freq, SN, N, Tobs):
        SN = _f64(SN)
        return self.L.ref_lnl_test(self.net.ptr, self.ptr, _f64(D), _f64(params).copy(), _f64(freq), SN,
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

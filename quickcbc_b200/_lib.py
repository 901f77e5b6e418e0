"""ctypes binding of libqcbc_gpu.so (the C ABI in include/qcbc_gpu.h and
include/qcbc_quickcbc.h).  There is no CPU fallback: if the library is missing
or no GPU is present the calls raise."""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("QCBC_LIB_PATH") or os.path.join(HERE, "libqcbc_gpu.so")

QCBC_OK = 0
QCBC_EDOM = 33
FP64 = 0
MIXED = 1


class QcbcError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"qcbc error {code}: {msg}")
        self.code = code


# ---- reference struct layouts (QuickCBC.h:13-51, IMRPhenomD_internals.h:649-665)
class Net(C.Structure):
    _fields_ = [("Nifo", C.c_int), ("Tobs", C.c_double), ("tmax", C.c_double), ("tmin", C.c_double),
                ("GMST", C.c_double), ("labels", C.POINTER(C.c_int)), ("tds", C.POINTER(C.c_double)),
                ("delays", C.POINTER(C.POINTER(C.c_double))), ("lstart", C.POINTER(C.c_int)),
                ("lstop", C.POINTER(C.c_int))]


class RealVector(C.Structure):
    _fields_ = [("data", C.POINTER(C.c_double)), ("length", C.c_size_t)]


class AmpPhaseFDWaveform(C.Structure):
    _fields_ = [("freq", C.POINTER(C.c_double)), ("amp", C.POINTER(C.c_double)),
                ("phase", C.POINTER(C.c_double)), ("length", C.c_size_t)]


_PD = C.POINTER(C.c_double)
_PPD = C.POINTER(_PD)
_PPPD = C.POINTER(_PPD)


class Het(C.Structure):
    _fields_ = [("M", C.c_int), ("MM", C.c_int), ("MN", C.c_int), ("ell", C.c_int), ("J", C.c_int),
                ("NR", C.c_int), ("hh", C.c_double), ("hr", C.c_double), ("logLb", C.c_double),
                ("IP", _PPPD), ("SL", _PPPD), ("amp", _PPD), ("phase", _PPD), ("rc", _PPD), ("rs", _PPD),
                ("aa", _PPD), ("lc", _PPPD), ("ls", _PPPD), ("pref", _PD), ("fgrid", C.POINTER(C.c_int)),
                ("freq", C.POINTER(RealVector))]


class HetTables(C.Structure):
    _fields_ = [("M", C.c_int), ("MN", C.c_int), ("MM", C.c_int), ("J", C.c_int), ("NR", C.c_int),
                ("logLb", C.c_double), ("fgrid", C.POINTER(C.c_int))] + \
               [(k, _PD) for k in ("freq", "amp", "phase", "IP", "SL", "lc", "ls", "aa", "rc", "rs")]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `python -m quickcbc_b200.build`")
        L = C.CDLL(LIB_PATH)
        i, d, vp, ll = C.c_int, C.c_double, C.c_void_p, C.c_longlong
        pi = C.POINTER(C.c_int)
        L.qcbc_last_error.restype = C.c_char_p
        L.qcbc_version.restype = C.c_char_p
        L.qcbc_launch_count.restype = ll
        L.qcbc_init.argtypes = [i]
        L.qcbc_set_qnm_table.argtypes = [_PD, _PD, _PD, i]
        L.qcbc_event_open.restype = vp
        L.qcbc_event_open.argtypes = [i, pi, d, d, i, _PD, i, _PD, i, d, d]
        L.qcbc_event_close.argtypes = [vp]
        L.qcbc_event_device_bytes.restype = ll
        L.qcbc_event_device_bytes.argtypes = [vp]
        # host arrays as plain addresses (a numpy array's .ctypes.data): the batched calls are
        # made per sampler step, and building a typed pointer per argument costs microseconds
        L.qcbc_lnl_full.argtypes = [vp, vp, i, vp, vp, i]
        L.qcbc_lnl_full_dev.argtypes = [vp, vp, i, vp, vp, i, vp]
        L.qcbc_lnl_full_noalloc.argtypes = [vp, vp, i, vp, vp, i, vp]
        L.qcbc_synchronize.argtypes = []
        L.qcbc_batch_create.restype = vp
        L.qcbc_batch_create.argtypes = [C.POINTER(vp), i]
        L.qcbc_batch_destroy.argtypes = [vp]
        L.qcbc_batch_set_slot.argtypes = [vp, i, vp]
        L.qcbc_batch_set_tiling.argtypes = [vp, i, i]
        L.qcbc_batch_get_tiling.argtypes = [vp, pi, pi]
        L.qcbc_batch_autotune.argtypes = [vp, pi, _PD, i, i]
        L.qcbc_lnl_multi.argtypes = [vp, pi, _PD, i, _PD, _PD, i]
        L.qcbc_time_lnl_multi.argtypes = [vp, i, i, i, i, C.POINTER(C.c_float)]
        L.qcbc_het_set.argtypes = [vp, C.POINTER(HetTables)]
        L.qcbc_het_setup.argtypes = [vp, _PD, pi, i, i, i, i]
        L.qcbc_het_sizes.argtypes = [vp, pi, pi, pi, pi, pi]
        L.qcbc_het_export.argtypes = [vp, pi] + [_PD] * 11
        L.qcbc_lnl_het.argtypes = [vp, vp, i, vp, i]
        L.qcbc_lnl_intrinsic.argtypes = [vp, _PD, i, _PD, _PD, i]
        L.qcbc_het_diff.argtypes = [vp, _PD, _PD, i, _PD]
        L.qcbc_het_fisher.argtypes = [vp, _PD, i, _PD]
        L.qcbc_het_space.argtypes = [vp, _PD, _PD, _PD, pi, pi, pi]
        L.qcbc_het_space_grid.argtypes = [vp, pi]
        L.qcbc_lnl_multi_het.argtypes = [vp, pi, _PD, i, _PD, i]
        L.qcbc_lnl_het_dev.argtypes = [vp, vp, i, vp, i, vp]
        L.qcbc_sky_ring_map.argtypes = [_PD, _PD, d, i, i, d, C.POINTER(d)]
        L.qcbc_set_full_launch.argtypes = [vp, i, i]
        L.qcbc_get_full_launch.argtypes = [vp, i, i, pi, pi]
        L.qcbc_device_alloc.restype = vp
        L.qcbc_device_alloc.argtypes = [ll]
        L.qcbc_device_free.argtypes = [vp]
        L.qcbc_memcpy_h2d.argtypes = [vp, vp, ll]
        L.qcbc_memcpy_d2h.argtypes = [vp, vp, ll]
        L.qcbc_time_lnl_full.argtypes = [vp, vp, i, i, i, i, C.POINTER(C.c_float), C.POINTER(C.c_float)]
        L.qcbc_time_lnl_het.argtypes = [vp, vp, i, i, i, i, C.POINTER(C.c_float)]
        # reference-signature entry points
        L.qcbc_set_band.argtypes = [d, d]
        L.qcbc_bind_data.argtypes = [C.POINTER(Net), _PPD, _PPD, i, d]
        L.log_likelihood_full.restype = d
        L.log_likelihood_full.argtypes = [C.POINTER(Net), _PPD, _PD, C.POINTER(RealVector), _PPD, _PD, i, d]
        L.log_likelihood_het.restype = d
        L.log_likelihood_het.argtypes = [C.POINTER(Net), C.POINTER(Het), _PD, d]
        L.qcbc_time_dropin.restype = i
        L.qcbc_time_dropin.argtypes = [i, C.POINTER(Net), C.POINTER(Het), _PPD, C.POINTER(RealVector), _PPD, i, d, _PD,
                                       i, i, i, _PD, _PD]
        L.heterodyne.restype = None
        L.heterodyne.argtypes = [C.POINTER(Net), C.POINTER(Het), _PPD, _PD, C.POINTER(RealVector), _PPD, i, d]
        L.fulltemplates.restype = None
        L.fulltemplates.argtypes = [C.POINTER(Net), _PPD, C.POINTER(RealVector), _PD, i]
        L.fullphaseamp.restype = None
        L.fullphaseamp.argtypes = [C.POINTER(Net), _PPD, _PPD, C.POINTER(RealVector), _PD, i]
        L.IMRPhenomDGenerateh22FDAmpPhase.restype = i
        L.IMRPhenomDGenerateh22FDAmpPhase.argtypes = [C.POINTER(C.POINTER(AmpPhaseFDWaveform)),
                                                       C.POINTER(RealVector)] + [d] * 7
        L.fourier_nwip.restype = d
        L.fourier_nwip.argtypes = [_PD, _PD, _PD, i, i, i]
        L.log_likelihood_intrinsic.restype = d
        L.log_likelihood_intrinsic.argtypes = [C.POINTER(Net), _PPD, _PD, C.POINTER(RealVector), _PPD, i, d]
        L.templates.restype = None
        L.templates.argtypes = [C.POINTER(Net), _PPD, C.POINTER(RealVector), _PD, i]
        L.AmpPhase.restype = None
        L.AmpPhase.argtypes = [_PD, _PD, C.POINTER(RealVector), _PD, i]
        L.het_diff.restype = d
        L.het_diff.argtypes = [C.POINTER(Net), C.POINTER(Het), _PD, _PD]
        L.het_space.restype = None
        L.het_space.argtypes = [C.POINTER(Net), C.POINTER(Het), _PD, _PD, _PD, C.POINTER(RealVector), _PPD, i, d]
        L.Fisher_Het.restype = None
        L.Fisher_Het.argtypes = [C.POINTER(Net), C.POINTER(Het), _PPD, _PD, d]
        # input stage (include/qcbc_ingest.h)
        cp = C.c_char_p
        L.qcbc_framed_length.argtypes = [cp, pi]
        L.qcbc_read_framed.argtypes = [cp, i, _PD, _PD]
        L.qcbc_read_spec.argtypes = [cp, i, _PD, _PD]
        L.qcbc_analysis_paths.argtypes = [cp, d, d, i, cp, cp, i]
        L.qcbc_condition_data.argtypes = [i, i, d, _PD, i, _PD, i]
        L.qcbc_load_analysis.argtypes = [cp, d, d, i, pi, i, _PD, i, _PD, _PD, i]
        L.qcbc_psd_model_open.restype = vp
        L.qcbc_psd_model_open.argtypes = [cp, i, pi]
        L.qcbc_psd_model_create.restype = vp
        L.qcbc_psd_model_create.argtypes = [i, pi, pi, i, i, i, _PD, _PD, _PD]
        L.qcbc_psd_model_info.argtypes = [vp, pi, pi, pi, pi]
        L.qcbc_psd_model_close.argtypes = [vp]
        L.qcbc_psd_draw.argtypes = [vp, i, d, i, _PD, i]
        L.qcbc_event_set_psd_sample.argtypes = [vp, vp, i]
        L.qcbc_event_set_psd.argtypes = [vp, _PD, i]
        L.makespec.restype = None
        L.makespec.argtypes = [i, i] + [_PD] * 8 + [d, i]
        _lib = L
    return _lib


def last_error() -> str:
    return lib().qcbc_last_error().decode()


def check(rc):
    if rc != QCBC_OK:
        raise QcbcError(rc, last_error())
    return rc


def launch_count() -> int:
    return int(lib().qcbc_launch_count())

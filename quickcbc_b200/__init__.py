"""B200-native likelihood hot path for QuickCBC.

IMRPhenomD frequency-domain amplitude/phase, detector projection with time and
phase shifts, and the PSD-weighted inner products behind the full and
heterodyned log-likelihoods, as hand-written sm_100a CUDA kernels behind a
C ABI (include/qcbc_gpu.h, include/qcbc_quickcbc.h).  See ``engine`` for the
host interface and ``synth`` for the seeded synthetic workloads.
"""
from ._lib import FP64, MIXED, QcbcError, launch_count  # noqa: F401
from .engine import (Event, Batch, DeviceBuffer, amp_phase, ampphase, fourier_nwip, fullphaseamp,  # noqa: F401
                     fulltemplates, templates, het_space, log_likelihood_full, log_likelihood_intrinsic, set_band,
                     LegacyHet, sky_ring_map,
                     time_lnl_full, time_lnl_het)

__all__ = ["FP64", "MIXED", "QcbcError", "Event", "Batch", "DeviceBuffer", "amp_phase", "ampphase", "fourier_nwip",
           "fullphaseamp", "fulltemplates", "templates", "het_space", "log_likelihood_full", "log_likelihood_intrinsic", "set_band",
           "LegacyHet", "sky_ring_map", "time_lnl_full", "time_lnl_het", "launch_count"]

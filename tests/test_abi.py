"""The C-ABI library loads without a GPU and exports every function that
include/*.h declares (no compute calls here)."""
import ctypes
import os
import re

import pytest

from conftest import ROOT


def declared_functions():
    names = set()
    for h in ("qcbc_gpu.h", "qcbc_quickcbc.h", "qcbc_serve.h"):
        text = open(os.path.join(ROOT, "include", h)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^[A-Za-z_][\w \*]*?\b([A-Za-z_]\w*)\s*\(", text, flags=re.M):
            name = m.group(1)
            if name not in ("defined",):
                names.add(name)
    return sorted(names)


def test_header_parse_sanity():
    names = declared_functions()
    for must in ("qcbc_event_open", "qcbc_lnl_full", "qcbc_lnl_het", "qcbc_het_setup", "log_likelihood_full",
                 "log_likelihood_het", "heterodyne", "fulltemplates", "fullphaseamp",
                 "IMRPhenomDGenerateh22FDAmpPhase", "fourier_nwip"):
        assert must in names


def test_library_exports_every_declared_symbol():
    from quickcbc_b200 import _lib
    lib = ctypes.CDLL(_lib.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, f"not exported: {missing}"


def test_library_is_sm100a_only():
    """The build targets sm_100a exclusively (no PTX for other targets)."""
    from quickcbc_b200 import build
    flags = " ".join(build.NVCC_FLAGS)
    assert "arch=compute_100a,code=sm_100a" in flags
    assert "compute_90" not in flags and "sm_90" not in flags


def test_no_gpu_gives_clear_error():
    """Without a usable GPU the engine raises instead of computing on the CPU."""
    from quickcbc_b200 import _lib
    lib = _lib.lib()
    if lib.qcbc_init(0) == 0:
        pytest.skip("a GPU is present")
    assert "CUDA" in _lib.last_error() or "device" in _lib.last_error()
    import quickcbc_b200 as q
    import numpy as np
    with pytest.raises(q.QcbcError):
        q.Event([0], 4.0, 0.0, 64, np.zeros((1, 64)), np.ones((1, 33)))

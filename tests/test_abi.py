"""The C-ABI library loads without a GPU and exports every function that
include/*.h declares (no compute calls here)."""
import ctypes
import os
import re

import pytest

from conftest import ROOT


def declared_functions():
    names = set()
    for h in sorted(f for f in os.listdir(os.path.join(ROOT, "include")) if f.endswith(".h")):
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
                 "IMRPhenomDGenerateh22FDAmpPhase", "fourier_nwip", "qcbc_condition_data", "makespec",
                 "qcbc_event_set_psd_sample", "qcbc_server_set_device_steps", "qcbc_lnl_multi_dev"):
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


def test_psd_model_without_gpu_fails_loudly():
    """The GPU-side input stage has no CPU path: without a device it reports an error."""
    from quickcbc_b200 import _lib, ingest
    import numpy as np
    if _lib.lib().qcbc_init(0) == 0:
        pytest.skip("a GPU is present")
    with pytest.raises(_lib.QcbcError):
        ingest.condition_data(np.zeros((1, 64)), 4.0)
    with pytest.raises(_lib.QcbcError):
        ingest.PsdModel(np.array([[0.0, 1.0, 2.0]]), np.zeros((1, 1, 3)), np.zeros((1, 1, 0, 5)))

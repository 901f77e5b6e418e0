import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built libqcbc_gpu.so")
    config.addinivalue_line("markers", "slow: long-running CPU test")


def _ensure_oracle():
    from oracle import ora
    if not ora.available():
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "oracle"], check=True,
                       stdout=subprocess.DEVNULL)
    return ora


@pytest.fixture(scope="session")
def ora():
    return _ensure_oracle()


@pytest.fixture(scope="session")
def refo():
    from oracle import ref
    if not ref.available():
        pytest.skip("reference oracle (oracle/_ref) not built on this machine")
    return ref


def load_golden(name):
    return dict(np.load(os.path.join(GOLDEN, name), allow_pickle=False))


@pytest.fixture(scope="session")
def golden():
    return load_golden


class GoldenEvent:
    """Event rebuilt from a golden fixture (same attributes as synth.Event)."""

    def __init__(self, z):
        self.labels = z["labels"].astype(np.int32)
        self.Tobs = float(z["Tobs"])
        self.fs = float(z["fs"])
        self.N = int(z["N"])
        self.fmin = float(z["fmin"])
        self.GMST = float(z["GMST"])
        self.D = z["D"]
        self.SN = z["SN"]
        self.inj = z["inj"]
        self.freq = np.arange(self.N // 2, dtype=np.float64) / self.Tobs
        self.freq[0] = 1.0 / self.Tobs          # the reference's grid (QuickCBC.c:418-419)
        self.freq[0] = 1.0 / self.Tobs

    @property
    def nifo(self):
        return len(self.labels)


@pytest.fixture(scope="session")
def cfg1_event():
    z = load_golden("cfg1.npz")
    return GoldenEvent(z), z


def oracle_template(ora):
    def t(info, p):
        return ora.fulltemplates(info["labels"], info["GMST"], info["freq"], p, info["N"])
    return t


def prior_bounds(Tobs):
    """MCMC_all's prior box (QuickCBC.c:1871-1896, ConstCBC.h:48-57), as the fixtures used."""
    from quickcbc_b200 import synth
    M, PC = synth.MSUN_SI, synth.PC_SI
    pmin = np.array([np.log(0.5 * M), np.log(0.5 * M), -0.85, -0.85, 0.0, max(Tobs - 3.5, 1.5),
                     np.log(1e6 * PC), 0.0, -1.0, 0.0, -1.0])
    pmax = np.array([np.log(160 * M), np.log(300 * M), 0.85, 0.85, 2 * np.pi, Tobs - 0.5,
                     np.log(1e10 * PC), 2 * np.pi, 1.0, np.pi, 1.0])
    return pmin, pmax

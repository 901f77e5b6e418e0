"""Input files on the host (no GPU): framed_/spec_ readers of include/qcbc_ingest.h against
the reference's own reading (QuickCBC.c:198-242) and numpy, including the row count's edge
cases, and the file names QuickCBC.c builds."""
import os

import numpy as np
import pytest

from quickcbc_b200 import ingest, synth
from quickcbc_b200._lib import QcbcError

ref = pytest.importorskip("oracle.ref")
if not ref.available():
    pytest.skip("oracle/_ref not built", allow_module_level=True)


@pytest.mark.parametrize("text", [
    "0 1.5\n1 -2.5e-21\n2 3\n",                    # trailing newline
    "0 1.5\n1 -2.5e-21\n2 3",                      # ends on the last number: one row fewer
    "0 1.5\n1 -2.5e-21\n2 3\n\n   \n",             # trailing blank lines
    "0 1.5\r\n1 -2.5e-21\r\n2 3\r\n",              # CRLF
    "  0\t1.5 1 -2.5E-21\n2 +3.0\n",               # free layout, as fscanf reads it
    "",                                            # empty
])
def test_framed_length_matches_reference_loop(tmp_path, text):
    p = tmp_path / "framed.dat"
    p.write_text(text)
    assert ingest.framed_length(p) == max(ref.framed_count(p), 0)


def test_framed_length_rejects_bad_content(tmp_path):
    p = tmp_path / "bad.dat"
    p.write_text("0 1\n1 x\n")
    assert ref.framed_count(p) == -2          # the reference's loop would not end on this file
    with pytest.raises(QcbcError):
        ingest.framed_length(p)
    p.write_text("0 1\n1\n")
    with pytest.raises(QcbcError):
        ingest.framed_length(p)
    with pytest.raises(QcbcError):
        ingest.framed_length(tmp_path / "missing.dat")


def test_readers_match_numpy(tmp_path):
    rng = np.random.default_rng(7)
    x = rng.normal(size=(2, 512)) * 1e-21
    SN = np.abs(rng.normal(size=(2, 256))) * 1e-46
    SM = SN * 0.5
    synth.write_analysis_files(str(tmp_path), [0, 2], 4.0, 1126259462.4, x, SN, SM)
    fr, sp = ingest.analysis_paths(str(tmp_path), 4.0, 1126259462.4, 2)
    assert os.path.basename(fr) == "framed_4_1126259462_2.dat" and os.path.basename(sp) == "spec_4_1126259462_2.dat"
    assert ingest.framed_length(fr) == 512 == ref.framed_count(fr)
    t, xr = ingest.read_framed(fr, 512)
    a = np.loadtxt(fr)
    assert np.array_equal(t, a[:, 0]) and np.array_equal(xr, a[:, 1])
    assert np.array_equal(xr, x[1]), "%.16e text round-trips every double"
    s1, s2 = ingest.read_spec(sp, 256)
    b = np.loadtxt(sp)
    assert np.array_equal(s1, b[:, 1]) and np.array_equal(s2, b[:, 2])
    np.testing.assert_allclose(s1, SN[1], rtol=1e-15)
    with pytest.raises(QcbcError):
        ingest.read_spec(sp, 257)                # fewer rows than asked for
    with pytest.raises(QcbcError):
        ingest.read_framed(fr, 513)

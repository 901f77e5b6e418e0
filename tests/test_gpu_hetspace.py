"""Heterodyne grid search het_space (QuickCBC.c:4570-4910) against the grids
the reference's own het_space produced (tests/golden/het1.npz for config 1,
grid3.npz for config 3), through the reference-signature drop-in and the
event API, and the grid feeding the GPU heterodyne setup."""
import numpy as np
import pytest

import quickcbc_b200 as q
from quickcbc_b200 import synth
from conftest import oracle_template, load_golden, prior_bounds

pytestmark = pytest.mark.gpu


def test_het_space_config1_matches_reference(cfg1_event, golden):
    ev, _ = cfg1_event
    h = golden("het1.npz")
    pmin, pmax = prior_bounds(ev.Tobs)
    g, MN, MM, J, NR = q.het_space(ev.labels, ev.GMST, ev.Tobs, ev.inj, pmin, pmax, ev.freq, ev.SN, ev.N)
    assert (MN, MM, J) == (int(h["MN"]), int(h["MM"]), int(h["J"]))
    assert np.array_equal(g, h["fgrid"])
    assert NR == (len(g) - 1) // J
    e = q.Event.from_synthetic(ev)
    g2, MN2, MM2 = e.het_space(ev.inj, pmin, pmax)
    assert np.array_equal(g2, g) and (MN2, MM2) == (MN, MM)
    # the grid drives the GPU heterodyne setup; its het lnL matches the reference's on that grid
    e.het_setup(ev.inj, g2, MN2, MM2, 2)
    L = e.lnl_het(h["params"], q.FP64)
    np.testing.assert_allclose(L, h["lnl"], rtol=0, atol=1e-8)
    e.close()


def test_het_space_config3_matches_reference(ora):
    g3 = load_golden("grid3.npz")
    ev = synth.config_event(3, oracle_template(ora))
    assert np.array_equal(ev.inj, g3["inj"])
    pmin, pmax = prior_bounds(ev.Tobs)
    e = q.Event.from_synthetic(ev)
    g, MN, MM = e.het_space(ev.inj, pmin, pmax)
    assert (MN, MM) == (int(g3["MN"]), int(g3["MM"]))
    assert np.array_equal(g, g3["fgrid"])
    e.close()

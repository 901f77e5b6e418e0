"""Host-side parameter-set generators (CPU only): the wrap into the reference's ranges and the
search for sets at given lnL drops that the config-3 fixtures and bench use."""
import numpy as np

from quickcbc_b200 import synth


def test_wrap_params_ranges_and_eta():
    rng = np.random.default_rng(1)
    P = rng.normal(size=(500, 11)) * 5.0
    P[:, 1] = 70.0 + rng.normal(size=500)
    P[:, 0] = P[:, 1] + 0.6 * np.log(rng.uniform(0.05, 0.45, size=500))   # some eta above 1/4
    W = synth.wrap_params(P)
    assert np.all((W[:, 4] >= 0) & (W[:, 4] < 2 * np.pi)) and np.all((W[:, 7] >= 0) & (W[:, 7] < 2 * np.pi))
    assert np.all((W[:, 9] >= 0) & (W[:, 9] < np.pi))
    assert np.all(np.abs(W[:, [8, 10]]) <= 1.0)
    assert np.all(np.abs(W[:, 2:4]) <= 0.85)
    eta = np.exp((W[:, 0] - W[:, 1]) / 0.6)
    assert np.all(eta <= 0.25)
    np.testing.assert_array_equal(W[:, 0], P[:, 0])               # chirp mass kept
    inside = np.exp((P[:, 0] - P[:, 1]) / 0.6) <= 0.25
    np.testing.assert_array_equal(W[inside, 1], P[inside, 1])     # only eta > 1/4 moves Mt
    # reflection about 1/4: 0.25 + d -> 0.25 - d
    d = np.exp((P[~inside, 0] - P[~inside, 1]) / 0.6) - 0.25
    np.testing.assert_allclose(eta[~inside], np.clip(0.25 - d, 0.05, 0.25), rtol=1e-9)


def test_cloud_at_drops_hits_the_targets_on_a_quadratic_likelihood():
    rng = np.random.default_rng(2)
    A = rng.normal(size=(11, 11))
    F = A @ A.T + np.diag(np.geomspace(10.0, 1e6, 11))
    c = np.array([69.9, 70.8, 0.03, -0.02, 2.0, 126.0, 56.0, 2.6, -0.6, 0.9, -0.65])

    def lnl(P):
        d = synth.wrap_params(P) - c
        return 400.0 - 0.5 * np.einsum("bi,ij,bj->b", d, F, d)
    drops = np.concatenate([rng.uniform(0.5, 10.0, 20), rng.uniform(100.0, 400.0, 10)])
    P = synth.cloud_at_drops(rng, c, F, drops, lnl)
    np.testing.assert_allclose(400.0 - lnl(P), drops, rtol=1e-6, atol=1e-6)
    # the steps follow the Fisher metric: sets lie along Fisher steps, not along one axis
    assert np.linalg.matrix_rank(P - c) >= 10

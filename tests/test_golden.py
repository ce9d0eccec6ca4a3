"""The oracle against its committed golden fixtures (tests/golden/tiny_inversion.npz,
made by tests/golden/make_golden.py), and the finite-difference pattern of
S4/Gradient_check.F90 in those fixtures.  No GPU."""
import os

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "tiny_inversion.npz")


@pytest.fixture(scope="module")
def golden():
    with np.load(GOLDEN) as d:
        return {k: d[k] for k in d.files}


def test_oracle_reproduces_the_fixtures(golden):
    import golden.make_golden as G
    now = G.compute()
    for k in ("ID", "store_eq", "fd_nodes"):
        assert np.array_equal(now[k], golden[k]), k
    for k in ("dis", "traces0", "g_lambda", "g_mu", "fd_mu", "fd_lambda"):
        ref = golden[k]
        assert np.linalg.norm(now[k] - ref) <= 1e-13 * np.linalg.norm(ref), k
    assert abs(float(now["misfit"]) - float(golden["misfit"])) <= 1e-13 * float(golden["misfit"])


def test_fixture_gradient_follows_finite_differences(golden):
    """Gradient_check pattern: the sign-flipped gradient before the gradient mass
    matches FD derivatives of the misfit (the OtD gradient is not the exact derivative
    of the discrete misfit, so to a few percent)."""
    fd = np.concatenate([golden["fd_mu"], golden["fd_lambda"]])
    adj = np.concatenate([golden["adj_mu"], golden["adj_lambda"]])
    cos = float(fd @ adj / (np.linalg.norm(fd) * np.linalg.norm(adj)))
    assert cos > 0.999
    big = np.abs(fd) > 0.1 * np.abs(fd).max()
    assert np.median(np.abs(fd[big] - adj[big]) / np.abs(fd[big])) < 0.1

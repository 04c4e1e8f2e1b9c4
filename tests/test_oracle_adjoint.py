"""The CPU adjoint oracle against the reference's own discrete adjoint and against finite differences.

Golden vectors (tests/golden/adjoint_*.npz) are the reference DifferentiableSimulation's signals and its
gradient of sum(weights * signals) on the CPU (tests/golden/make_golden.py)."""
import numpy as np
import pytest

from oracle.adjoint_oracle import AdjointOracle
from torchfdtd_b200 import Project
from torchfdtd_b200.plan import plan_grid

TOL = {'float32': 1e-6, 'float64': 1e-13}


def rel(a, b):
    return float(np.linalg.norm((np.asarray(a) - np.asarray(b)).ravel()) / np.linalg.norm(np.asarray(b).ravel()))


@pytest.mark.parametrize('name', ['2d_float32', '2d_float64', '3d_float32', '3d_float64', 'mesh2d_float32', 'mesh2d_float64',
                                  'mesh3d_float32', 'mesh3d_float64'])
def test_oracle_adjoint_matches_reference_adjoint(golden, name):
    d = np.load(golden / f'adjoint_{name}.npz')
    project = Project.model_validate_json(str(d['project']))
    plan = plan_grid(project, polarization='both')
    o = AdjointOracle(plan, d['epsilon'])
    np.testing.assert_array_equal(o.forward(), d['signals'])
    gradient = o.backward(d['weights'].astype(plan.dtype))
    assert rel(gradient, d['gradient']) <= TOL[project.region.precision]


def test_oracle_adjoint_matches_central_differences(golden):
    d = np.load(golden / 'adjoint_2d_float64.npz')
    project = Project.model_validate_json(str(d['project']))
    eps, w = d['epsilon'], d['weights']

    def objective(e):
        return float((AdjointOracle(plan_grid(project, polarization='both'), e).forward() * w).sum())
    o = AdjointOracle(plan_grid(project, polarization='both'), eps)
    o.forward()
    gradient = o.backward(w)
    rng = np.random.default_rng(3)
    big = np.argsort(np.abs(gradient).ravel())[-3:]
    for flat in list(big) + list(rng.integers(0, eps.size, 2)):
        idx = np.unravel_index(flat, eps.shape)
        h = 1e-6
        up, down = eps.copy(), eps.copy()
        up[idx] += h
        down[idx] -= h
        fd = (objective(up) - objective(down)) / (2 * h)
        assert abs(gradient[idx] - fd) <= 1e-5 * max(abs(fd), np.abs(gradient).max() * 1e-3)

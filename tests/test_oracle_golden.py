"""The CPU oracle (NumPy and C restatements) against the reference's own golden vectors.

tests/golden/*.npz were written by the reference's CPU path (tests/golden/make_golden.py);
the oracle, fed by this package's host planner, must reproduce them bitwise: E, H, every
CPML memory, point traces, the voxelized permittivity and the DFT planes.
"""
from pathlib import Path

import numpy as np
import pytest

from oracle.cpu import CpuOracle
from oracle.yee_oracle import YeeOracle
from torchfdtd_b200 import Project, Region
from torchfdtd_b200.plan import plan_grid

GOLDEN = Path(__file__).resolve().parent / 'golden'
SIMS = sorted(p.stem[4:] for p in GOLDEN.glob('sim_*.npz'))
STATES = sorted(p.stem[6:] for p in GOLDEN.glob('state_*.npz'))


def test_golden_files_present():
    assert len(SIMS) >= 7 and len(STATES) >= 8


@pytest.mark.parametrize('name', SIMS)
def test_numpy_oracle_reproduces_reference_simulation(name):
    d = np.load(GOLDEN / f'sim_{name}.npz')
    plan = plan_grid(Project.model_validate_json(str(d['project'])))
    np.testing.assert_array_equal(plan.epsilon, d['epsilon'])
    o = YeeOracle(plan).run()
    np.testing.assert_array_equal(o.E, d['E'])
    np.testing.assert_array_equal(o.H, d['H'])
    np.testing.assert_array_equal(o.traces, d['signals'])
    for k, entry in enumerate(o.planes):
        np.testing.assert_array_equal(entry['value'], d[f'plane{k}_fields'])


@pytest.mark.parametrize('name', [n for n in SIMS if not n.startswith(('tfsf', 'drude', 'frozen'))])
def test_c_oracle_reproduces_reference_simulation(name):
    """(The C oracle has no TFSF boxes or dispersive materials; the NumPy oracle checks those scenes.)"""
    d = np.load(GOLDEN / f'sim_{name}.npz')
    plan = plan_grid(Project.model_validate_json(str(d['project'])), polarization='both')
    o = CpuOracle(plan, threads=2).run()
    np.testing.assert_array_equal(o.E, d['E'])
    np.testing.assert_array_equal(o.H, d['H'])
    np.testing.assert_array_equal(o.traces, d['signals'])


@pytest.mark.parametrize('name', STATES)
@pytest.mark.parametrize('impl', ['numpy', 'c'])
def test_oracles_reproduce_reference_cpml_states(name, impl):
    d = np.load(GOLDEN / f'state_{name}.npz')
    region = Region.model_validate_json(str(d['region']))
    plan = plan_grid(Project(region=region), polarization='both')
    plan.inv_eps = d['init_inverse_permittivity']
    steps = int(d['steps'])
    if impl == 'numpy':
        o = YeeOracle(plan)
        o.E[:], o.H[:] = d['init_E'], d['init_H']
        for _ in range(steps):
            o.update_E()
            o.update_H()
    else:
        o = CpuOracle(plan, threads=2)
        o.E[:], o.H[:] = d['init_E'], d['init_H']
        o.run(steps)
    np.testing.assert_array_equal(o.E, d['E'])
    np.testing.assert_array_equal(o.H, d['H'])
    psi = [d[f'psi_{i}'] for i in range(len([k for k in d.files if k.startswith('psi_')]))]
    assert [s.shape for s in o.memory_states] == [s.shape for s in psi]
    for got, want in zip(o.memory_states, psi):
        np.testing.assert_array_equal(got, want)


def test_reference_fixture_itself_when_the_reference_tree_is_present(reference_tree):
    """The reference's own golden result (tests/fixtures/npz/tiny_2d_complete.npz), read in place."""
    root = reference_tree / 'tests' / 'fixtures'
    p = Project.load(root / 'projects' / 'tiny_result.json')
    d = np.load(root / 'npz' / 'tiny_2d_complete.npz')
    o = YeeOracle(plan_grid(p)).run()
    np.testing.assert_array_equal(o.E, d['E'])
    np.testing.assert_array_equal(o.H, d['H'])
    np.testing.assert_array_equal(o.traces, d['signals'])


def test_a_planted_mistake_in_the_oracle_is_caught():
    """A one-ulp change of the Courant number in the oracle breaks bitwise parity with the goldens."""
    d = np.load(GOLDEN / 'sim_tmz.npz')
    plan = plan_grid(Project.model_validate_json(str(d['project'])))
    plan.courant = float(np.nextafter(np.float32(plan.courant), np.float32(1)))
    o = YeeOracle(plan).run(60)
    assert not np.array_equal(o.E, YeeOracle(plan_grid(Project.model_validate_json(str(d['project'])))).run(60).E)

"""The 2D TMz tile kernel and batches of uneven 2D grids (one persistent launch per step).

Bar: bitwise equality of Ez, Hx, Hy, their CPML memories and traces with the reference's CPU path
(golden vectors) and with the oracle; batched runs bitwise equal to the same cases run one by one.
"""
import numpy as np
import pytest

from oracle.yee_oracle import YeeOracle
from torchfdtd_b200 import Project, Region
from torchfdtd_b200.plan import CURL_TERMS, plan_grid

pytestmark = pytest.mark.gpu

TM_FIELDS = (('E', 2), ('H', 0), ('H', 1))


def tm_psi_mask(plan):
    """Which entries of the reference memory_states order belong to the TMz terms."""
    mask = []
    for forward in (False, True):
        for axis, comp, out, _ in CURL_TERMS:
            if plan.shape[axis] == 1:
                continue
            for seg in plan.segments:
                if seg.forward == forward and seg.axis == axis:
                    mask.append(out == 2 if not forward else out in (0, 1))
    return mask


def native(plan, kernel, variant=0):
    from torchfdtd_b200.native import NativeGrid
    return NativeGrid(plan, kernel=kernel, variant=variant)


def assert_tm_equal(E, H, E_ref, H_ref):
    np.testing.assert_array_equal(E[..., 2], E_ref[..., 2])
    np.testing.assert_array_equal(H[..., 0], H_ref[..., 0])
    np.testing.assert_array_equal(H[..., 1], H_ref[..., 1])


@pytest.mark.parametrize('kernel', ['tile2d', 'gather'])
@pytest.mark.parametrize('precision', ['float32', 'float64'])
def test_tm_state_and_cpml_memories_match_reference_bitwise(golden, kernel, precision):
    """Random initial state of the reference's 2D CPML grid: the TMz components evolve on their own."""
    d = np.load(golden / f'state_pml2d_{precision}.npz')
    region = Region.model_validate_json(str(d['region']))
    plan = plan_grid(Project(region=region), polarization='TM')
    plan.inv_eps = d['init_inverse_permittivity']
    g = native(plan, kernel)
    assert g.kernel == kernel
    g.set_fields(d['init_E'], d['init_H'])
    g.step(int(d['steps']))
    E, H = g.get_fields()
    assert_tm_equal(E, H, d['E'], d['H'])
    assert (E[..., :2] == 0).all() and (H[..., 2] == 0).all()
    psi = g.get_psi()
    mask = tm_psi_mask(plan)
    assert len(psi) == len(mask)
    for k, (got, tm) in enumerate(zip(psi, mask)):
        if tm:
            np.testing.assert_array_equal(got, d[f'psi_{k}'])
        else:
            assert (got == 0).all()
    assert g.counter() == int(d['steps']) and g.device_status() == 0


def tm_project(size=(3.3, 2.5), mesh=.05, steps=24, precision='float32', pml=7, faces=None, monitors=(), sources=None):
    from torchfdtd_b200.models import BoundaryFace, Source, Structure
    region = Region(dimension='2d', size=(size[0], size[1], 1), mesh=mesh, pml_cells=pml, steps=steps,
                    precision=precision, backend='cuda')
    region.boundaries.x_min = BoundaryFace(layers=pml + 2, kappa=2, alpha=.04, alpha_polynomial=1)
    for name, face in (faces or {}).items():
        setattr(region.boundaries, name, face)
    if sources is None:
        sources = [Source(center=(-.05, .02, 0), component='Ez', pulse_cycles=1, wavelength=1.0),
                   Source(center=(.05, -.03, 0), component='Hy', pulse_cycles=1, wavelength=1.0, amplitude=.3)]
    return Project(region=region, structures=[Structure(kind='sphere', radius=.5, material='Si (constant n)')],
                   sources=sources, monitors=list(monitors))


def random_start(plan, oracle, seed):
    rng = np.random.default_rng(seed)
    oracle.E[:] = rng.normal(size=oracle.E.shape).astype(plan.dtype) * .01
    oracle.H[:] = rng.normal(size=oracle.H.shape).astype(plan.dtype) * .01


@pytest.mark.parametrize('precision', ['float32', 'float64'])
@pytest.mark.parametrize('shape', [(3.3, 2.5), (1.55, 1.0), (6.2, 0.95), (1.3, 4.1)])
def test_tile_kernel_ragged_shapes_match_oracle(precision, shape):
    """Shapes that leave partial tiles on both axes, kappa>1 CPML, E and H sources, random start."""
    from torchfdtd_b200.models import BoundaryFace
    project = tm_project(size=shape, precision=precision, faces={'y_max': BoundaryFace(kind='pec')})
    plan = plan_grid(project)
    assert plan.polarization == 'TM'
    full = plan_grid(project, polarization='both')
    oracle = YeeOracle(full)
    random_start(full, oracle, 3)
    g = native(plan, 'tile2d')
    g.set_fields(oracle.E, oracle.H)
    oracle.run()
    g.step(plan.steps)
    E, H = g.get_fields()
    assert_tm_equal(E, H, oracle.E, oracle.H)
    mask = tm_psi_mask(plan)
    for got, want, tm in zip(g.get_psi(), oracle.memory_states, mask):
        if tm:
            np.testing.assert_array_equal(got, want)


@pytest.mark.parametrize('ctas', [1, 5, 0])
def test_persistent_cta_count_does_not_change_results(ctas):
    project = tm_project(size=(4.1, 3.3), steps=20)
    plan = plan_grid(project)
    ref = native(plan, 'gather')
    ref.step(20)
    g = native(plan, 'tile2d', variant=ctas)
    g.step(20)
    for x, y in zip(ref.get_fields(), g.get_fields()):
        np.testing.assert_array_equal(x, y)
    np.testing.assert_array_equal(ref.get_traces(), g.get_traces())


def test_tile_kernel_graph_replay_equals_eager():
    import torch
    plan = plan_grid(tm_project(steps=30))
    a, b = native(plan, 'tile2d'), native(plan, 'tile2d')
    a.step(30)
    stream = torch.cuda.Stream()
    with torch.cuda.stream(stream):
        b.step(1, stream)
        b.reset()
        graph = torch.cuda.CUDAGraph()
        graph.capture_begin()
        b.step(3, stream)
        graph.capture_end()
        for _ in range(10):
            graph.replay()
    torch.cuda.synchronize()
    for x, y in zip(a.get_fields(), b.get_fields()):
        np.testing.assert_array_equal(x, y)
    assert b.counter() == 30


def uneven_cases(precision='float32', steps=(30, 30, 30, 30, 30)):
    from torchfdtd_b200.models import BoundaryFace, FieldMonitor, Monitor, Source, SpectrumSettings
    spec = SpectrumSettings(sampling='frequency', frequency_points=3, apodization='none')
    sizes = [(3.3, 2.5), (1.6, 4.05), (6.4, 1.2), (2.0, 2.0), (1.2, 0.9)]
    projects = []
    for k, (size, n) in enumerate(zip(sizes, steps)):
        faces = {'x_max': BoundaryFace(kind='pec')} if k == 3 else None
        mesh, pml = (.05 if k != 4 else .025), 5 + k
        monitors = [Monitor(center=(.2, .1, 0), component='Ez')]
        if k % 2 == 0:      # a plane across half of the non-PML interior
            monitors.append(FieldMonitor(center=(.1, 0, 0), size=(0, size[1] / 2 - pml * mesh, 1), spectrum=spec))
        src = [Source(center=(-.2 + .05 * k, .05, 0), component='Ez', pulse_cycles=1, wavelength=1.0 + .1 * k)]
        projects.append(tm_project(size=size, mesh=mesh, steps=n, precision=precision, pml=pml, faces=faces,
                                   monitors=monitors, sources=src))
    return projects


def assert_results_equal(a, b):
    np.testing.assert_array_equal(a.electric, b.electric)
    np.testing.assert_array_equal(a.magnetic, b.magnetic)
    np.testing.assert_array_equal(a.signals, b.signals)
    np.testing.assert_array_equal(a.frames, b.frames)
    np.testing.assert_array_equal(a.frame_steps, b.frame_steps)
    assert len(a.frequency_fields) == len(b.frequency_fields)
    for x, y in zip(a.frequency_fields, b.frequency_fields):
        np.testing.assert_array_equal(x['fields'], y['fields'])


@pytest.mark.parametrize('precision', ['float32', 'float64'])
def test_uneven_batch_equals_cases_run_alone(precision):
    from torchfdtd_b200 import Simulation
    from torchfdtd_b200.batch import run_tensor_batch
    projects = uneven_cases(precision)
    report = run_tensor_batch(projects, cuda_graph=True, cuda_graph_steps=4)
    assert report.successful and report.plan['tiles'] > len(projects)
    for p, item in zip(projects, report.items):
        alone = Simulation(p).run(kernel='tile2d')
        assert item.summary['cuda_kernel'] == 'fused_batch' and item.summary['kernel'] == 'tile2d'
        assert_results_equal(item.result, alone)


@pytest.mark.parametrize('precision', ['float32', 'float64'])
@pytest.mark.parametrize('graph', [False, True])
def test_persistent_batch_equals_cases_run_alone(precision, graph):
    """All steps of a replay in one cooperative launch over every member (uneven sizes, step counts, planes)."""
    from torchfdtd_b200 import Simulation
    from torchfdtd_b200.batch import run_tensor_batch
    projects = uneven_cases(precision, steps=(30, 12, 41, 10, 30))
    report = run_tensor_batch(projects, cuda_graph=graph, cuda_graph_steps=8 if graph else 1, launch=(0, 16, 1))
    assert report.successful and report.plan['launch'] == [0, 16, 1]
    for p, item in zip(projects, report.items):
        assert item.summary['steps'] == p.region.steps
        assert_results_equal(item.result, Simulation(p).run(kernel='tile2d'))


def test_batch_members_with_different_step_counts():
    from torchfdtd_b200 import Simulation
    from torchfdtd_b200.batch import run_tensor_batch
    projects = uneven_cases(steps=(30, 12, 41, 10, 30))
    report = run_tensor_batch(projects, cuda_graph=False)
    for p, item in zip(projects, report.items):
        assert item.summary['steps'] == p.region.steps
        assert_results_equal(item.result, Simulation(p).run(kernel='tile2d'))


def test_raw_batch_with_random_start_matches_oracle():
    """Every member from a random state through the C ABI batch entry points, each checked against the oracle."""
    from torchfdtd_b200.native import NativeBatch
    projects = uneven_cases()
    grids, oracles = [], []
    for k, p in enumerate(projects):
        plan = plan_grid(p)
        full = plan_grid(p, polarization='both')
        oracle = YeeOracle(full)
        random_start(full, oracle, 10 + k)
        g = native(plan, 'tile2d')
        g.set_fields(oracle.E, oracle.H)
        grids.append(g)
        oracles.append(oracle.run())
    batch = NativeBatch(grids)
    batch.set_launch(7, 9)
    assert batch.tiles() > len(grids)
    with pytest.raises(ValueError, match='batch'):
        grids[0].step(1)
    batch.step(30)
    batch.close()
    for g, o in zip(grids, oracles):
        assert g.counter() == 30
        E, H = g.get_fields()
        assert_tm_equal(E, H, o.E, o.H)
        np.testing.assert_array_equal(g.get_traces()[:, 0], o.traces[:, 0])


def test_batch_refuses_3d_and_started_plans():
    from torchfdtd_b200.native import NativeBatch
    p3 = plan_grid(Project(region=Region(dimension='3d', size=(1.2, 1.2, 1.2), mesh=.1, pml_cells=3, steps=10, backend='cuda')))
    with pytest.raises(ValueError, match='2D TMz'):
        NativeBatch([native(p3, 'auto')])
    g = native(plan_grid(tm_project()), 'tile2d')
    g.step(1)
    with pytest.raises(ValueError, match='step 0'):
        NativeBatch([g])


def test_grouped_batch_runs_mixed_cases_in_input_order():
    from torchfdtd_b200 import Simulation
    from torchfdtd_b200.batch import plan_grouped_batch, run_grouped_batch
    projects = uneven_cases()[:3]
    p3 = Project(region=Region(dimension='3d', size=(1.2, 1.2, 1.2), mesh=.1, pml_cells=3, steps=10, backend='cuda'))
    cases = [projects[0], p3, projects[1], projects[2]]
    plan = plan_grouped_batch(cases)
    assert [c['execution'] for c in plan['cohorts']] == ['fused_cuda_batch', 'simulation']
    report = run_grouped_batch(cases)
    assert [i.id for i in report.items] == [f'case-{k:04d}' for k in range(4)]
    assert report.items[1].summary['kernel'] in ('march', 'gather')
    assert_results_equal(report.items[2].result, Simulation(projects[1]).run(kernel='tile2d'))


def test_batch_tuner_picks_a_measured_cta_count_and_results_do_not_change():
    from torchfdtd_b200.batch import run_tensor_batch
    from torchfdtd_b200.tuning import tune_tensor_batch
    projects = uneven_cases()
    shapes = [(1, 8), (4, 0), (0, 12), (0, 0)]
    tuning = tune_tensor_batch(projects, candidates=shapes, steps=2, repeats=3)
    assert tuning.kind == 'batch' and tuple(tuning.choice[:2]) in shapes and tuning.choice[2] == 0
    assert sorted((r['ctas'], r['rows']) for r in tuning.candidates) == sorted(shapes)
    auto = run_tensor_batch(projects, launch='auto')
    plain = run_tensor_batch(projects)
    assert auto.plan['tuning']['kind'] == 'batch'
    for a, b in zip(auto.items, plain.items):
        assert_results_equal(a.result, b.result)


def test_batch_accepts_per_case_epsilon():
    from torchfdtd_b200 import Simulation
    from torchfdtd_b200.batch import run_tensor_batch
    projects = uneven_cases()[:3]
    rng = np.random.default_rng(4)
    eps = [None] + [rng.uniform(1, 4, size=tuple(plan_grid(p).shape)).astype(np.float32) for p in projects[1:]]
    report = run_tensor_batch(projects, epsilon=eps)
    for p, e, item in zip(projects, eps, report.items):
        assert_results_equal(item.result, Simulation(p, epsilon=e).run(kernel='tile2d'))

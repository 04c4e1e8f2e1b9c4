"""Scene model, host planning and the refusals of the drop-in boundary (no GPU)."""
import json
import math
from pathlib import Path

import numpy as np
import pytest

from torchfdtd_b200 import (Boundaries, BoundaryFace, FieldMonitor, Material, Monitor, Project, Region, Simulation, Source,
                            SpectrumSettings, Structure)
from torchfdtd_b200.plan import CURL_TERMS, cpml_segments, index_at, plan_grid, source_slice
from torchfdtd_b200.run_control import DecayDecision, observation_schedule, validate_graph_steps
from torchfdtd_b200.models import RunControl

GOLDEN = Path(__file__).resolve().parent / 'golden'
C0 = 299792458.0


def test_every_golden_project_round_trips_through_json():
    for path in GOLDEN.glob('sim_*.npz'):
        text = str(np.load(path)['project'])
        p = Project.model_validate_json(text)
        assert json.loads(p.model_dump_json()) == json.loads(text)


def test_reference_demo_projects_load_when_the_reference_tree_is_present(reference_tree):
    root = reference_tree / 'tests' / 'fixtures' / 'projects'
    for name in ('demo_3d.json', 'demo_waveguide.json', 'demo_scatterer.json', 'minimal_defaults.json', 'tiny_result.json'):
        p = Project.load(root / name)
        assert p.region.shape


def test_time_base_of_the_benchmark_configurations():
    r2 = Region(dimension='2d', size=(16, 12, 1), mesh=.05, pml_cells=16)
    assert r2.shape == (320, 240, 1)
    assert math.isclose(r2.time_step, 0.99 / math.sqrt(2) * .05e-6 / C0, rel_tol=1e-15) and math.isclose(r2.time_step, 1.1675e-16, rel_tol=1e-4)
    assert math.isclose(r2.rectangular_courant, .99 / math.sqrt(2))
    r3 = Region(dimension='3d', size=(8, 6, 2), mesh=.05, pml_cells=12)
    assert r3.shape == (160, 120, 40)
    assert math.isclose(r3.time_step, 9.5331e-17, rel_tol=1e-4)
    ra = Region(dimension='3d', size=(8, 8, 3.2), mesh=.04, pml_cells=12)
    assert ra.shape == (200, 200, 80) and math.isclose(ra.time_step, 7.626e-17, rel_tol=1e-3)


def test_cpml_slab_rows_and_grading_follow_the_reference_layout():
    r = Region(dimension='3d', size=(8, 6, 2), mesh=.05, pml_cells=12)
    segs = cpml_segments(r, r.rectangular_courant)
    # 23 rows per (family, axis): E targets 1..n-1 and H targets 0..n-2
    for forward in (False, True):
        for axis in range(3):
            rows = sum(s.hi - s.lo for s in segs if s.forward == forward and s.axis == axis)
            assert rows == 23
    psi = sum(int(np.prod(shape)) for _, shape in plan_grid(Project(region=r)).psi_shapes())
    assert psi == 2_796_800
    e0 = [s for s in segs if not s.forward and s.axis == 0 and s.side == 0][0]
    assert (e0.lo, e0.hi) == (1, 12)
    assert np.all(np.diff(e0.b) > 0)          # decay grows toward the interior
    assert np.all((e0.b > 0) & (e0.b < 1))


def test_baseline_cpml_parameters_map_to_the_reference_faces():
    """sigma_max = 0.8 (m+1)/(eta0 dx), m = 3 -> sigma_scale = 3.2 (L+1)/40 in the reference's normalisation."""
    L = 16
    face = BoundaryFace(sigma_scale=3.2 * (L + 1) / 40, kappa=1, alpha=.05, alpha_polynomial=1)
    r = Region(dimension='2d', size=(16, 12, 1), mesh=.05, pml_cells=L, boundaries=Boundaries(x_min=face))
    seg = [s for s in cpml_segments(r, r.rectangular_courant) if s.forward and s.axis == 0 and s.side == 0][0]
    rho_outer = (L - 1) / (L + 1)    # H target 0 sits one cell in: depth L - 0 - 1, graded over L + 1
    assert math.isclose(seg.sigma[0], face.sigma_scale * 40 * rho_outer**3 / (L + 1))
    assert math.isclose(seg.sigma[0], 3.2 * rho_outer**3, rel_tol=1e-12)


def test_source_and_monitor_indices():
    r = Region(dimension='2d', size=(16, 12, 1), mesh=.05, pml_cells=16)
    assert index_at((-2.5, 0, 0), r) == (110, 120, 0)
    src = Source(kind='plane', center=(-2.5, 0, 0), size=(0, 1.0, 0))
    loc = source_slice(src, r)
    assert (loc[0].start, loc[0].stop) == (110, 111) and loc[1].stop - loc[1].start == 20


@pytest.mark.parametrize('change,match', [
    (dict(backend='cpu'), 'backend="cuda"'),
    (dict(cuda_kernel='torch'), 'cuda_kernel="torch"'),
    (dict(cuda_monitor_kernel='torch'), 'cuda_monitor_kernel="torch"'),
])
def test_selector_refuses_other_paths_before_any_gpu_work(change, match):
    p = Project(region=Region(size=(2, 2, 1), mesh=.1, pml_cells=4, **change))
    with pytest.raises(ValueError, match=match):
        Simulation(p).run()


@pytest.mark.parametrize('build,match', [
    (lambda p: setattr(p.region.boundaries, 'y_min', BoundaryFace(kind='bloch')) or
     setattr(p.region.boundaries, 'y_max', BoundaryFace(kind='bloch')), 'Bloch'),
    (lambda p: setattr(p.region.boundaries, 'x_max', BoundaryFace(kind='pmc')), 'PMC'),
    (lambda p: p.materials.append(Material(name='aniso', model='tensor')) or
     p.structures.append(Structure(material='aniso', size=(.2, .2, 1))), 'tensor'),
    (lambda p: setattr(p.region, 'pml_dispersion', 'absorber') or p.materials.append(Material(name='metal', model='drude')) or
     p.structures.append(Structure(material='metal', size=(.2, .2, 1))), 'absorber'),
    (lambda p: p.sources.append(Source(kind='plane', injection='oneway', normal='x', size=(0, 2, 0), center=(-.5, 0, 0))),
     'periodic transverse'),
    (lambda p: setattr(p.region, 'interface_method', 'subpixel'), 'Subpixel'),
])
def test_unsupported_features_are_refused_by_name(build, match):
    p = Project(region=Region(size=(3, 3, 1), mesh=.1, pml_cells=4, material_sampling='yee'))
    try:
        build(p)
    except ValueError:
        pytest.skip('the scene model itself refuses this combination')
    with pytest.raises(ValueError, match=match):
        plan_grid(p)


def test_2d_polarization_follows_the_sources():
    base = dict(region=Region(size=(2, 2, 1), mesh=.1, pml_cells=4))
    assert plan_grid(Project(**base, sources=[Source(component='Ez')])).polarization == 'TM'
    assert plan_grid(Project(**base, sources=[Source(component='Hz')])).polarization == 'TE'
    both = plan_grid(Project(**base, sources=[Source(component='Ex', theta=60, phi=30)]))
    assert both.polarization == 'both'


def test_plane_plan_and_interpolation_corners():
    p = Project(region=Region(dimension='3d', size=(2, 2, 2), mesh=.1, pml_cells=4),
                monitors=[FieldMonitor(center=(.3, 0, 0), size=(0, .8, .6),
                                       spectrum=SpectrumSettings(sampling='frequency', frequency_points=3, apodization='none'))])
    plane = plan_grid(p).planes[0]
    assert plane.corner_cells.shape == (6, 8, 8 * 6)
    np.testing.assert_allclose(plane.corner_weights.astype(np.float64).sum(axis=1), 1, rtol=1e-6)
    assert plane.windows[0].dtype == np.float32 and len(plane.frequency) == 3


def test_observation_schedule_and_graph_width():
    assert list(observation_schedule(10, 4, {5})) == [(4, 4), (5, 1), (9, 4), (10, 1)]
    with pytest.raises(ValueError):
        validate_graph_steps(65)
    with pytest.raises(ValueError):
        validate_graph_steps(2, enabled=False)


def test_decay_decision_raises_on_divergence_and_stops_on_decay():
    control = RunControl(auto_shutoff=True, min_steps=10, consecutive_checks=2, decay_threshold=1e-3)
    d = DecayDecision(control, source_end_s=0, dt=1)
    assert not d.update(10, 1.0, 1.0)
    assert not d.update(20, 1e-4, 1.0)
    assert d.update(30, 1e-5, 1.0)
    with pytest.raises(FloatingPointError):
        DecayDecision(control, 0, 1).update(10, float('nan'), 1.0)
    grow = DecayDecision(RunControl(min_steps=10, growth_limit=10), 0, 1)
    grow.update(10, 1.0, 1.0)
    with pytest.raises(FloatingPointError, match='grew'):
        grow.update(20, 100.0, 1.0)


def test_curl_term_table_is_the_reference_order():
    assert CURL_TERMS == ((0, 2, 1, -1), (0, 1, 2, 1), (1, 2, 0, 1), (1, 0, 2, -1), (2, 1, 0, -1), (2, 0, 1, 1))

"""Parity of the fused CUDA path (through the C ABI) with the reference's CPU path.

Golden vectors in tests/golden were written by the reference's own CPU code
(tests/golden/make_golden.py); the reference pins its fused CUDA kernels to that
code bitwise in FP32 (reference tests/test_cuda_kernels.py:149-170) and to 3e-6
in general (:72-111). Bar here: fields, CPML memories and point traces bitwise
equal in FP32 and FP64 (the kernels keep the reference operation order and are
built with --fmad=false); DFT planes, whose accumulators are FP64 here and
complex64 in the reference, within relative L2 1e-5 (FP32 fields) and 1e-12
(FP64 fields).
"""
import json

import numpy as np
import pytest

from oracle.yee_oracle import YeeOracle
from torchfdtd_b200 import Project, Region
from torchfdtd_b200.plan import plan_grid

pytestmark = pytest.mark.gpu

KERNELS = ['gather', 'march', 'tile2d']
PLANE_TOL = {'float32': 1e-5, 'float64': 1e-12}


def rel_l2(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))


def native(plan, kernel):
    from torchfdtd_b200.native import NativeGrid
    return NativeGrid(plan, kernel=kernel)


def skip_unmarchable(plan_or_project, kernel):
    """The marching kernel tiles 3D grids (periodic x/y seams included), the 2D tile kernel 2D TMz grids without
    periodic x/y faces; other scenes run the gather kernel."""
    region = getattr(plan_or_project, 'region', None) or plan_or_project.project.region
    project = plan_or_project if hasattr(plan_or_project, 'region') else plan_or_project.project
    if kernel != 'gather' and project is not None and (
            any(s.enabled and s.kind == 'tfsf' for s in project.sources)
            or any(m.oscillators for m in project.materials if m.name in {s.material for s in project.structures if s.enabled})):
        pytest.skip('TFSF and dispersive scenes run the split gather kernels')
    periodic_xy = any(region.boundaries.pair(a)[0].kind == 'periodic' for a in (0, 1))
    if kernel == 'march' and region.dimension == '2d':
        pytest.skip('scene runs the gather kernel')
    if kernel == 'tile2d':
        plan = plan_or_project if hasattr(plan_or_project, 'psi_shapes') else plan_grid(plan_or_project)
        if region.dimension != '2d' or periodic_xy or plan.polarization != 'TM':
            pytest.skip('scene is not a 2D TMz grid with PML/PEC x/y faces')


def state_files(golden):
    return sorted(golden.glob('state_*.npz'))


@pytest.mark.parametrize('kernel', KERNELS)
@pytest.mark.parametrize('name', ['pml2d', 'pml3d', 'periodic', 'pec', 'graded', 'explicit'])
@pytest.mark.parametrize('precision', ['float32', 'float64'])
def test_random_state_and_every_cpml_memory_match_reference_bitwise(golden, kernel, name, precision):
    d = np.load(golden / f'state_{name}_{precision}.npz')
    region = Region.model_validate_json(str(d['region']))
    plan = plan_grid(Project(region=region), polarization='both')
    skip_unmarchable(plan, kernel)
    plan.inv_eps = d['init_inverse_permittivity']
    g = native(plan, kernel)
    g.set_fields(d['init_E'], d['init_H'])
    g.step(int(d['steps']))
    E, H = g.get_fields()
    np.testing.assert_array_equal(E, d['E'])
    np.testing.assert_array_equal(H, d['H'])
    psi = g.get_psi()
    expected = [d[f'psi_{i}'] for i in range(len([k for k in d.files if k.startswith('psi_')]))]
    assert len(psi) == len(expected)
    for got, want in zip(psi, expected):
        np.testing.assert_array_equal(got, want)
    assert g.counter() == int(d['steps'])
    assert g.device_status() == 0


SIMS = ['tmz', 'strip3d', 'strip3d_f64', 'yee_periodic', 'te2d', 'both2d', 'tiny', 'graded3d', 'graded2d', 'steps3d', 'explicit3d',
        'oneway3d', 'oneway2d', 'tfsf3d', 'tfsf2d', 'drude3d', 'frozen2d']


@pytest.mark.parametrize('kernel', KERNELS)
@pytest.mark.parametrize('name', SIMS)
def test_simulation_run_matches_reference_cpu_result(golden, kernel, name):
    from torchfdtd_b200 import Simulation
    d = np.load(golden / f'sim_{name}.npz')
    project = Project.model_validate_json(str(d['project']))
    project.region.backend = 'cuda'
    project.region.cuda_kernel = 'fused'
    skip_unmarchable(project, kernel)
    result = Simulation(project).run(kernel=kernel)
    assert result.summary['cuda_kernel'] == 'fused' and result.summary['kernel'] == kernel
    np.testing.assert_array_equal(result.electric, d['E'])
    np.testing.assert_array_equal(result.magnetic, d['H'])
    np.testing.assert_array_equal(result.signals, d['signals'])
    np.testing.assert_array_equal(result.frame_steps, d['frame_steps'])
    np.testing.assert_array_equal(result.frames, d['frames'])
    tol = PLANE_TOL[project.region.precision]
    for k, plane in enumerate(result.frequency_fields):
        assert rel_l2(plane['fields'], d[f'plane{k}_fields']) <= max(tol, 1e-12)
        if f'plane{k}_flux' in d.files:
            assert rel_l2(plane['flux'], d[f'plane{k}_flux']) <= 2 * max(tol, 1e-12)
    for k, spec in enumerate(result.spectra):
        np.testing.assert_allclose(spec['value'], d[f'spectrum{k}_value'], rtol=1e-12, atol=0)


@pytest.mark.parametrize('kernel', KERNELS)
def test_planes_match_oracle_with_float64_accumulators(golden, kernel):
    """FP64 accumulation stated against the same accumulation on the CPU."""
    from torchfdtd_b200 import Simulation
    d = np.load(golden / 'sim_strip3d.npz')
    project = Project.model_validate_json(str(d['project']))
    project.region.backend = 'cuda'
    plan = plan_grid(project)
    skip_unmarchable(plan, kernel)
    oracle = YeeOracle(plan, dft_float64=True).run()
    g = native(plan, kernel)
    g.step(plan.steps)
    for k in range(len(plan.planes)):
        assert rel_l2(g.get_plane(k), oracle.planes[k]['value']) <= 1e-12


def random_project(dimension, precision, sampling='cell', faces=None, steps=20):
    from torchfdtd_b200.models import BoundaryFace, Source, Structure
    region = Region(dimension=dimension, size=(3.3, 2.5, 2.05 if dimension == '3d' else 1), mesh=.05, pml_cells=7,
                    steps=steps, precision=precision, material_sampling=sampling, backend='cuda')
    region.boundaries.x_min = BoundaryFace(layers=9, kappa=2, alpha=.04, alpha_polynomial=1)
    for name, face in (faces or {}).items():
        setattr(region.boundaries, name, face)
    return Project(region=region, structures=[Structure(kind='sphere', radius=.5, material='Si (constant n)')],
                   sources=[Source(center=(-.6, .1, 0), component='Ez', pulse_cycles=1, wavelength=1.0),
                            Source(center=(.3, -.2, 0), component='Hy', pulse_cycles=1, wavelength=1.0, amplitude=.3)])


@pytest.mark.parametrize('kernel', KERNELS)
@pytest.mark.parametrize('dimension', ['2d', '3d'])
@pytest.mark.parametrize('precision', ['float32', 'float64'])
def test_odd_shapes_and_random_state_match_oracle(kernel, dimension, precision):
    """Ragged shapes (x not a multiple of the tile), kappa>1 CPML, sources on E and H, random start."""
    project = random_project(dimension, precision)
    plan = plan_grid(project, polarization='both')
    skip_unmarchable(plan, kernel)
    rng = np.random.default_rng(7)
    oracle = YeeOracle(plan)
    oracle.E[:] = rng.normal(size=oracle.E.shape).astype(plan.dtype) * .01
    oracle.H[:] = rng.normal(size=oracle.H.shape).astype(plan.dtype) * .01
    g = native(plan, kernel)
    g.set_fields(oracle.E, oracle.H)
    oracle.run()
    g.step(plan.steps)
    E, H = g.get_fields()
    np.testing.assert_array_equal(E, oracle.E)
    np.testing.assert_array_equal(H, oracle.H)
    for got, want in zip(g.get_psi(), oracle.memory_states):
        np.testing.assert_array_equal(got, want)


@pytest.mark.parametrize('kernel', KERNELS)
@pytest.mark.parametrize('zfaces', ['periodic', 'pec'])
def test_z_faces_periodic_and_pec_match_oracle(kernel, zfaces):
    """The marching kernel's chunk seams: periodic z wraps the halo plane, PEC z adds the H ghost."""
    from torchfdtd_b200.models import BoundaryFace
    faces = {'z_min': BoundaryFace(kind=zfaces), 'z_max': BoundaryFace(kind=zfaces),
             'y_max': BoundaryFace(kind='pec')}
    project = random_project('3d', 'float32', faces=faces, steps=16)
    plan = plan_grid(project)
    skip_unmarchable(plan, kernel)
    rng = np.random.default_rng(11)
    oracle = YeeOracle(plan)
    oracle.E[:] = rng.normal(size=oracle.E.shape).astype(plan.dtype) * .01
    oracle.H[:] = rng.normal(size=oracle.H.shape).astype(plan.dtype) * .01
    g = native(plan, kernel)
    g.set_fields(oracle.E, oracle.H)
    oracle.run()
    g.step(plan.steps)
    E, H = g.get_fields()
    np.testing.assert_array_equal(E, oracle.E)
    np.testing.assert_array_equal(H, oracle.H)
    for got, want in zip(g.get_psi(), oracle.memory_states):
        np.testing.assert_array_equal(got, want)


@pytest.mark.parametrize('kernel,variant', [(k, 0) for k in KERNELS] + [('march', 114), ('march', 314)])
@pytest.mark.parametrize('precision', ['float32', 'float64'])
def test_interior_and_boundary_tiles_match_oracle(kernel, variant, precision):
    """A grid large enough for interior tiles and boundary strips, with sources in the interior and a DFT
    plane. Variant 114 splits the march: the pure fast kernel over the interior tiles' planes outside the
    z slabs, the general kernel over their z-slab planes and over the boundary strips (concurrent launches);
    variant 314 runs both bodies in one launch, chosen per CTA."""
    from torchfdtd_b200.models import FieldMonitor, Source, SpectrumSettings, Structure
    region = Region(dimension='3d', size=(5.0, 3.0, 1.5), mesh=.05, pml_cells=6, steps=24, precision=precision, backend='cuda')
    project = Project(region=region, structures=[Structure(kind='sphere', radius=.6, material='Si (constant n)')],
                      sources=[Source(center=(-.4, .1, 0), component='Ez', pulse_cycles=1, wavelength=1.0),
                               Source(center=(.6, -.2, .1), component='Hx', pulse_cycles=1, wavelength=1.0, amplitude=.2)],
                      monitors=[FieldMonitor(center=(.9, 0, 0), size=(0, 1.2, .6),
                                             spectrum=SpectrumSettings(sampling='frequency', frequency_points=2, apodization='none'))])
    plan = plan_grid(project)
    skip_unmarchable(plan, kernel)
    rng = np.random.default_rng(5)
    oracle = YeeOracle(plan)
    oracle.E[:] = rng.normal(size=oracle.E.shape).astype(plan.dtype) * .01
    oracle.H[:] = rng.normal(size=oracle.H.shape).astype(plan.dtype) * .01
    if variant and precision == 'float64':
        variant = variant // 100 * 100 + 22       # FP64 runs D / MINB = 22
    from torchfdtd_b200.native import NativeGrid
    g = NativeGrid(plan, kernel=kernel, variant=variant)
    g.set_fields(oracle.E, oracle.H)
    oracle.run()
    g.step(plan.steps)
    E, H = g.get_fields()
    np.testing.assert_array_equal(E, oracle.E)
    np.testing.assert_array_equal(H, oracle.H)
    for got, want in zip(g.get_psi(), oracle.memory_states):
        np.testing.assert_array_equal(got, want)


@pytest.mark.parametrize('variant', [0, 314])
@pytest.mark.parametrize('zmax', ['pml', 'pec'])
@pytest.mark.parametrize('precision', ['float32', 'float64'])
def test_interior_block_on_z_slab_and_z_face_planes_matches_oracle(variant, zmax, precision):
    """The mixed launch's z-pure body: interior tiles on the chunks outside the pure z segment, with rows that
    meet only a z slab, the z-face planes (PML or PEC above) and, with PEC above, sources on E and H in the
    top plane."""
    from torchfdtd_b200.models import BoundaryFace, Source, Structure
    region = Region(dimension='3d', size=(5.0, 3.0, 1.5), mesh=.05, pml_cells=6, steps=20, precision=precision, backend='cuda')
    if zmax == 'pec':
        region.boundaries.z_max = BoundaryFace(kind='pec')
    zs = .72 if zmax == 'pec' else .3               # with PEC above: the top plane, in the last z segment
    project = Project(region=region, structures=[Structure(kind='sphere', radius=.6, material='Si (constant n)')],
                      sources=[Source(center=(-.4, .1, zs), component='Ez', pulse_cycles=1, wavelength=1.0),
                               Source(center=(.6, -.2, zs), component='Hx', pulse_cycles=1, wavelength=1.0, amplitude=.2)])
    plan = plan_grid(project)
    rng = np.random.default_rng(9)
    oracle = YeeOracle(plan)
    oracle.E[:] = rng.normal(size=oracle.E.shape).astype(plan.dtype) * .01
    oracle.H[:] = rng.normal(size=oracle.H.shape).astype(plan.dtype) * .01
    if variant and precision == 'float64':
        variant = variant // 100 * 100 + 22
    from torchfdtd_b200.native import NativeGrid
    g = NativeGrid(plan, kernel='march', variant=variant)
    g.set_fields(oracle.E, oracle.H)
    oracle.run()
    g.step(plan.steps)
    E, H = g.get_fields()
    np.testing.assert_array_equal(E, oracle.E)
    np.testing.assert_array_equal(H, oracle.H)
    for got, want in zip(g.get_psi(), oracle.memory_states):
        np.testing.assert_array_equal(got, want)


@pytest.mark.parametrize('zfaces', ['periodic', 'pec'])
def test_interior_block_with_periodic_or_pec_z_faces_matches_oracle(zfaces):
    """The mixed launch on a grid with interior tiles and no z slab: the first and last planes (periodic: with
    the wrapped neighbour plane; PEC: the H ghost above, no previous plane below) run the z-pure body, with
    sources on E and H in the first plane."""
    from torchfdtd_b200.models import BoundaryFace, Source, Structure
    region = Region(dimension='3d', size=(5.0, 3.0, 1.5), mesh=.05, pml_cells=6, steps=18, precision='float32', backend='cuda')
    region.boundaries.z_min = BoundaryFace(kind=zfaces)
    region.boundaries.z_max = BoundaryFace(kind=zfaces)
    project = Project(region=region, structures=[Structure(kind='sphere', radius=.6, material='Si (constant n)')],
                      sources=[Source(center=(-.4, .1, -.73), component='Ez', pulse_cycles=1, wavelength=1.0),
                               Source(center=(.6, -.2, -.73), component='Hy', pulse_cycles=1, wavelength=1.0, amplitude=.2)])
    plan = plan_grid(project)
    assert not [s for s in plan.segments if s.axis == 2]
    rng = np.random.default_rng(13)
    oracle = YeeOracle(plan)
    oracle.E[:] = rng.normal(size=oracle.E.shape).astype(plan.dtype) * .01
    oracle.H[:] = rng.normal(size=oracle.H.shape).astype(plan.dtype) * .01
    g = native(plan, 'march')
    g.set_fields(oracle.E, oracle.H)
    oracle.run()
    g.step(plan.steps)
    E, H = g.get_fields()
    np.testing.assert_array_equal(E, oracle.E)
    np.testing.assert_array_equal(H, oracle.H)
    for got, want in zip(g.get_psi(), oracle.memory_states):
        np.testing.assert_array_equal(got, want)


def seam_project(size, precision, sampling, steps=14):
    """Periodic x/y with z-CPML (the scene the reference's one-pass marching kernel admits), ragged tile
    counts, and sources on the seam cells (first column / row), which halo lanes recompute."""
    from torchfdtd_b200.models import BoundaryFace, Source, Structure
    region = Region(dimension='3d', size=size, mesh=.05, pml_cells=5, steps=steps, precision=precision,
                    material_sampling=sampling, backend='cuda')
    for name in ('x_min', 'x_max', 'y_min', 'y_max'):
        setattr(region.boundaries, name, BoundaryFace(kind='periodic'))
    hx, hy = size[0] / 2, size[1] / 2
    return Project(region=region, structures=[Structure(kind='sphere', radius=.3, material='Si (constant n)')],
                   sources=[Source(center=(-hx + .025, .05, 0), component='Ey', pulse_cycles=1, wavelength=1.0),
                            Source(center=(.1, -hy + .025, .05), component='Ex', pulse_cycles=1, wavelength=1.0),
                            Source(center=(-hx + .025, -hy + .025, -.05), component='Ez', pulse_cycles=1, wavelength=1.0),
                            Source(center=(.2, .1, 0), component='Hz', pulse_cycles=1, wavelength=1.0, amplitude=.2)])


@pytest.mark.parametrize('kernel', ['gather', 'march'])
@pytest.mark.parametrize('size,precision,sampling', [((3.3, 2.5, 1.2), 'float32', 'cell'), ((3.3, 2.5, 1.2), 'float64', 'cell'),
                                                     ((1.0, .8, 1.0), 'float32', 'yee'), ((1.6, .8, .9), 'float64', 'yee')])
def test_periodic_xy_seams_match_oracle(kernel, size, precision, sampling):
    """Seam tiles of the marching kernel patch the wrapped neighbours into their stages; narrow grids (one or
    two tiles per axis) put both seams in one tile."""
    project = seam_project(size, precision, sampling)
    plan = plan_grid(project)
    rng = np.random.default_rng(13)
    oracle = YeeOracle(plan)
    oracle.E[:] = rng.normal(size=oracle.E.shape).astype(plan.dtype) * .01
    oracle.H[:] = rng.normal(size=oracle.H.shape).astype(plan.dtype) * .01
    g = native(plan, kernel)
    assert g.kernel == kernel
    g.set_fields(oracle.E, oracle.H)
    oracle.run()
    g.step(plan.steps)
    E, H = g.get_fields()
    np.testing.assert_array_equal(E, oracle.E)
    np.testing.assert_array_equal(H, oracle.H)
    for got, want in zip(g.get_psi(), oracle.memory_states):
        np.testing.assert_array_equal(got, want)
    assert g.device_status() == 0


@pytest.mark.parametrize('kernel', KERNELS)
def test_graph_replay_equals_eager_steps(kernel):
    import torch
    project = random_project('3d', 'float32', steps=30)
    plan = plan_grid(project)
    skip_unmarchable(plan, kernel)
    a, b = native(plan, kernel), native(plan, kernel)
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


def test_diagnostics_slice_and_psi_round_trip():
    project = random_project('3d', 'float64', steps=25)
    plan = plan_grid(project)
    g = native(plan, 'gather')
    g.step(25)
    E, H = g.get_fields()
    inv = plan.inv_eps[..., None]
    energy, peak, finite = g.diagnose()
    assert finite
    assert peak == max(np.abs(E).max(), np.abs(H).max())
    np.testing.assert_allclose(energy, (E * E / inv).sum() + (H * H).sum(), rtol=1e-12)
    np.testing.assert_array_equal(g.get_slice('Ey', 2, 7), E[:, :, 7, 1])
    np.testing.assert_array_equal(g.get_slice('Hz', 0, 3), H[3, :, :, 2])
    psi = g.get_psi()
    g.set_psi([p * 0 + 1 for p in psi])
    assert all((p == 1).all() for p in g.get_psi())


def test_invalid_descriptor_is_refused_with_a_named_error():
    import ctypes
    from torchfdtd_b200 import native as nat
    plan = plan_grid(random_project('3d', 'float32'))
    g = native(plan, 'gather')
    desc = g.desc
    desc.precision = 3
    size = ctypes.c_size_t()
    with pytest.raises(ValueError, match='precision'):
        nat.check(nat.library().tfd_plan_bytes(ctypes.byref(desc), ctypes.byref(size)))


@pytest.mark.parametrize('variant', [14, 23, 32, 22, 114, 123, 214, 314, 4014, 7023])
def test_march_launch_variants_match_oracle(variant):
    """Every launch shape the autotuner may pick (prefetch depth, CTAs per SM, interior split, z-chunk)."""
    from torchfdtd_b200.native import NativeGrid
    project = random_project('3d', 'float32', steps=14)
    plan = plan_grid(project)
    rng = np.random.default_rng(variant)
    oracle = YeeOracle(plan)
    oracle.E[:] = rng.normal(size=oracle.E.shape).astype(plan.dtype) * .01
    oracle.H[:] = rng.normal(size=oracle.H.shape).astype(plan.dtype) * .01
    g = NativeGrid(plan, kernel='march', variant=variant)
    g.set_fields(oracle.E, oracle.H)
    oracle.run()
    g.step(plan.steps)
    E, H = g.get_fields()
    np.testing.assert_array_equal(E, oracle.E)
    np.testing.assert_array_equal(H, oracle.H)
    assert g.device_status() == 0


def test_invalid_launch_variant_is_refused():
    from torchfdtd_b200.native import NativeGrid
    plan = plan_grid(random_project('3d', 'float32'))
    with pytest.raises(ValueError, match='launch variant'):
        NativeGrid(plan, kernel='march', variant=15)
    plan64 = plan_grid(random_project('3d', 'float64'))
    with pytest.raises(ValueError, match='launch variant'):
        NativeGrid(plan64, kernel='march', variant=14)


def test_select_launch_measures_candidates_and_simulation_uses_the_winner():
    from torchfdtd_b200 import Simulation
    from torchfdtd_b200.tuning import select_launch
    project = random_project('3d', 'float32', steps=40)
    plan = plan_grid(project)
    tuning = select_launch(plan, candidates=[14, 23, 4014], steps=4, repeats=3)
    assert tuning.kind == 'grid' and tuning.choice in (14, 23, 4014)
    assert all(r['status'] == 'completed' and len(r['samples_ms_per_step']) == 3 for r in tuning.candidates)
    assert select_launch(plan, candidates=[14, 23, 4014], steps=4, repeats=3).cached
    tuned = Simulation(project).run(launch='auto')
    plain = Simulation(project).run()
    np.testing.assert_array_equal(tuned.electric, plain.electric)
    assert tuned.summary['launch_tuning']['kind'] == 'grid'


@pytest.mark.parametrize('precision', ['float32', 'float64'])
def test_persistent_2d_launch_equals_per_step_launches(golden, monkeypatch, precision):
    """Small 2D TMz grids step in one persistent cooperative launch (grid barrier between steps, observations
    of step n-1 taken during step n). Against the per-step launches: fields, CPML memories, traces, DFT planes
    and the step counter bitwise equal, for uneven step counts per call and a call that runs past the end."""
    from torchfdtd_b200.native import NativeGrid
    d = np.load(golden / 'sim_tmz.npz')
    project = Project.model_validate_json(str(d['project']))
    project.region.precision = precision
    plan = plan_grid(project)
    grids = {}
    for mode in ('0', '1'):
        monkeypatch.setenv('TFD_PERSIST2D', mode)
        grids[mode] = NativeGrid(plan, kernel='tile2d')
    for count in (1, 7, 64, 3, plan.steps):
        for g in grids.values():
            g.step(count)
    a, b = grids['0'], grids['1']
    assert a.counter() == b.counter() == plan.steps
    for x, y in zip(a.get_fields(), b.get_fields()):
        np.testing.assert_array_equal(x, y)
    for x, y in zip(a.get_psi(), b.get_psi()):
        np.testing.assert_array_equal(x, y)
    np.testing.assert_array_equal(a.get_traces(), b.get_traces())
    for k in range(len(plan.planes)):
        np.testing.assert_array_equal(a.get_plane(k), b.get_plane(k))
    assert a.device_status() == b.device_status() == 0


@pytest.mark.parametrize('kernel', ['gather', 'march'])
def test_steps_past_the_last_step_are_no_ops(kernel):
    """Stepping a plan past its configured step count changes nothing: fields, CPML memories (the H family's
    are updated in place), traces and the counter stay those of the last step."""
    project = random_project('3d', 'float32', steps=14)
    plan = plan_grid(project)
    a, b = native(plan, kernel), native(plan, kernel)
    a.step(14)
    b.step(10)
    b.step(9)
    b.step(2)
    assert a.counter() == b.counter() == 14
    for x, y in zip(a.get_fields(), b.get_fields()):
        np.testing.assert_array_equal(x, y)
    for x, y in zip(a.get_psi(), b.get_psi()):
        np.testing.assert_array_equal(x, y)
    np.testing.assert_array_equal(a.get_traces(), b.get_traces())


@pytest.mark.parametrize('precision', ['float32', 'float64'])
def test_device_permittivity_inversion_and_field_check(precision):
    """tfd_set_permittivity loads the same material as tfd_set_material(1 / eps) (bitwise equal fields after
    stepping), refuses non-finite or sub-unity values, and tfd_field_check reports the host's peak |E|."""
    project = random_project('3d', precision, sampling='yee')
    plan = plan_grid(project)
    eps = np.asarray(plan.epsilon, plan.dtype) * np.asarray(1 + .3 * np.random.default_rng(3).random(plan.epsilon.shape), plan.dtype)
    plan.epsilon, plan.inv_eps = eps, (1 / eps).astype(plan.dtype)
    a = native(plan, 'march')
    from torchfdtd_b200.native import NativeGrid
    b = NativeGrid(plan, kernel='march', permittivity=eps)
    a.step(plan.steps)
    b.step(plan.steps)
    for x, y in zip(a.get_fields(), b.get_fields()):
        np.testing.assert_array_equal(x, y)
    E, H = b.get_fields()
    peak, finite = b.field_check()
    assert finite and peak == float(np.max(np.abs(E)))
    for bad in (np.nan, np.inf, .5):
        wrong = eps.copy()
        wrong[3, 4, 5, 1] = bad
        with pytest.raises(ValueError, match='epsilon must be finite and at least 1'):
            b.set_permittivity(wrong)


def test_simulation_device_material_and_checks_equal_host_path(monkeypatch):
    """Simulation(project, epsilon).run() through the large-grid path (device permittivity inversion, device
    field check, result arrays prepared on a helper thread, staged download), with CUDA graphs, returns the
    host path's fields, traces and peak."""
    import torchfdtd_b200.simulation as sim
    project = random_project('3d', 'float32', steps=16)
    eps = np.asarray(plan_grid(project).epsilon, np.float32)
    want = sim.Simulation(project, epsilon=eps).run(cuda_graph=False)
    monkeypatch.setattr(sim, 'LARGE_FIELD_BYTES', 0)
    got = sim.Simulation(project, epsilon=eps).run(cuda_graph=True, cuda_graph_steps=4)
    np.testing.assert_array_equal(got.electric, want.electric)
    np.testing.assert_array_equal(got.magnetic, want.magnetic)
    np.testing.assert_array_equal(got.signals, want.signals)
    assert got.summary['field_peak'] == want.summary['field_peak']


@pytest.mark.parametrize('precision', ['float32', 'float64'])
@pytest.mark.parametrize('mesh', ['uniform', 'graded'])
def test_on_chip_cluster_2d_path_equals_the_strip_launches(monkeypatch, precision, mesh):
    """Small 2D TMz plans without planes run every step of a call in one thread-block cluster (fields in
    distributed shared memory): bitwise equal to the persistent strip launch and to the per-step launches, with
    E and H sources, a PEC face, CPML and (graded) metric factors; traces included."""
    from torchfdtd_b200 import Project, Region, Source, Monitor, Structure
    from torchfdtd_b200.models import BoundaryFace
    extra = dict(mesh_type='graded', mesh_max=.12, mesh_ppw=6, material_sampling='yee') if mesh == 'graded' else {}
    region = Region(dimension='2d', size=(4.8, 3.2, 1), mesh=.04, pml_cells=10, steps=180, precision=precision, backend='cuda', **extra)
    region.boundaries.y_max = BoundaryFace(kind='pec')
    project = Project(region=region, structures=[Structure(kind='circle', center=(.4, .2, 0), radius=.3, material='Si (constant n)')],
                      sources=[Source(center=(-.8, 0, 0), component='Ez', pulse_cycles=2, wavelength=1.6),
                               Source(center=(-.3, .3, 0), component='Hx', pulse_cycles=2, wavelength=1.6, amplitude=.4)],
                      monitors=[Monitor(center=(.9, .1, 0), component='Ez'), Monitor(center=(.2, -.4, 0), component='Hy')])
    out = {}
    for mode, env in (('cluster', {}), ('persistent', {'TFD_CLUSTER2D': '0'}), ('per_step', {'TFD_CLUSTER2D': '0', 'TFD_PERSIST2D': '0'})):
        for k in ('TFD_CLUSTER2D', 'TFD_PERSIST2D'):
            monkeypatch.delenv(k, raising=False)
        for k, v in env.items():
            monkeypatch.setenv(k, v)
        plan = plan_grid(project)
        g = native(plan, 'tile2d')
        g.step(70)
        g.step(110)
        out[mode] = (*g.get_fields(), g.get_traces(), g.get_psi(), g.counter())
        g.close()
    oracle = YeeOracle(plan_grid(project)).run()
    for mode in ('persistent', 'per_step'):
        for a, b in zip(out['cluster'][:3], out[mode][:3]):
            np.testing.assert_array_equal(a, b)
        for a, b in zip(out['cluster'][3], out[mode][3]):
            np.testing.assert_array_equal(a, b)
    np.testing.assert_array_equal(out['cluster'][0], oracle.E)
    np.testing.assert_array_equal(out['cluster'][1], oracle.H)
    np.testing.assert_array_equal(out['cluster'][2], oracle.traces)
    assert out['cluster'][4] == 180 and np.abs(out['cluster'][0]).max() > 0


"""Parity at the benchmark configurations' own sizes and step counts, through the public API.

The other parity tests pin the kernels on small scenes against golden vectors the reference
wrote. Here the workloads are those of bench.py at full size, checked against the C oracle
(oracle/yee_cpu.c, the reference's CPU update restated operation for operation and itself
pinned bitwise to the reference's goldens):

* config 0: 2D TMz 320 x 240, CPML 16, 2000 steps: Ez, Hx, Hy, the Ez trace and its DFT at 1.55 um;
* config 1: 3D 160 x 120 x 40 Si strip, CPML 12, 1000 steps, with the 96 x 16-point x-normal DFT plane;
* the 512 x 512 x 256 roofline scene for 8 steps through the default mixed march launch (pure, z-pure
  and general bodies over 17 x 35 x 23 CTAs and three z segments), every CPML memory included;
* 8 grids of the seeded 64-grid batch for its 3000 steps in one batched run.

Bars: fields, CPML memories and traces bitwise; DFT planes within 1e-12 of the oracle's FP64
accumulation. The FP32 run is also stated against an FP64 run of the same kernels
(``test_float32_against_float64_runs_of_the_same_kernels``).
"""
import numpy as np
import pytest

from bench import batch_workload, workload
from oracle.cpu import CpuOracle
from torchfdtd_b200.plan import plan_grid

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    a, b = np.asarray(a, dtype=np.complex128 if np.iscomplexobj(a) else np.float64), np.asarray(b)
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))


def config_project(name, steps, precision='float32'):
    project, eps, _ = workload(name, steps)
    project.region.precision = precision
    return project, eps


@pytest.mark.parametrize('precision', ['float32', 'float64'])
def test_config0_tmz_320x240_2000_steps(precision):
    from torchfdtd_b200 import Simulation
    project, _ = config_project('tmz2d', 2000, precision)
    result = Simulation(project).run()
    assert result.summary['steps'] == 2000 and tuple(result.summary['shape']) == (320, 240, 1)
    oracle = CpuOracle(plan_grid(project)).run()
    np.testing.assert_array_equal(result.electric, oracle.E)
    np.testing.assert_array_equal(result.magnetic, oracle.H)
    np.testing.assert_array_equal(result.signals, oracle.traces)
    from torchfdtd_b200.spectra import point_spectrum
    monitor = result.point_monitors[0]
    want = point_spectrum(result.times, oracle.traces[:, 0], monitor.spectrum)['value']
    np.testing.assert_array_equal(result.spectra[0]['value'], want)


@pytest.mark.parametrize('precision', ['float32', 'float64'])
def test_config1_strip_160x120x40_1000_steps_with_dft_plane(precision):
    from torchfdtd_b200 import Simulation
    project, _ = config_project('strip', 1000, precision)
    result = Simulation(project).run()
    assert tuple(result.summary['shape']) == (160, 120, 40) and result.summary['steps'] == 1000
    plan = plan_grid(project)
    assert plan.planes[0].corner_cells.shape[2] == 96 * 16
    oracle = CpuOracle(plan)
    planes = oracle.run_with_planes(dft_float64=True)
    np.testing.assert_array_equal(result.electric, oracle.E)
    np.testing.assert_array_equal(result.magnetic, oracle.H)
    plane = result.field_monitor('plane')
    order = [plane['accumulated_components'].index(c) for c in plane['components']]
    assert rel_l2(plane['fields'], planes[0][..., order]) <= 1e-12


def test_roofline_512x512x256_mixed_launch_8_steps_every_memory():
    from torchfdtd_b200.native import NativeGrid
    project, eps = config_project('roofline', 10)      # a Region runs at least 10 steps; 8 of them here
    plan = plan_grid(project)
    plan.epsilon, plan.inv_eps = eps, (1 / eps).astype(plan.dtype)
    grid = NativeGrid(plan)
    assert grid.kernel == 'march'
    grid.step(8)
    E, H = grid.get_fields()
    psi = grid.get_psi()
    traces = grid.get_traces()
    status = grid.device_status()
    grid.close()
    assert status == 0
    oracle = CpuOracle(plan).run(8)
    np.testing.assert_array_equal(E, oracle.E)
    np.testing.assert_array_equal(H, oracle.H)
    assert len(psi) == len(oracle.memory_states)
    for got, want in zip(psi, oracle.memory_states):
        np.testing.assert_array_equal(got, want)
    np.testing.assert_array_equal(traces[:8], oracle.traces[:8])
    assert np.abs(E).max() > 0


def test_batch64_subset_of_8_grids_3000_steps():
    from torchfdtd_b200.batch import run_tensor_batch
    projects, eps, _ = batch_workload(3000)
    picks = [0, 9, 18, 27, 36, 45, 54, 63]
    projects, eps = [projects[i] for i in picks], [eps[i] for i in picks]
    report = run_tensor_batch(projects, epsilon=eps, cuda_graph=True, cuda_graph_steps=16)
    report.raise_for_errors()
    assert len(report.items) == len(picks)
    for item, project, e in zip(report.items, projects, eps):
        plan = plan_grid(project)
        plan.epsilon, plan.inv_eps = e, (1 / e).astype(plan.dtype)
        oracle = CpuOracle(plan).run()
        np.testing.assert_array_equal(item.result.electric, oracle.E)
        np.testing.assert_array_equal(item.result.magnetic, oracle.H)
        np.testing.assert_array_equal(item.result.signals, oracle.traces)


def test_float32_against_float64_runs_of_the_same_kernels():
    """FP32 fields and spectra against an FP64 run of the same kernels on configs 0 and 1. After 2000 steps
    config 0's pulse has left the grid (the field norm is ~4e-5 of its peak), so its fields compare the
    rounding residue; its trace and spectrum, and config 1's fields and DFT plane, compare live signals."""
    from torchfdtd_b200 import Simulation
    out = {}
    for name, steps in (('tmz2d', 2000), ('strip', 1000)):
        runs = {p: Simulation(config_project(name, steps, p)[0]).run() for p in ('float32', 'float64')}
        a, b = runs['float32'], runs['float64']
        rec = {f'E{"xyz"[c]}': rel_l2(a.electric[..., c], b.electric[..., c]) for c in range(3) if np.any(b.electric[..., c])}
        rec.update({f'H{"xyz"[c]}': rel_l2(a.magnetic[..., c], b.magnetic[..., c]) for c in range(3) if np.any(b.magnetic[..., c])})
        if a.signals.size:
            rec['trace'] = rel_l2(a.signals, b.signals)
            rec['spectrum'] = rel_l2(a.spectra[0]['value'], b.spectra[0]['value'])
        for m, n in zip(a.frequency_fields, b.frequency_fields):
            rec['plane'] = rel_l2(m['fields'], n['fields'])
        out[name] = rec
    print('FP32 vs FP64 relative L2:', out)
    assert out['tmz2d']['trace'] < 1e-5 and out['tmz2d']['spectrum'] < 1e-5
    assert max(out['tmz2d'][k] for k in ('Ez', 'Hx', 'Hy')) < 5e-2
    assert max(v for v in out['strip'].values()) < 1e-5


@pytest.mark.parametrize('precision', ['float32', 'float64'])
def test_graded_mesh_306x306x172_metric_mixed_launch_every_memory(precision):
    """The graded-mesh workload (metric equidistribution, auto-refined box, physically graded CPML) for 10 steps
    through the metric mixed march launch: the pure body with metric factors on the interior block, the general
    metric body elsewhere; fields, every CPML memory and the traces bitwise against the C oracle."""
    from torchfdtd_b200.native import NativeGrid
    project, eps = config_project('graded', 10, precision)
    plan = plan_grid(project)
    if eps is not None:
        plan.epsilon, plan.inv_eps = eps, (1 / eps).astype(plan.dtype)
    assert plan.metrics, 'the workload must run on a nonuniform mesh'
    grid = NativeGrid(plan)
    assert grid.kernel == 'march'
    grid.step(10)
    E, H = grid.get_fields()
    psi = grid.get_psi()
    traces = grid.get_traces()
    status = grid.device_status()
    grid.close()
    assert status == 0
    oracle = CpuOracle(plan).run(10)
    np.testing.assert_array_equal(E, oracle.E)
    np.testing.assert_array_equal(H, oracle.H)
    assert len(psi) == len(oracle.memory_states)
    for got, want in zip(psi, oracle.memory_states):
        np.testing.assert_array_equal(got, want)
    np.testing.assert_array_equal(traces[:10], oracle.traces[:10])
    assert np.abs(E).max() > 0

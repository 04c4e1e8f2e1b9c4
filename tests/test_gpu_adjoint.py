"""The CUDA discrete adjoint (reverse-time kernel + sqrt(T) checkpoints) against the reference's adjoint,
the CPU oracle and central finite differences.

Bars: signals bitwise equal to the reference's (they are the fused forward path); gradients within relative
L2 1e-5 (FP32) and 1e-11 (FP64) of the reference adjoint and the oracle; FP64 gradients within 1e-6 of
central differences; identical gradients for every checkpoint count."""
import numpy as np
import pytest

from oracle.adjoint_oracle import AdjointOracle
from torchfdtd_b200 import Project, Region
from torchfdtd_b200.plan import plan_grid

pytestmark = pytest.mark.gpu

GRAD_TOL = {'float32': 1e-5, 'float64': 1e-11}


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))


def cuda_project(d):
    project = Project.model_validate_json(str(d['project']))
    project.region.backend = 'cuda'
    return project


@pytest.mark.parametrize('name', ['2d_float32', '2d_float64', '3d_float32', '3d_float64', 'mesh2d_float32', 'mesh2d_float64',
                                  'mesh3d_float32', 'mesh3d_float64'])
def test_gradient_matches_reference_adjoint(golden, name):
    import torch
    from torchfdtd_b200.adjoint import DifferentiableSimulation
    d = np.load(golden / f'adjoint_{name}.npz')
    project = cuda_project(d)
    dtype = torch.float32 if project.region.precision == 'float32' else torch.float64
    model = DifferentiableSimulation(project)
    epsilon = torch.tensor(d['epsilon'], dtype=dtype, device='cuda', requires_grad=True)
    result = model(epsilon)
    np.testing.assert_array_equal(result.signals.detach().cpu().numpy(), d['signals'])
    objective = (result.signals * torch.tensor(d['weights'], dtype=dtype, device='cuda')).sum()
    objective.backward()
    assert rel(epsilon.grad.cpu().numpy(), d['gradient']) <= GRAD_TOL[project.region.precision]
    assert result.report['replayed_steps'] > 0
    model.close()


def periodic_project(precision='float64', steps=26):
    from torchfdtd_b200.models import BoundaryFace, Monitor, Source
    region = Region(dimension='3d', size=(1.6, 1.4, 1.2), mesh=.1, pml_cells=3, steps=steps, precision=precision, backend='cuda')
    region.boundaries.y_min = BoundaryFace(kind='periodic')
    region.boundaries.y_max = BoundaryFace(kind='periodic')
    region.boundaries.z_max = BoundaryFace(kind='pec')
    return Project(region=region, sources=[Source(center=(-.1, .05, 0), component='Ey', pulse_cycles=1, wavelength=.6)],
                   monitors=[Monitor(center=(.2, .1, .1), component='Ey'), Monitor(center=(.1, -.1, 0), component='Hz'),
                             Monitor(center=(0, 0, .2), component='Ex')])


def test_periodic_pec_and_per_component_epsilon_match_oracle():
    import torch
    from torchfdtd_b200.adjoint import DifferentiableSimulation
    project = periodic_project()
    plan = plan_grid(project)
    rng = np.random.default_rng(9)
    eps = rng.uniform(1, 3, size=(*plan.shape, 3))
    w = rng.normal(size=(plan.steps, 3))
    oracle = AdjointOracle(plan, eps)
    signals = oracle.forward()
    expected = oracle.backward(w)
    model = DifferentiableSimulation(project)
    epsilon = torch.tensor(eps, device='cuda', requires_grad=True)
    result = model(epsilon)
    np.testing.assert_array_equal(result.signals.detach().cpu().numpy(), signals)
    (result.signals * torch.tensor(w, device='cuda')).sum().backward()
    assert rel(epsilon.grad.cpu().numpy(), expected) <= 1e-11


def test_every_checkpoint_count_gives_the_same_gradient():
    import torch
    from torchfdtd_b200.adjoint import AdjointOptions, DifferentiableSimulation
    project = periodic_project('float32', steps=23)
    shape = plan_grid(project).shape
    eps = np.random.default_rng(2).uniform(1, 2, size=shape)
    grads = []
    for checkpoints in (1, 3, 7, None, 23):
        model = DifferentiableSimulation(project, AdjointOptions(checkpoints=checkpoints))
        epsilon = torch.tensor(eps, dtype=torch.float32, device='cuda', requires_grad=True)
        model(epsilon).signals.square().sum().backward()
        grads.append(epsilon.grad.cpu().numpy())
        model.close()
    for g in grads[1:]:
        np.testing.assert_array_equal(g, grads[0])


def plane_project(precision='float64'):
    from torchfdtd_b200.models import FieldMonitor, Source, SpectrumSettings
    region = Region(dimension='3d', size=(2.0, 1.6, 1.4), mesh=.1, pml_cells=4, steps=60, precision=precision, backend='cuda')
    spec = SpectrumSettings(sampling='frequency', frequency_points=2, apodization='none', wavelength_start=1.0,
                            wavelength_stop=1.2)
    return Project(region=region, sources=[Source(center=(-.4, 0, 0), component='Ey', pulse_cycles=1, wavelength=1.1)],
                   monitors=[FieldMonitor(id='out', center=(.4, 0, 0), size=(0, .6, .3), spectrum=spec)])


def overlap_objective(model, epsilon):
    import torch
    fields = model(epsilon)['out'].fields                       # (F, P, 6)
    ey = fields[..., 1]
    mode = torch.exp(-torch.linspace(-1, 1, ey.shape[1], device=ey.device, dtype=torch.float64) ** 2).to(ey.dtype)
    return (torch.abs((ey * mode.conj()).sum(dim=1)) ** 2).sum()


def test_plane_overlap_gradient_matches_central_differences():
    import torch
    from torchfdtd_b200.adjoint import DifferentiablePlaneSimulation
    project = plane_project()
    model = DifferentiablePlaneSimulation(project)
    shape = model.plan.shape
    rng = np.random.default_rng(5)
    eps = rng.uniform(1, 2.5, size=shape)
    epsilon = torch.tensor(eps, device='cuda', requires_grad=True)
    overlap_objective(model, epsilon).backward()
    gradient = epsilon.grad.cpu().numpy()
    picks = list(np.argsort(np.abs(gradient).ravel())[-4:]) + list(rng.integers(0, eps.size, 2))
    for flat in picks:
        idx = np.unravel_index(flat, shape)
        h = 1e-5
        up, down = eps.copy(), eps.copy()
        up[idx] += h
        down[idx] -= h
        with torch.no_grad():
            fd = float(overlap_objective(model, torch.tensor(up, device='cuda')) -
                       overlap_objective(model, torch.tensor(down, device='cuda'))) / (2 * h)
        assert abs(gradient[idx] - fd) <= 1e-6 * max(abs(fd), np.abs(gradient).max() * 1e-2), (idx, gradient[idx], fd)


def test_plane_fields_match_the_forward_simulation_planes():
    import torch
    from torchfdtd_b200 import Simulation
    from torchfdtd_b200.adjoint import DifferentiablePlaneSimulation
    project = plane_project('float64')
    model = DifferentiablePlaneSimulation(project)
    eps = np.random.default_rng(8).uniform(1, 2, size=model.plan.shape)
    fields = model(torch.tensor(eps, device='cuda'))['out'].fields.detach().cpu().numpy()
    plane = Simulation(project, epsilon=eps).run().field_monitor('out')
    assert rel(fields, plane['fields']) <= 1e-12


@pytest.mark.parametrize('precision', ['float32', 'float64'])
def test_interior_tiles_fast_path_is_the_general_path(monkeypatch, precision):
    """A grid with whole interior tiles (80 x 40 x 30 cells, CPML 6): the reverse-step kernels' interior fast path
    gives the general path's gradient bitwise, and (FP64) the oracle's."""
    import torch
    from torchfdtd_b200.adjoint import DifferentiableSimulation
    from torchfdtd_b200.models import Monitor, Source
    region = Region(dimension='3d', size=(4.0, 2.0, 1.5), mesh=.05, pml_cells=6, steps=30, precision=precision, backend='cuda')
    project = Project(region=region, sources=[Source(center=(-.6, .05, 0), component='Ey', pulse_cycles=1, wavelength=.6)],
                      monitors=[Monitor(center=(.5, .1, .1), component='Ey'), Monitor(center=(.2, -.2, -.1), component='Hz')])
    plan = plan_grid(project)
    assert plan.shape == (80, 40, 30)
    dtype = torch.float32 if precision == 'float32' else torch.float64
    eps = np.random.default_rng(5).uniform(1, 3, size=plan.shape)
    w = np.random.default_rng(6).normal(size=(plan.steps, 2))
    grads = {}
    for fast in ('1', '0'):
        monkeypatch.setenv('TFD_ADJ_FAST', fast)
        model = DifferentiableSimulation(project)
        epsilon = torch.tensor(eps, dtype=dtype, device='cuda', requires_grad=True)
        result = model(epsilon)
        (result.signals * torch.tensor(w, dtype=dtype, device='cuda')).sum().backward()
        grads[fast] = epsilon.grad.cpu().numpy()
        model.close()
    np.testing.assert_array_equal(grads['1'], grads['0'])
    assert np.abs(grads['1']).max() > 0
    if precision == 'float64':
        oracle = AdjointOracle(plan, eps)
        oracle.forward()
        assert rel(grads['1'], oracle.backward(w)) <= 1e-11

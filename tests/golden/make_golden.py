"""Write the golden vectors in tests/golden/*.npz from the reference's own CPU path.

Run where the reference source tree (read-only) is present, given as the first argument, as
$TORCHFDTD_REFERENCE, or as a ``reference`` directory beside this repository:

    python tests/golden/make_golden.py [path/to/reference [states|scenes|adjoint|results ...]]

It imports the reference package, with ``tests/golden/fdtd_standin`` standing
in for the uninstalled third-party ``fdtd`` 0.2.2 (only its constructor and
allocators are used by the reference), and records:

- ``state_*.npz``: seeded random E, H and inverse permittivity advanced by the
  reference ``YeeGrid.update_E/update_H`` for 23 steps, with every CPML memory
  (the scene family of reference ``tests/test_cuda_kernels.py:72-111``: a
  kappa=3, alpha=0.03, alpha_polynomial=1 face, 2D/3D/periodic/PEC layouts,
  FP32 and FP64);
- ``sim_*.npz``: complete ``Simulation(project).run()`` results on the CPU
  (fields, point traces, DFT planes with flux) plus the voxelized permittivity,
  for small scenes shaped like the benchmark configurations;
- ``adjoint_*.npz``: the reference ``DifferentiableSimulation`` (discrete adjoint, CPU) on small 2D/3D
  scenes: seeded random epsilon, the point-monitor signals and the gradient of sum(weights * signals).

The engine and the GPU tests never read the reference; they read these files.
"""
import json
import os
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REFERENCE = Path(sys.argv[1] if len(sys.argv) > 1 else os.environ.get('TORCHFDTD_REFERENCE', HERE.parents[2] / 'reference'))
C0 = 299792458.0


def load_reference():
    sys.path.insert(0, str(HERE / 'fdtd_standin'))
    sys.path.insert(0, str(REFERENCE))
    import torchfdtd
    return torchfdtd


# BASELINE CPML grading mapped to the reference's dimensionless face parameters:
# sigma_max = 0.8 (m+1)/(eta0 dx), m = 3  ->  sigma_scale = 3.2 (L+1)/40; kappa_max 1; alpha_max 0.05 linear.
def baseline_face(ref, layers):
    return ref.BoundaryFace(sigma_scale=3.2 * (layers + 1) / 40, kappa=1, alpha=0.05, polynomial=3, alpha_polynomial=1)


def state_regions(ref):
    from torchfdtd.models import Boundaries, BoundaryFace
    out = {}
    for layout in ('pml2d', 'pml3d', 'periodic', 'pec'):
        r = ref.Region(dimension='2d' if layout == 'pml2d' else '3d', size=(1.8, 1.6, 1.4), mesh=.1, pml_cells=3,
                       backend='cpu')
        r.boundaries.x_min = BoundaryFace(layers=5, kappa=3, alpha=.03, alpha_polynomial=1)
        if layout == 'periodic':
            r.boundaries.y_min = BoundaryFace(kind='periodic')
            r.boundaries.y_max = BoundaryFace(kind='periodic')
        if layout == 'pec':
            r.boundaries.y_max = BoundaryFace(kind='pec')
            r.boundaries.z_max = BoundaryFace(kind='pec')
        out[layout] = r
    return out


def write_states(ref):
    import fdtd
    from torchfdtd.boundaries import YeeGrid
    for layout, region in state_regions(ref).items():
        for precision in ('float32', 'float64'):
            region = region.model_copy(update={'precision': precision})
            dtype = np.float32 if precision == 'float32' else np.float64
            fdtd.set_backend('numpy')
            from fdtd.backend import NumpyBackend

            class Precision(NumpyBackend):
                def zeros(self, shape, dtype_=None):
                    return np.zeros(shape, dtype=dtype)

                def ones(self, shape, dtype_=None):
                    return np.ones(shape, dtype=dtype)
            fdtd.backend.__class__ = Precision
            g = YeeGrid(region)
            rng = np.random.default_rng(615)
            init = {}
            for name in ('E', 'H', 'inverse_permittivity'):
                dst = getattr(g, name)
                values = rng.normal(size=dst.shape) * .02 if name != 'inverse_permittivity' else rng.uniform(.25, 1, dst.shape)
                dst[:] = values.astype(np.float32).astype(dtype)
                init[name] = dst.copy()
            for _ in range(23):
                g.update_E()
                g.update_H()
            arrays = {f'init_{k}': v for k, v in init.items()}
            arrays.update(E=g.E, H=g.H, **{f'psi_{i}': s for i, s in enumerate(g.memory_states)})
            np.savez_compressed(HERE / f'state_{layout}_{precision}.npz', region=region.model_dump_json(), steps=23, **arrays)
            fdtd.set_backend('numpy')


def scenes(ref):
    from torchfdtd.models import Boundaries, BoundaryFace
    P, R, S, M, F, St, Mat, Sp = (ref.Project, ref.Region, ref.Source, ref.Monitor, ref.FieldMonitor, ref.Structure,
                                  ref.Material, ref.SpectrumSettings)
    lam = 1.55
    custom = Sp(sampling='custom', custom_frequencies_hz=[C0 / (lam * 1e-6)], apodization='none')
    out = {}
    # Config-0 shaped 2D TMz: straight core eps=3.476^2 in eps=1.444^2, Gaussian Ez point source.
    L = 16
    b = Boundaries(**{f'{a}_{s}': baseline_face(ref, L) for a in 'xy' for s in ('min', 'max')})
    out['tmz'] = P(name='tmz', region=R(dimension='2d', size=(3.2, 2.4, 1), mesh=.05, pml_cells=L, background_index=1.444,
                                        steps=300, backend='cpu', boundaries=b),
                   materials=[Mat(name='core', index=3.476)],
                   structures=[St(id='core', name='core', size=(3.2, .5, 1), material='core')],
                   sources=[S(id='src', center=(-.5, 0, 0), component='Ez', wavelength=lam, pulse='gaussian',
                              time_definition='standard', pulse_length=35.3e-15, pulse_offset=45e-15)],
                   monitors=[M(id='probe', center=(.5, 0, 0), component='Ez', spectrum=custom),
                             F(id='plane', normal='x', center=(.4, 0, 0), size=(0, 0.6, 1),
                               spectrum=Sp(sampling='wavelength', wavelength_start=1.5, wavelength_stop=1.6, frequency_points=3,
                                           apodization='none'))])
    # Config-1 shaped 3D: Si strip in SiO2, Ey dipole, x-normal DFT plane in FP64.
    L = 5
    b3 = Boundaries(**{f'{a}_{s}': baseline_face(ref, L) for a in 'xyz' for s in ('min', 'max')})
    strip = dict(materials=[Mat(name='Si', index=12.08**.5)],
                 structures=[St(id='strip', name='strip', size=(1.6, .65, .4), material='Si')],
                 sources=[S(id='dip', center=(-.25, 0, 0), component='Ey', wavelength=lam, pulse='gaussian',
                            time_definition='standard', pulse_length=20e-15, pulse_offset=30e-15)],
                 monitors=[M(id='probe', center=(.2, 0.05, 0), component='Ey', spectrum=custom),
                           F(id='plane', normal='x', center=(.25, 0, 0), size=(0, .6, .3), dft_precision='float64',
                             spectrum=custom)])
    reg3 = dict(dimension='3d', size=(1.6, 1.2, 0.8), mesh=.05, pml_cells=L, background_index=2.085**.5, steps=150,
                backend='cpu', boundaries=b3)
    out['strip3d'] = P(name='strip3d', region=R(**reg3), **strip)
    out['strip3d_f64'] = P(name='strip3d_f64', region=R(**reg3, precision='float64'), **strip)
    # Yee sampling, periodic x, PEC y, a sphere, a plane Ex sheet and an Hz point source; decimated trace and
    # an apodized plane; E and H traces.
    b = Boundaries(x_min=BoundaryFace(kind='periodic'), x_max=BoundaryFace(kind='periodic'),
                   y_min=BoundaryFace(kind='pec'), y_max=BoundaryFace(kind='pec'),
                   z_min=BoundaryFace(layers=4, kappa=2, alpha=.02, alpha_polynomial=1), z_max=BoundaryFace(layers=4))
    out['yee_periodic'] = P(name='yee_periodic', region=R(dimension='3d', size=(1.2, 1.0, 1.4), mesh=.05, pml_cells=4, steps=120,
                                                          material_sampling='yee', backend='cpu', boundaries=b),
                            structures=[St(id='ball', name='ball', kind='sphere', radius=.22, material='Si (constant n)')],
                            sources=[S(id='sheet', kind='plane', center=(0, 0, -.3), size=(1.2, .6, 0), normal='z',
                                       component='Ex', wavelength=1.3, pulse_cycles=2),
                                     S(id='mag', center=(.1, .1, .1), component='Hz', wavelength=1.3, pulse_cycles=2, amplitude=.5)],
                            monitors=[M(id='e', center=(0, 0, .2), component='Ex', time_downsample=2,
                                        spectrum=Sp(sampling='frequency', frequency_points=4, apodization='none')),
                                      M(id='h', center=(0.05, -0.1, .2), component='Hy'),
                                      F(id='plane', normal='z', center=(0, 0, .25), size=(1.2, .8, 0), time_downsample=2,
                                        spectrum=Sp(sampling='frequency', frequency_points=2, apodization='full',
                                                    apodization_center=30e-15, apodization_time_width=15e-15))])
    # 2D TE: an Ey sheet and an Hz point source, kappa>1 CPML.
    b = Boundaries(x_min=BoundaryFace(layers=8, kappa=2.5, alpha=.04, alpha_polynomial=1), x_max=BoundaryFace(layers=8),
                   y_min=BoundaryFace(layers=6), y_max=BoundaryFace(layers=6, sigma_scale=1.5))
    out['te2d'] = P(name='te2d', region=R(dimension='2d', size=(2.4, 2.0, 1), mesh=.05, steps=200, backend='cpu', boundaries=b),
                    structures=[St(id='c', name='c', kind='circle', radius=.3, material='Si (constant n)')],
                    sources=[S(id='sheet', kind='plane', center=(-.5, 0, 0), size=(0, .8, 0), component='Ey', pulse_cycles=2),
                             S(id='mag', center=(.3, .2, 0), component='Hz', pulse_cycles=2)],
                    monitors=[M(id='p', center=(.4, -.1, 0), component='Hz'),
                              F(id='plane', normal='y', center=(0, .4, 0), size=(1.0, 0, 1),
                                spectrum=Sp(sampling='frequency', frequency_points=2, apodization='none'))])
    # 2D, both polarizations: a tilted electric dipole (Ex, Ey, Ez) and a ring.
    out['both2d'] = P(name='both2d', region=R(dimension='2d', size=(2.0, 2.0, 1), mesh=.05, pml_cells=6, steps=160, backend='cpu'),
                      structures=[St(id='r', name='r', kind='ring', radius=.4, inner_radius=.2, material='SiN (constant n)')],
                      sources=[S(id='tilt', center=(-.2, .1, 0), component='Ex', theta=60, phi=30, pulse_cycles=2)],
                      monitors=[M(id='ez', center=(.3, 0, 0), component='Ez'), M(id='hz', center=(.3, 0, 0), component='Hz')])
    # The reference's own tiny fixture scene (tests/fixtures/generate_fixtures.py:tiny_result_project).
    out['tiny'] = P(name='tiny 2D result', region=R(dimension='2d', size=(2, 2, .1), mesh=.1, pml_cells=3, steps=40,
                                                    snapshot_interval=10, backend='cpu'),
                    sources=[S(id='src', wavelength=1, pulse_cycles=1)], monitors=[M(id='probe', center=(.4, 0, 0))])
    return out


def write_scenes(ref):
    from torchfdtd.solver import voxelize
    for name, project in scenes(ref).items():
        result = ref.Simulation(project).run()
        eps, _ = voxelize(project)
        arrays = dict(E=result.electric, H=result.magnetic, signals=result.signals, times=result.times, epsilon=eps,
                      frame_steps=result.frame_steps, frames=result.frames)
        for k, plane in enumerate(result.frequency_fields):
            for key in ('fields', 'flux', 'poynting', 'points_um', 'weights', 'frequency_hz'):
                if plane.get(key) is not None:
                    arrays[f'plane{k}_{key}'] = plane[key]
        for k, spec in enumerate(result.spectra):
            arrays[f'spectrum{k}_frequency_hz'] = spec['frequency_hz']
            arrays[f'spectrum{k}_value'] = spec['value']
        np.savez_compressed(HERE / f'sim_{name}.npz', project=project.model_dump_json(), **arrays,
                            summary=json.dumps({k: result.summary[k] for k in ('steps', 'precision', 'slice_index')}))


def adjoint_scenes(ref):
    """Small scenes for the discrete adjoint: kappa > 1 CPML, a PEC face, E and H point monitors."""
    from torchfdtd.models import BoundaryFace, Monitor, Project, Region, Source
    out = {}
    for dim in ('2d', '3d'):
        for precision in ('float32', 'float64'):
            r = Region(dimension=dim, size=(1.6, 1.4, 1.2 if dim == '3d' else 1), mesh=.1, pml_cells=3, steps=30,
                       precision=precision, backend='cpu')
            r.boundaries.x_min = BoundaryFace(layers=4, kappa=2, alpha=.04, alpha_polynomial=1)
            r.boundaries.y_max = BoundaryFace(kind='pec')
            out[f'{dim}_{precision}'] = Project(
                name=f'adjoint {dim}', region=r,
                sources=[Source(id='src', center=(-.1, .05, 0), component='Ez', pulse_cycles=1, wavelength=.6)],
                monitors=[Monitor(id='ez', center=(.2, .1, 0), component='Ez'),
                          Monitor(id='hy', center=(.1, -.1, 0), component='Hy')])
    return out


def write_adjoint(ref):
    """Reference DifferentiableSimulation on the CPU: signals and d/d eps of sum(w * signals)."""
    import torch
    from torchfdtd.differentiable import AdjointOptions, DifferentiableSimulation
    for name, project in adjoint_scenes(ref).items():
        dtype = torch.float32 if project.region.precision == 'float32' else torch.float64
        rng = np.random.default_rng(17)
        shape = tuple(project.region.shape)
        eps = rng.uniform(1, 3, size=shape)
        weights = rng.normal(size=(project.region.steps, 2))
        model = DifferentiableSimulation(project, AdjointOptions(checkpoints=4))
        epsilon = torch.tensor(eps, dtype=dtype, requires_grad=True)
        result = model(epsilon)
        objective = (result.signals * torch.tensor(weights, dtype=dtype)).sum()
        objective.backward()
        np.savez_compressed(HERE / f'adjoint_{name}.npz', project=project.model_dump_json(), epsilon=eps.astype(np.float64),
                            weights=weights, signals=result.signals.detach().numpy(), gradient=epsilon.grad.numpy(),
                            objective=float(objective.detach()))


def write_results(ref):
    """The reference's own ``Result.save`` of complete CPU runs: the NPZ layout a result written here must
    reproduce and that ``Result.load`` here must read."""
    for name in ('strip3d', 'yee_periodic'):
        result = ref.Simulation(scenes(ref)[name]).run()
        result.save(HERE / f'result_{name}.npz')


WRITERS = {'states': write_states, 'scenes': write_scenes, 'adjoint': write_adjoint, 'results': write_results}

if __name__ == '__main__':
    # Optional names after the reference path select writers (default: all of them).
    ref = load_reference()
    for name in (sys.argv[2:] or WRITERS):
        WRITERS[name](ref)
    for path in sorted(HERE.glob('*.npz')):
        print(f'{path.name}: {path.stat().st_size/1024:.0f} KiB')

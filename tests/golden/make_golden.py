"""Write the golden vectors in tests/golden/*.npz from the reference's own CPU path.

Run where the reference source tree (read-only) is present, given as the first argument, as
$TORCHFDTD_REFERENCE, or as a ``reference`` directory beside this repository:

    python tests/golden/make_golden.py [path/to/reference [states|scenes|adjoint|results|mesh|sources ...]]

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


def mesh_state_regions(ref):
    """Nonuniform meshes for the random-state CPML goldens: a graded mesh (a refinement box, coarse gaps) with
    the kappa=3 face and a PEC face, and explicit coordinates with periodic x (the wrap metric) and physically
    graded CPML on y and z."""
    from torchfdtd.models import BoundaryFace, MeshRefinement
    out = {}
    r = ref.Region(dimension='3d', size=(3.0, 2.4, 2.0), mesh=.1, pml_cells=3, mesh_type='graded', mesh_max=.25,
                   mesh_grading=1.4, material_sampling='yee', backend='cpu',
                   mesh_refinements=[MeshRefinement(center=(.3, -.2, .1), size=(.4, .5, .3))])
    r.boundaries.x_min = BoundaryFace(layers=5, kappa=3, alpha=.03, alpha_polynomial=1)
    r.boundaries.z_max = BoundaryFace(kind='pec')
    out['graded'] = r
    rng = np.random.default_rng(77)
    coords = []
    for span, cells in ((1.6, 14), (1.4, 13), (1.2, 12)):
        w = rng.uniform(.7, 1.3, cells)
        w = w / w.sum() * span
        nodes = np.r_[0, np.cumsum(w)] - span / 2
        nodes[0], nodes[-1] = -span / 2, span / 2
        coords.append(tuple(float(v) for v in nodes))
    r = ref.Region(dimension='3d', size=(1.6, 1.4, 1.2), mesh=.1, pml_cells=3, mesh_type='explicit',
                   mesh_coordinates=tuple(coords), material_sampling='yee', backend='cpu')
    r.boundaries.x_min = BoundaryFace(kind='periodic')
    r.boundaries.x_max = BoundaryFace(kind='periodic')
    out['explicit'] = r
    return out


def write_states(ref, regions=None):
    import fdtd
    from torchfdtd.boundaries import YeeGrid
    for layout, region in (regions or state_regions(ref)).items():
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


def write_scenes(ref, projects=None):
    from torchfdtd.solver import voxelize
    for name, project in (projects or scenes(ref)).items():
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


def adjoint_mesh_scenes(ref):
    """The adjoint scenes on nonuniform meshes: graded (2D, with a refinement box) and explicit coordinates
    with a periodic axis (3D), FP32 and FP64."""
    from torchfdtd.models import BoundaryFace, MeshRefinement, Monitor, Project, Region, Source
    out = {}
    for dim in ('2d', '3d'):
        for precision in ('float32', 'float64'):
            if dim == '2d':
                r = Region(dimension='2d', size=(2.4, 2.0, 1), mesh=.08, pml_cells=3, steps=40, precision=precision,
                           backend='cpu', mesh_type='graded', mesh_max=.2, mesh_grading=1.4, material_sampling='yee',
                           mesh_refinements=[MeshRefinement(center=(.3, .2, 0), size=(.3, .3, 1))])
                r.boundaries.y_max = BoundaryFace(kind='pec')
            else:
                rng = np.random.default_rng(5)
                coords = []
                for span, cells in ((1.6, 16), (1.4, 14), (1.2, 12)):
                    w = rng.uniform(.8, 1.25, cells)
                    w = w / w.sum() * span
                    nodes = np.r_[0, np.cumsum(w)] - span / 2
                    nodes[0], nodes[-1] = -span / 2, span / 2
                    coords.append(tuple(float(v) for v in nodes))
                r = Region(dimension='3d', size=(1.6, 1.4, 1.2), mesh=.1, pml_cells=3, steps=30, precision=precision,
                           backend='cpu', mesh_type='explicit', mesh_coordinates=tuple(coords), material_sampling='yee')
                r.boundaries.x_min = BoundaryFace(kind='periodic')
                r.boundaries.x_max = BoundaryFace(kind='periodic')
            out[f'mesh{dim}_{precision}'] = Project(
                name=f'adjoint mesh {dim}', region=r,
                sources=[Source(id='src', center=(-.1, .05, 0), component='Ez', pulse_cycles=1, wavelength=.6)],
                monitors=[Monitor(id='ez', center=(.2, .1, 0), component='Ez'),
                          Monitor(id='hy', center=(.1, -.1, 0), component='Hy')])
    return out


def write_adjoint(ref, projects=None):
    """Reference DifferentiableSimulation on the CPU: signals and d/d eps of sum(w * signals)."""
    import torch
    from torchfdtd.differentiable import AdjointOptions, DifferentiableSimulation
    for name, project in (projects or adjoint_scenes(ref)).items():
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


def mesh_scenes(ref):
    """Complete runs on nonuniform meshes: graded (automatic refinement around the objects), axis-specific steps
    and explicit coordinates with a periodic axis; 3D and 2D TMz, E and H sources, point traces and DFT planes."""
    from torchfdtd.models import Boundaries, BoundaryFace, MeshRefinement
    P, R, S, M, F, St, Sp = (ref.Project, ref.Region, ref.Source, ref.Monitor, ref.FieldMonitor, ref.Structure,
                             ref.SpectrumSettings)
    lam = 1.55
    custom = Sp(sampling='custom', custom_frequencies_hz=[C0 / (lam * 1e-6)], apodization='none')
    out = {}
    out['graded3d'] = P(name='graded3d', region=R(dimension='3d', size=(3.2, 2.4, 2.0), mesh=.05, pml_cells=5, steps=160,
                                                  mesh_type='graded', mesh_max=.16, material_sampling='yee', backend='cpu',
                                                  background_index=1.444),
                        structures=[St(id='wg', name='wg', size=(3.2, .5, .3), material='Si (constant n)'),
                                    St(id='ball', name='ball', kind='sphere', center=(.6, .4, .2), radius=.2, material='Si (constant n)')],
                        sources=[S(id='dip', center=(-.9, 0, 0), component='Ey', wavelength=lam, pulse='gaussian',
                                   time_definition='standard', pulse_length=12e-15, pulse_offset=25e-15)],
                        monitors=[M(id='probe', center=(.9, 0, 0), component='Ey', spectrum=custom),
                                  F(id='plane', normal='x', center=(1.0, 0, 0), size=(0, .8, .6), dft_precision='float64',
                                    spectrum=custom)])
    b = Boundaries(**{f'{a}_{s}': BoundaryFace(layers=8) for a in 'xy' for s in ('min', 'max')})
    b.y_max = BoundaryFace(kind='pec')
    out['graded2d'] = P(name='graded2d', region=R(dimension='2d', size=(4.0, 3.0, 1), mesh=.04, pml_cells=8, steps=300,
                                                  mesh_type='graded', mesh_max=.12, mesh_grading=1.3, material_sampling='yee',
                                                  backend='cpu', boundaries=b,
                                                  mesh_refinements=[MeshRefinement(center=(.8, -.6, 0), size=(.3, .3, 1))]),
                        structures=[St(id='c', name='c', kind='circle', center=(.5, .3, 0), radius=.3, material='Si (constant n)')],
                        sources=[S(id='src', center=(-1.0, 0, 0), component='Ez', wavelength=1.3, pulse_cycles=2),
                                 S(id='mag', center=(-.5, .4, 0), component='Hx', wavelength=1.3, pulse_cycles=2, amplitude=.3)],
                        monitors=[M(id='probe', center=(1.0, -.2, 0), component='Ez'),
                                  F(id='plane', normal='x', center=(1.2, 0, 0), size=(0, 1.2, 1),
                                    spectrum=Sp(sampling='frequency', frequency_points=2, apodization='none'))])
    out['steps3d'] = P(name='steps3d', region=R(dimension='3d', size=(2.0, 1.6, 1.5), mesh=.05, mesh_steps=(.05, .04, .06),
                                                pml_cells=5, steps=120, material_sampling='yee', backend='cpu'),
                       structures=[St(id='blk', name='blk', size=(.6, .4, .3), material='Si (constant n)')],
                       sources=[S(id='src', center=(-.4, 0, 0), component='Ez', wavelength=1.3, pulse_cycles=2)],
                       monitors=[M(id='probe', center=(.4, .1, 0), component='Ez'),
                                 F(id='plane', normal='z', center=(0, 0, .2), size=(.8, .6, 0),
                                   spectrum=Sp(sampling='frequency', frequency_points=2, apodization='none'))])
    rng = np.random.default_rng(91)
    coords = []
    for span, cells in ((1.6, 30), (1.6, 34), (1.2, 26)):
        w = rng.uniform(.8, 1.25, cells)
        w = w / w.sum() * span
        nodes = np.r_[0, np.cumsum(w)] - span / 2
        nodes[0], nodes[-1] = -span / 2, span / 2
        coords.append(tuple(float(v) for v in nodes))
    b = Boundaries(x_min=BoundaryFace(kind='periodic'), x_max=BoundaryFace(kind='periodic'),
                   y_min=BoundaryFace(layers=5), y_max=BoundaryFace(layers=5), z_min=BoundaryFace(layers=4), z_max=BoundaryFace(layers=4))
    out['explicit3d'] = P(name='explicit3d', region=R(dimension='3d', size=(1.6, 1.6, 1.2), mesh=.05, mesh_type='explicit',
                                                      mesh_coordinates=tuple(coords), pml_cells=5, steps=120, material_sampling='yee',
                                                      backend='cpu', boundaries=b),
                          structures=[St(id='rod', name='rod', kind='circle', radius=.15, size=(1, 1, 1.2), material='Si (constant n)')],
                          sources=[S(id='sheet', kind='plane', center=(0, -.3, 0), size=(1.6, 0, .5), normal='y', component='Ex',
                                     wavelength=1.2, pulse_cycles=2)],
                          monitors=[M(id='h', center=(.1, .3, 0), component='Hz'),
                                    F(id='plane', normal='y', center=(0, .35, 0), size=(1.6, 0, .6),
                                      spectrum=Sp(sampling='frequency', frequency_points=2, apodization='none'))])
    return out


def write_mesh(ref):
    write_states(ref, mesh_state_regions(ref))
    write_scenes(ref, mesh_scenes(ref))
    write_adjoint(ref, adjoint_mesh_scenes(ref))


def source_scenes(ref):
    """One-way (Huygens) plane sources: 3D with periodic x/y and a dielectric slab downstream (Ex, travelling +z),
    and 2D TMz with periodic y (Ez, travelling -x); traces on both sides of the plane and a DFT plane."""
    from torchfdtd.models import Boundaries, BoundaryFace
    P, R, S, M, F, St, Sp = (ref.Project, ref.Region, ref.Source, ref.Monitor, ref.FieldMonitor, ref.Structure,
                             ref.SpectrumSettings)
    out = {}
    b = Boundaries(x_min=BoundaryFace(kind='periodic'), x_max=BoundaryFace(kind='periodic'),
                   y_min=BoundaryFace(kind='periodic'), y_max=BoundaryFace(kind='periodic'),
                   z_min=BoundaryFace(layers=8), z_max=BoundaryFace(layers=8))
    out['oneway3d'] = P(name='oneway3d', region=R(dimension='3d', size=(0.8, 0.6, 3.0), mesh=.05, pml_cells=8, steps=180,
                                                  backend='cpu', boundaries=b),
                        structures=[St(id='slab', name='slab', size=(0.8, 0.6, .3), center=(0, 0, .6), material='Si (constant n)')],
                        sources=[S(id='pw', kind='plane', injection='oneway', normal='z', direction='+', center=(0, 0, -.5),
                                   size=(0.8, 0.6, 0), component='Ex', wavelength=1.3, pulse_cycles=2)],
                        monitors=[M(id='up', center=(0, 0, .2), component='Ex'), M(id='down', center=(0, 0, -.9), component='Ex'),
                                  M(id='hy', center=(0.1, 0, .1), component='Hy'),
                                  F(id='plane', normal='z', center=(0, 0, 1.0), size=(0.8, 0.6, 0),
                                    spectrum=Sp(sampling='frequency', frequency_points=2, apodization='none'))])
    b = Boundaries(x_min=BoundaryFace(layers=10), x_max=BoundaryFace(layers=10),
                   y_min=BoundaryFace(kind='periodic'), y_max=BoundaryFace(kind='periodic'))
    out['oneway2d'] = P(name='oneway2d', region=R(dimension='2d', size=(4.0, 1.0, 1), mesh=.05, pml_cells=10, steps=260,
                                                  backend='cpu', boundaries=b),
                        structures=[St(id='c', name='c', kind='circle', center=(-1.0, 0, 0), radius=.2, material='Si (constant n)')],
                        sources=[S(id='pw', kind='plane', injection='oneway', normal='x', direction='-', center=(.5, 0, 0),
                                   size=(0, 1.0, 0), component='Ez', wavelength=1.2, pulse_cycles=2, amplitude=.7)],
                        monitors=[M(id='left', center=(-.5, 0, 0), component='Ez'), M(id='right', center=(1.2, 0, 0), component='Ez'),
                                  F(id='plane', normal='x', center=(-1.5, 0, 0), size=(0, 1.0, 1),
                                    spectrum=Sp(sampling='frequency', frequency_points=2, apodization='none'))])
    return out


def tfsf_scenes(ref):
    """TFSF boxes: 3D (Ey, travelling +x, a sphere inside the box) and 2D TMz (Ez, travelling -y, a circle
    inside); traces inside (total field) and outside (scattered field), a DFT plane in the scattered region."""
    P, R, S, M, F, St, Sp = (ref.Project, ref.Region, ref.Source, ref.Monitor, ref.FieldMonitor, ref.Structure,
                             ref.SpectrumSettings)
    out = {}
    out['tfsf3d'] = P(name='tfsf3d', region=R(dimension='3d', size=(2.4, 2.2, 2.0), mesh=.05, pml_cells=6, steps=150,
                                              backend='cpu'),
                      structures=[St(id='ball', name='ball', kind='sphere', radius=.25, material='Si (constant n)')],
                      sources=[S(id='box', kind='tfsf', normal='x', direction='+', center=(0, 0, 0), size=(1.0, 1.1, .9),
                                 component='Ey', wavelength=1.3, pulse_cycles=2)],
                      monitors=[M(id='inside', center=(-.3, .1, 0), component='Ey'),
                                M(id='outside', center=(-.8, .1, 0), component='Ey'),
                                M(id='hz', center=(.7, 0, .1), component='Hz'),
                                F(id='plane', normal='x', center=(.75, 0, 0), size=(0, 1.2, 1.0),
                                  spectrum=Sp(sampling='frequency', frequency_points=2, apodization='none'))])
    out['tfsf2d'] = P(name='tfsf2d', region=R(dimension='2d', size=(3.0, 3.0, 1), mesh=.04, pml_cells=10, steps=300,
                                              backend='cpu'),
                      structures=[St(id='c', name='c', kind='circle', radius=.3, center=(.1, 0, 0), material='Si (constant n)')],
                      sources=[S(id='box', kind='tfsf', normal='y', direction='-', center=(0, 0, 0), size=(1.4, 1.2, 0),
                                 component='Ez', wavelength=1.1, pulse_cycles=2, amplitude=.8)],
                      monitors=[M(id='inside', center=(.2, .3, 0), component='Ez'), M(id='outside', center=(.9, .2, 0), component='Ez'),
                                F(id='plane', normal='x', center=(-1.0, 0, 0), size=(0, 1.6, 1),
                                  spectrum=Sp(sampling='frequency', frequency_points=2, apodization='none'))])
    return out


def dispersive_scenes(ref):
    """Dispersive materials through the coupled trapezoidal ADE: 3D with a Drude sphere and a Lorentz slab (cell
    sampling); 2D TMz with a two-pole material reaching into the PML under pml_dispersion='frozen' and a Lorentz
    circle (Yee sampling)."""
    from torchfdtd.models import LorentzPole
    P, R, S, M, F, St, Sp, Mat = (ref.Project, ref.Region, ref.Source, ref.Monitor, ref.FieldMonitor, ref.Structure,
                                  ref.SpectrumSettings, ref.Material)
    out = {}
    metal = Mat(name='metal', model='drude', epsilon_inf=1.5, plasma_rad_s=9e15, collision_rad_s=1e14)
    glass = Mat(name='disp', model='lorentz', epsilon_inf=2.0, resonance_rad_s=3e15, linewidth_rad_s=2e14, delta_epsilon=1.2)
    out['drude3d'] = P(name='drude3d', region=R(dimension='3d', size=(2.0, 1.6, 1.4), mesh=.05, pml_cells=6, steps=160, backend='cpu'),
                       materials=[metal, glass],
                       structures=[St(id='ball', name='ball', kind='sphere', center=(.3, 0, 0), radius=.2, material='metal'),
                                   St(id='slab', name='slab', size=(.2, 1.6, 1.4), center=(-.35, 0, 0), material='disp')],
                       sources=[S(id='src', center=(-.6, .1, 0), component='Ey', wavelength=1.2, pulse_cycles=2)],
                       monitors=[M(id='probe', center=(.55, 0, 0), component='Ey'), M(id='in', center=(-.35, .1, .05), component='Ey'),
                                 F(id='plane', normal='x', center=(.6, 0, 0), size=(0, .8, .6),
                                   spectrum=Sp(sampling='frequency', frequency_points=2, apodization='none'))])
    multi = Mat(name='multi', model='multipole', epsilon_inf=1.8,
                poles=[LorentzPole(resonance_rad_s=2.5e15, strength_rad_s_squared=6e30, damping_rad_s=1e14),
                       LorentzPole(resonance_rad_s=0, strength_rad_s_squared=2e30, damping_rad_s=3e14)])
    lor = Mat(name='lor', model='lorentz', epsilon_inf=1.2, resonance_rad_s=4e15, linewidth_rad_s=1e14, delta_epsilon=2.0)
    out['frozen2d'] = P(name='frozen2d', region=R(dimension='2d', size=(3.0, 2.4, 1), mesh=.04, pml_cells=8, steps=300,
                                                  material_sampling='yee', pml_dispersion='frozen', backend='cpu'),
                        materials=[multi, lor],
                        structures=[St(id='bar', name='bar', size=(3.0, .3, 1), center=(0, -.5, 0), material='multi'),
                                    St(id='c', name='c', kind='circle', center=(.4, .3, 0), radius=.25, material='lor')],
                        sources=[S(id='src', center=(-.8, 0, 0), component='Ez', wavelength=1.3, pulse_cycles=2)],
                        monitors=[M(id='probe', center=(.9, .1, 0), component='Ez'), M(id='inbar', center=(0, -.5, 0), component='Ez')])
    return out


def write_sources(ref):
    write_scenes(ref, source_scenes(ref))
    write_scenes(ref, tfsf_scenes(ref))
    write_scenes(ref, dispersive_scenes(ref))


def write_results(ref):
    """The reference's own ``Result.save`` of complete CPU runs: the NPZ layout a result written here must
    reproduce and that ``Result.load`` here must read."""
    for name in ('strip3d', 'yee_periodic'):
        result = ref.Simulation(scenes(ref)[name]).run()
        result.save(HERE / f'result_{name}.npz')


WRITERS = {'states': write_states, 'scenes': write_scenes, 'adjoint': write_adjoint, 'results': write_results, 'mesh': write_mesh,
           'sources': write_sources}

if __name__ == '__main__':
    # Optional names after the reference path select writers (default: all of them).
    ref = load_reference()
    for name in (sys.argv[2:] or WRITERS):
        WRITERS[name](ref)
    for path in sorted(HERE.glob('*.npz')):
        print(f'{path.name}: {path.stat().st_size/1024:.0f} KiB')

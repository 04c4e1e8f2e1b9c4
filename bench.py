"""Benchmark of the fused Yee/CPML engine: Gcell-updates/s and HBM-roofline fraction.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload roofline|roofline256|strip|periodic|tmz2d|batch64|adjoint3d|surrogate|
                                adjoint_probe|surrogate_kernels]

Workload (default ``roofline``): 3D full-vector Yee + CPML, FP32, 512 x 512 x 256 cells
at 0.05 um, CPML 12 cells per face (cubic grading, sigma_max = 0.8 (m+1)/(eta0 dx),
kappa_max 1, alpha_max 0.05), seeded random piecewise-constant permittivity in [1, 12.1]
on 8^3-cell blocks, Ey dipole at the centre, one Ey point trace. ``strip`` is the
160 x 120 x 40 Si-strip scene with an x-normal DFT plane. ``periodic`` is 512 x 512 x 128 with
periodic x/y faces and CPML on z only, the scenes the reference's one-pass marching kernel admits;
its line adds ``restated_reference``, that kernel restated in CUDA (baseline/fused_eh_marching.cu)
and timed on the same device, scene and steps. All inputs are synthetic and
seeded. A bench step is one FDTD time step over the whole grid (one fused step launch
plus one observation launch).

* ``value``: device-timed (CUDA events on the launching stream) whole-job throughput,
  fields resident in HBM; inputs are larger than L2, so no flush is needed.
* ``e2e``: the same metric through the public call ``Simulation(project, epsilon).run()``,
  wall-clock from the call to its return (planning, host->device upload of the material,
  graph capture, the K steps, device->host copies of fields, traces and frames).
* ``roofline``: algorithmic bytes per step (each field component read and written once,
  the permittivity read once, each CPML memory read and written once) per average step
  time, against the measured HBM copy peak.
* ``cpu_baseline``: the C oracle (oracle/yee_cpu.c, same arithmetic, all host threads) on
  the same grid for a bounded number of steps.

``--impl reference`` times the reference's CPU algorithm (the C port of its NumPy path)
on the host cores. With torchrun (N>1) every rank runs its own replica (the benchmark
configurations are single-GPU; the engine does not shard a grid): scaling "weak", time
is the max over ranks.
"""
import argparse
import json
import math
import os
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = 'Gcell-updates/s'
C0 = 299792458.0
# DRAM bytes per cell-update of the step kernel(s) measured by ncu on the workload itself
# (dram__bytes_read.sum + dram__bytes_write.sum of one launch / cells; profiles/ has the commands):
# 512x512x256: 2.428 + 1.776 GB per k_step_march_mixed launch; batch64: 493.4 MB (k_step2d_interior) + 118.5 MB
# (k_step2d_general) per step at the tuned launch shape.
L2_NOTE = 'inputs larger than L2 (no flush needed)'
MEASURED_TRAFFIC_PER_CELL = {('roofline', 'march'): 4.175e9 / 67108864, ('batch64', 'tile2d'): 611.9e6 / 20187264}


def baseline_face(layers):
    from torchfdtd_b200 import BoundaryFace
    return BoundaryFace(sigma_scale=3.2 * (layers + 1) / 40, kappa=1, alpha=0.05, polynomial=3, alpha_polynomial=1)


def workload(name, steps, seed=2024):
    """(project, epsilon or None, description) of a benchmark workload."""
    from torchfdtd_b200 import Boundaries, FieldMonitor, Material, Monitor, Project, Region, Source, SpectrumSettings, Structure
    from torchfdtd_b200.models import BoundaryFace, RunControl
    lam = 1.55
    control = RunControl(divergence_check=False)
    src = dict(component='Ey', wavelength=lam, pulse='gaussian', time_definition='standard', pulse_length=20e-15, pulse_offset=40e-15)
    if name in ('roofline', 'roofline256'):
        # 'roofline256' is the same scene at 256^3 cells (about 1.3 GB on the device) for profiler captures.
        n = (512, 512, 256) if name == 'roofline' else (256, 256, 256)
        L = 12
        b = Boundaries(**{f'{a}_{s}': baseline_face(L) for a in 'xyz' for s in ('min', 'max')})
        region = Region(dimension='3d', size=tuple(v * .05 for v in n), mesh=.05, pml_cells=L, steps=steps, backend='cuda',
                        cuda_kernel='fused', boundaries=b, run_control=control, snapshot_interval=10000)
        project = Project(name=f'roofline {n[0]}x{n[1]}x{n[2]}', region=region, sources=[Source(id='dip', center=(0, 0, 0), **src)],
                          monitors=[Monitor(id='probe', center=(1.0, 0, 0), component='Ey')])
        rng = np.random.default_rng(seed)
        blocks = rng.uniform(1, 12.1, tuple(v // 8 for v in n)).astype(np.float32)
        eps = np.repeat(np.repeat(np.repeat(blocks, 8, 0), 8, 1), 8, 2)
        return project, eps, (f'3D Yee+CPML {n[0]}x{n[1]}x{n[2]} (0.05 um), CPML 12, seeded random piecewise-constant eps in '
                              '[1,12.1] on 8^3 blocks, Ey dipole at the centre, FP32')
    if name == 'periodic':
        # Periodic x/y, CPML on z only, E source: the scenes the reference's one-pass marching kernel
        # (FusedEHMarching) admits; its CTA holds all z, so nz stays within its 160-plane limit.
        n, L = (512, 512, 128), 12
        b = Boundaries(**{f'{a}_{s}': BoundaryFace(kind='periodic') for a in 'xy' for s in ('min', 'max')},
                       z_min=baseline_face(L), z_max=baseline_face(L))
        region = Region(dimension='3d', size=tuple(v * .05 for v in n), mesh=.05, pml_cells=L, steps=steps, backend='cuda',
                        cuda_kernel='fused', boundaries=b, run_control=control, snapshot_interval=10000)
        project = Project(name='periodic 512x512x128', region=region, sources=[Source(id='dip', center=(0, 0, 0), **src)])
        rng = np.random.default_rng(seed)
        blocks = rng.uniform(1, 12.1, tuple(v // 8 for v in n)).astype(np.float32)
        eps = np.repeat(np.repeat(np.repeat(blocks, 8, 0), 8, 1), 8, 2)
        return project, eps, ('3D Yee 512x512x128 (0.05 um), periodic x/y, CPML 12 on z, seeded random piecewise-constant eps '
                              'in [1,12.1] on 8^3 blocks, Ey dipole at the centre, FP32')
    if name == 'strip':
        L = 12
        b = Boundaries(**{f'{a}_{s}': baseline_face(L) for a in 'xyz' for s in ('min', 'max')})
        region = Region(dimension='3d', size=(8, 6, 2), mesh=.05, pml_cells=L, background_index=2.085**.5, steps=steps,
                        backend='cuda', cuda_kernel='fused', boundaries=b, run_control=control, snapshot_interval=10000)
        custom = SpectrumSettings(sampling='custom', custom_frequencies_hz=[C0 / (lam * 1e-6)], apodization='none')
        project = Project(name='Si strip 160x120x40', region=region, materials=[Material(name='Si', index=12.08**.5)],
                          structures=[Structure(id='strip', size=(8, .65, .4), material='Si')],
                          sources=[Source(id='dip', center=(-2.5, 0, 0), **src)],
                          monitors=[FieldMonitor(id='plane', normal='x', center=(2, 0, 0), size=(0, 4.8, .8), dft_precision='float64',
                                                 spectrum=custom)])
        return project, None, ('3D Yee+CPML 160x120x40 (0.05 um), CPML 12, Si strip 0.65x0.4 um in SiO2, Ey dipole, '
                               'x-normal DFT plane at 1.55 um, FP32')
    if name == 'graded':
        # A graded mesh (nonuniform x / y / z): fine 0.05 um lattice around a Si block, coarsened up to 0.15 um
        # (1.4 grading) between it and the PML; the march kernel's metric body.
        L = 12
        b = Boundaries(**{f'{a}_{s}': baseline_face(L) for a in 'xyz' for s in ('min', 'max')})
        region = Region(dimension='3d', size=(30.0, 30.0, 16.0), mesh=.05, pml_cells=L, steps=steps, backend='cuda',
                        cuda_kernel='fused', boundaries=b, run_control=control, snapshot_interval=10000, mesh_type='graded',
                        mesh_max=.15, mesh_grading=1.4, mesh_ppw=6, material_sampling='yee')
        project = Project(name='graded mesh', region=region, materials=[Material(name='Si', index=3.476)],
                          structures=[Structure(id='blk', size=(6, 6, 3), material='Si')],
                          sources=[Source(id='dip', center=(-2.0, 0, 0), **src)],
                          monitors=[Monitor(id='probe', center=(2.0, 0, 0), component='Ey')])
        return project, None, ('3D Yee+CPML on a graded mesh (30x30x16 um, 0.05 um lattice coarsened to 0.15 um at grading '
                               '1.4 outside a 6x6x3 um Si block), CPML 12, Yee sampling, Ey dipole, FP32')
    if name in ('tfsf', 'dispersive'):
        # 256^3 at 0.05 um, CPML 12: a TFSF box (plane wave along +x) around a Si sphere, or a Drude sphere and a
        # Lorentz slab lit by an Ey dipole; both run the split gather step.
        n, L = (256, 256, 256), 12
        b = Boundaries(**{f'{a}_{s}': baseline_face(L) for a in 'xyz' for s in ('min', 'max')})
        region = Region(dimension='3d', size=tuple(v * .05 for v in n), mesh=.05, pml_cells=L, steps=steps, backend='cuda',
                        cuda_kernel='fused', boundaries=b, run_control=control, snapshot_interval=10000)
        if name == 'tfsf':
            project = Project(name='TFSF 256^3', region=region, materials=[Material(name='Si', index=3.476)],
                              structures=[Structure(id='ball', kind='sphere', radius=2.0, material='Si')],
                              sources=[Source(id='box', kind='tfsf', normal='x', direction='+', size=(8, 8, 8), component='Ey',
                                              wavelength=lam, pulse='gaussian', time_definition='standard', pulse_length=20e-15,
                                              pulse_offset=40e-15)],
                              monitors=[Monitor(id='probe', center=(5.0, 0, 0), component='Ey')])
            return project, None, ('3D Yee+CPML 256^3 (0.05 um), CPML 12, an 8 um TFSF box (Ey plane wave along +x) around a '
                                   '2 um Si sphere, FP32')
        metal = Material(name='metal', model='drude', epsilon_inf=1.5, plasma_rad_s=9e15, collision_rad_s=1e14)
        glass = Material(name='disp', model='lorentz', epsilon_inf=2.0, resonance_rad_s=3e15, linewidth_rad_s=2e14, delta_epsilon=1.2)
        project = Project(name='dispersive 256^3', region=region, materials=[metal, glass],
                          structures=[Structure(id='ball', kind='sphere', center=(2.0, 0, 0), radius=1.5, material='metal'),
                                      Structure(id='slab', size=(1.0, 11.6, 11.6), center=(-2.0, 0, 0), material='disp')],
                          sources=[Source(id='dip', center=(-4.0, 0, 0), **src)],
                          monitors=[Monitor(id='probe', center=(4.5, 0, 0), component='Ey')])
        return project, None, ('3D Yee+CPML 256^3 (0.05 um), CPML 12, a 1.5 um Drude sphere and a 1 um Lorentz slab '
                               '(coupled trapezoidal ADE), Ey dipole, FP32')
    if name == 'tmz2d':
        # 2D TMz plain-method case: 16 x 12 um at 0.05 um (320 x 240 cells), CPML 16, Courant 0.99/sqrt(2).
        L = 16
        b = Boundaries(**{f'{a}_{s}': baseline_face(L) for a in 'xy' for s in ('min', 'max')})
        region = Region(dimension='2d', size=(16, 12, 1), mesh=.05, pml_cells=L, background_index=1.444, steps=steps,
                        backend='cuda', cuda_kernel='fused', boundaries=b, run_control=control, snapshot_interval=10000)
        custom = SpectrumSettings(sampling='custom', custom_frequencies_hz=[C0 / (lam * 1e-6)], apodization='none')
        pulse = dict(component='Ez', wavelength=lam, pulse='broadband', time_definition='wavelength',
                     wavelength_start=lam - .05, wavelength_stop=lam + .05)
        project = Project(name='TMz waveguide 320x240', region=region, materials=[Material(name='core', index=3.476)],
                          structures=[Structure(id='core', size=(16, .5, 1), material='core')],
                          sources=[Source(id='src', center=(-2.5, 0, 0), **pulse)],
                          monitors=[Monitor(id='probe', center=(2.5, 0, 0), component='Ez', spectrum=custom)])
        return project, None, ('2D TMz 320x240 (0.05 um), CPML 16, eps 1.444^2 background with a 0.5 um x-directed core '
                               'eps 3.476^2, Ez pulse at x=-2.5 um (1.50-1.60 um), Ez trace + DFT at 1.55 um, FP32')
    raise ValueError(name)


def batch_workload(steps, seed=2024, count=64, mesh=.05, layers=16):
    """64 independent 2D TMz grids, per-side cell counts drawn uniformly from 128 to 1024 (seeded), each with a
    2 x 2 um design region of seeded random binary density (Gaussian-filtered, sigma 2 cells, thresholded at
    0.5) mapping to eps in {2.085, 12.08} in an eps 2.085 background, CPML 16 cells, an Ez pulse 1.8 um left of
    the design and an Ez trace + DFT 1.8 um right of it. Returns (projects, epsilon arrays, description)."""
    from scipy.ndimage import gaussian_filter
    from torchfdtd_b200 import Boundaries, Monitor, Project, Region, Source, SpectrumSettings
    from torchfdtd_b200.models import RunControl
    rng = np.random.default_rng(seed)
    lam = 1.55
    sides = rng.integers(128, 1025, size=(count, 2))
    custom = SpectrumSettings(sampling='custom', custom_frequencies_hz=[C0 / (lam * 1e-6)], apodization='none')
    pulse = dict(component='Ez', wavelength=lam, pulse='broadband', time_definition='wavelength', wavelength_start=lam - .05,
                 wavelength_stop=lam + .05)
    projects, eps = [], []
    design = int(round(2.0 / mesh))
    for k, (nx, ny) in enumerate(sides):
        b = Boundaries(**{f'{a}_{s}': baseline_face(layers) for a in 'xy' for s in ('min', 'max')})
        region = Region(dimension='2d', size=(nx * mesh, ny * mesh, 1), mesh=mesh, pml_cells=layers,
                        background_index=2.085 ** .5, steps=steps, backend='cuda', cuda_kernel='fused', boundaries=b,
                        run_control=RunControl(divergence_check=False), snapshot_interval=10000)
        projects.append(Project(name=f'design {k}', region=region, sources=[Source(id='src', center=(-1.8, 0, 0), **pulse)],
                                monitors=[Monitor(id='probe', center=(1.8, 0, 0), component='Ez', spectrum=custom)]))
        rho = gaussian_filter(rng.integers(0, 2, size=(design, design)).astype(np.float64), 2.0) > .5
        e = np.full((int(nx), int(ny), 1), 2.085, dtype=np.float32)
        x0, y0 = int(nx) // 2 - design // 2, int(ny) // 2 - design // 2
        e[x0:x0 + design, y0:y0 + design, 0] = np.where(rho, 12.08, 2.085)
        eps.append(e)
    cells = int(sum(int(a) * int(b) for a, b in sides))
    return projects, eps, (f'{count} independent 2D TMz grids, sides uniform in [128, 1024] (seeded; {cells} cells in '
                           'all), 2x2 um seeded binary design region (Gaussian sigma 2 cells, threshold 0.5) eps in '
                           '{2.085, 12.08}, CPML 16, FP32, one persistent launch per step over all grids')


def measured_tensor_peak():
    path = ROOT / 'MEASURED_PEAKS.json'
    if path.exists():
        data = json.loads(path.read_text())
        return float(data.get('bf16_tflops', 1590.0)), 'measured (burst)'
    return 1590.0, 'fallback'


def measured_peaks():
    path = ROOT / 'MEASURED_PEAKS.json'
    if path.exists():
        data = json.loads(path.read_text())
        return float(data['hbm_gbs']), 'measured'
    return 6650.0, 'fallback'


class ClockSampler:
    """SM clock and throttle reasons through NVML every 20 ms while active."""
    REASONS = {0x4: 'sw_power_cap', 0x8: 'hw_slowdown', 0x20: 'sw_thermal_slowdown', 0x40: 'hw_thermal_slowdown',
               0x80: 'hw_power_brake_slowdown', 0x2: 'applications_clocks_setting', 0x1: 'gpu_idle'}

    def __init__(self, index):
        self.samples = []
        self.window = None
        self.ok = False
        try:
            import pynvml
            pynvml.nvmlInit()
            self.nvml = pynvml
            self.handle = pynvml.nvmlDeviceGetHandleByIndex(index)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self.handle, pynvml.NVML_CLOCK_SM)
            self.ok = True
        except Exception:  # noqa: BLE001 - no NVML: clocks are reported as unavailable
            self.max_mhz = None
        self.stop = threading.Event()
        self.thread = threading.Thread(target=self._run, daemon=True)

    def _run(self):
        while not self.stop.is_set():
            try:
                mhz = self.nvml.nvmlDeviceGetClockInfo(self.handle, self.nvml.NVML_CLOCK_SM)
                reasons = self.nvml.nvmlDeviceGetCurrentClocksEventReasons(self.handle)
                self.samples.append((time.time(), mhz, reasons))
            except Exception:  # noqa: BLE001
                pass
            time.sleep(0.02)

    def start(self):
        if self.ok:
            self.thread.start()

    def finish(self):
        self.stop.set()
        if self.ok:
            self.thread.join()
        if not self.samples:
            return {'sm_mhz': None, 'sm_max_mhz': self.max_mhz, 'reasons': [], 'samples': 0}
        lo, hi = self.window or (0, math.inf)
        inside = [s for s in self.samples if lo <= s[0] <= hi] or self.samples
        mask = 0
        for _, _, r in inside:
            mask |= r
        names = sorted({name for bit, name in self.REASONS.items() if mask & bit and name != 'gpu_idle'})
        return {'sm_mhz': float(np.median([s[1] for s in inside])), 'sm_max_mhz': self.max_mhz, 'reasons': names,
                'samples': len(inside)}


def cpu_rate(plan, budget_s=15.0, min_steps=2, max_steps=None, threads=None):
    """Gcell-updates/s of the C oracle on the same plan; steps run until the time budget is spent."""
    sys.path.insert(0, str(ROOT))
    from oracle.cpu import CpuOracle
    o = CpuOracle(plan, threads=threads)
    o.run(1)  # warm-up (first touch of the state)
    steps, t0 = 0, time.perf_counter()
    while True:
        o.run(1)
        steps += 1
        elapsed = time.perf_counter() - t0
        if (steps >= min_steps and elapsed >= budget_s) or (max_steps and steps >= max_steps):
            break
    return plan.cells * steps / elapsed / 1e9, steps, elapsed, o.threads


def dist_setup(args):
    world = int(os.environ.get('WORLD_SIZE', '1'))
    rank = int(os.environ.get('RANK', '0'))
    local = int(os.environ.get('LOCAL_RANK', '0'))
    if world > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta
        torch.cuda.set_device(local)
        dist.init_process_group('nccl', timeout=timedelta(seconds=600), device_id=torch.device('cuda', local))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(value, world):
    if world == 1:
        return value
    import torch
    import torch.distributed as dist
    t = torch.tensor([value], dtype=torch.float64, device='cuda')
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def run_reference(args, world, rank):
    from torchfdtd_b200.plan import plan_grid
    if rank != 0:
        return None
    project, eps, desc = workload(args.workload, max(10, args.steps))
    plan = plan_grid(project)
    if eps is not None:
        plan.epsilon, plan.inv_eps = eps, (1 / eps).astype(plan.dtype)
    # Each bench step is one full time step over the whole grid; the run is bounded to ~2 minutes.
    per_step_budget = 120.0 / max(1, args.steps + args.warmup)
    rate, steps, elapsed, threads = cpu_rate(plan, budget_s=per_step_budget * args.steps, min_steps=min(args.steps, 2),
                                             max_steps=args.steps)
    sample = (f'{steps} full time steps of the {plan.shape[0]}x{plan.shape[1]}x{plan.shape[2]} grid on {threads} host threads '
              f'(C port of the reference NumPy Yee/CPML update, bitwise equal to it), after 1 warm-up step')
    line = dict(metric=METRIC, value=rate, unit=METRIC, n_gpus=world, steps=args.steps, warmup=args.warmup,
                ms_per_step=elapsed / steps * 1e3, higher_is_better=True, scaling='weak', vs_baseline=None, dtype='f32',
                data='synthetic', impl='reference', parallelism='host threads',
                config=dict(workload=desc, cells=plan.cells, l2=L2_NOTE),
                cpu_baseline=dict(value=rate, unit=METRIC, cores=threads, kind='port', sample=sample),
                e2e=dict(value=rate, unit=METRIC, h2d_bytes_per_step=0, d2h_bytes_per_step=0))
    return line


def run_ours(args, world, rank, local):
    import torch
    from torchfdtd_b200 import Simulation
    from torchfdtd_b200.native import NativeGrid
    from torchfdtd_b200.plan import plan_grid
    from torchfdtd_b200.simulation import algorithmic_bytes_per_step
    device = torch.device('cuda', local)
    torch.cuda.set_device(device)
    total_steps = args.warmup + args.steps
    project, eps, desc = workload(args.workload, max(10, total_steps))
    plan = plan_grid(project)
    if eps is not None:
        plan.epsilon, plan.inv_eps = eps, (1 / eps).astype(plan.dtype)
    grid = NativeGrid(plan, kernel=args.kernel)
    stream = torch.cuda.Stream(device)
    sampler = ClockSampler(local)
    sampler.start()
    with torch.cuda.stream(stream):
        grid.step(args.warmup, stream)
        stream.synchronize()
        barrier(world)
        torch.cuda.synchronize()
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t_wall = time.time()
        start.record(stream)
        grid.step(args.steps, stream)
        end.record(stream)
        end.synchronize()
        t_wall_end = time.time()
    torch.cuda.synchronize()
    barrier(world)
    sampler.window = (t_wall, t_wall_end)
    clocks = sampler.finish()
    elapsed = max_over_ranks(start.elapsed_time(end) / 1e3, world)
    status = grid.device_status()
    kernel_used = grid.kernel
    launches = grid.step_launches(args.steps)
    grid.close()
    del grid
    torch.cuda.empty_cache()
    cells = plan.cells
    value = world * cells * args.steps / elapsed / 1e9
    bytes_step = algorithmic_bytes_per_step(plan)
    peak, peak_kind = measured_peaks()
    achieved = bytes_step * args.steps / elapsed / 1e9
    traffic = MEASURED_TRAFFIC_PER_CELL.get((args.workload, kernel_used))
    roofline = dict(bound='hbm', achieved=achieved, peak=peak, unit='GB/s', frac=achieved / peak,
                    traffic=None if traffic is None else traffic * cells, peak_source=peak_kind,
                    algorithmic_bytes_per_step=bytes_step, kernel=f'k_step_{kernel_used}',
                    note='achieved counts the whole step (fused step launch + observation launch)')
    # ---- end to end through the public API --------------------------------------------------
    e2e = None
    if not args.no_e2e:
        e2e_steps = max(10, args.steps)
        e2e_project, e2e_eps, _ = workload(args.workload, e2e_steps)
        barrier(world)
        t0 = time.perf_counter()
        result = Simulation(e2e_project, epsilon=e2e_eps).run(cuda_graph=True, cuda_graph_steps=16, kernel=args.kernel)
        e2e_s = max_over_ranks(time.perf_counter() - t0, world)
        real = np.dtype(plan.dtype).itemsize
        h2d = cells * plan.material_samples * real + sum(t.values.nbytes for t in plan.sources)
        d2h = result.electric.nbytes + result.magnetic.nbytes + result.signals.nbytes + result.frames.nbytes
        phases = dict(result.summary.get('phase_seconds', {}))
        phases['outside_phases'] = e2e_s - sum(phases.values())
        e2e = dict(value=world * cells * e2e_steps / e2e_s / 1e9, unit=METRIC, h2d_bytes_per_step=h2d / e2e_steps,
                   d2h_bytes_per_step=d2h / e2e_steps, seconds=e2e_s, steps=e2e_steps,
                   breakdown_s={k: round(v, 4) for k, v in phases.items()},
                   call='Simulation(project, epsilon).run(cuda_graph=True, cuda_graph_steps=16)')
    line = dict(metric=METRIC, value=value, unit=METRIC, n_gpus=world, steps=args.steps, warmup=args.warmup,
                ms_per_step=elapsed / args.steps * 1e3, higher_is_better=True, scaling='weak', vs_baseline=None, dtype='f32',
                data='synthetic (seeded)', config=dict(workload=desc, cells=cells, l2=L2_NOTE),
                parallelism=f'replicas x{world}' if world > 1 else 'single GPU', kernel=kernel_used,
                roofline=roofline, e2e=e2e, clocks=clocks, gpu_launches=launches, device_status=status)
    if args.workload == 'periodic':
        line['restated_reference'] = time_restated_marching(plan, args, device, bytes_step, peak)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        rate, steps, el, threads = cpu_rate(plan, budget_s=args.cpu_budget)
        line['cpu_baseline'] = dict(value=rate, unit=METRIC, cores=threads, kind='port',
                                    sample=f'{steps} full time steps of the same grid on {threads} host threads (C port of the '
                                           f'reference NumPy update), {el:.1f} s')
    return line if rank == 0 else None


def time_restated_marching(plan, args, device, bytes_step, peak):
    """The reference's one-pass marching kernel (FusedEHMarching, restated in baseline/fused_eh_marching.cu) on
    the same scene and device, timed like ours: CUDA events on its stream around the same K steps."""
    import torch
    from baseline.fused_eh_marching import RestatedMarching
    ref = RestatedMarching(plan, device=device)
    stream = torch.cuda.Stream(device)
    with torch.cuda.stream(stream):
        ref.step(args.warmup, stream)
        stream.synchronize()
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record(stream)
        ref.step(args.steps, stream)
        end.record(stream)
        end.synchronize()
    elapsed = start.elapsed_time(end) / 1e3
    a = ref.args
    out = dict(kernel='FusedEHMarching (reference torchfdtd/reversible_cuda_fused.py:259-326) restated in CUDA',
               value=plan.cells * args.steps / elapsed / 1e9, unit=METRIC, ms_per_step=elapsed / args.steps * 1e3,
               roofline_frac=bytes_step * args.steps / elapsed / 1e9 / peak,
               launch=dict(grid=[(a.ny + a.rows - 1) // a.rows, (a.nx + a.chunk - 1) // a.chunk], block=[a.zb, a.rows + 2]),
               note='same algorithmic bytes as ours for the fraction; the restated kernel also reads 3 inverse-permittivity '
                    'samples per cell (the reference layout), 8 B per cell more than ours')
    del ref
    torch.cuda.empty_cache()
    return out


def batch_cpu_rate(plans, budget_s, threads=None):
    """Cell-updates/s of the C oracle over a batch, one grid after another (as the reference's CPU path runs
    them), round-robin one step per grid until the budget is spent."""
    from oracle.cpu import CpuOracle
    oracles, cells, t0, k = {}, 0, None, 0
    while True:
        i = k % len(plans)
        if i not in oracles:
            oracles[i] = CpuOracle(plans[i], threads=threads)
            oracles[i].run(1)                      # first touch, untimed
        if t0 is None:
            t0 = time.perf_counter()
        oracles[i].run(1)
        cells += plans[i].cells
        k += 1
        elapsed = time.perf_counter() - t0
        if elapsed >= budget_s and k >= len(plans):
            break
        if elapsed >= budget_s * 2:
            break
    threads = next(iter(oracles.values())).threads
    return cells / elapsed / 1e9, k, elapsed, threads


def batch_plans(projects, eps):
    from torchfdtd_b200.simulation import Simulation
    return [Simulation(p, epsilon=e).plan for p, e in zip(projects, eps)]


def run_reference_batch(args, world, rank):
    if rank != 0:
        return None
    projects, eps, desc = batch_workload(max(10, args.steps))
    plans = batch_plans(projects, eps)
    budget = 120.0 * args.steps / max(1, args.steps + args.warmup)
    rate, steps, elapsed, threads = batch_cpu_rate(plans, budget)
    sample = (f'{steps} grid-steps (one time step of one grid each, round-robin over the {len(plans)} grids) on {threads} '
              f'host threads (C port of the reference NumPy Yee/CPML update), {elapsed:.1f} s')
    return dict(metric=METRIC, value=rate, unit=METRIC, n_gpus=world, steps=args.steps, warmup=args.warmup,
                ms_per_step=sum(p.cells for p in plans) / rate / 1e6, higher_is_better=True, scaling='weak',
                vs_baseline=None, dtype='f32', data='synthetic', impl='reference', parallelism='host threads',
                config=dict(workload=desc, cells=sum(p.cells for p in plans), l2=L2_NOTE),
                cpu_baseline=dict(value=rate, unit=METRIC, cores=threads, kind='port', sample=sample),
                e2e=dict(value=rate, unit=METRIC, h2d_bytes_per_step=0, d2h_bytes_per_step=0))


def run_ours_batch(args, world, rank, local):
    import torch
    from torchfdtd_b200.batch import run_tensor_batch
    from torchfdtd_b200.native import NativeBatch, NativeGrid
    from torchfdtd_b200.simulation import algorithmic_bytes_per_step
    from torchfdtd_b200.tuning import tune_tensor_batch
    device = torch.device('cuda', local)
    torch.cuda.set_device(device)
    total_steps = args.warmup + args.steps
    config_steps = 3000
    projects, eps, desc = batch_workload(max(config_steps, total_steps + 64))
    plans = batch_plans(projects, eps)
    cells = sum(p.cells for p in plans)
    if args.batch_launch:
        choice = [int(v) for v in args.batch_launch.split(',')]
        tuning = None
    else:
        tuning = tune_tensor_batch(projects, epsilon=eps, device=local)
        choice = tuning.choice
    grids = [NativeGrid(plan, kernel='tile2d') for plan in plans]
    batch = NativeBatch(grids)
    batch.set_launch(*choice[:2])
    batch.set_persistent(bool(choice[2]) if len(choice) > 2 else False)
    tiles = batch.tiles()
    stream = torch.cuda.Stream(device)
    sampler = ClockSampler(local)
    sampler.start()
    with torch.cuda.stream(stream):
        batch.step(args.warmup, stream)
        stream.synchronize()
        barrier(world)
        torch.cuda.synchronize()
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t_wall = time.time()
        start.record(stream)
        batch.step(args.steps, stream)
        end.record(stream)
        end.synchronize()
        t_wall_end = time.time()
    torch.cuda.synchronize()
    barrier(world)
    sampler.window = (t_wall, t_wall_end)
    clocks = sampler.finish()
    elapsed = max_over_ranks(start.elapsed_time(end) / 1e3, world)
    status = max(g.device_status() for g in grids)
    batch.close()
    for g in grids:
        g.close()
    del grids, batch
    torch.cuda.empty_cache()
    value = world * cells * args.steps / elapsed / 1e9
    bytes_step = sum(algorithmic_bytes_per_step(p) for p in plans)
    peak, peak_kind = measured_peaks()
    achieved = bytes_step * args.steps / elapsed / 1e9
    roofline = dict(bound='hbm', achieved=achieved, peak=peak, unit='GB/s', frac=achieved / peak,
                    traffic=(MEASURED_TRAFFIC_PER_CELL[('batch64', 'tile2d')] * cells
                             if ('batch64', 'tile2d') in MEASURED_TRAFFIC_PER_CELL else None), peak_source=peak_kind,
                    algorithmic_bytes_per_step=bytes_step, kernel='k_step2d_tm',
                    note='achieved counts the whole step (batched tile launch + batched observation launch)')
    # ---- end to end: the public batch call over the configured 3000 steps ------------------------------
    e2e = None
    if not args.no_e2e:
        e2e_projects, e2e_eps, _ = batch_workload(config_steps)
        barrier(world)
        t0 = time.perf_counter()
        report = run_tensor_batch(e2e_projects, epsilon=e2e_eps, cuda_graph=True, cuda_graph_steps=16, launch=choice)
        e2e_s = max_over_ranks(time.perf_counter() - t0, world)
        report.raise_for_errors()
        h2d = sum(p.cells * 4 + sum(t.values.nbytes for t in p.sources) for p in plans)
        d2h = sum(i.result.electric.nbytes + i.result.magnetic.nbytes + i.result.signals.nbytes + i.result.frames.nbytes
                  for i in report.items)
        e2e = dict(value=world * cells * config_steps / e2e_s / 1e9, unit=METRIC, h2d_bytes_per_step=h2d / config_steps,
                   d2h_bytes_per_step=d2h / config_steps, seconds=e2e_s, steps=config_steps,
                   loop_seconds=report.plan['loop_seconds'], setup_seconds=report.plan['setup_seconds'],
                   call='run_tensor_batch(projects, epsilon=eps, cuda_graph=True, cuda_graph_steps=16, launch=tuned)')
    line = dict(metric=METRIC, value=value, unit=METRIC, n_gpus=world, steps=args.steps, warmup=args.warmup,
                ms_per_step=elapsed / args.steps * 1e3, higher_is_better=True, scaling='weak', vs_baseline=None, dtype='f32',
                data='synthetic (seeded)',
                config=dict(workload=desc, cells=cells, l2=L2_NOTE),
                grids=len(plans), strips=tiles, launch=choice,
                tuning=[(r['ctas'], r['rows'], r.get('persistent', 0), r['strips'], round(r['median_ms_per_step'], 5))
                        for r in tuning.candidates] if tuning else 'fixed by --batch-launch',
                parallelism=f'replicas x{world}' if world > 1 else 'single GPU', kernel='tile2d',
                roofline=roofline, e2e=e2e, clocks=clocks,
                gpu_launches=1 if len(choice) > 2 and choice[2] else 2 * args.steps, device_status=status)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        rate, steps, el, threads = batch_cpu_rate(plans, args.cpu_budget)
        line['cpu_baseline'] = dict(value=rate, unit=METRIC, cores=threads, kind='port',
                                    sample=f'{steps} grid-steps round-robin over the {len(plans)} grids on {threads} host '
                                           f'threads (C port of the reference NumPy update), {el:.1f} s')
    return line if rank == 0 else None


def adjoint_workload(steps, precision='float32', seed=2024):
    """3D discrete-adjoint design scene: 200 x 200 x 80 cells at 0.04 um (8 x 8 x 3.2 um), CPML 12, SiO2
    background (eps 2.085) with a 2 x 2 x 0.22 um design region of density rho (seeded uniform noise,
    Gaussian-smoothed with sigma 2 cells, sigmoid projection beta 8 about 0.5), eps = 2.085 + rho (12.08 -
    2.085); an Ey dipole 2.5 um before the design and an x-normal DFT plane 2.5 um after it at 1.55 um.
    Returns (project, design index box, rho parameters as a numpy array)."""
    from scipy.ndimage import gaussian_filter
    from torchfdtd_b200 import Boundaries, FieldMonitor, Project, Region, Source, SpectrumSettings
    from torchfdtd_b200.models import RunControl
    lam, mesh, L = 1.55, .04, 12
    b = Boundaries(**{f'{a}_{s}': baseline_face(L) for a in 'xyz' for s in ('min', 'max')})
    region = Region(dimension='3d', size=(8, 8, 3.2), mesh=mesh, pml_cells=L, background_index=2.085 ** .5, steps=steps,
                    precision=precision, backend='cuda', cuda_kernel='fused', boundaries=b,
                    run_control=RunControl(divergence_check=False), snapshot_interval=10000)
    custom = SpectrumSettings(sampling='custom', custom_frequencies_hz=[C0 / (lam * 1e-6)], apodization='none')
    src = dict(component='Ey', wavelength=lam, pulse='gaussian', time_definition='standard', pulse_length=20e-15,
               pulse_offset=40e-15)
    project = Project(name='adjoint design 200x200x80', region=region, sources=[Source(id='dip', center=(-2.5, 0, 0), **src)],
                      monitors=[FieldMonitor(id='out', normal='x', center=(2.5, 0, 0), size=(0, 2.4, 1.2), spectrum=custom)])
    n = (200, 200, 80)
    dn = (int(round(2 / mesh)), int(round(2 / mesh)), int(round(.22 / mesh)))
    lo = tuple((a - d) // 2 for a, d in zip(n, dn))
    rng = np.random.default_rng(seed)
    raw = gaussian_filter(rng.uniform(0, 1, size=dn), 2.0)
    raw = (raw - raw.mean()) / max(raw.std(), 1e-12) * .15 + .5
    return project, (lo, dn), raw


def run_ours_adjoint(args, world, rank, local, precisions=('float32', 'float64')):
    """Gradient of |mode overlap|^2 of the output-plane Ey at 1.55 um with respect to the design density
    through the discrete adjoint, timed; then central differences on 16 seeded design voxels (float64)."""
    import torch
    from torchfdtd_b200.adjoint import AdjointOptions, DifferentiablePlaneSimulation
    torch.cuda.set_device(local)
    steps = 4000
    results = {}
    for precision in precisions:
        project, (lo, dn), raw = adjoint_workload(steps, precision)
        dtype = torch.float32 if precision == 'float32' else torch.float64
        model = DifferentiablePlaneSimulation(project, AdjointOptions())
        shape = model.plan.shape
        base = torch.full(shape, 2.085, dtype=dtype, device='cuda')
        sl = tuple(slice(a, a + d) for a, d in zip(lo, dn))
        theta = torch.tensor(raw, dtype=dtype, device='cuda', requires_grad=True)

        def objective(param):
            rho = torch.sigmoid(8 * (param - .5))
            eps = base.clone()
            eps[sl] = 2.085 + rho * (12.08 - 2.085)
            ey = model(eps)['out'].fields[..., 1]
            _, ny, nz = model._maps[0][0].plan['shape']
            y = torch.linspace(-1, 1, ny, device='cuda', dtype=torch.float64)[:, None]
            z = torch.linspace(-1, 1, nz, device='cuda', dtype=torch.float64)[None, :]
            mode = torch.exp(-(y / .5) ** 2 - (z / .5) ** 2).reshape(-1).to(ey.dtype)
            return (torch.abs((ey * mode.conj()).sum(dim=1)) ** 2).sum()
        for _ in range(1):                              # warm-up: plans, kernels, snapshot buffers
            objective(theta).backward()
        theta.grad = None
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        value = objective(theta)
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        value.backward()
        torch.cuda.synchronize()
        t2 = time.perf_counter()
        report = model.engine(base).report
        cells = int(np.prod(shape))
        entry = dict(objective=float(value.detach()), forward_s=t1 - t0, backward_s=t2 - t1, gradient_s=t2 - t0,
                     forward_gcells=cells * steps / (t1 - t0) / 1e9, checkpoints=report['checkpoints'],
                     segment_steps=report['segment_steps'], replayed_steps=report['replayed_steps'],
                     checkpoint_gb=report['checkpoint_bytes'] / 1e9, restart_mb=report['restart_bytes'] / 1e6)
        if precision == 'float64':
            grad = theta.grad.detach().cpu().numpy()
            rng = np.random.default_rng(16)
            picks = [tuple(int(rng.integers(0, d)) for d in dn) for _ in range(16)]
            h, errors = 1e-4, []
            with torch.no_grad():
                for idx in picks:
                    up, down = theta.detach().clone(), theta.detach().clone()
                    up[idx] += h
                    down[idx] -= h
                    fd = float(objective(up) - objective(down)) / (2 * h)
                    errors.append(abs(grad[idx] - fd) / max(abs(fd), 1e-3 * np.abs(grad).max()))
            entry.update(fd_voxels=16, fd_step=h, fd_max_rel_err=float(max(errors)), fd_median_rel_err=float(np.median(errors)))
        results[precision] = entry
        model.close()
    f32 = results['float32']
    cells = 200 * 200 * 80
    return dict(metric='adjoint gradient wall time', value=f32['gradient_s'], unit='s', n_gpus=world, steps=steps, warmup=1,
                ms_per_step=f32['gradient_s'] / steps * 1e3, higher_is_better=False, scaling='weak', vs_baseline=None,
                dtype='f32', data='synthetic (seeded)',
                config=dict(workload='3D discrete adjoint 200x200x80 at 0.04 um, 2x2x0.22 um design (sigmoid beta 8), '
                                     '|mode overlap of DFT Ey at 1.55 um|^2, 4000 steps, sqrt(T) checkpoints', cells=cells),
                adjoint=results)


def run_ours_surrogate(args, world, rank, local):
    """Learned surrogate configuration: 4096 density->spectrum pairs from the batched engine (400 x 400 TMz,
    100 x 100 design pixels at 0.02 um, 16 wavelengths 1.50-1.60 um), training of the 8-layer 64-channel
    network by the engine's BF16 kernels, then the plain adjoint loop against the surrogate-assisted loop to
    the plain loop's FOM (within 1 %, verified by FDTD)."""
    import torch
    from torchfdtd_b200.design import TransmissionProblem, adjoint_design, generate_dataset, surrogate_design
    from torchfdtd_b200.surrogate import ConvNeuralOperator
    torch.cuda.set_device(local)
    problem = TransmissionProblem()
    rhos, targets, gen_s = generate_dataset(problem, count=4096, seed=0)
    rho_t, y_t = torch.tensor(rhos, device='cuda'), torch.tensor(targets, device='cuda')
    train, val = slice(0, 3840), slice(3840, 4096)
    # The scene is mirror-symmetric about y = 0: a density flipped along y has the same transmission.
    rho_aug = torch.cat([rho_t[train], torch.flip(rho_t[train], dims=[2])])
    y_aug = torch.cat([y_t[train], y_t[train]])
    net = ConvNeuralOperator(outputs=32, seed=0)
    epochs = args.surrogate_epochs
    net.fit(rho_t[:64], y_t[:64], epochs=1, batch=64)            # warm-up: kernels, buffers
    net = ConvNeuralOperator(outputs=32, seed=0)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    history = net.fit(rho_aug, y_aug, epochs=epochs, batch=64, lr=2e-3)
    torch.cuda.synchronize()
    train_s = time.perf_counter() - t0
    pred = net.predict(rho_t[val])
    mse = float(((pred - y_t[val]) ** 2).mean())
    baseline = float(((y_t[val] - y_t[train].mean(dim=0)) ** 2).mean())
    flops = 3 * net.flops_per_sample * rho_aug.shape[0] * epochs
    # inference throughput on a batch of 256, on the tcgen05 kernels and on the mma.sync kernels
    from torchfdtd_b200.surrogate import device_status, set_tensor_path
    infer = {}
    for path in ('mma', 'tcgen05'):
        set_tensor_path(path)
        net.forward(rho_t[:256])
        torch.cuda.synchronize()
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record()
        for _ in range(20):
            net.forward(rho_t[:256])
        end.record()
        end.synchronize()
        infer[path] = start.elapsed_time(end) / 20 / 1e3
    set_tensor_path('tcgen05')
    infer_s = infer['tcgen05']
    peak_tf = measured_tensor_peak()
    # design loops
    iterations = args.design_iterations
    plain, theta = adjoint_design(problem, iterations=iterations, lr=.2)
    target = plain[-1][1]
    plain_time = plain[-1][0]
    reach = next((t for t, f in plain if f >= .99 * target), plain_time)
    hist, best, _ = surrogate_design(problem, net, target_fom=.99 * target, iterations=50 * iterations, lr=.2, verify_every=5,
                                     finetune_steps=10, data=(rho_aug, y_aug), max_seconds=2 * plain_time)
    sur_time = hist[-1][0] if hist else float('nan')
    reached = best >= .99 * target
    fallbacks = sum(1 for _, _, src in hist if src != 'surrogate')
    surrogate_phase = max((t for t, _, src in hist if src == 'surrogate'), default=0.0)
    surrogate_best = max((f for _, f, src in hist if src == 'surrogate'), default=float('nan'))
    result = dict(metric='surrogate-assisted design time to the plain adjoint FOM', value=sur_time, unit='s', n_gpus=world,
                  steps=problem.steps, warmup=1, ms_per_step=None, higher_is_better=False, scaling='weak', vs_baseline=None,
                  dtype='bf16', data='synthetic (seeded)',
                  config=dict(workload='learned surrogate: 400x400 2D TMz at 0.02 um, 100x100 design pixels, 4096 batched-engine '
                                       'samples, 16 wavelengths 1.50-1.60 um, 8-layer 64-channel CNO (BF16, FP32 accumulate)',
                              samples=4096, train='3840 (+ y-mirrored copies)', validation=256, epochs=epochs,
                              design_iterations=iterations),
                  dataset=dict(seconds=gen_s, cell_updates=4096 * problem.cells ** 2 * problem.steps,
                               gcells_per_s=4096 * problem.cells ** 2 * problem.steps / gen_s / 1e9),
                  training=dict(seconds=train_s, tflops=flops / train_s / 1e12, loss_first=history[0], loss_last=history[-1],
                                validation_mse=mse, mean_predictor_mse=baseline, r2=1 - mse / baseline,
                                inference_ms_per_256=infer_s * 1e3, inference_ms_per_256_mma_sync=infer['mma'] * 1e3,
                                status=device_status()),
                  roofline=dict(bound='tensor', achieved=256 * net.flops_per_sample / infer_s / 1e12, peak=peak_tf[0],
                                unit='TFLOP/s', frac=256 * net.flops_per_sample / infer_s / 1e12 / peak_tf[0],
                                peak_source=peak_tf[1], traffic=None,
                                note='conv-layer FLOPs of a 256-sample inference pass (8 layers; head, packing included in time)'),
                  design=dict(plain_fom=target, plain_seconds=plain_time, plain_seconds_to_99pct=reach,
                              surrogate_best_fom=best, surrogate_seconds=sur_time, reached=reached,
                              speedup_vs_plain=plain_time / sur_time if reached else None,
                              verifications=len(hist), adjoint_fallbacks=fallbacks, surrogate_phase_seconds=surrogate_phase,
                              surrogate_phase_best_fom=surrogate_best))
    return result


def run_adjoint_probe(args, world, rank, local):
    """Profiling case of the discrete adjoint: one gradient (no warm-up) of a small 3D scene (--probe-cells per side in
    x and y, half that in z, 0.05 um, CPML 8, an Ey dipole and an Ey point monitor, --steps steps), timed on the host."""
    import torch
    from torchfdtd_b200 import Monitor, Project, Region, Source
    from torchfdtd_b200.adjoint import DifferentiableSimulation
    torch.cuda.set_device(local)
    n, steps = args.probe_cells, args.steps
    region = Region(dimension='3d', size=(n * .05, n * .05, n * .025), mesh=.05, pml_cells=8, steps=steps, backend='cuda')
    project = Project(region=region, sources=[Source(center=(-.5, 0, 0), component='Ey', pulse_cycles=1, wavelength=1.0)],
                      monitors=[Monitor(center=(.5, 0, 0), component='Ey')])
    model = DifferentiableSimulation(project)
    eps = torch.full(tuple(region.shape), 2.0, device='cuda', requires_grad=True)
    torch.cuda.synchronize()
    t0 = time.perf_counter()                                # one cold gradient: the launch list of a profiler capture
    (model(eps).signals ** 2).sum().backward()
    torch.cuda.synchronize()
    seconds = time.perf_counter() - t0
    report = {k: v for k, v in model.engine(eps).report.items() if isinstance(v, (int, float, str))}
    cells = int(np.prod(region.shape))
    return dict(metric='adjoint gradient wall time', value=seconds, unit='s', n_gpus=world, steps=steps, warmup=1,
                ms_per_step=seconds / steps * 1e3, higher_is_better=False, scaling='weak', vs_baseline=None, dtype='f32',
                data='synthetic', config=dict(workload=f'3D adjoint probe {region.shape}, CPML 8, Ey dipole', cells=cells,
                                              l2=L2_NOTE), report=report)


def run_surrogate_kernels(args, world, rank, local):
    """Profiling case of the surrogate's kernels: forward and forward+backward passes of the 8-layer network on
    --probe-batch random densities, --steps passes, on the tcgen05 and on the mma.sync kernels."""
    import torch
    from torchfdtd_b200.surrogate import ConvNeuralOperator, device_status, set_tensor_path
    torch.cuda.set_device(local)
    batch, passes = args.probe_batch, args.steps
    net = ConvNeuralOperator(outputs=32, seed=0)
    rho = torch.rand((batch, 100, 100), device='cuda', generator=torch.Generator(device='cuda').manual_seed(0))
    target = torch.zeros((batch, 32), device='cuda')
    result = {}
    for path in ('tcgen05', 'mma'):
        set_tensor_path(path)
        net.forward(rho)
        torch.cuda.synchronize()
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record()
        for _ in range(passes):
            net.forward(rho)
        end.record()
        end.synchronize()
        fwd = start.elapsed_time(end) / passes
        start.record()
        for _ in range(passes):
            net.forward(rho)
            net.loss(target)
            net.backward(net._buffers[net._last]['dout'])
        end.record()
        end.synchronize()
        result[path] = dict(forward_ms=fwd, conv_tflops=batch * net.flops_per_sample / fwd / 1e9,
                            forward_backward_ms=start.elapsed_time(end) / passes)
    set_tensor_path('tcgen05')
    return dict(metric='surrogate forward time', value=result['tcgen05']['forward_ms'], unit='ms', n_gpus=world, steps=passes,
                warmup=1, ms_per_step=result['tcgen05']['forward_ms'], higher_is_better=False, scaling='weak', vs_baseline=None,
                dtype='bf16', data='synthetic', config=dict(workload=f'surrogate kernels, batch {batch} of 100x100 densities',
                                                            cells=batch * 100 * 100, l2=L2_NOTE),
                paths=result, device_status=device_status())


def device_rate(project, eps, steps, warmup, device, kernel='auto'):
    """Device-timed stepping of one workload through NativeGrid (CUDA events on the launching stream)."""
    import torch
    from torchfdtd_b200.native import NativeGrid
    from torchfdtd_b200.plan import plan_grid
    from torchfdtd_b200.simulation import algorithmic_bytes_per_step
    plan = plan_grid(project)
    if eps is not None:
        plan.epsilon, plan.inv_eps = eps, (1 / eps).astype(plan.dtype)
    grid = NativeGrid(plan, kernel=kernel)
    stream = torch.cuda.Stream(device)
    with torch.cuda.stream(stream):
        grid.step(warmup, stream)
        stream.synchronize()
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record(stream)
        grid.step(steps, stream)
        end.record(stream)
        end.synchronize()
    elapsed = start.elapsed_time(end) / 1e3
    out = dict(value=plan.cells * steps / elapsed / 1e9, unit=METRIC, ms_per_step=elapsed / steps * 1e3, steps=steps,
               kernel=grid.kernel, roofline_frac=algorithmic_bytes_per_step(plan) * steps / elapsed / 1e9 / measured_peaks()[0],
               device_status=grid.device_status(), gpu_launches=grid.step_launches(steps))
    grid.close()
    del grid
    torch.cuda.empty_cache()
    return plan, out


def extra_workloads(args, local):
    """The other benchmark configurations, device-timed in the same process (compact records; a failure is
    recorded, not raised): the periodic scene with the reference's marching kernel restated beside ours, the 2D
    TMz and Si-strip configurations at their own step counts, the 64-grid batch and the 3D adjoint gradient."""
    import copy
    import torch
    device = torch.device('cuda', local)
    extras = {}

    def attempt(name, fn):
        t0 = time.perf_counter()
        try:
            extras[name] = fn()
        except Exception as exc:  # noqa: BLE001 - one failed extra must not void the headline line
            extras[name] = dict(error=f'{type(exc).__name__}: {exc}')
        extras[name]['wall_s'] = round(time.perf_counter() - t0, 2)
        torch.cuda.empty_cache()

    def periodic():
        project, eps, desc = workload('periodic', args.warmup + args.steps)
        plan, ours = device_rate(project, eps, args.steps, args.warmup, device)
        from torchfdtd_b200.simulation import algorithmic_bytes_per_step
        ref = time_restated_marching(plan, args, device, algorithmic_bytes_per_step(plan), measured_peaks()[0])
        return dict(workload=desc, ours=ours, restated_reference=ref, speedup=ref['ms_per_step'] and ref['ms_per_step'] / ours['ms_per_step'])

    def fixed(name, steps, warmup):
        def run():
            project, eps, desc = workload(name, warmup + steps)
            _, out = device_rate(project, eps, steps, warmup, device)
            return dict(workload=desc, **out)
        return run

    def batch():
        a = copy.copy(args)
        a.no_e2e, a.no_cpu_baseline = True, True
        line = run_ours_batch(a, 1, 0, local)
        return dict(workload=line['config']['workload'], value=line['value'], unit=METRIC, ms_per_step=line['ms_per_step'],
                    roofline_frac=line['roofline']['frac'], launch=line['launch'], device_status=line['device_status'])

    def adjoint():
        line = run_ours_adjoint(args, 1, 0, local, precisions=('float32',))
        f32 = line['adjoint']['float32']
        return dict(workload=line['config']['workload'], gradient_s=f32['gradient_s'], forward_s=f32['forward_s'],
                    backward_s=f32['backward_s'], replayed_steps=f32['replayed_steps'], checkpoints=f32['checkpoints'])

    attempt('periodic', periodic)
    attempt('tmz2d', fixed('tmz2d', 2000, 100))
    attempt('strip', fixed('strip', 1000, 50))
    attempt('batch64', batch)
    attempt('adjoint3d', adjoint)
    for name in ('graded', 'tfsf', 'dispersive'):
        attempt(name, fixed(name, 100, 5))
    return extras


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--gpus', type=int, default=1)
    ap.add_argument('--steps', type=int, default=200)
    ap.add_argument('--warmup', type=int, default=10)
    ap.add_argument('--impl', choices=['ours', 'reference'], default='ours')
    ap.add_argument('--workload', choices=['roofline', 'roofline256', 'strip', 'periodic', 'tmz2d', 'batch64', 'adjoint3d', 'surrogate',
                                           'adjoint_probe', 'surrogate_kernels', 'graded', 'tfsf', 'dispersive'],
                    default='roofline')
    ap.add_argument('--probe-cells', type=int, default=128, help='adjoint_probe: cells per side in x and y')
    ap.add_argument('--probe-batch', type=int, default=256, help='surrogate_kernels: densities per pass')
    ap.add_argument('--surrogate-epochs', type=int, default=30)
    ap.add_argument('--design-iterations', type=int, default=30)
    ap.add_argument('--kernel', choices=['auto', 'march', 'gather', 'tile2d'], default='auto')
    ap.add_argument('--cpu-budget', type=float, default=15.0)
    ap.add_argument('--no-cpu-baseline', action='store_true')
    ap.add_argument('--no-e2e', action='store_true', help='skip the end-to-end leg (profiling runs)')
    ap.add_argument('--batch-launch', default=None, help='batch64: fixed "ctas,rows" instead of the autotuner')
    ap.add_argument('--no-extras', action='store_true',
                    help='roofline workload: skip the device-timed records of the other configurations')
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
    if args.impl == 'reference':
        # Rank 0 alone times the host-core reference; other ranks exit without work.
        world, rank, local = int(os.environ.get('WORLD_SIZE', '1')), int(os.environ.get('RANK', '0')), 0
        line = (run_reference_batch if args.workload == 'batch64' else run_reference)(args, world, rank)
        if line is not None:
            print(json.dumps(line), flush=True)
        return
    world, rank, local = dist_setup(args)
    try:
        runner = {'batch64': run_ours_batch, 'adjoint3d': run_ours_adjoint, 'surrogate': run_ours_surrogate,
                  'adjoint_probe': run_adjoint_probe, 'surrogate_kernels': run_surrogate_kernels}.get(args.workload, run_ours)
        line = runner(args, world, rank, local)
        if line is not None and args.workload == 'roofline' and world == 1 and not args.no_extras:
            line['extra_workloads'] = extra_workloads(args, local)
        if rank == 0 and line is not None:
            print(json.dumps(line), flush=True)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == '__main__':
    main()

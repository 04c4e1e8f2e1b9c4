"""``Simulation(project).run() -> Result`` on the fused B200 kernels.

Mirrors reference ``torchfdtd/solver.py``: ``Simulation`` :642-908 (run loop,
graph capture, observation barriers, diagnostics, frames, summary) and
``Result`` :511-639 (fields, traces, spectra, DFT planes, NPZ layout that
round-trips through ``Result.load``). The selector is
``Region(backend="cuda", cuda_kernel="fused")``; 'auto' resolves to the same
kernels. Any other choice, and every scene feature outside the fused
nondispersive path, is refused with a ``ValueError`` that names it.
"""
from __future__ import annotations

import hashlib
import json
import math
import threading
import time
from dataclasses import dataclass, field
from functools import cached_property
from pathlib import Path

import numpy as np

from .models import Project
from .plan import field_axes, index_at, plan_grid
from .run_control import DecayDecision, observation_schedule, source_end_time, validate_graph_steps
from .spectra import point_spectrum

C0 = 299792458.0
ENGINE_LOCK = threading.Lock()
ENGINE = 'TorchFDTD-B200 fused Yee/CPML (sm_100a)'


def algorithmic_bytes_per_step(plan):
    """Compulsory HBM bytes of one step: each advanced field component read and written once,
    each stored permittivity sample read once, each CPML memory and each dispersive pole state (P, Q) read and
    written once."""
    real = np.dtype(plan.dtype).itemsize
    comps = len(plan.active_components())
    samples = plan.material_samples if plan.dimension == '3d' else 1
    psi = sum(int(np.prod(s)) for (f, a, c, side), s in plan.psi_shapes() if _psi_active(plan, f, a, c))
    # Dispersive samples: P and Q of every pole read and written once.
    ade = sum(2 * st.poles * st.samples for st in getattr(plan, 'ade', []))
    return plan.cells * (2 * real * comps + real * samples) + 2 * real * psi + 2 * real * ade


def _psi_active(plan, forward, axis, comp):
    """Whether the curl term (axis, input comp) of a family writes an advanced component."""
    out = {(0, 2): 1, (0, 1): 2, (1, 2): 0, (1, 0): 2, (2, 1): 0, (2, 0): 1}[(axis, comp)]
    name = ('H' if forward else 'E') + 'xyz'[out]
    return name in plan.active_components()


def plane_result(monitor, plan, frequency, components, values, dimension):
    """Plane record from accumulated (frequency, point, component) DFT values
    (reference torchfdtd/field_monitors.py:167-183)."""
    values = np.asarray(values).astype(np.complex128)
    by_component = {c: values[..., i] for i, c in enumerate(components)}
    density = {}
    for axis in set(monitor.record_poynting) | ({monitor.normal} if monitor.record_flux else set()):
        i = 'xyz'.index(axis)
        b, c = 'xyz'[(i + 1) % 3], 'xyz'[(i + 2) % 3]
        density[axis] = .5 * np.real(by_component['E' + b] * by_component['H' + c].conj()
                                     - by_component['E' + c] * by_component['H' + b].conj())
    flux = density[monitor.normal] @ plan['weights'] if monitor.record_flux else None
    fields = values[..., [components.index(c) for c in monitor.record_fields]]
    poynting = (np.stack([density[c] for c in monitor.record_poynting], axis=-1) if monitor.record_poynting
                else np.empty((*values.shape[:2], 0)))
    return dict(id=monitor.id, name=monitor.name, frequency_hz=frequency, fields=fields, poynting=poynting, flux=flux, **plan,
                components=list(monitor.record_fields), poynting_components=list(monitor.record_poynting),
                accumulated_components=list(components), time_downsample=monitor.time_downsample,
                settings=monitor.model_dump(),
                flux_units='reduced E*H * s^2 * ' + ('m per invariant length' if dimension == '2d' else 'm^2'),
                field_units='reduced field * s', normal_axis=monitor.normal)


def run_signature(project, steps):
    r = project.region
    config = dict(region=r.model_dump(exclude={'backend', 'cuda_kernel', 'cuda_monitor_kernel', 'execution_mode', 'tiling',
                                               'resident_cell_limit', 'field', 'slice_axis', 'slice_position',
                                               'complex_display', 'snapshot_interval'}),
                  sources=[project.resolved_source(s).model_dump() for s in project.sources], steps=steps,
                  nodes=[a.tolist() for a in r.mesh_nodes])
    return hashlib.sha256(json.dumps(config, sort_keys=True).encode()).hexdigest()


@dataclass
class Result:
    project: Project
    summary: dict
    frames: np.ndarray
    frame_steps: np.ndarray
    epsilon: np.ndarray
    signals: np.ndarray
    times: np.ndarray
    electric: np.ndarray
    magnetic: np.ndarray
    frequency_fields: list = field(default_factory=list)
    endpoint_fields: dict | None = None

    @property
    def point_monitors(self):
        return [self.project.resolved_monitor(m) for m in self.project.monitors if m.enabled and m.kind == 'point']

    @cached_property
    def spectra(self):
        # H is sampled half a step after E.
        dt = self.times[1] - self.times[0] if len(self.times) > 1 else 0
        return [point_spectrum((self.times + (dt / 2 if m.component.startswith('H') else 0))[::m.time_downsample],
                               self.signals[::m.time_downsample, k], m.spectrum)
                for k, m in enumerate(self.point_monitors)]

    def save(self, path, format=None):
        """NPZ layout of the reference ``Result.save`` (torchfdtd/solver.py:536-564). The reference's chunked HDF5
        layout (``format='hdf5'`` or a .h5 / .hdf5 path, torchfdtd/result_store.py) needs h5py and is refused."""
        path = Path(path)
        _refuse_hdf5(path, format)
        path.parent.mkdir(parents=True, exist_ok=True)
        spectral_arrays, metadata, plane_metadata = {}, [], []
        for k, (m, spec) in enumerate(zip(self.point_monitors, self.spectra)):
            spectral_arrays[f'monitor_{k}_frequency_hz'] = spec['frequency_hz']
            spectral_arrays[f'monitor_{k}_spectrum'] = spec['value']
            metadata.append({'id': m.id, 'name': m.name, 'component': m.component, 'settings': m.spectrum.model_dump(),
                             'units': spec['units'], 'transform': spec['transform']})
        for k, result in enumerate(self.frequency_fields):
            plane_metadata.append({key: v for key, v in result.items() if not isinstance(v, np.ndarray)})
            for key, v in result.items():
                if isinstance(v, np.ndarray):
                    spectral_arrays[f'field_monitor_{k}_{key}'] = v
        if self.endpoint_fields is not None:
            spectral_arrays.update({'endpoint_' + key: value for key, value in self.endpoint_fields.items()})
        np.savez_compressed(path, project=self.project.model_dump_json(), summary=json.dumps(self.summary, default=str),
                            field_monitors=json.dumps(plane_metadata, default=str),
                            **{f'mesh_{a}_um': nodes for a, nodes in zip('xyz', self.project.region.mesh_nodes)},
                            frames=self.frames, frame_steps=self.frame_steps, epsilon=self.epsilon, signals=self.signals,
                            times=self.times, E=self.electric, H=self.magnetic, monitor_spectra=json.dumps(metadata),
                            **spectral_arrays)

    @classmethod
    def load(cls, path):
        """Read the NPZ layout (a reference-written file included; reference torchfdtd/solver.py:603-618)."""
        _refuse_hdf5(Path(path), None)
        with np.load(path, allow_pickle=False) as data:
            planes = json.loads(str(data['field_monitors'])) if 'field_monitors' in data else []
            for k, plane in enumerate(planes):
                prefix = f'field_monitor_{k}_'
                plane.update({key[len(prefix):]: data[key].copy() for key in data.files if key.startswith(prefix)})
            endpoint = ({key: data['endpoint_' + key].copy() for key in ('E_upper', 'H_upper')}
                        if 'endpoint_E_upper' in data.files else None)
            return cls(Project.model_validate_json(str(data['project'])), json.loads(str(data['summary'])),
                       *(data[key].copy() for key in ('frames', 'frame_steps', 'epsilon', 'signals', 'times', 'E', 'H')),
                       planes, endpoint)

    def field_monitor(self, name_or_id):
        matches = [m for m in self.frequency_fields if name_or_id in (m['id'], m['name'])]
        if len(matches) != 1:
            raise ValueError('Expected one enabled frequency plane with this name or id.')
        return matches[0]

    def flux_data(self):
        return [dict(id=m['id'], name=m['name'], normal=m['normal_axis'], frequency_thz=(m['frequency_hz'] * 1e-12).tolist(),
                     wavelength_um=(C0 / m['frequency_hz'] * 1e6).tolist(), flux=m['flux'].tolist(), units=m['flux_units'],
                     points=len(m['weights']), shape=m['shape'], settings=m['settings'])
                for m in self.frequency_fields if m['flux'] is not None]


def _refuse_hdf5(path, format):
    if format == 'hdf5' or (format is None and path.suffix.lower() in ('.h5', '.hdf5')):
        raise ValueError('The HDF5 result layout needs h5py, which this engine does not use; save and load results as NPZ.')
    if format not in (None, 'npz', 'hdf5'):
        raise ValueError(f'Unknown result format {format!r}; use "npz".')


def snapshot_frames(project):
    """Frame cadence against the shortest enabled source wavelength: a frame every max(snapshot_interval,
    ceil(steps / 100)) steps; fewer than four frames per optical period alias the carrier in playback."""
    r = project.region
    interval = max(r.snapshot_interval, math.ceil(r.steps / 100))
    lengths = [s.wavelength_start if s.time_definition in ('wavelength', 'frequency') else s.wavelength
               for s in map(project.resolved_source, project.sources) if s.enabled]
    shortest = min(lengths) if lengths else None
    period = shortest * 1e-6 / C0 / r.time_step if shortest else None
    per_period = period / interval if period else None
    return dict(interval=r.snapshot_interval, effective_interval=interval, frames=r.steps // interval,
                shortest_wavelength_um=shortest, period_steps=period, frames_per_period=per_period,
                aliased=bool(per_period is not None and per_period < 4))


def run_estimates(project, plan, arena_bytes):
    """The scene and memory keys of the reference's run summary (torchfdtd/solver.py:456-466, with the mesh
    summary of torchfdtd/mesh.py:100-107), computed for this engine: device memory is the plan's arena."""
    r = project.region
    dims = 2 if r.dimension == '2d' else 3
    widths = [np.diff(a) for a in r.mesh_nodes[:dims]]
    real = np.dtype(plan.dtype).itemsize
    cells = math.prod(r.shape)
    traces = 0
    for t in plan.traces:
        m = t.monitor
        samples = len(range(0, r.steps, m.time_downsample))
        traces += r.steps * real + 16 * (samples // 2 + 1 if m.spectrum.sampling == 'fft' else len(frequency_samples_of(m)))
    waveform = sum(t.values.size * real for t in plan.sources)
    host = 2 * cells * 3 * real + traces
    ratios = [max(float((w[1:] / w[:-1]).max()), float((w[:-1] / w[1:]).max())) if w.size > 1 else 1.0 for w in widths]
    return dict(mesh_type=r.mesh_type, material_sampling=r.material_sampling, uniform_reference_cells=math.prod(r.base_shape),
                cell_reduction_percent=100 * (1 - cells / math.prod(r.base_shape)),
                axis_min_step_um=[float(w.min()) for w in widths], axis_max_step_um=[float(w.max()) for w in widths],
                coarse_limit_um=getattr(r, '_coarse_limit', None) or r.reference_step, max_adjacent_ratio=max(ratios),
                shape=list(r.shape), actual_size_um=list(r.actual_size), cells=cells, dt_fs=r.time_step * 1e15,
                duration_fs=r.time_step * r.steps * 1e15, estimated_memory_mb=round((arena_bytes + waveform) / 2**20, 1),
                memory_model='fused_b200_arena', host_estimated_mb=round(host / 2**20, 1), oneway_planes=[], tfsf_boxes=[],
                tfsf_auxiliary_estimated_bytes=0, point_trace_estimated_bytes=traces,
                source_waveform_estimated_bytes=waveform, snapshot=snapshot_frames(project))


def frequency_samples_of(monitor):
    from .spectra import frequency_samples
    return frequency_samples(monitor.spectrum)


def resolve_selector(region):
    """Refuse every kernel/back-end choice other than the fused CUDA path (reference models.py:277,287-288)."""
    if region.backend == 'cpu':
        raise ValueError('The fused CUDA kernel requires backend="cuda" and a CUDA GPU; backend="cpu" is the reference '
                         "NumPy path, which this engine does not provide.")
    for name in ('cuda_kernel', 'cuda_monitor_kernel'):
        if getattr(region, name) == 'torch':
            raise ValueError(f'{name}="torch" selects the reference Torch kernels, which this engine does not provide; '
                             'use "fused" or "auto".')
    return 'fused'


class Observer:
    """Frames, divergence checks and the packaged ``Result`` of one grid during a run
    (reference torchfdtd/solver.py:806-908; per case in torchfdtd/tensor_batch.py:228-333)."""

    def __init__(self, project, plan, grid, label=''):
        r = project.region
        self.project, self.plan, self.grid, self.region = project, plan, grid, r
        self.label = label
        self.control = r.run_control
        self.source_end = source_end_time(project)
        self.decision = DecayDecision(self.control, self.source_end, r.time_step)
        self.diagnose = self.control.auto_shutoff or self.control.divergence_check
        self.warnings = list(plan.warnings)
        if self.control.auto_shutoff and not math.isfinite(self.source_end):
            self.warnings.append('Automatic decay shutoff is inactive while a continuous source is enabled.')
        self.axis = 'xyz'.index(r.slice_axis)
        self.plane_index = index_at(tuple(r.slice_position if i == self.axis else 0 for i in range(3)), r, r.field)[self.axis]
        component = 'xyz'.index(r.field[1].lower())
        # Nonuniform meshes: frames (and the permittivity plane) are sampled at the cells nearest to a uniform
        # grid of min(256, uniform cells) pixels per in-plane axis (reference torchfdtd/solver.py:810-818).
        self.display = None
        if r.mesh_type != 'uniform':
            self.display = []
            for i, coords in enumerate(field_axes(r, r.field)):
                if i == self.axis:
                    continue
                count = min(256, r.base_shape[i])
                pixels = (np.arange(count) + .5) * r.actual_size[i] / count - r.actual_size[i] / 2
                self.display.append(np.abs(coords[:, None] - pixels).argmin(axis=0))
        eps = plan.epsilon
        sl = [slice(None)] * 3
        sl[self.axis] = self.plane_index
        plane = (eps[..., component] if eps.ndim == 4 else eps)[tuple(sl)]
        if hasattr(plane, 'cpu'):                          # a permittivity tensor given to Simulation
            plane = plane.detach().cpu().numpy()
        self.eps_plane = np.array(self.decimate(np.asarray(plane, dtype=plan.dtype)))
        self.interval = max(r.snapshot_interval, math.ceil(r.steps / 100))
        self.frames, self.frame_steps = [], []
        self.host_fields = None                     # future of prefaulted (E, H) host arrays, large grids
        self.ring = None                            # future of the pinned download staging ring, large grids
        self.diagnostic_seconds = 0.

    def decimate(self, a):
        if self.display is not None:
            return a[self.display[0][:, None], self.display[1][None, :]]
        return a[::max(1, math.ceil(a.shape[0] / 256)), ::max(1, math.ceil(a.shape[1] / 256))]

    def barriers(self):
        """Steps after which this grid is observed on the host."""
        steps = self.region.steps
        due = set(range(self.interval, steps + 1, self.interval)) | {steps}
        if self.diagnose:
            due.update(range(self.control.check_interval, steps + 1, self.control.check_interval))
        return due

    def _where(self, text):
        return f'{self.label}{text}'

    def observe(self, completed, progress=None, started=None):
        """Observations due after ``completed`` steps; True when the decay shutoff fires."""
        r, control, stop = self.region, self.control, False
        if self.diagnose and (completed % control.check_interval == 0 or completed == r.steps):
            t0 = time.perf_counter()
            energy, peak, finite = self.grid.diagnose()
            if not finite:
                raise FloatingPointError(self._where(f'Non-finite CPML or incident-line memory detected. (diagnostic step {completed})'))
            try:
                stop = self.decision.update(completed, energy, peak)
            except FloatingPointError as exc:
                raise FloatingPointError(self._where(f'{exc} (diagnostic step {completed})')) from exc
            self.diagnostic_seconds += time.perf_counter() - t0
        if completed % self.interval == 0 or completed == r.steps or stop:
            frame = self.decimate(self.grid.get_slice(r.field, self.axis, self.plane_index))
            if not np.isfinite(frame).all():
                raise FloatingPointError(self._where('Fields diverged. Check mesh, sources and precision.'))
            frame = {'real': np.real, 'imag': np.imag, 'magnitude': np.abs, 'phase': np.angle}[r.complex_display](frame)
            self.frames.append(frame)
            self.frame_steps.append(completed)
            if progress:
                progress({'step': completed, 'total': r.steps, 'frame': frame.tolist(),
                          'elapsed': time.perf_counter() - started,
                          'termination_reason': 'decayed' if stop else None,
                          'diagnostics': self.decision.history[-1] if self.decision.history else None})
        return stop

    def large_fields(self):
        """Whether the field arrays take the device-side checks and the staged download."""
        return math.prod(self.plan.shape) * 3 * np.dtype(self.plan.dtype).itemsize > LARGE_FIELD_BYTES

    def result(self, completed, termination_reason, seconds, setup_seconds, phases=None, **extra):
        """Read the final state back and package it as the reference's ``Result``. ``phases``: the caller's
        per-phase host seconds; the field download and the rest of the packaging are added to it."""
        import torch
        from .native import download
        t_start = time.perf_counter()
        p, r, plan, grid = self.project, self.region, self.plan, self.grid
        status = grid.device_status()
        if status:
            raise RuntimeError(self._where(f'A fused kernel reported device status {status}.'))
        if self.large_fields():
            # Large grids: finiteness and the peak are checked on the device, and the fields come back through
            # a pinned staging ring (native.download). Small grids keep the host path, whose fixed costs are
            # lower than the first use of the device reductions.
            field_peak, finite = grid.field_check()
            if not finite:
                raise FloatingPointError(self._where('Non-finite fields detected.'))
            e_dev, h_dev = grid.fields_device()
            t_wait = time.perf_counter()
            e_out, h_out = self.host_fields.result() if self.host_fields is not None else (None, None)
            if self.ring is not None:
                self.ring.result()
            t_copy = time.perf_counter()
            e, h = download(e_dev, out=e_out), download(h_dev, out=h_out)
            t_done = time.perf_counter()
            del e_dev, h_dev
        else:
            t_wait = t_copy = time.perf_counter()
            e, h = grid.get_fields()
            t_done = time.perf_counter()
            if not np.isfinite(e).all() or not np.isfinite(h).all():
                raise FloatingPointError(self._where('Non-finite fields detected.'))
            field_peak = float(np.max(np.abs(e)))
        traces = grid.get_traces()[:completed]
        frequency_results = []
        for k, pp in enumerate(plan.planes):
            values = grid.get_plane(k)
            frequency_results.append(plane_result(pp.monitor, pp.plan, pp.frequency, list(pp.components), values, r.dimension))
        if frequency_results:
            signature = run_signature(p, completed)
            for m in frequency_results:
                m['run_signature'] = signature
        cells = math.prod(r.shape)
        if r.material_sampling == 'yee':
            from .plan import field_axes
            slice_position = float(field_axes(r, r.field)[self.axis][self.plane_index])
        else:
            slice_position = (0 if r.dimension == '2d' and self.axis == 2
                              else (self.plane_index + .5) * r.mesh - r.actual_size[self.axis] / 2)
        stats = run_estimates(p, plan, grid.arena_bytes)
        stats.update(warnings=self.warnings, plan_hash=run_signature(p, r.steps), backend='cuda', precision=r.precision,
                     gpu=torch.cuda.get_device_name(),
                     cuda_kernel='fused', cuda_monitor_kernel='fused', kernel=grid.kernel,
                     steps=completed, requested_steps=r.steps, cancelled=termination_reason == 'cancelled',
                     termination_reason=termination_reason, auto_shutoff=termination_reason == 'decayed',
                     diagnostics=self.decision.history, diagnostic_seconds=self.diagnostic_seconds,
                     diagnostic_backend='fused_cuda' if self.diagnose else None,
                     source_end_s=self.source_end if math.isfinite(self.source_end) else None,
                     seconds=seconds, setup_seconds=setup_seconds,
                     mcells_per_second=cells * completed / max(seconds, 1e-9) / 1e6,
                     gcells_per_s=cells * completed / max(seconds, 1e-9) / 1e9,
                     hbm_bytes_per_step=algorithmic_bytes_per_step(plan), arena_bytes=grid.arena_bytes,
                     field_peak=field_peak, slice_index=self.plane_index, slice_position=slice_position,
                     complex_fields=False, complex_display=r.complex_display,
                     material_update='trapezoidal ADE' if plan.ade else 'nondispersive',
                     dispersive_samples=sum(st.poles * st.samples for st in plan.ade), material_sampling=r.material_sampling,
                     epsilon_definition='instantaneous relative permittivity (epsilon-infinity for dispersive cells)',
                     boundaries=r.boundaries.model_dump(), bloch_phase=r.bloch_phase,
                     units='geometry: um; time: s; E/H: reduced fields; Bloch phase: rad', engine=ENGINE)
        stats.update(extra)
        if phases is not None:
            phases['field_check'] = t_wait - t_start
            phases['host_result_arrays_wait'] = t_copy - t_wait
            phases['field_download'] = t_done - t_copy
            phases['result_packaging'] = time.perf_counter() - t_done
            stats['phase_seconds'] = dict(phases)
        return Result(p, stats, np.array(self.frames), np.array(self.frame_steps), self.eps_plane, traces,
                      np.arange(1, completed + 1) * r.time_step, e, h, frequency_results)


# Field arrays above this size take the device-side checks and the staged download in Observer.result, and
# a given permittivity above it is checked and inverted on the device.
LARGE_FIELD_BYTES = 64 << 20


def capture_graphs(step, widths):
    """CUDA graphs of ``step(count)`` for each width, captured on the current stream."""
    import torch
    graphs = {}
    for count in sorted(set(widths)):
        g = torch.cuda.CUDAGraph()
        g.capture_begin()
        step(count)
        g.capture_end()
        graphs[count] = g
    return graphs


class Simulation:
    """Run the fused Yee/CPML kernels on a B200 for a ``Project``.

    Coordinates, spans, wavelength and mesh are micrometres; E/H are the reduced
    fields of the reference, not calibrated V/m or A/m."""

    def __init__(self, project: Project, epsilon=None):
        """``epsilon`` (optional) replaces the voxelized relative permittivity with an array of the
        grid shape, (nx, ny, nz) or (nx, ny, nz, 3): a material given at plan level instead of as
        structures (the reference's differentiable path takes the same, torchfdtd/differentiable.py:100)."""
        self.project = Project.model_validate(project.model_dump())
        self.project.region.require_resident()
        self.epsilon = epsilon

    @cached_property
    def plan(self):
        plan = plan_grid(self.project)
        if self.epsilon is not None:
            eps = np.asarray(self.epsilon, dtype=plan.dtype)
            if eps.shape not in (tuple(plan.shape), (*plan.shape, 3)):
                raise ValueError(f'epsilon must have shape {tuple(plan.shape)} or {(*plan.shape, 3)}, not {eps.shape}.')
            if not np.all(np.isfinite(eps)) or np.any(eps < 1):
                raise ValueError('epsilon must be finite and at least 1.')
            from .injection import validate_oneway_materials
            from .tfsf import validate_tfsf_materials
            validate_oneway_materials(self.project, eps)
            validate_tfsf_materials(self.project, eps)
            plan.epsilon = eps
            plan.inv_eps = (1 / eps).astype(plan.dtype)
        return plan

    def _run_plan(self):
        """(plan, permittivity) for ``run``. A large ``epsilon`` skips voxelization and the host pass: the
        library checks and inverts it on the device (IEEE division: the same values as the host's 1 / eps), and
        ``plan.inv_eps`` stays None."""
        if self.epsilon is None or np.size(self.epsilon) * 4 <= LARGE_FIELD_BYTES:
            return self.plan, None
        import torch
        plan = plan_grid(self.project, material=False)
        shape = tuple(np.shape(self.epsilon))
        if shape not in (tuple(plan.shape), (*plan.shape, 3)):
            raise ValueError(f'epsilon must have shape {tuple(plan.shape)} or {(*plan.shape, 3)}, not {shape}.')
        dtype = torch.float64 if plan.dtype == np.float64 else torch.float32
        if isinstance(self.epsilon, torch.Tensor) and self.epsilon.is_cuda:
            eps = self.epsilon.detach().to(device='cuda', dtype=dtype).contiguous()
        else:
            eps = np.ascontiguousarray(np.asarray(self.epsilon, dtype=plan.dtype))
        plan.epsilon = self.epsilon
        return plan, eps

    def run(self, progress=None, cancel=None, cuda_graph=True, cuda_graph_steps=1, kernel='auto', launch=None):
        """``kernel``: 'auto' (the marching kernel for 3D, the tile kernel for 2D TMz, else gather) or a name.
        ``launch``: None (default launch shape), an explicit launch variant, or 'auto' to measure the
        marching kernel's variants on scratch plans first (``tuning.select_launch``; cached per process)."""
        with ENGINE_LOCK:
            return self._run(progress, cancel, cuda_graph, cuda_graph_steps, kernel, launch)

    def _run(self, progress, cancel, cuda_graph, cuda_graph_steps, kernel, launch=None):
        import torch
        from .native import NativeGrid
        p, r = self.project, self.project.region
        resolve_selector(r)
        validate_graph_steps(cuda_graph_steps, cuda_graph)
        if not torch.cuda.is_available():
            raise RuntimeError('CUDA requested but unavailable. The fused B200 engine needs a CUDA GPU.')
        started = time.perf_counter()
        # Host seconds of each phase of the call (device work included where the phase waits for it).
        phases, mark = {}, [started]

        def lap(name):
            now = time.perf_counter()
            phases[name] = now - mark[0]
            mark[0] = now

        plan, permittivity = self._run_plan()
        lap('plan')
        helper, host_fields, ring = None, None, None
        shape, dtype = (*plan.shape, 3), np.dtype(plan.dtype)
        large = math.prod(shape) * dtype.itemsize > LARGE_FIELD_BYTES
        if large:
            # Helper threads pin the download's staging ring and map the result's host arrays while the device
            # steps. Both start once the graphs are captured: the ring is a CUDA host allocation, which a capture
            # must not see, and the page zeroing of either slowed the device arena allocation and the graph
            # instantiation when they ran beside them.
            from concurrent.futures import ThreadPoolExecutor
            from .native import host_buffer, staging_ring
            helper = ThreadPoolExecutor(max_workers=2)
        grid, graphs = None, {}
        try:
            variant, tuning = 0, None
            if launch == 'auto':
                if plan.dimension == '3d' and kernel in ('auto', 'march'):
                    from .tuning import select_launch
                    try:
                        tuning = select_launch(plan)
                        variant = tuning.choice
                    except ValueError as exc:          # too few steps to tune, or no marching kernel for this scene
                        tuning = dict(skipped=str(exc))
            elif launch is not None:
                variant = int(launch)
            if tuning is not None:
                lap('launch_tuning')
            grid = NativeGrid(plan, kernel=kernel, variant=variant, permittivity=permittivity)
            phases.update(grid.timing)
            mark[0] = time.perf_counter()
            free, _ = torch.cuda.mem_get_info()
            observer = Observer(p, plan, grid)
            lap('observer')
            width = 1
            stream = torch.cuda.Stream()
            stream.wait_stream(torch.cuda.current_stream())
            if cuda_graph:
                width = min(cuda_graph_steps, r.steps)
                with torch.cuda.stream(stream):
                    # One eager step loads the kernels before capture; the state is then zeroed.
                    grid.step(1, stream)
                    grid.reset()
                    stream.synchronize()
                    lap('warm_step_and_reset')
                    graphs = capture_graphs(lambda count: grid.step(count, stream), {1, width})
                torch.cuda.synchronize()
            torch.cuda.synchronize()
            lap('graph_capture')
            if large:
                ring = helper.submit(staging_ring, torch.float32 if dtype == np.float32 else torch.float64)
                host_fields = helper.submit(lambda: (host_buffer(shape, dtype), host_buffer(shape, dtype)))
                observer.host_fields, observer.ring = host_fields, ring
            setup_seconds = time.perf_counter() - started
            compute_start = time.perf_counter()
            completed, termination_reason, replays = 0, 'max_steps', 0
            with torch.cuda.stream(stream):
                for target, advance in observation_schedule(r.steps, width, observer.barriers()):
                    if cancel is not None and cancel.is_set():
                        termination_reason = 'cancelled'
                        break
                    if graphs:
                        graphs[advance].replay()
                        replays += 1
                    else:
                        grid.step(advance, stream)
                    completed = target
                    if observer.observe(completed, progress, compute_start):
                        termination_reason = 'decayed'
                        break
            torch.cuda.synchronize()
            seconds = time.perf_counter() - compute_start
            phases['stepping'] = seconds
            mark[0] = time.perf_counter()
            result = observer.result(completed, termination_reason, seconds, setup_seconds, phases, cuda_graph=bool(graphs),
                                     cuda_graph_steps=width, cuda_graph_replays=replays, free_device_bytes=free,
                                     launch_variant=variant or None,
                                     launch_tuning=tuning.as_dict() if hasattr(tuning, 'as_dict') else tuning)
        finally:
            # The helper threads (pinned staging ring, mapped result arrays) are joined on every path.
            if helper is not None:
                helper.shutdown(wait=True)
            graphs.clear()
            if grid is not None:
                grid.close()
        return result

"""Discrete adjoint of the fused Yee/CPML time loop behind ``torch.autograd.Function``.

Mirrors the reference's differentiable API (torchfdtd/differentiable.py): ``AdjointOptions`` (:28-68),
``DifferentiableResult`` with ``spectrum`` (:71-96), ``DifferentiableSimulation`` (:756-906, point monitors,
``forward`` and ``spectrum``) and ``DifferentiablePlaneSimulation`` (torchfdtd/adjoint_planes.py:154-285,
field-plane DFTs of all six components). The forward pass runs the fused kernels; the backward pass runs
the hand-written reverse-time kernel (``tfd_adjoint_step``: the transpose of one step with the CPML
memory transpose, accumulating the material sensitivity) over restart states recomputed from
checkpoints.

Checkpointing is the two-level square-root scheme: the forward pass stores K restart snapshots (default
K = ceil(sqrt(steps))) in device memory; the backward pass restores each segment's snapshot, replays the
segment once while saving its states, and transposes the segment's steps in reverse from those states.
Every forward step is therefore recomputed exactly once, and device memory holds about 2 sqrt(steps)
restart states (the reference's binomial schedule, differentiable.py:644-652, trades more replays for
fewer slots; on a 180 GB device the square-root schedule's memory is affordable and its replay count is
the minimum).

The gradient is with respect to the relative permittivity (per cell, or per Yee component with a
trailing axis of 3): dJ/d eps = -courant * S / eps^2 with S = sum over steps of e_bar * curl_b(H), as in the
reference's ``transpose_step``. Observations are point samples of the state after each step; spectra
and plane DFTs are linear torch operations on those samples, so autograd supplies their transpose.
"""
from __future__ import annotations

import math
import time
from dataclasses import dataclass, field, replace
from functools import cached_property

import numpy as np

from .models import Project
from .plan import Trace, plan_grid
from .simulation import ENGINE_LOCK, resolve_selector

COMPONENTS = ('Ex', 'Ey', 'Ez', 'Hx', 'Hy', 'Hz')


@dataclass(frozen=True)
class AdjointOptions:
    """``checkpoints``: restart snapshots kept by the forward pass (None: ceil(sqrt(steps)));
    ``storage``: 'device' (the only tier; snapshots stay in HBM)."""
    checkpoints: int | None = None
    storage: str = 'device'

    def __post_init__(self):
        if self.checkpoints is not None and (isinstance(self.checkpoints, bool) or not isinstance(self.checkpoints, int)
                                             or not 1 <= self.checkpoints <= 65536):
            raise ValueError('checkpoints must be None or an integer from 1 to 65536.')
        if self.storage != 'device':
            raise ValueError("Checkpoint storage 'device' is the only tier of the B200 engine (HBM holds the snapshots).")


@dataclass
class DifferentiableResult:
    signals: object               # torch (steps, monitors)
    time_step: float
    monitor_components: tuple
    report: dict = field(default_factory=dict)

    def spectrum(self, frequency_hz, *, window=None):
        """Time-integral DFT with the half-step H time convention (reference differentiable.py:78-96)."""
        import torch
        frequency = torch.as_tensor(frequency_hz, device=self.signals.device, dtype=self.signals.dtype).reshape(-1)
        if not bool(torch.isfinite(frequency).all()) or bool((frequency <= 0).any()):
            raise ValueError('Frequencies must be finite and positive.')
        if bool((frequency * self.time_step >= .5).any()):
            raise ValueError('Frequencies must be below temporal Nyquist.')
        t = (torch.arange(self.signals.shape[0], device=frequency.device, dtype=frequency.dtype) + 1) * self.time_step
        weights = torch.ones_like(t) if window is None else torch.as_tensor(window, device=t.device, dtype=t.dtype)
        if weights.shape != t.shape:
            raise ValueError('Window must have one weight per timestep.')
        values = []
        for i, comp in enumerate(self.monitor_components):
            times = t + (self.time_step / 2 if comp[0] == 'H' else 0)
            kernel = torch.exp(-2j * torch.pi * frequency[:, None] * times[None, :])
            values.append(kernel @ (self.signals[:, i] * weights).to(kernel.dtype) * self.time_step)
        return torch.stack(values, dim=-1)


@dataclass
class DifferentiablePlaneResult:
    fields: object                # torch complex (frequencies, points, 6): Ex, Ey, Ez, Hx, Hy, Hz
    frequency_hz: object
    points_um: object
    weights: object
    shape: tuple
    normal: str
    report: dict = field(default_factory=dict)


class _Engine:
    """Native plan + adjoint + snapshots of one fixed project; the observers are the plan's traces."""

    def __init__(self, plan, options):
        import torch
        from .native import NativeAdjoint, NativeGrid
        self.plan = plan
        self.options = options
        self.grid = NativeGrid(plan, kernel='auto')
        self.adjoint = NativeAdjoint(self.grid)
        self.state_bytes = self.grid.state_bytes()
        steps = plan.steps
        self.slots = min(steps, options.checkpoints or math.ceil(math.sqrt(steps)))
        self.segment = math.ceil(steps / self.slots)
        self.slots = math.ceil(steps / self.segment)
        device = self.grid.device
        self.checkpoints = torch.empty((self.slots, self.state_bytes), dtype=torch.uint8, device=device)
        self.replay = torch.empty((self.segment, self.state_bytes), dtype=torch.uint8, device=device)
        self.report = dict(adjoint='discrete Yee/CPML (fused CUDA transpose)', checkpoint_scheme='sqrt(T) two-level',
                           checkpoints=self.slots, segment_steps=self.segment, restart_bytes=self.state_bytes,
                           checkpoint_bytes=int(self.checkpoints.numel() + self.replay.numel()),
                           forward_kernel=self.grid.kernel)

    def set_material(self, epsilon):
        inv = 1 / epsilon.detach()
        self.grid.set_material(inv if inv.ndim == 3 else inv.contiguous())

    def forward(self, epsilon):
        import torch
        started = time.perf_counter()
        self.set_material(epsilon)
        self.grid.reset()
        steps = self.plan.steps
        for k in range(self.slots):
            self.grid.save_state(self.checkpoints[k])
            self.grid.step(min(self.segment, steps - k * self.segment))
        signals = self.grid.traces_device()
        torch.cuda.synchronize(self.grid.device)
        self.report['forward_seconds'] = time.perf_counter() - started
        return signals

    def backward(self, signal_bar, epsilon):
        import torch
        started = time.perf_counter()
        seeds = signal_bar.detach().to(self.grid.torch_dtype).contiguous()
        steps = self.plan.steps
        self.adjoint.reset()
        replayed = 0
        for k in range(self.slots - 1, -1, -1):
            start = k * self.segment
            end = min(start + self.segment, steps)
            self.grid.load_state(self.checkpoints[k])
            for j in range(end - start):
                self.grid.save_state(self.replay[j])
                if start + j + 1 < end:
                    self.grid.step(1)
                    replayed += 1
            for n in range(end - 1, start - 1, -1):
                self.adjoint.step(self.replay[n - start], seeds[n] if seeds.shape[1] else None)
        S = self.adjoint.sensitivity()
        eps = epsilon.detach()
        if eps.ndim == 3:
            S = S[..., 0] + S[..., 1] + S[..., 2]
        gradient = (-self.plan.courant) * S / (eps * eps)
        status = self.grid.device_status()
        if status:
            raise RuntimeError(f'A fused kernel reported device status {status}.')
        torch.cuda.synchronize(self.grid.device)
        self.report.update(backward_seconds=time.perf_counter() - started, replayed_steps=replayed)
        return gradient.to(epsilon.dtype)

    def close(self):
        self.adjoint.close()
        self.grid.close()


_FUNCTION = []


def _autograd_function():
    if _FUNCTION:
        return _FUNCTION[0]
    import torch

    class _FDTD(torch.autograd.Function):
        @staticmethod
        def forward(ctx, epsilon, engine):
            ctx.engine = engine
            ctx.save_for_backward(epsilon)
            return engine.forward(epsilon)

        @staticmethod
        def backward(ctx, signal_bar):
            if torch.is_grad_enabled():
                raise RuntimeError('Higher-order derivatives are not supported by the discrete adjoint.')
            epsilon, = ctx.saved_tensors
            return ctx.engine.backward(signal_bar, epsilon), None

    _FUNCTION.append(_FDTD)
    return _FDTD


def _check_epsilon(epsilon, plan):
    import torch
    if not isinstance(epsilon, torch.Tensor) or epsilon.dtype not in (torch.float32, torch.float64):
        raise ValueError('epsilon must be a real float32 or float64 torch Tensor.')
    if epsilon.device.type != 'cuda':
        raise ValueError('The B200 engine differentiates on the GPU: pass a CUDA epsilon tensor.')
    if tuple(epsilon.shape) not in (tuple(plan.shape), (*plan.shape, 3)):
        raise ValueError(f'epsilon shape must be {tuple(plan.shape)} or {(*plan.shape, 3)}.')
    if (epsilon.dtype == torch.float64) != (plan.dtype == np.float64):
        raise ValueError('epsilon dtype must match the project precision.')
    if not bool(torch.isfinite(epsilon).all()) or bool((epsilon < 1).any()):
        raise ValueError('This conservative CFL contract requires finite epsilon >= 1.')


def _unique_observers(observers):
    """Distinct (component, cell) observers and, per requested observer, its distinct column."""
    index, unique, columns = {}, [], []
    for component, cell in observers:
        key = (component, tuple(int(v) for v in cell))
        if key not in index:
            index[key] = len(unique)
            unique.append(key)
        columns.append(index[key])
    return unique, columns


def _observer_plan(plan, observers):
    traces = [Trace(None, component, cell) for component, cell in observers]
    return replace(plan, traces=traces, planes=[])


class _Differentiable:
    """Engine ownership shared by the point and plane models: one native engine per material layout
    (a per-cell epsilon, or per Yee component)."""
    _engine = None

    def engine(self, epsilon):
        samples = 3 if epsilon.ndim == 4 else 1
        if self._engine is not None and self._engine.plan.material_samples != samples:
            self.close()
        if self._engine is None:
            plan = self.plan
            inv = np.ones((*plan.shape, 3) if samples == 3 else plan.shape, dtype=plan.dtype)
            self._engine = _Engine(replace(plan, inv_eps=inv, epsilon=1 / inv), self.options)
        return self._engine

    def close(self):
        if self._engine is not None:
            self._engine.close()
            self._engine = None


class DifferentiableSimulation(_Differentiable):
    """Epsilon -> point-monitor signals with a discrete adjoint (reference differentiable.py:756-906).

    Epsilon has shape (Nx, Ny, Nz), or (Nx, Ny, Nz, 3) for per-component Yee values, on the GPU, in the
    project's precision. The result's ``signals`` are (steps, monitors), sampled after every step."""

    def __init__(self, project: Project, options: AdjointOptions | None = None):
        self.project = Project.model_validate(project.model_dump())
        self.options = options or AdjointOptions()
        p, r = self.project, self.project.region
        resolve_selector(r)
        if not any(m.enabled for m in p.monitors) or any(m.enabled and m.kind != 'point' for m in p.monitors):
            raise ValueError('The differentiable API currently requires point monitors only.')
        if r.run_control.auto_shutoff:
            raise ValueError('Differentiable simulations require a fixed number of timesteps.')

    @cached_property
    def plan(self):
        plan = plan_grid(self.project)
        if plan.tfsf:
            raise ValueError('TFSF boxes are not differentiated by the B200 engine; use soft or one-way sources.')
        observers = [(t.component, t.index) for t in plan.traces]
        unique, self._columns = _unique_observers(observers)
        return _observer_plan(plan, unique)

    def __call__(self, epsilon):
        return self.forward(epsilon)

    def forward(self, epsilon):
        import torch
        plan = self.plan
        _check_epsilon(epsilon, plan)
        with ENGINE_LOCK:
            engine = self.engine(epsilon)
            unique = _autograd_function().apply(epsilon, engine)
        signals = unique[:, torch.as_tensor(self._columns, device=unique.device)]
        comps = tuple(m.component for m in self.project.monitors if m.enabled)
        return DifferentiableResult(signals, self.project.region.time_step, comps, engine.report)

    def spectrum(self, epsilon, frequency_hz, *, window=None):
        """Point-monitor spectra (frequencies, monitors) of ``forward(epsilon)``, differentiable."""
        return self.forward(epsilon).spectrum(frequency_hz, window=window)


class DifferentiablePlaneSimulation(_Differentiable):
    """Epsilon -> DFT field planes (all six components) with a discrete adjoint
    (reference torchfdtd/adjoint_planes.py:154-285). Every enabled monitor must be a field plane with no
    apodization and time_downsample 1. The observers are the distinct Yee cells the planes' trilinear
    interpolation reads; their time samples are transformed and interpolated with torch operations."""

    def __init__(self, project: Project, options: AdjointOptions | None = None):
        self.project = Project.model_validate(project.model_dump())
        self.options = options or AdjointOptions()
        p, r = self.project, self.project.region
        resolve_selector(r)
        active = [m for m in p.monitors if m.enabled]
        if not active or any(m.kind != 'field' for m in active):
            raise ValueError('DifferentiablePlaneSimulation requires enabled field monitors only.')
        for raw in active:
            m = p.resolved_monitor(raw)
            if m.time_downsample != 1 or m.spectrum.apodization != 'none':
                raise ValueError('Differentiable planes require time_downsample=1 and no apodization.')
        if r.run_control.auto_shutoff:
            raise ValueError('Differentiable simulations require a fixed number of timesteps.')

    @cached_property
    def plan(self):
        plan = plan_grid(self.project)
        if plan.tfsf:
            raise ValueError('TFSF boxes are not differentiated by the B200 engine; use soft or one-way sources.')
        nx, ny, nz = plan.shape
        observers, self._maps = [], []
        for pp in plan.planes:
            maps = []
            for k, component in enumerate(pp.components):
                cells = np.asarray(pp.corner_cells[k], dtype=np.int64)        # (corners, points), flat (x*ny+y)*nz+z
                xyz = np.stack(np.unravel_index(cells.reshape(-1), (nx, ny, nz)), axis=-1)
                start = len(observers)
                observers.extend((component, tuple(c)) for c in xyz)
                maps.append((component, np.arange(start, len(observers)).reshape(cells.shape),
                             np.asarray(pp.corner_weights[k], dtype=np.float64)))
            self._maps.append((pp, maps))
        unique, columns = _unique_observers(observers)
        self._columns = np.asarray(columns, dtype=np.int64)
        return _observer_plan(plan, unique)

    def __call__(self, epsilon, frequency_hz=None):
        return self.forward(epsilon, frequency_hz)

    def forward(self, epsilon, frequency_hz=None):
        """{monitor id: DifferentiablePlaneResult}. ``frequency_hz``: override the monitors' frequencies."""
        import torch
        plan = self.plan
        _check_epsilon(epsilon, plan)
        with ENGINE_LOCK:
            engine = self.engine(epsilon)
            samples = _autograd_function().apply(epsilon, engine)            # (steps, distinct observers)
        dt = self.project.region.time_step
        cdtype = torch.complex128 if samples.dtype == torch.float64 else torch.complex64
        t = (torch.arange(samples.shape[0], device=samples.device, dtype=torch.float64) + 1) * dt
        out = {}
        columns = torch.as_tensor(self._columns, device=samples.device)
        for pp, maps in self._maps:
            freq = torch.as_tensor(pp.frequency if frequency_hz is None else np.atleast_1d(frequency_hz),
                                   device=samples.device, dtype=torch.float64)
            fields = []
            by_comp = {c: (idx, w) for c, idx, w in maps}
            for component in COMPONENTS:
                if component not in by_comp:
                    fields.append(torch.zeros((len(freq), pp.corner_cells.shape[2]), dtype=cdtype, device=samples.device))
                    continue
                idx, w = by_comp[component]
                times = t + (dt / 2 if component[0] == 'H' else 0)
                kernel = (torch.exp(2j * torch.pi * freq[:, None] * times[None, :]) * dt).to(cdtype)   # (F, T)
                obs = columns[torch.as_tensor(idx.reshape(-1), device=samples.device)]
                series = samples[:, obs].to(cdtype)                                                 # (T, K*P)
                spectra = (kernel @ series).reshape(len(freq), *idx.shape)                           # (F, K, P)
                weight = torch.as_tensor(w, device=samples.device).to(cdtype)
                fields.append((spectra * weight[None]).sum(dim=1))
            out[pp.monitor.id] = DifferentiablePlaneResult(
                torch.stack(fields, dim=-1), freq, torch.as_tensor(pp.plan['points_um']), torch.as_tensor(pp.plan['weights']),
                tuple(pp.plan['shape']), pp.monitor.normal, engine.report)
        return out


"""Batched runs: many independent 2D TMz Projects of uneven size advanced by one persistent launch per step.

Mirrors the reference's batch API: ``BatchCase`` / ``BatchItem`` / ``BatchReport``
(torchfdtd/batch.py:32-85), ``run_tensor_batch`` (torchfdtd/tensor_batch.py:45-113, per-cohort run :128-337),
``plan_grouped_batch`` / ``run_grouped_batch`` (torchfdtd/grouped_batch.py:38-146).

What differs, by design: the reference batches only cases of identical topology (shape, steps, time step,
boundaries; tensor_batch.py:32-42) and launches one kernel per cohort, so uneven grids run as successive
cohorts. Here every case of a cohort keeps its own plan (its own shape, time step, CPML, sources and
monitors) and the fused 2D step kernel walks one tile table over all of them, so a cohort of uneven grids
costs one step launch plus one monitor launch per time step, captured in CUDA graphs. Cases may even have
different step counts (a finished grid is skipped). What a cohort needs is one precision and the 2D TMz
fused kernel (2D, TM sources only, PML or PEC x/y faces); ``run_grouped_batch`` groups by precision and runs
any case outside that set on its own through ``Simulation`` (the reference likewise runs incompatible groups
successively). Results are bitwise identical to running each case alone.
"""
from __future__ import annotations

import hashlib
import json
import math
import os
import re
import time
from dataclasses import asdict, dataclass, field
from pathlib import Path

import numpy as np

from .models import Project
from .run_control import observation_schedule, validate_graph_steps
from .simulation import ENGINE_LOCK, Observer, Result, Simulation, capture_graphs, resolve_selector

MAX_COHORT = 64


@dataclass
class BatchCase:
    id: str
    project: Project
    parameters: dict = field(default_factory=dict)

    def __post_init__(self):
        if not re.fullmatch(r'[A-Za-z0-9][A-Za-z0-9_.-]{0,95}', self.id):
            raise ValueError('Case ids need 1-96 ASCII letters/digits/dot/underscore/hyphen, starting with a letter or digit.')
        self.project = Project.model_validate(self.project.model_dump())
        json.dumps(self.parameters, allow_nan=False)


@dataclass
class BatchItem:
    id: str
    status: str
    parameters: dict
    summary: dict = field(default_factory=dict)
    metrics: dict = field(default_factory=dict)
    output: str | None = None
    error: str | None = None
    pid: int | None = None
    device: str | None = None
    started: float | None = None
    finished: float | None = None
    resumed: bool = False
    result: Result | None = field(default=None, repr=False)

    def load(self):
        if self.result is not None:
            return self.result
        if self.output is None:
            raise ValueError('No saved or retained result. Set output_dir or keep_results=True.')
        return Result.load(self.output)

    def as_dict(self):
        d = asdict(self)
        d.pop('result')
        return d


@dataclass
class BatchReport:
    items: list
    seconds: float
    plan: dict

    @property
    def successful(self):
        return all(item.status == 'completed' for item in self.items)

    def raise_for_errors(self):
        errors = [f'{x.id}: {x.error or x.status}' for x in self.items if x.status != 'completed']
        if errors:
            raise RuntimeError('Batch did not complete: ' + '; '.join(errors))
        return self

    def as_dict(self):
        return dict(seconds=self.seconds, plan=self.plan, successful=self.successful,
                    items=[item.as_dict() for item in self.items])


def write_json(path, value):
    path = Path(path)
    temporary = path.with_suffix(path.suffix + '.tmp')
    temporary.write_text(json.dumps(value, indent=2, allow_nan=False, default=str), encoding='utf-8')
    temporary.replace(path)


def as_cases(cases):
    """Snapshot the input as BatchCase objects with unique ids (reference grouped_batch.py:24-35)."""
    result = [BatchCase(f'case-{i:04d}', c) if isinstance(c, Project) else c for i, c in enumerate(cases)]
    if not result:
        raise ValueError('A batch requires at least one case.')
    if any(not isinstance(c, BatchCase) for c in result):
        raise TypeError('Supply BatchCase or Project instances.')
    if len({c.id for c in result}) != len(result):
        raise ValueError('Duplicate case ids.')
    return [BatchCase(c.id, c.project, dict(c.parameters)) for c in result]


def batch_refusal(project):
    """Why a project cannot join a fused batch cohort (None when it can)."""
    from .plan import plan_grid
    r = project.region
    if r.backend == 'cpu':
        return 'a batch cannot execute a CPU project. Set backend="cuda" or "auto" explicitly.'
    if r.complex_fields:
        return 'batches require real fields.'
    if r.run_control.auto_shutoff:
        return 'batches require fixed-duration runs. Set auto_shutoff=False.'
    if r.dimension != '2d':
        return 'batch cohorts run 2D TMz grids; 3D projects run through Simulation.'
    if any(r.boundaries.pair(a)[0].kind == 'periodic' for a in (0, 1)):
        return 'batch cohorts need PML or PEC x/y faces (periodic 2D grids run through Simulation).'
    plan = plan_grid(project)
    if plan.polarization != 'TM':
        return f'batch cohorts run the TMz polarization (Ez, Hx, Hy); this project drives {plan.polarization}.'
    return None


def _check_cohort_size(cohort_size):
    if isinstance(cohort_size, bool) or not isinstance(cohort_size, int) or not 1 <= cohort_size <= MAX_COHORT:
        raise ValueError(f'cohort_size must be an integer from 1 to {MAX_COHORT}. Split larger ensembles explicitly.')


def _admit(cases, memory_fraction):
    projects = [Project.model_validate(c.project.model_dump()) for c in cases]
    for c, p in zip(cases, projects):
        p.region.require_resident()
        resolve_selector(p.region)
        why = batch_refusal(p)
        if why:
            raise ValueError(f'{c.id}: {why}')
    if len({p.region.precision for p in projects}) > 1:
        raise ValueError('A batch cohort shares one precision; group float32 and float64 cases separately.')
    if not 0 < memory_fraction <= .9:
        raise ValueError('memory_fraction must be positive and at most .9.')
    return projects


def run_tensor_batch(cases, *, objective=None, output_dir=None, keep_results=True, device=0, memory_fraction=.6,
                     cuda_graph=True, cancel=None, progress=None, cohort_size=None, cuda_graph_steps=1, launch=None,
                     epsilon=None):
    """Run independent 2D TMz projects in fused cohorts of 1-64 cases (reference tensor_batch.py:45-113).

    Shapes, time steps, CPML depths, sources, monitors and step counts may differ between cases; one
    precision per cohort. ``launch`` sets the step kernel's launch shape: None for the default (one warp per
    strip, strip rows sized to the cohort, one launch per step), a ``(ctas, strip_rows[, persistent])`` tuple (0
    keeps a default; persistent 1 runs every replayed width of steps as one cooperative launch), or 'auto' to
    measure candidates on scratch copies first (``tune_tensor_batch``).
    ``epsilon`` (optional): one permittivity array (or None) per case, replacing its voxelized structures as
    ``Simulation(project, epsilon)`` does. Auto shutoff is rejected, never silently disabled. A numerical
    failure aborts the cohort, an invalid objective marks only its item failed. Result summary seconds
    describe the whole cohort.
    """
    import torch
    validate_graph_steps(cuda_graph_steps, cuda_graph)
    cases = as_cases(list(cases))
    if cohort_size is None:
        cohort_size = len(cases)
    _check_cohort_size(cohort_size)
    root = Path(output_dir) if output_dir is not None else None
    if root and ((root / 'tensor-batch.json').exists() or any((root / (c.id + '.npz')).exists() for c in cases)):
        raise FileExistsError('Tensor batch output exists. Use a new directory.')
    projects = _admit(cases, memory_fraction)
    if epsilon is None:
        epsilon = [None] * len(cases)
    epsilon = list(epsilon)
    if len(epsilon) != len(cases):
        raise ValueError('epsilon needs one entry (an array or None) per case.')
    if not torch.cuda.is_available():
        raise RuntimeError('Tensor batch requires CUDA.')
    if isinstance(device, bool) or not isinstance(device, int) or not 0 <= device < torch.cuda.device_count():
        raise ValueError('Invalid CUDA device.')
    with ENGINE_LOCK, torch.cuda.device(device):
        start = time.perf_counter()
        items, plans = [], []
        for offset in range(0, len(cases), cohort_size):
            if cancel is not None and cancel.is_set() and offset:
                items.extend(BatchItem(c.id, 'cancelled', c.parameters) for c in cases[offset:])
                break

            def on_progress(state, offset=offset):
                progress(dict(state, cohort_offset=offset, total_cases=len(cases)))
            report = _run_cohort(cases[offset:offset + cohort_size], projects[offset:offset + cohort_size], objective, root,
                                 keep_results, memory_fraction, cuda_graph, cancel, on_progress if progress else None,
                                 cuda_graph_steps, launch, epsilon[offset:offset + cohort_size])
            items.extend(report.items)
            plans.append(report.plan)
        plan = plans[0] if len(plans) == 1 else dict(
            execution='fused_cuda_cohorts', cohorts=plans, batch_size=len(cases),
            loop_seconds=sum(p['loop_seconds'] for p in plans), setup_seconds=sum(p['setup_seconds'] for p in plans),
            resume=False)
        plan = dict(plan, total_cases=len(cases), cohort_size=cohort_size, cohorts_completed=len(plans))
        report = BatchReport(items, time.perf_counter() - start, plan)
        if root:
            root.mkdir(parents=True, exist_ok=True)
            write_json(root / 'tensor-batch.json', report.as_dict())
        return report


def _run_cohort(cases, projects, objective, root, keep_results, memory_fraction, cuda_graph, cancel, progress,
                cuda_graph_steps, launch, epsilon):
    import torch
    from .native import NativeBatch, NativeGrid
    started, wall_started = time.perf_counter(), time.time()
    tuning = None
    if launch == 'auto':
        from .tuning import tune_tensor_batch
        try:
            tuning = tune_tensor_batch(cases, device=torch.cuda.current_device(), epsilon=epsilon).as_dict()
            launch = tuning['choice']
        except ValueError as exc:                  # runs too short to tune on scratch state
            tuning, launch = dict(skipped=str(exc)), None
    sims = [Simulation(p, epsilon=e) for p, e in zip(projects, epsilon)]
    plans = [s.plan for s in sims]
    estimate = sum(NativeGrid.plan_bytes(plan) for plan in plans)
    free, _ = torch.cuda.mem_get_info()
    if estimate > free * memory_fraction:
        raise ValueError('Tensor cohort exceeds its GPU memory allowance. Split it into smaller cohorts.')
    grids = [NativeGrid(plan, kernel='tile2d') for plan in plans]
    observers = [Observer(p, plan, g, label=f'Case {c.id}: ') for c, p, plan, g in zip(cases, projects, plans, grids)]
    batch = NativeBatch(grids)
    try:
        if launch is not None:
            batch.set_launch(*launch[:2])
            batch.set_persistent(bool(launch[2]) if len(launch) > 2 else False)
        steps = max(p.region.steps for p in projects)
        stream = torch.cuda.Stream()
        stream.wait_stream(torch.cuda.current_stream())
        graphs, width = {}, 1
        if cuda_graph:
            width = min(cuda_graph_steps, steps)
            with torch.cuda.stream(stream):
                graphs = capture_graphs(lambda count: batch.step(count, stream), {1, width})
            torch.cuda.synchronize()
        events = {}
        for i, obs in enumerate(observers):
            for q in obs.barriers():
                events.setdefault(q, []).append(i)
        barriers = set(events)
        if progress:
            barriers.update(range(max(1, steps // 100), steps + 1, max(1, steps // 100)))
        setup_seconds = time.perf_counter() - started
        loop_start = time.perf_counter()
        completed, cancelled, replays = 0, False, 0
        with torch.cuda.stream(stream):
            for target, advance in observation_schedule(steps, width, barriers):
                if cancel is not None and cancel.is_set():
                    cancelled = True
                    break
                if graphs:
                    graphs[advance].replay()
                    replays += 1
                else:
                    batch.step(advance, stream)
                completed = target
                for i in events.get(completed, ()):
                    observers[i].observe(completed)
                if progress and (completed % max(1, steps // 100) == 0 or completed == steps):
                    progress(dict(step=completed, total=steps, cases=len(cases), elapsed=time.perf_counter() - loop_start))
        torch.cuda.synchronize()
        seconds = time.perf_counter() - loop_start
        tiles = batch.tiles()
    finally:
        batch.close()
    items = []
    if root:
        root.mkdir(parents=True, exist_ok=True)
    for i, (case, p, obs, grid) in enumerate(zip(cases, projects, observers, grids)):
        done = min(completed, p.region.steps)
        result = obs.result(done, 'cancelled' if cancelled else 'max_steps', seconds, setup_seconds,
                            cuda_kernel='fused_batch', batch_size=len(cases), batch_index=i, timing_scope='whole_cohort',
                            cuda_graph=bool(graphs), cuda_graph_steps=width, cuda_graph_replays=replays, batch_tiles=tiles)
        grid.close()
        item = BatchItem(case.id, 'cancelled' if cancelled else 'completed', case.parameters, summary=result.summary,
                         pid=os.getpid(), device=str(grid.device), started=wall_started)
        if root:
            path = root / (case.id + '.npz')
            result.save(path)
            item.output = str(path)
        if not cancelled and objective is not None:
            try:
                value = objective(result)
                if not isinstance(value, dict):
                    value = {'objective': value}
                metrics = {str(k): float(v) for k, v in value.items()}
                if not metrics or not all(math.isfinite(v) for v in metrics.values()):
                    raise ValueError('Objective must return finite nonempty scalar metrics.')
                item.metrics = metrics
            except Exception as exc:  # noqa: BLE001 - an objective failure marks only its own item
                item.status, item.error = 'failed', f'{type(exc).__name__}: {exc}'
        if keep_results:
            item.result = result
        item.finished = time.time()
        items.append(item)
    cells = sum(math.prod(p.region.shape) * min(completed, p.region.steps) for p in projects)
    plan = dict(execution='fused_cuda_batch', batch_size=len(cases), device=str(grids[0].device),
                estimated_memory_mb=estimate / 2**20, memory_fraction=memory_fraction, loop_seconds=seconds,
                setup_seconds=setup_seconds, graph=bool(graphs), cuda_graph_steps=width, cuda_graph_replays=replays,
                tiles=tiles, launch=list(launch) if launch is not None else None, tuning=tuning, gcells_per_s=cells / max(seconds, 1e-9) / 1e9, resume=False)
    return BatchReport(items, time.perf_counter() - started, plan)


def _plan(cases, cohort_size):
    _check_cohort_size(cohort_size)
    groups, solo = {}, []
    for index, case in enumerate(cases):
        r = case.project.region
        if r.backend == 'cpu':
            raise ValueError(f'{case.id}: grouped CUDA batch cannot execute a CPU project.')
        if r.complex_fields:
            raise ValueError(f'{case.id}: grouped CUDA batch requires real fields.')
        if r.run_control.auto_shutoff:
            raise ValueError(f'{case.id}: grouped CUDA batch requires fixed-duration runs.')
        if batch_refusal(case.project):
            solo.append(index)
            continue
        key = r.precision
        if key not in groups:
            groups[key] = dict(group=len(groups), signature=hashlib.sha256(repr(key).encode()).hexdigest(),
                               precision=r.precision, indices=[])
        groups[key]['indices'].append(index)
    cohorts = []
    for group in groups.values():
        idx = group['indices']
        for k in range(0, len(idx), cohort_size):
            cohorts.append(dict(group=group['group'], indices=idx[k:k + cohort_size], execution='fused_cuda_batch'))
    for index in solo:
        cohorts.append(dict(group=None, indices=[index], execution='simulation'))
    return dict(execution='grouped_fused_cuda', total_cases=len(cases), cohort_size=cohort_size, group_count=len(groups),
                groups=list(groups.values()), cohorts=cohorts, padding_cells=0, resume=False, result_order='input',
                objective_order='cohort execution')


def plan_grouped_batch(cases, *, cohort_size=MAX_COHORT):
    """Inspect the cohorts without initialising CUDA (reference grouped_batch.py:80-87)."""
    return _plan(as_cases(list(cases)), cohort_size)


def run_grouped_batch(cases, *, cohort_size=MAX_COHORT, objective=None, output_dir=None, keep_results=True, device=0,
                      memory_fraction=.6, cuda_graph=True, cuda_graph_steps=1, cancel=None, progress=None, launch=None):
    """Run mixed projects: batchable 2D TMz cases in fused cohorts by precision, the rest one by one
    through ``Simulation`` (reference grouped_batch.py:90-146). Items come back in input order."""
    import torch
    start = time.perf_counter()
    validate_graph_steps(cuda_graph_steps, cuda_graph)
    cases = as_cases(list(cases))
    plan = _plan(cases, cohort_size)
    if not 0 < memory_fraction <= .9:
        raise ValueError('memory_fraction must be positive and at most .9.')
    if not torch.cuda.is_available():
        raise RuntimeError('Grouped batch requires CUDA.')
    root = Path(output_dir) if output_dir is not None else None
    if root is not None and root.exists():
        raise FileExistsError('Grouped batch output directory exists. Use a new directory.')
    if root is not None:
        root.mkdir(parents=True)
        write_json(root / 'plan.json', plan)
    items, executions = {}, []
    for number, cohort in enumerate(plan['cohorts']):
        if cancel is not None and cancel.is_set():
            break
        chosen = [cases[i] for i in cohort['indices']]
        out = root / f'cohort-{number:04d}' if root else None
        if cohort['execution'] == 'simulation':
            case = chosen[0]
            item = BatchItem(case.id, 'running', case.parameters, pid=os.getpid(), device=f'cuda:{device}', started=time.time())
            with torch.cuda.device(device):
                result = Simulation(case.project).run(cancel=cancel, cuda_graph=cuda_graph, cuda_graph_steps=cuda_graph_steps)
            item.summary, item.status = result.summary, 'cancelled' if result.summary['cancelled'] else 'completed'
            if out is not None:
                out.mkdir(parents=True)
                result.save(out / (case.id + '.npz'))
                item.output = str(out / (case.id + '.npz'))
            if item.status == 'completed' and objective is not None:
                try:
                    value = objective(result)
                    value = value if isinstance(value, dict) else {'objective': value}
                    item.metrics = {str(k): float(v) for k, v in value.items()}
                except Exception as exc:  # noqa: BLE001
                    item.status, item.error = 'failed', f'{type(exc).__name__}: {exc}'
            if keep_results:
                item.result = result
            item.finished = time.time()
            items[case.id] = item
            executions.append(dict(cohort=number, execution='simulation', seconds=result.summary['seconds']))
            continue

        def on_progress(state, number=number, cohort=cohort):
            progress(dict(state, cohort=number, group=cohort['group'], input_indices=cohort['indices'], total_cases=len(cases)))
        report = run_tensor_batch(chosen, cohort_size=len(chosen), objective=objective, output_dir=out,
                                  keep_results=keep_results, device=device, memory_fraction=memory_fraction,
                                  cuda_graph=cuda_graph, cuda_graph_steps=cuda_graph_steps, cancel=cancel,
                                  progress=on_progress if progress else None, launch=launch)
        items.update((item.id, item) for item in report.items)
        executions.append(dict(cohort=number, **report.plan))
    ordered = [items.get(c.id, BatchItem(c.id, 'cancelled', c.parameters)) for c in cases]
    plan.update(executions=executions, cohorts_started=len(executions), seconds=time.perf_counter() - start)
    report = BatchReport(ordered, time.perf_counter() - start, plan)
    if root is not None:
        write_json(root / 'grouped-batch.json', report.as_dict())
    return report

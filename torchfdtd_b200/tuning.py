"""Launch autotuners: measured, interleaved candidate timing on scratch state.

Mirrors the reference's tuners: ``select_launch`` (torchfdtd/reversible_cuda_tuning.py:84-215; interleaved sweeps
of every candidate on scratch copies, winner by median, cached per device and source) and ``tune_tensor_batch``
(torchfdtd/tuning.py:63-160; full-ensemble trials in alternating order, every trial must reproduce identical
physical arrays, winner by median). The knobs here are the B200 kernels' own:

* a single 3D grid: the marching kernel's launch variant, ``lz * 1000 + split * 100 + D * 10 + MINB``
  (z-planes per CTA chunk, interior-tile split, TMA prefetch depth, CTAs per SM);
* a batch of 2D grids: the rows per strip of the batch's strip table (the tile size) and the CTA count of the
  kernel that walks it (one warp per strip, or a persistent grid).

Tuning has a visible up-front cost and never runs implicitly: ``Simulation.run(launch='auto')`` and
``run_tensor_batch(launch='auto')`` ask for it. Candidates run on scratch plans, never on the caller's state;
each candidate advances the same steps from the same zero state, and the tuner checks that every candidate
ends with bitwise identical fields before it reports a winner.
"""
from __future__ import annotations

import hashlib
import json
import statistics
import time
from dataclasses import asdict, dataclass, field

import numpy as np

_CACHE = {}


@dataclass
class LaunchTuning:
    kind: str                     # 'grid' (marching-kernel variant) or 'batch' (persistent CTA count)
    choice: object                # grid: launch variant (int); batch: [ctas, rows per strip]
    median_ms_per_step: float
    candidates: list = field(default_factory=list)
    repeats: int = 0
    steps_per_sample: int = 0
    seconds: float = 0.0
    workload_sha256: str = ''
    hardware: dict = field(default_factory=dict)
    cached: bool = False

    def as_dict(self):
        return asdict(self)


def _hardware(device):
    import torch
    props = torch.cuda.get_device_properties(device)
    return dict(device=device.index if hasattr(device, 'index') else device, gpu=props.name,
                capability=list(torch.cuda.get_device_capability(device)), sms=props.multi_processor_count,
                total_memory_bytes=props.total_memory, torch=torch.__version__, cuda=torch.version.cuda)


def _digest(arrays):
    h = hashlib.sha256()
    for a in arrays:
        a = np.ascontiguousarray(a)
        h.update(str((a.shape, a.dtype.str)).encode())
        h.update(a.tobytes())
    return h.hexdigest()


def _interleaved(runners, repeats, steps, stream):
    """Median ms per step of each runner, timed in alternating order with CUDA events on ``stream``."""
    import torch
    samples = {k: [] for k in runners}
    keys = list(runners)
    for k in keys:                      # warm-up: loads kernels, first touch of the arenas
        runners[k](steps)
    torch.cuda.synchronize()
    for sweep in range(repeats):
        for k in (keys if sweep % 2 == 0 else keys[::-1]):
            start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            start.record(stream)
            runners[k](steps)
            stop.record(stream)
            stop.synchronize()
            samples[k].append(start.elapsed_time(stop) / steps)
    return samples


def grid_candidates(plan):
    """Marching-kernel launch variants worth measuring for a plan."""
    nz = plan.shape[2]
    if plan.dtype == np.float64:
        base = [22, 122]
    else:
        base = [14, 23, 32, 22, 114, 314]
    lz = [v for v in (4, 8, 16) if v < nz]            # planes per chunk around the default (about 12)
    return base + [z * 1000 + 14 for z in lz] if plan.dtype != np.float64 else base + [z * 1000 + 22 for z in lz]


def select_launch(plan, candidates=None, *, steps=8, repeats=5, device=None):
    """Measure marching-kernel launch variants for ``plan`` (a 3D ``GridPlan``) and return a ``LaunchTuning``.

    Scratch plans are created per candidate (all at once when device memory allows, else one candidate at a
    time with the same number of sweeps). Results are cached per (GPU, plan shape, CPML layout, candidates)."""
    import torch
    from .native import NativeGrid
    if plan.dimension != '3d':
        raise ValueError('select_launch tunes the 3D marching kernel; 2D batches use tune_tensor_batch.')
    if isinstance(repeats, bool) or not isinstance(repeats, int) or repeats < 1:
        raise ValueError('repeats must be a positive integer.')
    device = torch.device('cuda', torch.cuda.current_device() if device is None else device)
    candidates = list(dict.fromkeys(candidates or grid_candidates(plan)))
    steps = min(steps, plan.steps // (repeats + 1))      # scratch runs stay within the plan's own steps
    if steps < 1:
        raise ValueError(f'Tuning needs {repeats + 1} steps of scratch state but the plan runs {plan.steps}.')
    key = ('grid', torch.cuda.get_device_name(device), tuple(plan.shape), str(plan.dtype), plan.material_samples,
           tuple((s.forward, s.axis, s.lo, s.hi) for s in plan.segments), tuple(candidates), steps, repeats)
    if key in _CACHE:
        return LaunchTuning(**dict(_CACHE[key], cached=True))
    started = time.perf_counter()
    stream = torch.cuda.Stream(device)
    records, grids = [], {}
    free, _ = torch.cuda.mem_get_info(device)
    together = NativeGrid.plan_bytes(plan) * len(candidates) < 0.6 * free
    with torch.cuda.device(device), torch.cuda.stream(stream):
        for v in candidates:
            try:
                grids[v] = NativeGrid(plan, kernel='march', variant=v)
            except ValueError as exc:
                records.append(dict(variant=v, status='unsupported', reason=str(exc)))
                continue
            if not together:
                grids[v].close()
                grids[v] = None
        if not grids:
            raise ValueError('No launch variant is supported for this plan.')
        if together:
            samples = _interleaved({v: (lambda n, g=g: g.step(n, stream)) for v, g in grids.items()}, repeats, steps, stream)
            digests = {v: _digest(g.get_fields()) for v, g in grids.items()}
            for g in grids.values():
                g.close()
        else:
            samples, digests = {}, {}
            for v in grids:
                g = NativeGrid(plan, kernel='march', variant=v)
                samples.update(_interleaved({v: lambda n: g.step(n, stream)}, repeats, steps, stream))
                digests[v] = _digest(g.get_fields())
                g.close()
    if len(set(digests.values())) != 1:
        raise ArithmeticError('Launch variants changed the physical fields; refusing to tune.')
    for v, s in samples.items():
        records.append(dict(variant=v, status='completed', samples_ms_per_step=s, median_ms_per_step=statistics.median(s)))
    winner = min((r for r in records if r['status'] == 'completed'), key=lambda r: (r['median_ms_per_step'], r['variant']))
    tuning = LaunchTuning('grid', winner['variant'], winner['median_ms_per_step'], records, repeats, steps,
                          time.perf_counter() - started, _plan_sha(plan), _hardware(device))
    _CACHE[key] = tuning.as_dict()
    return tuning


def _plan_sha(plan):
    return hashlib.sha256(json.dumps(plan.project.model_dump(), sort_keys=True, default=str).encode()).hexdigest()


def batch_candidates(sms):
    """Launch shapes worth measuring, as (CTA count, rows per strip, persistent) triples: one launch per step with
    one warp per strip (ctas 0) at 8-64 rows or with 4 or 8 CTAs per SM at the default rows (0); and all steps in
    one cooperative launch (persistent 1) at 16-64 rows."""
    return [(0, 8, 0), (0, 16, 0), (0, 32, 0), (0, 64, 0), (0, 0, 0), (4 * sms, 0, 0), (8 * sms, 0, 0),
            (0, 16, 1), (0, 32, 1), (0, 64, 1)]


def tune_tensor_batch(cases, candidates=None, *, steps=8, repeats=5, device=0, epsilon=None):
    """Measure the batch step kernel's launch shape (persistent CTA count, rows per strip) for a cohort of
    2D TMz projects.

    Each candidate runs on its own scratch copy of the cohort (same plans, zero state); all candidates must
    end with bitwise identical fields. Returns a ``LaunchTuning`` whose ``choice`` is the ``[ctas, rows,
    persistent]`` triple to pass as ``run_tensor_batch(..., launch=choice)``."""
    import torch
    from .batch import _admit, as_cases
    from .native import NativeBatch, NativeGrid
    from .simulation import Simulation
    if isinstance(repeats, bool) or not isinstance(repeats, int) or repeats < 1:
        raise ValueError('repeats must be a positive integer.')
    cases = as_cases(list(cases))
    projects = _admit(cases, .9)
    steps = min(steps, min(p.region.steps for p in projects) // (repeats + 1))
    if steps < 1:
        raise ValueError(f'Tuning needs {repeats + 1} steps of scratch state; every case must run at least that many.')
    plans = [Simulation(p, epsilon=e).plan for p, e in zip(projects, epsilon or [None] * len(projects))]
    dev = torch.device('cuda', device)
    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    candidates = [tuple(int(v) for v in (*c, 0)[:3]) for c in dict.fromkeys(tuple(c) for c in (candidates or batch_candidates(sms)))]
    key = ('batch', torch.cuda.get_device_name(dev), tuple(tuple(p.shape) for p in plans), str(plans[0].dtype),
           tuple(candidates), steps, repeats)
    if key in _CACHE:
        return LaunchTuning(**dict(_CACHE[key], cached=True))
    started = time.perf_counter()
    with torch.cuda.device(dev):
        stream = torch.cuda.Stream(dev)
        cohort_bytes = sum(NativeGrid.plan_bytes(plan) for plan in plans)
        free, _ = torch.cuda.mem_get_info(dev)
        together = cohort_bytes * len(candidates) < 0.6 * free
        samples, digests, strips = {}, {}, {}

        def scratch(c):
            grids = [NativeGrid(plan, kernel='tile2d') for plan in plans]
            b = NativeBatch(grids)
            b.set_launch(c[0], c[1], stream=stream)
            b.set_persistent(bool(c[2]), stream=stream)
            strips[c] = b.tiles()
            return grids, b

        def finish(c, grids, b):
            b.close()
            digests[c] = _digest([a for g in grids for a in g.get_fields()])
            for g in grids:
                g.close()

        with torch.cuda.stream(stream):
            if together:
                sets = {c: scratch(c) for c in candidates}
                samples = _interleaved({c: (lambda n, b=v[1]: b.step(n, stream)) for c, v in sets.items()}, repeats, steps, stream)
                for c, (grids, b) in sets.items():
                    finish(c, grids, b)
            else:
                for c in candidates:
                    grids, b = scratch(c)
                    samples.update(_interleaved({c: lambda n: b.step(n, stream)}, repeats, steps, stream))
                    finish(c, grids, b)
    if len(set(digests.values())) != 1:
        raise ArithmeticError('Launch shapes changed the physical fields; refusing to tune.')
    records = [dict(ctas=c[0], rows=c[1], persistent=c[2], strips=strips[c], status='completed', samples_ms_per_step=v,
                    median_ms_per_step=statistics.median(v)) for c, v in samples.items()]
    winner = min(records, key=lambda r: (r['median_ms_per_step'], -r['persistent'], r['ctas'], r['rows']))
    fingerprint = hashlib.sha256(json.dumps([p.model_dump() for p in projects], sort_keys=True, default=str).encode()).hexdigest()
    tuning = LaunchTuning('batch', [winner['ctas'], winner['rows'], winner['persistent']], winner['median_ms_per_step'], records,
                          repeats, steps,
                          time.perf_counter() - started, fingerprint, _hardware(dev))
    _CACHE[key] = tuning.as_dict()
    return tuning

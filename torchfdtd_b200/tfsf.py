"""Total-field / scattered-field boxes: planning of the live incident line and the surface corrections.

A TFSF box splits the grid into total field (inside the staggered box) and scattered field (outside). The
update of a field sample next to a box face reads a neighbour on the other side, which holds the other kind
of field; the correction adds (or removes) the incident field there, so both sides stay consistent:

    E_o gains  C / eps_b * (M_E curl(H_inc) - curl(M_H H_inc))
    H_o gains -C       * (M_H curl(E_inc) - curl(M_E E_inc))

with M_E, M_H the masks of the box on the E and H Yee lattices. The masks differ only along the derivative
axis of each curl term, so every correction sits on one of the two faces of that axis: a sparse list of
(target sample, incident sample, weight) per family, corner duplicates merged. The incident field is a live
scalar Yee line (field precision, thick CPML at both ends, soft drive 8 cells upstream of the first face)
stepped with the grid: before the grid's E corrections its E half-step runs (the corrections read its old
H); before the H corrections its H half-step runs (they read its new E).

Restates reference ``torchfdtd/tfsf.py:19-160`` (``tfsf_plan``, ``validate_tfsf_materials``,
``surface_maps``, ``line_coefficients``, ``IncidentLine``); the device side is ``csrc/tfsf.cuh``.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .mesh import local_uniform_step
from .plan import CURL_TERMS
from .waveforms import source_time_signal

DRIVE_OFFSET = 24      # drive cell: incident_pml_cells + 24
PROBE_OFFSET = 32      # first face's incident sample: incident_pml_cells + 32


def tfsf_plan(source, region):
    """(normal axis, lower node indices, upper node indices, direction) of a TFSF box after checking it: PML on
    every active face, positive spans, at least three cells per active axis, two interior cells between each
    face and the PML, and equal cell widths across each face."""
    s, r = source, region
    axis = 'xyz'.index(s.normal)
    active = 2 if r.dimension == '2d' else 3
    if axis >= active:
        raise ValueError(f'{s.name}: TFSF propagation must follow an active axis.')
    if any(face.kind != 'pml' for a in range(active) for face in r.boundaries.pair(a)):
        raise ValueError(f'{s.name}: the current isolated TFSF box requires PML on every active face.')
    lo, hi = [], []
    for a, nodes in enumerate(r.mesh_nodes):
        if a >= active:
            lo.append(0)
            hi.append(0)
            continue
        if s.size[a] <= 0:
            raise ValueError(f'{s.name}: TFSF spans must be positive on every active axis.')
        first = int(np.argmin(abs(nodes - (s.center[a] - s.size[a] / 2))))
        last = int(np.argmin(abs(nodes - (s.center[a] + s.size[a] / 2))))
        if last - first < 3:
            raise ValueError(f'{s.name}: the TFSF box needs at least three cells along each active axis.')
        if first < r.pml_layers(a, 0) + 2 or last > r.shape[a] - r.pml_layers(a, 1) - 2:
            raise ValueError(f'{s.name}: leave at least two interior cells between each TFSF face and PML.')
        local_uniform_step(r, a, first - 1, last + 2)
        lo.append(first)
        hi.append(last)
    return axis, tuple(lo), tuple(hi), 1 if s.direction == '+' else -1


def validate_tfsf_materials(project, epsilon):
    """Each face of a TFSF box, with one cell on either side, must hold the homogeneous background."""
    eps = np.asarray(epsilon)
    r = project.region
    active = 2 if r.dimension == '2d' else 3
    for raw in project.sources:
        if not raw.enabled or raw.kind != 'tfsf':
            continue
        _, lo, hi, _ = tfsf_plan(project.resolved_source(raw), r)
        for axis in range(active):
            for boundary in (lo[axis], hi[axis]):
                sl = [slice(l - 1, h + 2) if a < active else slice(None) for a, (l, h) in enumerate(zip(lo, hi))]
                sl[axis] = slice(boundary - 1, boundary + 2)
                if not np.allclose(eps[tuple(sl)], r.background_index**2, rtol=1e-7 if eps.dtype == np.float32 else 1e-13, atol=0):
                    raise ValueError(f'{raw.name}: the TFSF face neighborhood must be homogeneous background. '
                                     'Move the scatterer inside the box.')


def _courant(region, axis, lo, hi):
    return region.rectangular_courant * region.reference_step / local_uniform_step(region, axis, lo[axis] - 1, hi[axis] + 2)


def surface_maps(source, region):
    """{'E' | 'H': (target, sample, weight)}: the flat reference-layout element (cell * 3 + component) each
    correction adds to, the incident-line cell it reads and its float64 weight, sorted by target, with
    corrections of one target from one sample merged and zero weights dropped."""
    axis, lo, hi, d = tfsf_plan(source, region)
    active = 2 if region.dimension == '2d' else 3
    probe = source.incident_pml_cells + PROBE_OFFSET
    entry = lo[axis] if d == 1 else hi[axis]
    electric = {'xyz'.index(f[1]): w for f, w in source.polarization_components}
    magnetic = {3 - axis - c: d * w * (1 if (axis + 1) % 3 == c else -1) for c, w in electric.items()}
    out = {}
    for family, incident in (('E', magnetic), ('H', electric)):
        targets, samples, weights = [], [], []
        for a, c, o, sign in CURL_TERMS:
            if a >= active or c not in incident:
                continue
            courant = _courant(region, a, lo, hi)
            for side in (0, 1):
                # Tangential E faces lie on the lo / hi node planes, tangential H faces half a cell outside.
                face = (lo[a] if side == 0 else hi[a]) - (1 if family == 'H' and side == 0 else 0)
                ranges = []
                for b in range(3):
                    if b >= active:
                        ranges.append(np.array([0]))
                    elif b == a:
                        ranges.append(np.array([face]))
                    else:
                        # A component sits on half-integer positions along its own axis (E) or across it (H).
                        half = (b == o) if family == 'E' else (b != o)
                        ranges.append(np.arange(lo[b], hi[b] + (0 if half else 1)))
                grid = np.meshgrid(*ranges, indexing='ij')
                flat = np.ravel_multi_index(tuple(v.ravel() for v in grid), region.shape) * 3 + o
                j = grid[axis].ravel().copy()
                if a == axis and side == 0:
                    j += -1 if family == 'E' else 1
                sample = probe + d * (j - entry) - (1 if family == 'E' and d == -1 else 0)
                factor = courant / (region.background_index**2) if family == 'E' else courant
                orientation = (-1 if side == 0 else 1) if family == 'E' else (1 if side == 0 else -1)
                targets.append(flat)
                samples.append(sample)
                weights.append(np.full(len(flat), factor * sign * orientation * incident[c]))
        target, sample, weight = np.concatenate(targets), np.concatenate(samples), np.concatenate(weights)
        order = np.lexsort((sample, target))
        target, sample, weight = target[order], sample[order], weight[order]
        first = np.flatnonzero(np.r_[True, (np.diff(target) != 0) | (np.diff(sample) != 0)])
        weight = np.add.reduceat(weight, first)
        target, sample = target[first], sample[first]
        keep = weight != 0
        target, sample, weight = target[keep], sample[keep], weight[keep]
        if len(np.unique(target)) != len(target):
            raise AssertionError('A TFSF target unexpectedly needs multiple incident samples.')
        out[family] = (target, sample, weight)
    return out


def line_coefficients(count, layers, courant, index):
    """Decay b and coupling c of the line's E-family and H-family CPML (float64), cubic grading over
    layers + 1 cells at both ends, attenuation matched to the background wave speed."""
    out = []
    j = np.arange(count, dtype=float)
    for forward in (False, True):
        half = 1 if forward else .5
        depth = np.maximum(layers - j - half, j - (count - layers) + half)
        rho = np.maximum(depth, 0) / (layers + 1)
        sigma = 40 * rho**3 / (layers + 1)
        b = np.exp(-(sigma + 1e-8) * courant / index)
        out.append((b, (b - 1) * sigma / (sigma + 1e-8)))
    return out


@dataclass
class TfsfBox:
    """Everything the device needs for one box: the line and its drive (float64, rounded by the library) and
    the two correction maps."""
    source: object
    count: int
    drive_at: int
    courant: float              # the line's H factor; its E factor is courant / index^2
    index: float
    coefficients: list          # [(b, c) E family, (b, c) H family], float64 (count,)
    drive: np.ndarray           # float64 (steps,)
    maps: dict                  # 'E' / 'H' -> (target, sample, weight)
    norm_weight: float          # diagnostics weight of every line cell

    @property
    def courant_e(self):
        return self.courant / self.index**2


def tfsf_box(source, region):
    axis, lo, hi, _ = tfsf_plan(source, region)
    layers = source.incident_pml_cells
    count = 2 * layers + 64 + hi[axis] - lo[axis]
    courant = _courant(region, axis, lo, hi)
    index = region.background_index
    drive = source_time_signal(source, np.arange(1, region.steps + 1) * region.time_step)
    # The line stands for the whole box in the energy norm: its transverse area times its cell length, in
    # reference-step units.
    active = 2 if region.dimension == '2d' else 3
    area = 1.0
    for a in range(active):
        if a != axis:
            area *= (hi[a] - lo[a]) * local_uniform_step(region, a, lo[a] - 1, hi[a] + 2) / region.reference_step
    area *= local_uniform_step(region, axis, lo[axis] - 1, hi[axis] + 2) / region.reference_step
    return TfsfBox(source, count, layers + DRIVE_OFFSET, courant, index, line_coefficients(count, layers, courant, index),
                   np.asarray(drive, dtype=np.float64), surface_maps(source, region), area)

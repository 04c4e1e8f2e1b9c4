"""Rectilinear mesh nodes: uniform, axis-specific, explicit and graded.

The graded mesh keeps a fine lattice of step ``h`` (the region's ``mesh``, or its ``mesh_steps``)
wherever it must be fine (the PML cells and one interior cell next to them, the user's refinement
boxes, and the automatic boxes around enabled structures, sources and monitors) and coarsens only
the gaps between fine runs. In a gap of length L the requested spacing grows linearly, at rate
ln(grading), from h at either end towards the coarse limit; the nodes equidistribute the metric
s(x) = integral dx / spacing(x), whose ramp part is ln(1 + rate x / h) / rate, so neighbouring cells
differ by at most the grading ratio and no cell is smaller than h.

This is the reference's mesh (``torchfdtd/mesh.py:18-134``, ``configure_auto_mesh`` / ``coarse_gap`` /
``mesh_nodes`` / ``local_uniform_step``). The node coordinates decide every metric, material sample and
source index, so they are computed with the same floating-point operations, in the same order, as the
reference computes them: the results are bitwise equal (pinned by the golden vectors of
tests/golden/make_golden.py).
"""
from __future__ import annotations

import math

import numpy as np


def configure_auto_mesh(project):
    """Set ``region._auto_boxes`` (the fine boxes around enabled objects) and ``region._coarse_limit`` (the
    largest coarse step: ``mesh_max``, tightened to the shortest source wavelength over background index x
    points per wavelength, and never below the fine step)."""
    r = project.region
    boxes = []
    if r.mesh_type == 'graded' and r.mesh_auto_refine:
        from .geometry import object_bounds
        grow = r.axis_steps
        for obj in project.structures:
            if obj.enabled:
                center, size = object_bounds(obj)
                boxes.append((center, tuple(v + 4 * h for v, h in zip(size, grow))))
        for obj in list(project.sources) + list(project.monitors):
            if obj.enabled:
                # Planes keep their whole transverse support fine (a sheet on a coarse transverse grid would be
                # injected or sampled unevenly); points get a box of two fine cells on either side.
                size = obj.size if getattr(obj, 'kind', None) in ('plane', 'field', 'tfsf') else (0, 0, 0)
                boxes.append((tuple(obj.center), tuple(v + 4 * h for v, h in zip(size, grow))))
    r._auto_boxes = tuple(boxes)
    lengths = []
    for raw in project.sources:
        if raw.enabled:
            s = project.resolved_source(raw)
            lengths.append(s.wavelength_start if s.time_definition in ('wavelength', 'frequency') else s.wavelength)
    limit = min(r.mesh_max, min(lengths) / (r.background_index * r.mesh_ppw)) if lengths else r.mesh_max
    r._coarse_limit = max(r.reference_step, limit)


def coarse_gap(length, h, maximum, grading):
    """Node positions over a gap [0, length] of ``round(length / h)`` fine cells, both ends included.

    Falls back to the fine lattice when the gap is too short to coarsen (fewer than five cells, or a metric
    bin count that does not save a cell) or when the equidistributed nodes would break a bound: a cell
    below h, above ``maximum``, or a neighbour ratio above ``grading`` (ends compared with h)."""
    fine = round(length / h)
    lattice = np.arange(fine + 1) * h
    if fine < 5 or maximum <= h * (1 + 1e-12):
        return lattice
    rate = math.log(grading)
    half = length / 2
    ramp = min(half, (maximum - h) / rate)              # distance over which the spacing grows to `maximum`
    s_ramp = math.log1p(rate * ramp / h) / rate          # metric at the end of the ramp
    s_half = s_ramp + (half - ramp) / maximum            # metric at the middle of the gap
    bins = int(math.ceil(2 * s_half))
    if bins >= fine:
        return lattice
    s = np.linspace(0, 2 * s_half, bins + 1)
    folded = np.minimum(s, 2 * s_half - s)               # metric measured from the nearer end
    x = np.where(folded <= s_ramp,
                 h * np.expm1(rate * np.minimum(folded, s_ramp)) / rate,
                 ramp + (folded - s_ramp) * maximum)
    x = np.where(s <= s_half, x, length - x)
    widths = np.diff(x)
    padded = np.r_[h, widths, h]
    ratios = padded[1:] / padded[:-1]
    if (widths.min() < h * (1 - 1e-10) or widths.max() > maximum * (1 + 1e-10)
            or max(ratios.max(), 1 / ratios.min()) > grading * (1 + 1e-9)):
        return lattice
    x[0], x[-1] = 0, length
    return x


def _graded_axis(r, axis, n, boxes):
    h = r.axis_steps[axis]
    low = -n * h / 2
    fine = np.zeros(n, dtype=bool)
    fine[:r.pml_layers(axis, 0) + 1] = True
    fine[-r.pml_layers(axis, 1) - 1:] = True
    for center, size in boxes:
        first = max(0, min(n, math.floor((center[axis] - size[axis] / 2 - low) / h + 1e-10)))
        last = max(0, min(n, math.ceil((center[axis] + size[axis] / 2 - low) / h - 1e-10)))
        fine[first:last] = True
    # Runs of equal flags: fine runs keep the lattice, the others are coarsened.
    edges = np.flatnonzero(np.r_[True, fine[1:] != fine[:-1], True])
    coarse = max(h, min(r.mesh_max, r._coarse_limit or r.mesh_max))
    pieces = []
    for a, b in zip(edges[:-1], edges[1:]):
        run = np.arange(b - a + 1) * h if fine[a] else coarse_gap((b - a) * h, h, coarse, r.mesh_grading)
        pieces.append(low + a * h + run[:-1])
    return np.r_[np.concatenate(pieces), -low]


def mesh_nodes(region):
    """Node coordinates (um) of every axis, cached on the region until a mesh input changes."""
    r = region
    base = r.base_shape
    if r.mesh_type != 'explicit' and max(base) > 1_000_000:
        raise ValueError('Requested fine lattice exceeds one million cells on an axis.')
    boxes = tuple((tuple(b.center), tuple(b.size)) for b in r.mesh_refinements if b.enabled) + tuple(r._auto_boxes)
    key = (r.mesh_type, r.dimension, tuple(r.size), r.mesh, r.mesh_steps, r.mesh_coordinates, r.mesh_max, r.mesh_grading,
           r._coarse_limit, boxes, tuple(r.pml_layers(a, s) for a in range(3) for s in (0, 1)))
    if r._nodes is not None and r._nodes[0] == key:
        return r._nodes[1]
    out = []
    for axis, n in enumerate(base):
        if r.mesh_type == 'explicit':
            nodes = np.asarray(r.mesh_coordinates[axis], dtype=float)
        elif r.dimension == '2d' and axis == 2:
            nodes = np.array([-r.size[2] / 2, r.size[2] / 2])
        elif r.mesh_type == 'uniform':
            nodes = np.arange(n + 1) * r.axis_steps[axis] - n * r.axis_steps[axis] / 2
        else:
            nodes = _graded_axis(r, axis, n, boxes)
        nodes.setflags(write=False)
        out.append(nodes)
    r._nodes = (key, tuple(out))
    return r._nodes[1]


def local_uniform_step(region, axis, start, stop):
    """The spacing of cells [start, stop) on ``axis``, which must be equal: the fine step when they are fine,
    else their mean."""
    widths = np.diff(region.mesh_nodes[axis])[start:stop]
    if not widths.size or not np.allclose(widths, widths[0], rtol=1e-10, atol=0):
        raise ValueError('The source support and neighboring cells must have constant spacing along each active axis.')
    fine = region.axis_steps[axis]
    return fine if np.allclose(widths, fine, rtol=1e-10, atol=0) else float(np.mean(widths))

"""One-way (discrete Huygens) plane sources and the scalar incident line behind them.

A one-way plane launches a normal-incidence wave in one direction only: an E sheet on the Yee plane k and
an H sheet half a cell upstream carry the incident E and H that a wave travelling through the background
would have there, so the two sheets cancel on the upstream side. The incident pair is not a continuum
impedance guess: it is recorded from a scalar 1D Yee line with the grid's Courant number and background
index, driven softly by the source waveform eight cells upstream of the recording point and terminated by
thick CPML, so it carries the grid's own discrete dispersion and delay (reference
``torchfdtd/injection.py:14-116``: ``oneway_plan``, ``_incident_line``, ``oneway_tables``, ``source_terms``).

The line runs once on the host in float64; its E and H samples become two ordinary soft-source terms per
polarization component, added after each family's update like any other soft source.
"""
from __future__ import annotations

import math
from functools import lru_cache

import numpy as np

from .mesh import local_uniform_step
from .waveforms import source_time_signal

# The line: `layers` CPML cells at either end, the drive `layers + 24` cells in, the recording point 8 cells
# downstream of it.
DRIVE_OFFSET = 24
PROBE_OFFSET = 32


def oneway_plan(source, region):
    """(normal axis, E plane index k, direction +1/-1) of a one-way plane, after checking its geometry: PML at
    both ends of the normal axis, periodic transverse faces (zero Bloch phase), a sheet of zero normal span that
    covers the whole transverse cell and is centred on it, two interior cells between it and the PML, and equal
    cell widths around it."""
    r, s = region, source
    axis = 'xyz'.index(s.normal)
    active = 2 if r.dimension == '2d' else 3
    if axis >= active:
        raise ValueError(f'{s.name}: one-way propagation must be along an active axis.')
    if any(face.kind != 'pml' for face in r.boundaries.pair(axis)):
        raise ValueError(f'{s.name}: the propagation axis requires PML at both ends.')
    if s.size[axis] != 0:
        raise ValueError(f'{s.name}: the one-way plane must have zero span along its normal.')
    for a in range(active):
        if a == axis:
            continue
        if any(face.kind not in ('periodic', 'bloch') for face in r.boundaries.pair(a)) or r.bloch_phase[a] != 0:
            raise ValueError(f'{s.name}: normal-incidence planes require periodic transverse boundaries (zero Bloch phase).')
        if s.center[a] != 0 or not math.isclose(s.size[a], r.actual_size[a], rel_tol=1e-10, abs_tol=1e-12):
            raise ValueError(f'{s.name}: the plane must cover the complete transverse unit cell and be centered on it.')
    nodes = r.mesh_nodes[axis]
    k = int(np.argmin(abs(nodes[:-1] - s.center[axis])))
    lo, hi = r.interior_bounds(axis)
    if k < 2 or k + 2 >= len(nodes) or nodes[k - 1] < lo or nodes[k + 2] > hi:
        raise ValueError(f'{s.name}: leave at least two interior cells between the injection plane and PML.')
    local_uniform_step(r, axis, k - 1, k + 2)
    return axis, k, 1 if s.direction == '+' else -1


def _line_cpml(count, layers, courant, index):
    """Decay and coupling of the line's E-family (staggered half a cell) and H-family CPML: cubic grading
    over `layers + 1`, attenuation matched to the background wave speed courant / index."""
    out = []
    j = np.arange(count, dtype=float)
    for forward in (False, True):
        half = 1 if forward else .5
        depth = np.maximum(layers - j - half, j - (count - layers) + half)
        rho = np.maximum(depth, 0) / (layers + 1)
        sigma = 40 * rho**3 / (layers + 1)
        decay = np.exp(-(sigma + 1e-8) * courant / index)
        out.append((decay, np.divide((decay - 1) * sigma, sigma + 1e-8)))
    return out


@lru_cache(maxsize=8)
def incident_line(drive_bytes, courant, index, layers):
    """(E samples, H samples) per step of the scalar incident line (float64, read-only arrays).

    Per step n: the E sample is the line's old H just upstream of the recording point times courant / index^2
    (what the grid's E update will see), then the line's E update (its CPML memory first), the soft drive;
    the H sample is the new E at the recording point times the Courant number, then the line's H update."""
    drive = np.frombuffer(drive_bytes, dtype=np.float64)
    count = 2 * layers + 64
    at, probe = layers + DRIVE_OFFSET, layers + PROBE_OFFSET
    e, h, pe, ph = (np.zeros(count) for _ in range(4))
    (be, ce), (bh, ch) = _line_cpml(count, layers, courant, index)
    electric, magnetic = np.zeros(len(drive)), np.zeros(len(drive))
    ce_line = courant / index**2
    diff = np.zeros(count)
    for n, value in enumerate(drive):
        electric[n] = ce_line * h[probe - 1]
        diff[0] = 0
        diff[1:] = h[1:] - h[:-1]
        pe *= be
        pe += ce * diff
        e -= ce_line * (diff + pe)
        e[at] += value
        magnetic[n] = courant * e[probe]
        diff[:-1] = e[1:] - e[:-1]
        diff[-1] = 0
        ph *= bh
        ph += ch * diff
        h -= courant * (diff + ph)
    electric.setflags(write=False)
    magnetic.setflags(write=False)
    return electric, magnetic


def oneway_tables(source, region):
    """The incident E and H samples of a one-way source at steps 1..steps."""
    drive = source_time_signal(source, np.arange(1, region.steps + 1) * region.time_step)
    axis, k, _ = oneway_plan(source, region)
    courant = region.rectangular_courant * region.reference_step / local_uniform_step(region, axis, k - 1, k + 2)
    return incident_line(np.asarray(drive, dtype=np.float64).tobytes(), courant, region.background_index,
                         source.incident_pml_cells)


def oneway_terms(source, region):
    """Soft-source terms (component, lo, hi, values) of a one-way plane: per polarization component an E sheet on
    plane k and the H sheet of the crossed component on plane k-1 (travelling +) or k (travelling -), whose sign
    makes E x H point along the travel direction."""
    axis, k, direction = oneway_plan(source, region)
    e_values, h_values = oneway_tables(source, region)
    shape = region.shape
    h_at = k - 1 if direction == 1 else k
    out = []
    for component, weight in source.polarization_components:
        transverse = 'xyz'.index(component[1].lower())
        magnetic = 3 - axis - transverse
        cross = 1 if (axis + 1) % 3 == transverse else -1
        lo_e, hi_e = [0, 0, 0], list(shape)
        lo_e[axis], hi_e[axis] = k, k + 1
        lo_h, hi_h = [0, 0, 0], list(shape)
        lo_h[axis], hi_h[axis] = h_at, h_at + 1
        out.append((component, tuple(lo_e), tuple(hi_e), e_values * weight))
        out.append(('H' + 'xyz'[magnetic], tuple(lo_h), tuple(hi_h), h_values * (weight * direction * cross)))
    return out


def validate_oneway_materials(project, epsilon):
    """The three cells around a one-way plane must hold the homogeneous background permittivity."""
    for s in project.sources:
        if not s.enabled or s.injection != 'oneway' or s.kind == 'tfsf':
            continue
        axis, k, _ = oneway_plan(project.resolved_source(s), project.region)
        sl = [slice(None)] * 3
        sl[axis] = slice(k - 1, k + 2)
        expected = project.region.background_index**2
        eps = np.asarray(epsilon)
        if not np.allclose(eps[tuple(sl)], expected, rtol=1e-7 if eps.dtype == np.float32 else 1e-13, atol=0):
            raise ValueError(f'{s.name}: the injection neighborhood must match the homogeneous background index.')

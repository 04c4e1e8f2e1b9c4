"""Host planning: everything the fused kernels need, resolved once in float64.

``plan_grid(project)`` resolves a validated ``Project`` into a ``GridPlan``:
the Yee shape and time base, boundary kinds, the stretched-coordinate CPML
coefficient tables, the staircase permittivity, the soft-source terms with
their sampled waveforms, point traces and the DFT plane interpolation maps.
It restates the reference planners that feed the fused CUDA path:

- shape / dt / Courant: ``torchfdtd/models.py:352-417``;
- CPML segments: ``torchfdtd/boundaries.py:258-355`` (``_prepare_boundaries``);
- staircase permittivity: ``torchfdtd/solver.py:49-111`` (``voxelize``) and
  the inverse permittivity fill ``torchfdtd/solver.py:742-745``;
- source terms: ``torchfdtd/injection.py:117-141``, ``torchfdtd/solver.py:114-149``;
- point traces: ``torchfdtd/solver.py:765,790-796``;
- DFT planes: ``torchfdtd/field_monitors.py:14-79,121-164``.

Features outside the fused nondispersive path are refused here with a
``ValueError`` that names them; nothing falls back to another engine.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field, replace
from itertools import product

import numpy as np

from .geometry import contains, object_bounds
from .spectra import apodization_window, frequency_samples
from .waveforms import source_time_signal

COMPONENTS = ('Ex', 'Ey', 'Ez', 'Hx', 'Hy', 'Hz')
# (derivative axis, input component, output component, curl sign), the order in which the
# reference accumulates curl terms (torchfdtd/boundaries.py:21-23).
CURL_TERMS = ((0, 2, 1, -1), (0, 1, 2, 1),
              (1, 2, 0, 1), (1, 0, 2, -1),
              (2, 1, 0, -1), (2, 0, 1, 1))
FACE_CODES = {'pml': 0, 'periodic': 1, 'pec': 2, 'antisymmetric': 2}


@dataclass
class CPMLSegment:
    """Coefficients of one (family, axis, side) CPML slab over target cells [lo, hi) on ``axis``.

    E-family (backward difference) and H-family (forward difference) slabs have their own
    grading offsets; both curl terms that differentiate along ``axis`` share these tables
    and keep separate psi memories."""
    forward: bool
    axis: int
    side: int
    lo: int
    hi: int
    b: np.ndarray
    c: np.ndarray
    inv_kappa: np.ndarray
    kappa: np.ndarray
    sigma: np.ndarray
    alpha: np.ndarray


@dataclass
class SourceTerm:
    component: str
    lo: tuple
    hi: tuple
    values: np.ndarray          # float64 (steps,), waveform x polarization weight

    @property
    def family(self):
        return 0 if self.component[0] == 'E' else 1

    @property
    def comp(self):
        return 'xyz'.index(self.component[1].lower())


@dataclass
class Trace:
    monitor: object
    component: str
    index: tuple

    @property
    def family(self):
        return 0 if self.component[0] == 'E' else 1

    @property
    def comp(self):
        return 'xyz'.index(self.component[1].lower())


@dataclass
class PlanePlan:
    monitor: object
    plan: dict
    frequency: np.ndarray
    components: tuple
    corner_cells: np.ndarray     # int64 (C, K, P): flat cell index (x*ny+y)*nz+z of each interpolation corner
    corner_weights: np.ndarray   # field dtype (C, K, P)
    windows: tuple               # field dtype (steps,) for E and for H samples: apodization * dt * downsample mask
    complex_dtype: type

    @property
    def ne(self):
        return sum(c.startswith('E') for c in self.components)


@dataclass
class GridPlan:
    project: object
    shape: tuple
    dimension: str
    dtype: type
    courant: float
    time_step: float
    steps: int
    faces: tuple                 # per axis (low kind, high kind)
    pec_upper: dict
    segments: list
    epsilon: np.ndarray
    inv_eps: np.ndarray
    counts: dict
    sources: list
    traces: list
    planes: list
    polarization: str | None = None
    warnings: list = field(default_factory=list)
    metrics: dict = field(default_factory=dict)   # (forward, axis) -> (float64 (n-1,) interior values, wrap value)
    tfsf: list = field(default_factory=list)      # tfsf.TfsfBox per enabled TFSF source, in source order
    ade: list = field(default_factory=list)       # materials.ADEState per dispersive material state

    @property
    def cells(self):
        return math.prod(self.shape)

    @property
    def material_samples(self):
        return 1 if (self.inv_eps if self.inv_eps is not None else self.epsilon).ndim == 3 else 3

    def psi_shapes(self):
        """Shapes of every CPML memory, in the order the reference allocates them (``YeeGrid.memory_states``)."""
        shapes = []
        for forward in (False, True):
            for axis, comp, out, _ in CURL_TERMS:
                if self.shape[axis] == 1:
                    continue
                for seg in self.segments:
                    if seg.forward == forward and seg.axis == axis:
                        s = list(self.shape)
                        s[axis] = seg.hi - seg.lo
                        shapes.append(((forward, axis, comp, seg.side), tuple(s)))
        return shapes

    def metric_table(self, family, axis):
        """Per-target-cell metric factors of one family and axis (float64, length n), or None on an axis whose
        cells all have the reference step. E (family 0) at cell i differences H across the dual cell i-1/i: entry
        i >= 1 is the dual factor i-1, entry 0 the periodic wrap factor. H (family 1) at cell i differences E across
        cell i: entry i <= n-2 is that cell's factor, entry n-1 the wrap factor. A kernel multiplies the plain
        difference by the entry of the cell it updates, before the CPML terms."""
        forward = family == 1
        if (forward, axis) not in self.metrics:
            return None
        values, wrap = self.metrics[forward, axis]
        return np.r_[values, wrap] if forward else np.r_[wrap, values]

    def active_components(self):
        """Field components the kernels advance: all six in 3D, one 2D polarization (or both) in 2D."""
        if self.dimension == '3d' or self.polarization == 'both':
            return COMPONENTS
        return ('Ez', 'Hx', 'Hy') if self.polarization == 'TM' else ('Ex', 'Ey', 'Hz')


# ---- coordinates ---------------------------------------------------------------------------
def field_axes(region, component):
    """Yee sample coordinates (um) of a component: E on its own edge, H on its dual face."""
    axis = 'xyz'.index(component[1].lower())
    offsets = [(.5 if i == axis else 0.) if component[0] == 'E' else (0. if i == axis else .5) for i in range(3)]
    return [np.array([0.]) if region.dimension == '2d' and i == 2 else
            ((nodes[:-1] + nodes[1:]) / 2 if offsets[i] else nodes[:-1])
            for i, nodes in enumerate(region.mesh_nodes)]


def index_at(center, region, component=None):
    if component and region.material_sampling == 'yee':
        return tuple(int(np.argmin(abs(axis - c))) for axis, c in zip(field_axes(region, component), center))
    return tuple(0 if n == 1 else min(n - 1, max(0, int(math.floor((v + s / 2) / region.mesh))))
                 for v, s, n in zip(center, region.actual_size, region.shape))


def source_slice(src, r):
    if src.kind == 'point':
        return tuple(slice(i, i + 1) for i in index_at(src.center, r, src.component))
    parts = []
    if r.material_sampling == 'yee':
        for axis, c, span, n in zip(field_axes(r, src.component), src.center, src.size, r.shape):
            if n == 1:
                parts.append(slice(0, 1))
            elif span == 0:
                k = int(np.argmin(abs(axis - c)))
                parts.append(slice(k, k + 1))
            else:
                idx = np.flatnonzero((axis >= c - span / 2 - 1e-12) & (axis <= c + span / 2 + 1e-12))
                if len(idx) == 0:
                    raise ValueError(f'{src.name} is smaller than one mesh cell.')
                parts.append(slice(int(idx[0]), int(idx[-1]) + 1))
        return tuple(parts)
    for c, span, total, n in zip(src.center, src.size, r.actual_size, r.shape):
        if n == 1:
            parts.append(slice(0, 1))
        elif span == 0:
            k = min(n - 1, max(0, int((c + total / 2) / r.mesh)))
            parts.append(slice(k, k + 1))
        else:
            # Cell centres inside the requested support.
            lo = max(0, int(math.ceil((c - span / 2 + total / 2) / r.mesh - .5)))
            hi = min(n, int(math.floor((c + span / 2 + total / 2) / r.mesh - .5)) + 1)
            if hi <= lo:
                raise ValueError(f'{src.name} is smaller than one mesh cell.')
            parts.append(slice(lo, hi))
    return tuple(parts)


# ---- refusal of features outside the fused nondispersive path -------------------------------
def check_supported(project):
    r = project.region
    if r.interface_method != 'staircase':
        raise ValueError('Subpixel interfaces are not implemented by the fused B200 engine; use interface_method="staircase".')
    if r.complex_fields:
        raise ValueError('The fused CUDA kernel currently supports real fields. Bloch boundaries are not implemented.')
    for axis in range(3):
        for face in r.boundaries.pair(axis):
            if face.kind in ('pmc', 'symmetric'):
                raise ValueError('PMC/symmetric faces are not implemented by the fused B200 engine.')
    if r.pml_dispersion == 'absorber':
        raise ValueError('pml_dispersion="absorber" is not implemented by the fused B200 engine.')
    active = {s.material for s in project.structures if s.enabled}
    for m in project.materials:
        if m.name in active and m.model == 'tensor':
            raise ValueError(f'{m.name}: tensor materials are not implemented by the fused B200 engine.')
    for raw in project.sources:
        s = project.resolved_source(raw)
        if not s.enabled:
            continue
    r.require_resident()


# ---- nonuniform meshes ----------------------------------------------------------------------------
def mesh_metrics(region):
    """Difference scale factors of a nonuniform mesh (reference ``torchfdtd/boundaries.py:276-284``).

    The update works in units of the reference step: on an axis whose cell widths w are not all the reference
    step h, a forward (H) difference across cell i is scaled by h / w[i] and a backward (E) difference across
    the dual cell between centres i and i+1 by h / ((w[i] + w[i+1]) / 2); the periodic wrap uses the last cell
    (H) and the mean of the first and last cells (E). Returns {(forward, axis): (interior float64, wrap)}."""
    out = {}
    if region.mesh_type == 'uniform' and region.mesh_steps is None:
        return out
    h = region.reference_step
    for axis, nodes in enumerate(region.mesh_nodes):
        if region.shape[axis] == 1:
            continue
        widths = np.diff(nodes)
        if np.allclose(widths, h, rtol=1e-10, atol=0):
            continue
        out[True, axis] = (h / widths[:-1], float(h / widths[-1]))
        out[False, axis] = (h / ((widths[1:] + widths[:-1]) / 2), float(2 * h / (widths[0] + widths[-1])))
    return out


# ---- CPML ------------------------------------------------------------------------------------
def cpml_segments(region, courant):
    """The (family, axis, side) CPML slabs of ``YeeGrid._prepare_boundaries``, coefficients in float64."""
    segments = []
    for forward in (False, True):
        for axis in range(3):
            n = region.shape[axis]
            if n == 1:
                continue
            for side, face in enumerate(region.boundaries.pair(axis)):
                if face.kind != 'pml':
                    continue
                layers = region.pml_layers(axis, side)
                base = 0 if side == 0 else n - layers
                # E derivatives are backward differences (targets 1..n-1), H forward (targets 0..n-2).
                active_start, active_stop = (0, n - 1) if forward else (1, n)
                lo, hi = max(base, active_start), min(base + layers, active_stop)
                if lo >= hi:
                    continue
                target = np.arange(lo, hi) - base
                depth = layers - target - (1 if forward else .5) if side == 0 else target + (1 if forward else .5)
                rho = depth / (layers + 1)
                sigma = face.sigma_scale * 40 * rho**face.polynomial / (layers + 1)
                if region.mesh_type == 'explicit' or region.mesh_steps is not None:
                    # Physical grading: depth measured in um from the slab's inner interface, over the slab
                    # thickness plus one cell; sigma scaled by reference step / that length.
                    nodes = region.mesh_nodes[axis]
                    widths = np.diff(nodes)
                    where = nodes[lo + 1:hi + 1] if forward else (nodes[lo:hi] + nodes[lo + 1:hi + 1]) / 2
                    inner = nodes[layers] if side == 0 else nodes[base]
                    span = (nodes[layers] - nodes[0] + widths[layers]) if side == 0 else (nodes[-1] - nodes[base] + widths[base - 1])
                    rho = ((inner - where) if side == 0 else (where - inner)) / span
                    sigma = face.sigma_scale * 40 * region.reference_step / span * rho**face.polynomial
                kappa = 1 + (face.kappa - 1) * rho**face.polynomial
                alpha = face.alpha * (1 - rho)**face.alpha_polynomial
                decay = np.exp(-(sigma / kappa + alpha) * courant)
                denominator = sigma * kappa + alpha * kappa * kappa
                coupling = np.divide((decay - 1) * sigma, denominator, out=np.zeros_like(sigma), where=denominator != 0)
                segments.append(CPMLSegment(forward, axis, side, lo, hi, decay, coupling, 1 / kappa, kappa, sigma, alpha))
    return segments


# ---- material ----------------------------------------------------------------------------------
def _voxelize_at(project, axes, dtype):
    r = project.region
    shape = tuple(len(a) for a in axes)
    eps = np.full(shape, r.background_index**2, dtype=dtype)
    active = {obj.material for obj in project.structures if obj.enabled}
    materials = {m.name: m.instantaneous_epsilon for m in project.materials if m.name in active}
    ids = {m.name: i for i, m in enumerate(project.materials)}
    owner = np.full(shape, -1, dtype=np.int32)     # material index of each sample (-1: background)
    counts = {}
    # Lower mesh order wins; at equal order the later object wins.
    for obj in sorted(project.structures, key=lambda s: -s.mesh_order):
        if not obj.enabled:
            continue
        center, size = object_bounds(obj)
        slices = []
        for axis, c, span in zip(axes, center, size):
            tol = 128 * np.finfo(float).eps * max(abs(c), span, 1e-300)
            slices.append(slice(int(np.searchsorted(axis, c - span / 2 - tol, 'left')),
                                int(np.searchsorted(axis, c + span / 2 + tol, 'right'))))
        slices = tuple(slices)
        if any(s.start == s.stop for s in slices):
            counts[obj.id] = 0
            continue
        xyz = np.meshgrid(*(axis[s] for axis, s in zip(axes, slices)), indexing='ij', sparse=True)
        mask = contains(obj, *xyz)
        eps[slices][mask] = materials[obj.material]
        owner[slices][mask] = ids[obj.material]
        counts[obj.id] = int(np.count_nonzero(mask))
    return eps, counts, owner


def voxelize(project, dtype, with_ownership=False):
    """Staircase permittivity (and, with_ownership, the material index of every sample, -1 for background):
    (nx, ny, nz) at cell centres, or (nx, ny, nz, 3) at the E samples with Yee sampling."""
    r = project.region
    if r.material_sampling == 'yee':
        parts = [_voxelize_at(project, field_axes(r, c), dtype) for c in ('Ex', 'Ey', 'Ez')]
        eps = np.stack([p[0] for p in parts], axis=-1)
        counts = {k: max(p[1].get(k, 0) for p in parts) for k in parts[0][1]}
        owner = np.stack([p[2] for p in parts], axis=-1)
    else:
        axes = [(np.arange(n) + .5) * r.mesh - s / 2 for n, s in zip(r.shape, r.actual_size)]
        if r.dimension == '2d':
            axes[2] = np.array([0.])
        eps, counts, owner = _voxelize_at(project, axes, dtype)
    return (eps, counts, owner) if with_ownership else (eps, counts)


# ---- monitors ----------------------------------------------------------------------------------
def plane_plan(region, monitor):
    axes, widths = [], []
    normal = 'xyz'.index(monitor.normal)
    for a, nodes in enumerate(region.mesh_nodes):
        if region.dimension == '2d' and a == 2:
            axes.append(np.array([0.]))
            widths.append(np.array([1.]))
            continue
        if a == normal:
            position = monitor.center[a]
            if monitor.spatial_interpolation == 'nearest':
                position = nodes[np.argmin(abs(nodes - position))]
            axes.append(np.array([position]))
            widths.append(np.array([1.]))
            continue
        lo, hi = monitor.center[a] - monitor.size[a] / 2, monitor.center[a] + monitor.size[a] / 2
        edges = np.r_[lo, nodes[(nodes > lo + 1e-12) & (nodes < hi - 1e-12)], hi]
        stride = monitor.downsample_xyz[a] if monitor.downsample_xyz is not None else monitor.downsample
        edges = edges[np.r_[np.arange(0, len(edges) - 1, stride), len(edges) - 1]]
        axes.append((edges[:-1] + edges[1:]) / 2)
        widths.append(np.diff(edges) * 1e-6)
    points = np.stack([v.ravel() for v in np.meshgrid(*axes, indexing='ij')], axis=1)
    area = np.prod(np.stack(np.broadcast_arrays(*[v.reshape(tuple(-1 if a == i else 1 for a in range(3)))
                                                   for i, v in enumerate(widths)])), axis=0).ravel()
    return dict(points_um=points, weights=area, shape=tuple(len(a) for a in axes), normal=normal)


def interpolation_map(region, component, points):
    """Trilinear corners of each plane point: flat cell indices (K, P) and float64 weights (K, P)."""
    pairs = []
    for a, coords in enumerate(field_axes(region, component)):
        x = points[:, a]
        n = len(coords)
        if n == 1:
            pairs.append([(np.zeros(len(x), dtype=int), np.ones(len(x)))])
            continue
        low = np.searchsorted(coords, x, side='right') - 1
        high = low + 1
        if region.boundaries.pair(a)[0].kind == 'periodic':
            length = region.actual_size[a]
            lower = coords[low % n] - np.where(low < 0, length, 0)
            upper = coords[high % n] + np.where(high >= n, length, 0)
            q = (x - lower) / (upper - lower)
            pairs.append([(low % n, 1 - q), (high % n, q)])
        else:
            if np.any(x < coords[0] - 1e-10) or np.any(x > coords[-1] + 1e-10):
                raise ValueError('Monitor interpolation extends beyond the Yee grid.')
            low = np.clip(low, 0, n - 2)
            high = low + 1
            q = (x - coords[low]) / (coords[high] - coords[low])
            pairs.append([(low, 1 - q), (high, q)])
    ny, nz = region.shape[1:]
    cells, weights = [], []
    for terms in product(*pairs):
        cells.append((terms[0][0] * ny + terms[1][0]) * nz + terms[2][0])
        weights.append(terms[0][1] * terms[1][1] * terms[2][1])
    return np.array(cells, dtype=np.int64), np.array(weights)


def _plane(project, monitor, dtype):
    r = project.region
    plan = plane_plan(r, monitor)
    frequency = frequency_samples(monitor.spectrum)
    high = r.precision == 'float64' or monitor.dft_precision == 'float64'
    components = monitor.required_fields
    cells, weights = [], []
    for comp in components:
        c, w = interpolation_map(r, comp, plan['points_um'])
        cells.append(c)
        weights.append(w.astype(dtype))
    times = np.arange(1, r.steps + 1) * r.time_step
    mask = (np.arange(r.steps) % monitor.time_downsample == 0) * monitor.time_downsample
    windows = tuple((apodization_window(times + shift, monitor.spectrum) * r.time_step * mask).astype(dtype)
                    for shift in (0, r.time_step / 2))
    return PlanePlan(monitor, plan, frequency, components, np.stack(cells), np.stack(weights), windows,
                     np.complex128 if high else np.complex64)


# ---- the plan ----------------------------------------------------------------------------------
def plan_grid(project, polarization=None, material=True):
    """Resolve a project into a ``GridPlan`` for the fused kernels (refusing unsupported features).
    ``material=False`` skips voxelization (``epsilon`` / ``inv_eps`` stay None) for callers that supply the
    permittivity themselves."""
    check_supported(project)
    r = project.region
    dtype = np.float64 if r.precision == 'float64' else np.float32
    courant = r.rectangular_courant
    faces = tuple(tuple(f.kind for f in r.boundaries.pair(a)) for a in range(3))
    pec_upper = {a: float(r.reference_step / (r.mesh_nodes[a][-1] - r.mesh_nodes[a][-2]))
                 for a in range(3) if r.shape[a] > 1 and faces[a][1] in ('pec', 'antisymmetric')}
    segments = cpml_segments(r, courant)
    metrics = mesh_metrics(r)
    ade = []
    if material:
        eps, counts, owner = voxelize(project, dtype, with_ownership=True)
        from .injection import validate_oneway_materials
        from .tfsf import validate_tfsf_materials
        validate_oneway_materials(project, eps)
        validate_tfsf_materials(project, eps)
        inv_eps = (1 / eps).astype(dtype)
        from .materials import ade_states
        ade = ade_states(project, owner, inv_eps)
        warnings = [f'{obj.name}: no cells intersect this object. Refine mesh or reposition it.'
                    for obj in project.structures if obj.enabled and counts.get(obj.id) == 0]
    else:
        eps = inv_eps = None
        counts, warnings = {}, []
    sources, boxes = [], []
    times = np.arange(1, r.steps + 1) * r.time_step
    for raw in project.sources:
        s = project.resolved_source(raw)
        if not s.enabled:
            continue
        if s.kind == 'tfsf':
            from .tfsf import tfsf_box
            boxes.append(tfsf_box(s, r))
            continue
        if s.injection == 'oneway':
            # A one-way plane: E and H sheets fed by the incident line (injection.oneway_terms).
            from .injection import oneway_terms
            sources.extend(SourceTerm(c, lo, hi, v) for c, lo, hi, v in oneway_terms(s, r))
            continue
        waveform = source_time_signal(s, times + s.time_offset_steps * r.time_step)
        for component, weight in s.polarization_components:
            scalar = s.model_copy(update={'component': component, 'theta': None})
            loc = source_slice(scalar, r)
            sources.append(SourceTerm(component, tuple(p.start for p in loc), tuple(p.stop for p in loc), waveform * weight))
    traces = []
    planes = []
    for raw in project.monitors:
        if not raw.enabled:
            continue
        m = project.resolved_monitor(raw)
        if m.kind == 'point':
            traces.append(Trace(m, m.component, index_at(m.center, r, m.component)))
        else:
            planes.append(_plane(project, m, dtype))
    if r.dimension == '2d' and polarization is None:
        tm = any(t.component in ('Ez', 'Hx', 'Hy') for t in sources)
        te = any(t.component in ('Ex', 'Ey', 'Hz') for t in sources)
        polarization = 'both' if tm and te else ('TE' if te else 'TM')
    if r.dimension == '2d' and polarization != 'both':
        # A 2D polarization leaves the other E components at zero: their pole states stay zero too, so only the
        # samples of the advanced components carry an ADE state.
        keep = (2,) if polarization == 'TM' else (0, 1)
        ade = [st for st in (replace(st, target=st.target[np.isin(st.target % 3, keep)]) for st in ade) if st.samples]
    return GridPlan(project, tuple(r.shape), r.dimension, dtype, courant, r.time_step, r.steps, faces, pec_upper,
                    segments, eps, inv_eps, counts, sources, traces, planes,
                    polarization if r.dimension == '2d' else None, warnings, metrics, boxes, ade)

"""ctypes binding of the C ABI in include/tfdtd.h (libtfdtd.so, built in-tree).

``NativeGrid`` turns a host ``GridPlan`` into a device plan: it fills ``tfd_desc``,
lets PyTorch allocate the one device arena the library lays out (the reference
also keeps every array in torch, ``torchfdtd/cuda_kernels.py:120-128``) and wraps
the entry points. There is no CPU path: without the library or a GPU every entry
point raises.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIBRARY = HERE / 'libtfdtd.so'

TFD_ABI_VERSION = 2
TFD_DEVICE, TFD_HOST = 0, 1
KERNELS = {'auto': 0, 'march': 1, 'gather': 2, 'tile2d': 3}
FACE = {'pml': 0, 'periodic': 1, 'pec': 2, 'antisymmetric': 2}
MASK = {'3d': 0x3F, 'both': 0x3F, 'TM': 0x04 | 0x08 | 0x10, 'TE': 0x01 | 0x02 | 0x20}

c_i32, c_i64, c_dbl, c_vp = ctypes.c_int32, ctypes.c_int64, ctypes.c_double, ctypes.c_void_p
P_dbl = ctypes.POINTER(ctypes.c_double)
P_i32 = ctypes.POINTER(ctypes.c_int32)
P_i64 = ctypes.POINTER(ctypes.c_int64)


class CpmlSegment(ctypes.Structure):
    _fields_ = [('forward', c_i32), ('axis', c_i32), ('lo', c_i32), ('hi', c_i32),
                ('b', P_dbl), ('c', P_dbl), ('inv_kappa', P_dbl)]


class SourceTermC(ctypes.Structure):
    _fields_ = [('family', c_i32), ('component', c_i32), ('lo', c_i32 * 3), ('hi', c_i32 * 3), ('values', P_dbl)]


class TraceC(ctypes.Structure):
    _fields_ = [('family', c_i32), ('component', c_i32), ('index', c_i32 * 3)]


class PlaneC(ctypes.Structure):
    _fields_ = [('points', c_i32), ('frequencies', c_i32), ('components', c_i32), ('corners', c_i32),
                ('component_ids', P_i32), ('corner_cells', P_i64), ('corner_weights', P_dbl),
                ('frequency_hz', P_dbl), ('window_e', P_dbl), ('window_h', P_dbl)]


class TfsfC(ctypes.Structure):
    _fields_ = [('count', c_i32), ('drive_at', c_i32), ('courant_e', c_dbl), ('courant_h', c_dbl), ('index', c_dbl),
                ('norm_weight', c_dbl), ('b', P_dbl * 2), ('c', P_dbl * 2), ('drive', P_dbl), ('n_targets', c_i32 * 2),
                ('target', P_i64 * 2), ('sample', P_i64 * 2), ('weight', P_dbl * 2)]


class AdeC(ctypes.Structure):
    _fields_ = [('samples', c_i32), ('poles', c_i32), ('multiple', c_i32), ('target', P_i64), ('eps_inf', c_dbl),
                ('a', P_dbl), ('d', P_dbl), ('k', P_dbl), ('w0', P_dbl), ('strength', P_dbl), ('weight', P_dbl)]


class Desc(ctypes.Structure):
    _fields_ = [('abi_version', c_i32), ('nx', c_i32), ('ny', c_i32), ('nz', c_i32), ('precision', c_i32),
                ('material_samples', c_i32), ('components', c_i32), ('steps', c_i32), ('kernel', c_i32),
                ('launch_variant', c_i32),
                ('face', (c_i32 * 2) * 3), ('courant', c_dbl), ('time_step', c_dbl), ('pec_upper', c_dbl * 3),
                ('n_segments', c_i32), ('segments', ctypes.POINTER(CpmlSegment)),
                ('n_sources', c_i32), ('sources', ctypes.POINTER(SourceTermC)),
                ('n_traces', c_i32), ('traces', ctypes.POINTER(TraceC)),
                ('n_planes', c_i32), ('planes', ctypes.POINTER(PlaneC)), ('metric', (P_dbl * 3) * 2),
                ('volume', P_dbl * 3), ('n_tfsf', c_i32), ('tfsf', ctypes.POINTER(TfsfC)),
                ('n_ade', c_i32), ('ade', ctypes.POINTER(AdeC))]


# Every entry point of include/tfdtd.h with its ctypes signature.
SIGNATURES = {
    'tfd_plan_bytes': (ctypes.c_int, [ctypes.POINTER(Desc), ctypes.POINTER(ctypes.c_size_t)]),
    'tfd_plan_create': (ctypes.c_int, [ctypes.POINTER(Desc), c_vp, ctypes.c_size_t, c_vp, ctypes.POINTER(c_vp)]),
    'tfd_plan_destroy': (None, [c_vp]),
    'tfd_set_material': (ctypes.c_int, [c_vp, c_vp, ctypes.c_int, c_vp]),
    'tfd_set_permittivity': (ctypes.c_int, [c_vp, c_vp, ctypes.c_int, c_vp]),
    'tfd_field_check': (ctypes.c_int, [c_vp, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(c_i32), c_vp]),
    'tfd_set_fields': (ctypes.c_int, [c_vp, c_vp, c_vp, ctypes.c_int, c_vp]),
    'tfd_get_fields': (ctypes.c_int, [c_vp, c_vp, c_vp, ctypes.c_int, c_vp]),
    'tfd_psi_count': (ctypes.c_int, [c_vp, ctypes.POINTER(ctypes.c_size_t)]),
    'tfd_set_psi': (ctypes.c_int, [c_vp, c_vp, ctypes.c_int, c_vp]),
    'tfd_get_psi': (ctypes.c_int, [c_vp, c_vp, ctypes.c_int, c_vp]),
    'tfd_step': (ctypes.c_int, [c_vp, c_i32, c_vp]),
    'tfd_reset': (ctypes.c_int, [c_vp, c_vp]),
    'tfd_get_traces': (ctypes.c_int, [c_vp, c_vp, ctypes.c_int, c_vp]),
    'tfd_get_plane': (ctypes.c_int, [c_vp, c_i32, c_vp, ctypes.c_int, c_vp]),
    'tfd_get_slice': (ctypes.c_int, [c_vp, c_i32, c_i32, c_i32, c_vp, ctypes.c_int, c_vp]),
    'tfd_diagnose': (ctypes.c_int, [c_vp, P_dbl, c_vp]),
    'tfd_counter': (ctypes.c_int, [c_vp, P_i64, c_vp]),
    'tfd_device_status': (ctypes.c_int, [c_vp, P_i32, c_vp]),
    'tfd_kernel_in_use': (ctypes.c_int, [c_vp, P_i32]),
    'tfd_step_launches': (ctypes.c_int, [c_vp, ctypes.c_int32, ctypes.POINTER(ctypes.c_int64)]),
    'tfd_field_norm_static': (ctypes.c_int, [c_vp, c_vp, c_vp, c_i64, c_i32, c_i32, c_vp, c_vp]),
    'tfd_batch_bytes': (ctypes.c_int, [c_i32, ctypes.POINTER(c_vp), ctypes.POINTER(ctypes.c_size_t)]),
    'tfd_batch_create': (ctypes.c_int, [c_i32, ctypes.POINTER(c_vp), c_vp, ctypes.c_size_t, c_vp, ctypes.POINTER(c_vp)]),
    'tfd_batch_set_launch': (ctypes.c_int, [c_vp, c_i32, c_i32, c_vp]),
    'tfd_batch_set_persistent': (ctypes.c_int, [c_vp, c_i32, c_vp]),
    'tfd_batch_step': (ctypes.c_int, [c_vp, c_i32, c_vp]),
    'tfd_batch_tiles': (ctypes.c_int, [c_vp, P_i32]),
    'tfd_batch_destroy': (None, [c_vp]),
    'tfd_state_bytes': (ctypes.c_int, [c_vp, ctypes.POINTER(ctypes.c_size_t)]),
    'tfd_state_save': (ctypes.c_int, [c_vp, c_vp, c_vp]),
    'tfd_state_load': (ctypes.c_int, [c_vp, c_vp, c_vp]),
    'tfd_adjoint_bytes': (ctypes.c_int, [c_vp, ctypes.POINTER(ctypes.c_size_t)]),
    'tfd_adjoint_create': (ctypes.c_int, [c_vp, c_vp, ctypes.c_size_t, c_vp, ctypes.POINTER(c_vp)]),
    'tfd_adjoint_reset': (ctypes.c_int, [c_vp, c_vp]),
    'tfd_adjoint_step': (ctypes.c_int, [c_vp, c_vp, c_vp, c_vp]),
    'tfd_adjoint_sensitivity': (ctypes.c_int, [c_vp, c_vp, ctypes.c_int, c_vp]),
    'tfd_adjoint_destroy': (None, [c_vp]),
    'tfd_error_string': (ctypes.c_char_p, [ctypes.c_int]),
    'tfd_last_error': (ctypes.c_char_p, []),
}

_lib = None


def library():
    """Load libtfdtd.so once; raise when it has not been built (there is no fallback)."""
    global _lib
    if _lib is None:
        if not LIBRARY.exists():
            raise RuntimeError(f'{LIBRARY.name} is not built. Build it with `python __graft_entry__.py` (build()) or '
                               '`make -C torchfdtd_b200/csrc`; the fused B200 engine has no CPU fallback.')
        lib = ctypes.CDLL(str(LIBRARY))
        for name, (restype, argtypes) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = restype
            fn.argtypes = argtypes
        _lib = lib
    return _lib


class NativeError(RuntimeError):
    pass


def check(code):
    if code != 0:
        lib = library()
        message = lib.tfd_last_error().decode()
        kind = lib.tfd_error_string(code).decode()
        if code in (1, 2):
            raise ValueError(f'{kind}: {message}')
        raise NativeError(f'{kind}: {message}')


def _ptr(array, ctype):
    return array.ctypes.data_as(ctypes.POINTER(ctype))


def _stream(stream=None):
    import torch
    s = stream if stream is not None else torch.cuda.current_stream()
    return c_vp(s.cuda_stream)


_STAGING = {}


def staging_ring(dtype, chunk_bytes=32 << 20, depth=4):
    """The pinned staging buffers of ``download`` for a torch dtype (allocated once per process)."""
    import torch
    itemsize = torch.empty(0, dtype=dtype).element_size()
    step = max(1, chunk_bytes // itemsize)
    key = (dtype, step, depth)
    if key not in _STAGING:
        _STAGING[key] = [torch.empty(step, dtype=dtype, pin_memory=True) for _ in range(depth)]
    return _STAGING[key]


def host_buffer(shape, dtype, slab_bytes=64 << 20, workers=8):
    """A pageable host array whose pages are already mapped (one byte written per 4 KiB page, a slab at a
    time), so that a later ``download(..., out=...)`` copies without page faults. Large arrays come from an
    anonymous mapping advised for transparent huge pages where the kernel offers them (one fault per 2 MiB
    instead of per 4 KiB). The cost is the kernel zeroing each new page on the faulting core, so up to
    ``workers`` threads touch the slabs (numpy releases the GIL while it writes). Host memory only: meant to
    run on a helper thread while the device works."""
    import mmap
    import os
    dtype = np.dtype(dtype)
    nbytes = int(np.prod(shape)) * dtype.itemsize
    out = None
    if nbytes >= (64 << 20) and hasattr(mmap, 'MADV_HUGEPAGE'):
        try:
            region = mmap.mmap(-1, nbytes, flags=mmap.MAP_PRIVATE | mmap.MAP_ANONYMOUS)
            region.madvise(mmap.MADV_HUGEPAGE)
            out = np.frombuffer(region, dtype=dtype).reshape(shape)
        except (OSError, ValueError):
            out = None
    if out is None:
        out = np.empty(shape, dtype=dtype)
    raw = out.reshape(-1).view(np.uint8)
    slabs = range(0, raw.size, slab_bytes)

    def touch(a):
        raw[a:a + slab_bytes:4096] = 0

    workers = max(1, min(workers, len(os.sched_getaffinity(0)) if hasattr(os, 'sched_getaffinity') else os.cpu_count() or 1,
                         len(slabs)))
    if workers > 1:
        from concurrent.futures import ThreadPoolExecutor
        with ThreadPoolExecutor(workers) as pool:
            list(pool.map(touch, slabs))
    else:
        for a in slabs:
            touch(a)
    return out


def download(tensor, chunk_bytes=32 << 20, depth=4, direct_bytes=64 << 20, out=None):
    """A contiguous device tensor as a host numpy array. Up to ``direct_bytes``: one plain copy. Larger:
    device-to-host copies of chunk_bytes into a ring of ``depth`` pinned staging buffers (allocated once per
    process and dtype), each drained into the pageable result by a host thread while later chunks are in
    flight. Page-locking the whole result would cost more than it saves on a first call (about 0.5 s per GB
    here); a plain pageable copy runs at about 5 GB/s. ``out``: a C-contiguous host array of the tensor's shape
    and dtype to fill (``host_buffer``) instead of a new one."""
    import torch
    from concurrent.futures import ThreadPoolExecutor
    np_dtype = torch.empty(0, dtype=tensor.dtype).numpy().dtype
    if out is not None and (out.shape != tuple(tensor.shape) or out.dtype != np_dtype or not out.flags.c_contiguous):
        raise ValueError('out must be a C-contiguous host array of the tensor shape and dtype')
    if tensor.numel() * tensor.element_size() <= direct_bytes:
        if out is None:
            return tensor.detach().cpu().numpy()
        np.copyto(out, tensor.detach().cpu().numpy())
        return out
    src = tensor.detach().reshape(-1)
    if out is None:
        out = np.empty(tuple(tensor.shape), dtype=np_dtype)
    flat = out.reshape(-1)
    n = src.numel()
    if n == 0:
        return out
    step = max(1, chunk_bytes // src.element_size())
    ring = staging_ring(src.dtype, chunk_bytes, depth)
    views = [b.numpy() for b in ring]
    stream = torch.cuda.current_stream(src.device)
    pending = [None] * depth

    def drain(event, k, a, b):
        event.synchronize()
        np.copyto(flat[a:b], views[k][:b - a])

    with ThreadPoolExecutor(max_workers=depth) as pool:
        for i, a in enumerate(range(0, n, step)):
            b = min(n, a + step)
            k = i % depth
            if pending[k] is not None:
                pending[k].result()
            ring[k][:b - a].copy_(src[a:b], non_blocking=True)
            event = torch.cuda.Event()
            event.record(stream)
            pending[k] = pool.submit(drain, event, k, a, b)
        for f in pending:
            if f is not None:
                f.result()
    return out


def describe(plan, kernel='auto', variant=0):
    """The C descriptor of a plan and the host arrays it points into (keep them alive while it is used)."""
    keep = []
    desc = Desc()
    desc.abi_version = TFD_ABI_VERSION
    desc.nx, desc.ny, desc.nz = plan.shape
    desc.precision = 8 if plan.dtype == np.float64 else 4
    desc.material_samples = plan.material_samples
    desc.components = MASK['3d' if plan.dimension == '3d' else plan.polarization]
    desc.steps = plan.steps
    desc.kernel = KERNELS[kernel]
    desc.launch_variant = int(variant)
    for a in range(3):
        for s in range(2):
            desc.face[a][s] = FACE[plan.faces[a][s]]
        desc.pec_upper[a] = plan.pec_upper.get(a, 0.0)
    desc.courant = plan.courant
    desc.time_step = plan.time_step
    segs = (CpmlSegment * max(1, len(plan.segments)))()
    for k, s in enumerate(plan.segments):
        arrays = [np.ascontiguousarray(v, dtype=np.float64) for v in (s.b, s.c, s.inv_kappa)]
        keep.extend(arrays)
        segs[k] = CpmlSegment(int(s.forward), s.axis, s.lo, s.hi, *(_ptr(v, ctypes.c_double) for v in arrays))
    desc.n_segments, desc.segments = len(plan.segments), segs
    srcs = (SourceTermC * max(1, len(plan.sources)))()
    for k, t in enumerate(plan.sources):
        v = np.ascontiguousarray(t.values, dtype=np.float64)
        keep.append(v)
        srcs[k] = SourceTermC(t.family, t.comp, (c_i32 * 3)(*t.lo), (c_i32 * 3)(*t.hi), _ptr(v, ctypes.c_double))
    desc.n_sources, desc.sources = len(plan.sources), srcs
    traces = (TraceC * max(1, len(plan.traces)))()
    for k, t in enumerate(plan.traces):
        traces[k] = TraceC(t.family, t.comp, (c_i32 * 3)(*t.index))
    desc.n_traces, desc.traces = len(plan.traces), traces
    planes = (PlaneC * max(1, len(plan.planes)))()
    for k, p in enumerate(plan.planes):
        ids = np.array([['Ex', 'Ey', 'Ez', 'Hx', 'Hy', 'Hz'].index(c) for c in p.components], dtype=np.int32)
        cells = np.ascontiguousarray(p.corner_cells, dtype=np.int64)
        weights = np.ascontiguousarray(p.corner_weights, dtype=np.float64)
        freq = np.ascontiguousarray(p.frequency, dtype=np.float64)
        we = np.ascontiguousarray(p.windows[0], dtype=np.float64)
        wh = np.ascontiguousarray(p.windows[1], dtype=np.float64)
        keep.extend([ids, cells, weights, freq, we, wh])
        planes[k] = PlaneC(cells.shape[2], len(freq), len(ids), cells.shape[1], _ptr(ids, c_i32), _ptr(cells, c_i64),
                           _ptr(weights, ctypes.c_double), _ptr(freq, ctypes.c_double), _ptr(we, ctypes.c_double),
                           _ptr(wh, ctypes.c_double))
    desc.n_planes, desc.planes = len(plan.planes), planes
    for f in range(2):
        for a in range(3):
            table = plan.metric_table(f, a) if hasattr(plan, 'metric_table') else None
            if table is not None:
                table = np.ascontiguousarray(table, dtype=np.float64)
                keep.append(table)
                desc.metric[f][a] = _ptr(table, ctypes.c_double)
    region = plan.project.region if plan.project is not None else None
    if region is not None and (region.mesh_type != 'uniform' or region.mesh_steps is not None):
        # Diagnostics cell volumes of a nonuniform mesh: widths over the reference step, every axis.
        for a, nodes in enumerate(region.mesh_nodes):
            if plan.shape[a] > 1:
                w = np.ascontiguousarray(np.diff(nodes) / region.reference_step, dtype=np.float64)
                keep.append(w)
                desc.volume[a] = _ptr(w, ctypes.c_double)
    boxes = getattr(plan, 'tfsf', [])
    tf = (TfsfC * max(1, len(boxes)))()
    for k, box in enumerate(boxes):
        t = tf[k]
        t.count, t.drive_at = box.count, box.drive_at
        t.courant_e, t.courant_h, t.index, t.norm_weight = box.courant_e, box.courant, box.index, box.norm_weight
        drive = np.ascontiguousarray(box.drive, dtype=np.float64)
        keep.append(drive)
        t.drive = _ptr(drive, ctypes.c_double)
        for f, family in enumerate(('E', 'H')):
            b, c = (np.ascontiguousarray(v, dtype=np.float64) for v in box.coefficients[f])
            target, sample, weight = (np.ascontiguousarray(box.maps[family][0], dtype=np.int64),
                                      np.ascontiguousarray(box.maps[family][1], dtype=np.int64),
                                      np.ascontiguousarray(box.maps[family][2], dtype=np.float64))
            keep.extend([b, c, target, sample, weight])
            t.b[f], t.c[f] = _ptr(b, ctypes.c_double), _ptr(c, ctypes.c_double)
            t.n_targets[f] = len(target)
            t.target[f], t.sample[f], t.weight[f] = _ptr(target, c_i64), _ptr(sample, c_i64), _ptr(weight, ctypes.c_double)
    desc.n_tfsf, desc.tfsf = len(boxes), tf
    states = getattr(plan, 'ade', [])
    ade = (AdeC * max(1, len(states)))()
    nonuniform = region is not None and (region.mesh_type != 'uniform' or region.mesh_steps is not None)
    for k, st in enumerate(states):
        m = ade[k]
        m.samples, m.poles, m.multiple, m.eps_inf = st.samples, st.poles, int(st.multiple), st.eps_inf
        arrays = [np.ascontiguousarray(st.target, dtype=np.int64)] + [np.ascontiguousarray(getattr(st, f), dtype=np.float64)
                                                                      for f in ('a', 'd', 'k', 'w0', 'strength')]
        keep.extend(arrays)
        m.target = _ptr(arrays[0], c_i64)
        m.a, m.d, m.k, m.w0, m.strength = (_ptr(v, ctypes.c_double) for v in arrays[1:])
        if nonuniform:
            # The state norm weighs each sample by its cell's volume in reference-step units.
            widths = [np.diff(nodes) / region.reference_step if n > 1 else np.ones(1)
                      for nodes, n in zip(region.mesh_nodes, plan.shape)]
            cell = st.target // 3
            x, y, z = np.unravel_index(cell, plan.shape)
            w = np.ascontiguousarray(widths[0][x] * widths[1][y] * widths[2][z], dtype=np.float64)
            keep.append(w)
            m.weight = _ptr(w, ctypes.c_double)
    desc.n_ade, desc.ade = len(states), ade
    keep.extend([segs, srcs, traces, planes, tf, ade])
    return desc, keep


class NativeGrid:
    """A device plan built from a ``GridPlan`` (owns the arena tensor and the native handle)."""

    @staticmethod
    def plan_bytes(plan, kernel='auto'):
        """Device bytes the plan's arena needs (no device work)."""
        desc, keep = describe(plan, kernel)
        size = ctypes.c_size_t()
        check(library().tfd_plan_bytes(ctypes.byref(desc), ctypes.byref(size)))
        return size.value

    def __init__(self, plan, kernel='auto', device=None, variant=0, material=None, permittivity=None):
        """``material``: the inverse permittivity to load instead of ``plan.inv_eps`` (a host array or a device
        tensor, as for ``set_material``). ``permittivity``: the relative permittivity instead, checked and
        inverted on the device (``set_permittivity``)."""
        import time
        import torch
        if not torch.cuda.is_available():
            raise RuntimeError('CUDA requested but unavailable: the fused B200 engine runs on a CUDA GPU only.')
        t0 = time.perf_counter()
        lib = library()
        self.plan = plan
        self.device = torch.device('cuda', torch.cuda.current_device() if device is None else device)
        self.dtype = plan.dtype
        self.torch_dtype = torch.float64 if plan.dtype == np.float64 else torch.float32
        desc, self._keep = describe(plan, kernel, variant)
        self.desc = desc
        size = ctypes.c_size_t()
        check(lib.tfd_plan_bytes(ctypes.byref(desc), ctypes.byref(size)))
        self.arena_bytes = size.value
        with torch.cuda.device(self.device):
            self.arena = torch.empty(self.arena_bytes, dtype=torch.uint8, device=self.device)
            handle = c_vp()
            check(lib.tfd_plan_create(ctypes.byref(desc), c_vp(self.arena.data_ptr()), size, _stream(), ctypes.byref(handle)))
        self.handle = handle
        kernel_used = c_i32()
        check(lib.tfd_kernel_in_use(self.handle, ctypes.byref(kernel_used)))
        self.kernel = {v: k for k, v in KERNELS.items()}[kernel_used.value]
        torch.cuda.synchronize(self.device)
        t1 = time.perf_counter()
        if permittivity is not None:
            self.set_permittivity(permittivity)
        else:
            self.set_material(plan.inv_eps if material is None else material)
        torch.cuda.synchronize(self.device)
        # Host seconds of the set-up phases (device work included): arena allocation + plan creation, and the
        # material upload (with the permittivity check and inversion when it is done on the device).
        self.timing = {'arena_and_plan_create': t1 - t0, 'material_upload': time.perf_counter() - t1}

    # ---- restart states (checkpoints of the discrete adjoint) ------------------------------------
    def state_bytes(self):
        v = ctypes.c_size_t()
        check(library().tfd_state_bytes(self.handle, ctypes.byref(v)))
        return v.value

    def save_state(self, snapshot, stream=None):
        """Copy the restart state into ``snapshot`` (a 256-byte aligned uint8 device tensor)."""
        check(library().tfd_state_save(self.handle, c_vp(snapshot.data_ptr()), _stream(stream)))

    def load_state(self, snapshot, stream=None):
        check(library().tfd_state_load(self.handle, c_vp(snapshot.data_ptr()), _stream(stream)))

    def close(self):
        if getattr(self, 'batch', None) is not None:
            self.batch.close()
        if getattr(self, 'handle', None):
            library().tfd_plan_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001 - interpreter shutdown
            pass

    # ---- state transfer (reference layout, host numpy arrays) --------------------------------
    def set_material(self, inv_eps):
        """Inverse permittivity in the reference layout: a host array, or a contiguous device tensor of the
        plan's dtype (stream-ordered, no host copy)."""
        if hasattr(inv_eps, 'data_ptr'):
            t = inv_eps.contiguous()
            if t.dtype != self.torch_dtype or t.device != self.device:
                raise ValueError('device inverse permittivity must be a tensor of the plan dtype on its device')
            self._material_tensor = t
            check(library().tfd_set_material(self.handle, c_vp(t.data_ptr()), TFD_DEVICE, _stream()))
            return
        a = np.ascontiguousarray(inv_eps, dtype=self.dtype)
        check(library().tfd_set_material(self.handle, c_vp(a.ctypes.data), TFD_HOST, _stream()))

    def set_permittivity(self, eps):
        """Relative permittivity in the reference layout (a host array, or a contiguous device tensor of the
        plan's dtype): checked (finite, at least 1; ValueError otherwise) and inverted on the device."""
        if hasattr(eps, 'data_ptr'):
            t = eps.contiguous()
            if t.dtype != self.torch_dtype or t.device != self.device:
                raise ValueError('device permittivity must be a tensor of the plan dtype on its device')
            check(library().tfd_set_permittivity(self.handle, c_vp(t.data_ptr()), TFD_DEVICE, _stream()))
            return
        a = np.ascontiguousarray(eps, dtype=self.dtype)
        check(library().tfd_set_permittivity(self.handle, c_vp(a.ctypes.data), TFD_HOST, _stream()))

    def field_check(self):
        """(largest |E|, every E and H value finite) over the current fields, computed on the device."""
        peak, finite = ctypes.c_double(), c_i32()
        check(library().tfd_field_check(self.handle, ctypes.byref(peak), ctypes.byref(finite), _stream()))
        return peak.value, bool(finite.value)

    def set_fields(self, E=None, H=None):
        e = None if E is None else np.ascontiguousarray(E, dtype=self.dtype)
        h = None if H is None else np.ascontiguousarray(H, dtype=self.dtype)
        check(library().tfd_set_fields(self.handle, c_vp(e.ctypes.data) if e is not None else None,
                                       c_vp(h.ctypes.data) if h is not None else None, TFD_HOST, _stream()))

    def get_fields(self):
        shape = (*self.plan.shape, 3)
        E, H = np.empty(shape, self.dtype), np.empty(shape, self.dtype)
        check(library().tfd_get_fields(self.handle, c_vp(E.ctypes.data), c_vp(H.ctypes.data), TFD_HOST, _stream()))
        return E, H

    def fields_device(self):
        """E and H as torch tensors in the reference layout, on the device (no host copy)."""
        import torch
        shape = (*self.plan.shape, 3)
        E = torch.empty(shape, dtype=self.torch_dtype, device=self.device)
        H = torch.empty(shape, dtype=self.torch_dtype, device=self.device)
        check(library().tfd_get_fields(self.handle, c_vp(E.data_ptr()), c_vp(H.data_ptr()), TFD_DEVICE, _stream()))
        return E, H

    def psi_count(self):
        n = ctypes.c_size_t()
        check(library().tfd_psi_count(self.handle, ctypes.byref(n)))
        return n.value

    def get_psi(self):
        """Every CPML memory, as a list in the reference's memory_states order and shapes."""
        flat = np.empty(self.psi_count(), self.dtype)
        if flat.size:
            check(library().tfd_get_psi(self.handle, c_vp(flat.ctypes.data), TFD_HOST, _stream()))
        out, off = [], 0
        for _, shape in self.plan.psi_shapes():
            size = int(np.prod(shape))
            out.append(flat[off:off + size].reshape(shape))
            off += size
        return out

    def set_psi(self, arrays):
        flat = np.ascontiguousarray(np.concatenate([np.asarray(a, dtype=self.dtype).ravel() for a in arrays]))
        if flat.size != self.psi_count():
            raise ValueError('CPML memory count differs from the plan.')
        if flat.size:
            check(library().tfd_set_psi(self.handle, c_vp(flat.ctypes.data), TFD_HOST, _stream()))

    # ---- time stepping -------------------------------------------------------------------------
    def step(self, n=1, stream=None):
        check(library().tfd_step(self.handle, int(n), _stream(stream)))

    def reset(self):
        check(library().tfd_reset(self.handle, _stream()))

    def step_launches(self, n):
        """Kernel launches that ``step(n)`` issues."""
        v = c_i64()
        check(library().tfd_step_launches(self.handle, int(n), ctypes.byref(v)))
        return v.value

    def counter(self):
        v = c_i64()
        check(library().tfd_counter(self.handle, ctypes.byref(v), _stream()))
        return v.value

    def device_status(self):
        v = c_i32()
        check(library().tfd_device_status(self.handle, ctypes.byref(v), _stream()))
        return v.value

    # ---- observations ----------------------------------------------------------------------------
    def traces_device(self):
        """The (steps, traces) record as a torch tensor on the device."""
        import torch
        out = torch.zeros((self.plan.steps, len(self.plan.traces)), dtype=self.torch_dtype, device=self.device)
        if out.numel():
            check(library().tfd_get_traces(self.handle, c_vp(out.data_ptr()), TFD_DEVICE, _stream()))
        return out

    def get_traces(self):
        out = np.zeros((self.plan.steps, len(self.plan.traces)), self.dtype)
        if out.size:
            check(library().tfd_get_traces(self.handle, c_vp(out.ctypes.data), TFD_HOST, _stream()))
        return out

    def get_plane(self, k):
        p = self.plan.planes[k]
        out = np.zeros((len(p.frequency), p.corner_cells.shape[2], len(p.components)), np.complex128)
        if out.size:
            check(library().tfd_get_plane(self.handle, k, c_vp(out.ctypes.data), TFD_HOST, _stream()))
        return out

    def get_slice(self, component, axis, index):
        n = list(self.plan.shape)
        n.pop(axis)
        out = np.empty(n, self.dtype)
        c = ['Ex', 'Ey', 'Ez', 'Hx', 'Hy', 'Hz'].index(component) if isinstance(component, str) else int(component)
        check(library().tfd_get_slice(self.handle, c, axis, int(index), c_vp(out.ctypes.data), TFD_HOST, _stream()))
        return out

    def field_norm_static(self, E, H, inv_eps, out):
        """Energy and peak of device tensors E, H (cells x 3) and inv_eps through the allocation-free entry
        point; `out` is a 2-element float64 device tensor. For callers that must not allocate (see
        include/tfdtd.h)."""
        cells = E.numel() // 3
        samples = inv_eps.numel() // max(cells, 1)
        check(library().tfd_field_norm_static(c_vp(E.data_ptr()), c_vp(H.data_ptr()), c_vp(inv_eps.data_ptr()), cells, samples,
                                              E.element_size(), c_vp(out.data_ptr()), _stream()))

    def diagnose(self):
        out = (ctypes.c_double * 3)()
        check(library().tfd_diagnose(self.handle, out, _stream()))
        return float(out[0]), float(out[1]), bool(out[2] == 1.0)


class NativeBatch:
    """Independent 2D TMz plans advanced together: one persistent launch per step over all their tiles."""

    def __init__(self, grids):
        import torch
        lib = library()
        self.grids = list(grids)
        if not self.grids:
            raise ValueError('A batch needs at least one grid.')
        handles = (c_vp * len(self.grids))(*[g.handle.value for g in self.grids])
        self._handles = handles
        size = ctypes.c_size_t()
        check(lib.tfd_batch_bytes(len(self.grids), handles, ctypes.byref(size)))
        self.arena = torch.empty(size.value, dtype=torch.uint8, device=self.grids[0].device)
        handle = c_vp()
        check(lib.tfd_batch_create(len(self.grids), handles, c_vp(self.arena.data_ptr()), size, _stream(), ctypes.byref(handle)))
        self.handle = handle
        for g in self.grids:
            g.batch = self

    def set_launch(self, ctas=0, rows=0, stream=None):
        """Persistent CTA count (0: one warp per strip) and rows per strip (0: default) of the step kernel."""
        check(library().tfd_batch_set_launch(self.handle, int(ctas), int(rows), _stream(stream)))

    def set_persistent(self, on=True, stream=None):
        """All steps of a ``step`` call in one cooperative launch (True) or one launch per step (False)."""
        check(library().tfd_batch_set_persistent(self.handle, int(bool(on)), _stream(stream)))
        self.persistent = bool(on)

    def tiles(self):
        v = c_i32()
        check(library().tfd_batch_tiles(self.handle, ctypes.byref(v)))
        return v.value

    def step(self, n=1, stream=None):
        check(library().tfd_batch_step(self.handle, int(n), _stream(stream)))

    def close(self):
        if getattr(self, 'handle', None):
            library().tfd_batch_destroy(self.handle)
            self.handle = None
            for g in self.grids:
                g.batch = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001 - interpreter shutdown
            pass


class NativeAdjoint:
    """The discrete adjoint of a plan (its traces are the observers); owns its arena tensor."""

    def __init__(self, grid):
        import torch
        self.grid = grid
        lib = library()
        size = ctypes.c_size_t()
        check(lib.tfd_adjoint_bytes(grid.handle, ctypes.byref(size)))
        self.arena = torch.empty(size.value, dtype=torch.uint8, device=grid.device)
        handle = c_vp()
        check(lib.tfd_adjoint_create(grid.handle, c_vp(self.arena.data_ptr()), size, _stream(), ctypes.byref(handle)))
        self.handle = handle

    def reset(self, stream=None):
        check(library().tfd_adjoint_reset(self.handle, _stream(stream)))

    def step(self, snapshot, seeds=None, stream=None):
        """Transpose the step that left ``snapshot``'s state, after adding ``seeds`` (one per trace)."""
        check(library().tfd_adjoint_step(self.handle, c_vp(snapshot.data_ptr()),
                                         c_vp(seeds.data_ptr()) if seeds is not None else None, _stream(stream)))

    def sensitivity(self):
        """S = sum over steps of e_bar * curl_b(H), (nx, ny, nz, 3) torch tensor on the device."""
        import torch
        nx, ny, nz = self.grid.plan.shape
        out = torch.empty((nx, ny, nz, 3), dtype=self.grid.torch_dtype, device=self.grid.device)
        check(library().tfd_adjoint_sensitivity(self.handle, c_vp(out.data_ptr()), TFD_DEVICE, _stream()))
        return out

    def close(self):
        if getattr(self, 'handle', None):
            library().tfd_adjoint_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001 - interpreter shutdown
            pass

"""ctypes wrapper of the C oracle (TEST INFRASTRUCTURE and CPU baseline, not product code).

``CpuOracle(plan)`` holds the state in the reference layout and advances it with
oracle/yee_cpu.c on ``threads`` host threads; results are bitwise equal to
``oracle.yee_oracle.YeeOracle`` (same operation order, no contraction).
"""
import ctypes
import os

import numpy as np

from .build import TARGET, build

c_i32, c_dbl, c_vp = ctypes.c_int32, ctypes.c_double, ctypes.c_void_p
P_dbl = ctypes.POINTER(ctypes.c_double)


class Segment(ctypes.Structure):
    _fields_ = [('forward', c_i32), ('axis', c_i32), ('lo', c_i32), ('hi', c_i32), ('b', P_dbl), ('c', P_dbl), ('inv_kappa', P_dbl)]


class Source(ctypes.Structure):
    _fields_ = [('family', c_i32), ('component', c_i32), ('lo', c_i32 * 3), ('hi', c_i32 * 3), ('values', P_dbl)]


class Trace(ctypes.Structure):
    _fields_ = [('family', c_i32), ('component', c_i32), ('index', c_i32 * 3)]


class Desc(ctypes.Structure):
    _fields_ = [('nx', c_i32), ('ny', c_i32), ('nz', c_i32), ('steps', c_i32), ('material_samples', c_i32),
                ('courant', c_dbl), ('periodic', c_i32 * 3), ('pec_on', c_i32 * 3), ('pec_upper', c_dbl * 3),
                ('n_segments', c_i32), ('segments', ctypes.POINTER(Segment)), ('n_sources', c_i32),
                ('sources', ctypes.POINTER(Source)), ('n_traces', c_i32), ('traces', ctypes.POINTER(Trace)),
                ('metric', (P_dbl * 3) * 2)]


_lib = None


def library():
    global _lib
    if _lib is None:
        if not TARGET.exists():
            build()
        _lib = ctypes.CDLL(str(TARGET))
        for name in ('oc_run_f32', 'oc_run_f64'):
            fn = getattr(_lib, name)
            fn.restype = ctypes.c_int
            fn.argtypes = [ctypes.POINTER(Desc), c_vp, c_vp, c_vp, ctypes.POINTER(c_vp), ctypes.c_int64, c_i32, c_vp, c_i32]
    return _lib


def _p(a):
    return a.ctypes.data_as(P_dbl)


class CpuOracle:
    def __init__(self, plan, threads=None):
        if getattr(plan, 'tfsf', None) or getattr(plan, 'ade', None):
            raise ValueError('The C oracle does not implement TFSF boxes or dispersive materials; use oracle.yee_oracle.YeeOracle.')
        self.plan = plan
        self.threads = threads or os.cpu_count() or 1
        dt = plan.dtype
        shape = plan.shape
        self.E = np.zeros((*shape, 3), dt)
        self.H = np.zeros((*shape, 3), dt)
        self.inv_eps = np.ascontiguousarray(plan.inv_eps, dtype=dt)
        self.memory_states = [np.zeros(s, dt) for _, s in plan.psi_shapes()]
        self.traces = np.zeros((plan.steps, len(plan.traces)), dt)
        self.counter = 0
        self._keep = []
        d = Desc()
        d.nx, d.ny, d.nz = shape
        d.steps = plan.steps
        d.material_samples = plan.material_samples
        d.courant = plan.courant
        for a in range(3):
            d.periodic[a] = int(shape[a] > 1 and plan.faces[a][0] == 'periodic')
            d.pec_on[a] = int(a in plan.pec_upper)
            d.pec_upper[a] = plan.pec_upper.get(a, 0.)
        segs = (Segment * max(1, len(plan.segments)))()
        for k, s in enumerate(plan.segments):
            arrays = [np.ascontiguousarray(v, dtype=np.float64) for v in (s.b, s.c, s.inv_kappa)]
            self._keep += arrays
            segs[k] = Segment(int(s.forward), s.axis, s.lo, s.hi, *map(_p, arrays))
        d.n_segments, d.segments = len(plan.segments), segs
        srcs = (Source * max(1, len(plan.sources)))()
        for k, t in enumerate(plan.sources):
            v = np.ascontiguousarray(t.values, dtype=np.float64)
            self._keep.append(v)
            srcs[k] = Source(t.family, t.comp, (c_i32 * 3)(*t.lo), (c_i32 * 3)(*t.hi), _p(v))
        d.n_sources, d.sources = len(plan.sources), srcs
        trs = (Trace * max(1, len(plan.traces)))()
        for k, t in enumerate(plan.traces):
            trs[k] = Trace(t.family, t.comp, (c_i32 * 3)(*t.index))
        d.n_traces, d.traces = len(plan.traces), trs
        for f in range(2):
            for a in range(3):
                table = plan.metric_table(f, a)
                if table is not None:
                    table = np.ascontiguousarray(table, dtype=np.float64)
                    self._keep.append(table)
                    d.metric[f][a] = _p(table)
        self._keep += [segs, srcs, trs]
        self.desc = d

    def run_with_planes(self, steps=None, dft_float64=True):
        """Step one step at a time and accumulate the plan's DFT planes on the host after each step (the NumPy
        oracle's accumulation); returns the accumulators."""
        from .yee_oracle import accumulate_planes, plane_entries
        if not hasattr(self, 'planes'):
            self.planes = plane_entries(self.plan, dft_float64)
        for _ in range(self.plan.steps if steps is None else steps):
            n = self.counter
            self.run(1)
            accumulate_planes(self.planes, self.E, self.H, n)
        return [e['value'] for e in self.planes]

    def run(self, steps=None):
        n = self.plan.steps if steps is None else steps
        psi = (c_vp * max(1, len(self.memory_states)))(*[m.ctypes.data for m in self.memory_states])
        fn = library().oc_run_f64 if self.plan.dtype == np.float64 else library().oc_run_f32
        rc = fn(ctypes.byref(self.desc), c_vp(self.E.ctypes.data), c_vp(self.H.ctypes.data), c_vp(self.inv_eps.ctypes.data),
                psi, self.counter, n, c_vp(self.traces.ctypes.data), self.threads)
        if rc:
            raise RuntimeError('C oracle failed')
        self.counter += n
        return self

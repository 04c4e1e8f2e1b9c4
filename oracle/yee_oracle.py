"""CPU oracle of the fused Yee/CPML time loop (TEST INFRASTRUCTURE, not product code).

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg
use this module, and only as the checker. The engine never calls it.

It restates, operation for operation in the same floating-point order, the
reference CPU path that the reference's fused CUDA kernels are pinned to
(bitwise in FP32, reference ``tests/test_cuda_kernels.py:149-170``):

- ``YeeGrid.curl`` (reference ``torchfdtd/boundaries.py:363-394``): backward
  differences for E, forward for H, scaled by the nonuniform-mesh metric where the
  mesh has one, curl terms summed in ``CURL_TERMS`` order,
  CPML ``psi <- b*psi + c*d; d <- d/kappa + psi`` inside the slabs, periodic
  wrap, the PEC upper ghost for H;
- ``update_E`` / ``update_H`` (:413-438): ``E += (cn*inv_eps)*curl H``,
  ``H -= (cn*inv_mu)*curl E``;
- soft injection after each family update (``torchfdtd/solver.py:778-789``);
- point traces after the H update (:790-796) and the online plane DFT
  (``torchfdtd/field_monitors.py:144-160``).

The state layout is the reference's: E, H as (Nx, Ny, Nz, 3) with z fastest,
and the CPML memories in the reference's allocation order. It consumes a
``torchfdtd_b200.plan.GridPlan`` whose planning is itself pinned to the
reference by the golden vectors in ``tests/golden``.
"""
from __future__ import annotations

import numpy as np

CURL_TERMS = ((0, 2, 1, -1), (0, 1, 2, 1),
              (1, 2, 0, 1), (1, 0, 2, -1),
              (2, 1, 0, -1), (2, 0, 1, 1))


def _slice(axis, value, component=None):
    parts = [slice(None)] * 3
    parts[axis] = value
    if component is not None:
        parts.append(component)
    return tuple(parts)


def plane_entries(plan, dft_float64=False):
    """DFT accumulators of the plan's planes (reference torchfdtd/field_monitors.py:121-164)."""
    entries = []
    for p in plan.planes:
        cdtype = np.complex128 if dft_float64 else p.complex_dtype
        value = np.zeros((len(p.frequency), p.corner_cells.shape[2], len(p.components)), dtype=cdtype)
        omega = 2j * np.pi * p.frequency * plan.time_step
        half = np.exp(1j * np.pi * p.frequency * plan.time_step).astype(cdtype)
        entries.append(dict(plan=p, value=value, omega=omega, half=half))
    return entries


def accumulate_planes(entries, E, H, n):
    """One step of the online plane DFT after step n (reference torchfdtd/field_monitors.py:144-160): the
    trilinear sample of each component times the window, times exp(i w (n+1) dt), H half a step later."""
    for entry in entries:
        p = entry['plan']
        fields = []
        for k, comp in enumerate(p.components):
            family = int(comp.startswith('H'))
            flat = (H if family else E).reshape(-1)
            c = 'xyz'.index(comp[1].lower())
            sampled = (flat[p.corner_cells[k] * 3 + c] * p.corner_weights[k]).sum(axis=0)
            fields.append(sampled * p.windows[family][n])
        value = entry['value']
        phase = np.exp(entry['omega'] * (n + 1)).astype(value.dtype)
        values = np.stack(fields, axis=-1)
        ne = p.ne
        value[..., :ne] += phase[:, None, None] * values[None, :, :ne]
        value[..., ne:] += (phase * entry['half'])[:, None, None] * values[None, :, ne:]


class YeeOracle:
    def __init__(self, plan, dft_float64=False):
        self.plan = plan
        dtype = plan.dtype
        shape = plan.shape
        self.dtype = dtype
        self.E = np.zeros((*shape, 3), dtype=dtype)
        self.H = np.zeros((*shape, 3), dtype=dtype)
        inv = plan.inv_eps if plan.inv_eps.ndim == 4 else plan.inv_eps[..., None]
        self.inverse_permittivity = np.ones((*shape, 3), dtype=dtype)
        self.inverse_permittivity[:] = inv
        self.inverse_permeability = np.ones((1,), dtype=dtype)
        self.courant = plan.courant
        self.wrap = {a for a in range(3) if shape[a] > 1 and plan.faces[a][0] == 'periodic'}
        # Nonuniform mesh factors (reference torchfdtd/boundaries.py:276-284), stored in the field precision.
        self.metric = {}
        for (forward, axis), (values, wrap) in plan.metrics.items():
            shape_m = [1, 1, 1]
            shape_m[axis] = len(values)
            self.metric[forward, axis] = (values.reshape(shape_m).astype(dtype), wrap)
        self.pec_upper = dict(plan.pec_upper)
        self.cpml = {}
        self.memory_states = []
        for forward in (False, True):
            for axis, component, output, _ in CURL_TERMS:
                n = shape[axis]
                if n == 1:
                    continue
                active_start = 0 if forward else 1
                segments = []
                for seg in plan.segments:
                    if seg.forward != forward or seg.axis != axis:
                        continue
                    coeff_shape = [1, 1, 1]
                    coeff_shape[axis] = seg.hi - seg.lo
                    psi_shape = list(shape)
                    psi_shape[axis] = seg.hi - seg.lo
                    psi = np.zeros(psi_shape, dtype=dtype)
                    self.memory_states.append(psi)
                    segments.append(dict(slice=_slice(axis, slice(seg.lo - active_start, seg.hi - active_start)), psi=psi,
                                         b=seg.b.reshape(coeff_shape).astype(dtype), c=seg.c.reshape(coeff_shape).astype(dtype),
                                         inv_k=seg.inv_kappa.reshape(coeff_shape).astype(dtype)))
                self.cpml[forward, axis, component] = segments
        self.sources = {0: [], 1: []}
        for term in plan.sources:
            loc = tuple(slice(lo, hi) for lo, hi in zip(term.lo, term.hi))
            self.sources[term.family].append((term.values.astype(dtype), loc, term.comp))
        # TFSF boxes: the live incident line in the field precision and the two correction maps
        # (reference torchfdtd/tfsf.py:125-176).
        self.lines = []
        for box in plan.tfsf:
            line = dict(box=box, e=np.zeros(box.count, dtype), h=np.zeros(box.count, dtype), pe=np.zeros(box.count, dtype),
                        ph=np.zeros(box.count, dtype), diff=np.zeros(box.count, dtype),
                        coef=[tuple(v.astype(dtype) for v in pair) for pair in box.coefficients],
                        drive=box.drive.astype(dtype),
                        maps={f: (t, smp, w.astype(dtype)) for f, (t, smp, w) in box.maps.items()})
            self.lines.append(line)
        # Dispersive materials (reference torchfdtd/materials.py:29-88): per state its samples, P and Q per pole,
        # and the coefficients as the reference holds them (float64 scalars for one pole, the field precision for
        # several).
        self.ade = []
        for st in getattr(plan, 'ade', []):
            if st.multiple:
                coef = {k: getattr(st, k).reshape(-1, 1).astype(dtype) for k in ('a', 'd', 'k')}
                shape = (st.poles, st.samples)
            else:
                coef = {k: float(getattr(st, k)[0]) for k in ('a', 'd', 'k')}
                shape = (st.samples,)
            k_sum = coef['k'].sum(axis=0) if st.multiple else coef['k']
            self.ade.append(dict(state=st, P=np.zeros(shape, dtype), Q=np.zeros(shape, dtype), k_sum=k_sum, **coef))
        self.counter = 0
        self.traces = np.zeros((plan.steps, len(plan.traces)), dtype=dtype)
        self.planes = plane_entries(plan, dft_float64)

    # -- reference YeeGrid.curl ---------------------------------------------------------------
    def curl(self, field, forward):
        result = np.zeros(field.shape, dtype=self.dtype)
        for axis, component, output, sign in CURL_TERMS:
            if field.shape[axis] == 1:
                continue
            low = _slice(axis, slice(None, -1), component)
            high = _slice(axis, slice(1, None), component)
            derivative = field[high] - field[low]
            if (forward, axis) in self.metric:
                derivative *= self.metric[forward, axis][0]
            for segment in self.cpml[forward, axis, component]:
                data = derivative[segment['slice']]
                psi = segment['psi']
                psi *= segment['b']
                psi += segment['c'] * data
                data *= segment['inv_k']
                data += psi
            target = _slice(axis, slice(None, -1) if forward else slice(1, None), output)
            result[target] += sign * derivative
            if axis in self.wrap:
                first, last = _slice(axis, 0, component), _slice(axis, -1, component)
                edge = 1.0 * field[first] - field[last] if forward else field[first] - field[last] / 1.0
                if (forward, axis) in self.metric:
                    edge *= self.metric[forward, axis][1]
                result[_slice(axis, -1 if forward else 0, output)] += sign * edge
            elif forward and axis in self.pec_upper:
                edge = -self.pec_upper[axis] * field[_slice(axis, -1, component)]
                result[_slice(axis, -1, output)] += sign * edge
        return result

    def update_E(self):
        flat = self.E.reshape(-1)
        prepared = [(flat[m['state'].target], (m['Q'] - m['a'] * m['P']) / m['d']) for m in self.ade]
        self.E += self.courant * self.inverse_permittivity * self.curl(self.H, False)
        for m, (old, response) in zip(self.ade, prepared):
            free = flat[m['state'].target]
            total = response.sum(axis=0) if m['state'].multiple else response
            eps = m['state'].eps_inf
            new = (eps * free - m['k_sum'] * old - total) / (eps + m['k_sum'])
            delta = response + m['k'] * (new + old)
            m['P'] += delta
            m['Q'] *= -1
            m['Q'] += 2 * delta
            flat[m['state'].target] = new

    def update_H(self):
        self.H -= self.courant * self.inverse_permeability * self.curl(self.E, True)

    def inject(self, family):
        field = self.E if family == 0 else self.H
        for values, loc, component in self.sources[family]:
            field[loc + (component,)] += values[self.counter]
        for line in self.lines:
            self._tfsf(line, family)

    def _tfsf(self, line, family):
        """Advance the incident line by one half step of `family`, then add the corrections of that family."""
        box, forward = line['box'], family == 1
        e, h, diff = line['e'], line['h'], line['diff']
        if forward:
            diff[:-1] = e[1:] - e[:-1]
            diff[-1] = 0
        else:
            diff[1:] = h[1:] - h[:-1]
            diff[0] = 0
        b, c = line['coef'][int(forward)]
        psi = line['ph'] if forward else line['pe']
        psi *= b
        psi += c * diff
        field_line = h if forward else e
        field_line -= (box.courant if forward else box.courant_e) * (diff + psi)
        if not forward:
            e[box.drive_at] += line['drive'][self.counter]
        target, sample, weight = line['maps']['H' if forward else 'E']
        flat = (self.H if forward else self.E).reshape(-1)
        flat[target] += weight * (e if forward else h)[sample]

    def _planes(self):
        accumulate_planes(self.planes, self.E, self.H, self.counter)

    def step(self):
        self.update_E()
        self.inject(0)
        self.update_H()
        self.inject(1)
        self._planes()
        if self.plan.traces:
            self.traces[self.counter] = [(self.E if t.family == 0 else self.H)[t.index + (t.comp,)] for t in self.plan.traces]
        self.counter += 1

    def run(self, steps=None):
        for _ in range(self.plan.steps if steps is None else steps):
            self.step()
        return self

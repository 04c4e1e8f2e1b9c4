"""CPU oracle of the discrete Yee/CPML adjoint (TEST INFRASTRUCTURE, not product code).

Only ``tests/`` use this module, as the checker of the CUDA adjoint. It restates the reference's
transpose of one step (``_System.transpose_step``, reference torchfdtd/differentiable.py:489-519) and
of the CPML curl (``curl_faces_transpose`` :369-432, without PMC faces) in numpy on the state of
``oracle.yee_oracle.YeeOracle``:

- observation seeds are added to e_bar / h_bar first (the traces sample the state after the step);
- e_bar += curl_f^T(-cn h_bar), with the CPML memory transpose m = psi_bar + v; psi_bar <- b m;
  v <- v / kappa + c m; then, on a nonuniform mesh, v <- v * metric (the forward scales the difference
  before its CPML terms, so the transpose scales after them);
- dJ/d eps += -cn e_bar curl_b(H_n; psi_n) / eps^2, summed over components for a per-cell eps;
- h_bar += curl_b^T((cn / eps) e_bar).

The forward pass keeps every state (small grids only); the reverse pass walks the steps backwards.
"""
from __future__ import annotations

import numpy as np

from oracle.yee_oracle import CURL_TERMS, YeeOracle, _slice


class AdjointOracle:
    def __init__(self, plan, epsilon):
        """``plan``: a GridPlan whose traces are the observers; ``epsilon``: (nx, ny, nz) or (nx, ny, nz, 3)."""
        eps = np.asarray(epsilon, dtype=plan.dtype)
        plan.epsilon = eps
        plan.inv_eps = (1 / eps).astype(plan.dtype)
        self.plan = plan
        self.eps = eps
        self.eps4 = eps if eps.ndim == 4 else eps[..., None]
        self.fwd = YeeOracle(plan)
        self.keys = {}
        index = 0
        for key, segs in self.fwd.cpml.items():
            self.keys[key] = list(range(index, index + len(segs)))
            index += len(segs)

    def forward(self):
        o = self.fwd
        self.states = []
        for _ in range(self.plan.steps):
            self.states.append((o.E.copy(), o.H.copy(), [p.copy() for p in o.memory_states]))
            o.step()
        return o.traces.copy()

    def _segments(self, forward, axis, component):
        return [(i, seg) for i, seg in zip(self.keys[forward, axis, component], self.fwd.cpml[forward, axis, component])]

    def curl_state(self, H, psis):
        """Forward E curl of a stored state without touching its memories."""
        shape = H.shape[:3]
        result = np.zeros(H.shape, dtype=H.dtype)
        for axis, component, output, sign in CURL_TERMS:
            n = shape[axis]
            if n == 1:
                continue
            derivative = H[_slice(axis, slice(1, None), component)] - H[_slice(axis, slice(None, -1), component)]
            metric = self.fwd.metric.get((False, axis))
            if metric:
                derivative = derivative * metric[0]
            for i, seg in self._segments(False, axis, component):
                data = derivative[seg['slice']]
                psi = psis[i] * seg['b'] + seg['c'] * data
                derivative[seg['slice']] = data * seg['inv_k'] + psi
            result[_slice(axis, slice(1, None), output)] += sign * derivative
            if axis in self.fwd.wrap:
                edge = H[_slice(axis, 0, component)] - H[_slice(axis, -1, component)]
                if metric:
                    edge = edge * metric[1]
                result[_slice(axis, 0, output)] += sign * edge
        return result

    def curl_transpose(self, bar, psi_bar, forward):
        shape = bar.shape[:3]
        result = np.zeros(bar.shape, dtype=bar.dtype)
        previous = list(psi_bar)
        for axis, component, output, sign in CURL_TERMS:
            n = shape[axis]
            if n == 1:
                continue
            dst = bar[..., output]
            derivative = sign * dst[_slice(axis, slice(0, n - 1) if forward else slice(1, n))]
            for i, seg in self._segments(forward, axis, component):
                value = derivative[seg['slice']]
                memory_bar = psi_bar[i] + value
                previous[i] = seg['b'] * memory_bar
                derivative = derivative.copy()
                derivative[seg['slice']] = value * seg['inv_k'] + seg['c'] * memory_bar
            metric = self.fwd.metric.get((forward, axis))
            if metric:
                derivative = derivative * metric[0]
            src = result[..., component]
            src[_slice(axis, slice(1, n))] += derivative
            src[_slice(axis, slice(0, n - 1))] -= derivative
            if axis in self.fwd.wrap:
                edge = sign * dst[_slice(axis, n - 1 if forward else 0)]
                if metric:
                    edge = edge * metric[1]
                src[_slice(axis, 0)] += edge
                src[_slice(axis, n - 1)] -= edge
            elif forward and axis in self.fwd.pec_upper:
                src[_slice(axis, n - 1)] -= sign * self.fwd.pec_upper[axis] * dst[_slice(axis, n - 1)]
        return result, previous

    def backward(self, signal_bar):
        """Gradient of sum(signal_bar * traces) with respect to epsilon (its shape)."""
        o = self.fwd
        cn = o.courant
        dtype = self.plan.dtype
        e_bar = np.zeros_like(o.E)
        h_bar = np.zeros_like(o.H)
        psi_bar = [np.zeros_like(p) for p in o.memory_states]
        gradient = np.zeros(self.eps4.shape, dtype=dtype)
        for n in range(self.plan.steps - 1, -1, -1):
            for k, t in enumerate(self.plan.traces):
                (e_bar if t.family == 0 else h_bar)[t.index + (t.comp,)] += signal_bar[n, k]
            contribution, psi_bar = self.curl_transpose(-cn * h_bar, psi_bar, True)
            e_bar = e_bar + contribution
            E, H, psis = self.states[n]
            curl_e = self.curl_state(H, psis)
            full = -cn * (e_bar * curl_e) / np.square(self.eps4)
            gradient += full.sum(axis=-1, keepdims=True) if self.eps4.shape[-1] == 1 else full
            contribution, psi_bar = self.curl_transpose(cn / self.eps4 * e_bar, psi_bar, False)
            h_bar = h_bar + contribution
        self.e_bar, self.h_bar, self.psi_bar = e_bar, h_bar, psi_bar
        return gradient if self.eps.ndim == 4 else gradient[..., 0]

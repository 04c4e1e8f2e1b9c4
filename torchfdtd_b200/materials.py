"""Dispersive (Drude / Lorentz / multipole) materials: the coupled trapezoidal auxiliary-differential equation.

A dispersive material has eps(w) = eps_inf + sum_p strength_p / (w0_p^2 - w^2 - i damping_p w). Each E sample
it owns carries, per pole, the relative polarization P and Q = dt dP/dt. The E update first advances E with
1 / eps_inf (the voxelized permittivity of a dispersive cell is eps_inf), giving the "free" value; the
trapezoidal rule then solves E and the oscillators together:

    response_p = (Q_p - a_p P_p) / d_p                      (from the old state)
    E_new      = (eps_inf E_free - k_sum E_old - sum_p response_p) / (eps_inf + k_sum)
    delta_p    = response_p + k_p (E_new + E_old);  P_p += delta_p;  Q_p = -Q_p + 2 delta_p

with a = (w0 dt)^2 / 2, d = 1 + damping dt / 2 + (w0 dt)^2 / 4, k = strength dt^2 / (4 d), k_sum = sum_p k_p,
before the soft sources are added. With pml_dispersion='frozen' the samples inside the PML keep a constant
real permittivity (the material's at the pulsed sources' mean centre frequency, else its static limit)
instead of the oscillators.

Restates reference ``torchfdtd/materials.py`` (``permittivity`` :15-26, ``MaterialADE`` :29-88,
``configure_materials`` :117-193 for the 'ade' and 'frozen' modes). The arithmetic precision follows the
reference's: a single-pole material keeps a, d, k in float64 and the field precision rounds them at each use
(and rounds eps_inf + k once); a multipole material stores them in the field precision and sums in it.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np


def permittivity(material, frequency_hz, dt=0):
    """eps(f) of a material; with dt > 0 the trapezoidal rule's frequency warping (w -> 2/dt tan(pi f dt))."""
    f = np.asarray(frequency_hz, dtype=float)
    if np.any(~np.isfinite(f)) or np.any(f <= 0):
        raise ValueError('Material frequencies must be finite and positive.')
    if not np.isfinite(dt) or dt < 0 or (dt and np.any(f * dt >= .5)):
        raise ValueError('Material timestep must be nonnegative and frequencies below Nyquist.')
    omega = 2 * np.pi * f if not dt else 2 / dt * np.tan(np.pi * f * dt)
    eps = np.full(f.shape, material.instantaneous_epsilon, dtype=complex)
    for w0, strength, gamma in material.oscillators:
        with np.errstate(divide='ignore', invalid='ignore'):
            eps += strength / (w0 * w0 - omega * omega - 1j * gamma * omega)
    return eps


@dataclass
class ADEState:
    """The samples one dispersive material owns and its per-pole coefficients (float64)."""
    material: object
    target: np.ndarray          # int64: flat reference-layout element (cell * 3 + component) of each sample
    multiple: bool              # more than one pole: coefficients stored in the field precision
    a: np.ndarray               # (poles,)
    d: np.ndarray
    k: np.ndarray
    eps_inf: float
    w0: np.ndarray              # (poles,): diagnostics
    strength: np.ndarray

    @property
    def poles(self):
        return len(self.a)

    @property
    def samples(self):
        return len(self.target)


def _pml_mask(region, shape):
    mask = np.zeros(shape[:3], dtype=bool)
    for axis in range(3 if region.dimension == '3d' else 2):
        lo, hi = region.pml_layers(axis, 0), region.pml_layers(axis, 1)
        index = [slice(None)] * 3
        if lo:
            index[axis] = slice(0, lo)
            mask[tuple(index)] = True
        if hi:
            index[axis] = slice(shape[axis] - hi, None)
            mask[tuple(index)] = True
    return mask


def _frozen_frequency(project):
    from .waveforms import pulse_parameters
    values = [pulse_parameters(s).frequency_hz for s in map(project.resolved_source, project.sources)
              if s.enabled and s.amplitude != 0 and s.pulse != 'sampled']
    return float(np.mean(values)) if values else None


def ade_states(project, owner, inv_eps):
    """ADE states of the dispersive materials that own samples (``owner``: material index per sample, the shape of
    the permittivity). With pml_dispersion='frozen', ``inv_eps`` is overwritten in place on the PML samples."""
    r = project.region
    if r.pml_dispersion == 'absorber':
        raise ValueError('pml_dispersion="absorber" is not implemented by the fused B200 engine.')
    frozen = r.pml_dispersion == 'frozen'
    per_component = owner.ndim == 4
    pml = _pml_mask(r, owner.shape).reshape(-1) if frozen else None
    if frozen and per_component:
        pml = np.repeat(pml, 3)
    reference_hz = _frozen_frequency(project) if frozen else None
    dt = r.time_step
    states = []
    for i, m in enumerate(project.materials):
        if not m.oscillators or not np.any(owner == i):
            continue
        owned = owner.reshape(-1) == i
        if frozen and np.any(owned & pml):
            eps = float(permittivity(m, reference_hz).real if reference_hz else
                        m.instantaneous_epsilon + sum(s / (w0 * w0) for w0, s, _ in m.oscillators if w0))
            if eps <= 0:
                at = f'at the reference frequency {reference_hz:.6g} Hz' if reference_hz else 'in the static limit'
                raise ValueError(f'{m.name}: pml_dispersion="frozen" has no meaning for a real permittivity of {eps:.6g} '
                                 f'{at}. Keep the material out of the PML or use pml_dispersion="ade".')
            flat = inv_eps.reshape(-1) if per_component else inv_eps.reshape(-1)
            flat[np.flatnonzero(owned & pml)] = 1 / max(eps, 1e-3)
            owned = owned & ~pml
            if not np.any(owned):
                continue
        index = np.flatnonzero(owned)
        target = index if per_component else (index[:, None] * 3 + np.arange(3)).reshape(-1)
        poles = np.asarray(m.oscillators, dtype=float)
        w0, strength, gamma = poles[:, 0], poles[:, 1], poles[:, 2]
        d = 1 + .5 * gamma * dt + .25 * (w0 * dt)**2
        states.append(ADEState(m, target.astype(np.int64), len(poles) > 1, .5 * (w0 * dt)**2, d,
                               strength * dt * dt / (4 * d), float(m.epsilon_inf), w0, strength))
    return states

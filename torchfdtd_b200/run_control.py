"""Run control: source end time, decay/divergence decisions and the graph barrier schedule.

Restates reference ``torchfdtd/run_control.py:15-85`` (``source_end_time``,
``DecayDecision``) and ``torchfdtd/cuda_graph.py:12-29``
(``validate_graph_steps``, ``observation_schedule``). The state norm itself
is measured on the device by ``tfd_diagnose``.
"""
from __future__ import annotations

import math

from .waveforms import TAIL_OUTER, pulse_parameters


def source_end_time(project):
    cutoff = project.region.run_control.source_tail_amplitude
    ends = [0.]
    for source in project.sources:
        s = project.resolved_source(source)
        if not s.enabled or s.amplitude == 0:
            continue
        if s.pulse == 'continuous':
            return math.inf
        if s.pulse == 'sampled':
            ends.append(s.signal.time_s[-1])
            continue
        pulse = pulse_parameters(s)
        tail = TAIL_OUTER if s.eliminate_discontinuities else math.sqrt(-2 * math.log(cutoff))
        ends.append(pulse.offset_s + tail * pulse.sigma_s)
    return max(ends)


class DecayDecision:
    """Backend-independent decay and divergence decisions from (state norm, field peak) samples."""

    def __init__(self, control, source_end_s, dt):
        self.control, self.dt = control, dt
        self.eligible_time = source_end_s + control.after_source_s
        self.peak = 0.
        self.frozen_peak = None
        self.below = 0
        self.history = []

    def update(self, step, energy, field_peak):
        c = self.control
        if not math.isfinite(energy) or not math.isfinite(field_peak):
            raise FloatingPointError(f'Non-finite full-domain or auxiliary state at step {step}.')
        if c.divergence_check and c.field_limit is not None and field_peak > c.field_limit:
            raise FloatingPointError(f'Field magnitude limit exceeded at step {step}: {field_peak:.6g}.')
        eligible = step >= c.min_steps and step * self.dt >= self.eligible_time
        self.peak = max(self.peak, energy)
        if eligible and self.frozen_peak is None:
            self.frozen_peak = self.peak
        baseline = self.frozen_peak if self.frozen_peak is not None else self.peak
        ratio = energy / baseline if baseline else 0.
        if c.divergence_check and eligible and ratio > c.growth_limit:
            raise FloatingPointError(f'Post-source state norm grew by {ratio:.6g} at step {step}.')
        self.below = self.below + 1 if eligible and ratio <= c.decay_threshold else 0
        self.history.append(dict(step=step, time_s=step * self.dt, state_norm=energy, relative_norm=ratio,
                                 field_peak=field_peak, source_finished=eligible))
        return c.auto_shutoff and self.below >= c.consecutive_checks


def validate_graph_steps(value, enabled=True):
    if isinstance(value, bool) or not isinstance(value, int) or not 1 <= value <= 64:
        raise ValueError('cuda_graph_steps must be an integer from 1 to 64.')
    if value != 1 and not enabled:
        raise ValueError('cuda_graph_steps > 1 requires CUDA graph execution.')
    return value


def observation_schedule(steps, width, barriers=()):
    """Yield (completed steps, replay width), stopping at every host barrier."""
    completed = 0
    for end in sorted(set(barriers) | {steps}):
        if not 0 < end <= steps:
            raise ValueError('Observation barriers must lie within the run.')
        while completed < end:
            advance = width if end - completed >= width else 1
            completed += advance
            yield completed, advance

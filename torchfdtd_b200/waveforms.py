"""Source time signals, sampled on the host in float64.

Restates reference ``torchfdtd/waveforms.py``: ``pulse_parameters`` :28-42
(carrier, Gaussian sigma from the power FWHM, offset), ``gaussian_envelope``
:45-52 (with the optional C1 Hermite tail taper) and ``source_time_signal``
:55-74 (gaussian, continuous, sampled and chirped broadband pulses). The
sampled waveform is uploaded once and indexed by the device step counter, so
its formulas must agree with the reference sample for sample.
"""
import math
from dataclasses import dataclass

import numpy as np

C0 = 299792458.0
# Gaussian amplitude 1e-4 in units of sigma, and the end of the optional taper 10% later.
TAIL_INNER = math.sqrt(2 * math.log(1e4))
TAIL_OUTER = 1.1 * TAIL_INNER


@dataclass(frozen=True)
class PulseParameters:
    frequency_hz: float
    sigma_s: float
    offset_s: float
    frequency_span_hz: float
    chirped: bool


def pulse_parameters(source):
    frequency = C0 / (source.wavelength * 1e-6)
    span = source.chirp_bandwidth_hz if source.pulse == 'broadband' else 0.
    if source.time_definition in ('wavelength', 'frequency'):
        low, high = C0 / (source.wavelength_stop * 1e-6), C0 / (source.wavelength_start * 1e-6)
        frequency, span = (low + high) / 2, high - low
        length = (2 if source.optimize_for_short_pulse else 8) / (high + .01 * low)
        sigma = length / (2 * math.sqrt(math.log(2)))
        offset = TAIL_OUTER * sigma
        chirped = span > math.sqrt(math.log(2)) / (math.pi * sigma)
    elif source.time_definition == 'standard':
        sigma = source.pulse_length / (2 * math.sqrt(math.log(2)))
        offset = source.pulse_offset
        chirped = source.pulse == 'broadband'
    else:
        sigma = source.pulse_cycles / frequency
        offset, chirped = 4 * sigma, False
    return PulseParameters(frequency, sigma, offset, span, chirped)


def gaussian_envelope(u, smooth=False):
    envelope = np.exp(-.5 * u * u)
    if not smooth:
        return envelope
    h = TAIL_OUTER - TAIL_INNER
    distance = np.maximum(TAIL_OUTER - np.abs(u), 0)
    # Cubic in the distance to TAIL_OUTER matching value (1e-4) and slope at TAIL_INNER.
    alpha = (3e-4 - TAIL_INNER * 1e-4 * h) / (h * h)
    beta = (TAIL_INNER * 1e-4 * h - 2e-4) / (h * h * h)
    return np.where(np.abs(u) <= TAIL_INNER, envelope, alpha * distance**2 + beta * distance**3)


def source_time_signal(source, times):
    times = np.asarray(times, dtype=np.float64)
    if source.pulse == 'sampled':
        signal = source.signal
        amplitude = np.interp(times, signal.time_s, signal.amplitude, left=0, right=0)
        phase = np.interp(times, signal.time_s, signal.phase_rad) + math.radians(source.phase)
        return source.amplitude * amplitude * np.sin(phase)
    p = pulse_parameters(source)
    x = times - p.offset_s
    u = x / p.sigma_s
    omega = 2 * math.pi * p.frequency_hz
    phase = math.radians(source.phase)
    if source.pulse == 'continuous':
        envelope = 1 - np.exp(-(times / p.sigma_s)**2)
        carrier = omega * times
    else:
        envelope = gaussian_envelope(u, source.eliminate_discontinuities)
        carrier = omega * times if source.time_definition == 'cycles' else -omega * x
        if p.chirped:
            # Instantaneous frequency sweeps sinusoidally across the band within |u| <= 2.
            inside = p.frequency_span_hz * p.sigma_s * (4 * np.cos(np.pi * u / 4) - 2 * np.pi)
            outside = -np.pi * p.frequency_span_hz * np.abs(x)
            carrier = carrier + np.where(np.abs(u) <= 2, inside, outside)
    return source.amplitude * envelope * np.sin(carrier + phase)

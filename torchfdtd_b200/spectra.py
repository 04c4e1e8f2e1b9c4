"""Frequency samples, apodization windows and the host transform of point traces.

What the engine must reproduce is the reference's spectral convention (``torchfdtd/spectra.py``:
windows :14-27, sample grids :30-44, :54-73, transforms :76-116), written here from its definition:

* custom / wavelength / frequency / Chebyshev samples: ``X(f) = dt * sum_n x[n] w[n] exp(+2 pi i f t[n])``,
  a field integral in "reduced field * s";
* ``fft`` sampling: ``X(f_k) = s * sum_n x[n] w[n] exp(-2 pi i f_k t[n])`` at the positive FFT frequencies
  ``f_k = k / (N dt)``, ``s = 2/N`` for a real trace and ``1/N`` for a complex one (an amplitude spectrum,
  with no window-gain correction);
* windows: ``1``, a Hann taper, or a Gaussian in ``t - center`` whose ``|w|^2`` has the full width at half
  maximum ``apodization_time_width`` (``start`` / ``end`` keep it flat after / before the centre).

Point traces are recorded on the device every step and transformed here after the run.
"""
import numpy as np

C0 = 299792458.0
# Largest phase table the custom-sample transform builds at once (complex entries).
_PHASE_TABLE = 1 << 20


def apodization_window(times, settings):
    """Window samples at ``times`` (s) for a ``SpectrumSettings``."""
    t = np.asarray(times, dtype=np.float64)
    mode = settings.apodization
    if mode == 'none':
        return np.ones_like(t)
    if mode == 'hann':
        return np.hanning(t.size)
    offset = t - settings.apodization_center
    if mode in ('start', 'end'):
        # One-sided: the Gaussian acts only before ('start') or after ('end') the centre.
        offset = np.clip(offset, None, 0) if mode == 'start' else np.clip(offset, 0, None)
    # |w|^2 = exp(-4 ln2 (d / width)^2) has its half maximum at d = width / 2.
    return np.exp(-2 * np.log(2) * (offset / settings.apodization_time_width)**2)


def frequency_samples(settings):
    """The sample frequencies (Hz) of a non-FFT ``SpectrumSettings``."""
    if settings.sampling == 'custom':
        return np.asarray(settings.custom_frequencies_hz, dtype=np.float64)
    a, b, n = settings.wavelength_start, settings.wavelength_stop, settings.frequency_points
    if settings.sampling == 'fft':
        raise ValueError('FFT samples depend on the recorded time grid.')
    if settings.sampling == 'chebyshev':
        if settings.chebyshev_nodes == 'lobatto':
            u = np.array([.5]) if n == 1 else (1 - np.cos(np.pi * np.arange(n) / (n - 1))) / 2
        else:
            u = (1 - np.cos(np.pi * (np.arange(n) + .5) / n)) / 2
        if settings.chebyshev_wavelength:
            return C0 / ((a + (b - a) * u) * 1e-6)
        return C0 / (b * 1e-6) + (C0 / (a * 1e-6) - C0 / (b * 1e-6)) * u
    if n == 1:
        return np.array([C0 / (1e-6 * (a + b) / 2) if settings.sampling == 'wavelength' else .5 * C0 * 1e6 * (1 / a + 1 / b)])
    if settings.sampling == 'wavelength':
        return C0 / (np.linspace(a, b, n) * 1e-6)
    return np.linspace(C0 / (b * 1e-6), C0 / (a * 1e-6), n)


def frequency_count(settings):
    """How many samples ``frequency_samples`` returns, without building them."""
    if settings.sampling == 'fft':
        raise ValueError('FFT samples depend on the recorded time grid.')
    return settings.frequency_points if settings.sampling != 'custom' else len(settings.custom_frequencies_hz)


def highest_frequency(settings):
    if settings.sampling == 'fft':
        raise ValueError('FFT samples depend on the recorded time grid.')
    return float(np.max(frequency_samples(settings)))


def _uniform_step(t):
    """The step of a uniform, increasing time grid of at least two samples."""
    if t.ndim != 1 or t.size < 2:
        raise ValueError('A point spectrum needs a one-dimensional trace of two or more samples.')
    steps = np.diff(t)
    dt = steps[0]
    if not dt > 0 or np.any(np.abs(steps - dt) > 1e-7 * abs(dt)):
        raise ValueError('A point spectrum needs samples on a uniform, increasing time grid.')
    return dt


def direct_transform(times, signal, frequencies, window=None):
    """``dt * sum_n x[n] w[n] exp(+2 pi i f t[n])`` for each ``f`` (complex128).

    The sum runs over blocks of time samples, so the phase table stays bounded for long traces."""
    t = np.asarray(times, dtype=np.float64)
    f = np.asarray(frequencies, dtype=np.float64)
    x = np.asarray(signal)
    if x.shape != t.shape or f.ndim != 1:
        raise ValueError('A point spectrum needs one trace value per time sample and a list of frequencies.')
    dt = _uniform_step(t)
    if not np.all(np.isfinite(f)) or np.any(f <= 0) or np.any(f * dt >= .5):
        raise ValueError('Spectrum frequencies must be positive and below half the sampling rate 1/(2 dt).')
    weighted = x * np.asarray(window) if window is not None else x
    total = np.zeros(f.size, dtype=np.complex128)
    block = max(1, _PHASE_TABLE // max(1, f.size))
    omega = 2 * np.pi * f
    for lo in range(0, t.size, block):
        phase = np.multiply.outer(omega, t[lo:lo + block])
        total += np.exp(1j * phase) @ weighted[lo:lo + block]
    return total * dt


def _fft_amplitudes(times, signal, window):
    """Amplitude spectrum at the positive FFT frequencies, phase referred to t = 0."""
    t = np.asarray(times, dtype=np.float64)
    dt = t[1] - t[0]
    x = np.asarray(signal) * window
    n = x.size
    if np.iscomplexobj(x):
        freq, raw, scale = np.fft.fftfreq(n, dt), np.fft.fft(x), 1 / n
    else:
        freq, raw, scale = np.fft.rfftfreq(n, dt), np.fft.rfft(x), 2 / n
    # The FFT's sum runs over n dt; the samples sit at t[0] + n dt, hence the factor exp(-2 pi i f t[0]).
    value = raw * scale * np.exp(-2j * np.pi * freq * t[0])
    positive = freq > 0
    return freq[positive], value[positive]


def point_spectrum(times, signal, settings):
    """The spectrum record of one point trace: frequencies, values, units and the transform used."""
    window = apodization_window(times, settings)
    if len(times) < 2:
        return {'frequency_hz': np.array([]), 'value': np.array([], dtype=complex),
                'units': 'unavailable', 'transform': 'insufficient time samples'}
    if settings.sampling == 'fft':
        f, value = _fft_amplitudes(times, signal, window)
        return {'frequency_hz': f, 'value': value, 'units': 'reduced field',
                'transform': 'FFT exp(-2pi i f t); scale 2/N real or 1/N complex; no window-gain correction'}
    f = frequency_samples(settings)
    return {'frequency_hz': f, 'value': direct_transform(times, signal, f, window),
            'units': 'reduced field * s', 'transform': 'dt * sum(field * window * exp(+2pi i f t))'}

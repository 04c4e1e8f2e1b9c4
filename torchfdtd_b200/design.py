"""Inverse design of a 2D TMz transmission region: the plain adjoint loop and the surrogate-assisted loop.

The scene (the learned-surrogate benchmark configuration): a 400 x 400 cell 2D TMz grid at 0.02 um
(8 x 8 um, CPML 16, SiO2 background eps 2.085), a 0.4 um Si input waveguide (eps 12.08) from the left face and
an output waveguide to the right face, joined by a 2 x 2 um design region of 100 x 100 pixels (one pixel per
cell) with eps = 2.085 + rho (12.08 - 2.085). An Ez point source 3 um left of the centre (broadband pulse,
1.50-1.60 um) drives the input guide; an Ez point monitor 3 um right of the centre samples the output. The
complex transmission is t(lambda) = DFT_out(lambda) / DFT_ref(lambda) at 16 wavelengths in 1.50-1.60 um, the
reference being the straight guide (a 0.4 um strip across the design region). The figure of merit is the
mean of |t|^2 over the 16 wavelengths.

* ``generate_dataset``: seeded smoothed random densities simulated by the batched engine (cohorts of 64
  grids, one persistent launch per step) -> (rho, [Re t, Im t]) pairs.
* ``adjoint_design``: Adam on a latent theta (rho = sigmoid(theta)) with FDTD gradients from the discrete
  adjoint (``DifferentiableSimulation``).
* ``surrogate_design``: the same update with gradients of the trained network; every ``verify_every``-th
  iterate is simulated (FDTD judges every accepted design), the network is fine-tuned on the verified
  samples, and a verified drop below the best design falls back to an adjoint step from the best design.
"""
from __future__ import annotations

import math
import time
from dataclasses import dataclass, field

import numpy as np

C0 = 299792458.0
EPS_LOW, EPS_HIGH = 2.085, 12.08


@dataclass
class TransmissionProblem:
    cells: int = 400
    pixels: int = 100
    mesh: float = .02
    steps: int = 4000
    pml: int = 16
    guide_width: float = .4
    wavelengths: tuple = tuple(np.linspace(1.50, 1.60, 16))
    precision: str = 'float32'
    _cache: dict = field(default_factory=dict, repr=False)

    # ---- scene -------------------------------------------------------------------------------------------
    def project(self):
        from .models import Material, Monitor, Project, Region, Source, Structure
        size = self.cells * self.mesh
        region = Region(dimension='2d', size=(size, size, 1), mesh=self.mesh, pml_cells=self.pml, steps=self.steps,
                        background_index=EPS_LOW ** .5, precision=self.precision, backend='cuda', cuda_kernel='fused',
                        snapshot_interval=10000)
        region.run_control.divergence_check = False
        half = self.pixels * self.mesh / 2
        arm = size / 2 - half
        guides = [Structure(id='guide_in', center=(-(half + arm / 2), 0, 0), size=(arm, self.guide_width, 1), material='Si'),
                  Structure(id='guide_out', center=(half + arm / 2, 0, 0), size=(arm, self.guide_width, 1), material='Si')]
        lam = 1.55
        return Project(name='transmission design 400x400', region=region, materials=[Material(name='Si', index=EPS_HIGH ** .5)],
                       structures=guides,
                       sources=[Source(id='src', center=(-3.0, 0, 0), component='Ez', wavelength=lam, pulse='broadband',
                                       time_definition='wavelength', wavelength_start=1.50, wavelength_stop=1.60)],
                       monitors=[Monitor(id='probe', center=(3.0, 0, 0), component='Ez')])

    @property
    def design_slice(self):
        lo = (self.cells - self.pixels) // 2
        return slice(lo, lo + self.pixels), slice(lo, lo + self.pixels)

    def base_epsilon(self):
        if 'base' not in self._cache:
            from .plan import plan_grid
            self._cache['base'] = np.asarray(plan_grid(self.project()).epsilon, dtype=np.float64)
        return self._cache['base']

    def epsilon(self, rho):
        """Full (cells, cells, 1) permittivity of a design density (numpy)."""
        eps = self.base_epsilon().copy()
        sx, sy = self.design_slice
        eps[sx, sy, 0] = EPS_LOW + np.asarray(rho, dtype=np.float64) * (EPS_HIGH - EPS_LOW)
        return eps

    def epsilon_torch(self, rho):
        """The same map on a torch density (differentiable)."""
        import torch
        base = torch.as_tensor(self.base_epsilon(), device=rho.device, dtype=rho.dtype)
        sx, sy = self.design_slice
        eps = base.clone()
        eps[sx, sy, 0] = EPS_LOW + rho * (EPS_HIGH - EPS_LOW)
        return eps

    def straight(self):
        rho = np.zeros((self.pixels, self.pixels))
        w = int(round(self.guide_width / self.mesh / 2))
        rho[:, self.pixels // 2 - w:self.pixels // 2 + w] = 1
        return rho

    # ---- spectra -----------------------------------------------------------------------------------------
    def dft(self):
        """(16, steps) complex DFT rows: dt exp(2 pi i f t_n), t_n = (n + 1) dt (E samples)."""
        if 'dft' not in self._cache:
            r = self.project().region
            f = C0 / (np.asarray(self.wavelengths) * 1e-6)
            t = (np.arange(self.steps) + 1) * r.time_step
            self._cache['dft'] = np.exp(2j * np.pi * f[:, None] * t[None, :]) * r.time_step
        return self._cache['dft']

    def reference(self):
        if 'ref' not in self._cache:
            self._cache['ref'] = self.dft() @ self.trace(self.straight())
        return self._cache['ref']

    def simulate(self, rhos, launch=None):
        """Ez traces (n, steps) of the output monitor for a list of densities (batched engine, cohorts of 64)."""
        from .batch import run_tensor_batch
        project = self.project()
        traces = []
        for i in range(0, len(rhos), 64):
            chunk = rhos[i:i + 64]
            report = run_tensor_batch([project] * len(chunk), epsilon=[self.epsilon(r) for r in chunk],
                                      cuda_graph=True, cuda_graph_steps=16, launch=launch)
            report.raise_for_errors()
            traces.extend(item.result.signals[:, 0].astype(np.float64) for item in report.items)
        return np.asarray(traces)

    def transmission(self, rhos):
        """Complex t (n, 16): one density through a resident plan replayed from a CUDA graph, several through
        the batched engine."""
        rhos = list(rhos)
        traces = [self.trace(rhos[0])] if len(rhos) == 1 else self.simulate(rhos)
        return (np.asarray(traces) @ self.dft().T) / self.reference()[None, :]

    def trace(self, rho):
        """Ez trace of one density: material upload, reset and graph replays of a resident plan."""
        import torch
        from .native import NativeGrid
        from .plan import plan_grid
        if 'grid' not in self._cache:
            plan = plan_grid(self.project())
            grid = NativeGrid(plan, kernel='auto')
            stream = torch.cuda.Stream()
            stream.wait_stream(torch.cuda.current_stream())
            width = 16 if self.steps % 16 == 0 else 1
            with torch.cuda.stream(stream):
                grid.step(1, stream)
                grid.reset()
                graph = torch.cuda.CUDAGraph()
                graph.capture_begin()
                grid.step(width, stream)
                graph.capture_end()
            torch.cuda.synchronize()
            self._cache['grid'] = (grid, graph, stream, width)
        grid, graph, stream, width = self._cache['grid']
        with torch.cuda.stream(stream):
            grid.set_material((1 / self.epsilon(rho)).astype(np.float32 if self.precision == 'float32' else np.float64))
            grid.reset()
            for _ in range(self.steps // width):
                graph.replay()
        torch.cuda.synchronize()
        return grid.get_traces()[:, 0].astype(np.float64)

    @staticmethod
    def fom(t):
        """Mean |t|^2 over the wavelengths (numpy or torch, last axis)."""
        return (t.real ** 2 + t.imag ** 2).mean(axis=-1) if isinstance(t, np.ndarray) else (t.abs() ** 2).mean(dim=-1)


def random_densities(count, pixels=100, seed=0):
    """Seeded smoothed random patterns: Gaussian-filtered noise (sigma 2-8 px), sigmoid-projected with a random
    sharpness, a random fill level and a random share of straight-guide background."""
    from scipy.ndimage import gaussian_filter
    rng = np.random.default_rng(seed)
    out = np.empty((count, pixels, pixels), dtype=np.float32)
    y = np.arange(pixels) - pixels / 2 + .5
    guide = (np.abs(y) <= 10)[None, :].astype(np.float64) * np.ones((pixels, 1))
    for k in range(count):
        sigma = rng.uniform(2, 8)
        field = gaussian_filter(rng.normal(size=(pixels, pixels)), sigma)
        field = (field - field.mean()) / max(field.std(), 1e-12)
        beta = rng.uniform(1, 6)
        rho = 1 / (1 + np.exp(-beta * (field - rng.normal(0, .6))))
        mix = rng.uniform(0, .6)
        out[k] = np.clip((1 - mix) * rho + mix * guide, 0, 1)
    return out


def generate_dataset(problem, count=4096, seed=0, log=None):
    """(rho (count, P, P) float32, targets (count, 32) float32 = [Re t, Im t], seconds)."""
    rhos = random_densities(count, problem.pixels, seed)
    started = time.perf_counter()
    problem.reference()
    t = []
    for i in range(0, count, 512):
        t.append(problem.transmission(rhos[i:i + 512]))
        if log:
            log(i + len(t[-1]), time.perf_counter() - started)
    t = np.concatenate(t)
    targets = np.concatenate([t.real, t.imag], axis=1).astype(np.float32)
    return rhos, targets, time.perf_counter() - started


def _adjoint_value_and_grad(problem, model, theta):
    """FOM and d FOM / d theta through the discrete adjoint (rho = sigmoid(theta))."""
    import torch
    theta = theta.detach().requires_grad_(True)
    rho = torch.sigmoid(theta)
    eps = problem.epsilon_torch(rho.to(torch.float32)).contiguous()
    signals = model(eps).signals[:, 0].to(torch.float64)
    dft = torch.as_tensor(problem.dft(), device=signals.device)
    ref = torch.as_tensor(problem.reference(), device=signals.device)
    t = (dft @ signals.to(dft.dtype)) / ref
    fom = TransmissionProblem.fom(t)
    fom.backward()
    return float(fom.detach()), theta.grad.detach()


def adjoint_design(problem, iterations=30, lr=.2, seed=0, theta0=None, log=None):
    """Plain loop: Adam ascent on theta with discrete-adjoint gradients. Returns a history of
    (seconds, fom) after each iteration and the final theta."""
    import torch
    from .adjoint import DifferentiableSimulation
    model = DifferentiableSimulation(problem.project())
    theta = torch.zeros((problem.pixels, problem.pixels), dtype=torch.float64, device='cuda') if theta0 is None else theta0.clone()
    opt = torch.optim.Adam([theta.requires_grad_(True)], lr=lr)
    history, started = [], time.perf_counter()
    for k in range(iterations):
        fom, grad = _adjoint_value_and_grad(problem, model, theta)
        opt.zero_grad()
        theta.grad = -grad
        opt.step()
        history.append((time.perf_counter() - started, fom))
        if log:
            log(k, fom)
    final = problem.fom(problem.transmission([torch.sigmoid(theta.detach()).cpu().numpy()]))[0]
    history.append((time.perf_counter() - started, float(final)))
    model.close()
    return history, theta.detach()


def surrogate_design(problem, net, target_fom, iterations=200, lr=.2, verify_every=5, finetune_steps=10, data=None,
                     theta0=None, max_seconds=None, patience=2, adjoint_lr=.2, log=None):
    """Surrogate-assisted loop. Phase 1: Adam ascent on theta with the network's input gradient; every
    ``verify_every``-th iterate is simulated (FDTD judges every accepted design) and becomes training data for a
    short fine-tune; the best verified design is kept. When ``patience`` verifications in a row fail to improve
    on it, phase 2 falls back to the plain discrete-adjoint loop from the best verified design. Stops once a
    verified FOM reaches ``target_fom`` (or after ``max_seconds``). Returns (history of (seconds, verified fom,
    source), best verified fom, best theta)."""
    import torch
    from .adjoint import DifferentiableSimulation
    theta = torch.zeros((problem.pixels, problem.pixels), dtype=torch.float64, device='cuda') if theta0 is None else theta0.clone()
    opt = torch.optim.Adam([theta.requires_grad_(True)], lr=lr)
    half = net.outputs // 2
    best, best_theta, history = -math.inf, theta.detach().clone(), []
    verified_rho, verified_y = [], []
    rng = np.random.default_rng(0)
    started = time.perf_counter()
    stalled = 0

    def done():
        return best >= target_fom or (max_seconds and time.perf_counter() - started > max_seconds)
    for k in range(1, iterations + 1):
        with torch.no_grad():
            rho = torch.sigmoid(theta).to(torch.float32)[None]
        out = net.forward(rho)
        dout = torch.zeros_like(out)
        dout[:, :half] = 2 * out[:, :half] / half          # d mean|t|^2 / d Re t
        dout[:, half:] = 2 * out[:, half:] / half          # d mean|t|^2 / d Im t
        grad_rho = net.backward(dout, parameters=False, input_gradient=True)[0].to(torch.float64)
        with torch.no_grad():
            s = torch.sigmoid(theta)
            grad_theta = grad_rho * s * (1 - s)
        opt.zero_grad()
        theta.grad = -grad_theta
        opt.step()
        if k % verify_every:
            continue
        rho_np = torch.sigmoid(theta.detach()).cpu().numpy()
        t = problem.transmission([rho_np])[0]
        fom = float(problem.fom(t[None])[0])
        verified_rho.append(rho_np.astype(np.float32))
        verified_y.append(np.concatenate([t.real, t.imag]).astype(np.float32))
        if fom > best + 1e-4:
            best, best_theta, stalled = fom, theta.detach().clone(), 0
        else:
            stalled += 1
        history.append((time.perf_counter() - started, fom, 'surrogate'))
        if log:
            log(k, fom, 'surrogate')
        if done() or stalled >= patience:
            break
        if finetune_steps and data is not None:
            rho_train, y_train = data
            vr = torch.tensor(np.stack(verified_rho[-16:]), device='cuda')
            vy = torch.tensor(np.stack(verified_y[-16:]), device='cuda')
            for _ in range(finetune_steps):
                idx = torch.as_tensor(rng.integers(0, rho_train.shape[0], 64 - vr.shape[0]), device='cuda')
                net.train_step(torch.cat([rho_train[idx], vr]), torch.cat([y_train[idx], vy]), lr=3e-4)
    if not done():
        # Phase 2: the plain adjoint loop from the best verified design (each iterate is an FDTD evaluation).
        model = DifferentiableSimulation(problem.project())
        theta = best_theta.clone()
        opt = torch.optim.Adam([theta.requires_grad_(True)], lr=adjoint_lr)
        while not done():
            fom, grad = _adjoint_value_and_grad(problem, model, theta)
            if fom > best:
                best, best_theta = fom, theta.detach().clone()
            history.append((time.perf_counter() - started, fom, 'adjoint'))
            if log:
                log(len(history), fom, 'adjoint')
            if done():
                break
            opt.zero_grad()
            theta.grad = -grad
            opt.step()
        model.close()
    return history, best, best_theta

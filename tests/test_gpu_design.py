"""The design loops end to end on a reduced scene (160 x 160 cells at 0.05 um, 40 x 40 design pixels):
dataset generation through the batched engine, surrogate training, the plain adjoint loop and the
surrogate-assisted loop with FDTD verification."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def small_problem():
    from torchfdtd_b200.design import TransmissionProblem
    return TransmissionProblem(cells=160, pixels=40, mesh=.05, steps=1600)


def test_batched_dataset_is_normalised_to_the_straight_guide():
    from torchfdtd_b200.design import generate_dataset
    problem = small_problem()
    straight = problem.transmission([problem.straight(), problem.straight()])      # batched path, twice
    np.testing.assert_allclose(straight, 1.0, rtol=1e-12, atol=1e-12)               # bitwise the single-plan trace
    rhos, targets, seconds = generate_dataset(problem, count=96, seed=1)
    assert rhos.shape == (96, 40, 40) and targets.shape == (96, 32) and np.isfinite(targets).all()
    assert targets.std() > 1e-3


def test_adjoint_loop_improves_and_surrogate_loop_is_verified_by_fdtd():
    import torch
    from torchfdtd_b200.design import adjoint_design, generate_dataset, surrogate_design
    from torchfdtd_b200.surrogate import ConvNeuralOperator
    problem = small_problem()
    history, theta = adjoint_design(problem, iterations=6, lr=.3)
    foms = [f for _, f in history]
    assert foms[-1] > foms[0] + 1e-3
    rhos, targets, _ = generate_dataset(problem, count=256, seed=2)
    net = ConvNeuralOperator(outputs=32, seed=0, input_shape=(40, 40))
    rho_t, y_t = torch.tensor(rhos, device='cuda'), torch.tensor(targets, device='cuda')
    losses = net.fit(rho_t, y_t, epochs=8, batch=32, lr=2e-3)
    assert losses[-1] < losses[0]
    hist, best, best_theta = surrogate_design(problem, net, target_fom=foms[-1], iterations=40, lr=.3, verify_every=5,
                                              finetune_steps=5, data=(rho_t, y_t))
    assert len(hist) >= 1 and all(np.isfinite(f) for _, f, _ in hist)
    verified = problem.fom(problem.transmission([torch.sigmoid(best_theta).cpu().numpy()]))[0]
    assert abs(verified - best) <= 1e-5 * max(1, abs(best))                         # FDTD judged the best design


def test_surrogate_loop_reaches_the_plain_fom_in_less_time():
    """The race on the reduced scene, from the same start (theta = 0, rho = 0.5): the plain adjoint loop runs 20
    iterations; the surrogate-assisted loop, with a network trained on 1024 batched FDTD samples, must reach the
    plain loop's FDTD-verified FOM within 1 % in less wall time (every design it reports is FDTD-verified).
    Dataset generation and training are not timed: they are paid once for many designs."""
    import torch
    from torchfdtd_b200.design import adjoint_design, generate_dataset, surrogate_design
    from torchfdtd_b200.surrogate import ConvNeuralOperator
    problem = small_problem()
    rhos, targets, _ = generate_dataset(problem, count=1024, seed=2)
    net = ConvNeuralOperator(outputs=32, seed=0, input_shape=(40, 40))
    rho_t, y_t = torch.tensor(rhos, device='cuda'), torch.tensor(targets, device='cuda')
    net.fit(rho_t, y_t, epochs=20, batch=64, lr=2e-3)
    adjoint_design(problem, iterations=2, lr=.3)                                     # loads the kernels once
    history, _ = adjoint_design(problem, iterations=20, lr=.3)
    plain_seconds, plain_fom = history[-1]
    hist, best, best_theta = surrogate_design(problem, net, target_fom=0.99 * plain_fom, iterations=200, lr=.3,
                                              verify_every=5, finetune_steps=5, data=(rho_t, y_t), max_seconds=2 * plain_seconds)
    seconds = hist[-1][0]
    verified = problem.fom(problem.transmission([torch.sigmoid(best_theta).cpu().numpy()]))[0]
    assert abs(verified - best) <= 1e-5 * max(1, abs(best))
    assert best >= 0.99 * plain_fom, (best, plain_fom)
    assert seconds < plain_seconds, (seconds, plain_seconds)

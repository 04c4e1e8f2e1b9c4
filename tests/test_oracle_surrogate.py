"""The CPU network oracle (float64, no BF16 rounding) against central differences."""
import numpy as np

from oracle.surrogate_oracle import LAYERS, NetworkOracle


def random_params(k=6, seed=0, features=64):
    rng = np.random.default_rng(seed)
    p = {}
    for l, (ci, _) in enumerate(LAYERS):
        p[f'w{l}'] = rng.normal(size=(9, 64, ci)) * np.sqrt(2 / (9 * (4 if l == 0 else ci)))
        p[f'b{l}'] = rng.normal(size=64) * .1
    p['wh'] = rng.normal(size=(k, features)) / np.sqrt(features)
    p['bh'] = rng.normal(size=k) * .1
    return p


def test_network_oracle_gradients_match_central_differences():
    rng = np.random.default_rng(1)
    params = random_params(features=1 * 1 * 64)     # 11 x 9 input -> 1 x 1 after four stride-2 layers
    rho = rng.uniform(0, 1, size=(2, 11, 9))
    dout = rng.normal(size=(2, 6))
    net = NetworkOracle(params, bf16=False)
    net.forward(rho)
    grads = net.backward(dout, input_gradient=True)

    def objective(p=params, r=rho):
        return float((NetworkOracle(p, bf16=False).forward(r) * dout).sum())
    h = 1e-6
    for name, index in (('w0', (4, 3, 0)), ('w3', (0, 10, 20)), ('w7', (8, 63, 1)), ('b5', (7,)), ('wh', (2, 9)), ('bh', (1,))):
        up = {k: v.copy() for k, v in params.items()}
        down = {k: v.copy() for k, v in params.items()}
        up[name][index] += h
        down[name][index] -= h
        fd = (objective(up) - objective(down)) / (2 * h)
        assert abs(grads[name][index] - fd) <= 1e-6 * max(1.0, abs(fd)), (name, grads[name][index], fd)
    for index in ((0, 5, 4), (1, 0, 8)):
        up, down = rho.copy(), rho.copy()
        up[index] += h
        down[index] -= h
        fd = (objective(r=up) - objective(r=down)) / (2 * h)
        assert abs(grads['rho'][index] - fd) <= 1e-6 * max(1.0, abs(fd))

"""The surrogate's BF16 tensor-core kernels (forward, backward data, backward weight, head, loss, Adam)
against the CPU network oracle, which rounds the same operands to bfloat16 and accumulates in float64.

Bars: outputs within 1e-2 relative L2 and parameter and input gradients within 2e-2: activations,
pre-activations and their gradients are held in BF16, so wherever the GPU's FP32 sum and the oracle's FP64 sum
of the same BF16 operands fall on different sides of a BF16 rounding boundary the element moves by 2^-8,
and the flips compound over 8 layers; training lowers the loss."""
import numpy as np
import pytest

from oracle.surrogate_oracle import NetworkOracle

pytestmark = pytest.mark.gpu


def rel(a, b):
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-30))


@pytest.fixture(params=['tcgen05', 'tcgen05_gather', 'mma'])
def tensor_path(request):
    from torchfdtd_b200.surrogate import set_tensor_path
    set_tensor_path(request.param)
    yield request.param
    set_tensor_path('tcgen05')


@pytest.mark.parametrize('shape', [(3, 24, 20), (2, 33, 17), (5, 40, 40)])
def test_forward_and_every_gradient_match_the_oracle(shape, tensor_path):
    import torch
    from torchfdtd_b200.surrogate import ConvNeuralOperator, device_status
    net = ConvNeuralOperator(outputs=6, seed=3, input_shape=shape[1:])
    for k in net.params:
        if k.startswith('b'):
            net.params[k].copy_(torch.randn(net.params[k].shape, generator=torch.Generator().manual_seed(5)) * .1)
    net.cast_weights()
    rng = np.random.default_rng(2)
    rho = rng.uniform(0, 1, size=shape).astype(np.float32)
    dout = rng.normal(size=(shape[0], 6)).astype(np.float32)
    out = net.forward(torch.tensor(rho, device='cuda')).cpu().numpy()
    drho = net.backward(torch.tensor(dout, device='cuda'), input_gradient=True).cpu().numpy()
    oracle = NetworkOracle(net.state_dict(), bf16=True)
    expected = oracle.forward(rho)
    grads = oracle.backward(dout.astype(np.float64), input_gradient=True)
    assert rel(out, expected) <= 1e-2
    for k, g in net.grads.items():
        assert rel(g.cpu().numpy(), grads[k]) <= 2e-2, k
    assert rel(drho, grads['rho']) <= 2e-2
    assert device_status() == 0


def test_loss_and_adam_match_their_definitions():
    import torch
    from torchfdtd_b200.surrogate import ConvNeuralOperator
    net = ConvNeuralOperator(outputs=4, seed=1, input_shape=(16, 16))
    rho = torch.rand((2, 16, 16), device='cuda')
    y = torch.randn((2, 4), device='cuda')
    out = net.forward(rho).clone()
    loss = float(net.loss(y))
    assert abs(loss - float(((out - y) ** 2).mean())) <= 1e-6 * max(1, loss)
    before = {k: v.clone() for k, v in net.params.items()}
    g = {k: torch.randn_like(v) for k, v in net.params.items()}
    for k in g:
        net.grads[k].copy_(g[k])
    net.adam_step(lr=1e-2)
    for k, p in net.params.items():           # first Adam step: p - lr * g / (|g| + eps)
        expected = before[k] - 1e-2 * g[k] / (g[k].abs() + 1e-8)
        torch.testing.assert_close(p, expected, rtol=1e-5, atol=1e-6)


def test_training_fits_a_smooth_map():
    import torch
    from torchfdtd_b200.surrogate import ConvNeuralOperator
    gen = torch.Generator(device='cpu').manual_seed(0)
    rho = torch.rand((512, 20, 20), generator=gen).cuda()
    target = torch.stack([rho.mean(dim=(1, 2)), (rho[:, :10] - rho[:, 10:]).mean(dim=(1, 2))], dim=1) * 4
    net = ConvNeuralOperator(outputs=2, seed=0, input_shape=(20, 20))
    history = net.fit(rho, target, epochs=15, batch=64, lr=3e-3)
    assert history[-1] < .1 * history[0]


@pytest.mark.parametrize('ci,stride,shape', [(16, 1, (3, 24, 20)), (64, 2, (2, 33, 17)), (64, 1, (4, 40, 40)), (16, 1, (2, 61, 57))])
def test_backward_weight_paths_agree_and_match_float64(ci, stride, shape):
    """tfd_sg_conv_backward_weight on the tcgen05 kernel (taps stacked in M, MN-major operands, bias from a ones
    row) and on the mma.sync kernel, against dW[tap, co, ci] = sum_p dz[p, co] x[in(p, tap), ci] and
    dbias[co] = sum_p dz[p, co] summed in float64 over the same BF16 operands. Shapes with more than one
    4096-pixel chunk and a ragged last 32-pixel block are included."""
    import ctypes
    import torch
    from torchfdtd_b200.surrogate import WGRAD_CHUNK, _lib, device_status, out_size, set_tensor_path
    lib, check = _lib()
    n, h, w = shape
    ho, wo = out_size(h, stride), out_size(w, stride)
    gen = torch.Generator().manual_seed(ci + stride + h)
    x = torch.randn((n, h, w, ci), generator=gen).to(torch.bfloat16)
    dz = torch.randn((n, ho, wo, 64), generator=gen).to(torch.bfloat16)
    size = ctypes.c_size_t()
    check(lib.tfd_sg_wgrad_scratch(n, h, w, ci, stride, WGRAD_CHUNK, ctypes.byref(size)))
    scratch = torch.empty(size.value // 4 + 1, dtype=torch.float32, device='cuda')
    xd, dzd = x.cuda(), dz.cuda()
    results = {}
    for path in ('tcgen05', 'mma'):
        set_tensor_path(path)
        try:
            dw = torch.full((9, 64, ci), float('nan'), device='cuda')
            db = torch.full((64,), float('nan'), device='cuda')
            check(lib.tfd_sg_conv_backward_weight(ctypes.c_void_p(dzd.data_ptr()), ctypes.c_void_p(xd.data_ptr()),
                                                  ctypes.c_void_p(dw.data_ptr()), ctypes.c_void_p(db.data_ptr()),
                                                  ctypes.c_void_p(scratch.data_ptr()), size.value, n, h, w, ci, stride, WGRAD_CHUNK,
                                                  ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)))
            torch.cuda.synchronize()
            results[path] = (dw.cpu().numpy().astype(np.float64), db.cpu().numpy().astype(np.float64))
        finally:
            set_tensor_path('tcgen05')
    assert device_status() == 0
    xs, dzs = x.double().numpy(), dz.double().numpy().reshape(-1, 64)
    pad = np.zeros((n, h + 2, w + 2, ci))
    pad[:, 1:-1, 1:-1] = xs
    expected = np.empty((9, 64, ci))
    for t in range(9):
        ky, kx = divmod(t, 3)
        xt = pad[:, ky:ky + stride * (ho - 1) + 1:stride, kx:kx + stride * (wo - 1) + 1:stride].reshape(-1, ci)
        expected[t] = dzs.T @ xt
    expected_bias = dzs.sum(axis=0)
    for path, (dw, db) in results.items():
        assert rel(dw, expected) <= 1e-5, path
        assert rel(db, expected_bias) <= 1e-5, path
    assert rel(results['tcgen05'][0], results['mma'][0]) <= 1e-5


def _conv_reference(x, w, stride):
    """z[p, co] = sum_{tap, ci} x[in(p, tap), ci] w[tap, co, ci] in float64 (zero padding 1)."""
    n, h, wd, ci = x.shape
    ho, wo = (h - 1) // stride + 1, (wd - 1) // stride + 1
    pad = np.zeros((n, h + 2, wd + 2, ci))
    pad[:, 1:-1, 1:-1] = x
    z = np.zeros((n, ho, wo, w.shape[1]))
    for t in range(9):
        ky, kx = divmod(t, 3)
        z += pad[:, ky:ky + stride * (ho - 1) + 1:stride, kx:kx + stride * (wo - 1) + 1:stride] @ w[t].T
    return z


@pytest.mark.parametrize('ci,shape', [(16, (3, 24, 20)), (64, (2, 33, 17)), (64, (64, 40, 40)), (16, (5, 100, 100)), (64, (1, 9, 500))])
def test_shifted_window_conv_matches_the_gather_kernel_and_float64(ci, shape):
    """Stride-1 forward and backward data on the shifted-window tcgen05 kernel against the per-tap gather kernel
    and against float64 sums of the same BF16 operands: grids whose padded rows do not fill whole 128-row tiles,
    more tiles than CTAs (the persistent loop), and a 500-wide row whose patch exceeds shared memory (both paths
    then run the gather kernel)."""
    import ctypes
    import torch
    from torchfdtd_b200.surrogate import _lib, device_status, set_tensor_path
    lib, check = _lib()
    n, h, w = shape
    gen = torch.Generator().manual_seed(ci + h + w)
    x = torch.randn((n, h, w, ci), generator=gen).to(torch.bfloat16)
    wt = (torch.randn((9, 64, ci), generator=gen) / (3 * ci ** .5)).to(torch.bfloat16)
    wt_t = wt.transpose(1, 2).contiguous()                          # [tap][ci][co] for backward data
    bias = torch.randn(64, generator=gen) * .1
    dz = torch.randn((n, h, w, 64), generator=gen).to(torch.bfloat16)
    dev = {k: v.cuda() for k, v in dict(x=x, w=wt, wt=wt_t, bias=bias, dz=dz).items()}
    ptr = lambda t: ctypes.c_void_p(t.data_ptr())
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    out = {}
    for path in ('tcgen05', 'tcgen05_gather'):
        set_tensor_path(path)
        try:
            z = torch.empty((n, h, w, 64), dtype=torch.bfloat16, device='cuda')
            a = torch.empty_like(z)
            dx = torch.full((n, h, w, ci), float('nan'), device='cuda')
            check(lib.tfd_sg_conv_forward(ptr(dev['x']), ptr(dev['w']), ptr(dev['bias']), ptr(z), ptr(a), n, h, w, ci, 1, stream))
            check(lib.tfd_sg_conv_backward_data(ptr(dev['dz']), ptr(dev['wt']), None, ptr(dx), n, h, w, ci, 1, stream))
            torch.cuda.synchronize()
            out[path] = (z.float().cpu().numpy(), a.float().cpu().numpy(), dx.cpu().numpy())
        finally:
            set_tensor_path('tcgen05')
    assert device_status() == 0
    zref = _conv_reference(x.double().numpy(), wt.double().numpy(), 1) + bias.double().numpy()
    # backward data = the conv of dz with the taps flipped and the weights transposed
    dxref = _conv_reference(dz.double().numpy(), wt_t.double().numpy()[::-1], 1)
    for path, (z, a, dx) in out.items():
        assert rel(z, zref) <= 1e-2, path
        assert rel(dx, dxref) <= 1e-5, path
    assert rel(out['tcgen05'][0], out['tcgen05_gather'][0]) <= 1e-3
    assert rel(out['tcgen05'][1], out['tcgen05_gather'][1]) <= 1e-3
    assert rel(out['tcgen05'][2], out['tcgen05_gather'][2]) <= 1e-5


@pytest.mark.parametrize('ci,shape', [(64, (2, 33, 17)), (16, (3, 24, 20)), (64, (4, 50, 50)), (64, (1, 1, 7))])
def test_stride2_backward_data_by_parity_class_matches_float64(ci, shape):
    """Backward data of a stride-2 layer (the tcgen05 kernels run each parity class of input pixels with only the
    taps that reach it: as shifted windows of the dz image, and in the gather form) against the mma.sync kernel and
    against dx[2 oy + ky - 1, 2 ox + kx - 1] += dz[oy, ox] w[tap]
    summed in float64 over the same BF16 operands; odd sizes leave classes of different sizes, and a one-row image
    leaves two classes empty."""
    import ctypes
    import torch
    from torchfdtd_b200.surrogate import _lib, device_status, out_size, set_tensor_path
    lib, check = _lib()
    n, h, w = shape
    ho, wo = out_size(h, 2), out_size(w, 2)
    gen = torch.Generator().manual_seed(7 * ci + h)
    wt = (torch.randn((9, 64, ci), generator=gen) / 24).to(torch.bfloat16)
    wt_t = wt.transpose(1, 2).contiguous()
    dz = torch.randn((n, ho, wo, 64), generator=gen).to(torch.bfloat16)
    dzd, wtd = dz.cuda(), wt_t.cuda()
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    out = {}
    for path in ('tcgen05', 'tcgen05_gather', 'mma'):
        set_tensor_path(path)
        try:
            dx = torch.full((n, h, w, ci), float('nan'), device='cuda')
            check(lib.tfd_sg_conv_backward_data(ctypes.c_void_p(dzd.data_ptr()), ctypes.c_void_p(wtd.data_ptr()), None,
                                                ctypes.c_void_p(dx.data_ptr()), n, h, w, ci, 2, stream))
            torch.cuda.synchronize()
            out[path] = dx.cpu().numpy()
        finally:
            set_tensor_path('tcgen05')
    assert device_status() == 0
    d, wf = dz.double().numpy(), wt.double().numpy()
    pad = np.zeros((n, h + 2, w + 2, ci))
    for t in range(9):
        ky, kx = divmod(t, 3)
        pad[:, ky:ky + 2 * (ho - 1) + 1:2, kx:kx + 2 * (wo - 1) + 1:2] += d @ wf[t]
    expected = pad[:, 1:-1, 1:-1]
    for path, dx in out.items():
        assert np.isfinite(dx).all(), path
        assert rel(dx, expected) <= 1e-5, path


@pytest.mark.parametrize('shape', [(2, 33, 17), (3, 50, 50), (2, 100, 100), (1, 1, 7)])
def test_stride2_forward_phase_windows_match_the_gather_kernel_and_float64(shape):
    """Stride-2 forward of a 64-channel layer on the tcgen05 path (the per-tap gather kernel: the shifted-window form
    with the four row/column phases of the padded input as windows of one patch was measured slower, 821 against
    410 us on the 100x100 layer) against float64 sums of the same BF16 operands, on odd sizes and a one-row image."""
    import ctypes
    import torch
    from torchfdtd_b200.surrogate import _lib, device_status, out_size, set_tensor_path
    lib, check = _lib()
    n, h, w = shape
    ho, wo = out_size(h, 2), out_size(w, 2)
    gen = torch.Generator().manual_seed(h * w)
    x = torch.randn((n, h, w, 64), generator=gen).to(torch.bfloat16)
    wt = (torch.randn((9, 64, 64), generator=gen) / 24).to(torch.bfloat16)
    bias = torch.randn(64, generator=gen) * .1
    xd, wd, bd = x.cuda(), wt.cuda(), bias.cuda()
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    out = {}
    for path in ('tcgen05', 'tcgen05_gather'):
        set_tensor_path(path)
        try:
            z = torch.empty((n, ho, wo, 64), dtype=torch.bfloat16, device='cuda')
            a = torch.empty_like(z)
            check(lib.tfd_sg_conv_forward(ctypes.c_void_p(xd.data_ptr()), ctypes.c_void_p(wd.data_ptr()), ctypes.c_void_p(bd.data_ptr()),
                                          ctypes.c_void_p(z.data_ptr()), ctypes.c_void_p(a.data_ptr()), n, h, w, 64, 2, stream))
            torch.cuda.synchronize()
            out[path] = (z.float().cpu().numpy(), a.float().cpu().numpy())
        finally:
            set_tensor_path('tcgen05')
    assert device_status() == 0
    zref = _conv_reference(x.double().numpy(), wt.double().numpy(), 2) + bias.double().numpy()
    for path, (z, a) in out.items():
        assert rel(z, zref) <= 1e-2, path
    assert rel(out['tcgen05'][0], out['tcgen05_gather'][0]) <= 1e-3
    assert rel(out['tcgen05'][1], out['tcgen05_gather'][1]) <= 1e-3

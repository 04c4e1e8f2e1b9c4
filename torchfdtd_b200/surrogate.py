"""Learned surrogate: a convolutional neural operator trained by the engine's own BF16 kernels.

The network maps a design density rho (n, H, W) in [0, 1] to K real outputs (here the real and imaginary parts
of a complex transmission spectrum). Architecture: packed input (2 rho - 1, x, y, 1; 16 channels), 8 conv
layers of 64 channels (3x3, zero padding 1, strides 1, 2, 1, 2, 1, 2, 1, 2, GELU) and a linear head on the
flattened last feature map (positions stay distinct: the scenes are not translation invariant). Every op of
training and inference runs in ``csrc/surrogate.cu``: BF16 tensor-core implicit GEMMs with FP32 accumulation
for the convolutions (forward, backward data, backward weight), FP32 head, mean-squared loss and Adam with
FP32 master weights. Torch provides the device buffers only.
"""
from __future__ import annotations

import ctypes
import math

import numpy as np

LAYERS = ((16, 1), (64, 2), (64, 1), (64, 2), (64, 1), (64, 2), (64, 1), (64, 2))   # (input channels, stride)
CO = 64
WGRAD_CHUNK = 4096          # the most output pixels per weight-gradient partial sum (small layers use fewer)

_SIGNATURES = {
    'tfd_sg_pack_input': [ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p],
    'tfd_sg_conv_forward': [ctypes.c_void_p] * 5 + [ctypes.c_int32] * 5 + [ctypes.c_void_p],
    'tfd_sg_conv_backward_data': [ctypes.c_void_p] * 4 + [ctypes.c_int32] * 5 + [ctypes.c_void_p],
    'tfd_sg_wgrad_scratch': [ctypes.c_int32] * 6 + [ctypes.POINTER(ctypes.c_size_t)],
    'tfd_sg_conv_backward_weight': [ctypes.c_void_p] * 5 + [ctypes.c_size_t] + [ctypes.c_int32] * 6 + [ctypes.c_void_p],
    'tfd_sg_head_forward': [ctypes.c_void_p] * 4 + [ctypes.c_int32] * 3 + [ctypes.c_void_p],
    'tfd_sg_mse': [ctypes.c_void_p] * 4 + [ctypes.c_int32, ctypes.c_void_p],
    'tfd_sg_head_backward': [ctypes.c_void_p] * 7 + [ctypes.c_int32] * 3 + [ctypes.c_void_p],
    'tfd_sg_adam': [ctypes.c_void_p] * 4 + [ctypes.c_int64, ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_float,
                                            ctypes.c_int32, ctypes.c_void_p],
    'tfd_sg_cast_weights': [ctypes.c_void_p] * 3 + [ctypes.c_int32, ctypes.c_void_p],
    'tfd_sg_set_tensor_path': [ctypes.c_int32],
    'tfd_sg_status': [ctypes.POINTER(ctypes.c_int32)],
}


def _lib():
    from .native import check, library
    lib = library()
    if not getattr(lib, '_sg_bound', False):
        for name, args in _SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = ctypes.c_int
            fn.argtypes = args
        lib._sg_bound = True
    return lib, check


def set_tensor_path(mode):
    """'tcgen05' (default): conv forward, backward data and backward weight on the 5th-generation tensor cores with
    tensor-memory accumulators, stride-1 layers as shifted windows of a patch loaded once per tile (where the patch
    fits in shared memory); 'tcgen05_gather': the same kernels with a per-tap gather for every layer; 'mma': on
    warp-level mma.sync kernels."""
    lib, check = _lib()
    check(lib.tfd_sg_set_tensor_path({'mma': 0, 'tcgen05': 1, 'tcgen05_gather': 2}[mode]))


def device_status():
    """1 if a bounded tensor-core wait timed out since the last call, else 0 (reading clears it)."""
    lib, check = _lib()
    v = ctypes.c_int32()
    check(lib.tfd_sg_status(ctypes.byref(v)))
    return v.value


def _p(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


def _stream():
    import torch
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def out_size(n, stride):
    return (n - 1) // stride + 1


class ConvNeuralOperator:
    """The surrogate network with its Adam state; ``forward``, ``backward`` and ``train_step`` run the
    engine's kernels on CUDA tensors."""

    def __init__(self, outputs=32, seed=0, device='cuda', input_shape=(100, 100)):
        import torch
        self.outputs = outputs
        h, w = input_shape
        for _, stride in LAYERS:
            h, w = out_size(h, stride), out_size(w, stride)
        self.input_shape = tuple(input_shape)
        self.features = h * w * CO
        self.device = torch.device(device)
        g = torch.Generator(device='cpu').manual_seed(seed)
        self.params = {}
        for l, (ci, _) in enumerate(LAYERS):
            fan_in = 9 * (4 if l == 0 else ci)
            self.params[f'w{l}'] = (torch.randn((9, CO, ci), generator=g) * math.sqrt(2.0 / fan_in)).to(self.device)
            self.params[f'b{l}'] = torch.zeros(CO, device=self.device)
        self.params['wh'] = (torch.randn((outputs, self.features), generator=g) / math.sqrt(self.features)).to(self.device)
        self.params['bh'] = torch.zeros(outputs, device=self.device)
        self.adam = {k: (torch.zeros_like(v), torch.zeros_like(v)) for k, v in self.params.items()}
        self.grads = {k: torch.zeros_like(v) for k, v in self.params.items()}
        self.step_count = 0
        self.wb, self.wt = {}, {}
        for l, (ci, _) in enumerate(LAYERS):
            self.wb[l] = torch.empty((9, CO, ci), dtype=torch.bfloat16, device=self.device)
            self.wt[l] = torch.empty((9, ci, CO), dtype=torch.bfloat16, device=self.device)
        self._buffers = {}
        self.cast_weights()

    # ---- parameters ----------------------------------------------------------------------------------
    def cast_weights(self):
        lib, check = _lib()
        for l, (ci, _) in enumerate(LAYERS):
            check(lib.tfd_sg_cast_weights(_p(self.params[f'w{l}']), _p(self.wb[l]), _p(self.wt[l]), ci, _stream()))

    def state_dict(self):
        return {k: v.detach().cpu().numpy().copy() for k, v in self.params.items()}

    def load_state_dict(self, state):
        import torch
        for k, v in state.items():
            self.params[k].copy_(torch.as_tensor(v, device=self.device))
        self.cast_weights()

    @property
    def flops_per_sample(self):
        """Multiply-adds x 2 of the conv layers for one sample of the last input size (forward)."""
        h, w = self._hw
        total = 0
        for ci, stride in LAYERS:
            ho, wo = out_size(h, stride), out_size(w, stride)
            total += 2 * ho * wo * CO * 9 * ci
            h, w = ho, wo
        return total

    # ---- buffers -------------------------------------------------------------------------------------
    def _alloc(self, n, h, w):
        import torch
        key = (n, h, w)
        if key in self._buffers:
            return self._buffers[key]
        lib, check = _lib()
        b = dict(x=[], z=[], a=[], dz=[], shapes=[])
        b['x0'] = torch.empty((n, h, w, 16), dtype=torch.bfloat16, device=self.device)
        hh, ww = h, w
        scratch = 0
        for ci, stride in LAYERS:
            ho, wo = out_size(hh, stride), out_size(ww, stride)
            b['shapes'].append((hh, ww, ho, wo))
            b['z'].append(torch.empty((n, ho, wo, CO), dtype=torch.bfloat16, device=self.device))
            b['a'].append(torch.empty((n, ho, wo, CO), dtype=torch.bfloat16, device=self.device))
            b['dz'].append(torch.empty((n, ho, wo, CO), dtype=torch.bfloat16, device=self.device))
            size = ctypes.c_size_t()
            check(lib.tfd_sg_wgrad_scratch(n, hh, ww, ci, stride, WGRAD_CHUNK, ctypes.byref(size)))
            scratch = max(scratch, size.value)
            hh, ww = ho, wo
        b['scratch'] = torch.empty(max(1, scratch // 4), dtype=torch.float32, device=self.device)
        b['scratch_bytes'] = scratch
        b['out'] = torch.empty((n, self.outputs), dtype=torch.float32, device=self.device)
        b['dout'] = torch.empty((n, self.outputs), dtype=torch.float32, device=self.device)
        b['loss'] = torch.empty(1, dtype=torch.float32, device=self.device)
        b['dx0'] = torch.empty((n, h, w, 16), dtype=torch.float32, device=self.device)
        self._buffers = {key: b}          # one batch shape resident at a time
        return b

    # ---- passes --------------------------------------------------------------------------------------
    def forward(self, rho):
        """rho (n, H, W) float32 CUDA tensor in [0, 1] -> outputs (n, K) float32 (a view of an internal buffer)."""
        lib, check = _lib()
        rho = rho.contiguous().float()
        n, h, w = rho.shape
        if (h, w) != self.input_shape:
            raise ValueError(f'the network was built for {self.input_shape} inputs, not {(h, w)}')
        self._hw = (h, w)
        b = self._alloc(n, h, w)
        s = _stream()
        check(lib.tfd_sg_pack_input(_p(rho), n, h, w, _p(b['x0']), s))
        x = b['x0']
        for l, (ci, stride) in enumerate(LAYERS):
            hh, ww, _, _ = b['shapes'][l]
            check(lib.tfd_sg_conv_forward(_p(x), _p(self.wb[l]), _p(self.params[f'b{l}']), _p(b['z'][l]), _p(b['a'][l]),
                                          n, hh, ww, ci, stride, s))
            x = b['a'][l]
        check(lib.tfd_sg_head_forward(_p(x), _p(self.params['wh']), _p(self.params['bh']), _p(b['out']),
                                      n, self.features, self.outputs, s))
        self._last = (n, h, w)
        return b['out']

    def backward(self, dout, parameters=True, input_gradient=False):
        """Back-propagate d(objective)/d(outputs) of the last ``forward``: fills ``self.grads`` (parameters) and
        returns d/d rho (n, H, W) float32 when ``input_gradient``."""
        lib, check = _lib()
        n, h, w = self._last
        b = self._buffers[(n, h, w)]
        s = _stream()
        dout = dout.contiguous().float()
        check(lib.tfd_sg_head_backward(_p(dout), _p(b['a'][-1]), _p(self.params['wh']), _p(b['z'][-1]),
                                       _p(self.grads['wh']) if parameters else None, _p(self.grads['bh']) if parameters else None,
                                       _p(b['dz'][-1]), n, self.features, self.outputs, s))
        for l in range(len(LAYERS) - 1, -1, -1):
            ci, stride = LAYERS[l]
            hh, ww, _, _ = b['shapes'][l]
            x = b['x0'] if l == 0 else b['a'][l - 1]
            if parameters:
                check(lib.tfd_sg_conv_backward_weight(_p(b['dz'][l]), _p(x), _p(self.grads[f'w{l}']), _p(self.grads[f'b{l}']),
                                                      _p(b['scratch']), b['scratch_bytes'], n, hh, ww, ci, stride, WGRAD_CHUNK, s))
            if l > 0:
                check(lib.tfd_sg_conv_backward_data(_p(b['dz'][l]), _p(self.wt[l]), _p(b['z'][l - 1]), _p(b['dz'][l - 1]),
                                                    n, hh, ww, ci, stride, s))
            elif input_gradient:
                check(lib.tfd_sg_conv_backward_data(_p(b['dz'][0]), _p(self.wt[0]), None, _p(b['dx0']), n, hh, ww, ci, stride, s))
        if input_gradient:
            return 2 * b['dx0'][..., 0]
        return None

    def loss(self, target, gradient=True):
        """Mean-squared error of the last forward against ``target`` (n, K); fills the output gradient."""
        lib, check = _lib()
        n, h, w = self._last
        b = self._buffers[(n, h, w)]
        target = target.contiguous().float()
        check(lib.tfd_sg_mse(_p(b['out']), _p(target), _p(b['dout']) if gradient else None, _p(b['loss']), target.numel(), _stream()))
        return b['loss']

    def adam_step(self, lr=1e-3, b1=.9, b2=.999, eps=1e-8):
        lib, check = _lib()
        self.step_count += 1
        s = _stream()
        for k, p in self.params.items():
            m, v = self.adam[k]
            check(lib.tfd_sg_adam(_p(p), _p(self.grads[k]), _p(m), _p(v), p.numel(), lr, b1, b2, eps, self.step_count, s))
        self.cast_weights()

    def train_step(self, rho, target, lr=1e-3):
        """One Adam step on a batch; returns the loss tensor (device, before the step)."""
        self.forward(rho)
        loss = self.loss(target).clone()
        self.backward(self._buffers[self._last]['dout'])
        self.adam_step(lr)
        return loss

    def predict(self, rho, batch=256):
        import torch
        outs = []
        for i in range(0, rho.shape[0], batch):
            outs.append(self.forward(rho[i:i + batch]).clone())
        return torch.cat(outs)

    def input_gradient(self, rho, dout):
        """d(sum(dout * net(rho)))/d rho for a batch."""
        self.forward(rho)
        return self.backward(dout, parameters=False, input_gradient=True).clone()

    def fit(self, rho, target, epochs=20, batch=64, lr=2e-3, seed=0, lr_final=1e-4, log=None):
        """Shuffled mini-batch Adam over (rho, target) device tensors with a cosine learning-rate schedule."""
        import torch
        n = rho.shape[0]
        gen = torch.Generator(device='cpu').manual_seed(seed)
        steps = epochs * (n // batch)
        k = 0
        history = []
        for epoch in range(epochs):
            order = torch.randperm(n, generator=gen).to(rho.device)
            total = torch.zeros((), device=rho.device)
            for i in range(0, n - batch + 1, batch):
                idx = order[i:i + batch]
                rate = lr_final + .5 * (lr - lr_final) * (1 + math.cos(math.pi * k / max(1, steps)))
                total += self.train_step(rho[idx], target[idx], rate)[0]
                k += 1
            history.append(float(total) / max(1, n // batch))
            if log:
                log(epoch, history[-1])
        return history


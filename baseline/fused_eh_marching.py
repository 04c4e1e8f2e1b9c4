"""Host side of the restated reference marching kernel (fused_eh_marching.cu): build, bind, run.

The reference's FusedEHMarching (torchfdtd/reversible_cuda_fused.py:259-326) advances real FP32 fields
with periodic x/y faces, CPML on z only and soft E sources (its eligibility rules:
reversible_cuda_fused.py:45-78), on z extents whose CTA fits 1024 threads and 48 KB of shared memory
(:86-90, :268-269). ``RestatedMarching`` takes the same scenes from a ``GridPlan`` and refuses the rest with
the reference's reasons. It is the comparison kernel for the product's TMA z-march, not part of the engine.
"""
from __future__ import annotations

import ctypes
import math
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
SOURCE = HERE / 'fused_eh_marching.cu'
TARGET = HERE / 'libfused_eh_marching.so'
NVCC = os.environ.get('NVCC', '/usr/local/cuda/bin/nvcc')
FLAGS = ['-gencode', 'arch=compute_100a,code=sm_100a', '-O3', '-lineinfo', '--fmad=false', '-std=c++17',
         '-Xcompiler', '-fPIC', '-shared']
MAX_SLABS, MAX_SOURCES = 2, 8
P2 = ctypes.c_void_p * 2


class FemArgs(ctypes.Structure):
    _fields_ = [('Eo', ctypes.c_void_p), ('Ho', ctypes.c_void_p), ('En', ctypes.c_void_p), ('Hn', ctypes.c_void_p),
                ('inv', ctypes.c_void_p), ('cn', ctypes.c_float), ('cn_imu', ctypes.c_float),
                ('nx', ctypes.c_int), ('ny', ctypes.c_int), ('nz', ctypes.c_int), ('zb', ctypes.c_int),
                ('rows', ctypes.c_int), ('chunk', ctypes.c_int), ('n_eslab', ctypes.c_int), ('n_hslab', ctypes.c_int),
                ('elo', ctypes.c_int * 2), ('ehi', ctypes.c_int * 2), ('hlo', ctypes.c_int * 2), ('hhi', ctypes.c_int * 2),
                ('eb', P2), ('ec', P2), ('ek', P2), ('hb', P2), ('hc', P2), ('hk', P2),
                ('epo', P2 * 2), ('epn', P2 * 2), ('hpsi', P2 * 2),
                ('n_src', ctypes.c_int), ('src_comp', ctypes.c_int * MAX_SOURCES),
                ('src_lo', (ctypes.c_int * 3) * MAX_SOURCES), ('src_hi', (ctypes.c_int * 3) * MAX_SOURCES),
                ('src_w', ctypes.c_void_p * MAX_SOURCES)]


def build(force=False, verbose=False):
    if force or not TARGET.exists() or SOURCE.stat().st_mtime > TARGET.stat().st_mtime:
        cmd = [NVCC, *FLAGS, '-o', str(TARGET), str(SOURCE)]
        if verbose:
            print(' '.join(cmd))
        subprocess.run(cmd, check=True, cwd=HERE)
    return TARGET


_LIB = None


def library():
    global _LIB
    if _LIB is None:
        if not TARGET.exists():
            raise RuntimeError(f'{TARGET.name} is not built (baseline.fused_eh_marching.build())')
        lib = ctypes.CDLL(str(TARGET))
        lib.fem_args_size.restype = ctypes.c_int
        lib.fem_smem_bytes.restype = ctypes.c_int
        lib.fem_smem_bytes.argtypes = [ctypes.c_int, ctypes.c_int]
        lib.fem_step.restype = ctypes.c_int
        lib.fem_step.argtypes = [ctypes.POINTER(FemArgs), ctypes.c_int, ctypes.c_void_p]
        if lib.fem_args_size() != ctypes.sizeof(FemArgs):
            raise RuntimeError('fem_args layout differs between the library and its binding')
        _LIB = lib
    return _LIB


def eligibility_reason(plan):
    """None when the reference's marching kernel admits the scene, else its reason."""
    nz = plan.shape[2]
    zb = 32 * ((nz + 31) // 32)
    if plan.dimension != '3d' or np.dtype(plan.dtype) != np.float32:
        return 'Fused updates require real FP32 fields.'
    if any(plan.faces[a] != ('periodic', 'periodic') for a in (0, 1)):
        return 'Fused updates require uniform periodic x/y boundaries.'
    if min(plan.shape) < 2 or 3 * math.prod(plan.shape) >= 2**31:
        return 'Grid dimensions exceed the fused launch contract.'
    if any(seg.axis != 2 for seg in plan.segments):
        return 'Fused updates support CPML on z only.'
    if plan.pec_upper:
        return 'Fused updates do not support mirror boundaries.'
    if any(s.family != 0 for s in plan.sources):
        return 'Fused forward supports volume electric sources only.'
    if zb * 6 > 1024 or 4 * 6 * zb * 3 * 4 > 48 * 1024:
        return 'z extent too large for the marching kernel'
    if len(plan.sources) > MAX_SOURCES or sum(s.forward for s in plan.segments) > MAX_SLABS:
        return 'more sources or CPML slabs than the restated launch table holds'
    return None


class RestatedMarching:
    """The reference's marching kernel on a plan's scene, with its launch shape (TY = 4 rows per CTA,
    x chunks sized to about 8 CTAs per SM). Fields start at (E, H) given in (nx, ny, nz, 3) layout."""

    def __init__(self, plan, E=None, H=None, rows=4, chunks=None, device='cuda'):
        import torch
        reason = eligibility_reason(plan)
        if reason:
            raise ValueError(reason)
        self.torch = torch
        self.plan, self.device = plan, device
        nx, ny, nz = plan.shape
        f32 = dict(dtype=torch.float32, device=device)
        zeros = np.zeros((*plan.shape, 3), np.float32)
        self.E = [torch.tensor(zeros if E is None else np.asarray(E, np.float32), **f32), torch.zeros((*plan.shape, 3), **f32)]
        self.H = [torch.tensor(zeros if H is None else np.asarray(H, np.float32), **f32), torch.zeros((*plan.shape, 3), **f32)]
        inv = np.asarray(plan.inv_eps, np.float32)
        if inv.ndim == 3:
            inv = np.repeat(inv[..., None], 3, axis=3)
        self.inv = torch.tensor(np.ascontiguousarray(inv), **f32)
        self.keep = []

        def dev(a):
            t = torch.tensor(np.ascontiguousarray(np.asarray(a, np.float32)), **f32)
            self.keep.append(t)
            return t.data_ptr()

        a = FemArgs()
        a.cn = np.float32(plan.courant)
        a.cn_imu = np.float32(np.float32(plan.courant) * np.float32(1.0))
        a.nx, a.ny, a.nz = nx, ny, nz
        a.zb = 32 * ((nz + 31) // 32)
        a.rows = rows
        yblocks = (ny + rows - 1) // rows
        if chunks is None:
            sms = torch.cuda.get_device_properties(device).multi_processor_count
            chunks = max(1, min(nx, (8 * sms + yblocks - 1) // yblocks))
        a.chunk = (nx + chunks - 1) // chunks
        self.epsi = []                        # per E slab: [[old j0, old j1], [new j0, new j1]]
        self.hpsi = []
        for seg in sorted(plan.segments, key=lambda s: (s.forward, s.lo)):
            length = seg.hi - seg.lo
            if seg.forward:
                k = a.n_hslab
                a.hlo[k], a.hhi[k] = seg.lo, seg.hi
                a.hb[k], a.hc[k], a.hk[k] = dev(seg.b), dev(seg.c), dev(seg.inv_kappa)
                pair = [torch.zeros((nx, ny, length), **f32) for _ in range(2)]
                self.hpsi.append(pair)
                for j in range(2):
                    a.hpsi[k][j] = pair[j].data_ptr()
                a.n_hslab += 1
            else:
                k = a.n_eslab
                a.elo[k], a.ehi[k] = seg.lo, seg.hi
                a.eb[k], a.ec[k], a.ek[k] = dev(seg.b), dev(seg.c), dev(seg.inv_kappa)
                self.epsi.append([[torch.zeros((nx, ny, length), **f32) for _ in range(2)] for _ in range(2)])
                a.n_eslab += 1
        for q, src in enumerate(plan.sources):
            a.src_comp[q] = src.comp
            for ax in range(3):
                a.src_lo[q][ax], a.src_hi[q][ax] = src.lo[ax], src.hi[ax]
            a.src_w[q] = dev(src.values)
        a.n_src = len(plan.sources)
        self.args = a
        self.n = 0
        self.lib = library()

    def _bind(self):
        a, p = self.args, self.n & 1
        a.Eo, a.Ho = self.E[p].data_ptr(), self.H[p].data_ptr()
        a.En, a.Hn = self.E[1 - p].data_ptr(), self.H[1 - p].data_ptr()
        a.inv = self.inv.data_ptr()
        for k, pair in enumerate(self.epsi):
            for j in range(2):
                a.epo[k][j] = pair[p][j].data_ptr()
                a.epn[k][j] = pair[1 - p][j].data_ptr()

    def step(self, count=1, stream=None):
        torch = self.torch
        s = stream if stream is not None else torch.cuda.current_stream(self.device)
        for _ in range(count):
            self._bind()
            rc = self.lib.fem_step(ctypes.byref(self.args), self.n, ctypes.c_void_p(s.cuda_stream))
            if rc:
                raise RuntimeError(f'fem_step failed with CUDA error {rc}')
            self.n += 1

    def fields(self):
        p = self.n & 1
        return self.E[p].cpu().numpy(), self.H[p].cpu().numpy()

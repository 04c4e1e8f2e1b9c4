"""Build libtfdtd.so in-tree for sm_100a (nvcc cross-compiles; no GPU needed)."""
import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / 'csrc'
TARGET = HERE / 'libtfdtd.so'
NVCC = os.environ.get('NVCC', '/usr/local/cuda/bin/nvcc')
# --fmad=false: no multiply-add contraction, as in the reference's NVRTC build
# (torchfdtd/cuda_kernels.py:49-51), so FP32 results match the reference bitwise.
FLAGS = ['-gencode', 'arch=compute_100a,code=sm_100a', '-O3', '-lineinfo', '--fmad=false', '-std=c++17',
         '-Xcompiler', '-fPIC', '-shared']


def sources():
    return sorted(CSRC.glob('*.cu'))


def stale():
    if not TARGET.exists():
        return True
    newest = max(p.stat().st_mtime for p in list(CSRC.glob('*.cu')) + list(CSRC.glob('*.cuh')) + [HERE.parent / 'include' / 'tfdtd.h'])
    return newest > TARGET.stat().st_mtime


def build(force=False, verbose=False):
    if not force and not stale():
        return TARGET
    cmd = [NVCC, *FLAGS, '-o', str(TARGET), *map(str, sources())]
    if verbose:
        print(' '.join(cmd))
    subprocess.run(cmd, check=True, cwd=CSRC)
    return TARGET


if __name__ == '__main__':
    build(force='--force' in sys.argv, verbose=True)

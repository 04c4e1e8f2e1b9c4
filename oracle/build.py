"""Build the C oracle (test infrastructure / CPU baseline) into oracle/_build/."""
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
TARGET = HERE / '_build' / 'libyee_oracle.so'
# -ffp-contract=off: no fused multiply-add, so results equal the NumPy restatement bitwise.
FLAGS = ['-O3', '-march=x86-64-v2', '-fopenmp', '-ffp-contract=off', '-fno-fast-math', '-fPIC', '-shared', '-std=c11']


def build(force=False):
    src = HERE / 'yee_cpu.c'
    if not force and TARGET.exists() and TARGET.stat().st_mtime >= src.stat().st_mtime:
        return TARGET
    TARGET.parent.mkdir(exist_ok=True)
    subprocess.run(['gcc', *FLAGS, '-o', str(TARGET), str(src)], check=True)
    return TARGET


if __name__ == '__main__':
    print(build(force='--force' in sys.argv))

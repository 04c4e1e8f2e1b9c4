import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))
GOLDEN = Path(__file__).resolve().parent / 'golden'


def reference_root():
    """The TorchFDTD source tree, when it is present: $TORCHFDTD_REFERENCE, else a ``reference`` directory beside
    this repository. Tests that read it skip without it; the GPU tests never read it."""
    path = Path(os.environ.get('TORCHFDTD_REFERENCE', ROOT.parent / 'reference'))
    return path if (path / 'torchfdtd').is_dir() else None


def pytest_configure(config):
    config.addinivalue_line('markers', 'gpu: needs a CUDA GPU (B200); runs the fused kernels through the C-ABI')


@pytest.fixture(scope='session')
def golden():
    return GOLDEN


@pytest.fixture(scope='session')
def reference_tree():
    root = reference_root()
    if root is None:
        pytest.skip('TorchFDTD source tree not present (set TORCHFDTD_REFERENCE)')
    return root

"""Array allocators selected by name, as the reference expects of ``fdtd.backend``.

``fdtd.backend`` (the package attribute) is an allocator *instance* whose class
``set_backend`` swaps; ``fdtd.backend.NumpyBackend`` (this module) is importable
by name. The reference subclasses ``NumpyBackend`` and assigns the subclass to
``fdtd.backend.__class__`` (reference ``torchfdtd/solver.py:711-721``).
"""
import numpy as np


class NumpyBackend:
    float = np.float64

    def zeros(self, shape, dtype=None):
        return np.zeros(shape, dtype=dtype or self.float)

    def ones(self, shape, dtype=None):
        return np.ones(shape, dtype=dtype or self.float)


class TorchBackend:
    """CPU torch tensors (this stand-in never allocates on a GPU)."""
    float = None
    device = 'cpu'

    def _dtype(self, dtype):
        import torch
        return dtype or self.float or torch.float64

    def zeros(self, shape, dtype=None):
        import torch
        return torch.zeros(shape, dtype=self._dtype(dtype), device=self.device)

    def ones(self, shape, dtype=None):
        import torch
        return torch.ones(shape, dtype=self._dtype(dtype), device=self.device)


backend = NumpyBackend()


def set_backend(name):
    """'numpy' or 'torch[.cuda][.float32|.float64]'; only the CPU forms allocate here."""
    import sys
    package = sys.modules[__name__.rsplit('.', 1)[0]]
    current = package.backend
    if name == 'numpy':
        current.__class__ = NumpyBackend
        current.float = np.float64
        return
    if not name.startswith('torch'):
        raise ValueError(f'unknown backend {name!r}')
    import torch
    current.__class__ = TorchBackend
    current.float = torch.float64 if name.endswith('float64') else torch.float32
    current.device = 'cuda' if '.cuda' in name else 'cpu'

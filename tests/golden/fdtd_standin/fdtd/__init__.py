"""Minimal local stand-in for the names TorchFDTD takes from the third-party
``fdtd`` package (flaport/fdtd 0.2.2), which is not installed in this image.

Test infrastructure only: it lets ``tests/golden/make_golden.py`` import the
reference's CPU path to write golden vectors. TorchFDTD's hot-path arithmetic
(``YeeGrid.curl/update_E/update_H``) does not live in ``fdtd``: the reference
only calls the ``Grid`` constructor, the backend allocators and
``set_backend`` (reference ``torchfdtd/boundaries.py:225-240``,
``torchfdtd/solver.py:11-14,668-721``), and then overwrites every attribute
the constructor set. This module supplies exactly those names.
"""
from . import backend as _backend_module
from .backend import backend, set_backend
from .grid import Grid

__all__ = ['Grid', 'backend', 'set_backend']

"""The ``Grid`` base class the reference's ``YeeGrid`` extends.

The reference calls ``super().__init__(shape=..., grid_spacing=..., courant_number=...)``
on a 2x2x(1|2) grid and then replaces E, H, the material arrays, the Courant
number and the time step (reference ``torchfdtd/boundaries.py:233-244``).
"""
import math

SPEED_LIGHT = 299792458.0


class Grid:
    def __init__(self, shape, grid_spacing, permittivity=1.0, permeability=1.0, courant_number=None):
        from . import backend as _pkg_backend  # noqa: F401  (module import keeps the package initialised)
        import sys
        bk = sys.modules[__name__.rsplit('.', 1)[0]].backend
        self.grid_spacing = float(grid_spacing)
        self.Nx, self.Ny, self.Nz = (int(v) for v in shape)
        dims = sum(n > 1 for n in (self.Nx, self.Ny, self.Nz))
        self.courant_number = courant_number if courant_number is not None else 0.99 / math.sqrt(max(dims, 1))
        self.time_step = self.courant_number * self.grid_spacing / SPEED_LIGHT
        self.E = bk.zeros((self.Nx, self.Ny, self.Nz, 3))
        self.H = bk.zeros((self.Nx, self.Ny, self.Nz, 3))
        self.inverse_permittivity = bk.ones((self.Nx, self.Ny, self.Nz, 3)) / float(permittivity)
        self.inverse_permeability = bk.ones((self.Nx, self.Ny, self.Nz, 3)) / float(permeability)
        self.time_steps_passed = 0

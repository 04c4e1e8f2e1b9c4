"""The C ABI library loads without a GPU, exports every declared entry point and validates descriptors."""
import ctypes
import re
from pathlib import Path

import numpy as np
import pytest

from torchfdtd_b200 import Project, Region, Source, Structure
from torchfdtd_b200 import native
from torchfdtd_b200.plan import plan_grid

HEADER = Path(__file__).resolve().parents[1] / 'include' / 'tfdtd.h'


def declared():
    text = HEADER.read_text()
    return sorted(set(re.findall(r'^\s*(?:const\s+)?\w[\w\s\*]*?\b(tfd_\w+)\s*\(', text, flags=re.M)))


def test_every_declared_entry_point_is_exported():
    names = declared()
    assert len(names) >= 20
    lib = native.library()
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing
    assert set(names) == set(native.SIGNATURES)


def test_error_strings():
    lib = native.library()
    assert lib.tfd_error_string(0) == b'ok'
    assert lib.tfd_error_string(2) == b'unsupported feature'


def descriptor(project, **override):
    """The tfd_desc NativeGrid would build, without touching a GPU."""
    plan = plan_grid(project)
    keep = []
    d = native.Desc()
    d.abi_version = native.TFD_ABI_VERSION
    d.nx, d.ny, d.nz = plan.shape
    d.precision = 4
    d.material_samples = 1
    d.components = native.MASK['3d' if plan.dimension == '3d' else plan.polarization]
    d.steps = plan.steps
    d.courant = plan.courant
    d.time_step = plan.time_step
    segs = (native.CpmlSegment * len(plan.segments))()
    for k, s in enumerate(plan.segments):
        arrays = [np.ascontiguousarray(v) for v in (s.b, s.c, s.inv_kappa)]
        keep += arrays
        segs[k] = native.CpmlSegment(int(s.forward), s.axis, s.lo, s.hi, *(a.ctypes.data_as(native.P_dbl) for a in arrays))
    d.n_segments, d.segments = len(plan.segments), segs
    for k, v in override.items():
        setattr(d, k, v)
    return d, keep, plan


def project3d():
    return Project(region=Region(dimension='3d', size=(1.6, 1.2, 1.0), mesh=.05, pml_cells=5, steps=20),
                   structures=[Structure(size=(1.6, .4, .3))], sources=[Source(center=(-.3, 0, 0), component='Ey')])


def plan_bytes(d):
    size = ctypes.c_size_t()
    native.check(native.library().tfd_plan_bytes(ctypes.byref(d), ctypes.byref(size)))
    return size.value


def test_plan_bytes_counts_double_buffered_fields_and_cpml():
    d, keep, plan = descriptor(project3d())
    size = plan_bytes(d)
    pitch = -(-plan.shape[0] // 32) * 32
    comp = plan.shape[2] * plan.shape[1] * pitch * 4
    # six double-buffered components, one material sample, the CPML slabs and the stage buffer
    assert size > 12 * comp + comp
    d64, keep64, _ = descriptor(project3d(), precision=8)
    assert plan_bytes(d64) > 1.9 * size


@pytest.mark.parametrize('field,value,match', [('precision', 3, 'precision'), ('nx', 0, 'positive'),
                                              ('material_samples', 2, 'material_samples'), ('components', 5, '3D grids'),
                                              ('abi_version', 99, 'ABI')])
def test_invalid_descriptors_are_refused_by_name(field, value, match):
    d, keep, _ = descriptor(project3d(), **{field: value})
    with pytest.raises(ValueError, match=match):
        plan_bytes(d)


def test_cpml_segment_outside_the_derivative_range_is_refused():
    d, keep, _ = descriptor(project3d())
    d.segments[0].lo = 0   # E family starts at 1 (backward difference)
    with pytest.raises(ValueError, match='CPML segment'):
        plan_bytes(d)


def test_create_requires_an_aligned_arena_of_the_reported_size():
    d, keep, _ = descriptor(project3d())
    size = plan_bytes(d)
    handle = ctypes.c_void_p()
    code = native.library().tfd_plan_create(ctypes.byref(d), ctypes.c_void_p(0x1000 + 8), size, None, ctypes.byref(handle))
    assert code == 4 and b'arena' in native.library().tfd_last_error()
    code = native.library().tfd_plan_create(ctypes.byref(d), ctypes.c_void_p(0x100000), size - 256, None, ctypes.byref(handle))
    assert code == 4


def test_no_gpu_means_a_loud_error_not_a_fallback(monkeypatch):
    import torch
    from torchfdtd_b200 import Simulation
    monkeypatch.setattr(torch.cuda, 'is_available', lambda: False)
    p = project3d()
    p.region.backend = 'cuda'
    with pytest.raises(RuntimeError, match='CUDA'):
        Simulation(p).run()
    with pytest.raises(RuntimeError, match='CUDA'):
        native.NativeGrid(plan_grid(p))


def test_host_buffer_and_download_into_a_given_array():
    """The helpers of the large-grid result path: host_buffer returns a writable C-contiguous array of the
    requested shape and dtype (every page touched), and download(out=...) fills that array or refuses one of
    the wrong shape, dtype or layout. A CPU tensor takes the plain-copy branch here."""
    import torch
    a = native.host_buffer((5, 7, 300, 3), np.float32, slab_bytes=4096)
    assert a.shape == (5, 7, 300, 3) and a.dtype == np.float32 and a.flags.c_contiguous and a.flags.writeable
    t = torch.arange(a.size, dtype=torch.float32).reshape(a.shape)
    assert native.download(t, out=a) is a
    np.testing.assert_array_equal(a, t.numpy())
    for wrong in (np.empty((5, 7, 300, 3), np.float64), np.empty((5, 7, 299, 3), np.float32),
                  np.empty((3, 300, 7, 5), np.float32).T):
        with pytest.raises(ValueError, match='out must be'):
            native.download(t, out=wrong)

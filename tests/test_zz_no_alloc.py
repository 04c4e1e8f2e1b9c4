"""The allocation-free field-norm entry point against tfd_diagnose (collected last on purpose).

tfd_field_norm_static serves callers that cannot allocate device memory (a health check running after an
out-of-memory failure, or a host whose memory belongs to a pool it must not bypass): its scratch is a static
device array in the library. Two calls in a row on different states must each agree with tfd_diagnose, which
uses the plan's own arena: energy to the FP64 summation tolerance, peak exactly, in both field precisions
and with one (cell) or three (Yee) stored permittivity samples per cell.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize('precision', ['float32', 'float64'])
@pytest.mark.parametrize('sampling', ['cell', 'yee'])
def test_static_scratch_norm_matches_diagnose_on_two_calls_in_a_row(precision, sampling):
    import torch
    from torchfdtd_b200 import Project, Region, Source, Structure
    from torchfdtd_b200.native import NativeGrid
    from torchfdtd_b200.plan import plan_grid
    project = Project(region=Region(dimension='3d', size=(2.0, 1.6, 1.2), mesh=.05, pml_cells=6, steps=40, backend='cuda',
                                    precision=precision, material_sampling=sampling),
                      structures=[Structure(kind='sphere', radius=.4, material='Si (constant n)')],
                      sources=[Source(center=(-.3, .1, 0), component='Ey', pulse_cycles=1, wavelength=1.0)])
    plan = plan_grid(project)
    grid = NativeGrid(plan)
    inv_eps = torch.as_tensor(plan.inv_eps, device='cuda')
    out = torch.zeros(2, dtype=torch.float64, device='cuda')
    for steps in (20, 20):
        grid.step(steps)
        E, H = grid.fields_device()
        grid.field_norm_static(E, H, inv_eps, out)
        torch.cuda.synchronize()
        energy, peak = out.tolist()
        ref_energy, ref_peak, _ = grid.diagnose()
        assert ref_energy > 0
        np.testing.assert_allclose(energy, ref_energy, rtol=1e-12)
        assert peak == ref_peak
        out.zero_()


def test_sizes_beyond_the_static_limit_are_refused():
    import torch
    from torchfdtd_b200 import native
    lib = native.library()
    buf = torch.zeros(8, dtype=torch.float32, device='cuda')
    out = torch.zeros(2, dtype=torch.float64, device='cuda')
    code = lib.tfd_field_norm_static(native.c_vp(buf.data_ptr()), native.c_vp(buf.data_ptr()), native.c_vp(buf.data_ptr()),
                                     67_108_865, 1, 4, native.c_vp(out.data_ptr()), None)
    assert code == 1 and b'static scratch limit' in lib.tfd_last_error()

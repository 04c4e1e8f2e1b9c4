"""The restated reference marching kernel (baseline/fused_eh_marching.cu, the reference's FusedEHMarching):
its scene rules on the CPU, and on the GPU bitwise agreement with the product's TMA z-march kernel and the
oracle on the periodic-x/y, z-CPML scenes it admits (both keep the reference operation order, --fmad=false)."""
import numpy as np
import pytest

from torchfdtd_b200 import Project, Region
from torchfdtd_b200.plan import plan_grid


def scene(size=(3.5, 2.6, 1.6), precision='float32', zfaces='pml', sources=('Ey', 'Ex'), steps=12):
    from torchfdtd_b200.models import BoundaryFace, Source, Structure
    region = Region(dimension='3d', size=size, mesh=.05, pml_cells=6, steps=steps, precision=precision, backend='cuda')
    for name in ('x_min', 'x_max', 'y_min', 'y_max'):
        setattr(region.boundaries, name, BoundaryFace(kind='periodic'))
    for name in ('z_min', 'z_max'):
        setattr(region.boundaries, name, BoundaryFace(kind=zfaces))
    hx = size[0] / 2
    centres = [(-hx + .025, .1, 0), (.3, -size[1] / 2 + .025, .05), (.1, .1, -.1)]
    return Project(region=region, structures=[Structure(kind='sphere', radius=.4, material='Si (constant n)')],
                   sources=[Source(center=c, component=comp, pulse_cycles=1, wavelength=1.0) for c, comp in zip(centres, sources)])


def test_scene_rules_follow_the_reference():
    from baseline.fused_eh_marching import eligibility_reason
    assert eligibility_reason(plan_grid(scene())) is None
    assert 'FP32' in eligibility_reason(plan_grid(scene(precision='float64')))
    assert 'mirror' in eligibility_reason(plan_grid(scene(zfaces='pec')))
    assert 'electric sources' in eligibility_reason(plan_grid(scene(sources=('Ey', 'Hz'))))
    assert 'z extent' in eligibility_reason(plan_grid(scene(size=(1.5, 1.5, 9.0))))
    pml_xy = scene()
    pml_xy.region.boundaries.x_min.kind = 'pml'
    pml_xy.region.boundaries.x_max.kind = 'pml'
    assert 'periodic' in eligibility_reason(plan_grid(pml_xy))


@pytest.mark.gpu
@pytest.mark.parametrize('size', [(3.5, 2.6, 1.6), (1.0, .9, 3.2), (1.6, 2.2, .9)])
def test_restated_reference_kernel_equals_the_march_kernel_and_oracle(size):
    from baseline.fused_eh_marching import RestatedMarching, build
    from oracle.yee_oracle import YeeOracle
    from torchfdtd_b200.native import NativeGrid
    build()
    plan = plan_grid(scene(size))
    rng = np.random.default_rng(21)
    E0 = (rng.normal(size=(*plan.shape, 3)) * .01).astype(np.float32)
    H0 = (rng.normal(size=(*plan.shape, 3)) * .01).astype(np.float32)
    ours = NativeGrid(plan, kernel='march')
    ours.set_fields(E0, H0)
    ours.step(plan.steps)
    ref = RestatedMarching(plan, E0, H0)
    ref.step(plan.steps)
    oracle = YeeOracle(plan)
    oracle.E[:], oracle.H[:] = E0, H0
    oracle.run()
    E, H = ours.get_fields()
    rE, rH = ref.fields()
    np.testing.assert_array_equal(rE, oracle.E)
    np.testing.assert_array_equal(rH, oracle.H)
    np.testing.assert_array_equal(E, rE)
    np.testing.assert_array_equal(H, rH)
    assert ours.device_status() == 0

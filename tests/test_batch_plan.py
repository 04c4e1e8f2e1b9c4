"""Host-side batch logic: case admission, grouping and refusals (no GPU needed)."""
import pytest

from torchfdtd_b200 import Project, Region
from torchfdtd_b200.batch import BatchCase, BatchItem, BatchReport, as_cases, batch_refusal, plan_grouped_batch
from torchfdtd_b200.models import BoundaryFace, Source


def tmz(size=(2.0, 1.5), precision='float32', steps=20, component='Ez'):
    region = Region(dimension='2d', size=(size[0], size[1], 1), mesh=.05, pml_cells=6, steps=steps,
                    precision=precision, backend='cuda')
    return Project(region=region, sources=[Source(center=(0, 0, 0), component=component)])


def test_case_ids_are_validated_and_generated():
    cases = as_cases([tmz(), tmz()])
    assert [c.id for c in cases] == ['case-0000', 'case-0001']
    with pytest.raises(ValueError, match='Duplicate'):
        as_cases([BatchCase('a', tmz()), BatchCase('a', tmz())])
    with pytest.raises(ValueError, match='Case ids'):
        BatchCase('-bad', tmz())
    with pytest.raises(TypeError):
        as_cases([1])
    with pytest.raises(ValueError, match='at least one'):
        as_cases([])


def test_refusals_name_the_reason():
    assert batch_refusal(tmz()) is None
    assert 'TMz' in batch_refusal(tmz(component='Hz'))
    p = tmz()
    p.region.boundaries.x_min = BoundaryFace(kind='periodic')
    p.region.boundaries.x_max = BoundaryFace(kind='periodic')
    assert 'periodic' in batch_refusal(p)
    p3 = Project(region=Region(dimension='3d', size=(1.2, 1.2, 1.2), mesh=.1, pml_cells=3, steps=10, backend='cuda'))
    assert '3D' in batch_refusal(p3)
    p = tmz()
    p.region.run_control.auto_shutoff = True
    assert 'fixed-duration' in batch_refusal(p)


def test_grouped_plan_groups_by_precision_and_keeps_the_rest_solo():
    cases = [tmz((2, 1)), tmz((3, 2), 'float64'), tmz((1, 1)), tmz(component='Hz'), tmz((4, 1), steps=33)]
    plan = plan_grouped_batch(cases, cohort_size=2)
    cohorts = [(c['execution'], c['indices']) for c in plan['cohorts']]
    assert cohorts == [('fused_cuda_batch', [0, 2]), ('fused_cuda_batch', [4]), ('fused_cuda_batch', [1]),
                       ('simulation', [3])]
    assert plan['group_count'] == 2 and plan['padding_cells'] == 0
    with pytest.raises(ValueError, match='cohort_size'):
        plan_grouped_batch(cases, cohort_size=65)


def test_report_serialises_without_results():
    item = BatchItem('a', 'completed', {'w': 1}, summary={'steps': 3})
    report = BatchReport([item, BatchItem('b', 'failed', {}, error='boom')], 1.5, {'x': 1})
    d = report.as_dict()
    assert d['successful'] is False and 'result' not in d['items'][0]
    with pytest.raises(RuntimeError, match='boom'):
        report.raise_for_errors()

"""A result computed and saved here has the reference's on-disk layout and values.

The reference's ``Result.save`` of the same project on its CPU path is tests/golden/result_*.npz.
A ``Simulation.run()`` on the fused kernels, saved here, must hold the same keys with the same
dtypes and shapes; fields, traces, frames and the stored permittivity bitwise; DFT-plane values
within the plane bar of the parity tests (FP64 accumulators here, complex64 in the reference);
point spectra to 1e-12; and every key of the reference's run summary.
"""
import json

import numpy as np
import pytest

from torchfdtd_b200 import Project, Simulation

pytestmark = pytest.mark.gpu
BITWISE = ('E', 'H', 'signals', 'frames', 'frame_steps', 'times', 'epsilon', 'mesh_x_um', 'mesh_y_um', 'mesh_z_um')


def rel_l2(a, b):
    return float(np.linalg.norm((np.asarray(a) - b).ravel()) / max(np.linalg.norm(np.asarray(b).ravel()), 1e-300))


@pytest.mark.parametrize('name', ['strip3d', 'yee_periodic'])
def test_saved_result_matches_the_reference_file(golden, tmp_path, name):
    ref_path = golden / f'result_{name}.npz'
    with np.load(ref_path, allow_pickle=False) as raw:
        project = Project.model_validate_json(str(raw['project']))
    project.region.backend = 'cuda'
    project.region.cuda_kernel = 'fused'
    out = tmp_path / 'ours.npz'
    Simulation(project).run().save(out)
    with np.load(ref_path, allow_pickle=False) as want, np.load(out, allow_pickle=False) as got:
        assert sorted(got.files) == sorted(want.files)
        for key in want.files:
            if key not in ('project', 'summary'):     # JSON texts: compared field by field below
                assert got[key].dtype == want[key].dtype and got[key].shape == want[key].shape, key
        saved = json.loads(str(got['project']))
        assert saved['region'].pop('backend') == 'cuda' and saved['region'].pop('cuda_kernel') == 'fused'
        reference = json.loads(str(want['project']))
        reference['region'].pop('backend')
        reference['region'].pop('cuda_kernel', None)
        assert saved == reference
        for key in BITWISE:
            np.testing.assert_array_equal(got[key], want[key], err_msg=key)
        for key in want.files:
            if key.startswith('monitor_') and key.endswith('_spectrum'):
                np.testing.assert_allclose(got[key], want[key], rtol=1e-12, atol=0)
            elif key.startswith('field_monitor_') and key.endswith(('_fields', '_poynting', '_flux')):
                assert rel_l2(got[key], want[key]) <= 2e-5, key
            elif key.startswith('field_monitor_'):
                np.testing.assert_array_equal(got[key], want[key], err_msg=key)
        ours, theirs = json.loads(str(got['summary'])), json.loads(str(want['summary']))
        assert set(theirs) <= set(ours), sorted(set(theirs) - set(ours))
        for key in ('shape', 'cells', 'steps', 'requested_steps', 'precision', 'slice_index', 'termination_reason',
                    'material_sampling', 'mesh_type', 'dt_fs', 'snapshot'):
            assert ours[key] == theirs[key], key
        np.testing.assert_allclose(ours['slice_position'], theirs['slice_position'], rtol=1e-12)
        assert json.loads(str(got['monitor_spectra'])) == json.loads(str(want['monitor_spectra']))
        planes_ours, planes_ref = json.loads(str(got['field_monitors'])), json.loads(str(want['field_monitors']))
        assert planes_ours == planes_ref

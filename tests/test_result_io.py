"""The on-disk NPZ layout of ``Result`` against files the reference itself wrote.

tests/golden/result_*.npz are the reference's own ``Result.save`` of complete CPU runs
(tests/golden/make_golden.py, reference torchfdtd/solver.py:536-564). Here: ``Result.load``
reads them field for field, a loaded result saved again reproduces every key, dtype and
value of the reference file, and (with the reference tree present) a file saved here loads
in the reference's own ``Result.load`` (torchfdtd/solver.py:603-618).
"""
import json
import subprocess
import sys
import textwrap

import numpy as np
import pytest

from torchfdtd_b200 import Project
from torchfdtd_b200.simulation import Result

NAMES = ['strip3d', 'yee_periodic']
ARRAY_FIELDS = {'frames': 'frames', 'frame_steps': 'frame_steps', 'epsilon': 'epsilon', 'signals': 'signals',
                'times': 'times', 'E': 'electric', 'H': 'magnetic'}


def assert_same_array(a, b):
    assert a.dtype == b.dtype and a.shape == b.shape
    np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize('name', NAMES)
def test_load_reads_a_reference_written_result_field_for_field(golden, name):
    path = golden / f'result_{name}.npz'
    result = Result.load(path)
    with np.load(path, allow_pickle=False) as raw:
        for key, attr in ARRAY_FIELDS.items():
            assert_same_array(getattr(result, attr), raw[key])
        assert json.loads(result.project.model_dump_json()) == json.loads(str(raw['project']))
        assert result.summary == json.loads(str(raw['summary']))
        planes = json.loads(str(raw['field_monitors']))
        assert len(result.frequency_fields) == len(planes)
        for k, plane in enumerate(result.frequency_fields):
            for key, value in plane.items():
                if isinstance(value, np.ndarray):
                    assert_same_array(value, raw[f'field_monitor_{k}_{key}'])
                else:
                    assert json.loads(json.dumps(value)) == planes[k][key]
        # The point spectra this engine computes from the loaded traces are the ones the reference stored.
        for k, spec in enumerate(result.spectra):
            np.testing.assert_array_equal(spec['frequency_hz'], raw[f'monitor_{k}_frequency_hz'])
            np.testing.assert_allclose(spec['value'], raw[f'monitor_{k}_spectrum'], rtol=1e-12, atol=0)
        assert result.field_monitor('plane')['fields'].shape[-1] == len(result.field_monitor('plane')['components'])


@pytest.mark.parametrize('name', NAMES)
def test_save_reproduces_the_reference_layout(golden, tmp_path, name):
    path = golden / f'result_{name}.npz'
    out = tmp_path / 'again.npz'
    Result.load(path).save(out)
    with np.load(path, allow_pickle=False) as want, np.load(out, allow_pickle=False) as got:
        assert sorted(got.files) == sorted(want.files)
        for key in want.files:
            a, b = got[key], want[key]
            if a.dtype.kind == 'U':
                assert json.loads(str(a)) == json.loads(str(b)), key
            else:
                assert_same_array(a, b)


def test_hdf5_is_refused_by_name(golden, tmp_path):
    result = Result.load(golden / 'result_strip3d.npz')
    for kwargs, target in (({}, tmp_path / 'r.h5'), ({'format': 'hdf5'}, tmp_path / 'r.npz')):
        with pytest.raises(ValueError, match='HDF5'):
            result.save(target, **kwargs)
    with pytest.raises(ValueError, match='HDF5'):
        Result.load(tmp_path / 'r.hdf5')


def test_a_result_saved_here_loads_in_the_reference(golden, tmp_path, reference_tree):
    """The reference's own Result.load (run in a child process with the fdtd stand-in) reads a file saved here."""
    result = Result.load(golden / 'result_strip3d.npz')
    result.electric = result.electric * np.float32(2)          # a value the reference file does not hold
    out = tmp_path / 'ours.npz'
    result.save(out)
    script = textwrap.dedent(f'''
        import sys, numpy as np
        sys.path.insert(0, {str(golden / 'fdtd_standin')!r})
        sys.path.insert(0, {str(reference_tree)!r})
        from torchfdtd.solver import Result
        r = Result.load({str(out)!r})
        np.save({str(tmp_path / 'E.npy')!r}, r.electric)
        np.save({str(tmp_path / 'fields.npy')!r}, r.field_monitor('plane')['fields'])
        print(r.project.name, len(r.spectra), r.summary['steps'])
    ''')
    done = subprocess.run([sys.executable, '-c', script], capture_output=True, text=True, timeout=300)
    assert done.returncode == 0, done.stderr[-2000:]
    assert done.stdout.split() == [result.project.name, str(len(result.spectra)), str(result.summary['steps'])]
    np.testing.assert_array_equal(np.load(tmp_path / 'E.npy'), result.electric)
    np.testing.assert_array_equal(np.load(tmp_path / 'fields.npy'), result.field_monitor('plane')['fields'])


def test_loaded_project_is_the_reference_project(golden):
    with np.load(golden / 'result_yee_periodic.npz', allow_pickle=False) as raw:
        project = Project.model_validate_json(str(raw['project']))
        for axis, name in enumerate('xyz'):
            np.testing.assert_array_equal(project.region.mesh_nodes[axis], raw[f'mesh_{name}_um'])


@pytest.mark.parametrize('name', ['graded3d', 'graded2d', 'explicit3d', 'steps3d', 'strip3d'])
def test_frames_sample_the_reference_display_grid(golden, name):
    """The last stored frame and the permittivity plane are the reference's: on nonuniform meshes the cells
    nearest to a uniform pixel grid, else a stride decimation (reference torchfdtd/solver.py:810-828)."""
    from torchfdtd_b200.simulation import Observer, Simulation
    d = np.load(golden / f'sim_{name}.npz')
    project = Project.model_validate_json(str(d['project']))
    r = project.region
    plan = Simulation(project).plan

    class Final:                       # stands in for the device grid: the reference's final fields
        def get_slice(self, component, axis, index):
            field = (d['E'] if component[0] == 'E' else d['H'])[..., 'xyz'.index(component[1].lower())]
            return np.take(field, index, axis=axis)

    observer = Observer(project, plan, Final())
    np.testing.assert_array_equal(observer.decimate(Final().get_slice(r.field, observer.axis, observer.plane_index)),
                                  d['frames'][-1])
    assert observer.eps_plane.shape == d['frames'][-1].shape

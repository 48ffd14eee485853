"""Parameter files and recon dicts (no GPU): the YAML round trip of every geometry model
(tests/test_projectors.py:96-145 of the reference: to_file, from_file, compare_parameter_handlers), the
recon_dict layout of TomographyModel.get_recon_dict (tomography_model.py:333-410), and save/load_recon_hdf5
(tests/test_vcd.py:127-140) through a stand-in for h5py, which this image does not have."""
import io
import sys
import types

import numpy as np
import pytest

import mbirjax_b200 as mb
from cases import make_case


@pytest.mark.parametrize('kind', ['parallel', 'cone', 'translation'])
def test_to_file_from_file_round_trip(tmp_path, kind):
    model, _ = make_case(kind, views=12, rows=6, channels=24)
    model.set_params(granularity=[2, 8], qggmrf_nbr_wts=(1.0, 0.5, 2.0), sharpness=0.5, positivity_flag=True)
    fn = str(tmp_path / 'sub' / 'model.yaml')
    assert model.to_file(fn) is None
    new = type(model).from_file(fn)
    assert mb.ParameterHandler.compare_parameter_handlers(model, new, verbose=True)
    # the same from the YAML text and from a stream
    text = model.to_file(None)
    assert mb.ParameterHandler.compare_parameter_handlers(model, type(model).from_file(text))
    assert mb.ParameterHandler.compare_parameter_handlers(model, type(model).from_file(io.StringIO(text)))
    # view parameters are written as ':ARRAY:' strings with their shape and read back as arrays
    view_params = model.get_params('view_params_name')
    assert isinstance(new.get_params(view_params), np.ndarray)
    assert new.get_params(view_params).shape == np.asarray(model.get_params(view_params)).shape
    assert tuple(new.get_params('recon_shape')) == tuple(model.get_params('recon_shape'))
    with pytest.raises(ValueError):
        model.to_file(str(tmp_path / 'model.txt'))


def test_loading_reenables_auto_regularization_as_the_reference():
    # from_file sets sigma_* (which clears auto_regularize_flag) and sharpness / snr_db (which set it again),
    # all in one set_params call, so a loaded model always has auto-regularisation on (parameter_handler.py:486-502)
    model, _ = make_case('parallel', views=8, rows=4, channels=16)
    with pytest.warns(UserWarning):
        model.set_params(sigma_y=0.3)
    assert model.get_params('auto_regularize_flag') is False
    new = mb.ParallelBeamModel.from_file(model.to_file(None))
    assert new.get_params('auto_regularize_flag') is True
    assert new.get_params('sigma_y') == pytest.approx(0.3)


def test_compare_parameter_handlers_detects_differences():
    a, _ = make_case('cone', views=8, rows=4, channels=16)
    b, _ = make_case('cone', views=8, rows=4, channels=16)
    assert mb.ParameterHandler.compare_parameter_handlers(a, b)
    b.set_params(granularity=[1, 2])
    assert not mb.ParameterHandler.compare_parameter_handlers(a, b)


def test_parameter_file_written_by_the_reference_module_path_loads():
    # a file whose geometry_type names the reference's module loads into the same class here
    model, _ = make_case('parallel', views=8, rows=4, channels=16)
    text = model.to_file(None).replace("mbirjax_b200.parallel_beam.ParallelBeamModel",
                                       "mbirjax.parallel_beam.ParallelBeamModel")
    assert "<class 'mbirjax.parallel_beam.ParallelBeamModel'>" in text
    new = mb.ParallelBeamModel.from_file(text)
    assert tuple(new.get_params('sinogram_shape')) == (8, 4, 16)
    with pytest.raises((KeyError, ValueError)):
        mb.ConeBeamModel.from_file(text)   # a parallel-beam file lacks the cone's required parameters


def test_recon_dict_layout():
    model, _ = make_case('parallel', views=8, rows=4, channels=16)
    d = model.get_recon_dict()
    assert set(d) == {'recon_params', 'recon_log', 'notes', 'model_params'}
    assert d['recon_params'] == '# Recon params not saved.'
    assert d['notes'] == '# No notes saved'
    assert d['model_params']['sharpness'].val == model.get_params('sharpness')
    rp = {'num_iterations': 3, 'granularity': [4], 'fm_rmse': [1.0, 0.5, np.float32(0.25)],
          'regularization_params': {'sigma_y': 0.1}}
    s = model.get_recon_dict(rp, notes='n', save_log=False, save_model=True, str_format=True)
    assert all(isinstance(v, str) for v in s.values())
    assert s['recon_log'] == '# Log info not saved.'
    import yaml
    assert yaml.safe_load(s['recon_params'])['fm_rmse'] == [1.0, 0.5, 0.25]
    rebuilt = mb.ParallelBeamModel.from_file(s['model_params'])
    assert mb.ParameterHandler.compare_parameter_handlers(model, rebuilt)


class _FakeDataset:
    def __init__(self, data):
        self.data = np.array(data)
        self.attrs = {}

    def __getitem__(self, key):
        assert key == ()
        return self.data.copy()


class _FakeFile:
    """The part of the h5py.File API the HDF5 helpers use, kept in a dict by path."""
    store = {}

    def __init__(self, path, mode):
        self.path, self.mode = str(path), mode
        if mode == 'w':
            _FakeFile.store[self.path] = {}
        elif self.path not in _FakeFile.store:
            raise FileNotFoundError(self.path)

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        return False

    def create_dataset(self, name, data):
        ds = _FakeDataset(data)
        _FakeFile.store[self.path][name] = ds
        return ds

    def keys(self):
        return _FakeFile.store[self.path].keys()

    def __getitem__(self, name):
        return _FakeFile.store[self.path][name]


def test_save_load_recon_hdf5_through_the_h5py_api(monkeypatch, tmp_path):
    fake = types.ModuleType('h5py')
    fake.File = _FakeFile
    monkeypatch.setitem(sys.modules, 'h5py', fake)
    model, _ = make_case('cone', views=8, rows=4, channels=16)
    recon = np.random.default_rng(0).random(model.get_params('recon_shape')).astype(np.float32)
    rd = model.get_recon_dict({'num_iterations': 2, 'fm_rmse': [1.0, 0.5]}, notes='Testing save/load')
    fn = tmp_path / 'out' / 'recon.h5'
    model.save_recon_hdf5(fn, recon, rd)
    loaded, ld, new_model = mb.TomographyModel.load_recon_hdf5(str(fn), recreate_model=True)
    np.testing.assert_array_equal(loaded, recon)
    assert ld['notes'] == 'Testing save/load'
    assert isinstance(new_model, mb.ConeBeamModel)
    assert np.allclose(model.get_params('sigma_x'), new_model.get_params('sigma_x'))
    assert mb.ParameterHandler.compare_parameter_handlers(model, new_model)


def test_hdf5_without_h5py_says_so(monkeypatch, tmp_path):
    monkeypatch.setitem(sys.modules, 'h5py', None)
    model, _ = make_case('parallel', views=8, rows=4, channels=16)
    with pytest.raises(ImportError, match='h5py'):
        model.save_recon_hdf5(tmp_path / 'r.h5', np.zeros(model.get_params('recon_shape'), np.float32))


def test_array_string_conversions_round_trip():
    """ParameterHandler.convert_arrays_to_strings / convert_strings_to_arrays (parameter_handler.py:122-172): arrays
    to ':ARRAY:' strings with their shape and back, scalars normalised, other entries untouched."""
    ph = mb.ParameterHandler
    params = {'angles': mb.Param(np.linspace(0, 1, 6).reshape(2, 3), True), 'sharpness': mb.Param(np.float32(0.5), False),
              'granularity': mb.Param([1, 2], False)}
    out = ph.convert_arrays_to_strings(params)
    assert out['angles'].val.startswith(ph.array_prefix) and out['angles'].shape == (2, 3)
    assert type(out['sharpness'].val) is float and out['granularity'].val == [1, 2]
    back = ph.convert_strings_to_arrays(out)
    np.testing.assert_allclose(back['angles'].val, np.linspace(0, 1, 6).reshape(2, 3), atol=1e-7)
    assert not hasattr(back['angles'], 'shape')

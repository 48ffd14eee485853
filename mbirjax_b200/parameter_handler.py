"""Model parameters with the reference's names, defaults and recompile semantics.

Mirrors ``mbirjax/_utils.py:17-58`` (``Param`` and the default dictionaries) and
``ParameterHandler.set_params`` / ``get_params`` (``parameter_handler.py:433-559``): a change to a parameter
whose recompile flag is set invalidates the projector geometry (here: the ``mbx_geom`` record and any cached
device state), setting sigma_x / sigma_y / sigma_prox directly disables auto-regularisation, and setting
sharpness or snr_db re-enables it.

Parameter files (``parameter_handler.py:95-431``): ``save_params`` writes every parameter as a YAML mapping
``{val, recompile_flag}`` (arrays as ``':ARRAY:'`` + space-separated values with 7 decimals, plus their
``shape``; lists as sequences), and ``load_param_dict`` reads that format back from a file name, a YAML string
or a stream and splits off the constructor's required parameters.  The reference writes with ruamel.yaml, which
this image lacks; PyYAML writes and reads the same YAML document structure.
"""
from collections.abc import Iterable, Sized
import copy
import logging
import os
import io
import warnings
from dataclasses import dataclass
from typing import Any

import numpy as np
import yaml


@dataclass
class Param:
    val: Any
    recompile_flag: bool = True


_forward_model_defaults = {
    'geometry_type': Param(None, False),
    'file_format': Param(1.0, False),
    'sinogram_shape': Param(None, True),
    'delta_det_channel': Param(1.0, True),
    'delta_det_row': Param(1.0, True),
    'det_row_offset': Param(0.0, True),
    'det_channel_offset': Param(0.0, True),
    'sigma_y': Param(1.0, False),
}

_recon_model_defaults = {
    'recon_shape': Param(None, True),
    'delta_voxel': Param(None, True),
    'sigma_x': Param(1.0, False),
    'sigma_prox': Param(1.0, False),
    'p': Param(2.0, False),
    'q': Param(1.2, False),
    'T': Param(1.0, False),
    'qggmrf_nbr_wts': Param([1.0, 1.0, 1.0], False),
}

_reconstruction_defaults = {
    'auto_regularize_flag': Param(True, False),
    'positivity_flag': Param(False, False),
    'snr_db': Param(30.0, False),
    'sharpness': Param(1.0, False),
    'granularity': Param([1, 2, 4, 8, 16, 32, 64, 128, 256], False),
    'partition_sequence': Param([0, 2, 4, 6, 7], False),
    'verbose': Param(1, False),
    'use_gpu': Param('automatic', True),
}


def get_default_params():
    return copy.deepcopy({**_forward_model_defaults, **_recon_model_defaults, **_reconstruction_defaults})


def _class_name(geometry_type):
    """'ConeBeamModel' from "<class 'pkg.module.ConeBeamModel'>"."""
    return str(geometry_type).split("<class '")[-1].split("'>")[0].split('.')[-1]


def _is_tensor(val):
    return type(val).__module__.startswith('torch') and hasattr(val, 'detach')


def _as_numpy(val):
    return val.detach().cpu().numpy() if _is_tensor(val) else np.asarray(val)


def _to_yaml_sequence(val):
    """Tuples (nested too) as lists, which YAML writes as plain sequences."""
    if isinstance(val, (list, tuple)):
        return [_to_yaml_sequence(v) for v in val]
    return val


def _normalize_scalar(val):
    if isinstance(val, np.generic):
        return val.item()
    if isinstance(val, (list, tuple)):
        return type(val)(_normalize_scalar(v) for v in val)
    return val


class ParameterHandler:
    array_prefix = ':ARRAY:'

    def __init__(self):
        self.params = get_default_params()
        self.logger = None
        self.log_buffer = None

    def setup_logger(self, *, logfile_path='./logs/recon.log', print_logs=True):
        """parameter_handler.py:36-93: buffer, console and optional file handlers."""
        verbose = self.get_params('verbose')
        level = logging.WARNING if verbose < 1 else (logging.INFO if verbose < 2 else logging.DEBUG)
        logger = logging.getLogger(self.__class__.__name__ + '_b200')
        logger.setLevel(level)
        logger.propagate = False
        for h in list(logger.handlers):
            try:
                h.flush()
            finally:
                h.close()
                logger.removeHandler(h)
        self.log_buffer = io.StringIO()
        bh = logging.StreamHandler(self.log_buffer)
        bh.setLevel(level)
        logger.addHandler(bh)
        if print_logs:
            ch = logging.StreamHandler()
            ch.setLevel(level)
            logger.addHandler(ch)
        if logfile_path:
            d = os.path.dirname(logfile_path)
            if d:
                os.makedirs(d, exist_ok=True)
            fh = logging.FileHandler(logfile_path, mode='w')
            fh.setLevel(level)
            logger.addHandler(fh)
        self.logger = logger

    def set_params(self, no_warning=False, no_compile=False, **kwargs):
        """parameter_handler.py:433-510; returns True when the projector geometry must be rebuilt."""
        recompile = False
        regularization_change = False
        meta_change = False
        for key, val in kwargs.items():
            recompile_flag = True
            if key in self.params:
                recompile_flag = self.params[key].recompile_flag
            elif not no_warning:
                raise ValueError('{} is not a recognized parameter\nValid parameters are: \n{}'.format(
                    key, ''.join('   {}\n'.format(k) for k in self.params)))
            self.params[key] = Param(_normalize_scalar(val), recompile_flag)
            if recompile_flag:
                recompile = True
            elif key in ('sigma_y', 'sigma_x', 'sigma_prox'):
                regularization_change = True
            elif key in ('sharpness', 'snr_db'):
                meta_change = True
        if not no_warning:
            self.verify_valid_params()
        if regularization_change and not no_warning:
            self.set_params(auto_regularize_flag=False)
            warnings.warn('You are directly setting regularization parameters, sigma_x, sigma_y or sigma_prox. '
                          'This is an advanced feature that will disable auto-regularization.')
        if meta_change and self.get_params('auto_regularize_flag') is False:
            self.set_params(auto_regularize_flag=True)
            if not no_warning:
                warnings.warn('You have re-enabled auto-regularization by setting sharpness or snr_db. '
                              'It was previously disabled')
        return bool(recompile and not no_compile)

    def get_params(self, parameter_names):
        """parameter_handler.py:539-559."""
        if isinstance(parameter_names, str):
            if parameter_names not in self.params:
                raise NameError('"{}" is not a recognized argument'.format(parameter_names))
            return self.params[parameter_names].val
        values = []
        for name in parameter_names:
            if name not in self.params:
                raise NameError('"{}" is not a recognized argument'.format(name))
            values.append(self.params[name].val)
        return values

    # ------------------------------------------------------------------ parameter files
    @staticmethod
    def normalize_scalar(val):
        """NumPy scalars to Python scalars, recursively through lists and tuples (parameter_handler.py:175-192)."""
        return _normalize_scalar(val)

    @staticmethod
    def serialize_parameter(param_obj):
        """Param -> YAML-safe dict (parameter_handler.py:194-226)."""
        val = param_obj.val
        if isinstance(val, np.ndarray) or _is_tensor(val):
            arr = _as_numpy(val)
            return {'val': ParameterHandler.array_prefix + " ".join(f"{x:.7f}" for x in arr.flatten()),
                    'shape': list(arr.shape), 'recompile_flag': param_obj.recompile_flag}
        val = _normalize_scalar(val)
        return {'val': _to_yaml_sequence(val), 'recompile_flag': param_obj.recompile_flag}

    @staticmethod
    def deserialize_parameter(entry):
        """YAML dict -> Param; array strings become arrays of the saved shape (parameter_handler.py:228-250,
        148-173)."""
        val = entry['val']
        flag = entry.get('recompile_flag', True)
        if isinstance(val, str) and val.startswith(ParameterHandler.array_prefix):
            body = val[len(ParameterHandler.array_prefix):].replace('[', '').replace(']', '').split()
            arr = np.array([float(v) for v in body])
            if 'shape' in entry:
                arr = arr.reshape(tuple(entry['shape']))
            return Param(arr, flag)
        val = _normalize_scalar(val)
        if isinstance(val, list):
            val = tuple(val)
        return Param(val, flag)

    @staticmethod
    def convert_arrays_to_strings(cur_params):
        """{name: Param}: array values become the ':ARRAY:' string of their flattened values (7 decimals) with a
        ``shape`` attribute on the Param, other values lose their NumPy scalar types (parameter_handler.py:122-145).
        The reference's loop assigns the original value back after the string, so there arrays stay arrays; here
        they become strings, as its docstring says and as its file writer (serialize_parameter) does."""
        for entry in cur_params.values():
            val = entry.val
            if isinstance(val, np.ndarray) or _is_tensor(val):
                arr = _as_numpy(val)
                entry.val = ParameterHandler.array_prefix + " ".join(f"{x:.7f}" for x in arr.flatten())
                entry.shape = arr.shape
            else:
                entry.val = _normalize_scalar(val)
        return cur_params

    @staticmethod
    def convert_strings_to_arrays(cur_params):
        """{name: Param}: ':ARRAY:' strings become arrays of the Param's ``shape`` attribute, which is then
        removed (parameter_handler.py:147-172)."""
        prefix = ParameterHandler.array_prefix
        for entry in cur_params.values():
            val = entry.val
            if isinstance(val, str) and val.startswith(prefix):
                body = val[len(prefix):].replace('[', '').replace(']', '').split()
                entry.val = np.array([float(v) for v in body]).reshape(entry.shape)
                del entry.shape
        return cur_params

    @staticmethod
    def is_flat_iterable(x):
        return isinstance(x, Iterable) and isinstance(x, Sized) and not isinstance(x, (str, bytes))

    @staticmethod
    def compare_flat_iterables(v1, v2, atol=1e-6):
        """Same length and entries up to atol (parameter_handler.py:256-278)."""
        if len(v1) != len(v2):
            return False
        for a, b in zip(v1, v2):
            if isinstance(a, (int, float, np.generic)) and isinstance(b, (int, float, np.generic)):
                if not abs(float(a) - float(b)) <= atol:
                    return False
            elif a != b:
                return False
        return True

    @staticmethod
    def compare_parameter_handlers(ph1, ph2, atol=1e-6, verbose=False):
        """True when both handlers hold the same parameter names and values up to atol
        (parameter_handler.py:280-322)."""
        keys1, keys2 = set(ph1.params.keys()), set(ph2.params.keys())
        if keys1 != keys2:
            if verbose:
                print("Parameter key mismatch:")
                print("Only in ph1:", keys1 - keys2)
                print("Only in ph2:", keys2 - keys1)
            return False
        for key in keys1:
            val1, val2 = ph1.params[key].val, ph2.params[key].val
            if (isinstance(val1, np.ndarray) or _is_tensor(val1)) and (isinstance(val2, np.ndarray) or _is_tensor(val2)):
                a1, a2 = _as_numpy(val1), _as_numpy(val2)
                equal = a1.shape == a2.shape and np.allclose(a1, a2, atol=atol)
            elif isinstance(val1, (int, float, np.generic)) and isinstance(val2, (int, float, np.generic)):
                equal = abs(float(val1) - float(val2)) <= atol
            elif ParameterHandler.is_flat_iterable(val1) and ParameterHandler.is_flat_iterable(val2):
                equal = ParameterHandler.compare_flat_iterables(val1, val2, atol)
            else:
                equal = val1 == val2
            if not equal:
                if verbose:
                    print(f"Mismatch in key '{key}': {val1} != {val2}")
                return False
        return True

    @staticmethod
    def save_params(params, filename=None):
        """Parameters to YAML text, or to a .yml / .yaml file when filename is given (parameter_handler.py:
        324-358)."""
        output_params = {key: ParameterHandler.serialize_parameter(entry) for key, entry in params.items()}
        text = yaml.safe_dump(output_params, default_flow_style=False, sort_keys=False)
        if filename:
            if not filename.lower().endswith(('.yml', '.yaml')):
                raise ValueError(f"Filename must end in .yaml or .yml: {filename}")
            d = os.path.dirname(filename)
            if d:
                os.makedirs(d, exist_ok=True)
            with open(filename, 'w') as file:
                file.write(text)
            return None
        return text

    @staticmethod
    def load_param_dict(source, required_param_names=None, values_only=True):
        """Parameters from a YAML file name, a YAML string or a file-like object; returns (required_params,
        other_params) (parameter_handler.py:373-416)."""
        if isinstance(source, str):
            if os.path.exists(source):
                if not source.lower().endswith(('.yml', '.yaml')):
                    raise ValueError("Filename must end in .yml or .yaml")
                with open(source, 'r') as f:
                    contents = f.read()
            else:
                contents = source
        elif hasattr(source, 'read'):
            contents = source.read()
        else:
            raise TypeError("Invalid source type for load_param_dict. Must be str or file-like object.")
        param_dict = yaml.safe_load(contents)
        param_dict = {key: ParameterHandler.deserialize_parameter(val) for key, val in param_dict.items()}
        return ParameterHandler.get_required_params_from_dict(param_dict, required_param_names or [],
                                                              values_only=values_only)

    @staticmethod
    def get_required_params_from_dict(param_dict, required_param_names=None, values_only=True):
        """Split the named required parameters off a parameter dict (parameter_handler.py:418-431)."""
        required_params = dict()
        param_dict = param_dict.copy()
        for name in required_param_names or []:
            required_params[name] = param_dict[name]
            del param_dict[name]
        if values_only:
            required_params = {k: v.val for k, v in required_params.items()}
            param_dict = {k: v.val for k, v in param_dict.items()}
        return required_params, param_dict

    @staticmethod
    def get_params_from_dict(param_dict, parameter_names):
        """Values of the named entries of a Param dict (parameter_handler.py:513-537)."""
        if isinstance(parameter_names, str):
            if parameter_names not in param_dict:
                raise NameError('"{}" is not a recognized argument'.format(parameter_names))
            return param_dict[parameter_names].val
        values = []
        for name in parameter_names:
            if name not in param_dict:
                raise NameError('"{}" is not a recognized argument'.format(name))
            values.append(param_dict[name].val)
        return values

    def print_params(self):
        print('----')
        for key, entry in self.params.items():
            print('{} = {}'.format(key, entry.val))
        print('----')

    def get_magnification(self):
        raise NotImplementedError('get_magnification is not implemented.')

    def verify_valid_params(self):
        """parameter_handler.py:572-591."""
        sinogram_shape = self.get_params('sinogram_shape')
        if sinogram_shape is None or len(sinogram_shape) != 3:
            raise ValueError('sinogram_shape must be (views, rows, channels). \nGot {} for sinogram shape.'.format(
                sinogram_shape))
        geometry_type = self.get_params('geometry_type')
        # the class must match; the module path may differ, so that a parameter file written by mbirjax
        # ("<class 'mbirjax.cone_beam.ConeBeamModel'>") loads into the same class here
        if geometry_type is not None and _class_name(geometry_type) != _class_name(str(type(self))):
            raise ValueError('Parameters are associated with {}, but the current model is {}'.format(
                geometry_type, str(type(self))))

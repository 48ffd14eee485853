"""Model parameters with the reference's names, defaults and recompile semantics.

Mirrors ``mbirjax/_utils.py:17-58`` (``Param`` and the default dictionaries) and
``ParameterHandler.set_params`` / ``get_params`` (``parameter_handler.py:433-559``): a change to a parameter
whose recompile flag is set invalidates the projector geometry (here: the ``mbx_geom`` record and any cached
device state), setting sigma_x / sigma_y / sigma_prox directly disables auto-regularisation, and setting
sharpness or snr_db re-enables it.
"""
import copy
import logging
import os
import io
import warnings
from dataclasses import dataclass
from typing import Any

import numpy as np


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


def _normalize_scalar(val):
    if isinstance(val, np.generic):
        return val.item()
    if isinstance(val, (list, tuple)):
        return type(val)(_normalize_scalar(v) for v in val)
    return val


class ParameterHandler:

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
        if geometry_type is not None and geometry_type != str(type(self)):
            raise ValueError('Parameters are associated with {}, but the current model is {}'.format(
                geometry_type, str(type(self))))

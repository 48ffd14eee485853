"""TomographyModel: the reference's public model API on top of the mbirjax_b200 CUDA kernels.

Drop-in for ``mbirjax.TomographyModel`` (``tomography_model.py:36-1815``) on the hot path:
``set_params``/``get_params``, ``forward_project``/``back_project`` (``:531-574``),
``sparse_forward_project``/``sparse_back_project`` (``:576-677``), ``compute_hessian_diagonal`` (``:679-708``),
``auto_set_regularization_params`` (``:756-932``), ``direct_recon``/``direct_filter``, ``recon`` (``:966-1084``),
``vcd_recon`` (``:1086-1255``) and ``get_forward_model_loss`` (``:1633-1658``).

Arrays may be NumPy arrays or torch tensors; results are float32 torch tensors on the model's CUDA device
(the reference returns JAX device arrays).  Every projection, prior and VCD step runs in the CUDA library
through the C ABI (``mbirjax_b200._capi``); nothing here computes them on the CPU.  The host keeps only what
the reference keeps on the host: parameters, partitions (NumPy, same ``np.random`` call order),
auto-regularisation statistics and the iteration loop.
"""
import datetime
import inspect
import io
import warnings
from collections import namedtuple

import numpy as np
import torch
import yaml

from . import _capi
from .parameter_handler import ParameterHandler
from .vcd_utils import gen_full_indices, gen_set_of_pixel_partitions, gen_partition_sequence, morton_sorted_partition
from .qggmrf import get_b_from_nbr_wts

recon_param_names = ['num_iterations', 'granularity', 'partition_sequence', 'fm_rmse', 'prior_loss',
                     'regularization_params', 'stop_threshold_change_pct', 'alpha_values']
ReconParams = namedtuple('ReconParams', recon_param_names)


def _cuda_device():
    if not torch.cuda.is_available():
        raise _capi.MbxError('mbirjax_b200 needs a CUDA device; none is visible')
    return torch.device('cuda', torch.cuda.current_device())


class TomographyModel(ParameterHandler):
    """Base class of the geometry models; see ParallelBeamModel and ConeBeamModel."""

    DIRECT_RECON_VIEW_BATCH_SIZE = 100

    def __init__(self, sinogram_shape, **kwargs):
        super().__init__()
        self._geom = None
        self._angles_dev = None
        self._full_idx = None
        self.set_params(no_compile=True, no_warning=True, sinogram_shape=tuple(int(v) for v in sinogram_shape),
                        **kwargs)
        if self.get_params('delta_voxel') is None:
            delta_voxel = self.get_params('delta_det_channel') / self.get_magnification()
            self.set_params(no_compile=True, no_warning=True, delta_voxel=delta_voxel)
        self.use_ror_mask = True
        self.auto_set_recon_size(sinogram_shape, no_compile=True, no_warning=True)
        self.set_params(geometry_type=str(type(self)))
        self.verify_valid_params()
        self.main_device = self.sinogram_device = self.worker = None
        self.view_batch_size_for_vmap = 512
        self.pixel_batch_size_for_vmap = 2048
        self.transfer_pixel_batch_size = 100 * self.pixel_batch_size_for_vmap
        self.use_gpu = 'full'
        self.create_projectors()

    # ------------------------------------------------------------------ parameters / geometry
    def set_params(self, no_warning=False, no_compile=False, **kwargs):
        recompile = super().set_params(no_warning=no_warning, no_compile=no_compile, **kwargs)
        if any(self.params[k].recompile_flag for k in kwargs if k in self.params):
            self._geom = None  # geometry record and device angles are rebuilt on next use
        if recompile:
            self.create_projectors()

    def verify_valid_params(self):
        super().verify_valid_params()
        use_gpu = self.get_params('use_gpu')
        if use_gpu not in ['automatic', 'full', 'sinograms', 'projections', 'none']:
            raise ValueError("use_gpu must be one of 'automatic', 'full', 'sinograms', 'projections', 'none'")

    def create_projectors(self):
        """Counterpart of tomography_model.py:475-484: invalidates the cached mbx_geom record (built lazily)."""
        self._geom = None

    def get_geometry_parameters(self):
        raise NotImplementedError

    def auto_set_recon_size(self, sinogram_shape, no_compile=True, no_warning=False):
        """tomography_model.py:858-861: each geometry sets its own default recon size."""
        raise NotImplementedError('auto_set_recon_size must be implemented by each specific geometry model.')

    def get_projector_params(self):
        """(sinogram_shape, recon_shape, geometry_params): the projector_params argument of the per-view plugin
        functions, as the reference's Projectors builds it (projectors.py:44-53)."""
        sinogram_shape, recon_shape = self.get_params(['sinogram_shape', 'recon_shape'])
        return ProjectorParams(tuple(sinogram_shape), tuple(recon_shape), self.get_geometry_parameters())

    @staticmethod
    def forward_project_pixel_batch_to_one_view(voxel_values, pixel_indices, view_params, projector_params):
        """tomography_model.py:486-505: a geometry overrides this; the base class warns and returns None."""
        warnings.warn('Forward projector not implemented for TomographyModel.')
        return None

    @staticmethod
    def back_project_one_view_to_pixel_batch(sinogram_view, pixel_indices, single_view_params, projector_params,
                                             coeff_power=1):
        """tomography_model.py:507-529: a geometry overrides this; the base class warns and returns None."""
        warnings.warn('Back projector not implemented for TomographyModel.')
        return None

    def _kind(self):
        raise NotImplementedError

    def _device(self):
        return _cuda_device()

    def _geometry(self):
        """The mbx_geom record for the current parameters.  Its angle (or translation) pointer refers to a device
        tensor owned by this model, so the record is valid only while the model is alive and its geometry
        parameters unchanged."""
        if self._geom is None:
            dev = self._device()
            sinogram_shape, recon_shape = self.get_params(['sinogram_shape', 'recon_shape'])
            view_params = np.asarray(self.get_params(self.get_params('view_params_name')), dtype=np.float32)
            self._angles_dev = torch.as_tensor(view_params, device=dev).contiguous()
            gp = self.get_geometry_parameters()
            g = _capi.MbxGeom()
            g.kind = self._kind()
            g.num_views, g.num_det_rows, g.num_det_channels = (int(v) for v in sinogram_shape)
            g.num_recon_rows, g.num_recon_cols, g.num_recon_slices = (int(v) for v in recon_shape)
            g.psf_radius = int(gp.psf_radius)
            g.bp_psf_radius = int(getattr(gp, 'bp_psf_radius', 1))
            g.entries_per_cylinder_batch = int(getattr(gp, 'entries_per_cylinder_batch', 128))
            g.delta_det_channel = float(gp.delta_det_channel)
            g.delta_det_row = float(self.get_params('delta_det_row'))
            g.det_channel_offset = float(gp.det_channel_offset)
            g.det_row_offset = float(self.get_params('det_row_offset'))
            g.delta_voxel = float(gp.delta_voxel)
            g.recon_slice_offset = float(getattr(gp, 'recon_slice_offset', 0.0))
            g.source_detector_dist = float(getattr(gp, 'source_detector_dist', np.inf))
            g.magnification = float(getattr(gp, 'magnification', 1.0))
            if g.kind == _capi.MBX_GEOM_TRANSLATION:  # (num_views, 3) translation vectors
                g.translations = self._angles_dev.data_ptr()
                g.delta_recon_row = float(gp.delta_recon_row)
                g.max_magnification = float(self._max_magnification())
            else:
                g.angles = self._angles_dev.data_ptr()
            if g.psf_radius > _capi.MBX_MAX_PSF_RADIUS or g.bp_psf_radius > _capi.MBX_MAX_PSF_RADIUS:
                raise ValueError('psf radius %d / %d exceeds the supported maximum %d' % (
                    g.psf_radius, g.bp_psf_radius, _capi.MBX_MAX_PSF_RADIUS))
            self._geom = g
        return self._geom

    def _dev(self, x, dtype=torch.float32):
        dev = self._device()
        if isinstance(x, torch.Tensor):
            return x.to(device=dev, dtype=dtype).contiguous()
        return torch.as_tensor(np.ascontiguousarray(x), device=dev).to(dtype).contiguous()

    # ------------------------------------------------------------------ projections
    def get_voxels_at_indices(self, recon, indices):
        recon_shape = self.get_params('recon_shape')
        r = self._dev(recon).reshape((-1,) + tuple(recon_shape[2:]))
        return r[self._dev(indices, torch.int64)]

    def reshape_recon(self, recon):
        return recon.reshape(self.get_params('recon_shape'))

    def sparse_forward_project(self, voxel_values, pixel_indices, view_indices=None, output_device=None):
        """(N, S) voxel cylinders at pixel_indices -> sinogram (len(view_indices), R, C)."""
        recon_shape = self.get_params('recon_shape')
        vox = self._dev(voxel_values)
        pix = self._dev(pixel_indices, torch.int32)
        if vox.ndim != 2 or vox.shape[0] != pix.shape[0] or vox.shape[1] != recon_shape[2]:
            raise ValueError('voxel_values must have shape[0:2] = (num_indices, num_slices)')
        views = None if view_indices is None else self._dev(view_indices, torch.int32)
        out = _capi.forward_project(self._geometry(), vox, pix, views)
        return out.cpu() if output_device == 'cpu' else out

    def sparse_back_project(self, sinogram, pixel_indices, view_indices=None, coeff_power=1, output_device=None):
        """Full sinogram -> (N, S) at pixel_indices; view_indices select rows of sinogram and angles."""
        sinogram_shape = self.get_params('sinogram_shape')
        sino = self._dev(sinogram)
        if tuple(sino.shape) != tuple(sinogram_shape):
            raise ValueError('sinogram must have shape {}, got {}'.format(sinogram_shape, tuple(sino.shape)))
        pix = self._dev(pixel_indices, torch.int32)
        views = None if view_indices is None else self._dev(view_indices, torch.int32)
        out = _capi.back_project(self._geometry(), sino, pix, views, coeff_power=coeff_power)
        return out.cpu() if output_device == 'cpu' else out

    def _full_indices(self):
        """gen_full_indices(recon_shape, use_ror_mask) as an int32 device tensor.  The host call runs every time,
        because it draws from np.random as the reference's does (and so shapes the partitions drawn after it); its
        result (the sorted region of reconstruction) depends only on the shape and the mask, so the device copy
        is kept and reused: a host-to-device copy would wait for the GPU work queued before it."""
        recon_shape = tuple(self.get_params('recon_shape'))
        idx = gen_full_indices(recon_shape, use_ror_mask=self.use_ror_mask)
        key = (recon_shape, bool(self.use_ror_mask))
        if self._full_idx is None or self._full_idx[0] != key:
            self._full_idx = (key, torch.as_tensor(idx, dtype=torch.int32, device=self._device()))
        return self._full_idx[1]

    def forward_project(self, recon):
        full_indices = self._full_indices()
        voxel_values = self.get_voxels_at_indices(recon, full_indices)
        return self.sparse_forward_project(voxel_values, full_indices)

    def back_project(self, sinogram):
        recon_shape = self.get_params('recon_shape')
        full_indices = self._full_indices()
        cyl = self.sparse_back_project(sinogram, full_indices)
        recon = torch.zeros((recon_shape[0] * recon_shape[1], recon_shape[2]), dtype=torch.float32,
                            device=cyl.device)
        recon[full_indices.long()] = cyl
        return recon.reshape(recon_shape)

    def compute_hessian_diagonal(self, weights=None, output_device=None):
        """Back projection of the weights with squared coefficients over every pixel (no ROR mask)."""
        sinogram_shape, recon_shape = self.get_params(['sinogram_shape', 'recon_shape'])
        w = None
        if weights is not None:
            w = self._dev(weights)
            if tuple(w.shape) != tuple(sinogram_shape):
                raise ValueError('Weights must be constant or an array compatible with sinogram'
                                 '\nGot weights.shape = {}, but sinogram.shape = {}'.format(tuple(w.shape),
                                                                                           sinogram_shape))
        nr, nc, ns = recon_shape
        idx = torch.arange(nr * nc, dtype=torch.int32, device=self._device())
        # no sinogram: the library back-projects the weights, or ones for unit weights without a buffer of ones
        return _capi.back_project(self._geometry(), None, idx, coeff_power=2, weights=w).reshape((nr, nc, ns))

    # ------------------------------------------------------------------ direct recon
    def direct_filter(self, sinogram, filter_name='ramp', view_batch_size=DIRECT_RECON_VIEW_BATCH_SIZE):
        if filter_name not in ['ramp']:
            raise ValueError('Unsupported filter. Supported filters are: ramp.')
        return _capi.direct_filter(self._geometry(), self._dev(sinogram))

    def direct_recon(self, sinogram, filter_name='ramp', view_batch_size=DIRECT_RECON_VIEW_BATCH_SIZE):
        return self.back_project(self.direct_filter(sinogram, filter_name=filter_name,
                                                    view_batch_size=view_batch_size))

    # ------------------------------------------------------------------ regularisation
    def auto_set_regularization_params(self, sinogram, weights=None):
        """tomography_model.py:756-796 (host NumPy on at most 20 subsampled views)."""
        if self.get_params('auto_regularize_flag'):
            num_views = sinogram.shape[0]
            max_views_to_use = np.minimum(20, num_views)
            step_size = num_views // max_views_to_use
            small_sinogram = _to_numpy(sinogram[::step_size])
            small_weights = 1 if weights is None else _to_numpy(weights[::step_size])
            sino_indicator = self._get_sino_indicator(small_sinogram)
            self.auto_set_sigma_y(small_sinogram, sino_indicator, small_weights)
            recon_std = self._get_estimate_of_recon_std(small_sinogram, sino_indicator)
            self.auto_set_sigma_x(recon_std)
            self.auto_set_sigma_prox(recon_std)
        names = ['sigma_y', 'sigma_x', 'sigma_prox']
        return dict(zip(names, [float(v) for v in self.get_params(names)]))

    def auto_set_sigma_y(self, sinogram, sino_indicator, weights=1):
        snr_db = self.get_params('snr_db')
        magnification = self.get_magnification()
        delta_voxel, delta_det_channel = self.get_params(['delta_voxel', 'delta_det_channel'])
        signal_rms = float(np.average(weights * sinogram ** 2, None, sino_indicator) ** 0.5)
        rel_noise_std = 10 ** (-snr_db / 20)
        pixel_pitch_relative_to_default = delta_voxel / (delta_det_channel / magnification)
        sigma_y = np.float32(rel_noise_std * signal_rms * (pixel_pitch_relative_to_default ** 0.5))
        self.set_params(no_warning=True, sigma_y=sigma_y, auto_regularize_flag=True)

    def auto_set_sigma_x(self, recon_std):
        sigma_x = np.float32(0.2 * (2 ** self.get_params('sharpness')) * recon_std)
        self.set_params(no_warning=True, sigma_x=sigma_x, auto_regularize_flag=True)

    def auto_set_sigma_prox(self, recon_std):
        sigma_prox = np.float32(0.2 * (2 ** self.get_params('sharpness')) * recon_std)
        self.set_params(no_warning=True, sigma_prox=sigma_prox, auto_regularize_flag=True)

    @staticmethod
    def _get_sino_indicator(sinogram):
        return np.int8(sinogram > (0.01 * 5.0) * np.mean(np.fabs(sinogram)))

    def _get_estimate_of_recon_std(self, sinogram, sino_indicator):
        delta_det_channel, delta_voxel, recon_shape = self.get_params(['delta_det_channel', 'delta_voxel',
                                                                       'recon_shape'])
        magnification = self.get_magnification()
        typical_sinogram_value = np.average(np.abs(sinogram), weights=sino_indicator)
        path_space = (2 * recon_shape[0] * recon_shape[1]) / (recon_shape[0] + recon_shape[1]) * delta_voxel
        path_sino = sinogram.shape[-1] * delta_det_channel / magnification
        return typical_sinogram_value / np.minimum(path_space, path_sino)

    def _qggmrf_params(self):
        qggmrf_nbr_wts, sigma_x, p, q, T = self.get_params(['qggmrf_nbr_wts', 'sigma_x', 'p', 'q', 'T'])
        return get_b_from_nbr_wts(qggmrf_nbr_wts), float(sigma_x), float(p), float(q), float(T)

    # ------------------------------------------------------------------ reconstruction
    @staticmethod
    def get_forward_model_loss(error_sinogram, sigma_y, weights=None, normalize=True):
        """tomography_model.py:1633-1658 (float64 accumulation on the device)."""
        e = error_sinogram.double() if isinstance(error_sinogram, torch.Tensor) else torch.as_tensor(error_sinogram).double()
        if weights is None:
            w, avg = 1.0, 1.0
        else:
            w = weights.double() if isinstance(weights, torch.Tensor) else torch.as_tensor(weights).double()
            avg = w.mean()
        if normalize:
            return float(torch.sqrt((1.0 / sigma_y ** 2) * torch.mean((e * e) * (w / avg))))
        return float((1.0 / (2 * sigma_y ** 2)) * torch.sum((e * e) * w))

    def recon(self, sinogram, weights=None, init_recon=None, max_iterations=15, stop_threshold_change_pct=0.2,
              first_iteration=0, compute_prior_loss=False, num_iterations=None, logfile_path='./logs/recon.log',
              print_logs=True):
        """MBIR reconstruction by multi-granular VCD (tomography_model.py:966-1084)."""
        if num_iterations is not None:
            max_iterations = num_iterations
        if first_iteration == 0 or self.logger is None:
            self.setup_logger(logfile_path=logfile_path, print_logs=print_logs)
        regularization_params = self.auto_set_regularization_params(sinogram, weights=weights)
        recon_shape, granularity = self.get_params(['recon_shape', 'granularity'])
        partitions = gen_set_of_pixel_partitions(recon_shape, granularity, use_ror_mask=self.use_ror_mask)
        partition_sequence = gen_partition_sequence(self.get_params('partition_sequence'), max_iterations)
        partition_sequence = partition_sequence[first_iteration:]
        recon, loss_vectors = self.vcd_recon(sinogram, partitions, partition_sequence, stop_threshold_change_pct,
                                             weights=weights, init_recon=init_recon,
                                             compute_prior_loss=compute_prior_loss, first_iteration=first_iteration)
        fm_rmse = [float(v) for v in loss_vectors[0]]
        prior_loss = [float(v) for v in loss_vectors[1]] if compute_prior_loss else [0]
        recon_params = ReconParams(len(fm_rmse), granularity, [int(v) for v in partition_sequence], fm_rmse,
                                   prior_loss, regularization_params, [100 * float(v) for v in loss_vectors[2]],
                                   [float(v) for v in loss_vectors[3]])._asdict()
        notes = 'Reconstruction completed: {}\n\n'.format(datetime.datetime.now())
        return recon, self.get_recon_dict(recon_params, notes=notes)

    def prox_map(self, prox_input, sinogram, weights=None, init_recon=None, stop_threshold_change_pct=0.2,
                 max_iterations=3, first_iteration=0, logfile_path='./logs/recon.log', print_logs=True):
        """Proximal map for Plug-and-Play (tomography_model.py:1660-1697): VCD with the quadratic proximal prior
        centred on prox_input, using the model's current sigma_y and sigma_prox (no auto-regularisation).
        Returns (recon, loss_vectors) as the reference does."""
        recon_shape, granularity = self.get_params(['recon_shape', 'granularity'])
        partitions = gen_set_of_pixel_partitions(recon_shape, granularity)
        partition_sequence = gen_partition_sequence(self.get_params('partition_sequence'), max_iterations)
        partition_sequence = partition_sequence[first_iteration:]
        if first_iteration == 0 or self.logger is None:
            self.setup_logger(logfile_path=logfile_path, print_logs=print_logs)
        return self.vcd_recon(sinogram, partitions, partition_sequence, stop_threshold_change_pct, weights=weights,
                              init_recon=init_recon, prox_input=prox_input, first_iteration=first_iteration)

    # ------------------------------------------------------------------ parameter files and recon dicts
    @classmethod
    def get_required_param_names(cls):
        """Names of the constructor's parameters, in signature order (tomography_model.py:94-115)."""
        params = inspect.signature(cls.__init__).parameters.values()
        return [p.name for p in params if p.name != 'self' and
                p.kind not in (inspect.Parameter.VAR_POSITIONAL, inspect.Parameter.VAR_KEYWORD)]

    @classmethod
    def from_file(cls, source):
        """A model of this class from parameters saved by :meth:`to_file` (a .yml/.yaml file name, a YAML string
        or a stream) (tomography_model.py:296-317)."""
        required_params, params = ParameterHandler.load_param_dict(source, cls.get_required_param_names(),
                                                                   values_only=True)
        with warnings.catch_warnings():
            warnings.simplefilter("ignore")
            new_model = cls(**required_params)
            new_model.set_params(**params)
        return new_model

    def to_file(self, filename):
        """Every parameter to a .yml/.yaml file, or the YAML text when filename is None
        (tomography_model.py:319-331)."""
        return self.save_params(self.params, filename)

    def get_recon_dict(self, recon_params=None, notes=None, save_log=True, save_model=True, str_format=False):
        """Dict with 'recon_params', 'recon_log', 'notes' and 'model_params' (the Param dict, or its YAML text
        when str_format) (tomography_model.py:333-386)."""
        recon_dict = dict()
        recon_dict['recon_params'] = "# Recon params not saved." if recon_params is None else recon_params
        if self.log_buffer is None or not save_log:
            recon_dict['recon_log'] = "# Log info not saved."
        else:
            recon_dict['recon_log'] = self.log_buffer.getvalue()
        recon_dict['notes'] = '# No notes saved' if notes is None else notes
        recon_dict['model_params'] = self.params.copy() if save_model else '# Model not saved'
        if str_format:
            recon_dict = self.convert_subdicts_to_strings(recon_dict)
        return recon_dict

    @staticmethod
    def convert_subdicts_to_strings(recon_dict):
        """Every entry as a string: model_params as a parameter file, other dicts as YAML, the rest by str()
        (tomography_model.py:387-410)."""
        if not isinstance(recon_dict, dict):
            return recon_dict
        string_dict = recon_dict.copy()
        for key, value in string_dict.items():
            if key == 'model_params' and isinstance(value, dict):
                string_dict[key] = ParameterHandler.save_params(value)
            elif isinstance(value, dict):
                buf = io.StringIO()
                yaml.safe_dump(_yaml_plain(value), buf, default_flow_style=False, sort_keys=False)
                string_dict[key] = buf.getvalue()
            else:
                try:
                    string_dict[key] = str(value)
                except Exception:
                    raise ValueError('Entries in recon_dict must be strings or dicts that can be converted to strings')
        return string_dict

    def save_recon_hdf5(self, filepath, recon, recon_dict=None):
        """One dataset 'recon' with the recon_dict entries as string attributes (tomography_model.py:412-440).
        Needs h5py."""
        from .utilities import save_data_hdf5
        save_data_hdf5(filepath, _to_numpy(recon), 'recon', recon_dict)
        if self.logger:
            self.logger.info(f"Saved reconstruction and params to '{filepath}'")

    @staticmethod
    def load_recon_hdf5(filepath, recreate_model=False):
        """(recon, recon_dict) from :meth:`save_recon_hdf5`, plus the model rebuilt from its parameters when
        recreate_model (tomography_model.py:442-473).  Needs h5py."""
        from .utilities import load_data_hdf5
        recon, recon_dict = load_data_hdf5(filepath)
        if not recreate_model:
            return recon, recon_dict
        model_yaml = recon_dict['model_params']
        class_name = model_yaml.split("<class '")[1].split("'>")[0].split(".")[-1]
        import mbirjax_b200
        ct_model = getattr(mbirjax_b200, class_name).from_file(model_yaml)
        return recon, recon_dict, ct_model

    def vcd_recon(self, sinogram, partitions, partition_sequence, stop_threshold_change_pct, weights=None,
                  init_recon=None, prox_input=None, compute_prior_loss=False, first_iteration=0):
        """tomography_model.py:1086-1308; each subset update is one mbx_vcd_subset_step on the device."""
        positivity = bool(self.get_params('positivity_flag'))
        state = self._vcd_setup(sinogram, weights, init_recon)
        prox_flat, sigma_prox = None, 0.0
        if prox_input is not None:  # tomography_model.py:1158-1170
            recon_shape = self.get_params('recon_shape')
            prox = self._dev(prox_input)
            if tuple(prox.shape) != tuple(recon_shape):
                raise ValueError('prox_input does not have the correct size. \nExpected {}, but got shape {} for '
                                 'prox_input shape.'.format(recon_shape, tuple(prox.shape)))
            prox_flat = prox.reshape((-1, recon_shape[2])).contiguous()
            sigma_prox = float(self.get_params('sigma_prox'))
        recon_shape = self.get_params('recon_shape')
        dev = state['device']
        w, flat_recon, error_sinogram = state['weights'], state['flat_recon'], state['error_sinogram']
        fm_hessian, fm_constant, qp, sigma_y = (state['fm_hessian'], state['fm_constant'], state['qp'],
                                                state['sigma_y'])
        geom = self._geometry()
        # subsets in Z-order: same sets, spatially coherent processing order for the projectors
        dev_partitions = [torch.as_tensor(morton_sorted_partition(part, recon_shape[1]), device=dev,
                                          dtype=torch.int32).contiguous() for part in partitions]
        workspaces = {}
        max_subsets = max(part.shape[0] for part in partitions)
        stats = torch.zeros((max_subsets, 4), dtype=torch.float64, device=dev)
        n_iter = len(partition_sequence)
        fm_rmse, pm_loss, nmae_update, alpha_values = (np.zeros(n_iter) for _ in range(4))
        num_iters = 0
        if self.logger is not None:
            self.logger.info('Starting VCD iterations')
        for i in range(n_iter):
            part = dev_partitions[int(partition_sequence[i])]
            num_subsets, subset_size = part.shape
            if subset_size not in workspaces:
                workspaces[subset_size] = _capi.vcd_subset_step_workspace(geom, subset_size, dev)
            for j, index in enumerate(np.random.permutation(num_subsets)):
                _capi.vcd_subset_step(geom, flat_recon, error_sinogram, w, fm_hessian, part[int(index)], fm_constant,
                                      qp, stats[j], workspaces[subset_size], prox_input=prox_flat,
                                      sigma_prox=sigma_prox, positivity=positivity)
            st = stats[:num_subsets].cpu().numpy()
            ell1 = float(np.sum(st[:, 1]))
            alpha_values[i] = float(np.mean(st[:, 0]))
            fm_rmse[i] = self.get_forward_model_loss(error_sinogram, sigma_y, w)
            nmae_update[i] = ell1 / float(torch.sum(torch.abs(flat_recon.double())))
            if compute_prior_loss:
                loss, _ = _capi.qggmrf_loss_grad(flat_recon.reshape(recon_shape), qp, need_grad=False)
                pm_loss[i] = float(loss) / flat_recon.numel()
            if self.logger is not None:
                self.logger.info('After iteration {} of a max of {}: Pct change={:.4f}, Forward loss={:.4f}'.format(
                    i + first_iteration, n_iter + first_iteration, 100 * nmae_update[i], fm_rmse[i]))
            num_iters += 1
            if nmae_update[i] < stop_threshold_change_pct / 100:
                if self.logger is not None:
                    self.logger.warning('Change threshold stopping condition reached')
                break
        self.last_error_sinogram = error_sinogram
        return flat_recon.reshape(recon_shape), (fm_rmse[:num_iters], pm_loss[:num_iters], nmae_update[:num_iters],
                                                 alpha_values[:num_iters])

    def _vcd_setup(self, sinogram, weights=None, init_recon=None):
        """Device state for VCD iterations (tomography_model.py:1110-1192): initial recon (direct recon when
        init_recon is None), alpha-rescaled error sinogram, Hessian diagonal, fm constant and qGGMRF record."""
        recon_shape = self.get_params('recon_shape')
        num_slices = recon_shape[2]
        dev = self._device()
        sino = self._dev(sinogram)
        w = None if weights is None else self._dev(weights)
        if init_recon is None:
            init = self.direct_recon(sino)
        elif isinstance(init_recon, int) and init_recon == 0:
            init = torch.zeros(recon_shape, dtype=torch.float32, device=dev)
        else:
            init = self._dev(init_recon)
        if tuple(init.shape) != tuple(recon_shape):
            raise ValueError('init_recon does not have the correct shape. \nExpected {}, but got shape {} for '
                             'init_recon shape.'.format(recon_shape, tuple(init.shape)))
        # alpha minimising (1/2)||y - alpha A x||_W^2 (tomography_model.py:1137-1152), kept on the device (float64
        # sums, applied in float32) so that setting up queues GPU work without waiting for it
        error_sinogram = self.forward_project(init)
        wes = error_sinogram if w is None else w * error_sinogram
        norm = torch.sum(wes.double() * error_sinogram.double())
        num = torch.sum(wes.double() * sino.double())
        alpha = torch.where(norm > 0, num / torch.where(norm > 0, norm, torch.ones_like(norm)),
                            torch.ones_like(norm)).float()
        error_sinogram = (sino - alpha * error_sinogram).contiguous()
        flat_recon = (alpha * init).reshape((-1, num_slices)).contiguous()
        del wes, norm, num
        sigma_y = float(self.get_params('sigma_y'))
        fm_hessian = self.compute_hessian_diagonal(weights=w).reshape((-1, num_slices)).contiguous()
        b, sigma_x, p, q, T = self._qggmrf_params()
        return {'device': dev, 'weights': w, 'flat_recon': flat_recon, 'error_sinogram': error_sinogram,
                'fm_hessian': fm_hessian, 'fm_constant': 1.0 / (sigma_y ** 2.0), 'sigma_y': sigma_y,
                'qp': _capi.qggmrf_params(b, sigma_x, p, q, T)}

    # ------------------------------------------------------------------ misc reference helpers
    def gen_weights(self, sinogram, weight_type):
        """tomography_model.py:1727-1764."""
        s = self._dev(sinogram)
        if weight_type == 'unweighted':
            return torch.ones_like(s)
        if weight_type == 'transmission':
            return torch.exp(-s)
        if weight_type == 'transmission_root':
            return torch.exp(-s / 2)
        if weight_type == 'emission':
            return 1.0 / (torch.abs(s) + 0.1)
        raise Exception('gen_weights: undefined weight_type {}'.format(weight_type))

    def gen_modified_3d_sl_phantom(self):
        """tomography_model.py:1766-1775: the low-dynamic-range 3D Shepp-Logan phantom of the recon shape, on the
        model's GPU (on the host when none is visible, since it is test data rather than compute)."""
        from .utilities import generate_3d_shepp_logan_low_dynamic_range
        device = self._device() if torch.cuda.is_available() else torch.device('cpu')
        return generate_3d_shepp_logan_low_dynamic_range(self.get_params('recon_shape'), device=device)

    def scale_recon_shape(self, row_scale=1.0, col_scale=1.0, slice_scale=1.0):
        old_rows, old_cols, old_slices = self.get_params('recon_shape')
        new = (int(old_rows * row_scale), int(old_cols * col_scale), int(old_slices * slice_scale))
        self.set_params(recon_shape=new)
        return new[0] - old_rows, new[1] - old_cols, new[2] - old_slices


def _yaml_plain(value):
    """Tuples as lists and NumPy scalars as Python scalars, recursively, for a YAML dump."""
    if isinstance(value, dict):
        return {k: _yaml_plain(v) for k, v in value.items()}
    if isinstance(value, (list, tuple)):
        return [_yaml_plain(v) for v in value]
    if isinstance(value, np.generic):
        return value.item()
    if isinstance(value, np.ndarray):
        return value.tolist()
    return value


def _to_numpy(x):
    if isinstance(x, torch.Tensor):
        return x.detach().cpu().numpy()
    return np.asarray(x)


# ---------------------------------------------------------------------- the reference's per-view plugin functions
ProjectorParams = namedtuple('ProjectorParams', ['sinogram_shape', 'recon_shape', 'geometry_params'])


def translation_max_magnification(delta_recon_row, num_recon_rows, min_ty, magnification, source_detector_dist):
    """An upper bound of mag = 1 / (1/M - y/D) over every pixel row of a translation geometry, y = delta_recon_row
    (row - (Nr-1)/2) - ty, for views whose smallest ty is min_ty, with a small margin; 0 when some pixel reaches
    the source plane.  The fast back projector sizes its detector-row cache from it."""
    y_max = delta_recon_row * 0.5 * (num_recon_rows - 1) - float(min_ty)
    inv = 1.0 / magnification - y_max / source_detector_dist
    return 0.0 if inv <= 1e-6 else 1.001 / inv


def one_view_geometry(kind, projector_params, view_params):
    """The mbx_geom record of one view of a geometry, from the arguments of the reference's per-view plugin
    functions: projector_params = (sinogram_shape, recon_shape, geometry_params), the namedtuple the reference's
    Projectors builds (projectors.py:44-53), and the view's angle or translation vector.  Geometry parameters the
    namedtuple of a geometry does not carry take their defaults (a parallel beam has no row spacing or offset).
    Returns (record, the device tensor of the view parameters that the record points to)."""
    sinogram_shape, recon_shape, gp = projector_params
    translation = kind == _capi.MBX_GEOM_TRANSLATION
    vp = np.asarray(_to_numpy(view_params), dtype=np.float32).reshape(-1)
    if translation and vp.shape != (3,):
        raise ValueError('translation_vector must hold (x, y, z); got {} values'.format(vp.size))
    if not translation and vp.shape != (1,):
        raise ValueError('angle must be one value; got {} values'.format(vp.size))
    view_dev = torch.as_tensor(vp.reshape(1, -1) if translation else vp, device=_cuda_device()).contiguous()
    g = _capi.MbxGeom()
    g.kind = kind
    g.num_views = 1
    g.num_det_rows, g.num_det_channels = int(sinogram_shape[1]), int(sinogram_shape[2])
    g.num_recon_rows, g.num_recon_cols, g.num_recon_slices = (int(v) for v in recon_shape)
    g.psf_radius = int(gp.psf_radius)
    g.bp_psf_radius = int(getattr(gp, 'bp_psf_radius', 1))
    g.entries_per_cylinder_batch = int(getattr(gp, 'entries_per_cylinder_batch', 128))
    g.delta_det_channel = float(gp.delta_det_channel)
    g.delta_det_row = float(getattr(gp, 'delta_det_row', 1.0))
    g.det_channel_offset = float(gp.det_channel_offset)
    g.det_row_offset = float(getattr(gp, 'det_row_offset', 0.0))
    g.delta_voxel = float(gp.delta_voxel)
    g.recon_slice_offset = float(getattr(gp, 'recon_slice_offset', 0.0))
    g.source_detector_dist = float(getattr(gp, 'source_detector_dist', np.inf))
    g.magnification = float(getattr(gp, 'magnification', 1.0))
    if translation:
        g.translations = view_dev.data_ptr()
        g.delta_recon_row = float(gp.delta_recon_row)
        g.max_magnification = float(translation_max_magnification(gp.delta_recon_row, recon_shape[0], vp[1],
                                                                   gp.magnification, gp.source_detector_dist))
    else:
        g.angles = view_dev.data_ptr()
    if g.psf_radius > _capi.MBX_MAX_PSF_RADIUS or g.bp_psf_radius > _capi.MBX_MAX_PSF_RADIUS:
        raise ValueError('psf radius %d / %d exceeds the supported maximum %d' % (
            g.psf_radius, g.bp_psf_radius, _capi.MBX_MAX_PSF_RADIUS))
    return g, view_dev


def forward_project_one_view(kind, voxel_values, pixel_indices, view_params, projector_params):
    """The reference's forward_project_pixel_batch_to_one_view: (N, S) voxel cylinders at pixel_indices ->
    the (R, C) view, through mbx_sparse_forward_project on a one-view geometry."""
    g, view_dev = one_view_geometry(kind, projector_params, view_params)
    dev = view_dev.device
    vox = _on_device(voxel_values, dev, torch.float32)
    pix = _on_device(pixel_indices, dev, torch.int32)
    if vox.ndim != 2 or pix.ndim != 1 or vox.shape[0] != pix.shape[0] or vox.shape[1] != g.num_recon_slices:
        raise ValueError('voxel_values must have shape[0:2] = (num_indices, num_slices)')
    return _capi.forward_project(g, vox, pix)[0]


def back_project_one_view(kind, sinogram_view, pixel_indices, view_params, projector_params, coeff_power=1):
    """The reference's back_project_one_view_to_pixel_batch: the (R, C) view -> (N, S) voxel cylinders at
    pixel_indices with coefficients A_ij ** coeff_power, through mbx_sparse_back_project on a one-view
    geometry."""
    g, view_dev = one_view_geometry(kind, projector_params, view_params)
    dev = view_dev.device
    view = _on_device(sinogram_view, dev, torch.float32)
    pix = _on_device(pixel_indices, dev, torch.int32)
    if tuple(view.shape) != (g.num_det_rows, g.num_det_channels):
        raise ValueError('sinogram_view must have shape {}, got {}'.format(
            (g.num_det_rows, g.num_det_channels), tuple(view.shape)))
    if pix.ndim != 1:
        raise ValueError('pixel_indices must be a 1D array')
    if coeff_power not in (1, 2):
        raise ValueError('coeff_power must be 1 or 2')
    return _capi.back_project(g, view.reshape((1,) + tuple(view.shape)), pix, coeff_power=coeff_power)


def _on_device(x, device, dtype):
    if isinstance(x, torch.Tensor):
        return x.to(device=device, dtype=dtype).contiguous()
    return torch.as_tensor(np.ascontiguousarray(x), device=device).to(dtype).contiguous()

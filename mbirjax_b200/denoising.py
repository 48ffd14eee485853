"""qGGMRF denoiser (denoising.py of the reference) on the B200 kernels.

``QGGMRFDenoiser`` keeps the reference's interface and host logic: the noise estimate from 4-neighbour standard
deviations (denoising.py:80-136), the regularisation hooks (sigma_y = sigma_noise), one fixed partition of
``granularity[partition_sequence[0]]`` subsets drawn with ``np.random`` (no region-of-reconstruction mask by
default), and subsets visited in order in every iteration (denoising.py:213-260) until the relative change falls
below the threshold (denoising.py:266-330).  Each subset update is one ``mbx_qggmrf_denoise_step`` on the device.
``median_filter3d`` is the 27-point median with edge replication (denoising.py:414-490).
"""
import datetime

import numpy as np
import torch

from . import _capi
from .tomography_model import TomographyModel, ReconParams, _to_numpy
from .vcd_utils import gen_set_of_pixel_partitions
from .qggmrf import get_b_from_nbr_wts


class QGGMRFDenoiser(TomographyModel):
    """The qGGMRF proximal-map denoiser; the primary interface is :meth:`denoise`."""

    def __init__(self, image_shape):
        super().__init__(image_shape, view_params_name='None', sigma_noise=None)
        self.use_ror_mask = False
        self.set_params(sharpness=0)  # the denoiser's default sharpness
        self.set_params(granularity=[16], partition_sequence=[0])

    def get_magnification(self):
        return 1.0

    def verify_valid_params(self):
        super().verify_valid_params()
        sinogram_shape = self.get_params('sinogram_shape')
        image_shape = self.get_params('recon_shape')
        if image_shape is not None and tuple(image_shape) != tuple(sinogram_shape):
            raise ValueError('image_shape and sinogram_shape must be the same. \n'
                             'Got {} for image_shape and {} for sinogram_shape'.format(image_shape, sinogram_shape))

    def get_geometry_parameters(self):
        raise NotImplementedError('get_geometry_parameters is not implemented for QGGMRFDenoiser.')

    def create_projectors(self):
        pass

    def auto_set_recon_size(self, sinogram_shape, no_compile=True, no_warning=False):
        self.set_params(no_compile=no_compile, no_warning=no_warning, recon_shape=tuple(sinogram_shape))

    def auto_set_sigma_y(self, sinogram, sino_indicator, weights=1):
        self.set_params(no_warning=True, sigma_y=self.get_params('sigma_noise'), auto_regularize_flag=True)

    def estimate_image_noise_std(self, image):
        """Noise standard deviation from the image: 4-neighbour std over a support mask, twice (denoising.py:80-91)."""
        image = _to_numpy(image)
        support_indicator = self._get_sino_indicator(image, sigma_noise=0.0)
        sigma_noise = self._get_estimate_of_recon_std(image, support_indicator)
        support_indicator = self._get_sino_indicator(image, sigma_noise=sigma_noise)
        return self._get_estimate_of_recon_std(image, support_indicator)

    def _get_estimate_of_recon_std(self, noisy_image, support_indicator):
        """Mean over the support of the std of each voxel and its three lower neighbours (denoising.py:93-116)."""
        noisy_image = _to_numpy(noisy_image)
        inds = np.where(support_indicator)
        inds = [np.clip(inds[j], 1, None) for j in range(len(inds))]
        vals = np.stack([noisy_image[inds[0], inds[1], inds[2]],
                         noisy_image[inds[0] - 1, inds[1], inds[2]],
                         noisy_image[inds[0], inds[1] - 1, inds[2]],
                         noisy_image[inds[0], inds[1], inds[2] - 1]], axis=0)
        return np.mean(np.std(vals, axis=0))

    def _get_sino_indicator(self, noisy_image, sigma_noise=None):
        """Support mask: voxels above 5% of the mean magnitude plus sigma_noise (denoising.py:118-136)."""
        noisy_image = _to_numpy(noisy_image)
        if sigma_noise is None:
            sigma_noise = self.get_params('sigma_noise')
        percent_noise_floor = 5.0
        threshold = (0.01 * percent_noise_floor) * np.mean(np.fabs(noisy_image)) + sigma_noise
        threshold = min(threshold, np.amax(noisy_image))
        return np.int8(noisy_image >= threshold)

    def recon(self, *args, **kwargs):
        raise NotImplementedError('recon is not implemented for QGGMRFDenoiser.  Use `denoise` instead.')

    def denoise(self, image, sigma_noise=None, use_ror_mask=False, init_image=None, max_iterations=15,
                stop_threshold_change_pct=0.2, first_iteration=0, logfile_path='./logs/recon.log', print_logs=True):
        """MAP estimate of the clean volume under the qGGMRF prior for additive white noise of std sigma_noise
        (estimated from the image when None).  Returns (denoised_image, denoiser_dict) as the reference."""
        self.use_ror_mask = use_ror_mask
        if sigma_noise is None:
            sigma_noise = self.estimate_image_noise_std(image)
        self.set_params(sigma_noise=float(sigma_noise))
        if first_iteration == 0 or self.logger is None:
            self.setup_logger(logfile_path=logfile_path, print_logs=print_logs)
        if self.logger is not None:
            self.logger.info('Initializing QGGMRFDenoiser')
        regularization_params = self.auto_set_regularization_params(image)

        image_shape, granularity = self.get_params(['recon_shape', 'granularity'])
        partition_sequence = self.get_params('partition_sequence')
        partition_index = partition_sequence[0]
        partition = gen_set_of_pixel_partitions(image_shape, [granularity[partition_index]],
                                                use_ror_mask=self.use_ror_mask)[0]

        img = self._dev(image)
        init = img.clone() if init_image is None else self._dev(init_image)
        ns = image_shape[2]
        flat_error = (img - init).reshape((-1, ns)).contiguous()
        flat_image = init.reshape((-1, ns)).contiguous()
        del img, init
        fm_constant = 1.0 / (float(self.get_params('sigma_y')) ** 2.0)
        qggmrf_nbr_wts, sigma_x, p, q, T = self.get_params(['qggmrf_nbr_wts', 'sigma_x', 'p', 'q', 'T'])
        qp = _capi.qggmrf_params(get_b_from_nbr_wts(qggmrf_nbr_wts), sigma_x, p, q, T)

        dev = flat_image.device
        subsets = torch.as_tensor(partition, device=dev, dtype=torch.int32).contiguous()
        k = subsets.shape[0]
        stats = torch.zeros((k, 4), dtype=torch.float64, device=dev)
        workspace = _capi._workspace(_capi.load_library().mbx_qggmrf_denoise_step_workspace_bytes(
            int(subsets.shape[1]), ns), dev)
        stop_thresh = stop_threshold_change_pct / 100.0
        nmae_update, alpha_values = [], []
        if self.logger is not None:
            self.logger.info('Starting VCD iterations')
        for i in range(max_iterations):
            for j in range(k):  # subsets in order, as the reference's fori_loop
                _capi.qggmrf_denoise_step(flat_image, flat_error, image_shape, subsets[j], fm_constant, qp, stats[j],
                                          workspace)
            st = stats.cpu().numpy()
            nmae = float(np.sum(st[:, 1])) / float(torch.sum(torch.abs(flat_image.double())))
            nmae_update.append(nmae)
            alpha_values.append(float(np.mean(st[:, 0])))
            if self.logger is not None and i % 5 == 0:
                self.logger.info('After iteration {} of a max of {}: Pct change={:.4f}'.format(
                    i + first_iteration, max_iterations, 100 * nmae))
            if nmae < stop_thresh:
                break
        recon_params = ReconParams(len(nmae_update), granularity, partition_sequence, None, None,
                                   regularization_params, [100 * v for v in nmae_update], alpha_values)._asdict()
        notes = 'Reconstruction completed: {}\n\n'.format(datetime.datetime.now())
        return self.reshape_recon(flat_image), self.get_recon_dict(recon_params, notes=notes)


def median_filter3d(x, max_block_gb=4.0):
    """27-point (3x3x3) median filter with replicated edges, same shape, float32 on the device
    (denoising.py:414-490; max_block_gb is accepted for interface compatibility: one kernel pass needs no
    blocking)."""
    dev = torch.device('cuda', torch.cuda.current_device()) if torch.cuda.is_available() else None
    if dev is None:
        raise _capi.MbxError('median_filter3d needs a CUDA device')
    t = x.to(device=dev, dtype=torch.float32) if isinstance(x, torch.Tensor) else torch.as_tensor(
        np.ascontiguousarray(x), device=dev).to(torch.float32)
    return _capi.median_filter3d(t.contiguous())

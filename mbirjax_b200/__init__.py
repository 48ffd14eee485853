"""mbirjax_b200: the MBIR hot path of mbirjax (v0.6.7) re-built for NVIDIA B200 (sm_100a).

Public API mirrors the reference: ``ParallelBeamModel``, ``ConeBeamModel``, ``TranslationModel`` (all
``TomographyModel``s with
``set_params``, ``forward_project``, ``back_project``, ``sparse_forward_project``, ``sparse_back_project``,
``compute_hessian_diagonal``, ``recon``, ``direct_recon``), the pixel-partition utilities and the qGGMRF
prior.  ``mbirjax_b200.autograd`` wraps the projector pair as torch autograd functions and
``mbirjax_b200.batched`` reconstructs many scans of uneven geometry together.  ``QGGMRFDenoiser`` and
``median_filter3d`` are the reference's denoising tools.

All compute runs in the CUDA library ``mbirjax_b200/_lib/libmbirjax_b200.so`` (C ABI:
``include/mbirjax_b200.h``), built by ``mbirjax_b200.build()``.
"""
import os
import subprocess

from .parameter_handler import ParameterHandler, Param
from .tomography_model import TomographyModel
from .parallel_beam import ParallelBeamModel
from .cone_beam import ConeBeamModel
from .translation_model import TranslationModel
from .denoising import QGGMRFDenoiser, median_filter3d
from .vcd_utils import (get_2d_ror_mask, gen_pixel_partition, gen_set_of_pixel_partitions, gen_partition_sequence,
                        gen_full_indices)
from .qggmrf import get_b_from_nbr_wts, qggmrf_gradient_and_hessian_at_indices, qggmrf_loss, qggmrf_loss_and_grad
from ._capi import MbxError, load_library, lib_path, version

_CSRC = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'csrc')


def build(jobs=8, verbose=False):
    """Compile the CUDA library for sm_100a in-tree (make -C mbirjax_b200/csrc)."""
    cmd = ['make', '-C', _CSRC, '-j%d' % jobs]
    res = subprocess.run(cmd, capture_output=not verbose, text=True)
    if res.returncode != 0:
        raise RuntimeError('building the mbirjax_b200 CUDA library failed:\n%s\n%s' % (res.stdout, res.stderr))
    return lib_path()

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

_HERE = os.path.dirname(os.path.abspath(__file__))
_CSRC = os.path.join(_HERE, 'csrc')
TORCH_OPS_SOURCE = os.path.join(_HERE, 'csrc_torch', 'mbx_torch_ops.cpp')
TORCH_OPS_LIB = os.path.join(_HERE, '_lib', 'libmbirjax_b200_torch.so')


def build(jobs=8, verbose=False, torch_ops=True):
    """Compile the CUDA library for sm_100a in-tree (make -C mbirjax_b200/csrc), then the PyTorch operator
    library over its C ABI (mbirjax_b200/_lib/libmbirjax_b200_torch.so)."""
    cmd = ['make', '-C', _CSRC, '-j%d' % jobs]
    res = subprocess.run(cmd, capture_output=not verbose, text=True)
    if res.returncode != 0:
        raise RuntimeError('building the mbirjax_b200 CUDA library failed:\n%s\n%s' % (res.stdout, res.stderr))
    if torch_ops:
        build_torch_ops(verbose)
    return lib_path()


def build_torch_ops(verbose=False):
    """g++ of the TORCH_LIBRARY operators (csrc_torch/mbx_torch_ops.cpp) against the installed torch, linked to the
    CUDA library beside it; skipped when the output is newer than its source and the CUDA library."""
    import torch
    import torch.utils.cpp_extension as ext
    src, out, lib = TORCH_OPS_SOURCE, TORCH_OPS_LIB, lib_path()
    if os.path.exists(out) and os.path.getmtime(out) >= max(os.path.getmtime(src), os.path.getmtime(lib)):
        return out
    cuda_home = ext.CUDA_HOME or '/usr/local/cuda'
    incs = [os.path.join(os.path.dirname(torch.__file__), 'include'),
            os.path.join(os.path.dirname(torch.__file__), 'include', 'torch', 'csrc', 'api', 'include'),
            os.path.join(cuda_home, 'include')]
    libdirs = [os.path.join(os.path.dirname(torch.__file__), 'lib'), os.path.join(cuda_home, 'lib64'),
               os.path.dirname(lib)]
    abi = int(torch._C._GLIBCXX_USE_CXX11_ABI)
    cmd = (['g++', '-O2', '-std=c++17', '-fPIC', '-shared', '-D_GLIBCXX_USE_CXX11_ABI=%d' % abi, src, '-o', out] +
           ['-I' + d for d in incs] + ['-L' + d for d in libdirs] +
           ['-lmbirjax_b200', '-ltorch', '-ltorch_cpu', '-ltorch_cuda', '-lc10', '-lc10_cuda', '-lcudart',
            '-Wl,-rpath,$ORIGIN'])
    res = subprocess.run(cmd, capture_output=not verbose, text=True)
    if res.returncode != 0:
        raise RuntimeError('building the mbirjax_b200 torch operators failed:\n%s\n%s' % (res.stdout, res.stderr))
    return out

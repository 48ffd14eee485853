"""The allocation-free back projection entry point (mbx_sparse_back_project_noalloc).

It exists for callers that cannot allocate GPU memory at call time, such as code running inside JAX (which
the reference configures to reserve 98% of the GPU for its own allocator).  Its scratch is a static device
array inside the library.  These checks call it through the C ABI on cases where the back projector splits the
views and so needs scratch, two calls in a row, and compare it with mbx_sparse_back_project given a caller
workspace.  The file is named to be collected last.
"""
import ctypes

import numpy as np
import pytest
import torch

from mbirjax_b200 import _capi
from cases import make_case, rel_l2

pytestmark = pytest.mark.gpu


def _case(kind, seed, views, rows, channels):
    model, geom = make_case(kind, views=views, rows=rows, channels=channels)
    nr, nc, ns = geom.recon_shape
    rng = np.random.default_rng(seed)
    idx = torch.as_tensor(np.sort(rng.choice(nr * nc, nr * nc // 3, replace=False)).astype(np.int32), device='cuda')
    sino = torch.as_tensor(rng.standard_normal(geom.sinogram_shape).astype(np.float32), device='cuda')
    w = torch.as_tensor(rng.random(geom.sinogram_shape).astype(np.float32), device='cuda')
    return model, sino, w, idx  # the model owns the device angle table the geometry record points to


def test_noalloc_back_projection_matches_workspace_version(cuda):
    lib = _capi.load_library()
    cases = [('parallel', 1, 96, 16, 64, 1, False), ('cone', 2, 80, 12, 48, 2, True)]  # two calls in a row
    for kind, seed, v, r, c, cp, weighted in cases:
        model, sino, w, idx = _case(kind, seed, v, r, c)
        g = model._geometry()
        need = lib.mbx_back_project_workspace_bytes(ctypes.byref(g), int(idx.shape[0]), g.num_views)
        assert 0 < need <= 16 << 20  # the case exercises the scratch
        wts = w if weighted else None
        ref = _capi.back_project(g, sino, idx, coeff_power=cp, weights=wts)
        got = _capi.back_project_noalloc(g, sino, idx, coeff_power=cp, weights=wts)
        torch.cuda.synchronize()
        assert rel_l2(got.cpu().numpy(), ref.cpu().numpy()) <= 1e-6

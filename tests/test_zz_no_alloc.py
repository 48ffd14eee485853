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


def test_noalloc_rejects_bad_calls_before_any_launch(cuda):
    """Argument errors come back as codes before any launch, and the output buffer keeps its contents."""
    lib = _capi.load_library()
    model, sino, w, idx = _case('parallel', 3, 40, 8, 32)
    g = model._geometry()
    out = torch.full((int(idx.shape[0]), g.num_recon_slices), 7.0, device='cuda')
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    args = (ctypes.byref(g), ctypes.c_void_p(sino.data_ptr()), None)
    # pixel indices missing for a non-empty pixel list
    rc = lib.mbx_sparse_back_project_noalloc(*args, None, int(idx.shape[0]), None, g.num_views, 1, 1.0,
                                             ctypes.c_void_p(out.data_ptr()), stream)
    assert rc == _capi.MBX_ERR_INVALID_ARG
    # coefficient power other than 1 or 2
    rc = lib.mbx_sparse_back_project_noalloc(*args, ctypes.c_void_p(idx.data_ptr()), int(idx.shape[0]), None,
                                             g.num_views, 3, 1.0, ctypes.c_void_p(out.data_ptr()), stream)
    assert rc == _capi.MBX_ERR_UNSUPPORTED
    # more views than the geometry has, without a view list
    rc = lib.mbx_sparse_back_project_noalloc(*args, ctypes.c_void_p(idx.data_ptr()), int(idx.shape[0]), None,
                                             g.num_views + 1, 1, 1.0, ctypes.c_void_p(out.data_ptr()), stream)
    assert rc == _capi.MBX_ERR_INVALID_ARG
    torch.cuda.synchronize()
    assert bool(torch.all(out == 7.0))


def test_noalloc_scratch_covers_the_largest_split_on_this_gpu(cuda):
    """The back projector splits views over CTAs only while its pixel-by-slice-tile grid is under a few waves of
    the device, so the split scratch has a ceiling (about 2 x 4 x SMs x 128 x 16 floats, 9.7 MB on 148 SMs).
    Over a sweep of pixel counts around the split thresholds no call needs more than the static array, and the
    sweep's largest parallel-beam request runs through the allocation-free entry point and matches the workspace
    version.  (A request above MBX_NOALLOC_SCRATCH_BYTES would return MBX_ERR_WORKSPACE before any launch; no
    geometry reaches it on this GPU.)"""
    lib = _capi.load_library()
    worst = {}
    for kind in ('parallel', 'cone'):
        for rows in (8, 16, 40, 64):
            model, geom = make_case(kind, views=64, rows=rows, channels=48)
            g = model._geometry()
            for n in range(64, 76000, 997):
                need = lib.mbx_back_project_workspace_bytes(ctypes.byref(g), n, 4096)
                assert need <= _capi.MBX_NOALLOC_SCRATCH_BYTES, (kind, rows, n, need)
                if kind == 'parallel' and need > worst.get('need', 0):
                    worst = dict(need=need, rows=rows, n=n)
    assert worst['need'] > 0
    model, geom = make_case('parallel', views=64, rows=worst['rows'], channels=48)
    g = model._geometry()
    nr, nc, ns = geom.recon_shape
    rng = np.random.default_rng(6)
    idx = torch.as_tensor(rng.integers(0, nr * nc, worst['n']).astype(np.int32), device='cuda')
    views = torch.as_tensor(np.arange(4096) % 64, dtype=torch.int32, device='cuda')
    sino = torch.as_tensor(rng.standard_normal(geom.sinogram_shape).astype(np.float32), device='cuda')
    ref = _capi.back_project(g, sino, idx, view_indices=views)
    got = _capi.back_project_noalloc(g, sino, idx, view_indices=views)
    torch.cuda.synchronize()
    assert rel_l2(got.cpu().numpy(), ref.cpu().numpy()) <= 1e-6

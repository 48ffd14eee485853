"""ctypes binding of the mbirjax_b200 C ABI (``include/mbirjax_b200.h``).

The shared library ``mbirjax_b200/_lib/libmbirjax_b200.so`` is built in-tree by ``mbirjax_b200.build``
(``make -C mbirjax_b200/csrc``).  Device buffers are torch CUDA tensors; only their raw pointers and the
current torch stream cross the boundary.  There is no CPU fallback: if the library or a GPU is missing,
every compute call raises.
"""
import ctypes
import os

import torch

_LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), '_lib', 'libmbirjax_b200.so')

MBX_GEOM_PARALLEL = 0
MBX_GEOM_CONE = 1
MBX_GEOM_TRANSLATION = 2
MBX_MAX_PSF_RADIUS = 4
MBX_OK, MBX_ERR_INVALID_ARG, MBX_ERR_UNSUPPORTED, MBX_ERR_CUDA, MBX_ERR_WORKSPACE = 0, -1, -2, -3, -4
MBX_NOALLOC_SCRATCH_BYTES = 16 << 20

c_int32, c_int64, c_float, c_size_t, c_void_p = (ctypes.c_int32, ctypes.c_int64, ctypes.c_float, ctypes.c_size_t,
                                                 ctypes.c_void_p)


class MbxGeom(ctypes.Structure):
    """Mirror of ``mbx_geom``."""
    _fields_ = [('kind', c_int32), ('num_views', c_int32), ('num_det_rows', c_int32), ('num_det_channels', c_int32),
                ('num_recon_rows', c_int32), ('num_recon_cols', c_int32), ('num_recon_slices', c_int32),
                ('psf_radius', c_int32), ('bp_psf_radius', c_int32), ('entries_per_cylinder_batch', c_int32),
                ('delta_det_channel', c_float), ('delta_det_row', c_float), ('det_channel_offset', c_float),
                ('det_row_offset', c_float), ('delta_voxel', c_float), ('recon_slice_offset', c_float),
                ('source_detector_dist', c_float), ('magnification', c_float), ('angles', c_void_p),
                ('delta_recon_row', c_float), ('translations', c_void_p), ('max_magnification', c_float)]


class MbxQggmrfParams(ctypes.Structure):
    """Mirror of ``mbx_qggmrf_params``."""
    _fields_ = [('b', c_float * 6), ('sigma_x', c_float), ('p', c_float), ('q', c_float), ('T', c_float)]


class MbxScan(ctypes.Structure):
    """Mirror of ``mbx_scan``."""
    _fields_ = [('geom', MbxGeom), ('flat_recon', c_void_p), ('error_sinogram', c_void_p), ('weights', c_void_p),
                ('fm_hessian', c_void_p), ('partition', c_void_p), ('partition_order', c_void_p),
                ('num_subsets', c_int32), ('subset_size', c_int32), ('fm_constant', c_float),
                ('qp', MbxQggmrfParams), ('sinogram', c_void_p), ('full_indices', c_void_p),
                ('num_full_indices', c_int32)]


class MbxBatchedPlan(ctypes.Structure):
    """Mirror of ``mbx_batched_plan`` (opaque)."""
    _fields_ = [('opaque', ctypes.c_uint64 * 128)]


# name -> (restype, argtypes); must match include/mbirjax_b200.h
_SIGNATURES = {
    'mbx_version': (ctypes.c_char_p, []),
    'mbx_error_string': (ctypes.c_char_p, [ctypes.c_int]),
    'mbx_last_cuda_error': (ctypes.c_int, []),
    'mbx_get_device_error': (ctypes.c_int, [ctypes.POINTER(ctypes.c_int)]),
    'mbx_launch_count': (ctypes.c_uint64, []),
    'mbx_set_autotune': (ctypes.c_int, [ctypes.c_int]),
    'mbx_forward_project_workspace_bytes': (c_size_t, [ctypes.POINTER(MbxGeom), c_int64, c_int32]),
    'mbx_sparse_forward_project': (ctypes.c_int, [ctypes.POINTER(MbxGeom), c_void_p, c_void_p, c_int64, c_void_p,
                                                  c_int32, c_void_p, c_void_p, c_size_t, c_void_p]),
    'mbx_back_project_workspace_bytes': (c_size_t, [ctypes.POINTER(MbxGeom), c_int64, c_int32]),
    'mbx_sparse_back_project': (ctypes.c_int, [ctypes.POINTER(MbxGeom), c_void_p, c_void_p, c_void_p, c_int64,
                                               c_void_p, c_int32, c_int32, c_float, c_void_p, c_void_p, c_size_t,
                                               c_void_p]),
    'mbx_sparse_back_project_noalloc': (ctypes.c_int, [ctypes.POINTER(MbxGeom), c_void_p, c_void_p, c_void_p,
                                                       c_int64, c_void_p, c_int32, c_int32, c_float, c_void_p,
                                                       c_void_p]),
    'mbx_qggmrf_grad_hess': (ctypes.c_int, [c_void_p, c_int32, c_int32, c_int32, c_void_p, c_int64,
                                            ctypes.POINTER(MbxQggmrfParams), c_void_p, c_void_p, c_void_p]),
    'mbx_qggmrf_loss_grad_workspace_bytes': (c_size_t, [c_int32, c_int32, c_int32]),
    'mbx_qggmrf_loss_grad': (ctypes.c_int, [c_void_p, c_int32, c_int32, c_int32, ctypes.POINTER(MbxQggmrfParams),
                                            c_void_p, c_void_p, c_void_p, c_size_t, c_void_p]),
    'mbx_vcd_subset_step_workspace_bytes': (c_size_t, [ctypes.POINTER(MbxGeom), c_int64]),
    'mbx_vcd_subset_step': (ctypes.c_int, [ctypes.POINTER(MbxGeom), c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
                                           c_int64, c_float, ctypes.POINTER(MbxQggmrfParams), c_void_p, c_void_p,
                                           c_size_t, c_void_p]),
    'mbx_vcd_subset_step_ex': (ctypes.c_int, [ctypes.POINTER(MbxGeom), c_void_p, c_void_p, c_void_p, c_void_p,
                                              c_void_p, c_int64, c_float, ctypes.POINTER(MbxQggmrfParams), c_void_p,
                                              c_float, c_int32, c_void_p, c_void_p, c_size_t, c_void_p]),
    'mbx_qggmrf_denoise_step_workspace_bytes': (c_size_t, [c_int64, c_int32]),
    'mbx_qggmrf_denoise_step': (ctypes.c_int, [c_void_p, c_void_p, c_int32, c_int32, c_int32, c_void_p, c_int64,
                                               c_float, ctypes.POINTER(MbxQggmrfParams), c_void_p, c_void_p,
                                               c_size_t, c_void_p]),
    'mbx_median_filter3d': (ctypes.c_int, [c_void_p, c_int32, c_int32, c_int32, c_void_p, c_void_p]),
    'mbx_vcd_batched_workspace_bytes': (c_size_t, [ctypes.POINTER(MbxScan), c_int32, c_int32]),
    'mbx_vcd_batched_workspace_bytes2': (c_size_t, [ctypes.POINTER(MbxScan), c_int32, c_int32, c_int32]),
    'mbx_vcd_batched_prepare2': (ctypes.c_int, [ctypes.POINTER(MbxScan), c_int32, c_void_p, c_int32, c_int32,
                                                c_void_p, c_void_p, c_void_p, c_size_t, c_int32,
                                                ctypes.POINTER(MbxBatchedPlan), c_void_p]),
    'mbx_vcd_batched_prepare': (ctypes.c_int, [ctypes.POINTER(MbxScan), c_int32, c_void_p, c_int32, c_int32,
                                               c_void_p, c_void_p, c_void_p, c_size_t,
                                               ctypes.POINTER(MbxBatchedPlan), c_void_p]),
    'mbx_vcd_batched_step': (ctypes.c_int, [ctypes.POINTER(MbxBatchedPlan), c_int32, c_void_p]),
    'mbx_vcd_batched_iteration_stats': (ctypes.c_int, [ctypes.POINTER(MbxBatchedPlan), c_int32, c_void_p]),
    'mbx_vcd_batched_stage': (ctypes.c_int, [ctypes.POINTER(MbxBatchedPlan), c_int32, c_int32, c_void_p]),
    'mbx_vcd_batched_setup': (ctypes.c_int, [ctypes.POINTER(MbxBatchedPlan), c_void_p]),
    'mbx_vcd_batched_update': (ctypes.c_int, [ctypes.POINTER(MbxBatchedPlan), ctypes.POINTER(MbxScan), c_int32,
                                              c_void_p, c_void_p]),
    'mbx_vcd_batched_refresh': (ctypes.c_int, [ctypes.POINTER(MbxBatchedPlan), c_void_p]),
    'mbx_direct_filter': (ctypes.c_int, [ctypes.POINTER(MbxGeom), c_void_p, c_void_p, c_void_p]),
}

_lib = None


class MbxError(RuntimeError):
    pass


def lib_path():
    return _LIB_PATH


def load_library():
    """Load the CUDA library (raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(_LIB_PATH):
        raise MbxError('mbirjax_b200 CUDA library not found at %s; run mbirjax_b200.build()' % _LIB_PATH)
    lib = ctypes.CDLL(_LIB_PATH)
    for name, (restype, argtypes) in _SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = restype
        fn.argtypes = argtypes
    _lib = lib
    return lib


def exported_symbols():
    return list(_SIGNATURES)


def _check(rc, what):
    if rc != 0:
        lib = load_library()
        msg = lib.mbx_error_string(rc).decode()
        if rc == -3:
            msg += ' (cudaError %d)' % lib.mbx_last_cuda_error()
        raise MbxError('%s failed: %s [%d]' % (what, msg, rc))


def _require_cuda(*tensors):
    for t in tensors:
        if t is None:
            continue
        if not t.is_cuda:
            raise MbxError('mbirjax_b200 kernels need CUDA tensors (got a %s tensor)' % t.device)
        if not t.is_contiguous():
            raise MbxError('mbirjax_b200 kernels need contiguous tensors')


def _ptr(t):
    return None if t is None else ctypes.c_void_p(t.data_ptr())


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _workspace(nbytes, device):
    if nbytes == 0:
        return None, 0
    return torch.empty(int(nbytes), dtype=torch.uint8, device=device), int(nbytes)


def version():
    return load_library().mbx_version().decode()


def set_autotune(mode):
    """0: default projector plans; 1 (default): time the candidate plans once per call shape and keep the
    fastest; k >= 2: always candidate k-1 (a test hook).  Returns the previous mode."""
    old = load_library().mbx_set_autotune(int(mode))
    if old < 0:
        raise ValueError('mode must be >= 0')
    return old


def get_device_error():
    flags = ctypes.c_int(0)
    _check(load_library().mbx_get_device_error(ctypes.byref(flags)), 'mbx_get_device_error')
    return flags.value


def forward_project(geom, voxel_values, pixel_indices, view_indices=None, out=None):
    """voxel_values (N, S) float32, pixel_indices (N,) int32 -> sinogram (len(view_indices) or V, R, C)."""
    lib = load_library()
    _require_cuda(voxel_values, pixel_indices, view_indices)
    n = int(pixel_indices.shape[0])
    nv = int(view_indices.shape[0]) if view_indices is not None else geom.num_views
    if out is None:
        out = torch.empty((nv, geom.num_det_rows, geom.num_det_channels), dtype=torch.float32,
                          device=voxel_values.device)
    nbytes = lib.mbx_forward_project_workspace_bytes(ctypes.byref(geom), n, nv)
    ws, nbytes = _workspace(nbytes, voxel_values.device)
    rc = lib.mbx_sparse_forward_project(ctypes.byref(geom), _ptr(voxel_values), _ptr(pixel_indices), n,
                                        _ptr(view_indices), nv, _ptr(out), _ptr(ws), nbytes, _stream())
    _check(rc, 'mbx_sparse_forward_project')
    return out


def back_project(geom, sinogram, pixel_indices, view_indices=None, coeff_power=1, weights=None, scale=1.0, out=None):
    """Full sinogram (V, R, C) -> (N, S) at pixel_indices.  sinogram None: back-projects the weights, or ones when
    weights is None too (the unit-weight Hessian diagonal with coeff_power=2, with no buffer of ones)."""
    lib = load_library()
    _require_cuda(sinogram, pixel_indices, view_indices, weights)
    n = int(pixel_indices.shape[0])
    nv = int(view_indices.shape[0]) if view_indices is not None else geom.num_views
    if out is None:
        out = torch.empty((n, geom.num_recon_slices), dtype=torch.float32, device=pixel_indices.device)
    nbytes = lib.mbx_back_project_workspace_bytes(ctypes.byref(geom), n, nv)
    ws, nbytes = _workspace(nbytes, pixel_indices.device)
    rc = lib.mbx_sparse_back_project(ctypes.byref(geom), _ptr(sinogram), _ptr(weights), _ptr(pixel_indices), n,
                                     _ptr(view_indices), nv, int(coeff_power), float(scale), _ptr(out), _ptr(ws),
                                     nbytes, _stream())
    _check(rc, 'mbx_sparse_back_project')
    return out


def back_project_noalloc(geom, sinogram, pixel_indices, view_indices=None, coeff_power=1, weights=None, scale=1.0,
                         out=None):
    """Same result as back_project, through the entry point that allocates nothing: its scratch is a static
    device array inside the library (for callers that cannot allocate GPU memory at call time).  Calls whose GPU
    work overlaps share that array and must not run concurrently."""
    lib = load_library()
    _require_cuda(sinogram, pixel_indices, view_indices, weights)
    n = int(pixel_indices.shape[0])
    nv = int(view_indices.shape[0]) if view_indices is not None else geom.num_views
    if out is None:
        out = torch.empty((n, geom.num_recon_slices), dtype=torch.float32, device=pixel_indices.device)
    rc = lib.mbx_sparse_back_project_noalloc(ctypes.byref(geom), _ptr(sinogram), _ptr(weights), _ptr(pixel_indices),
                                             n, _ptr(view_indices), nv, int(coeff_power), float(scale), _ptr(out),
                                             _stream())
    _check(rc, 'mbx_sparse_back_project_noalloc')
    return out


def qggmrf_params(b, sigma_x, p, q, T):
    qp = MbxQggmrfParams()
    for i in range(6):
        qp.b[i] = float(b[i])
    qp.sigma_x, qp.p, qp.q, qp.T = float(sigma_x), float(p), float(q), float(T)
    return qp


def qggmrf_grad_hess(flat_recon, recon_shape, pixel_indices, qp):
    lib = load_library()
    _require_cuda(flat_recon, pixel_indices)
    n = int(pixel_indices.shape[0])
    ns = int(recon_shape[2])
    grad = torch.empty((n, ns), dtype=torch.float32, device=flat_recon.device)
    hess = torch.empty_like(grad)
    rc = lib.mbx_qggmrf_grad_hess(_ptr(flat_recon), int(recon_shape[0]), int(recon_shape[1]), ns,
                                  _ptr(pixel_indices), n, ctypes.byref(qp), _ptr(grad), _ptr(hess), _stream())
    _check(rc, 'mbx_qggmrf_grad_hess')
    return grad, hess


def qggmrf_loss_grad(recon, qp, need_grad=True):
    """recon (Nr, Nc, S) float32 -> (loss as a device float64 scalar tensor, gradient or None)."""
    lib = load_library()
    _require_cuda(recon)
    nr, nc, ns = (int(v) for v in recon.shape)
    loss = torch.empty((), dtype=torch.float64, device=recon.device)
    grad = torch.empty_like(recon) if need_grad else None
    nbytes = lib.mbx_qggmrf_loss_grad_workspace_bytes(nr, nc, ns)
    ws, nbytes = _workspace(nbytes, recon.device)
    rc = lib.mbx_qggmrf_loss_grad(_ptr(recon), nr, nc, ns, ctypes.byref(qp), _ptr(loss), _ptr(grad), _ptr(ws), nbytes,
                                  _stream())
    _check(rc, 'mbx_qggmrf_loss_grad')
    return loss, grad


def vcd_subset_step_workspace(geom, num_pixels, device):
    nbytes = load_library().mbx_vcd_subset_step_workspace_bytes(ctypes.byref(geom), int(num_pixels))
    return _workspace(nbytes, device)


def vcd_subset_step(geom, flat_recon, error_sinogram, weights, fm_hessian, pixel_indices, fm_constant, qp, stats,
                    workspace=None, prox_input=None, sigma_prox=0.0, positivity=False):
    """One device-resident VCD subset update; stats is a device float64 tensor with >= 4 entries.  prox_input
    (flat like flat_recon) selects the proximal-map prior, positivity the clip of the reference's updater."""
    lib = load_library()
    _require_cuda(flat_recon, error_sinogram, weights, fm_hessian, pixel_indices, stats, prox_input)
    n = int(pixel_indices.shape[0])
    if workspace is None:
        workspace = vcd_subset_step_workspace(geom, n, flat_recon.device)
    ws, nbytes = workspace
    if prox_input is None and not positivity:
        rc = lib.mbx_vcd_subset_step(ctypes.byref(geom), _ptr(flat_recon), _ptr(error_sinogram), _ptr(weights),
                                     _ptr(fm_hessian), _ptr(pixel_indices), n, float(fm_constant), ctypes.byref(qp),
                                     _ptr(stats), _ptr(ws), nbytes, _stream())
        _check(rc, 'mbx_vcd_subset_step')
        return
    rc = lib.mbx_vcd_subset_step_ex(ctypes.byref(geom), _ptr(flat_recon), _ptr(error_sinogram), _ptr(weights),
                                    _ptr(fm_hessian), _ptr(pixel_indices), n, float(fm_constant), ctypes.byref(qp),
                                    _ptr(prox_input), float(sigma_prox), 1 if positivity else 0, _ptr(stats),
                                    _ptr(ws), nbytes, _stream())
    _check(rc, 'mbx_vcd_subset_step_ex')


def qggmrf_denoise_step(flat_image, flat_error_image, image_shape, pixel_indices, fm_constant, qp, stats,
                        workspace=None):
    """One subset update of the qGGMRF denoiser on flat (Nr*Nc, S) device images."""
    lib = load_library()
    _require_cuda(flat_image, flat_error_image, pixel_indices, stats)
    nr, nc, ns = (int(v) for v in image_shape)
    n = int(pixel_indices.shape[0])
    if workspace is None:
        workspace = _workspace(lib.mbx_qggmrf_denoise_step_workspace_bytes(n, ns), flat_image.device)
    ws, nbytes = workspace
    rc = lib.mbx_qggmrf_denoise_step(_ptr(flat_image), _ptr(flat_error_image), nr, nc, ns, _ptr(pixel_indices), n,
                                     float(fm_constant), ctypes.byref(qp), _ptr(stats), _ptr(ws), nbytes, _stream())
    _check(rc, 'mbx_qggmrf_denoise_step')


def median_filter3d(x, out=None):
    """3x3x3 median with edge replication of a float32 (d0, d1, d2) device volume."""
    lib = load_library()
    _require_cuda(x)
    if x.dim() != 3:
        raise ValueError('median_filter3d needs a 3-D array')
    if out is None:
        out = torch.empty_like(x)
    rc = lib.mbx_median_filter3d(_ptr(x), *(int(v) for v in x.shape), _ptr(out), _stream())
    _check(rc, 'mbx_median_filter3d')
    return out


def direct_filter(geom, sinogram, out=None):
    lib = load_library()
    _require_cuda(sinogram)
    if out is None:
        out = torch.empty_like(sinogram)
    _check(lib.mbx_direct_filter(ctypes.byref(geom), _ptr(sinogram), _ptr(out), _stream()), 'mbx_direct_filter')
    return out


MBX_BATCHED_PLAN_FORWARD = 1


def vcd_batched_workspace_bytes(scans, num_steps, flags=0):
    n = len(scans)
    arr = (MbxScan * n)(*scans)
    return int(load_library().mbx_vcd_batched_workspace_bytes2(arr, n, int(num_steps), int(flags)))


def vcd_batched_prepare(scans, schedule, num_iterations, step_stats, iter_stats, device, flags=0):
    """scans: list of MbxScan; schedule: int32 numpy (num_steps, num_scans); flags: MBX_BATCHED_PLAN_FORWARD or 0.
    Returns (plan, workspace)."""
    import numpy as np
    lib = load_library()
    n = len(scans)
    arr = (MbxScan * n)(*scans)
    sched = np.ascontiguousarray(schedule, dtype=np.int32)
    num_steps = int(sched.shape[0])
    nbytes = lib.mbx_vcd_batched_workspace_bytes2(arr, n, num_steps, int(flags))
    if nbytes == 0:
        raise MbxError('mbx_vcd_batched_workspace_bytes: batch not supported (mixed geometry kinds, psf radius '
                       'other than 1, or invalid scans)')
    ws = torch.empty(int(nbytes), dtype=torch.uint8, device=device)
    plan = MbxBatchedPlan()
    rc = lib.mbx_vcd_batched_prepare2(arr, n, sched.ctypes.data_as(c_void_p), num_steps, int(num_iterations),
                                      _ptr(step_stats), _ptr(iter_stats), _ptr(ws), int(nbytes), int(flags),
                                      ctypes.byref(plan), _stream())
    _check(rc, 'mbx_vcd_batched_prepare')
    return plan, ws


def vcd_batched_step(plan, step):
    _check(load_library().mbx_vcd_batched_step(ctypes.byref(plan), int(step), _stream()), 'mbx_vcd_batched_step')


def vcd_batched_iteration_stats(plan, iteration):
    _check(load_library().mbx_vcd_batched_iteration_stats(ctypes.byref(plan), int(iteration), _stream()),
           'mbx_vcd_batched_iteration_stats')


def vcd_batched_setup(plan):
    _check(load_library().mbx_vcd_batched_setup(ctypes.byref(plan), _stream()), 'mbx_vcd_batched_setup')


def vcd_batched_update(plan, scans, schedule):
    """New fm constants / qGGMRF parameters (read from the MbxScan records) and subset schedule of a prepared
    batch, copied to its device tables on the current stream."""
    import numpy as np
    n = len(scans)
    arr = (MbxScan * n)(*scans)
    sched = np.ascontiguousarray(schedule, dtype=np.int32)
    _check(load_library().mbx_vcd_batched_update(ctypes.byref(plan), arr, n, sched.ctypes.data_as(c_void_p),
                                                  _stream()), 'mbx_vcd_batched_update')


def vcd_batched_refresh(plan):
    _check(load_library().mbx_vcd_batched_refresh(ctypes.byref(plan), _stream()), 'mbx_vcd_batched_refresh')


BATCHED_STAGES = ('bp', 'delta', 'fp', 'linquad', 'alpha', 'apply', 'error', 'l1')


def vcd_batched_stage(plan, step, stage):
    _check(load_library().mbx_vcd_batched_stage(ctypes.byref(plan), int(step), int(stage), _stream()),
           'mbx_vcd_batched_stage')

// PyTorch dispatcher operators over the mbirjax_b200 C ABI (include/mbirjax_b200.h).
//
// Each operator checks dtype, contiguity and device of its tensors (TORCH_CHECK raises a Python error), allocates
// its outputs and workspace with the caching allocator, and calls the C entry point on the current CUDA stream
// (at::cuda::getCurrentCUDAStream()), so the ops compose with torch streams, CUDA graphs and torch.compile
// tracing like any other op.  They are registered for the CUDA dispatch key only: there is no CPU kernel, so a
// call with host tensors fails in the dispatcher.  The C ABI stays the boundary a non-Python caller binds (the
// ctypes layer in mbirjax_b200/_capi.py binds it directly).
//
// Geometry: the mbx_geom record is passed as two scalar lists and the per-view parameter tensor,
//   geom_ints   = [kind, num_views, num_det_rows, num_det_channels, num_recon_rows, num_recon_cols,
//                  num_recon_slices, psf_radius, bp_psf_radius, entries_per_cylinder_batch]
//   geom_floats = [delta_det_channel, delta_det_row, det_channel_offset, det_row_offset, delta_voxel,
//                  recon_slice_offset, source_detector_dist, magnification, delta_recon_row, max_magnification]
//   view_params = angles (num_views,) or translations (num_views, 3), float32 on the device;
// qGGMRF parameters as qparams = [b0..b5, sigma_x, p, q, T].
#include <ATen/ATen.h>
#include <ATen/cuda/CUDAContext.h>
#include <c10/cuda/CUDAGuard.h>
#include <torch/library.h>

#include "../../include/mbirjax_b200.h"

namespace {

void check_rc(int rc, const char *what) {
    TORCH_CHECK(rc == MBX_OK, what, " failed: ", mbx_error_string(rc), " [", rc, "]",
                rc == MBX_ERR_CUDA ? " (cudaError " + std::to_string(mbx_last_cuda_error()) + ")" : std::string());
}

void check_tensor(const at::Tensor &t, at::ScalarType dtype, const char *name, const at::Device &dev) {
    TORCH_CHECK(t.is_cuda(), name, " must be a CUDA tensor");
    TORCH_CHECK(t.device() == dev, name, " must be on ", dev, " (got ", t.device(), ")");
    TORCH_CHECK(t.scalar_type() == dtype, name, " must be ", dtype, " (got ", t.scalar_type(), ")");
    TORCH_CHECK(t.is_contiguous(), name, " must be contiguous");
}

void check_opt(const c10::optional<at::Tensor> &t, at::ScalarType dtype, const char *name, const at::Device &dev) {
    if (t.has_value() && t->defined()) check_tensor(*t, dtype, name, dev);
}

template <class T>
const T *opt_ptr(const c10::optional<at::Tensor> &t) {
    return (t.has_value() && t->defined()) ? t->data_ptr<T>() : nullptr;
}

mbx_geom make_geom(at::IntArrayRef gi, at::ArrayRef<double> gf, const at::Tensor &view_params, const at::Device &dev) {
    TORCH_CHECK(gi.size() == 10, "geom_ints must hold 10 values");
    TORCH_CHECK(gf.size() == 10, "geom_floats must hold 10 values");
    check_tensor(view_params, at::kFloat, "view_params", dev);
    mbx_geom g{};
    g.kind = (int32_t)gi[0];
    g.num_views = (int32_t)gi[1];
    g.num_det_rows = (int32_t)gi[2];
    g.num_det_channels = (int32_t)gi[3];
    g.num_recon_rows = (int32_t)gi[4];
    g.num_recon_cols = (int32_t)gi[5];
    g.num_recon_slices = (int32_t)gi[6];
    g.psf_radius = (int32_t)gi[7];
    g.bp_psf_radius = (int32_t)gi[8];
    g.entries_per_cylinder_batch = (int32_t)gi[9];
    g.delta_det_channel = (float)gf[0];
    g.delta_det_row = (float)gf[1];
    g.det_channel_offset = (float)gf[2];
    g.det_row_offset = (float)gf[3];
    g.delta_voxel = (float)gf[4];
    g.recon_slice_offset = (float)gf[5];
    g.source_detector_dist = (float)gf[6];
    g.magnification = (float)gf[7];
    g.delta_recon_row = (float)gf[8];
    g.max_magnification = (float)gf[9];
    const int64_t per_view = g.kind == MBX_GEOM_TRANSLATION ? 3 : 1;
    TORCH_CHECK(view_params.numel() == per_view * g.num_views, "view_params must hold ", per_view,
                " value(s) per view");
    if (g.kind == MBX_GEOM_TRANSLATION)
        g.translations = view_params.data_ptr<float>();
    else
        g.angles = view_params.data_ptr<float>();
    return g;
}

mbx_qggmrf_params make_qparams(at::ArrayRef<double> q) {
    TORCH_CHECK(q.size() == 10, "qparams must hold b[6], sigma_x, p, q, T");
    mbx_qggmrf_params p{};
    for (int i = 0; i < 6; ++i) p.b[i] = (float)q[i];
    p.sigma_x = (float)q[6];
    p.p = (float)q[7];
    p.q = (float)q[8];
    p.T = (float)q[9];
    return p;
}

at::Tensor workspace(size_t bytes, const at::Tensor &like) {
    return at::empty({(int64_t)std::max<size_t>(bytes, 1)}, like.options().dtype(at::kByte));
}

void *stream() { return at::cuda::getCurrentCUDAStream().stream(); }

at::Tensor sparse_forward_project(at::IntArrayRef gi, at::ArrayRef<double> gf, const at::Tensor &view_params,
                                  const at::Tensor &voxel_values, const at::Tensor &pixel_indices,
                                  const c10::optional<at::Tensor> &view_indices) {
    const at::Device dev = voxel_values.device();
    c10::cuda::CUDAGuard guard(dev);
    check_tensor(voxel_values, at::kFloat, "voxel_values", dev);
    check_tensor(pixel_indices, at::kInt, "pixel_indices", dev);
    check_opt(view_indices, at::kInt, "view_indices", dev);
    const mbx_geom g = make_geom(gi, gf, view_params, dev);
    const int64_t n = pixel_indices.numel();
    TORCH_CHECK(voxel_values.dim() == 2 && voxel_values.size(0) == n && voxel_values.size(1) == g.num_recon_slices,
                "voxel_values must have shape (num_pixels, num_recon_slices)");
    const int32_t nv = view_indices.has_value() ? (int32_t)view_indices->numel() : g.num_views;
    auto out = at::empty({nv, g.num_det_rows, g.num_det_channels}, voxel_values.options());
    const size_t wb = mbx_forward_project_workspace_bytes(&g, n, nv);
    auto ws = workspace(wb, voxel_values);
    check_rc(mbx_sparse_forward_project(&g, voxel_values.data_ptr<float>(), pixel_indices.data_ptr<int32_t>(), n,
                                        opt_ptr<int32_t>(view_indices), nv, out.data_ptr<float>(),
                                        wb ? ws.data_ptr() : nullptr, wb, stream()),
             "mbx_sparse_forward_project");
    return out;
}

at::Tensor sparse_back_project(at::IntArrayRef gi, at::ArrayRef<double> gf, const at::Tensor &view_params,
                               const c10::optional<at::Tensor> &sinogram, const at::Tensor &pixel_indices,
                               const c10::optional<at::Tensor> &view_indices, int64_t coeff_power,
                               const c10::optional<at::Tensor> &weights, double scale) {
    const at::Device dev = pixel_indices.device();
    c10::cuda::CUDAGuard guard(dev);
    check_tensor(pixel_indices, at::kInt, "pixel_indices", dev);
    check_opt(sinogram, at::kFloat, "sinogram", dev);
    check_opt(weights, at::kFloat, "weights", dev);
    check_opt(view_indices, at::kInt, "view_indices", dev);
    const mbx_geom g = make_geom(gi, gf, view_params, dev);
    const int64_t sino_elems = (int64_t)g.num_views * g.num_det_rows * g.num_det_channels;
    if (sinogram.has_value()) TORCH_CHECK(sinogram->numel() == sino_elems, "sinogram must have the geometry's shape");
    if (weights.has_value()) TORCH_CHECK(weights->numel() == sino_elems, "weights must have the geometry's shape");
    const int64_t n = pixel_indices.numel();
    const int32_t nv = view_indices.has_value() ? (int32_t)view_indices->numel() : g.num_views;
    auto out = at::empty({n, g.num_recon_slices}, pixel_indices.options().dtype(at::kFloat));
    const size_t wb = mbx_back_project_workspace_bytes(&g, n, nv);
    auto ws = workspace(wb, out);
    check_rc(mbx_sparse_back_project(&g, opt_ptr<float>(sinogram), opt_ptr<float>(weights),
                                     pixel_indices.data_ptr<int32_t>(), n, opt_ptr<int32_t>(view_indices), nv,
                                     (int32_t)coeff_power, (float)scale, out.data_ptr<float>(),
                                     wb ? ws.data_ptr() : nullptr, wb, stream()),
             "mbx_sparse_back_project");
    return out;
}

at::Tensor direct_filter(at::IntArrayRef gi, at::ArrayRef<double> gf, const at::Tensor &view_params,
                         const at::Tensor &sinogram) {
    const at::Device dev = sinogram.device();
    c10::cuda::CUDAGuard guard(dev);
    check_tensor(sinogram, at::kFloat, "sinogram", dev);
    const mbx_geom g = make_geom(gi, gf, view_params, dev);
    TORCH_CHECK(sinogram.numel() == (int64_t)g.num_views * g.num_det_rows * g.num_det_channels,
                "sinogram must have the geometry's shape");
    auto out = at::empty_like(sinogram);
    check_rc(mbx_direct_filter(&g, sinogram.data_ptr<float>(), out.data_ptr<float>(), stream()), "mbx_direct_filter");
    return out;
}

std::tuple<at::Tensor, at::Tensor> qggmrf_grad_hess(const at::Tensor &flat_recon, at::IntArrayRef recon_shape,
                                                    const at::Tensor &pixel_indices, at::ArrayRef<double> qparams) {
    const at::Device dev = flat_recon.device();
    c10::cuda::CUDAGuard guard(dev);
    check_tensor(flat_recon, at::kFloat, "flat_recon", dev);
    check_tensor(pixel_indices, at::kInt, "pixel_indices", dev);
    TORCH_CHECK(recon_shape.size() == 3, "recon_shape must be (rows, cols, slices)");
    TORCH_CHECK(flat_recon.numel() == recon_shape[0] * recon_shape[1] * recon_shape[2],
                "flat_recon must hold recon_shape voxels");
    const mbx_qggmrf_params qp = make_qparams(qparams);
    const int64_t n = pixel_indices.numel();
    auto grad = at::empty({n, recon_shape[2]}, flat_recon.options());
    auto hess = at::empty({n, recon_shape[2]}, flat_recon.options());
    check_rc(mbx_qggmrf_grad_hess(flat_recon.data_ptr<float>(), (int32_t)recon_shape[0], (int32_t)recon_shape[1],
                                  (int32_t)recon_shape[2], pixel_indices.data_ptr<int32_t>(), n, &qp,
                                  grad.data_ptr<float>(), hess.data_ptr<float>(), stream()),
             "mbx_qggmrf_grad_hess");
    return {grad, hess};
}

std::tuple<at::Tensor, at::Tensor> qggmrf_loss_grad(const at::Tensor &recon, at::ArrayRef<double> qparams) {
    const at::Device dev = recon.device();
    c10::cuda::CUDAGuard guard(dev);
    check_tensor(recon, at::kFloat, "recon", dev);
    TORCH_CHECK(recon.dim() == 3, "recon must be (rows, cols, slices)");
    const mbx_qggmrf_params qp = make_qparams(qparams);
    auto loss = at::empty({}, recon.options().dtype(at::kDouble));
    auto grad = at::empty_like(recon);
    const int32_t r = (int32_t)recon.size(0), c = (int32_t)recon.size(1), s = (int32_t)recon.size(2);
    const size_t wb = mbx_qggmrf_loss_grad_workspace_bytes(r, c, s);
    auto ws = workspace(wb, recon);
    check_rc(mbx_qggmrf_loss_grad(recon.data_ptr<float>(), r, c, s, &qp, loss.data_ptr<double>(),
                                  grad.data_ptr<float>(), wb ? ws.data_ptr() : nullptr, wb, stream()),
             "mbx_qggmrf_loss_grad");
    return {loss, grad};
}

void vcd_subset_step(at::IntArrayRef gi, at::ArrayRef<double> gf, const at::Tensor &view_params,
                     const at::Tensor &flat_recon, const at::Tensor &error_sinogram,
                     const c10::optional<at::Tensor> &weights, const at::Tensor &fm_hessian,
                     const at::Tensor &pixel_indices, double fm_constant, at::ArrayRef<double> qparams,
                     const at::Tensor &stats) {
    const at::Device dev = flat_recon.device();
    c10::cuda::CUDAGuard guard(dev);
    check_tensor(flat_recon, at::kFloat, "flat_recon", dev);
    check_tensor(error_sinogram, at::kFloat, "error_sinogram", dev);
    check_opt(weights, at::kFloat, "weights", dev);
    check_tensor(fm_hessian, at::kFloat, "fm_hessian", dev);
    check_tensor(pixel_indices, at::kInt, "pixel_indices", dev);
    check_tensor(stats, at::kDouble, "stats", dev);
    TORCH_CHECK(stats.numel() >= 4, "stats must hold 4 doubles");
    const mbx_geom g = make_geom(gi, gf, view_params, dev);
    const int64_t nrecon = (int64_t)g.num_recon_rows * g.num_recon_cols * g.num_recon_slices;
    TORCH_CHECK(flat_recon.numel() == nrecon && fm_hessian.numel() == nrecon, "flat_recon / fm_hessian size");
    TORCH_CHECK(error_sinogram.numel() == (int64_t)g.num_views * g.num_det_rows * g.num_det_channels,
                "error_sinogram must have the geometry's shape");
    const mbx_qggmrf_params qp = make_qparams(qparams);
    const int64_t n = pixel_indices.numel();
    const size_t wb = mbx_vcd_subset_step_workspace_bytes(&g, n);
    auto ws = workspace(wb, flat_recon);
    check_rc(mbx_vcd_subset_step(&g, flat_recon.data_ptr<float>(), error_sinogram.data_ptr<float>(),
                                 opt_ptr<float>(weights), fm_hessian.data_ptr<float>(),
                                 pixel_indices.data_ptr<int32_t>(), n, (float)fm_constant, &qp,
                                 stats.data_ptr<double>(), wb ? ws.data_ptr() : nullptr, wb, stream()),
             "mbx_vcd_subset_step");
}

}  // namespace

TORCH_LIBRARY(mbirjax_b200, m) {
    m.def("sparse_forward_project(int[] geom_ints, float[] geom_floats, Tensor view_params, Tensor voxel_values, "
          "Tensor pixel_indices, Tensor? view_indices=None) -> Tensor");
    m.def("sparse_back_project(int[] geom_ints, float[] geom_floats, Tensor view_params, Tensor? sinogram, "
          "Tensor pixel_indices, Tensor? view_indices=None, int coeff_power=1, Tensor? weights=None, "
          "float scale=1.0) -> Tensor");
    m.def("direct_filter(int[] geom_ints, float[] geom_floats, Tensor view_params, Tensor sinogram) -> Tensor");
    m.def("qggmrf_grad_hess(Tensor flat_recon, int[] recon_shape, Tensor pixel_indices, float[] qparams) "
          "-> (Tensor, Tensor)");
    m.def("qggmrf_loss_grad(Tensor recon, float[] qparams) -> (Tensor, Tensor)");
    m.def("vcd_subset_step(int[] geom_ints, float[] geom_floats, Tensor view_params, Tensor(a!) flat_recon, "
          "Tensor(b!) error_sinogram, Tensor? weights, Tensor fm_hessian, Tensor pixel_indices, float fm_constant, "
          "float[] qparams, Tensor(c!) stats) -> ()");
}

TORCH_LIBRARY_IMPL(mbirjax_b200, CUDA, m) {
    m.impl("sparse_forward_project", &sparse_forward_project);
    m.impl("sparse_back_project", &sparse_back_project);
    m.impl("direct_filter", &direct_filter);
    m.impl("qggmrf_grad_hess", &qggmrf_grad_hess);
    m.impl("qggmrf_loss_grad", &qggmrf_loss_grad);
    m.impl("vcd_subset_step", &vcd_subset_step);
}

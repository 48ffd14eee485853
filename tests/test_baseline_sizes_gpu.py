"""GPU parity at the benchmark sizes, against the oracle run on all host cores (``oracle.pool.OraclePool``).

* Plain cone-beam configuration: sinogram 256 views x 128 rows x 256 channels, source_detector_dist =
  source_iso_dist = 1024, recon 256 x 256 x 128 of 20 seeded ellipsoids with 1% noise.  One VCD subset update
  (1 of 4 subsets), the unit-weight Hessian diagonal and the FDK direct recon, each within 1e-5 of the oracle.
* Batched parallel-beam configuration: the 24 uneven scans of the batched benchmark.  The first subset update of
  every scan through the batched stage kernels against the oracle's update from the same state, and full
  10-iteration recons of two scans, the largest among them, by the batched and the plain path, each within 1e-4
  NRMSE of the oracle's recon.
* Differentiable cone-beam configuration (the plain cone geometry and phantom, W = exp(-y / max y)): the autograd
  gradient of 0.5 ||W^(1/2)(A x - y)||^2 + qGGMRF(x) against central differences of the float64 oracle at 64
  voxels (eps = 1e-3), and 100 steps of projected gradient descent.

The oracle's projections are spread over the host's cores by view; the float64 finite differences are evaluated
exactly where the loss changes (see ``test_config2_gradient_matches_central_differences``)."""
import numpy as np
import pytest
import torch

import mbirjax_b200 as mb
from mbirjax_b200 import _capi
from mbirjax_b200 import autograd as AG
from mbirjax_b200.batched import BatchedVCD
from mbirjax_b200.utilities import add_noise, batched_scan_shapes, gen_ellipsoid_phantom, uniform_angles
import oracle as O
from oracle import vcd as OV
from oracle.pool import OraclePool
from cases import oracle_geometry, rel_l2

pytestmark = pytest.mark.gpu

CONE = dict(views=256, rows=128, channels=256, sdd=1024.0, sid=1024.0, ellipsoids=20, seed=1)
QPARAMS = (O.get_b_from_nbr_wts([1, 1, 1]), 2.0, 1.2, 1.0)  # b, p, q, T (sigma_x from the data)


@pytest.fixture(scope='module')
def pool():
    with OraclePool() as p:
        yield p


@pytest.fixture(scope='module')
def cone_case(cuda):
    """The plain cone-beam configuration: model, oracle geometry, phantom (host) and noisy sinogram (host)."""
    ang = np.linspace(0, 2 * np.pi, CONE['views'], endpoint=False).astype(np.float32)
    model = mb.ConeBeamModel((CONE['views'], CONE['rows'], CONE['channels']), ang,
                             source_detector_dist=CONE['sdd'], source_iso_dist=CONE['sid'])
    assert tuple(model.get_params('recon_shape')) == (256, 256, 128)
    geom = oracle_geometry(model)
    ph = gen_ellipsoid_phantom(geom.recon_shape, CONE['ellipsoids'], CONE['seed'], device=cuda)
    np.random.seed(CONE['seed'])
    sino = add_noise(model.forward_project(ph), 0.01, CONE['seed'])
    return model, geom, ph.cpu().numpy(), sino.cpu().numpy()


def test_config1_subset_update_and_hessian_match_oracle(cuda, cone_case, pool):
    model, geom, ph, sino = cone_case
    nr, nc, ns = geom.recon_shape
    rng = np.random.default_rng(0)
    flat = (0.9 * ph + 0.05 * rng.random(ph.shape)).astype(np.float32).reshape(-1, ns)
    np.random.seed(1)
    err = (sino - model.forward_project(flat.reshape(geom.recon_shape)).cpu().numpy()).astype(np.float32)
    hess = model.compute_hessian_diagonal().cpu().numpy()
    assert rel_l2(hess, pool.compute_hessian_diagonal(geom)) <= 1e-5
    hess = hess.reshape(-1, ns)
    sigma_y, sigma_x, _ = OV.auto_regularization(geom, sino, sharpness=0.0)
    params = (QPARAMS[0], sigma_x) + QPARAMS[1:]
    fm = 1.0 / sigma_y ** 2
    np.random.seed(2)
    subset = O.gen_pixel_partition(geom.recon_shape, 4)[0]
    r_ref, e_ref, l1_ref, a_ref = OV.vcd_subset_update(geom, flat, err, None, hess, subset, fm, params, proj=pool)

    dev = torch.device('cuda')
    flat_d = torch.as_tensor(flat, device=dev).contiguous()
    err_d = torch.as_tensor(err, device=dev).contiguous()
    stats = torch.zeros(4, dtype=torch.float64, device=dev)
    _capi.vcd_subset_step(model._geometry(), flat_d, err_d, None, torch.as_tensor(hess, device=dev),
                          torch.as_tensor(subset, device=dev), fm, _capi.qggmrf_params(*params), stats)
    st = stats.cpu().numpy()
    assert st[0] == pytest.approx(a_ref, rel=1e-5)
    assert st[1] == pytest.approx(l1_ref, rel=1e-5)
    assert rel_l2(flat_d.cpu().numpy(), r_ref) <= 1e-6
    assert rel_l2(err_d.cpu().numpy(), e_ref) <= 1e-5


def test_config1_fdk_matches_oracle(cuda, cone_case, pool):
    model, geom, ph, sino = cone_case
    gpu = model.direct_recon(torch.as_tensor(sino, device='cuda')).cpu().numpy()
    np.random.seed(0)
    ref = OV.direct_recon(geom, sino, proj=pool)
    assert rel_l2(gpu, ref) <= 1e-5


def _batched_scans(device, which=None):
    """The scans of the batched benchmark (scan i: seed i; views U{60..720}, rows U{8..64}, channels U{96..512},
    10 ellipsoids, 1% noise), as (models, sinograms on the device)."""
    models, sinos = [], []
    shapes = batched_scan_shapes(24)
    for i in (range(24) if which is None else which):
        v, r, c = shapes[i]
        model = mb.ParallelBeamModel((v, r, c), uniform_angles(v))
        model.set_params(sharpness=0.0, snr_db=30.0, granularity=[4], partition_sequence=[0], verbose=0)
        ph = gen_ellipsoid_phantom(model.get_params('recon_shape'), 10, i, device=device)
        np.random.seed(i)
        sinos.append(add_noise(model.forward_project(ph), 0.01, i).contiguous())
        models.append(model)
    return models, sinos


def _qparams_tuple(qp):
    return np.array(list(qp.b), dtype=np.float32), qp.sigma_x, qp.p, qp.q, qp.T


def test_config3_first_batched_subset_update_of_every_scan_matches_oracle(cuda, pool):
    models, sinos = _batched_scans(cuda)
    b = BatchedVCD(models, sinos, seeds=list(range(24)))
    scans, sched = b._setup(1)
    n = len(scans)
    step_stats = torch.zeros((sched.shape[0], n, 4), dtype=torch.float64, device=cuda)
    iter_stats = torch.zeros((1, n, 4), dtype=torch.float64, device=cuda)
    plan, ws = _capi.vcd_batched_prepare(scans, sched, 1, step_stats, iter_stats, cuda)
    before = [(st['flat_recon'].cpu().numpy(), st['error_sinogram'].cpu().numpy(), st['fm_hessian'].cpu().numpy())
              for st in b.states]
    _capi.vcd_batched_step(plan, 0)
    torch.cuda.synchronize()
    alphas = step_stats[0, :, 0].cpu().numpy()
    for s, (model, state) in enumerate(zip(models, b.states)):
        geom = oracle_geometry(model)
        flat, err, hess = before[s]
        subset = b.partitions[s][sched[0, s]]
        r_ref, e_ref, _, a_ref = OV.vcd_subset_update(geom, flat, err, None, hess, subset, state['fm_constant'],
                                                      _qparams_tuple(state['qp']), proj=pool)
        assert alphas[s] == pytest.approx(a_ref, rel=1e-5), 'scan %d' % s
        assert rel_l2(state['flat_recon'].cpu().numpy(), r_ref) <= 1e-6, 'scan %d' % s
        assert rel_l2(state['error_sinogram'].cpu().numpy(), e_ref) <= 1e-5, 'scan %d' % s
    del plan, ws


def test_config3_two_full_recons_match_oracle(cuda, pool):
    """Scan 13 (652 x 57 x 437, the largest sinogram of the batch) and scan 23 (83 x 47 x 272): 10 iterations of 4
    subsets with FBP initialisation, by the batched path and by the plain path, within 1e-4 NRMSE of the oracle."""
    which = [13, 23]
    models, sinos = _batched_scans(cuda, which)
    batched, _ = BatchedVCD(models, sinos, seeds=which).recon(max_iterations=10)
    for model, sino, seed, rb in zip(models, sinos, which, batched):
        np.random.seed(seed)
        rp, _ = model.recon(sino, max_iterations=10, stop_threshold_change_pct=0, logfile_path=None, print_logs=False)
        geom = oracle_geometry(model)
        np.random.seed(seed)
        ref, _ = OV.recon(geom, sino.cpu().numpy(), granularity=[4], partition_sequence=[0], max_iterations=10,
                          sharpness=0.0, snr_db=30.0, stop_threshold_change_pct=0, proj=pool)
        eb, ep = rel_l2(rb.cpu().numpy(), ref), rel_l2(rp.cpu().numpy(), ref)
        assert eb <= 1e-4, 'batched, scan %d: %.3g' % (seed, eb)
        assert ep <= 1e-4, 'plain, scan %d: %.3g' % (seed, ep)


def _config2_data(model, ph_dev):
    y = AG.forward_project(ph_dev, model).detach()
    y = add_noise(y, 0.01, CONE['seed'])
    w = torch.exp(-y / y.max())
    return y, w


def test_config2_gradient_matches_central_differences(cuda, cone_case, pool):
    """Central differences (eps = 1e-3) of the float64 oracle loss at 64 voxels of the region of reconstruction.
    The loss is a quadratic data term plus the qGGMRF prior, so each difference is evaluated where it changes: the
    data term through the residual r = A x - y (one pooled float64 forward projection) and the voxel's own column
    a of A (the oracle's forward projection of that one voxel), 0.5 sum W (r +- eps a)^2; the prior on the voxel's
    3x3x3 neighbourhood, which holds every clique that contains it."""
    model, geom, ph, _ = cone_case
    nr, nc, ns = geom.recon_shape
    ph_dev = torch.as_tensor(ph, device=cuda)
    y, w = _config2_data(model, ph_dev)
    x = (0.5 * ph + 0.02 * O.get_2d_ror_mask(geom.recon_shape)[:, :, None]).astype(np.float32)
    b, p, q, T = QPARAMS
    params = (b, 0.3, p, q, T)
    xt = torch.tensor(x, device=cuda, requires_grad=True)
    loss = AG.weighted_ls_qggmrf_loss(xt, model, y, w, params, view_chunk=32)
    (grad,) = torch.autograd.grad(loss, xt)
    grad = grad.cpu().numpy()

    yh, wh = y.cpu().numpy().astype(np.float64), w.cpu().numpy().astype(np.float64)
    np.random.seed(0)
    r = pool.forward_project(geom, x.astype(np.float64), dtype=np.float64) - yh
    x64 = x.astype(np.float64)
    rng = np.random.default_rng(5)
    ror = np.argwhere(np.broadcast_to(O.get_2d_ror_mask(geom.recon_shape)[:, :, None], geom.recon_shape))
    picks = ror[rng.choice(len(ror), 64, replace=False)]
    eps = 1e-3
    fd, ag = [], []
    for i, j, k in picks:
        cyl = np.zeros((1, ns), dtype=np.float64)
        cyl[0, k] = 1.0
        a = O.sparse_forward_project(geom, cyl, np.array([i * nc + j], dtype=np.int32), dtype=np.float64)
        sup = a != 0
        rs, ws, as_ = r[sup], wh[sup], a[sup]
        data = (0.5 * np.sum(ws * (rs + eps * as_) ** 2) - 0.5 * np.sum(ws * (rs - eps * as_) ** 2)) / (2 * eps)
        lo = [max(v - 1, 0) for v in (i, j, k)]
        crop = x64[lo[0]:i + 2, lo[1]:j + 2, lo[2]:k + 2].copy()
        c = (i - lo[0], j - lo[1], k - lo[2])
        crop[c] += eps
        lp = O.qggmrf_loss(crop, params)
        crop[c] -= 2 * eps
        lm = O.qggmrf_loss(crop, params)
        fd.append(data + (lp - lm) / (2 * eps))
        ag.append(grad[i, j, k])
    fd, ag = np.array(fd), np.array(ag)
    assert np.linalg.norm(ag - fd) <= 1e-3 * np.linalg.norm(fd)


def test_config2_projected_gradient_descent_100_steps(cuda, cone_case):
    model, geom, ph, _ = cone_case
    ph_dev = torch.as_tensor(ph, device=cuda)
    y, w = _config2_data(model, ph_dev)
    b, p, q, T = QPARAMS
    params = (b, 0.3, p, q, T)
    v = torch.rand_like(ph_dev)
    for _ in range(10):  # power iteration for the Lipschitz constant of A^T W A
        v = AG.back_project(w * AG.forward_project(v, model), model)
        lip = float(torch.linalg.norm(v))
        v = v / lip
    x, losses = AG.projected_gradient_descent(model, y, w, params, torch.zeros_like(ph_dev), steps=100,
                                              step_size=1.0 / (1.1 * lip), view_chunk=32)
    losses = losses.cpu().numpy()
    assert len(losses) == 100 and np.all(np.isfinite(losses))
    assert float(x.min()) >= 0.0
    assert losses[-1] < 0.2 * losses[0]

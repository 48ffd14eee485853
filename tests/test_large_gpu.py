"""Full-size parity by a size-independent property: the large cone-beam configuration (720 views x 512 rows x
1024 channels, source-detector = source-iso = 4096, recon 1024 x 1024 x 512, 2 GiB) is far too large for the
oracle, so the forward and back projectors are checked for adjointness, <A x, y> = <x, A^T y>, with the inner
products in float64 on the device."""
import numpy as np
import pytest
import torch

import mbirjax_b200 as mb

pytestmark = pytest.mark.gpu


def test_large_cone_projectors_are_adjoint(cuda):
    V, R, C = 720, 512, 1024
    angles = np.linspace(0, 2 * np.pi, V, endpoint=False).astype(np.float32)
    model = mb.ConeBeamModel((V, R, C), angles, 4096.0, 4096.0)
    shape = tuple(model.get_params('recon_shape'))
    assert shape == (1024, 1024, 512)
    gen = torch.Generator(device='cuda').manual_seed(0)
    x = torch.rand(shape, device='cuda', generator=gen)
    y = torch.rand((V, R, C), device='cuda', generator=gen)
    ax = model.forward_project(x)
    lhs = float(torch.sum(ax.double() * y.double()))
    del ax
    aty = model.back_project(y)
    rhs = float(torch.sum(x.double() * aty.double()))
    assert lhs > 0
    assert abs(lhs - rhs) / abs(lhs) <= 1e-5


def test_large_cone_subset_update_on_a_cropped_view_set_matches_oracle(cuda):
    """Values at the large size, where the oracle can afford them: the large cone geometry (detector 512 x 1024,
    sdd = sid = 4096, recon 1024 x 1024 x 512) restricted to 6 of its 720 views, one VCD subset update of 1 of 8
    subsets from a phantom-like state, against the oracle on all host cores from the same state.  Every per-view
    quantity (magnification, 128-row batch anchors of the forward fan, 128-slice batches of the back fan) is that of
    the full geometry."""
    from cases import oracle_geometry, rel_l2
    from oracle import vcd as OV
    from oracle.pool import OraclePool
    import oracle as O
    from mbirjax_b200 import _capi
    from mbirjax_b200.utilities import gen_ellipsoid_phantom
    views = np.linspace(0, 2 * np.pi, 720, endpoint=False).astype(np.float32)[::120]
    model = mb.ConeBeamModel((len(views), 512, 1024), views, 4096.0, 4096.0)
    model.set_params(recon_shape=(1024, 1024, 512), no_warning=True)
    geom = oracle_geometry(model)
    nr, nc, ns = geom.recon_shape
    ph = gen_ellipsoid_phantom(geom.recon_shape, 40, 2, device='cuda')
    y = model.forward_project(ph)
    rng = np.random.default_rng(0)
    flat = (0.9 * ph).reshape(-1, ns)
    flat += 0.02 * torch.as_tensor(rng.random(flat.shape, dtype=np.float32), device='cuda')
    err = (y - model.forward_project(flat.reshape(geom.recon_shape))).contiguous()
    hess = model.compute_hessian_diagonal().reshape(-1, ns).contiguous()
    np.random.seed(4)
    subset = O.gen_pixel_partition(geom.recon_shape, 8)[3]
    params = (O.get_b_from_nbr_wts([1, 1, 1]), 0.05, 2.0, 1.2, 1.0)
    fm = 1.0 / 0.5 ** 2
    flat_h, err_h, hess_h = flat.cpu().numpy(), err.cpu().numpy(), hess.cpu().numpy()
    stats = torch.zeros(4, dtype=torch.float64, device='cuda')
    _capi.vcd_subset_step(model._geometry(), flat, err, None, hess, torch.as_tensor(subset, device='cuda'), fm,
                          _capi.qggmrf_params(*params), stats)
    torch.cuda.synchronize()
    with OraclePool() as pool:
        r_ref, e_ref, l1_ref, a_ref = OV.vcd_subset_update(geom, flat_h, err_h, None, hess_h, subset, fm, params,
                                                           proj=pool)
    st = stats.cpu().numpy()
    assert st[0] == pytest.approx(a_ref, rel=1e-5)
    assert st[1] == pytest.approx(l1_ref, rel=1e-5)
    assert rel_l2(flat.cpu().numpy()[subset], r_ref[subset]) <= 1e-6
    assert rel_l2(err.cpu().numpy(), e_ref) <= 1e-5

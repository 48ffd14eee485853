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

"""CPU oracle for the MBIR hot path: TEST INFRASTRUCTURE ONLY.

This package restates, in NumPy, the arithmetic of the mbirjax reference (v0.6.7) for the functions
on the hot path: parallel-beam, cone-beam and translation sparse forward/back projection, the qGGMRF surrogate
gradient/Hessian and loss, pixel partitions, the VCD subset update and FBP/FDK filtering.  Every
function cites the reference file:line it follows.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` may import it,
and only as the checker (or the timed CPU baseline).  The product package ``mbirjax_b200`` never
imports it: its compute path is the CUDA library and fails loudly when that library is missing.

Parity pins: the qGGMRF restatement is checked against the reference's golden gradient/Hessian
vectors (``tests/golden/qggmrf_golden.json``, extracted from the reference test file by
``tests/golden/make_qggmrf_golden.py``).  The projectors are pinned by the reference's structural
tests (adjointness, Hessian finite difference, view batching) and by its end-to-end acceptance bounds (FBP,
FDK, VCD and the denoiser against their phantoms at the reference's own sizes,
``tests/golden/acceptance_bounds.json``), because the reference itself (JAX) is not installable offline.
"""

from .geometry import OracleGeometry, parallel_geometry, cone_geometry, translation_geometry  # noqa: F401
from .projectors import (  # noqa: F401
    sparse_forward_project, sparse_back_project, forward_project, back_project,
    compute_hessian_diagonal, forward_project_one_view, back_project_one_view,
)
from .qggmrf import (  # noqa: F401
    get_b_from_nbr_wts, get_2_b_tilde, qggmrf_gradient_and_hessian_at_indices, qggmrf_loss,
    qggmrf_loss_grad, compute_qggmrf_grad_and_hessian, b_tilde_by_definition,
)
from .partitions import (  # noqa: F401
    get_2d_ror_mask, gen_pixel_partition, gen_set_of_pixel_partitions, gen_partition_sequence,
    gen_full_indices,
)
from .filters import generate_direct_recon_filter, fbp_filter, fdk_filter  # noqa: F401
from .vcd import vcd_recon, vcd_subset_update, auto_regularization, prox_map  # noqa: F401

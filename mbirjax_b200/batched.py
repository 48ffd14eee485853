"""Batched VCD: reconstruct many scans of uneven geometry together on one GPU.

For each scan this does exactly what ``TomographyModel.recon`` does (``tomography_model.py:966-1084``), in the
same ``np.random`` order: auto-regularisation, partition, direct-recon initialisation with the alpha rescale,
Hessian diagonal, then per iteration ``np.random.permutation`` of the subsets.  The difference is how the subset
updates run: instead of one chain of launches per scan, every stage of a subset update is ONE persistent kernel
over a packed work list of all scans (``mbx_vcd_batched_step``), and all iterations of all scans are captured
in a single CUDA graph and replayed, so the host issues no launches and reads nothing back until the end.

Restrictions of the batched path: all scans share one geometry kind (parallel or cone beam; translation
geometry runs through ``TomographyModel.recon`` only), have psf radius 1, and use a single partition with the
same number of subsets (``granularity=[K]``, ``partition_sequence=[0]``).
"""
import numpy as np
import torch

from . import _capi
from .vcd_utils import gen_set_of_pixel_partitions, gen_partition_sequence, morton_order, morton_sorted_partition


class BatchedVCD:
    """recon() of many models at once.

    models: list of ParallelBeamModel or ConeBeamModel (one kind), sinograms / weights: per-scan arrays or
    tensors (weights entries may be None), seeds: per-scan np.random seeds applied before each scan's partition
    draw (None: use the global stream as is, scan after scan), init_recons: per-scan init (None: direct recon).
    """

    def __init__(self, models, sinograms, weights=None, seeds=None, init_recons=None):
        if len(models) == 0 or len(models) != len(sinograms):
            raise ValueError('models and sinograms must be non-empty lists of equal length')
        self.models = list(models)
        self.sinograms = list(sinograms)
        self.weights = list(weights) if weights is not None else [None] * len(models)
        self.seeds = seeds
        self.init_recons = list(init_recons) if init_recons is not None else [None] * len(models)
        self.graph = None

    def _setup(self, max_iterations):
        scans, schedules, self.states, self.partitions, self.reg = [], [], [], [], []
        num_subsets = None
        # the auto-regularisation statistics use at most ~20 views of each sinogram on the host: copy those views
        # of every scan first, so that the per-scan host work below overlaps the GPU setup work queued before it
        # (subsampling the subsample again selects the same views)
        small = [_view_subsample(sino) for sino in self.sinograms]
        small_w = [None if w is None else _view_subsample(w) for w in self.weights]
        for i, model in enumerate(self.models):
            if self.seeds is not None:
                np.random.seed(int(self.seeds[i]))
            reg = model.auto_set_regularization_params(small[i], weights=small_w[i])
            recon_shape, granularity = model.get_params(['recon_shape', 'granularity'])
            seq = gen_partition_sequence(model.get_params('partition_sequence'), max_iterations)
            if len(set(int(v) for v in seq)) != 1:
                raise ValueError('the batched path needs one partition per scan (e.g. granularity=[K], '
                                 'partition_sequence=[0])')
            partitions = gen_set_of_pixel_partitions(recon_shape, granularity, use_ror_mask=model.use_ror_mask)
            part = partitions[int(seq[0])]
            if num_subsets is None:
                num_subsets = part.shape[0]
            elif part.shape[0] != num_subsets:
                raise ValueError('all scans of a batch need the same number of subsets')
            state = model._vcd_setup(self.sinograms[i], self.weights[i], self.init_recons[i])
            schedules.append(np.stack([np.random.permutation(num_subsets) for _ in range(max_iterations)]))
            dev = state['device']
            part = morton_sorted_partition(part, recon_shape[1])  # spatially coherent processing order
            # from pinned memory, so that the copy does not wait for the setup work queued before it
            part_d = torch.from_numpy(np.ascontiguousarray(part, dtype=np.int32)).pin_memory().to(
                dev, non_blocking=True)
            rec = _capi.MbxScan()
            rec.geom = model._geometry()
            rec.flat_recon = state['flat_recon'].data_ptr()
            rec.error_sinogram = state['error_sinogram'].data_ptr()
            rec.weights = state['weights'].data_ptr() if state['weights'] is not None else None
            rec.fm_hessian = state['fm_hessian'].data_ptr()
            rec.partition = part_d.data_ptr()
            rec.partition_order = None
            rec.num_subsets = int(part.shape[0])
            rec.subset_size = int(part.shape[1])
            rec.fm_constant = float(state['fm_constant'])
            rec.qp = state['qp']
            state['partition_d'] = part_d
            scans.append(rec)
            self.states.append(state)
            self.partitions.append(part)
            self.reg.append(reg)
        self.num_subsets = num_subsets
        # schedule[step, scan] with step = iteration * K + j
        sched = np.stack(schedules, axis=-1).reshape(max_iterations * num_subsets, len(self.models))
        return scans, sched

    def recon(self, max_iterations=10, use_graph=True):
        """Returns (list of recons, list of recon_params dicts)."""
        scans, sched = self._setup(max_iterations)
        dev = self.states[0]['device']
        n, steps = len(scans), sched.shape[0]
        self.step_stats = torch.zeros((steps, n, 4), dtype=torch.float64, device=dev)
        self.iter_stats = torch.zeros((max_iterations, n, 4), dtype=torch.float64, device=dev)
        self.plan, self.workspace = _capi.vcd_batched_prepare(scans, sched, max_iterations, self.step_stats,
                                                              self.iter_stats, dev)
        K = self.num_subsets

        def run_all():
            for it in range(max_iterations):
                for j in range(K):
                    _capi.vcd_batched_step(self.plan, it * K + j)
                _capi.vcd_batched_iteration_stats(self.plan, it)

        if use_graph:
            # captured on a side stream that first waits for the setup work; capture_begin / capture_end directly
            # rather than torch.cuda.graph(), whose entry synchronises, runs the garbage collector and empties the
            # caching allocator (so that every later allocation goes back to cudaMalloc)
            self.graph = torch.cuda.CUDAGraph()
            main = torch.cuda.current_stream()
            side = torch.cuda.Stream()
            side.wait_stream(main)
            with torch.cuda.stream(side):
                self.graph.capture_begin()
                try:
                    run_all()
                finally:
                    self.graph.capture_end()
            main.wait_stream(side)
            self.graph.replay()
        else:
            run_all()
        out = self._results(max_iterations)  # reads the statistics back (synchronises)
        # release the graph and the scratch now rather than whenever the object is collected, so that the
        # next reconstruction finds its memory in the caching allocator instead of allocating afresh
        if self.graph is not None:
            self.graph.reset()
            self.graph = None
        self.workspace = None
        self.plan = None  # its tables lived in the workspace
        return out

    def _results(self, max_iterations):
        step = self.step_stats.cpu().numpy()
        it = self.iter_stats.cpu().numpy()
        K = self.num_subsets
        recons, dicts = [], []
        for s, (model, state) in enumerate(zip(self.models, self.states)):
            recon_shape = model.get_params('recon_shape')
            st = step[:, s, :].reshape(max_iterations, K, 4)
            ell1 = st[:, :, 1].sum(axis=1)
            alphas = st[:, :, 0].mean(axis=1)
            w = state['weights']
            sino_size = state['error_sinogram'].numel()
            if w is None:
                wmean = 1.0
            else:
                wmean = float(torch.mean(w.double()))
            sigma_y = state['sigma_y']
            fm_rmse = np.sqrt((1.0 / sigma_y ** 2) * it[:, s, 0] / (sino_size * wmean))
            nmae = ell1 / it[:, s, 1]
            recons.append(state['flat_recon'].reshape(recon_shape))
            dicts.append({'num_iterations': max_iterations, 'granularity': model.get_params('granularity'),
                          'fm_rmse': [float(v) for v in fm_rmse], 'regularization_params': self.reg[s],
                          'stop_threshold_change_pct': [100 * float(v) for v in nmae],
                          'alpha_values': [float(v) for v in alphas]})
        return recons, dicts


def _view_subsample(x):
    """The views auto_set_regularization_params reads (tomography_model.py:766-770), on the host."""
    num_views = x.shape[0]
    step = num_views // min(20, num_views)
    sub = x[::step]
    return sub.cpu().numpy() if isinstance(sub, torch.Tensor) else np.asarray(sub)

"""Batched VCD: reconstruct many scans of uneven geometry together on one GPU.

For each scan this does what ``TomographyModel.recon`` does (``tomography_model.py:966-1255``), in the same
``np.random`` order: auto-regularisation, partition, direct-recon initialisation with the alpha rescale, Hessian
diagonal, then per iteration ``np.random.permutation`` of the subsets.  The difference is how the device work runs:
every stage of the set-up and of a subset update is ONE persistent kernel over a packed work list of all scans
(``mbx_vcd_batched_setup`` / ``mbx_vcd_batched_step``), and the host issues no launches and reads nothing back
until the end.

The device state of a batch shape (per-scan buffers, the prepared plan with its tuned work lists, and two CUDA
graphs: the set-up of all scans, and all iterations of all scans) is built by the first ``recon`` of that shape
and kept in a small cache, so later calls of the same shape only copy their sinograms in, replay the set-up graph,
run the host part (auto-regularisation statistics and the reference's partition and subset-order draws) while the
set-up runs on the device, upload the new parameters and partitions, and replay the iteration graph.

Restrictions of the batched path: all scans share one geometry kind (parallel, cone or translation), have psf
radius 1, and use a single partition with the same number of subsets (``granularity=[K]``,
``partition_sequence=[0]``).  Translation scans start from zeros, as ``TranslationModel.recon`` does (the reference
has no direct recon for that geometry).
"""
import collections
import warnings

import numpy as np
import torch

from . import _capi
from .vcd_utils import (gen_full_indices, gen_partition_sequence, gen_set_of_pixel_partitions, morton_order,
                        morton_sorted_partition)

__all__ = ['BatchedVCD', 'release_batched_sessions', 'morton_order']

_REPLAYED = [0]  # kernel launches replayed from the batched CUDA graphs (mbx_launch_count counts host launches)


def replayed_launches():
    """Kernels of this library launched by replays of the batched CUDA graphs so far (each replay launches every
    kernel node its capture recorded; mbx_launch_count counts only launches the host submits)."""
    return _REPLAYED[0]


_SESSIONS = collections.OrderedDict()  # batch key -> _Session, most recently used last
_MAX_SESSIONS = 2
PLAN_FORWARD = True               # plan the subset forward projections of a batch when it fits (see _Session)
PLAN_FORWARD_MAX_FRACTION = 0.5   # of the free device memory the plan's workspace may take


_POOL = None


def _draw_pool():
    """Host threads for the per-scan draws."""
    global _POOL
    if _POOL is None:
        import concurrent.futures
        import os
        _POOL = concurrent.futures.ThreadPoolExecutor(max_workers=min(16, os.cpu_count() or 1))
    return _POOL


def release_batched_sessions():
    """Free the device state (buffers, plans, graphs) kept for the batch shapes reconstructed so far."""
    while _SESSIONS:
        _SESSIONS.popitem(last=False)[1].close()


class BatchedVCD:
    """recon() of many models at once.

    models: list of ParallelBeamModel, ConeBeamModel or TranslationModel (one kind), sinograms / weights: per-scan arrays or
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

    # ---------------------------------------------------------------- host part of a reconstruction
    def _host_subsamples(self):
        """The views of every sinogram (and weights) that auto-regularisation reads, on the host."""
        return ([_view_subsample(sino) for sino in self.sinograms],
                [None if w is None else _view_subsample(w) for w in self.weights])

    def _scan_draws(self, i, max_iterations, small, small_w, rng):
        """Host part of scan i, in the reference's np.random order on the stream rng (None: the global stream):
        auto-regularisation (on the host subsamples), the partition, the region-of-reconstruction draws of the
        set-up (direct recon's back projection and the initial forward projection) and the subset order of every
        iteration.  Returns (regularisation dict, Morton-sorted partition, schedule (iterations, K), fm constant,
        qGGMRF record, sigma_y)."""
        model = self.models[i]
        reg = model.auto_set_regularization_params(small[i], weights=small_w[i])
        recon_shape, granularity = model.get_params(['recon_shape', 'granularity'])
        seq = gen_partition_sequence(model.get_params('partition_sequence'), max_iterations)
        if len(set(int(v) for v in seq)) != 1:
            raise ValueError('the batched path needs one partition per scan (e.g. granularity=[K], '
                             'partition_sequence=[0])')
        part = gen_set_of_pixel_partitions(recon_shape, granularity, use_ror_mask=model.use_ror_mask,
                                           rng=rng)[int(seq[0])]
        # translation geometry has no direct recon (zeros, no draw); the others draw for its back projection
        draws = 1 if model._kind() == _capi.MBX_GEOM_TRANSLATION else 2
        for _ in range(draws):
            gen_full_indices(recon_shape, use_ror_mask=model.use_ror_mask, rng=rng)
        src = np.random if rng is None else rng
        num_subsets = part.shape[0]
        schedule = np.stack([src.permutation(num_subsets) for _ in range(max_iterations)])
        part = morton_sorted_partition(part, recon_shape[1])  # spatially coherent processing order
        sigma_y = float(model.get_params('sigma_y'))
        b, sigma_x, p, q, T = model._qggmrf_params()
        return reg, part, schedule, 1.0 / (sigma_y ** 2.0), _capi.qggmrf_params(b, sigma_x, p, q, T), sigma_y

    def _host_draws(self, max_iterations, small, small_w):
        """The host part of every scan (see _scan_draws).  With per-scan seeds each scan draws from its own
        RandomState, which is the stream np.random.seed(seed) gives, so the scans run on a pool of host threads
        and the global stream is left where the plain path leaves it, after the last scan's draws.  (The legacy
        shuffles, most of this time, hold the GIL, so the threads overlap only the sorts and array work; the
        whole host part runs while the set-up graph runs on the device.)  Without seeds the scans draw from the
        global stream one after another.
        Returns (regularisation dicts, partitions, schedule (steps, scans), fm constants, qGGMRF records, sigmas)."""
        n = len(self.models)
        for model in self.models:
            if model._kind() == _capi.MBX_GEOM_TRANSLATION:
                warnings.warn('direct_recon not implemented for TomographyModel.')
        if self.seeds is None:
            out = [self._scan_draws(i, max_iterations, small, small_w, None) for i in range(n)]
        else:
            rngs = [np.random.RandomState(int(sd)) for sd in self.seeds]
            out = list(_draw_pool().map(
                lambda i: self._scan_draws(i, max_iterations, small, small_w, rngs[i]), range(n)))
            np.random.set_state(rngs[-1].get_state())
        regs, parts, schedules, fms, qps, sigmas = (list(v) for v in zip(*out))
        num_subsets = parts[0].shape[0]
        if any(p.shape[0] != num_subsets for p in parts):
            raise ValueError('all scans of a batch need the same number of subsets')
        # schedule[step, scan] with step = iteration * K + j
        sched = np.stack(schedules, axis=-1).reshape(max_iterations * num_subsets, n)
        return regs, parts, sched.astype(np.int32), fms, qps, sigmas

    # ---------------------------------------------------------------- reconstruction
    def recon(self, max_iterations=10, use_graph=True):
        """Returns (list of recons, list of recon_params dicts)."""
        if any(init is not None for init in self.init_recons):
            return self._recon_host_setup(max_iterations, use_graph)
        key = _batch_key(self.models, self.weights, max_iterations)
        sess = _SESSIONS.get(key)
        fresh = sess is None
        # the host copies of the auto-regularisation views come before any device work of this call is queued, so
        # that they wait for nothing of it
        small, small_w = self._host_subsamples()
        regs, parts, sched, fms, qps, sigmas = None, None, None, None, None, None
        if fresh:
            # the host draws come first: the plan is prepared (and tuned) on real partitions
            regs, parts, sched, fms, qps, sigmas = self._host_draws(max_iterations, small, small_w)
            sess = _Session(self.models, self.weights, parts, sched, fms, qps, max_iterations)
            _SESSIONS[key] = sess
            while len(_SESSIONS) > _MAX_SESSIONS:
                _SESSIONS.popitem(last=False)[1].close()
        _SESSIONS.move_to_end(key)
        sess.load_inputs(self.sinograms, self.weights)
        sess.run_setup(use_graph)
        if not fresh:  # the host part overlaps the set-up queued above
            regs, parts, sched, fms, qps, sigmas = self._host_draws(max_iterations, small, small_w)
            sess.load_parameters(parts, sched, fms, qps)
        sess.run_iterations(use_graph)
        return sess.results(self.models, regs, sigmas)

    # ---------------------------------------------------------------- explicit initial recons
    def _setup(self, max_iterations):
        """Host-driven set-up (each scan through TomographyModel._vcd_setup, which accepts an initial recon) and
        the MbxScan records of the batch.  Returns (records, schedule)."""
        scans, schedules, self.states, self.partitions, self.reg = [], [], [], [], []
        num_subsets = None
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
            part = morton_sorted_partition(part, recon_shape[1])
            part_d = torch.from_numpy(np.ascontiguousarray(part, dtype=np.int32)).pin_memory().to(
                dev, non_blocking=True)
            rec = _scan_record(model._geometry(), state['flat_recon'], state['error_sinogram'], state['weights'],
                               state['fm_hessian'], part_d, float(state['fm_constant']), state['qp'])
            state['partition_d'] = part_d
            scans.append(rec)
            self.states.append(state)
            self.partitions.append(part)
            self.reg.append(reg)
        self.num_subsets = num_subsets
        sched = np.stack(schedules, axis=-1).reshape(max_iterations * num_subsets, len(self.models))
        return scans, sched

    def _recon_host_setup(self, max_iterations, use_graph):
        scans, sched = self._setup(max_iterations)
        dev = self.states[0]['device']
        n, steps = len(scans), sched.shape[0]
        step_stats = torch.zeros((steps, n, 4), dtype=torch.float64, device=dev)
        iter_stats = torch.zeros((max_iterations, n, 4), dtype=torch.float64, device=dev)
        plan, workspace = _capi.vcd_batched_prepare(scans, sched, max_iterations, step_stats, iter_stats, dev)
        K = self.num_subsets

        def run_all():
            for it in range(max_iterations):
                for j in range(K):
                    _capi.vcd_batched_step(plan, it * K + j)
                _capi.vcd_batched_iteration_stats(plan, it)

        graph = None
        if use_graph:
            graph, kernels = _capture_counted(run_all)
            graph.replay()
            _REPLAYED[0] += kernels
        else:
            run_all()
        step = step_stats.cpu().numpy()  # synchronises
        it = iter_stats.cpu().numpy()
        del graph, plan, workspace
        return _results(self.models, [st['flat_recon'] for st in self.states],
                        [st['error_sinogram'].numel() for st in self.states],
                        [st['weights'] for st in self.states], [st['sigma_y'] for st in self.states], self.reg,
                        step, it, max_iterations, K, clone=False)


class _Session:
    """Device state of one batch shape: per-scan buffers (sinogram, weights, error sinogram, flat recon, Hessian,
    partition, region-of-reconstruction list), session-owned geometry records, the prepared plan and its
    workspace, statistics, and the set-up and iteration graphs."""

    def __init__(self, models, weights, parts, sched, fms, qps, max_iterations):
        dev = models[0]._device()
        self.device = dev
        self.max_iterations = max_iterations
        self.num_subsets = parts[0].shape[0]
        self.recon_shapes = [tuple(m.get_params('recon_shape')) for m in models]
        self.geoms, self.angles = [], []
        self.y, self.w, self.err, self.flat, self.hess, self.part, self.full = [], [], [], [], [], [], []
        scans = []
        for i, model in enumerate(models):
            g0 = model._geometry()
            g = _capi.MbxGeom.from_buffer_copy(g0)
            view_params = np.asarray(model.get_params(model.get_params('view_params_name')), dtype=np.float32)
            ang = torch.as_tensor(view_params, device=dev).contiguous()
            if g.kind == _capi.MBX_GEOM_TRANSLATION:
                g.translations = ang.data_ptr()
            else:
                g.angles = ang.data_ptr()
            self.geoms.append(g)
            self.angles.append(ang)
            V, R, C = (int(v) for v in model.get_params('sinogram_shape'))
            nr, nc, ns = self.recon_shapes[i]
            self.y.append(torch.empty((V, R, C), dtype=torch.float32, device=dev))
            self.w.append(None if weights[i] is None else torch.empty((V, R, C), dtype=torch.float32, device=dev))
            self.err.append(torch.empty((V, R, C), dtype=torch.float32, device=dev))
            self.flat.append(torch.empty((nr * nc, ns), dtype=torch.float32, device=dev))
            self.hess.append(torch.empty((nr * nc, ns), dtype=torch.float32, device=dev))
            self.part.append(torch.as_tensor(np.ascontiguousarray(parts[i], dtype=np.int32), device=dev))
            full = gen_full_indices_no_draw(self.recon_shapes[i], model.use_ror_mask)
            self.full.append(torch.as_tensor(full, dtype=torch.int32, device=dev))
            rec = _scan_record(g, self.flat[i], self.err[i], self.w[i], self.hess[i], self.part[i], fms[i], qps[i])
            rec.sinogram = self.y[i].data_ptr()
            rec.full_indices = self.full[i].data_ptr()
            rec.num_full_indices = int(self.full[i].shape[0])
            scans.append(rec)
        self.scans = scans
        n, steps = len(scans), sched.shape[0]
        self.step_stats = torch.zeros((steps, n, 4), dtype=torch.float64, device=dev)
        self.iter_stats = torch.zeros((max_iterations, n, 4), dtype=torch.float64, device=dev)
        # pinned staging of the per-call partitions
        self.part_host = [torch.empty(tuple(p.shape), dtype=torch.int32).pin_memory() for p in self.part]
        # planned forward projections (each subset's sorted record passes, built once per reconstruction and
        # replayed by every iteration) when their storage leaves most of the device free
        flags = _capi.MBX_BATCHED_PLAN_FORWARD if PLAN_FORWARD else 0
        if flags:
            need = _capi.vcd_batched_workspace_bytes(scans, sched.shape[0], flags)
            free = torch.cuda.mem_get_info(dev)[0]
            if need == 0 or need > PLAN_FORWARD_MAX_FRACTION * free:
                flags = 0
        self.planned_forward = bool(flags)
        self.plan, self.workspace = _capi.vcd_batched_prepare(scans, sched, max_iterations, self.step_stats,
                                                              self.iter_stats, dev, flags)
        self.setup_graph = None
        self.iter_graph = None

    def close(self):
        self.setup_graph = None
        self.iter_graph = None
        self.plan = None
        self.workspace = None

    def load_inputs(self, sinograms, weights):
        for i, s in enumerate(sinograms):
            _copy_in(self.y[i], s)
            if self.w[i] is not None:
                _copy_in(self.w[i], weights[i])

    def load_parameters(self, parts, sched, fms, qps):
        for i, p in enumerate(parts):
            self.part_host[i].numpy()[...] = p
            self.part[i].copy_(self.part_host[i], non_blocking=True)
        for rec, fm, qp in zip(self.scans, fms, qps):
            rec.fm_constant = fm
            rec.qp = qp
        _capi.vcd_batched_update(self.plan, self.scans, sched)

    def _setup_launches(self):
        _capi.vcd_batched_setup(self.plan)

    def _iteration_launches(self):
        _capi.vcd_batched_refresh(self.plan)  # chunk boxes of the partitions written for this call
        K = self.num_subsets
        for it in range(self.max_iterations):
            for j in range(K):
                _capi.vcd_batched_step(self.plan, it * K + j)
            _capi.vcd_batched_iteration_stats(self.plan, it)

    def run_setup(self, use_graph):
        if not use_graph:
            self._setup_launches()
            return
        if self.setup_graph is None:
            self.setup_graph, self.setup_kernels = _capture_counted(self._setup_launches)
        self.setup_graph.replay()
        _REPLAYED[0] += self.setup_kernels

    def run_iterations(self, use_graph):
        if not use_graph:
            self._iteration_launches()
            return
        if self.iter_graph is None:
            self.iter_graph, self.iter_kernels = _capture_counted(self._iteration_launches)
        self.iter_graph.replay()
        _REPLAYED[0] += self.iter_kernels

    def results(self, models, regs, sigmas):
        step = self.step_stats.cpu().numpy()  # synchronises
        it = self.iter_stats.cpu().numpy()
        return _results(models, self.flat, [e.numel() for e in self.err], self.w, sigmas, regs, step, it,
                        self.max_iterations, self.num_subsets, clone=True)


def _results(models, flats, sino_sizes, weights, sigmas, regs, step, it, max_iterations, K, clone):
    recons, dicts = [], []
    for s, model in enumerate(models):
        recon_shape = model.get_params('recon_shape')
        st = step[:, s, :].reshape(max_iterations, K, 4)
        ell1 = st[:, :, 1].sum(axis=1)
        alphas = st[:, :, 0].mean(axis=1)
        w = weights[s]
        wmean = 1.0 if w is None else float(torch.mean(w.double()))
        fm_rmse = np.sqrt((1.0 / sigmas[s] ** 2) * it[:, s, 0] / (sino_sizes[s] * wmean))
        nmae = ell1 / it[:, s, 1]
        rec = flats[s].clone() if clone else flats[s]
        recons.append(rec.reshape(recon_shape))
        dicts.append({'num_iterations': max_iterations, 'granularity': model.get_params('granularity'),
                      'fm_rmse': [float(v) for v in fm_rmse], 'regularization_params': regs[s],
                      'stop_threshold_change_pct': [100 * float(v) for v in nmae],
                      'alpha_values': [float(v) for v in alphas]})
    return recons, dicts


def _scan_record(geom, flat, err, w, hess, part_d, fm_constant, qp):
    rec = _capi.MbxScan()
    rec.geom = geom
    rec.flat_recon = flat.data_ptr()
    rec.error_sinogram = err.data_ptr()
    rec.weights = w.data_ptr() if w is not None else None
    rec.fm_hessian = hess.data_ptr()
    rec.partition = part_d.data_ptr()
    rec.partition_order = None
    rec.num_subsets = int(part_d.shape[0])
    rec.subset_size = int(part_d.shape[1])
    rec.fm_constant = float(fm_constant)
    rec.qp = qp
    rec.sinogram = None
    rec.full_indices = None
    rec.num_full_indices = 0
    return rec


def _capture(launches):
    """A CUDA graph of the library launches that `launches` enqueues, captured on a side stream that first waits
    for the work queued so far (capture_begin / capture_end directly rather than torch.cuda.graph(), whose entry
    synchronises, runs the garbage collector and empties the caching allocator)."""
    graph = torch.cuda.CUDAGraph()
    main = torch.cuda.current_stream()
    side = torch.cuda.Stream()
    side.wait_stream(main)
    with torch.cuda.stream(side):
        graph.capture_begin()
        try:
            launches()
        finally:
            graph.capture_end()
    main.wait_stream(side)
    return graph


def _capture_counted(launches):
    """_capture, and the number of library kernels the graph holds (counted while capturing)."""
    lib = _capi.load_library()
    n0 = lib.mbx_launch_count()
    graph = _capture(launches)
    return graph, int(lib.mbx_launch_count() - n0)


def _copy_in(dst, src):
    """src (host array, host tensor or device tensor) into the device buffer dst, on the current stream."""
    if isinstance(src, torch.Tensor):
        src = src.detach()
        if src.dtype != torch.float32:
            src = src.float()
        dst.copy_(src.reshape(dst.shape), non_blocking=src.is_cuda or src.is_pinned())
    else:
        dst.copy_(torch.as_tensor(np.ascontiguousarray(src, dtype=np.float32)).reshape(dst.shape))


def gen_full_indices_no_draw(recon_shape, use_ror_mask):
    """The sorted region-of-reconstruction pixels of a grid without advancing np.random (the set is the same for
    every draw): the stream state is saved around the draw and restored."""
    state = np.random.get_state()
    try:
        return np.asarray(gen_full_indices(recon_shape, use_ror_mask=use_ror_mask), dtype=np.int32)
    finally:
        np.random.set_state(state)


def _batch_key(models, weights, max_iterations):
    """The batch shape: every scan's geometry record (pointers left out) and view parameters, which scans carry
    weights, and the iteration count."""
    items = []
    for model, w in zip(models, weights):
        g = _capi.MbxGeom.from_buffer_copy(model._geometry())
        g.angles = None
        g.translations = None
        view_params = np.asarray(model.get_params(model.get_params('view_params_name')), dtype=np.float32)
        items.append((bytes(g), view_params.tobytes(), w is not None, tuple(model.get_params('granularity')),
                      bool(model.use_ror_mask)))
    return (tuple(items), int(max_iterations))


def _view_subsample(x):
    """The views auto_set_regularization_params reads (tomography_model.py:766-770), on the host."""
    num_views = x.shape[0]
    step = num_views // min(20, num_views)
    sub = x[::step]
    return sub.cpu().numpy() if isinstance(sub, torch.Tensor) else np.asarray(sub)

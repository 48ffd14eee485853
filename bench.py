#!/usr/bin/env python
"""Benchmark of the MBIR hot path on B200.

Default workload (``--workload batched``): 24 independent parallel-beam scans of uneven geometry.  Scan i (seed i)
draws views U{60..720} on [0, pi), det_rows U{8..64} and det_channels U{96..512}; its volume is channels x
channels x rows holding 10 seeded random ellipsoids (centres in the inner 70%, semi-axes U[5,40] voxels,
densities U[0.1,1], summed where they overlap), forward-projected with 1% Gaussian noise; qGGMRF p=2, q=1.2, T=1,
sharpness 0, 4 pixel subsets, 10 VCD iterations with FBP initialisation.  A step is one reconstruction of all 24
scans; the value is recons/s of the batched path (``mbirjax_b200.batched.BatchedVCD``: one persistent work-list
kernel per stage over all scans, all iterations in one CUDA graph).  The same line reports the plain per-scan GPU
path (``ParallelBeamModel.recon`` scan after scan) measured the same way, and their ratio.

``--workload cone``: plain cone-beam VCD on one scan (256 views x 128 rows x 256 channels, sdd = sid = 1024,
recon 256x256x128 from 20 ellipsoids, 20 iterations x 4 subsets, FDK init).

``--workload large``: plain cone-beam VCD at the large size (720 views x 512 rows x 1024 channels, about 1.5 GB,
sdd = sid = 4096, recon 1024x1024x512 (2 GiB) from 40 ellipsoids, 10 iterations x 8 subsets, FDK init), plus one FDK
direct recon and one autograd gradient of the differentiable loss with 32-view backward chunks; the line adds the
peak device memory.  Defaults to 1 warm-up and 1 timed step (a step takes tens of seconds).

``--workload translation``: plain translation-geometry VCD on the setup of the reference's translation experiment
(experiments/translation/exp_translation.py: a 7 x 7 raster of translations 22 ALU apart = 49 views, 128 x 128
detector, sdd = sid = 64, recon 21x196x196 from the model's own sizing, sharpness 1, zero init, 15 iterations),
with 10 seeded ellipsoids in place of the rendered-text phantom and 4 subsets per iteration.

Synthetic data stands in for measured scans (the reference publishes no benchmark dataset).
Timing: W untimed warm-up steps, then exactly K steps between barriers + device synchronisations, timed with
CUDA events on the launching stream; max over ranks.  L2 is flushed (a 256 MB write) before every step, inside
the timed region (the batched inputs, about 1 GB, exceed L2 anyway).  SM clocks and throttle reasons are sampled
with nvidia-smi during the timed region.  ``e2e`` repeats the measurement through the public API with the
sinograms in pinned host memory and the recons copied back each step.  ``roofline`` times the dominant kernels
(the back- and forward-projection stages of a subset update) live with CUDA events and divides their algorithmic
bytes, 4 (V N S + V R C) summed over scans, by the measured HBM copy bandwidth.  ``cpu_baseline`` times the
oracle's restatement of the reference arithmetic on all host cores for one whole reconstruction of one batch scan
(auto-regularisation, FBP init, Hessian, all iterations) and scales it across scans by the same work model.  ``autograd`` times one gradient of the differentiable
cone-beam loss (weighted least squares + qGGMRF, backward through the matched back projector in 32-view chunks)
against one forward projection on the same geometry.

``--impl reference`` times the reference arithmetic (the oracle port: JAX is not installable offline, so the
reference's own JAX CPU path cannot run) on the host cores on the same workload and metric.
Multi-GPU (torchrun, one process per GPU): independent replicas, no collective on the data path.
"""
import argparse
import json
import os
import re
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = 'batched vs plain recons/s at 1e-4 NRMSE; proj HBM GB/s; autograd/fwd time'
CONE = dict(views=256, rows=128, channels=256, sdd=1024.0, sid=1024.0, ellipsoids=20, seed=1, subsets=4,
            iterations=20)
BATCH = dict(num_scans=24, ellipsoids=10, subsets=4, iterations=10, cpu_sample_scan=0)
LARGE = dict(views=720, rows=512, channels=1024, sdd=4096.0, sid=4096.0, ellipsoids=40, seed=2, subsets=8,
             iterations=10)
TRANS = dict(nx=7, nz=7, spacing=22.0, rows=128, channels=128, sdd=64.0, sid=64.0, ellipsoids=10, seed=2, subsets=4,
             iterations=15, sharpness=1.0)


def sig(x, digits=4):
    """x rounded to a number of significant digits (throughputs here span 1e-5 to 1e2 recons/s)."""
    return float('%.*g' % (digits, x))


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument('--gpus', type=int, default=1)
    ap.add_argument('--steps', type=int, default=None, help='timed steps (default 5; 1 for --workload large)')
    ap.add_argument('--warmup', type=int, default=None, help='warm-up steps (default 3; 1 for --workload large)')
    ap.add_argument('--impl', default='mbirjax_b200', choices=['mbirjax_b200', 'reference'])
    ap.add_argument('--workload', default='batched', choices=['batched', 'cone', 'translation', 'large'])
    ap.add_argument('--no-e2e', action='store_true')
    ap.add_argument('--no-cpu-baseline', action='store_true')
    ap.add_argument('--scans', type=int, default=None,
                    help='batched workload: the first N scans only (a small case for profiling; default 24)')
    ap.add_argument('--iterations', type=int, default=None, help='VCD iterations per scan (default 10 / 20 / 15)')
    ap.add_argument('--cpu-sample-scan', type=int, default=None,
                    help='batched workload: the batch scan whose whole oracle reconstruction is the CPU sample '
                         '(default 0)')
    ap.add_argument('--autotune', type=int, default=1, choices=[0, 1],
                    help='1: tune the projector plans (default); 0: default plans, no tuning launches (for profiling)')
    ap.add_argument('--no-plan-forward', action='store_true',
                    help='batched path: scan, sort and walk every forward projection instead of replaying stored '
                         'record passes (for comparison and profiling)')
    args = ap.parse_args()
    if args.steps is None:
        args.steps = 1 if args.workload == 'large' else 5
    if args.warmup is None:
        args.warmup = 1 if args.workload == 'large' else 3
    if args.scans is not None:
        BATCH['num_scans'] = args.scans
    if args.cpu_sample_scan is not None:
        BATCH['cpu_sample_scan'] = args.cpu_sample_scan
    if args.iterations is not None:
        BATCH['iterations'] = args.iterations
        CONE['iterations'] = args.iterations
        TRANS['iterations'] = args.iterations
        LARGE['iterations'] = args.iterations
    return args


# ----------------------------------------------------------------------------------------------- helpers
def load_peaks():
    try:
        with open(os.path.join(ROOT, 'MEASURED_PEAKS.json')) as f:
            d = json.load(f)
        return float(d['hbm_gbs']), 'measured'
    except Exception:
        return 6650.0, 'fallback'


class ClockSampler:
    """nvidia-smi sampling of SM clock and throttle reasons while the timed region runs.  Every 500 ms: at 200 ms
    the NVML queries were seen to stall a batched reconstruction now and then (0.4 - 1.1 s in 1.8 s)."""

    FIELDS = ('index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,'
              'clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,'
              'clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap')

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix='.csv')
        os.close(fd)
        try:
            self.proc = subprocess.Popen(['nvidia-smi', '-i', str(self.gpu), '--query-gpu=' + self.FIELDS,
                                          '--format=csv,noheader,nounits', '-lms', '500'],
                                         stdout=open(self.path, 'w'), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {'sm_mhz': None, 'sm_max_mhz': None, 'reasons': ['nvidia-smi unavailable']}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ['hw_slowdown', 'hw_thermal_slowdown', 'sw_thermal_slowdown', 'sw_power_cap']
        for line in open(self.path):
            parts = [p.strip() for p in line.split(',')]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for name, val in zip(names, parts[5:9]):
                if val.lower() == 'active':
                    reasons.add(name)
        os.unlink(self.path)
        return {'sm_mhz': statistics.median(sm) if sm else None, 'sm_max_mhz': smax, 'reasons': sorted(reasons),
                'samples': len(sm)}


def dist_setup(n_gpus):
    import torch
    world = int(os.environ.get('WORLD_SIZE', '1'))
    rank = int(os.environ.get('RANK', '0'))
    local = int(os.environ.get('LOCAL_RANK', '0'))
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group('nccl', timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device('cuda', local))
    elif torch.cuda.is_available():
        torch.cuda.set_device(0)
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(value, world):
    if world == 1:
        return value
    import torch
    import torch.distributed as dist
    # the NCCL group reduces device tensors; a gloo group (the CPU tests of this logic) host tensors
    device = 'cuda' if dist.get_backend() == 'nccl' else 'cpu'
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ----------------------------------------------------------------------------------------------- workload
def cone_angles(spec=CONE):
    return np.linspace(0, 2 * np.pi, spec['views'], endpoint=False).astype(np.float32)


def cone_model(spec=CONE):
    import mbirjax_b200 as mb
    return mb.ConeBeamModel((spec['views'], spec['rows'], spec['channels']), cone_angles(spec),
                            source_detector_dist=spec['sdd'], source_iso_dist=spec['sid'])


def build_cone_workload(device, spec=CONE):
    """The cone model, its noisy sinogram (forward projection of the seeded ellipsoid phantom + 1% noise) and the
    phantom."""
    from mbirjax_b200.utilities import gen_ellipsoid_phantom, add_noise
    model = cone_model(spec)
    model.set_params(sharpness=0.0, snr_db=30.0, granularity=[spec['subsets']], partition_sequence=[0], verbose=0)
    phantom = gen_ellipsoid_phantom(model.get_params('recon_shape'), spec['ellipsoids'], spec['seed'], device=device)
    np.random.seed(spec['seed'])
    sino = add_noise(model.forward_project(phantom), 0.01, spec['seed']).contiguous()
    return model, sino, phantom


def recon_once(model, sino, spec=CONE):
    np.random.seed(spec['seed'])
    rec, _ = model.recon(sino, max_iterations=spec['iterations'], stop_threshold_change_pct=0, logfile_path=None,
                         print_logs=False)
    return rec


def translation_vectors():
    from mbirjax_b200.utilities import gen_translation_vectors
    return gen_translation_vectors(TRANS['nx'], TRANS['nz'], TRANS['spacing'], TRANS['spacing'])


def build_translation_workload(device):
    import mbirjax_b200 as mb
    from mbirjax_b200.utilities import gen_ellipsoid_phantom, add_noise
    tv = translation_vectors()
    model = mb.TranslationModel((tv.shape[0], TRANS['rows'], TRANS['channels']), tv,
                                source_detector_dist=TRANS['sdd'], source_iso_dist=TRANS['sid'])
    model.set_params(sharpness=TRANS['sharpness'], snr_db=30.0, granularity=[TRANS['subsets']],
                     partition_sequence=[0], verbose=0)
    phantom = gen_ellipsoid_phantom(model.get_params('recon_shape'), TRANS['ellipsoids'], TRANS['seed'], device=device)
    np.random.seed(TRANS['seed'])
    sino = add_noise(model.forward_project(phantom), 0.01, TRANS['seed']).contiguous()
    return model, sino, phantom


def translation_recon_once(model, sino):
    np.random.seed(TRANS['seed'])
    rec, _ = model.recon(sino, init_recon=0, max_iterations=TRANS['iterations'], stop_threshold_change_pct=0,
                         logfile_path=None, print_logs=False)
    return rec


def build_batched_workload(device):
    import mbirjax_b200 as mb
    from mbirjax_b200.utilities import gen_ellipsoid_phantom, add_noise, batched_scan_shapes, uniform_angles
    models, sinos = [], []
    for i, (v, r, c) in enumerate(batched_scan_shapes(BATCH['num_scans'])):
        model = mb.ParallelBeamModel((v, r, c), uniform_angles(v))
        model.set_params(sharpness=0.0, snr_db=30.0, granularity=[BATCH['subsets']], partition_sequence=[0],
                         verbose=0)
        phantom = gen_ellipsoid_phantom(model.get_params('recon_shape'), BATCH['ellipsoids'], i, device=device)
        np.random.seed(i)
        sinos.append(add_noise(model.forward_project(phantom), 0.01, i).contiguous())
        models.append(model)
        del phantom
    return models, sinos


def batched_recon(models, sinos):
    from mbirjax_b200.batched import BatchedVCD
    recons, _ = BatchedVCD(models, sinos, seeds=list(range(len(models)))).recon(max_iterations=BATCH['iterations'])
    return recons


def plain_recon(models, sinos):
    recons = []
    for i, (model, sino) in enumerate(zip(models, sinos)):
        np.random.seed(i)
        rec, _ = model.recon(sino, max_iterations=BATCH['iterations'], stop_threshold_change_pct=0,
                             logfile_path=None, print_logs=False)
        recons.append(rec)
    return recons


def batched_roofline(models, sinos, peak_gbs, peak_kind):
    """Average duration of each batched stage of a subset step (CUDA events, the K steps of one iteration), on the
    device state the benchmark's reconstructions use: after one recon() call of the batch, whose refresh built the
    planned forward projections, the stages of steps 0..K-1 are launched one by one.  Also the duration of that
    refresh (chunk boxes and the build of the planned forward projections, once per reconstruction)."""
    import torch
    from mbirjax_b200 import _capi
    from mbirjax_b200 import batched as B
    b = B.BatchedVCD(models, sinos, seeds=list(range(len(models))))
    b.recon(max_iterations=BATCH['iterations'])
    sess = B._SESSIONS[B._batch_key(models, b.weights, BATCH['iterations'])]
    plan, K = sess.plan, sess.num_subsets

    def timed(fn):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        fn()
        e.record()
        torch.cuda.synchronize()
        return s.elapsed_time(e)

    build_ms = timed(lambda: _capi.vcd_batched_refresh(plan))
    times = {k: 0.0 for k in _capi.BATCHED_STAGES}
    for step in range(K):
        for stage, name in enumerate(_capi.BATCHED_STAGES):
            times[name] += timed(lambda: _capi.vcd_batched_stage(plan, step, stage))
    alg = 0.0
    for m, part in zip(models, sess.part):
        V, R, C = m.get_params('sinogram_shape')
        S = m.get_params('recon_shape')[2]
        alg += 4.0 * (V * int(part.shape[1]) * S + V * R * C)
    res = {}
    for name in ('bp', 'fp'):
        ms = times[name] / K
        res[name] = {'ms': ms, 'gbs': alg / (ms * 1e-3) / 1e9}
    dom = max(res, key=lambda k: res[k]['ms'])
    kernel = {'bp': 'b_bp', 'fp': 'b_fp_replay' if sess.planned_forward else 'b_fp'}
    traffic = profile_traffic(kernel[dom])
    share = {k: round(v / sum(times.values()), 4) for k, v in times.items()}
    return {'kernel': kernel[dom], 'bound': 'hbm', 'achieved': round(res[dom]['gbs'], 1), 'peak': peak_gbs,
            'peak_kind': peak_kind, 'unit': 'GB/s', 'frac': round(res[dom]['gbs'] / peak_gbs, 4),
            'traffic': traffic, 'launch_ms': round(res[dom]['ms'], 4), 'alg_bytes_per_launch': alg,
            'other': {kernel[k]: {'launch_ms': round(v['ms'], 4), 'achieved_gbs': round(v['gbs'], 1),
                                  'frac': round(v['gbs'] / peak_gbs, 4)}
                      for k, v in res.items() if k != dom},
            'planned_forward': bool(sess.planned_forward), 'plan_build_ms_per_recon': round(build_ms, 3),
            'stage_time_share': share}


def batched_work(v, r, c, S=None):
    """Algorithmic bytes of one full forward or back projection of a batch scan, 4 V (N S + R C) with N its
    region-of-reconstruction pixel count (the work model that scales a one-scan CPU sample to the batch)."""
    import oracle as O
    n = int(np.sum(O.get_2d_ror_mask((c, c, r))))
    return 4.0 * v * (n * r + r * c)


class CpuBatchedSample:
    """A whole reconstruction of one scan of the batch by the oracle on all host cores, as the plain GPU path
    runs it (tomography_model.py:966-1255): auto-regularisation, partition draws, FBP initialisation with the
    alpha rescale, Hessian diagonal and 10 iterations of 4 subset updates.  The sinogram is the oracle's forward
    projection of the scan's seeded phantom with 1% noise (made once, untimed).  ``run()`` returns the seconds of
    one whole reconstruction; ``scale`` converts it to the 24-scan workload by the work model (the only
    extrapolation: across scans, not within a reconstruction)."""

    def __init__(self, scan=None, workers=None):
        import oracle as O
        from oracle.pool import OraclePool
        from mbirjax_b200.utilities import batched_scan_shapes, gen_ellipsoid_phantom, uniform_angles
        self.scan = BATCH['cpu_sample_scan'] if scan is None else scan
        shapes = batched_scan_shapes(BATCH['num_scans'])
        v, r, c = shapes[self.scan]
        self.shape = (v, r, c)
        self.geom = O.parallel_geometry((v, r, c), uniform_angles(v))
        self.pool = OraclePool(workers=workers)
        ph = gen_ellipsoid_phantom(self.geom.recon_shape, BATCH['ellipsoids'], self.scan).numpy()
        np.random.seed(self.scan)
        sino = self.pool.forward_project(self.geom, ph)
        rng = np.random.default_rng(self.scan + 1000)
        self.sino = (sino + rng.normal(0, 0.01 * np.abs(sino).max(), sino.shape)).astype(np.float32)
        self.scale = sum(batched_work(*sh) for sh in shapes) / batched_work(v, r, c)
        self.workers = self.pool.workers

    def run(self):
        from oracle import vcd as OV
        np.random.seed(self.scan)
        t0 = time.perf_counter()
        OV.recon(self.geom, self.sino, granularity=[BATCH['subsets']], partition_sequence=[0],
                 max_iterations=BATCH['iterations'], sharpness=0.0, snr_db=30.0, stop_threshold_change_pct=0,
                 proj=self.pool)
        return time.perf_counter() - t0

    def describe(self, seconds):
        v, r, c = self.shape
        return ('whole reconstruction of scan %d (%d views x %d rows x %d channels: auto-regularisation, FBP init, '
                'Hessian, %d iterations x %d subsets) by the oracle NumPy port on %d processes, %.2f s, scaled '
                'x%.2f across scans by the 4 V (N S + R C) work model' % (
                    self.scan, v, r, c, BATCH['iterations'], BATCH['subsets'], self.workers, seconds, self.scale))

    def close(self):
        self.pool.close()


def timed_steps(step_fn, steps, warmup, world, flush):
    import torch
    for _ in range(warmup):
        step_fn()
    torch.cuda.synchronize()
    barrier(world)
    torch.cuda.synchronize()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record()
    for _ in range(steps):
        flush()
        step_fn()
    end.record()
    torch.cuda.synchronize()
    barrier(world)
    torch.cuda.synchronize()
    return start.elapsed_time(end)


def autograd_cost(model, sino, phantom, reps=10, label='cone 256x128x256, recon 256x256x128'):
    """One gradient of 0.5 ||W^(1/2) (A x - y)||^2 + qGGMRF(x) through torch.autograd (forward projection, loss,
    backward through the matched back projector in 32-view chunks and the qGGMRF gradient kernel) against one
    forward projection of the same recon.  Data as in the differentiable configuration: y the workload's noisy
    sinogram of its phantom, W = exp(-y / max y), x = half the phantom (an iterate away from the solution).  CUDA
    events, reps repetitions each after warm-ups."""
    import torch
    import mbirjax_b200 as mb
    from mbirjax_b200 import autograd as AG
    y = sino
    w = torch.exp(-y / y.max())
    x = (0.5 * phantom).detach().clone().requires_grad_(True)
    params = (mb.get_b_from_nbr_wts([1, 1, 1]), 0.3, 2.0, 1.2, 1.0)

    def fwd():
        with torch.no_grad():
            AG.forward_project(x, model)

    def grad():
        loss = AG.weighted_ls_qggmrf_loss(x, model, y, w, params, view_chunk=32)
        torch.autograd.grad(loss, x)

    res = {}
    for name, fn in (('fp_ms', fwd), ('grad_ms', grad)):
        for _ in range(2 if reps < 10 else 3):
            fn()
        torch.cuda.synchronize()
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        for _ in range(reps):
            fn()
        e.record()
        torch.cuda.synchronize()
        res[name] = round(s.elapsed_time(e) / reps, 4)
    res['grad_over_fp'] = round(res['grad_ms'] / res['fp_ms'], 3)
    res['config'] = label + ', W = exp(-y / max y), x = phantom / 2, backward in 32-view chunks'
    return res


def kernel_roofline(model, sino, peak_gbs, peak_kind, prefix='cone', spec=CONE, reps=20):
    """Average duration of one VCD subset's back and forward projection (CUDA events, 20 launches each)."""
    import torch
    from mbirjax_b200 import _capi
    import mbirjax_b200 as mb
    g = model._geometry()
    V, R, C = model.get_params('sinogram_shape')
    S = model.get_params('recon_shape')[2]
    np.random.seed(spec['seed'])
    from mbirjax_b200.vcd_utils import morton_sorted_partition
    # the subset in the Z-order the VCD path processes it in
    subset = morton_sorted_partition(mb.gen_pixel_partition(model.get_params('recon_shape'), spec['subsets']),
                                     model.get_params('recon_shape')[1])[0]
    pix = torch.as_tensor(subset, device='cuda')
    n = int(pix.shape[0])
    vox = torch.rand((n, S), device='cuda')
    out_fp = torch.empty((V, R, C), device='cuda')
    out_bp = torch.empty((n, S), device='cuda')
    res = {}
    for name, fn in (('bp_' + prefix, lambda: _capi.back_project(g, sino, pix, out=out_bp)),
                     ('fp_' + prefix, lambda: _capi.forward_project(g, vox, pix, out=out_fp))):
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        for _ in range(reps):
            fn()
        e.record()
        torch.cuda.synchronize()
        ms = s.elapsed_time(e) / reps
        alg_bytes = 4.0 * (V * n * S + V * R * C)
        achieved = alg_bytes / (ms * 1e-3) / 1e9
        res[name] = {'ms': ms, 'alg_bytes': alg_bytes, 'achieved_gbs': achieved}
    dom = max(res, key=lambda k: res[k]['ms'])
    d = res[dom]
    traffic = profile_traffic(dom)
    return {'kernel': dom, 'bound': 'hbm', 'achieved': round(d['achieved_gbs'], 1), 'peak': peak_gbs,
            'peak_kind': peak_kind, 'unit': 'GB/s', 'frac': round(d['achieved_gbs'] / peak_gbs, 4),
            'traffic': traffic, 'launch_ms': round(d['ms'], 4),
            'alg_bytes_per_launch': d['alg_bytes'],
            'other': {k: {'launch_ms': round(v['ms'], 4), 'achieved_gbs': round(v['achieved_gbs'], 1)}
                      for k, v in res.items() if k != dom}}


def profile_traffic(kernel):
    """DRAM bytes per launch of the kernel, from the committed ncu summary (profiles/<kernel>_*.md)."""
    pdir = os.path.join(ROOT, 'profiles')
    if not os.path.isdir(pdir):
        return None
    for fn in sorted(os.listdir(pdir)):
        if fn.startswith(kernel) and fn.endswith('.md'):
            m = re.search(r'traffic_bytes_per_launch:\s*([0-9.eE+]+)', open(os.path.join(pdir, fn)).read())
            if m:
                return float(m.group(1))
    return None


def cpu_reference_sample(workers=None, workload='cone'):
    """One VCD subset update of the workload with the oracle on all host cores; returns (seconds, cores)."""
    import oracle as O
    from oracle.pool import OraclePool, vcd_subset_update_pooled
    if workload == 'translation':
        tv = translation_vectors()
        geom = O.translation_geometry((tv.shape[0], TRANS['rows'], TRANS['channels']), tv, TRANS['sdd'], TRANS['sid'])
        spec = TRANS
    elif workload == 'large':  # evenly spaced views of the large scan: the per-view work is the same
        ang = cone_angles(LARGE)[:: LARGE['views'] // LARGE_CPU_VIEWS][:LARGE_CPU_VIEWS]
        geom = O.cone_geometry((len(ang), LARGE['rows'], LARGE['channels']), ang, LARGE['sdd'], LARGE['sid'],
                               recon_shape=(1024, 1024, 512))
        spec = LARGE
    else:
        geom = O.cone_geometry((CONE['views'], CONE['rows'], CONE['channels']), cone_angles(), CONE['sdd'],
                               CONE['sid'])
        spec = CONE
    nr, nc, ns = geom.recon_shape
    rng = np.random.default_rng(0)
    flat = rng.random((nr * nc, ns)).astype(np.float32) * 0.1
    err = rng.standard_normal(geom.sinogram_shape).astype(np.float32)
    hess = np.full((nr * nc, ns), 1000.0, dtype=np.float32)
    np.random.seed(spec['seed'])
    subset = O.gen_pixel_partition(geom.recon_shape, spec['subsets'])[0]
    params = (O.get_b_from_nbr_wts([1, 1, 1]), 0.05, 2.0, 1.2, 1.0)
    pool = OraclePool(geom, workers)
    try:
        vcd_subset_update_pooled(pool, flat, err, None, hess, subset[:256], 100.0, params)  # start workers
        t0 = time.perf_counter()
        vcd_subset_update_pooled(pool, flat, err, None, hess, subset, 100.0, params)
        dt = time.perf_counter() - t0
    finally:
        pool.close()
    return dt, pool.workers


def cpu_sample_scale(workload):
    """Subset updates of a whole reconstruction per sampled one (the initialisation and Hessian are not counted),
    times the views left out of the large scan's sample."""
    spec = single_scan_spec(workload)[0]
    scale = spec['subsets'] * spec['iterations']
    if workload == 'large':
        scale *= LARGE['views'] / LARGE_CPU_VIEWS
    return scale


# ----------------------------------------------------------------------------------------------- arms
def batched_config(world):
    return {'workload': '%d uneven parallel-beam scans (views U{60..720}, rows U{8..64}, channels U{96..512}, '
                        'seed i), 10 ellipsoids each, %d VCD iterations x %d subsets, FBP init; batched path'
                        % (BATCH['num_scans'], BATCH['iterations'], BATCH['subsets']),
            'num_scans': BATCH['num_scans'], 'iterations': BATCH['iterations'], 'subsets': BATCH['subsets'],
            'parallelism': 'replicas x%d' % world, 'l2': 'flushed before every step (inputs ~1 GB > L2)'}


def translation_config(world):
    tv = translation_vectors()
    return {'workload': 'plain translation VCD, %d x %d translations %g ALU apart (%d views), detector %dx%d, '
                        'sdd=sid=%g, %d iterations x %d subsets, zero init, sharpness %g'
                        % (TRANS['nx'], TRANS['nz'], TRANS['spacing'], tv.shape[0], TRANS['rows'], TRANS['channels'],
                           TRANS['sdd'], TRANS['iterations'], TRANS['subsets'], TRANS['sharpness']),
            'views': int(tv.shape[0]), 'det_rows': TRANS['rows'], 'det_channels': TRANS['channels'],
            'iterations': TRANS['iterations'], 'subsets': TRANS['subsets'], 'parallelism': 'replicas x%d' % world,
            'l2': 'flushed before every step'}


def single_scan_spec(workload):
    """(spec, config function, cpu sample label) of a single-scan workload."""
    if workload == 'translation':
        return TRANS, translation_config, 'the translation scan'
    if workload == 'large':
        return LARGE, large_config, 'the large cone scan on %d of its %d views' % (LARGE_CPU_VIEWS, LARGE['views'])
    return CONE, cone_config, 'the cone scan'


LARGE_CPU_VIEWS = 16  # views of the large cone scan in its CPU sample (evenly spaced; scaled by views)


def large_config(world):
    return {'workload': 'plain cone-beam VCD, sinogram 720x512x1024, recon 1024x1024x512 of 40 ellipsoids, '
                        '%d iterations x %d subsets, FDK init, sdd=sid=4096; plus one FDK and one autograd gradient'
                        % (LARGE['iterations'], LARGE['subsets']),
            'views': LARGE['views'], 'det_rows': LARGE['rows'], 'det_channels': LARGE['channels'],
            'recon_shape': [1024, 1024, 512], 'iterations': LARGE['iterations'], 'subsets': LARGE['subsets'],
            'parallelism': 'replicas x%d' % world, 'l2': 'inputs (1.5 GB sinogram, 2 GiB recon) exceed L2'}


def cone_config(world):
    return {'workload': 'plain cone-beam VCD, sinogram 256x128x256, recon 256x256x128, %d iterations x %d subsets, '
                        'FDK init, sdd=sid=1024' % (CONE['iterations'], CONE['subsets']), 'views': CONE['views'], 'det_rows': CONE['rows'],
            'det_channels': CONE['channels'], 'recon_shape': [256, 256, 128], 'iterations': CONE['iterations'],
            'subsets': CONE['subsets'], 'parallelism': 'replicas x%d' % world, 'l2': 'flushed before every step'}


def run_reference(args):
    world = int(os.environ.get('WORLD_SIZE', '1'))
    rank = int(os.environ.get('RANK', '0'))
    if rank != 0:
        return
    samples, cores, scale = [], None, 1.0
    if args.workload == 'batched':
        # each timed step is one whole oracle reconstruction of one batch scan (about 10-20 s on 16 host
        # processes); the warm-up starts the worker processes and runs one subset update's projections, so that
        # the default 20 timed steps end within a few minutes
        cs = CpuBatchedSample()
        try:
            for _ in range(args.warmup):
                cs.pool.sparse_back_project(cs.geom, cs.sino, np.arange(64, dtype=np.int32))
            for _ in range(args.steps):
                samples.append(cs.run())
        finally:
            cs.close()
        cores, scale = cs.workers, cs.scale
        mean = float(np.mean(samples))
        value = BATCH['num_scans'] / (mean * scale)
        sample = 'per step: ' + cs.describe(mean) + ' (mean of %d steps)' % len(samples)
    else:
        for i in range(args.warmup + args.steps):
            spec = single_scan_spec(args.workload)[0]
            dt, cores = cpu_reference_sample(workload=args.workload)
            scale = cpu_sample_scale(args.workload)
            if i >= args.warmup:
                samples.append(dt)
        mean = float(np.mean(samples))
        value = 1.0 / (mean * scale)
        sample = ('one VCD subset update of %s per step, oracle NumPy port on %d processes, scaled x%.1f to the '
                  'whole reconstruction' % (single_scan_spec(args.workload)[2], cores, scale))
    line = {'impl': 'reference', 'metric': METRIC, 'value': value, 'unit': 'recons/s', 'n_gpus': args.gpus,
            'steps': args.steps, 'warmup': args.warmup, 'ms_per_step': mean * 1e3, 'higher_is_better': True,
            'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f32', 'data': 'synthetic',
            'config': (batched_config(world) if args.workload == 'batched'
                       else single_scan_spec(args.workload)[1](world)),
            'cpu_baseline': {'value': value, 'unit': 'recons/s', 'cores': cores, 'kind': 'port', 'sample': sample},
            'e2e': {'value': value, 'unit': 'recons/s', 'h2d_bytes_per_step': 0, 'd2h_bytes_per_step': 0},
            'note': 'reference JAX CPU path unavailable (jax not installable offline); oracle NumPy port timed'}
    print(json.dumps(line), flush=True)


def run_gpu(args):
    import torch
    from mbirjax_b200 import _capi
    world, rank, local = dist_setup(args.gpus)
    device = torch.device('cuda', local)
    lib = _capi.load_library()
    _capi.set_autotune(args.autotune)
    if args.no_plan_forward:
        from mbirjax_b200 import batched as B
        B.PLAN_FORWARD = False
    peak_gbs, peak_kind = load_peaks()
    flush_buf = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=device)

    def flush():
        flush_buf.zero_()

    if args.workload == 'batched':
        models, sinos = build_batched_workload(device)
        units = BATCH['num_scans']
        config = batched_config(world)

        def step():
            batched_recon(models, sinos)
    elif args.workload == 'translation':
        model, sino, phantom = build_translation_workload(device)
        units = 1
        config = translation_config(world)
        recon_fn = translation_recon_once

        def step():
            recon_fn(model, sino)
    elif args.workload == 'large':
        model, sino, phantom = build_cone_workload(device, LARGE)
        units = 1
        config = large_config(world)

        def recon_fn(m, y):
            return recon_once(m, y, LARGE)

        def step():
            recon_fn(model, sino)
    else:
        model, sino, phantom = build_cone_workload(device)
        units = 1
        config = cone_config(world)
        recon_fn = recon_once

        def step():
            recon_fn(model, sino)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    from mbirjax_b200 import batched as _batched

    def kernel_launches():  # host-submitted launches plus the kernels of replayed batched graphs
        return int(lib.mbx_launch_count()) + _batched.replayed_launches()

    launches0 = kernel_launches()
    ms = timed_steps(step, args.steps, 0, world, flush)
    launches = kernel_launches() - launches0
    clk = clocks.stop()
    ms = max_over_ranks(ms, world)
    value = world * units * args.steps / (ms * 1e-3)
    line = {'metric': METRIC, 'value': sig(value), 'unit': 'recons/s', 'n_gpus': world, 'steps': args.steps,
            'warmup': args.warmup, 'ms_per_step': round(ms / args.steps, 3), 'higher_is_better': True,
            'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f32', 'data': 'synthetic', 'config': config,
            'gpu_launches': int(launches), 'clocks': clk}

    if args.workload == 'batched':
        # the plain per-scan GPU path on the same scans, measured the same way
        for _ in range(1):
            plain_recon(models, sinos)
        p_ms = timed_steps(lambda: plain_recon(models, sinos), args.steps, 0, world, flush)
        p_ms = max_over_ranks(p_ms, world)
        plain_value = world * units * args.steps / (p_ms * 1e-3)
        rb = batched_recon(models, sinos)
        rp = plain_recon(models, sinos)
        diff = max(float(torch.linalg.norm(a - b) / torch.linalg.norm(b)) for a, b in zip(rb, rp))
        line['plain_recons_per_s'] = sig(plain_value)
        line['batched_over_plain'] = round(value / plain_value, 3)
        line['max_rel_l2_batched_vs_plain'] = diff
        del rb, rp

    if not args.no_e2e:
        if args.workload == 'batched':
            host_sinos = [s_.cpu().pin_memory() for s_ in sinos]
            outs = [torch.empty(tuple(m.get_params('recon_shape')), dtype=torch.float32).pin_memory() for m in models]

            def e2e_step():
                recs = batched_recon(models, host_sinos)   # H2D of every sinogram inside the public API
                for o, r in zip(outs, recs):
                    o.copy_(r, non_blocking=True)            # D2H of every recon
            h2d = sum(int(h.numel()) * 4 for h in host_sinos)
            d2h = sum(int(o.numel()) * 4 for o in outs)
        else:
            host_sino = sino.cpu().pin_memory()
            out_host = torch.empty(tuple(model.get_params('recon_shape')), dtype=torch.float32).pin_memory()

            def e2e_step():
                r = recon_fn(model, host_sino)
                out_host.copy_(r, non_blocking=True)
            h2d, d2h = int(host_sino.numel()) * 4, int(out_host.numel()) * 4
        e_ms = timed_steps(e2e_step, args.steps, 1, world, flush)
        e_ms = max_over_ranks(e_ms, world)
        line['e2e'] = {'value': sig(world * units * args.steps / (e_ms * 1e-3)), 'unit': 'recons/s',
                       'h2d_bytes_per_step': h2d, 'd2h_bytes_per_step': d2h}

    if args.workload == 'batched':
        line['roofline'] = batched_roofline(models, sinos, peak_gbs, peak_kind)
    else:
        line['roofline'] = kernel_roofline(model, sino, peak_gbs, peak_kind, args.workload,
                                           single_scan_spec(args.workload)[0],
                                           reps=5 if args.workload == 'large' else 20)

    if args.workload == 'large':
        # one FDK direct recon at this size, the peak device memory of the whole run, and the gradient below
        for _ in range(1):
            model.direct_recon(sino)
        torch.cuda.synchronize()
        s_, e_ = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s_.record()
        model.direct_recon(sino)
        e_.record()
        torch.cuda.synchronize()
        line['fdk_ms'] = round(s_.elapsed_time(e_), 3)
        line['autograd'] = autograd_cost(model, sino, phantom, reps=2,
                                         label='cone 720x512x1024, recon 1024x1024x512')
        line['peak_memory_gb'] = round(torch.cuda.max_memory_allocated(device) / 1e9, 3)
    elif args.workload == 'cone':
        line['autograd'] = autograd_cost(model, sino, phantom)
    elif args.workload == 'batched':
        c_model, c_sino, c_phantom = build_cone_workload(device)
        line['autograd'] = autograd_cost(c_model, c_sino, c_phantom)
        del c_model, c_sino, c_phantom

    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        if args.workload == 'batched':
            cs = CpuBatchedSample()
            try:
                dt = cs.run()
            finally:
                cs.close()
            line['cpu_baseline'] = {'value': sig(units / (dt * cs.scale)), 'unit': 'recons/s',
                                    'cores': cs.workers, 'kind': 'port', 'sample': cs.describe(dt)}
        else:
            spec = single_scan_spec(args.workload)[0]
            dt, cores = cpu_reference_sample(workload=args.workload)
            scale = cpu_sample_scale(args.workload)
            line['cpu_baseline'] = {'value': sig(units / (dt * scale)), 'unit': 'recons/s', 'cores': cores,
                                    'kind': 'port',
                                    'sample': 'one VCD subset update of %s (oracle NumPy port, %d processes), %.2f s, '
                                              'scaled x%.1f to the whole reconstruction' % (
                                                  single_scan_spec(args.workload)[2], cores, dt, scale)}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def main():
    args = parse_args()
    if args.impl == 'reference':
        run_reference(args)
    else:
        run_gpu(args)


if __name__ == '__main__':
    main()

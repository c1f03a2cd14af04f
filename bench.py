'''Benchmark: batched Levenberg-Marquardt fits of 201x201 hologram crops.

A step fits one batch of B = 256 single-sphere features (201x201 crops,
a_p = 0.75 um, n_p = 1.42, z_p = 200 px, noise 0.05, start perturbed by
5 % / +0.02 / +10 px) with the device-resident fitter (FP64 Mie
coefficients, FP32 per-pixel sums, analytic Jacobian, MINPACK LM steps on
the device).  Inputs are synthetic (seeded; see pylorenzmie_b200.workloads).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Prints one JSON line (rank 0).  ``value`` is whole-job features/s with the
inputs resident in HBM; ``e2e`` is the same metric through the public API
on host numpy crops (Optimizer.optimize_stream over the batches: packing,
host-to-device copies, the fits and the device-to-host reads of the
results inside the timed region; e2e.optimize_batch gives the one-call-
per-batch figure).  ``--impl reference`` times the reference algorithm (the
FP64 numpy oracle with scipy's lm fit, all host cores) on a bounded sample
of the same workload.  Multi-GPU runs (torchrun) shard features across
ranks with no data-path collective (weak scaling).
'''
import argparse
import json
import os
import statistics
import sys
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = 'features fitted/s (LM, 201² crops)'
UNIT = 'features/s'
WORKLOAD = ('batched LM fit, 201x201 single-sphere crops (a_p 0.75 um, n_p '
            '1.42, z_p 200 px, start +5%/+0.02/+10 px)')
BATCH = 256
SHAPE = (201, 201)
ROTATE = 4  # distinct input batches cycled through (4 x 41 MB > 126 MB L2)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument('--gpus', type=int, default=1)
    ap.add_argument('--steps', type=int, default=20)
    ap.add_argument('--warmup', type=int, default=3)
    ap.add_argument('--impl', default='b200', choices=['b200', 'reference'])
    ap.add_argument('--batch', type=int, default=BATCH)
    ap.add_argument('--no-cpu-baseline', action='store_true')
    ap.add_argument('--no-extras', action='store_true')
    ap.add_argument('--tile-config', type=int, default=None,
                    help='fixed evaluation launch shape (default: autotune)')
    return ap.parse_args()


def dist_env():
    return (int(os.environ.get('RANK', 0)),
            int(os.environ.get('WORLD_SIZE', 1)),
            int(os.environ.get('LOCAL_RANK', 0)))


# ---------------------------------------------------------------------------
# CPU side: the reference algorithm (oracle) on the host cores

def _import_reference():
    '''Pool initializer: import the reference (baseline/_ref) once per
    worker, before anything is timed.'''
    try:
        _reference_modules()
    except Exception:  # pragma: no cover - reported by the fit itself
        pass


def _reference_modules():
    import types
    ref = ROOT / 'baseline' / '_ref'
    if not (ref / 'pylorenzmie').is_dir():
        return None
    if str(ref) not in sys.path:
        sys.path.insert(0, str(ref))
    sys.modules.setdefault('trackpy', types.ModuleType('trackpy'))
    from pylorenzmie.theory.LorenzMie import LorenzMie
    from pylorenzmie.theory import Sphere, Instrument
    from pylorenzmie.analysis.Optimizer import Optimizer
    from pylorenzmie.analysis.Hologram import Hologram
    return LorenzMie, Sphere, Instrument, Optimizer, Hologram


def _reference_fit_201(data, start):
    '''One 201x201 fit by the reference's own Optimizer, installed in
    baseline/_ref: its numpy LorenzMie (theory/LorenzMie.py) and
    scipy least_squares with the forward-difference Jacobian
    (analysis/Optimizer.py:196-222), default variables and settings.
    Returns the fitted values and success, or None without the install.'''
    import numpy as np
    mods = _reference_modules()
    if mods is None:
        return None
    RefLorenzMie, RefSphere, RefInstrument, RefOptimizer, RefHologram = mods
    inst = RefInstrument()
    inst.magnification, inst.wavelength, inst.n_m = 0.048, 0.447, 1.340
    part = RefSphere()
    part.r_p = list(start[:3])
    part.a_p, part.n_p, part.k_p = start[3], start[4], start[5]
    model = RefLorenzMie(particle=part, instrument=inst)
    opt = RefOptimizer(model=model)
    r = opt.optimize(RefHologram(np.asarray(data).reshape(201, 201)))
    keys = ('x_p', 'y_p', 'z_p', 'a_p', 'n_p')
    return {**{k: float(r[k]) for k in keys}, 'success': bool(r['success'])}


def cpu_fit_rate(nfeat, seed=0, reference=False):
    '''features/s of the oracle fit over a spawn pool of all host cores.
    With reference, the reference's own Optimizer (baseline/_ref) also fits
    the same crops in the same pool; its rate and its largest parameter
    differences from the oracle's fits are returned as a fifth item (None
    without the install).'''
    import multiprocessing as mp
    import numpy as np
    from pylorenzmie_b200 import workloads
    from oracle import bench_tasks
    cores = os.cpu_count() or 1
    truth, start = workloads.batch_201(nfeat, seed)
    # one thread per worker process: BLAS/OpenMP threads would oversubscribe
    for var in ('OMP_NUM_THREADS', 'MKL_NUM_THREADS', 'OPENBLAS_NUM_THREADS'):
        os.environ[var] = '1'
    ctx = mp.get_context('spawn')
    ref = None
    with ctx.Pool(cores,
                  initializer=_import_reference if reference else None) as pool:
        data = pool.starmap(bench_tasks.render_201,
                            [(truth[i], 1000 + i) for i in range(nfeat)])
        t0 = time.perf_counter()
        res = pool.starmap(bench_tasks.fit_201,
                           [(data[i], start[i]) for i in range(nfeat)])
        dt = time.perf_counter() - t0
        if reference:
            t1 = time.perf_counter()
            rres = pool.starmap(_reference_fit_201,
                                [(data[i], start[i]) for i in range(nfeat)])
            rdt = time.perf_counter() - t1
            if all(r is not None for r in rres):
                keys = ('x_p', 'y_p', 'z_p', 'a_p', 'n_p')
                ref = {'value': nfeat / rdt, 'unit': UNIT, 'cores': cores,
                       'kind': 'reference',
                       'sample': f'the same {nfeat} crops, {rdt:.1f} s wall '
                                 f'on {cores} processes',
                       'success_fraction': float(np.mean(
                           [r['success'] for r in rres])),
                       'max_abs_diff_vs_port': {
                           k: float(max(abs(r[k] - o[k])
                                        for r, o in zip(rres, res)))
                           for k in keys}}
    ok = float(np.mean([r['success'] for r in res]))
    if reference:
        return nfeat / dt, cores, dt, ok, ref
    return nfeat / dt, cores, dt, ok


def reference_arm(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    cores = os.cpu_count() or 1
    sample = max(cores, 8)
    for _ in range(max(args.warmup, 0)):
        cpu_fit_rate(sample, seed=7)
    rates, times = [], []
    for k in range(args.steps):
        r, cores, dt, ok = cpu_fit_rate(sample, seed=100 + k)
        rates.append(r)
        times.append(dt)
    value = sample * len(times) / sum(times)
    line = {
        'metric': METRIC, 'value': value, 'unit': UNIT, 'impl': 'reference',
        'n_gpus': world, 'steps': args.steps, 'warmup': args.warmup,
        'ms_per_step': 1e3 * sum(times) / len(times),
        'higher_is_better': True, 'scaling': 'weak', 'vs_baseline': None,
        'dtype': 'f64', 'data': 'synthetic (seeded)',
        'config': {'workload': WORKLOAD + ', FP64 model + scipy lm with a '
                               'forward-difference Jacobian (the reference '
                               'algorithm)',
                   'global_batch': sample, 'crop': '201x201',
                   'sample': f'{sample} features per step (a bounded sample '
                             'of the GPU arm\'s 256-feature batch)',
                   'parallelism': f'{cores} host processes'},
        'cpu_baseline': {'value': value, 'unit': UNIT, 'cores': cores,
                         'kind': 'port',
                         'sample': f'{sample} features per step x '
                                   f'{args.steps} steps, oracle FP64 model '
                                   '+ scipy lm (FD Jacobian)'},
        'e2e': {'value': value, 'unit': UNIT, 'h2d_bytes_per_step': 0,
                'd2h_bytes_per_step': 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
# clocks under load (NVML, read only)

class ClockSampler:
    REASONS = {0x1: 'gpu_idle', 0x2: 'applications_clocks_setting',
               0x4: 'sw_power_cap', 0x8: 'hw_slowdown', 0x10: 'sync_boost',
               0x20: 'sw_thermal_slowdown', 0x40: 'hw_thermal_slowdown',
               0x80: 'hw_power_brake_slowdown'}

    def __init__(self, index):
        self.samples, self.reasons, self.max_mhz = [], 0, None
        self._stop = threading.Event()
        try:
            import pynvml
            pynvml.nvmlInit()
            self.nv = pynvml
            self.h = pynvml.nvmlDeviceGetHandleByIndex(index)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(
                self.h, pynvml.NVML_CLOCK_SM)
        except Exception:
            self.nv = None

    def _run(self):
        nv = self.nv
        while not self._stop.is_set():
            try:
                self.samples.append(nv.nvmlDeviceGetClockInfo(
                    self.h, nv.NVML_CLOCK_SM))
                self.reasons |= int(
                    nv.nvmlDeviceGetCurrentClocksEventReasons(self.h))
            except Exception:
                pass
            time.sleep(0.005)

    def start(self):
        if self.nv is not None:
            self.t = threading.Thread(target=self._run, daemon=True)
            self.t.start()

    def stop(self):
        if self.nv is not None:
            self._stop.set()
            self.t.join()

    def summary(self):
        if not self.samples:
            return {'sm_mhz': None, 'sm_max_mhz': self.max_mhz,
                    'reasons': ['unavailable']}
        return {'sm_mhz': statistics.median(self.samples),
                'sm_max_mhz': self.max_mhz,
                'reasons': [v for k, v in self.REASONS.items()
                            if self.reasons & k],
                'samples': len(self.samples)}


# ---------------------------------------------------------------------------

def b200_arm(args):
    rank, world, local = dist_env()
    cpu_base = None
    if (rank == 0 and world == 1 and not args.no_cpu_baseline):
        # before the first GPU call: the pool uses spawn anyway
        cores = os.cpu_count() or 1
        sample = min(max(2 * cores, 8), 64)
        rate, cores, dt, ok, ref_opt = cpu_fit_rate(sample, seed=3,
                                                    reference=True)
        cpu_base = {'value': rate, 'unit': UNIT, 'cores': cores,
                    'kind': 'port',
                    'sample': f'{sample} features of the same workload, '
                              f'oracle FP64 model + scipy lm (FD Jacobian), '
                              f'{dt:.1f} s wall on {cores} processes',
                    # the reference's own Optimizer on the same crops
                    'reference_optimizer': ref_opt or {
                        'unavailable': 'reference not installed in '
                                       'baseline/_ref'}}

    import ctypes
    import numpy as np
    import torch
    import torch.distributed as tdist
    from pylorenzmie_b200 import _native, workloads, Hologram, Optimizer, \
        LorenzMie, Instrument
    from pylorenzmie_b200.analysis import _fit

    torch.cuda.set_device(local)
    dev = torch.device('cuda', local)
    if world > 1:
        from datetime import timedelta
        tdist.init_process_group('nccl', timeout=timedelta(seconds=120),
                                 device_id=dev)

    def barrier():
        if world > 1:
            tdist.barrier()

    def max_over_ranks(x):
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        tdist.all_reduce(t, op=tdist.ReduceOp.MAX)
        return float(t.item())

    lib = _native.load()
    inst = Instrument()
    variables = ['x_p', 'y_p', 'z_p', 'a_p', 'n_p']
    B = args.batch
    npix = SHAPE[0] * SHAPE[1]

    # device-resident inputs: ROTATE distinct batches
    batches = []
    for r in range(ROTATE):
        seed = 1000 * rank + r
        truth, start = workloads.batch_201(B, seed)
        data = workloads.render(truth, SHAPE, seed=seed, device=dev)
        items = [(data[i].cpu().numpy(), (0., 0., SHAPE[0], SHAPE[1]), None)
                 for i in range(B)]
        packed = _fit.PackedFeatures(items)
        d_feat, d_data, d_coords, d_params = _fit.upload(packed, start, dev)
        cap = _fit.fit_capacity(start, inst.n_m, inst.wavelength)
        batches.append(dict(packed=packed, start=start, truth=truth,
                            d_feat=d_feat, d_data=d_data,
                            d_params0=d_params.clone(), d_params=d_params,
                            cap=cap))

    def step(i, stats=False):
        b = batches[i % ROTATE]
        b['d_params'].copy_(b['d_params0'])
        return _fit.fit_device(b['d_feat'], b['d_data'], None, b['d_params'],
                               B, npix * B, inst, variables, None, b['cap'],
                               b['start'], stats, tile_config=tile_config)

    from pylorenzmie_b200 import autotune
    b0 = batches[0]
    if args.tile_config is None:
        tile_config = autotune.tune(b0['packed'], b0['start'], inst,
                                    variables, b0['cap'], None, dev)
    else:
        tile_config = int(args.tile_config)

    peak = ctypes.c_double()
    _native.check(lib.lmb_measure_fp32_peak(ctypes.byref(peak),
                                            torch.cuda.current_stream().cuda_stream),
                  'lmb_measure_fp32_peak')

    for i in range(args.warmup):
        step(i)
    torch.cuda.synchronize()

    clocks = ClockSampler(torch.cuda.current_device())
    stats = []
    barrier()
    torch.cuda.synchronize()
    clocks.start()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for i in range(args.steps):
        _, fs = step(i, stats=True)
        stats.append(fs)
    e1.record()
    torch.cuda.synchronize()
    clocks.stop()
    barrier()
    ms = max_over_ranks(e0.elapsed_time(e1))
    value = world * B * args.steps / (ms * 1e-3)

    # results of the last timed step: converged?
    res = step(args.steps - 1)[0]
    resv = res[:B * _native.RESULT_DTYPE.itemsize].cpu().numpy().view(
        _native.RESULT_DTYPE)
    success = float(resv['success'].mean())
    nfev = float(resv['nfev'].mean())

    eval_ms = sum(s.eval_ms for s in stats)
    launches = sum(s.eval_launches for s in stats)
    pixels = sum(s.pixels for s in stats)
    porders = sum(s.pixel_orders for s in stats)
    flop_per_launch = (292. * porders + 476. * pixels) / launches
    avg_ms = eval_ms / launches
    achieved = flop_per_launch / (avg_ms * 1e-3) / 1e12
    peak_tf = peak.value / 1e12
    traffic = None
    tfile = ROOT / 'profiles' / 'traffic.json'
    if tfile.exists():
        try:
            t = json.loads(tfile.read_text()).get('k_fit_eval')
            if t:
                traffic = t['bytes_per_launch_full_batch']
        except Exception:
            traffic = None
    roofline = {'bound': 'fp32', 'achieved': achieved, 'peak': peak_tf,
                'unit': 'TFLOP/s', 'frac': achieved / peak_tf,
                'traffic': traffic, 'kernel': 'k_fit_eval',
                'peak_source': 'measured FP32 FMA throughput of this GPU '
                               '(lmb_measure_fp32_peak, same run); '
                               'MEASURED_PEAKS.json has no FP32 CUDA-core '
                               'figure',
                'flop_per_launch': flop_per_launch,
                'avg_launch_ms': avg_ms,
                'work': '292 FLOP per pixel-order + 476 FLOP per pixel '
                        '(value + 6-column Jacobian + normal equations)'}
    gpu_launches = sum(s.kernel_launches for s in stats)

    # end to end through the public API with host crops
    opt = Optimizer(model=LorenzMie(coordinates=np.zeros((2, 1)),
                                    instrument=inst, device=dev))
    host_sets = []
    for r in range(ROTATE):
        b = batches[r]
        holos = [Hologram(b['packed'].data[i * npix:(i + 1) * npix]
                          .reshape(SHAPE).astype(np.float64))
                 for i in range(B)]
        host_sets.append((holos, b['start']))
    # (1) the stream API: batch after batch (frames of a video, say), the
    # host work of one overlapping the fit of the previous
    def stream(n, offset=0):
        return iter([host_sets[(offset + i) % ROTATE] for i in range(n)])
    for _ in opt.optimize_stream(stream(max(args.warmup, 2))):
        pass
    barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    nrows = 0
    for df in opt.optimize_stream(stream(args.steps)):
        nrows += len(df)
    torch.cuda.synchronize()
    e2e_s = max_over_ranks(time.perf_counter() - t0)
    barrier()
    assert nrows == B * args.steps
    # (2) one synchronous optimize_batch call per batch
    for i in range(max(args.warmup, 1)):
        opt.optimize_batch(host_sets[i % ROTATE][0],
                           starts=host_sets[i % ROTATE][1])
    barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for i in range(args.steps):
        df = opt.optimize_batch(host_sets[i % ROTATE][0],
                                starts=host_sets[i % ROTATE][1])
    torch.cuda.synchronize()
    sync_s = max_over_ranks(time.perf_counter() - t0)
    barrier()
    h2d = B * npix * 4 + B * 40 + B * 48
    d2h = B * 48 + B * _native.RESULT_DTYPE.itemsize
    e2e = {'value': world * B * args.steps / e2e_s, 'unit': UNIT,
           'h2d_bytes_per_step': h2d, 'd2h_bytes_per_step': d2h,
           'api': 'Optimizer.optimize_stream(iter of (list[Hologram], '
                  'starts)): host crops in, DataFrames out, pipelined',
           'optimize_batch': {'value': world * B * args.steps / sync_s,
                              'unit': UNIT,
                              'api': 'Optimizer.optimize_batch(list['
                                     'Hologram], starts), one call per '
                                     'batch, synchronous'}}

    extras = {}
    if rank == 0 and world == 1 and not args.no_extras:
        extras = run_extras(dev, inst, value)
    ns = target_figures(value, extras)
    ref_opt = (cpu_base or {}).get('reference_optimizer', {})
    if 'max_abs_diff_vs_port' in ref_opt:
        # the oracle's restatement of the fit against the reference's own
        # Optimizer on the same crops (the pin of the CPU baseline)
        ns['reference_optimizer_vs_oracle_fit_max_abs'] = \
            ref_opt['max_abs_diff_vs_port']

    # the FP32 peak from the clock: SMs x 128 FP32 lanes x 2 FLOP x MHz
    csum = clocks.summary()
    if csum.get('sm_mhz'):
        sms = torch.cuda.get_device_properties(dev).multi_processor_count
        clk_peak = sms * 128 * 2 * csum['sm_mhz'] * 1e6 / 1e12
        roofline['peak_clock_derived'] = clk_peak
        roofline['frac_clock_derived'] = achieved / clk_peak
        roofline['sm_mhz_median'] = csum['sm_mhz']

    if world > 1:
        tdist.destroy_process_group()
    if rank != 0:
        return 0
    line = {
        'metric': METRIC, 'value': value, 'unit': UNIT, 'n_gpus': world,
        'steps': args.steps, 'warmup': args.warmup,
        'ms_per_step': ms / args.steps, 'higher_is_better': True,
        'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f32',
        'data': 'synthetic (seeded); rendered by the FP64 kernel + N(0, 0.05)',
        'config': {'workload': WORKLOAD + ', FP64 Mie coefficients + FP32 '
                               'sums + analytic Jacobian',
                   'global_batch': B * world, 'per_gpu_batch': B,
                   'crop': '201x201', 'parallelism': f'features sharded '
                   f'over {world} GPU(s), no collective',
                   'l2': f'{ROTATE} rotating input batches '
                         f'({ROTATE * B * npix * 4 / 1e6:.0f} MB) > 126 MB L2',
                   'tile_config': tile_config},
        'fit_quality': {'success_fraction': success, 'mean_nfev': nfev},
        'roofline': roofline,
        'cpu_baseline': cpu_base,
        'e2e': e2e,
        'gpu_launches': gpu_launches,
        'clocks': csum,
        'target_figures': ns,
        'extras': extras,
    }
    print(json.dumps(line), flush=True)
    return 0


def run_extras(dev, inst, chosen_value):
    '''Secondary figures on one GPU: the plain-FP64 path, hologram Mpx/s of
    a full frame, and mixed-crop batched fits.'''
    import numpy as np
    import torch
    from scipy.optimize import least_squares
    from pylorenzmie_b200 import workloads, LorenzMie, Hologram, Optimizer
    from pylorenzmie_b200.analysis import _fit
    out = {}

    # plain FP64: FP64 field kernel + forward-difference Jacobian + host LM,
    # one feature at a time (the reference Optimizer's loop on our kernel)
    nplain = 8
    truth, start = workloads.batch_201(nplain, 77)
    data = workloads.render(truth, SHAPE, seed=77, device=dev).cpu().numpy()
    model = LorenzMie(coordinates=LorenzMie.meshgrid(SHAPE), instrument=inst,
                      double_precision=True, device=dev)
    names = ('x_p', 'y_p', 'z_p', 'a_p', 'n_p')

    def plain_fit(d, s):
        def resid(v):
            model.properties = dict(zip(names, v))
            return (model.hologram() - d) / inst.noise
        model.particle = workloads.spheres(s)[0]
        return least_squares(resid, s[:5], method='lm', ftol=1e-4, xtol=1e-6,
                             gtol=1e-6, max_nfev=2000, diff_step=1e-5,
                             x_scale='jac')
    plain_fit(data[0].ravel().astype(float), start[0])  # warm-up
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for i in range(nplain):
        plain_fit(data[i].ravel().astype(float), start[i])
    plain = nplain / (time.perf_counter() - t0)
    out['plain_fp64_gpu'] = {
        'value': plain, 'unit': UNIT,
        'method': 'FP64 field kernel + forward-difference Jacobian + host '
                  'scipy lm, one feature at a time',
        'chosen_over_plain': chosen_value / plain}

    # the reference's own GPU path for holograms beside ours
    out['reference_gpu_batch_hologram'] = reference_batch_hologram(dev)

    # hologram throughput of a 1280x1024 frame with 16 spheres
    p = workloads.bench_frame()
    frames = {}
    for fp64 in (False, True):
        m = LorenzMie(coordinates=LorenzMie.meshgrid((1024, 1280)),
                      particle=workloads.spheres(p), instrument=inst,
                      double_precision=fp64, device=dev)
        frames[fp64] = m.hologram(device=True).double()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        reps = 10
        e0.record()
        for _ in range(reps):
            m.hologram(device=True)
        e1.record()
        torch.cuda.synchronize()
        sec = e0.elapsed_time(e1) / reps * 1e-3
        out['frame_fp64' if fp64 else 'frame_fp32'] = {
            'value': 1280 * 1024 * p.shape[0] / sec / 1e6,
            'unit': 'Mpx/s (pixel-particles)', 'spheres': int(p.shape[0]),
            'ms_per_frame': sec * 1e3}
    diff = (frames[False] - frames[True]).abs()
    out['frame_fp32']['max_abs_error_vs_fp64'] = float(diff.max())
    out['frame_fp32']['max_rel_error_vs_fp64'] = float(
        (diff / frames[True].abs().clamp_min(1.)).max())
    out['frame_fp32']['max_hologram'] = float(frames[True].max())

    # differentiation workload: 64 crops of 401x401, a_p 3-6 um
    from pylorenzmie_b200.theory import autograd as ag
    from pylorenzmie_b200.theory import _kernels as K
    P = torch.tensor(workloads.large(64, seed=11), dtype=torch.float64,
                     device=dev)
    coords = LorenzMie.meshgrid((401, 401))
    ag.jacobian(P, coords)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    H, J = ag.jacobian(P, coords)
    torch.cuda.synchronize()
    tj = time.perf_counter() - t0
    Pg = P.clone().requires_grad_(True)
    d = (H.float() + 0.05 * torch.randn(H.shape, device=dev)).detach()
    ((ag.hologram(Pg, coords) - d) ** 2).sum().backward()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    Pg.grad = None
    ((ag.hologram(Pg, coords) - d) ** 2).sum().backward()
    torch.cuda.synchronize()
    tg = time.perf_counter() - t0
    out['jacobian_401'] = {
        'value': 64 / tj, 'unit': 'Jacobian evaluations/s (401x401 crop, '
                                  '6 columns)',
        'grad_chi2_per_s': 64 / tg,
        'mean_nmax': float(K.wiscombe_yang(
            P[:, 3].cpu().numpy(), P[:, 4].cpu().numpy(), 0., inst.n_m,
            inst.wavelength).mean())}
    del H, J

    # layered spheres from a video stream: frames of 32 features each,
    # 8 frames per device batch, four distinct batches pipelined by
    # optimize_stream (its default for layered streams: 4 fits at once)
    nbatch = 4
    stream_sets = []
    for b in range(nbatch):
        sb = workloads.layered(256, seed=13 + b)
        pb = workloads.layered_spheres(sb[1], sb[3], sb[4])
        ib = workloads.render_particles(pb, [(s, s) for s in sb[0]],
                                        seed=13 + b, device=dev)
        stream_sets.append(
            (sb, ib, ([Hologram(im.astype(np.float64)) for im in ib],
                      workloads.layered_spheres(sb[2], sb[3], sb[4]))))
    sides, truth, start, frac, core = stream_sets[0][0]
    imgs = stream_sets[0][1]
    opt = Optimizer(model=LorenzMie(coordinates=np.zeros((2, 1)),
                                    instrument=inst, device=dev))
    for _ in opt.optimize_stream(iter([stream_sets[0][2]])):
        pass
    # three timed passes over the same four batches (the fits are
    # deterministic); the median is reported, with the spread
    runs = []
    for _ in range(3):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        dfs = list(opt.optimize_stream(iter([x[2] for x in stream_sets])))
        torch.cuda.synchronize()
        runs.append(time.perf_counter() - t0)
    dt = float(np.median(runs))
    df = dfs[0]
    err = np.abs(df['a_p'].to_numpy() - truth[:, 3])
    sub = list(range(0, 256, 32))          # one feature per frame
    ref = oracle_fits([(imgs[i], (sides[i], sides[i]), start[i], frac[i],
                        core[i]) for i in sub])
    out['layered_stream_e2e'] = {
        'value': 256 * nbatch / dt, 'unit': UNIT,
        'frames_per_s': 8 * nbatch / dt,
        'runs_features_per_s': [256 * nbatch / t for t in runs],
        'api': 'Optimizer.optimize_stream, 4 distinct batches of 8 frames x '
               '32 features (median of 3 timed passes)',
        'max_nfev_per_batch': [int(d['nfev'].max()) for d in dfs],
        'features': 256 * nbatch, 'layers': 3,
        'success_fraction': float(df['success'].mean()),
        'mean_nfev': float(df['nfev'].mean()),
        'max_nfev': int(df['nfev'].max()),
        'median_abs_a_p_error_vs_truth_um': float(np.median(err)),
        'vs_oracle_fit': compare_fits(df.iloc[sub].reset_index(drop=True),
                                      ref),
        'per_feature': layered_parity(opt, inst, dev, imgs, sides, start,
                                      frac, core, sub, df, ref)}

    # global estimates of a frame's features (DEEstimator defaults: 2 % of
    # each 121x121 crop's pixels, popsize 10, tol 0.01): the searches side
    # by side (Frame.estimate, one lmb_chi2_crops launch per generation of
    # all of them) against one feature at a time (one lmb_chi2_batch
    # launch per generation of each), both with and without scipy's own
    # per-candidate code (a callback that never stops the search selects
    # it), and the
    # oracle's numpy search
    from pylorenzmie_b200 import Frame
    from oracle import estimate as oest, field as ofield
    nest = 32
    P, fdata, boxes = workloads.estimate_frame(nest, 21, inst, dev)

    def _no_stop(xk, convergence):
        return False

    def estimate_frame(side, scipy_code=False, device=False):
        f = Frame(instrument=inst)
        f.data = fdata
        f.bboxes = boxes
        for i, feat in enumerate(f.features):
            feat.estimator.seed = 40 + i
            feat.estimator.device_search = device
            if scipy_code:
                feat.estimator.settings = dict(feat.estimator.settings,
                                               callback=_no_stop)
        np.random.seed(41)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        if side:
            f.estimate()
        else:
            for feat in f.features:
                feat.estimate()
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        return dt, np.array([[ft.particle.z_p, ft.particle.a_p,
                              ft.particle.n_p] for ft in f.features]), f
    estimate_frame(True)                           # warm-up
    # three passes over the same inputs (estimates, then the rest of the
    # reference's frame workflow, Frame.analyze without detection: every
    # estimated feature fitted in one device call); medians reported
    sides, fits = [], []
    for rep in range(3):
        t_s, est_s, f_s = estimate_frame(True)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        res_s = f_s.optimize()
        torch.cuda.synchronize()
        sides.append(t_s)
        fits.append(time.perf_counter() - t0)
        if rep == 0:
            est_side, f, fres = est_s, f_s, res_s
    t_side, t_fit = float(np.median(sides)), float(np.median(fits))
    t_one, est_one, _ = estimate_frame(False)
    estimate_frame(True, device=True)                 # warm-up
    t_dev, est_dev, _ = estimate_frame(True, device=True)
    t_side_sp, est_side_sp, _ = estimate_frame(True, True)
    t_one_sp, est_one_sp, _ = estimate_frame(False, True)
    nref = 2
    np.random.seed(41)
    t0 = time.perf_counter()
    for ft in f.features[:nref]:
        oest.de_estimate(ft.data, ft.coordinates,
                         dict(zip(('x_p', 'y_p', 'z_p', 'a_p', 'n_p', 'k_p'),
                                  [0., 0., 100., 1., 1.5, 0.])),
                         ofield.DEFAULT_INSTRUMENT, exclude=ft.mask.exclude,
                         seed=40 + f.features.index(ft))
    t_ref = time.perf_counter() - t0
    out['frame_estimate'] = {
        'value': nest / t_side, 'unit': 'feature estimates/s',
        'api': 'Frame.estimate, 32 features of 121x121 px, DEEstimator '
               'defaults, searches side by side',
        'one_by_one_per_s': nest / t_one,
        'scipy_code_side_by_side_per_s': nest / t_side_sp,
        'scipy_code_one_by_one_per_s': nest / t_one_sp,
        'identical_all_four': bool(
            np.array_equal(est_side, est_one) and
            np.array_equal(est_side, est_side_sp) and
            np.array_equal(est_side, est_one_sp)),
        'oracle_numpy_per_s': nref / t_ref,
        'median_abs_a_p_error_vs_truth_um': float(
            np.median(np.abs(est_side[:, 1] - P[:, 3]))),
        'device_search': {
            'per_s': nest / t_dev,
            'api': 'the same estimators with device_search=True (the '
                   'search on the GPU, its own random stream)',
            'median_abs_a_p_error_vs_truth_um': float(
                np.median(np.abs(est_dev[:, 1] - P[:, 3]))),
            'median_abs_z_p_error_vs_truth_px': float(
                np.median(np.abs(est_dev[:, 0] - P[:, 2]))),
            'scipy_median_abs_z_p_error_vs_truth_px': float(
                np.median(np.abs(est_side[:, 0] - P[:, 2])))},
        'then_frame_optimize': {
            'features_per_s': nest / t_fit,
            'runs_features_per_s': [nest / t for t in fits],
            'estimate_plus_optimize_frames_per_s': 1. / (t_side + t_fit),
            'success_fraction': float(fres['success'].mean()),
            'median_abs_a_p_error_vs_truth_um': float(np.median(np.abs(
                fres['a_p'].to_numpy() - P[:, 3])))}}

    # spherical aberration (s = 1.5 wavelengths, fixed: a calibrated
    # instrument): 256 aberrated 201x201 crops through optimize_batch,
    # beside the ideal model on the ideal rendering of the same spheres
    from pylorenzmie_b200 import AberratedLorenzMie
    truth, start = workloads.batch_201(256, seed=31)
    grid = LorenzMie.meshgrid(SHAPE)
    ma = AberratedLorenzMie(coordinates=grid, instrument=inst, spherical=1.5,
                            double_precision=True, device=dev)
    ha = ma.batch_hologram([[s] for s in workloads.spheres(truth)],
                           device=True)
    gen = torch.Generator(device=dev)
    gen.manual_seed(31)
    ha = (ha + inst.noise * torch.randn(ha.shape, generator=gen, device=dev,
                                        dtype=ha.dtype)).cpu().numpy()
    holo_a = [Hologram(ha[i].reshape(SHAPE)) for i in range(256)]
    hi = workloads.render(truth, SHAPE, seed=31, device=dev).cpu().numpy()
    holo_i = [Hologram(hi[i].astype(np.float64)) for i in range(256)]
    opt_a = Optimizer(model=AberratedLorenzMie(
        coordinates=np.zeros((2, 1)), instrument=inst, spherical=1.5,
        device=dev))
    opt_a.fixed = opt_a.fixed + ['spherical']
    opt_i = Optimizer(model=LorenzMie(coordinates=np.zeros((2, 1)),
                                      instrument=inst, device=dev))
    rates = {}
    for name, o, hs in (('aberrated', opt_a, holo_a), ('ideal', opt_i, holo_i)):
        o.optimize_batch(hs, starts=start)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        reps = 3
        for _ in range(reps):
            df = o.optimize_batch(hs, starts=start)
        torch.cuda.synchronize()
        rates[name] = (256 * reps / (time.perf_counter() - t0), df)
    dfa = rates['aberrated'][1]
    out['aberrated_fit'] = {
        'value': rates['aberrated'][0], 'unit': UNIT,
        'api': 'Optimizer.optimize_batch, AberratedLorenzMie (spherical 1.5 '
               'fixed), 256 x 201x201 crops',
        'ideal_same_call_per_s': rates['ideal'][0],
        'success_fraction': float(dfa['success'].mean()),
        'mean_nfev': float(dfa['nfev'].mean()),
        'median_abs_a_p_error_vs_truth_um': float(np.median(np.abs(
            dfa['a_p'].to_numpy() - truth[:, 3]))),
        'median_abs_z_p_error_vs_truth_px': float(np.median(np.abs(
            dfa['z_p'].to_numpy() - truth[:, 2])))}

    # mixed crop sizes 51..301, 256 features per launch
    sides, truth, start = workloads.mixed_crops(256, seed=9)
    holos, raw = [], []
    for i in range(256):
        s = int(sides[i])
        d = workloads.render(truth[i:i + 1], (s, s), seed=i, device=dev)[0]
        raw.append(d.cpu().numpy().astype(np.float64))
        holos.append(Hologram(raw[-1]))
    opt = Optimizer(model=LorenzMie(coordinates=np.zeros((2, 1)),
                                    instrument=inst, device=dev))
    opt.optimize_batch(holos, starts=start)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    reps = 5
    for _ in range(reps):
        df = opt.optimize_batch(holos, starts=start)
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    sub = list(range(0, 256, 16))
    ref = oracle_fits([(raw[i], (sides[i], sides[i]), start[i], None, None)
                       for i in sub])
    out['mixed_crops_e2e'] = {
        'value': 256 * reps / dt, 'unit': UNIT,
        'success_fraction': float(df['success'].mean()),
        'mean_pixels': float(np.mean(sides.astype(float) ** 2)),
        'vs_oracle_fit': compare_fits(df.iloc[sub].reset_index(drop=True),
                                      ref)}
    return out


def reference_batch_hologram(dev, reps=5):
    '''The reference's batched GPU holograms (TorchLorenzMieBatch.batch_
    hologram: host Mie coefficients, one Triton launch per particle slot,
    theory/torchLorenzMieBatch.py:258-431) against ours through the same
    public call, on the reference's speed example (128 holograms of the
    same 4 spheres, 201x201 px, devel/speed_example.py).  Both return numpy
    float64 (B, npts); timed end to end, synchronized.  Runs the reference
    installed in baseline/_ref.'''
    import types
    import numpy as np
    import torch
    ref = ROOT / 'baseline' / '_ref'
    if not (ref / 'pylorenzmie').is_dir():
        return {'unavailable': 'reference not installed in baseline/_ref'}
    if str(ref) not in sys.path:
        sys.path.insert(0, str(ref))
    sys.modules.setdefault('trackpy', types.ModuleType('trackpy'))
    try:
        from pylorenzmie.theory.torchLorenzMieBatch import \
            TorchLorenzMieBatch
        from pylorenzmie.theory import Sphere as RefSphere
        from pylorenzmie.theory import Instrument as RefInstrument
    except Exception as e:  # pragma: no cover - missing dependency
        return {'unavailable': f'reference import failed: {e!r}'}
    from pylorenzmie_b200 import LorenzMie, Sphere, Instrument
    spheres = [(100, 100, 200, 0.5, 1.45), (80, 120, 300, 1.0, 1.40),
               (150, 50, 250, 0.75, 1.42), (60, 160, 350, 1.2, 1.43)]
    shape, N = (201, 201), 128

    def make(cls):
        out = []
        for x, y, z, a, n in spheres:
            p = cls()
            p.r_p = [x, y, z]
            p.a_p, p.n_p = a, n
            out.append(p)
        return out

    rinst = RefInstrument()
    rinst.magnification, rinst.wavelength, rinst.n_m = 0.048, 0.447, 1.340
    rmodel = TorchLorenzMieBatch(
        coordinates=TorchLorenzMieBatch.meshgrid(shape), instrument=rinst)
    rlists = [make(RefSphere)] * N
    bmodel = LorenzMie(coordinates=LorenzMie.meshgrid(shape),
                       instrument=Instrument(), device=dev)
    blists = [make(Sphere)] * N

    def timed(fn):
        fn()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(reps):
            h = fn()
        torch.cuda.synchronize()
        return h, (time.perf_counter() - t0) / reps

    href, tref = timed(lambda: rmodel.batch_hologram(rlists))
    hb, tb = timed(lambda: bmodel.batch_hologram(blists))
    px = N * len(spheres) * shape[0] * shape[1]
    return {'shape': '128 x 4 spheres x 201x201',
            'reference_ms': tref * 1e3, 'b200_ms': tb * 1e3,
            'reference_mpx_per_s': px / tref / 1e6,
            'b200_mpx_per_s': px / tb / 1e6, 'speedup': tref / tb,
            'max_abs_diff': float(np.abs(href - hb).max()),
            'max_abs_hologram': float(np.abs(hb).max())}


TIGHT = {'method': 'lm', 'ftol': 1e-10, 'xtol': 1e-10, 'gtol': 1e-10,
         'loss': 'linear', 'max_nfev': 2000, 'diff_step': 1e-5,
         'x_scale': 'jac'}
FIT_TARGETS = {'x_p': 0.02, 'y_p': 0.02, 'z_p': 0.02, 'a_p': 1e-3,
               'n_p': 1e-4}


def layered_parity(opt, inst, dev, imgs, sides, start, frac, core, sub, df,
                   ref):
    '''Per feature of the layered subset: device and oracle reduced chi^2
    and whether the fits meet the targets, with the default settings and
    converged tightly (ftol = xtol = gtol = 1e-10) from the same starts.
    Where the tight fits still differ, the oracle is restarted from the
    device's point: if it stays there (within the targets, chi^2 no lower)
    both share that minimum and the first oracle fit stopped short of it.'''
    import numpy as np
    from pylorenzmie_b200 import Optimizer, LorenzMie, Hologram, workloads
    opt_t = Optimizer(model=LorenzMie(coordinates=np.zeros((2, 1)),
                                      instrument=inst, device=dev),
                      settings=dict(TIGHT))
    dft = opt_t.optimize_batch(
        [Hologram(imgs[i].astype(np.float64)) for i in sub],
        particles=workloads.layered_spheres(start[sub], frac[sub], core[sub]))
    ref_t = oracle_fits([(imgs[i], (sides[i], sides[i]), start[i], frac[i],
                          core[i], TIGHT) for i in sub])

    def meets(d, o):
        return all(abs(float(d[k]) - o[k]) <= t
                   for k, t in FIT_TARGETS.items())

    rows, again = [], []
    for j, i in enumerate(sub):
        d0 = df.iloc[i]
        d1 = dft.iloc[j]
        row = {'feature': int(i),
               'default': {'device_redchi': float(d0['redchi']),
                           'oracle_redchi': ref[j]['redchi'],
                           'meets_targets': meets(d0, ref[j])},
               'tight': {'device_redchi': float(d1['redchi']),
                         'oracle_redchi': ref_t[j]['redchi'],
                         'oracle_status': ref_t[j]['status'],
                         'meets_targets': meets(d1, ref_t[j])}}
        if not row['tight']['meets_targets']:
            p = start[i].copy()
            for n, k in enumerate(('x_p', 'y_p', 'z_p', 'a_p', 'n_p')):
                p[n] = float(d1[k])
            again.append((j, (imgs[i], (sides[i], sides[i]), p, frac[i],
                              core[i], TIGHT)))
        rows.append(row)
    if again:
        res = oracle_fits([t for _, t in again])
        for (j, _), r in zip(again, res):
            d1 = dft.iloc[j]
            rows[j]['tight']['oracle_restarted_at_device'] = {
                'redchi': r['redchi'], 'status': r['status'],
                'meets_targets': meets(d1, r)}
    shared = sum(1 for r in rows if r['tight']['meets_targets'] or
                 r['tight'].get('oracle_restarted_at_device', {})
                 .get('meets_targets', False))
    return {'features': len(rows),
            'meet_targets_default': sum(r['default']['meets_targets']
                                        for r in rows),
            'meet_targets_tight': sum(r['tight']['meets_targets']
                                      for r in rows),
            'same_minimum_tight': shared, 'rows': rows}


def target_figures(chosen, extras):
    '''The target figures of the hot path, beside their targets: the
    chosen form against plain FP64 on the same GPU, the FP32 frame
    hologram's error against FP64, and the fits against the oracle's.'''
    ns = {'chosen_features_per_s': chosen,
          'targets': {'chosen_over_plain': 50., 'hologram_abs_error': 2e-5,
                      'a_p_um': 1e-3, 'n_p': 1e-4, 'z_p_px': 0.02}}
    if not extras:
        return ns
    plain = extras.get('plain_fp64_gpu', {})
    ns['plain_fp64_gpu_features_per_s'] = plain.get('value')
    ns['chosen_over_plain'] = plain.get('chosen_over_plain')
    refgpu = extras.get('reference_gpu_batch_hologram', {})
    if 'speedup' in refgpu:
        ns['batch_hologram_vs_reference_triton'] = {
            k: refgpu[k] for k in ('reference_mpx_per_s', 'b200_mpx_per_s',
                                   'speedup', 'max_abs_diff')}
    frame = extras.get('frame_fp32', {})
    ns['frame_fp32_mpx_per_s'] = frame.get('value')
    ns['frame_fp32_max_abs_error_vs_fp64'] = frame.get(
        'max_abs_error_vs_fp64')
    for key in ('mixed_crops_e2e', 'layered_stream_e2e'):
        cmp = extras.get(key, {}).get('vs_oracle_fit')
        if cmp:
            ns[key + '_vs_oracle_fit_max_abs'] = {
                k: cmp[k]['max_abs'] for k in ('x_p', 'y_p', 'z_p', 'a_p',
                                                'n_p')}
    per = extras.get('layered_stream_e2e', {}).get('per_feature')
    if per:
        ns['layered_subset_same_minimum'] = {
            k: per[k] for k in ('features', 'meet_targets_default',
                                'meet_targets_tight', 'same_minimum_tight')}
    return ns


def oracle_fits(tasks):
    '''The reference fitting algorithm (oracle) on a subset of crops,
    over a spawn pool of the host cores: tasks of (data, shape, start,
    fractions or None, core indices or None).'''
    import multiprocessing as mp
    from oracle import bench_tasks
    for var in ('OMP_NUM_THREADS', 'MKL_NUM_THREADS', 'OPENBLAS_NUM_THREADS'):
        os.environ[var] = '1'
    with mp.get_context('spawn').Pool(min(len(tasks), os.cpu_count() or 1)
                                      ) as pool:
        return pool.starmap(bench_tasks.fit_crop, tasks)


def compare_fits(df, ref):
    '''Largest |device - oracle| per fitted parameter over a subset, in
    its units and in units of the oracle's uncertainty.'''
    import numpy as np
    out = {'features': len(ref),
           'oracle_success': float(np.mean([r['success'] for r in ref])),
           'max_redchi_rel_diff': float(np.max(np.abs(
               df['redchi'].to_numpy() / np.array([r['redchi'] for r in ref])
               - 1.)))}
    for k in ('x_p', 'y_p', 'z_p', 'a_p', 'n_p'):
        d = np.abs(df[k].to_numpy() - np.array([r[k] for r in ref]))
        sig = np.array([r['d' + k] for r in ref])
        out[k] = {'max_abs': float(d.max()),
                  'max_in_sigma': float((d / np.maximum(sig, 1e-300)).max())}
    return out


def main():
    args = parse()
    if args.impl == 'reference':
        return reference_arm(args)
    return b200_arm(args)


if __name__ == '__main__':
    sys.exit(main())

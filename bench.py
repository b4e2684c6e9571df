"""Benchmark: P_ell spectra/s of the mesh power-spectrum path on B200.

Workload (one step = one spectrum): a lognormal mock on a 512^3 mesh in a 1000 Mpc/h
box, P(k) = 2e4 (k/0.1)^-1.5 exp(-(k/0.5)^2), Poisson-sampled at nbar = 5e-3
(~5e6 float32 positions, unit weights); paint TSC with interlacing 3 and compensation,
global line of sight 'z', ells (0, 2, 4), k edges step 0.005 up to k_Nyq.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints one JSON line (rank 0).  ``value``: spectra/s with positions resident in HBM;
``e2e``: the same through the public API with positions copied from pinned host
memory every step and the multipoles read back.  ``--impl reference`` times the
CPU oracle (a NumPy/SciPy restatement of the reference's JAX code, which cannot run
here: no jax) on a bounded sample of the same workload.  Multi-GPU runs are
replicas (weak scaling): each rank computes its own spectra, no collective on the
data path.
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
for _p in (ROOT, os.path.join(ROOT, 'jax-power_b200')):
    if _p not in sys.path:
        sys.path.insert(0, _p)

METRIC = 'P_l spectra/s @512^3 (batched+learned vs plain GPU, <=1e-3 rel); %HBM peak'
WORKLOAD = dict(workload='lognormal mock 512^3, ~5e6 particles, TSC, interlacing 3, compensate, los z, '
                         'ells (0,2,4), k step 0.005', meshsize=512, boxsize=1000., nbar=5e-3, resampler='tsc',
                interlacing=3, compensate=True, los='z', ells=[0, 2, 4], k_step=0.005, seed=42)

# kernel launches issued by each C-ABI entry point (ours, including CUB's scan kernels)
LAUNCHES = {'pk_paint': 5, 'pk_interlace_compensate': 1, 'pk_bin_global': 2, 'pk_bin_firstpoint': 2,
            'pk_bin_modes': 2, 'pk_bin_mesh': 2, 'pk_scale_real': 1, 'pk_ylm_premultiply': 1, 'pk_read': 1}


def measured_peaks():
    path = os.path.join(ROOT, 'MEASURED_PEAKS.json')
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d['hbm_gbs']), 'measured'
    return 6650., 'fallback'


def algorithmic_bytes(name, npart, meshsize, interlacing, nells):
    nr = float(meshsize)**3
    nc = float(meshsize)**2 * (meshsize // 2 + 1)
    if name == 'pk_paint':  # read positions (+weights) once, write one float32 mesh per shift
        return 16. * npart + 4. * nr * interlacing
    if name == 'pk_interlace_compensate':
        return 8. * nc * (interlacing + 1)
    if name in ('pk_bin_global', 'pk_bin_mesh'):
        return 8. * nc
    return None


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    FIELDS = ('clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,'
              'clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,'
              'clocks_event_reasons.sw_power_cap')

    def __init__(self, index):
        self.index = index
        self.proc = None

    def __enter__(self):
        self.file = tempfile.NamedTemporaryFile('w+', suffix='.csv', delete=False)
        try:
            self.proc = subprocess.Popen(['nvidia-smi', '-i', str(self.index), '--query-gpu=' + self.FIELDS,
                                          '--format=csv,noheader,nounits', '-lms', '100'],
                                         stdout=self.file, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        self.file.flush()
        rows = []
        with open(self.file.name) as f:
            for line in f:
                parts = [p.strip() for p in line.split(',')]
                if len(parts) == 7:
                    rows.append(parts)
        os.unlink(self.file.name)
        if not rows:
            return {'sm_mhz': None, 'sm_max_mhz': None, 'reasons': ['unsampled']}
        sm = [float(r[0]) for r in rows if r[0].replace('.', '').isdigit()]
        names = ['hw_slowdown', 'hw_thermal_slowdown', 'sw_thermal_slowdown', 'sw_power_cap']
        reasons = sorted({n for r in rows for n, v in zip(names, r[3:]) if v.lower().startswith('active')})
        return {'sm_mhz': float(np.median(sm)) if sm else None, 'sm_max_mhz': float(rows[0][1]),
                'power_w_max': max(float(r[2]) for r in rows if r[2].replace('.', '').isdigit()),
                'samples': len(rows), 'reasons': reasons}


# ----------------------------------------------------------------------------- CPU arm

def cpu_sample(meshsize=256, seed=0):
    """Time the oracle's float32 pipeline on a scaled sample of the workload; return
    (seconds extrapolated to one full 512^3 spectrum, description, threads)."""
    from oracle.coords import Geometry
    from oracle import paint as opaint
    from oracle.spectrum import Bins, compute_mesh2_spectrum
    full = WORKLOAD['meshsize']
    scale_n = (full / meshsize)**3
    npart = int(round(5.0e6 / scale_n))
    rng = np.random.default_rng(seed)
    box = WORKLOAD['boxsize']
    pos = (rng.uniform(-0.5, 0.5, (npart, 3)) * box).astype('f4')
    geom = Geometry(meshsize, box, 0.)
    t0 = time.perf_counter()
    mesh = opaint.paint(geom, pos, None, 'tsc', 3, True, 'complex')
    t1 = time.perf_counter()
    bins = Bins(geom, step=WORKLOAD['k_step'], ells=(0, 2, 4))
    t2 = time.perf_counter()
    compute_mesh2_spectrum(mesh, bins, los='z', accum='f64')
    t3 = time.perf_counter()
    # paint+FFT scale with N_p and N log N, binning with the number of modes
    fft_factor = scale_n * np.log(full**3) / np.log(meshsize**3)
    seconds = (t1 - t0) * fft_factor + (t3 - t2) * scale_n
    desc = ('oracle float32 pipeline (numpy serial paint, scipy.fft workers=all) on a {m}^3 mesh with {n} '
            'uniform particles ({f:.0f}x fewer cells/particles), per-stage times scaled to 512^3 / 5e6 '
            '(paint+FFT by N log N, binning by modes); bin setup excluded').format(m=meshsize, n=npart, f=scale_n)
    return seconds, desc, os.cpu_count()


def run_reference(args):
    rank = int(os.environ.get('RANK', 0))
    if rank != 0:
        return
    times = []
    for step in range(args.warmup + args.steps):
        seconds, desc, cores = cpu_sample(meshsize=args.cpu_meshsize, seed=step)
        if step >= args.warmup:
            times.append(seconds)
    value = 1. / float(np.mean(times))
    line = {'impl': 'reference', 'metric': METRIC, 'value': value, 'unit': 'spectra/s', 'n_gpus': args.gpus,
            'steps': args.steps, 'warmup': args.warmup, 'ms_per_step': 1e3 / value, 'higher_is_better': True,
            'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f32', 'data': 'synthetic', 'config': WORKLOAD,
            'cpu_baseline': {'value': value, 'unit': 'spectra/s', 'cores': cores, 'kind': 'port', 'sample': desc},
            'e2e': {'value': value, 'unit': 'spectra/s', 'h2d_bytes_per_step': 0, 'd2h_bytes_per_step': 0}}
    print(json.dumps(line), flush=True)


# ----------------------------------------------------------------------------- batched mocks

BATCHED = dict(workload='256 lognormal periodic mocks, N_p log-uniform in [1e5, 4e6], meshsize in {128, 192, 256}, '
                        'box 1000, TSC, interlacing 2, compensate, los z, ells (0,2,4), k step 0.005 up to k_Nyq(128)',
               nmocks=256, meshsizes=[128, 192, 256], np_range=[1e5, 4e6], boxsize=1000., interlacing=2, seed=7)


def run_batched(nmocks=256, fp64_subset=3, group=32):
    """Plain per-mock GPU loop vs batched launches (CUDA graph) on the same mocks."""
    import torch
    import jaxpower_b200 as jp
    from jaxpower_b200.mock import lognormal_particles, power_law_pk
    from jaxpower_b200.batch import BatchedSpectra
    B = BATCHED
    rng = np.random.default_rng(B['seed'])
    lo, hi = np.log(B['np_range'][0]), np.log(B['np_range'][1])
    targets = np.exp(rng.uniform(lo, hi, nmocks))
    sizes = rng.choice(B['meshsizes'], nmocks)
    kmax = float(np.pi * min(B['meshsizes']) / B['boxsize'])
    edges = np.arange(0., kmax, 0.005)
    mocks = []
    for i in range(nmocks):
        attrs = jp.MeshAttrs(meshsize=int(sizes[i]), boxsize=B['boxsize'])
        pos = lognormal_particles(attrs, power_law_pk(), targets[i] / B['boxsize']**3, seed=1000 + i)
        mocks.append((int(sizes[i]), pos))
    bins = {n: jp.BinMesh2SpectrumPoles(jp.MeshAttrs(meshsize=n, boxsize=B['boxsize']), edges=edges, ells=(0, 2, 4))
            for n in B['meshsizes']}
    attrs_of = {n: jp.MeshAttrs(meshsize=n, boxsize=B['boxsize']) for n in B['meshsizes']}
    torch.cuda.synchronize()

    def plain(i):
        n, pos = mocks[i]
        mesh = jp.ParticleField(pos, attrs=attrs_of[n]).paint(resampler='tsc', interlacing=B['interlacing'],
                                                             compensate=True, out='complex')
        return np.array([p.num_raw for p in jp.compute_mesh2_spectrum(mesh, bin=bins[n], los='z')])

    for i in range(3):
        plain(i)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    plain_out = [plain(i) for i in range(nmocks)]
    torch.cuda.synchronize()
    t_plain = time.perf_counter() - t0
    # batched: groups of `group` mocks of the same mesh size, one graph each
    runners, inputs = [], []
    for n in B['meshsizes']:
        idx = [i for i in range(nmocks) if mocks[i][0] == n]
        for start in range(0, len(idx), group):
            sel = idx[start:start + group]
            counts = [mocks[i][1].shape[0] for i in sel]
            bs = BatchedSpectra(attrs_of[n], bins[n], counts, resampler='tsc', interlacing=B['interlacing'])
            runners.append((sel, bs))
            inputs.append(torch.cat([mocks[i][1] for i in sel]))
    for (sel, bs), x in zip(runners, inputs):  # warm-up replays
        bs.positions.copy_(x)
        bs()
    torch.cuda.synchronize()
    batched_out = [None] * nmocks
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record()
    results = []
    for (sel, bs), x in zip(runners, inputs):
        results.append(bs(x))
    end.record()
    torch.cuda.synchronize()
    t_batched = start.elapsed_time(end) / 1e3
    for (sel, bs), r in zip(runners, results):
        r = r.cpu().numpy()
        for j, i in enumerate(sel):
            batched_out[i] = r[j]
    plain_arr, batched_arr = np.array(plain_out), np.array(batched_out)
    norm = np.array([[(n / B['boxsize'])**3 * n**3] for n, _ in mocks])  # N^3 / V_cell
    p_plain = (plain_arr / norm[:, :, None]).reshape(nmocks, -1)
    p_batched = (batched_arr / norm[:, :, None]).reshape(nmocks, -1)
    scale0 = np.abs(p_plain[:, :len(edges) - 1]).max()
    rel_batched = float(np.abs(p_batched - p_plain).max() / scale0)
    cov_plain, cov_batched = np.cov(p_plain.T), np.cov(p_batched.T)
    cov_rel = float(np.abs(cov_batched - cov_plain).max() / np.abs(np.diag(cov_plain)).max())
    # float64 per-mock oracle loop on a subset of the smallest catalogs
    from oracle.coords import Geometry
    from oracle import paint as opaint
    from oracle.spectrum import Bins, compute_mesh2_spectrum
    order = sorted(range(nmocks), key=lambda i: (mocks[i][0], mocks[i][1].shape[0]))[:fp64_subset]
    err64 = 0.
    for i in order:
        n, pos = mocks[i]
        geom = Geometry(n, B['boxsize'], 0., dtype=np.float64)
        ref = compute_mesh2_spectrum(opaint.paint(geom, pos.cpu().numpy().astype('f8'), None, 'tsc', B['interlacing'], True,
                                                  'complex'), Bins(geom, edges=edges, ells=(0, 2, 4)), los='z')['num_raw']
        err64 = max(err64, float(np.abs(batched_arr[i] - ref).max() / np.abs(ref[0]).max()))
    return dict(B, nparticles_total=int(sum(m[1].shape[0] for m in mocks)),
                plain_spectra_per_s=nmocks / t_plain, batched_spectra_per_s=nmocks / t_batched,
                speedup=t_plain / t_batched, batched_vs_plain_max_rel=rel_batched,
                covariance_max_rel_vs_plain=cov_rel, fp64_subset=len(order), fp64_max_rel=err64,
                tile_configs=sorted({bs.tile_config for _, bs in runners}), graphs=len(runners),
                timing='plain: wall clock of the per-mock public-API loop (host-synchronous per mock); '
                       'batched: CUDA events around the graph replays (inputs resident)')


# ----------------------------------------------------------------------------- GPU arm

def run_ours(args):
    import torch
    import torch.distributed as dist
    import jaxpower_b200 as jp
    from jaxpower_b200.mock import lognormal_particles, power_law_pk
    from jaxpower_b200.tracing import Timeline

    world = int(os.environ.get('WORLD_SIZE', 1))
    rank = int(os.environ.get('RANK', 0))
    local = int(os.environ.get('LOCAL_RANK', 0))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group('nccl', timeout=timedelta(seconds=120), device_id=torch.device('cuda', local))

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x):
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device='cuda')
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    W = dict(WORKLOAD)
    if args.meshsize:  # smaller case of the same workload (profiling): same nbar and box
        W['meshsize'] = args.meshsize
    attrs = jp.MeshAttrs(meshsize=W['meshsize'], boxsize=W['boxsize'], boxcenter=0.)
    positions = lognormal_particles(attrs, power_law_pk(), W['nbar'], seed=W['seed'] + rank)
    npart = positions.shape[0]
    bins = jp.BinMesh2SpectrumPoles(attrs, edges={'step': W['k_step']}, ells=tuple(W['ells']))
    torch.cuda.synchronize()

    def step(pos):
        mesh = jp.ParticleField(pos, attrs=attrs).paint(resampler=W['resampler'], interlacing=W['interlacing'],
                                                        compensate=W['compensate'], out='complex')
        return jp.compute_mesh2_spectrum(mesh, bin=bins, los=W['los'])

    for _ in range(args.warmup):
        step(positions)
    # ---- device-resident throughput
    barrier()
    timeline = Timeline()
    with ClockSampler(local) as clocks, timeline:
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record()
        for _ in range(args.steps):
            result = step(positions)
        end.record()
        torch.cuda.synchronize()
    elapsed = max_over_ranks(start.elapsed_time(end) / 1e3)
    stages = timeline.summary()
    value = world * args.steps / elapsed
    # ---- end to end: pinned host positions -> device each step, multipoles back to host
    e2e_value = None
    if not args.no_e2e:
        host = torch.empty(positions.shape, dtype=torch.float32, pin_memory=True)
        host.copy_(positions)
        for _ in range(args.warmup):
            step(host.to('cuda', non_blocking=True))
        barrier()
        start2, end2 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start2.record()
        for _ in range(args.steps):
            res = step(host.to('cuda', non_blocking=True))
            _ = res.value()
        end2.record()
        torch.cuda.synchronize()
        elapsed2 = max_over_ranks(start2.elapsed_time(end2) / 1e3)
        e2e_value = world * args.steps / elapsed2
    nbins = bins.nbins

    # roofline of the dominant kernel (ours; cuFFT excluded)
    peak, peak_kind = measured_peaks()
    ours = {k: v for k, v in stages.items() if k != 'pk_fft_exec' and k in LAUNCHES}
    dominant = max(ours, key=lambda k: ours[k]['total_ms'])
    abytes = algorithmic_bytes(dominant, npart, W['meshsize'], W['interlacing'], len(W['ells']))
    achieved = abytes / (ours[dominant]['mean_ms'] * 1e-3) / 1e9
    launches = sum(LAUNCHES.get(k, 0) * v['calls'] for k, v in stages.items())
    stage_report = {k: {'calls': v['calls'], 'mean_ms': round(v['mean_ms'], 4),
                        'share': round(v['total_ms'] / (elapsed * 1e3), 4)} for k, v in stages.items()}
    line = {'metric': METRIC, 'value': value, 'unit': 'spectra/s', 'n_gpus': world, 'steps': args.steps,
            'warmup': args.warmup, 'ms_per_step': elapsed * 1e3 / args.steps, 'higher_is_better': True,
            'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f32', 'data': 'synthetic',
            'config': dict(W, nparticles=int(npart), parallelism='replicas' if world > 1 else 'single',
                           l2='inputs larger than L2 (512 MiB meshes per shift)', out='complex'),
            'roofline': {'bound': 'hbm', 'kernel': dominant, 'achieved': achieved, 'peak': peak,
                         'peak_kind': peak_kind, 'unit': 'GB/s', 'frac': achieved / peak,
                         'algorithmic_bytes': abytes, 'traffic': None},
            'e2e': {'value': e2e_value, 'unit': 'spectra/s', 'h2d_bytes_per_step': int(npart * 12),
                    'd2h_bytes_per_step': int(len(W['ells']) * nbins * 8)},
            'gpu_launches': int(launches), 'stages': stage_report, 'clocks': clocks.summary()}
    if rank == 0 and world == 1 and not args.no_batched:
        line['batched'] = run_batched()
    if rank == 0 and world == 1 and not args.no_cpu:
        seconds, desc, cores = cpu_sample(meshsize=args.cpu_meshsize)
        line['cpu_baseline'] = {'value': 1. / seconds, 'unit': 'spectra/s', 'cores': cores, 'kind': 'port',
                                'sample': desc}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def main():
    parser = argparse.ArgumentParser(description=__doc__.split('\n')[0])
    parser.add_argument('--gpus', type=int, default=1)
    parser.add_argument('--steps', type=int, default=20)
    parser.add_argument('--warmup', type=int, default=5)
    parser.add_argument('--impl', default='ours', choices=['ours', 'reference'])
    parser.add_argument('--cpu-meshsize', type=int, default=256)
    parser.add_argument('--no-cpu', action='store_true', help='skip the CPU baseline sample')
    parser.add_argument('--no-e2e', action='store_true', help='skip the end-to-end (host buffers) measurement')
    parser.add_argument('--meshsize', type=int, default=0, help='smaller mesh of the same workload (profiling)')
    parser.add_argument('--no-batched', action='store_true', help='skip the batched-mocks measurement')
    args = parser.parse_args()
    if args.impl == 'reference':
        run_reference(args)
    else:
        run_ours(args)


if __name__ == '__main__':
    main()

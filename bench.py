"""Benchmark: P_ell spectra/s of the mesh power-spectrum path on B200.

Workload (one step = one spectrum): a lognormal mock on a 512^3 mesh in a 1000 Mpc/h
box, P(k) = 2e4 (k/0.1)^-1.5 exp(-(k/0.5)^2), Poisson-sampled at nbar = 5e-3
(~5e6 float32 positions, unit weights); paint TSC with interlacing 3 and compensation,
global line of sight 'z', ells (0, 2, 4), k edges step 0.005 up to k_Nyq.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints one JSON line (rank 0).  ``value``: spectra/s with positions resident in HBM;
``e2e``: the same through the public API with positions copied from pinned host
memory every step and the multipoles read back.  ``--impl reference`` times the
CPU oracle (a NumPy/SciPy/C restatement of the reference's JAX code, which cannot run
here: no jax) on whole 512^3 spectra of the same catalog (the catalog is made on the
host with NumPy, so both arms read the same positions).  Multi-GPU runs are
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

LEARNED = dict(workload='learned aliasing correction: lognormal mocks (benchmark P(k), N~1e6, box 1000), CIC at '
                        '128^3 corrected towards the same catalog at 512^3; no interlacing, compensate, los z, '
                        'ells (0,2,4), k step 0.01', low=128, high=512, gen_meshsize=256, boxsize=1000., nbar=1e-3,
               resampler='cic', interlacing=0, kstep=0.01, ntrain=4096, nheld=512, steps=4000, batch=4096,
               kmax_fraction_eval=0.8, seed0=100000)

CUTSKY = dict(workload='cut-sky FKP, first-point los, with adjoint: ~2e6 clustered data (lognormal) and 2e7 randoms, '
                       'r in [1000, 2000] Mpc/h, 60 deg cap, Gaussian n(r) (1500, 250), FKP weights 1/(1+n 1e4), '
                       'boxpad 2, meshsize 512, TSC, interlacing 3, compensate, ells (0,2,4), k step 0.005',
              ndata=2e6, nrandoms=2e7, meshsize=512, boxpad=2., resampler='tsc', interlacing=3, ells=(0, 2, 4),
              k_step=0.005, ell_weights=(1., 0.5, 0.25), fd_step=0.25, seed=11)

# kernel launches issued by each C-ABI entry point (ours, including CUB's scan kernels)
LAUNCHES = {'pk_paint': 6, 'pk_paint_batch': 6, 'pk_interlace_compensate': 1, 'pk_interlace_compensate_batch': 1,
            'pk_bin_global': 2, 'pk_bin_global_batch': 2, 'pk_bin_global_interlaced': 2, 'pk_bin_firstpoint': 2,
            'pk_bin_modes': 2, 'pk_bin_mesh': 2, 'pk_scale_real': 1, 'pk_ylm_premultiply': 1, 'pk_read': 1,
            'pk_read_interlaced': 3}


# ncu DRAM read + write of one pk_paint call of the 512^3 workload above (its counting, column
# scan, placement and per-shift tile kernels, one-pass metrics on the full-size workload); the
# event timing supplies the duration
PAINT_TRAFFIC_512 = (60061696 + 256768) + (9705984 + 0) + (73378304 + 70682368) + (123594240 + 1547215360)

C0 = dict(workload='uniform catalog 1e5 particles in a 1000 Mpc/h cube (seed 0), meshsize 64, CIC, no interlacing, '
                   'compensate, los z, ells (0,2,4), k step 0.01', nparticles=100000, meshsize=64, boxsize=1000.,
          resampler='cic', interlacing=0, compensate=True, k_step=0.01, seed=0)


def run_c0(reps=50):
    """The reference's CPU-runnable configuration: GPU spectra/s through the public API
    (positions resident) beside the oracle's float32 pipeline on the host, and their
    difference (parity of the two on these inputs)."""
    import torch
    import jaxpower_b200 as jp
    from oracle.coords import Geometry
    from oracle import paint as opaint
    from oracle.spectrum import Bins, compute_mesh2_spectrum as ospectrum
    c = C0
    rng = np.random.default_rng(c['seed'])
    pos = (rng.uniform(0., c['boxsize'], (c['nparticles'], 3))).astype('f4')
    attrs = jp.MeshAttrs(meshsize=c['meshsize'], boxsize=c['boxsize'], boxcenter=c['boxsize'] / 2.)
    b = jp.BinMesh2SpectrumPoles(attrs, edges={'step': c['k_step']}, ells=(0, 2, 4))
    dpos = torch.as_tensor(pos).cuda()

    def gpu():
        mesh = jp.ParticleField(dpos, attrs=attrs).paint(resampler=c['resampler'], interlacing=c['interlacing'],
                                                         compensate=c['compensate'], out='complex')
        return jp.compute_mesh2_spectrum(mesh, bin=b, los='z')

    for _ in range(3):
        gpu()
    torch.cuda.synchronize()
    t = time.perf_counter()
    for _ in range(reps):
        res = gpu()
    torch.cuda.synchronize()
    t_gpu = (time.perf_counter() - t) / reps
    geom = Geometry(c['meshsize'], c['boxsize'], c['boxsize'] / 2.)
    t = time.perf_counter()
    ref = ospectrum(opaint.paint(geom, pos, None, c['resampler'], c['interlacing'], c['compensate'], 'complex'),
                    Bins(geom, step=c['k_step'], ells=(0, 2, 4)), los='z')['num_raw']
    t_cpu = time.perf_counter() - t
    got = np.array([p.num_raw for p in res])
    geom64 = Geometry(c['meshsize'], c['boxsize'], c['boxsize'] / 2., dtype=np.float64)
    ref64 = ospectrum(opaint.paint(geom64, pos.astype('f8'), None, c['resampler'], c['interlacing'], c['compensate'],
                                   'complex'), Bins(geom64, step=c['k_step'], ells=(0, 2, 4)), los='z')
    same = np.asarray(b.nmodes) == ref64['nmodes']
    return dict(c, gpu_spectra_per_s=1. / t_gpu, cpu_oracle_spectra_per_s=1. / t_cpu, cpu_cores=cpu_cores(),
                max_rel_diff_vs_oracle=float(np.abs(got - ref).max() / np.abs(ref[0]).max()),
                max_rel_diff_vs_fp64_oracle=float(np.abs(got[:, same] - ref64['num_raw'][:, same]).max()
                                                  / np.abs(ref64['num_raw'][0][same]).max()),
                timing='GPU: wall clock per spectrum through the public API with host read-back (positions '
                       'resident); CPU: the oracle float32 pipeline, one run')


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
    if name in ('pk_paint', 'pk_paint_batch'):  # read positions (+weights) once, write one float32 mesh per shift
        return 16. * npart + 4. * nr * interlacing
    if name == 'pk_interlace_compensate':
        return 8. * nc * (interlacing + 1)
    if name in ('pk_bin_global', 'pk_bin_mesh'):
        return 8. * nc
    if name == 'pk_bin_global_interlaced':  # the shifted meshes read once
        return 8. * nc * interlacing
    return None


def binning_roofline(stages, bins, W, peak):
    """The fused interlace + compensate + binning pass against the HBM peak: on the whole shifted
    meshes (8 N_c I bytes, the algorithmic figure) and on the stored modes below the last edge,
    the only ones it reads (8 I bytes each)."""
    st = stages.get('pk_bin_global_interlaced')
    if not st:
        return None
    n = int(W['meshsize'])
    kf = 2. * np.pi / float(W['boxsize'])
    k = np.fft.fftfreq(n, 1. / n) * kf
    kz2 = (np.arange(n // 2 + 1) * kf) ** 2
    klast2 = float(bins._edges1d[-1]) ** 2
    kxy = (k[:, None] ** 2 + k[None, :] ** 2).ravel()
    in_range = int(np.searchsorted(kz2, klast2 - kxy, side='left').sum())
    t = st['mean_ms'] * 1e-3
    whole = 8. * n * n * (n // 2 + 1) * W['interlacing']
    needed = 8. * W['interlacing'] * in_range
    return {'kernel': 'pk_bin_global_interlaced', 'bound': 'hbm', 'unit': 'GB/s', 'peak': peak,
            'algorithmic_bytes': whole, 'achieved': whole / t / 1e9, 'frac': whole / t / 1e9 / peak,
            'in_range_bytes': needed, 'achieved_in_range': needed / t / 1e9, 'frac_in_range': needed / t / 1e9 / peak}


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


# ----------------------------------------------------------------------------- benchmark catalog

def lognormal_catalog(meshsize=512, boxsize=1000., nbar=5e-3, seed=42, amplitude=2e4, k0=0.1, index=-1.5,
                      kcut=0.5):
    """The benchmark catalog, made on the host with NumPy/SciPy so that both arms (GPU and CPU)
    read the same float32 positions: a Gaussian field with P(k) = A (k/k0)^index exp(-(k/kcut)^2)
    (white noise, r2c, times sqrt(P / V_cell), c2r with 1/N^3), the lognormal transform
    1 + delta_LN = exp(delta - sigma^2 / 2), Poisson counts of mean nbar V_cell (1 + delta_LN)
    per cell and positions uniform within each cell (the recipe of ``jaxpower_b200.mock``)."""
    import scipy.fft
    rng = np.random.default_rng(seed)
    n = int(meshsize)
    cell = boxsize / n
    vcell = cell**3
    noise = rng.standard_normal((n, n, n), dtype=np.float32)
    c = scipy.fft.rfftn(noise, workers=-1)
    del noise
    kf = 2. * np.pi / boxsize
    kx = (np.fft.fftfreq(n, 1. / n) * kf).astype('f4')
    kz = (np.fft.rfftfreq(n, 1. / n) * kf).astype('f4')
    for i in range(n):  # plane by plane: small temporaries
        k = np.sqrt(kx[i]**2 + kx[:, None]**2 + kz[None, :]**2)
        safe = np.where(k > 0, k, 1.)
        p = np.where(k > 0, amplitude * (safe / k0)**index * np.exp(-(safe / kcut)**2), 0.)
        c[i] *= np.sqrt(p / vcell).astype('f4')
    delta = scipy.fft.irfftn(c, s=(n, n, n), workers=-1).astype('f4')
    del c
    sigma2 = float(np.mean(delta.astype('f8')**2))
    lam = np.exp(delta - np.float32(0.5 * sigma2), dtype=np.float32)
    del delta
    lam *= np.float32(nbar * vcell)
    counts = rng.poisson(lam.ravel())
    del lam
    cells = np.repeat(np.arange(n**3, dtype=np.int64), counts)
    ijk = np.stack([cells // (n * n), (cells // n) % n, cells % n], axis=1).astype('f4')
    del cells
    u = rng.random(ijk.shape, dtype=np.float32)
    return ((ijk + u) * np.float32(cell) - np.float32(boxsize / 2.)).astype('f4')


def benchmark_catalog(seed=None, meshsize=None):
    W = WORKLOAD
    return lognormal_catalog(meshsize=meshsize or W['meshsize'], boxsize=W['boxsize'], nbar=W['nbar'],
                             seed=W['seed'] if seed is None else seed)


# ----------------------------------------------------------------------------- CPU arm

def oracle_pipeline(meshsize=None, catalog=None, dtype=np.float32):
    """The oracle's pipeline for the benchmark workload on the host: (one-spectrum callable,
    positions).  float32: the reference's operation order (serial float32 scatter in C,
    scipy.fft with all host cores, float64 bin sums); float64: the same in float64."""
    from oracle.coords import Geometry
    from oracle import paint as opaint
    from oracle.spectrum import Bins, compute_mesh2_spectrum
    W = WORKLOAD
    n = meshsize or W['meshsize']
    pos = benchmark_catalog(meshsize=n) if catalog is None else catalog
    geom = Geometry(n, W['boxsize'], 0., dtype=dtype)
    bins = Bins(geom, step=W['k_step'], ells=tuple(W['ells']))  # bin setup, once (as the reference's)
    x = pos.astype(dtype)

    def spectrum():
        mesh = opaint.paint(geom, x, None, W['resampler'], W['interlacing'], W['compensate'], 'complex')
        return compute_mesh2_spectrum(mesh, bins, los=W['los'], accum='f64')

    return spectrum, pos


def cpu_cores():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count()


ORACLE_SAMPLE = ('oracle float32 pipeline on the benchmark catalog itself, 512^3 (C scatter in the reference\'s '
                 'serial order, scipy.fft on all host cores, bin sums in float64), measured whole spectra, no scaling')


def run_reference(args):
    """The CPU arm: the oracle's restatement of the reference's JAX CPU path (the reference itself
    needs jax, absent here), timed on whole 512^3 spectra of the benchmark catalog.  A spectrum
    takes tens of seconds, so one warm-up step is run and the timed steps stop at ``--ref-budget``
    seconds (at least one); the line reports the steps actually run."""
    rank = int(os.environ.get('RANK', 0))
    if rank != 0:
        return
    spectrum, pos = oracle_pipeline()
    warmup = min(args.warmup, 1)
    for _ in range(warmup):
        spectrum()
    times = []
    t_all = time.perf_counter()
    while len(times) < args.steps and (not times or time.perf_counter() - t_all < args.ref_budget):
        t0 = time.perf_counter()
        spectrum()
        times.append(time.perf_counter() - t0)
    value = len(times) / float(np.sum(times))
    cores = cpu_cores()
    line = {'impl': 'reference', 'metric': METRIC, 'value': value, 'unit': 'spectra/s', 'n_gpus': args.gpus,
            'steps': len(times), 'warmup': warmup, 'steps_requested': args.steps, 'warmup_requested': args.warmup,
            'ms_per_step': 1e3 / value, 'higher_is_better': True, 'scaling': 'weak', 'vs_baseline': None,
            'dtype': 'f32', 'data': 'synthetic', 'config': dict(WORKLOAD, nparticles=int(pos.shape[0])),
            'cpu_baseline': {'value': value, 'unit': 'spectra/s', 'cores': cores, 'kind': 'port',
                             'sample': ORACLE_SAMPLE + '; {} timed spectra'.format(len(times))},
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

    for i in range(nmocks):  # warm-up pass: plans, tile autotuning per (mesh, particle-count) key
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
        results.append(bs(x, check=False))
    end.record()
    torch.cuda.synchronize()
    t_batched = start.elapsed_time(end) / 1e3
    assert not any(bs.status() for _, bs in runners), 'a batched mock dropped particles'
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


def run_sharded_mocks(world, rank, barrier, max_over_ranks, group=32):
    """The batched-mocks workload (256 lognormal mocks, mesh sizes 128 / 192 / 256) shared out over
    the ranks: each rank measures its cost-balanced share (``sharding.ShardedMocks``: one
    BatchedSpectra graph per mesh size and group) and one NCCL all_reduce assembles every mock's
    multipoles on every rank.  Timed with CUDA events, max over ranks, the gather included; rank 0
    checks two of its mocks against the plain public API."""
    import torch
    import jaxpower_b200 as jp
    from jaxpower_b200.mock import lognormal_particles, power_law_pk
    from jaxpower_b200.sharding import ShardedMocks, covariance
    B = BATCHED
    nmocks = B['nmocks']
    rng = np.random.default_rng(B['seed'])
    lo, hi = np.log(B['np_range'][0]), np.log(B['np_range'][1])
    targets = np.exp(rng.uniform(lo, hi, nmocks))
    sizes = rng.choice(B['meshsizes'], nmocks)
    kmax = float(np.pi * min(B['meshsizes']) / B['boxsize'])
    edges = np.arange(0., kmax, 0.005)
    attrs_of = {n: jp.MeshAttrs(meshsize=n, boxsize=B['boxsize']) for n in B['meshsizes']}
    bins = {n: jp.BinMesh2SpectrumPoles(attrs_of[n], edges=edges, ells=(0, 2, 4)) for n in B['meshsizes']}
    sharded = ShardedMocks([(int(m), float(t)) for m, t in zip(sizes, targets)], bins, resampler='tsc',
                           interlacing=B['interlacing'], group=group)
    cats = {i: lognormal_particles(attrs_of[int(sizes[i])], power_law_pk(), targets[i] / B['boxsize']**3,
                                   seed=1000 + i) for i in sharded.mine}  # this rank's mocks only
    sharded(cats.__getitem__)  # warm-up: autotuning, graph capture
    barrier()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record()
    full = sharded(cats.__getitem__)
    end.record()
    torch.cuda.synchronize()
    seconds = max_over_ranks(start.elapsed_time(end) / 1e3)
    check = None
    if rank == 0:
        errs = []
        for i in sharded.mine[:2]:
            n = int(sizes[i])
            mesh = jp.ParticleField(cats[i], attrs=attrs_of[n]).paint(resampler='tsc', interlacing=B['interlacing'],
                                                                      compensate=True, out='complex')
            ref = np.array([p.num_raw for p in jp.compute_mesh2_spectrum(mesh, bin=bins[n], los='z')])
            got = full[i].cpu().numpy()
            errs.append(float(np.abs(got - ref).max() / np.abs(ref[0]).max()))
        check = max(errs) if errs else None
    cov = covariance(full.cpu())
    return dict(workload=B['workload'], nmocks=nmocks, ranks=world, mocks_per_s=nmocks / seconds, seconds=seconds,
                mocks_on_rank0=len(sharded.mine), batches_on_rank0=len(sharded.batches),
                max_rel_vs_public_api=check, covariance_shape=list(cov.shape),
                timing='CUDA events around this rank\'s batched graphs and the NCCL all_reduce of all multipoles, '
                       'max over ranks; catalogs resident')


def run_cutsky(reps=3):
    """Cut-sky FKP first-point multipoles at 512^3 and the gradient of sum_l w_l P_l with
    respect to the data positions (hand-written adjoints), checked by central differences."""
    import torch
    import jaxpower_b200 as jp
    from jaxpower_b200.mock import cutsky_particles
    from jaxpower_b200.autodiff import paint_value, spectrum_value
    C = dict(CUTSKY)
    data, randoms, wd, wr = cutsky_particles(ndata=C['ndata'], nrandoms=C['nrandoms'], seed=C['seed'])
    attrs = jp.get_mesh_attrs(data, randoms, meshsize=C['meshsize'], boxpad=C['boxpad'])
    b = jp.BinMesh2SpectrumPoles(attrs, edges={'step': C['k_step']}, ells=C['ells'])
    fkp = jp.FKPField(jp.ParticleField(data, wd, attrs=attrs), jp.ParticleField(randoms, wr, attrs=attrs))
    norm = jp.compute_fkp2_normalization(fkp, bin=b)
    shotnoise = jp.compute_fkp2_shotnoise(fkp, bin=b)

    def forward():
        mesh = fkp.paint(resampler=C['resampler'], interlacing=C['interlacing'], compensate=True, out='real')
        return jp.compute_mesh2_spectrum(mesh, bin=b, los='firstpoint')

    def events(fn, n):
        fn()
        torch.cuda.synchronize()
        a, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(n):
            out = fn()
        e.record()
        torch.cuda.synchronize()
        return a.elapsed_time(e) / 1e3 / n, out

    t_fwd, poles = events(forward, reps)
    alpha = float(wd.double().sum() / wr.double().sum())
    weights = torch.cat([wd, -alpha * wr])
    coef = torch.tensor(C['ell_weights'], dtype=torch.float64, device='cuda')[:, None]
    scale = 1. / float(np.abs(poles.get(0).num_raw).max())

    def loss(xd):
        mesh = paint_value(torch.cat([xd, randoms]), weights, attrs, C['resampler'], C['interlacing'], True, 'real')
        return (coef * spectrum_value(mesh, attrs, b, 'firstpoint')).sum() * scale

    def fwd_bwd():
        xd = data.clone().requires_grad_(True)
        value = loss(xd)
        value.backward()
        return value.detach(), xd.grad

    t_grad, (value, grad) = events(fwd_bwd, reps)
    g = torch.Generator(device='cuda').manual_seed(5)
    v = torch.randn(data.shape, generator=g, device='cuda')
    v /= torch.linalg.norm(v, dim=1, keepdim=True)
    h = C['fd_step']
    with torch.no_grad():
        lp, lm = float(loss(data + h * v)), float(loss(data - h * v))
    fd = (lp - lm) / (2 * h)
    ad = float((grad.double() * v.double()).sum())
    consistency = float(abs(value.item() - float(
        (coef.cpu().numpy() * np.array([p.num_raw for p in poles])).sum() * scale)))
    from jaxpower_b200.mesh2 import _term_batches
    return dict(C, ndata=int(data.shape[0]), nrandoms=int(randoms.shape[0]), boxsize=[float(x) for x in attrs.boxsize],
                nbins=int(b.nbins), term_batches=[len(t) for t in _term_batches(attrs, C['ells'])],
                spectra_per_s=1. / t_fwd, seconds_forward=t_fwd,
                seconds_forward_backward=t_grad, norm=float(np.mean(norm)),
                shotnoise_ell0=float(np.mean(shotnoise[0])) if np.ndim(shotnoise) > 1 else float(np.mean(shotnoise)),
                gradient_check={'directional_ad': ad, 'directional_fd': fd, 'rel_err': abs(ad - fd) / abs(fd),
                                'fd_step_mpc': h, 'direction': 'random unit vector per data particle'},
                value_api_vs_autodiff_abs=consistency,
                timing='CUDA events, positions resident; forward = FKPField.paint + compute_mesh2_spectrum; '
                       'forward_backward = differentiable paint + spectrum + backward to data positions')


def run_paint_only(meshsize=None, reps=3, config=4):
    """Profiling aid: the benchmark catalog (made at 512^3) painted with TSC and 3
    interlacing shifts at ``meshsize`` through pk_paint_batch with tile configuration ``config``,
    one warm-up and ``reps`` timed calls; nothing else is on the device meanwhile."""
    import torch
    import jaxpower_b200 as jp
    from jaxpower_b200.mesh import _paint_call
    from jaxpower_b200.mock import lognormal_particles, power_law_pk
    W = WORKLOAD
    pos = torch.as_tensor(benchmark_catalog()).cuda()
    n = meshsize or W['meshsize']
    attrs = jp.MeshAttrs(meshsize=n, boxsize=W['boxsize'], boxcenter=0.)
    out = torch.empty((W['interlacing'], n, n, n), dtype=torch.float32, device='cuda')
    status = torch.zeros(1, dtype=torch.int32, device='cuda')
    _paint_call(attrs, pos, None, 3, W['interlacing'], 0, W['interlacing'], out, status, config)  # warm-up
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(reps):
        _paint_call(attrs, pos, None, 3, W['interlacing'], 0, W['interlacing'], out, status, config)
    b.record()
    torch.cuda.synchronize()
    return dict(nparticles=int(pos.shape[0]), meshsize=n, tile_config=config, ms_per_paint=a.elapsed_time(b) / reps,
                status=int(status.item()))


def run_window_only(meshsize=None, reps=2):
    """Profiling aid: window matrices of the global-los multipoles (0, 2, 4), ells_in (0, 2, 4), on
    a (2000 Mpc/h)^3 box at ``meshsize`` (default 512), output k step 0.005: a selection function
    (uniform random W in [0.5, 1.5]) with 20 input bins of width 0.01 (60 columns), and the
    periodic box with the same input bins (one merged pass) and with the output bins as input
    (diagonal).  One warm-up and ``reps`` timed calls each, device time by CUDA events, with the
    per-entry-point split of the selection window (``tracing.Timeline``)."""
    import torch
    import jaxpower_b200 as jp
    from jaxpower_b200.tracing import Timeline
    n = meshsize or 512
    attrs = jp.MeshAttrs(meshsize=n, boxsize=2000.)
    b = jp.BinMesh2SpectrumPoles(attrs, edges={'step': 0.005}, ells=(0, 2, 4))
    gen = torch.Generator(device='cuda').manual_seed(0)
    sel = attrs.create(kind='real', fill=torch.rand((n, n, n), generator=gen, device='cuda') + 0.5)
    edgesin = np.linspace(0.001, 0.201, 21)
    cases = {'selection_60_columns': lambda: jp.compute_mesh2_spectrum_window(sel, edgesin=edgesin, ellsin=(0, 2, 4),
                                                                              bin=b, los='z'),
             'periodic_60_columns': lambda: jp.compute_mesh2_spectrum_window(attrs, edgesin=edgesin, ellsin=(0, 2, 4),
                                                                             bin=b, los='z'),
             'periodic_diagonal': lambda: jp.compute_mesh2_spectrum_window(attrs, edgesin=b._edges1d,
                                                                           ellsin=(0, 2, 4), bin=b, los='z')}
    out = dict(meshsize=n)
    for name, fn in cases.items():
        fn()
        torch.cuda.synchronize()
        a, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(reps):
            fn()
        e.record()
        torch.cuda.synchronize()
        out[name + '_ms'] = a.elapsed_time(e) / reps
    with Timeline() as tl:
        cases['selection_60_columns']()
    torch.cuda.synchronize()
    out['selection_split_ms'] = {k: round(v['total_ms'], 3) for k, v in tl.summary().items()}
    return out


def run_cutsky_forward_only(meshsize=None, reps=3):
    """Profiling aid: the cut-sky FKP first-point forward pipeline (paint + spectrum) ``reps``
    times, at ``meshsize`` (default that of the cut-sky workload)."""
    import torch
    import jaxpower_b200 as jp
    from jaxpower_b200.mock import cutsky_particles
    C = dict(CUTSKY)
    data, randoms, wd, wr = cutsky_particles(ndata=C['ndata'], nrandoms=C['nrandoms'], seed=C['seed'])
    attrs = jp.get_mesh_attrs(data, randoms, meshsize=meshsize or C['meshsize'], boxpad=C['boxpad'])
    b = jp.BinMesh2SpectrumPoles(attrs, edges={'step': C['k_step']}, ells=C['ells'])
    fkp = jp.FKPField(jp.ParticleField(data, wd, attrs=attrs), jp.ParticleField(randoms, wr, attrs=attrs))
    a, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for r in range(reps + 1):
        if r == 1:
            a.record()
        mesh = fkp.paint(resampler=C['resampler'], interlacing=C['interlacing'], compensate=True, out='real')
        poles = jp.compute_mesh2_spectrum(mesh, bin=b, los='firstpoint')
        del mesh
    e.record()
    torch.cuda.synchronize()
    return dict(meshsize=int(attrs.meshsize[0]), ms_per_spectrum=a.elapsed_time(e) / reps,
                p0_sum=float(np.sum(poles.get(0).num_raw)))


def run_mlp_forward(batch=1 << 20, reps=20):
    """Throughput of the correction network's tcgen05 forward pass on a batch of random
    feature rows (dense FLOPs 2 (16 + 2 x 128 + 16) x 128 per row; the padded output layer
    counts at its computed width 16)."""
    import torch
    from jaxpower_b200.learned import MLP
    mlp = MLP(seed=3)
    x = torch.randn((batch, 16), generator=torch.Generator(device='cuda').manual_seed(4), device='cuda')
    for _ in range(3):
        mlp(x)
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(reps):
        mlp(x)
    b.record()
    torch.cuda.synchronize()
    mlp.check()
    seconds = a.elapsed_time(b) / 1e3 / reps
    flops = 2. * (16 + 2 * 128 + 16) * 128 * batch
    return dict(batch=batch, seconds=seconds, rows_per_s=batch / seconds, tflops=flops / seconds / 1e12,
                timing='CUDA events around %d forward passes (inputs resident)' % reps)


def run_learned(ntrain=None, nheld=None, steps=None):
    """Train the learned correction on the GPU and evaluate it on held-out mocks."""
    import torch
    import jaxpower_b200 as jp
    from jaxpower_b200.learned import (LearnedCorrection, mock_spectra, spectrum_errors, ensemble_bias,
                                      ensemble_bias_significance, ensemble_bias_chi2)
    L = dict(LEARNED)
    ntrain = ntrain or L['ntrain']
    nheld = nheld or L['nheld']
    t0 = time.perf_counter()
    data = mock_spectra(range(L['seed0'], L['seed0'] + ntrain + nheld), meshsizes=(L['low'], L['high']),
                        boxsize=L['boxsize'], nbar=L['nbar'], gen_meshsize=L['gen_meshsize'],
                        resampler=L['resampler'], interlacing=L['interlacing'], kstep=L['kstep'], group=16)
    torch.cuda.synchronize()
    t_data = time.perf_counter() - t0
    train = dict(data, nparticles=data['nparticles'][:ntrain],
                 spectra={n: v[:ntrain] for n, v in data['spectra'].items()})
    t0 = time.perf_counter()
    corr, report = LearnedCorrection.train(train, L['low'], L['high'], steps=steps or L['steps'], batch=L['batch'],
                                           resampler=L['resampler'], interlacing=L['interlacing'])
    torch.cuda.synchronize()
    t_train = time.perf_counter() - t0
    low, high = data['spectra'][L['low']][ntrain:], data['spectra'][L['high']][ntrain:]
    npart = data['nparticles'][ntrain:]
    fixed = corr(low, npart)
    kmax = L['kmax_fraction_eval'] * np.pi * L['low'] / L['boxsize']
    e_plain, _ = spectrum_errors(low, high, data['k'], kmax)
    e_corr, _ = spectrum_errors(fixed, high, data['k'], kmax)
    # table baseline: the training-set mean of (P_fine - P_coarse) / P0_coarse per (ell, bin)
    tl, th = train['spectra'][L['low']], train['spectra'][L['high']]
    table = ((th - tl) / tl[:, :1]).mean(axis=0)
    e_table, _ = spectrum_errors(low + table[None] * low[:, :1], high, data['k'], kmax)
    bias_corr, bias_plain = ensemble_bias(fixed, high, data['k'], kmax), ensemble_bias(low, high, data['k'], kmax)
    _, bin_corr = spectrum_errors(fixed, high, data['k'], kmax)
    _, bin_plain = spectrum_errors(low, high, data['k'], kmax)
    _, bin_table = spectrum_errors(low + table[None] * low[:, :1], high, data['k'], kmax)

    # time per spectrum, one catalog resident on the device, public API, host-synchronous
    from jaxpower_b200.mock import lognormal_particles, power_law_pk
    attrs_lo = jp.MeshAttrs(meshsize=L['low'], boxsize=L['boxsize'])
    attrs_hi = jp.MeshAttrs(meshsize=L['high'], boxsize=L['boxsize'])
    pos = lognormal_particles(jp.MeshAttrs(meshsize=L['gen_meshsize'], boxsize=L['boxsize']), power_law_pk(),
                              L['nbar'], seed=7)
    b_lo = jp.BinMesh2SpectrumPoles(attrs_lo, edges=data['edges'], ells=(0, 2, 4))
    b_hi = jp.BinMesh2SpectrumPoles(attrs_hi, edges=data['edges'], ells=(0, 2, 4))

    def plain(attrs, b):
        mesh = jp.ParticleField(pos, attrs=attrs).paint(resampler=L['resampler'], interlacing=L['interlacing'],
                                                        compensate=True, out='complex')
        return np.array([p.value() for p in jp.compute_mesh2_spectrum(mesh, bin=b, los='z')])

    norm_lo = float(np.prod([L['low']] * 3))**2 / pos.shape[0]**2

    def learned():
        return corr(plain(attrs_lo, b_lo) * norm_lo, pos.shape[0])

    def timed(fn, reps):
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        t = time.perf_counter()
        for _ in range(reps):
            fn()
        torch.cuda.synchronize()
        return (time.perf_counter() - t) / reps

    t_hi = timed(lambda: plain(attrs_hi, b_hi), 20)
    t_lo = timed(lambda: plain(attrs_lo, b_lo), 50)
    t_learned = timed(learned, 50)
    # batched: 16 resident catalogs per CUDA-graph replay, timed with CUDA events; the
    # correction runs on the device on the batch's multipoles
    from jaxpower_b200.batch import BatchedSpectra
    from jaxpower_b200.learned import spectrum_norm
    gen = jp.MeshAttrs(meshsize=L['gen_meshsize'], boxsize=L['boxsize'])
    cats = [lognormal_particles(gen, power_law_pk(), L['nbar'], seed=900 + i) for i in range(16)]
    counts = [c.shape[0] for c in cats]
    allpos = torch.cat(cats)
    bs_lo = BatchedSpectra(attrs_lo, b_lo, counts, resampler=L['resampler'], interlacing=L['interlacing'])
    bs_hi = BatchedSpectra(attrs_hi, b_hi, counts, resampler=L['resampler'], interlacing=L['interlacing'])
    nrm_lo = torch.as_tensor(spectrum_norm(attrs_lo.meshsize, L['boxsize'], counts), device='cuda')[:, None, None]
    npart16 = np.array(counts, dtype='f8')

    def events(fn, reps):
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(reps):
            out = fn()
        b.record()
        torch.cuda.synchronize()
        return a.elapsed_time(b) / 1e3 / reps / 16, out

    bs_lo(allpos), bs_hi(allpos)
    tb_hi, _ = events(lambda: bs_hi(check=False), 5)
    tb_lo, _ = events(lambda: bs_lo(check=False), 20)
    tb_learned, _ = events(lambda: corr(bs_lo(check=False) * nrm_lo, npart16), 20)
    return dict(L, ntrain=ntrain, nheld=nheld, nbins=int(len(data['k'])),
                train_samples=int(report['ntrain'] * 3 * len(data['k'])),
                corrected_bins=report['corrected_bins'], total_bins=report['total_bins'],
                final_loss=float(report['loss_history'][-1]),
                heldout_max_rel_err={'learned': {'median': float(np.median(e_corr)),
                                                 'p95': float(np.percentile(e_corr, 95)), 'max': float(e_corr.max())},
                                     'plain_128': {'median': float(np.median(e_plain)),
                                                   'p95': float(np.percentile(e_plain, 95)),
                                                   'max': float(e_plain.max())},
                                     'mean_table_128': {'median': float(np.median(e_table)),
                                                        'p95': float(np.percentile(e_table, 95)),
                                                        'max': float(e_table.max())}},
                frac_heldout_within_0p5pct=float((e_corr <= 5e-3).mean()),
                heldout_bias_max={'learned': float(bias_corr.max()), 'plain_128': float(bias_plain.max()),
                                  'mean_table_128': float(ensemble_bias(low + table[None] * low[:, :1], high,
                                                                        data['k'], kmax).max()),
                                  'per_ell_learned': [float(b) for b in bias_corr.max(axis=1)],
                                  'per_ell_plain_128': [float(b) for b in bias_plain.max(axis=1)]},
                heldout_bias_in_standard_errors={
                    'learned': ensemble_bias_significance(fixed, high, data['k'], kmax),
                    'plain_128': ensemble_bias_significance(low, high, data['k'], kmax),
                    'mean_table_128': ensemble_bias_significance(low + table[None] * low[:, :1], high, data['k'],
                                                                 kmax)},
                heldout_bias_chi2_per_bin={
                    'learned': ensemble_bias_chi2(fixed, high, data['k'], kmax),
                    'plain_128': ensemble_bias_chi2(low, high, data['k'], kmax),
                    'mean_table_128': ensemble_bias_chi2(low + table[None] * low[:, :1], high, data['k'], kmax)},
                heldout_rms_rel_err_per_ell={'learned': [float(v) for v in np.sqrt((bin_corr**2).mean(axis=(0, 2)))],
                                             'plain_128': [float(v) for v in np.sqrt((bin_plain**2).mean(axis=(0, 2)))],
                                             'mean_table_128': [float(v) for v in
                                                                np.sqrt((bin_table**2).mean(axis=(0, 2)))]},
                heldout_median_rel_err_worst_bin={
                    'learned': float(np.median(bin_corr, axis=0).max()),
                    'plain_128': float(np.median(bin_plain, axis=0).max()),
                    'mean_table_128': float(np.median(bin_table, axis=0).max())},
                bias_definition='max over (ell, k <= 0.8 k_Nyq(128)) of |mean over held-out mocks of '
                                '(P_ell - P_ell(512^3))| / mean P_0(512^3)',
                error_definition='per held-out mock: max over k <= 0.8 k_Nyq(128) and ell in (0,2,4) of '
                                 '|P_ell - P_ell(512^3)| / P_0(512^3)',
                seconds_per_spectrum={'plain_512': t_hi, 'plain_128': t_lo, 'learned_128': t_learned},
                speedup_learned_vs_plain_512=t_hi / t_learned,
                batched_seconds_per_spectrum={'plain_512': tb_hi, 'plain_128': tb_lo, 'learned_128': tb_learned},
                batched_speedup_learned_vs_plain_512=tb_hi / tb_learned,
                seconds_data_generation=t_data, seconds_training=t_train,
                timing='seconds_per_spectrum: wall clock through the public API (paint + spectrum + host '
                       'read-back), one resident catalog; batched_*: CUDA events around BatchedSpectra graph '
                       'replays of 16 resident catalogs (+ the on-device correction), per spectrum')


def run_mlp_training(batch=4096, rows=1 << 20, reps=20):
    """The correction network's backward pass (tcgen05, and the mma.sync formulation beside it)
    on ``rows`` random feature rows, and one whole training step (tcgen05 forward with stored
    activations, loss, tcgen05 backward, CTA-order reduction, AdamW) at the training batch,
    replayed from a CUDA graph.  Backward dense FLOPs per row: 2 x 128 x (16 + 2 x 128) for the
    weight gradients and 2 x 128 x 2 x 128 for the activation gradients."""
    import torch
    from jaxpower_b200 import _lib
    from jaxpower_b200.learned import MLP
    mlp = MLP(seed=5)
    gen = torch.Generator(device='cuda').manual_seed(6)
    stream = _lib.stream_handle()

    def events(fn, n):
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(n):
            fn()
        b.record()
        torch.cuda.synchronize()
        return a.elapsed_time(b) / 1e3 / n

    x = torch.randn((rows, 16), generator=gen, device='cuda')
    dy = torch.randn(rows, generator=gen, device='cuda') / rows
    y = torch.empty(rows, device='cuda')
    z = torch.empty((3, rows, 128), device='cuda')
    h = torch.empty_like(z)
    grad = torch.empty(mlp.nparams, device='cuda')
    nbytes = _lib.c_size_t()
    _lib.call('pk_mlp_backward_workspace_size', rows, _lib.ctypes.byref(nbytes))
    ws = torch.empty(nbytes.value, dtype=torch.uint8, device='cuda')
    _lib.call('pk_mlp_forward_tc', stream, _lib.ptr(x), None, rows, _lib.ptr(mlp.wb), _lib.ptr(mlp.w), _lib.ptr(y),
              _lib.ptr(z), _lib.ptr(h), _lib.ptr(mlp.status))
    common = (_lib.ptr(x), None, rows, _lib.ptr(mlp.wb), _lib.ptr(z), _lib.ptr(h), _lib.ptr(dy), _lib.ptr(grad),
              _lib.ptr(ws), ws.numel())
    t_tc = events(lambda: _lib.call('pk_mlp_backward_tc', stream, *common, _lib.ptr(mlp.status)), reps)
    t_mma = events(lambda: _lib.call('pk_mlp_backward', stream, *common), reps)
    flops = 2. * 128 * (16 + 2 * 128) * rows + 2. * 128 * 2 * 128 * rows
    del z, h, y, ws
    # one training step at the training batch, as a graph of `reps` steps
    n = 16 * batch
    xt = torch.randn((n, 16), generator=gen, device='cuda')
    target = torch.randn(n, generator=gen, device='cuda')
    mlp.fit(xt, target, steps=16, batch=batch, graph=False)  # warm-up, kernel attributes
    torch.cuda.synchronize()
    step_s = mlp.fit_step_seconds(xt, target, batch=batch, steps=reps)
    mlp.check()
    return dict(backward_rows=rows, backward_seconds_tc=t_tc, backward_seconds_mma_sync=t_mma,
                backward_tflops_tc=flops / t_tc / 1e12, backward_tflops_mma_sync=flops / t_mma / 1e12,
                training_batch=batch, training_step_ms=step_s * 1e3,
                timing='CUDA events; backward: %d calls on resident rows and stored activations; training step: '
                       'a CUDA graph of %d steps (forward, loss, backward, reduction, AdamW) replayed' % (reps, reps))


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
    catalog = benchmark_catalog(seed=W['seed'] + rank, meshsize=W['meshsize'])
    positions = torch.as_tensor(catalog).cuda()
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
        # every step copies its positions from pinned host memory and reads its multipoles
        # back to the host; the copy of step k + 1 runs on a copy stream while step k computes
        # (two device buffers, events order the copy after the step that last used the buffer),
        # and step k's multipoles are read back (prefetch: a side-stream copy) while step k + 1
        # runs: the host waits for them after enqueuing step k + 1, the last one before the
        # timing event
        host = torch.empty(positions.shape, dtype=torch.float32, pin_memory=True)
        host.copy_(positions)
        bufs = [torch.empty_like(positions) for _ in range(2)]
        copied = [torch.cuda.Event() for _ in range(2)]
        used = [torch.cuda.Event() for _ in range(2)]
        copy_stream = torch.cuda.Stream()
        compute = torch.cuda.current_stream()

        def issue_copy(k):
            with torch.cuda.stream(copy_stream):
                copy_stream.wait_event(used[k % 2])
                bufs[k % 2].copy_(host, non_blocking=True)
                copied[k % 2].record(copy_stream)

        def run_steps(n):
            copy_stream.wait_stream(compute)  # the first copy starts after the timing event
            issue_copy(0)
            prev = None
            for k in range(n):
                if k + 1 < n:
                    issue_copy(k + 1)
                compute.wait_event(copied[k % 2])
                res = step(bufs[k % 2])
                used[k % 2].record(compute)
                res.prefetch()
                if prev is not None:
                    _ = prev.value()
                prev = res
            if prev is not None:
                _ = prev.value()

        for e in used:
            e.record(compute)
        run_steps(args.warmup)
        barrier()
        start2, end2 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start2.record()
        run_steps(args.steps)
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
    achieved = abytes / (ours[dominant]['mean_ms'] * 1e-3) / 1e9 if abytes else None
    launches = sum(LAUNCHES.get(k, 0) * v['calls'] for k, v in stages.items())
    stage_report = {k: {'calls': v['calls'], 'mean_ms': round(v['mean_ms'], 4),
                        'share': round(v['total_ms'] / (elapsed * 1e3), 4)} for k, v in stages.items()}
    line = {'metric': METRIC, 'value': value, 'unit': 'spectra/s', 'n_gpus': world, 'steps': args.steps,
            'warmup': args.warmup, 'ms_per_step': elapsed * 1e3 / args.steps, 'higher_is_better': True,
            'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f32', 'data': 'synthetic',
            'config': dict(W, nparticles=int(npart), parallelism='replicas' if world > 1 else 'single',
                           l2='inputs larger than L2 (512 MiB meshes per shift)', out='complex'),
            'roofline': {'bound': 'hbm', 'kernel': dominant, 'achieved': achieved, 'peak': peak,
                         'peak_kind': peak_kind, 'unit': 'GB/s', 'frac': achieved / peak if achieved else None,
                         'algorithmic_bytes': abytes,
                         'traffic': float(PAINT_TRAFFIC_512) if (dominant in ('pk_paint', 'pk_paint_batch')
                                                                 and W['meshsize'] == 512) else None,
                         'traffic_source': 'ncu dram read+write of the pk_paint kernels (bucket count, column scan, '
                                           'placement, per-shift tiles), this workload at 512^3'},
            'roofline_binning': binning_roofline(stages, bins, W, peak),
            'e2e': {'value': e2e_value, 'unit': 'spectra/s', 'h2d_bytes_per_step': int(npart * 12),
                    'd2h_bytes_per_step': int(len(W['ells']) * nbins * 8)},
            'gpu_launches': int(launches), 'stages': stage_report, 'clocks': clocks.summary()}
    details = {}
    if (world > 1 or args.sharded_mocks) and not args.no_batched:  # every rank: mocks shared out, one gather
        line['sharded_mocks'] = run_sharded_mocks(world, rank, barrier, max_over_ranks)
    if rank == 0 and world == 1 and not args.no_batched:
        details['batched'] = run_batched()
        line['batched'] = summary(details['batched'], ('plain_spectra_per_s', 'batched_spectra_per_s', 'speedup',
                                                       'covariance_max_rel_vs_plain', 'fp64_max_rel'))
    if rank == 0 and world == 1 and not args.no_cutsky:
        details['cutsky'] = run_cutsky()
        line['cutsky'] = summary(details['cutsky'], ('spectra_per_s', 'seconds_forward', 'seconds_forward_backward'))
        line['cutsky']['gradient_rel_err'] = details['cutsky']['gradient_check']['rel_err']
    if rank == 0 and world == 1 and not args.no_learned:
        details['learned'] = run_learned()
        details['learned']['mlp_forward'] = run_mlp_forward()
        details['learned']['mlp_training'] = run_mlp_training()
        line['learned'] = learned_summary(details['learned'])
    if rank == 0 and world == 1 and not args.no_cpu:
        # the CPU oracle on the same catalog: one whole 512^3 spectrum, timed (no scaling)
        spectrum, _ = oracle_pipeline(meshsize=W['meshsize'], catalog=catalog)
        t0 = time.perf_counter()
        ref32 = spectrum()
        seconds = time.perf_counter() - t0
        line['cpu_baseline'] = {'value': 1. / seconds, 'unit': 'spectra/s', 'cores': cpu_cores(), 'kind': 'port',
                                'sample': ORACLE_SAMPLE + '; 1 timed spectrum'}
        got = np.array([p.num_raw for p in result])
        scale = np.abs(ref32['num_raw'][0]).max()
        parity = {'c1_max_rel_vs_fp32_oracle': float(np.abs(got - ref32['num_raw']).max() / scale),
                  'c1_nmodes_exact': bool(np.array_equal(np.asarray(bins.nmodes), ref32['nmodes']))}
        if not args.no_fp64:
            parity.update(fp64_errors(W, catalog, got, bins))
        details['c0'] = run_c0()
        parity['c0_max_rel_vs_fp32_oracle'] = details['c0']['max_rel_diff_vs_oracle']
        parity['c0_max_rel_vs_fp64_oracle'] = details['c0']['max_rel_diff_vs_fp64_oracle']
        line['c0'] = summary(details['c0'], ('gpu_spectra_per_s', 'cpu_oracle_spectra_per_s'))
        line['parity'] = parity
    if rank == 0:
        if args.details:
            with open(args.details, 'w') as f:
                json.dump(details, f, indent=1)
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def summary(report, keys):
    return {k: report[k] for k in keys if k in report}


def learned_summary(r):
    """Scalar figures of the learned-correction report (the full report goes to --details)."""
    out = {'heldout_bias_max_learned': r['heldout_bias_max']['learned'],
           'heldout_bias_max_table': r['heldout_bias_max']['mean_table_128'],
           'heldout_bias_max_plain_128': r['heldout_bias_max']['plain_128'],
           'heldout_bias_sigma_learned': r['heldout_bias_in_standard_errors']['learned'],
           'heldout_bias_sigma_table': r['heldout_bias_in_standard_errors']['mean_table_128'],
           'heldout_bias_chi2_per_bin_learned': r['heldout_bias_chi2_per_bin']['learned'],
           'heldout_bias_chi2_per_bin_table': r['heldout_bias_chi2_per_bin']['mean_table_128'],
           'per_mock_max_rel_err_median_learned': r['heldout_max_rel_err']['learned']['median'],
           'per_mock_max_rel_err_median_table': r['heldout_max_rel_err']['mean_table_128']['median'],
           'frac_heldout_within_0p5pct': r['frac_heldout_within_0p5pct'],
           'per_mock_target_0p5pct_met': r['frac_heldout_within_0p5pct'] >= 0.5,
           'batched_speedup_learned_vs_plain_512': r['batched_speedup_learned_vs_plain_512'],
           'seconds_training': r['seconds_training'],
           'mlp_forward_tflops': r['mlp_forward']['tflops']}
    if 'mlp_training' in r:
        t = r['mlp_training']
        out.update(mlp_backward_tflops_tc=t['backward_tflops_tc'], mlp_backward_tflops_mma_sync=t['backward_tflops_mma_sync'],
                   training_step_ms=t['training_step_ms'])
    for k in ('heldout_rms_gain_vs_table_sigma',):
        if k in r:
            out[k] = r[k]
    return out


def fp64_errors(W, catalog, got, bins):
    """Error of the GPU multipoles against the oracle's float64 pipeline: the benchmark catalog
    (512^3), and the cut-sky first-point configuration at 256^3 (its full catalog), as
    max |P_gpu - P_fp64| / max |P_0 fp64| over the bins whose float32 and float64 mode counts agree."""
    spectrum64, _ = oracle_pipeline(meshsize=W['meshsize'], catalog=catalog, dtype=np.float64)
    ref = spectrum64()
    same = np.asarray(bins.nmodes) == ref['nmodes']
    out = {'c1_max_rel_vs_fp64_oracle': float(np.abs(got[:, same] - ref['num_raw'][:, same]).max()
                                              / np.abs(ref['num_raw'][0][same]).max()),
           'c1_bins_with_other_fp64_nmodes': int((~same).sum())}
    out.update(cutsky_fp64_error(meshsize=256))
    return out


def cutsky_fp64_error(meshsize=256):
    import torch
    import jaxpower_b200 as jp
    from jaxpower_b200.mock import cutsky_particles
    from oracle.coords import Geometry
    from oracle import paint as opaint
    from oracle.spectrum import Bins, compute_mesh2_spectrum, fkp_particles
    C = CUTSKY
    data, randoms, wd, wr = cutsky_particles(ndata=C['ndata'], nrandoms=C['nrandoms'], seed=C['seed'])
    attrs = jp.get_mesh_attrs(data, randoms, meshsize=meshsize, boxpad=C['boxpad'])
    b = jp.BinMesh2SpectrumPoles(attrs, edges={'step': C['k_step']}, ells=C['ells'])
    fkp = jp.FKPField(jp.ParticleField(data, wd, attrs=attrs), jp.ParticleField(randoms, wr, attrs=attrs))
    mesh = fkp.paint(resampler=C['resampler'], interlacing=C['interlacing'], compensate=True, out='real')
    got = np.array([p.num_raw for p in jp.compute_mesh2_spectrum(mesh, bin=b, los='firstpoint')])
    host = [t.cpu().numpy() for t in (data, wd, randoms, wr)]
    del mesh, fkp, data, randoms
    torch.cuda.empty_cache()
    geom = Geometry(attrs.meshsize, attrs.boxsize, attrs.boxcenter, dtype=np.float64)
    pos, w, _ = fkp_particles(*host, dtype=np.float64)
    ref = compute_mesh2_spectrum(opaint.paint(geom, pos, w, C['resampler'], C['interlacing'], True, 'real'),
                                 Bins(geom, step=C['k_step'], ells=C['ells']), los='firstpoint')
    same = np.asarray(b.nmodes) == ref['nmodes']
    return {'c2_meshsize': meshsize,
            'c2_max_rel_vs_fp64_oracle': float(np.abs(got[:, same] - ref['num_raw'][:, same]).max()
                                               / np.abs(ref['num_raw'][0][same]).max()),
            'c2_bins_with_other_fp64_nmodes': int((~same).sum())}


def main():
    parser = argparse.ArgumentParser(description=__doc__.split('\n')[0])
    parser.add_argument('--gpus', type=int, default=1)
    parser.add_argument('--steps', type=int, default=20)
    parser.add_argument('--warmup', type=int, default=5)
    parser.add_argument('--impl', default='ours', choices=['ours', 'reference'])
    parser.add_argument('--ref-budget', type=float, default=240.,
                        help='--impl reference: stop the timed oracle spectra after this many seconds (>= 1 step)')
    parser.add_argument('--no-cpu', action='store_true', help='skip the CPU baseline and parity against the oracle')
    parser.add_argument('--no-fp64', action='store_true', help='skip the float64-oracle errors')
    parser.add_argument('--details', default='', help='write the full sub-reports (JSON) to this file')
    parser.add_argument('--no-e2e', action='store_true', help='skip the end-to-end (host buffers) measurement')
    parser.add_argument('--meshsize', type=int, default=0, help='smaller mesh of the same workload (profiling)')
    parser.add_argument('--no-batched', action='store_true', help='skip the batched-mocks measurement')
    parser.add_argument('--sharded-mocks', action='store_true',
                        help='run the sharded-mocks measurement (every N > 1 run does) also with one GPU')
    parser.add_argument('--no-learned', action='store_true', help='skip training / evaluating the learned correction')
    parser.add_argument('--no-cutsky', action='store_true', help='skip the cut-sky FKP first-point measurement')
    parser.add_argument('--mlp-forward-only', action='store_true',
                        help='only time the correction network forward pass (profiling aid)')
    parser.add_argument('--mlp-training-only', action='store_true',
                        help='only time the correction network backward pass and training step (profiling aid)')
    parser.add_argument('--paint-only', action='store_true',
                        help='only paint the benchmark catalog (at --meshsize if given; profiling aid)')
    parser.add_argument('--paint-config', type=int, default=4, help='tile configuration of --paint-only')
    parser.add_argument('--window-only', action='store_true',
                        help='only time window matrices (at --meshsize if given; profiling aid)')
    parser.add_argument('--cutsky-forward-only', action='store_true',
                        help='only run the cut-sky first-point forward pipeline (at --meshsize if given; profiling aid)')
    args = parser.parse_args()
    if args.mlp_forward_only:
        print(json.dumps({'mlp_forward': run_mlp_forward()}), flush=True)
        return
    if args.mlp_training_only:
        print(json.dumps({'mlp_training': run_mlp_training()}), flush=True)
        return
    if args.paint_only:
        print(json.dumps({'paint': run_paint_only(args.meshsize or None, config=args.paint_config)}), flush=True)
        return
    if args.window_only:
        print(json.dumps({'window': run_window_only(args.meshsize or None)}), flush=True)
        return
    if args.cutsky_forward_only:
        print(json.dumps({'cutsky_forward': run_cutsky_forward_only(args.meshsize or None)}), flush=True)
        return
    if args.impl == 'reference':
        run_reference(args)
    else:
        run_ours(args)


if __name__ == '__main__':
    main()

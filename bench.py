#!/usr/bin/env python
"""Benchmark: particle-steps/s of the FLIP sub-step, batched against plain, on one GPU per rank.

Default workload (`--workload batch`): 64 independent tanks of uneven sizes, each grid axis drawn from
{16, 24, 32, 48, 64} cells, h = 1 m / (vertical cells), a bottom block filled to U[0.2, 0.6] at 8 particles
per cell, 0-3 random obstacles (sphere, box or cylinder; face fractions from analytic SDFs), 80 SOR
iterations at ω = 1.7, FLIP 0.95, dt = 1/240 s (11.7M particles, 3.7M cells; seed = tank index). A step is
one sub-step of all 64 tanks: binning, P2G, forces and divergence, the pressure solve, projection, G2P with
collisions and drop/whitewater logic, advanced together by the batched, graph-captured launches with the
form of the pressure solve picked by the autotuner. `value` is the batch's particle-steps/s; the same 64
scenes stepped one by one on the plain path give `plain_sequential`. At one GPU the line also carries
`serving`: p50/p99 request latency of the serving loop over a short Poisson run at 10 requests/s
(`--serve-sample` seconds). Synthetic seeded data.

Other workloads: `obstacles_inflow` (one 128×64×64 tank with obstacles, a faucet and a drain),
`full_scene` (256×128×128 with rain and the 1024×512 ripple layer), `frame_export` (that scene's per-frame
surface mesh and light/surface maps), `serve` (Poisson scene requests).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl suiri|reference] [--workload ...]

Under torchrun each rank advances its own replica of the workload (tanks do not interact: no collective in
the data path); the time is the max over ranks and the value counts every rank's particles. `--impl
reference` times the reference's CPU solver (its NumPy restatement, pinned bit-exact against it) on the
same workload on this host's cores.
"""
import argparse
import importlib
import json
import math
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
METRIC = 'particle-steps/s'
L2_FLUSH_BYTES = 256 << 20          # larger than the 126 MB L2; written between timed steps
DT = 1 / 240


def pkg():
    return importlib.import_module('hahenn-_b200')


def peaks():
    try:
        with open(os.path.join(ROOT, 'MEASURED_PEAKS.json')) as f:
            p = json.load(f)
        return float(p['hbm_gbs']), 'measured'
    except Exception:
        return 6650.0, 'fallback'


def profile_figure(name):
    """A figure from a committed ncu summary under profiles/ (None if absent)."""
    try:
        with open(os.path.join(ROOT, 'profiles', name)) as f:
            return json.load(f)
    except Exception:
        return None


class Clocks:
    """SM clock and throttle reasons sampled every 5 ms during the timed region (NVML reads only; the
    nvidia-smi query loop is the fallback)."""
    Q = 'clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,' \
        'clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap'
    BITS = {'sw_power_cap': 0x4, 'hw_slowdown': 0x8, 'sw_thermal_slowdown': 0x20, 'hw_thermal_slowdown': 0x40}

    def __init__(self, device):
        self.device, self.rows, self.proc = device, [], None
        self.stop_flag = threading.Event()
        self.nv = None

    def _handle(self):
        import pynvml
        pynvml.nvmlInit()
        try:
            import torch
            pr = torch.cuda.get_device_properties(self.device)
            bus = f'{int(pr.pci_domain_id):08X}:{int(pr.pci_bus_id):02X}:{int(pr.pci_device_id):02X}.0'
        except Exception:
            bus = None
        if bus is not None:      # the PCI id as NVML spells it ("00000000:1B:00.0"); a non-string here would crash NVML
            try:
                return pynvml, pynvml.nvmlDeviceGetHandleByPciBusId(bus.encode())
            except Exception:
                pass
        return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.device)

    def start(self):
        try:
            self.nv = self._handle()
            threading.Thread(target=self._poll, daemon=True).start()
            return
        except Exception:
            self.nv = None
        try:
            self.proc = subprocess.Popen(['nvidia-smi', f'--query-gpu={self.Q}', '--format=csv,noheader,nounits',
                                          '-lms', '200', '-i', str(self.device)], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            threading.Thread(target=self._read, daemon=True).start()
        except Exception:
            self.proc = None

    def _poll(self):
        nv, h = self.nv
        mx = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
        while not self.stop_flag.is_set():
            try:
                sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
                r = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
            except Exception:
                break
            act = ['Active' if r & self.BITS[k] else 'Not Active'
                   for k in ('hw_slowdown', 'hw_thermal_slowdown', 'sw_thermal_slowdown', 'sw_power_cap')]
            self.rows.append([str(sm), str(mx)] + act)
            time.sleep(0.005)

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(',')])

    def stop(self):
        self.stop_flag.set()
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        time.sleep(0.02)
        rows = list(self.rows)
        sm = [float(r[0]) for r in rows if r and r[0].replace('.', '').isdigit()]
        mx = [float(r[1]) for r in rows if len(r) > 1 and r[1].replace('.', '').isdigit()]
        names = ['hw_slowdown', 'hw_thermal_slowdown', 'sw_thermal_slowdown', 'sw_power_cap']
        reasons = sorted({names[i] for r in rows for i in range(4) if len(r) > 2 + i and r[2 + i] == 'Active'})
        return dict(sm_mhz=float(np.median(sm)) if sm else None, sm_max_mhz=max(mx) if mx else None,
                    reasons=reasons, samples=len(sm), source='nvml' if self.nv else 'nvidia-smi')


# ------------------------------------------------------------------ workloads
def make_tank(P, w, device, host_inflow=False):
    """The single-tank workload (obstacles and inflow) on the plain path."""
    prm = w['params']
    t = P.Tank(nx=w['nx'], ny=w['ny'], nz=w['nz'], h=w['h'], flip=prm['flip'], omega=prm['omega'], iters=prm['iters'],
               gravity=prm['g'], whitewater=True, ripple=None, capacity=int(len(w['pos']) * 1.25) + 100000,
               device=device, sdf_mode='analytic')
    t.set_objects(w['objects'])
    t.add_particles(w['pos'])
    if not host_inflow:
        t.set_emitters([dict(shape='disc', pos=e['pos'], dir=e['dir'], radius=e['radius'], speed=e['speed'],
                             count=e['count']) for e in w['emitters']])
    return t


def faucet_particles(e, dt, rng):
    """The faucet's particles of one sub-step generated on the host (for the end-to-end measurement)."""
    n = e['count']
    d = np.array(e['dir'], float); d /= np.linalg.norm(d)
    ref = np.array([0.0, 1.0, 0.0]) if abs(d[1]) < 0.95 else np.array([1.0, 0.0, 0.0])
    u = np.cross(d, ref); u /= np.linalg.norm(u)
    w = np.cross(d, u)
    rr = e['radius'] * np.sqrt(rng.random(n)); th = 2 * math.pi * rng.random(n)
    p = np.array(e['pos']) + (np.cos(th)[:, None] * u + np.sin(th)[:, None] * w) * rr[:, None] \
        + d * (rng.random(n) * e['speed'] * dt)[:, None]
    v = d * e['speed'] + (rng.random((n, 3)) - 0.5) * (0.02 * e['speed'])
    return p.astype(np.float32), v.astype(np.float32)


def batch_specs(n):
    return pkg().workloads.batch_tanks(n)


def batch_config(specs):
    """The batching workload's config, identical in both arms."""
    return dict(workload=f'batch_{len(specs)}_tanks', tanks=len(specs),
                particles=int(sum(len(w['pos']) for w in specs)),
                cells=int(sum(w['nx'] * w['ny'] * w['nz'] for w in specs)),
                axes=[16, 24, 32, 48, 64], sor_iters=80, omega=1.7, flip=0.95, dt=DT, sdf_mode='analytic',
                whitewater=True, seed='tank index')


def plain_config(w):
    prm = w['params']
    return dict(workload=w['name'], particles=int(len(w['pos'])), cells=w['nx'] * w['ny'] * w['nz'],
                sor_iters=prm['iters'], omega=prm['omega'], flip=prm['flip'], dt=prm['dt'], sdf_mode='analytic',
                inflow_per_step=w['emitters'][0]['count'], whitewater=True)


def make_batch_tanks(P, specs, device, add=True):
    ts = []
    for w in specs:
        prm = w['params']
        t = P.Tank(nx=w['nx'], ny=w['ny'], nz=w['nz'], h=w['h'], flip=prm['flip'], omega=prm['omega'],
                   iters=prm['iters'], gravity=prm['g'], whitewater=True, ripple=None,
                   capacity=int(len(w['pos']) * 1.2) + 1000, ww_capacity=20000, device=device, sdf_mode='analytic')
        t.set_objects(w['objects'])
        if add:
            t.add_particles(w['pos'])
        ts.append(t)
    return ts


def size_lanes(specs):
    """Each tank's size lane as the library forms them (under 2^16 cells, under 2^19, larger; occupied lanes
    in that order) and the number of lanes."""
    raw = [0 if c < 1 << 16 else (1 if c < 1 << 19 else 2) for c in (w['nx'] * w['ny'] * w['nz'] for w in specs)]
    occ = sorted(set(raw))
    return [occ.index(r) for r in raw], len(occ)


def launches_per_substep(sor_mode, iters, residual=False, g2p_form=0):
    """Kernels of one sub-step graph of a group (bin, scan ×2, scatter and the rest: 10) plus the solve's, and
    the deferred pass of G2P form 2."""
    sor = {0: 2 * iters, 1: 1, 2: 1 + iters + (iters & 1), 3: -(-2 * iters // 4) + (-(-2 * iters // 4) & 1), 4: 1}[sor_mode]
    return 10 + (sor if iters > 0 else 0) + (2 if residual else 0) + (1 if g2p_form == 2 else 0)


# ------------------------------------------------------------------ the CPU oracle (reference arm, cpu_baseline)
def _port_tank(w, ww_cap=140000):
    """The CPU oracle (NumPy restatement of the reference solver) set up on a workload tank, obstacles as the
    web version's analytic shapes, as the GPU arm uses them."""
    from oracle import flip as of
    from oracle import sdf as sdfm
    prm = w['params']
    t = of.Tank(w['nx'], w['ny'], w['nz'], w['h'], origin=w['origin'], flip=prm['flip'], omega=prm['omega'],
                iters=prm['iters'], g=prm['g'], whitewater=True, rng_mode='hash', sdf_mode='analytic', ww_cap=ww_cap)
    objs = []
    for it in w['objects']:
        if it['kind'] == 'obstacle':
            objs.append(sdfm.make_obstacle(it['shape'], it['pos'], tuple(it['rot']), **it['dims']))
        else:
            objs.append(sdfm.make_drain(it['pos'], it['r'], tuple(it['rot'])))
    t.set_objects(objs)
    t.add_particles(w['pos'].astype(np.float64))
    return t


def _port_steps(tanks, specs, steps, rng):
    """`steps` sub-steps of every oracle tank (faucet particles added on the host); returns particle-steps."""
    n_ps = 0
    for _ in range(steps):
        for t, w in zip(tanks, specs):
            for e in w['emitters']:
                p, v = faucet_particles(e, w['params']['dt'], rng)
                t.add_particles(p.astype(np.float64), v.astype(np.float64))
            n_ps += len(t.pos)
            t.frame += 1
            t.substep(w['params']['dt'])
    return n_ps


def _workload_specs(workload, n_tanks):
    P = pkg()
    if workload == 'batch':
        return P.workloads.batch_tanks(n_tanks)
    return [P.workloads.obstacles_inflow()]


def _port_worker(workload, n_tanks, idx, steps, warm, barrier, out, k):
    """One CPU process (spawned): its share of the workload's tanks, warmed up, then `steps` timed sub-steps
    of all of them from a common start."""
    sys.path.insert(0, ROOT)
    specs = [_workload_specs(workload, n_tanks)[i] for i in idx]
    ww = 20000 if workload == 'batch' else 140000
    tanks = [_port_tank(w, ww) for w in specs]
    rng = np.random.default_rng(1 + k)
    if warm:
        _port_steps(tanks, specs, warm, rng)
    barrier.wait(timeout=900)
    t0 = time.perf_counter()
    n_ps = _port_steps(tanks, specs, steps, rng)
    out.put((n_ps, time.perf_counter() - t0))


def cpu_processes():
    """One process per usable core, at most 32, and at most one per 2 GB of available memory."""
    cores = len(os.sched_getaffinity(0))
    avail_gb = 0.0
    try:
        with open('/proc/meminfo') as f:
            for line in f:
                if line.startswith('MemAvailable:'):
                    avail_gb = int(line.split()[1]) / 1e6
    except OSError:
        avail_gb = 2.0
    return max(1, min(cores, 32, int(avail_gb // 2)))


def partition(sizes, parts):
    """Indices split into `parts` groups of near-equal total size (largest first onto the lightest group)."""
    groups, load = [[] for _ in range(parts)], [0] * parts
    for i in sorted(range(len(sizes)), key=lambda i: -sizes[i]):
        g = load.index(min(load))
        groups[g].append(i)
        load[g] += sizes[i]
    return [g for g in groups if g]


def cpu_parallel_rate(workload, n_tanks, steps, warm, procs):
    """The workload on `procs` processes of one core each, timed together from a common start: all processes'
    particle-steps ÷ the slowest process's time. The batch's tanks are partitioned over the processes; the
    single-tank workload runs one replica per process."""
    import multiprocessing as mp
    specs = _workload_specs(workload, n_tanks)
    if workload == 'batch':
        groups = partition([len(w['pos']) for w in specs], procs)
    else:
        groups = [[0] for _ in range(procs)]
    ctx = mp.get_context('spawn')
    barrier, out = ctx.Barrier(len(groups)), ctx.Queue()
    env = {k: os.environ.get(k) for k in ('OMP_NUM_THREADS', 'OPENBLAS_NUM_THREADS', 'MKL_NUM_THREADS')}
    for k in env:
        os.environ[k] = '1'
    ps = [ctx.Process(target=_port_worker, args=(workload, n_tanks, g, steps, warm, barrier, out, k))
          for k, g in enumerate(groups)]
    for p in ps:
        p.start()
    res = [out.get(timeout=3600) for _ in ps]
    for p in ps:
        p.join(timeout=60)
    for k, v in env.items():
        if v is None:
            os.environ.pop(k, None)
        else:
            os.environ[k] = v
    el = max(r[1] for r in res)
    return sum(r[0] for r in res) / el, el, len(groups)


def cpu_sample_rate(specs, steps=1, every=4):
    """The oracle on one core over a bounded sample of the workload: every `every`-th tank, `steps`
    sub-steps (setup untimed). Returns particle-steps/s, seconds and the sample's description."""
    sub = specs[::every]
    tanks = [_port_tank(w, 20000 if len(specs) > 1 else 140000) for w in sub]
    rng = np.random.default_rng(1)
    t0 = time.perf_counter()
    n_ps = _port_steps(tanks, sub, steps, rng)
    el = time.perf_counter() - t0
    what = (f'{len(sub)} of the {len(specs)} tanks (every {every}th, {sum(len(w["pos"]) for w in sub)} particles)'
            if len(specs) > 1 else 'the tank')
    return n_ps / el, el, f'{what} × {steps} sub-step(s) on the host, 1 core of {os.cpu_count()} (NumPy ' \
                          f'restatement of the reference solver, {el:.1f} s)'


def run_reference(args, rank):
    """The reference's CPU path (its NumPy solver, restated and pinned bit-exact against it) on the same
    workload, on this host's cores: rank 0 only; other ranks exit at once."""
    if rank != 0:
        return
    workload = 'batch' if args.workload == 'batch' else 'obstacles_inflow'
    specs = _workload_specs(workload, args.tanks)
    cfg = batch_config(specs) if workload == 'batch' else plain_config(specs[0])
    steps, warm = max(1, args.steps), max(0, args.warmup)
    procs = cpu_processes()
    rate, el, used = cpu_parallel_rate(workload, args.tanks, steps, warm, procs)
    if workload == 'batch':
        sample = (f'all {len(specs)} tanks partitioned over {used} processes (one core each, balanced by particle '
                  f'count), each stepping all of its tanks {steps} timed sub-steps after {warm} warm-up')
    else:
        sample = f'{used} replicas of the tank, one process and one core each, {steps} timed sub-steps after {warm}'
    line = dict(impl='reference', metric=METRIC, value=rate, unit=METRIC, n_gpus=args.gpus, steps=steps, warmup=warm,
                ms_per_step=1000 * el / steps, higher_is_better=True, scaling='weak', vs_baseline=None, dtype='f64',
                data='synthetic (seeded particles, analytic obstacles)', config=cfg,
                cpu_baseline=dict(value=rate, unit=METRIC, cores=used, kind='port',
                                  sample=sample + ' (NumPy restatement of the reference solver, pinned bit-exact '
                                                  'against it; NumPy runs one core per process)'),
                e2e=dict(value=rate, unit=METRIC, h2d_bytes_per_step=0, d2h_bytes_per_step=0))
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------ multi-rank bookkeeping
def reduce_ranks(ms, particles, sor_launch_ms, device):
    """Whole-job figures of the replicas: the slowest rank's step and SOR-launch times (max over ranks) and
    the particles of all ranks (sum), so value = all ranks' particle-steps ÷ the slowest rank's time."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([ms, particles, sor_launch_ms], dtype=torch.float64, device=device)
    mx = t.clone()
    dist.all_reduce(mx, op=dist.ReduceOp.MAX)
    tot = t.clone()
    dist.all_reduce(tot, op=dist.ReduceOp.SUM)
    return float(mx[0]), float(tot[1]), float(mx[2])


def reduce_e2e(rate, world, device):
    """End-to-end rate of the whole job: the slowest rank's rate times the number of ranks."""
    import torch
    import torch.distributed as dist
    x = torch.tensor([rate], dtype=torch.float64, device=device)
    dist.all_reduce(x, op=dist.ReduceOp.MIN)
    return float(x[0]) * world


def init_ranks(world, local):
    import torch
    import torch.distributed as dist
    if world > 1:
        import datetime
        dist.init_process_group('nccl', timeout=datetime.timedelta(seconds=120))
    torch.cuda.set_device(local)


# ------------------------------------------------------------------ the batching workload (default)
def e2e_batch(P, specs, device, best, steps, workers=8):
    """The job end to end through the public API with host buffers: every scene's particles added from host
    arrays (page-locked, copied by the copy engine), `steps` batched sub-steps with each scene's stats
    read back every sub-step (pollStats), and every scene's particles read back into page-locked host arrays
    (the ABI's pos4/vel4 layout) at the end. The scenes are uploaded and read back from `workers` host threads, one
    scene per thread at a time (handles are per thread; the ctypes calls release the interpreter lock).
    Wall clock around all of it, after two untimed runs of the same job (graph capture, and the two pinned
    staging buffers a tank alternates between, as a loop that keeps uploading scenes has them)."""
    from concurrent.futures import ThreadPoolExecutor
    tanks = make_batch_tanks(P, specs, device, add=False)
    b = P.Batch(tanks)
    for k, knobs in enumerate(best):
        b.tune_lane(k, *knobs)
    import torch
    # the scenes' positions and the read-back live in page-locked arrays, allocated once as a client that
    # uploads and reads every run keeps them: the copy engine reads and writes them directly (pageable arrays
    # go through the tanks' pinned buffers and a host copy)
    host = [torch.from_numpy(np.ascontiguousarray(w['pos'], np.float32)).pin_memory().numpy() for w in specs]
    pinned = [tuple(torch.empty((len(p) + 64, 4), dtype=torch.float32, pin_memory=True) for _ in range(2)) for p in host]
    outs = [(a.numpy(), b.numpy()) for a, b in pinned]
    readback = int(P.native.lib().suiri_stats_readback_bytes())
    pool = ThreadPoolExecutor(max_workers=workers)

    split = {}

    def job(n_steps):
        t0 = time.perf_counter()
        list(pool.map(lambda tp: tp[0].add_particles(tp[1]), zip(tanks, host)))
        h2d = sum(12 * len(p) for p in host)          # the positions, copied packed (3 float32 per particle)
        d2h = 0
        t1 = time.perf_counter()
        for _ in range(n_steps):
            b.substep(DT)
            for t in tanks:
                t.poll_stats()
                d2h += readback
        b.sync()
        t2 = time.perf_counter()
        res = list(pool.map(lambda to: to[0].particles4(to[1]), zip(tanks, outs)))
        n_end = sum(len(r[0]) for r in res)
        split.update(upload_s=t1 - t0, substeps_s=t2 - t1, readback_s=time.perf_counter() - t2)
        return h2d, d2h + 32 * n_end, n_end

    for _ in range(2):      # untimed: graph capture, and both pinned staging buffers each tank alternates between
        job(3)
        for t in tanks:
            t.clear_water()
        b.sync()
    t0 = time.perf_counter()
    h2d, d2h, n_end = job(steps)
    el = time.perf_counter() - t0
    pool.shutdown()
    n0 = sum(len(p) for p in host)
    b.close()
    for t in tanks:
        t.close()
    return dict(value=0.5 * (n0 + n_end) * steps / el, unit=METRIC, h2d_bytes_per_step=h2d // steps,
                d2h_bytes_per_step=d2h // steps, wall_s=el, host_threads=workers, split=dict(split),
                job=f'{len(specs)} scenes uploaded from host arrays, {steps} batched sub-steps with every scene\'s '
                    f'stats read back each sub-step, every scene\'s particles read back at the end')


def solve_residual(target, tanks, dt):
    """The FP64 residual of one more sub-step's pressure solve (after the timed region), per tank: max
    |h²·div − A·p| over the active cells, relative to max |h²·div|; the largest over the tanks."""
    target.residual(True)
    target.substep(dt)
    target.sync()
    st = [t.stats() for t in tanks]
    target.residual(False)
    rel = [s['residual_max'] / s['rhs_max'] for s in st if s['rhs_max'] > 0]
    return dict(max_abs=max(s['residual_max'] for s in st), max_rel=max(rel) if rel else 0.0,
                rms_max=max(s['residual_rms'] for s in st), tanks=len(st),
                note='FP64 residual r = sum C p_nb - h^2 div - (sum C) p of the solve, float64 from the float32 operands, '
                     'over the active cells, one sub-step after the timed region; rel = max|r| / max|h^2 div| per tank')


def run_batch(args, rank, world, local):
    import torch
    import torch.distributed as dist
    init_ranks(world, local)
    P = pkg()
    autotune_batch = importlib.import_module('hahenn-_b200.autotune').autotune_batch
    specs = batch_specs(args.tanks)
    cfg = batch_config(specs)
    lane_of, nlanes = size_lanes(specs)
    dev = f'cuda:{local}'

    # the same scenes one by one on the plain path (each tank's own sub-step graph and stream)
    plain = make_batch_tanks(P, specs, local)
    for t in plain:
        t.substep(DT)                                # GEOM and graph capture, untimed
    steps_plain = max(3, min(args.steps, 20))
    ms_plain = sum(t.time_substeps(DT, steps_plain) / steps_plain for t in plain)
    for t in plain:
        t.close()

    tanks = make_batch_tanks(P, specs, local)
    b = P.Batch(tanks)
    best, timings = autotune_batch(b, DT)          # per lane: (blocks per SM, solve form, tile, G2P form)
    b.profile(True)
    stream = torch.cuda.ExternalStream(b.stream())
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=dev)
    for _ in range(max(args.warmup, 3)):
        b.substep(DT)
    b.sync()
    n0 = sum(t.stats()['count'] for t in tanks)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    phases = []
    clocks = Clocks(local)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    for k in range(args.steps):
        with torch.cuda.stream(stream):
            flush.zero_()                          # L2 flush, outside the timed interval
        ev[k][0].record(stream)
        b.substep(DT)
        ev[k][1].record(stream)
        phases.append([b.phase_ms(l) for l in range(nlanes)])
    torch.cuda.synchronize()
    clk = clocks.stop()
    if world > 1:
        dist.barrier()
    step_ms = [a.elapsed_time(c) for a, c in ev]
    st = [t.stats() for t in tanks]
    n1 = sum(s['count'] for s in st)
    ms = float(np.mean(step_ms))
    particles = 0.5 * (n0 + n1)
    sor_lane = [float(np.mean([ph[l]['pressure_solve'] for ph in phases])) for l in range(nlanes)]
    sor_ms = max(sor_lane)
    if world > 1:
        ms, particles, sor_ms = reduce_ranks(ms, particles, sor_ms, dev)
    value = particles * 1000.0 / ms
    b.profile(False)
    residual = solve_residual(b, tanks, DT)
    b.close()
    for t in tanks:
        t.close()
    e2e = e2e_batch(P, specs, local, best, args.steps)
    if world > 1:
        e2e['value'] = reduce_e2e(e2e['value'], world, dev)
    if rank == 0:
        peak, kind = peaks()
        iters = cfg['sor_iters']
        lanes = []
        for l in range(nlanes):
            idx = [i for i in range(len(specs)) if lane_of[i] == l]
            parts = sum(st[i]['count'] for i in idx)
            nodes = sum((specs[i]['nx'] + 1) * (specs[i]['ny'] + 1) * (specs[i]['nz'] + 1) for i in idx)
            active = sum(st[i]['active_cells'] for i in idx)
            cells = sum(specs[i]['nx'] * specs[i]['ny'] * specs[i]['nz'] for i in idx)
            ph = {k: float(np.mean([p[l][k] for p in phases])) for k in P.native.PHASES}
            fig = {}
            # algorithmic bytes per phase: binning 32 B read + 4 B rank, scan 12 B per cell, scatter 64 + 4 B;
            # P2G 32 B per particle + 48 B flush per node; node pass 88 B read + 104 B written per node, cell
            # pass 40 B per cell + 16 B per active list entry; the solve 20 B per active cell and colour sweep;
            # projection 40 B per node; G2P 64 B per particle + 24 B of node gathers per node
            for name, alg in (('bin_sort', 104.0 * parts + 12.0 * cells), ('p2g', 32.0 * parts + 48.0 * nodes),
                              ('grid_passes', 192.0 * nodes + 40.0 * cells + 16.0 * active),
                              ('pressure_solve', 20.0 * active * iters), ('projection', 40.0 * nodes),
                              ('g2p', 64.0 * parts + 24.0 * nodes)):
                gbs = alg / (ph[name] * 1e-3) / 1e9
                fig[name] = dict(alg_bytes=alg, ms=ph[name], achieved_gbs=gbs, frac=gbs / peak)
            lanes.append(dict(tanks=len(idx), particles=parts, nodes=nodes, active_cells=active, phases_ms=ph,
                              kernels=fig, tuned=dict(zip(('blocks_per_sm', 'sor_mode', 'piece_kb', 'g2p_form'),
                                                          best[l]))))
        dom = max(range(nlanes), key=lambda l: lanes[l]['phases_ms']['pressure_solve'])
        sol = lanes[dom]['kernels']['pressure_solve']
        mode = best[dom][1]
        per_launch = 1 if mode in (1, 4) else 2 * iters
        tr = profile_figure('sor_cluster_batch_traffic.json' if mode == 4 else 'sor_batch_traffic.json') or {}
        tr_kind = 'warm' if 'dram_bytes_per_launch' in tr else ('cold' if 'dram_bytes_per_launch_cold' in tr else None)
        roofline = dict(bound='hbm', kernel='k_sor_cluster (whole solve, one launch per lane)' if mode == 4 else
                        f'sor mode {mode}', achieved=sol['achieved_gbs'], peak=peak, unit='GB/s',
                        frac=sol['achieved_gbs'] / peak, peak_kind=kind,
                        traffic=tr.get('dram_bytes_per_launch', tr.get('dram_bytes_per_launch_cold')),
                        traffic_kind=tr_kind, traffic_source='profiles/' + ('sor_cluster_batch_traffic.json' if mode == 4
                                                                             else 'sor_batch_traffic.json'),
                        alg_bytes_per_launch=sol['alg_bytes'] / per_launch, launch_ms=sol['ms'] / per_launch,
                        lane=dom, active_cells=lanes[dom]['active_cells'], iters=iters,
                        unit_bytes='20 B per active cell per colour sweep',
                        note='the solve\'s operands stay on chip (shared memory) or in L2, so the algorithmic '
                             'rate may exceed the HBM copy rate; traffic is the DRAM bytes ncu measured per launch '
                             '(warm: caches kept as in the step; cold: ncu flushed them before the launch)')
        cpu_rate, cpu_el, cpu_what = cpu_sample_rate(specs)
        launches = args.steps * sum(launches_per_substep(best[l][1], iters, g2p_form=best[l][3]) for l in range(nlanes))
        serving = serving_sample(args.serve_sample, local) if world == 1 and args.serve_sample > 0 else None
        line = dict(metric=METRIC, value=value, unit=METRIC, n_gpus=world, steps=args.steps, warmup=args.warmup,
                    ms_per_step=ms, higher_is_better=True, scaling='weak', vs_baseline=None, dtype='f32',
                    data='synthetic (seeded particles, analytic obstacles)', config=cfg,
                    l2='flushed (256 MiB write) between timed steps', parallelism=f'replicas{world}',
                    tuned=[dict(zip(('blocks_per_sm', 'sor_mode', 'piece_kb', 'g2p_form'), b)) for b in best],
                    tuning_ms={f'lane{l}': {'x'.join(str(v) for v in k): v for k, v in t.items()}
                               for l, t in timings.items()},
                    plain_sequential=dict(value=particles / world * 1000.0 / ms_plain, ms_per_step=ms_plain,
                                          note='the same scenes one by one, device time summed'),
                    batched_over_plain=ms_plain / ms if world == 1 else None,
                    roofline=roofline, kernels=dict(peak_gbs=peak, lanes=lanes),
                    cpu_baseline=dict(value=cpu_rate, unit=METRIC, cores=1, kind='port', sample=cpu_what),
                    e2e=e2e, gpu_launches=launches, clocks=clk, residual_f64=residual, serving=serving)
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


def serving_sample(duration, local, rate=10.0):
    """The metric's latency figures beside the batch: the serving loop (`--workload serve`) run for `duration`
    seconds of Poisson arrivals at `rate` requests/s, the load one B200 serves as it comes (at the serving
    configuration's 200/s the offered load is several times what it delivers, and the latencies measure the
    queue: `--workload serve --rate 200`). Latencies are wall-clock request times from submission to the
    finished result."""
    from importlib import import_module
    r = import_module('hahenn-_b200.serve').poisson_run(rate=rate, duration=duration, steps=120, budget_bytes=150e9,
                                                        device=local)
    keep = ('requests', 'completed', 'failed', 'p50_ms', 'p99_ms', 'particle_steps_per_s',
            'offered_particle_steps_per_s', 'mean_active', 'wall_s')
    return dict(workload='serving_poisson', rate_per_s=rate, duration_s=duration, steps_per_request=120,
                budget_gb=150, **{k: r[k] for k in keep})


# ------------------------------------------------------------------ the single-tank workload
def run_plain(args, rank, world, local):
    import torch
    import torch.distributed as dist
    init_ranks(world, local)
    P = pkg()
    w = P.workloads.obstacles_inflow()
    prm = w['params']
    dt = prm['dt']
    tank = make_tank(P, w, local)
    autotune = importlib.import_module('hahenn-_b200.autotune').autotune
    best, timings = autotune(tank, dt)
    tank.profile(True)
    stream = torch.cuda.ExternalStream(tank.stream())
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=f'cuda:{local}')
    for _ in range(max(args.warmup, 3)):
        tank.substep(dt)
    tank.sync()
    n0 = tank.stats()['count']
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    phases = []
    clocks = Clocks(local)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    for k in range(args.steps):
        with torch.cuda.stream(stream):
            flush.zero_()
        ev[k][0].record(stream)
        tank.substep(dt)
        ev[k][1].record(stream)
        phases.append(tank.phase_ms())
    torch.cuda.synchronize()
    clk = clocks.stop()
    if world > 1:
        dist.barrier()
    st = tank.stats()
    ms = float(np.mean([a.elapsed_time(b) for a, b in ev]))
    particles = 0.5 * (n0 + st['count'])
    ph = {k: float(np.mean([p[k] for p in phases])) for k in P.native.PHASES}
    sor_launch_ms = ph['pressure_solve'] / (2 * prm['iters'])
    if world > 1:
        ms, particles, sor_launch_ms = reduce_ranks(ms, particles, sor_launch_ms, f'cuda:{local}')
    value = particles * 1000.0 / ms
    tank.profile(False)
    residual = solve_residual(tank, [tank], dt)

    # end-to-end through the C ABI: host inflow particles (pinned) up, stats back, every step
    t2 = make_tank(P, w, local, host_inflow=True)
    t2.tune_piece(best[2])
    t2.tune(best[0], best[1])
    t2.tune_g2p(best[3])
    rng = np.random.default_rng(7)
    for _ in range(3):
        for e in w['emitters']:
            p, v = faucet_particles(e, dt, rng)
            t2.add_particles(p, v)
        t2.substep(dt)
        t2.stats()
    nA = t2.stats()['count']
    h2d = d2h = 0
    readback = int(P.native.lib().suiri_stats_readback_bytes())
    t0 = time.perf_counter()
    for _ in range(args.steps):
        for e in w['emitters']:
            p, v = faucet_particles(e, dt, rng)
            t2.add_particles(p, v)
            h2d += 24 * len(p)          # positions and velocities, copied packed (6 float32 per particle)
        t2.substep(dt)
        t2.poll_stats()
        d2h += readback
    t2.sync()
    el = time.perf_counter() - t0
    nB = t2.stats()['count']
    e2e_rate = 0.5 * (nA + nB) * args.steps / el
    if world > 1:
        e2e_rate = reduce_e2e(e2e_rate, world, f'cuda:{local}')
    e2e = dict(value=e2e_rate, unit=METRIC, h2d_bytes_per_step=h2d // args.steps, d2h_bytes_per_step=d2h // args.steps)
    t2.close()

    if rank == 0:
        peak, kind = peaks()
        active = st['active_cells']
        alg = 20.0 * active / 2                      # one colour sweep: read p 4 + fractions 12 + rhs 2 + write 2 per cell
        achieved = alg / (sor_launch_ms * 1e-3) / 1e9
        tr = profile_figure('sor_sweep_traffic.json')
        cpu_rate, cpu_el, cpu_what = cpu_sample_rate([w], steps=args.cpu_steps)
        line = dict(metric=METRIC, value=value, unit=METRIC, n_gpus=world, steps=args.steps, warmup=args.warmup,
                    ms_per_step=ms, higher_is_better=True, scaling='weak', vs_baseline=None, dtype='f32',
                    data='synthetic (seeded particles, analytic obstacles)', config=plain_config(w),
                    l2='flushed (256 MiB write) between timed steps', parallelism=f'replicas{world}',
                    roofline=dict(bound='hbm', kernel='k_sor (one colour sweep)', achieved=achieved, peak=peak,
                                  unit='GB/s', frac=achieved / peak, peak_kind=kind,
                                  traffic=None if tr is None else tr.get('dram_bytes_per_launch'),
                                  alg_bytes_per_launch=alg, launch_ms=sor_launch_ms, active_cells=active,
                                  unit_bytes='20 B per active cell per colour sweep'),
                    phases_ms=ph, tuned=dict(blocks_per_sm=best[0], sor_mode=best[1], piece_kb=best[2], g2p_form=best[3]),
                    cpu_baseline=dict(value=cpu_rate, unit=METRIC, cores=1, kind='port', sample=cpu_what),
                    e2e=e2e, gpu_launches=launches_per_substep(best[1], prm['iters'], g2p_form=best[3]) * args.steps,
                    clocks=clk,
                    residual_f64=residual)
        print(json.dumps(line), flush=True)
    tank.close()
    if world > 1:
        dist.destroy_process_group()


def run_full_scene(args, local):
    """Full scene: 256×128(up)×128 cells at h = 1/128 m, ≈8.39M particles, rain of 2000 drops/s over the
    top (each drop one particle with the free-flight mark, merging as ripple impulses and crowns), ripple
    layer 1024×512 (mirrored FFT 2048×1024, σ = 0.072 N/m, ρ = 1000 kg/m³, d = 0.1 m), 100 SOR iterations at
    ω = 1.8. A step here is one frame of 1/240 s: CFL sub-steps, whitewater, top height, ripple update."""
    import torch
    P = pkg()
    w = P.workloads.full_scene()
    prm = w['params']
    t = P.Tank(nx=w['nx'], ny=w['ny'], nz=w['nz'], h=w['h'], flip=prm['flip'], omega=prm['omega'], iters=prm['iters'],
               whitewater=True, ripple=w['ripple'], wmap=512, capacity=int(len(w['pos']) * 1.1) + 200000,
               ww_capacity=400000, ripple_sigma=prm['sigma'], ripple_rho=prm['rho'], ripple_depth=prm['depth'], device=local,
               drop_d=prm['drop_d'])
    t.add_particles(w['pos'])
    t.set_emitters(w['emitters'])
    stream = torch.cuda.ExternalStream(t.stream())
    for _ in range(args.warmup):
        t.step(prm['dt'])
    t.sync()
    n0 = t.stats()['count']
    subs, ms = 0, 0.0
    for _ in range(args.steps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        subs += t.step(prm['dt'])
        b.record(stream)
        b.synchronize()
        ms += a.elapsed_time(b)
    st = t.stats()
    particles = 0.5 * (n0 + st['count'])
    line = dict(metric=METRIC, value=particles * subs * 1000 / ms, unit=METRIC, n_gpus=1, steps=args.steps,
                warmup=args.warmup, ms_per_step=ms / args.steps, higher_is_better=True, scaling='weak', vs_baseline=None,
                dtype='f32', data='synthetic',
                config=dict(workload=w['name'], particles=int(particles), cells=w['nx'] * w['ny'] * w['nz'],
                            ripple=list(w['ripple']), substeps=subs, impacts=st['impacts'], whitewater=st['ww_count'],
                            sor_iters=prm['iters'], dt=prm['dt'], drop_d_median=prm['drop_d'][0],
                            drop_d_sigma_log=prm['drop_d'][1]))
    print(json.dumps(line), flush=True)
    t.close()


EXPORT_SUN = (0.35, 0.85, 0.25)


def _export_bytes(info, particles, nodes, W):
    """Algorithmic bytes of each phase of one frame export: what each kernel must read and write once.
    classify 16 B/particle position + 1 B class (+ the 27 cell counts, cached); distance field 4 B/node
    fill + 16 B/body particle; blur 3 passes × (4 B read + 4 B write)/node; surface nets 4 B/node phi
    reads in the count, cell and quad passes + 4 B/cell vertex index + 24 B/vertex + 16 B/quad + 1 B/particle
    class ×2; finish 24 B/body vertex + 24 B/vertex out; light maps 8 B/texel top + 16 B/ripple vertex
    (cached) + 8 B/texel fixed-point sums ×3 + 16 B/texel maps."""
    V, Q, nb, nl = len(info['verts']), len(info['quads']), int(info['body_verts']), int(info['lone'])
    return dict(classify=17 * particles, distance_field=4 * nodes + 16 * particles, blur=24 * nodes,
                surface_nets=12 * nodes + 4 * nodes + 24 * nb + 16 * Q + 2 * particles + 4 * nl,
                finish=24 * nb + 24 * V, light_maps=(8 + 24 + 16) * W * W)


def _cpu_export_rate(P, steps_frames=3):
    """The oracle's export (surface mesh, settling, vertex velocity, floor light) timed on the host for the
    same scene at a quarter of each axis, advanced on the GPU for the same frames: particles exported per
    second on one core (NumPy)."""
    from oracle import flip as of, meshing as om, ripple as orp
    w = P.workloads.full_scene(scale=4)
    prm = w['params']
    t = P.Tank(nx=w['nx'], ny=w['ny'], nz=w['nz'], h=w['h'], flip=prm['flip'], omega=prm['omega'], iters=prm['iters'],
               whitewater=True, ripple=w['ripple'], wmap=128, capacity=len(w['pos']) + 20000,
               ripple_sigma=prm['sigma'], ripple_rho=prm['rho'], ripple_depth=prm['depth'], drop_d=prm['drop_d'])
    t.add_particles(w['pos'])
    t.set_emitters(w['emitters'])
    for _ in range(steps_frames):
        t.step(prm['dt'])
    ora = of.Tank(w['nx'], w['ny'], w['nz'], w['h'], origin=w['origin'], ripple=w['ripple'], wmap=128)
    pos, vel, air, ids = t.particles()
    ora.pos, ora.vel, ora.air, ora.pid = pos.astype(float), vel.astype(float), air.astype(float), ids.astype(np.int64)
    ora.count = t.grid(P.native.FIELD_CELL_COUNT).astype(np.int64)
    top = t.ripple_field(P.native.FIELD_TOP64, (128, 128), np.float64)
    velg = t.grid(P.native.FIELD_VEL).astype(np.float64)
    field = t.ripple_field(P.native.FIELD_RIPPLE, (w['ripple'][1] + 1, w['ripple'][0] + 1, 3), np.float32).astype(float)
    n = len(pos)
    t.close()
    t0 = time.perf_counter()
    v, q, tr = om.surface(ora)
    om.settle_on_top(ora, v, top)
    om.vertex_velocity(ora, v, velg)
    orp.caustics(top, field, w['nx'] * w['h'], w['nz'] * w['h'], EXPORT_SUN)
    sec = time.perf_counter() - t0
    return n / sec, n, sec


def run_frame_export(args, local):
    """The per-frame export of the full scene (256×128(up)×128 cells at h = 1/128 m, ≈8.4M particles, rain,
    1024×512 ripple layer, 512² maps) after 8 frames of 1/240 s: a step is one frame's export, the surface
    mesh (lone drops as spheres, surface nets of the blurred distance field on the 2 mm lattice, settling,
    vertex velocity) and the floor light and surface maps. `value` is the device time of the export's kernels
    (the state resident in HBM); `e2e` is the export through the public calls into host arrays (mesh build,
    its read-back, the maps' build and read-back)."""
    import torch
    P = pkg()
    w = P.workloads.full_scene()
    prm = w['params']
    W = 512
    t = P.Tank(nx=w['nx'], ny=w['ny'], nz=w['nz'], h=w['h'], flip=prm['flip'], omega=prm['omega'], iters=prm['iters'],
               whitewater=True, ripple=w['ripple'], wmap=W, capacity=int(len(w['pos']) * 1.1) + 200000,
               ww_capacity=400000, ripple_sigma=prm['sigma'], ripple_rho=prm['rho'], ripple_depth=prm['depth'], device=local,
               drop_d=prm['drop_d'])
    t.add_particles(w['pos'])
    t.set_emitters(w['emitters'])
    for _ in range(8):
        t.step(prm['dt'])
    t.sync()
    stream = torch.cuda.ExternalStream(t.stream())
    particles = t.stats()['count']
    for _ in range(args.warmup):
        m = t.surface_mesh()
        t.frame_maps(EXPORT_SUN)
    phases = {k: 0.0 for k in P.native.MESH_PHASES}
    light_ms = 0.0
    clocks = Clocks(local)
    clocks.start()
    for _ in range(args.steps):
        m = t.surface_mesh()
        for k, v in m['phase_ms'].items():
            phases[k] += v / args.steps
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        t.frame_maps(EXPORT_SUN, read=False)
        b.record(stream)
        b.synchronize()
        light_ms += a.elapsed_time(b) / args.steps
    clk = clocks.stop()
    dev_ms = sum(phases.values()) + light_ms
    # end to end: the public calls into host arrays
    out = np.empty((W, W, 4), np.float32)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        m = t.surface_mesh()
        t.frame_maps(EXPORT_SUN, out)
    e2e_s = (time.perf_counter() - t0) / args.steps
    d2h = m['verts'].nbytes + m['vel'].nbytes + m['quads'].nbytes + m['tris'].nbytes + out.nbytes
    nodes = int(np.prod(m['lattice']))
    alg = _export_bytes(m, particles, nodes, W)
    times = dict(phases, light_maps=light_ms)
    top = max(times, key=times.get)
    peak, kind = peaks()
    prof = profile_figure('frame_export_traffic.json') or {}
    ach = alg[top] / (times[top] * 1e-3) / 1e9
    cpu_rate, cpu_n, cpu_s = _cpu_export_rate(P)
    line = dict(metric='exported particles/s', value=particles * 1000 / dev_ms, unit='particles/s', n_gpus=1,
                steps=args.steps, warmup=args.warmup, ms_per_step=dev_ms, higher_is_better=True, scaling='weak',
                vs_baseline=None, dtype='f32/f64', data='synthetic (seeded particles, rain)',
                config=dict(workload='frame_export_256x128x128', particles=int(particles), wmap=W,
                            lattice=list(m['lattice']), verts=int(len(m['verts'])), quads=int(len(m['quads'])),
                            lone=int(m['lone']), l2='state larger than L2 (particles 268 MB, lattice '
                            f'{nodes * 16 / 1e6:.0f} MB); no flush'),
                phases_ms=times,
                roofline=dict(bound='hbm', kernel=top, achieved=ach, peak=peak, unit='GB/s', frac=ach / peak,
                              peak_kind=kind, traffic=prof.get(top), alg_bytes_per_launch=alg[top]),
                alg_bytes=alg,
                cpu_baseline=dict(value=cpu_rate, unit='particles/s', cores=1, kind='port',
                                  sample=f'the oracle export (surface mesh, settling, vertex velocity, floor light) '
                                         f'of the scene at a quarter of each axis ({cpu_n} particles, 128² maps), '
                                         f'{cpu_s:.1f} s on one core'),
                e2e=dict(value=particles / e2e_s, unit='particles/s', h2d_bytes_per_step=0, d2h_bytes_per_step=int(d2h)),
                # per export: 4 of the cell count, 13 of the mesh (classify, fill, cell order, tile splat,
                # 3 blur passes, count, scan, cells, quads, lone, finish), 2 of the light maps
                gpu_launches=19 * args.steps, clocks=clk)
    print(json.dumps(line), flush=True)
    t.close()


def run_serve(args, local):
    """Serving workload: Poisson arrivals of seeded scene solves (axes up to 128, 10 % with a faucet), each
    asking for `--req-steps` sub-steps, admitted under a 150 GB HBM budget and co-scheduled in shared
    batched launches. Reports p50/p99 request latency and aggregate particle-steps/s."""
    from importlib import import_module
    serve = import_module('hahenn-_b200.serve')
    r = serve.poisson_run(rate=args.rate, duration=args.duration, steps=args.req_steps, budget_bytes=150e9, device=local)
    line = dict(metric=METRIC, value=r['particle_steps_per_s'], unit=METRIC, n_gpus=1, steps=args.req_steps, warmup=0,
                ms_per_step=None, higher_is_better=True, scaling='weak', vs_baseline=None, dtype='f32', data='synthetic',
                config=dict(workload='serving_poisson', rate_per_s=args.rate, duration_s=args.duration,
                            steps_per_request=args.req_steps, budget_gb=150),
                latency=dict(p50_ms=r['p50_ms'], p99_ms=r['p99_ms'], p50_all_ms=r['p50_all_ms'], p99_all_ms=r['p99_all_ms']),
                serving=r)
    print(json.dumps(line), flush=True)


def run_for_profiler(args, local):
    """A fixed launch sequence for ncu: the workload set up (the batch tuned to --sor-mode), stepped 3 + N
    sub-steps and synchronised; no timing, no JSON line."""
    P = pkg()
    if args.workload == 'batch':
        specs = batch_specs(args.tanks)
        tanks = make_batch_tanks(P, specs, local)
        b = P.Batch(tanks)
        b.tune(args.bps, args.sor_mode)
        b.tune_g2p(args.g2p_form)
        for _ in range(3 + args.ncu_steps):
            b.substep(DT)
        b.sync()
        print('sub-steps', 3 + args.ncu_steps, 'particles', sum(t.stats()['count'] for t in tanks))
        b.close()
        for t in tanks:
            t.close()
        return
    if args.workload == 'frame_export':
        # the full scene's shape at 1/--scale of each axis (default a quarter: 131k particles, 128² maps),
        # 3 frames, then N exports (mesh and maps)
        w = P.workloads.full_scene(scale=args.scale)
        prm = w['params']
        t = P.Tank(nx=w['nx'], ny=w['ny'], nz=w['nz'], h=w['h'], flip=prm['flip'], omega=prm['omega'],
                   iters=prm['iters'], whitewater=True, ripple=w['ripple'], wmap=512 // args.scale,
                   capacity=int(len(w['pos']) * 1.1) + 20000,
                   ripple_sigma=prm['sigma'], ripple_rho=prm['rho'], ripple_depth=prm['depth'], drop_d=prm['drop_d'],
                   device=local)
        t.add_particles(w['pos'])
        t.set_emitters(w['emitters'])
        for _ in range(3):
            t.step(prm['dt'])
        for _ in range(args.ncu_steps):
            t.surface_mesh()
            t.frame_maps(EXPORT_SUN, read=False)
        t.sync()
        print('exports', args.ncu_steps, 'particles', t.stats()['count'])
        t.close()
        return
    w = P.workloads.obstacles_inflow()
    t = make_tank(P, w, local)
    t.tune(args.bps, args.sor_mode if args.sor_mode != 4 else 0)
    t.tune_g2p(args.g2p_form)
    for _ in range(3 + args.ncu_steps):
        t.substep(w['params']['dt'])
    t.sync()
    print('sub-steps', 3 + args.ncu_steps, 'particles', t.stats()['count'])
    t.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--gpus', type=int, default=1)
    ap.add_argument('--steps', type=int, default=20)
    ap.add_argument('--warmup', type=int, default=5)
    ap.add_argument('--impl', default='suiri', choices=['suiri', 'reference'])
    ap.add_argument('--workload', default='batch',
                    choices=['batch', 'obstacles_inflow', 'serve', 'full_scene', 'frame_export'])
    ap.add_argument('--cpu-steps', type=int, default=2, help='sub-steps of the single-tank CPU baseline sample')
    ap.add_argument('--tanks', type=int, default=64)
    ap.add_argument('--rate', type=float, default=200.0)
    ap.add_argument('--duration', type=float, default=60.0)
    ap.add_argument('--req-steps', type=int, default=120)
    ap.add_argument('--serve-sample', type=float, default=20.0,
                    help='batch workload at one GPU: seconds of serving at 10 requests/s for its p50/p99 (0: none)')
    ap.add_argument('--ncu-steps', type=int, default=0,
                    help='profiler run: 3 warm-up and N more sub-steps of the workload, no timing, no JSON line')
    ap.add_argument('--bps', type=int, default=2, help='profiler run: particle blocks per SM')
    ap.add_argument('--g2p-form', type=int, default=0, help='profiler run: form of the grid-to-particle pass')
    ap.add_argument('--sor-mode', type=int, default=4, help='profiler run: form of the pressure solve')
    ap.add_argument('--scale', type=int, default=4, help='profiler run of the frame export: 1/scale of each axis')
    args = ap.parse_args()
    rank, world = int(os.environ.get('RANK', 0)), int(os.environ.get('WORLD_SIZE', 1))
    local = int(os.environ.get('LOCAL_RANK', 0))
    if args.impl == 'reference':
        return run_reference(args, rank)
    if args.ncu_steps:
        return run_for_profiler(args, local)
    if args.workload == 'batch':
        return run_batch(args, rank, world, local)
    if args.workload == 'serve':
        return run_serve(args, local)
    if args.workload == 'full_scene':
        return run_full_scene(args, local)
    if args.workload == 'frame_export':
        return run_frame_export(args, local)
    return run_plain(args, rank, world, local)


if __name__ == '__main__':
    main()

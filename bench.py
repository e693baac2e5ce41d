#!/usr/bin/env python
"""Benchmark: particle-steps/s of the FLIP sub-step on the obstacles-and-inflow workload.

Workload (one GPU): 128×64(up)×64 cells at h = 1/64 m, ≈1.70M particles (bottom 26 layers at 8 per cell),
a sphere, a turned box and a cylinder (face fractions from analytic SDFs), a 2 cm faucet at 1.5 m/s
emitting 10 particles per sub-step, one floor drain, 100 SOR iterations at ω = 1.8, FLIP 0.95,
dt = 1/240 s. A step is one sub-step of the liquid: binning, P2G, forces and divergence, the pressure
solve, projection, G2P with collisions, drains and drop/whitewater logic. Synthetic seeded data.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl suiri|reference]

Under torchrun each rank advances its own replica of the workload (tanks do not interact: no collective
in the data path); the time is the max over ranks and the value counts every rank's particles.
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


def pkg():
    return importlib.import_module('hahenn-_b200')


def peaks():
    try:
        with open(os.path.join(ROOT, 'MEASURED_PEAKS.json')) as f:
            p = json.load(f)
        return float(p['hbm_gbs']), 'measured'
    except Exception:
        return 6650.0, 'fallback'


def sor_traffic():
    """DRAM bytes per SOR sweep launch from the committed ncu summary (null if none)."""
    try:
        with open(os.path.join(ROOT, 'profiles', 'sor_sweep_traffic.json')) as f:
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


def make_tank(P, w, device, host_inflow=False):
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


def _port_tank(w):
    """The CPU oracle (NumPy restatement of the reference solver) set up on the workload."""
    from oracle import flip as of
    from oracle import sdf as sdfm
    prm = w['params']
    t = of.Tank(w['nx'], w['ny'], w['nz'], w['h'], origin=w['origin'], flip=prm['flip'], omega=prm['omega'],
                iters=prm['iters'], g=prm['g'], whitewater=True, rng_mode='hash', sdf_mode='lattice')
    objs = []
    for it in w['objects']:
        if it['kind'] == 'obstacle':
            objs.append(sdfm.make_obstacle(it['shape'], it['pos'], tuple(it['rot']), **it['dims']))
        else:
            objs.append(sdfm.make_drain(it['pos'], it['r'], tuple(it['rot'])))
    t.set_objects(objs)
    t.add_particles(w['pos'].astype(np.float64))
    return t


def _port_steps(t, w, steps, rng):
    """`steps` sub-steps with the faucet's particles added on the host; returns the particle-steps."""
    dt = w['params']['dt']
    n_ps = 0
    for _ in range(steps):
        for e in w['emitters']:
            p, v = faucet_particles(e, dt, rng)
            t.add_particles(p.astype(np.float64), v.astype(np.float64))
        n_ps += len(t.pos)
        t.frame += 1
        t.substep(dt)
    return n_ps


def cpu_port_rate(w, steps):
    """The CPU oracle on one core for `steps` sub-steps of the workload: particle-steps/s."""
    t = _port_tank(w)
    rng = np.random.default_rng(1)
    t0 = time.perf_counter()
    n_ps = _port_steps(t, w, steps, rng)
    el = time.perf_counter() - t0
    return n_ps / el, el


def _port_replica(steps, warm, barrier, out, k):
    """One CPU replica (a spawned process): set up, warm up, wait for the others, time `steps` sub-steps."""
    sys.path.insert(0, ROOT)
    P = pkg()
    w = P.workloads.obstacles_inflow()
    t = _port_tank(w)
    rng = np.random.default_rng(1 + k)
    if warm:
        _port_steps(t, w, warm, rng)
    barrier.wait(timeout=900)
    t0 = time.perf_counter()
    n_ps = _port_steps(t, w, steps, rng)
    out.put((n_ps, time.perf_counter() - t0))


def cpu_replicas_count():
    """One replica per usable core, at most 32, and at most one per 2 GB of available memory (a replica of
    the 1.7M-particle workload peaks near 1.1 GB)."""
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


def cpu_replicas_rate(steps, warm, procs):
    """`procs` independent replicas of the CPU oracle, one process (one core) each, timed together from a
    common start: all replicas' particle-steps ÷ the slowest replica's time."""
    import multiprocessing as mp
    ctx = mp.get_context('spawn')
    barrier, out = ctx.Barrier(procs), ctx.Queue()
    env = {k: os.environ.get(k) for k in ('OMP_NUM_THREADS', 'OPENBLAS_NUM_THREADS', 'MKL_NUM_THREADS')}
    for k in env:
        os.environ[k] = '1'
    ps = [ctx.Process(target=_port_replica, args=(steps, warm, barrier, out, k)) for k in range(procs)]
    for p in ps:
        p.start()
    res = [out.get(timeout=1800) for _ in ps]
    for p in ps:
        p.join(timeout=60)
    for k, v in env.items():
        if v is None:
            os.environ.pop(k, None)
        else:
            os.environ[k] = v
    return sum(r[0] for r in res) / max(r[1] for r in res), max(r[1] for r in res)


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


def run_reference(args, rank):
    """The reference's CPU path (its NumPy solver, restated and pinned bit-exact against it) on this host's
    cores: one independent replica of the workload per core, as many as the process may use. Rank 0 only;
    other ranks exit at once."""
    if rank != 0:
        return
    w = pkg().workloads.obstacles_inflow()
    steps, warm = max(1, min(args.steps, 3)), min(args.warmup, 3)   # ≈4 s a sub-step per core
    procs = cpu_replicas_count()
    rate, el = cpu_replicas_rate(steps, warm, procs)
    line = dict(impl='reference', metric=METRIC, value=rate, unit=METRIC, n_gpus=args.gpus, steps=steps, warmup=warm,
                ms_per_step=1000 * el / steps, higher_is_better=True, scaling='weak', vs_baseline=None, dtype='f64',
                data='synthetic',
                config=dict(workload=w['name'], particles=len(w['pos']), cells=w['nx'] * w['ny'] * w['nz'],
                            sor_iters=w['params']['iters'], omega=w['params']['omega'], dt=w['params']['dt']),
                cpu_baseline=dict(value=rate, unit=METRIC, cores=procs, kind='port',
                                  sample=f'{procs} replicas × {steps} sub-steps of the full workload, one process '
                                         f'and one core each (NumPy restatement of the reference solver, pinned '
                                         f'bit-exact against it; NumPy runs one core per process)'),
                e2e=dict(value=rate, unit=METRIC, h2d_bytes_per_step=0, d2h_bytes_per_step=0))
    print(json.dumps(line), flush=True)


def run_batch(args, local):
    """Batching workload: 64 tanks of uneven sizes (axes from {16,24,32,48,64}, h = 1/ny, fill U[0.2,0.6],
    0-3 obstacles, 80 SOR iterations at ω = 1.7) advanced together in one set of batched, graph-captured
    launches, against the same 64 scenes run one by one on the plain path. Both paths compute identical
    results (the batch is bit-for-bit the plain path), so the divergence residual is equal by construction."""
    import torch
    from importlib import import_module
    P = pkg()
    autotune = import_module('hahenn-_b200.autotune').autotune
    specs = P.workloads.batch_tanks(args.tanks)
    dt = 1 / 240

    def make():
        ts = []
        for w in specs:
            t = P.Tank(nx=w['nx'], ny=w['ny'], nz=w['nz'], h=w['h'], flip=0.95, omega=1.7, iters=80, whitewater=True,
                       ripple=None, capacity=int(len(w['pos']) * 1.2) + 1000, ww_capacity=20000, device=local)
            t.set_objects(w['objects'])
            t.add_particles(w['pos'])
            ts.append(t)
        return ts
    particles = sum(len(w['pos']) for w in specs)
    cells = sum(w['nx'] * w['ny'] * w['nz'] for w in specs)
    plain = make()
    for t in plain:
        t.substep(dt)
    torch.cuda.synchronize()
    ms_plain = 0.0
    for t in plain:
        ms_plain += t.time_substeps(dt, args.steps) / args.steps
    for t in plain:
        t.close()
    tanks = make()
    b = P.Batch(tanks)
    best, timings = autotune(b, dt)
    for _ in range(args.warmup):
        b.substep(dt)
    ms_batch = b.time_substeps(dt, args.steps) / args.steps
    rate_b, rate_p = particles * 1000 / ms_batch, particles * 1000 / ms_plain
    line = dict(metric=METRIC, value=rate_b, unit=METRIC, n_gpus=1, steps=args.steps, warmup=args.warmup, ms_per_step=ms_batch,
                higher_is_better=True, scaling='weak', vs_baseline=None, dtype='f32', data='synthetic',
                config=dict(workload=f'batch_{len(specs)}_tanks', tanks=len(specs), particles=particles, cells=cells,
                            sor_iters=80, omega=1.7, dt=dt, tuned=dict(blocks_per_sm=best[0], sor_mode=best[1]),
                            tuning_ms={f'{k[0]}x{k[1]}': v for k, v in timings.items()}),
                plain_sequential=dict(value=rate_p, ms_per_step=ms_plain), batched_over_plain=rate_b / rate_p)
    print(json.dumps(line), flush=True)
    b.close()
    for t in tanks:
        t.close()


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
               ww_capacity=400000, ripple_sigma=prm['sigma'], ripple_rho=prm['rho'], ripple_depth=prm['depth'], device=local)
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
                            sor_iters=prm['iters'], dt=prm['dt']))
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


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--gpus', type=int, default=1)
    ap.add_argument('--steps', type=int, default=200)
    ap.add_argument('--warmup', type=int, default=5)
    ap.add_argument('--impl', default='suiri', choices=['suiri', 'reference'])
    ap.add_argument('--workload', default='obstacles_inflow', choices=['obstacles_inflow', 'batch', 'serve', 'full_scene'])
    ap.add_argument('--cpu-steps', type=int, default=2, help='sub-steps of the CPU baseline sample')
    ap.add_argument('--tanks', type=int, default=64)
    ap.add_argument('--rate', type=float, default=200.0)
    ap.add_argument('--duration', type=float, default=60.0)
    ap.add_argument('--req-steps', type=int, default=120)
    ap.add_argument('--ncu-steps', type=int, default=0,
                    help='profiler run: 3 warm-up and N more sub-steps of the workload, no timing, no JSON line')
    args = ap.parse_args()
    rank, world = int(os.environ.get('RANK', 0)), int(os.environ.get('WORLD_SIZE', 1))
    local = int(os.environ.get('LOCAL_RANK', 0))
    if args.impl == 'reference':
        return run_reference(args, rank)
    if args.workload == 'batch':
        return run_batch(args, local)
    if args.workload == 'serve':
        return run_serve(args, local)
    if args.workload == 'full_scene':
        return run_full_scene(args, local)
    if args.ncu_steps:
        return run_for_profiler(args, local)
    import torch
    import torch.distributed as dist
    if world > 1:
        import datetime
        dist.init_process_group('nccl', timeout=datetime.timedelta(seconds=120))
    torch.cuda.set_device(local)
    P = pkg()
    w = P.workloads.obstacles_inflow()
    prm = w['params']
    dt = prm['dt']
    ncell = w['nx'] * w['ny'] * w['nz']
    tank = make_tank(P, w, local)
    tank.profile(True)
    stream = torch.cuda.ExternalStream(tank.stream())
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=f'cuda:{local}')
    for _ in range(max(args.warmup, 3)):
        tank.substep(dt)
    tank.sync()
    n0 = tank.stats()['count']
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    step_ms, sor_ms = [], []
    clocks = Clocks(local)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    for k in range(args.steps):
        with torch.cuda.stream(stream):
            flush.zero_()                          # L2 flush, outside the timed interval
        ev[k][0].record(stream)
        tank.substep(dt)
        ev[k][1].record(stream)
        sor_ms.append(tank.sor_phase_ms())
    torch.cuda.synchronize()
    clk = clocks.stop()
    if world > 1:
        dist.barrier()
    step_ms = [a.elapsed_time(b) for a, b in ev]
    n1 = tank.stats()['count']
    ms = float(np.mean(step_ms))
    particles = 0.5 * (n0 + n1)
    sor_launch_ms = float(np.mean(sor_ms)) / (2 * prm['iters'])
    if world > 1:
        ms, particles, sor_launch_ms = reduce_ranks(ms, particles, sor_launch_ms, f'cuda:{local}')
    value = particles * 1000.0 / ms

    # end-to-end through the C ABI: host inflow particles (pinned) up, stats back, every step
    e2e = None
    if rank == 0 or world > 1:
        t2 = make_tank(P, w, local, host_inflow=True)
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
                h2d += 32 * len(p)            # staged as two float4 per particle
            t2.substep(dt)
            t2.poll_stats()                   # the step's stats read, collected without waiting (pollStats)
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
        alg_bytes = 20.0 * ncell                 # one colour sweep: read p 4 + 3 fractions 12 + rhs 2 + write p 2 per cell
        achieved = alg_bytes / (sor_launch_ms * 1e-3) / 1e9
        tr = sor_traffic()
        cpu_rate, cpu_el = cpu_port_rate(w, args.cpu_steps)
        launches_per_step = 10 + 2 * prm['iters']  # the sub-step graph; dt is constant, so it is uploaded once
        line = dict(metric=METRIC, value=value, unit=METRIC, n_gpus=world, steps=args.steps, warmup=args.warmup,
                    ms_per_step=ms, higher_is_better=True, scaling='weak', vs_baseline=None, dtype='f32',
                    data='synthetic (seeded particles, analytic obstacles)',
                    config=dict(workload=w['name'], particles=int(particles / world), cells=ncell,
                                sor_iters=prm['iters'], omega=prm['omega'], flip=prm['flip'], dt=dt,
                                inflow_per_step=w['emitters'][0]['count'], l2='flushed (256 MiB write) between timed steps',
                                parallelism=f'replicas{world}'),
                    roofline=dict(bound='hbm', kernel='k_sor (one colour sweep)', achieved=achieved, peak=peak,
                                  unit='GB/s', frac=achieved / peak, peak_kind=kind,
                                  traffic=None if tr is None else tr.get('dram_bytes_per_launch'),
                                  alg_bytes_per_launch=alg_bytes, launch_ms=sor_launch_ms,
                                  sor_share=float(np.mean(sor_ms)) / ms),
                    cpu_baseline=dict(value=cpu_rate, unit=METRIC, cores=1, kind='port',
                                      sample=f'{args.cpu_steps} sub-steps of the same workload on the host (NumPy '
                                             f'restatement of the reference solver, {cpu_el:.1f} s, 1 core of {os.cpu_count()})'),
                    e2e=e2e, gpu_launches=launches_per_step * args.steps, clocks=clk)
        print(json.dumps(line), flush=True)
    tank.close()
    if world > 1:
        dist.destroy_process_group()


def run_for_profiler(args, local):
    """The obstacles-and-inflow tank stepped 3 + N times and synchronised: a fixed launch sequence for ncu
    (per sub-step: 10 kernels + 2 per SOR iteration)."""
    P = pkg()
    w = P.workloads.obstacles_inflow()
    t = make_tank(P, w, local)
    for _ in range(3 + args.ncu_steps):
        t.substep(w['params']['dt'])
    t.sync()
    print('sub-steps', 3 + args.ncu_steps, 'particles', t.stats()['count'])
    t.close()


if __name__ == '__main__':
    main()

"""Serving: scene-solve requests admitted by HBM budget and co-scheduled in shared batched launches.

``Server`` wraps the native request loop (``suiri_server_*``): a worker thread in libsuiri_cuda.so admits
requests FIFO as device memory frees up, advances all resident scenes with one batched sub-step at a time
(one CUDA graph per batch composition) and retires finished scenes at sub-step boundaries.

``poisson_run`` is the serving workload: requests arrive as a Poisson process, each a seeded scene drawn
like the batching workload (axes up to 128, 10 % with a faucet), each asking for a number of sub-steps;
it reports p50/p99 request latency and the aggregate particle-steps/s.
"""
import ctypes as C
import json
import math
import time

import numpy as np

from . import native as N

AXES_SERVE = (16, 24, 32, 48, 64, 96, 128)


def estimate_bytes(scene, params=None):
    """Device bytes a scene solve would take (the server admits by this figure)."""
    L = N.lib()
    p = N.Params()
    N.check(L.suiri_params_default(C.byref(p)))
    keep = []
    for k, v in (params or {}).items():
        if k == 'quality':
            v = v.encode()
            keep.append(v)
        setattr(p, k, v)
    b = C.c_double()
    js = (scene if isinstance(scene, str) else json.dumps(scene)).encode()
    N.check(L.suiri_estimate_bytes(js, C.byref(p), C.byref(b)))
    return b.value


class Server:
    def __init__(self, budget_bytes=150e9, dt=1 / 240, device=0):
        h = C.c_void_p()
        N.check(N.lib().suiri_server_create(int(device), float(budget_bytes), float(dt), C.byref(h)))
        self._h = h

    def close(self):
        if getattr(self, '_h', None):
            N.lib().suiri_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def submit(self, scene, params=None, emitters=(), steps=120, keep_result=False):
        """Queue a scene solve; returns its id. `params` are suiri_params fields (grid, physics)."""
        L = N.lib()
        p = N.Params()
        N.check(L.suiri_params_default(C.byref(p)))
        keep = []
        for k, v in (params or {}).items():
            if k == 'quality':
                v = v.encode()
                keep.append(v)
            setattr(p, k, v)
        em = (N.Emitter * max(1, len(emitters)))()
        for i, e in enumerate(emitters):
            em[i].shape = {'disc': 0, 'rain': 3}[e.get('shape', 'disc')]
            em[i].airborne = 1 if e.get('airborne') else 0
            em[i].pos[:] = [float(x) for x in e['pos']]
            em[i].dir[:] = [float(x) for x in e.get('dir', (0.0, -1.0, 0.0))]
            em[i].radius, em[i].speed, em[i].per_substep = float(e['radius']), float(e['speed']), float(e['count'])
        js = (scene if isinstance(scene, str) else json.dumps(scene)).encode()
        r = N.Request(size=C.sizeof(N.Request), params=C.pointer(p), scene_json=js, emitters=em,
                      n_emitters=len(emitters), steps=int(steps), keep_result=1 if keep_result else 0)
        i = C.c_int64()
        N.check(L.suiri_server_submit(self._h, C.byref(r), C.byref(i)))
        return i.value

    def poll(self, rid):
        st, lat, cnt = C.c_int32(), C.c_double(), C.c_int64()
        N.check(N.lib().suiri_server_poll(self._h, int(rid), C.byref(st), C.byref(lat), C.byref(cnt)))
        return dict(state=('queued', 'running', 'done', 'failed')[st.value], latency_ms=lat.value, count=cnt.value)

    def wait(self, rid, timeout_s=600.0):
        N.check(N.lib().suiri_server_wait(self._h, int(rid), float(timeout_s)))

    def result(self, rid):
        n = C.c_int64()
        N.check(N.lib().suiri_server_result(self._h, int(rid), None, None, 0, C.byref(n)))
        P = np.empty((n.value, 4), np.float32)
        V = np.empty((n.value, 4), np.float32)
        N.check(N.lib().suiri_server_result(self._h, int(rid), C.c_void_p(P.ctypes.data), C.c_void_p(V.ctypes.data),
                                            n.value, C.byref(n)))
        return P, V

    def stats(self):
        s = N.ServerStats()
        N.check(N.lib().suiri_server_get_stats(self._h, C.byref(s)))
        return {k: getattr(s, k) for k, _ in N.ServerStats._fields_}


def scene_request(seed, axes=AXES_SERVE, faucet_p=0.1, iters=80, omega=1.7):
    """A seeded scene like the batching workload (axes from `axes`, fill U[0.2, 0.6] as a bottom block,
    0–3 obstacles), as scene JSON + grid parameters + emitters. Water is emitted on the device."""
    rng = np.random.default_rng(seed)
    nx, ny, nz = (int(rng.choice(axes)) for _ in range(3))
    h = 1.0 / ny
    W, H, D = nx * h, ny * h, nz * h
    frac = rng.uniform(0.2, 0.6)
    layers = max(1, int(round(frac * ny)))
    items = []
    for _ in range(int(rng.integers(0, 4))):
        shape = ['sphere', 'box', 'cylinder'][int(rng.integers(0, 3))]
        s = rng.uniform(0.1, 0.3, size=3) * np.array([W, H, D])
        pos = [float(rng.uniform(-W / 2 + s[0] / 2, W / 2 - s[0] / 2)), float(rng.uniform(s[1] / 2, H - s[1] / 2)),
               float(rng.uniform(-D / 2 + s[2] / 2, D / 2 - s[2] / 2))]
        if shape == 'sphere':
            dims = dict(r=float(min(s) / 2))
        elif shape == 'box':
            dims = dict(w=float(s[0]), h=float(s[1]), d=float(s[2]))
        else:
            dims = dict(r=float(min(s[0], s[2]) / 2), h=float(s[1]))
        items.append(dict(kind='obstacle', shape=shape, pos=pos, rot=[0.0, float(rng.uniform(0, 90)), 0.0], dims=dims))
    items.append(dict(kind='block', pos=[0.0, layers * h / 2, 0.0], dims=dict(w=W, h=layers * h, d=D)))
    scene = dict(v=1, app='suiri-lab', scene=dict(tank=dict(w=W, h=H, d=D), items=items))
    n_fill = nx * nz * layers * 8
    params = dict(nx=nx, ny=ny, nz=nz, h=h, clamp_tank=0, flip=0.95, omega=omega, iters=iters, ripple_rx=-1,
                  ripple_rz=-1, capacity=int(n_fill * 1.2) + 20000, ww_capacity=20000)
    emitters = []
    if rng.random() < faucet_p:
        emitters.append(dict(shape='disc', pos=[0.0, 0.9 * H, 0.0], dir=[0.0, -1.0, 0.0], radius=0.01, speed=1.5,
                             count=max(1, int(round(8 * math.pi * 0.01 ** 2 / (h * h))))))
    return scene, params, emitters, dict(nx=nx, ny=ny, nz=nz, cells=nx * ny * nz, particles=n_fill)


def poisson_run(rate=200.0, duration=60.0, steps=120, budget_bytes=150e9, seed=0, axes=AXES_SERVE, faucet_p=0.1,
                drain_timeout=10.0, device=0):
    """Submit requests at Poisson arrival times for `duration` seconds, give the outstanding ones up to
    `drain_timeout` more seconds, and report over that window:
      * throughput: particle-steps/s done by the server (every resident scene's particles, counted at
        admission, per batched sub-step), beside the load offered (the requests' fill particles × steps ÷
        duration);
      * latency: p50/p99 of the completed requests, and p50/p99 over every request with the unfinished ones
        counted at the time they had waited when the window closed (a lower bound: under overload the queue
        grows and this is what a client sees)."""
    srv = Server(budget_bytes=budget_bytes, device=device)
    rng = np.random.default_rng(seed)
    t0 = time.perf_counter()
    t_next = t0
    ids = []
    offered = 0.0
    k = 0
    while True:
        t_next += rng.exponential(1.0 / rate)
        if t_next - t0 > duration:
            break
        while time.perf_counter() < t_next:
            time.sleep(min(0.002, max(0.0, t_next - time.perf_counter())))
        scene, params, em, info = scene_request(seed * 1000003 + k, axes, faucet_p)
        ids.append(srv.submit(scene, params, em, steps))
        offered += info['particles'] * steps
        k += 1
    submit_end = time.perf_counter()
    deadline = submit_end + drain_timeout
    while time.perf_counter() < deadline and srv.stats()['completed'] + srv.stats()['failed'] < len(ids):
        time.sleep(0.05)
    el = time.perf_counter() - t0
    st = srv.stats()
    lat, all_lat, failed, pending = [], [], 0, 0
    for i in ids:
        s = srv.poll(i)
        all_lat.append(s['latency_ms'])
        if s['state'] == 'done':
            lat.append(s['latency_ms'])
        elif s['state'] == 'failed':
            failed += 1
        else:
            pending += 1
    srv.close()
    pc = lambda a, q: float(np.percentile(np.array(a), q)) if len(a) else None
    return dict(requests=len(ids), completed=len(lat), failed=failed, pending_at_end=pending, rate=rate,
                duration_s=duration, wall_s=el, submit_s=submit_end - t0,
                p50_ms=pc(lat, 50), p99_ms=pc(lat, 99), p50_all_ms=pc(all_lat, 50), p99_all_ms=pc(all_lat, 99),
                particle_steps=st['particle_steps'], particle_steps_per_s=st['particle_steps'] / el,
                offered_particle_steps_per_s=offered / duration, mean_active=st['mean_active'],
                rebuilds=int(st['rebuilds']), substeps=int(st['substeps']))

"""Seeded synthetic scenes for the benchmark and parity workloads.

Solver coordinates are y up (metres, floor at y = 0, tank centred on x = z = 0), as in the reference
(``blender_addon/suiri_lab/solver.py:5-7``, ``src/js/50-sim.js:38``). The workload descriptions use
"z up", so a description's z is the solver's y.

The reference fills water blocks with a jittered half-cell lattice (``solver.py:317-343``,
``src/js/55-emit.js:83-106``). The workloads here instead put 8 particles per cell uniformly at random
inside each cell from ``numpy.random.default_rng(seed)``, stored as float32; the same arrays are given to
the CUDA path and to the CPU solver, so both start from identical particles.
"""
import math
import numpy as np


def grid_origin(nx, nz, h):
    """Minimum corner of the grid: the tank is centred on x = z = 0 (``solver.py:67``)."""
    return np.array([-nx * h / 2, 0.0, -nz * h / 2])


def fill_cells(cells, h, origin, ppc=8, seed=0):
    """`ppc` particles uniformly inside each cell of `cells` (M,3 int) → float32 (M·ppc, 3)."""
    rng = np.random.default_rng(seed)
    cells = np.asarray(cells, np.int64).reshape(-1, 3)
    u = rng.random((len(cells), ppc, 3))
    p = origin + (cells[:, None, :] + u) * h
    return p.reshape(-1, 3).astype(np.float32)


def block_cells(nx, ny, nz, pred_ijk):
    """Cells (i, j, k) for which pred_ijk(i, j, k) (broadcast arrays) holds, in x-fastest order."""
    k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing='ij')
    m = pred_ijk(i, j, k)
    return np.stack([i[m], j[m], k[m]], 1)


# ------------------------------------------------------------------ the five workloads
def dam_break(n=32, seed=0):
    """Plain dam break, 32³ MAC at h = 1/32 m, liquid in cells whose centre has x − x0 < 0.4 m and
    height < 0.5 m: 13·16·32 = 6,656 cells × 8 = 53,248 particles. g = −9.81, dt = 1/240, FLIP 0.95,
    60 SOR iterations at ω = 1.7, no obstacles."""
    h = 1.0 / n
    o = grid_origin(n, n, h)
    cells = block_cells(n, n, n, lambda i, j, k: ((i + 0.5) * h < 0.4) & ((j + 0.5) * h < 0.5))
    pos = fill_cells(cells, h, o, 8, seed)
    return dict(name='dam_break_32', nx=n, ny=n, nz=n, h=h, origin=o, pos=pos,
                params=dict(flip=0.95, omega=1.7, iters=60, g=9.81, dt=1 / 240), objects=[], emitters=[], steps=200)


def obstacles_inflow(seed=0, scale=1):
    """Obstacles and inflow: 128×64(up)×64 cells at h = 1/64 m (a 2 × 1 × 1 m tank), bottom 26 layers
    filled (128·64·26 = 212,992 cells × 8 ≈ 1.70M particles, those inside obstacles dropped). Obstacles:
    sphere r = 0.15 at the tank centre, a 0.3 × 0.1 × 0.2 box turned 30° about the vertical axis, a
    vertical cylinder r = 0.05, height 0.3. A 2 cm faucet at 1.5 m/s pointing down, 8 particles per cell
    of outlet area per step (10 per step). One floor drain of radius 2h. 100 SOR iterations at ω = 1.8.

    `scale` divides every axis (scale 2 → 64×32×32) for parity-test sized versions of the same scene."""
    nx, ny, nz = 128 // scale, 64 // scale, 64 // scale
    h = 1.0 / ny
    o = grid_origin(nx, nz, h)
    fill_layers = int(round(26 / scale))
    cells = block_cells(nx, ny, nz, lambda i, j, k: j < fill_layers)
    pos = fill_cells(cells, h, o, 8, seed)
    objects = [
        dict(kind='obstacle', shape='sphere', pos=[0.0, 0.5, 0.0], rot=[0, 0, 0], dims=dict(r=0.15)),
        dict(kind='obstacle', shape='box', pos=[0.55, 0.2, -0.2], rot=[0, 30, 0], dims=dict(w=0.3, h=0.1, d=0.2)),
        dict(kind='obstacle', shape='cylinder', pos=[-0.55, 0.15, 0.25], rot=[0, 0, 0], dims=dict(r=0.05, h=0.3)),
        dict(kind='drain', pos=[0.8, 0.0, 0.3], rot=[0, 0, 0], r=2 * h),
    ]
    outlet = math.pi * 0.01 ** 2
    n_emit = int(round(8 * outlet / (h * h)))
    emitters = [dict(shape='disc', pos=[-0.7, 0.9, -0.3], dir=[0.0, -1.0, 0.0], radius=0.01, speed=1.5,
                     count=n_emit)]
    return dict(name=f'obstacles_inflow_{nx}x{ny}x{nz}', nx=nx, ny=ny, nz=nz, h=h, origin=o, pos=pos,
                params=dict(flip=0.95, omega=1.8, iters=100, g=9.81, dt=1 / 240), objects=objects,
                emitters=emitters, steps=500)


def full_scene(seed=0, scale=1):
    """Full scene: 256×128(up)×128 cells at h = 1/128 m, bottom 32 layers filled (25 %, ≈8.39M particles),
    ripple layer 1024×512 (σ = 0.072 N/m, ρ = 1000 kg/m³, d = 0.1 m), rain of 2000 drops/s over the top,
    100 SOR iterations at ω = 1.8 (unspecified in the workload; recorded as chosen)."""
    nx, ny, nz = 256 // scale, 128 // scale, 128 // scale
    h = 1.0 / ny
    o = grid_origin(nx, nz, h)
    cells = block_cells(nx, ny, nz, lambda i, j, k: j < 32 // scale)
    pos = fill_cells(cells, h, o, 8, seed)
    W, H, D = nx * h, ny * h, nz * h
    # every sub-grid drop is one particle carrying the free-flight mark; its impulse and crown use the drop's
    # own diameter, lognormal with median 2 mm and σ_log 0.4 (drop_d; the reference's rule, the particle mass
    # 998·(h/2)³ of 31-wgsl-sim2.js:224, is drop_d=None)
    rain = dict(shape='rain', pos=[0.0, 0.98 * H, 0.0], radius=W / 2, radius_z=D / 2, speed=4.0,
                count=2000.0 / 240.0, airborne=True)
    return dict(name=f'full_scene_{nx}x{ny}x{nz}', nx=nx, ny=ny, nz=nz, h=h, origin=o, pos=pos,
                params=dict(flip=0.95, omega=1.8, iters=100, g=9.81, dt=1 / 240, sigma=0.072, rho=1000.0, depth=0.1,
                            drop_d=(0.002, 0.4)),
                objects=[], emitters=[rain], ripple=(1024 // scale, 512 // scale), steps=300)


AXES_BATCH = (16, 24, 32, 48, 64)


def random_tank(seed, axes=AXES_BATCH, faucet_p=0.0):
    """One tank of the batching workload: each axis from `axes`, h = 1 m / (vertical size), a bottom
    block filled to a fraction U[0.2, 0.6] at 8 particles per cell, 0–3 random obstacles (sphere, box or
    cylinder, sizes U[0.1, 0.3] of the tank), 80 SOR iterations at ω = 1.7. Seed = tank index."""
    rng = np.random.default_rng(seed)
    nx, ny, nz = (int(rng.choice(axes)) for _ in range(3))
    h = 1.0 / ny
    o = grid_origin(nx, nz, h)
    frac = rng.uniform(0.2, 0.6)
    layers = max(1, int(round(frac * ny)))
    W, H, D = nx * h, ny * h, nz * h
    objects = []
    for _ in range(int(rng.integers(0, 4))):
        shape = ['sphere', 'box', 'cylinder'][int(rng.integers(0, 3))]
        s = rng.uniform(0.1, 0.3, size=3) * np.array([W, H, D])
        pos = [rng.uniform(-W / 2 + s[0] / 2, W / 2 - s[0] / 2), rng.uniform(s[1] / 2, H - s[1] / 2),
               rng.uniform(-D / 2 + s[2] / 2, D / 2 - s[2] / 2)]
        if shape == 'sphere':
            dims = dict(r=float(min(s) / 2))
        elif shape == 'box':
            dims = dict(w=float(s[0]), h=float(s[1]), d=float(s[2]))
        else:
            dims = dict(r=float(min(s[0], s[2]) / 2), h=float(s[1]))
        objects.append(dict(kind='obstacle', shape=shape, pos=[float(v) for v in pos],
                            rot=[0.0, float(rng.uniform(0, 90)), 0.0], dims=dims))
    cells = block_cells(nx, ny, nz, lambda i, j, k: j < layers)
    pos = fill_cells(cells, h, o, 8, seed)
    emitters = []
    if faucet_p > 0 and rng.random() < faucet_p:
        emitters.append(dict(shape='disc', pos=[0.0, 0.9 * H, 0.0], dir=[0.0, -1.0, 0.0], radius=0.01, speed=1.5,
                             count=max(1, int(round(8 * math.pi * 0.01 ** 2 / (h * h))))))
    return dict(name=f'tank{seed}_{nx}x{ny}x{nz}', nx=nx, ny=ny, nz=nz, h=h, origin=o, pos=pos,
                params=dict(flip=0.95, omega=1.7, iters=80, g=9.81, dt=1 / 240), objects=objects,
                emitters=emitters, steps=200)


def batch_tanks(n=64, first_seed=0):
    """The batching workload: `n` tanks of uneven sizes (seed = tank index)."""
    return [random_tank(first_seed + t) for t in range(n)]

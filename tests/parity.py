"""Helpers shared by the parity tests: the same seeded inputs to the CUDA path and to the oracle, and the
comparisons with their tolerances.

Tolerances (stated once, used everywhere):
  * binning / cell counts / classification / valid-face masks: bit-exact;
  * face fractions: float32 of the same float64 value — bit-exact;
  * P2G face velocities, pressure, projected velocities: |a - b| <= 1e-5·|b| + 1e-5·max|b| (the GPU sums
    in 64-bit fixed point and stores float32; the CPU solver sums in float64);
  * particles after a sub-step (matched by id): positions within 1e-6 m + 1e-6 relative,
    velocities within 1e-5 relative + 1e-5·max|v|;
  * ripple layer (float32 FFT against float64 numpy.fft): 1e-4 relative to the field's max.
"""
import numpy as np

from oracle import flip as of
from oracle import sdf as sdfm

RTOL = 1e-5


def f32(a):
    return np.asarray(a, np.float32).astype(np.float64)


def oracle_from(nx, ny, nz, h, origin, *, flip, omega, iters, g=9.81, whitewater=False, rng_mode='hash', sdf_mode='analytic',
                ripple=(16, 16), wmap=32, seed=1, ww_cap=140000, advect='euler'):
    return of.Tank(nx, ny, nz, h, origin=origin, flip=flip, omega=omega, iters=iters, g=g, whitewater=whitewater,
                   rng_mode=rng_mode, sdf_mode=sdf_mode, ripple=ripple, wmap=wmap, seed=seed, ww_cap=ww_cap,
                   advect=advect)


def gpu_from(pkg, nx, ny, nz, h, *, flip, omega, iters, g=9.81, whitewater=False, ripple=None, wmap=32, capacity=None,
             sdf_mode='analytic', ww_capacity=140000, seed=1, advect='euler'):
    n = capacity or max(64, nx * ny * nz * 12)
    return pkg.Tank(nx=nx, ny=ny, nz=nz, h=h, flip=flip, omega=omega, iters=iters, gravity=g, whitewater=whitewater,
                    capacity=n, ripple=ripple, wmap=wmap, sdf_mode=sdf_mode, ww_capacity=ww_capacity, seed=seed,
                    advect=advect)


def assert_close_field(a, b, rtol=RTOL, what='', atol=0.0):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    assert a.shape == b.shape, (what, a.shape, b.shape)
    scale = max(float(np.abs(b).max()) if b.size else 0.0, 1e-30)
    err = np.abs(a - b)
    lim = rtol * np.abs(b) + rtol * scale + atol
    bad = err > lim
    if bad.any():
        w = np.unravel_index(int(np.argmax(np.where(bad, err - lim, -np.inf))), b.shape)
        raise AssertionError(f'{what}: {int(bad.sum())} of {b.size} beyond tolerance, max err {err.max():.3e} '
                             f'(scale {scale:.3e}); worst at {tuple(int(i) for i in w)}: {a[w]:.9e} against {b[w]:.9e}')


def by_id(pos, vel, air, ids):
    o = np.argsort(ids, kind='stable')
    return pos[o], vel[o], air[o], ids[o]


def assert_particles(gpu, ora, what='', vel_rtol=RTOL, floor_y=None):
    """Particles matched by id: ids, airborne marks, positions, velocities. With floor_y given, particles lying
    within 1e-9 m of that height (the floor clamp, x_y = floor + 0.32h with v_y = max(v_y, 0)) have their
    vertical velocity left out: there the clamp is a step in v_y, and whether the float32 sums of the GPU and
    the float64 sums of the oracle land on one side of it or the other is a tie either can break."""
    gp, gv, ga, gi = gpu.particles()
    gp, gv, ga, gi = by_id(gp, gv, ga, gi.astype(np.int64))
    op, ov, oa, oi = by_id(ora.pos, ora.vel, ora.air, ora.pid)
    assert len(gi) == len(oi), f'{what}: {len(gi)} particles on the GPU, {len(oi)} in the oracle'
    np.testing.assert_array_equal(gi, oi)
    np.testing.assert_array_equal(ga, oa, err_msg=f'{what}: airborne marks')
    perr = np.abs(gp - op) - (1e-6 + 1e-6 * np.abs(op))
    if op.size and perr.max() > 0:
        k = int(np.argmax(perr.max(1)))
        raise AssertionError(f'{what}: position of particle id {int(oi[k])} (airborne {oa[k]:.0f}): {gp[k]} on the GPU, '
                             f'{op[k]} in the oracle, velocity {gv[k]} / {ov[k]}; {int((perr.max(1) > 0).sum())} particles '
                             f'beyond 1e-6 m + 1e-6 relative')
    verr = np.abs(gv - ov) - (vel_rtol * np.abs(ov) + vel_rtol * max(float(np.abs(ov).max()) if ov.size else 0.0, 1e-30))
    if floor_y is not None:
        verr[np.abs(op[:, 1] - floor_y) < 1e-9, 1] = -1.0
    if ov.size and verr.max() > 0:
        k = int(np.argmax(verr.max(1)))
        raise AssertionError(f'{what}: velocity of particle id {int(oi[k])} at {op[k]} (airborne {oa[k]:.0f}): '
                             f'{gv[k]} on the GPU, {ov[k]} in the oracle; {int((verr.max(1) > 0).sum())} particles beyond '
                             f'{vel_rtol:g} relative + {vel_rtol:g} of the largest')


def sync_oracle_particles(gpu, ora):
    """Continue the oracle from the GPU's float32 particle state (step-wise parity over many steps)."""
    gp, gv, ga, gi = gpu.particles()
    o = np.argsort(gi)
    ora.pos, ora.vel, ora.air, ora.pid = gp[o].astype(np.float64), gv[o].astype(np.float64), ga[o].astype(np.float64), gi[o].astype(np.int64)


def gpu_max_divergence(pkg, gpu):
    """Post-projection max |div| over the GPU's liquid cells, from its own face velocities and fractions, as
    the oracle's max_divergence forms it (static solids: the solid velocity is zero)."""
    N = pkg.native
    nx, ny, nz, h = gpu.nx, gpu.ny, gpu.nz, gpu.h
    vel = gpu.grid(N.FIELD_VEL).astype(np.float64)
    frac = gpu.grid(N.FIELD_FRAC).astype(np.float64)
    cnt = gpu.grid(N.FIELD_CELL_COUNT)
    F = [frac[a] * vel[a] for a in range(3)]
    div = (F[0][1:nx + 1, :ny, :nz] - F[0][:nx, :ny, :nz] + F[1][:nx, 1:ny + 1, :nz] - F[1][:nx, :ny, :nz]
           + F[2][:nx, :ny, 1:nz + 1] - F[2][:nx, :ny, :nz]) / h
    return float(np.abs(div[cnt > 0]).max()) if (cnt > 0).any() else 0.0


def obstacle_items():
    """Scene items (JSON form) with the oracle objects made from them."""
    items = [dict(kind='obstacle', shape='sphere', pos=[0.15, 0.18, 0.0], rot=[0, 0, 0], dims=dict(r=0.09)),
             dict(kind='obstacle', shape='box', pos=[-0.25, 0.1, 0.12], rot=[0, 30, 0], dims=dict(w=0.16, h=0.1, d=0.12)),
             dict(kind='obstacle', shape='cone', pos=[-0.05, 0.1, -0.2], rot=[10, 0, 20], dims=dict(r=0.08, h=0.14)),
             dict(kind='drain', pos=[0.38, 0.0, -0.28], rot=[0, 0, 0], r=0.06)]
    return items, objs_from_items(items)


def objs_from_items(items):
    out = []
    for it in items:
        if it['kind'] == 'obstacle':
            out.append(sdfm.make_obstacle(it['shape'], it['pos'], tuple(it['rot']), **it['dims']))
        elif it['kind'] == 'drain':
            out.append(sdfm.make_drain(it['pos'], it['r'], tuple(it['rot'])))
    return out


def assert_mesh_matches_oracle(pkg, gpu, ora, smooth=0.8):
    """The GPU's surface mesh against the oracle's on the GPU's own state: the particles in the order the GPU
    holds them (the order of its lone-particle spheres), its cell counts, top-view height map, projected face
    velocity, and the blur weights it used (the reference forms them with NumPy's exp, which may differ from
    the C library's in the last bit). Body vertices, quads, triangles and body velocities are equal; the
    icosphere table of the drops is normalised by a different dot product, so their vertices and velocities
    agree to float32 rounding."""
    from oracle import meshing as om
    m = gpu.surface_mesh(smooth)
    P, V, A, ids = gpu.particles()
    ora.pos, ora.vel, ora.air = P.astype(np.float64), V.astype(np.float64), A.astype(np.float64)
    ora.pid = ids.astype(np.int64)
    ora.count = gpu.grid(pkg.native.FIELD_CELL_COUNT).astype(np.int64)
    W = gpu.stats()['wmap']
    top = gpu.ripple_field(pkg.native.FIELD_TOP64, (W, W), np.float64)
    velg = gpu.grid(pkg.native.FIELD_VEL).astype(np.float64)
    verts, quads, tris = om.surface(ora, smooth, weights=m['weights'])
    om.settle_on_top(ora, verts, top)
    vel = om.vertex_velocity(ora, verts, velg)
    nb = m['body_verts']
    assert m['verts'].shape == verts.shape, (m['verts'].shape, verts.shape)
    assert m['lone'] * 42 == len(verts) - nb
    np.testing.assert_array_equal(m['quads'], quads)
    np.testing.assert_array_equal(m['tris'], tris)
    np.testing.assert_array_equal(m['verts'][:nb], verts[:nb].astype(np.float32))
    np.testing.assert_array_equal(m['vel'][:nb], vel[:nb].astype(np.float32))
    np.testing.assert_allclose(m['verts'][nb:], verts[nb:], rtol=2e-7, atol=1e-9)
    np.testing.assert_allclose(m['vel'][nb:], vel[nb:], rtol=1e-6, atol=1e-9)
    return m


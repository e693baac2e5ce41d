"""System tests on the GPU: scene JSON, reset and snapshots, serving (alone vs in the mix), the long dam-break
run against the oracle, and size-independent properties at the full obstacles-and-inflow size."""
import json

import numpy as np
import pytest

from oracle import flip as of
from parity import (assert_close_field, assert_particles, f32, gpu_max_divergence, objs_from_items, oracle_from,
                    sync_oracle_particles)

pytestmark = pytest.mark.gpu


def dam_scene():
    return dict(v=1, app='suiri-lab', scene=dict(
        tank=dict(w=0.6, h=0.32, d=0.4),
        items=[dict(id=1, kind='block', name='water', pos=[-0.2, 0.11, 0.0], dims=dict(w=0.18, h=0.22, d=0.38)),
               dict(id=2, kind='obstacle', shape='cylinder', pos=[0.08, 0.06, 0.04], rot=[0, 0, 0], dims=dict(r=0.035, h=0.12)),
               dict(id=3, kind='obstacle', shape='box', pos=[0.12, 0.025, -0.1], rot=[0, 30, 0], dims=dict(w=0.08, h=0.05, d=0.08))]),
        cam={})


def test_scene_json_sizing_reset_and_errors(pkg):
    t = pkg.Tank(dam_scene(), quality='low', whitewater=False, ripple=None)
    # FluidSim sizing (src/js/50-sim.js:33-37): n = max(8, round(size / 0.012)), h = min(size / n)
    assert (t.nx, t.ny, t.nz) == (50, 27, 33)
    assert abs(t.h - min(0.6 / 50, 0.32 / 27, 0.4 / 33)) < 1e-15
    n0 = t.stats()['count']
    sp = t.h / 2
    # the block's half-cell lattice (src/js/55-emit.js:83-106)
    n_lat = int(np.floor(0.18 / sp)) * int(np.floor(0.22 / sp)) * int(np.floor(0.38 / sp))
    assert 0 < n0 <= n_lat
    for _ in range(3):
        t.step(1 / 60)
    st = t.stats()
    assert st['count'] > 0.98 * n0 and st['time'] > 0.04
    t.reset()
    t.substep(1 / 240)
    assert abs(t.stats()['count'] - n0) <= n0 * 0.001
    with pytest.raises(pkg.native.SuiriError) as e:
        pkg.Tank('{"scene": {"tank": {"w": -1}}}')
    assert e.value.code in (-5, -1)
    t.close()


def test_set_objects_moving_obstacle_velocity(pkg):
    t = pkg.Tank(nx=16, ny=16, nz=16, h=1 / 32, whitewater=False, ripple=None, capacity=10000, iters=4)
    box = dict(id=7, kind='obstacle', shape='box', pos=[0.0, 0.2, 0.0], rot=[0, 0, 0], dims=dict(w=0.1, h=0.1, d=0.1))
    assert not t.set_objects([box], 0.0)
    box2 = dict(box, pos=[0.01, 0.2, 0.0])
    assert t.set_objects([box2], 0.01)            # moved 1 cm in 10 ms: 1 m/s
    t.close()


def test_serving_result_alone_equals_result_in_mix(pkg):
    """Each request gives the same particles alone and co-scheduled with others (the step is deterministic:
    integer P2G sums, id-keyed randomness), here bit for bit; the 48³ scene runs in another size lane (its
    own stream and batch) beside the small ones."""
    from importlib import import_module
    serve = import_module('hahenn-_b200.serve')
    reqs = [serve.scene_request(s, axes=(16, 24, 32), faucet_p=0.5 if s == 2 else 0.0) for s in (1, 2, 3)]
    reqs.append(serve.scene_request(4, axes=(48,)))
    srv = serve.Server(budget_bytes=8e9)
    alone = []
    for sc, prm, em, _ in reqs:
        i = srv.submit(sc, prm, em, steps=12, keep_result=True)
        srv.wait(i)
        alone.append(srv.result(i))
    ids = [srv.submit(sc, prm, em, steps=12, keep_result=True) for sc, prm, em, _ in reqs]
    for i in ids:
        srv.wait(i)
    st = srv.stats()
    assert st['mean_active'] > 1.0 and st['completed'] == 8
    for (Pa, Va), i in zip(alone, ids):
        Pm, Vm = srv.result(i)
        ka, km = Va[:, 3].view(np.uint32), Vm[:, 3].view(np.uint32)
        oa, om = np.argsort(ka), np.argsort(km)
        np.testing.assert_array_equal(ka[oa], km[om])
        np.testing.assert_array_equal(Pa[oa], Pm[om])
        np.testing.assert_array_equal(Va[oa], Vm[om])
    srv.close()


def test_serving_budget_admission(pkg):
    """A budget that fits one scene at a time still completes every request (FIFO, one resident)."""
    from importlib import import_module
    serve = import_module('hahenn-_b200.serve')
    sc, prm, em, info = serve.scene_request(5, axes=(16,))
    one = 1.5 * serve.estimate_bytes(sc, prm)
    srv = serve.Server(budget_bytes=one)
    ids = [srv.submit(sc, prm, em, steps=4) for _ in range(3)]
    for i in ids:
        srv.wait(i)
    st = srv.stats()
    assert st['completed'] == 3 and st['mean_active'] == 1.0
    big = dict(prm, nx=128, ny=128, nz=128, h=1 / 128, capacity=20_000_000)
    j = srv.submit(sc, big, em, steps=1)
    assert srv.poll(j)['state'] == 'failed'
    # a malformed scene is refused at submission with a parse error; the server keeps serving
    with pytest.raises(pkg.native.SuiriError) as e:
        srv.submit('{"scene": {"tank": ', prm, em, steps=1)
    assert e.value.code == -5
    k = srv.submit(sc, prm, em, steps=2)
    srv.wait(k)
    assert srv.poll(k)['state'] == 'done'
    srv.close()


def test_bounded_wait_gives_up_reports_and_serving_fails_the_request(pkg):
    """The cooperative solve (sor_mode 1) with a poll limit of 0: a block that finds a grid barrier not yet
    passed gives up at once (32³ and 32–48-cell tanks, so the solve has several blocks to wait for). The
    sub-step returns, the tank's stats carry error bit 1, and with the per-sweep form the next sub-steps run
    cleanly. In the server a request whose solve gave up is reported failed with the reason, and the next
    request completes."""
    from importlib import import_module
    serve = import_module('hahenn-_b200.serve')
    w = pkg.workloads.dam_break(32)
    t = pkg.Tank(nx=32, ny=32, nz=32, h=w['h'], iters=20, whitewater=False, ripple=None, capacity=len(w['pos']) * 2,
                 sor_mode=1, watchdog_polls=0)
    t.add_particles(w['pos'])
    t.substep(1 / 240)
    assert t.stats()['errors'] & 1
    t.tune(4, 0)
    for _ in range(2):
        t.substep(1 / 240)
    st = t.stats()
    assert st['count'] == len(w['pos']) and np.isfinite(t.grid(pkg.native.FIELD_PRES)).all()
    t.close()
    sc, prm, em, _ = serve.scene_request(6, axes=(32, 48))
    srv = serve.Server(budget_bytes=4e9)
    bad = srv.submit(sc, dict(prm, sor_mode=1, watchdog_polls=0), em, steps=3)
    with pytest.raises(pkg.native.SuiriError, match='grid-barrier wait'):
        srv.wait(bad)
    assert srv.poll(bad)['state'] == 'failed'
    good = srv.submit(sc, prm, em, steps=3)
    srv.wait(good)
    assert srv.poll(good)['state'] == 'done'
    st = srv.stats()
    assert st['failed'] == 1 and st['completed'] == 1
    srv.close()


def test_dam_break_long_run(pkg):
    """The 32³ dam break: 200 sub-steps. Step-wise parity with the oracle for the first 10 sub-steps (oracle
    continued from the GPU state after each), then the free-running run compared on volume, kinetic energy
    and the post-projection divergence."""
    w = pkg.workloads.dam_break()
    prm = w['params']
    gpu = pkg.Tank(nx=32, ny=32, nz=32, h=w['h'], flip=prm['flip'], omega=prm['omega'], iters=prm['iters'],
                   whitewater=False, ripple=None, capacity=len(w['pos']) * 2)
    ora = oracle_from(32, 32, 32, w['h'], w['origin'], flip=prm['flip'], omega=prm['omega'], iters=prm['iters'])
    gpu.add_particles(w['pos'])
    ora.add_particles(f32(w['pos']))
    for s in range(1, 11):
        gpu.substep(prm['dt'])
        ora.frame = s
        ora.substep(prm['dt'])
        assert_particles(gpu, ora, f'dam break sub-step {s}')
        # same state: the post-projection divergence equals the oracle's (velocities agree to 1e-5 relative)
        dg, do = gpu_max_divergence(pkg, gpu), ora.max_divergence()
        assert abs(dg - do) <= 1e-3 * do, (s, dg, do)
        sync_oracle_particles(gpu, ora)
    free = oracle_from(32, 32, 32, w['h'], w['origin'], flip=prm['flip'], omega=prm['omega'], iters=prm['iters'])
    free.pos, free.vel, free.air, free.pid = ora.pos.copy(), ora.vel.copy(), ora.air.copy(), ora.pid.copy()
    free.pres = ora.pres.copy()
    ke_g, ke_o = [], []
    for s in range(11, 201):
        gpu.substep(prm['dt'])
        free.frame = s
        free.substep(prm['dt'])
        if s % 38 == 0 or s == 200:
            _, v, _, _ = gpu.particles()
            ke_g.append(0.5 * 998 * (w['h'] / 2) ** 3 * float(np.sum(v.astype(np.float64) ** 2)))
            ke_o.append(free.kinetic_energy())
    st = gpu.stats()
    assert st['count'] == len(w['pos']) == len(free.pos)           # closed tank: volume conserved exactly
    ke_g, ke_o = np.array(ke_g), np.array(ke_o)
    assert np.all(np.abs(ke_g - ke_o) <= 0.1 * ke_o + 1e-6), (ke_g, ke_o)
    # after 190 free-running sub-steps the two flows have drifted apart (chaotic), so their post-projection
    # divergences are compared as figures of the same solve: within a factor of 2 of each other
    dg, do = gpu_max_divergence(pkg, gpu), free.max_divergence()
    assert 0.5 * do <= dg <= 2.0 * do, (dg, do)
    gpu.close()


def test_full_size_obstacles_inflow_properties(pkg):
    """At the full 128×64×64 / 1.7M-particle size: face fractions equal the oracle's (float32 of the same
    float64), cell counts equal a float64 binning of the GPU's own particles, and volume is conserved up to
    the inflow and the drain."""
    w = pkg.workloads.obstacles_inflow()
    prm = w['params']
    t = pkg.Tank(nx=w['nx'], ny=w['ny'], nz=w['nz'], h=w['h'], flip=prm['flip'], omega=prm['omega'], iters=prm['iters'],
                 whitewater=True, ripple=None, capacity=int(len(w['pos']) * 1.25))
    t.set_objects(w['objects'])
    t.add_particles(w['pos'])
    t.set_emitters([dict(shape='disc', pos=e['pos'], dir=e['dir'], radius=e['radius'], speed=e['speed'], count=e['count'])
                    for e in w['emitters']])
    n_first = t.stats()['count']
    for _ in range(4):
        t.substep(prm['dt'])
    N = pkg.native
    ora = of.Tank(w['nx'], w['ny'], w['nz'], w['h'], origin=w['origin'], sdf_mode='analytic')
    ora.set_objects(objs_from_items(w['objects']))
    np.testing.assert_array_equal(t.grid(N.FIELD_FRAC), ora.frac.astype(np.float32))
    # the counts of the last binning are of the particles as they were before the last G2P: re-bin now
    pos, vel, air, ids = t.particles()
    t.substep(prm['dt'])
    cnt = t.grid(N.FIELD_CELL_COUNT)
    g = (pos.astype(np.float64) - w['origin']) / w['h']
    ing = np.all((g >= 0) & (g < [w['nx'], w['ny'], w['nz']]), axis=1)
    c = g[ing].astype(np.int64)
    ref = np.zeros((w['nx'], w['ny'], w['nz']), np.int64)
    np.add.at(ref, (c[:, 0], c[:, 1], c[:, 2]), 1)
    # particles emitted for the last sub-step are binned too; the faucet is above the liquid, count them out
    diff = cnt - ref
    assert diff.min() >= 0 and diff.sum() <= 10
    st = t.stats()
    assert st['count'] <= n_first + 5 * 10 and st['count'] >= n_first - 5000
    assert np.isfinite(t.grid(N.FIELD_PRES)).all() and np.isfinite(vel).all()
    t.close()


def test_empty_tank_steps_cleanly(pkg):
    """A tank with no liquid steps without error: no particles, zero pressure, nothing spawned."""
    t = pkg.Tank(nx=24, ny=16, nz=20, h=1 / 32, whitewater=True, ripple=None, capacity=1000, iters=10)
    for _ in range(4):
        t.substep(1 / 240)
    st = t.stats()
    assert st['count'] == 0 and st['ww_count'] == 0 and st['errors'] == 0 and st['full'] == 0
    assert not np.any(t.grid(pkg.native.FIELD_PRES))
    t.step(1 / 60)
    assert t.stats()['count'] == 0
    t.close()


def test_read_back_skips_the_drained_and_keeps_pending_adds(pkg):
    """The read-back (compacted on the device): particles a drain took in the last sub-step are left out, the
    rest keep their order, particles added since come after them with their ids, marks and velocities, a
    read with no arrays returns the same count, and a read into page-locked arrays gives the same particles."""
    import ctypes as C
    w = pkg.workloads.dam_break()
    t = pkg.Tank(nx=w['nx'], ny=w['ny'], nz=w['nz'], h=w['h'], whitewater=False, ripple=None,
                 capacity=len(w['pos']) + 4096, iters=20)
    t.set_objects([dict(kind='drain', pos=[-0.3, 0.0, 0.0], rot=[0, 0, 0], r=0.12)])
    t.add_particles(w['pos'])
    n0 = len(w['pos'])
    for _ in range(3):
        t.substep(1 / 240)
    p1, v1 = t.particles4()
    assert 0 < len(p1) < n0                                    # the drain took some
    assert len(np.unique(v1[:, 3].view(np.uint32))) == len(p1)
    rng = np.random.default_rng(5)
    add = (np.array([0.1, 0.6, 0.1]) + rng.uniform(-0.05, 0.05, (1000, 3))).astype(np.float32)
    vel = rng.uniform(-1, 1, (1000, 3)).astype(np.float32)
    air = (rng.random(1000) < 0.5).astype(np.float32)
    first = t.add_particles(add, vel, air)
    p2, v2 = t.particles4()
    assert len(p2) == len(p1) + 1000
    np.testing.assert_array_equal(p2[:len(p1)], p1)
    np.testing.assert_array_equal(v2[:len(p1)], v1)
    np.testing.assert_array_equal(p2[len(p1):, :3], add)
    np.testing.assert_array_equal(p2[len(p1):, 3], air)
    np.testing.assert_array_equal(v2[len(p1):, :3], vel)
    np.testing.assert_array_equal(v2[len(p1):, 3].view(np.uint32), first + np.arange(1000, dtype=np.uint32))
    n = C.c_int64()
    pkg.native.check(pkg.native.lib().suiri_read_particles(t.handle, None, None, 0, C.byref(n)))
    assert n.value == len(p2)
    # into page-locked arrays (written by the copy engine directly): the same particles
    import torch
    pp = torch.full((len(p2) + 10, 4), -7.0, dtype=torch.float32, pin_memory=True).numpy()
    pv = torch.full((len(p2) + 10, 4), -7.0, dtype=torch.float32, pin_memory=True).numpy()
    p3, v3 = t.particles4((pp, pv))
    np.testing.assert_array_equal(p3, p2)
    np.testing.assert_array_equal(v3, v2)
    assert np.all(pp[len(p2):] == -7.0)
    t.close()


def test_adds_from_page_locked_arrays_equal_adds_from_pageable_ones(pkg):
    """Particles added from page-locked arrays (read by the copy engine directly) arrive exactly as those added
    from ordinary arrays (staged first), with their velocities, marks and ids, and the caller's arrays are
    left as they were."""
    import torch
    rng = np.random.default_rng(8)
    pos = (np.array([0.0, 0.3, 0.0]) + rng.uniform(-0.2, 0.2, (5000, 3))).astype(np.float32)
    vel = rng.uniform(-1, 1, (5000, 3)).astype(np.float32)
    air = (rng.random(5000) < 0.3).astype(np.float32)
    out = []
    for pinned in (False, True):
        t = pkg.Tank(nx=32, ny=32, nz=32, h=1 / 32, whitewater=False, ripple=None, capacity=8192, iters=20)
        args = [torch.from_numpy(a.copy()).pin_memory().numpy() if pinned else a.copy() for a in (pos, vel, air)]
        t.sync()                       # nothing queued: the page-locked arrays go to the device directly
        first = t.add_particles(*args)
        for a, b in zip(args, (pos, vel, air)):
            np.testing.assert_array_equal(a, b)
        out.append((first,) + t.particles4())
        t.substep(1 / 240)
        out[-1] += t.particles4()
        t.close()
    assert out[0][0] == out[1][0]
    np.testing.assert_array_equal(out[0][1], out[1][1])          # as added: in the order given
    np.testing.assert_array_equal(out[0][2], out[1][2])
    np.testing.assert_array_equal(out[1][1][:, :3], pos)
    np.testing.assert_array_equal(out[1][2][:, :3], vel)
    np.testing.assert_array_equal(out[1][1][:, 3], air)
    # after a sub-step the order within a cell follows the binning's atomics: compare by id
    o0, o1 = (np.argsort(o[4][:, 3].view(np.uint32)) for o in out)
    np.testing.assert_array_equal(out[0][3][o0], out[1][3][o1])
    np.testing.assert_array_equal(out[0][4][o0], out[1][4][o1])
    # the library's own page-locked arrays (suiri_host_alloc) for both directions
    t = pkg.Tank(nx=32, ny=32, nz=32, h=1 / 32, whitewater=False, ripple=None, capacity=8192, iters=20)
    hp = pkg.native.host_empty((5000, 3))
    hp[:] = pos
    t.sync()
    t.add_particles(hp, vel, air)
    rp, rv = pkg.native.host_empty((5010, 4)), pkg.native.host_empty((5010, 4))
    p4, v4 = t.particles4((rp, rv))
    np.testing.assert_array_equal(p4, out[1][1])
    np.testing.assert_array_equal(v4, out[1][2])
    t.close()
    with pytest.raises(pkg.native.SuiriError):
        pkg.native.check(pkg.native.lib().suiri_host_free(pkg.native.C.c_void_p(hp.ctypes.data + 16)))


def test_poll_stats_and_pipelined_particle_adds(pkg):
    """Non-blocking stats (pollStats): the first call only starts a read; a read started once the stream is
    idle returns exactly what the blocking read returns. Particles added every sub-step through the two
    staging buffers, without waits in between, all arrive with their ids and values."""
    w = pkg.workloads.dam_break()
    t = pkg.Tank(nx=w['nx'], ny=w['ny'], nz=w['nz'], h=w['h'], whitewater=False, ripple=None,
                 capacity=len(w['pos']) + 4096, iters=20)
    t.add_particles(w['pos'])
    assert t.poll_stats() is None
    rng = np.random.default_rng(3)
    added = []
    for _ in range(12):
        p = (np.array([0.0, 0.8, 0.0]) + rng.uniform(-0.05, 0.05, (7, 3))).astype(np.float32)
        v = np.tile(np.float32([0.0, -1.0, 0.0]), (7, 1))
        added.append(p)
        t.add_particles(p, v)
        t.substep(1 / 240)
        t.poll_stats()
    t.sync()
    t.poll_stats()          # collects the read in flight (it may date from an earlier step), starts one now
    t.sync()
    st = t.poll_stats()
    ref = t.stats()
    assert st is not None and st == ref
    assert ref['count'] == len(w['pos']) + 12 * 7 and ref['frame'] == 12
    pos, vel, air, ids = t.particles()
    assert len(np.unique(ids)) == len(ids) and ids.max() == len(w['pos']) + 12 * 7 - 1
    t.close()
    # the same adds, staged one at a time with a sync after each, give the same particles bit for bit
    u = pkg.Tank(nx=w['nx'], ny=w['ny'], nz=w['nz'], h=w['h'], whitewater=False, ripple=None,
                 capacity=len(w['pos']) + 4096, iters=20)
    u.add_particles(w['pos'])
    for p in added:
        u.add_particles(p, np.tile(np.float32([0.0, -1.0, 0.0]), (7, 1)))
        u.sync()
        u.substep(1 / 240)
        u.sync()
    pu, vu, au, iu = u.particles()
    o, ou = np.argsort(ids), np.argsort(iu)
    np.testing.assert_array_equal(pos[o], pu[ou])
    np.testing.assert_array_equal(vel[o], vu[ou])
    u.close()


def test_emitters_switched_on_and_off_after_capture(pkg):
    """Fixed emitters set and cleared once the sub-step graph exists: emission follows at once (the graph
    reads the emitter count on the device), 20 particles a sub-step, none lost in the closed tank."""
    t = pkg.Tank(nx=16, ny=16, nz=16, h=1 / 32, whitewater=False, ripple=None, capacity=20000, iters=10)
    for _ in range(3):
        t.substep(1 / 240)
    assert t.stats()['count'] == 0
    t.set_emitters([dict(shape='disc', pos=[0.0, 0.4, 0.0], dir=[0.0, -1.0, 0.0], radius=0.05, speed=1.0, count=20)])
    for _ in range(5):
        t.substep(1 / 240)
    assert t.stats()['count'] == 100
    t.set_emitters([])
    for _ in range(3):
        t.substep(1 / 240)
    assert t.stats()['count'] == 100
    t.close()


def test_capacity_reached_sets_full_and_caps_the_count(pkg):
    """An emitter that outruns the particle capacity: emission stops at the capacity (minus its margin),
    the full flag is raised, and the step keeps running."""
    cap = 3000
    t = pkg.Tank(nx=16, ny=16, nz=16, h=1 / 32, whitewater=False, ripple=None, capacity=cap, iters=10)
    t.set_emitters([dict(shape='disc', pos=[0.0, 0.4, 0.0], dir=[0.0, -1.0, 0.0], radius=0.06, speed=1.0, count=400)])
    for _ in range(20):
        t.substep(1 / 240)
    st = t.stats()
    assert st['full'] == 1
    assert 0.9 * cap < st['count'] <= cap
    pos, vel, air, ids = t.particles()
    assert len(ids) == st['count'] and len(np.unique(ids)) == len(ids)
    assert np.all(np.isfinite(pos)) and np.all(np.isfinite(vel))
    t.close()


def test_obstacles_long_run(pkg):
    """The obstacles scene at quarter resolution (32×16×16, h = 1/16 m: the same 2 m tank, sphere, turned
    box and cylinder), its liquid kept in the left half so that it breaks around the obstacles, closed (no
    faucet or drain, so volume is conserved), for the reference scene's 500 sub-steps. The GPU and a
    free-running oracle start from the same particles and are compared on volume (exactly), kinetic energy
    every 100 sub-steps (15 %: the flow past the obstacles is chaotic) and the error bits."""
    w = pkg.workloads.obstacles_inflow(scale=4)
    prm = w['params']
    items = [it for it in w['objects'] if it['kind'] != 'drain']
    nx, ny, nz, h = w['nx'], w['ny'], w['nz'], w['h']
    pos = w['pos'][w['pos'][:, 0] < -0.2]
    gpu = pkg.Tank(nx=nx, ny=ny, nz=nz, h=h, flip=prm['flip'], omega=prm['omega'], iters=prm['iters'],
                   whitewater=False, ripple=None, capacity=len(pos) * 2)
    gpu.set_objects(items)
    ora = oracle_from(nx, ny, nz, h, w['origin'], flip=prm['flip'], omega=prm['omega'], iters=prm['iters'])
    ora.set_objects(objs_from_items(items))
    gpu.add_particles(pos)
    ora.add_particles(f32(pos))
    n0 = gpu.stats()['count']
    ke_g, ke_o = [], []
    for s in range(1, 501):
        gpu.substep(prm['dt'])
        ora.frame = s
        ora.substep(prm['dt'])
        if s % 100 == 0:
            _, v, _, _ = gpu.particles()
            ke_g.append(0.5 * 998 * (h / 2) ** 3 * float(np.sum(v.astype(np.float64) ** 2)))
            ke_o.append(ora.kinetic_energy())
    assert gpu.stats()['count'] == n0 == len(ora.pos)
    ke_g, ke_o = np.array(ke_g), np.array(ke_o)
    assert ke_o.min() > 1e-3, ke_o                 # the liquid is moving
    assert np.all(np.abs(ke_g - ke_o) <= 0.15 * ke_o), (ke_g, ke_o)
    assert gpu.stats()['errors'] == 0
    gpu.close()

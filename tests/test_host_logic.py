"""Host-side logic that needs no GPU: the autotuner's choice (with a stand-in for a tank or batch) and the
synthetic workloads' shapes and seeding."""
import importlib

import numpy as np
import pytest

autotune = importlib.import_module('hahenn-_b200.autotune')
workloads = importlib.import_module('hahenn-_b200.workloads')


class FakeTarget:
    """Times each (blocks per SM, sor_mode, piece_kb) from a table; a None entry cannot be launched. Its
    "state" is a counter of the sub-steps run, saved and restored like the tanks' water copies."""

    def __init__(self, table):
        self.table, self.current, self.applied = table, None, []
        self.piece, self.substeps, self.saves, self.g2p = 0, 0, [], 0

    def tune(self, bps, mode):
        self.current = (bps, mode, self.piece)
        self.applied.append(self.current)

    def key(self):
        return self.current + (self.g2p,)

    def tune_piece(self, kb):
        self.piece = kb

    def tune_g2p(self, form):
        self.g2p = form

    def time_substeps(self, dt, steps):
        self.substeps += steps
        ms = self.table[self.key()]
        if ms is None:
            raise RuntimeError(f'{self.current} cannot be launched')
        return ms * steps

    def save_state(self):
        self.saves.append(self.substeps)
        return len(self.saves) - 1

    def restore_state(self, k):
        self.substeps = self.saves[k]


def test_autotune_keeps_the_fastest_and_skips_shapes_that_fail():
    table = {c + (f,): 5.0 for c in autotune.CANDIDATES for f in autotune.G2P_FORMS}
    table[(2, 4, 128, 0)] = 3.0
    table[(2, 4, 128, 1)] = 2.5          # the brick G2P form is faster with the best solve shape
    table[(4, 0, 0, 1)] = 1.0            # never timed: G2P forms are tried with the best shape only
    table[(4, 1, 0, 0)] = None
    t = FakeTarget(table)
    t.substeps = 7
    best, timings = autotune.autotune(t, 1 / 240)
    assert best == (2, 4, 128, 1) and t.key() == (2, 4, 128, 1)
    assert timings[(4, 1, 0, 0)] == float('inf') and timings[(2, 4, 128, 0)] == pytest.approx(3.0)
    assert set(timings) == {c + (0,) for c in autotune.CANDIDATES} | {(2, 4, 128, f) for f in autotune.G2P_FORMS}
    assert t.substeps == 7              # the tuning sub-steps were rolled back
    assert {c[1] for c in autotune.CANDIDATES} >= {0, 1, 2, 3, 4}
    assert len({c[2] for c in autotune.CANDIDATES if c[1] == 4}) >= 3     # tile sizes of the cluster solve


class NoisyTarget(FakeTarget):
    """Like FakeTarget, but a key listed in `swings` reads fast the first time it is timed and slow after."""

    def __init__(self, table, swings):
        super().__init__(table)
        self.swings, self.seen = swings, set()

    def time_substeps(self, dt, steps):
        ms = super().time_substeps(dt, steps)
        if steps > 1 and self.key() in self.swings:
            if self.key() in self.seen:
                return self.swings[self.key()] * steps
            self.seen.add(self.key())
        return ms


def test_autotune_keeps_the_default_over_marginal_or_swinging_winners():
    table = {c + (f,): 5.0 for c in autotune.CANDIDATES for f in autotune.G2P_FORMS}
    table[(4, 4, 0, 0)] = 4.98           # 0.4 % faster: inside the margin
    best, _ = autotune.autotune(FakeTarget(table), 1 / 240)
    assert best == autotune.CANDIDATES[0] + (0,)
    table[(4, 4, 0, 0)] = 4.0            # fast on its first reading only
    t = NoisyTarget(table, {(4, 4, 0, 0): 6.0})
    best, timings = autotune.autotune(t, 1 / 240)
    assert best == autotune.CANDIDATES[0] + (0,) and t.key() == best
    assert timings[(4, 4, 0, 0)] == pytest.approx(4.0)
    t = NoisyTarget(table, {(4, 4, 0, 0): 4.2})       # slower later, but still clear of the margin
    assert autotune.autotune(t, 1 / 240)[0] == (4, 4, 0, 0)


def test_autotune_raises_when_nothing_launches():
    t = FakeTarget({c + (f,): None for c in autotune.CANDIDATES for f in autotune.G2P_FORMS})
    with pytest.raises(RuntimeError):
        autotune.autotune(t, 1 / 240)


def test_workloads_shapes_and_seeds():
    w = workloads.obstacles_inflow()
    assert (w['nx'], w['ny'], w['nz']) == (128, 64, 64)
    assert 1.69e6 < len(w['pos']) < 1.71e6 and w['pos'].dtype == np.float32
    lo, hi = w['origin'], w['origin'] + w['h'] * np.array([w['nx'], w['ny'], w['nz']])
    assert np.all(w['pos'] >= lo) and np.all(w['pos'] <= hi)    # float32 may round onto the upper wall
    np.testing.assert_array_equal(workloads.obstacles_inflow()['pos'], w['pos'])          # seeded
    specs = workloads.batch_tanks(64)
    assert len(specs) == 64
    assert all(a in workloads.AXES_BATCH for s in specs for a in (s['nx'], s['ny'], s['nz']))
    assert len({(s['nx'], s['ny'], s['nz']) for s in specs}) > 10                        # uneven sizes


class FakeBatch:
    """Two size lanes whose sub-step time is the slower lane's; lane 0 is fastest with the cluster-resident
    solve, lane 1 with one launch per sweep. State: a sub-step counter, saved and restored."""

    def __init__(self):
        self.knobs = [None, None]
        self.substeps, self.saves = 0, []

    def lanes(self):
        return 2

    def tune_lane(self, k, bps, mode, piece, g2p):
        self.knobs[k] = (bps, mode, piece, g2p)

    def lane(self, k):
        from importlib import import_module
        return import_module('hahenn-_b200.tank')._LaneTarget(self, k)

    def time_substeps(self, dt, steps):
        self.substeps += steps
        cost = [{4: 1.0}.get(self.knobs[0][1], 2.0), {0: 1.5}.get(self.knobs[1][1], 3.0)]
        return max(cost) * steps

    def save_state(self):
        self.saves.append(self.substeps)
        return len(self.saves) - 1

    def restore_state(self, k):
        self.substeps = self.saves[k]


def test_batch_tuned_lane_by_lane():
    b = FakeBatch()
    best, timings = autotune.autotune_batch(b, 1 / 240)
    assert [k[1] for k in best] == [4, 0] and b.knobs[0][1] == 4 and b.knobs[1][1] == 0
    assert b.substeps == 0 and set(timings) == {0, 1}


def test_balanced_lanes_keep_sizes_together_and_balance_particles():
    from importlib import import_module
    tk = import_module('hahenn-_b200.tank')
    cells = [100, 100, 200, 400, 800, 800, 1600, 3200]
    parts = [c * 8 for c in cells]
    lane = tk.balanced_lanes(cells, parts, 2)
    assert lane[0] == lane[1] and lane[4] == lane[5]          # equal sizes share a lane
    assert list(lane) == sorted(lane)                          # contiguous in size
    assert set(lane) == {0, 1}
    tot = [sum(p for p, l in zip(parts, lane) if l == k) for k in (0, 1)]
    assert max(tot) <= 0.75 * sum(parts)


def _local_box(o):
    d = o['dims']
    t = o['type']
    if t in (0, 6):
        return np.array([d[0], d[1], d[2]])
    if t in (2, 3, 5):
        return np.array([d[0], d[1], d[0]])
    if t == 4:
        return np.array([d[0] + d[1], d[1], d[0] + d[1]])
    return np.array([d[0], d[0], d[0]])


def _reach_bits(objs, c, h, rc):
    """The per-cell reach rule of the geometry pass, restated: bit 1 an obstacle's cull may hold within
    reach·h of the centre c, bit 2 a drain's bound may (reach = √3/2 + 0.98 + 1e-3)."""
    from oracle import sdf as sdfm
    reach = (0.8660254037844387 + 0.98 + 1e-3) * h + 1e-6
    bits = np.zeros(len(c), np.uint8)
    for o in objs:
        e2 = ((c - o['pos']) ** 2).sum(1)
        if o['flag'] == 2:
            bits |= np.where(e2 <= (o['bound'] + reach) ** 2, 2, 0).astype(np.uint8)
            continue
        if o['type'] == 7:
            bits |= 1
            continue
        inside = e2 < (rc + o['bound'] + 1e-6 + reach) ** 2
        if o['type'] != 1:
            q = sdfm.to_local(o, c)
            out = np.maximum(np.abs(q) - _local_box(o), 0.0)
            inside &= (out ** 2).sum(1) < (rc + 1e-6 + reach) ** 2
        bits |= inside.astype(np.uint8)
    return bits


def _ball(rng, n, r):
    v = rng.normal(size=(n, 3))
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    return v * (r * rng.random((n, 1)) ** (1 / 3))


def test_reach_rule_leaves_out_only_cells_no_collision_or_drain_can_come_from():
    """The reach map's rule on the reference's own shape distances (the oracle's restatement of the WGSL
    library): from a cell it leaves out, no point a particle can reach in the sub-step (within √3/2·h of the
    centre, then at most 0.98h) is within the collision radius of an obstacle or inside a drain. A gutter
    anywhere marks every cell."""
    from oracle import sdf as sdfm
    from parity import objs_from_items
    from test_gpu_parity import ALL_SHAPES
    h = 1 / 40
    rc = 0.32 * h
    items = [it for it in ALL_SHAPES if it['shape'] != 'gutter']
    objs = objs_from_items(items) + [sdfm.make_drain([0.05, 0.0, 0.1], 0.05)]
    rng = np.random.default_rng(4)
    lo, hi = np.array([-0.3, 0.0, -0.2]), np.array([0.3, 0.3, 0.2])
    cells = lo + rng.random((6000, 3)) * (hi - lo)
    bits = _reach_bits(objs, cells, h, rc)
    assert 0 < (bits & 1).sum() < len(cells) and 0 < (bits & 2).sum() < len(cells)
    far_o, far_d = cells[(bits & 1) == 0], cells[(bits & 2) == 0]
    reach = (0.8660254037844387 + 0.98) * h
    for c0, test in ((far_o, lambda p: sdfm.scene_sdf(objs, p, cull=True) >= rc),
                     (far_d, lambda p: ~sdfm.in_drain_analytic(objs, p))):
        p = np.repeat(c0, 16, 0) + _ball(rng, len(c0) * 16, reach)
        assert np.all(test(p))
    # the cells it keeps include ones a collision does come from
    near = cells[(bits & 1) == 1][:2000]
    p = np.repeat(near, 16, 0) + _ball(rng, len(near) * 16, reach)
    assert np.any(sdfm.scene_sdf(objs, p, cull=True) < rc)
    gut = objs_from_items([it for it in ALL_SHAPES if it['shape'] == 'gutter'])
    assert np.all(_reach_bits(gut, cells[:100], h, rc) & 1)


def test_nearest_obstacle_normal_samples_equal_the_scene_distance():
    """The collision normal's shortcut, on the reference's shape distances: where the culled scene loop at p
    puts every obstacle but the nearest more than d + 2e (+1e-6) away (computed distance, or bounding-sphere
    distance where the cull skipped it), the scene distance at each of the six samples p ± e·axis equals the
    nearest obstacle's own distance bit for bit."""
    from oracle import sdf as sdfm
    from parity import objs_from_items
    from test_gpu_parity import ALL_SHAPES
    objs = [o for o in objs_from_items([it for it in ALL_SHAPES if it['shape'] != 'gutter'])]
    rng = np.random.default_rng(6)
    lo, hi = np.array([-0.3, 0.0, -0.2]), np.array([0.3, 0.3, 0.2])
    p = lo + rng.random((200000, 3)) * (hi - lo)
    d_all = np.stack([sdfm.shape_sdf(o, p) for o in objs], 1)
    p = p[np.abs(d_all.min(1)) < 0.01][:20000]             # near a surface, as colliding particles are
    e = 0.0006
    # the culled loop, tracking the nearest and a lower bound on the others
    best = np.full(len(p), sdfm.BIG)
    near = np.full(len(p), -1)
    other = np.full(len(p), sdfm.BIG)
    for i, o in enumerate(objs):
        c = np.linalg.norm(p - o['pos'], axis=1) - o['bound']
        d = sdfm.shape_sdf(o, p)
        culled = c > best
        other = np.where(culled, np.minimum(other, c), other)
        better = ~culled & (d < best)
        other = np.where(better & (near >= 0), np.minimum(other, best), other)
        other = np.where(~culled & ~better, np.minimum(other, d), other)
        near = np.where(better, i, near)
        best = np.where(better, d, best)
    np.testing.assert_array_equal(best, sdfm.scene_sdf(objs, p, cull=True))
    ok = (near >= 0) & (other > best + 2 * e + 1e-6)
    assert ok.mean() > 0.5 and (~ok).any()
    for axis in range(3):
        for sgn in (1.0, -1.0):
            q = p.copy()
            q[:, axis] = p[:, axis] + sgn * e
            scene = sdfm.scene_sdf(objs, q, cull=True)
            own = np.choose(near.clip(0), [sdfm.shape_sdf(o, q) for o in objs])
            np.testing.assert_array_equal(scene[ok], own[ok])

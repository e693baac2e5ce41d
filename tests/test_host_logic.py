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

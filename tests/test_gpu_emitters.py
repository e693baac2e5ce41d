"""Scene sources emitted on the device by step(): per-mode particle counts follow the reference's
accumulators exactly (src/js/55-emit.js:13-69, solver.py:345-413), positions fall where the source
puts them."""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def js_round(x):
    return math.floor(x + 0.5)


def expected_counts(src, vp, dt, steps):
    """Particles emitted per sub-step by one source, restating sourceEmits' state machine."""
    acc = timer = liters = 0.0
    fired = False
    out = []
    for _ in range(steps):
        n = 0
        mode = src['mode']
        if mode in ('stream', 'shower'):
            acc += (src['flow'] / 60000 * dt) / vp
            n = math.floor(acc)
            acc -= n
        elif mode == 'drops':
            timer -= dt
            if timer <= 0:
                timer += 1 / min(max(src['dropRate'], 0.05), 60)
                timer = max(timer, 0)
                d = min(max(src['dropD'], 1), 40) / 1000
                n = max(1, js_round(math.pi / 6 * d * d * d / vp))
        elif mode == 'burst':
            if not fired:
                fired = True
                n = max(1, js_round(min(max(src['burst'], 0.01), 50) / 1000 / vp))
        elif mode == 'rain':
            side = min(max(src['rainSize'], 0.05), 2)
            acc += ((min(max(src['rainRate'], 1), 500) / 3.6e6) * side * side * dt) / vp
            n = math.floor(acc)
            acc -= n
        out.append(n)
    return out


SOURCES = [
    dict(mode='stream', flow=3.0, speed=0.6, pos=[0.0, 0.25, 0.0], pitch=-90, yaw=0),
    dict(mode='shower', flow=4.0, speed=0.8, spread=18, pos=[0.05, 0.25, 0.0], pitch=-90, yaw=0),
    dict(mode='drops', dropD=6, dropRate=30, speed=0.0, pos=[0.0, 0.25, 0.05], pitch=-90, yaw=0),
    dict(mode='burst', burst=0.05, speed=0.5, pos=[0.0, 0.2, 0.0], pitch=-90, yaw=0),
    dict(mode='rain', rainRate=400, rainSize=0.2, pos=[0.0, 0.28, 0.0], pitch=-90, yaw=0),
]


@pytest.mark.parametrize('src', SOURCES, ids=[s['mode'] for s in SOURCES])
def test_source_counts_and_placement(pkg, src):
    scene = dict(v=1, app='suiri-lab', scene=dict(tank=dict(w=0.4, h=0.3, d=0.3),
                                                  items=[dict(kind='source', id=5, enabled=True, **src)]))
    t = pkg.Tank(scene, quality='low', whitewater=False, ripple=None)
    dt, steps = 1 / 240, 12
    exp = expected_counts(src, (t.h / 2) ** 3, dt, steps)
    total = 0
    for k in range(steps):
        assert t.step(dt) == 1
        total += exp[k]
        assert t.stats()['count'] == total, (k, t.stats()['count'], total)
    pos, vel, air, ids = t.particles()
    assert total > 0 and len(pos) == total
    p = np.array(src['pos'])
    if src['mode'] in ('stream', 'shower'):
        # the outlet disc 2 mm below the nozzle, particles moving down
        assert np.all(np.hypot(pos[:, 0] - p[0], pos[:, 2] - p[2]) < 0.03)
        assert np.all(vel[:, 1] < 0)
    if src['mode'] == 'rain':
        assert np.all(np.abs(pos[:, [0, 2]] - p[[0, 2]]) <= 0.1 + 1e-6)
        assert np.all(air == 1)                  # rain drops carry the free-flight mark
    t.close()

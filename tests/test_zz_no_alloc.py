"""suiri_eval_sdf_static — obstacle distances for callers that cannot allocate device memory when they ask
(a host whose device memory is fully committed to resident scenes, or a per-frame picking/placement loop
that must keep the allocator off its path). It stages points and distances in one fixed array inside the
library instead of allocating per call.

Checked through the C ABI on two calls in a row with different points: against suiri_eval_sdf, which
allocates its staging per call (the same kernel computes both, so the distances must agree exactly), and
against the oracle's distances, so the second call's results are its own points' distances and not
staging left from the first. After a warm-up call, several calls leave the device's free memory and its
default memory pool's used and reserved bytes unchanged. This file is collected last so that a run
stopping at the first failure has already run every other test; it also passes alone in a fresh process."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MAX_POINTS = 65536

SCENE_ITEMS = [
    dict(kind='obstacle', shape='sphere', pos=[0.1, 0.15, 0.0], rot=[0, 0, 0], dims=dict(r=0.06)),
    dict(kind='obstacle', shape='gutter', pos=[-0.1, 0.2, -0.05], rot=[0, 0, -14], dims=dict(len=0.28, r=0.03, t=0.006)),
    dict(kind='obstacle', shape='container', pos=[0.15, 0.04, -0.1], rot=[0, 20, 0], dims=dict(w=0.14, h=0.06, d=0.1, t=0.008)),
]


def call_static(pkg, tank, pts):
    L = pkg.native.lib()
    p = np.ascontiguousarray(pts, np.float64)
    b = np.full(len(p), np.nan)
    pkg.native.check(L.suiri_eval_sdf_static(tank.handle, C.c_void_p(p.ctypes.data), len(p), C.c_void_p(b.ctypes.data)),
                     tank.handle)
    return b


def eval_both(pkg, tank, pts):
    L = pkg.native.lib()
    p = np.ascontiguousarray(pts, np.float64)
    a = np.full(len(p), np.nan)
    pkg.native.check(L.suiri_eval_sdf(tank.handle, C.c_void_p(p.ctypes.data), len(p), C.c_void_p(a.ctypes.data)), tank.handle)
    return a, call_static(pkg, tank, pts)


def device_memory(dev):
    """(free bytes of the device, used and reserved bytes of its default memory pool)."""
    from cuda.bindings import runtime as rt
    err, free, _ = rt.cudaMemGetInfo()
    assert err == rt.cudaError_t.cudaSuccess
    err, pool = rt.cudaDeviceGetDefaultMemPool(dev)
    assert err == rt.cudaError_t.cudaSuccess
    out = [free]
    for attr in (rt.cudaMemPoolAttr.cudaMemPoolAttrUsedMemCurrent, rt.cudaMemPoolAttr.cudaMemPoolAttrReservedMemCurrent):
        err, v = rt.cudaMemPoolGetAttribute(pool, attr)
        assert err == rt.cudaError_t.cudaSuccess
        out.append(int(v))
    return tuple(out)


@pytest.mark.parametrize('mode', ['analytic', 'lattice'])
def test_static_staging_matches_allocating_entry_point(pkg, mode):
    from oracle import flip as of
    from parity import objs_from_items
    t = pkg.Tank(nx=24, ny=12, nz=16, h=1 / 40, whitewater=False, ripple=None, capacity=1024, sdf_mode=mode)
    t.set_objects(SCENE_ITEMS)
    ora = of.Tank(24, 12, 16, 1 / 40, origin=t.origin, sdf_mode=mode)
    ora.set_objects(objs_from_items(SCENE_ITEMS))
    if mode == 'lattice':
        t.set_lattice(ora.lat)
    rng = np.random.default_rng(21)
    span = np.array([24, 12, 16]) / 40
    first = t.origin + rng.random((50000, 3)) * span
    second = t.origin + rng.random((1234, 3)) * span
    for pts in (first, second):
        a, b = eval_both(pkg, t, pts)
        assert np.isfinite(a).all()
        np.testing.assert_array_equal(b, a)
        np.testing.assert_array_equal(b, ora.sdf_at(pts))
    t.close()


def test_static_staging_allocates_nothing(pkg):
    t = pkg.Tank(nx=24, ny=12, nz=16, h=1 / 40, whitewater=False, ripple=None, capacity=1024)
    t.set_objects(SCENE_ITEMS)
    rng = np.random.default_rng(22)
    pts = t.origin + rng.random((MAX_POINTS, 3)) * (np.array([24, 12, 16]) / 40)
    call_static(pkg, t, pts[:100])                         # warm-up: the per-device address lookup
    before = device_memory(0)
    for n in (MAX_POINTS, 17, 4096, MAX_POINTS):
        call_static(pkg, t, pts[:n])
    assert device_memory(0) == before
    t.close()


def test_static_staging_rejects_more_than_its_size(pkg):
    t = pkg.Tank(nx=8, ny=8, nz=8, h=1 / 16, whitewater=False, ripple=None, capacity=64)
    t.set_objects(SCENE_ITEMS[:1])
    L = pkg.native.lib()
    p = np.zeros((MAX_POINTS + 1, 3))
    out = np.zeros(MAX_POINTS + 1)
    rc = L.suiri_eval_sdf_static(t.handle, C.c_void_p(p.ctypes.data), len(p), C.c_void_p(out.ctypes.data))
    assert rc == -1
    assert b'at most 65536' in L.suiri_last_error(t.handle)
    # exactly the maximum is accepted
    rc = L.suiri_eval_sdf_static(t.handle, C.c_void_p(p.ctypes.data), MAX_POINTS, C.c_void_p(out.ctypes.data))
    assert rc == 0
    t.close()

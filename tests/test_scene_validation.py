"""Scene-JSON validation as the reference's editor does it when it opens a scene file (validScene,
src/js/80-ui.js:430-459): field by field against a fresh item of the same kind (src/js/10-scene.js:56-86),
the tank clamped to the editor's limits, ids kept or renumbered. Through the C ABI (suiri_scene_validate,
no GPU needed)."""
import ctypes as C
import json
import math

import pytest

from conftest import package


@pytest.fixture(scope='module')
def N():
    return package().native


def scene(items, tank=None):
    return dict(v=1, app='suiri-lab', scene=dict(tank=tank or dict(w=0.6, h=0.32, d=0.4), items=items), cam={})


def test_tank_clamped_to_the_editor_limits(N):
    out = N.validate_scene(scene([], dict(w=5.0, h=0.01, d=0.4)))
    assert out['tank'] == dict(w=1.2, h=0.1, d=0.4)
    out = N.validate_scene(scene([], dict(w=0.1, h=2.0, d=0.05)))
    assert out['tank'] == dict(w=0.2, h=0.6, d=0.15)
    # the explicit-grid path reads the tank as given
    out = N.validate_scene(scene([], dict(w=5.0, h=0.01, d=0.4)), clamp_tank=False)
    assert out['tank'] == dict(w=5.0, h=0.01, d=0.4)


@pytest.mark.parametrize('doc', [
    '{"scene": {"tank": {"w": 0.6, "h": 0.3, "d": 0.4}, "items": [}}',        # malformed JSON
    json.dumps(dict(scene=dict(tank=dict(w=0.6, h=0.0, d=0.4), items=[]))),   # tank size not positive
    json.dumps(dict(scene=dict(tank=dict(w=0.6, h='0.3', d=0.4), items=[]))),  # tank size not a number
    json.dumps(dict(scene=dict(tank=dict(w=0.6, h=0.3), items=[]))),          # a tank size missing
    json.dumps(dict(scene=dict(tank=dict(w=0.6, h=0.3, d=0.4), items={}))),   # items not an array
    json.dumps(dict(scene=dict(items=[]))),                                     # no tank
])
def test_unusable_documents_are_refused_with_a_parse_error(N, doc):
    n = C.c_size_t()
    assert N.lib().suiri_scene_validate(doc.encode(), 1, None, 0, C.byref(n)) == -5
    assert N.lib().suiri_last_error(None)


def test_every_field_of_every_kind_falls_back_to_a_fresh_item(N):
    items = [
        dict(id=1, kind='obstacle', shape='teapot', pos=[0.1, 'x', 0.0], rot=[0, 10], dims=dict(w=0.2, h=None),
             material='gold', color='', name=5),
        dict(id=2, kind='obstacle', shape='cylinder', pos=[0.1, 0.2, 0.3], rot=[0, 30, 0], dims=dict(r=0.05, q=1),
             material='metal', color='#112233', name='post'),
        dict(id=3, kind='source', mode='laser', flow=12, enabled='yes', pitch=float('nan'), total=2.5),
        dict(id=4, kind='source', mode='rain', enabled=False, rainRate=120, rainSize=0.5),
        dict(id=5, kind='drain', r='wide', pos=[0.2, 0.0, -0.1, 9]),
        dict(id=6, kind='block', dims=dict(w=0.3), pos=[0.0, 0.1, 0.0]),
    ]
    out = N.validate_scene(json.dumps(scene(items)).replace('NaN', '"nan"'))['items']
    assert [it['kind'] for it in out] == ['obstacle', 'obstacle', 'source', 'source', 'drain', 'block']
    box, cyl, src, rain, drain, block = out
    # an unknown shape is a box; its fields come from a fresh box where the item's are unusable
    assert box['shape'] == 'box' and box['name'] == '箱' and box['material'] == 'ceramic' and box['color'] == '#c9c2b4'
    assert box['pos'] == [0, 0.05, 0] and box['rot'] == [0, 0, 0]
    assert box['dims'] == dict(w=0.2, h=0.06, d=0.08)
    # usable fields are kept; dims are the shape's own keys only
    assert cyl['shape'] == 'cylinder' and cyl['name'] == 'post' and cyl['material'] == 'metal' and cyl['color'] == '#112233'
    assert cyl['pos'] == [0.1, 0.2, 0.3] and cyl['rot'] == [0, 30, 0] and cyl['dims'] == dict(r=0.05, h=0.12)
    fresh_src = dict(name='水源', pos=[0, 0.4, 0], pitch=-90, yaw=0, mode='stream', enabled=True, flow=3.0, speed=0.6,
                     dropD=5, dropRate=3, spread=18, burst=0.5, burstEvery=0, rainRate=60, rainSize=0.3, total=0)
    assert {k: src[k] for k in fresh_src} == dict(fresh_src, flow=12, total=2.5)
    assert rain['mode'] == 'rain' and rain['enabled'] is False and rain['rainRate'] == 120 and rain['rainSize'] == 0.5
    assert drain['r'] == 0.025 and drain['pos'] == [0, 0, 0] and drain['name'] == '排水口'
    assert block['dims'] == dict(w=0.3, h=0.1, d=0.16) and block['pos'] == [0, 0.1, 0]


def test_ids_kept_or_numbered_on_from_the_largest(N):
    items = [dict(id=7, kind='block'), dict(id=7, kind='drain'), dict(kind='source'), dict(id=2.5, kind='block'),
             dict(id=-1, kind='drain'), dict(id=3, kind='obstacle', shape='sphere'), 'text', dict(kind='alien'),
             dict(id=1, kind='unknown')]
    out = N.validate_scene(scene(items))['items']
    assert [it['id'] for it in out] == [7, 8, 9, 10, 11, 3]
    assert [it['kind'] for it in out] == ['block', 'drain', 'source', 'block', 'drain', 'obstacle']


def test_validation_is_idempotent_and_the_buffer_is_checked(N):
    items = [dict(kind='obstacle', shape='torus', dims=dict(R=0.07)), dict(kind='source', mode='drops', dropD=3)]
    once = N.validate_scene(scene(items, dict(w=2.0, h=0.5, d=0.3)))
    assert once == N.validate_scene(once)
    assert math.isclose(once['items'][0]['dims']['r'], 0.014) and once['items'][0]['dims']['R'] == 0.07
    js = json.dumps(scene(items)).encode()
    n = C.c_size_t()
    assert N.lib().suiri_scene_validate(js, 1, None, 0, C.byref(n)) == 0 and n.value > 0
    small = C.create_string_buffer(n.value)            # no room for the terminating NUL
    assert N.lib().suiri_scene_validate(js, 1, small, n.value, C.byref(n)) == -1

"""ctypes binding of libsuiri_cuda.so (include/suiri.h).

The library is the only implementation: there is no CPU fallback. Loading fails loudly when the in-tree
build is missing; build it with ``python hahenn-_b200/build.py``.
"""
import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, 'libsuiri_cuda.so')

OK = 0
ERR = {-1: 'invalid argument', -2: 'CUDA error', -3: 'out of memory', -4: 'capacity reached', -5: 'parse error',
       -6: 'invalid state'}

FIELD_CELL_COUNT, FIELD_FRAC, FIELD_VEL, FIELD_VELOLD, FIELD_MASK, FIELD_PRES, FIELD_RHS = range(7)
FIELD_RIPPLE_SRC, FIELD_RIPPLE, FIELD_TOP, FIELD_RIPPLE_STATE, FIELD_RIPPLE_MASK, FIELD_TOP64 = 7, 8, 9, 10, 11, 12


class Params(C.Structure):
    _fields_ = [('size', C.c_uint32), ('nx', C.c_int32), ('ny', C.c_int32), ('nz', C.c_int32), ('h', C.c_double),
                ('quality', C.c_char_p), ('clamp_tank', C.c_int32), ('extra_height', C.c_double),
                ('flip', C.c_double), ('omega', C.c_double), ('iters', C.c_int32), ('gravity', C.c_double),
                ('friction', C.c_double), ('ppc', C.c_double), ('drift', C.c_double), ('ww_rate', C.c_double),
                ('whitewater', C.c_int32), ('capacity', C.c_int64), ('ww_capacity', C.c_int64),
                ('ripple_rx', C.c_int32), ('ripple_rz', C.c_int32), ('wmap', C.c_int32), ('sdf_mode', C.c_int32),
                ('device', C.c_int32), ('seed', C.c_uint32), ('ripple_sigma', C.c_double), ('ripple_rho', C.c_double),
                ('ripple_depth', C.c_double), ('advect', C.c_int32), ('drop_d_median', C.c_double),
                ('drop_d_sigma_log', C.c_double), ('sor_mode', C.c_int32), ('watchdog_polls', C.c_int64)]


class Stats(C.Structure):
    _fields_ = [('count', C.c_int64), ('ww_count', C.c_int64), ('impacts', C.c_int64), ('vmax', C.c_double),
                ('time', C.c_double), ('liters', C.c_double), ('full', C.c_int32), ('frame', C.c_int32),
                ('errors', C.c_int32), ('pad', C.c_int32), ('nx', C.c_int32), ('ny', C.c_int32), ('nz', C.c_int32), ('h', C.c_double),
                ('origin', C.c_double * 3), ('active_cells', C.c_int64), ('residual_max', C.c_double),
                ('residual_rms', C.c_double), ('rhs_max', C.c_double), ('ripple_rx', C.c_int32), ('ripple_rz', C.c_int32),
                ('wmap', C.c_int32), ('pad2', C.c_int32)]


PHASES = ('bin_sort', 'p2g', 'grid_passes', 'pressure_solve', 'projection', 'g2p')


class Object(C.Structure):
    _fields_ = [('type', C.c_int32), ('flag', C.c_int32), ('pos', C.c_double * 3), ('rot', C.c_double * 9),
                ('dims', C.c_double * 4), ('lin', C.c_double * 3), ('ang', C.c_double * 3)]


class Emitter(C.Structure):
    _fields_ = [('shape', C.c_int32), ('airborne', C.c_int32), ('pos', C.c_double * 3), ('dir', C.c_double * 3),
                ('radius', C.c_double), ('speed', C.c_double), ('per_substep', C.c_double), ('radius_z', C.c_double)]


class MeshInfo(C.Structure):
    _fields_ = [('verts', C.c_int64), ('quads', C.c_int64), ('tris', C.c_int64), ('body_verts', C.c_int64),
                ('lone', C.c_int64), ('lattice', C.c_int32 * 3), ('taps', C.c_int32), ('lo', C.c_double * 3),
                ('spacing', C.c_double), ('smooth', C.c_double), ('weights', C.c_double * 33),
                ('phase_ms', C.c_double * 5)]


MESH_PHASES = ('classify', 'distance_field', 'blur', 'surface_nets', 'finish')


class Request(C.Structure):
    _fields_ = [('size', C.c_uint32), ('params', C.POINTER(Params)), ('scene_json', C.c_char_p),
                ('emitters', C.POINTER(Emitter)), ('n_emitters', C.c_int32), ('steps', C.c_int32),
                ('keep_result', C.c_int32)]


class ServerStats(C.Structure):
    _fields_ = [('completed', C.c_int64), ('queued', C.c_int64), ('running', C.c_int64), ('failed', C.c_int64),
                ('rebuilds', C.c_int64), ('substeps', C.c_int64), ('particle_steps', C.c_double),
                ('elapsed_s', C.c_double), ('used_bytes', C.c_double), ('budget_bytes', C.c_double),
                ('p50_ms', C.c_double), ('p99_ms', C.c_double), ('mean_active', C.c_double)]


P = C.c_void_p
# name: (restype, argtypes) for every entry point of include/suiri.h
SIGNATURES = {
    'suiri_server_create': (C.c_int, [C.c_int32, C.c_double, C.c_double, C.POINTER(P)]),
    'suiri_server_destroy': (C.c_int, [P]),
    'suiri_server_submit': (C.c_int, [P, C.POINTER(Request), C.POINTER(C.c_int64)]),
    'suiri_server_poll': (C.c_int, [P, C.c_int64, C.POINTER(C.c_int32), C.POINTER(C.c_double), C.POINTER(C.c_int64)]),
    'suiri_server_wait': (C.c_int, [P, C.c_int64, C.c_double]),
    'suiri_server_result': (C.c_int, [P, C.c_int64, P, P, C.c_int64, C.POINTER(C.c_int64)]),
    'suiri_server_get_stats': (C.c_int, [P, C.POINTER(ServerStats)]),
    'suiri_set_emitters': (C.c_int, [P, C.POINTER(Emitter), C.c_int32]),
    'suiri_tune': (C.c_int, [P, C.c_int32, C.c_int32]),
    'suiri_eval_sdf': (C.c_int, [P, P, C.c_int64, P]),
    'suiri_eval_sdf_static': (C.c_int, [P, P, C.c_int64, P]),
    'suiri_estimate_bytes': (C.c_int, [C.c_char_p, C.POINTER(Params), C.POINTER(C.c_double)]),
    'suiri_profile': (C.c_int, [P, C.c_int32]),
    'suiri_sor_phase_ms': (C.c_int, [P, C.POINTER(C.c_double)]),
    'suiri_batch_profile': (C.c_int, [P, C.c_int32]),
    'suiri_batch_sor_phase_ms': (C.c_int, [P, C.POINTER(C.c_double)]),
    'suiri_params_default': (C.c_int, [C.POINTER(Params)]),
    'suiri_create': (C.c_int, [C.c_char_p, C.POINTER(Params), C.POINTER(P)]),
    'suiri_destroy': (C.c_int, [P]),
    'suiri_last_error': (C.c_char_p, [P]),
    'suiri_reset': (C.c_int, [P]),
    'suiri_clear': (C.c_int, [P]),
    'suiri_set_objects': (C.c_int, [P, C.c_char_p, C.c_double, C.POINTER(C.c_int32)]),
    'suiri_set_obstacles': (C.c_int, [P, C.POINTER(Object), C.c_int32]),
    'suiri_set_lattice': (C.c_int, [P, P, P, C.c_int32, C.c_int32, C.c_int32]),
    'suiri_add_particles': (C.c_int, [P, P, P, P, C.c_int64, C.POINTER(C.c_uint32)]),
    'suiri_emit_block': (C.c_int, [P, C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_int32]),
    'suiri_substep': (C.c_int, [P, C.c_double]),
    'suiri_step': (C.c_int, [P, C.c_double, C.POINTER(C.c_int32)]),
    'suiri_sync': (C.c_int, [P]),
    'suiri_read_particles': (C.c_int, [P, P, P, C.c_int64, C.POINTER(C.c_int64)]),
    'suiri_read_whitewater': (C.c_int, [P, P, P, C.c_int64, C.POINTER(C.c_int64)]),
    'suiri_read_grid': (C.c_int, [P, C.c_int32, P, C.c_size_t]),
    'suiri_frame_maps': (C.c_int, [P, P, P, C.c_size_t]),
    'suiri_frame_end': (C.c_int, [P, C.c_double]),
    'suiri_surface_mesh': (C.c_int, [P, C.c_double, P]),
    'suiri_surface_mesh_read': (C.c_int, [P, P, P, P, P, C.c_int64, C.c_int64, C.c_int64]),
    'suiri_get_stats': (C.c_int, [P, C.POINTER(Stats)]),
    'suiri_poll_stats': (C.c_int, [P, C.POINTER(Stats), C.POINTER(C.c_int32)]),
    'suiri_stats_readback_bytes': (C.c_size_t, []),
    'suiri_snapshot': (C.c_int, [P, C.POINTER(C.c_int32)]),
    'suiri_restore': (C.c_int, [P, C.c_int32]),
    'suiri_stream': (C.c_int, [P, C.POINTER(P)]),
    'suiri_use_graphs': (C.c_int, [P, C.c_int32]),
    'suiri_batch_create': (C.c_int, [C.POINTER(P), C.c_int32, C.POINTER(P)]),
    'suiri_batch_create_lanes': (C.c_int, [C.POINTER(P), C.c_int32, P, C.POINTER(P)]),
    'suiri_batch_destroy': (C.c_int, [P]),
    'suiri_batch_substep': (C.c_int, [P, C.c_double]),
    'suiri_host_alloc': (C.c_int, [C.c_size_t, C.POINTER(C.c_void_p)]),
    'suiri_host_free': (C.c_int, [P]),
    'suiri_batch_sync': (C.c_int, [P]),
    'suiri_batch_tune': (C.c_int, [P, C.c_int32, C.c_int32]),
    'suiri_batch_stream': (C.c_int, [P, C.POINTER(P)]),
    'suiri_time_substeps': (C.c_int, [P, C.c_double, C.c_int32, C.POINTER(C.c_double)]),
    'suiri_batch_time_substeps': (C.c_int, [P, C.c_double, C.c_int32, C.POINTER(C.c_double)]),
    'suiri_time_sor': (C.c_int, [P, C.c_int32, C.POINTER(C.c_double)]),
    'suiri_add_whitewater': (C.c_int, [P, P, P, C.c_int64]),
    'suiri_scene_validate': (C.c_int, [C.c_char_p, C.c_int32, C.c_char_p, C.c_size_t, C.POINTER(C.c_size_t)]),
    'suiri_tune_piece': (C.c_int, [P, C.c_int32]),
    'suiri_tune_g2p': (C.c_int, [P, C.c_int32]),
    'suiri_batch_tune_g2p': (C.c_int, [P, C.c_int32]),
    'suiri_batch_tune_lane': (C.c_int, [P, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32]),
    'suiri_batch_tune_piece': (C.c_int, [P, C.c_int32]),
    'suiri_residual': (C.c_int, [P, C.c_int32]),
    'suiri_batch_residual': (C.c_int, [P, C.c_int32]),
    'suiri_phase_ms': (C.c_int, [P, C.POINTER(C.c_double)]),
    'suiri_batch_lanes': (C.c_int, [P, C.POINTER(C.c_int32)]),
    'suiri_batch_phase_ms': (C.c_int, [P, C.c_int32, C.POINTER(C.c_double)]),
}

_lib = None


class SuiriError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f'{ERR.get(code, code)}: {msg}')
        self.code = code


def lib():
    """The loaded library (declares every signature on first use)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f'{LIB_PATH} is missing: build it with `python hahenn-_b200/build.py`')
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype, f.argtypes = res, args
        _lib = L
    return _lib


def validate_scene(scene, clamp_tank=True):
    """The scene (JSON text or a dict) as the library reads it (suiri_scene_validate): a dict {tank, items}."""
    import json
    js = (scene if isinstance(scene, (str, bytes)) else json.dumps(scene))
    js = js.encode() if isinstance(js, str) else js
    n = C.c_size_t()
    check(lib().suiri_scene_validate(js, 1 if clamp_tank else 0, None, 0, C.byref(n)))
    buf = C.create_string_buffer(n.value + 1)
    check(lib().suiri_scene_validate(js, 1 if clamp_tank else 0, buf, n.value + 1, C.byref(n)))
    return json.loads(buf.value.decode())


def host_empty(shape, dtype='float32'):
    """An uninitialised NumPy array in page-locked host memory from the library (suiri_host_alloc), released
    to the library's cache when the array and its views are gone. Particle adds and read-backs with such
    arrays are copied by the copy engine directly."""
    import weakref
    import numpy as np
    dt = np.dtype(dtype)
    n = max(1, int(np.prod(shape)) * dt.itemsize)
    ptr = C.c_void_p()
    check(lib().suiri_host_alloc(n, C.byref(ptr)))
    buf = (C.c_char * n).from_address(ptr.value)
    weakref.finalize(buf, lib().suiri_host_free, C.c_void_p(ptr.value))
    return np.frombuffer(buf, dtype=dt, count=int(np.prod(shape))).reshape(shape)


def check(rc, handle=None):
    if rc != OK:
        msg = lib().suiri_last_error(handle)
        raise SuiriError(rc, msg.decode(errors='replace') if msg else '')
    return rc

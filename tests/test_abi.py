"""The C-ABI library loads and exports every entry point that include/suiri.h declares (no GPU needed:
nothing here calls into CUDA beyond the parameter defaults)."""
import ctypes
import os
import re

from conftest import ROOT


def declared():
    text = open(os.path.join(ROOT, 'include', 'suiri.h')).read()
    text = re.sub(r'/\*.*?\*/', '', text, flags=re.S)
    return sorted(set(re.findall(r'\b(suiri_[a-z_0-9]+)\s*\(', text)))


def test_header_declares_entry_points():
    names = declared()
    for n in ('suiri_create', 'suiri_step', 'suiri_substep', 'suiri_reset', 'suiri_set_objects', 'suiri_read_grid',
              'suiri_batch_create', 'suiri_batch_substep'):
        assert n in names


def test_library_exports_every_declared_symbol(pkg):
    lib = pkg.native.lib()
    missing = [n for n in declared() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_the_header(pkg):
    assert set(pkg.native.SIGNATURES) == set(declared())


def test_params_default_and_struct_layout(pkg):
    N = pkg.native
    p = N.Params()
    assert N.lib().suiri_params_default(ctypes.byref(p)) == 0
    assert p.size == ctypes.sizeof(N.Params)
    assert p.quality == b'standard' and abs(p.flip - 0.96) < 1e-15 and abs(p.omega - 1.6) < 1e-15
    assert p.whitewater == 1 and p.clamp_tank == 1


def test_bad_arguments_fail_with_codes_not_crashes(pkg):
    N = pkg.native
    L = N.lib()
    assert L.suiri_destroy(None) == -1
    assert L.suiri_substep(None, 0.01) == -1
    assert b'null' in L.suiri_last_error(None)
    p = N.Params()
    L.suiri_params_default(ctypes.byref(p))
    p.size = 3
    h = ctypes.c_void_p()
    assert L.suiri_create(None, ctypes.byref(p), ctypes.byref(h)) == -1
    assert b'size' in L.suiri_last_error(None)

"""The C ABI library: loads without a GPU and exports every entry point
declared in include/irbc.h.  No compute calls are made here."""
import ctypes as C
import os
import subprocess

import pytest

import irbc_b200 as G


def test_library_exports_every_declared_symbol():
    L = G.lib()
    names = G.exported_names()
    assert len(names) >= 30
    missing = [n for n in names if not hasattr(L, n)]
    assert missing == []


def test_nm_lists_the_same_symbols():
    out = subprocess.run(["nm", "-D", "--defined-only", G.LIB_PATH], capture_output=True, text=True).stdout
    exported = {l.split()[-1] for l in out.splitlines() if " T " in l}
    assert set(G.exported_names()) <= exported


def test_struct_layouts_match_header():
    # field counts/offsets of the ctypes mirror follow include/irbc.h
    assert C.sizeof(G.Params) % 8 == 0
    assert G.View.step.offset % 8 == 0
    import oracle as O
    assert C.sizeof(G.View) == C.sizeof(O.View)
    for (a, _), (b, _) in zip(G.View._fields_, O.View._fields_):
        assert a == b and getattr(G.View, a).offset == getattr(O.View, b).offset


def test_default_params_are_define_h():
    p = G.default_params()
    assert (p.Lx, p.Ly, p.Lz, p.Ns, p.Nt) == (60.0, 40.0, 40.0, 960000, 600)
    assert (p.dtcd, p.dtmd, p.navg, p.walls) == (0.02, 0.002, 10.0, 3.0)
    assert p.cosalpha == -0.70710678118 and p.sinalpha == 0.70710678118
    assert (p.kappasa, p.kappad, p.kappav, p.kappab, p.ks) == (60000.0, 1200.0, 6000.0, 100.0, 6000.0)
    assert p.Pi == 3.141592653 and p.randno == 12345678


def test_footprint_grows_with_box():
    L = G.lib()
    p = G.default_params()
    small = L.irbc_footprint_bytes(C.byref(p), 600, 1794, 1196)
    p.Lx, p.Ly, p.Lz, p.Ns = 128.0, 64.0, 64.0, 5242880
    big = L.irbc_footprint_bytes(C.byref(p), 2562, 7680, 5120)
    assert 0 < small < big < 4 * 10**9


def test_create_rejects_bad_parameters():
    L = G.lib()
    p = G.default_params()
    p.a = 0.5
    h = C.c_void_p()
    assert L.irbc_create(C.byref(p), C.byref(h)) == -1
    p = G.default_params()
    p.precision = 7
    assert L.irbc_create(C.byref(p), C.byref(h)) == -1


@pytest.mark.skipif(os.environ.get("CUDA_VISIBLE_DEVICES", None) is not None and False, reason="")
def test_create_without_device_fails_cleanly():
    from helpers import gpu_available
    if gpu_available():
        pytest.skip("a GPU is present")
    L = G.lib()
    p = G.default_params()
    p.Ns = 1000
    h = C.c_void_p()
    assert L.irbc_create(C.byref(p), C.byref(h)) == -2

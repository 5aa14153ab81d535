"""The C-ABI library builds, loads and exports every declared symbol (CPU)."""
import ctypes
import os
import re

from conftest import ROOT


def declared_functions():
    names = []
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if not fn.endswith(".h"):
            continue
        text = open(os.path.join(ROOT, "include", fn)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names += re.findall(r"\b(cbp_[A-Za-z_0-9]+)\s*\(", text)
    return sorted(set(names))


def test_library_exports_all_declared_symbols():
    from cother_b200 import build
    path = build.build_main()
    lib = ctypes.CDLL(path)
    names = declared_functions()
    assert len(names) >= 15
    for n in names:
        assert hasattr(lib, n), n


def test_defaults_and_errors_without_gpu():
    import cother_b200 as cb
    o = cb.Options.defaults()
    assert abs(o.ssswgt - 0.12) < 1e-7 and abs(o.ddmswgt - 0.2) < 1e-7 and o.dstsegm == 6
    lib = cb.load_library()
    # creating a context with an invalid option must fail with a message,
    # never abort the process
    bad = cb.Options.defaults()
    bad.cvswgt = 1.5             # CVSWGT is in [0, 1) (MOptions.cpp)
    h = ctypes.c_void_p()
    import numpy as np
    t = np.zeros((30, 30), np.float32)
    rc = lib.cbp_create(0, ctypes.byref(bad), t.ctypes.data, 0, ctypes.byref(h))
    assert rc != 0
    assert b"CVSWGT" in lib.cbp_last_error()


def test_slab_bytes_is_host_only():
    """The slab planner's charge needs no device: linear in the slab's
    positions, growing with the query length."""
    import cother_b200 as cb
    a, b = cb.slab_bytes(400, 1000), cb.slab_bytes(400, 2000)
    assert 0 < a < b and b - a == cb.slab_bytes(400, 1000) - cb.slab_bytes(400, 0)
    assert cb.slab_bytes(800, 1000) > a

"""The C ABI: the library loads, exports every symbol the headers in include/ declare, and its
parameter block matches the oracle's layout.  No compute call is made here."""
import ctypes
import os
import re

from conftest import ROOT


def _declared(header="acs.h", prefix="acs_"):
    src = open(os.path.join(ROOT, "include", header)).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(" + prefix + r"[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol(pkg):
    L = pkg.lib()
    names = _declared()
    assert len(names) >= 25
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    assert set(pkg.EXPORTED) <= set(names)


def test_library_exports_every_network_kernel(pkg):
    L = pkg.lib()
    names = _declared("unet.h", "unet_")
    assert len(names) >= 15
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    from importlib import import_module
    sig = import_module(pkg.__name__ + ".unet")._SIG
    assert set(sig) == set(names)    # the Python binding declares every kernel

def test_param_block_layout_matches_oracle(pkg, orc):
    a = [(n, t) for n, t in pkg.AcsParams._fields_]
    b = [(n, t) for n, t in orc.OrcParams._fields_]
    assert a == b
    assert ctypes.sizeof(pkg.AcsParams) == ctypes.sizeof(orc.OrcParams)


def test_version_and_errors_without_device(pkg):
    L = pkg.lib()
    assert b"sm_100a" in L.acs_version()
    # invalid arguments are rejected before any device work
    assert L.acs_create(None, None, None) != 0
    assert L.acs_batch_create(None, None, 0, None) != 0
    assert pkg.reference_jmax(51) == 84


def test_static_solve_u_checks_parameters_like_acs_create(pkg):
    """The allocation-free solve_U rejects what acs_create rejects (here: a Darcy number of 0,
    which would put sqrt(eps*Da) = 0 under a division) and the FAST arithmetic it does not
    compute in, before it touches the device (the pointers are never dereferenced)."""
    L = pkg.lib()
    prm, mesh, _, _ = pkg.configs.channel_case(20, 16)
    g = pkg.AcsGrid()
    g.imax, g.jmax = prm.imax, prm.jmax
    dummy = (ctypes.c_double * 1)()
    g.x = g.y = g.xm = g.ym = g.epsilon1 = g.liga_poros = ctypes.cast(dummy, ctypes.POINTER(ctypes.c_double))
    r = ctypes.c_double()
    from dataclasses import replace
    for bad in (replace(prm, Da=0.0), replace(prm, Re=-1.0), replace(prm, itc_max=1),
                replace(prm, continuity=3), replace(prm, arith=pkg.ARITH_FAST)):
        p = bad.struct()
        code = L.acs_solve_u_static(ctypes.byref(p), ctypes.byref(g), 1, 1, 1, 1, 1, ctypes.byref(r), None)
        assert code == pkg.ACS_E_ARG, (bad, code)

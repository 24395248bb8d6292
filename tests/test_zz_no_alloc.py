"""acs_solve_u_static, the allocation-free solve_U, against the handle-based acs_solve_u.

Some callers cannot allocate device memory: their device memory belongs to another allocator,
or they must not allocate once they are running.  acs_solve_u_static serves them from a fixed
static scratch array inside the library; the caller passes device inputs and outputs only.  This
test allocates those inputs and outputs itself (with torch) and checks, on two calls in a row,
that the residual and every output array are bit-identical to acs_solve_u on the same inputs
(the tolerance of the EXACT-arithmetic parity tests).  The file sorts last so a run that stops
at the first failure has run every other test before it.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import mask_dead

pytestmark = pytest.mark.gpu


def _dev(torch, a):
    return torch.from_numpy(np.asarray(a, np.float64).ravel(order="F").copy()).cuda()


def _host(t, shape):
    return t.cpu().numpy().reshape(shape, order="F")


def _cases(pkg):
    cfg = pkg.configs
    prm, mesh, _, _, _ = cfg.reference_case(23)
    yield "reference", prm, mesh
    prm, mesh, _, _ = cfg.channel_case(37, 26, scheme=pkg.SCHEME_QUICK, block=cfg.centred_block(2, 1, 0.3),
                                       porosity=0.4, Da=1e-3, Cf=0.55, Ri=1.0, scalars=True)
    yield "channel", prm, mesh


def _compare_calls(pkg, torch, name, prm, mesh, rng, calls):
    """`calls` calls of the allocation-free solve_U, each compared with acs_solve_u."""
    L = pkg.lib()
    nx, ny = prm.imax, prm.jmax
    handle = pkg.Case(prm, mesh)
    # grid on the device, in the acs_grid layout
    keep = [_dev(torch, mesh[k]) for k in ("x", "y", "xm", "ym", "eps", "liga")]
    g = pkg.AcsGrid()
    g.imax, g.jmax = nx, ny
    ptrs = [C.cast(C.c_void_p(t.data_ptr()), C.POINTER(C.c_double)) for t in keep]
    g.x, g.y, g.xm, g.ym, g.epsilon1, g.liga_poros = ptrs
    p = prm.struct()
    for call in range(calls):
        um = np.asfortranarray(rng.uniform(-1, 1, (nx + 1, ny)))
        um_tau = np.asfortranarray(rng.uniform(-1, 1, (nx + 1, ny)))
        vm_tau = np.asfortranarray(rng.uniform(-1, 1, (nx, ny + 1)))
        pn = np.asfortranarray(rng.uniform(-2, 2, (nx, ny)))
        # existing entry point (host arrays, handle)
        vt_h = vm_tau.copy(order="F")
        un_h = np.zeros((nx + 1, ny), order="F")
        res_h = handle.solve_U(um, None, None, um_tau, vt_h, un_h, pn)
        # allocation-free entry point (device arrays allocated here by the caller)
        d_um, d_ut, d_vt, d_pn = (_dev(torch, a) for a in (um, um_tau, vm_tau, pn))
        d_un = torch.zeros((nx + 1) * ny, dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        res_s = C.c_double(-1.0)
        code = L.acs_solve_u_static(C.byref(p), C.byref(g), d_um.data_ptr(), d_ut.data_ptr(), d_vt.data_ptr(),
                                    d_pn.data_ptr(), d_un.data_ptr(), C.byref(res_s), None)
        assert code == 0, L.acs_last_error().decode()
        assert res_s.value == res_h, (name, call, res_s.value, res_h)
        un_s = _host(d_un, (nx + 1, ny))
        vt_s = _host(d_vt, (nx, ny + 1))
        assert np.array_equal(un_s, un_h), (name, call)
        assert np.array_equal(mask_dead("vm_tau", vt_s, prm.bc), mask_dead("vm_tau", vt_h, prm.bc)), (name, call)
    handle.close()


@pytest.mark.parametrize("which", [0, 1])
def test_static_solve_u_matches_handle(gpu, which):
    import torch
    name, prm, mesh = list(_cases(gpu))[which]
    # two calls in a row share the static scratch
    _compare_calls(gpu, torch, name, prm, mesh, np.random.default_rng(100 + which), 2)


def test_static_solve_u_large_then_small(gpu):
    """A smaller case right after a larger one: nothing the larger call left in the shared
    scratch (padding, rows past jmax) may reach the smaller call's result."""
    import torch
    cases = list(_cases(gpu))
    big, small = sorted(cases, key=lambda c: -(c[1].imax + 1) * (c[1].jmax + 1))
    rng = np.random.default_rng(7)
    _compare_calls(gpu, torch, *big, rng, 1)
    _compare_calls(gpu, torch, *small, rng, 1)


def test_static_solve_u_rejects_oversize(gpu):
    pkg = gpu
    L = pkg.lib()
    prm, mesh, _, _ = pkg.configs.channel_case(300, 300)
    g = pkg.AcsGrid()
    g.imax = g.jmax = 300
    dummy = (C.c_double * 1)()
    g.x = g.y = g.xm = g.ym = g.epsilon1 = g.liga_poros = C.cast(dummy, C.POINTER(C.c_double))
    p = prm.struct()
    r = C.c_double()
    code = L.acs_solve_u_static(C.byref(p), C.byref(g), 1, 1, 1, 1, 1, C.byref(r), None)
    assert code == pkg.ACS_E_SIZE
    assert b"static scratch" in L.acs_last_error()

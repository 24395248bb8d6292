"""The product's host helpers (mesh, noise, case builders) against the oracle's restatement."""
import numpy as np
import pytest


@pytest.mark.parametrize("imax", [10, 12, 26, 51, 102])
def test_reference_mesh_bit_exact(pkg, orc, imax):
    a, b = pkg.mesh_reference(imax), orc.mesh_reference(imax)
    assert (a["nx"], a["ny"]) == (b["nx"], b["ny"])
    for k in ("x", "y", "xm", "ym", "flag", "eps", "liga"):
        assert np.array_equal(a[k], b[k]), k


@pytest.mark.parametrize("nx,ny,block", [
    (51, 51, None), (102, 102, (0.45, 1.55, 0.226, 0.774)), (37, 23, (0.0, 0.7, 0.3, 1.0)),
    (64, 40, (1.3, 2.0, 0.0, 0.4))])
def test_channel_mesh_bit_exact(pkg, orc, nx, ny, block):
    a = pkg.mesh_channel(nx, ny, 2.0, 1.0, 1.5, block, 0.4)
    b = orc.mesh_channel(nx, ny, 2.0, 1.0, 1.5, block, 0.4)
    for k in ("x", "y", "xm", "ym", "flag", "eps", "liga"):
        assert np.array_equal(a[k], b[k]), k
    # tanh clustering toward the walls: the first and last y spacings are the smallest
    dy = np.diff(a["y"])
    assert dy[0] <= dy.min() * (1 + 1e-12) and dy[-1] < dy[len(dy) // 2]


def test_noise_bit_exact(pkg, orc):
    for args in [(0, 0, 1, 0), (1, 7, 2, 12345), (2**40, 255, 100, 3)]:
        a = pkg.noise(*args, 1e-3)
        assert a == orc.noise(*args, 1e-3)
        assert -1e-3 <= a < 1e-3


def test_block_area_and_batch_parameters(pkg):
    cfg = pkg.configs
    b = cfg.centred_block(2.0, 1.0, 0.3)
    assert abs((b[1] - b[0]) * (b[3] - b[2]) - 0.6) < 1e-12
    seen = set()
    for c in range(64):
        q = cfg.batch_case_params(c, 0)
        assert q["nx"] in (51, 102, 153, 204) and q["ny"] in (51, 102, 153, 204)
        assert 50 <= q["Re"] <= 500 and 1e-5 <= q["Da"] <= 1e-2
        assert 0.3 <= q["porosity"] <= 0.9 and 0 <= q["Ri"] <= 2
        x0, x1, y0, y1 = q["block"]
        assert x0 >= -1e-12 and x1 <= 2 + 1e-12 and y0 >= -1e-12 and y1 <= 1 + 1e-12
        seen.add((q["nx"], q["ny"]))
    assert len(seen) > 8


def test_reference_case_setup(pkg):
    prm, mesh, st, itc, n = pkg.configs.reference_case(51)
    assert (prm.imax, prm.jmax, itc, n) == (51, 84, 1, 200)
    assert prm.beta == 1300.0 and prm.dtau == 0.05 and prm.dt == 0.005 and prm.eps == 1e-4
    assert (st["vm"] == 5e-4).all() and (st["p"] == 1.0).all() and (st["pn"] == 0).all()
    assert (st["T_tau"] == 0).all() and (st["C"][mesh["flag"] != 0] == 1.0).all()


def test_channel_noise_only_on_update_region(pkg):
    prm, mesh, st, itc, n = pkg.configs.cfg_plain()
    um, vm = st["um"], st["vm"]
    assert (um[:2, :] == 0).all() and (um[-2:, :] == 0).all() and (um[:, 0] == 0).all()
    assert (vm[:, :2] == 0).all() and (vm[0, :] == 0).all()
    assert 0 < np.abs(um).max() <= 1e-3 and 0 < np.abs(vm).max() <= 1e-3
    assert n == 200 and prm.beta == 1.0 and prm.eps == 1e-6 and prm.continuity == 1


def test_noise_array_matches_scalar_and_oracle(pkg, orc):
    import numpy as np
    idx = np.array([0, 1, 5, 1000, 2**33 + 7], dtype=np.uint64)
    a = pkg.noise_array(3, 9, 2, idx, 1e-3)
    for k, i in enumerate(idx):
        assert a[k] == pkg.noise(3, 9, 2, int(i), 1e-3) == orc.noise(3, 9, 2, int(i), 1e-3)


def test_channel_noise_matches_oracle_generator(pkg, orc):
    """The vectorised initial condition equals element-wise calls of the oracle's generator."""
    prm, mesh, st, itc = pkg.configs.channel_case(13, 11, seed=4, case_id=2)
    nx, ny = 13, 11
    for j in range(2, ny):
        for i in range(3, nx):
            assert st["um"][i - 1, j - 1] == orc.noise(4, 2, 1, (i - 1) + (j - 1) * (nx + 1), 1e-3)
    for j in range(3, ny):
        for i in range(2, nx):
            assert st["vm"][i - 1, j - 1] == orc.noise(4, 2, 2, (i - 1) + (j - 1) * nx, 1e-3)


def test_oracle_generators_build_identical_cases(pkg, orc):
    """The case builders with the oracle's mesh and noise generators (what a run that must not
    load the package's library uses) give the same cases bit for bit as with the package's own."""
    a, _ = pkg.configs.cfg_batch(3, seed=101, sizes=(31, 45), arith=pkg.ARITH_FAST)
    pkg.configs.use_backend(orc)
    try:
        b, _ = pkg.configs.cfg_batch(3, seed=101, sizes=(31, 45), arith=pkg.ARITH_FAST)
    finally:
        pkg.configs.use_backend(None)
    for (p1, m1, s1, i1), (p2, m2, s2, i2) in zip(a, b):
        assert p1 == p2 and i1 == i2
        for k in m1:
            assert np.array_equal(np.asarray(m1[k]), np.asarray(m2[k])), k
        for k in s1:
            assert np.array_equal(s1[k], s2[k]), k


@pytest.mark.gpu
@pytest.mark.parametrize("geom", [(37, 26, 1.5, 1), (153, 153, 1.5, 1), (64, 31, 0.0, 2), (20, 45, 1.5, 0)])
def test_device_channel_mesh_equals_host(gpu, geom):
    """acs_mesh_channel_device (porous flag, its dilation sweeps, epsilon1 and liga on the device)
    equals acs_mesh_channel bit for bit: one box, two boxes, none, stretched and uniform y."""
    import ctypes as C
    import torch
    pkg = gpu
    nx, ny, s, nbox = geom
    cfg = pkg.configs
    boxes = [cfg.centred_block(2.0, 1.0, 0.3), (0.1, 0.6, 0.2, 0.55)][:nbox] if nbox else []
    host = pkg.mesh_channel(nx, ny, 2.0, 1.0, s, boxes[0] if nbox > 0 else None, 0.45,
                            boxes[1] if nbox > 1 else None)
    dev = {k: torch.zeros(n, dtype=torch.float64, device="cuda")
           for k, n in (("x", nx), ("y", ny), ("xm", nx + 1), ("ym", ny + 1), ("eps", nx * ny), ("liga", nx * ny))}
    flag = torch.zeros(nx * ny, dtype=torch.int32, device="cuda")
    b = [np.array(bx, float) for bx in boxes] + [None] * (2 - len(boxes))
    ptr = lambda a: a.ctypes.data_as(C.POINTER(C.c_double)) if a is not None else None
    code = pkg.lib().acs_mesh_channel_device(nx, ny, 2.0, 1.0, s, ptr(b[0]), ptr(b[1]), 0.45,
                                             *(dev[k].data_ptr() for k in ("x", "y", "xm", "ym")),
                                             flag.data_ptr(), dev["eps"].data_ptr(), dev["liga"].data_ptr(), None)
    assert code == 0, pkg.lib().acs_last_error()
    for k in ("x", "y", "xm", "ym"):
        assert np.array_equal(dev[k].cpu().numpy(), host[k]), k
    assert np.array_equal(flag.cpu().numpy().reshape((nx, ny), order="F"), host["flag"])
    for k in ("eps", "liga"):
        assert np.array_equal(dev[k].cpu().numpy().reshape((nx, ny), order="F"), host[k]), k
    assert (host["flag"] == 3).any() == (nbox > 0)


@pytest.mark.gpu
def test_case_created_from_device_grid_runs_like_host_grid(gpu):
    """acs_create given a grid whose arrays are the device arrays of acs_mesh_channel_device runs
    the same two physical steps as the case created from the host mesh, bit for bit."""
    import ctypes as C
    import torch
    pkg = gpu
    params, mesh, state, itc = pkg.configs.channel_case(40, 30, seed=5, Re=150.0, block=pkg.configs.centred_block(2.0, 1.0, 0.3),
                                                        porosity=0.45, Da=1e-3, Cf=0.55, Ri=1.0, scalars=True)
    nx, ny = params.imax, params.jmax
    box = np.array(pkg.configs.centred_block(2.0, 1.0, 0.3), float)
    dev = {k: torch.zeros(n, dtype=torch.float64, device="cuda")
           for k, n in (("x", nx), ("y", ny), ("xm", nx + 1), ("ym", ny + 1), ("eps", nx * ny), ("liga", nx * ny))}
    flag = torch.zeros(nx * ny, dtype=torch.int32, device="cuda")
    L = pkg.lib()
    code = L.acs_mesh_channel_device(nx, ny, 2.0, 1.0, 1.5, box.ctypes.data_as(C.POINTER(C.c_double)), None, 0.45,
                                     *(dev[k].data_ptr() for k in ("x", "y", "xm", "ym")), flag.data_ptr(),
                                     dev["eps"].data_ptr(), dev["liga"].data_ptr(), None)
    assert code == 0, L.acs_last_error()
    assert np.array_equal(dev["eps"].cpu().numpy().reshape((nx, ny), order="F"), mesh["eps"])
    g = pkg.AcsGrid()
    g.imax, g.jmax = nx, ny
    D = C.POINTER(C.c_double)
    g.x, g.y, g.xm, g.ym, g.epsilon1, g.liga_poros = [C.cast(C.c_void_p(dev[k].data_ptr()), D)
                                                      for k in ("x", "y", "xm", "ym", "eps", "liga")]
    p = params.struct()
    h = C.c_void_p()
    assert L.acs_create(C.byref(g), C.byref(p), C.byref(h)) == 0, L.acs_last_error()
    a = pkg.Case.__new__(pkg.Case)
    a.params, a.nx, a.ny, a._keep, a._p, a.h = params, nx, ny, [], p, h
    b = pkg.Case(params, mesh)
    out = []
    for c in (a, b):
        c.set_state(state)
        out.append((c.physical_steps(2, itc)[:2], c.get_state()))
        c.close()
    assert np.array_equal(out[0][0][1], out[1][0][1])
    for k in out[0][1]:
        assert np.array_equal(out[0][1][k], out[1][1][k]), k

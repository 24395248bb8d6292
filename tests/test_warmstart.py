"""Learned warm start: the device hooks against host restatements, and the ablation.

* a plain-policy start leaves the loop bit-identical to a run without the hooks;
* the feature canvas holds the downloaded fields and increments at their staggered pixels;
* the extrapolated start is fields + increment (or the quadratic through the last three step
  starts) with the oracle's boundary passes, bit for bit;
* the initial residuals are the oracle's stage-1 momentum and pressure residual maxima;
* ablation: a network trained on snapshots of eight cases starts two held-out cases; the
  pseudo-iterations per step are compared with the plain start (the method without the
  network) and with the extrapolated start, and the final fields with the plain run's.
"""
import numpy as np
import pytest

from conftest import mask_dead

pytestmark = pytest.mark.gpu

NX = NY = 24


@pytest.fixture(scope="module")
def ws_mod(gpu):
    import importlib
    return importlib.import_module("solver_cfd_b200.warmstart")


def _case(pkg, seed=0, case_id=0, nx=NX, ny=NY, Re=200.0, Ri=1.0, por=0.4, itc_max=300000):
    cfg = pkg.configs
    return cfg.channel_case(nx, ny, seed=seed, case_id=case_id, Re=Re, scheme=pkg.SCHEME_QUICK,
                            block=cfg.centred_block(2.0, 1.0, 0.3), porosity=por, Da=1e-3, Cf=0.55, Ri=Ri,
                            scalars=True, itc_max=itc_max)


def _batch(pkg, cases):
    b = pkg.Batch([c[0] for c in cases], [c[1] for c in cases])
    for k, c in enumerate(cases):
        b.set_state(k, c[2])
    return b


def test_plain_policy_is_bit_identical(gpu, ws_mod):
    import torch
    pkg = gpu
    cases = [_case(pkg, case_id=k) for k in range(2)]
    a = _batch(pkg, cases)
    a.set_stream(torch.cuda.current_stream().cuda_stream)
    b = _batch(pkg, cases)
    w = ws_mod.WarmStart(b, 32, 32)
    itc_a = itc_b = np.ones(2, np.int32)
    for _ in range(4):
        itc_a, ia, _, _ = a.run(1, itc_a)
        w.features()
        chosen, res0 = b.set_start(None, 8, None, pkg.POLICY_PLAIN)
        assert not chosen.any()
        itc_b, ib, _, _ = b.run(1, itc_b)
        assert np.array_equal(ia, ib)
    for c in range(2):
        sa, sb = a.get_state(c), b.get_state(c)
        for k in sa:
            assert np.array_equal(mask_dead(k, sa[k], 1), mask_dead(k, sb[k], 1)), k


def _download_canvas(t, n, H, W, ch):
    return t.cpu().numpy().reshape(n, H, W, ch)


def test_features_and_extrapolated_start(gpu, orc, ws_mod):
    pkg = gpu
    prm, mesh, st, itc = _case(pkg)
    b = _batch(pkg, [(prm, mesh, st)])
    H, W = 32, 32
    w = ws_mod.WarmStart(b, H, W)
    itc = np.ones(1, np.int32)
    w.features()
    itc, _, _, _ = b.run(1, itc)
    prev = b.get_state(0)
    w.features()
    itc, _, _, _ = b.run(1, itc)
    cur = b.get_state(0)
    X = _download_canvas(w.features(), 1, H, W, 11)[0]
    scale = w.inc_scale.cpu().numpy()
    nx, ny = NX, NY
    for f, name, (sw, sh) in ((0, "um", (nx + 1, ny)), (1, "vm", (nx, ny + 1)), (2, "pn", (nx, ny)),
                              (3, "T", (nx, ny)), (4, "C", (nx, ny))):
        # pressure: the buffer the momentum routines read (the reference's pn)
        val = cur[name].T.astype(np.float32)
        d = cur[name] - prev[name]
        s_ref = np.sqrt(np.mean(d * d))
        s_ref = s_ref if s_ref > 0 else 1.0
        assert abs(scale[f] - s_ref) <= 1e-6 * s_ref, (name, scale[f], s_ref)
        assert np.array_equal(X[:sh, :sw, f], val), name
        assert np.allclose(X[:sh, :sw, 6 + f], (d / s_ref).T, rtol=1e-6, atol=1e-30), name
        assert not X[sh:, :, f].any() and not X[:, sw:, f].any()
    assert np.array_equal(X[:ny, :nx, 5], mesh["liga"].T.astype(np.float32))
    # extrapolated start, forced: fields + increment, then the boundary passes
    chosen, res0 = b.set_start(None, 8, None, pkg.POLICY_PREDICTED)
    assert chosen[0] == 1
    got = b.get_state(0)
    oc = orc.OracleCase(prm, mesh)
    ut = np.asfortranarray(cur["um"] + (cur["um"] - prev["um"]))
    vt = np.asfortranarray(cur["vm"] + (cur["vm"] - prev["vm"]))
    oc.bc_uv(ut, vt)
    pp = np.asfortranarray(cur["pn"] + (cur["pn"] - prev["pn"]))
    oc.bc_p(pp)
    Tt = np.asfortranarray(cur["T"] + (cur["T"] - prev["T"]))
    oc.bc_z(Tt)
    Ct = np.asfortranarray(cur["C"] + (cur["C"] - prev["C"]))
    oc.bc_c(Ct)
    assert np.array_equal(got["um_tau"], ut)
    assert np.array_equal(mask_dead("vm", got["vm_tau"], 1), mask_dead("vm", vt, 1))
    assert np.array_equal(got["p"], pp) and np.array_equal(got["pn"], pp)
    assert np.array_equal(got["T_tau"], Tt) and np.array_equal(got["C_tau"], Ct)
    # initial residual of the predicted start against the oracle's residual routines
    r_ref = _initial_residual(oc, prm, mesh, cur, ut, vt, pp)
    assert abs(res0[0, 1] - r_ref) <= 1e-13 * r_ref, (res0[0, 1], r_ref)
    r_plain = _initial_residual(oc, prm, mesh, cur, cur["um_tau"], cur["vm_tau"], cur["pn"])
    assert abs(res0[0, 0] - r_plain) <= 1e-13 * r_plain, (res0[0, 0], r_plain)
    assert np.isnan(res0[0, 2])


def _expected_start(oc, ut, vt, pp, Tt, Ct):
    ut, vt, pp, Tt, Ct = (np.asfortranarray(a) for a in (ut, vt, pp, Tt, Ct))
    oc.bc_uv(ut, vt)
    oc.bc_p(pp)
    oc.bc_z(Tt)
    oc.bc_c(Ct)
    return ut, vt, pp, Tt, Ct


def _assert_start(got, exp):
    ut, vt, pp, Tt, Ct = exp
    assert np.array_equal(got["um_tau"], ut)
    assert np.array_equal(mask_dead("vm", got["vm_tau"], 1), mask_dead("vm", vt, 1))
    assert np.array_equal(got["p"], pp) and np.array_equal(got["pn"], pp)
    assert np.array_equal(got["T_tau"], Tt) and np.array_equal(got["C_tau"], Ct)


def test_quadratic_extrapolated_start(gpu, orc, ws_mod):
    """ACS_OPT_EXTRAP_ORDER = 2: with two increments (three feature calls) the extrapolated
    candidate is x2 + (2 (x2 - x1) - (x1 - x0)) with the oracle's boundary passes, bit for bit;
    with one increment it is still the linear x1 + (x1 - x0)."""
    pkg = gpu
    prm, mesh, st, itc0 = _case(pkg)
    oc = orc.OracleCase(prm, mesh)
    keys = ("um", "vm", "pn", "T", "C")
    # one increment: linear
    b = _batch(pkg, [(prm, mesh, st)])
    b.set_option(pkg.OPT_EXTRAP_ORDER, 2)
    w = ws_mod.WarmStart(b, 32, 32)
    x0 = b.get_state(0)
    w.features()
    itc, _, _, _ = b.run(1, np.ones(1, np.int32))
    x1 = b.get_state(0)
    w.features()
    chosen, _ = b.set_start(None, 8, None, pkg.POLICY_PREDICTED)
    assert chosen[0] == 1
    _assert_start(b.get_state(0), _expected_start(oc, *(x1[k] + (x1[k] - x0[k]) for k in keys)))
    b.close()
    # two increments: quadratic
    b = _batch(pkg, [(prm, mesh, st)])
    b.set_option(pkg.OPT_EXTRAP_ORDER, 2)
    with pytest.raises(pkg.AcsError):
        b.set_option(pkg.OPT_EXTRAP_ORDER, 3)
    w = ws_mod.WarmStart(b, 32, 32)
    w.features()
    itc, _, _, _ = b.run(1, np.ones(1, np.int32))
    w.features()
    itc, _, _, _ = b.run(1, itc)
    x2 = b.get_state(0)
    w.features()
    chosen, res0 = b.set_start(None, 8, None, pkg.POLICY_PREDICTED)
    assert chosen[0] == 1
    exp = _expected_start(oc, *(x2[k] + (2.0 * (x2[k] - x1[k]) - (x1[k] - x0[k])) for k in keys))
    _assert_start(b.get_state(0), exp)
    r_ref = _initial_residual(oc, prm, mesh, x2, exp[0], exp[1], exp[2])
    assert abs(res0[0, 1] - r_ref) <= 1e-13 * r_ref, (res0[0, 1], r_ref)
    _, it, _, status = b.run(1, itc)
    assert status[0] == pkg.CASE_DONE and it[0, 0] >= 1
    b.close()


def _initial_residual(oc, prm, mesh, cur, ut, vt, pn):
    """max of |dtau ((u - u_tau) + RESU dt)| (U interior), the same for V, and |dtau RP beta|."""
    nx, ny = prm.imax, prm.jmax
    RU = oc.resu(ut, vt, pn)
    RV = oc.resv(ut, vt, pn, cur["T"])
    ru = np.abs(((cur["um"] - ut) + RU * prm.dt) * prm.dtau)[2:nx - 1, 1:ny - 1].max()
    rv = np.abs(((cur["vm"] - vt) + RV * prm.dt) * prm.dtau)[1:nx - 1, 2:ny - 1].max()
    xm, ym = mesh["xm"], mesh["ym"]   # 0-based: xm[k] is the reference's xm(k+1)
    i = np.arange(2, nx)[:, None]     # the reference's 1-based i = 2..nx-1
    j = np.arange(2, ny)[None, :]
    Aew = ym[j] - ym[j - 1]
    Ans = xm[i] - xm[i - 1]
    dudx = ut[i, j - 1] * Aew - ut[i - 1, j - 1] * Aew
    dvdy = vt[i - 1, j] * Ans - vt[i - 1, j - 1] * Ans
    RP = -(dudx + dvdy)
    if prm.continuity == 1:
        RP = RP / (Aew * Ans)
    rp = np.abs(prm.dtau * RP * prm.beta).max()
    return max(ru, rv, rp)


def test_warm_start_ablation(gpu, ws_mod, capsys):
    pkg = gpu
    from solver_cfd_b200.unet import UNet
    H = W = 32
    Re = [150.0, 200.0, 250.0, 300.0, 180.0, 270.0, 220.0, 160.0, 280.0, 240.0]
    Ri = [0.5, 1.0, 1.5, 0.8, 1.2, 0.6, 1.1, 0.9, 1.4, 0.7]
    cases = [_case(pkg, seed=3, case_id=k, Re=Re[k], Ri=Ri[k]) for k in range(10)]
    train_cases, test_cases = cases[:8], cases[8:]
    # snapshots from the solver itself (extrapolated start; the loop iterates to tolerance)
    b = _batch(pkg, train_cases)
    X, T, Wt, it_gen = ws_mod.generate(b, H, W, 24, 1, skip=2)
    b.close()
    norm = ws_mod.Normalizer.from_samples(X.cpu().numpy().reshape(-1, H, W, 11),
                                          T.cpu().numpy().reshape(-1, H, W, 8), Wt.cpu().numpy().reshape(-1, H, W, 8))
    net = UNet(11, 5, 32, 4, seed=0)
    losses = ws_mod.train(net, X, T, Wt, H, W, norm, epochs=300, batch=8, lr=1e-3)
    assert losses[-1] < 0.2 * losses[0], losses[::50]

    def make():
        return _batch(pkg, test_cases)

    steps = 14
    out = ws_mod.evaluate(make, H, W, steps, 1, net, norm)
    tot = {m: int(out[m]["iters"][:, 3:].sum()) for m in out}
    err = [ws_mod.field_error(out["learned"]["fields"][c], out["plain"]["fields"][c]) for c in range(2)]
    kept = out["learned"]["kept"][3:].mean(axis=0)
    with capsys.disabled():
        print("\nwarm start ablation, pseudo-iterations over steps 3..13 of 2 held-out 24x24 cases:", tot,
              "training losses", [round(x, 4) for x in losses[::50]],
              "starts plain/extrap/learned", kept, "final-field error vs plain", err)
    # Against the reference's (plain) start the warm start saves more than half the work.
    assert tot["learned"] < tot["plain"] / 2.0, tot
    # The method without the network is the extrapolated start (the network's head starts at zero,
    # so an untrained network gives exactly that start).  Negative result: the trained network
    # does not reliably beat it.  Its start has the smallest initial residual on most steps, but
    # the pseudo-iteration count over these steps was below the extrapolated start's in 2 of 7
    # training runs (26,019 and 72,275 against 72,625) and above it in 5 (73,162 to 119,959): the
    # count depends on smooth start errors that the max-norm residual barely sees, and training is
    # not bit-reproducible (the split-K gradient sums are not ordered).  Printed above, not asserted.
    assert kept[2] >= 0.5, kept
    # the loop iterates to the same tolerance from either start: velocities and scalars agree with
    # the plain run to 1e-4; the pressure, which converges slowest in pseudo time, to 1e-2 (observed
    # 8.7e-5 .. 8.3e-4 over training runs)
    for e in err:
        assert max(e["um"], e["vm"], e["T"], e["C"]) < 1e-4, e
        assert e["pn"] < 1e-2, e


def test_final_fields_against_tightly_converged_run(gpu, ws_mod, capsys):
    """How far runs at residual 1e-6 end from the converged solution: the plain and the
    extrapolated-start runs of two 24 x 24 cases, 10 physical steps each, against the same cases
    iterated to residual 1e-10 with the plain start, and the extrapolated start again with its
    warm-started steps iterated to 1e-7 (the warm-tolerance policy)."""
    pkg = gpu
    from dataclasses import replace
    cases = [_case(pkg, seed=3, case_id=k, Re=[280.0, 240.0][k], Ri=[1.4, 0.7][k], itc_max=2000000)
             for k in range(2)]
    H = W = 32
    steps = 10

    def run(eps, mode, warm_eps=None):
        b = _batch(pkg, [(replace(c[0], eps=eps),) + tuple(c[1:]) for c in cases])
        w = ws_mod.WarmStart(b, H, W)
        itc = np.ones(2, np.int32)
        total = 0
        for _ in range(steps):
            itc, it, _, _ = w.step(itc, mode, warm_eps=warm_eps)
            total += int(it.sum())
        out = [b.get_state(c, ("um", "vm", "pn", "T", "C")) for c in range(2)]
        b.close()
        return out, total

    ref, n_ref = run(1e-10, "plain")
    runs = {"plain 1e-6": run(1e-6, "plain"), "extrap 1e-6": run(1e-6, "extrap"),
            "extrap 1e-7": run(1e-6, "extrap", warm_eps=1e-7)}
    err = {name: {k: max(ws_mod.field_error(o[c], ref[c])[k] for c in range(2)) for k in ("um", "vm", "pn", "T", "C")}
           for name, (o, _) in runs.items()}
    with capsys.disabled():
        print(f"\nfinal fields after {steps} steps against the run converged to 1e-10 ({n_ref} pseudo-iterations),"
              " relative max-norm difference:")
        for name, e in err.items():
            print(f"   {name} ({runs[name][1]} pseudo-iterations)", {k: f"{v:.2e}" for k, v in e.items()})
    worst = {name: max(e.values()) for name, e in err.items()}
    # every run at 1e-6 ends close to the converged solution; the extrapolated start's error is of
    # the order of the plain run's own, and a tighter tolerance on its warm-started steps reduces it
    for name, w in worst.items():
        assert w < 1e-2, (name, err[name])
    assert worst["extrap 1e-6"] < 10.0 * worst["plain 1e-6"], err
    assert worst["extrap 1e-7"] < worst["extrap 1e-6"], err
    assert runs["extrap 1e-6"][1] < runs["plain 1e-6"][1], {k: v[1] for k, v in runs.items()}

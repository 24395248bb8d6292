"""CUDA path (EXACT arithmetic) against the CPU oracle, bit for bit, through the C ABI."""
import os

import numpy as np
import pytest

from conftest import GOLDEN, fcopy, mask_dead

pytestmark = pytest.mark.gpu


def _rand_state(pkg, nx, ny, seed):
    rng = np.random.default_rng(seed)
    st = pkg.configs.zero_state(nx, ny)
    for k, a in st.items():
        if k.startswith("T"):
            a[:] = rng.uniform(0.5, 1.5, a.shape)
        elif k.startswith("C"):
            a[:] = rng.uniform(0.0, 1.0, a.shape)
        elif k.startswith("p"):
            a[:] = rng.uniform(-2.0, 2.0, a.shape)
        else:
            a[:] = rng.uniform(-1.0, 1.0, a.shape)
    return st


def _cases(pkg):
    cfg = pkg.configs
    out = []
    prm, mesh, _, _, _ = cfg.reference_case(12)
    out.append(("reference-12", prm, mesh))
    prm, mesh, _, _, _ = cfg.reference_case(23, b_art=0.3)
    out.append(("reference-23-bart", prm, mesh))
    prm, mesh, _, _ = cfg.channel_case(33, 21, scheme=pkg.SCHEME_QUICK, block=cfg.centred_block(2, 1, 0.3),
                                       porosity=0.4, Da=1e-3, Cf=0.55, Ri=1.0, scalars=True)
    out.append(("channel-quick-porous", prm, mesh))
    prm, mesh, _, _ = cfg.channel_case(29, 17, scheme=pkg.SCHEME_UPWIND, continuity=0)
    out.append(("channel-upwind", prm, mesh))
    return out


@pytest.mark.parametrize("which", range(4))
def test_routines_bit_exact(gpu, orc, which):
    """solve_U/V/P/Z/C on random fields: every output array and residual bit-identical."""
    pkg = gpu
    name, prm, mesh = _cases(pkg)[which]
    nx, ny = prm.imax, prm.jmax
    g = pkg.Case(prm, mesh)
    o = orc.OracleCase(prm, mesh)
    for rep in range(2):
        s = _rand_state(pkg, nx, ny, 10 * which + rep)
        a, b = fcopy(s), fcopy(s)
        ru_g = g.solve_U(a["um"], a["vm"], None, a["um_tau"], a["vm_tau"], a["um_n_tau"], a["pn"])
        ru_o = o.solve_u(b["um"], b["um_tau"], b["vm_tau"], b["pn"], b["um_n_tau"])
        rv_g = g.solve_V(a["um"], a["vm"], None, a["um_tau"], a["vm_tau"], a["vm_n_tau"], a["pn"], a["T"])
        rv_o = o.solve_v(b["vm"], b["um_tau"], b["vm_tau"], b["pn"], b["T"], b["vm_n_tau"])
        rp_g = g.solve_P(a["p"], a["um_n_tau"], a["vm_n_tau"], a["pn"])
        rp_o = o.solve_p(b["p"], b["um_n_tau"], b["vm_n_tau"], b["pn"])
        g.solve_Z(a["um_n_tau"], a["vm_n_tau"], a["T"], a["T_n_tau"], a["T_tau"])
        o.solve_z(b["um_n_tau"], b["vm_n_tau"], b["T"], b["T_n_tau"], b["T_tau"])
        g.solve_C(a["um_n_tau"], a["vm_n_tau"], a["C"], a["C_n_tau"], a["C_tau"])
        o.solve_c(b["um_n_tau"], b["vm_n_tau"], b["C"], b["C_n_tau"], b["C_tau"])
        assert (ru_g, rv_g, rp_g) == (ru_o, rv_o, rp_o), name
        for k in ("um_n_tau", "vm_tau", "vm_n_tau", "um_tau", "pn", "T_n_tau", "C_n_tau"):
            x, y = mask_dead(k, a[k], prm.bc), mask_dead(k, b[k], prm.bc)
            assert np.array_equal(x, y), (name, k, float(np.nanmax(np.abs(x - y))))


ENGINES = pytest.mark.parametrize("engine", [0, 1], ids=["cluster", "graph"])


def _loop_compare(pkg, orc, prm, mesh, st, itc, nsteps, engine=0, nodes_per_cta=None):
    g = pkg.Case(prm, mesh)
    g.set_option(pkg.OPT_ENGINE, engine)
    if nodes_per_cta:
        g.set_option(pkg.OPT_NODES_PER_CTA, nodes_per_cta)
    g.set_state(st)
    itc_g, it_g, er_g, status = g.physical_steps(nsteps, itc)
    out = g.get_state()
    ost = fcopy(st)
    itc_o, it_o, er_o = orc.OracleCase(prm, mesh).run(ost, nsteps, itc)
    assert status == pkg.CASE_DONE
    assert list(it_g) == list(it_o) and itc_g == itc_o
    assert np.array_equal(er_g, er_o)
    for k in pkg.FIELDS:
        x, y = mask_dead(k, out[k], prm.bc), mask_dead(k, ost[k], prm.bc)
        assert np.array_equal(x, y), (k, float(np.abs(x - y).max()))
    assert g.launch_count() > 0
    return it_g


@ENGINES
def test_loop_reference_small(gpu, orc, engine):
    prm, mesh, st, itc, _ = gpu.configs.reference_case(12, itc_max=5000)
    it = _loop_compare(gpu, orc, prm, mesh, st, itc, 6, engine)
    assert it[0] >= 2


@ENGINES
def test_loop_channel_plain(gpu, orc, engine):
    """cfg-plain shape (51 x 51, upwind, beta=1) with the pseudo loop capped at 1500 per step."""
    prm, mesh, st, itc, _ = gpu.configs.cfg_plain(itc_max=1500)
    _loop_compare(gpu, orc, prm, mesh, st, itc, 2, engine)


@ENGINES
def test_loop_channel_full_physics(gpu, orc, engine):
    """QUICK, porous block, buoyancy, both scalars; 2 steps of a 40 x 30 channel."""
    cfg = gpu.configs
    prm, mesh, st, itc = cfg.channel_case(40, 30, seed=3, Re=200.0, scheme=gpu.SCHEME_QUICK,
                                          block=cfg.centred_block(2, 1, 0.3), porosity=0.4, Da=1e-3,
                                          Cf=0.55, Ri=1.0, scalars=True, itc_max=1200)
    _loop_compare(gpu, orc, prm, mesh, st, itc, 2, engine)


@pytest.mark.parametrize("nodes_per_cta", [64, 300, 100000])
def test_cluster_sizes_bit_exact(gpu, orc, nodes_per_cta):
    """The engine's result does not depend on how a case is split into strips (1..16 CTAs)."""
    cfg = gpu.configs
    prm, mesh, st, itc = cfg.channel_case(37, 70, seed=5, Re=150.0, scheme=gpu.SCHEME_QUICK,
                                          block=cfg.centred_block(2, 1, 0.3), porosity=0.5, Da=1e-2,
                                          Cf=0.55, Ri=0.5, scalars=True, itc_max=500)
    _loop_compare(gpu, orc, prm, mesh, st, itc, 2, 0, nodes_per_cta)


def test_per_case_cluster_sizes_bit_exact(gpu):
    """acs_batch_set_cluster_size changes how cases are split into CTAs, not the results: a batch
    with per-case cluster sizes (1, 5, 16, and back to the default) equals the default batch."""
    pkg = gpu
    cfg = pkg.configs
    cases = [cfg.channel_case(30 + 6 * k, 40, seed=11, case_id=k, Re=120.0 + 40 * k, scheme=pkg.SCHEME_QUICK,
                              block=cfg.centred_block(2, 1, 0.3), porosity=0.5, Da=1e-2, Cf=0.55, Ri=0.5,
                              scalars=True, itc_max=400) for k in range(4)]

    def run(sizes):
        b = pkg.Batch([c[0] for c in cases], [c[1] for c in cases])
        for k, c in enumerate(cases):
            b.set_state(k, c[2])
            if sizes is not None:
                b.set_cluster_size(k, sizes[k])
        _, it, _, st = b.run(2, np.array([c[3] for c in cases], np.int32))
        out = [b.get_state(k) for k in range(len(cases))]
        b.close()
        return it, st, out

    it0, st0, out0 = run(None)
    it1, st1, out1 = run([1, 5, 16, 0])
    assert np.array_equal(it0, it1) and (st0 == pkg.CASE_DONE).all() and (st1 == pkg.CASE_DONE).all()
    for a, b in zip(out0, out1):
        for k in a:
            assert np.array_equal(a[k], b[k]), k


@ENGINES
def test_per_case_tolerance_bit_exact(gpu, orc, engine):
    """acs_batch_set_tolerance between steps: each case equals an oracle run that switches to the
    same tolerance after the first step (a tighter one, a looser one, an unchanged one)."""
    from dataclasses import replace
    cfg = gpu.configs
    items = [cfg.reference_case(n, itc_max=6000, scheme=s)[:4]
             for n, s in ((12, gpu.SCHEME_QUICK), (14, gpu.SCHEME_UPWIND), (16, gpu.SCHEME_QUICK))]
    new_eps = [items[0][0].eps / 5, items[1][0].eps * 5, items[2][0].eps]
    b = gpu.Batch([x[0] for x in items], [x[1] for x in items])
    b.set_option(gpu.OPT_ENGINE, engine)
    for c, x in enumerate(items):
        b.set_state(c, x[2])
    itc_g, it1, _, _ = b.run(1, [x[3] for x in items])
    for c in range(3):
        b.set_tolerance(c, new_eps[c])
    itc_g, it2, _, st_g = b.run(2, itc_g)
    assert (st_g == gpu.CASE_DONE).all()
    for c, (prm, mesh, st, itc) in enumerate(items):
        ost = fcopy(st)
        itc_o, it_o1, _ = orc.OracleCase(prm, mesh).run(ost, 1, itc)
        itc_o, it_o2, _ = orc.OracleCase(replace(prm, eps=new_eps[c]), mesh).run(ost, 2, itc_o)
        assert list(it1[c]) == list(it_o1) and list(it2[c]) == list(it_o2) and itc_g[c] == itc_o, c
        out = b.get_state(c)
        for k in gpu.FIELDS:
            assert np.array_equal(mask_dead(k, out[k], prm.bc), mask_dead(k, ost[k], prm.bc)), (c, k)
        if c < 2:   # the change is visible: the case's own tolerance gives other counts
            ref = fcopy(st)
            _, it_ref, _ = orc.OracleCase(prm, mesh).run(ref, 3, itc)
            assert (it_ref[1:].sum() < it2[c].sum()) == (new_eps[c] < prm.eps), c
    for bad in (0.0, -1e-6, float("nan"), float("inf")):
        with pytest.raises(gpu.AcsError):
            b.set_tolerance(0, bad)
    with pytest.raises(gpu.AcsError):
        b.set_tolerance(3, 1e-6)
    b.close()


@ENGINES
def test_batch_equals_oracle_per_case(gpu, orc, engine):
    """Ragged batch (sizes, schemes, both boundary variants, converging and capped cases) in one
    graph launch; each case bit-identical to its own oracle run."""
    cfg = gpu.configs
    items = []
    prm, mesh, st, itc, _ = cfg.reference_case(12, itc_max=4000)
    items.append((prm, mesh, st, itc))
    prm, mesh, st, itc, _ = cfg.reference_case(14, itc_max=4000, scheme=gpu.SCHEME_UPWIND)
    items.append((prm, mesh, st, itc))
    for c in range(4):
        q = cfg.batch_case_params(c, 0, sizes=(17, 24, 31))
        items.append(cfg.channel_case(q["nx"], q["ny"], seed=0, case_id=c, Re=q["Re"], block=q["block"],
                                      porosity=q["porosity"], Da=q["Da"], Cf=0.55, Ri=q["Ri"],
                                      scalars=True, itc_max=700))
    b = gpu.Batch([x[0] for x in items], [x[1] for x in items])
    b.set_option(gpu.OPT_ENGINE, engine)
    for c, x in enumerate(items):
        b.set_state(c, x[2])
    nsteps = 3
    itc_g, it_g, er_g, st_g = b.run(nsteps, [x[3] for x in items])
    assert (st_g == gpu.CASE_DONE).all()
    for c, (prm, mesh, st, itc) in enumerate(items):
        ost = fcopy(st)
        itc_o, it_o, er_o = orc.OracleCase(prm, mesh).run(ost, nsteps, itc)
        assert list(it_g[c]) == list(it_o) and itc_g[c] == itc_o, c
        out = b.get_state(c)
        for k in gpu.FIELDS:
            x, y = mask_dead(k, out[k], prm.bc), mask_dead(k, ost[k], prm.bc)
            assert np.array_equal(x, y), (c, k)
    assert b.launch_count() > 0


def test_failed_case_is_isolated(gpu):
    """A NaN in one case's input marks that case FAILED and leaves the others untouched."""
    cfg = gpu.configs
    prm, mesh, st, itc, _ = cfg.reference_case(12, itc_max=3000)
    good = fcopy(st)
    bad = fcopy(st)
    bad["um_tau"][5, 7] = np.nan
    b = gpu.Batch([prm, prm], [mesh, mesh])
    b.set_state(0, good)
    b.set_state(1, bad)
    itc_g, it_g, er_g, status = b.run(3, [itc, itc])
    assert status[0] == gpu.CASE_DONE and status[1] == gpu.CASE_FAILED
    solo = gpu.Case(prm, mesh)
    solo.set_state(good)
    _, it_s, _, st_s = solo.physical_steps(3, itc)
    assert list(it_s) == list(it_g[0])
    a, c = solo.get_state(), b.get_state(0)
    for k in ("um", "vm", "p"):
        assert np.array_equal(a[k], c[k])


def test_reference_run_51x84_matches_golden(gpu):
    """The reference's default run (51 x 84, 200 steps, ~315k pseudo-iterations) on the GPU
    against the end state written by the reference's OpenMP build."""
    prm, mesh, st, itc, nsteps = gpu.configs.reference_case(51)
    g = gpu.Case(prm, mesh)
    g.set_state(st)
    itc_g, it_g, er_g, status = g.physical_steps(nsteps, itc)
    assert status == gpu.CASE_DONE
    out = g.get_state()
    ref = np.load(os.path.join(GOLDEN, "reference_51x84.npz"))
    for k in ("um", "vm", "p", "T", "C"):
        rel = np.abs(out[k] - ref[k]).max() / np.abs(ref[k]).max()
        assert rel < 1e-12, (k, rel)
    assert int(it_g.sum()) == 314712


def _fast_compare(pkg, orc, prm, mesh, st, itc, nsteps, tol=1e-10, l1=0, nodes_per_cta=None, engine=0):
    from dataclasses import replace
    g = pkg.Case(replace(prm, arith=pkg.ARITH_FAST), mesh)
    g.set_option(pkg.OPT_ENGINE, engine)
    g.set_option(pkg.OPT_L1_LOADS, l1)
    if nodes_per_cta:
        g.set_option(pkg.OPT_NODES_PER_CTA, nodes_per_cta)
    g.set_state(st)
    itc_g, it_g, er_g, status = g.physical_steps(nsteps, itc)
    out = g.get_state()
    ost = fcopy(st)
    itc_o, it_o, er_o = orc.OracleCase(prm, mesh).run(ost, nsteps, itc)
    assert status == pkg.CASE_DONE
    assert list(it_g) == list(it_o), (list(it_g), list(it_o))
    worst = 0.0
    for k in ("um", "vm", "p", "T", "C", "um_tau", "vm_tau", "pn"):
        x, y = mask_dead(k, out[k], prm.bc), mask_dead(k, ost[k], prm.bc)
        rel = float(np.abs(x - y).max() / max(np.abs(y).max(), 1e-300))
        worst = max(worst, rel)
        assert rel < tol, (k, rel)
    return worst


@pytest.mark.parametrize("l1", [0, 1], ids=["l2-loads", "l1-loads"])
def test_fast_engine_reference_case(gpu, orc, l1):
    """FAST arithmetic, converged steps of the reference case: same pseudo-iteration count in
    every step as the oracle and every field within 1e-10 relative max-norm."""
    prm, mesh, st, itc, _ = gpu.configs.reference_case(12, itc_max=20000)
    _fast_compare(gpu, orc, prm, mesh, st, itc, 8, l1=l1, nodes_per_cta=64)


@pytest.mark.parametrize("l1", [0, 1], ids=["l2-loads", "l1-loads"])
def test_fast_engine_channel_full_physics(gpu, orc, l1):
    cfg = gpu.configs
    prm, mesh, st, itc = cfg.channel_case(30, 22, seed=7, Re=120.0, scheme=gpu.SCHEME_QUICK,
                                          block=cfg.centred_block(2, 1, 0.3), porosity=0.45, Da=1e-3,
                                          Cf=0.55, Ri=1.0, scalars=True, eps=1e-5, itc_max=60000)
    _fast_compare(gpu, orc, prm, mesh, st, itc, 3, l1=l1, nodes_per_cta=64)


def test_fast_graph_engine(gpu, orc):
    """FAST arithmetic in the graph engine's per-stage kernels: the reference case and a
    full-physics channel case, same iteration counts as the oracle, fields within 1e-10."""
    prm, mesh, st, itc, _ = gpu.configs.reference_case(12, itc_max=20000)
    _fast_compare(gpu, orc, prm, mesh, st, itc, 8, engine=1)
    cfg = gpu.configs
    prm, mesh, st, itc = cfg.channel_case(30, 22, seed=7, Re=120.0, scheme=gpu.SCHEME_QUICK,
                                          block=cfg.centred_block(2, 1, 0.3), porosity=0.45, Da=1e-3,
                                          Cf=0.55, Ri=1.0, scalars=True, eps=1e-5, itc_max=60000)
    _fast_compare(gpu, orc, prm, mesh, st, itc, 3, engine=1)


@ENGINES
def test_large_case_fast(gpu, orc, engine):
    """The 1024 x 512 case in FAST arithmetic on both engines: capped steps, fields within
    1e-10 of the oracle."""
    prm, mesh, st, itc, _ = gpu.configs.cfg_large(itc_max=25)
    _fast_compare(gpu, orc, prm, mesh, st, itc, 2, engine=engine)


@ENGINES
def test_large_case_bit_exact(gpu, orc, engine):
    """The combined configuration's single 1024 x 512 case (two porous blocks, full scalars),
    the largest grid of the benchmark configurations: two physical steps capped at itc_max = 25
    (so each ends on the itc_max path) on the GPU against the oracle, bit for bit."""
    pkg = gpu
    prm, mesh, st, itc, _ = pkg.configs.cfg_large(itc_max=25)
    g = pkg.Case(prm, mesh)
    g.set_option(pkg.OPT_ENGINE, engine)
    g.set_state(st)
    itc_g, it_g, er_g, status = g.physical_steps(2, itc)
    out = g.get_state()
    ost = fcopy(st)
    itc_o, it_o, er_o = orc.OracleCase(prm, mesh).run(ost, 2, itc)
    assert status == pkg.CASE_DONE
    assert list(it_g) == list(it_o) == [24, 25]   # step 1 starts at itc = 1 (main.f90:77)
    for k in ("um", "vm", "p", "pn", "T", "C", "um_tau", "vm_tau", "T_tau", "C_tau"):
        assert np.array_equal(out[k], ost[k]), k

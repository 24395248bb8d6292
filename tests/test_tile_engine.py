"""The tile engine (TMA-loaded 32 x 32-node tiles, FAST arithmetic) against the CPU oracle.

Every case must take the same number of pseudo-iterations in every physical step as the oracle,
and every field must agree to 1e-10 relative max-norm (the FAST arithmetic's bound; the oracle
follows the reference's operation order).  The geometries are chosen so that tile edges fall
everywhere a boundary pass can be split: overlapping last tiles in x and y, a pitch that is an
exact multiple of the tile, cases smaller than one tile, both boundary variants, QUICK and upwind.
"""
from dataclasses import replace

import numpy as np
import pytest

from conftest import fcopy, mask_dead

pytestmark = pytest.mark.gpu

TILE = 2
TOL = 1e-10


def _rel(x, y):
    return float(np.abs(x - y).max() / max(np.abs(y).max(), 1e-300))


def _compare_case(pkg, prm, out, ost, tol=TOL):
    worst = 0.0
    for k in ("um", "vm", "p", "pn", "T", "C", "um_tau", "vm_tau", "T_tau", "C_tau"):
        x, y = mask_dead(k, out[k], prm.bc), mask_dead(k, ost[k], prm.bc)
        r = _rel(x, y)
        worst = max(worst, r)
        assert r < tol, (k, r)
    return worst


def _tile_vs_oracle(pkg, orc, items, nsteps, tol=TOL):
    fast = [replace(x[0], arith=pkg.ARITH_FAST) for x in items]
    b = pkg.Batch(fast, [x[1] for x in items])
    b.set_option(pkg.OPT_ENGINE, TILE)
    for c, x in enumerate(items):
        b.set_state(c, x[2])
    itc_g, it_g, _, st_g = b.run(nsteps, [x[3] for x in items])
    assert (st_g == pkg.CASE_DONE).all(), st_g
    worst = 0.0
    for c, (prm, mesh, st, itc) in enumerate(items):
        ost = fcopy(st)
        itc_o, it_o, _ = orc.OracleCase(prm, mesh).run(ost, nsteps, itc)
        assert list(it_g[c]) == list(it_o) and itc_g[c] == itc_o, (c, list(it_g[c]), list(it_o))
        worst = max(worst, _compare_case(pkg, prm, b.get_state(c), ost, tol))
    assert b.launch_count() > 0
    b.close()
    return worst


def test_tile_engine_reference_case(gpu, orc):
    """Reference boundary variant (inflow at the bottom), converged steps."""
    prm, mesh, st, itc, _ = gpu.configs.reference_case(12, itc_max=20000)
    w = _tile_vs_oracle(gpu, orc, [(prm, mesh, st, itc)], 8)
    print("max rel diff", w)


def test_tile_engine_channel_full_physics(gpu, orc):
    cfg = gpu.configs
    item = cfg.channel_case(30, 22, seed=7, Re=120.0, scheme=gpu.SCHEME_QUICK, block=cfg.centred_block(2, 1, 0.3),
                            porosity=0.45, Da=1e-3, Cf=0.55, Ri=1.0, scalars=True, eps=1e-5, itc_max=60000)
    print("max rel diff", _tile_vs_oracle(gpu, orc, [item], 3))


GEOMETRIES = [
    # (nx, ny): pitch = round_up(nx+1, 4) and ny+1 decide the tile table
    (61, 45),    # pitch 64 = two whole tiles in x; y: tiles at 0 and 14 (overlap)
    (70, 33),    # pitch 72: x tiles 0, 32, 40; y: 0, 2
    (95, 97),    # y: 0, 32, 64, 66
    (40, 64),    # ny+1 = 65: y tiles 0, 32, 33
    (20, 26),    # one tile, smaller than the box
]


@pytest.mark.parametrize("geom", GEOMETRIES, ids=[f"{a}x{b}" for a, b in GEOMETRIES])
def test_tile_engine_geometries(gpu, orc, geom):
    """Channel variant, QUICK, porous block, both scalars, capped steps (every step ends on the
    itc_max path or converges) on tile tables with overlapping and partial tiles."""
    cfg = gpu.configs
    nx, ny = geom
    item = cfg.channel_case(nx, ny, seed=nx, Re=150.0, scheme=gpu.SCHEME_QUICK, block=cfg.centred_block(2, 1, 0.3),
                            porosity=0.5, Da=1e-3, Cf=0.55, Ri=0.8, scalars=True, itc_max=300)
    print(geom, "max rel diff", _tile_vs_oracle(gpu, orc, [item], 2))


@pytest.mark.parametrize("imax", [23, 40])
def test_tile_engine_reference_variant_sizes(gpu, orc, imax):
    """Reference boundary variant with b_art and upwind at sizes spanning several tiles."""
    cfg = gpu.configs
    items = [cfg.reference_case(imax, itc_max=400, b_art=0.3)[:4],
             cfg.reference_case(imax, itc_max=400, scheme=gpu.SCHEME_UPWIND)[:4]]
    print(imax, "max rel diff", _tile_vs_oracle(gpu, orc, items, 2))


def test_tile_engine_ragged_batch(gpu, orc):
    """Ragged batch in one graph launch: cases converge and leave at different iterations, each
    stays within the bound of its own oracle run."""
    cfg = gpu.configs
    items = [cfg.reference_case(12, itc_max=4000)[:4], cfg.reference_case(14, itc_max=4000, scheme=gpu.SCHEME_UPWIND)[:4]]
    for c in range(4):
        q = cfg.batch_case_params(c, 0, sizes=(17, 24, 31, 45))
        items.append(cfg.channel_case(q["nx"], q["ny"], seed=0, case_id=c, Re=q["Re"], block=q["block"],
                                      porosity=q["porosity"], Da=q["Da"], Cf=0.55, Ri=q["Ri"], scalars=True,
                                      itc_max=700))
    print("max rel diff", _tile_vs_oracle(gpu, orc, items, 3))


def test_tile_engine_equals_graph_engine_fast(gpu):
    """The tile engine and the FAST per-stage graph engine on the same 153 x 153 cases of the
    batched configuration: same iteration counts, fields within 1e-12."""
    pkg = gpu
    items, _ = pkg.configs.cfg_batch(3, seed=101, sizes=(153,), arith=pkg.ARITH_FAST, itc_max=400)
    outs, its = [], []
    for eng in (1, TILE):
        b = pkg.Batch([x[0] for x in items], [x[1] for x in items])
        b.set_option(pkg.OPT_ENGINE, eng)
        for c, x in enumerate(items):
            b.set_state(c, x[2])
        _, it, _, st = b.run(2, [x[3] for x in items])
        assert (st == pkg.CASE_DONE).all()
        its.append(it)
        outs.append([b.get_state(c) for c in range(len(items))])
        b.close()
    assert np.array_equal(its[0], its[1])
    worst = 0.0
    for c, (prm, *_rest) in enumerate(items):
        for k in ("um", "vm", "p", "pn", "T", "C"):
            x, y = mask_dead(k, outs[1][c][k], prm.bc), mask_dead(k, outs[0][c][k], prm.bc)
            worst = max(worst, _rel(x, y))
    print("tile vs graph max rel diff", worst)
    assert worst < 1e-12


def test_tile_engine_large_case(gpu, orc):
    """The combined configuration's 1024 x 512 case (two porous blocks, full scalars), two steps
    capped at 25 pseudo-iterations."""
    prm, mesh, st, itc, _ = gpu.configs.cfg_large(itc_max=25)
    print("max rel diff", _tile_vs_oracle(gpu, orc, [(prm, mesh, st, itc)], 2))


def test_tile_engine_needs_fast_arithmetic(gpu):
    prm, mesh, st, itc, _ = gpu.configs.reference_case(12)
    g = gpu.Case(prm, mesh)
    with pytest.raises(gpu.AcsError):
        g.set_option(gpu.OPT_ENGINE, TILE)


def test_tile_engine_upload_between_steps_changes_nothing(gpu):
    """A driver that keeps the state on the host downloads every field after a physical step and
    uploads it before the next.  The upload marks um_tau / vm_tau as possibly not satisfying the
    boundary passes, and the next iteration follows the reference's order for them -- with the
    same kernels as every other iteration, so the trajectory is bit-identical to an uninterrupted
    run (same iteration counts, same fields)."""
    pkg = gpu
    items, _ = pkg.configs.cfg_batch(3, seed=7, sizes=(37, 52), arith=pkg.ARITH_FAST, itc_max=4000)
    itc0 = np.array([x[3] for x in items], np.int32)

    def make():
        b = pkg.Batch([x[0] for x in items], [x[1] for x in items])
        b.set_option(pkg.OPT_ENGINE, TILE)
        for c, x in enumerate(items):
            b.set_state(c, x[2])
        return b

    a = make()
    itc_a, it_a, _, st_a = a.run(3, itc0)
    b = make()
    itc = itc0.copy()
    its = []
    for k in range(3):
        states = [b.get_state(c) for c in range(len(items))]
        for c in range(len(items)):
            b.set_state(c, states[c])
        itc, it, _, st = b.run(1, itc)
        its.append(it[:, 0])
    assert (st_a == pkg.CASE_DONE).all()
    assert np.array_equal(np.stack(its, axis=1), it_a) and np.array_equal(itc, itc_a)
    for c, (prm, *_r) in enumerate(items):
        x, y = a.get_state(c), b.get_state(c)
        for k in pkg.FIELDS:
            assert np.array_equal(mask_dead(k, x[k], prm.bc), mask_dead(k, y[k], prm.bc)), (c, k)
    a.close()
    b.close()

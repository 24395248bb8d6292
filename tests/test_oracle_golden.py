"""The CPU oracle pinned against the reference's own shipped outputs (tests/golden/)."""
import os

import numpy as np
import pytest

from conftest import GOLDEN


def _golden(name="reference_51x84.npz"):
    return np.load(os.path.join(GOLDEN, name))


def test_reference_jmax(orc):
    # comum.f90:44-46 for the two shipped builds (mesh.dat: 51 84, 10 16)
    assert orc.reference_jmax(51) == 84
    assert orc.reference_jmax(10) == 16


@pytest.mark.parametrize("imax,name", [(51, "reference_51x84.npz"), (10, "doconcurrent_10x16.npz")])
def test_mesh_matches_reference_grid_files(orc, imax, name):
    """x, y, xm, ym of nonsymetric_mesh.f90 against grid_u.dat / grid_v.dat (printed with 16
    significant digits) of the OpenMP build (imax 51) and of the do-concurrent build (imax 10).
    The files hold 16 significant digits, and the stretched half of y goes through tanh, whose
    last bits differ between libm implementations: every coordinate agrees to a few ulp of the
    largest one (measured: at most 5.6e-16 of max |coordinate|)."""
    g = _golden(name)
    assert (int(g["imax"]), int(g["jmax"])) == (imax, orc.reference_jmax(imax))
    m = orc.mesh_reference(imax)
    for k in ("x", "y", "xm", "ym"):
        ref = g[k]
        assert m[k].shape == ref.shape
        assert np.abs(m[k] - ref).max() <= 2e-15 * np.abs(ref).max(), k
    # xm(1) = -(x(2)+x(1))/2 is the reference's quirk: positive, e.g. +5.88 for x(1) = -6, x(2) = -5.76
    assert m["xm"][0] == pytest.approx(-0.5 * (g["x"][1] + g["x"][0]), abs=1e-14) and m["xm"][0] > 0


def test_porous_flag_of_reference_mesh(orc):
    m = orc.mesh_reference(51)
    x, y, flag = m["x"], m["y"], m["flag"]
    block = (x[:, None] <= -4.0) & (y[None, :] >= 0.5)
    # every block node is flagged, and fluid cells next to the block boundary are flagged too
    assert (flag[block] != 0).all()
    assert (flag[~block] == 3).sum() > 0
    assert ((flag != 0) == (m["liga"] == 1.0)).all()
    assert (m["eps"][flag != 0] == 0.5).all() and (m["eps"][flag == 0] == 1.0).all()


@pytest.mark.slow
def test_oracle_reproduces_reference_run_51x84(orc, pkg):
    """Whole reference run (default inputs: beta=1300, eps=1e-4, dt=0.005, 200 physical steps,
    about 315k pseudo-iterations) against the end state the reference's OpenMP build wrote to
    data/restart/.  Agreement to ~1e-14 relative requires the same pseudo-iteration count in
    every one of the 200 steps."""
    prm, mesh, st, itc, nsteps = pkg.configs.reference_case(51)
    assert nsteps == 200
    c = orc.OracleCase(prm, orc.mesh_reference(51))
    itc, iters, err = c.run(st, nsteps, itc)
    assert iters[0] > 1000 and (iters >= 1).all()
    g = _golden()
    for name in ("um", "vm", "p", "T", "C"):
        a, b = st[name], g[name]
        rel = np.abs(a - b).max() / np.abs(b).max()
        assert rel < 1e-12, (name, rel)

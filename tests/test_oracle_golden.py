"""The CPU oracle pinned against the reference's own shipped outputs (tests/golden/)."""
import os

import numpy as np
import pytest

from conftest import GOLDEN


def _golden():
    return np.load(os.path.join(GOLDEN, "reference_51x84.npz"))


def test_reference_jmax(orc):
    # comum.f90:44-46 for the two shipped builds (mesh.dat: 51 84, 10 16)
    assert orc.reference_jmax(51) == 84
    assert orc.reference_jmax(10) == 16


def test_mesh_matches_reference_grid_files(orc):
    """x, y, xm, ym of nonsymetric_mesh.f90 against grid_u.dat / grid_v.dat (printed with 16
    significant digits).  x is exact; the stretched half of y goes through tanh, whose last bits
    differ between libm implementations, so y agrees to a few ulp (1e-14 relative)."""
    g = _golden()
    m = orc.mesh_reference(51)
    for k in ("x", "y", "xm", "ym"):
        ref = g[k]
        assert m[k].shape == ref.shape
        np.testing.assert_allclose(m[k], ref, rtol=1e-14, atol=1e-15, err_msg=k)
    # xm(1) = -(x(2)+x(1))/2 is the reference's quirk: +5.88 for x(1) = -6, x(2) = -5.76
    assert m["xm"][0] == pytest.approx(5.88, abs=1e-14)


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

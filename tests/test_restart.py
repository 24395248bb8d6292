"""Restart / output files in the reference driver's formats.

Pins: the cell-centred velocities and the p, T, C columns of the reference's own
output_variables.dat (OpenMp_Multicore 51 x 84 and OpenMp_DoConcurrent 10 x 16, written by
output.f90 from the state in data/restart/) against comp_mean of that state; exact write/read round trips; the reader order of
initial.f90's restart(); and, on the GPU, a checkpoint/resume through restart files that stays
bit-identical to the oracle resuming from the same files.
"""
import os

import numpy as np
import pytest

from conftest import GOLDEN


@pytest.fixture(scope="module")
def rs(pkg):
    import importlib
    return importlib.import_module(pkg.__name__ + ".restart")


def _golden(name="reference_51x84.npz"):
    return np.load(os.path.join(GOLDEN, name))


@pytest.mark.parametrize("name", ["reference_51x84.npz", "doconcurrent_10x16.npz"])
def test_comp_mean_matches_reference_output_file(rs, name):
    """comp_mean of a run's restart files against the same run's output_variables.dat: the OpenMP
    build at 51 x 84 and the do-concurrent build at 10 x 16."""
    g = _golden(name)
    out = g["output_variables"]          # [imax][jmax][x, y, u, v, p, T, C], i outer (output.f90:12-18)
    u, v = rs.comp_mean(g["um"], g["vm"])
    for k, a in ((2, u), (3, v), (4, g["p"]), (5, g["T"]), (6, g["C"])):
        ref = out[:, :, k]
        rel = np.abs(a - ref).max() / np.abs(ref).max()
        assert rel < 1e-12, (k, rel)
    assert np.allclose(out[:, 0, 0], g["x"], rtol=1e-14) and np.allclose(out[0, :, 1], g["y"], rtol=1e-14)


def test_write_read_round_trip_and_layout(rs, tmp_path):
    g = _golden()
    rs.write_restart(str(tmp_path), g["um"], g["vm"], g["p"], g["T"], g["C"])
    back = rs.read_restart(str(tmp_path), 51, 84)
    for k in ("um", "vm", "p", "T", "C"):
        assert np.array_equal(back[k], g[k]), k
    lines = open(tmp_path / "restartU.dat").read().splitlines()
    assert len(lines) == 52 * 84 and float(lines[1]) == g["um"][0, 1]   # i outer, j inner
    ptc = open(tmp_path / "restartPTC.dat").read().splitlines()
    assert len(ptc) == 51 * 84 and [float(t) for t in ptc[0].split()] == [g["p"][0, 0], g["T"][0, 0], g["C"][0, 0]]
    rs.write_output_variables(str(tmp_path / "ov.dat"), g["x"], g["y"], g["um"], g["vm"], g["p"], g["T"], g["C"])
    ov = np.loadtxt(tmp_path / "ov.dat").reshape(51, 84, 7)
    assert np.abs(ov - g["output_variables"]).max() <= 1e-12 * np.abs(g["output_variables"]).max()


def test_reader_order_of_initial_f90(rs, tmp_path):
    imax, jmax = 4, 6
    um = np.arange((imax + 1) * jmax, dtype=float).reshape(imax + 1, jmax)
    vm = 100 + np.arange(imax * (jmax + 1), dtype=float).reshape(imax, jmax + 1)
    p = 1000 + np.arange(imax * jmax, dtype=float).reshape(imax, jmax)
    rs.write_restart(str(tmp_path), um, vm, p, p + 1, p + 2)
    r = rs.read_restart(str(tmp_path), imax, jmax, order="reader")
    seq = um.ravel()                       # file order
    for i in range(imax + 1):
        for j in range(jmax):
            assert r["um"][i, j] == seq[j * (imax + 1) + i]   # do j; do i; read (initial.f90:62-66)
    seqp = p.ravel()
    assert r["p"][2, 3] == seqp[3 * imax + 2]
    st = rs.restart_state(rs.read_restart(str(tmp_path), imax, jmax))
    assert np.array_equal(st["um_tau"], um) and np.array_equal(st["vm_tau"], vm)
    assert not st["pn"].any() and not st["T_tau"].any() and not st["um_n_tau"].any()


@pytest.mark.gpu
def test_checkpoint_resume_through_restart_files(gpu, orc, rs, tmp_path):
    """Run, save the restart files, resume a fresh device case from them, and compare with the
    oracle resuming from the same files: identical iteration counts and bit-identical fields."""
    pkg = gpu
    prm, mesh, st, itc, _ = pkg.configs.reference_case(12, itc_max=400)
    g = pkg.Case(prm, mesh)
    g.set_state(st)
    g.physical_steps(2, itc)
    rs.save_case(g, str(tmp_path))
    h = pkg.Case(prm, mesh)
    loaded = rs.load_case(h, str(tmp_path), prm.imax, prm.jmax)
    itc_g, it_g, _, status = h.physical_steps(2, 1)
    out = h.get_state()
    ost = {k: np.asfortranarray(v.copy()) for k, v in loaded.items()}
    itc_o, it_o, _ = orc.OracleCase(prm, orc.mesh_reference(12)).run(ost, 2, 1)
    assert status == pkg.CASE_DONE
    assert list(it_g) == list(it_o)
    for k in ("um", "p", "T", "C"):
        assert np.array_equal(out[k], ost[k]), k
    a, b = out["vm"].copy(), ost["vm"].copy()
    a[-1, -1] = b[-1, -1] = 0.0   # vm(imax, jmax+1) is never read by the loop
    assert np.array_equal(a, b)


def test_vtk_writer_reproduces_the_reference_file(pkg):
    """transient.f90:55-104 writes data/paraview_output<n>.vtk; the writer, given the final
    arrays of the reference's 10 x 16 run (its restart files) and the cell-centred velocities of
    comp_mean, reproduces the ParaView file that run shipped, character for character."""
    from importlib import import_module
    r = import_module(pkg.__name__ + ".restart")
    z = np.load(os.path.join(GOLDEN, "doconcurrent_10x16.npz"))
    u, v = r.comp_mean(z["um"], z["vm"])
    assert r.vtk_text(z["x"], z["y"], u, v, z["T"], z["p"]) == str(z["paraview_vtk"])


@pytest.mark.gpu
def test_cell_fields_on_device_equal_comp_mean(gpu):
    """acs_batch_cell_fields: comp_mean and the velocity magnitude on the device, bit for bit the
    host's (the reference's expression order, no fused multiply-add)."""
    from importlib import import_module
    r = import_module(gpu.__name__ + ".restart")
    cfg = gpu.configs
    items = [cfg.channel_case(37, 26, seed=3, scalars=True), cfg.reference_case(14)[:4]]
    b = gpu.Batch([x[0] for x in items], [x[1] for x in items])
    rng = np.random.default_rng(5)
    for c, (prm, mesh, st, itc) in enumerate(items):
        st = dict(st)
        st["um"] = np.asfortranarray(rng.uniform(-1, 1, st["um"].shape))
        st["vm"] = np.asfortranarray(rng.uniform(-1, 1, st["vm"].shape))
        b.set_state(c, st)
        u, v, mag = b.cell_fields(c)
        uh, vh = r.comp_mean(st["um"], st["vm"])
        assert np.array_equal(u, uh) and np.array_equal(v, vh)
        assert np.array_equal(mag, np.sqrt(uh * uh + vh * vh))
    b.close()

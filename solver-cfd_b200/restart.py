"""Restart and output files in the reference driver's formats (host side).

Checkpoint/resume of the device state through the Fortran driver: the driver's restart files
are plain text, one value (or one ``p T C`` triple) per line, written with list-directed output.

* ``write_restart`` writes ``restartU.dat``, ``restartV.dat``, ``restartPTC.dat`` as
  ``SUBROUTINE output`` does (output.f90:20-43): i in the outer loop, j in the inner loop.
* ``read_restart`` reads them back.  ``order="writer"`` (default) undoes the writer's loop order,
  so a file written by the reference (or by ``write_restart``) gives the arrays that were
  written.  ``order="reader"`` reproduces ``SUBROUTINE restart`` (initial.f90:52-87), which reads
  with j in the outer loop: for imax+1 != jmax that is a different assignment of the same
  numbers, and it is what the unmodified driver would load.
* ``comp_mean`` is comp_mean.f90:1-25 (cell-centred u, v) and ``write_output_variables`` writes
  data/output_variables.dat as output.f90:12-18 does (x, y, u, v, p, T, C per cell, i outer).
* ``vtk_text`` / ``write_vtk`` are the ParaView output of transient.f90:55-104;
  ``write_case_vtk`` writes it for a device case, with comp_mean computed on the device.
* ``restart_state`` turns restart arrays into a loop state the way ``PROGRAM main`` continues
  after ``CALL restart`` (main.f90:97-109): um_tau = um, vm_tau = vm, every other loop array 0.
* ``save_case`` / ``load_case`` move a case's state between the device (``Case`` or one case of
  a ``Batch``) and a restart directory.
"""
from __future__ import annotations

import os

import numpy as np

FILES = ("restartU.dat", "restartV.dat", "restartPTC.dat")
LOOP_FIELDS = ("um", "vm", "um_tau", "vm_tau", "um_n_tau", "vm_n_tau", "p", "pn",
               "T", "T_tau", "T_n_tau", "C", "C_tau", "C_n_tau")


def _fmt(v: float) -> str:
    # 17 significant digits: reading the text back gives the same double
    return f"{v: .17E}"


def write_restart(directory: str, um, vm, p, T, C) -> None:
    """output.f90:20-43 (i outer, j inner; one value per line, p T C on one line)."""
    um, vm, p, T, C = (np.asarray(a, np.float64) for a in (um, vm, p, T, C))
    imax, jmax = p.shape
    assert um.shape == (imax + 1, jmax) and vm.shape == (imax, jmax + 1)
    assert T.shape == p.shape and C.shape == p.shape
    os.makedirs(directory, exist_ok=True)
    with open(os.path.join(directory, FILES[0]), "w") as f:
        f.write("".join(_fmt(v) + "\n" for v in um.ravel(order="C")))
    with open(os.path.join(directory, FILES[1]), "w") as f:
        f.write("".join(_fmt(v) + "\n" for v in vm.ravel(order="C")))
    trip = np.stack([p, T, C], axis=-1).reshape(-1, 3)
    with open(os.path.join(directory, FILES[2]), "w") as f:
        f.write("".join(f"{_fmt(a)} {_fmt(b)} {_fmt(c)}\n" for a, b, c in trip))


def _numbers(path):
    with open(path) as f:
        return np.array(f.read().split(), dtype=np.float64)


def read_restart(directory: str, imax: int, jmax: int, order: str = "writer") -> dict:
    """The three restart files as Fortran-ordered arrays {um, vm, p, T, C}.

    order="writer": the arrays output.f90 wrote (i outer, j inner in the files);
    order="reader": the arrays initial.f90's restart() fills (j outer, i inner)."""
    if order not in ("writer", "reader"):
        raise ValueError("order must be 'writer' or 'reader'")
    u = _numbers(os.path.join(directory, FILES[0]))
    v = _numbers(os.path.join(directory, FILES[1]))
    ptc = _numbers(os.path.join(directory, FILES[2]))
    need = ((imax + 1) * jmax, imax * (jmax + 1), 3 * imax * jmax)
    for got, n, name in zip((u.size, v.size, ptc.size), need, FILES):
        if got < n:
            raise ValueError(f"{name}: {got} numbers, {n} needed for imax={imax}, jmax={jmax}")
    u, v, ptc = u[:need[0]], v[:need[1]], ptc[:need[2]].reshape(imax * jmax, 3)
    if order == "writer":
        um = u.reshape(imax + 1, jmax)
        vm = v.reshape(imax, jmax + 1)
        pp, TT, CC = (ptc[:, k].reshape(imax, jmax) for k in range(3))
    else:
        um = u.reshape(jmax, imax + 1).T
        vm = v.reshape(jmax + 1, imax).T
        pp, TT, CC = (ptc[:, k].reshape(jmax, imax).T for k in range(3))
    return {k: np.asfortranarray(a) for k, a in (("um", um), ("vm", vm), ("p", pp), ("T", TT), ("C", CC))}


def comp_mean(um, vm):
    """comp_mean.f90:1-25: u(i,j) = (um(i+1,j) + um(i,j)) / 2, v(i,j) = (vm(i,j+1) + vm(i,j)) / 2."""
    um, vm = np.asarray(um, np.float64), np.asarray(vm, np.float64)
    u = (um[1:, :] + um[:-1, :]) * 0.5
    v = (vm[:, 1:] + vm[:, :-1]) * 0.5
    return np.asfortranarray(u), np.asfortranarray(v)


def write_output_variables(path: str, x, y, um, vm, p, T, C) -> None:
    """output.f90:12-18: one line `x(i) y(j) u v p T C` per cell, i outer, j inner."""
    u, v = comp_mean(um, vm)
    imax, jmax = u.shape
    with open(path, "w") as f:
        for i in range(imax):
            for j in range(jmax):
                f.write(" ".join(_fmt(a) for a in (x[i], y[j], u[i, j], v[i, j], p[i, j], T[i, j], C[i, j])) + "\n")


def _fortran_int(v: int, width: int) -> str:
    """Fortran Iw: right-justified in `width` columns.  (A value wider than the field is written in
    full; the reference's I3 / I6 would print asterisks there, which no reader accepts.)"""
    return f"{int(v):{width}d}"


def vtk_text(x, y, u, v, T, P, title: str = "Droplet Combustion") -> str:
    """The ParaView file of transient.f90:55-104 as text: a STRUCTURED_GRID of the imax x jmax
    cell nodes (x(i), y(j)), i outer and j inner, with the velocity magnitude, T and P as point
    scalars and (u, v, 0) as vectors, every value in the reference's F14.4 format.  u, v are the
    cell-centred velocities of comp_mean."""
    x, y = np.asarray(x, np.float64), np.asarray(y, np.float64)
    u, v, T, P = (np.asarray(a, np.float64) for a in (u, v, T, P))
    imax, jmax = u.shape
    f14 = lambda a: f"{a:14.4f}"
    out = ["# vtk DataFile Version 3.0", title, "ASCII", "DATASET STRUCTURED_GRID",
           "DIMENSIONS" + " " + _fortran_int(jmax, 3) + " " + _fortran_int(imax, 3) + " " + "1",
           "POINTS" + " " + _fortran_int(jmax * imax, 6) + " " + "float"]
    for i in range(imax):
        for j in range(jmax):
            out.append(f14(x[i]) + f14(y[j]) + f14(0.0))
    out.append("POINT_DATA" + " " + _fortran_int(imax * jmax, 6))
    out += ["SCALARS VEL_MAGNITUDE float", "LOOKUP_TABLE default"]
    mag = np.sqrt(u * u + v * v)
    out += [f14(mag[i, j]) for i in range(imax) for j in range(jmax)]
    out += ["SCALARS T float", "LOOKUP_TABLE default"]
    out += [f14(T[i, j]) for i in range(imax) for j in range(jmax)]
    out += ["SCALARS P float", "LOOKUP_TABLE default"]
    out += [f14(P[i, j]) for i in range(imax) for j in range(jmax)]
    out += ["", "", "VECTORS Vectors float"]
    out += [f14(u[i, j]) + f14(v[i, j]) + f14(0.0) for i in range(imax) for j in range(jmax)]
    return "\n".join(out) + "\n"


def write_vtk(path: str, x, y, u, v, T, P, title: str = "Droplet Combustion") -> None:
    """Write `vtk_text` to `path` (the reference names it data/paraview_output<n>.vtk)."""
    with open(path, "w") as f:
        f.write(vtk_text(x, y, u, v, T, P, title))


def write_case_vtk(path: str, solver, mesh: dict, case: int = 0, title: str = "Droplet Combustion") -> None:
    """The ParaView file of a device case (a ``Case``, or case `case` of a ``Batch``): u, v and
    the velocity magnitude from comp_mean computed on the device, T and P downloaded."""
    if hasattr(solver, "cell_fields") and hasattr(solver, "physical_steps"):
        u, v, _ = solver.cell_fields()
        st = solver.get_state(("T", "p"))
    else:
        u, v, _ = solver.cell_fields(case)
        st = solver.get_state(case, ("T", "p"))
    write_vtk(path, mesh["x"], mesh["y"], u, v, st["T"], st["p"], title)


def restart_state(arrays: dict) -> dict:
    """Loop state after `CALL restart` (main.f90:97-109): um_tau = um, vm_tau = vm; pn, the
    n_tau arrays, T_tau and C_tau are the driver's uninitialised static arrays, i.e. zero."""
    imax, jmax = arrays["p"].shape
    st = {}
    for n in LOOP_FIELDS:
        shape = (imax + 1, jmax) if n.startswith("um") else (imax, jmax + 1) if n.startswith("vm") else (imax, jmax)
        st[n] = np.zeros(shape, order="F")
    for n in ("um", "vm", "p", "T", "C"):
        st[n][:] = arrays[n]
    st["um_tau"][:] = st["um"]
    st["vm_tau"][:] = st["vm"]
    return st


def save_case(obj, directory: str, case: int | None = None) -> None:
    """Write the restart files of a device case (a Case, or case `case` of a Batch)."""
    names = ("um", "vm", "p", "T", "C")
    st = obj.get_state(case, names) if case is not None else obj.get_state(names)
    write_restart(directory, st["um"], st["vm"], st["p"], st["T"], st["C"])


def load_case(obj, directory: str, imax: int, jmax: int, case: int | None = None, order: str = "writer") -> dict:
    """Read a restart directory and upload the resulting loop state to a device case; returns it."""
    st = restart_state(read_restart(directory, imax, jmax, order))
    if case is not None:
        obj.set_state(case, st)
    else:
        obj.set_state(st)
    return st

"""Generate the golden fixtures in this folder from the reference's shipped output files.

Run once in a checkout where the reference project is available (read-only), e.g.
    python tests/golden/make_golden.py /path/to/solver-cfd
The fixtures are plain numbers copied from the reference's own output files; nothing here is
computed.  Sources (paths relative to the reference project):
  OpenMp_Multicore/data/restart/restart{U,V,PTC}.dat   end state of the OpenMP build, 51 x 84,
      default inputs (input/iterations.dat: beta=1300, eps=1e-4, final_time=1 -> 200 steps),
      written by output.f90:20-43 (i outer, j inner);
  OpenMp_Multicore/data/grid_u.dat, grid_v.dat, mesh.dat  mesh of the same run
      (nonsymetric_mesh.f90:149-163): (xm(i), y(j)) and (x(i), ym(j)) pairs, i outer;
  OpenMp_Multicore/data/output_variables.dat             x, y, u, v, p, T, C (output.f90:10-15);
  OpenMp_DoConcurrent/data/output_variables.dat, restart/restart{U,V,PTC}.dat, grid_u.dat,
  grid_v.dat                                             10 x 16 run of the do-concurrent build.
      Its mesh is that of nonsymetric_mesh.f90 at imax = 10; its fields were written by sources or
      inputs other than the shipped ones (the porous block holds C = 0.05 and T relaxes from 0.05 towards
      a bottom wall at 1, where the shipped initial.f90 and comum.f90 set both to 1), so only the
      geometry and the file layout of that run pin anything.
"""
import os
import sys

import numpy as np


def read_numbers(path):
    with open(path) as f:
        return np.array(f.read().split(), dtype=np.float64)


def main(ref_root):
    here = os.path.dirname(os.path.abspath(__file__))
    mp = os.path.join(ref_root, "OpenMp_Multicore", "data")
    nx, ny, h = read_numbers(os.path.join(mp, "mesh.dat"))
    nx, ny = int(nx), int(ny)
    U = read_numbers(os.path.join(mp, "restart", "restartU.dat")).reshape(nx + 1, ny)
    V = read_numbers(os.path.join(mp, "restart", "restartV.dat")).reshape(nx, ny + 1)
    PTC = read_numbers(os.path.join(mp, "restart", "restartPTC.dat")).reshape(nx, ny, 3)
    gu = read_numbers(os.path.join(mp, "grid_u.dat")).reshape(nx + 1, ny, 2)
    gv = read_numbers(os.path.join(mp, "grid_v.dat")).reshape(nx, ny + 1, 2)
    out = read_numbers(os.path.join(mp, "output_variables.dat")).reshape(nx, ny, 7)
    np.savez_compressed(
        os.path.join(here, "reference_51x84.npz"),
        imax=nx, jmax=ny, Hvert=h,
        um=U, vm=V, p=PTC[:, :, 0], T=PTC[:, :, 1], C=PTC[:, :, 2],
        xm=gu[:, 0, 0], y=gu[0, :, 1], x=gv[:, 0, 0], ym=gv[0, :, 1],
        output_variables=out)
    dc = os.path.join(ref_root, "OpenMp_DoConcurrent", "data")
    nx, ny = 10, 16
    out10 = read_numbers(os.path.join(dc, "output_variables.dat")).reshape(nx, ny, 7)
    U = read_numbers(os.path.join(dc, "restart", "restartU.dat")).reshape(nx + 1, ny)
    V = read_numbers(os.path.join(dc, "restart", "restartV.dat")).reshape(nx, ny + 1)
    PTC = read_numbers(os.path.join(dc, "restart", "restartPTC.dat")).reshape(nx, ny, 3)
    gu = read_numbers(os.path.join(dc, "grid_u.dat")).reshape(nx + 1, ny, 2)
    gv = read_numbers(os.path.join(dc, "grid_v.dat")).reshape(nx, ny + 1, 2)
    # the ParaView file the same run wrote at its end (transient.f90:55-104), kept as text
    with open(os.path.join(dc, "paraview_output100.vtk")) as f:
        vtk10 = f.read()
    np.savez_compressed(
        os.path.join(here, "doconcurrent_10x16.npz"),
        imax=nx, jmax=ny, output_variables=out10, paraview_vtk=np.array(vtk10),
        um=U, vm=V, p=PTC[:, :, 0], T=PTC[:, :, 1], C=PTC[:, :, 2],
        xm=gu[:, 0, 0], y=gu[0, :, 1], x=gv[:, 0, 0], ym=gv[0, :, 1])
    print("wrote fixtures to", here)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        raise SystemExit("usage: python make_golden.py <root of the reference project checkout>")
    main(sys.argv[1])

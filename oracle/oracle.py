"""ctypes binding of the CPU oracle (``oracle/acs_oracle.cpp``).

TEST INFRASTRUCTURE ONLY: imported by tests/, by ``__graft_entry__.smoke()`` and by the CPU
baseline leg of ``bench.py``, always as the checker or the timed CPU baseline.  The product
(``solver-cfd_b200``) never imports it.

Arrays follow the Fortran reference: column-major, so a field ``um(1:imax+1, 1:jmax)`` is a
numpy array of shape ``(imax+1, jmax)`` with ``order='F'`` and ``um[i-1, j-1]`` is ``um(i,j)``.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liborc.so")
_lib = None


def build(force: bool = False) -> str:
    """Compile the oracle with its Makefile (g++, -ffp-contract=off, OpenMP)."""
    if force or not os.path.exists(_LIB_PATH) or (
        os.path.getmtime(_LIB_PATH) < os.path.getmtime(os.path.join(_HERE, "acs_oracle.cpp"))
    ):
        subprocess.run(["make", "-C", _HERE, "-B" if force else "all"], check=True,
                       stdout=subprocess.DEVNULL)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        _lib = C.CDLL(_LIB_PATH)
        _declare(_lib)
    return _lib


class OrcParams(C.Structure):
    _fields_ = [
        ("imax", C.c_int), ("jmax", C.c_int), ("scheme", C.c_int), ("bc", C.c_int),
        ("solve_scalars", C.c_int), ("itc_max", C.c_int),
        ("Re", C.c_double), ("Pe", C.c_double), ("Sc", C.c_double), ("Da", C.c_double),
        ("Cf", C.c_double), ("g", C.c_double), ("InvFr2", C.c_double), ("v_in", C.c_double),
        ("T_in", C.c_double), ("C_in", C.c_double), ("b_art", C.c_double), ("beta", C.c_double),
        ("dt", C.c_double), ("dtau", C.c_double), ("eps", C.c_double),
        ("arith", C.c_int), ("continuity", C.c_int),
    ]


class OrcState(C.Structure):
    _fields_ = [(n, C.POINTER(C.c_double)) for n in (
        "um", "vm", "um_tau", "vm_tau", "um_n_tau", "vm_n_tau", "p", "pn",
        "T", "T_tau", "T_n_tau", "C", "C_tau", "C_n_tau")]


_D = C.POINTER(C.c_double)
_I = C.POINTER(C.c_int)


def _declare(L):
    L.orc_reference_jmax.argtypes = [C.c_int]
    L.orc_reference_jmax.restype = C.c_int
    L.orc_mesh_reference.argtypes = [C.c_int, C.c_double, _D, _D, _D, _D, _I, _D, _D]
    L.orc_mesh_reference.restype = C.c_int
    L.orc_mesh_channel.argtypes = [C.c_int, C.c_int] + [C.c_double] * 12 + [_D, _D, _D, _D, _I, _D, _D]
    L.orc_mesh_channel.restype = C.c_int
    L.orc_noise.argtypes = [C.c_uint64] * 4 + [C.c_double]
    L.orc_noise.restype = C.c_double
    L.orc_noise_array.argtypes = [C.c_uint64] * 3 + [C.POINTER(C.c_uint64), C.c_longlong, C.c_double, _D]
    L.orc_create.argtypes = [C.POINTER(OrcParams), _D, _D, _D, _D, _D, _D]
    L.orc_create.restype = C.c_void_p
    L.orc_destroy.argtypes = [C.c_void_p]
    L.orc_resu.argtypes = [C.c_void_p, _D, _D, _D, _D]
    L.orc_resv.argtypes = [C.c_void_p, _D, _D, _D, _D, _D]
    L.orc_resz.argtypes = [C.c_void_p, _D, _D, _D, _D]
    L.orc_resc.argtypes = [C.c_void_p, _D, _D, _D, _D]
    L.orc_solve_u.argtypes = [C.c_void_p, _D, _D, _D, _D, _D]
    L.orc_solve_u.restype = C.c_double
    L.orc_solve_v.argtypes = [C.c_void_p, _D, _D, _D, _D, _D, _D]
    L.orc_solve_v.restype = C.c_double
    L.orc_solve_p.argtypes = [C.c_void_p, _D, _D, _D, _D]
    L.orc_solve_p.restype = C.c_double
    L.orc_solve_z.argtypes = [C.c_void_p, _D, _D, _D, _D, _D]
    L.orc_solve_c.argtypes = [C.c_void_p, _D, _D, _D, _D, _D]
    for n in ("orc_bc_uv",):
        getattr(L, n).argtypes = [C.c_void_p, _D, _D]
    for n in ("orc_bc_p", "orc_bc_z", "orc_bc_c"):
        getattr(L, n).argtypes = [C.c_void_p, _D]
    L.orc_run.argtypes = [C.c_void_p, C.POINTER(OrcState), C.c_int, _I, _I, _D]
    L.orc_run.restype = C.c_long


def _p(a: np.ndarray):
    assert a.dtype == np.float64 and (a.flags.f_contiguous or a.ndim == 1)
    return a.ctypes.data_as(_D)


def _pi(a: np.ndarray):
    assert a.dtype == np.int32
    return a.ctypes.data_as(_I)


def params_struct(prm) -> OrcParams:
    """Build the ctypes block from any object with the same attribute names."""
    s = OrcParams()
    for name, _ in OrcParams._fields_:
        setattr(s, name, getattr(prm, name))
    return s


def reference_jmax(imax: int) -> int:
    return lib().orc_reference_jmax(imax)


def mesh_reference(imax: int, porosity: float = 0.5) -> dict:
    """nonsymetric_mesh.f90 for the compiled-in domain of comum.f90 (12 x 20, Py=1.6, Q=1)."""
    ny = reference_jmax(imax)
    m = _alloc_mesh(imax, ny)
    lib().orc_mesh_reference(imax, porosity, _p(m["x"]), _p(m["y"]), _p(m["xm"]), _p(m["ym"]),
                             _pi(m["flag"]), _p(m["eps"]), _p(m["liga"]))
    return m


def mesh_channel(nx, ny, Lx, Ly, stretch, block, porosity, block2=None) -> dict:
    bx0, bx1, by0, by1 = block if block is not None else (1.0, -1.0, 1.0, -1.0)
    cx0, cx1, cy0, cy1 = block2 if block2 is not None else (1.0, -1.0, 1.0, -1.0)
    m = _alloc_mesh(nx, ny)
    lib().orc_mesh_channel(nx, ny, Lx, Ly, stretch, bx0, bx1, by0, by1, cx0, cx1, cy0, cy1,
                           porosity, _p(m["x"]), _p(m["y"]), _p(m["xm"]), _p(m["ym"]),
                           _pi(m["flag"]), _p(m["eps"]), _p(m["liga"]))
    return m


def _alloc_mesh(nx, ny):
    return dict(nx=nx, ny=ny, x=np.zeros(nx), y=np.zeros(ny), xm=np.zeros(nx + 1),
                ym=np.zeros(ny + 1), flag=np.zeros((nx, ny), np.int32, order="F"),
                eps=np.zeros((nx, ny), order="F"), liga=np.zeros((nx, ny), order="F"))


def noise(seed, case_id, field, index, amp):
    return lib().orc_noise(seed, case_id, field, index, amp)


def noise_array(seed, case_id, field, index: np.ndarray, amp) -> np.ndarray:
    idx = np.ascontiguousarray(index, dtype=np.uint64)
    out = np.zeros(idx.size)
    lib().orc_noise_array(seed, case_id, field, idx.ctypes.data_as(C.POINTER(C.c_uint64)), idx.size, amp, _p(out))
    return out


STATE_FIELDS = ("um", "vm", "um_tau", "vm_tau", "um_n_tau", "vm_n_tau", "p", "pn",
                "T", "T_tau", "T_n_tau", "C", "C_tau", "C_n_tau")


def field_shape(name: str, nx: int, ny: int):
    if name.startswith("um"):
        return (nx + 1, ny)
    if name.startswith("vm"):
        return (nx, ny + 1)
    return (nx, ny)


class OracleCase:
    """One case: the metric arrays, the porous fields and the parameter block."""

    def __init__(self, prm, mesh: dict):
        self.prm = params_struct(prm)
        self.nx, self.ny = self.prm.imax, self.prm.jmax
        assert (mesh["nx"], mesh["ny"]) == (self.nx, self.ny)
        self._keep = [np.ascontiguousarray(mesh[k], dtype=np.float64) for k in ("x", "y", "xm", "ym")]
        self._keep += [np.asfortranarray(mesh[k], dtype=np.float64) for k in ("eps", "liga")]
        self.h = lib().orc_create(C.byref(self.prm), *[_p(a) for a in self._keep])

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.orc_destroy(self.h)
            self.h = None

    def zeros(self, name):
        return np.zeros(field_shape(name, self.nx, self.ny), order="F")

    # per-routine entry points (same argument meaning as the Fortran subroutines)
    def resu(self, um, vm, p):
        RU = self.zeros("um"); lib().orc_resu(self.h, _p(um), _p(vm), _p(p), _p(RU)); return RU

    def resv(self, um, vm, p, T):
        RV = self.zeros("vm"); lib().orc_resv(self.h, _p(um), _p(vm), _p(p), _p(T), _p(RV)); return RV

    def resz(self, um, vm, Z):
        R = self.zeros("p"); lib().orc_resz(self.h, _p(um), _p(vm), _p(Z), _p(R)); return R

    def resc(self, um, vm, Cf):
        R = self.zeros("p"); lib().orc_resc(self.h, _p(um), _p(vm), _p(Cf), _p(R)); return R

    def solve_u(self, um, um_tau, vm_tau, p, um_n_tau):
        return lib().orc_solve_u(self.h, _p(um), _p(um_tau), _p(vm_tau), _p(p), _p(um_n_tau))

    def solve_v(self, vm, um_tau, vm_tau, p, T, vm_n_tau):
        return lib().orc_solve_v(self.h, _p(vm), _p(um_tau), _p(vm_tau), _p(p), _p(T), _p(vm_n_tau))

    def solve_p(self, p, um_n, vm_n, pn):
        return lib().orc_solve_p(self.h, _p(p), _p(um_n), _p(vm_n), _p(pn))

    def solve_z(self, um_n, vm_n, Z, Z_n_tau, Z_tau):
        lib().orc_solve_z(self.h, _p(um_n), _p(vm_n), _p(Z), _p(Z_n_tau), _p(Z_tau))

    def solve_c(self, um_n, vm_n, Cc, C_n_tau, C_tau):
        lib().orc_solve_c(self.h, _p(um_n), _p(vm_n), _p(Cc), _p(C_n_tau), _p(C_tau))

    def bc_uv(self, um, vm):
        lib().orc_bc_uv(self.h, _p(um), _p(vm))

    def bc_p(self, p):
        lib().orc_bc_p(self.h, _p(p))

    def bc_z(self, z):
        lib().orc_bc_z(self.h, _p(z))

    def bc_c(self, z):
        lib().orc_bc_c(self.h, _p(z))

    def run(self, state: dict, n_steps: int, itc: int):
        """main.f90:116-186 for n_steps; state arrays are updated in place.

        Returns (itc_after, iters[n_steps], err[n_steps])."""
        st = OrcState()
        for n in STATE_FIELDS:
            a = state[n]
            assert a.shape == field_shape(n, self.nx, self.ny) and a.flags.f_contiguous
            setattr(st, n, _p(a))
        itc_c = C.c_int(itc)
        iters = np.zeros(n_steps, np.int32)
        err = np.zeros(n_steps)
        lib().orc_run(self.h, C.byref(st), n_steps, C.byref(itc_c), _pi(iters), _p(err))
        return itc_c.value, iters, err


def set_threads(n: int) -> None:
    """OpenMP thread count of the oracle (affects speed only, never the results)."""
    os.environ["OMP_NUM_THREADS"] = str(n)
    try:
        C.CDLL("libgomp.so.1").omp_set_num_threads(int(n))
    except OSError:
        pass


__all__ = [
    "OracleCase", "mesh_reference", "mesh_channel", "reference_jmax", "noise", "build",
    "STATE_FIELDS", "field_shape", "OrcParams", "set_threads"]

"""solver-cfd_b200 -- host layer of the B200 artificial-compressibility pseudo-time solver.

This package is a thin ctypes binding of ``libacs_b200.so`` (C ABI in ``include/acs.h``) plus a
Python mirror of the reference driver's interface for the hot path (paths relative to the
reference project, OpenMp_Multicore/):

* ``solve_U``, ``solve_V``, ``solve_P``, ``solve_Z``, ``solve_C`` -- same names, argument order
  and in/out meaning as the Fortran subroutines (equations.f90:244, 546, 607, 669, 769), on
  column-major numpy arrays; each call is one trip through the CUDA kernels;
* ``Case.physical_steps`` -- the loop of main.f90:116-186 on the device;
* ``Batch`` -- many independent cases in one graph launch.

There is no CPU fallback: if the CUDA library or a device is missing, calls raise
``AcsError``.  Arrays follow the Fortran layout: ``um`` has shape ``(imax+1, jmax)`` with
``order='F'`` and ``um[i-1, j-1]`` is the reference's ``um(i,j)``.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import asdict, dataclass, field, fields, replace

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libacs_b200.so")
_lib = None

ACS_OK, ACS_E_ARG, ACS_E_SIZE, ACS_E_CUDA, ACS_E_NOMEM, ACS_E_STATE, ACS_E_UNSUPPORTED = range(7)
SCHEME_QUICK, SCHEME_UPWIND = 0, 1
BC_REFERENCE, BC_CHANNEL = 0, 1
ARITH_EXACT, ARITH_FAST = 0, 1
CASE_RUNNING, CASE_DONE, CASE_FAILED = 0, 1, 2

FIELDS = ("um", "vm", "um_tau", "vm_tau", "um_n_tau", "vm_n_tau", "p", "pn",
          "T", "T_tau", "T_n_tau", "C", "C_tau", "C_n_tau")
FIELD_ID = {n: k for k, n in enumerate(FIELDS)}

EXPORTED = (
    "acs_last_error", "acs_version", "acs_device_count", "acs_reference_jmax",
    "acs_mesh_reference", "acs_mesh_channel", "acs_noise", "acs_noise_array", "acs_create", "acs_destroy",
    "acs_set_stream", "acs_solve_u", "acs_solve_v", "acs_solve_p", "acs_solve_z", "acs_solve_c",
    "acs_set_field", "acs_get_field", "acs_physical_steps", "acs_batch_create",
    "acs_batch_destroy", "acs_batch_set_stream", "acs_batch_set_field", "acs_batch_get_field",
    "acs_batch_run", "acs_batch_launch_count", "acs_launch_count", "acs_batch_time_kernel",
    "acs_batch_set_option", "acs_set_option", "acs_solve_u_static",
    "acs_batch_ws_enable", "acs_batch_ws_features", "acs_batch_ws_target", "acs_batch_set_start",
    "acs_batch_set_cluster_size", "acs_batch_set_tolerance", "acs_batch_cell_fields", "acs_cell_fields",
    "acs_mesh_channel_device",
)
WS_IN, WS_OUT = 11, 8
POLICY_BEST, POLICY_PREDICTED, POLICY_PLAIN = 0, 1, 2
START_PLAIN, START_EXTRAP, START_LEARNED = 0, 1, 2
OPT_ENGINE, OPT_NODES_PER_CTA, OPT_L1_LOADS, OPT_THREADS, OPT_CTAS_PER_SM, OPT_STAGED = 1, 2, 3, 4, 5, 6
OPT_EXTRAP_ORDER = 7
ENGINE_CLUSTER, ENGINE_GRAPH, ENGINE_TILE = 0, 1, 2


class AcsError(RuntimeError):
    def __init__(self, code: int, where: str):
        msg = _lib.acs_last_error().decode() if _lib is not None else ""
        super().__init__(f"{where} failed with code {code}: {msg}")
        self.code = code


class AcsParams(C.Structure):
    _fields_ = [
        ("imax", C.c_int), ("jmax", C.c_int), ("scheme", C.c_int), ("bc", C.c_int),
        ("solve_scalars", C.c_int), ("itc_max", C.c_int),
        ("Re", C.c_double), ("Pe", C.c_double), ("Sc", C.c_double), ("Da", C.c_double),
        ("Cf", C.c_double), ("g", C.c_double), ("InvFr2", C.c_double), ("v_in", C.c_double),
        ("T_in", C.c_double), ("C_in", C.c_double), ("b_art", C.c_double), ("beta", C.c_double),
        ("dt", C.c_double), ("dtau", C.c_double), ("eps", C.c_double),
        ("arith", C.c_int), ("continuity", C.c_int),
    ]


_D = C.POINTER(C.c_double)
_I = C.POINTER(C.c_int)


class AcsGrid(C.Structure):
    _fields_ = [("imax", C.c_int), ("jmax", C.c_int), ("x", _D), ("y", _D), ("xm", _D), ("ym", _D),
                ("epsilon1", _D), ("liga_poros", _D)]


def lib():
    """Load libacs_b200.so.  Raises (never falls back) when it is missing."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `python {_HERE}/build.py`")
        L = C.CDLL(LIB_PATH)
        _declare(L)
        _lib = L
    return _lib


def _declare(L):
    V = C.c_void_p
    L.acs_last_error.restype = C.c_char_p
    L.acs_version.restype = C.c_char_p
    L.acs_device_count.argtypes = [_I]
    L.acs_reference_jmax.argtypes = [C.c_int]
    L.acs_mesh_reference.argtypes = [C.c_int, C.c_double, _D, _D, _D, _D, _I, _D, _D]
    L.acs_mesh_channel.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, _D, _D,
                                   C.c_double, _D, _D, _D, _D, _I, _D, _D]
    L.acs_mesh_channel_device.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, _D, _D,
                                          C.c_double] + [C.c_void_p] * 8
    L.acs_noise.argtypes = [C.c_uint64] * 4 + [C.c_double]
    L.acs_noise.restype = C.c_double
    L.acs_noise_array.argtypes = [C.c_uint64] * 3 + [C.POINTER(C.c_uint64), C.c_longlong, C.c_double, _D]
    L.acs_create.argtypes = [C.POINTER(AcsGrid), C.POINTER(AcsParams), C.POINTER(V)]
    L.acs_destroy.argtypes = [V]
    L.acs_set_stream.argtypes = [V, V]
    L.acs_solve_u.argtypes = [V, _D, _D, _D, _D, _D, _D]
    L.acs_solve_v.argtypes = [V, _D, _D, _D, _D, _D, _D, _D]
    L.acs_solve_p.argtypes = [V, _D, _D, _D, _D, _D]
    L.acs_solve_z.argtypes = [V, _D, _D, _D, _D, _D]
    L.acs_solve_c.argtypes = [V, _D, _D, _D, _D, _D]
    L.acs_set_field.argtypes = [V, C.c_int, _D]
    L.acs_get_field.argtypes = [V, C.c_int, _D]
    L.acs_physical_steps.argtypes = [V, C.c_int, _I, _I, _D, _I]
    L.acs_batch_create.argtypes = [C.POINTER(AcsGrid), C.POINTER(AcsParams), C.c_int, C.POINTER(V)]
    L.acs_batch_destroy.argtypes = [V]
    L.acs_batch_set_stream.argtypes = [V, V]
    L.acs_batch_set_field.argtypes = [V, C.c_int, C.c_int, _D]
    L.acs_batch_get_field.argtypes = [V, C.c_int, C.c_int, _D]
    L.acs_batch_run.argtypes = [V, C.c_int, _I, _I, _D, _I]
    L.acs_batch_launch_count.argtypes = [V, C.POINTER(C.c_longlong)]
    L.acs_launch_count.argtypes = [V, C.POINTER(C.c_longlong)]
    L.acs_batch_time_kernel.argtypes = [V, C.c_int, C.c_int, _D, C.POINTER(C.c_longlong)]
    L.acs_batch_set_option.argtypes = [V, C.c_int, C.c_longlong]
    L.acs_set_option.argtypes = [V, C.c_int, C.c_longlong]
    L.acs_solve_u_static.argtypes = [C.POINTER(AcsParams), C.POINTER(AcsGrid), V, V, V, V, V, _D, V]
    L.acs_batch_set_cluster_size.argtypes = [V, C.c_int, C.c_int]
    L.acs_batch_cell_fields.argtypes = [V, C.c_int, _D, _D, _D]
    L.acs_cell_fields.argtypes = [V, _D, _D, _D]
    L.acs_batch_set_tolerance.argtypes = [V, C.c_int, C.c_double]
    L.acs_batch_ws_enable.argtypes = [V, C.c_int, C.c_int]
    L.acs_batch_ws_features.argtypes = [V, V, V]
    L.acs_batch_ws_target.argtypes = [V, V, V]
    L.acs_batch_set_start.argtypes = [V, V, C.c_int, V, C.c_int, _I, _D]


def _check(code: int, where: str):
    if code != ACS_OK:
        raise AcsError(code, where)


def _dp(a: np.ndarray):
    if a.dtype != np.float64 or not (a.flags.f_contiguous or a.ndim == 1):
        raise ValueError("arrays must be float64 and Fortran-contiguous")
    return a.ctypes.data_as(_D)


def device_count() -> int:
    n = C.c_int(0)
    _check(lib().acs_device_count(C.byref(n)), "acs_device_count")
    return n.value


# ---------------------------------------------------------------------------------------------
# Parameters
# ---------------------------------------------------------------------------------------------
@dataclass
class Params:
    """Constants of the loop.  Defaults are the reference's (comum.f90, input/iterations.dat,
    main.f90:105-106) for imax = 51."""
    imax: int = 51
    jmax: int = 84
    scheme: int = SCHEME_QUICK
    bc: int = BC_REFERENCE
    solve_scalars: int = 1
    itc_max: int = 800000
    Re: float = 1.0
    Pe: float = 1.0
    Sc: float = 1.0
    Da: float = 1.0e-2
    Cf: float = 1.75 / (150.0 * 0.5 ** 3) ** 0.5
    g: float = 9.80665
    InvFr2: float = 1.0
    v_in: float = 0.5
    T_in: float = 1.0
    C_in: float = 0.0
    b_art: float = 0.0
    beta: float = 1300.0
    dt: float = 0.5e-2
    dtau: float = 5.0e-2
    eps: float = 1.0e-4
    arith: int = ARITH_EXACT
    continuity: int = 0

    def struct(self) -> AcsParams:
        s = AcsParams()
        for k, v in asdict(self).items():
            setattr(s, k, v)
        return s


def reference_jmax(imax: int) -> int:
    return lib().acs_reference_jmax(imax)


def _alloc_mesh(nx, ny):
    return dict(nx=nx, ny=ny, x=np.zeros(nx), y=np.zeros(ny), xm=np.zeros(nx + 1),
                ym=np.zeros(ny + 1), flag=np.zeros((nx, ny), np.int32, order="F"),
                eps=np.zeros((nx, ny), order="F"), liga=np.zeros((nx, ny), order="F"))


def mesh_reference(imax: int, porosity: float = 0.5) -> dict:
    """The reference driver's `CALL mesh` (nonsymetric_mesh.f90:1-218)."""
    ny = reference_jmax(imax)
    m = _alloc_mesh(imax, ny)
    _check(lib().acs_mesh_reference(imax, porosity, _dp(m["x"]), _dp(m["y"]), _dp(m["xm"]),
                                    _dp(m["ym"]), m["flag"].ctypes.data_as(_I), _dp(m["eps"]),
                                    _dp(m["liga"])), "acs_mesh_reference")
    return m


def mesh_channel(nx, ny, Lx, Ly, stretch, block, porosity, block2=None) -> dict:
    m = _alloc_mesh(nx, ny)
    b1 = np.array(block, float) if block is not None else None
    b2 = np.array(block2, float) if block2 is not None else None
    _check(lib().acs_mesh_channel(
        nx, ny, Lx, Ly, stretch, b1.ctypes.data_as(_D) if b1 is not None else None,
        b2.ctypes.data_as(_D) if b2 is not None else None, porosity, _dp(m["x"]), _dp(m["y"]),
        _dp(m["xm"]), _dp(m["ym"]), m["flag"].ctypes.data_as(_I), _dp(m["eps"]), _dp(m["liga"])),
        "acs_mesh_channel")
    return m


def noise(seed, case_id, field_id, index, amp) -> float:
    return lib().acs_noise(seed, case_id, field_id, index, amp)


def noise_array(seed, case_id, field_id, index: np.ndarray, amp) -> np.ndarray:
    idx = np.ascontiguousarray(index, dtype=np.uint64)
    out = np.zeros(idx.size)
    _check(lib().acs_noise_array(seed, case_id, field_id, idx.ctypes.data_as(C.POINTER(C.c_uint64)),
                                 idx.size, amp, out.ctypes.data_as(_D)), "acs_noise_array")
    return out


def field_shape(name: str, nx: int, ny: int):
    if name.startswith("um"):
        return (nx + 1, ny)
    if name.startswith("vm"):
        return (nx, ny + 1)
    return (nx, ny)


def _grid_struct(mesh: dict, keep: list) -> AcsGrid:
    arrs = [np.ascontiguousarray(mesh[k], np.float64) for k in ("x", "y", "xm", "ym")]
    arrs += [np.asfortranarray(mesh[k], np.float64) for k in ("eps", "liga")]
    keep.extend(arrs)
    g = AcsGrid()
    g.imax, g.jmax = mesh["nx"], mesh["ny"]
    g.x, g.y, g.xm, g.ym, g.epsilon1, g.liga_poros = [_dp(a) for a in arrs]
    return g


# ---------------------------------------------------------------------------------------------
# One case
# ---------------------------------------------------------------------------------------------
class Case:
    """One case on the device (acs_handle)."""

    def __init__(self, params: Params, mesh: dict):
        self.params = params
        self.nx, self.ny = params.imax, params.jmax
        self._keep: list = []
        g = _grid_struct(mesh, self._keep)
        self._p = params.struct()
        h = C.c_void_p()
        _check(lib().acs_create(C.byref(g), C.byref(self._p), C.byref(h)), "acs_create")
        self.h = h

    def close(self):
        if getattr(self, "h", None) and self.h.value and _lib is not None:
            _lib.acs_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        self.close()

    def zeros(self, name):
        return np.zeros(field_shape(name, self.nx, self.ny), order="F")

    def set_stream(self, stream_ptr: int):
        _check(lib().acs_set_stream(self.h, C.c_void_p(stream_ptr)), "acs_set_stream")

    def set_option(self, option: int, value: int):
        _check(lib().acs_set_option(self.h, option, value), "acs_set_option")

    # -- per-routine entry points (equations.f90) --
    def solve_U(self, um, vm, um_n, um_tau, vm_tau, um_n_tau, p) -> float:
        """solve_U(um,vm,um_n,um_tau,vm_tau,um_n_tau,p,residual_u): writes um_n_tau, rewrites
        the boundary of vm_tau (bcUV), returns residual_u.  vm and um_n are unused, as in the
        reference."""
        r = C.c_double()
        _check(lib().acs_solve_u(self.h, _dp(um), _dp(um_tau), _dp(vm_tau), _dp(p), _dp(um_n_tau),
                                 C.byref(r)), "acs_solve_u")
        return r.value

    def solve_V(self, um, vm, vm_n, um_tau, vm_tau, vm_n_tau, p, T) -> float:
        r = C.c_double()
        _check(lib().acs_solve_v(self.h, _dp(vm), _dp(um_tau), _dp(vm_tau), _dp(p), _dp(T),
                                 _dp(vm_n_tau), C.byref(r)), "acs_solve_v")
        return r.value

    def solve_P(self, p, um_n, vm_n, pn) -> float:
        r = C.c_double()
        _check(lib().acs_solve_p(self.h, _dp(p), _dp(um_n), _dp(vm_n), _dp(pn), C.byref(r)),
               "acs_solve_p")
        return r.value

    def solve_Z(self, um_n, vm_n, Z, Z_n_tau, Z_tau) -> None:
        _check(lib().acs_solve_z(self.h, _dp(um_n), _dp(vm_n), _dp(Z), _dp(Z_n_tau), _dp(Z_tau)),
               "acs_solve_z")

    def solve_C(self, um_n, vm_n, Cc, C_n_tau, C_tau) -> None:
        _check(lib().acs_solve_c(self.h, _dp(um_n), _dp(vm_n), _dp(Cc), _dp(C_n_tau), _dp(C_tau)),
               "acs_solve_c")

    # -- device-resident loop --
    def set_state(self, state: dict):
        for n, a in state.items():
            _check(lib().acs_set_field(self.h, FIELD_ID[n], _dp(np.asfortranarray(a))), "acs_set_field")

    def get_state(self, names=FIELDS) -> dict:
        out = {}
        for n in names:
            a = self.zeros(n)
            _check(lib().acs_get_field(self.h, FIELD_ID[n], _dp(a)), "acs_get_field")
            out[n] = a
        return out

    def physical_steps(self, n_steps: int, itc: int):
        """main.f90:116-186 for n_steps steps.  Returns (itc, iters[n], err[n], status)."""
        itc_c = C.c_int(itc)
        iters = np.zeros(n_steps, np.int32)
        err = np.zeros(n_steps)
        st = C.c_int(0)
        code = lib().acs_physical_steps(self.h, n_steps, C.byref(itc_c),
                                        iters.ctypes.data_as(_I), _dp(err), C.byref(st))
        if code not in (ACS_OK, ACS_E_STATE) or (code == ACS_E_STATE and st.value != CASE_FAILED):
            _check(code, "acs_physical_steps")
        return itc_c.value, iters, err, st.value

    def launch_count(self) -> int:
        n = C.c_longlong(0)
        _check(lib().acs_launch_count(self.h, C.byref(n)), "acs_launch_count")
        return n.value

    def cell_fields(self):
        """comp_mean on the device: cell-centred (u, v) and the velocity magnitude."""
        out = [np.zeros((self.nx, self.ny), order="F") for _ in range(3)]
        _check(lib().acs_cell_fields(self.h, *(_dp(a) for a in out)), "acs_cell_fields")
        return tuple(out)


# ---------------------------------------------------------------------------------------------
# Batch of independent cases
# ---------------------------------------------------------------------------------------------
class Batch:
    """Many independent cases advanced together (acs_batch)."""

    def __init__(self, params_list, meshes):
        assert len(params_list) == len(meshes) and len(meshes) > 0
        self.params = list(params_list)
        self.n = len(meshes)
        self._keep: list = []
        grids = (AcsGrid * self.n)(*[_grid_struct(m, self._keep) for m in meshes])
        prms = (AcsParams * self.n)(*[p.struct() for p in params_list])
        self._grids, self._prms = grids, prms
        h = C.c_void_p()
        _check(lib().acs_batch_create(grids, prms, self.n, C.byref(h)), "acs_batch_create")
        self.h = h

    def close(self):
        if getattr(self, "h", None) and self.h.value and _lib is not None:
            _lib.acs_batch_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        self.close()

    def set_stream(self, stream_ptr: int):
        _check(lib().acs_batch_set_stream(self.h, C.c_void_p(stream_ptr)), "acs_batch_set_stream")

    def set_option(self, option: int, value: int):
        _check(lib().acs_batch_set_option(self.h, option, value), "acs_batch_set_option")

    def zeros(self, c, name):
        p = self.params[c]
        return np.zeros(field_shape(name, p.imax, p.jmax), order="F")

    def set_state(self, c: int, state: dict):
        for n, a in state.items():
            _check(lib().acs_batch_set_field(self.h, c, FIELD_ID[n], _dp(np.asfortranarray(a))),
                   "acs_batch_set_field")

    def get_state(self, c: int, names=FIELDS, out=None) -> dict:
        """Download fields of case c (into the arrays of `out` when given)."""
        res = {}
        for n in names:
            a = out[n] if out is not None else self.zeros(c, n)
            _check(lib().acs_batch_get_field(self.h, c, FIELD_ID[n], _dp(a)), "acs_batch_get_field")
            res[n] = a
        return res

    def run(self, n_steps: int, itc):
        """Advance every case n_steps physical steps.  Returns (itc[n], iters[n, n_steps],
        err[n, n_steps], status[n])."""
        itc_a = np.ascontiguousarray(np.broadcast_to(np.asarray(itc, np.int32), (self.n,))).copy()
        iters = np.zeros((self.n, n_steps), np.int32)
        err = np.zeros((self.n, n_steps))
        st = np.zeros(self.n, np.int32)
        code = lib().acs_batch_run(self.h, n_steps, itc_a.ctypes.data_as(_I),
                                   iters.ctypes.data_as(_I), err.ctypes.data_as(_D),
                                   st.ctypes.data_as(_I))
        if code != ACS_OK and not (code == ACS_E_STATE and (st == CASE_FAILED).any()):
            _check(code, "acs_batch_run")
        return itc_a, iters, err, st

    def launch_count(self) -> int:
        n = C.c_longlong(0)
        _check(lib().acs_batch_launch_count(self.h, C.byref(n)), "acs_batch_launch_count")
        return n.value

    def cell_fields(self, c: int):
        """comp_mean of case c on the device: cell-centred (u, v) and the velocity magnitude."""
        p = self.params[c]
        out = [np.zeros((p.imax, p.jmax), order="F") for _ in range(3)]
        _check(lib().acs_batch_cell_fields(self.h, c, *(_dp(a) for a in out)), "acs_batch_cell_fields")
        return tuple(out)

    def set_cluster_size(self, c: int, ctas: int):
        """CTAs of case c's cluster in the persistent engine (0: from OPT_NODES_PER_CTA)."""
        _check(lib().acs_batch_set_cluster_size(self.h, c, ctas), "acs_batch_set_cluster_size")

    def set_tolerance(self, c: int, eps: float):
        """Pseudo-time residual tolerance of case c for the following steps (initially its
        params' eps)."""
        _check(lib().acs_batch_set_tolerance(self.h, c, float(eps)), "acs_batch_set_tolerance")

    def balance_clusters(self, iterations, slots: int, kmin: int = 1):
        """Give each case CTAs in proportion to its pseudo-iteration count (e.g. of the last
        step), within `slots` resident CTAs (SMs x CTAs per SM); returns the sizes."""
        it = np.maximum(np.asarray(iterations, np.float64), 1.0)
        k = np.clip(np.floor(slots * it / it.sum()), kmin, 16).astype(int)
        while k.sum() > slots and (k > kmin).any():
            k[np.argmax(np.where(k > kmin, k / it, -1))] -= 1
        while k.sum() < slots and (k < 16).any():   # the rest to the most loaded CTAs
            k[np.argmax(np.where(k < 16, it / k, -1))] += 1
        for c in range(self.n):
            self.set_cluster_size(c, int(k[c]))
        return k

    # ---- learned warm start (device pointers: torch tensors' data_ptr()) -------------------
    def ws_enable(self, H: int, W: int):
        _check(lib().acs_batch_ws_enable(self.h, H, W), "acs_batch_ws_enable")

    def ws_features(self, X_ptr: int, scale_ptr: int = 0):
        _check(lib().acs_batch_ws_features(self.h, C.c_void_p(X_ptr), C.c_void_p(scale_ptr or 0)),
               "acs_batch_ws_features")

    def ws_target(self, T_ptr: int, W_ptr: int):
        _check(lib().acs_batch_ws_target(self.h, C.c_void_p(T_ptr), C.c_void_p(W_ptr)), "acs_batch_ws_target")

    def set_start(self, Y_ptr, ldy: int, scale_ptr, policy: int):
        """Choose the start of the next pseudo-time loop; returns (chosen[n], res0[n, 3]):
        chosen = 0 plain, 1 extrapolated, 2 learned; res0 = the three initial residuals (NaN for
        the learned one when Y_ptr is None)."""
        chosen = np.zeros(self.n, np.int32)
        res0 = np.zeros((self.n, 3))
        _check(lib().acs_batch_set_start(self.h, C.c_void_p(Y_ptr or 0), ldy, C.c_void_p(scale_ptr or 0), policy,
                                         chosen.ctypes.data_as(_I), res0.ctypes.data_as(_D)),
               "acs_batch_set_start")
        return chosen, res0

    def time_kernel(self, kernel: int, reps: int = 20):
        """Mean duration (ms) of one launch of a loop kernel and the nodes it updates."""
        ms = C.c_double(0.0)
        cells = C.c_longlong(0)
        _check(lib().acs_batch_time_kernel(self.h, kernel, reps, C.byref(ms), C.byref(cells)),
               "acs_batch_time_kernel")
        return ms.value, cells.value


from . import configs  # noqa: E402  (uses the names above)

__all__ = ["Params", "Case", "Batch", "AcsError", "mesh_reference", "mesh_channel", "noise",
           "reference_jmax", "FIELDS", "field_shape", "configs", "lib", "device_count"]

"""Case builders: the reference driver's set-up and the synthetic channel configurations.

``reference_case`` mirrors what ``PROGRAM main`` does before its loop (main.f90:34-109,
initial.f90:30-43): compiled-in constants, the reference mesh, the initial condition
(vm = 1e-3 v_i, um = 0, p = 1, T = Tinf, C = 0, T = C = 1 in porous cells), um_tau = um and
vm_tau = vm, and every other loop array zero (they are uninitialised static arrays in the
reference, i.e. zero).

``channel_case`` builds the synthetic channel configurations: a rectangular domain with aspect
ratio Lx:Ly = 2:1, inflow u = 1 on the left, outflow on the right and no-slip walls, y clustered
toward the walls by a tanh map, an optional centred (or placed) porous block, and seeded uniform
noise on the interior velocities.  Their loop state starts from the initial condition (tau and
n_tau copies equal to it, pn = p).  Dataset stand-ins: these are seeded synthetic inputs with the
shapes, sizes and parameter ranges of the benchmark configurations; there is no public dataset.
"""
from __future__ import annotations

import math
from dataclasses import replace

import numpy as np

from . import (ARITH_EXACT, BC_CHANNEL, SCHEME_QUICK, SCHEME_UPWIND, Params, field_shape,
               mesh_channel, mesh_reference, noise, noise_array, reference_jmax)

# The case builders draw meshes and noise from a generator backend: by default this package's C
# ABI (acs_mesh_channel, acs_noise, acs_noise_array); any module with the same mesh_channel(nx, ny,
# Lx, Ly, stretch, block, porosity, block2), noise(seed, case_id, field, index, amp) and
# noise_array(seed, case_id, field, index, amp) functions can stand in (the CPU oracle has all
# three, so a run that must not load this package's library can still build the identical cases).
_backend = None


def use_backend(module) -> None:
    """Make the case builders draw meshes and noise from `module` (None: this package)."""
    global _backend
    _backend = module


def _mesh_channel(*a, **k):
    return (_backend.mesh_channel if _backend is not None else mesh_channel)(*a, **k)


def _noise_array(*a, **k):
    return (_backend.noise_array if _backend is not None else noise_array)(*a, **k)


def _noise(*a, **k):
    return (_backend.noise if _backend is not None else noise)(*a, **k)

# field ids of the noise generator (shared by specification with the oracle tests)
NOISE_U, NOISE_V, NOISE_PARAM = 1, 2, 100


def n_physical_steps(final_time: float, dt: float) -> int:
    """Number of passes of `DO WHILE (time .LT. final_time); time = time + dt` (main.f90:116-117)."""
    t, n = 0.0, 0
    while t < final_time:
        t = t + dt
        n += 1
    return n


def zero_state(nx: int, ny: int) -> dict:
    names = ("um", "vm", "um_tau", "vm_tau", "um_n_tau", "vm_n_tau", "p", "pn",
             "T", "T_tau", "T_n_tau", "C", "C_tau", "C_n_tau")
    return {n: np.zeros(field_shape(n, nx, ny), order="F") for n in names}


def reference_case(imax: int = 51, **overrides):
    """Reference driver set-up.  Returns (params, mesh, state, itc0, n_steps)."""
    jmax = reference_jmax(imax)
    prm = replace(Params(imax=imax, jmax=jmax), **overrides)
    mesh = mesh_reference(imax, porosity=0.5)
    st = zero_state(imax, jmax)
    st["vm"][:] = 1.0e-3 * prm.v_in
    st["um"][:] = 0.0
    st["p"][:] = 1.0
    st["T"][:] = prm.T_in  # T = Tinf
    st["C"][:] = 0.0
    porous = mesh["flag"] != 0
    st["T"][porous] = 1.0  # Temp_cylinder
    st["C"][porous] = 1.0  # concentracao_inicial
    st["um_tau"][:] = st["um"]
    st["vm_tau"][:] = st["vm"]
    return prm, mesh, st, 1, n_physical_steps(1.0, prm.dt)


def centred_block(Lx, Ly, frac):
    w, h = math.sqrt(frac) * Lx, math.sqrt(frac) * Ly
    return (0.5 * (Lx - w), 0.5 * (Lx + w), 0.5 * (Ly - h), 0.5 * (Ly + h))


def stable_dtau(mesh, beta, dt, safety=0.85):
    """Largest pseudo step the three-stage Runge-Kutta loop tolerates for the artificial-
    compressibility (pressure-velocity) mode: with the volume-divided continuity its eigenvalues
    are about +-i sqrt(beta dt) 2 sqrt(1/dx^2 + 1/dy^2) per unit pseudo time, and SSP-RK3 is
    stable on the imaginary axis up to sqrt(3).  `safety` < 1 keeps a margin."""
    dx = np.diff(mesh["x"]).min()
    dy = np.diff(mesh["y"]).min()
    lam = math.sqrt(beta * dt) * 2.0 * math.sqrt(1.0 / dx ** 2 + 1.0 / dy ** 2)
    return float(np.float64(safety * math.sqrt(3.0) / lam).round(6))


def channel_case(nx, ny, *, seed=0, case_id=0, Re=100.0, scheme=SCHEME_QUICK, block=None,
                 block2=None, porosity=1.0, Da=1.0, Cf=0.0, Ri=0.0, Pr=0.7, Sc=1.0,
                 scalars=False, beta=1.0, dt=1.0e-3, dtau=None, eps=1.0e-6, itc_max=1000000,
                 noise_amp=1.0e-3, T_block=2.0, Lx=2.0, Ly=1.0, stretch=1.5, arith=ARITH_EXACT,
                 continuity=1):
    """Channel configuration.  Returns (params, mesh, state, itc0).  dtau=None picks
    stable_dtau() for the mesh."""
    mesh = _mesh_channel(nx, ny, Lx, Ly, stretch, block, porosity, block2)
    if dtau is None:
        dtau = stable_dtau(mesh, beta, dt)
    prm = Params(imax=nx, jmax=ny, scheme=scheme, bc=BC_CHANNEL, solve_scalars=int(scalars),
                 itc_max=itc_max, Re=Re, Pe=Re * Pr, Sc=Sc, Da=Da, Cf=Cf, g=0.0, InvFr2=Ri,
                 v_in=1.0, T_in=1.0, C_in=1.0, b_art=0.0, beta=beta, dt=dt, dtau=dtau, eps=eps,
                 arith=arith, continuity=continuity)
    st = zero_state(nx, ny)
    um, vm = st["um"], st["vm"]
    # u update region i = 3..nx-1, j = 2..ny-1; v update region i = 2..nx-1, j = 3..ny-1;
    # noise index = the Fortran linear index (i-1) + (j-1)*leading dimension
    I, J = np.meshgrid(np.arange(3, nx), np.arange(2, ny), indexing="ij")
    um[I - 1, J - 1] = _noise_array(seed, case_id, NOISE_U, ((I - 1) + (J - 1) * (nx + 1)).ravel(),
                                   noise_amp).reshape(I.shape)
    I, J = np.meshgrid(np.arange(2, nx), np.arange(3, ny), indexing="ij")
    vm[I - 1, J - 1] = _noise_array(seed, case_id, NOISE_V, ((I - 1) + (J - 1) * nx).ravel(),
                                   noise_amp).reshape(I.shape)
    porous = mesh["flag"] != 0
    st["T"][:] = 1.0
    st["T"][porous] = T_block if scalars else 1.0
    st["C"][:] = 0.0
    st["C"][porous] = 1.0 if scalars else 0.0
    for a, b in (("um_tau", "um"), ("vm_tau", "vm"), ("um_n_tau", "um"), ("vm_n_tau", "vm"),
                 ("pn", "p"), ("T_tau", "T"), ("T_n_tau", "T"), ("C_tau", "C"), ("C_n_tau", "C")):
        st[a][:] = st[b]
    return prm, mesh, st, 1


# ---- benchmark configurations ---------------------------------------------------------------
def cfg_plain(n=51, **kw):
    """Plain method, FP64, isothermal, no porous block, no scalars: 51 x 51 stretched mesh of a
    2:1 channel, inflow u=1, Re=100, first-order upwind, beta=1, dt=1e-3, residual 1e-6,
    200 physical steps from rest plus seeded 1e-3 uniform noise (seed 0)."""
    args = dict(seed=0, Re=100.0, scheme=SCHEME_UPWIND, scalars=False, beta=1.0, dt=1.0e-3, eps=1.0e-6)
    args.update(kw)
    prm, mesh, st, itc = channel_case(n, n, **args)
    return prm, mesh, st, itc, 200


def cfg_full(n=102, **kw):
    """Full equation set, QUICK: n x n stretched mesh, centred porous block over 30% of the
    domain (porosity 0.4, Da=1e-3, Cf=0.55), buoyancy Ri=1, Pr=0.7, scalars T and C with
    inflow value 1, Re=200, 500 physical steps, seed 1."""
    Lx, Ly = 2.0, 1.0
    args = dict(seed=1, Re=200.0, scheme=SCHEME_QUICK, block=centred_block(Lx, Ly, 0.3), porosity=0.4,
                Da=1.0e-3, Cf=0.55, Ri=1.0, Pr=0.7, Sc=1.0, scalars=True, beta=1.0, dt=1.0e-3, eps=1.0e-6)
    args.update(kw)
    prm, mesh, st, itc = channel_case(n, n, **args)
    return prm, mesh, st, itc, 500


def uniform01(seed, case_id, k):
    return 0.5 * (_noise(seed, case_id, NOISE_PARAM + k, 0, 1.0) + 1.0)


def batch_case_params(case_id, seed=0, sizes=(51, 102, 153, 204)):
    """Parameters of one case of the batched configuration: nx, ny uniform over `sizes`,
    Re ~ U[50,500], Da ~ logU[1e-5,1e-2], porosity ~ U[0.3,0.9], Ri ~ U[0,2], a porous block of
    30% area whose centre is uniform over the positions that keep it inside the domain."""
    u = [uniform01(seed, case_id, k) for k in range(8)]
    ns = len(sizes)
    nx = sizes[min(int(u[0] * ns), ns - 1)]
    ny = sizes[min(int(u[1] * ns), ns - 1)]
    Re = 50.0 + 450.0 * u[2]
    Da = 10.0 ** (-5.0 + 3.0 * u[3])
    por = 0.3 + 0.6 * u[4]
    Ri = 2.0 * u[5]
    Lx, Ly = 2.0, 1.0
    w, h = math.sqrt(0.3) * Lx, math.sqrt(0.3) * Ly
    cx = 0.5 * w + (Lx - w) * u[6]
    cy = 0.5 * h + (Ly - h) * u[7]
    block = (cx - 0.5 * w, cx + 0.5 * w, cy - 0.5 * h, cy + 0.5 * h)
    return dict(nx=nx, ny=ny, Re=Re, Da=Da, porosity=por, Ri=Ri, block=block)


def cfg_batch(n_cases=256, seed=0, sizes=(51, 102, 153, 204), **kw):
    """Batched configuration: n_cases independent seeded cases with the full equation set, QUICK,
    200 physical steps each.  Returns a list of (params, mesh, state, itc) and the step count."""
    out = []
    for c in range(n_cases):
        q = batch_case_params(c, seed, sizes)
        args = dict(seed=seed, case_id=c, Re=q["Re"], scheme=SCHEME_QUICK, block=q["block"],
                    porosity=q["porosity"], Da=q["Da"], Cf=0.55, Ri=q["Ri"], Pr=0.7, Sc=1.0,
                    scalars=True, beta=1.0, dt=1.0e-3, eps=1.0e-6)
        args.update(kw)
        out.append(channel_case(q["nx"], q["ny"], **args))
    return out, 200


def cfg_large(nx=1024, ny=512, **kw):
    """The combined configuration's single large case: nx x ny stretched 2:1 channel with two
    porous blocks (each 10 % of the area, centred at x = Lx/4 and 3Lx/4), porosity 0.4, Da 1e-3,
    Cf 0.55, Ri 1, Pr 0.7, Sc 1, scalars T and C with inflow value 1, Re 400, QUICK, 1000
    physical steps, seed 2.  Returns (params, mesh, state, itc, n_steps)."""
    Lx, Ly = 2.0, 1.0
    w, h = math.sqrt(0.1) * Lx, math.sqrt(0.1) * Ly

    def box(cx):
        return (cx - 0.5 * w, cx + 0.5 * w, 0.5 * (Ly - h), 0.5 * (Ly + h))

    args = dict(seed=2, Re=400.0, scheme=SCHEME_QUICK, block=box(0.25 * Lx), block2=box(0.75 * Lx),
                porosity=0.4, Da=1.0e-3, Cf=0.55, Ri=1.0, Pr=0.7, Sc=1.0, scalars=True, beta=1.0,
                dt=1.0e-3, eps=1.0e-6)
    args.update(kw)
    prm, mesh, st, itc = channel_case(nx, ny, **args)
    return prm, mesh, st, itc, 1000

"""The reference's module functions, re-expressed over liblbm3d.so.

Each function keeps the name (without Julia's `!`), argument order, argument meaning
and error behaviour of its counterpart in LBM3D_BB's src/ modules, so that a driver
written against the reference runs unchanged in spirit:

  read_params_input  Parameters.jl:87-164      gen_lattice_sets  Utilities.jl:945-993
  MotionLaw          Motion.jl:14-21           motion_at         Motion.jl:26-36
  motion             Motion.jl:41-122          collision         Collision.jl:14-45
  streaming          Streaming.jl:116-137      periodic_BC       OtherBC.jl:87-107
  solid_BC           SolidBC.jl:129-153        velocity_BC       OtherBC.jl:174-219
  compute_aero       MEA.jl:14-71              compute_macros    ComputeMacro.jl:53-83
  ref_area_lat       Utilities.jl:931-938      measure_Mlups     Utilities.jl:903-926
  main_simulation    MainCore.jl:48-395 (one partition, no MPI: rank 1 is the worker)

The populations live in the library (one fused kernel per step), so `f_old` and
`f_new` are handles on that storage (`PopulationHandle`).  `collision` runs the whole
fused step — collision, streaming, periodic copy, solid and face conditions, momentum
exchange and moments — so `streaming`, `periodic_BC`, `solid_BC` and `velocity_BC`
validate their arguments and return.  Every function is a no-op on rank 0 (the
reference's master), as in the reference.
"""
from __future__ import annotations

import math
import time
from dataclasses import dataclass, field
from typing import Callable, Optional

import numpy as np

from . import abi
from .domain import Domain, read_params

F32 = np.float32

COLLISIONS = ("BGK", "TRT")
# Solid boundary conditions of solid_BC!'s dispatch table (SolidBC.jl:99-123).
# "IBB" runs the bounce-back that IBB!_gpu executes for every link of the reference's
# bodies: it evaluates phi at x_b - c_dir (SolidBC.jl:290-292), the fluid node behind the
# boundary node, so for a convex body (cylinder, symmetric NACA band) phi_s >= 0 holds,
# no_brkt is true and the kernel takes its fallback (SolidBC.jl:306-319), which is the
# SBB!_gpu formula term for term (wall point x_b - c/2, local rho, 2 w rho (c.u_w)/cs^2).
# Its interpolating branch would need EPS_Q, defined nowhere in the reference, so it
# cannot execute as shipped.
SOLID_BCS = ("SBB", "IBB")


# ---- parameters ---------------------------------------------------------------------------
@dataclass
class LBMParams:
    """Parameters.jl:8-47 (FP32 fields, derived nu/omega_p/omega_m as the constructor)."""

    Nx: int
    Ny: int
    Nz: int
    h: np.float32
    R: np.float32
    x_c: np.float32
    y_c: np.float32
    theta0: np.float32
    q: int
    Re: np.float32
    U_inf: np.float32
    V_inf: np.float32
    W_inf: np.float32
    rho_inf: np.float32
    dt: np.float32
    n_max: int
    n_save: int
    nu: np.float32
    omega_p: np.float32
    omega_m: np.float32
    Lambda: np.float32
    bc: str
    coll: str
    shape: str  # "CYL" or "AIR"
    naca_code: Optional[str]
    chord: np.float32


def read_params_input(path: str) -> LBMParams:
    """read_params_input (Parameters.jl:87-164); raises LbmError(status 5) where the
    reference raises its AssertionError."""
    p = read_params(path)
    return LBMParams(p.Nx, p.Ny, p.Nz, F32(p.h), F32(p.R), F32(p.x_c), F32(p.y_c), F32(p.theta0), p.q, F32(p.Re),
                     F32(p.U_inf), F32(p.V_inf), F32(p.W_inf), F32(p.rho_inf), F32(p.dt), p.n_max, p.n_save,
                     F32(p.nu), F32(p.omega_p), F32(p.omega_m), F32(p.Lambda), p.bc.decode(), p.coll.decode(),
                     "CYL" if p.shape == 1 else "AIR", p.naca_code.decode() or None, F32(p.chord))


def gen_lattice_sets(params: LBMParams):
    """(c_x, c_y, c_z, W, bbOpp) with the reference's 1-based bbOpp (Utilities.jl:949-960)."""
    if params.q not in (19, 27):
        raise ValueError("Invalid q value!" if params.q != 3 else "q=3: D1Q3 is not implemented by liblbm3d")
    from .domain import lattice

    cx, cy, cz, w, op = lattice(params.q)
    return cx, cy, cz, w, (op + 1).astype(np.int8)


def ref_area_lat(shape: str, R, chord, Nz: int, h) -> np.float32:
    """Utilities.jl:931-938."""
    Lz = F32(Nz)
    return (F32(2) * F32(R) / F32(h)) * Lz if shape == "CYL" else (F32(chord) / F32(h)) * Lz


def measure_Mlups(t_start_ns: int, t_end_ns: int, t_ini_ns: int, Nx: int, Ny: int, Nz: int, n_max: int) -> float:
    """Utilities.jl:903-926: all cells, wall time of the loop."""
    s = (t_end_ns - t_start_ns) / 1e9
    return Nx * Ny * Nz * n_max / (s * 1e6)


# ---- motion -------------------------------------------------------------------------------
@dataclass
class MotionLaw:
    """Motion.jl:14-21: closures of t (physical time) for the planar rigid motion."""

    x: Callable
    xdot: Callable
    y: Callable
    ydot: Callable
    theta: Callable
    thetadot: Callable


def motion_at(n: int, dt, m: MotionLaw, offset=0.0) -> dict:
    """Motion.jl:26-36: pose at t = (n-1+offset)*dt, every field rounded to Float32."""
    t = (F32(n - 1) + F32(offset)) * F32(dt)
    return dict(x_c=F32(m.x(t)), y_c=F32(m.y(t)), theta=F32(m.theta(t)), U_c=F32(m.xdot(t)), V_c=F32(m.ydot(t)),
                omega=F32(m.thetadot(t)))


def main_core_law(params: LBMParams) -> MotionLaw:
    """The heaving law of MainCore.jl:72-80 (FP32)."""
    R, U = params.R, params.U_inf
    Ae = F32(0.2) * F32(2) * R
    fe = F32(0.154) * U / (F32(2) * R)
    we = F32(2) * F32(math.pi) * fe
    return MotionLaw(lambda t: params.x_c, lambda t: F32(0), lambda t: params.y_c - Ae * np.sin(we * F32(t)),
                     lambda t: -Ae * we * np.cos(we * F32(t)), lambda t: params.theta0, lambda t: F32(0))


# ---- population handles -----------------------------------------------------------------------
@dataclass
class PopulationHandle:
    """Stands for f_old / f_new: both name the library's population storage."""

    domain: Domain
    role: str = "f_old"


@dataclass
class SolidBCStruct:
    """SolidBC.jl:13-43, the fields the fused step uses (half-step kinematics)."""

    U_c_lat: np.float32 = F32(0)
    V_c_lat: np.float32 = F32(0)
    omega_lat: np.float32 = F32(0)
    x_c_lat: np.float32 = F32(0)
    y_c_lat: np.float32 = F32(0)
    nnz: int = 0


def _worker(rank: int) -> bool:
    return rank != 0


def motion(state: Domain, R, x_c, y_c, dt, h, bcstruct: SolidBCStruct, law: MotionLaw, n: int, rank: int):
    """motion! (Motion.jl:41-122): pose at (n-1)dt for the flags, half-step kinematics in
    lattice units for the moving-wall bounce-back (Motion.jl:96-100)."""
    if not _worker(rank):
        return
    pn = motion_at(n, dt, law, 0.0)
    ph = motion_at(n, dt, law, 0.5)
    th = pn["theta"]
    ct, st = F32(np.cos(th)), F32(np.sin(th))
    bcstruct.U_c_lat = ph["U_c"] * F32(dt) / F32(h)
    bcstruct.V_c_lat = ph["V_c"] * F32(dt) / F32(h)
    bcstruct.omega_lat = ph["omega"] * F32(dt)
    bcstruct.x_c_lat = ph["x_c"] / F32(h)
    bcstruct.y_c_lat = ph["y_c"] / F32(h)
    pose_n = abi.make_pose(center=(float(pn["x_c"]), float(pn["y_c"]), 0.0), cos_theta=float(ct), sin_theta=float(st))
    # half-time orientation for phi (the interpolated bounce-back, Motion.jl:117-119)
    th_h = ph["theta"]
    pose_h = abi.make_pose(center=(float(bcstruct.x_c_lat), float(bcstruct.y_c_lat), 0.0),
                           cos_theta=float(F32(np.cos(th_h))), sin_theta=float(F32(np.sin(th_h))),
                           vel=(float(bcstruct.U_c_lat), float(bcstruct.V_c_lat), 0.0),
                           omega=(0.0, 0.0, float(bcstruct.omega_lat)))
    state.update_body(pose_n, pose_h)


def collision(f_old: PopulationHandle, f_new: PopulationHandle, rho, u, v, w, c_x, c_y, c_z, wvec, bbOpp,
              omega_p, omega_m, coll: str, N_owned: int, rank: int):
    """collision! (Collision.jl:14-45): unknown methods raise as the reference's error();
    runs the fused step (collision through moments) once."""
    if coll not in COLLISIONS:
        raise ValueError(f"\nUnknown collision method: {coll}.\n")
    if not _worker(rank):
        return
    f_old.domain.step(1)


def streaming(f_pre, f_post, stream_lidxs, stream_mask, q: int, N_owned: int, rank: int):
    """streaming! (Streaming.jl:116-137): fused into `collision`."""
    return None


def periodic_BC(f_old, f_new, per_dest, per_dir, per_src, rank: int):
    """periodic_BC! (OtherBC.jl:87-107): fused into `collision`."""
    return None


def solid_BC(f_old, f_new, rho, wvec, c_x, c_y, x_lli_lat, y_lli_lat, bcstruct, params, bc: str, rank: int):
    """solid_BC! (SolidBC.jl:129-153): fused into `collision`; unknown BCs raise."""
    if rank == 0:
        return None
    if bc not in SOLID_BCS:
        raise ValueError(f"\n\nsolid_BC!: Unknown or unimplemented boundary condition: {bc}.\n\n")
    return None


def velocity_BC(f_old, f_new, vel_lidxs, vel_dirs, pres_lidxs, pres_dirs, bbOpp, c_x, c_y, c_z, wvec, rho, u, v, w,
                U_inf, V_inf, W_inf, rank: int):
    """velocity_BC! (OtherBC.jl:174-219): fused into `collision`."""
    return None


def compute_aero(step: int, n_save: int, n_max: int, f_new: PopulationHandle, f_old: PopulationHandle,
                 bcstruct: SolidBCStruct, bbOpp, c_x, c_y, c_z, CL, CD, CZ, fc_aero, comm, rank: int):
    """compute_aero! (MEA.jl:14-71): momentum-exchange force of this step (FP64 on the
    device), normalised in FP32 as CD = Px*fc, CL = Py*fc, CZ = Pz*fc; one partition,
    so the Allreduce is the identity.  Stores into CL/CD/CZ[step-1]."""
    if not _worker(rank):
        return None
    P = f_new.domain.force(step)
    fc = F32(fc_aero)
    CD[step - 1] = F32(P[0]) * fc
    CL[step - 1] = F32(P[1]) * fc
    CZ[step - 1] = F32(P[2]) * fc
    return P


def compute_macros(f: PopulationHandle, rho, u, v, w, c_x, c_y, c_z, rank: int):
    """compute_macros! (ComputeMacro.jl:53-83): rho, u, v, w of the current state into the
    caller's arrays (torch CUDA tensors: device copy; numpy arrays: host copy)."""
    if not _worker(rank):
        return None
    if hasattr(rho, "is_cuda") and rho.is_cuda:
        f.domain.macros_into(rho, u, v, w)
        return None
    r, uu, vv, ww = f.domain.macros(np.float32)
    for dst, src in ((rho, r), (u, uu), (v, vv), (w, ww)):
        if dst is not None:
            dst[...] = src.ravel()
    return None


# ---- the driver --------------------------------------------------------------------------------
@dataclass
class SimulationResult:
    CL: np.ndarray
    CD: np.ndarray
    CZ: np.ndarray
    snapshots: list = field(default_factory=list)  # (step, rho, u, v, w) every n_save steps
    mlups: float = 0.0
    domain: Optional[Domain] = None


def _shape_body(params: LBMParams) -> abi.LbmBody:
    """init_solid_mask_state (Geometry.jl:26-39)."""
    if params.shape == "CYL":
        return abi.make_body(abi.BODY_CYLINDER_Z, (float(params.x_c), float(params.y_c), 0.0),
                             radius=float(params.R), moving=True)
    code = params.naca_code or "0012"
    m, p, t = int(code[0]) / 100.0, int(code[1]) / 10.0, (10 * int(code[2]) + int(code[3])) / 100.0
    return abi.make_body(abi.BODY_NACA_Z, (float(params.x_c), float(params.y_c), 0.0), moving=True,
                         chord=float(params.chord), naca=(float(F32(m)), float(F32(p)), float(F32(t))),
                         x_int=float(F32(1.0089304)), x_le_offset=float(F32(0.25) * params.chord))


def main_simulation(params: LBMParams, *, n_max: Optional[int] = None, law: Optional[MotionLaw] = None,
                    seed: Optional[int] = 0, storage: str = "fp32", macros_every_step: bool = False,
                    device: int = 0, rank: int = 1, interpolated_ibb: bool = False) -> SimulationResult:
    """MainCore.jl:48-395 for one partition.  The reference's unseeded 20% velocity
    noise (Initialization.jl:27-32, 70) is drawn from numpy with `seed` (None: no
    noise).  Field snapshots are kept in memory every n_save steps instead of HDF5.
    BC "IBB" runs what the reference executes (its SBB fallback, see SOLID_BCS) unless
    `interpolated_ibb` asks for the interpolated bounce-back IBB!_gpu is written to be
    (lbm_config.solid_bc = LBM_SOLID_IBB)."""
    n_max = params.n_max if n_max is None else n_max
    law = law or main_core_law(params)
    if params.coll not in COLLISIONS:
        raise ValueError(f"\nUnknown collision method: {params.coll}.\n")
    if params.bc not in SOLID_BCS:
        raise ValueError(f"\n\ninit: Unknown or unimplemented boundary condition: {params.bc}.\n\n")
    t_ini = time.perf_counter_ns()
    Nx, Ny, Nz = params.Nx, params.Ny, params.Nz
    N = Nx * Ny * Nz
    A_ref = ref_area_lat(params.shape, params.R, params.chord, Nz, params.h)
    fc_aero = F32(1) / (F32(0.5) * params.rho_inf * (params.U_inf * params.U_inf) * A_ref)
    dom = Domain(Nx, Ny, Nz, mode="reference", collision=params.coll, storage=storage, omega_p=float(params.omega_p),
                 omega_m=float(params.omega_m), u_inf=(float(params.U_inf), float(params.V_inf), float(params.W_inf)),
                 h=float(params.h), force_history=max(16, min(n_max, 4096)), device=device,
                 solid_bc="IBB" if (interpolated_ibb and params.bc == "IBB") else "SBB", q=params.q)
    dom.add_body(_shape_body(params))
    if seed is None:
        r = np.zeros(N, np.float32)
    else:
        r = (F32(2) * np.random.default_rng(seed).random(N, dtype=np.float32) - F32(1)).astype(np.float32)
    fac = F32(1) + F32(0.2) * r
    dom.init_equilibrium(rho=np.full(N, float(params.rho_inf)), u=(params.U_inf * fac).astype(np.float64),
                         v=(params.V_inf * fac).astype(np.float64), w=(params.W_inf * fac).astype(np.float64))
    f_old, f_new = PopulationHandle(dom, "f_old"), PopulationHandle(dom, "f_new")
    bcs = SolidBCStruct()
    c_x, c_y, c_z, wvec, bbOpp = gen_lattice_sets(params)
    CL = np.zeros(n_max, np.float32)
    CD = np.zeros(n_max, np.float32)
    CZ = np.zeros(n_max, np.float32)
    rho = np.zeros(N, np.float32)
    u = np.zeros(N, np.float32)
    v = np.zeros(N, np.float32)
    w = np.zeros(N, np.float32)
    res = SimulationResult(CL, CD, CZ, domain=dom)
    dom.synchronize()
    t0 = time.perf_counter_ns()
    for n in range(1, n_max + 1):
        motion(dom, params.R, params.x_c, params.y_c, params.dt, params.h, bcs, law, n, rank)
        collision(f_old, f_new, rho, u, v, w, c_x, c_y, c_z, wvec, bbOpp, params.omega_p, params.omega_m,
                  params.coll, N, rank)
        streaming(f_new, f_old, None, None, params.q, N, rank)
        periodic_BC(f_old, f_new, None, None, None, rank)
        solid_BC(f_old, f_new, rho, wvec, c_x, c_y, None, None, bcs, params, params.bc, rank)
        velocity_BC(f_old, f_new, None, None, None, None, bbOpp, c_x, c_y, c_z, wvec, rho, u, v, w,
                    params.U_inf, params.V_inf, params.W_inf, rank)
        compute_aero(n, params.n_save, n_max, f_new, f_old, bcs, bbOpp, c_x, c_y, c_z, CL, CD, CZ, fc_aero, None, rank)
        if macros_every_step or n % params.n_save == 0:
            compute_macros(f_old, rho, u, v, w, c_x, c_y, c_z, rank)
        if n % params.n_save == 0:
            res.snapshots.append((n, rho.copy(), u.copy(), v.copy(), w.copy()))
    dom.synchronize()
    t1 = time.perf_counter_ns()
    res.mlups = measure_Mlups(t0, t1, t_ini, Nx, Ny, Nz, n_max)
    return res

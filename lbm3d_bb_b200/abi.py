"""ctypes mirrors of the structs and enums in include/lbm3d.h.

Importing this module loads no shared library; ``_capi`` binds the functions.
"""
from __future__ import annotations

import ctypes as C

ABI_VERSION = 1

# status codes
LBM_OK = 0
LBM_ERR_ARG = 1
LBM_ERR_CUDA = 2
LBM_ERR_STATE = 3
LBM_ERR_UNSUPPORTED = 4
LBM_ERR_PARSE = 5
LBM_ERR_NUMERIC = 6
LBM_ERR_CAPACITY = 7
LBM_ERR_TIMEOUT = 8

# solid boundary rule of the reference-mode step (lbm_config.solid_bc)
SOLID_SBB = 0
SOLID_IBB = 1
SOLID_BC = {"SBB": SOLID_SBB, "IBB": SOLID_IBB}

MODE_REFERENCE = 0
MODE_CONFIG = 1
COLL_BGK = 0
COLL_TRT = 1
STORE_FP32 = 0
STORE_FP64 = 1
STORE_FP16DEV = 2

FACE_PERIODIC = 0
FACE_WALL = 1
FACE_EQ_INLET = 2
FACE_OUTFLOW = 3
FACE_PRESSURE = 4
FACE_HALO = 5

BODY_CYLINDER_Z = 1
BODY_NACA_Z = 2
BODY_SPHERE = 3
BODY_ELLIPSOID = 4

LAYOUT_SOA = 0
LAYOUT_REFERENCE = 1
DTYPE_F32 = 0
DTYPE_F64 = 1
HOST = 0
DEVICE = 1

STORAGE = {"fp32": STORE_FP32, "fp64": STORE_FP64, "fp16dev": STORE_FP16DEV}
COLLISION = {"BGK": COLL_BGK, "TRT": COLL_TRT}
FACES = {"periodic": FACE_PERIODIC, "wall": FACE_WALL, "inlet": FACE_EQ_INLET, "outflow": FACE_OUTFLOW,
         "pressure": FACE_PRESSURE, "halo": FACE_HALO}


class LbmConfig(C.Structure):
    _fields_ = [
        ("nx", C.c_int32),
        ("ny", C.c_int32),
        ("nz", C.c_int32),
        ("q", C.c_int32),
        ("mode", C.c_int32),
        ("collision", C.c_int32),
        ("storage", C.c_int32),
        ("face", C.c_int32 * 6),
        ("compute_force", C.c_int32),
        ("omega_p", C.c_double),
        ("omega_m", C.c_double),
        ("rho0", C.c_double),
        ("face_u", (C.c_double * 3) * 6),
        ("accel", C.c_double * 3),
        ("u_inf", C.c_double * 3),
        ("h", C.c_double),
        ("force_history", C.c_int32),
        ("solid_bc", C.c_int32),
    ]


class LbmBody(C.Structure):
    _fields_ = [
        ("kind", C.c_int32),
        ("moving", C.c_int32),
        ("center", C.c_double * 3),
        ("radius", C.c_double),
        ("semi", C.c_double * 3),
        ("rot", C.c_double * 9),
        ("chord", C.c_double),
        ("naca_m", C.c_double),
        ("naca_p", C.c_double),
        ("naca_t", C.c_double),
        ("x_int", C.c_double),
        ("x_le_offset", C.c_double),
    ]


class LbmPose(C.Structure):
    _fields_ = [
        ("center", C.c_double * 3),
        ("cos_theta", C.c_double),
        ("sin_theta", C.c_double),
        ("rot", C.c_double * 9),
        ("vel", C.c_double * 3),
        ("omega", C.c_double * 3),
    ]


class LbmParams(C.Structure):
    _fields_ = [
        ("Nx", C.c_int32),
        ("Ny", C.c_int32),
        ("Nz", C.c_int32),
        ("h", C.c_float),
        ("R", C.c_float),
        ("x_c", C.c_float),
        ("y_c", C.c_float),
        ("theta0", C.c_float),
        ("q", C.c_int32),
        ("Re", C.c_float),
        ("U_inf", C.c_float),
        ("V_inf", C.c_float),
        ("W_inf", C.c_float),
        ("rho_inf", C.c_float),
        ("dt", C.c_float),
        ("n_max", C.c_int32),
        ("n_save", C.c_int32),
        ("nu", C.c_float),
        ("omega_p", C.c_float),
        ("omega_m", C.c_float),
        ("Lambda", C.c_float),
        ("bc", C.c_char * 16),
        ("coll", C.c_char * 16),
        ("shape", C.c_int32),
        ("naca_code", C.c_char * 8),
        ("chord", C.c_float),
    ]


def make_pose(center=(0.0, 0.0, 0.0), theta=None, cos_theta=None, sin_theta=None, rot=None, vel=(0.0, 0.0, 0.0),
              omega=(0.0, 0.0, 0.0)) -> LbmPose:
    """Builds an LbmPose; planar rotation from theta (or explicit cos/sin)."""
    import math

    p = LbmPose()
    for k in range(3):
        p.center[k] = float(center[k]) if k < len(center) else 0.0
        p.vel[k] = float(vel[k]) if k < len(vel) else 0.0
        p.omega[k] = float(omega[k]) if k < len(omega) else 0.0
    if cos_theta is None:
        th = 0.0 if theta is None else float(theta)
        cos_theta, sin_theta = math.cos(th), math.sin(th)
    p.cos_theta = float(cos_theta)
    p.sin_theta = float(sin_theta)
    if rot is None:
        rot = (cos_theta, -sin_theta, 0.0, sin_theta, cos_theta, 0.0, 0.0, 0.0, 1.0)
    for k in range(9):
        p.rot[k] = float(rot[k])
    return p


def make_body(kind: int, center, radius=0.0, semi=(0.0, 0.0, 0.0), rot=None, moving=False, chord=0.0, naca=(0.0, 0.0, 0.0),
              x_int=1.0089304, x_le_offset=0.0) -> LbmBody:
    b = LbmBody()
    b.kind = int(kind)
    b.moving = 1 if moving else 0
    for k in range(3):
        b.center[k] = float(center[k]) if k < len(center) else 0.0
        b.semi[k] = float(semi[k])
    b.radius = float(radius)
    if rot is not None:
        for k in range(9):
            b.rot[k] = float(rot[k])
    b.chord = float(chord)
    b.naca_m, b.naca_p, b.naca_t = (float(v) for v in naca)
    b.x_int = float(x_int)
    b.x_le_offset = float(x_le_offset)
    return b


def make_config(nx, ny, nz, *, mode=MODE_CONFIG, collision="BGK", storage="fp32", faces=("periodic",) * 6,
                omega_p=1.0, omega_m=None, rho0=1.0, face_u=None, accel=(0.0, 0.0, 0.0), u_inf=(0.0, 0.0, 0.0),
                h=1.0, compute_force=True, force_history=1024, solid_bc="SBB", q=19) -> LbmConfig:
    c = LbmConfig()
    c.nx, c.ny, c.nz = int(nx), int(ny), int(nz)
    c.q = int(q)
    c.mode = int(mode)
    c.collision = COLLISION[collision] if isinstance(collision, str) else int(collision)
    c.storage = STORAGE[storage] if isinstance(storage, str) else int(storage)
    for k in range(6):
        f = faces[k]
        c.face[k] = FACES[f] if isinstance(f, str) else int(f)
    c.compute_force = 1 if compute_force else 0
    c.omega_p = float(omega_p)
    c.omega_m = float(omega_m if omega_m is not None else omega_p)
    c.rho0 = float(rho0)
    if face_u is not None:
        for k in range(6):
            for a in range(3):
                c.face_u[k][a] = float(face_u[k][a])
    for a in range(3):
        c.accel[a] = float(accel[a])
        c.u_inf[a] = float(u_inf[a])
    c.h = float(h)
    c.force_history = int(force_history)
    c.solid_bc = SOLID_BC[solid_bc] if isinstance(solid_bc, str) else int(solid_bc)
    return c

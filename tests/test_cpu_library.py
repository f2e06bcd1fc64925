"""CPU checks of the C ABI: the library loads without a GPU, exports every entry point
include/lbm3d.h declares, reads params.txt exactly as read_params_input does
(Parameters.jl:87-164 with the LBMParams constructor, Parameters.jl:49-81), and refuses to
run without a CUDA device instead of falling back to the CPU.
"""
import ctypes
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

from lbm3d_bb_b200 import abi
from lbm3d_bb_b200._capi import LIB_PATH, LbmError, exported_symbols, lib
from lbm3d_bb_b200.domain import read_params

ROOT = Path(__file__).resolve().parent.parent
GOLDEN = Path(__file__).resolve().parent / "golden"


def _declared():
    text = (ROOT / "include" / "lbm3d.h").read_text()
    return sorted(set(re.findall(r"^\s*(?:int32_t|int64_t|const char\*)\s+(lbm_\w+)\s*\(", text, re.M)))


def test_header_entry_points_are_exported():
    if not LIB_PATH.exists():
        from lbm3d_bb_b200 import build

        build.build()
    declared = _declared()
    assert len(declared) >= 28
    nm = subprocess.run(["nm", "-D", "--defined-only", str(LIB_PATH)], capture_output=True, text=True).stdout
    exported = set(re.findall(r"\sT\s(lbm_\w+)$", nm, re.M))
    assert set(declared) <= exported, set(declared) - exported
    assert set(declared) == set(exported_symbols())
    L = lib()  # binds every prototype; no GPU needed to load
    for name in declared:
        assert getattr(L, name) is not None
    assert L.lbm_abi_version() == abi.ABI_VERSION


def test_unet_header_entry_points_are_exported():
    from lbm3d_bb_b200 import build, unet

    if not unet.LIB_PATH.exists():
        build.build_unet()
    text = (ROOT / "include" / "unet3d.h").read_text()
    declared = sorted(set(re.findall(r"^\s*(?:int32_t|const char\*)\s+(nn_\w+)\s*\(", text, re.M)))
    nm = subprocess.run(["nm", "-D", "--defined-only", str(unet.LIB_PATH)], capture_output=True, text=True).stdout
    exported = set(re.findall(r"\sT\s(nn_\w+)$", nm, re.M))
    assert set(declared) <= exported, set(declared) - exported
    assert set(declared) == set(unet.exported_symbols())
    L = unet.lib()
    assert L.nn_abi_version() == 1


def test_lattice_constants():
    from lbm3d_bb_b200 import lattice

    cx, cy, cz, w, op = lattice()
    # gen_lattice_sets D3Q19 (Utilities.jl:950-960), 0-based opposites
    assert list(cx) == [1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 0, 0, 1, -1, 1, -1, 0, 0, 0]
    assert list(cy) == [0, 0, 1, -1, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 1, -1, 0]
    assert list(cz) == [0, 0, 0, 0, 1, -1, 0, 0, 1, -1, 1, -1, 0, 0, -1, 1, -1, 1, 0]
    assert list(op) == [1, 0, 3, 2, 5, 4, 7, 6, 9, 8, 11, 10, 13, 12, 15, 14, 17, 16, 18]
    assert w[0] == np.float32(1) / np.float32(18) and w[6] == np.float32(1) / np.float32(36)
    assert w[18] == np.float32(1) / np.float32(3)
    for d in range(19):
        o = op[d]
        assert (cx[o], cy[o], cz[o]) == (-cx[d], -cy[d], -cz[d])


def test_lattice_d3q27_constants_and_isotropy():
    from lbm3d_bb_b200 import lattice

    cx, cy, cz, w, op = lattice(27)
    # gen_lattice_sets D3Q27 (Utilities.jl:962-976), 0-based opposites
    assert list(cx) == [1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 0, 0, 1, -1, 1, -1, 0, 0, 1, -1, 1, -1, 1, -1, -1, 1, 0]
    assert list(cy) == [0, 0, 1, -1, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 1, -1, 1, -1, 1, -1, -1, 1, 1, -1, 0]
    assert list(cz) == [0, 0, 0, 0, 1, -1, 0, 0, 1, -1, 1, -1, 0, 0, -1, 1, -1, 1, 1, -1, -1, 1, 1, -1, 1, -1, 0]
    assert list(op) == [d ^ 1 for d in range(26)] + [26]
    F = np.float32
    assert w[0] == F(2) / F(27) and w[6] == F(1) / F(54) and w[18] == F(1) / F(216) and w[26] == F(8) / F(27)
    c = np.stack([cx, cy, cz]).astype(np.float64)
    wd = w.astype(np.float64)
    # all 27 velocities distinct; the moments of a lattice with c_s^2 = 1/3
    assert len({(a, b, e) for a, b, e in zip(cx, cy, cz)}) == 27
    assert abs(wd.sum() - 1) < 1e-6
    assert np.allclose(c @ wd, 0, atol=1e-7)
    assert np.allclose((c * wd) @ c.T, np.eye(3) / 3, atol=1e-7)
    for d in range(27):
        o = op[d]
        assert (cx[o], cy[o], cz[o]) == (-cx[d], -cy[d], -cz[d])
    from lbm3d_bb_b200 import reference_api as ra

    p = ra.read_params_input(Path(__file__).resolve().parent / "golden" / "params_d3q27.txt")
    assert p.q == 27
    _, _, _, _, bbopp = ra.gen_lattice_sets(p)
    assert list(bbopp) == [2, 1, 4, 3, 6, 5, 8, 7, 10, 9, 12, 11, 14, 13, 16, 15, 18, 17, 20, 19, 22, 21, 24, 23, 26,
                           25, 27]


def _julia_read_params(path):
    """Restatement of read_params_input + LBMParams in Python/float32 (test oracle)."""
    F = np.float32
    values, bc, coll, shape, naca = [], None, None, "CYL", None
    num = re.compile(r"[+-]?\d+(?:\.\d*)?(?:[eE][+-]?\d+)?")
    for raw in Path(path).read_text().splitlines():
        line = raw.strip()
        if not line or line.startswith("#"):
            continue
        if line.startswith("BC:"):
            bc = re.match(r"^BC:\s*\|?\s*([A-Za-z0-9_+\-]+)", line).group(1)
        elif line.startswith("Coll:"):
            coll = re.match(r"^Coll:\s*\|?\s*([A-Za-z0-9_+\-]+)", line).group(1)
        elif line.startswith("Shape:"):
            shape = re.match(r"^Shape:\s*\|?\s*([A-Za-z]+)", line).group(1).upper()
            assert shape in ("CYL", "AIR")
        elif line.startswith("NACA:"):
            naca = re.match(r"^NACA:\s*\|?\s*([0-9]{4})", line).group(1)
        else:
            values.append(F(num.search(line).group(0)))
    assert len(values) == 19 and bc is not None
    coll = coll or "BGK"
    if shape == "AIR" and naca is None:
        naca = "0012"
    v = values
    h, R, chord, U, Re, Lam = v[3], v[4], v[8], v[11], v[10], v[16]
    L = ((F(2) * R) if shape == "CYL" else chord) / h
    nu = (U * L) / Re
    tau_p = F(0.5) + F(3) * nu
    tau_m = F(0.5) + Lam / (tau_p - F(0.5))
    return dict(Nx=int(v[0]), Ny=int(v[1]), Nz=int(v[2]), h=h, R=R, x_c=v[5], y_c=v[6],
                theta0=v[7] * (F(np.pi) / F(180)), chord=chord, q=int(v[9]), Re=Re, U_inf=U, V_inf=v[12],
                W_inf=v[13], rho_inf=v[14], dt=v[15], Lambda=Lam, n_max=int(v[17]), n_save=int(v[18]), nu=nu,
                omega_p=F(1) / tau_p, omega_m=F(1) / tau_m, bc=bc, coll=coll, shape=1 if shape == "CYL" else 2,
                naca=naca or "")


@pytest.mark.parametrize("name", ["params_cylinder.txt", "params_airfoil_defaults.txt"])
def test_read_params_matches_reference_semantics(name):
    p = read_params(GOLDEN / name)
    e = _julia_read_params(GOLDEN / name)
    for k in ("Nx", "Ny", "Nz", "q", "n_max", "n_save", "shape"):
        assert getattr(p, k) == e[k], k
    for k in ("h", "R", "x_c", "y_c", "theta0", "chord", "Re", "U_inf", "V_inf", "W_inf", "rho_inf", "dt",
              "Lambda", "nu", "omega_p", "omega_m"):
        assert np.float32(getattr(p, k)) == e[k], k  # bit-exact FP32
    assert p.bc.decode() == e["bc"] and p.coll.decode() == e["coll"] and p.naca_code.decode() == e["naca"]


def test_read_params_known_answers():
    p = read_params(GOLDEN / "params_cylinder.txt")
    # L = 2R/h = 33, nu = 0.05*33/150 = 0.011, tau+ = 0.533, tau- = 0.5 + 0.1875/0.033
    assert abs(p.nu - 0.011) < 1e-7 and abs(1 / p.omega_p - 0.533) < 1e-6
    assert abs(1 / p.omega_m - (0.5 + 0.1875 / 0.033)) < 1e-4
    assert p.coll == b"TRT" and p.naca_code == b"2412"
    q = read_params(GOLDEN / "params_airfoil_defaults.txt")
    assert q.shape == 2 and q.naca_code == b"0012" and q.coll == b"BGK" and q.Re == 1000.0


@pytest.mark.parametrize("name,msg", [
    ("params_missing_bc.txt", "Missing BC line"),
    ("params_17_numbers.txt", "Expected 19 numeric parameters, got 17"),
    ("params_noninteger.txt", "InexactError"),
    ("params_bad_shape.txt", "Shape must be CYL or AIR"),
])
def test_read_params_errors(name, msg):
    with pytest.raises(LbmError) as ei:
        read_params(GOLDEN / name)
    assert ei.value.status == abi.LBM_ERR_PARSE and msg in str(ei.value)


def test_invalid_config_rejected_before_device_use():
    L = lib()
    h = ctypes.c_void_p()
    bad = abi.make_config(8, 8, 8, faces=("periodic", "wall", "periodic", "periodic", "periodic", "periodic"))
    assert L.lbm_create(ctypes.byref(bad), 0, ctypes.byref(h)) == abi.LBM_ERR_ARG
    assert b"both faces periodic" in L.lbm_global_error()
    q27 = abi.make_config(8, 8, 8)
    q27.q = 27
    assert L.lbm_create(ctypes.byref(q27), 0, ctypes.byref(h)) == abi.LBM_ERR_UNSUPPORTED


def test_no_cpu_fallback_without_gpu():
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    from lbm3d_bb_b200 import Domain

    with pytest.raises(LbmError) as ei:
        Domain(16, 16, 16)
    assert ei.value.status == abi.LBM_ERR_CUDA

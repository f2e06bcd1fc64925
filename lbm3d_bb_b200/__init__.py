"""lbm3d_bb_b200 — sm_100a implementation of the LBM3D_BB single-domain time step.

The compute path is liblbm3d.so (CUDA C++ for sm_100a, C ABI in include/lbm3d.h).
``Domain`` is the Python handle on one lattice; ``reference_api`` mirrors the
reference's Julia module functions (collision!, streaming!, ...) on top of it.
"""
from .abi import make_body, make_config, make_pose  # noqa: F401
from .domain import Domain, LbmError, lattice, read_params  # noqa: F401

__all__ = ["Domain", "LbmError", "lattice", "read_params", "make_body", "make_config", "make_pose"]

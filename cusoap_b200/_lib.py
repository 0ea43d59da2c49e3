"""ctypes binding of libsoapb200.so (the C ABI declared in include/soapb200.h).

The library is the only compute path: importing this module without the
built library raises, so nothing silently falls back to a CPU implementation.
"""
from __future__ import annotations

import ctypes
import os
from ctypes import POINTER, c_char_p, c_double, c_int32, c_int64, c_void_p

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libsoapb200.so")

OK, ERR_ARG, ERR_CUDA, ERR_CAPACITY, ERR_UNSUPPORTED, ERR_ACCURACY = range(6)
OUT_PS, OUT_CC, OUT_RAW = 0, 1, 2
NL_CREATE, NL_ALL = 0, 1
RBF_GTO, RBF_POLY = 0, 1
W_NONE, W_W0, W_POLY, W_POW, W_EXP = range(5)

# Every symbol include/soapb200.h declares (checked by the CPU test suite).
EXPORTS = (
    "soapb_basis_plan", "soapb_basis_build", "soapb_basis_download",
    "soapb_neighbors_workspace", "soapb_neighbors_count", "soapb_neighbors_fill", "soapb_neighbors_status",
    "soapb_neighbors_stats", "soapb_neighbors_clamp", "soapb_neighbors_noalloc",
    "soapb_descriptor", "soapb_jacobian_workspace", "soapb_jacobian", "soapb_forces_workspace", "soapb_forces",
    "soapb_forces_status", "soapb_check_bounded_wait", "soapb_last_error", "soapb_version",
    "soapb_kernel_launches",
)


class Basis(ctypes.Structure):
    _fields_ = [
        ("n_max", c_int32), ("l_max", c_int32), ("n_species", c_int32), ("crossover", c_int32),
        ("r_cut", c_double), ("sigma", c_double),
        ("rbf", c_int32), ("weighting", c_int32),
        ("w_r0", c_double), ("w_c", c_double), ("w_d", c_double), ("w_m", c_double), ("w_w0", c_double),
        ("quad_n", c_int32), ("seg_hint", c_int32), ("tune", c_int32 * 4), ("h_poly", c_void_p),
        ("eta", c_double), ("cutoff", c_double), ("seg_width", c_double),
        ("n_seg", c_int32), ("n_keys", c_int32), ("n_feat_ps", c_int32), ("n_feat_cc", c_int32),
        ("bytes", c_int64),
        ("off_alpha", c_int64), ("off_beta", c_int64), ("off_tab_b", c_int64), ("off_tab_bh", c_int64),
        ("off_ftab", c_int64), ("off_widx", c_int64), ("off_err", c_int64),
        ("off_tabf", c_int64), ("off_self", c_int64), ("off_poly", c_int64),
        ("dev", c_void_p),
    ]


class Structs(ctypes.Structure):
    _fields_ = [
        ("n_struct", c_int32), ("n_atoms", c_int64),
        ("d_atom_off", c_void_p), ("d_positions", c_void_p), ("d_species", c_void_p),
        ("d_cells", c_void_p), ("d_pbc", c_void_p),
    ]


class Centres(ctypes.Structure):
    _fields_ = [("n_centres", c_int64), ("d_xyz", c_void_p), ("d_struct", c_void_p), ("d_atom", c_void_p)]


class SoapbError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"soapb status {status}: {message}")
        self.status = status


_lib = None


def load() -> ctypes.CDLL:
    """Load the shared library (once); raise if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `python -m cusoap_b200.build` "
                          "(there is no CPU fallback)")
    lib = ctypes.CDLL(LIB_PATH)
    P = c_void_p
    sig = {
        "soapb_basis_plan": [POINTER(Basis)],
        "soapb_basis_build": [POINTER(Basis), P, P],
        "soapb_basis_download": [POINTER(Basis), P, P, P, P],
        "soapb_neighbors_workspace": [POINTER(Basis), POINTER(Structs), POINTER(Centres), POINTER(c_int64)],
        "soapb_neighbors_count": [POINTER(Basis), POINTER(Structs), POINTER(Centres), c_int32, P, c_int64, P, P],
        "soapb_neighbors_fill": [POINTER(Basis), POINTER(Structs), POINTER(Centres), c_int32, P, c_int64, P, P,
                                 c_int64, P],
        "soapb_neighbors_status": [POINTER(Basis), POINTER(Structs), POINTER(Centres), P, POINTER(c_int32), P],
        "soapb_neighbors_stats": [POINTER(Basis), POINTER(Structs), POINTER(Centres), P, P, P, P],
        "soapb_neighbors_clamp": [P, c_int64, c_int64, P, P],
        "soapb_neighbors_noalloc": [POINTER(Basis), POINTER(Structs), POINTER(Centres), c_int32, P, P, c_int64, P,
                                    P],
        "soapb_descriptor": [POINTER(Basis), c_int64, P, P, c_int32, P, P, P, P],
        "soapb_jacobian_workspace": [POINTER(Basis), c_int64, c_int64, c_int64, c_int32, POINTER(c_int64)],
        "soapb_jacobian": [POINTER(Basis), c_int64, P, P, c_int64, P, P, c_int64, P, c_int32, c_int32, c_int32, P,
                           P, c_int64, P, P],
        "soapb_forces_workspace": [POINTER(Basis), c_int64, POINTER(c_int64)],
        "soapb_forces": [POINTER(Basis), c_int64, P, P, P, P, c_int32, P, c_int32, P, P, c_int64, P, P],
        "soapb_forces_status": [POINTER(Basis), c_int64, P, POINTER(c_int32), P],
        "soapb_check_bounded_wait": [P, P],
    }
    for name, args in sig.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = c_int32
    lib.soapb_last_error.argtypes = []
    lib.soapb_last_error.restype = c_char_p
    lib.soapb_version.argtypes = []
    lib.soapb_version.restype = c_char_p
    lib.soapb_kernel_launches.argtypes = []
    lib.soapb_kernel_launches.restype = c_int64
    _lib = lib
    return lib


def check(status: int) -> None:
    if status != OK:
        msg = load().soapb_last_error().decode(errors="replace")
        raise SoapbError(status, msg)


def version() -> str:
    return load().soapb_version().decode()


def kernel_launches() -> int:
    """Kernels launched by the library in this process so far."""
    return int(load().soapb_kernel_launches())

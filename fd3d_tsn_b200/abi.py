"""ctypes view of the C ABI in ``include/fd3d_gpu.h``.

Only the structures and the library loader live here; ``solver.py`` holds the
Python mirror of the reference's interface built on top of it.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libfd3d_gpu.so")

FD3D_OK = 0
ERRORS = {
    -1: "FD3D_ERR_ARG", -2: "FD3D_ERR_CFL", -3: "FD3D_ERR_CUDA", -4: "FD3D_ERR_NOMEM",
    -5: "FD3D_ERR_NEWTON", -6: "FD3D_ERR_NONFINITE", -7: "FD3D_ERR_STATE", -8: "FD3D_ERR_IO",
    -9: "FD3D_ERR_NODEV", -10: "FD3D_ERR_BUSY",
}
LAW_SW, LAW_FVW = 0, 1
PREC_F32, PREC_F64 = 0, 1
MAX_STATIONS = 10
HIST_NAMES = ["sliprateX", "sliprateZ", "shearstressX", "shearstressZ", "psi"]
FIELDS = {"u": 0, "v": 1, "w": 2, "xx": 3, "yy": 4, "zz": 5, "xy": 6, "yz": 7, "xz": 8}
PLANES = {"tx": 0, "tz": 1, "slipX": 2, "slipZ": 3, "ruptime": 4, "rise": 5, "sliptime": 6,
          "distX": 7, "distZ": 8, "psiX": 9, "psiZ": 10, "T0X": 11, "T0Z": 12,
          "schangeX": 13, "schangeZ": 14, "rvel": 15, "czone": 16}
NKERNELS = 8
KERNEL_NAMES = ["vel_interior", "vel_fault", "vel_pml", "vel_fs",
                "str_interior", "str_fault", "str_pml", "fault_bc"]


class Fd3dError(RuntimeError):
    def __init__(self, code: int, where: str = ""):
        self.code = code
        super().__init__(f"{where}: {ERRORS.get(code, code)}")


class Params(C.Structure):
    _fields_ = [
        ("nxt", C.c_int), ("nyt", C.c_int), ("nzt", C.c_int),
        ("nabc", C.c_int), ("nfs", C.c_int), ("ntfd", C.c_int),
        ("dh", C.c_double), ("dt", C.c_double), ("damp_s", C.c_double),
        ("pml_vp", C.c_double), ("pml_fact", C.c_double), ("vp_max", C.c_double),
        ("law", C.c_int), ("precision", C.c_int), ("nstations", C.c_int),
        ("staX", C.c_int * MAX_STATIONS), ("staY", C.c_int * MAX_STATIONS), ("staZ", C.c_int * MAX_STATIONS),
        ("history_stride", C.c_int), ("history_capacity", C.c_int), ("fspace", C.c_int),
    ]


_DP = C.POINTER(C.c_double)


class Fault(C.Structure):
    _fields_ = [
        ("striniX", _DP), ("striniZ", _DP), ("Dc", _DP),
        ("peak_xz", _DP), ("dyn_xz", _DP), ("coh", _DP),
        ("a", _DP), ("b", _DP), ("psi", _DP), ("vw", _DP),
        ("aX", _DP), ("bX", _DP), ("psiX", _DP), ("vwX", _DP),
        ("fwZ", _DP), ("fwX", _DP),
        ("Sn", C.c_double), ("v0", C.c_double), ("f0", C.c_double), ("fw", C.c_double),
        ("uini", C.c_double), ("wini", C.c_double),
        ("nucleation", C.c_int),
        ("hx0", C.c_double), ("hz0", C.c_double), ("perturb", C.c_double), ("RR2", C.c_double),
        ("TT2", C.c_double), ("strinixI", C.c_double),
    ]


def fortran_plane(a) -> np.ndarray:
    """(nxt,nzt) array -> contiguous float64 buffer in Fortran order."""
    return np.asfortranarray(np.asarray(a, dtype=np.float64)).ravel(order="F")


def make_params(cfg: dict) -> Params:
    p = Params()
    for k in ("nxt", "nyt", "nzt", "nabc", "ntfd"):
        setattr(p, k, int(cfg[k]))
    p.fspace = 1 if cfg.get("fspace", False) else 0
    p.nfs = int(cfg.get("nfs", p.nabc if p.fspace else 2))
    for k in ("dh", "dt", "damp_s", "pml_vp", "pml_fact"):
        setattr(p, k, float(cfg[k]))
    p.vp_max = float(cfg.get("vp_max", 0.0))
    p.law = LAW_FVW if cfg.get("law", "sw") == "fvw" else LAW_SW
    p.precision = PREC_F64 if cfg.get("precision", "f32") == "f64" else PREC_F32
    st = cfg.get("stations", [])
    p.nstations = len(st)
    for s, (x, y, z) in enumerate(st):
        p.staX[s], p.staY[s], p.staZ[s] = int(x), int(y), int(z)
    p.history_stride = int(cfg.get("history_stride", 1))
    p.history_capacity = int(cfg.get("history_capacity", 0))
    return p


class FaultBuffers:
    """Keeps the float64 Fortran-order buffers alive while a Fault struct points at them."""

    SW_KEYS = ("striniX", "striniZ", "Dc", "peak_xz", "dyn_xz", "coh")
    FVW_KEYS = ("striniX", "striniZ", "Dc", "a", "b", "psi", "vw", "aX", "bX", "psiX", "vwX", "fwZ", "fwX")
    SCALARS = ("Sn", "v0", "f0", "fw", "uini", "wini", "hx0", "hz0", "perturb", "RR2", "TT2", "strinixI")

    def __init__(self, fault: dict):
        self.bufs = {}
        self.s = Fault()
        keys = self.FVW_KEYS if fault.get("law", "sw") == "fvw" else self.SW_KEYS
        for k in keys:
            if fault.get(k) is None:
                continue
            b = fortran_plane(fault[k])
            self.bufs[k] = b
            setattr(self.s, k, b.ctypes.data_as(_DP))
        for k in self.SCALARS:
            setattr(self.s, k, float(fault.get(k, 0.0)))
        self.s.nucleation = int(fault.get("nucleation", 0))


def load_library(path: str | None = None) -> C.CDLL:
    path = path or LIB_PATH
    if not os.path.exists(path):
        raise FileNotFoundError(
            f"{path} is missing: build it with `python -m fd3d_tsn_b200.build` (there is no CPU fallback)")
    lib = C.CDLL(path)
    i, vp, dp, fp = C.c_int, C.c_void_p, _DP, C.POINTER(C.c_float)
    sig = {
        "fd3d_version": (C.c_char_p, []),
        "fd3d_struct_sizes": (i, [C.POINTER(C.c_size_t), C.POINTER(C.c_size_t)]),
        "fd3d_status_string": (C.c_char_p, [i]),
        "fd3d_device_count": (i, [C.POINTER(i)]),
        "fd3d_set_device": (i, [i]),
        "fd3d_ctx_create": (i, [C.POINTER(Params), C.POINTER(vp)]),
        "fd3d_ctx_destroy": (i, [vp]),
        "fd3d_upload_medium": (i, [vp, vp, vp, vp, i]),
        "fd3d_upload_medium_layers": (i, [vp, dp, dp, dp]),
        "fd3d_upload_fault": (i, [vp, C.POINTER(Fault)]),
        "fd3d_reset": (i, [vp]),
        "fd3d_run": (i, [vp, i]),
        "fd3d_sync": (i, [vp]),
        "fd3d_steps_done": (i, [vp, C.POINTER(i)]),
        "fd3d_fetch_history": (i, [vp, i, i, i, vp, i]),
        "fd3d_history_records": (i, [vp, C.POINTER(i)]),
        "fd3d_fetch_stations": (i, [vp, i, i, dp]),
        "fd3d_fetch_field": (i, [vp, i, vp, i]),
        "fd3d_fetch_plane": (i, [vp, i, dp]),
        "fd3d_fetch_final": (i, [vp, dp, dp, dp, dp, dp]),
        "fd3d_write_results": (i, [vp, C.c_char_p, i]),
        "fd3d_last_run_ms": (i, [vp, fp]),
        "fd3d_set_profiling": (i, [vp, i]),
        "fd3d_kernel_times": (i, [vp, fp, C.POINTER(i)]),
        "fd3d_ctx_info": (i, [vp, C.POINTER(i), C.POINTER(i)]),
        "fd3d_read_deck": (i, [C.c_char_p, C.POINTER(Params), C.POINTER(dp), C.POINTER(dp), C.POINTER(dp)]),
        "fd3d_read_deck_ex": (i, [C.c_char_p, i, C.POINTER(Params), C.POINTER(dp), C.POINTER(dp), C.POINTER(dp)]),
        "fd3d_free": (None, [vp]),
        "fd3d_check_division": (i, [fp, i, C.POINTER(C.c_ulonglong), C.POINTER(C.c_uint)]),
        "fd3d_check_waits": (i, [C.POINTER(i), C.POINTER(i)]),
        "fd3d_checkpoint": (i, [vp, C.c_char_p]),
        "fd3d_restore": (i, [C.c_char_p, C.POINTER(vp)]),
        "fd3d_fetch_moment_rate": (i, [vp, i, i, dp]),
        "fd3d_post_process": (i, [vp, dp]),
        "fd3d_upload_fault_model": (i, [vp, i, i, dp, dp, dp, C.c_double, i]),
        "fd3d_ctx_create_slab": (i, [C.POINTER(Params), i, i, C.POINTER(vp)]),
        "fd3d_slab_range": (i, [vp, C.POINTER(i), C.POINTER(i)]),
        "fd3d_slab_plan": (i, [C.POINTER(Params), i, C.POINTER(i), C.POINTER(i)]),
        "fd3d_slab_halo_plan": (i, [i, i, i, C.POINTER(i), C.POINTER(i)]),
        "fd3d_slab_group_create": (i, [C.POINTER(vp), i, C.POINTER(vp)]),
        "fd3d_slab_group_run": (i, [vp, i]),
        "fd3d_slab_group_sync": (i, [vp, fp]),
        "fd3d_slab_group_destroy": (i, [vp]),
        "fd3d_nccl_unique_id": (i, [C.c_char_p]),
        "fd3d_slab_connect": (i, [vp, C.c_char_p, i, i]),
        "fd3d_slab_run": (i, [vp, i]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


def header_symbols(header: str) -> list[str]:
    """Function names declared in a C header (for the export check)."""
    import re
    txt = open(header).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:const\s+)?\w+\**\s+\**(fd3d_\w+)\s*\(", txt, flags=re.M)))

"""ctypes wrapper of the CPU oracle -- TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this
module, and only as the checker / the timed CPU restatement.  The GPU product never
imports it.  The oracle restates src/fd3d_deriv.f90 and src/fd3d_theo.f90 loop by
loop (see fd3d_oracle.cpp); parity is unpinned against the reference's own output
because the reference ships no golden outputs and no Fortran compiler is available.

Variants: 0 = FP32 fields + FP64 accumulators (the GPU FP32 build's arithmetic),
1 = all FP64 (the reference built with -r8), 2 = all FP32 (built without -r8).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle_fd3d.so")
MIXED, F64, F32 = 0, 1, 2

_LIB = None


def lib():
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            subprocess.run(["make", "-s", "-C", HERE], check=True)
        # the ctypes structures are shared with the product's ABI module
        from fd3d_tsn_b200 import abi
        L = C.CDLL(LIB_PATH)
        vp, dp = C.c_void_p, C.POINTER(C.c_double)
        L.oracle_create.restype = vp
        L.oracle_create.argtypes = [C.POINTER(abi.Params), C.c_int]
        L.oracle_destroy.argtypes = [vp]
        L.oracle_set_medium.argtypes = [vp, dp, dp, dp]
        L.oracle_set_fault.argtypes = [vp, C.POINTER(abi.Fault)]
        L.oracle_reset.argtypes = [vp]
        L.oracle_step.argtypes = [vp, C.c_int, dp, dp]
        L.oracle_get_field.argtypes = [vp, C.c_int, dp]
        L.oracle_get_plane.argtypes = [vp, C.c_int, dp]
        L.oracle_steps_done.argtypes = [vp]
        L.oracle_steps_done.restype = C.c_int
        L.oracle_moment_rate.argtypes = [vp, C.c_int, C.c_int, dp]
        L.oracle_post.argtypes = [vp, dp, dp, dp]
        L.oracle_set_fault_model.argtypes = [vp, C.c_int, C.c_int, dp, dp, dp, C.c_double, C.c_int]
        L.oracle_num_threads.restype = C.c_int
        L.oracle_set_threads.argtypes = [C.c_int]
        _LIB = L
    return _LIB


class Oracle:
    def __init__(self, model: dict, variant: int = MIXED):
        from fd3d_tsn_b200 import abi
        self.abi = abi
        self.model = model
        self.p = abi.make_params(model)
        self.h = lib().oracle_create(C.byref(self.p), variant)
        if not self.h:
            raise ValueError("oracle_create rejected the parameters")
        shp = (model["nxt"], model["nyt"], model["nzt"])
        lam, mu, d = (np.asfortranarray(np.broadcast_to(np.asarray(a, dtype=np.float64)[None, None, :], shp))
                      for a in model["medium"])
        dp = C.POINTER(C.c_double)
        lib().oracle_set_medium(self.h, lam.ctypes.data_as(dp), mu.ctypes.data_as(dp), d.ctypes.data_as(dp))
        if "fault_model" in model:  # control points of forwardmodel.dat
            fm = model["fault_model"]
            self.set_fault_model(fm["T0I"], fm["TsI"], fm["DcI"], dip=fm.get("dip", 90.0),
                                 dipslip=fm.get("dipslip", False))
        else:
            fb = abi.FaultBuffers(model["fault"])
            lib().oracle_set_fault(self.h, C.byref(fb.s))
        lib().oracle_reset(self.h)
        self.nxT = model["nxt"] - 2 * model["nabc"]
        self.nzT = model["nzt"] - model["nfs"] - model["nabc"]
        self.nst = len(model.get("stations", []))

    def set_medium_arrays(self, lam, mu, d):
        dp = C.POINTER(C.c_double)
        arrs = [np.asfortranarray(a, dtype=np.float64) for a in (lam, mu, d)]
        lib().oracle_set_medium(self.h, *(a.ctypes.data_as(dp) for a in arrs))

    def step(self, nsteps: int, history: bool = True):
        """Runs nsteps; returns (hist (nsteps,5,nztT,nxtT), seis (nsteps,nst,3)) or (None, None)."""
        dp = C.POINTER(C.c_double)
        hist = np.zeros((nsteps, 5, self.nzT, self.nxT)) if history else None
        seis = np.zeros((nsteps, max(self.nst, 1), 3)) if history else None
        rc = lib().oracle_step(self.h, int(nsteps), hist.ctypes.data_as(dp) if history else None,
                               seis.ctypes.data_as(dp) if history else None)
        self.last_rc = rc
        if history:
            seis = seis[:, :self.nst]
        return hist, seis

    def field(self, name):
        shp = (self.model["nxt"], self.model["nyt"], self.model["nzt"])
        out = np.empty(shp, order="F")
        lib().oracle_get_field(self.h, self.abi.FIELDS[name], out.ctypes.data_as(C.POINTER(C.c_double)))
        return out

    def plane(self, name):
        out = np.empty((self.model["nxt"], self.model["nzt"]), order="F")
        lib().oracle_get_plane(self.h, self.abi.PLANES[name], out.ctypes.data_as(C.POINTER(C.c_double)))
        return out

    def final(self):
        out = {k: self.plane(k) for k in ("slipX", "slipZ", "ruptime", "rise", "sliptime")}
        out["rise"] = out["rise"] - out["ruptime"]
        return out

    def set_fault_model(self, T0I, TsI, DcI, dip=90.0, dipslip=False):
        """Fault from control points (readinversionresult + inversion_modeltofd3d)."""
        arrs = [np.asfortranarray(a, dtype=np.float64) for a in (T0I, TsI, DcI)]
        nli, nwi = arrs[0].shape
        dp = C.POINTER(C.c_double)
        lib().oracle_set_fault_model(self.h, nli, nwi, *(a.ctypes.data_as(dp) for a in arrs), float(dip),
                                     int(dipslip))
        lib().oracle_reset(self.h)

    def steps_done(self) -> int:
        return int(lib().oracle_steps_done(self.h))

    def moment_rate(self, first: int = 0, n: int | None = None) -> np.ndarray:
        """Moment rate per step (fd3d_theo.f90:574-578 with dtseis = dt)."""
        n = self.steps_done() - first if n is None else n
        out = np.empty(n)
        rc = lib().oracle_moment_rate(self.h, first, n, out.ctypes.data_as(C.POINTER(C.c_double)))
        if rc:
            raise ValueError("oracle_moment_rate: bad range")
        return out

    def post(self):
        """Post-loop quantities (fd3d_theo.f90:604-749): summary (average rupture speed,
        seismic moment, rupture area = 0, average stress drop) and the rvel, czone planes."""
        n2 = self.model["nxt"] * self.model["nzt"]
        out, rv, cz = np.empty(4), np.empty(n2), np.empty(n2)
        dp = C.POINTER(C.c_double)
        lib().oracle_post(self.h, out.ctypes.data_as(dp), rv.ctypes.data_as(dp), cz.ctypes.data_as(dp))
        shp = (self.model["nxt"], self.model["nzt"])
        return out, rv.reshape(shp, order="F"), cz.reshape(shp, order="F")

    def close(self):
        if self.h:
            lib().oracle_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def set_threads(n: int):
    lib().oracle_set_threads(int(n))


def num_threads() -> int:
    return lib().oracle_num_threads()

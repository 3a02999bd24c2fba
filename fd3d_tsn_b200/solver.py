"""Python mirror of the reference's time-stepping interface over the C ABI.

The reference runs ``fd3d()`` (src/fd3d_theo.f90:22) on module state and writes the
result files; here one :class:`Solver` owns one forward model on the GPU:

    s = Solver(model)          # fd3d_init + forwardspecial* + init_pml/interp_fric
    s.run(model["ntfd"])       # the time loop, enqueued on the GPU
    s.sync()                   # raises Fd3dError on a device error (NEWTON, NONFINITE)
    s.write_results("result")  # sliprateX/Z.res, shearstressX/Z.res, stan*.txt, ...

Everything runs through ``libfd3d_gpu.so``; if the library is missing the import of
the solver fails loudly (there is no CPU path).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import abi

_LIB = None


def lib() -> C.CDLL:
    global _LIB
    if _LIB is None:
        _LIB = abi.load_library()
    return _LIB


def _ck(rc: int, where: str):
    if rc != abi.FD3D_OK:
        raise abi.Fd3dError(rc, where)


def device_count() -> int:
    n = C.c_int(0)
    _ck(lib().fd3d_device_count(C.byref(n)), "fd3d_device_count")
    return n.value


class Solver:
    def __init__(self, model: dict, medium3d: bool = False, slab: tuple[int, int] | None = None):
        """slab = (k_lo, k_hi): a context for those planes of the model only (a z-slab,
        stepped by :class:`fd3d_tsn_b200.slab.SlabSolver`)."""
        self.model = model
        self.p = abi.make_params(model)
        self.h = C.c_void_p()
        if slab is None:
            _ck(lib().fd3d_ctx_create(C.byref(self.p), C.byref(self.h)), "fd3d_ctx_create")
        else:
            _ck(lib().fd3d_ctx_create_slab(C.byref(self.p), int(slab[0]), int(slab[1]), C.byref(self.h)),
                "fd3d_ctx_create_slab")
        self.nxT = model["nxt"] - 2 * model["nabc"]
        self.nzT = model["nzt"] - model["nfs"] - model["nabc"]
        self.nf = 5 if model.get("law", "sw") == "fvw" else 4
        self.upload_medium(medium3d)
        if "fault_model" in model:  # control points of forwardmodel.dat (readinversionresult)
            self.upload_fault_model(**model["fault_model"])
        else:
            self.upload_fault(model["fault"])

    # ------------------------------------------------------------ inputs
    def upload_medium(self, medium3d: bool = False):
        lam, mu, d = (np.ascontiguousarray(a, dtype=np.float64) for a in self.model["medium"])
        if not medium3d:
            dp = C.POINTER(C.c_double)
            _ck(lib().fd3d_upload_medium_layers(self.h, lam.ctypes.data_as(dp), mu.ctypes.data_as(dp),
                                                d.ctypes.data_as(dp)), "fd3d_upload_medium_layers")
            return
        shp = (self.model["nxt"], self.model["nyt"], self.model["nzt"])
        arrs = [np.asfortranarray(np.broadcast_to(a[None, None, :], shp)) for a in (lam, mu, d)]
        _ck(lib().fd3d_upload_medium(self.h, *(a.ctypes.data for a in arrs), 8), "fd3d_upload_medium")

    def upload_medium_arrays(self, lam, mu, d, real_kind=8):
        dt = np.float64 if real_kind == 8 else np.float32
        arrs = [np.asfortranarray(a, dtype=dt) for a in (lam, mu, d)]
        _ck(lib().fd3d_upload_medium(self.h, *(a.ctypes.data for a in arrs), real_kind), "fd3d_upload_medium")

    def upload_fault(self, fault: dict):
        fb = abi.FaultBuffers(fault)
        _ck(lib().fd3d_upload_fault(self.h, C.byref(fb.s)), "fd3d_upload_fault")

    def upload_fault_model(self, T0I, TsI, DcI, dip: float = 90.0, dipslip: bool = False):
        """Fault from the control points of forwardmodel.dat (interpolated on the device)."""
        arrs = [np.asfortranarray(a, dtype=np.float64) for a in (T0I, TsI, DcI)]
        nli, nwi = arrs[0].shape
        dp = C.POINTER(C.c_double)
        _ck(lib().fd3d_upload_fault_model(self.h, nli, nwi, *(a.ctypes.data_as(dp) for a in arrs), float(dip),
                                          int(dipslip)), "fd3d_upload_fault_model")

    # ------------------------------------------------------------ checkpoint / resume
    def checkpoint(self, path: str):
        """Write the whole state of the run to one file (waits for the enqueued steps)."""
        _ck(lib().fd3d_checkpoint(self.h, path.encode()), "fd3d_checkpoint")

    @classmethod
    def restore(cls, path: str, model: dict) -> "Solver":
        """A solver resuming the run saved in path; model is the model that run was made
        from (its sizes and law; the medium and fault come from the file)."""
        self = cls.__new__(cls)
        self.model = model
        self.p = abi.make_params(model)
        self.h = C.c_void_p()
        _ck(lib().fd3d_restore(path.encode(), C.byref(self.h)), "fd3d_restore")
        self.nxT = model["nxt"] - 2 * model["nabc"]
        self.nzT = model["nzt"] - model["nfs"] - model["nabc"]
        self.nf = 5 if model.get("law", "sw") == "fvw" else 4
        return self

    # ------------------------------------------------------------ time loop
    def reset(self):
        _ck(lib().fd3d_reset(self.h), "fd3d_reset")

    def run(self, nsteps: int):
        _ck(lib().fd3d_run(self.h, int(nsteps)), "fd3d_run")

    def sync(self):
        _ck(lib().fd3d_sync(self.h), "fd3d_sync")

    def steps_done(self) -> int:
        n = C.c_int()
        _ck(lib().fd3d_steps_done(self.h, C.byref(n)), "fd3d_steps_done")
        return n.value

    def last_run_ms(self) -> float:
        v = C.c_float()
        _ck(lib().fd3d_last_run_ms(self.h, C.byref(v)), "fd3d_last_run_ms")
        return v.value

    def set_profiling(self, on: bool):
        _ck(lib().fd3d_set_profiling(self.h, int(on)), "fd3d_set_profiling")

    def kernel_times(self):
        ms = (C.c_float * abi.NKERNELS)()
        n = (C.c_int * abi.NKERNELS)()
        _ck(lib().fd3d_kernel_times(self.h, ms, n), "fd3d_kernel_times")
        return {abi.KERNEL_NAMES[k]: (ms[k], n[k]) for k in range(abi.NKERNELS)}

    INTERIOR_VARIANTS = {0: "point", 1: "tiled", 2: "pipe", 3: "tma"}

    def info(self) -> dict:
        """Which interior sweep runs ("tma" unless the tensor maps could not be encoded or
        FD3D_INTERIOR chose another) and whether the medium is read as a 1-D profile."""
        v, lay = C.c_int(), C.c_int()
        _ck(lib().fd3d_ctx_info(self.h, C.byref(v), C.byref(lay)), "fd3d_ctx_info")
        return dict(interior_variant=self.INTERIOR_VARIANTS.get(v.value, str(v.value)), layered_medium=bool(lay.value))

    # ------------------------------------------------------------ outputs
    def history_records(self) -> int:
        n = C.c_int()
        _ck(lib().fd3d_history_records(self.h, C.byref(n)), "fd3d_history_records")
        return n.value

    def history(self, field, rec0: int = 0, nrec: int | None = None, real_kind: int = 8) -> np.ndarray:
        """(nrec, nztT, nxtT) planes of one history file (x fastest, as written)."""
        fi = abi.HIST_NAMES.index(field) if isinstance(field, str) else int(field)
        if nrec is None:
            nrec = self.history_records() - rec0
        out = np.empty((nrec, self.nzT, self.nxT), dtype=np.float64 if real_kind == 8 else np.float32)
        _ck(lib().fd3d_fetch_history(self.h, fi, rec0, nrec, out.ctypes.data, real_kind), "fd3d_fetch_history")
        return out

    def stations(self, rec0: int = 0, nrec: int | None = None) -> np.ndarray:
        if nrec is None:
            nrec = self.history_records() - rec0
        ns = max(1, self.p.nstations)
        out = np.empty((nrec, ns, 3))
        _ck(lib().fd3d_fetch_stations(self.h, rec0, nrec, out.ctypes.data_as(C.POINTER(C.c_double))),
            "fd3d_fetch_stations")
        return out[:, :self.p.nstations]

    def field(self, name: str) -> np.ndarray:
        shp = (self.model["nxt"], self.model["nyt"], self.model["nzt"])
        out = np.empty(shp, dtype=np.float64, order="F")
        _ck(lib().fd3d_fetch_field(self.h, abi.FIELDS[name], out.ctypes.data, 8), "fd3d_fetch_field")
        return out

    def plane(self, name: str) -> np.ndarray:
        out = np.empty((self.model["nxt"], self.model["nzt"]), dtype=np.float64, order="F")
        _ck(lib().fd3d_fetch_plane(self.h, abi.PLANES[name], out.ctypes.data_as(C.POINTER(C.c_double))),
            "fd3d_fetch_plane")
        return out

    def moment_rate(self, rec0: int = 0, nrec: int | None = None) -> np.ndarray:
        """Moment rate of the history records still in the device ring
        (MomentRate of fd3d_theo.f90:574-578 with the seismogram step equal to dt)."""
        if nrec is None:
            nrec = self.history_records() - rec0
        out = np.empty(nrec)
        _ck(lib().fd3d_fetch_moment_rate(self.h, rec0, nrec, out.ctypes.data_as(C.POINTER(C.c_double))),
            "fd3d_fetch_moment_rate")
        return out

    def post_process(self) -> dict:
        """The reference's post-loop block on the device: average rupture speed, seismic
        moment, rupture area (0, as the reference leaves it) and average stress drop, and
        the rupture-velocity and cohesive-zone planes."""
        out = np.empty(4)
        _ck(lib().fd3d_post_process(self.h, out.ctypes.data_as(C.POINTER(C.c_double))), "fd3d_post_process")
        return dict(rupture_speed=out[0], moment=out[1], area=out[2], stress_drop=out[3],
                    rvel=self.plane("rvel"), czone=self.plane("czone"))

    def final(self) -> dict:
        shp = (self.model["nxt"], self.model["nzt"])
        out = {k: np.empty(shp, order="F") for k in ("slipX", "slipZ", "ruptime", "rise", "sliptime")}
        dp = C.POINTER(C.c_double)
        _ck(lib().fd3d_fetch_final(self.h, *(out[k].ctypes.data_as(dp) for k in
                                             ("slipX", "slipZ", "ruptime", "rise", "sliptime"))),
            "fd3d_fetch_final")
        return out

    def write_results(self, outdir: str, real_kind: int = 4):
        _ck(lib().fd3d_write_results(self.h, outdir.encode(), real_kind), "fd3d_write_results")

    def close(self):
        if self.h:
            lib().fd3d_ctx_destroy(self.h)
            self.h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def read_deck(path: str, fspace: bool = False):
    """fd3d_init + readcrustalmodel through the C ABI: (params dict, lam1, mu1, d1);
    fspace reads the deck as the FSPACE build does (nfs = nabc)."""
    p = abi.Params()
    dp = C.POINTER(C.c_double)
    bl, bm, bd = dp(), dp(), dp()
    _ck(lib().fd3d_read_deck_ex(path.encode(), int(fspace), C.byref(p), C.byref(bl), C.byref(bm), C.byref(bd)),
        "fd3d_read_deck_ex")
    n = p.nxt * p.nyt * p.nzt
    arrs = []
    for b in (bl, bm, bd):
        a = np.ctypeslib.as_array(b, shape=(n,)).copy().reshape((p.nxt, p.nyt, p.nzt), order="F")
        lib().fd3d_free(C.cast(b, C.c_void_p))
        arrs.append(a)
    cfg = {f: getattr(p, f) for f, _ in abi.Params._fields_ if f not in ("staX", "staY", "staZ")}
    cfg["stations"] = [(p.staX[s], p.staY[s], p.staZ[s]) for s in range(p.nstations)]
    return cfg, arrs[0], arrs[1], arrs[2]

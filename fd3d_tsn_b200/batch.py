"""Python view of the batched C ABI (fd3d_batch_*): many forward models, one launch."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import abi
from .solver import _ck, lib

_SIG = False
SCHEDULES = {"persistent": 0, "graph": 1}


def _bind():
    global _SIG
    if _SIG:
        return
    L = lib()
    i, vp, dp, sz = C.c_int, C.c_void_p, C.POINTER(C.c_double), C.c_size_t
    sig = {
        "fd3d_batch_create": (i, [sz, i, C.POINTER(vp)]),
        "fd3d_batch_destroy": (i, [vp]),
        "fd3d_batch_bytes_needed": (i, [C.POINTER(abi.Params), C.POINTER(sz)]),
        "fd3d_batch_add": (i, [vp, C.POINTER(abi.Params), dp, dp, dp, C.POINTER(abi.Fault), C.POINTER(i)]),
        "fd3d_batch_remove": (i, [vp, i]),
        "fd3d_batch_reset": (i, [vp, i]),
        "fd3d_batch_run": (i, [vp, i]),
        "fd3d_batch_sync": (i, [vp]),
        "fd3d_batch_model_status": (i, [vp, i]),
        "fd3d_batch_last_run_ms": (i, [vp, C.POINTER(C.c_float)]),
        "fd3d_batch_steps_done": (i, [vp, i, C.POINTER(i)]),
        "fd3d_batch_live": (i, [vp, C.POINTER(i), C.POINTER(sz)]),
        "fd3d_batch_fetch_plane": (i, [vp, i, i, dp]),
        "fd3d_batch_fetch_final": (i, [vp, i, dp, dp, dp, dp, dp]),
        "fd3d_batch_fetch_history": (i, [vp, i, i, i, i, dp]),
        "fd3d_batch_set_tuning": (i, [vp, i, i]),
        "fd3d_batch_get_tuning": (i, [vp, C.POINTER(i), C.POINTER(i), C.POINTER(i)]),
        "fd3d_batch_autotune": (i, [vp, i, C.c_char_p, C.c_char_p]),
        "fd3d_batch_set_schedule": (i, [vp, i]),
        "fd3d_batch_get_schedule": (i, [vp, C.POINTER(i)]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _SIG = True


def bytes_needed(model: dict) -> int:
    _bind()
    p = abi.make_params(model)
    n = C.c_size_t()
    _ck(lib().fd3d_batch_bytes_needed(C.byref(p), C.byref(n)), "fd3d_batch_bytes_needed")
    return n.value


class Batch:
    def __init__(self, arena_bytes: int, max_models: int = 512):
        _bind()
        self.h = C.c_void_p()
        _ck(lib().fd3d_batch_create(int(arena_bytes), int(max_models), C.byref(self.h)), "fd3d_batch_create")
        self.models = {}

    def add(self, model: dict) -> int:
        p = abi.make_params(model)
        lam, mu, d = (np.ascontiguousarray(a, dtype=np.float64) for a in model["medium"])
        fb = abi.FaultBuffers(model["fault"])
        slot = C.c_int()
        dp = C.POINTER(C.c_double)
        _ck(lib().fd3d_batch_add(self.h, C.byref(p), lam.ctypes.data_as(dp), mu.ctypes.data_as(dp),
                                 d.ctypes.data_as(dp), C.byref(fb.s), C.byref(slot)), "fd3d_batch_add")
        self.models[slot.value] = model
        return slot.value

    def try_add(self, model: dict):
        """add() that returns None when the arena or the slot table is full."""
        try:
            return self.add(model)
        except abi.Fd3dError as e:
            if e.code in (-4, -10):
                return None
            raise

    def remove(self, slot: int):
        _ck(lib().fd3d_batch_remove(self.h, slot), "fd3d_batch_remove")
        self.models.pop(slot, None)

    def reset(self, slot: int):
        _ck(lib().fd3d_batch_reset(self.h, slot), "fd3d_batch_reset")

    def run(self, nsteps: int):
        _ck(lib().fd3d_batch_run(self.h, int(nsteps)), "fd3d_batch_run")

    def sync(self):
        _ck(lib().fd3d_batch_sync(self.h), "fd3d_batch_sync")

    def model_status(self, slot: int) -> int:
        return lib().fd3d_batch_model_status(self.h, slot)

    def last_run_ms(self) -> float:
        v = C.c_float()
        _ck(lib().fd3d_batch_last_run_ms(self.h, C.byref(v)), "fd3d_batch_last_run_ms")
        return v.value

    def steps_done(self, slot: int) -> int:
        n = C.c_int()
        _ck(lib().fd3d_batch_steps_done(self.h, slot, C.byref(n)), "fd3d_batch_steps_done")
        return n.value

    def live(self):
        n = C.c_int()
        b = C.c_size_t()
        _ck(lib().fd3d_batch_live(self.h, C.byref(n), C.byref(b)), "fd3d_batch_live")
        return n.value, b.value

    def plane(self, slot: int, name: str) -> np.ndarray:
        m = self.models[slot]
        out = np.empty((m["nxt"], m["nzt"]), order="F")
        _ck(lib().fd3d_batch_fetch_plane(self.h, slot, abi.PLANES[name], out.ctypes.data_as(C.POINTER(C.c_double))),
            "fd3d_batch_fetch_plane")
        return out

    def final(self, slot: int) -> dict:
        m = self.models[slot]
        shp = (m["nxt"], m["nzt"])
        keys = ("slipX", "slipZ", "ruptime", "rise", "sliptime")
        out = {k: np.empty(shp, order="F") for k in keys}
        dp = C.POINTER(C.c_double)
        _ck(lib().fd3d_batch_fetch_final(self.h, slot, *(out[k].ctypes.data_as(dp) for k in keys)),
            "fd3d_batch_fetch_final")
        return out

    def history(self, slot: int, field: int, rec0: int, nrec: int) -> np.ndarray:
        m = self.models[slot]
        nxT = m["nxt"] - 2 * m["nabc"]
        nzT = m["nzt"] - m["nfs"] - m["nabc"]
        out = np.empty((nrec, nzT, nxT))
        _ck(lib().fd3d_batch_fetch_history(self.h, slot, field, rec0, nrec, out.ctypes.data_as(C.POINTER(C.c_double))),
            "fd3d_batch_fetch_history")
        return out

    def set_tuning(self, kchunk: int, ctas_per_sm: int = 0):
        _ck(lib().fd3d_batch_set_tuning(self.h, kchunk, ctas_per_sm), "fd3d_batch_set_tuning")

    def set_schedule(self, mode: str):
        """"persistent" (one cooperative kernel per run) or "graph" (CUDA graphs of
        per-region kernels over all models)."""
        _ck(lib().fd3d_batch_set_schedule(self.h, SCHEDULES[mode]), "fd3d_batch_set_schedule")

    def tuning(self):
        a, b, c = C.c_int(), C.c_int(), C.c_int()
        _ck(lib().fd3d_batch_get_tuning(self.h, C.byref(a), C.byref(b), C.byref(c)), "fd3d_batch_get_tuning")
        mode = C.c_int()
        _ck(lib().fd3d_batch_get_schedule(self.h, C.byref(mode)), "fd3d_batch_get_schedule")
        names = {v: k for k, v in SCHEDULES.items()}
        return dict(schedule=names[mode.value], kchunk=a.value, ctas_per_sm=b.value, max_ctas_per_sm=c.value)

    def autotune(self, steps: int = 10, cache_path: str | None = None, key: str | None = None):
        _ck(lib().fd3d_batch_autotune(self.h, steps, cache_path.encode() if cache_path else None,
                                      key.encode() if key else None), "fd3d_batch_autotune")
        return self.tuning()

    def close(self):
        if self.h:
            lib().fd3d_batch_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

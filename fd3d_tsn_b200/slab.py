"""One forward model over several GPU contexts: z-slabs stepped as a group.

The reference runs one model in one process on one GPU (src/dynamicsolver.f90:66).  A
model too slow for one GPU is split here into slabs of consecutive planes k; each slab
is a context of its own (one device each, or several on one device), and the group
exchanges two halo planes (or fault-plane rows) with the neighbouring slabs after the
velocity sweeps, the stress sweeps, the trial traction and the friction law.  The
results are the same bits as one :class:`~fd3d_tsn_b200.solver.Solver`'s:

    s = SlabSolver(model, nslabs=4, devices=[0, 1, 2, 3])
    s.run(model["ntfd"])
    s.sync()
    slip = s.final()["slipX"]

Every slab holds its own planes of the wave field and medium plus three halo planes on
either side, and the whole fault plane and PML split-component pool; the fault-plane
post-processing (moment rate, rupture speed, stress drop) is not available on slabs.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import abi
from .solver import Solver, _ck, lib


NCCL_ID_BYTES = 128


def plan(model: dict, nslabs: int) -> list[tuple[int, int]]:
    """The plane ranges (k_lo, k_hi) of nslabs slabs of about equal cost."""
    p = abi.make_params(model)
    lo, hi = (C.c_int * nslabs)(), (C.c_int * nslabs)()
    _ck(lib().fd3d_slab_plan(C.byref(p), int(nslabs), lo, hi), "fd3d_slab_plan")
    return [(lo[r], hi[r]) for r in range(nslabs)]


class SlabSolver:
    def __init__(self, model: dict, nslabs: int = 2, devices: list[int] | None = None,
                 ranges: list[tuple[int, int]] | None = None, medium3d: bool = False):
        self.model = model
        self.ranges = list(ranges) if ranges is not None else plan(model, nslabs)
        self.slabs: list[Solver] = []
        self.g = C.c_void_p()
        for r, rng in enumerate(self.ranges):
            if devices is not None:
                _ck(lib().fd3d_set_device(int(devices[r % len(devices)])), "fd3d_set_device")
            self.slabs.append(Solver(model, medium3d=medium3d, slab=rng))
        hs = (C.c_void_p * len(self.slabs))(*[s.h.value for s in self.slabs])
        _ck(lib().fd3d_slab_group_create(hs, len(self.slabs), C.byref(self.g)), "fd3d_slab_group_create")
        self.nxT, self.nzT, self.nf = self.slabs[0].nxT, self.slabs[0].nzT, self.slabs[0].nf
        self._ms = 0.0

    # ------------------------------------------------------------ time loop
    def run(self, nsteps: int):
        _ck(lib().fd3d_slab_group_run(self.g, int(nsteps)), "fd3d_slab_group_run")

    def sync(self):
        ms = C.c_float()
        _ck(lib().fd3d_slab_group_sync(self.g, C.byref(ms)), "fd3d_slab_group_sync")
        self._ms = ms.value

    def last_run_ms(self) -> float:
        """The longest slab's device time of the last run."""
        return self._ms

    def steps_done(self) -> int:
        return self.slabs[0].steps_done()

    # ------------------------------------------------------------ outputs, merged
    def _owner(self, k: int) -> int:
        for r, (a, b) in enumerate(self.ranges):
            if a <= k <= b:
                return r
        raise ValueError(k)

    def _rows(self, arrays: list[np.ndarray], axis: int, k_of_index) -> np.ndarray:
        """Merge per-slab arrays along `axis`, index q taken from the slab owning k_of_index(q)."""
        out = np.array(arrays[0], copy=True)
        for q in range(out.shape[axis]):
            r = self._owner(k_of_index(q))
            if r:
                idx = [slice(None)] * out.ndim
                idx[axis] = q
                out[tuple(idx)] = arrays[r][tuple(idx)]
        return out

    def history_records(self) -> int:
        return self.slabs[0].history_records()

    def history(self, field, rec0: int = 0, nrec: int | None = None, real_kind: int = 8) -> np.ndarray:
        parts = [s.history(field, rec0, nrec, real_kind) for s in self.slabs]
        nab = self.model["nabc"]
        return self._rows(parts, 1, lambda kk: nab + 1 + kk)

    def stations(self, rec0: int = 0, nrec: int | None = None) -> np.ndarray:
        parts = [s.stations(rec0, nrec) for s in self.slabs]
        out = np.array(parts[0], copy=True)
        for st, (_, _, k) in enumerate(self.model.get("stations", [])):
            out[:, st] = parts[self._owner(k)][:, st]
        return out

    def field(self, name: str) -> np.ndarray:
        shp = (self.model["nxt"], self.model["nyt"], self.model["nzt"])
        out = np.zeros(shp, dtype=np.float64, order="F")
        for s in self.slabs:  # each slab writes its own planes
            _ck(lib().fd3d_fetch_field(s.h, abi.FIELDS[name], out.ctypes.data, 8), "fd3d_fetch_field")
        return out

    def plane(self, name: str) -> np.ndarray:
        return self._rows([s.plane(name) for s in self.slabs], 1, lambda q: q + 1)

    def final(self) -> dict:
        parts = [s.final() for s in self.slabs]
        return {k: self._rows([p[k] for p in parts], 1, lambda q: q + 1) for k in parts[0]}

    def close(self):
        if self.g:
            lib().fd3d_slab_group_destroy(self.g)
            self.g = C.c_void_p()
        for s in self.slabs:
            s.close()
        self.slabs = []

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def nccl_id() -> bytes:
    """A fresh NCCL unique id (made by rank 0 and passed to every rank)."""
    buf = C.create_string_buffer(NCCL_ID_BYTES)
    _ck(lib().fd3d_nccl_unique_id(buf), "fd3d_nccl_unique_id")
    return buf.raw


def rank_setup(model: dict, rank: int, world: int, broadcast, make_id=nccl_id):
    """This rank's plane range and the id every rank connects with: rank 0 makes the id
    and `broadcast` (a list broadcast from rank 0, e.g. torch.distributed's
    broadcast_object_list) hands it to the others."""
    ranges = plan(model, world)
    obj = [make_id() if rank == 0 else None]
    broadcast(obj)
    return ranges[rank], obj[0]


class SlabRank:
    """This process's slab of one model decomposed over torch.distributed ranks, one GPU
    each (rank r holds the r-th slab from the bottom); the halos travel over NCCL between
    neighbouring ranks.  The solver's outputs are this slab's (its planes, fault rows and
    stations); gather_final() puts the whole fault plane's results on every rank."""

    def __init__(self, model: dict, medium3d: bool = False):
        import torch.distributed as dist
        self.model = model
        self.rank, self.world = dist.get_rank(), dist.get_world_size()
        self.range, uid = rank_setup(model, self.rank, self.world, lambda o: dist.broadcast_object_list(o, src=0))
        self.ranges = plan(model, self.world)
        self.solver = Solver(model, medium3d=medium3d, slab=self.range)
        _ck(lib().fd3d_slab_connect(self.solver.h, uid, self.rank, self.world), "fd3d_slab_connect")

    def run(self, nsteps: int):
        _ck(lib().fd3d_slab_run(self.solver.h, int(nsteps)), "fd3d_slab_run")

    def sync(self):
        self.solver.sync()

    def last_run_ms(self) -> float:
        return self.solver.last_run_ms()

    def gather_final(self) -> dict:
        """The whole fault plane's final slip, rupture time, ... on every rank."""
        import torch.distributed as dist
        parts = [None] * self.world
        dist.all_gather_object(parts, self.solver.final())
        out = {}
        for k in parts[0]:
            a = np.array(parts[0][k], copy=True)
            for r, (lo, hi) in enumerate(self.ranges):
                a[:, lo - 1:hi] = parts[r][k][:, lo - 1:hi]
            out[k] = a
        return out

    def close(self):
        self.solver.close()

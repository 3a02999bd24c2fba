"""Writes tests/golden/oracle_tiny.json: SHA-256 digests of the CPU oracle's outputs on three
small seeded slip-weakening models (FP32 fields with FP64 accumulators, the all-FP64 build, and
the FSPACE build), 40 steps each.

These are fixtures made by the oracle, not by the reference: the reference is Fortran and no
Fortran compiler exists here, and its repository ships input decks but no outputs.  They pin
the oracle against drift (tests/test_oracle_cpu.py) and give the GPU path fixed vectors to meet
bit for bit (tests/test_gpu_parity.py).  Run from the repository root:

    python tests/golden/make_golden.py
"""
import hashlib
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

STEPS = 40
PLANES = ("tx", "tz", "slipX", "slipZ", "ruptime", "distX", "distZ")
FIELDS = ("u", "w", "xz", "yy")


def cases():
    """name -> (model, oracle variant name)"""
    from fd3d_tsn_b200 import configs
    return {
        "tiny_sw_f32": (configs.tiny_sw(seed=5, nsteps=STEPS), "MIXED"),
        "tiny_sw_f64": (configs.tiny_sw(seed=5, nsteps=STEPS, precision="f64"), "F64"),
        "tiny_sw_fspace_f32": (configs.tiny_sw(seed=31, nsteps=STEPS, fspace=True), "MIXED"),
    }


def digest(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(np.asarray(a, dtype=np.float64)).tobytes()).hexdigest()


def outputs_digests(hist, stations, field, plane) -> dict:
    """hist (steps, >=4, nztT, nxtT), stations (steps, nst, 3); field(name), plane(name) -> arrays"""
    out = {f"history{f}": digest(hist[:, f]) for f in range(4)}
    out["stations"] = digest(stations)
    out.update({f"field_{n}": digest(field(n)) for n in FIELDS})
    out.update({f"plane_{n}": digest(plane(n)) for n in PLANES})
    return out


def main():
    from oracle.oracle import F64, MIXED, Oracle
    variants = {"MIXED": MIXED, "F64": F64}
    doc = {"steps": STEPS, "made_by": "the CPU oracle (oracle/fd3d_oracle.cpp) through oracle/oracle.py",
           "cases": {}}
    for name, (m, var) in cases().items():
        o = Oracle(m, variants[var])
        hist, seis = o.step(STEPS)
        d = outputs_digests(hist, seis, o.field, o.plane)
        d["variant"] = var
        d["max_slip_rate"] = float(np.abs(hist[:, 0]).max())
        d["max_slipX"] = float(np.abs(o.plane("slipX")).max())
        doc["cases"][name] = d
        o.close()
    with open(os.path.join(ROOT, "tests", "golden", "oracle_tiny.json"), "w") as f:
        json.dump(doc, f, indent=1, sort_keys=True)
        f.write("\n")


if __name__ == "__main__":
    main()

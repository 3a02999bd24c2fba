"""CPU-side checks of the C ABI library: exports, argument validation, deck reading.

No kernel is launched here; everything runs without a GPU.
"""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

from fd3d_tsn_b200 import abi, configs, solver

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
# the reference's examples/ directory (input decks), when a copy is at hand
REF_EXAMPLES = os.environ.get("FD3D_REFERENCE_EXAMPLES", "")


def test_library_exports_every_header_symbol():
    lib = abi.LIB_PATH
    out = subprocess.run(["nm", "-D", "--defined-only", lib], capture_output=True, text=True, check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if line.strip()}
    inc = os.path.join(ROOT, "include")
    declared = []
    for h in sorted(os.listdir(inc)):
        if h.endswith(".h"):
            declared += abi.header_symbols(os.path.join(inc, h))
    assert len(declared) >= 20
    missing = [s for s in declared if s not in exported]
    assert not missing, missing


def test_library_loads_and_reports_version():
    L = solver.lib()
    assert b"sm_100a" in L.fd3d_version()
    assert L.fd3d_status_string(-2).startswith(b"CFL")


def test_cfl_violation_rejected_before_any_device_work():
    m = configs.tiny_sw()
    p = abi.make_params(m)
    p.dt = 0.3 * p.dh / p.vp_max
    h = C.c_void_p()
    assert solver.lib().fd3d_ctx_create(C.byref(p), C.byref(h)) == -2


@pytest.mark.parametrize("field,val", [("nabc", 2), ("nfs", 3), ("law", 7), ("precision", 5), ("nstations", 11)])
def test_bad_arguments_rejected(field, val):
    p = abi.make_params(configs.tiny_sw())
    setattr(p, field, val)
    h = C.c_void_p()
    assert solver.lib().fd3d_ctx_create(C.byref(p), C.byref(h)) == -1


def test_no_device_is_reported_on_cpu():
    if solver.device_count() > 0:
        pytest.skip("a GPU is present")
    p = abi.make_params(configs.tiny_sw())
    h = C.c_void_p()
    assert solver.lib().fd3d_ctx_create(C.byref(p), C.byref(h)) == -9


def test_read_synthetic_deck(tmp_path):
    rng = np.random.default_rng(7)
    lay = configs.layered(rng, 4, 30 * 100.0)
    m = configs.sw_model(30, 12, 30, 100.0, 1.0, 3, layers=lay, nstations=2)
    configs.write_deck(m, str(tmp_path), lay)
    cfg, lam, mu, d = solver.read_deck(str(tmp_path))
    for k in ("nxt", "nyt", "nzt", "nabc", "ntfd"):
        assert cfg[k] == m[k], k
    assert cfg["dt"] == m["dt"] and cfg["dh"] == m["dh"]
    assert cfg["stations"] == [tuple(s) for s in m["stations"]]
    ml, mm, md = m["medium"]
    np.testing.assert_allclose(lam[0, 0, :], ml, rtol=1e-12)
    np.testing.assert_allclose(mu[5, 3, :], mm, rtol=1e-12)
    np.testing.assert_allclose(d[-1, -1, :], md, rtol=1e-12)
    assert np.all(lam == lam[:1, :1, :])


def test_deck_cfl_stop(tmp_path):
    lay = dict(depth=[0.0], vp=[6000.0], vs=[3464.0], rho=[2670.0])
    m = configs.sw_model(20, 10, 20, 100.0, 1.0, 3, layers=lay, nstations=0)
    m["dt"] = 0.26 * 100.0 / 6000.0
    configs.write_deck(m, str(tmp_path), lay)
    with pytest.raises(abi.Fd3dError) as e:
        solver.read_deck(str(tmp_path))
    assert e.value.code == -2


@pytest.mark.skipif(not (REF_EXAMPLES and os.path.isdir(REF_EXAMPLES)),
                    reason="FD3D_REFERENCE_EXAMPLES does not name the reference's examples directory")
@pytest.mark.parametrize("deck", ["TPV5", "TPV104", "TPV9", "Amatrice2016"])
def test_reference_decks_parse(deck):
    d = os.path.join(REF_EXAMPLES, deck)
    cfg, lam, mu, dd = solver.read_deck(d)
    py = configs.read_inputfd3d(os.path.join(d, "inputfd3d.dat"))
    for k in ("nxt", "nyt", "nzt", "nabc", "ntfd"):
        assert cfg[k] == py[k]
    assert cfg["stations"] == py["stations"]
    cr = configs.read_crustal(os.path.join(d, "crustal.dat"))
    L, M, D, vpm = configs.crustal_medium(py["nzt"], py["dh"], py["dip"], cr["depth"], cr["vp"], cr["vs"], cr["rho"])
    np.testing.assert_allclose(lam[3, 2, :], L, rtol=1e-12)
    np.testing.assert_allclose(mu[3, 2, :], M, rtol=1e-12)
    np.testing.assert_allclose(dd[3, 2, :], D, rtol=1e-12)


def test_struct_layouts_match_the_library():
    """The ctypes mirrors of fd3d_params and fd3d_fault have the library's sizes."""
    lib = abi.load_library()
    pb, fb = C.c_size_t(), C.c_size_t()
    assert lib.fd3d_struct_sizes(C.byref(pb), C.byref(fb)) == 0
    assert pb.value == C.sizeof(abi.Params)
    assert fb.value == C.sizeof(abi.Fault)


def test_fortran_module_matches_the_library():
    """include/fd3d_gpu.f90 (not compiled here: no Fortran compiler in the image) binds only
    exported functions, and its derived types list the C structs' fields in their order."""
    import re
    src = open(os.path.join(ROOT, "include", "fd3d_gpu.f90")).read()
    out = subprocess.run(["nm", "-D", "--defined-only", abi.LIB_PATH], capture_output=True, text=True,
                         check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if line.strip()}
    bound = re.findall(r"function\s+(fd3d_\w+)\s*\(", src)
    assert len(bound) >= 15
    assert not [f for f in bound if f not in exported]

    def fields(type_name):
        body = re.search(r"type, bind\(C\) :: " + type_name + r"\n(.*?)end type", src, re.S).group(1)
        names = []
        for line in body.splitlines():
            if "::" not in line:
                continue
            decl = line.split("::")[1]
            names += [re.sub(r"\(.*\)", "", n).strip().lower() for n in decl.split(",")]
        return names

    assert fields("fd3d_params") == [n.lower() for n, _ in abi.Params._fields_]
    assert fields("fd3d_fault") == [n.lower() for n, _ in abi.Fault._fields_]

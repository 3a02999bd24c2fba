"""Model set-up on the host: synthetic workloads and the reference's input decks.

A *model* is a dict with the grid / run parameters of ``fd3d_params`` plus

* ``medium``: ``(lam_k, mu_k, d_k)``, one value per k of the padded grid (the 1-D
  layered medium that ``readcrustalmodel`` builds, src/fd3d_init.f90:241-265), and
* ``fault``: the per-node friction / prestress planes of shape (nxt, nzt), indexed
  [i-1, k-1] like the reference's Fortran arrays.

Workloads (all seeded with ``numpy.random.default_rng``):

* ``sw_small``   160x80x120 cells, h=200 m, homogeneous, 120x60-node patch, 8 s
* ``sw_large``   1000x400x500 cells (~214 M padded), h=50 m, 5 seeded layers, 12 s
* ``fvw_medium`` 600x300x400 cells, h=100 m, rate-and-state with nucleation ramp, 10 s
* ``batch_model`` the small uneven models of the batched / serving workloads
* tiny variants of the above for the parity tests.

Sizes follow the reference's convention: the simulated box is nxtT x nytT x nztT and
the padded grid adds 2*nabc cells in x, nabc in y (one side of the fault only, fault
at j = nyt) and nabc + 2 in z (PML below, two ghost rows above the free surface).
"""
from __future__ import annotations

import math
import os

import numpy as np

NABC = 10
NFS = 2
PML_VP = 6000.0
PML_FACT = 28.0
DAMP_S = 0.3


# ---------------------------------------------------------------- media
def crustal_medium(nzt: int, dh: float, dip: float, depth, vp, vs, rho, nfs: int = NFS):
    """readcrustalmodel (src/fd3d_init.f90:241-265): per-k lam, mu, rho and vp_max.

    depth in m (layer tops), vp/vs in m/s, rho in kg/m^3.  z is upside down: k = nzt-nfs
    is the free surface and the cell depth is dh*(nzt-nfs-k) + dh/2 (times sin(dip)).
    """
    depth, vp, vs, rho = (np.asarray(a, dtype=np.float64) for a in (depth, vp, vs, rho))
    nd = len(depth)
    lam = np.zeros(nzt); mu = np.zeros(nzt); d = np.zeros(nzt)
    vpmax = 0.0
    for k in range(nzt, 0, -1):
        dum = (dh * (nzt - nfs - k) + dh / 2.0) * math.sin(dip / 180.0 * 3.1415926535)
        if dum > depth[nd - 1]:
            q = nd - 1
        else:
            j = 2
            while j <= nd and not (dum < depth[j - 1]):
                j += 1
            q = j - 2
        vpp, vss, dd = vp[q], vs[q], rho[q]
        vpmax = max(vpmax, vpp)
        lam[k - 1] = dd * (vpp ** 2 - 2.0 * vss ** 2)
        mu[k - 1] = dd * vss ** 2
        d[k - 1] = dd
    return lam, mu, d, vpmax


def medium_3d(model: dict):
    """Full (nxt,nyt,nzt) Fortran-order arrays of the layered medium."""
    lam, mu, d = model["medium"]
    shp = (model["nxt"], model["nyt"], model["nzt"])
    out = []
    for a in (lam, mu, d):
        out.append(np.broadcast_to(np.asarray(a)[None, None, :], shp))
    return out


def gaussian_field(rng, nx, nz, corr_nodes, mean, std):
    """Seeded Gaussian random field: white noise filtered by a Gaussian kernel of the
    given correlation length (in nodes), rescaled to the requested mean and std."""
    noise = rng.standard_normal((nx, nz))
    kx = np.fft.fftfreq(nx)[:, None]
    kz = np.fft.fftfreq(nz)[None, :]
    filt = np.exp(-0.5 * (2 * np.pi * corr_nodes) ** 2 * (kx ** 2 + kz ** 2) / 2.0)
    f = np.real(np.fft.ifft2(np.fft.fft2(noise) * filt))
    f = (f - f.mean()) / (f.std() + 1e-30)
    return mean + std * f


def fortran_planes(fault: dict) -> dict:
    """Fault planes in Fortran order (x fastest), as a Fortran host holds them: the C ABI
    takes them without a copy."""
    return {k: (np.asfortranarray(v, dtype=np.float64) if isinstance(v, np.ndarray) and v.ndim == 2 else v)
            for k, v in fault.items()}


def _grid(nxT, nyT, nzT, h, dt, ntfd, nabc=NABC, fspace=False):
    """Padded grid of fd3d_init.f90:161-169; fspace: the FSPACE build (a PML strip of
    nabc cells above the model instead of the free surface, nfs = nabc)."""
    nfs = nabc if fspace else NFS
    return dict(nxt=nxT + 2 * nabc, nyt=nyT + nabc, nzt=nzT + nabc + nfs, nabc=nabc, nfs=nfs, fspace=bool(fspace),
                dh=float(h), dt=float(dt), ntfd=int(ntfd), damp_s=DAMP_S, pml_vp=PML_VP, pml_fact=PML_FACT)


def _stations(rng, m, n):
    st = []
    for _ in range(n):
        i = int(rng.integers(m["nabc"] + 3, m["nxt"] - m["nabc"] - 2))
        j = int(rng.integers(m["nabc"] + 3, m["nyt"] - 4))
        k = int(rng.integers(m["nabc"] + 3, m["nzt"] - m["nfs"]))
        st.append((i, j, k))
    return st


def sw_fault(m, rng, patch, sn=120e6, mus=0.68, mud=0.52, dc=0.4, t0_mean=70e6, t0_std=5e6,
             corr_m=2000.0, nuc_m=3000.0, dc_patch_m=None, dc_range=None, border_mus=10000.0):
    """Slip-weakening planes: a frictional patch (i0,i1,k0,k1) (1-based, inclusive) with a
    seeded Gaussian prestress clipped below static strength and a central overstressed
    square nucleation patch; outside the patch the static friction is `border_mus`
    (the TPV5 set-up uses 10000, src/fd3d_init.f90:581-590)."""
    nxt, nzt, h = m["nxt"], m["nzt"], m["dh"]
    i0, i1, k0, k1 = patch
    peak = np.full((nxt, nzt), sn * border_mus)
    dyn = np.full((nxt, nzt), sn * mud)
    Dc = np.full((nxt, nzt), dc)
    peak[i0 - 1:i1, k0 - 1:k1] = sn * mus
    if dc_patch_m is not None:
        npch = max(1, int(round(dc_patch_m / h)))
        nbx, nbz = (nxt + npch - 1) // npch, (nzt + npch - 1) // npch
        blocks = rng.uniform(dc_range[0], dc_range[1], size=(nbx, nbz))
        Dc = np.repeat(np.repeat(blocks, npch, axis=0), npch, axis=1)[:nxt, :nzt].copy()
    t0 = gaussian_field(rng, nxt, nzt, corr_m / h, t0_mean, t0_std)
    t0 = np.minimum(t0, 0.99 * sn * mus)
    ic, kc = (i0 + i1) // 2, (k0 + k1) // 2
    half = max(1, int(round(nuc_m / h / 2)))
    t0[ic - 1 - half:ic - 1 + half + 1, kc - 1 - half:kc - 1 + half + 1] = 1.015 * sn * mus
    return dict(law="sw", striniX=t0, striniZ=np.zeros((nxt, nzt)), Dc=Dc, peak_xz=peak, dyn_xz=dyn,
                coh=np.zeros((nxt, nzt)))


def sw_model(nxT, nyT, nzT, h, sim_time, seed, layers=None, patch_nodes=None, nstations=4, corr_m=2000.0,
             dc_patch_m=None, dc_range=None, history_stride=1, precision="f32", ntfd=None, fspace=False, nabc=NABC):
    rng = np.random.default_rng(seed)
    if layers is None:
        layers = dict(depth=[0.0], vp=[6000.0], vs=[3464.0], rho=[2670.0])
    dip = 90.0
    vpmax = max(layers["vp"])
    dt = 0.25 * h / vpmax * (1.0 - 1e-6)  # strict CFL check of fd3d_init.f90:274-278
    nsteps = int(round(sim_time / dt)) if ntfd is None else ntfd
    m = _grid(nxT, nyT, nzT, h, dt, nsteps, nabc=nabc, fspace=fspace)
    lam, mu, d, vpm = crustal_medium(m["nzt"], h, dip, layers["depth"], layers["vp"], layers["vs"], layers["rho"],
                                     nfs=m["nfs"])
    m.update(medium=(lam, mu, d), vp_max=vpm, law="sw", precision=precision, history_stride=history_stride)
    if patch_nodes is None:
        patch_nodes = (nxT * 3 // 4, nzT // 2)
    px, pz = patch_nodes
    nab = m["nabc"]
    i0 = nab + 1 + (nxT - px) // 2
    k0 = nab + 1 + (nzT - pz) // 2
    m["fault"] = fortran_planes(sw_fault(m, rng, (i0, i0 + px - 1, k0, k0 + pz - 1), corr_m=corr_m,
                                         dc_patch_m=dc_patch_m, dc_range=dc_range))
    m["stations"] = _stations(rng, m, nstations)
    m["seed"] = seed
    return m


def layered(rng, nlayers, zmax, vs_lo=2000.0, vs_hi=3600.0):
    """Seeded 1-D layering: vs increasing with depth, vp = sqrt(3) vs, rho = 1700 + 0.2 vp."""
    vs = np.sort(rng.uniform(vs_lo, vs_hi, size=nlayers))
    tops = np.concatenate([[0.0], np.sort(rng.uniform(0.05, 0.8, size=nlayers - 1)) * zmax])
    vp = np.sqrt(3.0) * vs
    rho = 1700.0 + 0.2 * vp
    return dict(depth=tops, vp=vp, vs=vs, rho=rho)


# ---------------------------------------------------------------- named workloads
def sw_small(seed=1, **kw):
    """160x80x120 cells, h=200 m, 8 s, 120x60 patch, 4 stations."""
    return sw_model(160, 80, 120, 200.0, 8.0, seed, patch_nodes=(120, 60), **kw)


def sw_large(seed=2, **kw):
    """1000x400x500 cells, h=50 m, 5 seeded layers, 800x400 patch, 1 km correlation,
    Dc uniform in [0.3, 0.6] m per 1 km patch, 12 s."""
    rng = np.random.default_rng(seed + 1000)
    lay = layered(rng, 5, 500 * 50.0)
    return sw_model(1000, 400, 500, 50.0, 12.0, seed, layers=lay, patch_nodes=(800, 400), corr_m=1000.0,
                    dc_patch_m=1000.0, dc_range=(0.3, 0.6), **kw)


def fvw_model(nxT, nyT, nzT, h, sim_time, seed, fault_m=(48e3, 24e3), dt=None, history_stride=5,
              precision="f32", nstations=4, border_m=3000.0, perturb=45e6, R=3000.0, TT=1.0, ntfd=None,
              fspace=False):
    """Fast-velocity-weakening model: a uniform in [0.008,0.012] inside, ramping to 0.02
    over the border; b=0.014; L in [0.2,0.5]; f0=0.6; V0=1e-6; fw in [0.1,0.2]; Vw 0.1
    ramping to 1.0 in the border; initial slip rate 1e-16 (uini = 0.5e-16, as the TPV104
    deck); steady-state psi (src/fd3d_init.f90:466,496); sigma_n 120 MPa, tau 40 MPa +/- a
    seeded 5 MPa field; smooth nucleation bump of the reference (src/fd3d_theo.f90:515-541)."""
    rng = np.random.default_rng(seed)
    vp, vs, rho = 6000.0, 3464.0, 2670.0
    dt = dt if dt is not None else 0.002 * h / 100.0
    nsteps = int(round(sim_time / dt)) if ntfd is None else ntfd
    m = _grid(nxT, nyT, nzT, h, dt, nsteps, fspace=fspace)
    lam, mu, d, vpm = crustal_medium(m["nzt"], h, 90.0, [0.0], [vp], [vs], [rho], nfs=m["nfs"])
    m.update(medium=(lam, mu, d), vp_max=vpm, law="fvw", precision=precision, history_stride=history_stride)
    nxt, nzt = m["nxt"], m["nzt"]
    nab = m["nabc"]
    Sn, v0, f0, b, uini = 120e6, 1e-6, 0.6, 0.014, 0.5e-16
    # fault box in nodes, centred in x, top at the free surface
    fx, fz = int(round(fault_m[0] / h)), int(round(fault_m[1] / h))
    fx, fz = min(fx, nxT), min(fz, nzT)
    i0 = nab + 1 + (nxT - fx) // 2
    k1 = nzt - m["nfs"]
    k0 = k1 - fz + 1
    bw = border_m / h

    def taper(ii, kk):
        dx = np.minimum(ii - i0, i0 + fx - 1 - ii)
        dz = kk - k0  # the border runs along the sides and the bottom
        dist = np.minimum(dx, dz).astype(np.float64)
        return np.clip(1.0 - dist / bw, 0.0, 1.0)  # 0 inside, 1 at the edge and outside

    ii, kk = np.meshgrid(np.arange(1, nxt + 1), np.arange(1, nzt + 1), indexing="ij")
    B = taper(ii, kk)
    a_in = rng.uniform(0.008, 0.012, size=(nxt, nzt))
    a = a_in + (0.02 - a_in) * B
    vw = 0.1 + 0.9 * B
    L = rng.uniform(0.2, 0.5, size=(nxt, nzt))
    fw = rng.uniform(0.1, 0.2, size=(nxt, nzt))
    tau = 40e6 + 5e6 * np.clip(gaussian_field(rng, nxt, nzt, 2000.0 / h, 0.0, 1.0), -3, 3) / 3.0
    psi = a * (np.log(2 * v0 / (2 * uini)) + np.log(np.sinh(tau / (a * Sn))))
    fault = dict(law="fvw", striniX=tau, striniZ=np.zeros((nxt, nzt)), Dc=L, a=a, b=np.full((nxt, nzt), b),
                 psi=psi, vw=vw, aX=a.copy(), bX=np.full((nxt, nzt), b), psiX=psi.copy(), vwX=vw.copy(),
                 fwZ=fw, fwX=fw.copy(), Sn=Sn, v0=v0, f0=f0, fw=0.15, uini=uini, wini=0.0,
                 nucleation=2, hx0=(i0 + fx // 2) * h, hz0=(k1 - fz // 2) * h, perturb=perturb, RR2=R * R,
                 TT2=TT, strinixI=float(np.mean(tau)))
    m["fault"] = fortran_planes(fault)
    m["stations"] = _stations(rng, m, nstations)
    m["seed"] = seed
    return m


def fvw_medium(seed=3, **kw):
    """600x300x400 cells, h=100 m, 48x24 km fault, 10 s, histories every 5 steps."""
    return fvw_model(600, 300, 400, 100.0, 10.0, seed, **kw)


def batch_model(rng, seed, h=200.0, sim_time=8.0, precision="f32", ntfd=None):
    """One model of the batched workload: fault length U[8,24] km, depth U[6,14] km,
    padded by 30 cells in x on each side and 30 below, nytT=30, 10-cell PML; mu_s, mu_d,
    Dc and prestress drawn as in sw_small."""
    L = rng.uniform(8e3, 24e3)
    W = rng.uniform(6e3, 14e3)
    fx, fz = int(round(L / h)), int(round(W / h))
    nxT, nzT, nyT = fx + 60, fz + 30, 30
    return sw_model(nxT, nyT, nzT, h, sim_time, seed, patch_nodes=(fx, fz), nstations=2, precision=precision,
                    ntfd=ntfd)


def batch_set(n=256, seed=2024, sim_time=8.0, ntfd=None):
    """The batched workload: n seeded models of uneven size (batch_model)."""
    rng = np.random.default_rng(seed)
    return [batch_model(rng, seed * 1000 + q, sim_time=sim_time, ntfd=ntfd) for q in range(n)]


def large_serving_model(rng, seed, sim_time=8.0, ntfd=None):
    """The large request of the serving stream: h=100 m, 40x20 km fault, padded as
    batch_model, 5 seeded layers as sw_large."""
    h = 100.0
    fx, fz = 400, 200
    lay = layered(np.random.default_rng(seed + 7), 5, (fz + 30) * h)
    return sw_model(fx + 60, 30, fz + 30, h, sim_time, seed, layers=lay, patch_nodes=(fx, fz), nstations=2,
                    ntfd=ntfd)


def serving_stream(n=2000, seed=4242, rate=30.0, large_frac=0.05, sim_time=8.0):
    """Poisson arrivals (seeded rate in requests/s): (arrival_s, model) pairs; a fraction
    large_frac of the requests are large_serving_model, the rest batch_model."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, size=n))
    out = []
    for q in range(n):
        if rng.uniform() < large_frac:
            m = large_serving_model(rng, seed * 10000 + q, sim_time=sim_time)
        else:
            m = batch_model(rng, seed * 10000 + q, sim_time=sim_time)
        m["request"] = q
        out.append((float(t[q]), m))
    return out


def fspace_variant(m: dict) -> dict:
    """The same model in the FSPACE build's padding: nfs = nabc, so nabc-2 more planes on
    top, where the fifth PML strip lies (fd3d_init.f90:161-169).  Medium and fault planes
    keep their values for k <= nzt-nfs+2 and repeat the last plane above, so both builds
    see the same model below the former free surface."""
    nab = m["nabc"]
    extra = nab - m["nfs"]
    f = dict(m, fspace=True, nfs=nab, nzt=m["nzt"] + extra)
    f["medium"] = tuple(np.concatenate([np.asarray(a), np.repeat(np.asarray(a)[-1:], extra)]) for a in m["medium"])
    f["fault"] = fortran_planes({k: (np.concatenate([v, np.repeat(v[:, -1:], extra, axis=1)], axis=1)
                                     if isinstance(v, np.ndarray) and v.ndim == 2 else v)
                                 for k, v in m["fault"].items()})
    return f


def tiny_sw(seed=5, nxT=40, nyT=14, nzT=28, h=200.0, nsteps=60, precision="f32", nstations=3, stride=1,
            fspace=False, layers=None, nabc=NABC):
    """Parity-test model: rupture starts on step 1 from an overstressed nucleation patch."""
    return sw_model(nxT, nyT, nzT, h, 1.0, seed, layers=layers, patch_nodes=(nxT - 8, nzT - 8), nstations=nstations,
                    precision=precision, ntfd=nsteps, history_stride=stride, corr_m=600.0, fspace=fspace, nabc=nabc)


def tiny_fvw(seed=6, nxT=40, nyT=14, nzT=28, h=200.0, nsteps=60, precision="f32", stride=1, fspace=False):
    return fvw_model(nxT, nyT, nzT, h, 1.0, seed, fault_m=(6000.0, 4000.0), dt=0.004, history_stride=stride,
                     precision=precision, ntfd=nsteps, border_m=800.0, R=1200.0, TT=0.1, fspace=fspace)


# ---------------------------------------------------------------- reference decks
def _tokens(line, n):
    t = line.split()[:n]
    return [x.replace("d", "e").replace("D", "e") for x in t]


def read_inputfd3d(path):
    """inputfd3d.dat as read by fd3d_init (src/fd3d_init.f90:145-173)."""
    lines = open(path).read().splitlines()
    it = iter(lines)
    nxT, nyT, nzT = (int(x) for x in _tokens(next(it), 3))
    dh = float(_tokens(next(it), 1)[0])
    ntfd = int(_tokens(next(it), 1)[0])
    dt = float(_tokens(next(it), 1)[0])
    dip = float(_tokens(next(it), 1)[0])
    t = _tokens(next(it), 3)
    nabc, pml_vp, pml_fact = int(t[0]), float(t[1]), float(t[2])
    damp_s = float(_tokens(next(it), 1)[0])
    nst = int(_tokens(next(it), 1)[0])
    st = [tuple(int(x) for x in _tokens(next(it), 3)) for _ in range(nst)]
    m = dict(nxt=nxT + 2 * nabc, nyt=nyT + nabc, nzt=nzT + nabc + NFS, nabc=nabc, nfs=NFS, dh=dh, dt=dt,
             ntfd=ntfd, damp_s=damp_s, pml_vp=pml_vp, pml_fact=pml_fact, stations=st, dip=dip)
    return m


def read_crustal(path):
    lines = open(path).read().splitlines()
    nd = int(lines[2].split()[0])
    rows = [[float(x) for x in lines[5 + q].split()[:4]] for q in range(nd)]
    a = np.array(rows)
    return dict(depth=a[:, 0] * 1e3, vp=a[:, 1] * 1e3, vs=a[:, 2] * 1e3, rho=a[:, 3] * 1e3)


def write_deck(model: dict, outdir: str, crustal: dict):
    """Write inputfd3d.dat / crustal.dat for a model in the reference's format."""
    os.makedirs(outdir, exist_ok=True)
    nab = model["nabc"]
    with open(os.path.join(outdir, "inputfd3d.dat"), "w") as f:
        f.write(f"{model['nxt'] - 2 * nab} {model['nyt'] - nab} {model['nzt'] - nab - NFS}\n")
        f.write(f"{model['dh']!r}\n{model['ntfd']}\n{model['dt']!r}\n{model.get('dip', 90.0)!r} -0.\n")
        f.write(f"{nab} {model['pml_vp']!r} {model['pml_fact']!r}\n{model['damp_s']!r}\n")
        st = model.get("stations", [])
        f.write(f"{len(st)}\n")
        for s in st:
            f.write(f"{s[0]} {s[1]} {s[2]}\n")
        f.write("0\n")
    with open(os.path.join(outdir, "crustal.dat"), "w") as f:
        f.write("Crustal model (free format)\nnumber of layers\n")
        f.write(f"  {len(crustal['depth'])}\nParameters of the layers\n")
        f.write("depth of layer top(km)   Vp(km/s)    Vs(km/s)    Rho(g/cm**3)    Qp     Qs\n")
        for dpt, vp, vs, rho in zip(crustal["depth"], crustal["vp"], crustal["vs"], crustal["rho"]):
            f.write(f"{float(dpt) / 1e3!r} {float(vp) / 1e3!r} {float(vs) / 1e3!r} {float(rho) / 1e3!r} 800. 400.\n")


def _scec_sw(scec_path):
    """The scecmodel.dat of the slip-weakening SCEC set-ups (forwardspecialTPV5/8/9,
    src/fd3d_init.f90:549-558, 630-639, 719-728)."""
    lines = open(scec_path).read().splitlines()
    t = _tokens(lines[0], 7)
    r = dict(no0=int(t[0]))
    r.update(zip(("hx0", "hz0", "h1x0", "h1z0", "h2x0", "h2z0"), (float(x) for x in t[1:])))
    r["hdelta"] = float(_tokens(lines[1], 1)[0])
    r.update(zip(("T0", "T0n", "T0h1", "T0h2"), (float(x) for x in _tokens(lines[2], 4))))
    r["sn"] = float(_tokens(lines[3], 1)[0])
    r["mus"], r["muso"] = (float(x) for x in _tokens(lines[4], 2))
    r["mud"] = float(_tokens(lines[5], 1)[0])
    r["d0h"] = float(_tokens(lines[6], 1)[0])
    return r


def _in_box(x, z, cx, cz, hdelta):
    return (x - cx >= -hdelta / 2) & (x - cx <= hdelta / 2) & (z - cz >= -hdelta / 2) & (z - cz <= hdelta / 2)


def _tpv89_fault(m, scec_path, dip_slip):
    """forwardspecialTPV8 (src/fd3d_init.f90:706-783) and forwardspecialTPV9 (:619-704):
    depth-dependent normal stress sigma_n = sn*dh*(nzt-2-k) (+0.5 for TPV8), cohesion
    1 MPa, prestress T0*sigma_n (strike slip in TPV8, dip slip in TPV9) with a
    nucleation square at T0n*mus*sigma_n + coh, the TPV9 surface row at 1/4 and the
    ghost rows mirrored with a sign change of the prestress.  In FP64 (the -r8 build)."""
    r = _scec_sw(scec_path)
    nxt, nzt, dh = m["nxt"], m["nzt"], float(m["dh"])
    shape = (nxt, nzt)
    peak, dyn, Dc, T = (np.zeros(shape) for _ in range(4))
    coh = np.full(shape, 1.e6)
    i = np.arange(1, nxt + 1, dtype=np.float64)[:, None]
    k = np.arange(2, nzt - 1, dtype=np.float64)[None, :]  # k = 2..nzt-2
    sig = r["sn"] * dh * ((nzt - 2 - k) + (0.0 if dip_slip else 0.5))
    ks = slice(1, nzt - 2)
    peak[:, ks] = sig * r["muso"]
    dyn[:, ks] = sig * r["mud"]
    nuc = _in_box((i - 1.0) * dh, (k - 1.0) * dh, r["hx0"], r["hz0"], r["hdelta"])
    T[:, ks] = np.where(nuc, r["T0n"] * r["mus"] * sig + 1.e6, r["T0"] * sig)
    Dc[:, ks] = r["d0h"]
    no0 = r["no0"]
    peak[no0:nxt - no0, no0:nzt - 2] = (sig * r["mus"] + 0.0 * i)[no0:nxt - no0, no0 - 1:]
    if dip_slip:  # TPV9: the surface row k = nzt-2 at a quarter (src/fd3d_init.f90:670-675)
        for a in (peak, dyn, T):
            a[:, nzt - 3] = 0.25 * a[:, nzt - 4]
        Dc[:, nzt - 3] = r["d0h"]
    for a in (peak, dyn, Dc):
        a[:, nzt - 2] = a[:, nzt - 3]
        a[:, nzt - 1] = a[:, nzt - 4]
    T[:, nzt - 2] = -T[:, nzt - 3]
    T[:, nzt - 1] = -T[:, nzt - 4]
    zero = np.zeros(shape)
    sX, sZ = (zero, T) if dip_slip else (T, zero)
    return dict(law="sw", striniX=sX, striniZ=sZ, Dc=Dc, peak_xz=peak, dyn_xz=dyn, coh=coh)


def tpv8_fault(m, scec_path):
    return _tpv89_fault(m, scec_path, dip_slip=False)


def tpv9_fault(m, scec_path):
    """TPV9 is built with -DDIPSLIP (examples/TPV9/compile.sh)."""
    return _tpv89_fault(m, scec_path, dip_slip=True)


def tpv10x_fault(m, scec_path, variant=104):
    """forwardspecialTPV103 / forwardspecialTPV104 (src/fd3d_init.f90:283-501): rate-and-state
    fast-velocity-weakening fault whose a and Vw rise outside a smooth box
    B(x)B(z) (tanh transition of width trans), steady-state psi for the initial slip
    rate, and the TPV103/104 nucleation ramp.  TPV104 tapers only below the
    hypocentre row (its z test is one-sided, the tanh argument uses |z - z0| as there).
    In FP64 (the -r8 build)."""
    lines = open(scec_path).read().splitlines()
    wfx, wfz, hx0t, hz0t, trans, fringe = (float(x) for x in _tokens(lines[0], 6))
    val = [float(_tokens(lines[q], 1)[0]) for q in range(1, 15)]
    f0, v0, a0, b, d0h, fw, vw0, vwd, vini, Tini, Sn, perturb, RRini, TT2 = val
    nxt, nzt, dh, nabc = m["nxt"], m["nzt"], float(m["dh"]), m["nabc"]
    hx0 = hx0t + fringe + nabc * dh
    hz0 = hz0t + fringe + nabc * dh

    def box(d, w, one_sided_dist=None):
        t = np.abs(d) if one_sided_dist is None else one_sided_dist
        ad = np.abs(d)
        mid = (t > w) & (t < w + trans)
        with np.errstate(divide="ignore", invalid="ignore"):
            ramp = 0.5 * (1.0 + np.tanh(trans / (ad - w - trans) + trans / (ad - w)))
        return np.where(t >= w + trans, 0.0, np.where(mid, ramp, 1.0))

    def taper(off):
        hx = np.arange(1, nxt + 1, dtype=np.float64)[:, None] * dh + off
        hz = np.arange(1, nzt + 1, dtype=np.float64)[None, :] * dh + off
        bx = box(hx - hx0, wfx)
        bz = box(hz - hz0, wfz, -(hz - hz0) if variant == 104 else None)
        return bx * bz

    shape = (nxt, nzt)
    T = np.full(shape, Tini)
    Bz_, Bx_ = taper(0.0), taper(dh / 2)
    a = a0 + a0 * (1.0 - Bz_)
    vw = vw0 + vwd * (1.0 - Bz_)
    aX = a0 + a0 * (1.0 - Bx_)
    vwX = vw0 + vwd * (1.0 - Bx_)
    psi = a * (np.log(2 * v0 / (2 * vini)) + np.log(np.sinh(T / (a * Sn))))
    psiX = aX * (np.log(2 * v0 / (2 * vini)) + np.log(np.sinh(T / (aX * Sn))))
    return dict(law="fvw", striniX=T, striniZ=np.zeros(shape), Dc=np.full(shape, d0h), a=a, b=np.full(shape, b),
                psi=psi, vw=vw, aX=aX, bX=np.full(shape, b), psiX=psiX, vwX=vwX, Sn=Sn, v0=v0, f0=f0, fw=fw,
                uini=vini, wini=0.0, nucleation=1, hx0=hx0, hz0=hz0, perturb=perturb, RR2=RRini * RRini, TT2=TT2,
                strinixI=Tini)


def read_forward_model(deck_dir):
    """inversion_init + readinversionresult (src/fd3d_init.f90:786-800, 839-857): the
    NLI x NWI control points of prestress T0I, static friction TsI and Dc from
    forwardmodel.dat (the first two values are skipped as there), Fortran order."""
    lines = open(os.path.join(deck_dir, "inputinv.dat")).read().splitlines()
    nli, nwi = (int(x) for x in _tokens(lines[1], 2))
    vals = [float(x.replace("d", "e").replace("D", "e"))
            for x in open(os.path.join(deck_dir, "forwardmodel.dat")).read().split()]
    n = nli * nwi
    if len(vals) < 2 + 3 * n:
        raise ValueError(f"forwardmodel.dat holds {len(vals)} values, {2 + 3 * n} needed")
    T0I, TsI, DcI = (np.asarray(vals[2 + q * n:2 + (q + 1) * n]).reshape((nli, nwi), order="F") for q in range(3))
    return T0I, TsI, DcI


def inversion_example(deck_dir, dipslip=False, precision="f32"):
    """A model as dynamicsolver builds it without -DSCEC (src/dynamicsolver.f90:56-58):
    the deck's grid and medium, and the fault from the control points of forwardmodel.dat,
    which Solver uploads with fd3d_upload_fault_model (interpolation on the device)."""
    m = read_inputfd3d(os.path.join(deck_dir, "inputfd3d.dat"))
    cr = read_crustal(os.path.join(deck_dir, "crustal.dat"))
    lam, mu, d, vpm = crustal_medium(m["nzt"], m["dh"], m["dip"], cr["depth"], cr["vp"], cr["vs"], cr["rho"])
    T0I, TsI, DcI = read_forward_model(deck_dir)
    m.update(medium=(lam, mu, d), vp_max=vpm, precision=precision, history_stride=1, law="sw",
             fault_model=dict(T0I=T0I, TsI=TsI, DcI=DcI, dip=m["dip"], dipslip=dipslip))
    return m


SCEC_SETUPS = {"TPV5": None, "TPV8": tpv8_fault, "TPV9": tpv9_fault,
               "TPV103": lambda m, p: tpv10x_fault(m, p, 103), "TPV104": lambda m, p: tpv10x_fault(m, p, 104)}


def reference_example(deck_dir, setup, precision="f32", fspace=False):
    """A model from one of the reference's example directories (inputfd3d.dat,
    crustal.dat, scecmodel.dat), as dynamicsolver builds it with -DSCEC -D<setup>
    (src/dynamicsolver.f90:39-57): fd3d_init, readcrustalmodel and forwardspecial<setup>."""
    m = read_inputfd3d(os.path.join(deck_dir, "inputfd3d.dat"))
    if fspace:
        nab = m["nabc"]
        m.update(fspace=True, nfs=nab, nzt=m["nzt"] + nab - NFS)
    cr = read_crustal(os.path.join(deck_dir, "crustal.dat"))
    lam, mu, d, vpm = crustal_medium(m["nzt"], m["dh"], m["dip"], cr["depth"], cr["vp"], cr["vs"], cr["rho"],
                                     nfs=m["nfs"])
    m.update(medium=(lam, mu, d), vp_max=vpm, precision=precision, history_stride=1)
    scec = os.path.join(deck_dir, "scecmodel.dat")
    fault = tpv5_fault(m, scec) if setup == "TPV5" else SCEC_SETUPS[setup](m, scec)
    m["fault"] = fortran_planes(fault)
    m["law"] = fault["law"]
    return m


def tpv5_fault(m, scec_path):
    """forwardspecialTPV5 (src/fd3d_init.f90:535-617) from scecmodel.dat."""
    lines = open(scec_path).read().splitlines()
    t = _tokens(lines[0], 7)
    no0 = int(t[0]); hx0, hz0, h1x0, h1z0, h2x0, h2z0 = (float(x) for x in t[1:])
    hdelta = float(_tokens(lines[1], 1)[0])
    T0, T0n, T0h1, T0h2 = (float(x) for x in _tokens(lines[2], 4))
    sn = float(_tokens(lines[3], 1)[0])
    mus, muso = (float(x) for x in _tokens(lines[4], 2))
    mud = float(_tokens(lines[5], 1)[0])
    d0h = float(_tokens(lines[6], 1)[0])
    nxt, nzt, dh = m["nxt"], m["nzt"], np.float64(m["dh"])
    sX = np.zeros((nxt, nzt)); peak = np.zeros((nxt, nzt)); dyn = np.zeros((nxt, nzt)); Dc = np.zeros((nxt, nzt))
    for i in range(1, nxt + 1):
        for k in range(1, nzt - 1):
            x = (i - 1.0) * dh; z = (k - 1.0) * dh
            v = T0
            for cx, cz, val in ((hx0, hz0, T0n), (h1x0, h1z0, T0h1), (h2x0, h2z0, T0h2)):
                if -hdelta / 2 <= x - cx <= hdelta / 2 and -hdelta / 2 <= z - cz <= hdelta / 2:
                    v = val
            sX[i - 1, k - 1] = v
            peak[i - 1, k - 1] = sn * muso
            dyn[i - 1, k - 1] = sn * mud
            Dc[i - 1, k - 1] = d0h
    peak[no0:nxt - no0, no0:nzt - 2] = sn * mus
    for a in (peak, dyn, Dc, sX):
        a[:, nzt - 2] = a[:, nzt - 3]
        a[:, nzt - 1] = a[:, nzt - 4]
    return dict(law="sw", striniX=sX, striniZ=np.zeros((nxt, nzt)), Dc=Dc, peak_xz=peak, dyn_xz=dyn,
                coh=np.zeros((nxt, nzt)))

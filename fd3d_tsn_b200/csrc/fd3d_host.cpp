// fd3d_host.cpp -- input decks and result files in the reference's formats.
//
//   inputfd3d.dat  read as fd3d_init does (src/fd3d_init.f90:145-173)
//   crustal.dat    read and turned into lam1/mu1/d1 as readcrustalmodel does
//                  (src/fd3d_init.f90:211-279), including the CFL stop
//   result/*.res   unformatted stream of `real` planes, x fastest
//                  (src/fd3d_theo.f90:133-145, 546-553)
//   stan<i>.txt    list-directed "u v w" per step (src/fd3d_theo.f90:117-128, 555-557)
//   post-loop planes as text, one value per line (src/fd3d_theo.f90:687-708)
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>
#include "fd3d_host.h"

namespace {

bool read_tokens(std::ifstream& in, int n, std::vector<std::string>& out) {
    std::string line;
    if (!std::getline(in, line)) return false;
    std::istringstream ss(line);
    out.clear();
    std::string t;
    while ((int)out.size() < n && ss >> t) out.push_back(t);
    return (int)out.size() == n;
}

// Fortran list-directed numbers may carry a d/D exponent
double num(const std::string& s) {
    std::string t = s;
    for (char& ch : t) if (ch == 'd' || ch == 'D') ch = 'e';
    char* end = nullptr;
    const double v = std::strtod(t.c_str(), &end);
    if (end == t.c_str()) return std::nan("");  // not a number: the caller reports FD3D_ERR_IO
    return v;
}

std::string path(const char* dir, const char* name) {
    std::string d(dir);
    if (!d.empty() && d.back() != '/') d += '/';
    return d + name;
}

}  // namespace

namespace fd3d {

int write_results(fd3d_ctx* ctx, const fd3d_params& p, int nf, int& rec_written, const char* dir, int rk) {
    int have = 0;
    int rc = fd3d_history_records(ctx, &have);
    if (rc) return rc;
    const int nxT = p.nxt - 2 * p.nabc, nzT = p.nzt - p.nfs - p.nabc;
    const size_t plane = (size_t)nxT * nzT;
    static const char* names[5] = {"sliprateX.res", "sliprateZ.res", "shearstressX.res", "shearstressZ.res", "psi.res"};
    const char* mode = rec_written == 0 ? "wb" : "ab";
    std::vector<char> buf(plane * (size_t)rk);
    for (int fld = 0; fld < nf; ++fld) {
        FILE* fp = std::fopen(path(dir, names[fld]).c_str(), mode);
        if (!fp) return FD3D_ERR_IO;
        for (int r = rec_written; r < have; ++r) {
            rc = fd3d_fetch_history(ctx, fld, r, 1, buf.data(), rk);
            if (rc) { std::fclose(fp); return rc; }
            if (std::fwrite(buf.data(), 1, buf.size(), fp) != buf.size()) { std::fclose(fp); return FD3D_ERR_IO; }
        }
        std::fclose(fp);
    }
    if (p.nstations > 0 && have > rec_written) {
        std::vector<double> s((size_t)(have - rec_written) * 3 * p.nstations);
        rc = fd3d_fetch_stations(ctx, rec_written, have - rec_written, s.data());
        if (rc) return rc;
        for (int st = 0; st < p.nstations; ++st) {
            char nm[32];
            std::snprintf(nm, sizeof nm, "stan%d.txt", st);
            FILE* fp = std::fopen(path(dir, nm).c_str(), rec_written == 0 ? "w" : "a");
            if (!fp) return FD3D_ERR_IO;
            for (int r = 0; r < have - rec_written; ++r) {
                const double* v = s.data() + ((size_t)r * p.nstations + st) * 3;
                std::fprintf(fp, " %23.15E %23.15E %23.15E\n", v[0], v[1], v[2]);
            }
            std::fclose(fp);
        }
    }
    rec_written = have;
    int done = 0;
    fd3d_steps_done(ctx, &done);
    if (done >= p.ntfd && p.ntfd > 0) {
        const size_t n2 = (size_t)p.nxt * p.nzt;
        std::vector<double> sx(n2), sz(n2), rt(n2), ri(n2), stt(n2), cx(n2), cz(n2), t0x(n2), t0z(n2);
        rc = fd3d_fetch_final(ctx, sx.data(), sz.data(), rt.data(), ri.data(), stt.data());
        rc |= fd3d_fetch_plane(ctx, FD3D_PLANE_SCHANGEX, cx.data());
        rc |= fd3d_fetch_plane(ctx, FD3D_PLANE_SCHANGEZ, cz.data());
        rc |= fd3d_fetch_plane(ctx, FD3D_PLANE_T0X, t0x.data());
        rc |= fd3d_fetch_plane(ctx, FD3D_PLANE_T0Z, t0z.data());
        if (rc) return FD3D_ERR_CUDA;
        struct Out { const char* name; std::vector<double>* v; const std::vector<double>* minus; };
        Out outs[] = {{"risetime.res", &ri, nullptr}, {"ruptime.res", &rt, nullptr}, {"slipX.res", &sx, nullptr},
                      {"slipZ.res", &sz, nullptr}, {"stressdropX.res", &cx, &t0x}, {"stressdropZ.res", &cz, &t0z}};
        const bool f32 = p.precision == FD3D_PREC_F32;
        for (const Out& o : outs) {
            FILE* fp = std::fopen(path(dir, o.name).c_str(), "w");
            if (!fp) return FD3D_ERR_IO;
            for (int k = p.nabc + 1; k <= p.nzt - p.nfs; ++k)
                for (int i = p.nabc + 1; i <= p.nxt - p.nabc; ++i) {
                    const size_t q = (size_t)(i - 1) + (size_t)p.nxt * (k - 1);
                    double v = (*o.v)[q];
                    if (o.minus)  // SCHANGE - T0 in `real` (fd3d_theo.f90:604-605)
                        v = f32 ? (double)((float)v - (float)(*o.minus)[q]) : v - (*o.minus)[q];
                    std::fprintf(fp, " %23.15E\n", v);
                }
            std::fclose(fp);
        }
        // rupture contour, cohesive zone and rupture velocity (fd3d_theo.f90:710-749),
        // the last two computed on the device by fd3d_post_process
        double summary[4];
        std::vector<double> rvel(n2), czone(n2);
        if (fd3d_post_process(ctx, summary) || fd3d_fetch_plane(ctx, FD3D_PLANE_RVEL, rvel.data()) ||
            fd3d_fetch_plane(ctx, FD3D_PLANE_CZONE, czone.data()))
            return FD3D_ERR_CUDA;
        FILE* fc = std::fopen(path(dir, "contour.res").c_str(), "w");
        FILE* fz = std::fopen(path(dir, "czone.res").c_str(), "w");
        FILE* fv = std::fopen(path(dir, "rvel.res").c_str(), "w");
        if (!fc || !fz || !fv) {
            if (fc) std::fclose(fc);
            if (fz) std::fclose(fz);
            if (fv) std::fclose(fv);
            return FD3D_ERR_IO;
        }
        std::fprintf(fc, " j k t\n");
        for (int k = p.nabc + 1; k <= p.nzt - p.nfs; ++k)
            for (int i = p.nabc + 1; i <= p.nxt - p.nabc; ++i) {
                const size_t q = (size_t)(i - 1) + (size_t)p.nxt * (k - 1);
                double x, z;
                if (f32) {
                    const float dh = (float)p.dh;
                    x = (double)(((float)(i - p.nabc - 1) - (float)(p.nxt - 2 * p.nabc) / 2.f) * dh);
                    z = (double)((float)(p.nzt - k - p.nabc - 1) * dh);
                } else {
                    x = ((double)(i - p.nabc - 1) - (double)(p.nxt - 2 * p.nabc) / 2.) * p.dh;
                    z = (double)(p.nzt - k - p.nabc - 1) * p.dh;
                }
                std::fprintf(fc, " %23.15E %23.15E %23.15E\n", x, z, rt[q]);
                std::fprintf(fz, " %23.15E\n", czone[q]);
                std::fprintf(fv, " %23.15E\n", rvel[q]);
            }
        std::fclose(fc);
        std::fclose(fz);
        std::fclose(fv);
    }
    return FD3D_OK;
}

}  // namespace fd3d

extern "C" {

void fd3d_free(void* p) { std::free(p); }

int fd3d_read_deck(const char* dir, fd3d_params* p, double** lam1, double** mu1, double** d1) {
    return fd3d_read_deck_ex(dir, 0, p, lam1, mu1, d1);
}

int fd3d_read_deck_ex(const char* dir, int fspace, fd3d_params* p, double** lam1, double** mu1, double** d1) {
    if (!dir || !p || (fspace != 0 && fspace != 1)) return FD3D_ERR_ARG;
    std::ifstream in(path(dir, "inputfd3d.dat"));
    if (!in) return FD3D_ERR_IO;
    std::vector<std::string> t;
    std::memset(p, 0, sizeof *p);
    if (!read_tokens(in, 3, t)) return FD3D_ERR_IO;
    const int nxtT = std::atoi(t[0].c_str()), nytT = std::atoi(t[1].c_str()), nztT = std::atoi(t[2].c_str());
    if (!read_tokens(in, 1, t)) return FD3D_ERR_IO;
    p->dh = num(t[0]);
    if (!(p->dh > 0)) return FD3D_ERR_IO;
    if (!read_tokens(in, 1, t)) return FD3D_ERR_IO;
    p->ntfd = std::atoi(t[0].c_str());
    if (!read_tokens(in, 1, t)) return FD3D_ERR_IO;
    p->dt = num(t[0]);
    if (!(p->dt > 0)) return FD3D_ERR_IO;
    if (!read_tokens(in, 1, t)) return FD3D_ERR_IO;
    const double dip = num(t[0]);
    if (!read_tokens(in, 3, t)) return FD3D_ERR_IO;
    p->nabc = std::atoi(t[0].c_str());
    p->pml_vp = num(t[1]);
    p->pml_fact = num(t[2]);
    if (!read_tokens(in, 1, t)) return FD3D_ERR_IO;
    p->damp_s = num(t[0]);
    if (!read_tokens(in, 1, t)) return FD3D_ERR_IO;
    p->nstations = std::atoi(t[0].c_str());
    if (p->nstations < 0 || p->nstations > FD3D_MAX_STATIONS) return FD3D_ERR_ARG;
    for (int s = 0; s < p->nstations; ++s) {
        if (!read_tokens(in, 3, t)) return FD3D_ERR_IO;
        p->staX[s] = std::atoi(t[0].c_str()); p->staY[s] = std::atoi(t[1].c_str()); p->staZ[s] = std::atoi(t[2].c_str());
    }
    p->fspace = fspace;
    p->nfs = fspace ? p->nabc : 2;  // fd3d_init.f90:161-165
    p->nxt = nxtT + 2 * p->nabc;
    p->nyt = nytT + p->nabc;
    p->nzt = nztT + p->nabc + p->nfs;
    p->law = FD3D_LAW_SW;
    p->precision = FD3D_PREC_F32;
    p->history_stride = 1;

    std::ifstream cr(path(dir, "crustal.dat"));
    if (!cr) return FD3D_ERR_IO;
    std::string line;
    std::getline(cr, line); std::getline(cr, line);
    if (!read_tokens(cr, 1, t)) return FD3D_ERR_IO;
    const int nd = std::atoi(t[0].c_str());
    if (nd < 1) return FD3D_ERR_IO;
    std::getline(cr, line); std::getline(cr, line);
    std::vector<double> depth(nd), vp(nd), vs(nd), rho(nd);
    for (int k = 0; k < nd; ++k) {
        if (!read_tokens(cr, 4, t)) return FD3D_ERR_IO;
        depth[k] = num(t[0]) * 1.e3; vp[k] = num(t[1]) * 1.e3; vs[k] = num(t[2]) * 1.e3; rho[k] = num(t[3]) * 1.e3;
        if (!std::isfinite(depth[k] + vp[k] + vs[k] + rho[k])) return FD3D_ERR_IO;
    }
    const int nxt = p->nxt, nyt = p->nyt, nzt = p->nzt, nfs = p->nfs;
    const size_t n3 = (size_t)nxt * nyt * nzt;
    double* L = (double*)std::malloc(n3 * sizeof(double));
    double* M = (double*)std::malloc(n3 * sizeof(double));
    double* D = (double*)std::malloc(n3 * sizeof(double));
    if (!L || !M || !D) { std::free(L); std::free(M); std::free(D); return FD3D_ERR_NOMEM; }
    const double PI = 3.1415926535;
    double vpmax = 0;
    for (int k = nzt; k >= 1; --k) {  // fd3d_init.f90:241-265
        const double dum = (p->dh * (double)(nzt - nfs - k) + p->dh / 2.) * std::sin(dip / 180. * PI);
        double vpp, vss, dd;
        if (dum > depth[nd - 1]) { vpp = vp[nd - 1]; vss = vs[nd - 1]; dd = rho[nd - 1]; }
        else {
            int j = 2;
            for (; j <= nd; ++j) if (dum < depth[j - 1]) break;
            vpp = vp[j - 2]; vss = vs[j - 2]; dd = rho[j - 2];
        }
        vpmax = std::max(vpmax, vpp);
        const double l = dd * (vpp * vpp - 2. * vss * vss), m = dd * vss * vss;
        for (size_t q = (size_t)nxt * nyt * (k - 1); q < (size_t)nxt * nyt * k; ++q) { L[q] = l; M[q] = m; D[q] = dd; }
    }
    p->vp_max = vpmax;
    if (vpmax * p->dt / p->dh > 0.25) { std::free(L); std::free(M); std::free(D); return FD3D_ERR_CFL; }
    if (lam1) *lam1 = L; else std::free(L);
    if (mu1) *mu1 = M; else std::free(M);
    if (d1) *d1 = D; else std::free(D);
    return FD3D_OK;
}

}  // extern "C"

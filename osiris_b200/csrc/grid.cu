// Host side of the grid path: model upload, per-component and geometric
// constants, the property sweeps, and their C-ABI entry points.
#include <cuda_runtime.h>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>
#include "osiris_b200.h"

#include "grid_internal.h"

namespace osr {

static osr_status gfail(cudaError_t) { return OSR_ERR_CUDA; }

#define GRID_CUDA(call)                             \
    do {                                            \
        cudaError_t e_ = (call);                    \
        if (e_ != cudaSuccess) return gfail(e_);    \
    } while (0)

GridScalars grid_scalars(const osr_grid &g) {
    GridScalars s;
    s.nx = g.nx;
    s.ny = g.ny;
    s.nz = g.nz;
    s.cells = g.cells;
    s.wat_ro = g.wat_ro;
    s.wat_mu = g.wat_mu;
    s.refp = g.refp;
    s.cpor = g.cpor;
    s.dcpor = g.dcpor;
    s.const_dif = g.const_dif;
    s.cdif = g.cdif;
    s.swt = g.d_swt;
    s.sgt = g.d_sgt;
    s.nswt = (int)g.swt.size() / 4;
    s.nsgt = (int)g.sgt.size() / 4;
    return s;
}

template <int N>
static osr_status update_n(osr_grid &g, cudaStream_t st) {
    GridArgs<N> a;
    make_grid_fluid<N>(g, a.g);
    a.s = grid_scalars(g);
    a.geo = GridGeom{g.di, g.dj, g.dk, g.blockH};
    a.m[0] = g.m[0];
    a.m[1] = g.m[1];
    long blocks = (g.cells + 127) / 128;
    if (blocks > 148L * 16) blocks = 148L * 16;
    cell_props_kernel<N><<<dim3((unsigned)blocks, 2), 128, 0, st>>>(a);
    GRID_CUDA(cudaGetLastError());
    face_trans_kernel<N><<<dim3((unsigned)blocks, 2), 128, 0, st>>>(a);
    GRID_CUDA(cudaGetLastError());
    return OSR_OK;
}

osr_status grid_update(osr_grid &g, cudaStream_t s) {
    switch (g.nc) {
#define GRID_NC(K) \
    case K: return update_n<K>(g, s);
        GRID_NC(1) GRID_NC(2) GRID_NC(3) GRID_NC(4) GRID_NC(5) GRID_NC(6) GRID_NC(7) GRID_NC(8) GRID_NC(9)
        GRID_NC(10) GRID_NC(11) GRID_NC(12) GRID_NC(13) GRID_NC(14) GRID_NC(15) GRID_NC(16)
#undef GRID_NC
        default: return OSR_ERR_NC;
    }
}

// Geometry of IFK_Calc (compsim/Init_Calcs.cpp:21-46) and CalcBlockHeight
// (:993-1011), on the host once per model.
static void geometry(const osr_grid &g, const double *di, const double *dj, const double *dk, const double *por,
                     const double *perm, std::vector<double> &ift, std::vector<double> &blockH) {
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    const long n = g.cells;
    const double SI_C = 9.869232667160128e-13;
    ift.assign(3 * n, 0.0);
    blockH.assign(n, 0.0);
    for (int i = 0; i < nx; i++)
        for (int j = 0; j < ny; j++)
            for (int k = 0; k < nz; k++) {
                long c = i + (long)nx * (j + (long)ny * k);
                long cx = c + 1, cy = c + nx, cz = c + (long)nx * ny;
                if ((nx != 1) && (i != nx - 1) && (por[c] > 1e-10) && (por[cx] > 1e-10))
                    ift[c] = SI_C * 2 * dj[j] * dk[k] / (di[i] / perm[c] + di[i + 1] / perm[cx]);
                if ((ny != 1) && (j != ny - 1) && (por[c] > 1e-10) && (por[cy] > 1e-10))
                    ift[n + c] = SI_C * 2 * di[i] * dk[k] / (dj[j] / perm[n + c] + dj[j + 1] / perm[n + cy]);
                if ((nz != 1) && (k != nz - 1) && (por[c] > 1e-10) && (por[cz] > 1e-10))
                    ift[2 * n + c] = SI_C * 2 * di[i] * dj[j] / (dk[k] / perm[2 * n + c] + dk[k + 1] / perm[2 * n + cz]);
            }
    for (int i = 0; i < nx; i++)
        for (int j = 0; j < ny; j++) {
            double h = 0;
            for (int k = nz - 1; k >= 0; k--) {
                if (k == nz - 1) h = 0.5 * dk[nz - 1];
                else h += 0.5 * (dk[k] + dk[k + 1]);
                blockH[i + (long)nx * (j + (long)ny * k)] = h;
            }
        }
}

}  // namespace osr

using namespace osr;

// Field table: name -> (medium member offset, count of [cells] planes, type)
namespace {
struct FieldRef {
    double *d;
    signed char *c;
    long planes;
};

FieldRef find_field(osr_grid *g, const std::string &name) {
    FieldRef r{nullptr, nullptr, 0};
    if (name.size() < 3 || name[1] != '.' || (name[0] != 'm' && name[0] != 'f')) return r;
    osr::MediumFields &F = g->m[name[0] == 'f' ? 1 : 0];
    std::string k = name.substr(2);
    const long nc = g->nc;
    if (k == "P") r = {F.P, nullptr, 3};
    else if (k == "sat") r = {F.sat, nullptr, 3};
    else if (k == "x") r = {F.x, nullptr, nc};
    else if (k == "y") r = {F.y, nullptr, nc};
    else if (k == "z") r = {F.z, nullptr, nc};
    else if (k == "label") r = {nullptr, F.label, 1};
    else if (k == "rho") r = {F.rho, nullptr, 2};
    else if (k == "pc") r = {F.pc, nullptr, 2};
    else if (k == "mu") r = {F.mu, nullptr, 2};
    else if (k == "gam") r = {F.gam, nullptr, 2};
    else if (k == "kr") r = {F.kr, nullptr, 3};
    else if (k == "dkr") r = {F.dkr, nullptr, 5};
    else if (k == "dE") r = {F.dE, nullptr, 2 * (nc + 1)};
    else if (k == "pre") r = {F.pre, nullptr, nc + 1};
    else if (k == "diff") r = {F.diff, nullptr, 2 * nc};
    else if (k == "ift") r = {F.ift, nullptr, 1};
    else if (k == "trans") r = {F.trans, nullptr, 36};
    else if (k == "transS") r = {nullptr, F.transS, 9};
    else if (k == "wtran") r = {F.wtran, nullptr, 3};
    else if (k == "dwtran") r = {F.dwtran, nullptr, 3};
    else if (k == "por") r = {F.por, nullptr, 1};
    else if (k == "perm") r = {F.perm, nullptr, 3};
    else if (k == "iftran") r = {F.iftran, nullptr, 3};
    return r;
}
}  // namespace


namespace osr {

// Per cell-medium check of the primary state: every pressure, saturation
// and phase composition finite, the oil pressure positive.  The first bad
// block (matrix blocks 0..cells-1, then fracture) is kept by an atomic min.
__global__ void grid_status_kernel(MediumFields m0, MediumFields m1, long n, int nc, unsigned long long *first,
                                   unsigned *codes) {
    for (long b = (long)blockIdx.x * blockDim.x + threadIdx.x; b < 2 * n; b += (long)gridDim.x * blockDim.x) {
        const MediumFields &F = b >= n ? m1 : m0;
        const long c = b >= n ? b - n : b;
        unsigned code = 0;
        for (int p = 0; p < 3; p++) {
            if (!isfinite(F.P[(long)p * n + c]) || !isfinite(F.sat[(long)p * n + c])) code |= 1u;
        }
        for (int i = 0; i < nc; i++)
            if (!isfinite(F.x[(long)i * n + c]) || !isfinite(F.y[(long)i * n + c])) code |= 1u;
        if (!(F.P[n + c] > 0)) code |= 2u;
        if (code) {
            atomicMin(first, (unsigned long long)b);
            atomicOr(codes, code);
        }
    }
}

}  // namespace osr

extern "C" {

osr_status osr_grid_create(const osr_model *md, osr_grid **out) {
    if (!md || !out) return OSR_ERR_ARG;
    *out = nullptr;
    if (md->nx < 1 || md->ny < 1 || md->nz < 1) return OSR_ERR_ARG;
    if (md->nc < 1 || md->nc > OSR_MAX_NC) return OSR_ERR_NC;
    if (md->eos != OSR_EOS_PR && md->eos != OSR_EOS_SRK) return OSR_ERR_ARG;
    if (!md->di || !md->dj || !md->dk || !md->por || !md->fpor || !md->perm || !md->fperm || !md->mw || !md->tc ||
        !md->pc || !md->vc || !md->acf || !md->zc || !md->kij || !md->swt || !md->sgt || md->nswt < 1 ||
        md->nsgt < 1)
        return OSR_ERR_ARG;
    osr_grid *g = new osr_grid();
    g->nx = md->nx;
    g->ny = md->ny;
    g->nz = md->nz;
    g->nc = md->nc;
    g->eos = md->eos;
    g->cells = (long)md->nx * md->ny * md->nz;
    g->T = md->restemp;
    g->wat_ro = md->wat_ro;
    g->wat_mu = md->wat_mu;
    g->refp = md->refp;
    g->cpor = md->cpor;
    g->dcpor = md->dcpor;
    g->lf = md->lf;
    g->re_f = md->re_f;
    g->sigma = md->sigma;
    g->const_dif = md->has_cdif;
    g->cdif = md->cdif;
    const int nc = md->nc;
    auto cp = [&](std::vector<double> &v, const double *p, long n) { v.assign(p, p + n); };
    cp(g->mw, md->mw, nc);
    cp(g->tc, md->tc, nc);
    cp(g->pc, md->pc, nc);
    cp(g->vc, md->vc, nc);
    cp(g->acf, md->acf, nc);
    cp(g->zc, md->zc, nc);
    if (md->parachor) cp(g->parachor, md->parachor, nc);
    else g->parachor.assign(nc, 0.0);
    cp(g->kij, md->kij, (long)nc * nc);
    cp(g->swt, md->swt, 4L * md->nswt);
    cp(g->sgt, md->sgt, 4L * md->nsgt);
    g->nwells = md->nwells;
    if (md->nwells > 0 && md->wells_i && md->wells_f) {
        g->wells_i.assign(md->wells_i, md->wells_i + 5L * md->nwells);
        g->wells_f.assign(md->wells_f, md->wells_f + (long)(nc + 6) * md->nwells);
    }
    // one device block for everything
    const long n = g->cells;
    const long nd_med = n * (3 + 3 + 3L * nc + 2 * 4 + 3 + 5 + 2L * (nc + 1) + (nc + 1) + 2L * nc + 1 + 36 + 3 + 3 +
                             1 + 3 + 3);
    const long nb_med = n * (1 + 9);  // label, transS
    const long nd = 2 * nd_med + md->nx + md->ny + md->nz + n + 4L * md->nswt + 4L * md->nsgt;
    size_t bytes = (size_t)nd * 8 + (size_t)(2 * nb_med) + 4096;
    if (cudaMalloc((void **)&g->block, bytes) != cudaSuccess) {
        delete g;
        return OSR_ERR_CUDA;
    }
    g->block_bytes = bytes;
    cudaMemset(g->block, 0, bytes);
    double *p = (double *)g->block;
    auto take = [&](long k) { double *r = p; p += k; return r; };
    for (int m = 0; m < 2; m++) {
        osr::MediumFields &F = g->m[m];
        F.P = take(3 * n);
        F.sat = take(3 * n);
        F.x = take(nc * n);
        F.y = take(nc * n);
        F.z = take(nc * n);
        F.rho = take(2 * n);
        F.pc = take(2 * n);
        F.mu = take(2 * n);
        F.gam = take(2 * n);
        F.kr = take(3 * n);
        F.dkr = take(5 * n);
        F.dE = take(2L * (nc + 1) * n);
        F.pre = take((nc + 1) * n);
        F.diff = take(2L * nc * n);
        F.ift = take(n);
        F.trans = take(36 * n);
        F.wtran = take(3 * n);
        F.dwtran = take(3 * n);
        F.por = take(n);
        F.perm = take(3 * n);
        F.iftran = take(3 * n);
    }
    g->di = take(md->nx);
    g->dj = take(md->ny);
    g->dk = take(md->nz);
    g->blockH = take(n);
    g->d_swt = take(4L * md->nswt);
    g->d_sgt = take(4L * md->nsgt);
    signed char *q = (signed char *)p;
    for (int m = 0; m < 2; m++) {
        g->m[m].label = q;
        q += n;
        g->m[m].transS = q;
        q += 9 * n;
    }
    // static fields
    std::vector<double> ift, bh;
    cudaError_t e = cudaSuccess;
    auto up = [&](void *dst, const void *src, size_t b) {
        if (e == cudaSuccess) e = cudaMemcpy(dst, src, b, cudaMemcpyHostToDevice);
    };
    for (int m = 0; m < 2; m++) {
        const double *por = m ? md->fpor : md->por, *perm = m ? md->fperm : md->perm;
        osr::geometry(*g, md->di, md->dj, md->dk, por, perm, ift, bh);
        up(g->m[m].por, por, n * 8);
        up(g->m[m].perm, perm, 3 * n * 8);
        up(g->m[m].iftran, ift.data(), 3 * n * 8);
    }
    up(g->blockH, bh.data(), n * 8);
    up(g->di, md->di, md->nx * 8);
    up(g->dj, md->dj, md->ny * 8);
    up(g->dk, md->dk, md->nz * 8);
    up(g->d_swt, md->swt, 4L * md->nswt * 8);
    up(g->d_sgt, md->sgt, 4L * md->nsgt * 8);
    if (e != cudaSuccess) {
        cudaFree(g->block);
        delete g;
        return osr::gfail(e);
    }
    osr_status st = osr::grid_assembly_init(*g, md);
    if (st != OSR_OK) {
        osr::grid_assembly_free(*g);
        cudaFree(g->block);
        delete g;
        return st;
    }
    *out = g;
    return OSR_OK;
}

osr_status osr_grid_destroy(osr_grid *g) {
    if (!g) return OSR_ERR_ARG;
    osr::grid_assembly_free(*g);
    if (g->block) cudaFree(g->block);
    delete g;
    return OSR_OK;
}

osr_status osr_grid_set_pressures(osr_grid *g, int medium, const double *P) {
    if (!g || (medium != 0 && medium != 1) || !P) return OSR_ERR_ARG;
    if (cudaMemcpy(g->m[medium].P, P, 3 * g->cells * 8, cudaMemcpyHostToDevice) != cudaSuccess)
        return OSR_ERR_CUDA;
    return OSR_OK;
}

osr_status osr_grid_set_state(osr_grid *g, int medium, const double *P_oil, const double *sat, const double *x,
                              const double *y, const double *z, const signed char *label, const double *rho) {
    if (!g || (medium != 0 && medium != 1) || !P_oil || !sat || !x || !y || !z || !label) return OSR_ERR_ARG;
    osr::MediumFields &F = g->m[medium];
    const long n = g->cells, nc = g->nc;
    cudaError_t e = cudaSuccess;
    auto up = [&](void *dst, const void *src, size_t b) {
        if (e == cudaSuccess) e = cudaMemcpy(dst, src, b, cudaMemcpyHostToDevice);
    };
    up(F.P + n, P_oil, n * 8);
    up(F.sat, sat, 3 * n * 8);
    up(F.x, x, nc * n * 8);
    up(F.y, y, nc * n * 8);
    up(F.z, z, nc * n * 8);
    up(F.label, label, n);
    if (rho) up(F.rho, rho, 2 * n * 8);
    if (e != cudaSuccess) return osr::gfail(e);
    return OSR_OK;
}

osr_status osr_grid_update_dependencies(osr_grid *g, void *stream) {
    if (!g) return OSR_ERR_ARG;
    return osr::grid_update(*g, (cudaStream_t)stream);
}

long osr_grid_field_size(osr_grid *g, const char *field) {
    if (!g || !field) return -1;
    FieldRef r = find_field(g, field);
    if (!r.d && !r.c) return -1;
    return r.planes * g->cells;
}

osr_status osr_grid_get(osr_grid *g, const char *field, double *out) {
    if (!g || !field || !out) return OSR_ERR_ARG;
    FieldRef r = find_field(g, field);
    if (!r.d && !r.c) return OSR_ERR_ARG;
    const long cnt = r.planes * g->cells;
    if (r.d) {
        if (cudaMemcpy(out, r.d, cnt * 8, cudaMemcpyDeviceToHost) != cudaSuccess) return osr::gfail(cudaGetLastError());
    } else {
        std::vector<signed char> tmp(cnt);
        if (cudaMemcpy(tmp.data(), r.c, cnt, cudaMemcpyDeviceToHost) != cudaSuccess)
            return osr::gfail(cudaGetLastError());
        for (long i = 0; i < cnt; i++) out[i] = tmp[i];
    }
    return OSR_OK;
}

osr_status osr_grid_dims(osr_grid *g, int *dims) {
    if (!g || !dims) return OSR_ERR_ARG;
    dims[0] = g->nx;
    dims[1] = g->ny;
    dims[2] = g->nz;
    dims[3] = g->nc;
    return OSR_OK;
}

osr_status osr_grid_status(osr_grid *g, int *code, long *first_bad_block) {
    if (!g || !code || !first_bad_block) return OSR_ERR_ARG;
    unsigned long long *d = nullptr;
    if (cudaMalloc((void **)&d, 16) != cudaSuccess) return osr::gfail(cudaGetLastError());
    const unsigned long long init[2] = {~0ull, 0ull};
    cudaError_t e = cudaMemcpy(d, init, 16, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        long blocks = (2 * g->cells + 255) / 256;
        if (blocks > 148 * 16) blocks = 148 * 16;
        osr::grid_status_kernel<<<(unsigned)blocks, 256>>>(g->m[0], g->m[1], g->cells, g->nc, d, (unsigned *)(d + 1));
        e = cudaGetLastError();
    }
    unsigned long long h[2] = {0, 0};
    if (e == cudaSuccess) e = cudaMemcpy(h, d, 16, cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess) return osr::gfail(e);
    const unsigned bits = (unsigned)h[1];
    *code = (bits & 1u) ? OSR_CELL_NAN : (bits & 2u) ? OSR_CELL_RANGE : OSR_CELL_OK;
    *first_bad_block = bits ? (long)h[0] : -1;
    return OSR_OK;
}

}  // extern "C"

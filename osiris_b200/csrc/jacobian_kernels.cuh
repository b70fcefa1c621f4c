// Analytic Jacobian of the dual-porosity residual (FP64).
//
// The reference assembles its Jacobian row by row (IteratorJacobian,
// compsim/Petsc_Functions.cpp:6898-42073) from hand-derived derivatives of
// every residual term: flux mobilities through dRho/dP, dRho/dx (dE),
// viscosity derivatives (DiffVisco, compsim/Mass_Tran.cpp:307-399) and
// diffusion-coefficient derivatives (DifDiffusion, :107-305), the saturation
// factors of the face transmissibilities, and the matrix-fracture transfer.
// Those derivatives are not the exact derivatives of the residual in every
// term (some sign slips, swapped gravity factors and omitted factors are part
// of the reference's matrix), so each term here restates the reference's
// expression; the direction-dependent deviations are kept as explicit flags.
//
// Output layout (the compact canonical block row).  Every block row (one
// cell of one continuum) places its unknowns at fixed canonical positions
// whatever its phase state: x_0..x_{N-1}, y_0..y_{N-1}, P, Sw, So, Sg
// (bs = 2N+4 columns), and its rows at fixed positions: fugacity rows
// 0..N-1, component rows N..2N-2, the total row 2N-1, the water row 2N and
// the constraint rows 2N+1 (sum x), 2N+2 (sum y), 2N+3 (sum S).  A one-phase
// cell's N+3 reference rows and unknowns map onto these positions; its unused
// rows hold a unit entry in an unused column.  Eight block slots per block
// row: this cell, the -x, +x, -y, +y, -z, +z neighbours, and the same cell of
// the other continuum.  Only the entries that can be nonzero are stored:
//   F  fugacity rows, own slot, columns 0..2N          N (2N+1)
//   C  component and total rows, 8 slots, all columns  N 8 (2N+4)
//   W  water row, 8 slots, columns P and Sw            16
//   K  constraint rows, own slot, all columns          3 (2N+4)
//   O  eight entries the reference places in the block after a neighbour's
//      (its total rows' -y and -z face columns, counted from the following
//      block's row offset)                              8
// i.e. 1,500 values per block row at N = 8 (the reference's structural count
// for an interior two-phase cell is 18N^2+35N+19 = 1,451).  Values are stored
// in chunks of 32 block rows, vals[chunk][entry][32]: the 32 lanes of a warp
// (32 consecutive block rows) store 256 contiguous bytes per entry, and a
// chunk's values are one contiguous run (a layout with the whole grid between
// consecutive entries puts every entry of a warp on its own page).  Each
// entry is written exactly once per call (zeros included, and zeros for the
// lanes of the last chunk beyond the grid): no clearing pass, no
// read-modify-write.
//
// Work decomposition: a warp takes 32 consecutive block rows and one task --
// a composition column k of all component and total rows, their pressure
// and saturation columns, or the fugacity, water and constraint rows.  The
// face factors of a (face, phase, column) are shared by all rows, so a
// column task evaluates them once and applies them row by row.  Viscosity
// derivatives and the composition sums of the diffusion-coefficient
// derivatives are tabulated per cell-medium by a preparation kernel, so an
// entry costs O(1).
//
// The code is plain C++ over a view of device arrays, so the same source also
// compiles for the host.
#pragma once
#include <cmath>

#if defined(__CUDACC__)
#define OSR_HD __host__ __device__
#else
#define OSR_HD
#endif

namespace osrj {

constexpr double kSIC = 9.869232667160128e-13;   // SI_C
constexpr double kGAcc = 9.80665;                // G_ACC
constexpr double kGAccG = 9.80665e-3;            // G_ACCG
constexpr double kWatMRo = 55.5084;              // WAT_M_RO
constexpr double kR = 8.3144621;                 // RGAS
constexpr double kSqrt2 = 1.4142135623730950488016887;
constexpr int kMaxNc = 16;
constexpr int kOverflow = 8;

template <class T>
OSR_HD inline T ld(const T *p) {
#if defined(__CUDA_ARCH__)
    return __ldg(p);
#else
    return *p;
#endif
}

// Fields of one continuum ([planes][cells], cell fastest).
struct JMed {
    const double *P, *sat, *x, *y, *rho, *mu, *gam, *kr, *dkr, *pc, *dE, *diff, *trans, *wtran, *dwtran, *por,
        *perm, *iftran;
    const signed char *label, *transS;
};

struct JacView {
    int nx, ny, nz, nc;
    long n;
    const double *di, *dj, *dk, *blockH, *tor;
    // per-component constants
    double sa[kMaxNc], b[kMaxNc], bic[kMaxNc * kMaxNc], mw[kMaxNc], smw[kMaxNc], mui[kMaxNc], vcm[kMaxNc],
        tc[kMaxNc], pc[kMaxNc], pcr_atm[kMaxNc], vc53[kMaxNc], vc23[kMaxNc], pD[kMaxNc * kMaxNc],
        ipD[kMaxNc * kMaxNc];   // 1 / pD
    double T;
    int srk;
    // scalars
    double cpor, dcpor, refp, wat_ro, wat_mu, sigma, lf, pcoeff, dt;
    // per-pass controls in device memory ([dt, time, PCoeff]), read in place
    // of dt and pcoeff when set (a Newton step replayed as one CUDA graph)
    const double *ctl;
    int diff_off;   // CDIF present and zero: diffusive shape factors vanish
    int const_dif;  // CDIF present: diffusion-coefficient derivatives vanish
    JMed m[2];
    const long *rowoff;
    // wells (rates at the linearisation point, per cell-medium; optional)
    const double *well_pi;    // [2 cells][3] PIw, PIo, PIg or null
    const int *well_comp;     // [2 cells] index of the injection well whose stream sets the component split, -1
    const double *well_q;     // [2 cells][3] Qw, Qo, Qg or null
    const double *stream_y;   // [wells][kMaxNc] injected gas composition
    // derivative tables (written by the preparation kernel)
    double *dmu;   // [2 phases][N+1][2 cells]: d mu / d w_k (k < N), d mu / d P (k = N)
    double *dh;    // [2 phases][8+2N][2 cells]: factors of d D / d w (see prep_cell)
    // output
    double *vals;  // [chunks of 32 block rows][entries][32]
    int entries;   // values per block row
};

OSR_HD inline double jdt(const JacView &v) { return v.ctl ? v.ctl[0] : v.dt; }
OSR_HD inline double jpc(const JacView &v) { return v.ctl ? v.ctl[2] : v.pcoeff; }

// Entry indices of the compact block row (see the file comment).
struct Layout {
    int N, BS, EF, EC, EW, EK, E, ET;
    OSR_HD explicit Layout(int n)
        : N(n), BS(2 * n + 4), EF(n * (2 * n + 1)), EC(n * 8 * (2 * n + 4)), EW(16), EK(3 * (2 * n + 4)),
          E(n * (2 * n + 1) + n * 8 * (2 * n + 4) + 16 + 3 * (2 * n + 4)),
          ET(n * (2 * n + 1) + n * 8 * (2 * n + 4) + 16 + 3 * (2 * n + 4) + kOverflow) {}
    OSR_HD int f(int r, int c) const { return r * (2 * N + 1) + c; }
    OSR_HD int cr(int r, int s, int c) const { return EF + ((r - N) * 8 + s) * BS + c; }
    OSR_HD int w(int s, int c) const { return EF + EC + 2 * s + (c - 2 * N); }
    OSR_HD int k(int r, int c) const { return EF + EC + EW + (r - 2 * N - 1) * BS + c; }
    OSR_HD int o(int j) const { return E + j; }
};

// Index of value e of block row b in the chunked layout.
OSR_HD inline long value_index(long b, int e, int entries) { return ((b >> 5) * entries + e) * 32 + (b & 31); }

struct Out {
    double *vals;
    int entries;
    long b;
    OSR_HD void st(int e, double x) const {
#if defined(__CUDA_ARCH__)
        __stcs(vals + value_index(b, e, entries), x);
#else
        vals[value_index(b, e, entries)] = x;
#endif
    }
};

// Canonical column of the unit entry of canonical row r in a block row whose
// rows carry no equation of their own: the reference's diagonal for an
// inactive cell-medium, and for the rows a one-phase block does not use, a
// column it does not use either.
OSR_HD inline int unit_col(int N, int lab, int r) {
    if (lab == 0) return r;
    const bool oil = lab == 1;
    if (r < N) return oil ? N + r : r;
    if (r < 2 * N) return oil ? r - N : r;
    if (r == 2 * N) return 2 * N;
    if (r == 2 * N + 1) return oil ? 2 * N + 1 : 2 * N + 2;
    if (r == 2 * N + 2) return oil ? 2 * N + 3 : 2 * N + 1;
    return oil ? 2 * N + 2 : 2 * N + 3;
}

// Reference-local row of canonical row r for phase state lab (-1: unused).
OSR_HD inline int ref_row(int N, int lab, int r) {
    if (lab == 0) return r;
    if (r < N) return -1;
    if (r < 2 * N) return r - N;
    if (r == 2 * N) return N;
    if (r == 2 * N + 1) return lab == 1 ? N + 1 : -1;
    if (r == 2 * N + 2) return lab == -1 ? N + 1 : -1;
    return N + 2;
}

// Reference-local column of canonical column cc for phase state lab (-1:
// unused).  The reference packs a one-phase cell's unknowns as
// [w_0..w_{N-1}, P, Sw, S_h].
OSR_HD inline int ref_col(int N, int lab, int cc) {
    if (lab == 0) return cc;
    const bool oil = lab == 1;
    if (cc < N) return oil ? cc : -1;
    if (cc < 2 * N) return oil ? -1 : cc - N;
    if (cc == 2 * N) return N;
    if (cc == 2 * N + 1) return N + 1;
    if (cc == 2 * N + 2) return oil ? N + 2 : -1;
    return oil ? -1 : N + 2;
}

// ---------------------------------------------------------------------------
// Small accessors
// ---------------------------------------------------------------------------
struct Cell {
    const JacView *v;
    const JMed *F;
    long c;
    int med;
    OSR_HD long bm() const { return med ? v->n + c : c; }
    OSR_HD double P(int p) const { return ld(F->P + p * v->n + c); }
    OSR_HD double S(int p) const { return ld(F->sat + p * v->n + c); }
    OSR_HD double w(int ph, int i) const { return ld((ph ? F->y : F->x) + (long)i * v->n + c); }
    OSR_HD double rho(int ph) const { return ld(F->rho + ph * v->n + c); }
    OSR_HD double mu(int ph) const { return ld(F->mu + ph * v->n + c); }
    OSR_HD double gam(int ph) const { return ld(F->gam + ph * v->n + c); }
    OSR_HD double kr(int p) const { return ld(F->kr + p * v->n + c); }
    OSR_HD double dkr(int p) const { return ld(F->dkr + p * v->n + c); }
    OSR_HD double pc(int p) const { return ld(F->pc + p * v->n + c); }
    OSR_HD double dE(int k, int ph) const { return ld(F->dE + (long)(2 * k + ph) * v->n + c); }
    OSR_HD double D(int i, int ph) const { return ld(F->diff + (long)(2 * i + ph) * v->n + c); }
    OSR_HD double por() const { return ld(F->por + c); }
    OSR_HD int label() const { return ld(F->label + c); }
    OSR_HD double porpor() const {
        const double dp = P(1) - v->refp;
        return por() * (1 + v->cpor * dp + v->dcpor * dp * dp);
    }
    OSR_HD double dpordp() const { return por() * (v->cpor + 2 * v->dcpor * (P(1) - v->refp)); }
};

// ---------------------------------------------------------------------------
// Derivative tables
// ---------------------------------------------------------------------------

// One cell-medium's tables.  dmu: d mu / d w_k (k < N) or d mu / d P (k == N)
// of each phase (DiffVisco / fDiffVisco, compsim/Mass_Tran.cpp:307-399).
// dh: the factors of the diffusion-coefficient derivative (DifDiffusion /
// fDifDiffusion, compsim/Mass_Tran.cpp:107-305) that do not depend on the
// column: s1 = sum w_j Vc_j^(5/3), s2 = sum w_j Vc_j^(2/3), s1/s2, 1/s2^2,
// cA = dAA/dEr at Er = rho s1/s2, AA(Er), 1/rho^2, rho/AA, and per component
// i, a2_i = Sm_i rho/AA with Sm_i = sum_{j != i} w_j / pD_ji, and 1/a2_i^2.
template <int N>
OSR_HD inline void prep_cell(const JacView &v, long bm) {
    const int med = bm >= v.n;
    const long c = med ? bm - v.n : bm;
    const Cell q{&v, &v.m[med], c, med};
    const long nb2 = 2 * v.n;
    for (int ph = 0; ph < 2; ph++) {
        double w[N];
#pragma unroll
        for (int n = 0; n < N; n++) w[n] = q.w(ph, n);
        double s1 = 0, s2 = 0, ro = 0, tcm = 0, pcm = 0, mwm = 0;
#pragma unroll
        for (int n = 0; n < N; n++) {
            const double t = w[n] * v.smw[n];
            s1 += t * v.mui[n];
            s2 += t;
            ro += w[n] * v.vcm[n];
            tcm += w[n] * v.tc[n];
            pcm += w[n] * v.pcr_atm[n];
            mwm += w[n] * v.mw[n];
        }
        const double rho = q.rho(ph);
        const double Er = rho * ro;
        const double eA = pow(tcm, 1.0 / 6), eB = sqrt(mwm), eC = pow(pcm, 2.0 / 3);
        const double eta = eA / (eB * eC);
        const double r1 = 0.10230 + 0.023364 * Er + 0.058533 * Er * Er - 0.040758 * Er * Er * Er + 0.0093324 * Er * Er * Er * Er;
        const double t56 = pow(tcm, -5.0 / 6.0), p13 = pow(pcm, -1.0 / 3.0);
        const double r4 = r1 * r1 * r1 * r1 - 1e-4;
#pragma unroll
        for (int k = 0; k <= N; k++) {
            double dMuS, dEta, dEr;
            if (k < N) {
                dMuS = (v.mui[k] * v.smw[k] * s2 - v.smw[k] * s1) / (s2 * s2);
                dEta = ((1.0 / 6.0) * t56 * v.tc[k] * eB * eC -
                        eA * (0.5 * v.mw[k] * eC / eB + (2.0 / 3.0) * p13 * v.pc[k] * eB / 101325)) /
                       (eB * eB * eC * eC);
                dEr = q.dE(k, ph) * ro + rho * v.vcm[k];
            } else {
                dMuS = 0;
                dEta = 0;
                dEr = q.dE(N, ph) * ro;
            }
            const double dMM = 4 * r1 * r1 * r1 * (0.023364 * dEr + 0.117066 * dEr * Er - 0.122274 * dEr * Er * Er + 0.0373296 * dEr * Er * Er * Er);
            v.dmu[(long)(ph * (N + 1) + k) * nb2 + bm] = (dMM * eta - r4 * dEta) / (eta * eta) + dMuS;
        }
        if (v.const_dif) continue;
        double d1 = 0, d2 = 0;
#pragma unroll
        for (int j = 0; j < N; j++) {
            d1 += w[j] * v.vc53[j];
            d2 += w[j] * v.vc23[j];
        }
        const double Ed = rho * d1 / d2;
        const double AA = 0.99589 + 0.096016 * Ed - 0.22035 * Ed * Ed + 0.032874 * Ed * Ed * Ed;
        const double iroRD = 1 / (AA / rho);
        double *h = v.dh + (long)ph * (8 + 2 * N) * nb2 + bm;
        h[0] = d1;
        h[nb2] = d2;
        h[2 * nb2] = d1 / d2;
        h[3 * nb2] = 1 / (d2 * d2);
        h[4 * nb2] = 0.096016 - 0.4407 * Ed + 0.098622 * Ed * Ed;
        h[5 * nb2] = AA;
        h[6 * nb2] = 1 / (rho * rho);
        h[7 * nb2] = iroRD;
        for (int i = 0; i < N; i++) {
            double sm = 0;
#pragma unroll
            for (int j = 0; j < N; j++)
                if (j != i) sm += w[j] / v.pD[j * N + i];
            const double a2 = sm * iroRD;
            h[(8 + 2 * i) * nb2] = a2;
            h[(9 + 2 * i) * nb2] = 1 / (a2 * a2);
        }
    }
}

OSR_HD inline double dmu(const Cell &q, int k, int ph) {
    const int N = q.v->nc;
    return ld(q.v->dmu + (long)(ph * (N + 1) + k) * (2 * q.v->n) + q.bm());
}

// d D_i / d w_k (k < N) or d D_i / d P (k == N) of one phase.  With
// G = (dAA rho - dRho AA) / rho^2 the reference's sums over j != i factor as
//   a2 = Sm_i / (AA/rho),  a1 = [k != i] / (pD_ki AA/rho) - G Sm_i / (AA/rho)^2,
//   dD = -(a2 [k == i] + a1 (1 - w_i)) / a2^2.
// Unlike the coefficient itself (CalcDiffusion) it carries no 1e-4 factor.
// DCol is the part of one (cell-medium, phase, k): G and rho/AA; a row adds
// a2_i, 1/a2_i^2 and w_i (dd_col).
struct DCol {
    double G, iroRD;
    bool zero;
};

OSR_HD inline DCol make_dcol(const Cell &q, int k, int ph, double dEk) {
    const JacView &v = *q.v;
    DCol d;
    if (v.const_dif) {
        d.zero = true;
        return d;
    }
    const int N = v.nc;
    const long nb2 = 2 * v.n;
    const double *h = v.dh + (long)ph * (8 + 2 * N) * nb2 + q.bm();
    const double s1 = ld(h), s2 = ld(h + nb2), r12 = ld(h + 2 * nb2), is22 = ld(h + 3 * nb2), cA = ld(h + 4 * nb2);
    const double AA = ld(h + 5 * nb2), irho2 = ld(h + 6 * nb2);
    const double rho = q.rho(ph);
    double dEr = dEk * r12;
    if (k < N) dEr += rho * (v.vc53[k] * s2 - v.vc23[k] * s1) * is22;
    d.G = (dEr * cA * rho - dEk * AA) * irho2;
    d.iroRD = ld(h + 7 * nb2);
    d.zero = AA < 0;
    return d;
}

OSR_HD inline double dd_col(const JacView &v, const DCol &d, const Cell &q, int i, int k, int ph) {
    if (d.zero) return 0;
    const int N = v.nc;
    const long nb2 = 2 * v.n;
    const double *h = v.dh + (long)ph * (8 + 2 * N) * nb2 + q.bm();
    const double a2 = ld(h + (8 + 2 * i) * nb2);
    if (a2 == 0) return 0;
    const double ia2sq = ld(h + (9 + 2 * i) * nb2), omw = 1 - q.w(ph, i);
    double a1 = -d.G * a2 * d.iroRD;
    if (k < N && k != i) a1 += v.ipD[k * N + i] * d.iroRD;
    if (k == i) return -(a2 + a1 * omw) * ia2sq;
    return -a1 * omw * ia2sq;
}

// ---------------------------------------------------------------------------
// Faces
// ---------------------------------------------------------------------------

// One face of a cell: neighbour, the cell holding the face's
// transmissibilities (tc), direction and sign, block slot, the two block
// sizes along the direction and twice the cross-section.
struct JFace {
    long nb, tc;
    int d, sgn, slot;
    double dl, dn, area2;
};

OSR_HD inline int jac_faces(const JacView &v, long c, JFace *f) {
    const int ix = (int)(c % v.nx), iy = (int)((c / v.nx) % v.ny), iz = (int)(c / ((long)v.nx * v.ny));
    const long sx = 1, sy = v.nx, sz = (long)v.nx * v.ny;
    const double di = ld(v.di + ix), dj = ld(v.dj + iy), dk = ld(v.dk + iz);
    int k = 0;
    if (ix < v.nx - 1) f[k++] = JFace{c + sx, c, 0, 1, 2, di, ld(v.di + ix + 1), 2 * dj * dk};
    if (ix > 0) f[k++] = JFace{c - sx, c - sx, 0, -1, 1, di, ld(v.di + ix - 1), 2 * dj * dk};
    if (iy < v.ny - 1) f[k++] = JFace{c + sy, c, 1, 1, 4, dj, ld(v.dj + iy + 1), 2 * di * dk};
    if (iy > 0) f[k++] = JFace{c - sy, c - sy, 1, -1, 3, dj, ld(v.dj + iy - 1), 2 * di * dk};
    if (iz < v.nz - 1) f[k++] = JFace{c + sz, c, 2, 1, 6, dk, ld(v.dk + iz + 1), 2 * di * dj};
    if (iz > 0) f[k++] = JFace{c - sz, c - sz, 2, -1, 5, dk, ld(v.dk + iz - 1), 2 * di * dj};
    return k;
}

struct FaceData {
    // transmissibility factors of the face (stored at tc), upstream flags
    double T[12], ift;
    int ts[3];
    double dP[3];   // phase pressure differences in the residual's orientation (nb - c for + faces, c - nb for -)
    double dH;      // likewise for block heights
};

OSR_HD inline FaceData face_data(const JacView &v, const JMed &F, long c, const JFace &e) {
    FaceData fd;
    const long n = v.n;
    for (int t = 0; t < 12; t++) fd.T[t] = ld(F.trans + (long)(t * 3 + e.d) * n + e.tc);
    for (int p = 0; p < 3; p++) fd.ts[p] = ld(F.transS + (long)(p * 3 + e.d) * n + e.tc);
    fd.ift = ld(F.iftran + (long)e.d * n + e.tc);
    for (int p = 0; p < 3; p++) {
        const double a = ld(F.P + p * n + e.nb), b = ld(F.P + p * n + c);
        fd.dP[p] = e.sgn > 0 ? a - b : b - a;
    }
    const double hn = ld(v.blockH + e.nb), hc = ld(v.blockH + c);
    fd.dH = e.sgn > 0 ? hn - hc : hc - hn;
    return fd;
}

// upstream cell of phase p (0 oil, 1 gas, 2 water) across the face
OSR_HD inline long upstream(const JFace &e, const FaceData &fd, long c, int p) {
    if (e.sgn > 0) return fd.ts[p] ? e.nb : c;
    return fd.ts[p] ? c : e.nb;
}

// Which of a cell's own unknowns the reference's rows address by phase state
// (its reCol / reCol3 offsets): a one-phase cell has no column for the
// absent phase's composition and saturation, and an oil-only or gas-only cell
// emits its own saturation derivatives only for the phases it carries.
struct OwnLayout {
    bool swso, sg, x, y;
};

OSR_HD inline OwnLayout own_layout(int lab) {
    if (lab == 0) return OwnLayout{true, true, true, true};
    if (lab == 1) return OwnLayout{true, false, true, false};
    return OwnLayout{false, true, false, true};
}

// One phase of one cell as the mobility factors see it.
struct Side {
    double rho, mu, gam;
};

// Mobility-ratio derivative factors of one phase across a face: the
// derivatives of (rho_c dl + rho_n dn C) / (mu_c dl + mu_n dn C) and of the
// face-averaged gravity with respect to a variable of this cell (M, MG) and
// of the neighbour (B, BG).  comp: a composition variable with molar mass
// mwk (else pressure).
struct Mob {
    double Sur, Mak, M, B, MG, BG, tempdx;
};

OSR_HD inline Mob mobility(const Side &q, const Side &nb, double dEq, double dEn, bool comp, double mwk, const JFace &e,
                           double coef, double dmu_c, double dmu_n) {
    Mob m;
    m.Sur = q.rho * e.dl + nb.rho * e.dn * coef;
    m.Mak = q.mu * e.dl + nb.mu * e.dn * coef;
    m.M = (dEq * e.dl * m.Mak - dmu_c * e.dl * m.Sur) / (m.Mak * m.Mak);
    m.B = (dEn * e.dn * coef * m.Mak - dmu_n * e.dn * coef * m.Sur) / (m.Mak * m.Mak);
    const double gk_c = comp ? kGAccG * q.rho * mwk : 0.0;
    const double gk_n = comp ? kGAccG * nb.rho * mwk : 0.0;
    m.MG = e.dl * (gk_c + q.gam * dEq / q.rho) / (e.dl + e.dn * coef);
    m.BG = coef * e.dn * (gk_n + nb.gam * dEn / nb.rho) / (e.dl + e.dn * coef);
    m.tempdx = (q.gam * e.dl + nb.gam * e.dn * coef) / (e.dl + e.dn * coef);
    return m;
}

// ---------------------------------------------------------------------------
// Matrix-fracture transfer quantities of a cell (the "sadeq" region of the
// reference's rows): porosities, averaged viscosities, the relative
// permeability of the upstream continuum and its saturation derivatives.
// ---------------------------------------------------------------------------
struct Transfer {
    double pm, pf, dpm, dpf;         // porosities at the linearisation point and d/dP
    double Do, Dg;                   // mu_m pm + mu_f pf per phase
    double kro, krg, krw;            // upstream relative permeabilities
    double dkm[5], dkf[5];           // d kr / dS terms of the matrix / fracture side (zero when not upstream)
    double dPo, dPg, dPw;            // fracture - matrix potential differences
    double SF1, SF2, SF3, Vb;
};

OSR_HD inline Transfer transfer_terms(const JacView &v, long c) {
    Transfer t;
    const Cell M{&v, &v.m[0], c, 0}, F{&v, &v.m[1], c, 1};
    t.pm = M.porpor();
    t.pf = F.porpor();
    t.dpm = M.dpordp();
    t.dpf = F.dpordp();
    t.Do = M.mu(0) * t.pm + F.mu(0) * t.pf;
    t.Dg = M.mu(1) * t.pm + F.mu(1) * t.pf;
    const bool mo = M.P(1) >= F.P(1), mg = M.P(2) >= F.P(2), mw = M.P(0) >= F.P(0);
    t.kro = mo ? M.kr(1) : F.kr(1);
    t.krg = mg ? M.kr(2) : F.kr(2);
    t.krw = mw ? M.kr(0) : F.kr(0);
    for (int j = 0; j < 5; j++) t.dkm[j] = t.dkf[j] = 0;
    // oil: d/dSw, d/dSg, d/dSo; gas: d/dSg; water: d/dSw
    if (mo) { t.dkm[1] = M.dkr(1); t.dkm[2] = M.dkr(2); t.dkm[4] = M.dkr(4); }
    else { t.dkf[1] = F.dkr(1); t.dkf[2] = F.dkr(2); t.dkf[4] = F.dkr(4); }
    if (mg) t.dkm[3] = M.dkr(3);
    else t.dkf[3] = F.dkr(3);
    if (mw) t.dkm[0] = M.dkr(0);
    else t.dkf[0] = F.dkr(0);
    t.dPo = F.P(1) - M.P(1);
    t.dPg = (F.P(2) - M.P(2)) + (F.pc(1) - M.pc(1));
    t.dPw = (F.P(0) - M.P(0)) + (M.pc(0) - F.pc(0));
    const int ix = (int)(c % v.nx), iy = (int)((c / v.nx) % v.ny), iz = (int)(c / ((long)v.nx * v.ny));
    const double di = ld(v.di + ix), dj = ld(v.dj + iy), dk = ld(v.dk + iz);
    t.Vb = di * dj * dk;
    t.SF2 = 4 * v.sigma * (ld(M.F->perm + c) / (di * di) + ld(M.F->perm + v.n + c) / (dj * dj) + ld(M.F->perm + 2 * v.n + c) / (dk * dk));
    t.SF1 = v.diff_off ? 0.0 : 4 * v.sigma * ((1 / (di * di)) + (1 / (dj * dj)) + (1 / (dk * dk)));
    t.SF3 = v.diff_off ? 0.0 : 4 * v.sigma * ((1 / di) + (1 / dj) + (1 / dk)) / v.lf;
    return t;
}

// Diffusive-transfer targets of a matrix row for phase ph: for each pairing of
// the two continua's phase states the reference adds zero, one or two terms
// toward the fracture composition (t = 1) or the interface composition
// (t = 0, which is identically zero).  Returns the number of terms; kinds[j]
// is 1 for the fracture composition, 0 for the interface.
OSR_HD inline int matrix_diff_targets(int lm, int lf, int ph, int *kinds) {
    int n = 0;
    if (ph == 0) {
        if (lm == 1 && lf == 1) kinds[n++] = 1;
        if (lm == 0 && lf == 0) kinds[n++] = 1;
        if (lm == 1 && lf == -1) kinds[n++] = 0;
        if (lm == 0 && lf == 1) kinds[n++] = 1;
        if (lm == 0 && lf == -1) kinds[n++] = 0;
        if (lm == 1 && lf == 0) { kinds[n++] = 0; kinds[n++] = 1; }
    } else {
        if (lm == -1 && lf == -1) kinds[n++] = 1;
        if (lm == 0 && lf == 0) kinds[n++] = 1;
        if (lm == -1 && lf == 1) kinds[n++] = 0;
        if (lm == 0 && lf == 1) kinds[n++] = 0;
        if (lm == 0 && lf == -1) kinds[n++] = 1;
        if (lm == -1 && lf == 0) { kinds[n++] = 1; kinds[n++] = 0; }
    }
    return n;
}

// Fracture-side diffusive transfer pairings.  fsf1: the matrix-side (SF1)
// terms toward the fracture composition a fracture row carries for phase ph;
// fsf3: the interface (SF3) terms of the fracture's own phase ph.
OSR_HD inline bool fsf1(int lm, int lf, int ph) {
    if (lm == 0 && lf == 0) return true;
    if (ph == 0) return (lm == 1 && lf == 1) || (lm == 0 && lf == 1) || (lm == 1 && lf == 0);
    return (lm == -1 && lf == -1) || (lm == 0 && lf == -1) || (lm == -1 && lf == 0);
}
OSR_HD inline bool fsf3(int lm, int lf, int ph) {
    if (ph == 0) return (lm == -1 && lf == 1) || (lm == 0 && lf == 1) || (lm == -1 && lf == 0);
    return (lm == 1 && lf == -1) || (lm == 0 && lf == -1) || (lm == 1 && lf == 0);
}

// Direction-dependent deviations of the reference's face blocks.
struct FaceQuirks {
    bool gas_dB_assign_up;     // - faces, gas upstream = this cell: dB = ... instead of dB -= ...
    bool gas_dB_assign_down;   // - faces, gas upstream = neighbour
    bool ift_y_in_diag_grav;   // +z face, k == i, oil upstream = neighbour: y-face transmissibility
    bool gas_coef_any_1ph;     // k != i, gas: neighbour weight zero for any one-phase neighbour
    bool oil_grav_assign_down; // - faces, oil upstream = neighbour: gravity term assigned to dB
    bool shifted_block;        // neighbour P / S columns counted from the block after the neighbour's
};

// the total rows' pressure / saturation face blocks
OSR_HD inline FaceQuirks total_quirks(const JFace &e) {
    FaceQuirks q{false, false, false, false, false, false};
    if (e.sgn < 0 && e.d == 1) { q.gas_dB_assign_down = true; q.oil_grav_assign_down = true; q.shifted_block = true; }
    if (e.sgn < 0 && e.d == 2) q.shifted_block = true;
    return q;
}

// the component rows' face blocks (both continua)
OSR_HD inline FaceQuirks comp_quirks(const JFace &e) {
    FaceQuirks q{false, false, false, false, false, false};
    if (e.sgn < 0 && e.d == 0) { q.gas_dB_assign_up = true; q.gas_dB_assign_down = true; q.gas_coef_any_1ph = true; }
    if (e.sgn > 0 && e.d == 2) q.ift_y_in_diag_grav = true;
    return q;
}

// k-independent factors of one phase across one face for the composition
// derivatives (the mobility-ratio and gravity denominators, the upstream
// weights and the diffusion factors) at neighbour weight coef.
struct PhFace {
    double coef, Sur, Mak, iMak2, iden, tempdx, SurMak, gq, gn;
    double BBd, iBB, MMd;
};

OSR_HD inline PhFace ph_face(const Side &sq, const Side &sn, const JFace &e, double coef, double dC, double Sq,
                             double Sn, double tor_c, double tor_n, double pm, double pn) {
    PhFace P;
    P.coef = coef;
    P.Sur = sq.rho * e.dl + sn.rho * e.dn * coef;
    P.Mak = sq.mu * e.dl + sn.mu * e.dn * coef;
    P.iMak2 = 1 / (P.Mak * P.Mak);
    P.iden = 1 / (e.dl + e.dn * coef);
    P.tempdx = (sq.gam * e.dl + sn.gam * e.dn * coef) * P.iden;
    P.SurMak = P.Sur / P.Mak;
    P.gq = sq.gam / sq.rho;
    P.gn = sn.gam / sn.rho;
    double AAd = sn.rho * e.dn * coef + sq.rho * e.dl * dC;
    AAd *= (Sn * e.dn * coef + Sq * e.dl * dC) / (e.dn + e.dl);
    P.BBd = tor_n * e.dn * coef / pn + tor_c * e.dl * dC / pm;
    P.iBB = 1 / P.BBd;
    P.MMd = AAd * P.iBB;
    return P;
}

// Well rates of a completion cell at the linearisation point (written by the
// residual path's well pass) and the gas-phase composition its component
// balance uses: the injected stream of an injection well, else the cell's own.
struct WellAt {
    double Qw, Qo, Qg, PIw, PIo, PIg, gcomp;
    int iwell;
};

OSR_HD inline WellAt well_at(const JacView &v, int med, long c, int i, double own_y) {
    WellAt w{0, 0, 0, 0, 0, 0, own_y, -1};
    if (!v.well_q) return w;
    const long b = med ? v.n + c : c;
    w.Qw = ld(v.well_q + 3 * b);
    w.Qo = ld(v.well_q + 3 * b + 1);
    w.Qg = ld(v.well_q + 3 * b + 2);
    w.PIw = ld(v.well_pi + 3 * b);
    w.PIo = ld(v.well_pi + 3 * b + 1);
    w.PIg = ld(v.well_pi + 3 * b + 2);
    w.iwell = ld(v.well_comp + b);
    if (w.iwell >= 0) w.gcomp = ld(v.stream_y + w.iwell * kMaxNc + i);
    return w;
}

// This cell's P and saturation entries of a component or total row; unused
// columns of a one-phase cell are stored as zeros.
OSR_HD inline void store_own_ps(int N, const Out &out, int row, int lab, double P, double Sw, double So, double Sg) {
    const Layout L(N);
    const OwnLayout O = own_layout(lab);
    out.st(L.cr(row, 0, 2 * N), P);
    out.st(L.cr(row, 0, 2 * N + 1), O.swso ? Sw : 0.0);
    out.st(L.cr(row, 0, 2 * N + 2), O.swso ? So : 0.0);
    out.st(L.cr(row, 0, 2 * N + 3), O.sg ? Sg : 0.0);
}

// The other continuum's block of a component or total row (slot 7): P, Sw,
// the saturation(s) and compositions its phase state carries.
OSR_HD inline void store_other_ps(int N, const Out &out, int row, int lo, double P, double Sw, double So, double Sg) {
    const Layout L(N);
    out.st(L.cr(row, 7, 2 * N), P);
    out.st(L.cr(row, 7, 2 * N + 1), Sw);
    out.st(L.cr(row, 7, 2 * N + 2), lo == -1 ? 0.0 : So);
    out.st(L.cr(row, 7, 2 * N + 3), lo == 1 ? 0.0 : Sg);
}

OSR_HD inline void store_other_x(int N, const Out &out, int row, int lo, int k, double xl, double xg) {
    const Layout L(N);
    out.st(L.cr(row, 7, k), lo == -1 ? 0.0 : xl);
    out.st(L.cr(row, 7, N + k), lo == 1 ? 0.0 : xg);
}

// ---------------------------------------------------------------------------
// Column decomposition of the component and total rows.
//
// Canonical rows N..2N-1 of a block row are the component balances i = 0..N-2
// and the total row (i = N-1).  Their face terms share one factor set per
// (face, phase, column): the mobility-ratio and gravity derivatives depend on
// the two cells and the column, not on the row.  A column task computes the
// x_k and y_k columns of all N rows in every block (own, six faces, the other
// continuum), evaluating those factors once per (face, phase) and applying
// them row by row; the pressure-saturation task does the same for the P, Sw,
// So, Sg columns and the eight shifted entries.  Per-row sums are kept in
// shared memory (SmemVec), in the order the reference adds their terms.
// ---------------------------------------------------------------------------

// A per-thread vector in shared memory: element j at p[j * stride].
struct SmemVec {
    double *p;
    int stride;
    OSR_HD double &operator[](int j) const { return p[j * stride]; }
};

// This cell's factors of one phase across a face for column k at neighbour
// weight coef: d(mobility ratio)/d w_k of this cell (M) and the neighbour (B)
// and the gravity-weighted forms gM, gB.
struct ColFac {
    PhFace P;
    double M, B, gM, gB;
};

OSR_HD inline ColFac col_fac(const Side &sq, const Side &sn, const JFace &e, double coef, double dC, double Sq,
                             double Sn, double tor_c, double tor_n, double pm, double pn, double dEq, double dEn,
                             double dmq, double dmn, double mwk) {
    ColFac f;
    f.P = ph_face(sq, sn, e, coef, dC, Sq, Sn, tor_c, tor_n, pm, pn);
    const PhFace &P = f.P;
    f.M = (dEq * e.dl * P.Mak - dmq * e.dl * P.Sur) * P.iMak2;
    f.B = (dEn * e.dn * coef * P.Mak - dmn * e.dn * coef * P.Sur) * P.iMak2;
    const double MG = e.dl * (kGAccG * sq.rho * mwk + P.gq * dEq) * P.iden;
    const double BG = coef * e.dn * (kGAccG * sn.rho * mwk + P.gn * dEn) * P.iden;
    f.gM = f.M * P.tempdx + MG * P.SurMak;
    f.gB = f.B * P.tempdx + BG * P.SurMak;
    return f;
}

// Column k (x_k and y_k) of all component and total rows of block row
// (med, c): the transfer terms, the other continuum's block, every face, and
// this cell's block.  accX, accY, accZ: N doubles each.
OSR_HD inline void column_task(const JacView &v, int med, long c, int k, const Out &out, SmemVec accX, SmemVec accY,
                               SmemVec accZ) {
    const int N = v.nc;
    const Layout L(N);
    const Cell M{&v, &v.m[0], c, 0}, Fr{&v, &v.m[1], c, 1};
    const Cell &q = med ? Fr : M;
    const int lm = M.label(), lf = Fr.label(), lq = q.label(), lo = med ? lm : lf;
    const Transfer t = transfer_terms(v, c);
    const double Vb = t.Vb, SF1 = t.SF1, SF2 = t.SF2, SF3 = t.SF3, pm = t.pm, pf = t.pf;
    const double tor = ld(v.tor + c);
    const double mubar_o = t.Do / (pm + pf), mubar_g = t.Dg / (pm + pf);
    const double ro = M.rho(0), rg = M.rho(1);
    const double dEkM[2] = {M.dE(k, 0), M.dE(k, 1)}, dEkF[2] = {Fr.dE(k, 0), Fr.dE(k, 1)};
    const double dmM[2] = {dmu(M, k, 0), dmu(M, k, 1)}, dmF[2] = {dmu(Fr, k, 0), dmu(Fr, k, 1)};
    const bool idiff = !v.diff_off;
    DCol dcM[2], dcF[2];
    for (int ph = 0; ph < 2; ph++) {
        dcM[ph] = make_dcol(M, k, ph, dEkM[ph]);
        dcF[ph] = make_dcol(Fr, k, ph, dEkF[ph]);
    }
    // 1) transfer terms of every row and the other continuum's block
    for (int i = 0; i < N; i++) {
        const int row = N + i;
        const bool total = i == N - 1, diag = !total && i == k;
        double rx[2], ox[2];
        if (total) {
            const double sg = med ? -1.0 : 1.0;
            const double t1o = kSIC * SF2 * Vb * t.kro / mubar_o * t.dPo;
            const double t2o = -kSIC * ro * SF2 * Vb * t.kro * pm / (t.Do * t.Do) * t.dPo * (pm + pf);
            const double t3o = -kSIC * ro * SF2 * Vb * t.kro * pf / (t.Do * t.Do) * t.dPo * (pm + pf);
            const double t1g = kSIC * SF2 * Vb * t.krg / mubar_g * t.dPg;
            const double t2g = -kSIC * rg * SF2 * Vb * t.krg * pm / (t.Dg * t.Dg) * t.dPg * (pm + pf);
            const double t3g = -kSIC * rg * SF2 * Vb * t.krg * pf / (t.Dg * t.Dg) * t.dPg * (pm + pf);
            const double xm = dEkM[0] * t1o + dmM[0] * t2o, xf = dmF[0] * t3o;
            const double ym = dEkM[1] * t1g + dmM[1] * t2g, yf = dmF[1] * t3g;
            rx[0] = sg * (med ? xf : xm);
            rx[1] = sg * (med ? yf : ym);
            ox[0] = sg * (med ? xm : xf);
            ox[1] = sg * (med ? ym : yf);
        } else if (med == 0) {
            // matrix component row i
            const double xi = M.w(0, i), yi = M.w(1, i);
            for (int ph = 0; ph < 2; ph++) {
                const double w = ph ? yi : xi, rho = ph ? rg : ro, kr = ph ? t.krg : t.kro, mub = ph ? mubar_g : mubar_o;
                const double Dd = ph ? t.Dg : t.Do, dPp = ph ? t.dPg : t.dPo;
                const double cdg = kSIC * rho * SF2 * Vb * kr / mub * dPp;
                const double cx1 = kSIC * w * SF2 * Vb * kr / mub * dPp;
                const double cx2 = -kSIC * w * rho * SF2 * Vb * kr * pm / (Dd * Dd) * dPp * (pm + pf);
                const double cf2 = -kSIC * w * rho * SF2 * Vb * kr * pf / (Dd * Dd) * dPp * (pm + pf);
                double dR = (diag ? cdg : 0.0) + dEkM[ph] * cx1 + dmM[ph] * cx2;
                double dRf = dmF[ph] * cf2;
                if (idiff) {
                    int kinds[2];
                    const int nt = matrix_diff_targets(lm, lf, ph, kinds);
                    const double sat = M.S(1 + ph), D = M.D(i, ph);
                    if (nt) {
                        double cd1 = 0, cdd = 0, cd2 = 0;
                        for (int j = 0; j < nt; j++) {
                            const double tgt = kinds[j] ? Fr.w(ph, i) : 0.0;
                            cd1 += SF1 * sat * pm * Vb / tor * D * (tgt - w);
                            cdd += -SF1 * sat * pm * Vb / tor * rho * D;
                            cd2 += SF1 * sat * pm * Vb / tor * rho * (tgt - w);
                        }
                        dR += dEkM[ph] * cd1 + (diag ? cdd : 0.0) + dd_col(v, dcM[ph], M, i, k, ph) * cd2;
                    }
                    if (diag) {
                        // towards the fracture composition of the same phase
                        bool on = (lm == 0 && lf == 0);
                        if (ph == 0) on = on || (lm == 1 && lf == 1) || (lm == 0 && lf == 1) || (lm == 1 && lf == 0);
                        else on = on || (lm == -1 && lf == -1) || (lm == 0 && lf == -1) || (lm == -1 && lf == 0);
                        if (on) dRf += SF1 * sat * pm * Vb / tor * rho * D;
                    }
                }
                rx[ph] = dR;
                ox[ph] = dRf;
            }
        } else {
            // fracture component row i
            const double xi = M.w(0, i), yi = M.w(1, i);
            for (int ph = 0; ph < 2; ph++) {
                const double w = ph ? yi : xi, rho = ph ? rg : ro, kr = ph ? t.krg : t.kro, mub = ph ? mubar_g : mubar_o;
                const double Dd = ph ? t.Dg : t.Do, dPp = ph ? t.dPg : t.dPo;
                const double cdg = kSIC * rho * SF2 * Vb * kr / mub * dPp;
                const double cx1 = kSIC * w * SF2 * Vb * kr / mub * dPp;
                const double cx2 = -kSIC * w * rho * SF2 * Vb * kr * pm / (Dd * Dd) * dPp * (pf + pm);
                const double cf2 = -kSIC * w * rho * SF2 * Vb * kr * pf / (Dd * Dd) * dPp * (pf + pm);
                double dRM = -((diag ? cdg : 0.0) + dEkM[ph] * cx1 + dmM[ph] * cx2);
                double dR = -(dmF[ph] * cf2);
                if (idiff && fsf1(lm, lf, ph)) {
                    const double msat = M.S(1 + ph), mD = M.D(i, ph), dlt = Fr.w(ph, i) - w;
                    const double m1 = SF1 * msat * pm * Vb / tor * mD * dlt;
                    const double mdd = -SF1 * msat * pm * Vb / tor * rho * mD;
                    const double m2 = SF1 * msat * pm * Vb / tor * rho * dlt;
                    dRM -= dEkM[ph] * m1 + (diag ? mdd : 0.0) + dd_col(v, dcM[ph], M, i, k, ph) * m2;
                    if (diag) dR -= SF1 * msat * pm * Vb / tor * rho * mD;
                }
                if (idiff && fsf3(lm, lf, ph)) {
                    const double fsat = Fr.S(1 + ph), frho = Fr.rho(ph), fD = Fr.D(i, ph), fw = Fr.w(ph, i);
                    const double f3 = SF3 * fsat * pf * Vb / tor * fD * (fw - 0.0);
                    const double f3d = SF3 * fsat * pf * Vb / tor * frho * fD;
                    const double f32 = SF3 * fsat * pf * Vb / tor * frho * (fw - 0.0);
                    dR -= dEkF[ph] * f3 + (diag ? f3d : 0.0) + dd_col(v, dcF[ph], Fr, i, k, ph) * f32;
                }
                rx[ph] = dR;
                ox[ph] = dRM;
            }
        }
        accX[i] = rx[0];
        accY[i] = rx[1];
        store_other_x(N, out, row, lo, k, ox[0], ox[1]);
    }
    // 2) faces: one factor set per (face, phase), applied to every row
    JFace fc[6];
    const int nf = jac_faces(v, c, fc);
    unsigned present = 0;
    const double ift_y = ld(q.F->iftran + v.n + c);
    const double mwk = v.mw[k];
    for (int f = 0; f < nf; f++) {
        const JFace &e = fc[f];
        present |= 1u << e.slot;
        const Cell nb{&v, q.F, e.nb, med};
        const FaceData fd = face_data(v, *q.F, c, e);
        const int lnb = nb.label();
        const FaceQuirks qk = comp_quirks(e);   // component rows; the total row has none
        const double s = e.sgn;
        const double tor_c = med ? 1.0 : tor, tor_n = med ? 1.0 : ld(v.tor + e.nb);
        const double pq = q.porpor(), pn = nb.porpor();
        const double NNd = e.area2 / (e.dn + e.dl);
        for (int ph = 0; ph < 2; ph++) {
            const bool up_nb = upstream(e, fd, c, ph) == e.nb;
            const Side sq{q.rho(ph), q.mu(ph), q.gam(ph)}, sn{nb.rho(ph), nb.mu(ph), nb.gam(ph)};
            const double krq = q.kr(1 + ph), krn = nb.kr(1 + ph), Sq = q.S(1 + ph), Sn = nb.S(1 + ph);
            const double dC = ph == 0 ? (lq == -1 ? 0.0 : 1.0) : (lq == 1 ? 0.0 : 1.0);
            // neighbour weight: standard (total row, diagonal row), and off the diagonal of the
            // component rows, where the -x gas term drops any one-phase neighbour
            const double coef_d = ph == 0 ? (lnb == -1 ? 0.0 : 1.0) : (lnb == 1 ? 0.0 : 1.0);
            const double coef_nd = (ph == 1 && qk.gas_coef_any_1ph) ? (lnb != 0 ? 0.0 : 1.0) : coef_d;
            const double dEq = q.dE(k, ph), dEn = nb.dE(k, ph), dmq = dmu(q, k, ph), dmn = dmu(nb, k, ph);
            const ColFac fs = col_fac(sq, sn, e, coef_d, dC, Sq, Sn, tor_c, tor_n, pq, pn, dEq, dEn, dmq, dmn, mwk);
            DCol dcn;
            dcn.zero = true;
            if (idiff) dcn = make_dcol(nb, k, ph, dEn);
            const DCol &dcq = med ? dcF[ph] : dcM[ph];
            const double dPp = fd.dP[1 + ph];
            const bool to_x = ph == 0 ? lnb != -1 : lnb == 1;
            for (int i = 0; i < N; i++) {
                const int row = N + i;
                const bool total = i == N - 1, diag = !total && i == k;
                ColFac F = fs;
                if (!total && !diag && coef_nd != coef_d)
                    F = col_fac(sq, sn, e, coef_nd, dC, Sq, Sn, tor_c, tor_n, pq, pn, dEq, dEn, dmq, dmn, mwk);
                const double coef = F.P.coef;
                const double wc = total ? 1.0 : q.w(ph, i), wn = total ? 1.0 : nb.w(ph, i);
                const double ac = wc * fd.ift * krq, an = wn * fd.ift * krn;
                const double Tp = diag ? fd.T[ph] : 0.0, Tg = diag ? fd.T[2 + ph] : 0.0;
                double dR = 0, dB;
                if (up_nb) {
                    dR += s * (an * F.M * dPp);
                    dB = s * ((Tp + an * F.B) * dPp);
                } else {
                    dR += s * ((Tp + ac * F.M) * dPp);
                    dB = s * (ac * F.B * dPp);
                }
                // gravity (nonzero across z faces only)
                if (e.sgn > 0) {
                    if (up_nb) {
                        const double ift_r = (diag && ph == 0 && qk.ift_y_in_diag_grav) ? ift_y : fd.ift;
                        dR += wn * ift_r * krn * F.gM * fd.dH;
                        dB += (Tg + an * F.gB) * fd.dH;
                    } else {
                        dR += (Tg + ac * F.gM) * fd.dH;
                        dB += ac * F.gB * fd.dH;
                    }
                } else {
                    // - faces: the gas terms exchange the two cells' factors; with k != i
                    // the oil terms of a downstream cell change sign
                    const double g1 = ph == 1 ? F.gB : F.gM, g2 = ph == 1 ? F.gM : F.gB;
                    if (!up_nb) {
                        dR -= (Tg + ac * g1) * fd.dH;
                        dB -= ac * g2 * fd.dH;
                    } else {
                        const double flip = (!diag && !total && ph == 0) ? -1.0 : 1.0;
                        dR -= flip * (an * g1 * fd.dH);
                        dB -= flip * ((Tg + an * g2) * fd.dH);
                    }
                }
                // intra-continuum diffusion (component rows only)
                if (idiff && !total && coef != 0 && dC != 0) {
                    const bool dn_up = wn > wc;
                    const double Dup = dn_up ? nb.D(i, ph) : q.D(i, ph);
                    const double dDx = dn_up ? dd_col(v, dcn, nb, i, k, ph) : dd_col(v, dcq, q, i, k, ph);
                    const double dDdx = dn_up ? 0.0 : dDx, dDdx2 = dn_up ? dDx : 0.0;
                    const double DX = wn - wc;
                    const double dMM = dEq * e.dl * dC * F.P.iBB, dMM2 = dEn * e.dn * coef * F.P.iBB;
                    dR += s * NNd * ((diag ? -F.P.MMd * Dup : 0.0) + dDdx * F.P.MMd * DX + dMM * Dup * DX);
                    dB += s * NNd * ((diag ? F.P.MMd * Dup : 0.0) + dDdx2 * F.P.MMd * DX + dMM2 * Dup * DX);
                }
                const double nv = -dB * coef;
                if (ph == 0) {
                    accX[i] += dR;
                    if (lnb == 0) out.st(L.cr(row, e.slot, k), nv);
                    else accZ[i] = nv;
                } else {
                    accY[i] += dR;
                    if (lnb == 0) {
                        out.st(L.cr(row, e.slot, N + k), nv);
                    } else {
                        // both phases land in the neighbour's one composition column
                        const double w = accZ[i] + nv;
                        out.st(L.cr(row, e.slot, k), to_x ? w : 0.0);
                        out.st(L.cr(row, e.slot, N + k), to_x ? 0.0 : w);
                    }
                }
            }
        }
    }
    for (int sl = 1; sl <= 6; sl++)
        if (!(present & (1u << sl)))
            for (int i = 0; i < N; i++) {
                out.st(L.cr(N + i, sl, k), 0.0);
                out.st(L.cr(N + i, sl, N + k), 0.0);
            }
    // 3) this cell's block
    const OwnLayout O = own_layout(lq);
    const WellAt W = well_at(v, med, c, 0, 0.0);
    for (int i = 0; i < N; i++) {
        const int row = N + i;
        const bool total = i == N - 1, diag = !total && i == k;
        double X, Y;
        if (total) {
            const double po_ = med ? pf : pm;
            const double dEq0 = med ? dEkF[0] : dEkM[0], dEq1 = med ? dEkF[1] : dEkM[1];
            X = (Vb / jdt(v)) * po_ * q.S(1) * dEq0 - accX[i];
            Y = (Vb / jdt(v)) * po_ * q.S(2) * dEq1 - accY[i];
        } else {
            const double dQxl = (diag && W.iwell < 0) ? W.Qo : 0.0, dQxg = (diag && W.iwell < 0) ? W.Qg : 0.0;
            if (med == 0) {
                const double xi = M.w(0, i), yi = M.w(1, i);
                const double dLxl = diag ? ro + xi * dEkM[0] : xi * dEkM[0];
                const double dLxg = diag ? rg + yi * dEkM[1] : yi * dEkM[1];
                X = (Vb / jdt(v)) * pm * M.S(1) * dLxl - dQxl - accX[i];
                Y = (Vb / jdt(v)) * pm * M.S(2) * dLxg - dQxg - accY[i];
            } else {
                const double fxi = Fr.w(0, i), fyi = Fr.w(1, i);
                const double dLxl = diag ? Fr.rho(0) + fxi * dEkF[0] : fxi * dEkF[0];
                const double dLxg = diag ? Fr.rho(1) + fyi * dEkF[1] : fyi * dEkF[1];
                X = (Vb / jdt(v)) * pf * Fr.S(1) * dLxl - dQxl - accX[i];
                Y = (Vb / jdt(v)) * pf * Fr.S(2) * dLxg - dQxg - accY[i];
            }
        }
        out.st(L.cr(row, 0, k), O.x ? X : 0.0);
        out.st(L.cr(row, 0, N + k), O.y ? Y : 0.0);
    }
}

// The pressure and saturation columns (P, Sw, So, Sg) of all component and
// total rows of block row (med, c) in every block, and the total row's eight
// shifted entries.  dp, dSw, dSo, dSg: N doubles each.
OSR_HD inline void ps_task(const JacView &v, int med, long c, const Out &out, SmemVec dp, SmemVec dSw, SmemVec dSo,
                           SmemVec dSg) {
    const int N = v.nc;
    const Layout L(N);
    const Cell M{&v, &v.m[0], c, 0}, Fr{&v, &v.m[1], c, 1};
    const Cell &q = med ? Fr : M;
    const int lm = M.label(), lf = Fr.label(), lq = q.label(), lo = med ? lm : lf;
    const Transfer t = transfer_terms(v, c);
    const double pm = t.pm, pf = t.pf, dpm = t.dpm, dpf = t.dpf;
    const double Vb = t.Vb, SF1 = t.SF1, SF2 = t.SF2, SF3 = t.SF3;
    const double tor = ld(v.tor + c);
    const double ro = M.rho(0), rg = M.rho(1);
    const double mubar_o = t.Do / (pm + pf), mubar_g = t.Dg / (pm + pf);
    const bool idiff = !v.diff_off;
    // pressure parts of the diffusion-coefficient derivatives of both cells
    DCol dpM[2], dpF[2];
    for (int ph = 0; ph < 2; ph++) {
        dpM[ph] = make_dcol(M, N, ph, M.dE(N, ph));
        dpF[ph] = make_dcol(Fr, N, ph, Fr.dE(N, ph));
    }
    // 1) transfer terms of every row (this cell's accumulations) and the other continuum's block
    for (int i = 0; i < N; i++) {
        const int row = N + i;
        const bool total = i == N - 1;
        double a_dp = 0, a_dSw = 0, a_dSo = 0, a_dSg = 0;
        double oP, oSw, oSo, oSg;
        if (total) {
            double tm = 0, tf = 0;
            tm += kSIC * M.dE(N, 0) * SF2 * Vb * t.kro / mubar_o * t.dPo;
            tm += -kSIC * ro * SF2 * Vb * t.kro / mubar_o;
            tm += -kSIC * (dmu(M, N, 0) * pm + dpm * M.mu(0)) * ro * SF2 * Vb * t.kro / (t.Do * t.Do) * t.dPo * (pm + pf);
            tm += kSIC * dpm * ro * SF2 * Vb * t.kro / t.Do * t.dPo;
            tm += kSIC * M.dE(N, 1) * SF2 * Vb * t.krg / mubar_g * t.dPg;
            tm += -kSIC * rg * SF2 * Vb * t.krg / mubar_g;
            tm += -kSIC * (dmu(M, N, 1) * pm + dpm * M.mu(1)) * rg * SF2 * Vb * t.krg / (t.Dg * t.Dg) * t.dPg * (pm + pf);
            tm += kSIC * dpm * rg * SF2 * Vb * t.krg / t.Dg * t.dPg;
            tf += kSIC * ro * SF2 * Vb * t.kro / mubar_o;
            tf += -kSIC * (dmu(Fr, N, 0) * pf + dpf * Fr.mu(0)) * ro * SF2 * Vb * t.kro / (t.Do * t.Do) * t.dPo * (pm + pf);
            tf += kSIC * dpf * ro * SF2 * Vb * t.kro / t.Do * t.dPo;
            tf += kSIC * rg * SF2 * Vb * t.krg / mubar_g;
            tf += -kSIC * (dmu(Fr, N, 1) * pf + dpf * Fr.mu(1)) * rg * SF2 * Vb * t.krg / (t.Dg * t.Dg) * t.dPg * (pm + pf);
            tf += kSIC * dpf * rg * SF2 * Vb * t.krg / t.Dg * t.dPg;
            const double sg = med ? -1.0 : 1.0;
            a_dp += sg * (med ? tf : tm);
            oP = sg * (med ? tm : tf);
            const double po = ro * SF2 * Vb / mubar_o * t.dPo, pg = rg * SF2 * Vb / mubar_g * t.dPg;
            const double smSo = kSIC * t.dkm[4] * po, sfSo = kSIC * t.dkf[4] * po;
            const double smSg = kSIC * t.dkm[2] * po + kSIC * t.dkm[3] * pg, sfSg = kSIC * t.dkf[2] * po + kSIC * t.dkf[3] * pg;
            const double smSw = kSIC * t.dkm[1] * po, sfSw = kSIC * t.dkf[1] * po;
            a_dSo += sg * (med ? sfSo : smSo);
            a_dSg += sg * (med ? sfSg : smSg);
            a_dSw += sg * (med ? sfSw : smSw);
            oSo = sg * (med ? smSo : sfSo);
            oSg = sg * (med ? smSg : sfSg);
            oSw = sg * (med ? smSw : sfSw);
        } else if (med == 0) {
            // matrix component row i
            const double xi = M.w(0, i), yi = M.w(1, i);
            double dRfdp = 0;
            a_dp += kSIC * M.dE(N, 0) * xi * SF2 * Vb * t.kro / mubar_o * t.dPo;
            a_dp += -kSIC * xi * ro * SF2 * Vb * t.kro / mubar_o;
            a_dp += -kSIC * (dmu(M, N, 0) * pm + dpm * M.mu(0)) * xi * ro * SF2 * Vb * t.kro / (t.Do * t.Do) * t.dPo * (pm + pf);
            a_dp += kSIC * dpm * xi * ro * SF2 * Vb * t.kro / t.Do * t.dPo;
            a_dp += kSIC * M.dE(N, 1) * yi * SF2 * Vb * t.krg / mubar_g * t.dPg;
            a_dp += -kSIC * yi * rg * SF2 * Vb * t.krg / mubar_g;
            a_dp += -kSIC * (dmu(M, N, 1) * pm + dpm * M.mu(1)) * yi * rg * SF2 * Vb * t.krg / (t.Dg * t.Dg) * t.dPg * (pm + pf);
            a_dp += kSIC * dpm * yi * rg * SF2 * Vb * t.krg / t.Dg * t.dPg;
            for (int ph = 0; ph < 2 && idiff; ph++) {
                int kinds[2];
                const int nt = matrix_diff_targets(lm, lf, ph, kinds);
                if (!nt) continue;
                const double sat = M.S(1 + ph), rho = M.rho(ph), D = M.D(i, ph), w = M.w(ph, i);
                const double dDdp = dd_col(v, dpM[ph], M, i, N, ph);
                for (int j = 0; j < nt; j++) {
                    const double tgt = kinds[j] ? Fr.w(ph, i) : 0.0;
                    a_dp += dpm * SF1 * sat * Vb / tor * rho * D * (tgt - w);
                    a_dp += M.dE(N, ph) * SF1 * sat * pm * Vb / tor * D * (tgt - w);
                    a_dp += dDdp * SF1 * sat * pm * Vb / tor * rho * (tgt - w);
                }
            }
            dRfdp += kSIC * xi * ro * SF2 * Vb * t.kro / mubar_o;
            dRfdp += -kSIC * (dmu(Fr, N, 0) * pf + dpf * Fr.mu(0)) * xi * ro * SF2 * Vb * t.kro / (t.Do * t.Do) * t.dPo * (pm + pf);
            dRfdp += kSIC * dpf * xi * ro * SF2 * Vb * t.kro / t.Do * t.dPo;
            dRfdp += kSIC * yi * rg * SF2 * Vb * t.krg / mubar_g;
            dRfdp += -kSIC * (dmu(Fr, N, 1) * pf + dpf * Fr.mu(1)) * yi * rg * SF2 * Vb * t.krg / (t.Dg * t.Dg) * t.dPg * (pm + pf);
            dRfdp += kSIC * dpf * yi * rg * SF2 * Vb * t.krg / t.Dg * t.dPg;
            double dRfdSw = 0, dRfdSo = 0, dRfdSg = 0;
            const double po = xi * ro * SF2 * Vb / mubar_o * t.dPo, pg = yi * rg * SF2 * Vb / mubar_g * t.dPg;
            a_dSo += kSIC * t.dkm[4] * po;
            if (idiff) {
                int kinds[2];
                const int nt = matrix_diff_targets(lm, lf, 0, kinds);
                for (int j = 0; j < nt; j++) {
                    const double tgt = kinds[j] ? Fr.w(0, i) : 0.0;
                    a_dSo += SF1 * Vb * pm / tor * ro * M.D(i, 0) * (tgt - xi);
                }
            }
            dRfdSo += kSIC * t.dkf[4] * po;
            a_dSg += kSIC * t.dkm[2] * po;
            a_dSg += kSIC * t.dkm[3] * pg;
            if (idiff) {
                // the gas saturation derivative omits the two-phase matrix / oil fracture pairing
                int kinds[2];
                int nt = matrix_diff_targets(lm, lf, 1, kinds);
                if (lm == 0 && lf == 1) nt = 0;
                for (int j = 0; j < nt; j++) {
                    const double tgt = kinds[j] ? Fr.w(1, i) : 0.0;
                    a_dSg += SF1 * Vb * pm / tor * rg * M.D(i, 1) * (tgt - yi);
                }
            }
            dRfdSg += kSIC * t.dkf[2] * po;
            dRfdSg += kSIC * t.dkf[3] * pg;
            a_dSw += kSIC * t.dkm[1] * po;
            dRfdSw += kSIC * t.dkf[1] * po;
            oP = dRfdp;
            oSw = dRfdSw;
            oSo = dRfdSo;
            oSg = dRfdSg;
        } else {
            // fracture component row i
            const double xi = M.w(0, i), yi = M.w(1, i);
            const double fxi = Fr.w(0, i), fyi = Fr.w(1, i);
            double dRMdp = 0;
            dRMdp -= kSIC * M.dE(N, 0) * xi * SF2 * Vb * t.kro / mubar_o * t.dPo;
            dRMdp -= -kSIC * xi * ro * SF2 * Vb * t.kro / mubar_o;
            dRMdp -= -kSIC * (dmu(M, N, 0) * pm + dpm * M.mu(0)) * xi * ro * SF2 * Vb * t.kro / (t.Do * t.Do) * t.dPo * (pf + pm);
            dRMdp -= kSIC * dpm * xi * ro * SF2 * Vb * t.kro / t.Do * t.dPo;
            dRMdp -= kSIC * M.dE(N, 1) * yi * SF2 * Vb * t.krg / mubar_g * t.dPg;
            dRMdp -= -kSIC * yi * rg * SF2 * Vb * t.krg / mubar_g;
            dRMdp -= -kSIC * (dmu(M, N, 1) * pm + dpm * M.mu(1)) * yi * rg * SF2 * Vb * t.krg / (t.Dg * t.Dg) * t.dPg * (pf + pm);
            dRMdp -= kSIC * dpm * yi * rg * SF2 * Vb * t.krg / t.Dg * t.dPg;
            for (int ph = 0; ph < 2 && idiff; ph++) {
                if (!fsf1(lm, lf, ph)) continue;
                const double sat = M.S(1 + ph), rho = M.rho(ph), D = M.D(i, ph), dlt = Fr.w(ph, i) - M.w(ph, i);
                dRMdp -= dpm * SF1 * sat * Vb / tor * rho * D * dlt;
                dRMdp -= M.dE(N, ph) * SF1 * sat * pm * Vb / tor * D * dlt;
                dRMdp -= dd_col(v, dpM[ph], M, i, N, ph) * SF1 * sat * pm * Vb / tor * rho * dlt;
            }
            a_dp -= kSIC * xi * ro * SF2 * Vb * t.kro / mubar_o;
            a_dp -= -kSIC * (dmu(Fr, N, 0) * pf + dpf * Fr.mu(0)) * xi * ro * SF2 * Vb * t.kro / (t.Do * t.Do) * t.dPo * (pf + pm);
            a_dp -= kSIC * dpf * xi * ro * SF2 * Vb * t.kro / t.Do * t.dPo;
            a_dp -= kSIC * yi * rg * SF2 * Vb * t.krg / mubar_g;
            a_dp -= -kSIC * (dmu(Fr, N, 1) * pf + dpf * Fr.mu(1)) * yi * rg * SF2 * Vb * t.krg / (t.Dg * t.Dg) * t.dPg * (pf + pm);
            a_dp -= kSIC * dpf * yi * rg * SF2 * Vb * t.krg / t.Dg * t.dPg;
            for (int ph = 0; ph < 2 && idiff; ph++) {
                if (!fsf3(lm, lf, ph)) continue;
                const double sat = Fr.S(1 + ph), rho = Fr.rho(ph), D = Fr.D(i, ph), w = Fr.w(ph, i);
                a_dp -= dpf * SF3 * sat * Vb / tor * rho * D * (w - 0.0);
                a_dp -= Fr.dE(N, ph) * SF3 * sat * pf * Vb / tor * D * (w - 0.0);
                a_dp -= dd_col(v, dpF[ph], Fr, i, N, ph) * SF3 * sat * pf * Vb / tor * rho * (w - 0.0);
            }
            double dRMdSo = 0, dRMdSg = 0, dRMdSw = 0;
            const double po = xi * ro * SF2 * Vb / mubar_o * t.dPo, pg = yi * rg * SF2 * Vb / mubar_g * t.dPg;
            dRMdSo -= kSIC * t.dkm[4] * po;
            if (idiff && fsf1(lm, lf, 0)) dRMdSo -= SF1 * Vb * pm / tor * ro * M.D(i, 0) * (fxi - xi);
            a_dSo -= kSIC * t.dkf[4] * po;
            if (idiff && fsf3(lm, lf, 0)) a_dSo -= SF3 * Vb * pf / tor * Fr.rho(0) * Fr.D(i, 0) * (fxi - 0.0);
            dRMdSg -= kSIC * t.dkm[2] * po;
            dRMdSg -= kSIC * t.dkm[3] * pg;
            if (idiff && fsf1(lm, lf, 1)) dRMdSg -= SF1 * Vb * pm / tor * rg * M.D(i, 1) * (fyi - yi);
            a_dSg -= kSIC * t.dkf[2] * po;
            a_dSg -= kSIC * t.dkf[3] * pg;
            if (idiff && fsf3(lm, lf, 1)) a_dSg -= SF3 * Vb * pf / tor * Fr.rho(1) * Fr.D(i, 1) * (fyi - 0.0);
            dRMdSw -= kSIC * t.dkm[1] * po;
            a_dSw -= kSIC * t.dkf[1] * po;
            oP = dRMdp;
            oSw = dRMdSw;
            oSo = dRMdSo;
            oSg = dRMdSg;
        }
        dp[i] = a_dp;
        dSw[i] = a_dSw;
        dSo[i] = a_dSo;
        dSg[i] = a_dSg;
        store_other_ps(N, out, row, lo, jpc(v) * oP, oSw, oSo, oSg);
    }
    // 2) faces
    JFace fc[6];
    const int nf = jac_faces(v, c, fc);
    unsigned present = 0;
    for (int f = 0; f < nf; f++) present |= 1u << fc[f].slot;
    // advective flux, this cell's pressure
    for (int ph = 0; ph < 2; ph++)
        for (int f = 0; f < nf; f++) {
            const FaceData fd = face_data(v, *q.F, c, fc[f]);
            const double T = fd.T[ph];
            const Cell U{&v, q.F, upstream(fc[f], fd, c, ph), med};
            for (int i = 0; i < N; i++) dp[i] += i == N - 1 ? T : U.w(ph, i) * T;
        }
    double ov[kOverflow];
    for (int j = 0; j < kOverflow; j++) ov[j] = 0;
    const double tor_c = med ? 1.0 : tor;
    const double pq = q.porpor(), dpq = q.dpordp();
    const bool q_inactive = q.por() < 1e-10;
    for (int f = 0; f < nf; f++) {
        const JFace &e = fc[f];
        const Cell nb{&v, q.F, e.nb, med};
        const FaceData fd = face_data(v, *q.F, c, e);
        const int lnb = nb.label();
        const double s = e.sgn;
        const bool nb_o = upstream(e, fd, c, 0) == e.nb, nb_g = upstream(e, fd, c, 1) == e.nb;
        const double tor_n = med ? 1.0 : ld(v.tor + e.nb);
        const double pn = nb.porpor(), dpn = nb.dpordp();
        const double NNd = e.area2 / (e.dn + e.dl);
        const bool inactive = q_inactive || nb.por() < 1e-10;
        // the pressure factors of both phases (shared by every row)
        Mob m[2];
        double coefs[2], dCs[2], MMd[2], dMM[2], dMM2[2];
        DCol dcnb[2];
        for (int ph = 0; ph < 2; ph++) {
            const double coef = ph == 0 ? (lnb == -1 ? 0.0 : 1.0) : (lnb == 1 ? 0.0 : 1.0);
            const double dC = ph == 0 ? (lq == -1 ? 0.0 : 1.0) : (lq == 1 ? 0.0 : 1.0);
            const Side sq{q.rho(ph), q.mu(ph), q.gam(ph)}, sn{nb.rho(ph), nb.mu(ph), nb.gam(ph)};
            const double dEq = q.dE(N, ph), dEn = nb.dE(N, ph);
            m[ph] = mobility(sq, sn, dEq, dEn, false, 0.0, e, coef, dmu(q, N, ph), dmu(nb, N, ph));
            dcnb[ph].zero = true;
            if (idiff) dcnb[ph] = make_dcol(nb, N, ph, dEn);
            coefs[ph] = coef;
            dCs[ph] = dC;
            double AAd = sn.rho * e.dn * coef + sq.rho * e.dl * dC;
            AAd *= (nb.S(1 + ph) * e.dn * coef + q.S(1 + ph) * e.dl * dC) / (e.dn + e.dl);
            const double BBd = tor_n * e.dn * coef / pn + tor_c * e.dl * dC / pq;
            MMd[ph] = AAd / BBd;
            const double dAA = dEq * e.dl * dC, dAA2 = dEn * e.dn * coef;
            const double dBB = -dpq * tor_c * e.dl * dC / (pq * pq), dBB2 = -dpn * tor_n * e.dn * coef / (pn * pn);
            dMM[ph] = (dAA * BBd - dBB * AAd) / (BBd * BBd);
            dMM2[ph] = (dAA2 * BBd - dBB2 * AAd) / (BBd * BBd);
        }
        const int cS2 = lnb == -1 ? 3 : 2, cS3 = lnb == 1 ? 2 : 3;
        for (int i = 0; i < N; i++) {
            const int row = N + i;
            const bool total = i == N - 1;
            const FaceQuirks qk = total ? total_quirks(e) : comp_quirks(e);
            const double xo = total ? 1.0 : (nb_o ? nb : q).w(0, i), yg = total ? 1.0 : (nb_g ? nb : q).w(1, i);
            double ps[4] = {0, 0, 0, 0}, ovl[4] = {0, 0, 0, 0};
            auto put = [&](int tt, int cc, double val) {
                if (qk.shifted_block) ovl[tt] = val;
                else ps[cc] += val;
            };
            // saturation factors
            const double dsw = s * (xo * fd.T[4] * fd.dP[1] + xo * fd.T[6] * fd.dH);
            if (nb_o) put(1, 1, dsw);
            else dSw[i] += dsw;
            const double dso = s * (xo * fd.T[10] * fd.dP[1] + xo * fd.T[11] * fd.dH);
            if (nb_o) put(2, cS2, lnb == -1 ? 0.0 : dso);
            else dSo[i] += dso;
            const double dsgo = s * (xo * fd.T[8] * fd.dP[1] + xo * fd.T[9] * fd.dH);
            const double dsgg = s * (yg * fd.T[5] * fd.dP[2] + yg * fd.T[7] * fd.dH);
            double vsg = 0;
            if (nb_o) vsg = lnb == 1 ? 0.0 : dsgo;
            else dSg[i] += dsgo;
            if (nb_g) vsg += lnb == 1 ? 0.0 : dsgg;
            else dSg[i] += dsgg;
            put(3, cS3, vsg);
            // mobility and diffusion derivatives with respect to the two pressures
            double dB = 0;
            for (int ph = 0; ph < 2; ph++) {
                const Mob &mb = m[ph];
                const bool up_nb = ph == 0 ? nb_o : nb_g;
                const Cell &U = up_nb ? nb : q;
                const double wk = total ? 1.0 : U.w(ph, i), krk = U.kr(1 + ph);
                const double dPp = fd.dP[1 + ph];
                const double a = wk * fd.ift * krk;
                dp[i] -= s * (a * mb.M * dPp);
                const double vB = s * (a * mb.B * dPp);
                if (ph == 1 && e.sgn < 0) {
                    const bool assign = up_nb ? qk.gas_dB_assign_down : qk.gas_dB_assign_up;
                    dB = assign ? vB : dB + vB;
                    // the reference exchanges this cell's and the neighbour's gravity factors here
                    dp[i] -= s * (a * (mb.B * mb.tempdx + mb.BG * mb.Sur / mb.Mak) * fd.dH);
                    dB += s * (a * (mb.M * mb.tempdx + mb.MG * mb.Sur / mb.Mak) * fd.dH);
                } else {
                    dB = ph == 0 ? vB : dB + vB;
                    dp[i] -= s * (a * (mb.M * mb.tempdx + mb.MG * mb.Sur / mb.Mak) * fd.dH);
                    const double gB = s * (a * (mb.B * mb.tempdx + mb.BG * mb.Sur / mb.Mak) * fd.dH);
                    if (ph == 0 && e.sgn < 0 && up_nb && qk.oil_grav_assign_down) dB = gB;
                    else dB += gB;
                }
                if (total || !idiff) continue;
                // intra-continuum diffusion
                const double wq = q.w(ph, i), wn = nb.w(ph, i);
                double Dup, dDdp, dDdp2;
                if (wn > wq) {
                    Dup = nb.D(i, ph);
                    dDdp = 0;
                    dDdp2 = dd_col(v, dcnb[ph], nb, i, N, ph);
                } else {
                    Dup = q.D(i, ph);
                    dDdp = dd_col(v, med ? dpF[ph] : dpM[ph], q, i, N, ph);
                    dDdp2 = 0;
                }
                if (inactive) Dup = dDdp = dDdp2 = 0;
                const double DX = wn - wq;
                if (coefs[ph] != 0 && dCs[ph] != 0) {
                    dp[i] += -NNd * DX * (MMd[ph] * dDdp + Dup * dMM[ph]);
                    dB += NNd * DX * (MMd[ph] * dDdp2 + Dup * dMM2[ph]);
                }
            }
            put(0, 0, jpc(v) * (-xo * fd.T[0] - yg * fd.T[1] - dB));
            for (int tt = 0; tt < 4; tt++) out.st(L.cr(row, e.slot, 2 * N + tt), ps[tt]);
            if (total && qk.shifted_block)
                for (int tt = 0; tt < 4; tt++) ov[(e.d == 1 ? 0 : 4) + tt] = ovl[tt];
        }
    }
    for (int sl = 1; sl <= 6; sl++)
        if (!(present & (1u << sl)))
            for (int i = 0; i < N; i++)
                for (int tt = 0; tt < 4; tt++) out.st(L.cr(N + i, sl, 2 * N + tt), 0.0);
    for (int j = 0; j < kOverflow; j++) out.st(L.o(j), ov[j]);
    // 3) this cell's block, with the accumulation and the completion's productivity terms
    for (int i = 0; i < N; i++) {
        const int row = N + i;
        double dLdp, dLdSo, dLdSg, well;
        if (i == N - 1) {
            const double po_ = med ? pf : pm, dpo_ = med ? dpf : dpm;
            dLdp = (Vb / jdt(v)) * (q.S(1) * (q.rho(0) * dpo_ + q.dE(N, 0) * po_) + q.S(2) * (q.rho(1) * dpo_ + q.dE(N, 1) * po_));
            dLdSo = (Vb / jdt(v)) * (po_ * q.rho(0));
            dLdSg = (Vb / jdt(v)) * (po_ * q.rho(1));
            const WellAt W = well_at(v, med, c, 0, 0.0);
            well = W.PIo + W.PIg;
        } else if (med == 0) {
            const double xi = M.w(0, i), yi = M.w(1, i);
            dLdp = (Vb / jdt(v)) * (xi * M.S(1) * (ro * dpm + M.dE(N, 0) * pm) + yi * M.S(2) * (rg * dpm + M.dE(N, 1) * pm));
            dLdSo = (Vb / jdt(v)) * (xi * pm * ro);
            dLdSg = (Vb / jdt(v)) * (yi * pm * rg);
            const WellAt W = well_at(v, 0, c, i, yi);
            well = xi * W.PIo + W.gcomp * W.PIg;
        } else {
            const double fxi = Fr.w(0, i), fyi = Fr.w(1, i);
            dLdp = (Vb / jdt(v)) * (fxi * Fr.S(1) * (Fr.rho(0) * dpf + Fr.dE(N, 0) * pf) + fyi * Fr.S(2) * (Fr.rho(1) * dpf + Fr.dE(N, 1) * pf));
            dLdSo = (Vb / jdt(v)) * (fxi * pf * Fr.rho(0));
            dLdSg = (Vb / jdt(v)) * (fyi * pf * Fr.rho(1));
            const WellAt W = well_at(v, 1, c, i, fyi);
            well = fxi * W.PIo + W.gcomp * W.PIg;
        }
        store_own_ps(N, out, row, lq, jpc(v) * (dLdp + dp[i] + well), -dSw[i], dLdSo - dSo[i], dLdSg - dSg[i]);
    }
}

// Inactive cell-media (porosity < 1e-10): the unit entries of the reference's
// diagonal in the columns a task owns, zeros elsewhere.
OSR_HD inline void inactive_column(int N, const Out &out, int lab, int k) {
    const Layout L(N);
    for (int i = 0; i < N; i++) {
        const int row = N + i, uc = unit_col(N, lab, row);
        for (int sl = 0; sl < 8; sl++) {
            out.st(L.cr(row, sl, k), (sl == 0 && uc == k) ? 1.0 : 0.0);
            out.st(L.cr(row, sl, N + k), (sl == 0 && uc == N + k) ? 1.0 : 0.0);
        }
    }
}

OSR_HD inline void zero_ps(int N, const Out &out) {
    const Layout L(N);
    for (int i = 0; i < N; i++)
        for (int sl = 0; sl < 8; sl++)
            for (int tt = 0; tt < 4; tt++) out.st(L.cr(N + i, sl, 2 * N + tt), 0.0);
    for (int j = 0; j < kOverflow; j++) out.st(L.o(j), 0.0);
}

OSR_HD inline void zero_column(int N, const Out &out, int k) {
    const Layout L(N);
    for (int i = 0; i < N; i++)
        for (int sl = 0; sl < 8; sl++) {
            out.st(L.cr(N + i, sl, k), 0.0);
            out.st(L.cr(N + i, sl, N + k), 0.0);
        }
}

OSR_HD inline void zero_misc(int N, const Out &out) {
    const Layout L(N);
    for (int e = 0; e < L.EF; e++) out.st(e, 0.0);
    for (int e = L.EF + L.EC; e < L.E; e++) out.st(e, 0.0);
}

// ---------------------------------------------------------------------------
// Water row (canonical 2N).
// ---------------------------------------------------------------------------
OSR_HD inline void water_row(const JacView &v, int med, long c, const Out &out) {
    const int N = v.nc;
    const Layout L(N);
    const Cell M{&v, &v.m[0], c, 0}, Fr{&v, &v.m[1], c, 1};
    const Cell &O = med ? Fr : M;
    const JMed &F = v.m[med];
    const Transfer t = transfer_terms(v, c);
    const double wr = v.wat_ro * kWatMRo;
    const double po_ = med ? t.pf : t.pm, dpo_ = med ? t.dpf : t.dpm;
    const double sg = med ? -1.0 : 1.0;
    const double dLdp = (t.Vb / jdt(v)) * wr * O.S(0) * dpo_;
    const double dLdSw = (t.Vb / jdt(v)) * (po_ * wr);
    const double tr = kSIC * v.wat_ro * kWatMRo * t.SF2 * t.krw / v.wat_mu * t.Vb;
    // both continua's water rows take -tr for their own pressure, +tr for the other's
    double dRdp = -tr;
    const double dROdp = tr;
    JFace fc[6];
    const int nf = jac_faces(v, c, fc);
    const long n = v.n;
    for (int q = 0; q < nf; q++) dRdp += ld(F.wtran + (long)fc[q].d * n + fc[q].tc);
    const WellAt W = well_at(v, med, c, 0, 0.0);
    out.st(L.w(0, 2 * N), jpc(v) * (dLdp + dRdp + W.PIw));
    const double smw = kSIC * kWatMRo * t.dkm[0] * v.wat_ro * t.SF2 / v.wat_mu * t.Vb * t.dPw;
    const double sfw = kSIC * kWatMRo * t.dkf[0] * v.wat_ro * t.SF2 / v.wat_mu * t.Vb * t.dPw;
    double dRdSw = sg * (med ? sfw : smw);
    const double dROSw = sg * (med ? smw : sfw);
    unsigned present = 0;
    for (int q = 0; q < nf; q++) {
        const JFace &e = fc[q];
        present |= 1u << e.slot;
        const FaceData fd = face_data(v, F, c, e);
        const double Tw = ld(F.wtran + (long)e.d * n + e.tc), dTw = ld(F.dwtran + (long)e.d * n + e.tc);
        out.st(L.w(e.slot, 2 * N), jpc(v) * (-Tw));
        const double dsw = e.sgn * (dTw * fd.dP[0] + kGAcc * v.wat_ro * dTw * fd.dH);
        const bool up_nb = upstream(e, fd, c, 2) == e.nb;
        out.st(L.w(e.slot, 2 * N + 1), up_nb ? dsw : 0.0);
        if (!up_nb) dRdSw += dsw;
    }
    for (int s = 1; s <= 6; s++)
        if (!(present & (1u << s))) {
            out.st(L.w(s, 2 * N), 0.0);
            out.st(L.w(s, 2 * N + 1), 0.0);
        }
    out.st(L.w(0, 2 * N + 1), dLdSw - dRdSw);
    out.st(L.w(7, 2 * N), jpc(v) * dROdp);
    out.st(L.w(7, 2 * N + 1), dROSw);
}

// ---------------------------------------------------------------------------
// Fugacity rows of a two-phase cell (compsim/Petsc_Functions.cpp:30240-30406
// for the matrix): x_i P_o phi_i^L - y_i P_g phi_i^V with Z from the stored
// density and dZ from dE.
// ---------------------------------------------------------------------------
OSR_HD inline void fugacity_rows(const JacView &v, const Cell &q, const Out &out) {
    const int N = v.nc;
    const Layout L(N);
    const double RT = kR * v.T;
    const double Pl = q.P(1), Pg = q.P(2);
    double xl[kMaxNc], yg[kMaxNc], tl[kMaxNc], tg[kMaxNc];
    for (int i = 0; i < N; i++) {
        xl[i] = q.w(0, i);
        yg[i] = q.w(1, i);
    }
    double Al = 0, Bl = 0, Ag = 0, Bg = 0;
    for (int i = 0; i < N; i++) {
        Bl += xl[i] * v.b[i];
        Bg += yg[i] * v.b[i];
        for (int j = 0; j < N; j++) {
            const double t = v.sa[i] * v.sa[j] * v.bic[i * N + j];
            Al += xl[i] * xl[j] * t;
            Ag += yg[i] * yg[j] * t;
        }
    }
    // sum_j w_j sqrt(a_i a_j) bic_ij of each component
    for (int i = 0; i < N; i++) {
        double a = 0, g = 0;
        for (int j = 0; j < N; j++) {
            const double t = v.sa[i] * v.sa[j] * v.bic[i * N + j];
            a += xl[j] * t;
            g += yg[j] * t;
        }
        tl[i] = a;
        tg[i] = g;
    }
    const double Cal = Al, Cbl = Bl, Cag = Ag, Cbg = Bg;
    Al *= Pl / (RT * RT);
    Bl *= Pl / RT;
    Ag *= Pg / (RT * RT);
    Bg *= Pg / RT;
    const double dAdpl = Cal / (RT * RT), dAdpg = Cag / (RT * RT), dBdpl = Cbl / RT, dBdpg = Cbg / RT;
    const double Zl = Pl / (q.rho(0) * RT), Zg = Pg / (q.rho(1) * RT);
    const double dZdpl = (1 - q.dE(N, 0) * RT * Zl) * (Zl / Pl), dZdpg = (1 - q.dE(N, 1) * RT * Zg) * (Zg / Pg);
    const double d1 = v.srk ? 1.0 : 1 + kSqrt2, d2 = v.srk ? 0.0 : 1 - kSqrt2;
    const double DDl = Al / (Bl * (d1 - d2)), DDg = Ag / (Bg * (d1 - d2));
    const double FFl = log((Zl + d2 * Bl) / (Zl + d1 * Bl)), FFg = log((Zg + d2 * Bg) / (Zg + d1 * Bg));
    const double lZBl = log(Zl - Bl), lZBg = log(Zg - Bg);
    // Denominators of the composition derivatives that do not depend on the
    // entry, inverted once per cell (the reference divides in every entry).
    const double iCb2l = 1 / (Cbl * Cbl), iCb2g = 1 / (Cbg * Cbg), iCbl = 1 / Cbl, iCbg = 1 / Cbg;
    const double iBB2l = 1 / (Bl * Bl * (d1 - d2)), iBB2g = 1 / (Bg * Bg * (d1 - d2));
    const double iZd2l = 1 / (Zl + d2 * Bl), iZd2g = 1 / (Zg + d2 * Bg);
    const double iZd1l = 1 / (Zl + d1 * Bl), iZd1g = 1 / (Zg + d1 * Bg);
    const double iZBl = 1 / (Zl - Bl), iZBg = 1 / (Zg - Bg);
    const double iCal = 1 / Cal, iCag = 1 / Cag;
    const double iPCal2 = 1 / (Pl * Cal * Cal), iPCag2 = 1 / (Pg * Cag * Cag);
    const double ZZPl = Zl * Zl / Pl, ZZPg = Zg * Zg / Pg;
    // d Z / d w_k of each phase (the reference's -dE RT Z^2 / P)
    double dzl[kMaxNc], dzg[kMaxNc];
    for (int k = 0; k < N; k++) {
        dzl[k] = -q.dE(k, 0) * RT * ZZPl;
        dzg[k] = -q.dE(k, 1) * RT * ZZPg;
    }
    for (int i = 0; i < N; i++) {
        const double t1l = v.b[i] / Cbl, t1g = v.b[i] / Cbg;
        const double EEl = 2 * tl[i] / Cal - t1l, EEg = 2 * tg[i] / Cag - t1g;
        const double phiL = exp(t1l * (Zl - 1) - lZBl + DDl * EEl * FFl);
        const double phiG = exp(t1g * (Zg - 1) - lZBg + DDg * EEg * FFg);
        const double dAAl = v.b[i] * dZdpl / Cbl, dAAg = v.b[i] * dZdpg / Cbg;
        const double dBBl = (dBdpl - dZdpl) / (Zl - Bl), dBBg = (dBdpg - dZdpg) / (Zg - Bg);
        const double dDDl = (Bl * dAdpl - Al * dBdpl) / (Bl * Bl * (d1 - d2)), dDDg = (Bg * dAdpg - Ag * dBdpg) / (Bg * Bg * (d1 - d2));
        const double dFFl = (dZdpl + d2 * dBdpl) / (Zl + d2 * Bl) - (dZdpl + d1 * dBdpl) / (Zl + d1 * Bl);
        const double dFFg = (dZdpg + d2 * dBdpg) / (Zg + d2 * Bg) - (dZdpg + d1 * dBdpg) / (Zg + d1 * Bg);
        const double dPhil = phiL * (dAAl + dBBl + EEl * (dDDl * FFl + DDl * dFFl));
        const double dPhig = phiG * (dAAg + dBBg + EEg * (dDDg * FFg + DDg * dFFg));
        const double xi = xl[i], yi = yg[i];
        out.st(L.f(i, 2 * N), jpc(v) * (xi * (phiL + Pl * dPhil) - yi * (phiG + Pg * dPhig)));
        const double bi = v.b[i], tli = tl[i], tgi = tg[i];
        for (int k = 0; k < N; k++) {
            const double dAl = tl[k] * (2 * Pl / (RT * RT)), dAg = tg[k] * (2 * Pg / (RT * RT));
            const double dBl = v.b[k] * Pl / RT, dBg = v.b[k] * Pg / RT;
            const double dZl = dzl[k], dZg = dzg[k];
            const double dAAxl = -v.b[k] * bi * (Zl - 1) * iCb2l + bi * dZl * iCbl;
            const double dAAxg = -v.b[k] * bi * (Zg - 1) * iCb2g + bi * dZg * iCbg;
            const double dBBxl = (dBl - dZl) * iZBl, dBBxg = (dBg - dZg) * iZBg;
            const double dDDxl = (dAl * Bl - dBl * Al) * iBB2l, dDDxg = (dAg * Bg - dBg * Ag) * iBB2g;
            const double dFFxl = (dZl + d2 * dBl) * iZd2l - (dZl + d1 * dBl) * iZd1l;
            const double dFFxg = (dZg + d2 * dBg) * iZd2g - (dZg + d1 * dBg) * iZd1g;
            const double tik = v.sa[i] * v.sa[k] * v.bic[i * N + k];
            const double dEEl = 2 * (tik * iCal - dAl * RT * RT * tli * iPCal2) + bi * v.b[k] * iCb2l;
            const double dEEg = 2 * (tik * iCag - dAg * RT * RT * tgi * iPCag2) + bi * v.b[k] * iCb2g;
            const double dPxl = phiL * (dAAxl + dBBxl + dDDxl * EEl * FFl + DDl * dEEl * FFl + DDl * EEl * dFFxl);
            const double dPxg = phiG * (dAAxg + dBBxg + dDDxg * EEg * FFg + DDg * dEEg * FFg + DDg * EEg * dFFxg);
            if (i == k) {
                out.st(L.f(i, k), Pl * phiL + Pl * xi * dPxl);
                out.st(L.f(i, N + k), -(Pg * phiG + Pg * yi * dPxg));
            } else {
                out.st(L.f(i, k), Pl * xi * dPxl);
                out.st(L.f(i, N + k), -Pg * yi * dPxg);
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Row tasks
// ---------------------------------------------------------------------------

// Task N: the fugacity rows (or a one-phase cell's unused rows), the water row
// and the constraint rows.
OSR_HD inline void misc_rows(const JacView &v, int med, long c, const Out &out) {
    const int N = v.nc;
    const Layout L(N);
    const Cell q{&v, &v.m[med], c, med};
    const int lab = q.label();
    const bool inactive = q.por() < 1e-10;
    // F region
    if (lab == 0 && !inactive) {
        fugacity_rows(v, q, out);
    } else {
        for (int r = 0; r < N; r++) {
            const int uc = unit_col(N, lab, r);
            for (int cc = 0; cc <= 2 * N; cc++) out.st(L.f(r, cc), cc == uc ? 1.0 : 0.0);
        }
    }
    // W region
    if (inactive) {
        for (int s = 0; s < 8; s++) {
            out.st(L.w(s, 2 * N), s == 0 ? 1.0 : 0.0);
            out.st(L.w(s, 2 * N + 1), 0.0);
        }
    } else {
        water_row(v, med, c, out);
    }
    // K region: the constraint rows, or unit entries where a row is unused
    for (int r = 2 * N + 1; r <= 2 * N + 3; r++) {
        const bool used = ref_row(N, lab, r) >= 0;
        const int uc = unit_col(N, lab, r);
        for (int cc = 0; cc < L.BS; cc++) {
            double val;
            if (inactive || !used) val = cc == uc ? 1.0 : 0.0;
            else if (r == 2 * N + 3) val = (cc == 2 * N + 1 || (cc == 2 * N + 2 && lab != -1) || (cc == 2 * N + 3 && lab != 1)) ? 1.0 : 0.0;
            else if (r == 2 * N + 1) val = cc < N ? 1.0 : 0.0;           // sum x (an oil-only cell's sum w)
            else val = (cc >= N && cc < 2 * N) ? 1.0 : 0.0;              // sum y (a gas-only cell's sum w)
            out.st(L.k(r, cc), val);
        }
    }
}

// Task kinds, one code path per launch: 0 matrix columns (task k = 0..N-1),
// 1 fracture columns, 2 matrix pressure-saturation columns (one task), 3
// fracture pressure-saturation columns, 4 fugacity / water / constraint rows.
// A kind's lanes only; lanes of the last chunk beyond the grid store zeros.
// smem: the thread's shared-memory column (3N or 4N doubles at stride).
template <int KIND>
OSR_HD inline void jacobian_task_kind(const JacView &v, long bm, int task, double *smem, int stride) {
    const int N = v.nc;
    const long nb = 2 * v.n;
    const Out out{v.vals, v.entries, bm};
    const int med = bm >= v.n;
    if (KIND == 4) {
        if (bm >= nb) zero_misc(N, out);
        else misc_rows(v, med, med ? bm - v.n : bm, out);
        return;
    }
    const int want = (KIND == 1 || KIND == 3) ? 1 : 0;
    if (bm >= nb) {
        if (KIND == 1) zero_column(N, out, task);
        if (KIND == 3) zero_ps(N, out);
        return;
    }
    if (med != want) return;
    const long c = med ? bm - v.n : bm;
    const Cell q{&v, &v.m[med], c, med};
    const SmemVec s0{smem, stride}, s1{smem + N * stride, stride}, s2{smem + 2 * N * stride, stride},
        s3{smem + 3 * N * stride, stride};
    if (KIND <= 1) {
        if (q.por() < 1e-10) inactive_column(N, out, q.label(), task);
        else column_task(v, med, c, task, out, s0, s1, s2);
    } else {
        if (q.por() < 1e-10) zero_ps(N, out);
        else ps_task(v, med, c, out, s0, s1, s2, s3);
    }
}

// Reference (global row, global column) of entry e of block row bm, or -1 for
// an entry the reference does not have (unit entries of unused rows, absent
// neighbours and unknowns).  rowoff: the row offsets of the row layout;
// lab_m, lab_f: per cell phase state of the two continua.
OSR_HD inline void entry_position(int N, int nx, int ny, int nz, long n, const long *rowoff, const signed char *lab_m,
                                  const signed char *lab_f, long bm, int e, long *grow, long *gcol) {
    const Layout L(N);
    *grow = *gcol = -1;
    const int med = bm >= n;
    const long c = med ? bm - n : bm;
    const signed char *lab = med ? lab_f : lab_m;
    const int lb = lab[c];
    const int ix = (int)(c % nx), iy = (int)((c / nx) % ny), iz = (int)(c / ((long)nx * ny));
    const long sy = nx, sz = (long)nx * ny;
    if (e >= L.E) {
        // shifted entries of the total row: face -y (0..3) or -z (4..7)
        const int j = e - L.E, f = j / 4, t = j % 4;
        if (f == 0 ? iy == 0 : iz == 0) return;
        const long stride = f == 0 ? sy : sz;
        const int lnb = lab[c - stride];
        const int nbase = lnb ? -N : 0, reCol4 = lnb ? 1 : 0;
        const int col = nbase + 2 * N + (t == 3 ? 3 - reCol4 : t);
        *grow = rowoff[bm] + ref_row(N, lb, 2 * N - 1);
        *gcol = rowoff[bm - stride + 1] + col;
        return;
    }
    int r, s, cc;
    if (e < L.EF) {
        r = e / (2 * N + 1);
        cc = e % (2 * N + 1);
        s = 0;
    } else if (e < L.EF + L.EC) {
        const int q = e - L.EF;
        r = N + q / (8 * L.BS);
        s = (q / L.BS) % 8;
        cc = q % L.BS;
    } else if (e < L.EF + L.EC + L.EW) {
        const int q = e - L.EF - L.EC;
        r = 2 * N;
        s = q / 2;
        cc = 2 * N + q % 2;
    } else {
        const int q = e - L.EF - L.EC - L.EW;
        r = 2 * N + 1 + q / L.BS;
        s = 0;
        cc = q % L.BS;
    }
    const int rr = ref_row(N, lb, r);
    if (rr < 0) return;
    long tb;   // target block row (cell-medium)
    switch (s) {
        case 0: tb = bm; break;
        case 1: if (ix == 0) return; tb = bm - 1; break;
        case 2: if (ix == nx - 1) return; tb = bm + 1; break;
        case 3: if (iy == 0) return; tb = bm - sy; break;
        case 4: if (iy == ny - 1) return; tb = bm + sy; break;
        case 5: if (iz == 0) return; tb = bm - sz; break;
        case 6: if (iz == nz - 1) return; tb = bm + sz; break;
        default: tb = med ? c : n + c; break;
    }
    const int lt = tb >= n ? lab_f[tb - n] : lab_m[tb];
    const int rc = ref_col(N, lt, cc);
    if (rc < 0) return;
    *grow = rowoff[bm] + rr;
    *gcol = rowoff[tb] + rc;
}

}  // namespace osrj

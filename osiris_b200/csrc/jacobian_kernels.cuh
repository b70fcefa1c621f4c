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
// One thread owns one cell of one continuum and writes its whole block row
// of a uniform block-sparse matrix: block size bs = 2N+4, eight block slots
// per block row (this cell, -x, +x, -y, +y, -z, +z neighbours, the other
// continuum's cell), values [block row][slot][bs][bs] row-major.  Rows and
// columns beyond a one-phase cell's N+3 unknowns stay zero.
//
// The code is plain C++ over a view of device arrays, so the same source is
// compiled for the GPU and, for testing, for the host.
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
        tc[kMaxNc], pc[kMaxNc], pcr_atm[kMaxNc], vc53[kMaxNc], vc23[kMaxNc], pD[kMaxNc * kMaxNc];
    double T;
    int srk;
    // scalars
    double cpor, dcpor, refp, wat_ro, wat_mu, sigma, lf, pcoeff, dt;
    int diff_off;   // CDIF present and zero: diffusive shape factors vanish
    int const_dif;  // CDIF present: diffusion-coefficient derivatives vanish
    JMed m[2];
    const long *rowoff;
    // wells (rates at the linearisation point, per cell-medium; optional)
    const double *well_pi;    // [2 cells][3] PIw, PIo, PIg or null
    const int *well_comp;     // [2 cells] index of the injection well whose stream sets the component split, -1
    const double *well_q;     // [2 cells][3] Qw, Qo, Qg or null
    const double *stream_y;   // [wells][kMaxNc] injected gas composition
    // output
    double *vals;
    int bs;
    // entries the reference places outside the eight-block pattern:
    // [block row][kOverflow] (local row, global column, value), count per block row
    int *ovf_row;
    long *ovf_col;
    double *ovf_val;
    int *ovf_n;
};

constexpr int kOverflow = 16;

// ---------------------------------------------------------------------------
// Small accessors
// ---------------------------------------------------------------------------
struct Cell {
    const JacView *v;
    const JMed *F;
    long c;
    OSR_HD double P(int p) const { return F->P[p * v->n + c]; }
    OSR_HD double S(int p) const { return F->sat[p * v->n + c]; }
    OSR_HD double w(int ph, int i) const { return (ph ? F->y : F->x)[(long)i * v->n + c]; }
    OSR_HD double rho(int ph) const { return F->rho[ph * v->n + c]; }
    OSR_HD double mu(int ph) const { return F->mu[ph * v->n + c]; }
    OSR_HD double gam(int ph) const { return F->gam[ph * v->n + c]; }
    OSR_HD double kr(int p) const { return F->kr[p * v->n + c]; }
    OSR_HD double dkr(int p) const { return F->dkr[p * v->n + c]; }
    OSR_HD double pc(int p) const { return F->pc[p * v->n + c]; }
    OSR_HD double dE(int k, int ph) const { return F->dE[(long)(2 * k + ph) * v->n + c]; }
    OSR_HD double D(int i, int ph) const { return F->diff[(long)(2 * i + ph) * v->n + c]; }
    OSR_HD double por() const { return F->por[c]; }
    OSR_HD int label() const { return F->label[c]; }
    OSR_HD double porpor() const {
        const double dp = P(1) - v->refp;
        return por() * (1 + v->cpor * dp + v->dcpor * dp * dp);
    }
    OSR_HD double dpordp() const { return por() * (v->cpor + 2 * v->dcpor * (P(1) - v->refp)); }
};

// d mu / d w_k (k < N) or d mu / d P (k == N) of one phase (DiffVisco /
// fDiffVisco, compsim/Mass_Tran.cpp:307-399).
OSR_HD inline double visc_deriv(const Cell &q, int k, int ph) {
    const JacView &v = *q.v;
    const int N = v.nc;
    double s1 = 0, s2 = 0, ro = 0, tcm = 0, pcm = 0, mwm = 0;
    for (int n = 0; n < N; n++) {
        const double w = q.w(ph, n);
        const double t = w * v.smw[n];
        s1 += t * v.mui[n];
        s2 += t;
        ro += w * v.vcm[n];
        tcm += w * v.tc[n];
        pcm += w * v.pcr_atm[n];
        mwm += w * v.mw[n];
    }
    const double rho = q.rho(ph);
    const double Er = rho * ro;
    const double eA = pow(tcm, 1.0 / 6), eB = sqrt(mwm), eC = pow(pcm, 2.0 / 3);
    const double eta = eA / (eB * eC);
    const double r1 = 0.10230 + 0.023364 * Er + 0.058533 * Er * Er - 0.040758 * Er * Er * Er + 0.0093324 * Er * Er * Er * Er;
    double dMuS, dEta, dEr;
    if (k < N) {
        dMuS = (v.mui[k] * v.smw[k] * s2 - v.smw[k] * s1) / (s2 * s2);
        dEta = ((1.0 / 6.0) * pow(tcm, -5.0 / 6.0) * v.tc[k] * eB * eC -
                eA * (0.5 * v.mw[k] * eC / sqrt(mwm) + (2.0 / 3.0) * pow(pcm, -1.0 / 3.0) * v.pc[k] * eB / 101325)) /
               (eB * eB * eC * eC);
        dEr = q.dE(k, ph) * ro + rho * v.vcm[k];
    } else {
        dMuS = 0;
        dEta = 0;
        dEr = q.dE(N, ph) * ro;
    }
    const double dMM = 4 * r1 * r1 * r1 * (0.023364 * dEr + 0.117066 * dEr * Er - 0.122274 * dEr * Er * Er + 0.0373296 * dEr * Er * Er * Er);
    return (dMM * eta - (r1 * r1 * r1 * r1 - 1e-4) * dEta) / (eta * eta) + dMuS;
}

// d D_i / d w_k (k < N) or d D_i / d P (k == N) of one phase (DifDiffusion /
// fDifDiffusion, compsim/Mass_Tran.cpp:107-305).  Unlike the coefficient
// itself (CalcDiffusion) it carries no 1e-4 factor.
OSR_HD inline double diff_deriv(const Cell &q, int i, int k, int ph) {
    const JacView &v = *q.v;
    const int N = v.nc;
    if (v.const_dif) return 0;
    double s1 = 0, s2 = 0;
    for (int j = 0; j < N; j++) {
        s1 += q.w(ph, j) * v.vc53[j];
        s2 += q.w(ph, j) * v.vc23[j];
    }
    const double rho = q.rho(ph);
    const double Er = rho * s1 / s2;
    const double AA = 0.99589 + 0.096016 * Er - 0.22035 * Er * Er + 0.032874 * Er * Er * Er;
    double dEr;
    if (k < N) dEr = q.dE(k, ph) * s1 / s2 + rho * (v.vc53[k] * s2 - v.vc23[k] * s1) / (s2 * s2);
    else dEr = q.dE(N, ph) * s1 / s2;
    const double dAA = 0.096016 * dEr - 0.4407 * Er * dEr + 0.098622 * Er * Er * dEr;
    const double roRD = AA / rho;
    const double dRho = q.dE(k < N ? k : N, ph);
    double a1 = 0, a2 = 0;
    for (int j = 0; j < N; j++) {
        if (j == i) continue;
        const double pDij = v.pD[j * N + i];
        const double Dij = pDij * roRD;
        if (k < N && k != i && j == k) a1 += 1.0 / (pDij * roRD);
        const double dD = pDij * (dAA * rho - dRho * AA) / (rho * rho);
        a1 += q.w(ph, j) * (-dD / (Dij * Dij));
        a2 += q.w(ph, j) / Dij;
    }
    if (AA < 0 || a2 == 0) return 0;
    if (k == i) return -(a2 + a1 * (1 - q.w(ph, i))) / (a2 * a2);
    return -a1 * (1 - q.w(ph, i)) / (a2 * a2);
}

// ---------------------------------------------------------------------------
// Output
// ---------------------------------------------------------------------------
struct BlockRow {
    const JacView *v;
    long b;
    OSR_HD void add(int slot, int r, int col, double val) const {
        const int bs = v->bs;
        v->vals[(((long)b * 8 + slot) * bs + r) * bs + col] += val;
    }
    // an entry at an arbitrary global column (kept in the overflow list)
    OSR_HD void add_global(int r, long col, double val) const {
        int k = v->ovf_n[b];
        if (k < kOverflow) {
            v->ovf_row[b * kOverflow + k] = r;
            v->ovf_col[b * kOverflow + k] = col;
            v->ovf_val[b * kOverflow + k] = val;
            v->ovf_n[b] = k + 1;
        }
    }
};

// One face of a cell for the Jacobian: neighbour, the cell holding the face's
// transmissibilities (tc), direction and sign, the two block sizes along the
// direction and twice the cross-section.
struct JFace {
    long nb, tc;
    int d, sgn, slot;
    double dl, dn, area2;
};

OSR_HD inline int jac_faces(const JacView &v, long c, JFace *f) {
    const int ix = (int)(c % v.nx), iy = (int)((c / v.nx) % v.ny), iz = (int)(c / ((long)v.nx * v.ny));
    const long sx = 1, sy = v.nx, sz = (long)v.nx * v.ny;
    int k = 0;
    if (ix < v.nx - 1) f[k++] = JFace{c + sx, c, 0, 1, 2, v.di[ix], v.di[ix + 1], 2 * v.dj[iy] * v.dk[iz]};
    if (ix > 0) f[k++] = JFace{c - sx, c - sx, 0, -1, 1, v.di[ix], v.di[ix - 1], 2 * v.dj[iy] * v.dk[iz]};
    if (iy < v.ny - 1) f[k++] = JFace{c + sy, c, 1, 1, 4, v.dj[iy], v.dj[iy + 1], 2 * v.di[ix] * v.dk[iz]};
    if (iy > 0) f[k++] = JFace{c - sy, c - sy, 1, -1, 3, v.dj[iy], v.dj[iy - 1], 2 * v.di[ix] * v.dk[iz]};
    if (iz < v.nz - 1) f[k++] = JFace{c + sz, c, 2, 1, 6, v.dk[iz], v.dk[iz + 1], 2 * v.di[ix] * v.dj[iy]};
    if (iz > 0) f[k++] = JFace{c - sz, c - sz, 2, -1, 5, v.dk[iz], v.dk[iz - 1], 2 * v.di[ix] * v.dj[iy]};
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
    for (int t = 0; t < 12; t++) fd.T[t] = F.trans[(long)(t * 3 + e.d) * n + e.tc];
    for (int p = 0; p < 3; p++) fd.ts[p] = F.transS[(long)(p * 3 + e.d) * n + e.tc];
    fd.ift = F.iftran[(long)e.d * n + e.tc];
    for (int p = 0; p < 3; p++) fd.dP[p] = e.sgn > 0 ? F.P[p * n + e.nb] - F.P[p * n + c] : F.P[p * n + c] - F.P[p * n + e.nb];
    fd.dH = e.sgn > 0 ? v.blockH[e.nb] - v.blockH[c] : v.blockH[c] - v.blockH[e.nb];
    return fd;
}

// upstream cell of phase p (0 oil, 1 gas, 2 water) across the face
OSR_HD inline long upstream(const JFace &e, const FaceData &fd, long c, int p) {
    if (e.sgn > 0) return fd.ts[p] ? e.nb : c;
    return fd.ts[p] ? c : e.nb;
}

// Columns of a cell's own unknowns by phase state (the reference's reCol /
// reCol3 offsets): a one-phase cell has no column for the absent phase's
// composition and saturation, and an oil-only or gas-only cell emits its own
// saturation derivatives only for the phases it carries.
struct OwnLayout {
    int P, Sw, So, Sg, X, Y;
    bool swso, sg, x, y;
};

OSR_HD inline OwnLayout own_layout(int N, int lab) {
    if (lab == 0) return OwnLayout{2 * N, 2 * N + 1, 2 * N + 2, 2 * N + 3, 0, N, true, true, true, true};
    if (lab == 1) return OwnLayout{N, N + 1, N + 2, -1, 0, -1, true, false, true, false};
    return OwnLayout{N, N + 1, -1, N + 2, -1, 0, false, true, false, true};
}

// Mobility-ratio derivative factors of one phase across a face: the
// derivatives of (rho_c dl + rho_n dn C) / (mu_c dl + mu_n dn C) and of the
// face-averaged gravity with respect to a variable of this cell (M, MG) and
// of the neighbour (B, BG).  k = N: pressure; k < N: component k.
struct Mob {
    double Sur, Mak, M, B, MG, BG, tempdx;
};

OSR_HD inline Mob mobility(const Cell &q, const Cell &nb, const JFace &e, int ph, int k, double coef, double dmu_c,
                           double dmu_n, bool coef_in_bg) {
    const int N = q.v->nc;
    Mob m;
    m.Sur = q.rho(ph) * e.dl + nb.rho(ph) * e.dn * coef;
    m.Mak = q.mu(ph) * e.dl + nb.mu(ph) * e.dn * coef;
    m.M = (q.dE(k, ph) * e.dl * m.Mak - dmu_c * e.dl * m.Sur) / (m.Mak * m.Mak);
    m.B = (nb.dE(k, ph) * e.dn * coef * m.Mak - dmu_n * e.dn * coef * m.Sur) / (m.Mak * m.Mak);
    const double gk_c = k < N ? kGAccG * q.rho(ph) * q.v->mw[k] : 0.0;
    const double gk_n = k < N ? kGAccG * nb.rho(ph) * q.v->mw[k] : 0.0;
    m.MG = e.dl * (gk_c + q.gam(ph) * q.dE(k, ph) / q.rho(ph)) / (e.dl + e.dn * coef);
    m.BG = (coef_in_bg ? coef : 1.0) * e.dn * (gk_n + nb.gam(ph) * nb.dE(k, ph) / nb.rho(ph)) / (e.dl + e.dn * coef);
    m.tempdx = (q.gam(ph) * e.dl + nb.gam(ph) * e.dn * coef) / (e.dl + e.dn * coef);
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
    const Cell M{&v, &v.m[0], c}, F{&v, &v.m[1], c};
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
    const double di = v.di[ix], dj = v.dj[iy], dk = v.dk[iz];
    t.Vb = di * dj * dk;
    t.SF2 = 4 * v.sigma * (M.F->perm[c] / (di * di) + M.F->perm[v.n + c] / (dj * dj) + M.F->perm[2 * v.n + c] / (dk * dk));
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

// Direction-dependent deviations of the reference's face blocks.
struct FaceQuirks {
    bool gas_dB_assign_up;     // - faces, gas upstream = this cell: dB = ... instead of dB -= ...
    bool gas_dB_assign_down;   // - faces, gas upstream = neighbour
    bool ift_y_in_diag_grav;   // +z face, k == i, oil upstream = neighbour: y-face transmissibility
    bool gas_coef_any_1ph;     // k != i, gas: neighbour weight zero for any one-phase neighbour
    bool oil_grav_assign_down; // - faces, oil upstream = neighbour: gravity term assigned to dB
    bool shifted_block;        // neighbour P / S columns counted from the block after the neighbour's
    bool matrix_kr_offdiag_up; // k != i, oil upstream = this cell: the matrix relative permeability
};

OSR_HD inline FaceQuirks matrix_total_quirks(const JFace &e) {
    FaceQuirks q{false, false, false, false, false, false, false};
    if (e.sgn < 0 && e.d == 1) { q.gas_dB_assign_down = true; q.oil_grav_assign_down = true; q.shifted_block = true; }
    if (e.sgn < 0 && e.d == 2) q.shifted_block = true;
    return q;
}

OSR_HD inline FaceQuirks fracture_comp_quirks(const JFace &e);

OSR_HD inline FaceQuirks matrix_comp_quirks(const JFace &e) {
    FaceQuirks q{false, false, false, false, false, false, false};
    if (e.sgn < 0 && e.d == 0) { q.gas_dB_assign_up = true; q.gas_dB_assign_down = true; q.gas_coef_any_1ph = true; }
    if (e.sgn > 0 && e.d == 2) q.ift_y_in_diag_grav = true;
    return q;
}


// ---------------------------------------------------------------------------
// Component balance rows of a cell (matrix continuum).
// ---------------------------------------------------------------------------

OSR_HD inline FaceQuirks fracture_comp_quirks(const JFace &e) {
    return matrix_comp_quirks(e);
}

// Derivatives of row i's face terms with respect to the neighbour's pressure
// and saturations (emitted) and this cell's pressure and saturations
// (accumulated): the first face block of the reference's component rows.
struct OwnPS {
    double dp, dSw, dSo, dSg;
};

OSR_HD inline void comp_face_ps(const JacView &v, const Cell &q, int i, const JFace &e, const FaceQuirks &qk,
                                const BlockRow &out, int row, OwnPS &acc, bool fracture, bool total = false) {
    const int N = v.nc;
    const JMed &F = *q.F;
    const Cell nb{&v, &F, e.nb};
    const FaceData fd = face_data(v, F, q.c, e);
    const double s = e.sgn;
    const int lnb = nb.label();
    const int nbase = lnb ? -N : 0, reCol4 = lnb ? 1 : 0;
    const long upo = upstream(e, fd, q.c, 0), upg = upstream(e, fd, q.c, 1);
    const bool nb_o = upo == e.nb, nb_g = upg == e.nb;
    const Cell Uo{&v, &F, upo}, Ug{&v, &F, upg};
    const double xo = total ? 1.0 : Uo.w(0, i), yg = total ? 1.0 : Ug.w(1, i);
    // the emitted neighbour columns; the reference counts some from the next block's offset
    auto put = [&](int col, double val) {
        if (qk.shifted_block) out.add_global(row, v.rowoff[(e.nb + (q.F == &v.m[1] ? v.n : 0)) + 1] + col, val);
        else out.add(e.slot, row, col, val);
    };
    // saturation factors
    const double dsw = s * (xo * fd.T[4] * fd.dP[1] + xo * fd.T[6] * fd.dH);
    if (nb_o) put(nbase + 2 * N + 1, dsw);
    else acc.dSw += dsw;
    const double dso = s * (xo * fd.T[10] * fd.dP[1] + xo * fd.T[11] * fd.dH);
    if (nb_o) put(nbase + 2 * N + 2, lnb == -1 ? 0.0 : dso);
    else acc.dSo += dso;
    const double dsgo = s * (xo * fd.T[8] * fd.dP[1] + xo * fd.T[9] * fd.dH);
    const double dsgg = s * (yg * fd.T[5] * fd.dP[2] + yg * fd.T[7] * fd.dH);
    double vsg = 0;
    if (nb_o) vsg = lnb == 1 ? 0.0 : dsgo;
    else acc.dSg += dsgo;
    if (nb_g) vsg += lnb == 1 ? 0.0 : dsgg;
    else acc.dSg += dsgg;
    put(nbase + 2 * N + 3 - reCol4, vsg);
    // mobility and diffusion derivatives with respect to the two pressures
    const double tor_c = fracture ? 1.0 : v.tor[q.c], tor_n = fracture ? 1.0 : v.tor[e.nb];
    const double pm = q.porpor(), dpm = q.dpordp();
    const double pn = nb.porpor(), dpn = nb.dpordp();
    const double NNd = e.area2 / (e.dn + e.dl);
    double dB = 0;
    for (int ph = 0; ph < 2; ph++) {
        const double coef = ph == 0 ? (lnb == -1 ? 0.0 : 1.0) : (lnb == 1 ? 0.0 : 1.0);
        const double dC = ph == 0 ? (q.label() == -1 ? 0.0 : 1.0) : (q.label() == 1 ? 0.0 : 1.0);
        const Mob m = mobility(q, nb, e, ph, N, coef, visc_deriv(q, N, ph), visc_deriv(nb, N, ph), true);
        const bool up_nb = ph == 0 ? nb_o : nb_g;
        const Cell &U = up_nb ? nb : q;
        const double wk = total ? 1.0 : U.w(ph, i), krk = U.kr(1 + ph);
        const double dPp = fd.dP[1 + ph];
        const double a = wk * fd.ift * krk;
        acc.dp -= s * (a * m.M * dPp);
        double vB = s * (a * m.B * dPp);
        if (ph == 1 && e.sgn < 0) {
            const bool assign = up_nb ? qk.gas_dB_assign_down : qk.gas_dB_assign_up;
            dB = assign ? vB : dB + vB;
            // the reference exchanges this cell's and the neighbour's gravity factors here
            acc.dp -= s * (a * (m.B * m.tempdx + m.BG * m.Sur / m.Mak) * fd.dH);
            dB += s * (a * (m.M * m.tempdx + m.MG * m.Sur / m.Mak) * fd.dH);
        } else {
            dB = ph == 0 ? vB : dB + vB;
            acc.dp -= s * (a * (m.M * m.tempdx + m.MG * m.Sur / m.Mak) * fd.dH);
            const double gB = s * (a * (m.B * m.tempdx + m.BG * m.Sur / m.Mak) * fd.dH);
            if (ph == 0 && e.sgn < 0 && up_nb && qk.oil_grav_assign_down) dB = gB;
            else dB += gB;
        }
        if (total) continue;
        // intra-continuum diffusion
        double Dup, dDdp, dDdp2;
        if (nb.w(ph, i) > q.w(ph, i)) {
            Dup = nb.D(i, ph);
            dDdp = 0;
            dDdp2 = diff_deriv(nb, i, N, ph);
        } else {
            Dup = q.D(i, ph);
            dDdp = diff_deriv(q, i, N, ph);
            dDdp2 = 0;
        }
        if (q.por() < 1e-10 || nb.por() < 1e-10) Dup = dDdp = dDdp2 = 0;
        double AAd = nb.rho(ph) * e.dn * coef + q.rho(ph) * e.dl * dC;
        AAd *= (nb.S(1 + ph) * e.dn * coef + q.S(1 + ph) * e.dl * dC) / (e.dn + e.dl);
        const double BBd = tor_n * e.dn * coef / pn + tor_c * e.dl * dC / pm;
        const double MMd = AAd / BBd;
        const double DX = nb.w(ph, i) - q.w(ph, i);
        const double dAA = q.dE(N, ph) * e.dl * dC, dAA2 = nb.dE(N, ph) * e.dn * coef;
        const double dBB = -dpm * tor_c * e.dl * dC / (pm * pm), dBB2 = -dpn * tor_n * e.dn * coef / (pn * pn);
        const double dMM = (dAA * BBd - dBB * AAd) / (BBd * BBd), dMM2 = (dAA2 * BBd - dBB2 * AAd) / (BBd * BBd);
        if (coef != 0 && dC != 0) {
            acc.dp += -NNd * DX * (MMd * dDdp + Dup * dMM);
            dB += NNd * DX * (MMd * dDdp2 + Dup * dMM2);
        }
    }
    put(nbase + 2 * N, v.pcoeff * (-xo * fd.T[0] - yg * fd.T[1] - dB));
}

// Derivatives of row i's face terms with respect to component k of both
// cells (the second and third face blocks: k == i and k != i).
OSR_HD inline void comp_face_x(const JacView &v, const Cell &q, int i, int k, const JFace &e, const FaceQuirks &qk,
                               const BlockRow &out, int row, double &dRxl, double &dRxg, bool fracture,
                               bool total = false) {
    const int N = v.nc;
    const JMed &F = *q.F;
    const Cell nb{&v, &F, e.nb};
    const FaceData fd = face_data(v, F, q.c, e);
    const double s = e.sgn;
    const bool diag = !total && k == i;
    const int lnb = nb.label();
    const double tor_c = fracture ? 1.0 : v.tor[q.c], tor_n = fracture ? 1.0 : v.tor[e.nb];
    const double pm = q.porpor(), pn = nb.porpor();
    const double NNd = e.area2 / (e.dn + e.dl);
    for (int ph = 0; ph < 2; ph++) {
        double coef;
        if (ph == 0) coef = lnb == -1 ? 0.0 : 1.0;
        else if (!diag && qk.gas_coef_any_1ph) coef = lnb != 0 ? 0.0 : 1.0;
        else coef = lnb == 1 ? 0.0 : 1.0;
        const double dC = ph == 0 ? (q.label() == -1 ? 0.0 : 1.0) : (q.label() == 1 ? 0.0 : 1.0);
        const Mob m = mobility(q, nb, e, ph, k, coef, visc_deriv(q, k, ph), visc_deriv(nb, k, ph), true);
        const bool up_nb = upstream(e, fd, q.c, ph) == e.nb;
        const double Tp = diag ? fd.T[ph] : 0.0, Tg = diag ? fd.T[2 + ph] : 0.0;
        const double dPp = fd.dP[1 + ph];
        double dR = 0, dB;
        const double wc = total ? 1.0 : q.w(ph, i), wn = total ? 1.0 : nb.w(ph, i);
        const double krc = (ph == 0 && !diag && !total && qk.matrix_kr_offdiag_up) ? v.m[0].kr[v.n + q.c] : q.kr(1 + ph);
        const double ac = wc * fd.ift * krc, an = wn * fd.ift * nb.kr(1 + ph);
        const double gM = m.M * m.tempdx + m.MG * m.Sur / m.Mak, gB = m.B * m.tempdx + m.BG * m.Sur / m.Mak;
        if (up_nb) {
            dR += s * (an * m.M * dPp);
            dB = s * ((Tp + an * m.B) * dPp);
        } else {
            dR += s * ((Tp + ac * m.M) * dPp);
            dB = s * (ac * m.B * dPp);
        }
        // gravity (nonzero across z faces only)
        if (e.sgn > 0) {
            if (up_nb) {
                const double ift_r = (diag && ph == 0 && qk.ift_y_in_diag_grav)
                                         ? F.iftran[v.n + q.c] : fd.ift;
                dR += wn * ift_r * nb.kr(1 + ph) * gM * fd.dH;
                dB += (Tg + an * gB) * fd.dH;
            } else {
                dR += (Tg + ac * gM) * fd.dH;
                dB += ac * gB * fd.dH;
            }
        } else {
            // - faces: the gas terms exchange the two cells' factors; with k != i
            // the oil terms of a downstream cell change sign
            const double g1 = ph == 1 ? gB : gM, g2 = ph == 1 ? gM : gB;
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
        double Dup = 0, dDdx = 0, dDdx2 = 0;
        if (total) {
        } else if (wn > wc) {
            Dup = nb.D(i, ph);
            dDdx = 0;
            dDdx2 = diff_deriv(nb, i, k, ph);
        } else {
            Dup = q.D(i, ph);
            dDdx = diff_deriv(q, i, k, ph);
            dDdx2 = 0;
        }
        double AAd = nb.rho(ph) * e.dn * coef + q.rho(ph) * e.dl * dC;
        AAd *= (nb.S(1 + ph) * e.dn * coef + q.S(1 + ph) * e.dl * dC) / (e.dn + e.dl);
        const double BBd = tor_n * e.dn * coef / pn + tor_c * e.dl * dC / pm;
        const double MMd = AAd / BBd;
        const double DX = wn - wc;
        const double dMM = q.dE(k, ph) * e.dl * dC / BBd, dMM2 = nb.dE(k, ph) * e.dn * coef / BBd;
        if (!total && coef != 0 && dC != 0) {
            dR += s * NNd * ((diag ? -MMd * Dup : 0.0) + dDdx * MMd * DX + dMM * Dup * DX);
            dB += s * NNd * ((diag ? MMd * Dup : 0.0) + dDdx2 * MMd * DX + dMM2 * Dup * DX);
        }
        if (ph == 0) {
            dRxl += dR;
            out.add(e.slot, row, k, -dB * coef);
        } else {
            dRxg += dR;
            out.add(e.slot, row, (lnb ? -N : 0) + k + N, -dB * coef);
        }
    }
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
    w.Qw = v.well_q[3 * b];
    w.Qo = v.well_q[3 * b + 1];
    w.Qg = v.well_q[3 * b + 2];
    w.PIw = v.well_pi[3 * b];
    w.PIo = v.well_pi[3 * b + 1];
    w.PIg = v.well_pi[3 * b + 2];
    w.iwell = v.well_comp[b];
    if (w.iwell >= 0) w.gcomp = v.stream_y[w.iwell * kMaxNc + i];
    return w;
}

// Component balance row i (0 <= i < N-1) of a two-phase matrix cell.
OSR_HD inline void matrix_comp_row_2ph(const JacView &v, long c, int i, const BlockRow &out, int row) {
    const int N = v.nc;
    const Cell M{&v, &v.m[0], c}, Fr{&v, &v.m[1], c};
    const Transfer t = transfer_terms(v, c);
    const double pm = t.pm, pf = t.pf, dpm = t.dpm, dpf = t.dpf;
    const double Vb = t.Vb, SF1 = t.SF1, SF2 = t.SF2;
    const double tor = v.tor[c];
    const int lm = M.label(), lf = Fr.label();
    const double xi = M.w(0, i), yi = M.w(1, i);
    const double ro = M.rho(0), rg = M.rho(1);
    const double mubar_o = t.Do / (pm + pf), mubar_g = t.Dg / (pm + pf);
    const double dLdp = (Vb / v.dt) * (xi * M.S(1) * (ro * dpm + M.dE(N, 0) * pm) + yi * M.S(2) * (rg * dpm + M.dE(N, 1) * pm));
    const double dLdSo = (Vb / v.dt) * (xi * pm * ro), dLdSg = (Vb / v.dt) * (yi * pm * rg);
    double dRfdp = 0;
    OwnPS a{0, 0, 0, 0};
    // transfer, this cell's pressure
    a.dp += kSIC * M.dE(N, 0) * xi * SF2 * Vb * t.kro / mubar_o * t.dPo;
    a.dp += -kSIC * xi * ro * SF2 * Vb * t.kro / mubar_o;
    a.dp += -kSIC * (visc_deriv(M, N, 0) * pm + dpm * M.mu(0)) * xi * ro * SF2 * Vb * t.kro / (t.Do * t.Do) * t.dPo * (pm + pf);
    a.dp += kSIC * dpm * xi * ro * SF2 * Vb * t.kro / t.Do * t.dPo;
    a.dp += kSIC * M.dE(N, 1) * yi * SF2 * Vb * t.krg / mubar_g * t.dPg;
    a.dp += -kSIC * yi * rg * SF2 * Vb * t.krg / mubar_g;
    a.dp += -kSIC * (visc_deriv(M, N, 1) * pm + dpm * M.mu(1)) * yi * rg * SF2 * Vb * t.krg / (t.Dg * t.Dg) * t.dPg * (pm + pf);
    a.dp += kSIC * dpm * yi * rg * SF2 * Vb * t.krg / t.Dg * t.dPg;
    // diffusive transfer, this cell's pressure
    for (int ph = 0; ph < 2; ph++) {
        int kinds[2];
        const int nt = matrix_diff_targets(lm, lf, ph, kinds);
        const double sat = M.S(1 + ph), rho = M.rho(ph), D = M.D(i, ph), w = M.w(ph, i);
        const double dDdp = diff_deriv(M, i, N, ph);
        for (int j = 0; j < nt; j++) {
            const double tgt = kinds[j] ? Fr.w(ph, i) : 0.0;
            a.dp += dpm * SF1 * sat * Vb / tor * rho * D * (tgt - w);
            a.dp += M.dE(N, ph) * SF1 * sat * pm * Vb / tor * D * (tgt - w);
            a.dp += dDdp * SF1 * sat * pm * Vb / tor * rho * (tgt - w);
        }
    }
    // transfer, the fracture's pressure
    dRfdp += kSIC * xi * ro * SF2 * Vb * t.kro / mubar_o;
    dRfdp += -kSIC * (visc_deriv(Fr, N, 0) * pf + dpf * Fr.mu(0)) * xi * ro * SF2 * Vb * t.kro / (t.Do * t.Do) * t.dPo * (pm + pf);
    dRfdp += kSIC * dpf * xi * ro * SF2 * Vb * t.kro / t.Do * t.dPo;
    dRfdp += kSIC * yi * rg * SF2 * Vb * t.krg / mubar_g;
    dRfdp += -kSIC * (visc_deriv(Fr, N, 1) * pf + dpf * Fr.mu(1)) * yi * rg * SF2 * Vb * t.krg / (t.Dg * t.Dg) * t.dPg * (pm + pf);
    dRfdp += kSIC * dpf * yi * rg * SF2 * Vb * t.krg / t.Dg * t.dPg;
    // advective flux, this cell's pressure
    JFace fc[6];
    const int nf = jac_faces(v, c, fc);
    for (int ph = 0; ph < 2; ph++)
        for (int q = 0; q < nf; q++) {
            const FaceData fd = face_data(v, v.m[0], c, fc[q]);
            const Cell U{&v, &v.m[0], upstream(fc[q], fd, c, ph)};
            a.dp += U.w(ph, i) * fd.T[ph];
        }
    // saturations (transfer and diffusive transfer)
    double dRfdSw = 0, dRfdSo = 0, dRfdSg = 0;
    const double po = xi * ro * SF2 * Vb / mubar_o * t.dPo, pg = yi * rg * SF2 * Vb / mubar_g * t.dPg;
    a.dSo += kSIC * t.dkm[4] * po;
    {
        int kinds[2];
        const int nt = matrix_diff_targets(lm, lf, 0, kinds);
        for (int j = 0; j < nt; j++) {
            const double tgt = kinds[j] ? Fr.w(0, i) : 0.0;
            a.dSo += SF1 * Vb * pm / tor * ro * M.D(i, 0) * (tgt - xi);
        }
    }
    dRfdSo += kSIC * t.dkf[4] * po;
    a.dSg += kSIC * t.dkm[2] * po;
    a.dSg += kSIC * t.dkm[3] * pg;
    {
        // the gas saturation derivative omits the two-phase matrix / oil fracture pairing
        int kinds[2];
        int nt = matrix_diff_targets(lm, lf, 1, kinds);
        if (lm == 0 && lf == 1) nt = 0;
        for (int j = 0; j < nt; j++) {
            const double tgt = kinds[j] ? Fr.w(1, i) : 0.0;
            a.dSg += SF1 * Vb * pm / tor * rg * M.D(i, 1) * (tgt - yi);
        }
    }
    dRfdSg += kSIC * t.dkf[2] * po;
    dRfdSg += kSIC * t.dkf[3] * pg;
    a.dSw += kSIC * t.dkm[1] * po;
    dRfdSw += kSIC * t.dkf[1] * po;
    // faces: neighbour pressures and saturations
    for (int q = 0; q < nf; q++) comp_face_ps(v, M, i, fc[q], matrix_comp_quirks(fc[q]), out, row, a, false);
    // this cell's pressure and saturations (with the completion's productivity terms)
    const WellAt W = well_at(v, 0, c, i, yi);
    const OwnLayout L = own_layout(N, lm);
    out.add(0, row, L.P, v.pcoeff * (dLdp + a.dp + xi * W.PIo + W.gcomp * W.PIg));
    if (L.swso) {
        out.add(0, row, L.Sw, -a.dSw);
        out.add(0, row, L.So, dLdSo - a.dSo);
    }
    if (L.sg) out.add(0, row, L.Sg, dLdSg - a.dSg);
    // the fracture's pressure and saturations
    const int rf = lf ? N : 0;
    if (lf == 1) out.add(7, row, 2 * N + 2 - rf, dRfdSo);
    else if (lf == -1) out.add(7, row, 2 * N + 2 - rf, dRfdSg);
    else {
        out.add(7, row, 2 * N + 2, dRfdSo);
        out.add(7, row, 2 * N + 3, dRfdSg);
    }
    out.add(7, row, 2 * N - rf, v.pcoeff * dRfdp);
    out.add(7, row, 2 * N + 1 - rf, dRfdSw);
    // compositions
    for (int k = 0; k < N; k++) {
        double dRxl = 0, dRxg = 0, dRfxl = 0, dRfxg = 0;
        const bool diag = k == i;
        for (int ph = 0; ph < 2; ph++) {
            const double w = M.w(ph, i), rho = M.rho(ph), kr = ph ? t.krg : t.kro, mub = ph ? mubar_g : mubar_o;
            const double Dd = ph ? t.Dg : t.Do, dPp = ph ? t.dPg : t.dPo;
            double &dR = ph ? dRxg : dRxl;
            double &dRf = ph ? dRfxg : dRfxl;
            if (diag) dR += kSIC * rho * SF2 * Vb * kr / mub * dPp;
            dR += kSIC * M.dE(k, ph) * w * SF2 * Vb * kr / mub * dPp;
            dR += -kSIC * visc_deriv(M, k, ph) * w * rho * SF2 * Vb * kr * pm / (Dd * Dd) * dPp * (pm + pf);
            int kinds[2];
            const int nt = matrix_diff_targets(lm, lf, ph, kinds);
            const double sat = M.S(1 + ph), D = M.D(i, ph), dDdx = diff_deriv(M, i, k, ph);
            for (int j = 0; j < nt; j++) {
                const double tgt = kinds[j] ? Fr.w(ph, i) : 0.0;
                dR += M.dE(k, ph) * SF1 * sat * pm * Vb / tor * D * (tgt - w);
                if (diag) dR += -SF1 * sat * pm * Vb / tor * rho * D;
                dR += dDdx * SF1 * sat * pm * Vb / tor * rho * (tgt - w);
            }
            dRf += -kSIC * visc_deriv(Fr, k, ph) * w * rho * SF2 * Vb * kr * pf / (Dd * Dd) * dPp * (pm + pf);
            if (diag) {
                // towards the fracture composition of the same phase
                bool on = (lm == 0 && lf == 0);
                if (ph == 0) on = on || (lm == 1 && lf == 1) || (lm == 0 && lf == 1) || (lm == 1 && lf == 0);
                else on = on || (lm == -1 && lf == -1) || (lm == 0 && lf == -1) || (lm == -1 && lf == 0);
                if (on) dRf += SF1 * sat * pm * Vb / tor * rho * D;
            }
        }
        const double dLxl = diag ? ro + xi * M.dE(k, 0) : xi * M.dE(k, 0);
        const double dLxg = diag ? rg + yi * M.dE(k, 1) : yi * M.dE(k, 1);
        const double dQxl = (diag && W.iwell < 0) ? W.Qo : 0.0, dQxg = (diag && W.iwell < 0) ? W.Qg : 0.0;
        for (int q = 0; q < nf; q++) comp_face_x(v, M, i, k, fc[q], matrix_comp_quirks(fc[q]), out, row, dRxl, dRxg, false);
        if (lf == 1) out.add(7, row, k, dRfxl);
        else if (lf == -1) out.add(7, row, k, dRfxg);
        else {
            out.add(7, row, k, dRfxl);
            out.add(7, row, N + k, dRfxg);
        }
        if (L.x) out.add(0, row, L.X + k, (Vb / v.dt) * pm * M.S(1) * dLxl - dQxl - dRxl);
        if (L.y) out.add(0, row, L.Y + k, (Vb / v.dt) * pm * M.S(2) * dLxg - dQxg - dRxg);
    }
}

// Fugacity rows of a two-phase cell (compsim/Petsc_Functions.cpp:30240-30406
// for the matrix): x_i P_o phi_i^L - y_i P_g phi_i^V with Z from the stored
// density and dZ from dE.
OSR_HD inline void fugacity_rows(const JacView &v, const Cell &q, const BlockRow &out) {
    const int N = v.nc;
    const double RT = kR * v.T;
    const double Pl = q.P(1), Pg = q.P(2);
    double Al = 0, Bl = 0, Ag = 0, Bg = 0;
    for (int i = 0; i < N; i++) {
        Bl += q.w(0, i) * v.b[i];
        Bg += q.w(1, i) * v.b[i];
        for (int j = 0; j < N; j++) {
            const double t = v.sa[i] * v.sa[j] * v.bic[i * N + j];
            Al += q.w(0, i) * q.w(0, j) * t;
            Ag += q.w(1, i) * q.w(1, j) * t;
        }
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
    for (int i = 0; i < N; i++) {
        double tl = 0, tg = 0;
        for (int j = 0; j < N; j++) {
            const double t = v.sa[i] * v.sa[j] * v.bic[i * N + j];
            tl += q.w(0, j) * t;
            tg += q.w(1, j) * t;
        }
        const double t1l = v.b[i] / Cbl, t1g = v.b[i] / Cbg;
        const double EEl = 2 * tl / Cal - t1l, EEg = 2 * tg / Cag - t1g;
        const double DDl = Al / (Bl * (d1 - d2)), DDg = Ag / (Bg * (d1 - d2));
        const double FFl = log((Zl + d2 * Bl) / (Zl + d1 * Bl)), FFg = log((Zg + d2 * Bg) / (Zg + d1 * Bg));
        const double phiL = exp(t1l * (Zl - 1) - log(Zl - Bl) + DDl * EEl * FFl);
        const double phiG = exp(t1g * (Zg - 1) - log(Zg - Bg) + DDg * EEg * FFg);
        const double dAAl = v.b[i] * dZdpl / Cbl, dAAg = v.b[i] * dZdpg / Cbg;
        const double dBBl = (dBdpl - dZdpl) / (Zl - Bl), dBBg = (dBdpg - dZdpg) / (Zg - Bg);
        const double dDDl = (Bl * dAdpl - Al * dBdpl) / (Bl * Bl * (d1 - d2)), dDDg = (Bg * dAdpg - Ag * dBdpg) / (Bg * Bg * (d1 - d2));
        const double dFFl = (dZdpl + d2 * dBdpl) / (Zl + d2 * Bl) - (dZdpl + d1 * dBdpl) / (Zl + d1 * Bl);
        const double dFFg = (dZdpg + d2 * dBdpg) / (Zg + d2 * Bg) - (dZdpg + d1 * dBdpg) / (Zg + d1 * Bg);
        const double dPhil = phiL * (dAAl + dBBl + EEl * (dDDl * FFl + DDl * dFFl));
        const double dPhig = phiG * (dAAg + dBBg + EEg * (dDDg * FFg + DDg * dFFg));
        const double xi = q.w(0, i), yi = q.w(1, i);
        out.add(0, i, 2 * N, v.pcoeff * (xi * (phiL + Pl * dPhil) - yi * (phiG + Pg * dPhig)));
        for (int k = 0; k < N; k++) {
            double dAl = 0, dAg = 0;
            for (int n = 0; n < N; n++) {
                const double t = v.sa[k] * v.sa[n] * v.bic[k * N + n];
                dAl += q.w(0, n) * t;
                dAg += q.w(1, n) * t;
            }
            dAl *= 2 * Pl / (RT * RT);
            dAg *= 2 * Pg / (RT * RT);
            const double dBl = v.b[k] * Pl / RT, dBg = v.b[k] * Pg / RT;
            const double dZl = -q.dE(k, 0) * RT * Zl * Zl / Pl, dZg = -q.dE(k, 1) * RT * Zg * Zg / Pg;
            const double dAAxl = -v.b[k] * v.b[i] * (Zl - 1) / (Cbl * Cbl) + v.b[i] * dZl / Cbl;
            const double dAAxg = -v.b[k] * v.b[i] * (Zg - 1) / (Cbg * Cbg) + v.b[i] * dZg / Cbg;
            const double dBBxl = (dBl - dZl) / (Zl - Bl), dBBxg = (dBg - dZg) / (Zg - Bg);
            const double dDDxl = (dAl * Bl - dBl * Al) / (Bl * Bl * (d1 - d2)), dDDxg = (dAg * Bg - dBg * Ag) / (Bg * Bg * (d1 - d2));
            const double dFFxl = (dZl + d2 * dBl) / (Zl + d2 * Bl) - (dZl + d1 * dBl) / (Zl + d1 * Bl);
            const double dFFxg = (dZg + d2 * dBg) / (Zg + d2 * Bg) - (dZg + d1 * dBg) / (Zg + d1 * Bg);
            const double tik = v.sa[i] * v.sa[k] * v.bic[i * N + k];
            const double dEEl = 2 * (tik / Cal - dAl * RT * RT * tl / (Pl * Cal * Cal)) + v.b[i] * v.b[k] / (Cbl * Cbl);
            const double dEEg = 2 * (tik / Cag - dAg * RT * RT * tg / (Pg * Cag * Cag)) + v.b[i] * v.b[k] / (Cbg * Cbg);
            const double dPxl = phiL * (dAAxl + dBBxl + dDDxl * EEl * FFl + DDl * dEEl * FFl + DDl * EEl * dFFxl);
            const double dPxg = phiG * (dAAxg + dBBxg + dDDxg * EEg * FFg + DDg * dEEg * FFg + DDg * EEg * dFFxg);
            if (i == k) {
                out.add(0, i, k, Pl * phiL + Pl * xi * dPxl);
                out.add(0, i, N + k, -(Pg * phiG + Pg * yi * dPxg));
            } else {
                out.add(0, i, k, Pl * xi * dPxl);
                out.add(0, i, N + k, -Pg * yi * dPxg);
            }
        }
    }
}

// Rows sum x - 1, sum y - 1, sum S - 1 of a two-phase cell.
OSR_HD inline void constraint_rows_2ph(const JacView &v, const BlockRow &out) {
    const int N = v.nc;
    for (int k = 0; k < N; k++) {
        out.add(0, 2 * N + 1, k, 1.0);
        out.add(0, 2 * N + 2, N + k, 1.0);
    }
    for (int j = 0; j < 3; j++) out.add(0, 2 * N + 3, 2 * N + 1 + j, 1.0);
}


// Total hydrocarbon row (2N-1) of a two-phase cell.  The matrix-fracture
// transfer derivatives are formed from the matrix side; a fracture row takes
// them negated with the roles of the two continua exchanged.
OSR_HD inline void total_row_2ph(const JacView &v, int med, long c, const BlockRow &out, int row) {
    const int N = v.nc;
    const Cell M{&v, &v.m[0], c}, Fr{&v, &v.m[1], c};
    const Cell &O = med ? Fr : M;          // this row's continuum
    const Transfer t = transfer_terms(v, c);
    const double pm = t.pm, pf = t.pf, dpm = t.dpm, dpf = t.dpf;
    const double Vb = t.Vb, SF2 = t.SF2;
    const double po_ = med ? pf : pm, dpo_ = med ? dpf : dpm;
    const int lo = (med ? M : Fr).label();   // the other continuum's label
    const double ro = M.rho(0), rg = M.rho(1);
    const double mubar_o = t.Do / (pm + pf), mubar_g = t.Dg / (pm + pf);
    const double dLdp = (Vb / v.dt) * (O.S(1) * (O.rho(0) * dpo_ + O.dE(N, 0) * po_) + O.S(2) * (O.rho(1) * dpo_ + O.dE(N, 1) * po_));
    const double dLdSo = (Vb / v.dt) * (po_ * O.rho(0)), dLdSg = (Vb / v.dt) * (po_ * O.rho(1));
    // matrix-side derivatives of the (matrix-row) transfer terms
    double tm = 0, tf = 0;
    tm += kSIC * M.dE(N, 0) * SF2 * Vb * t.kro / mubar_o * t.dPo;
    tm += -kSIC * ro * SF2 * Vb * t.kro / mubar_o;
    tm += -kSIC * (visc_deriv(M, N, 0) * pm + dpm * M.mu(0)) * ro * SF2 * Vb * t.kro / (t.Do * t.Do) * t.dPo * (pm + pf);
    tm += kSIC * dpm * ro * SF2 * Vb * t.kro / t.Do * t.dPo;
    tm += kSIC * M.dE(N, 1) * SF2 * Vb * t.krg / mubar_g * t.dPg;
    tm += -kSIC * rg * SF2 * Vb * t.krg / mubar_g;
    tm += -kSIC * (visc_deriv(M, N, 1) * pm + dpm * M.mu(1)) * rg * SF2 * Vb * t.krg / (t.Dg * t.Dg) * t.dPg * (pm + pf);
    tm += kSIC * dpm * rg * SF2 * Vb * t.krg / t.Dg * t.dPg;
    tf += kSIC * ro * SF2 * Vb * t.kro / mubar_o;
    tf += -kSIC * (visc_deriv(Fr, N, 0) * pf + dpf * Fr.mu(0)) * ro * SF2 * Vb * t.kro / (t.Do * t.Do) * t.dPo * (pm + pf);
    tf += kSIC * dpf * ro * SF2 * Vb * t.kro / t.Do * t.dPo;
    tf += kSIC * rg * SF2 * Vb * t.krg / mubar_g;
    tf += -kSIC * (visc_deriv(Fr, N, 1) * pf + dpf * Fr.mu(1)) * rg * SF2 * Vb * t.krg / (t.Dg * t.Dg) * t.dPg * (pm + pf);
    tf += kSIC * dpf * rg * SF2 * Vb * t.krg / t.Dg * t.dPg;
    const double sg = med ? -1.0 : 1.0;
    OwnPS a{0, 0, 0, 0};
    a.dp += sg * (med ? tf : tm);
    const double dROdp = sg * (med ? tm : tf);   // the other continuum's pressure
    JFace fc[6];
    const int nf = jac_faces(v, c, fc);
    for (int ph = 0; ph < 2; ph++)
        for (int q = 0; q < nf; q++) a.dp += face_data(v, v.m[med], c, fc[q]).T[ph];
    const double po = ro * SF2 * Vb / mubar_o * t.dPo, pg = rg * SF2 * Vb / mubar_g * t.dPg;
    const double smSo = kSIC * t.dkm[4] * po, sfSo = kSIC * t.dkf[4] * po;
    const double smSg = kSIC * t.dkm[2] * po + kSIC * t.dkm[3] * pg, sfSg = kSIC * t.dkf[2] * po + kSIC * t.dkf[3] * pg;
    const double smSw = kSIC * t.dkm[1] * po, sfSw = kSIC * t.dkf[1] * po;
    a.dSo += sg * (med ? sfSo : smSo);
    a.dSg += sg * (med ? sfSg : smSg);
    a.dSw += sg * (med ? sfSw : smSw);
    const double dROSo = sg * (med ? smSo : sfSo), dROSg = sg * (med ? smSg : sfSg), dROSw = sg * (med ? smSw : sfSw);
    for (int q = 0; q < nf; q++) comp_face_ps(v, O, 0, fc[q], matrix_total_quirks(fc[q]), out, row, a, med == 1, true);
    const WellAt W = well_at(v, med, c, 0, 0.0);
    const OwnLayout L = own_layout(N, O.label());
    out.add(0, row, L.P, v.pcoeff * (dLdp + a.dp + W.PIo + W.PIg));
    if (L.swso) {
        out.add(0, row, L.Sw, -a.dSw);
        out.add(0, row, L.So, dLdSo - a.dSo);
    }
    if (L.sg) out.add(0, row, L.Sg, dLdSg - a.dSg);
    const int rf = lo ? N : 0;
    if (lo == 1) out.add(7, row, 2 * N + 2 - rf, dROSo);
    else if (lo == -1) out.add(7, row, 2 * N + 2 - rf, dROSg);
    else {
        out.add(7, row, 2 * N + 2, dROSo);
        out.add(7, row, 2 * N + 3, dROSg);
    }
    out.add(7, row, 2 * N - rf, v.pcoeff * dROdp);
    out.add(7, row, 2 * N + 1 - rf, dROSw);
    for (int k = 0; k < N; k++) {
        double xm = 0, ym = 0;
        xm += kSIC * M.dE(k, 0) * SF2 * Vb * t.kro / mubar_o * t.dPo;
        xm += -kSIC * visc_deriv(M, k, 0) * ro * SF2 * Vb * t.kro * pm / (t.Do * t.Do) * t.dPo * (pm + pf);
        const double xf = -kSIC * visc_deriv(Fr, k, 0) * ro * SF2 * Vb * t.kro * pf / (t.Do * t.Do) * t.dPo * (pm + pf);
        ym += kSIC * M.dE(k, 1) * SF2 * Vb * t.krg / mubar_g * t.dPg;
        ym += -kSIC * visc_deriv(M, k, 1) * rg * SF2 * Vb * t.krg * pm / (t.Dg * t.Dg) * t.dPg * (pm + pf);
        const double yf = -kSIC * visc_deriv(Fr, k, 1) * rg * SF2 * Vb * t.krg * pf / (t.Dg * t.Dg) * t.dPg * (pm + pf);
        double dRxl = sg * (med ? xf : xm), dRxg = sg * (med ? yf : ym);
        const double dROxl = sg * (med ? xm : xf), dROxg = sg * (med ? ym : yf);
        const FaceQuirks none{false, false, false, false, false, false, false};
        for (int q = 0; q < nf; q++) comp_face_x(v, O, 0, k, fc[q], none, out, row, dRxl, dRxg, med == 1, true);
        if (L.x) out.add(0, row, L.X + k, (Vb / v.dt) * po_ * O.S(1) * O.dE(k, 0) - dRxl);
        if (L.y) out.add(0, row, L.Y + k, (Vb / v.dt) * po_ * O.S(2) * O.dE(k, 1) - dRxg);
        if (lo == 1) out.add(7, row, k, dROxl);
        else if (lo == -1) out.add(7, row, k, dROxg);
        else {
            out.add(7, row, k, dROxl);
            out.add(7, row, N + k, dROxg);
        }
    }
}

// Water row (2N) of a two-phase cell.
OSR_HD inline void water_row_2ph(const JacView &v, int med, long c, const BlockRow &out, int row) {
    const int N = v.nc;
    const Cell M{&v, &v.m[0], c}, Fr{&v, &v.m[1], c};
    const Cell &O = med ? Fr : M;
    const JMed &F = v.m[med];
    const Transfer t = transfer_terms(v, c);
    const double wr = v.wat_ro * kWatMRo;
    const double po_ = med ? t.pf : t.pm, dpo_ = med ? t.dpf : t.dpm;
    const double sg = med ? -1.0 : 1.0;
    const double dLdp = (t.Vb / v.dt) * wr * O.S(0) * dpo_;
    const double dLdSw = (t.Vb / v.dt) * (po_ * wr);
    const double tr = kSIC * v.wat_ro * kWatMRo * t.SF2 * t.krw / v.wat_mu * t.Vb;
    // both continua's water rows take -tr for their own pressure, +tr for the other's
    double dRdp = -tr;
    const double dROdp = tr;
    JFace fc[6];
    const int nf = jac_faces(v, c, fc);
    const long n = v.n;
    for (int q = 0; q < nf; q++) dRdp += F.wtran[(long)fc[q].d * n + fc[q].tc];
    const WellAt W = well_at(v, med, c, 0, 0.0);
    const OwnLayout L = own_layout(N, O.label());
    out.add(0, row, L.P, v.pcoeff * (dLdp + dRdp + W.PIw));
    const double smw = kSIC * kWatMRo * t.dkm[0] * v.wat_ro * t.SF2 / v.wat_mu * t.Vb * t.dPw;
    const double sfw = kSIC * kWatMRo * t.dkf[0] * v.wat_ro * t.SF2 / v.wat_mu * t.Vb * t.dPw;
    double dRdSw = sg * (med ? sfw : smw);
    const double dROSw = sg * (med ? smw : sfw);
    for (int q = 0; q < nf; q++) {
        const JFace &e = fc[q];
        const FaceData fd = face_data(v, F, c, e);
        const int lnb = F.label[e.nb];
        const int nbase = lnb ? -N : 0;
        const double Tw = F.wtran[(long)e.d * n + e.tc], dTw = F.dwtran[(long)e.d * n + e.tc];
        out.add(e.slot, row, nbase + 2 * N, v.pcoeff * (-Tw));
        const double dsw = e.sgn * (dTw * fd.dP[0] + kGAcc * v.wat_ro * dTw * fd.dH);
        if (upstream(e, fd, c, 2) == e.nb) out.add(e.slot, row, nbase + 2 * N + 1, dsw);
        else dRdSw += dsw;
    }
    out.add(0, row, L.P + 1, dLdSw - dRdSw);
    const int rf = (med ? M : Fr).label() ? N : 0;
    out.add(7, row, 2 * N - rf, v.pcoeff * dROdp);
    out.add(7, row, 2 * N + 1 - rf, dROSw);
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

// Component balance row i of a two-phase fracture cell (the fracture case of
// IteratorJacobian, compsim/Petsc_Functions.cpp:12756-18666).
OSR_HD inline void fracture_comp_row_2ph(const JacView &v, long c, int i, const BlockRow &out, int row) {
    const int N = v.nc;
    const Cell M{&v, &v.m[0], c}, Fr{&v, &v.m[1], c};
    const Transfer t = transfer_terms(v, c);
    const double pm = t.pm, pf = t.pf, dpm = t.dpm, dpf = t.dpf;
    const double Vb = t.Vb, SF1 = t.SF1, SF2 = t.SF2, SF3 = t.SF3;
    const double tor = v.tor[c];
    const int lm = M.label(), lf = Fr.label();
    const double xi = M.w(0, i), yi = M.w(1, i);         // matrix compositions (transfer terms)
    const double fxi = Fr.w(0, i), fyi = Fr.w(1, i);
    const double ro = M.rho(0), rg = M.rho(1);
    const double mubar_o = t.Do / (pf + pm), mubar_g = t.Dg / (pf + pm);
    const double dLdp = (Vb / v.dt) * (fxi * Fr.S(1) * (Fr.rho(0) * dpf + Fr.dE(N, 0) * pf) + fyi * Fr.S(2) * (Fr.rho(1) * dpf + Fr.dE(N, 1) * pf));
    const double dLdSo = (Vb / v.dt) * (fxi * pf * Fr.rho(0)), dLdSg = (Vb / v.dt) * (fyi * pf * Fr.rho(1));
    double dRMdp = 0;
    OwnPS a{0, 0, 0, 0};
    // transfer, the matrix pressure
    dRMdp -= kSIC * M.dE(N, 0) * xi * SF2 * Vb * t.kro / mubar_o * t.dPo;
    dRMdp -= -kSIC * xi * ro * SF2 * Vb * t.kro / mubar_o;
    dRMdp -= -kSIC * (visc_deriv(M, N, 0) * pm + dpm * M.mu(0)) * xi * ro * SF2 * Vb * t.kro / (t.Do * t.Do) * t.dPo * (pf + pm);
    dRMdp -= kSIC * dpm * xi * ro * SF2 * Vb * t.kro / t.Do * t.dPo;
    dRMdp -= kSIC * M.dE(N, 1) * yi * SF2 * Vb * t.krg / mubar_g * t.dPg;
    dRMdp -= -kSIC * yi * rg * SF2 * Vb * t.krg / mubar_g;
    dRMdp -= -kSIC * (visc_deriv(M, N, 1) * pm + dpm * M.mu(1)) * yi * rg * SF2 * Vb * t.krg / (t.Dg * t.Dg) * t.dPg * (pf + pm);
    dRMdp -= kSIC * dpm * yi * rg * SF2 * Vb * t.krg / t.Dg * t.dPg;
    for (int ph = 0; ph < 2; ph++) {
        if (!fsf1(lm, lf, ph)) continue;
        const double sat = M.S(1 + ph), rho = M.rho(ph), D = M.D(i, ph), dlt = Fr.w(ph, i) - M.w(ph, i);
        dRMdp -= dpm * SF1 * sat * Vb / tor * rho * D * dlt;
        dRMdp -= M.dE(N, ph) * SF1 * sat * pm * Vb / tor * D * dlt;
        dRMdp -= diff_deriv(M, i, N, ph) * SF1 * sat * pm * Vb / tor * rho * dlt;
    }
    // transfer, this (fracture) cell's pressure
    a.dp -= kSIC * xi * ro * SF2 * Vb * t.kro / mubar_o;
    a.dp -= -kSIC * (visc_deriv(Fr, N, 0) * pf + dpf * Fr.mu(0)) * xi * ro * SF2 * Vb * t.kro / (t.Do * t.Do) * t.dPo * (pf + pm);
    a.dp -= kSIC * dpf * xi * ro * SF2 * Vb * t.kro / t.Do * t.dPo;
    a.dp -= kSIC * yi * rg * SF2 * Vb * t.krg / mubar_g;
    a.dp -= -kSIC * (visc_deriv(Fr, N, 1) * pf + dpf * Fr.mu(1)) * yi * rg * SF2 * Vb * t.krg / (t.Dg * t.Dg) * t.dPg * (pf + pm);
    a.dp -= kSIC * dpf * yi * rg * SF2 * Vb * t.krg / t.Dg * t.dPg;
    for (int ph = 0; ph < 2; ph++) {
        if (!fsf3(lm, lf, ph)) continue;
        const double sat = Fr.S(1 + ph), rho = Fr.rho(ph), D = Fr.D(i, ph), w = Fr.w(ph, i);
        a.dp -= dpf * SF3 * sat * Vb / tor * rho * D * (w - 0.0);
        a.dp -= Fr.dE(N, ph) * SF3 * sat * pf * Vb / tor * D * (w - 0.0);
        a.dp -= diff_deriv(Fr, i, N, ph) * SF3 * sat * pf * Vb / tor * rho * (w - 0.0);
    }
    JFace fc[6];
    const int nf = jac_faces(v, c, fc);
    for (int ph = 0; ph < 2; ph++)
        for (int q = 0; q < nf; q++) {
            const FaceData fd = face_data(v, v.m[1], c, fc[q]);
            const Cell U{&v, &v.m[1], upstream(fc[q], fd, c, ph)};
            a.dp += U.w(ph, i) * fd.T[ph];
        }
    // saturations
    double dRMdSo = 0, dRMdSg = 0, dRMdSw = 0;
    const double po = xi * ro * SF2 * Vb / mubar_o * t.dPo, pg = yi * rg * SF2 * Vb / mubar_g * t.dPg;
    dRMdSo -= kSIC * t.dkm[4] * po;
    if (fsf1(lm, lf, 0)) dRMdSo -= SF1 * Vb * pm / tor * ro * M.D(i, 0) * (fxi - xi);
    a.dSo -= kSIC * t.dkf[4] * po;
    if (fsf3(lm, lf, 0)) a.dSo -= SF3 * Vb * pf / tor * Fr.rho(0) * Fr.D(i, 0) * (fxi - 0.0);
    dRMdSg -= kSIC * t.dkm[2] * po;
    dRMdSg -= kSIC * t.dkm[3] * pg;
    if (fsf1(lm, lf, 1)) dRMdSg -= SF1 * Vb * pm / tor * rg * M.D(i, 1) * (fyi - yi);
    a.dSg -= kSIC * t.dkf[2] * po;
    a.dSg -= kSIC * t.dkf[3] * pg;
    if (fsf3(lm, lf, 1)) a.dSg -= SF3 * Vb * pf / tor * Fr.rho(1) * Fr.D(i, 1) * (fyi - 0.0);
    dRMdSw -= kSIC * t.dkm[1] * po;
    a.dSw -= kSIC * t.dkf[1] * po;
    for (int q = 0; q < nf; q++) comp_face_ps(v, Fr, i, fc[q], fracture_comp_quirks(fc[q]), out, row, a, true);
    const WellAt W = well_at(v, 1, c, i, fyi);
    const OwnLayout L = own_layout(N, lf);
    out.add(0, row, L.P, v.pcoeff * (dLdp + a.dp + fxi * W.PIo + W.gcomp * W.PIg));
    if (L.swso) {
        out.add(0, row, L.Sw, -a.dSw);
        out.add(0, row, L.So, dLdSo - a.dSo);
    }
    if (L.sg) out.add(0, row, L.Sg, dLdSg - a.dSg);
    const int rm = lm ? N : 0;
    if (lm == 1) out.add(7, row, 2 * N + 2 - rm, dRMdSo);
    else if (lm == -1) out.add(7, row, 2 * N + 2 - rm, dRMdSg);
    else {
        out.add(7, row, 2 * N + 2, dRMdSo);
        out.add(7, row, 2 * N + 3, dRMdSg);
    }
    out.add(7, row, 2 * N - rm, v.pcoeff * dRMdp);
    out.add(7, row, 2 * N + 1 - rm, dRMdSw);
    for (int k = 0; k < N; k++) {
        double dRxl = 0, dRxg = 0, dRMxl = 0, dRMxg = 0;
        const bool diag = k == i;
        for (int ph = 0; ph < 2; ph++) {
            const double w = M.w(ph, i), rho = M.rho(ph), kr = ph ? t.krg : t.kro, mub = ph ? mubar_g : mubar_o;
            const double Dd = ph ? t.Dg : t.Do, dPp = ph ? t.dPg : t.dPo;
            double &dR = ph ? dRxg : dRxl;
            double &dRM = ph ? dRMxg : dRMxl;
            if (diag) dRM -= kSIC * rho * SF2 * Vb * kr / mub * dPp;
            dRM -= kSIC * M.dE(k, ph) * w * SF2 * Vb * kr / mub * dPp;
            dRM -= -kSIC * visc_deriv(M, k, ph) * w * rho * SF2 * Vb * kr * pm / (Dd * Dd) * dPp * (pf + pm);
            if (fsf1(lm, lf, ph)) {
                const double sat = M.S(1 + ph), D = M.D(i, ph), dlt = Fr.w(ph, i) - w;
                dRM -= M.dE(k, ph) * SF1 * sat * pm * Vb / tor * D * dlt;
                if (diag) dRM -= -SF1 * sat * pm * Vb / tor * rho * D;
                dRM -= diff_deriv(M, i, k, ph) * SF1 * sat * pm * Vb / tor * rho * dlt;
            }
            dR -= -kSIC * visc_deriv(Fr, k, ph) * w * rho * SF2 * Vb * kr * pf / (Dd * Dd) * dPp * (pf + pm);
            // the fracture's own SF1 / SF3 composition dependences, in the reference's order
            const double msat = M.S(1 + ph), mD = M.D(i, ph);
            const double fsat = Fr.S(1 + ph), frho = Fr.rho(ph), fD = Fr.D(i, ph), fw = Fr.w(ph, i);
            const bool s1 = fsf1(lm, lf, ph) && diag, s3 = fsf3(lm, lf, ph);
            auto sf1_term = [&]() { if (s1) dR -= SF1 * msat * pm * Vb / tor * rho * mD; };
            auto sf3_term = [&]() {
                if (!s3) return;
                dR -= Fr.dE(k, ph) * SF3 * fsat * pf * Vb / tor * fD * (fw - 0.0);
                if (diag) dR -= SF3 * fsat * pf * Vb / tor * frho * fD;
                dR -= diff_deriv(Fr, i, k, ph) * SF3 * fsat * pf * Vb / tor * frho * (fw - 0.0);
            };
            // both-phase pairings list the interface term first
            if ((ph == 0 && lm == 0 && lf == 1) || (ph == 1 && lm == 0 && lf == -1)) {
                if (ph == 0) { sf3_term(); sf1_term(); }
                else { sf1_term(); sf3_term(); }
            } else {
                sf1_term();
                sf3_term();
            }
        }
        const double dLxl = diag ? Fr.rho(0) + fxi * Fr.dE(k, 0) : fxi * Fr.dE(k, 0);
        const double dLxg = diag ? Fr.rho(1) + fyi * Fr.dE(k, 1) : fyi * Fr.dE(k, 1);
        const double dQxl = (diag && W.iwell < 0) ? W.Qo : 0.0, dQxg = (diag && W.iwell < 0) ? W.Qg : 0.0;
        for (int q = 0; q < nf; q++) comp_face_x(v, Fr, i, k, fc[q], fracture_comp_quirks(fc[q]), out, row, dRxl, dRxg, true);
        if (lm == 1) out.add(7, row, k, dRMxl);
        else if (lm == -1) out.add(7, row, k, dRMxg);
        else {
            out.add(7, row, k, dRMxl);
            out.add(7, row, N + k, dRMxg);
        }
        if (L.x) out.add(0, row, L.X + k, (Vb / v.dt) * pf * Fr.S(1) * dLxl - dQxl - dRxl);
        if (L.y) out.add(0, row, L.Y + k, (Vb / v.dt) * pf * Fr.S(2) * dLxg - dQxg - dRxg);
    }
}

// Block row b (cell-medium) of the Jacobian.  Returns false when this
// cell-medium's case is not covered.
OSR_HD inline bool jacobian_block(const JacView &v, long b) {
    const int N = v.nc;
    const int med = b >= v.n;
    const long c = med ? b - v.n : b;
    const BlockRow out{&v, b};
    const Cell q{&v, &v.m[med], c};
    const int lab = q.label();
    const int rows = lab == 0 ? 2 * N + 4 : N + 3;
    if (q.por() < 1e-10) {
        // an inactive cell-medium: unit diagonal
        for (int r = 0; r < rows; r++) out.add(0, r, r, 1.0);
        return true;
    }
    const int r0 = lab == 0 ? N : 0;
    if (lab == 0) fugacity_rows(v, q, out);
    if (med == 0)
        for (int i = 0; i < N - 1; i++) matrix_comp_row_2ph(v, c, i, out, r0 + i);
    else
        for (int i = 0; i < N - 1; i++) fracture_comp_row_2ph(v, c, i, out, r0 + i);
    total_row_2ph(v, med, c, out, r0 + N - 1);
    water_row_2ph(v, med, c, out, r0 + N);
    if (lab == 0) {
        constraint_rows_2ph(v, out);
    } else {
        const OwnLayout L = own_layout(N, lab);
        for (int k = 0; k < N; k++) out.add(0, N + 1, (lab == 1 ? L.X : L.Y) + k, 1.0);
        out.add(0, N + 2, L.Sw, 1.0);
        out.add(0, N + 2, lab == 1 ? L.So : L.Sg, 1.0);
    }
    return true;
}

}  // namespace osrj

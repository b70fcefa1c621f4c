/* C entry points into the reference simulator compiled unmodified from its
 * own sources (test infrastructure only: oracle/_ref/libosiris_ref.so).
 *
 * Each entry point sets the reference's global state the way its own
 * initialisation does, calls the reference function, and copies the
 * results out into flat arrays.  Nothing here re-implements reference
 * arithmetic; the restated oracle lives in oracle/flash_oracle.c.
 *
 * Layout of the flat arrays (shared with the restated oracle and the CUDA
 * library): per-cell scalars are [n]; per-component fields are
 * component-major [nc][n]. */
#include <chrono>
#include <fstream>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <cmath>
#include "Functions.h"

namespace {

int g_alloc_nc = -1;

/* Allocate the reference's global arrays for a 1x1x1 grid with nc
 * components, through the reference's own Allocation()
 * (compsim/Data_Input.cpp:1351).  Called once per component count. */
void ensure_single_cell(int nc) {
    if (g_alloc_nc == nc) return;
    Nx = Ny = Nz = 1;
    PNc = nc;
    UNc = 0;
    Nc = nc;
    Nswt = 2;
    Nsgt = 2;
    wellNO = 0;
    NOOptionsDB = 0;
    MPIsize = 1;
    MPIRank = 0;
    Allocation();
    g_alloc_nc = nc;
}

/* Component table and binary interaction: fluidProp columns as set by the
 * COMPNAME library (compsim/Data_Input.cpp:653-952), bic = 1 - kij as the
 * BIC keyword stores it (compsim/Data_Input.cpp:977-990). */
void set_fluid(int nc, int eos, const double *tc, const double *pc, const double *acf, const double *kij) {
    PR = (eos == 0);
    SRK = (eos != 0);
    for (int i = 0; i < nc; i++) {
        for (int c = 0; c < COMP_PROPS; c++) fluidProp[i][c] = 0;
        fluidProp[i][TCRIT] = tc[i];
        fluidProp[i][PCRIT] = pc[i];
        fluidProp[i][AC] = acf[i];
        fluidProp[i][MW] = 100.0;
        fluidProp[i][ZCRIT] = 0.28;
        for (int j = 0; j < nc; j++) bic[i][j] = 1 - kij[i * nc + j];
    }
}

/* EOS_Init divides VCRIT by 1e6 on every call (compsim/Init_Calcs.cpp:75),
 * so the driver restores it before each per-temperature call. */
void eos_at(int nc, double T) {
    for (int i = 0; i < nc; i++) fluidProp[i][VCRIT] = 300.0;
    resTemp = T;
    EOS_Init();
}

}  // namespace

extern "C" {

/* Flash n independent cells with the reference's SuccFalsh
 * (compsim/Init_Calcs.cpp:571-738): Wilson K, successive substitution with an
 * inner Rachford-Rice Newton, phase label from L.  Water saturation is 0, so
 * sat_o/sat_g are the hydrocarbon volume fractions.  kij is [nc][nc]. */
int ref_flash_batch(int nc, int eos, const double *tc, const double *pc, const double *acf, const double *kij,
                    long n, const double *P, const double *T, const double *z, double *x, double *y,
                    signed char *label, double *sat_o, double *sat_g, double *rho_o, double *rho_g) {
    if (nc < 1 || nc > 64) return -1;
    ensure_single_cell(nc);
    set_fluid(nc, eos, tc, pc, acf, kij);
    double lastT = -1;
    for (long c = 0; c < n; c++) {
        if (T[c] != lastT) {
            eos_at(nc, T[c]);
            lastT = T[c];
        }
        ::P[1][1][1][1] = P[c];
        sat[0][0][0][0] = 0;
        for (int i = 0; i < nc; i++) {
            comp[0][0][0][i][2] = z[(long)i * n + c];
            comp[0][0][0][i][0] = 0;
            comp[0][0][0][i][1] = 0;
        }
        SuccFalsh(0, 0, 0);
        for (int i = 0; i < nc; i++) {
            x[(long)i * n + c] = comp[0][0][0][i][0];
            y[(long)i * n + c] = comp[0][0][0][i][1];
        }
        label[c] = phaseStat[0][0][0];
        sat_o[c] = sat[0][0][0][1];
        sat_g[c] = sat[0][0][0][2];
        rho_o[c] = blockFProps[0][0][0][RO][0];
        rho_g[c] = blockFProps[0][0][0][RO][1];
    }
    return 0;
}

/* The reference's cubic root rule (compsim/Globals.cpp:212-264), exposed for
 * the root-selection tests. */
double ref_solve_z(double a1, double a2, double a3, int gas) { return Solve_Z(a1, a2, a3, gas ? 'g' : 'l'); }

/* EOS parameters a_i(T), b_i from the reference's EOS_Init
 * (compsim/Init_Calcs.cpp:66-97). */
int ref_eos_params(int nc, int eos, const double *tc, const double *pc, const double *acf, double T, double *a,
                   double *b) {
    if (nc < 1 || nc > 64) return -1;
    ensure_single_cell(nc);
    double zero[64 * 64] = {0};
    set_fluid(nc, eos, tc, pc, acf, zero);
    eos_at(nc, T);
    for (int i = 0; i < nc; i++) {
        a[i] = fluidProp[i][EOS_A];
        b[i] = fluidProp[i][EOS_B];
    }
    return 0;
}

}  // extern "C"

/* ------------------------------------------------------------------------
 * Deck-driven entry points: the reference reads a Data_Input deck and runs
 * the initialisation of its main program (compsim/PrimeSim.cpp:35-85); the
 * driver then exposes its state and property arrays, and evaluates the
 * PETSc callbacks (FormFunction, FormJacobian, InitGuess2, UpdateAll) on
 * caller-owned vectors through the PETSc-lite shim.
 *
 * Field layout of every dump: cell index c = Ix + Nx*(Iy + Ny*Iz) fastest,
 * then the array's trailing index (component, phase, direction), e.g.
 * "m.x" -> [nc][cells], "m.dE" -> [nc+1][2][cells], "m.trans" ->
 * [12][3][cells].  Prefix "m." = matrix, "f." = fracture.
 * ------------------------------------------------------------------------ */
#include "shim_types.h"
#include "MIfstream.h"

namespace {

long ncell() { return (long)Nx * Ny * Nz; }

template <class F>
void each_cell(F f) {
    for (int Iz = 0; Iz < Nz; Iz++)
        for (int Iy = 0; Iy < Ny; Iy++)
            for (int Ix = 0; Ix < Nx; Ix++) f(Ix, Iy, Iz, (long)Ix + (long)Nx * (Iy + (long)Ny * Iz));
}

}  // namespace

extern "C" {

/* Read a deck and initialise as main() does before its time loop. */
int ref_deck_open(const char *path) {
    MIfstream fin;
    fin.open(path, std::ios::in);
    if (!fin.is_open()) return -1;
    g_alloc_nc = -1;
    MPIsize = 1;
    MPIRank = 0;
    /* time-control state as a fresh process starts with it */
    incCount = 0;
    TSMCtrl = 0;
    repStat = 0;
    maxNR = 0;
    Data_Input(fin);
    fin.close();
    ManageTSMarker();
    IFK_Calc();
    Tr_Mu();
    QInitValue();
    Edge_Trans();
    Edge_fTrans();
    InitWells();
    WellCompSadeq_cum[0] = WellCompSadeq_cum[1] = WellCompSadeq_cum[2] = 0;
    SMethQ = 0;
    /* UpdateDependencies(true) starts with PhaseCtrl, whose test for a
     * gas-only cell reads the gas-phase pressure (compsim/Do_Cycle.cpp:1579)
     * before anything has written it: the deck sets only the oil pressure.
     * In a fresh process that memory reads zero; in a process that has
     * allocated and freed memory before, it holds whatever was left there,
     * and the start-up state changes from one opening to the next.  Pin it
     * to the fresh-process value. */
    for (int i = 0; i < Nx; i++)
        for (int j = 0; j < Ny; j++)
            for (int k = 0; k < Nz; k++) {
                P[i + 1][j + 1][k + 1][0] = P[i + 1][j + 1][k + 1][2] = 0;
                fP[i + 1][j + 1][k + 1][0] = fP[i + 1][j + 1][k + 1][2] = 0;
            }
    UpdateDependencies(true);
    return 0;
}

/* Nx, Ny, Nz, Nc, PR, MatrixSize, wellNO, Nswt, Nsgt, IsConstDif */
void ref_deck_info(int *info) {
    info[0] = Nx; info[1] = Ny; info[2] = Nz; info[3] = Nc; info[4] = PR;
    info[5] = MatrixSize; info[6] = wellNO; info[7] = Nswt; info[8] = Nsgt; info[9] = IsConstDif ? 1 : 0;
}

double ref_scalar(const char *name) {
    std::string s(name);
    if (s == "PCoeff") return PCoeff;
    if (s == "resTemp") return resTemp;
    if (s == "watRo") return watRo;
    if (s == "watMu") return watMu;
    if (s == "refP") return refP;
    if (s == "cpor") return cpor;
    if (s == "dcpor") return dcpor;
    if (s == "Lf") return Lf;
    if (s == "Re_f") return Re_f;
    if (s == "SigmaMF") return SigmaMF;
    if (s == "CDiffCoef") return CDiffCoef;
    if (s == "Dt") return Dt;
    if (s == "SMethQ") return SMethQ;
    return 0.0 / 0.0;
}

/* Copy a named array into out (layout above); returns values written or -1. */
long ref_get(const char *name, double *out) {
    std::string s(name);
    const long n = ncell();
    bool fr = s.size() > 2 && s[0] == 'f' && s[1] == '.';
    std::string k = s.size() > 2 ? s.substr(2) : s;
    FType *****cp = fr ? fcomp : comp;
    FType ****pp = fr ? fP : P;
    FType ****st = fr ? fsat : sat;
    signed char ***ps = fr ? fphaseStat : phaseStat;
    FType *****bp = fr ? fblockFProps : blockFProps;
    FType ****kr = fr ? frelPerm : relPerm;
    FType ****dkr = fr ? fdRelPerm : dRelPerm;
    FType *****de = fr ? fdE : dE;
    FType ****pre = fr ? fpreProp : preProp;
    FType *****dif = fr ? fdiffusion : diffusion;
    FType ***ift = fr ? fBift : Bift;
    FType *****tr = fr ? ftrans : trans;
    char *****trs = fr ? ftransS : transS;
    FType ****wt = fr ? fWtran : Wtran;
    FType ****dwt = fr ? fdWtran : dWtran;
    FType ****ift3 = fr ? fIFTran : IFTran;
    FType ***por = fr ? fporosity : porosity;
    FType ****perm4 = fr ? fperm : perm;
    long w = 0;
    if (k == "P") {
        for (int p = 0; p < 3; p++) each_cell([&](int i, int j, int l, long c) { out[p * n + c] = pp[i + 1][j + 1][l + 1][p]; });
        w = 3 * n;
    } else if (k == "sat") {
        for (int p = 0; p < 3; p++) each_cell([&](int i, int j, int l, long c) { out[p * n + c] = st[i][j][l][p]; });
        w = 3 * n;
    } else if (k == "x" || k == "y" || k == "z") {
        int ph = k == "x" ? 0 : (k == "y" ? 1 : 2);
        for (int q = 0; q < Nc; q++) each_cell([&](int i, int j, int l, long c) { out[q * n + c] = cp[i][j][l][q][ph]; });
        w = (long)Nc * n;
    } else if (k == "label") {
        each_cell([&](int i, int j, int l, long c) { out[c] = ps[i][j][l]; });
        w = n;
    } else if (k == "rho" || k == "pc" || k == "mu" || k == "gam") {
        int f = k == "rho" ? RO : (k == "pc" ? BLOCK_PC : (k == "mu" ? BMU : BGAM));
        for (int p = 0; p < 2; p++) each_cell([&](int i, int j, int l, long c) { out[p * n + c] = bp[i][j][l][f][p]; });
        w = 2 * n;
    } else if (k == "kr") {
        for (int p = 0; p < 3; p++) each_cell([&](int i, int j, int l, long c) { out[p * n + c] = kr[i][j][l][p]; });
        w = 3 * n;
    } else if (k == "dkr") {
        for (int p = 0; p < 5; p++) each_cell([&](int i, int j, int l, long c) { out[p * n + c] = dkr[i][j][l][p]; });
        w = 5 * n;
    } else if (k == "dE") {
        for (int q = 0; q <= Nc; q++)
            for (int p = 0; p < 2; p++) each_cell([&](int i, int j, int l, long c) { out[(q * 2 + p) * n + c] = de[i][j][l][q][p]; });
        w = (long)(Nc + 1) * 2 * n;
    } else if (k == "pre") {
        for (int q = 0; q <= Nc; q++) each_cell([&](int i, int j, int l, long c) { out[q * n + c] = pre[i][j][l][q]; });
        w = (long)(Nc + 1) * n;
    } else if (k == "diff") {
        for (int q = 0; q < Nc; q++)
            for (int p = 0; p < 2; p++) each_cell([&](int i, int j, int l, long c) { out[(q * 2 + p) * n + c] = dif[i][j][l][q][p]; });
        w = (long)Nc * 2 * n;
    } else if (k == "ift") {
        each_cell([&](int i, int j, int l, long c) { out[c] = ift[i][j][l]; });
        w = n;
    } else if (k == "trans") {
        for (int t = 0; t < 12; t++)
            for (int d = 0; d < 3; d++) each_cell([&](int i, int j, int l, long c) { out[(t * 3 + d) * n + c] = tr[i + 1][j + 1][l + 1][t][d]; });
        w = 36 * n;
    } else if (k == "transS") {
        for (int t = 0; t < 3; t++)
            for (int d = 0; d < 3; d++) each_cell([&](int i, int j, int l, long c) { out[(t * 3 + d) * n + c] = trs[i + 1][j + 1][l + 1][t][d]; });
        w = 9 * n;
    } else if (k == "wtran" || k == "dwtran") {
        FType ****a = k == "wtran" ? wt : dwt;
        for (int d = 0; d < 3; d++) each_cell([&](int i, int j, int l, long c) { out[d * n + c] = a[i + 1][j + 1][l + 1][d]; });
        w = 3 * n;
    } else if (k == "iftran") {
        for (int d = 0; d < 3; d++) each_cell([&](int i, int j, int l, long c) { out[d * n + c] = ift3[i][j][l][d]; });
        w = 3 * n;
    } else if (k == "por") {
        each_cell([&](int i, int j, int l, long c) { out[c] = por[i][j][l]; });
        w = n;
    } else if (k == "perm") {
        for (int d = 0; d < 3; d++) each_cell([&](int i, int j, int l, long c) { out[d * n + c] = perm4[i][j][l][d]; });
        w = 3 * n;
    } else if (k == "blockH") {
        each_cell([&](int i, int j, int l, long c) { out[c] = blockH[i + 1][j + 1][l + 1]; });
        w = n;
    } else if (s == "gridDim") {
        for (int q = 0; q < Nx + Ny + Nz; q++) out[q] = gridDim[q];
        w = Nx + Ny + Nz;
    } else if (s == "fluid") {  /* [nc][15] fluidProp */
        for (int q = 0; q < Nc; q++)
            for (int f = 0; f < COMP_PROPS; f++) out[q * COMP_PROPS + f] = fluidProp[q][f];
        w = (long)Nc * COMP_PROPS;
    } else if (s == "bic") {
        for (int q = 0; q < Nc; q++)
            for (int r = 0; r < Nc; r++) out[q * Nc + r] = bic[q][r];
        w = (long)Nc * Nc;
    } else if (s == "rowoff") {  /* preConRow[0..2*cells] */
        for (long q = 0; q <= 2 * n; q++) out[q] = preConRow[q];
        w = 2 * n + 1;
    } else {
        return -1;
    }
    return w;
}

/* Overwrite a named state array (the layout of ref_get): m./f. + P, sat,
 * x, y, z, label or rho.  Returns the values read, or -1. */
long ref_set(const char *name, const double *in) {
    std::string s(name);
    const long n = ncell();
    bool fr = s.size() > 2 && s[0] == 'f' && s[1] == '.';
    std::string k = s.size() > 2 ? s.substr(2) : s;
    FType *****cp = fr ? fcomp : comp;
    FType ****pp = fr ? fP : P;
    FType ****st = fr ? fsat : sat;
    signed char ***ps = fr ? fphaseStat : phaseStat;
    if (k == "P") {
        for (int p = 0; p < 3; p++) each_cell([&](int i, int j, int l, long c) { pp[i + 1][j + 1][l + 1][p] = in[p * n + c]; });
        return 3 * n;
    }
    if (k == "sat") {
        for (int p = 0; p < 3; p++) each_cell([&](int i, int j, int l, long c) { st[i][j][l][p] = in[p * n + c]; });
        return 3 * n;
    }
    if (k == "x" || k == "y" || k == "z") {
        int ph = k == "x" ? 0 : (k == "y" ? 1 : 2);
        for (int q = 0; q < Nc; q++) each_cell([&](int i, int j, int l, long c) { cp[i][j][l][q][ph] = in[q * n + c]; });
        return (long)Nc * n;
    }
    if (k == "label") {
        each_cell([&](int i, int j, int l, long c) { ps[i][j][l] = (signed char)in[c]; });
        return n;
    }
    if (k == "rho") {  /* phase molar densities, read by the next CalcIFT */
        FType *****bp = fr ? fblockFProps : blockFProps;
        for (int p = 0; p < 2; p++) each_cell([&](int i, int j, int l, long c) { bp[i][j][l][RO][p] = in[p * n + c]; });
        return 2 * n;
    }
    return -1;
}

/* Saturation pressure of cell c of one continuum as PhaseCtrl computes it
 * (Bubl_Succ / Dew_Succ, or the fracture's fBubl_Succ / fDew_Succ,
 * compsim/Minor_NR.cpp:491-2015) by its phase label; xm receives Xm[0..Nc-1].
 * Two-phase cells return 0. */
double ref_sat_pressure(int med, long c, double *xm) {
    const int Ix = (int)(c % Nx), Iy = (int)((c / Nx) % Ny), Iz = (int)(c / ((long)Nx * Ny));
    const int lab = med ? fphaseStat[Ix][Iy][Iz] : phaseStat[Ix][Iy][Iz];
    double p = 0;
    if (lab == 1) p = med ? fBubl_Succ(Ix, Iy, Iz) : Bubl_Succ(Ix, Iy, Iz);
    else if (lab == -1) p = med ? fDew_Succ(Ix, Iy, Iz) : Dew_Succ(Ix, Iy, Iz);
    for (int i = 0; i < Nc; i++) xm[i] = lab ? Xm[i] : 0.0;
    return p;
}

/* Bubl_NR (kind 0, an oil-only cell), Dew_NR (kind 1) or LowerDew_Succ
 * (kind 2, a gas-only cell) on matrix cell c (compsim/Minor_NR.cpp:33-489,
 * 2017-2136); xm receives Xm[0..Nc-1].  Bubl_NR and Dew_NR iterate without a
 * cap, so callers pass only cells whose restated iteration stopped. */
double ref_sat_pressure_nr(int kind, long c, double *xm) {
    const int Ix = (int)(c % Nx), Iy = (int)((c / Nx) % Ny), Iz = (int)(c / ((long)Nx * Ny));
    double p = kind == 0 ? Bubl_NR(Ix, Iy, Iz) : kind == 1 ? Dew_NR(Ix, Iy, Iz) : LowerDew_Succ(Ix, Iy, Iz);
    for (int i = 0; i < Nc; i++) xm[i] = Xm[i];
    return p;
}

/* critTest on matrix cell c (compsim/Minor_NR.cpp:2138-2308), as its
 * commented call site applies it to one-phase cells
 * (compsim/Do_Cycle.cpp:1576); returns the cell's label afterwards. */
int ref_crit_test(long c) {
    const int Ix = (int)(c % Nx), Iy = (int)((c / Nx) % Ny), Iz = (int)(c / ((long)Nx * Ny));
    if (phaseStat[Ix][Iy][Iz]) critTest(Ix, Iy, Iz);
    return phaseStat[Ix][Iy][Iz];
}

/* PhaseCtrl and fPhaseCtrl (compsim/Do_Cycle.cpp:1558-1721). */
int ref_phase_ctrl(void) {
    PhaseCtrl();
    fPhaseCtrl();
    return 0;
}

/* UpdateAll(x, full) (compsim/PetscAUX.cpp:176-498). */
int ref_update_all(double *x, int full) {
    _p_Vec v{x, MatrixSize};
    UpdateAll(&v, full != 0);
    return 0;
}

/* Calc_Re of well i at its first completion (compsim/Minor_NR.cpp:2700). */
double ref_calc_re(int i) {
    if (i < 0 || i >= wellNO) return -1;
    return Calc_Re(welli[i][1], welli[i][2], welli[i][3], i);
}

/* The WellCondition latch of well i (compsim/Do_Cycle.cpp:1745). */
int ref_set_well_condition(int i, int v) {
    if (i < 0 || i >= wellNO) return -1;
    WellCondition[i] = v != 0;
    return 0;
}

/* InitGuess2: state -> x (compsim/PetscAUX.cpp:878-964). */
int ref_init_guess(double *x) {
    _p_Vec v{x, MatrixSize};
    InitGuess2(nullptr, &v, nullptr);
    return 0;
}

/* Replace the component table of an opened deck (fluidProp columns as the
 * COMPNAME library sets them, compsim/Data_Input.cpp:653-952; bic = 1 - kij as
 * the BIC keyword stores it, compsim/Data_Input.cpp:977-990) and redo the
 * per-component initialisation that depends on it: EOS_Init (which divides
 * VCRIT, given here in cm3/mol, by 1e6) and Tr_Mu
 * (compsim/Init_Calcs.cpp:48-97).  The reference's own user-component path
 * recomputes Tc, Pc and omega from SG/TB correlations (CPlus_Props), so a
 * seeded table can only enter this way.  Call before setting the state. */
int ref_override_fluid(int nc, const double *tc, const double *pc, const double *acf, const double *mw,
                       const double *vc, const double *zc, const double *parachor, const double *kij) {
    if (nc != Nc) return -1;
    for (int i = 0; i < nc; i++) {
        fluidProp[i][TCRIT] = tc[i];
        fluidProp[i][PCRIT] = pc[i];
        fluidProp[i][AC] = acf[i];
        fluidProp[i][MW] = mw[i];
        fluidProp[i][VCRIT] = vc[i];
        fluidProp[i][ZCRIT] = zc[i];
        fluidProp[i][PARACHOR] = parachor[i];
        for (int j = 0; j < nc; j++) bic[i][j] = 1 - kij[i * nc + j];
    }
    EOS_Init();
    Tr_Mu();
    return 0;
}

/* PCoeff and the row layout of the current phase labels (CalcPCoeff, PJac),
 * as UpdateAll(x, true) runs them after phase control
 * (compsim/PetscAUX.cpp:505-506); for states set through ref_set. */
long ref_relayout(void) {
    CalcPCoeff();
    PJac();
    return MatrixSize;
}

/* Evaluate IteratorFunction (which = 0) or IteratorJacobian (which = 1) for
 * the k listed global rows, as FormFunction / FormJacobian do for every row
 * (compsim/PetscAUX.cpp:59-173), after the caller's UpdateAll; returns the
 * wall time of the loop in seconds.  Values go to f (which = 0, MatrixSize
 * doubles) or to a scratch matrix that is cleared first. */
double ref_time_rows(const long *rows, long k, double *x, double *f, double t, int which) {
    _p_Vec vx{x, MatrixSize}, vf{f, MatrixSize};
    _p_Mat m;
    SSimTime = t;
    userData.SimulationTime = t;
    const auto t0 = std::chrono::steady_clock::now();
    for (long q = 0; q < k; q++) {
        userData.GlobalIndex = (int)rows[q];
        userData.LocalIndex = (int)rows[q];
        if (which == 0) IteratorFunction(&vx, &vf, &userData);
        else IteratorJacobian(&vx, &m, &userData);
    }
    const auto t1 = std::chrono::steady_clock::now();
    return std::chrono::duration<double>(t1 - t0).count();
}

/* CreateBackups (compsim/Do_Time_Step.cpp:86-159). */
int ref_create_backups(double t) {
    CreateBackups(t);
    return 0;
}

/* TimeStepCtrl (compsim/Do_Time_Step.cpp:391-470) after a pass whose solve was
 * accepted (rejected = 0) or not (rejected = 1), as the main loop sets
 * repStat (compsim/PrimeSim.cpp:95-101): advances *t, updates Dt, and after a
 * rejection restores the backups and the row layout.  Returns its flag
 * (1 when the last time marker is reached). */
int ref_time_step_ctrl(double *t, int rejected) {
    repStat = rejected ? 1 : 0;
    return (int)TimeStepCtrl(t);
}

/* The time markers (TStepMarker[0..TSMSize), after ManageTSMarker) and the
 * index of the next one; returns TSMSize. */
int ref_time_markers(double *out, int *ctrl) {
    for (int i = 0; i < TSMSize; i++) out[i] = TStepMarker[i];
    if (ctrl) *ctrl = TSMCtrl;
    return TSMSize;
}

/* WriteRST (compsim/Do_Time_Step.cpp:179-234): the restart file "test.rst"
 * in the current directory, at simulation time t. */
int ref_write_rst(double t) {
    WriteRST(t);
    return 0;
}

/* PrintAll (compsim/ViewAssist.Cpp:39-88) of the current state at time t,
 * appended to one stream kept open across calls as the main program keeps
 * its output file (path opens it, a null path closes it). */
int ref_print_all(const char *path, double t) {
    static std::ofstream out;
    if (!path) {
        if (out.is_open()) out.close();
        return 0;
    }
    if (!out.is_open()) out.open(path, std::ios::out);
    if (!out.is_open()) return -1;
    PrintAll(out, t);
    return 0;
}

/* FormFunction(x) -> f (compsim/PetscAUX.cpp:59-104) at simulation time t. */
int ref_form_function(double *x, double *f, double t) {
    _p_Vec vx{x, MatrixSize}, vf{f, MatrixSize};
    SSimTime = t;
    return FormFunction(nullptr, &vx, &vf, &userData);
}

/* FormJacobian(x) (compsim/PetscAUX.cpp:106-173): the (row, col, value)
 * triplets MatSetValues received, in call order.  Returns their count, or
 * -(count) when cap was too small. */
long ref_form_jacobian(double *x, double t, long cap, int *rows, int *cols, double *vals) {
    _p_Vec vx{x, MatrixSize};
    _p_Mat m;
    SSimTime = t;
    FormJacobian(nullptr, &vx, &m, &m, &userData);
    long cnt = (long)m.v.size();
    if (cnt > cap) return -cnt;
    for (long q = 0; q < cnt; q++) {
        rows[q] = m.r[q];
        cols[q] = m.c[q];
        vals[q] = m.v[q];
    }
    return cnt;
}

}  // extern "C"

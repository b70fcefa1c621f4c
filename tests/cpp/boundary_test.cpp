// Boundary test from a compiled C++ caller (test infrastructure).
//
// One process links the reference simulator compiled from its own sources
// (oracle/_ref/libosiris_ref.so, with the oracle's PETSc-lite Vec and Mat)
// and libosiris_b200.so, and for each deck given on the command line:
//   1. opens it with the reference's Data_Input + start-up (ref_deck_open) and
//      with osr_create (the library's C++ reader + device start-up);
//   2. checks the row layout (equal) and InitGuess2 (OsrInitGuess against
//      the reference's, within 1e-9: the two start-ups flash independently);
//   3. perturbs the unknowns, then runs the reference's FormFunction and
//      FormJacobian and the adapter's OsrFormFunction / OsrSetJacobianPattern /
//      OsrFormJacobian (include/osiris_b200_petsc.hpp) on the same Vec and
//      Mat types;
//   4. compares: residual rows within 1e-10 of each row's sum of |terms|
//      (osr_grid_residual reports it), Jacobian entries within 1e-9 of the
//      reference row's largest entry (duplicates summed), NaN only where the
//      reference has NaN, and the VPBJacobi block sizes both hand to
//      MatSetVariableBlockSizes.
// Prints one line per deck and exits 0 only if every check passed.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <map>
#include <utility>
#include <vector>
#include <petscsnes.h>
#include "petsc_cuda_lite.h"
#include "shim_types.h"
#include "osiris_b200_petsc.hpp"

int CreateAllocationTable(void);   // the reference's own (compsim/PetscAUX.cpp:1081-1099)

extern "C" {
int ref_deck_open(const char *path);
void ref_deck_info(int *info);
int ref_init_guess(double *x);
int ref_form_function(double *x, double *f, double t);
long ref_form_jacobian(double *x, double t, long cap, int *rows, int *cols, double *vals);
}

// Block sizes every caller hands to MatSetVariableBlockSizes, per Mat.  This
// definition in the executable interposes the oracle library's no-op, so the
// reference's own FormJacobian reports its sizes here too.
static std::map<Mat, std::vector<PetscInt>> g_blocks;
static std::vector<PetscInt> g_last_blocks;
PetscErrorCode MatSetVariableBlockSizes(Mat m, PetscInt n, PetscInt *bs) {
    g_blocks[m] = std::vector<PetscInt>(bs, bs + n);
    g_last_blocks = g_blocks[m];
    return 0;
}

static int check_deck(const char *path, double t) {
    int fails = 0;
    auto fail = [&](const char *what, double a, double b, long where) {
        if (fails < 8) std::printf("  FAIL %s at %ld: %.17g vs %.17g\n", what, where, a, b);
        fails++;
    };
    if (ref_deck_open(path) != 0) {
        std::printf("%s: reference could not open the deck\n", path);
        return 1;
    }
    int info[10];
    ref_deck_info(info);
    const long n = info[5];
    osr_grid *g = nullptr;
    osr_status st = osr_create(path, nullptr, &g);
    if (st != OSR_OK) {
        std::printf("%s: osr_create failed: %s (%s)\n", path, osr_status_string(st), osr_deck_error());
        return 1;
    }
    long rows = 0;
    double pcoeff = 0;
    osr_grid_layout(g, &rows, &pcoeff);
    if (rows != n) fail("row count", (double)rows, (double)n, -1);

    OsrSnesCtx c;
    c.g = g;
    c.sim_time = t;
    std::vector<double> x0((size_t)n), xg((size_t)n), f((size_t)n), fr((size_t)n), scale((size_t)n);
    ref_init_guess(x0.data());
    _p_Vec X{xg.data(), (int)n}, F{f.data(), (int)n};
    if (OsrInitGuess(nullptr, &X, &c) != 0) fail("OsrInitGuess status", (double)c.last, 0, -1);
    // the two start-ups flash the cells independently, so the unknowns agree
    // to the flash's rounding, not bit for bit
    double worst_x = 0;
    for (long r = 0; r < n; r++) {
        const double e = std::fabs(xg[(size_t)r] - x0[(size_t)r]) / std::fmax(1.0, std::fabs(x0[(size_t)r]));
        if (!(e <= 1e-9)) fail("InitGuess2", xg[(size_t)r], x0[(size_t)r], r);
        else if (e > worst_x) worst_x = e;
    }

    // the same perturbed unknowns on both sides
    unsigned s = 12345u;
    for (long r = 0; r < n; r++) {
        s = s * 1664525u + 1013904223u;
        const double u = (double)(s >> 8) / (double)(1u << 24) * 2 - 1;
        x0[(size_t)r] *= 1 + 1e-2 * u;
    }
    std::vector<double> xr = x0;   // the reference may write into its copy
    xg = x0;
    ref_form_function(xr.data(), fr.data(), t);
    if (OsrFormFunction(nullptr, &X, &F, &c) != 0) fail("OsrFormFunction status", (double)c.last, 0, -1);
    // each row's sum of |terms| from the device residual at the same state
    double *d_f = nullptr, *d_s = nullptr;
    cudaMalloc((void **)&d_f, (size_t)n * sizeof(double));
    cudaMalloc((void **)&d_s, (size_t)n * sizeof(double));
    osr_grid_residual(g, d_f, d_s, t, nullptr);
    cudaMemcpy(scale.data(), d_s, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost);
    cudaFree(d_f);
    cudaFree(d_s);
    double worst_f = 0;
    for (long r = 0; r < n; r++) {
        const double e = std::fabs(f[(size_t)r] - fr[(size_t)r]) / (scale[(size_t)r] + 1e-300);
        if (std::isnan(f[(size_t)r]) && std::isnan(fr[(size_t)r])) continue;   // the reference's own NaN rows
        if (!(e <= 1e-10)) fail("residual row", f[(size_t)r], fr[(size_t)r], r);
        else if (e > worst_f) worst_f = e;
    }

    // Jacobian: reference triplets and the adapter's COO values, both summed
    const long cap = n * 10 * (2 * info[3] + 4);
    std::vector<int> rr((size_t)cap), rc((size_t)cap);
    std::vector<double> rv((size_t)cap);
    xr = x0;
    g_last_blocks.clear();
    CreateAllocationTable();   // SolveNonLinear's set-up of the rank's block sizes (compsim/PetscAUX.cpp:589)
    const long cnt = ref_form_jacobian(xr.data(), t, cap, rr.data(), rc.data(), rv.data());
    const std::vector<PetscInt> ref_blocks = g_last_blocks;
    _p_Mat B;
    if (OsrSetJacobianPattern(&B, &c) != 0) fail("OsrSetJacobianPattern status", (double)c.last, 0, -1);
    const std::vector<PetscInt> our_blocks = g_blocks[&B];
    xg = x0;
    if (OsrFormJacobian(nullptr, &X, &B, &B, &c) != 0) fail("OsrFormJacobian status", (double)c.last, 0, -1);
    std::map<std::pair<int, int>, double> Jr, Jg;
    for (long q = 0; q < cnt; q++) Jr[{rr[(size_t)q], rc[(size_t)q]}] += rv[(size_t)q];
    for (size_t q = 0; q < B.v.size(); q++) Jg[{B.r[q], B.c[q]}] += B.v[q];
    std::vector<double> rowmax((size_t)n, 0.0);
    for (const auto &kv : Jr)
        if (std::isfinite(kv.second))
            rowmax[(size_t)kv.first.first] = std::fmax(rowmax[(size_t)kv.first.first], std::fabs(kv.second));
    double worst_j = 0;
    long compared = 0;
    for (const auto &kv : Jr) {
        const auto it = Jg.find(kv.first);
        const double mine = it == Jg.end() ? 0.0 : it->second;
        const double ref = kv.second;
        compared++;
        if (std::isnan(ref) && std::isnan(mine)) continue;
        const double e = std::fabs(mine - ref) / (rowmax[(size_t)kv.first.first] + 1e-300);
        if (!(e <= 1e-9)) fail("Jacobian entry", mine, ref, (long)kv.first.first * n + kv.first.second);
        else if (e > worst_j) worst_j = e;
    }
    for (const auto &kv : Jg)   // entries the reference does not hold must be zero
        if (!Jr.count(kv.first) && kv.second != 0) fail("extra entry", kv.second, 0, (long)kv.first.first * n + kv.first.second);
    if (ref_blocks.empty()) fail("reference block sizes not captured", 0, 0, -1);
    if (our_blocks != ref_blocks) fail("VPBJacobi block sizes", (double)our_blocks.size(), (double)ref_blocks.size(), -1);
    OsrSnesCtxRelease(&c);
    osr_grid_destroy(g);
    std::printf("%s: %ld rows, %ld Jacobian entries; unknowns worst %.3e, residual worst %.3e of the row's |terms|, "
                "Jacobian worst %.3e of the row maximum, %zu block sizes equal: %s\n",
                path, n, compared, worst_x, worst_f, worst_j, our_blocks.size(), fails ? "FAIL" : "ok");
    return fails ? 1 : 0;
}

int main(int argc, char **argv) {
    if (argc < 2) {
        std::printf("usage: %s deck.dat [deck2.dat ...]\n", argv[0]);
        return 2;
    }
    int bad = 0;
    for (int i = 1; i < argc; i++) bad += check_deck(argv[i], 3600.0);
    return bad ? 1 : 0;
}

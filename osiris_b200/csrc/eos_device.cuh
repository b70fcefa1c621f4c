// Device-side cubic equation-of-state primitives (FP64, sm_100a).
//
// Every routine restates one piece of the reference simulator's thermodynamics
// (khazali/Osiris, compsim/) and cites it.  Compositions are processed one
// cell per thread with the component count N a compile-time constant, so the
// per-component arrays live in registers and the loops unroll.
//
// Component tables are per-launch constants (kernel parameters, read through
// the constant cache): critical pressure/temperature, the Wilson exponent
// coefficient 5.37 (1 + omega), the temperature-independent parts of a_i(T)
// (a_c and m), b_i, and the binary-interaction multipliers 1 - k_ij.
#pragma once
#include <cstdint>

namespace osr {

constexpr double kR = 8.3144621;                          // RGAS, compsim/Functions.h:216
constexpr double kSqrt2 = 1.4142135623730950488016887;    // SQRT2, compsim/Functions.h:219
constexpr double kPi = 3.1415926535897932384626433;       // PI, compsim/Functions.h:218
constexpr double kRRTol = 1e-8;                           // NEWTON_TOL, compsim/Functions.h:236
constexpr double kSSTol = 1e-14;                          // FLASH_TOL, compsim/Functions.h:237
constexpr double kLZero = 1e-20;                          // DZERO, compsim/Functions.h:239
constexpr int kRRMaxIt = 100;                             // MAX_FLASH_N_ITR, compsim/Functions.h:126
constexpr int kSSMaxIt = 500;                             // compsim/Init_Calcs.cpp:714
constexpr int kMaxNc = 16;

// Branch-free FP64 reciprocal and quotient.  The IEEE operator is compiled
// with an out-of-line slow path, and every such branch splits the code so
// that independent divisions cannot overlap (a Rachford-Rice step measured
// 4x its arithmetic latency).  Method: Newton-Raphson refinement of the
// hardware reciprocal seed (rcp.approx.ftz.f64), r' = r + r (1 - b r), then a
// residual-corrected quotient q' = q + r (a - b q) with the residual formed
// by a fused multiply-add (P. Markstein, "Computation of elementary functions
// on the IBM RISC System/6000 processor", IBM J. Res. Dev. 34(1), 1990).
// qrcp takes two refinement steps, qdiv one step and the correction; both
// are within one ulp of the IEEE result for operands inside qdiv_ok's range
// (tests/test_quotients_gpu.py checks this on random and edge operands).
// The callers gather qdiv_ok() over a whole step and redo that step with
// IEEE division when any operand is out of range (zeros, infinities, NaN,
// magnitudes beyond 2^+-1000), so special values follow the reference
// exactly.
__device__ __forceinline__ bool qdiv_ok(double a, double b) {
    double mb = fabs(b);
    return mb > 9.33e-302 && mb < 1.07e301 && fabs(a) < 1.07e301;
}

__device__ __forceinline__ double qrcp(double b) {
    double r;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(b));
    double e = fma(-b, r, 1.0);
    r = fma(r, e, r);
    e = fma(-b, r, 1.0);
    return fma(r, e, r);
}

__device__ __forceinline__ double qdiv(double a, double b) {
    double r;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(b));
    r = fma(r, fma(-b, r, 1.0), r);
    double q = a * r;
    return fma(fma(-b, q, a), r, q);
}

// Quotient by an exact constant divisor (9, 54, 3): reciprocal folded at
// compile time, one residual correction.
__device__ __forceinline__ double qdivc(double a, double b, double rb) {
    double q = a * rb;
    return fma(fma(-b, q, a), rb, q);
}

// Host-prepared component table for one fluid (one EOS, nc components).
template <int N>
struct FluidTable {
    double pc[N];      // critical pressure [Pa]
    double tc[N];      // critical temperature [K]
    double wil[N];     // 5.37 (1 + omega): Wilson K exponent, compsim/Init_Calcs.cpp:587
    double ac[N];      // Omega_a R^2 Tc^2 / Pc, compsim/Init_Calcs.cpp:83,91
    double m[N];       // alpha-function slope, compsim/Init_Calcs.cpp:84,92
    double b[N];       // Omega_b R Tc / Pc, compsim/Init_Calcs.cpp:86,94
    double bic[N * N]; // 1 - k_ij, compsim/Data_Input.cpp:985
    int srk;           // 0 = Peng-Robinson, 1 = Soave-Redlich-Kwong
};

// sqrt(a_i(T)) for every component: a_i = a_c (1 + m (1 - sqrt(T/Tc)))^2
// (compsim/Init_Calcs.cpp:85,93).  The reference mixes with sqrt(a_i a_j);
// this form, sqrt(a_i) sqrt(a_j), agrees to rounding and lets the mixing rule
// run as one matrix-vector product.
template <int N>
__device__ __forceinline__ void sqrt_a(const FluidTable<N> &f, double T, double *sa) {
#pragma unroll
    for (int i = 0; i < N; i++) {
        double s = 1 + f.m[i] * (1 - sqrt(T / f.tc[i]));
        sa[i] = sqrt(f.ac[i] * s * s);
    }
}

// Cubic root with the reference's selection rule (compsim/Globals.cpp:212-264):
// three real roots (D < 0) by the trigonometric form, vapour = largest,
// liquid = smallest positive (else the third); otherwise Cardano.  The three
// cosines come from one sincos and the angle-addition identities, and cube
// roots use cbrt; both agree with the reference's cos/pow(.,1/3) to rounding.
__device__ __forceinline__ double solve_z(double a1, double a2, double a3, bool gas) {
    double Q = qdivc(3 * a2 - a1 * a1, 9.0, 1.0 / 9.0);
    double J = qdivc(9 * a1 * a2 - 27 * a3 - 2 * a1 * a1 * a1, 54.0, 1.0 / 54.0);
    double D = Q * Q * Q + J * J;
    double Z;
    if (D < 0) {
        double s = 2 * sqrt(-Q);
        double a13 = qdivc(a1, 3.0, 1.0 / 3.0);
        double t = qdivc(acos(J / sqrt(-Q * Q * Q)), 3.0, 1.0 / 3.0);
        double st, ct;
        sincos(t, &st, &ct);
        // cos(t + 2pi/3) and cos(t + 4pi/3)
        constexpr double c23 = -0.5;
        constexpr double s23 = 0.86602540378443864676;  // sin(2 pi / 3)
        double r1 = s * ct - a13;
        double r2 = s * (ct * c23 - st * s23) - a13;
        double r3 = s * (ct * c23 + st * s23) - a13;
        if (gas) {
            if ((r1 >= r2) && (r1 >= r3)) Z = r1;
            else if ((r2 >= r1) && (r2 >= r3)) Z = r2;
            else Z = r3;
        } else {
            if ((r1 <= r2) && (r1 <= r3) && (r1 > 0)) Z = r1;
            else if ((r2 <= r1) && (r2 <= r3) && (r2 > 0)) Z = r2;
            else Z = r3;
        }
    } else if (D == 0) {
        double t = cbrt(J);
        double r1 = 2 * t - qdivc(a1, 3.0, 1.0 / 3.0);
        double r2 = -t - qdivc(a1, 3.0, 1.0 / 3.0);
        if (gas) Z = (r2 >= r1) ? r2 : r1;
        else Z = ((r2 <= r1) && (r2 > 0)) ? r2 : r1;
    } else {
        double s = sqrt(D);
        Z = cbrt(J + s) + cbrt(J - s) - qdivc(a1, 3.0, 1.0 / 3.0);
    }
    return Z;
}

// Cubic coefficients for Z^3 + a1 Z^2 + a2 Z + a3 with U, W the EOS's
// (PR: U = 2B, W = B; SRK: U = B, W = 0), compsim/Init_Calcs.cpp:657-675.
__device__ __forceinline__ double phase_z(double A, double B, bool srk, bool gas) {
    double U = srk ? B : 2 * B;
    double W = srk ? 0.0 : B;
    return solve_z(-(1 + B - U), A - B * U - U - W * W, -(A * B - B * W * W - W * W), gas);
}

}  // namespace osr

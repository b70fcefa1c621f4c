"""Algorithmic FP64 operation counts of the flash, frozen from the kernel source
(osiris_b200/csrc/flash_kernels.cuh, eos_device.cuh).

Counting convention (one FP64 "flop" unit):
  add, sub, mul, compare-free select ... 1
  fused multiply-add ..................... 2
  divide, sqrt ........................... 4   (hardware seed + Newton refinement)
  exp, log, cbrt ......................... 20  (range reduction + polynomial)
  acos, sincos ........................... 30
Every cubic solve is charged the three-real-root (trigonometric) branch.
Counts are per cell and depend on the kernel-reported iteration numbers:

  flops(cell) = INIT(N) + n_ss * SS(N) + n_rr * RR(N) [+ DERIV(N)]

with n_ss the successive-substitution steps and n_rr the Rachford-Rice
Newton steps that cell took.  The roofline's achieved rate is the sum over
all cells divided by the kernels' measured time; ncu's executed FP64
instruction counts are the cross-check.
"""
from __future__ import annotations

import numpy as np

W_DIV = 4
W_SQRT = 4
W_EXPLOG = 20
W_TRIG = 30


def rr_step(n: int) -> int:
    """One Newton step on the Rachford-Rice function: per component
    (1-K) 1, L+(1-L)K fma 2, divide, z*td 1, F+= 1, dF fma 2; plus (1-L),
    F/dF, L-=t, t*t."""
    return n * (1 + 2 + W_DIV + 1 + 1 + 2) + 1 + W_DIV + 1 + 1


def cubic() -> int:
    """Coefficients (8), Q (4 + div), J (7 + div), D (3), 2 sqrt, a1/3 div,
    acos, /3 div, sincos, three roots (9), selection (3)."""
    return 8 + (4 + W_DIV) + (7 + W_DIV) + 3 + 2 * W_SQRT + W_DIV + W_TRIG + W_DIV + W_TRIG + 9 + 3


def ss_step(n: int) -> int:
    """Clamp and |dL| (3); x, y (per component fma + divide + mul, plus 1-L);
    u (2N); v = (1-k) u for both phases (2N^2 fma); Ca, Cb (4N fma); P/(RT)^2,
    P/(RT) (3 mul + 2 div); A, B (4); two cubics; DD (2 mul + 2 div), FF
    (2 x (2 fma + div + log)), log(Z-B) (2 x (1 + log)), four reciprocals,
    DD*FF (2); per component: t1 (2), EE (2 x (mul + fma)), exponent
    (2 x (1 + fma + 1)), two exp, f = w phi (2), K *= fL/fG (div + mul)."""
    per_comp = 2 + 2 * (1 + 2) + 2 * (1 + 2 + 1) + 2 * W_EXPLOG + 2 + (W_DIV + 1)
    return (3 + n * (2 + W_DIV + 1) + 1 + 2 * n + 2 * (2 * n * n) + 4 * (2 * n) + (3 + 2 * W_DIV) + 4
            + 2 * cubic() + (2 + 2 * W_DIV) + 2 * (4 + W_DIV + W_EXPLOG) + 2 * (1 + W_EXPLOG) + 4 * W_DIV + 2
            + n * per_comp)


def init(n: int) -> int:
    """Wilson K (P div, Tc/T div, 1-., mul, exp, mul) and sqrt(a_i(T))
    (T/Tc div, sqrt, 1-., fma, 2 mul, sqrt) per component."""
    return n * ((W_DIV + W_DIV + 1 + 1 + W_EXPLOG + 1) + (W_DIV + W_SQRT + 1 + 2 + 2 + W_SQRT))


def deriv_phase(n: int) -> int:
    """One phase of the derivative pass: sqrt(a_i(T)) (as in init), u (N),
    v (N^2 fma), Ca/Cb (2N fma), scalar set-up (~4 div + log + 40), per k
    (dA, dB, dZ, dDD, dFF, P1..P4: ~34), per i (t, t1, EE, dP row, g: ~20),
    per (i, k) (4 fma + 2 mul = 10)."""
    return (n * (W_DIV + W_SQRT + 1 + 2 + 2 + W_SQRT) + n + 2 * n * n + 4 * n + (9 * W_DIV + W_EXPLOG + 40)
            + 34 * n + 20 * n + 10 * n * n)


def flash_flops(n: int, iters, rr_iters, derivs: bool = True) -> float:
    """Total algorithmic FP64 flops of a flash batch from per-cell counters."""
    iters = np.asarray(iters, dtype=np.float64)
    rr_iters = np.asarray(rr_iters, dtype=np.float64)
    cells = iters.shape[0]
    tot = cells * init(n) + iters.sum() * ss_step(n) + rr_iters.sum() * rr_step(n)
    if derivs:
        tot += cells * 2 * deriv_phase(n)
    return float(tot)


def flash_kernel_flops(n: int, iters, rr_iters) -> float:
    """Flops of the iteration kernel alone (no derivative pass)."""
    return flash_flops(n, iters, rr_iters, derivs=False)


def deriv_kernel_flops(n: int, cells: int) -> float:
    return float(cells * 2 * deriv_phase(n))

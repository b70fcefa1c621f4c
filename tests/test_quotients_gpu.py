"""Accuracy of the flash kernels' branch-free quotient and reciprocal.

qdiv / qrcp (osiris_b200/csrc/eos_device.cuh) refine the hardware
reciprocal seed by Newton-Raphson and correct the quotient with its residual
(Markstein).  Through osr_probe_quotients they run on 10^7 random operand
pairs (magnitudes log-uniform over 1e-300..1e300, both signs) and on the
edge bands of the range their callers accept without the IEEE fallback
(|b| just above 9.33e-302 and just below 1.07e301, |a| just below 1.07e301,
quotients in the subnormal range, |b| near powers of two).  Bar: within one
ulp of IEEE a / b and 1 / b for every pair inside that range whose quotient
does not overflow (a quotient beyond the largest double is outside the
flash's values; the callers' operands are compositions, K-values and
Rachford-Rice terms).  The predicate itself must match its definition.
"""
import numpy as np
import pytest

import osiris_b200 as osr

pytestmark = pytest.mark.gpu

N_RANDOM = 10_000_000


def _ulps(got, ref):
    """ulp distance of finite doubles (ordered integer representation)."""
    def key(v):
        i = v.view(np.int64)
        return np.where(i < 0, np.int64(-0x8000000000000000) - i, i)
    return np.abs(key(got) - key(ref))


def _operands(rng):
    def logu(n, lo, hi):
        return np.exp(rng.uniform(np.log(lo), np.log(hi), n)) * rng.choice([-1.0, 1.0], n)
    a = [logu(N_RANDOM, 1e-300, 1e300)]
    b = [logu(N_RANDOM, 1e-300, 1e300)]
    m = 200_000
    lo_b, hi_b, hi_a = 9.33e-302, 1.07e301, 1.07e301
    # |b| just inside both ends of the accepted range, with ordinary numerators
    a += [logu(m, 1e-3, 1e3), logu(m, 1e-3, 1e3)]
    b += [lo_b * (1 + rng.uniform(1e-15, 1e-3, m)) * rng.choice([-1.0, 1.0], m),
          hi_b * (1 - rng.uniform(1e-15, 1e-3, m)) * rng.choice([-1.0, 1.0], m)]
    # |a| just below its bound over large divisors (no overflow)
    a.append(hi_a * (1 - rng.uniform(1e-15, 1e-3, m)) * rng.choice([-1.0, 1.0], m))
    b.append(logu(m, 1e2, 1e300))
    # quotients in the subnormal range and at the normal/subnormal boundary
    a.append(logu(m, 1e-300, 1e-290))
    b.append(logu(m, 1e10, 1e30))
    # divisors at and next to powers of two (seed table boundaries)
    e = rng.integers(-990, 990, m).astype(np.float64)
    b.append(np.ldexp(1.0, e.astype(int)) * (1 + rng.choice([0.0, 2.0 ** -52, -2.0 ** -53, 2.0 ** -30], m)))
    a.append(logu(m, 1e-3, 1e3))
    return np.concatenate(a), np.concatenate(b)


def test_quotients_within_one_ulp_of_ieee(cuda_device):
    import torch
    rng = np.random.default_rng(11)
    a, b = _operands(rng)
    n = len(a)
    da, db = torch.from_numpy(a).to(cuda_device), torch.from_numpy(b).to(cuda_device)
    q = torch.empty_like(da)
    r = torch.empty_like(da)
    ok = torch.empty(n, dtype=torch.int8, device=cuda_device)
    rc = osr.lib().osr_probe_quotients(da.data_ptr(), db.data_ptr(), n, q.data_ptr(), r.data_ptr(), ok.data_ptr(),
                                       torch.cuda.current_stream().cuda_stream)
    assert rc == 0, osr.lib().osr_status_string(rc)
    torch.cuda.synchronize()
    q, r, ok = q.cpu().numpy(), r.cpu().numpy(), ok.cpu().numpy().astype(bool)
    with np.errstate(over="ignore", under="ignore"):
        qi, ri = a / b, 1.0 / b
    expect_ok = (np.abs(b) > 9.33e-302) & (np.abs(b) < 1.07e301) & (np.abs(a) < 1.07e301)
    assert np.array_equal(ok, expect_ok)
    use = ok & np.isfinite(qi)
    # pairs whose quotient overflows (about 12% of the log-uniform draw) are
    # outside the flash's values and are left out
    assert use.sum() > 0.85 * n
    dq = _ulps(q[use], qi[use])
    dr = _ulps(r[use], ri[use])
    print(f"{use.sum()} pairs: qdiv exact {np.mean(dq == 0):.6f}, max {dq.max()} ulp; "
          f"qrcp exact {np.mean(dr == 0):.6f}, max {dr.max()} ulp")
    assert dq.max() <= 1, [(a[use][i], b[use][i], q[use][i], qi[use][i]) for i in np.argsort(-dq)[:4]]
    assert dr.max() <= 1, [(b[use][i], r[use][i], ri[use][i]) for i in np.argsort(-dr)[:4]]

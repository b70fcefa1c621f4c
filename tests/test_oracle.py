"""CPU tests of the restated oracle (oracle/flash_oracle.c).

The oracle is pinned two ways: bit for bit against the golden fixtures made
by the reference's own SuccFalsh (tests/golden/make_golden.py), and, where
the reference library was built in this checkout, against it directly on
fresh seeded cells.  Its fugacity derivatives, which the reference never
exposes on their own, are pinned by central finite differences of its own
ln(phi).
"""
import numpy as np
import pytest

import oracle
from osiris_b200 import workloads


def _fluid(g):
    return oracle.Fluid(g["tc"], g["pc"], g["acf"], g["kij"], int(g["eos"]))


@pytest.mark.parametrize("name", ["golden_srk6", "golden_pr3"])
def test_oracle_matches_reference_golden_bitwise(name, request):
    g = request.getfixturevalue(name)
    fl = _fluid(g)
    o = oracle.flash_batch(fl, g["P"], g["T"], g["z"])
    assert np.array_equal(o["label"], g["label"])
    assert np.array_equal(o["x"], g["x"])
    assert np.array_equal(o["y"], g["y"])
    so, sg, ro, rg = oracle.derived_sat_rho(o, g["P"], g["T"])
    assert np.array_equal(so, g["sat_o"])
    assert np.array_equal(sg, g["sat_g"])
    assert np.array_equal(ro, g["rho_o"])
    assert np.array_equal(rg, g["rho_g"])


def test_golden_covers_all_phase_states(golden_srk6, golden_pr3):
    for g in (golden_srk6, golden_pr3):
        assert set(np.unique(g["label"])) == {-1, 0, 1}


@pytest.mark.skipif(not oracle.ref_available(), reason="reference library not built here")
@pytest.mark.parametrize("eos", [0, 1])
def test_oracle_matches_reference_fresh_cells(eos):
    tc, pc, acf, kij = workloads.flash_table(8, 21 + eos)
    fl = oracle.Fluid(tc, pc, acf, kij, eos)
    P, T, z = workloads.flash_cells(1500, 8, seed=31 + eos)
    o = oracle.flash_batch(fl, P, T, z)
    r = oracle.ref_flash_batch(fl, P, T, z)
    assert np.array_equal(o["label"], r["label"])
    assert np.array_equal(o["x"], r["x"])
    assert np.array_equal(o["y"], r["y"])


@pytest.mark.skipif(not oracle.ref_available(), reason="reference library not built here")
def test_solve_z_matches_reference_root_rule():
    rng = np.random.default_rng(5)
    for _ in range(3000):
        A = rng.uniform(0.01, 3.0)
        B = rng.uniform(0.001, 0.3)
        for srk in (0, 1):
            U, W = (B, 0.0) if srk else (2 * B, B)
            a1, a2, a3 = -(1 + B - U), A - B * U - U - W * W, -(A * B - B * W * W - W * W)
            for gas in (False, True):
                assert oracle.solve_z(a1, a2, a3, gas) == oracle.ref_solve_z(a1, a2, a3, gas)


@pytest.mark.skipif(not oracle.ref_available(), reason="reference library not built here")
@pytest.mark.parametrize("eos", [0, 1])
def test_eos_params_match_reference(eos):
    tc, pc, acf, kij = workloads.flash_table(6, 2)
    fl = oracle.Fluid(tc, pc, acf, kij, eos)
    for T in (300.0, 377.7, 450.0):
        a, b = oracle.eos_params(fl, T)
        ra, rb = oracle.ref_eos_params(fl, T)
        assert np.array_equal(a, ra) and np.array_equal(b, rb)


def _phase_z(fl, P, T, w, gas):
    a, b = oracle.eos_params(fl, T)
    aij = np.sqrt(np.outer(a, a)) * (1 - fl.kij)
    R = oracle.R_GAS
    A = (w @ aij @ w) * P / (R * R * T * T)
    B = (w @ b) * P / (R * T)
    U, W = (B, 0.0) if fl.eos else (2 * B, B)
    return oracle.solve_z(-(1 + B - U), A - B * U - U - W * W, -(A * B - B * W * W - W * W), gas)


@pytest.mark.parametrize("eos", [0, 1])
def test_fugacity_derivatives_central_fd(eos):
    """d ln(phi)/dw_k and d ln(phi)/dP of the oracle against central
    differences of its own ln(phi) (relative step 1e-6)."""
    tc, pc, acf, kij = workloads.flash_table(5, 9)
    fl = oracle.Fluid(tc, pc, acf, kij, eos)
    rng = np.random.default_rng(13)
    checked = 0
    for _ in range(40):
        P = rng.uniform(5e6, 40e6)
        T = rng.uniform(300, 450)
        w = rng.dirichlet(np.ones(5))
        for gas in (False, True):
            Z = _phase_z(fl, P, T, w, gas)
            if not np.isfinite(Z) or Z <= 0:
                continue
            _, dx, dp = oracle.fugacity(fl, P, T, w, Z)
            for k in range(5):
                h = 1e-6 * max(w[k], 1e-3)
                wp, wm = w.copy(), w.copy()
                wp[k] += h
                wm[k] -= h
                lp, _, _ = oracle.fugacity(fl, P, T, wp, _phase_z(fl, P, T, wp, gas))
                lm, _, _ = oracle.fugacity(fl, P, T, wm, _phase_z(fl, P, T, wm, gas))
                fd = (lp - lm) / (2 * h)
                np.testing.assert_allclose(dx[:, k], fd, rtol=2e-5, atol=2e-6 * np.abs(fd).max())
            hP = 1e-6 * P
            lp, _, _ = oracle.fugacity(fl, P + hP, T, w, _phase_z(fl, P + hP, T, w, gas))
            lm, _, _ = oracle.fugacity(fl, P - hP, T, w, _phase_z(fl, P - hP, T, w, gas))
            np.testing.assert_allclose(dp, (lp - lm) / (2 * hP), rtol=2e-5, atol=1e-16)
            checked += 1
    assert checked > 40


def test_oracle_empty_batch():
    tc, pc, acf, kij, eos = workloads.flash_fluid_srk6()
    fl = oracle.Fluid(tc, pc, acf, kij, eos)
    o = oracle.flash_batch(fl, np.zeros(0), np.zeros(0), np.zeros((6, 0)))
    assert o["label"].shape == (0,)


def test_reference_algorithm_rounding_sensitivity_meets_the_bar(golden_srk6):
    """The restated oracle compiled with fused multiply-add (a pure rounding
    change) meets the same two-tier bar the CUDA path is held to, and moves
    some cells beyond 1e-10: the bar's loose tier is the reference algorithm's
    own reproducibility, not slack for the GPU."""
    from osiris_b200 import workloads as w
    moved = 0
    for eos, nc, seed in [(1, 6, 3), (0, 8, 4), (0, 12, 6)]:
        tc, pc, acf, kij = w.flash_table(nc, 100 + seed)
        fl = oracle.Fluid(tc, pc, acf, kij, eos)
        P, T, z = w.flash_cells(6000, nc, seed=seed)
        o = oracle.flash_batch(fl, P, T, z)
        f = oracle.flash_batch(fl, P, T, z, fma=True)
        r = oracle.flash_parity(f, o)
        assert r["ok"], r
        moved += r["margin"].size
    assert moved > 0

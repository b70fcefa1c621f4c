"""The flash adjoint (osr_flash_adjoint) behind a torch.autograd.Function,
checked against central finite differences and against the oracle's
restatement.

The device flash's result u = (x, y, L) of a two-phase cell solves the
equal-fugacity, material-balance and Rachford-Rice equations to the
reference's stopping tolerances; the adjoint differentiates that equilibrium.
Finite differences of the reference's iteration itself carry the noise of
its stopping rules (a Rachford-Rice Newton truncated at step^2 <= 1e-8 moves
compositions by ~1e-9, more than h^2), so the finite differences here are of
the oracle's flash polished to rounding by Newton's method on the same
equations (oracle.flash_polish): the derivatives of the exact equilibrium.

Workload: SRK, 6 components (the batched flash's seeded table), 3,000 cells
of the batched flash's P/T/z draw; objective = sum of seeded random
cotangents times x, y, L over two-phase cells plus the present phase of
one-phase cells (whose composition is the feed).  Bars:
  * directional derivatives along 32 seeded kij directions (zero diagonal)
    against central differences with h = 1e-6, within 1e-6 of the
    direction's scale sum |g_ij V_ij| (the size of the terms the derivative
    sums; a direction whose derivative cancels to a small fraction of it
    magnifies the differences' rounding and the state's distance from the
    equilibrium by as much -- the relative error is printed as well): the
    device adjoint evaluated at the polished equilibrium, and the gradient
    through the autograd function at the device flash's own result
    (stopped by the reference's tolerances, ~1e-9 from the equilibrium);
  * z and P directions through the autograd function within 1e-5 relative;
  * the device's kij_bar, z_bar and P_bar within 1e-10 of the oracle's
    adjoint at the same state.
"""
import numpy as np
import pytest

import oracle
import osiris_b200 as osr
from osiris_b200 import workloads

pytestmark = pytest.mark.gpu

H = 1e-6
N_DIRECTIONS = 32


class FlashEquilibrium:
    """torch.autograd.Function over the device flash: (kij, z, P) -> (x, y, L)
    with the backward pass through osr_flash_adjoint.  Test harness only."""

    @staticmethod
    def make(tc, pc, acf, eos, T):
        import torch

        class Fn(torch.autograd.Function):
            @staticmethod
            def forward(ctx, kij, z, P):
                fl = osr.Fluid(tc, pc, acf, kij.detach().cpu().numpy(), eos)
                out = osr.flash(fl, P.detach().contiguous(), T, z.detach().contiguous(), derivs=False)
                ctx.fl, ctx.out = fl, out
                ctx.save_for_backward(z, P)
                return out["x"].clone(), out["y"].clone(), out["L"].clone()

            @staticmethod
            def backward(ctx, gx, gy, gL):
                z, P = ctx.saved_tensors
                r = osr.flash_adjoint(ctx.fl, P.detach().contiguous(), T, z.detach().contiguous(), ctx.out,
                                      gx.contiguous(), gy.contiguous(), gL.contiguous())
                assert r["singular"] == 0
                return r["kij_bar"].cpu(), r["z_bar"], r["P_bar"]

        return Fn


def _workload():
    tc, pc, acf, kij, eos = workloads.flash_fluid_srk6()
    P, T, z = workloads.flash_cells(3000, 6, seed=23)
    return tc, pc, acf, kij, eos, P, T, z


def _cotangents(label, nc, seed=7):
    """Seeded cotangents on the values that depend smoothly on the inputs:
    everything of a two-phase cell, the present phase of a one-phase cell."""
    rng = np.random.default_rng(seed)
    n = label.shape[0]
    xb, yb, Lb = rng.standard_normal((nc, n)), rng.standard_normal((nc, n)), rng.standard_normal(n)
    xb[:, label < 0] = 0
    yb[:, label > 0] = 0
    Lb[label != 0] = 0
    return xb, yb, Lb


def _polished(fl, P, T, z):
    r = oracle.flash_batch(fl, P, T, z)
    bad = oracle.flash_polish(fl, P, T, z, r)
    assert bad == 0
    return r


def _objective(r, xb, yb, Lb):
    return float((xb * r["x"]).sum() + (yb * r["y"]).sum() + (Lb * r["L"]).sum())


@pytest.fixture(scope="module")
def setup(cuda_device):
    import torch
    tc, pc, acf, kij, eos, P, T, z = _workload()
    fl = oracle.Fluid(tc, pc, acf, kij, eos)
    base = oracle.flash_batch(fl, P, T, z)
    # cells that stopped at the 500-step cap are not at the equilibrium
    keep = base["iters"] < 500
    P, T, z = P[keep], T[keep], np.ascontiguousarray(z[:, keep])
    ref = _polished(fl, P, T, z)
    dev = cuda_device
    tP, tT, tz = (torch.from_numpy(a).to(dev) for a in (P, T, z))
    xb, yb, Lb = _cotangents(ref["label"], 6)
    return dict(tc=tc, pc=pc, acf=acf, kij=kij, eos=eos, P=P, T=T, z=z, tP=tP, tT=tT, tz=tz, ref=ref, xb=xb, yb=yb,
                Lb=Lb, dev=dev)


def _directions(seed=5):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(N_DIRECTIONS):
        V = rng.standard_normal((6, 6))
        np.fill_diagonal(V, 0)
        out.append(V)
    return out


def _fd(s, V):
    fp = oracle.Fluid(s["tc"], s["pc"], s["acf"], s["kij"] + H * V, s["eos"])
    fm = oracle.Fluid(s["tc"], s["pc"], s["acf"], s["kij"] - H * V, s["eos"])
    rp, rm = _polished(fp, s["P"], s["T"], s["z"]), _polished(fm, s["P"], s["T"], s["z"])
    assert np.array_equal(rp["label"], s["ref"]["label"]) and np.array_equal(rm["label"], s["ref"]["label"])
    return (_objective(rp, s["xb"], s["yb"], s["Lb"]) - _objective(rm, s["xb"], s["yb"], s["Lb"])) / (2 * H)


def test_device_adjoint_at_equilibrium_matches_central_differences(setup):
    """osr_flash_adjoint at the polished equilibrium against central
    differences of the polished flash: 32 kij directions, 1e-6 relative."""
    import torch
    s = setup
    d = s["dev"]
    fl = osr.Fluid(s["tc"], s["pc"], s["acf"], s["kij"], s["eos"])
    st = {k: torch.from_numpy(np.ascontiguousarray(s["ref"][k])).to(d) for k in ("label", "L", "x", "y", "Zl", "Zg")}
    r = osr.flash_adjoint(fl, s["tP"], s["tT"], s["tz"], st, torch.from_numpy(s["xb"]).to(d),
                          torch.from_numpy(s["yb"]).to(d), torch.from_numpy(s["Lb"]).to(d))
    g = r["kij_bar"].cpu().numpy()
    worst = worst_rel = 0.0
    for q, V in enumerate(_directions()):
        fd = _fd(s, V)
        ad = float((g * V).sum())
        err = abs(ad - fd) / float(np.abs(g * V).sum())
        worst = max(worst, err)
        worst_rel = max(worst_rel, abs(ad - fd) / abs(fd))
        assert err <= 1e-6, (q, ad, fd, err)
    print(f"kij at the equilibrium: {N_DIRECTIONS} directions, worst difference {worst:.2e} of the direction's "
          f"scale ({worst_rel:.2e} of the derivative)")


def test_kij_gradient_matches_central_differences(setup):
    import torch
    s = setup
    Fn = FlashEquilibrium.make(s["tc"], s["pc"], s["acf"], s["eos"], s["tT"])
    k = torch.tensor(s["kij"], dtype=torch.float64, requires_grad=True)
    zt = s["tz"].clone().requires_grad_(True)
    Pt = s["tP"].clone().requires_grad_(True)
    x, y, L = Fn.apply(k, zt, Pt)
    d = s["dev"]
    obj = (torch.from_numpy(s["xb"]).to(d) * x).sum() + (torch.from_numpy(s["yb"]).to(d) * y).sum() + \
        (torch.from_numpy(s["Lb"]).to(d) * L).sum()
    obj.backward()
    g = k.grad.numpy()
    worst = worst_rel = 0.0
    for q, V in enumerate(_directions()):
        fd = _fd(s, V)
        ad = float((g * V).sum())
        scale = float(np.abs(g * V).sum())
        err = abs(ad - fd) / scale
        worst = max(worst, err)
        worst_rel = max(worst_rel, abs(ad - fd) / abs(fd))
        assert err <= 1e-6, (q, ad, fd, err)
    print(f"kij through autograd at the flash's result: {N_DIRECTIONS} directions, worst difference {worst:.2e} of "
          f"the direction's scale ({worst_rel:.2e} of the derivative)")
    rng = np.random.default_rng(6)
    # z and P through the same autograd graph
    # P steps of about 1 Pa on 5-40 MPa: smaller steps drown in the polish's rounding
    for name, t, scale in (("z", zt, 1e-3), ("P", Pt, 1e6)):
        grad = t.grad.cpu().numpy()
        V = rng.standard_normal(grad.shape) * scale
        base = s[name]
        fl = oracle.Fluid(s["tc"], s["pc"], s["acf"], s["kij"], s["eos"])
        args_p = dict(P=s["P"], T=s["T"], z=s["z"])
        args_m = dict(args_p)
        args_p[name] = base + H * V
        args_m[name] = base - H * V
        rp = _polished(fl, args_p["P"], args_p["T"], np.ascontiguousarray(args_p["z"]))
        rm = _polished(fl, args_m["P"], args_m["T"], np.ascontiguousarray(args_m["z"]))
        fd = (_objective(rp, s["xb"], s["yb"], s["Lb"]) - _objective(rm, s["xb"], s["yb"], s["Lb"])) / (2 * H)
        ad = float((grad * V).sum())
        err = abs(ad - fd) / abs(fd)
        print(f"{name}: adjoint {ad:.12e}, central difference {fd:.12e}, relative {err:.2e}")
        assert err <= 1e-5, (name, ad, fd)


def test_device_adjoint_matches_oracle_restatement(setup):
    import torch
    s = setup
    fl = osr.Fluid(s["tc"], s["pc"], s["acf"], s["kij"], s["eos"])
    out = osr.flash(fl, s["tP"], s["tT"], s["tz"], derivs=False)
    d = s["dev"]
    r = osr.flash_adjoint(fl, s["tP"], s["tT"], s["tz"], out, torch.from_numpy(s["xb"]).to(d),
                          torch.from_numpy(s["yb"]).to(d), torch.from_numpy(s["Lb"]).to(d))
    torch.cuda.synchronize()
    st = {k: v.cpu().numpy() for k, v in out.items()}
    kb, zb, pb, bad = oracle.flash_adjoint(oracle.Fluid(s["tc"], s["pc"], s["acf"], s["kij"], s["eos"]), s["P"],
                                           s["T"], s["z"], st, s["xb"], s["yb"], s["Lb"])
    assert bad == 0 and r["singular"] == 0
    g = r["kij_bar"].cpu().numpy()
    assert np.abs(g - kb).max() <= 1e-10 * np.abs(kb).max(), np.abs(g - kb).max() / np.abs(kb).max()
    zg, pg = r["z_bar"].cpu().numpy(), r["P_bar"].cpu().numpy()
    assert np.abs(zg - zb).max() <= 1e-10 * np.abs(zb).max()
    assert np.abs(pg - pb).max() <= 1e-10 * np.abs(pb).max()
    # one-phase cells: the present phase's cotangent goes to the feed
    lab = st["label"]
    assert np.array_equal(zg[:, lab > 0], s["xb"][:, lab > 0])
    assert np.array_equal(zg[:, lab < 0], s["yb"][:, lab < 0])
    # the kij sum is deterministic
    r2 = osr.flash_adjoint(fl, s["tP"], s["tT"], s["tz"], out, torch.from_numpy(s["xb"]).to(d),
                           torch.from_numpy(s["yb"]).to(d), torch.from_numpy(s["Lb"]).to(d))
    assert torch.equal(r2["kij_bar"], r["kij_bar"])


@pytest.mark.parametrize("eos,nc,seed", [(0, 8, 31), (1, 3, 32), (0, 12, 33)])
def test_adjoint_other_component_counts(eos, nc, seed, cuda_device):
    """PR with 8 and 12 components, SRK with 3: the device adjoint equals the
    oracle's restatement, and one kij direction matches central differences."""
    import torch
    tc, pc, acf, kij = workloads.flash_table(nc, 200 + seed)
    P, T, z = workloads.flash_cells(1500, nc, seed=seed)
    fo = oracle.Fluid(tc, pc, acf, kij, eos)
    base = oracle.flash_batch(fo, P, T, z)
    keep = base["iters"] < 500
    P, T, z = P[keep], T[keep], np.ascontiguousarray(z[:, keep])
    dev = cuda_device
    fl = osr.Fluid(tc, pc, acf, kij, eos)
    tP, tT, tz = (torch.from_numpy(a).to(dev) for a in (P, T, z))
    out = osr.flash(fl, tP, tT, tz, derivs=False)
    st = {k: v.cpu().numpy() for k, v in out.items()}
    xb, yb, Lb = _cotangents(st["label"], nc, seed)
    r = osr.flash_adjoint(fl, tP, tT, tz, out, *(torch.from_numpy(a).to(dev) for a in (xb, yb, Lb)))
    kb, _, _, bad = oracle.flash_adjoint(fo, P, T, z, st, xb, yb, Lb)
    g = r["kij_bar"].cpu().numpy()
    assert bad == 0 and r["singular"] == 0
    assert np.abs(g - kb).max() <= 1e-10 * np.abs(kb).max()
    rng = np.random.default_rng(seed)
    V = rng.standard_normal((nc, nc))
    np.fill_diagonal(V, 0)
    rp = _polished(oracle.Fluid(tc, pc, acf, kij + H * V, eos), P, T, z)
    rm = _polished(oracle.Fluid(tc, pc, acf, kij - H * V, eos), P, T, z)
    fd = (_objective(rp, xb, yb, Lb) - _objective(rm, xb, yb, Lb)) / (2 * H)
    ad = float((g * V).sum())
    assert abs(ad - fd) <= 1e-6 * abs(fd), (ad, fd)

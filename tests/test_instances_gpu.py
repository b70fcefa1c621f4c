"""GPU parity of the multi-instance batched flash (osr_flash_batch_instances).

Instances of every component count 3..12 with both equations of state, each
with its own seeded component table and an uneven cell count (a few to a
few hundred cells), flashed in one batched call per component count.  Each
instance's slice must agree with osr_flash_batch on that slice with that
instance's fluid: labels identical and the flash bar of the single-fluid
tests (the two kernel instantiations read the table from different memory
spaces, so the compiler's multiply-add contraction may differ by an ulp);
fugacity derivatives within 1e-10 of each block's largest entry.  A sample
of instances is also held to the oracle bar.
"""
import numpy as np
import pytest

import oracle
import osiris_b200 as osr
from osiris_b200 import workloads

pytestmark = pytest.mark.gpu

STATE = ("label", "L", "x", "y", "Zl", "Zg")


def _slice(v, a, b):
    return v[..., a:b]


def _assert_agree(mine, ref, where):
    n = mine["label"].shape[-1]
    r = oracle.flash_parity({k: mine[k] for k in STATE}, {k: ref[k] for k in STATE})
    assert r["labels_equal"] and r["wide_ok"], where
    assert len(r["margin"]) <= max(1, 0.005 * n), (where, r["margin"][:5])


@pytest.mark.parametrize("nc", list(range(3, 13)))
def test_instances_match_single_fluid_calls(nc, cuda_device):
    import torch
    insts = [d for d in workloads.batched_instances(n_inst=200, seed=11, cells_lo=3, cells_hi=400) if d["nc"] == nc]
    assert len(insts) >= 2 and len({d["eos"] for d in insts}) == 2
    members, start, P, T, z = workloads.instance_group(insts, nc, seed=7)
    dev = cuda_device
    tP, tT, tz = (torch.from_numpy(a).to(dev) for a in (P, T, z))
    fluids = [osr.Fluid(d["tc"], d["pc"], d["acf"], d["kij"], d["eos"]) for d in members]
    out = osr.flash_instances(fluids, start, tP, tT, tz, derivs=True)
    torch.cuda.synchronize()
    got = {k: v.cpu().numpy() for k, v in out.items()}
    for i, f in enumerate(fluids):
        a, b = int(start[i]), int(start[i + 1])
        one = osr.flash(f, tP[a:b].contiguous(), tT[a:b].contiguous(), tz[:, a:b].contiguous(), derivs=True)
        torch.cuda.synchronize()
        ref = {k: v.cpu().numpy() for k, v in one.items()}
        mine = {k: _slice(v, a, b) for k, v in got.items()}
        _assert_agree(mine, ref, (nc, i, "single-fluid call"))
        # derivatives against the oracle at this path's own converged state
        d = members[i]
        ofl = oracle.Fluid(d["tc"], d["pc"], d["acf"], d["kij"], d["eos"])
        dx, dp = oracle.flash_derivs(ofl, P[a:b], T[a:b], mine["x"], mine["y"], mine["Zl"], mine["Zg"])
        finite = np.isfinite(dx).all(axis=(0, 1, 2))
        ex = np.abs(mine["dlnphi_dx"] - dx)[..., finite] / np.abs(dx).max(axis=(1, 2), keepdims=True)[..., finite]
        ep = np.abs(mine["dlnphi_dP"] - dp)[..., finite] / np.abs(dp).max(axis=1, keepdims=True)[..., finite]
        assert ex.size == 0 or ex.max() <= 1e-10, (nc, i, ex.max())
        assert ep.size == 0 or ep.max() <= 1e-10, (nc, i, ep.max())
        if i % 3 == 0:
            o = oracle.flash_batch(ofl, P[a:b], T[a:b], z[:, a:b])
            _assert_agree(mine, o, (nc, i, "oracle"))


def test_instance_offsets_are_validated(cuda_device):
    import torch
    insts = workloads.batched_instances(n_inst=40, seed=3, cells_lo=5, cells_hi=20)
    nc = insts[0]["nc"]
    members, start, P, T, z = workloads.instance_group(insts, nc)
    fluids = [osr.Fluid(d["tc"], d["pc"], d["acf"], d["kij"], d["eos"]) for d in members]
    tP, tT, tz = (torch.from_numpy(a).to(cuda_device) for a in (P, T, z))
    bad = start.copy()
    bad[-1] += 1
    with pytest.raises(osr.OsrError):
        osr.flash_instances(fluids, bad, tP, tT, tz)


def test_plan_graph_equals_per_group_calls(cuda_device):
    """osr_flash_plan: instance groups of every component count 3..12 as one
    CUDA graph.  Every output of every group equals the group's own
    osr_flash_batch_instances call bit for bit (the same kernels and launch
    shapes), on the first run, on a repeat, and after the inputs are
    refilled in place with another seed."""
    import torch
    insts = workloads.batched_instances(n_inst=120, seed=13, cells_lo=20, cells_hi=3000)
    dev = cuda_device
    groups, refs = [], []
    for nc in sorted({d["nc"] for d in insts}):
        members, start, P, T, z = workloads.instance_group([d for d in insts if d["nc"] == nc], nc, seed=5)
        fluids = [osr.Fluid(d["tc"], d["pc"], d["acf"], d["kij"], d["eos"]) for d in members]
        g = dict(fluids=fluids, start=start, P=torch.from_numpy(P).to(dev), T=torch.from_numpy(T).to(dev),
                 z=torch.from_numpy(z).to(dev))
        g["out"] = osr.alloc_flash_outputs(nc, int(P.shape[0]), True, dev)
        groups.append(g)
    assert len(groups) == 10
    plan = osr.FlashPlan(groups)

    def check():
        torch.cuda.synchronize()
        for g in groups:
            ref = osr.flash_instances(g["fluids"], g["start"], g["P"], g["T"], g["z"], derivs=True)
            torch.cuda.synchronize()
            for k, v in ref.items():
                a, b = g["out"][k], v
                assert torch.equal(torch.nan_to_num(a, nan=7.0), torch.nan_to_num(b, nan=7.0)), k

    plan.run()
    check()
    for g in groups:
        for k in g["out"]:
            g["out"][k].zero_()
    plan.run()
    check()
    for i, g in enumerate(groups):
        _, _, P, T, z = workloads.instance_group([d for d in insts if d["nc"] == g["fluids"][0].nc],
                                                 g["fluids"][0].nc, seed=40 + i)
        g["P"].copy_(torch.from_numpy(P))
        g["T"].copy_(torch.from_numpy(T))
        g["z"].copy_(torch.from_numpy(z))
    plan.run()
    check()
    plan.close()


def test_persistent_launch_equals_graph(cuda_device):
    """osr_flash_plan_run_persistent: the same groups as ONE cooperative
    kernel launch with the device work table.  Every output equals the
    graph form's bit for bit, on repeated runs and on a plan whose groups
    include very small ones (passes that park no cell open and close without
    work), and no wait runs past its bound."""
    import torch
    dev = cuda_device
    for seed, lo, hi in ((13, 20, 3000), (17, 1, 40)):
        insts = workloads.batched_instances(n_inst=120, seed=seed, cells_lo=lo, cells_hi=hi)
        groups = []
        for nc in sorted({d["nc"] for d in insts}):
            members, start, P, T, z = workloads.instance_group([d for d in insts if d["nc"] == nc], nc, seed=5)
            fluids = [osr.Fluid(d["tc"], d["pc"], d["acf"], d["kij"], d["eos"]) for d in members]
            g = dict(fluids=fluids, start=start, P=torch.from_numpy(P).to(dev), T=torch.from_numpy(T).to(dev),
                     z=torch.from_numpy(z).to(dev))
            g["out"] = osr.alloc_flash_outputs(nc, int(P.shape[0]), True, dev)
            groups.append(g)
        plan = osr.FlashPlan(groups)
        plan.run()
        torch.cuda.synchronize()
        ref = [{k: v.clone() for k, v in g["out"].items()} for g in groups]
        for rep in range(3):
            for g in groups:
                for k in g["out"]:
                    g["out"][k].fill_(-7 if g["out"][k].dtype in (torch.int8, torch.int32) else float("nan"))
            plan.run_persistent()
            torch.cuda.synchronize()
            assert plan.persistent_error() == 0
            for g, r in zip(groups, ref):
                for k, v in r.items():
                    assert torch.equal(torch.nan_to_num(g["out"][k], nan=7.0), torch.nan_to_num(v, nan=7.0)), \
                        (seed, rep, g["fluids"][0].nc, k)
        plan.close()

"""GPU parity on the assembly workload's own deck family: the seeded
8-component PR fluid and the two-phase flash state of the dual-porosity
assembly bench, on small grids.

The reference reads the same grid, rock and tables from deck text
(``workloads.assembly_spec``); its component table is then replaced by the
seeded one (``RefDeck.override_fluid``, which redoes EOS_Init and Tr_Mu), and
both sides receive the state the device flash produced
(``workloads.assembly_state``), the reference through its state arrays and
PJac.  Row layout, PCoeff and the unknown vector must agree exactly; residual
rows within 1e-10 of the sum of each row's absolute terms; Jacobian entries
within 1e-9 of the largest entry of the reference's row.  The same setup
gives the bench its sampled-row reference timing.
"""
import os

import numpy as np
import pytest

import oracle
import osiris_b200 as osr
from osiris_b200 import deck, workloads

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not oracle.ref_available(), reason="reference library missing")]

CASES = {
    "6x5x4_cdif0": (6, 5, 4, 0.0),
    "5x4x3_diffusion": (5, 4, 3, None),
}


def open_pair(tmp_path, name, device):
    nx, ny, nz, cdif = CASES[name]
    d = workloads.assembly_deck(nx, ny, nz, cdif=cdif)
    G = osr.Grid(d)
    workloads.assembly_state(G, d, device)
    path = os.path.join(str(tmp_path), name + ".dat")
    deck.write_deck(path, workloads.assembly_spec(d))
    R = oracle.RefDeck(path)
    R.override_fluid(d)
    for mi, m in enumerate("mf"):
        for key in ("P", "sat", "x", "y", "z", "label", "rho"):
            R.set(f"{m}.{key}", G.get(f"{m}.{key}"))
    R.relayout()
    return d, R, G


@pytest.mark.parametrize("name", list(CASES))
def test_assembly_deck_matches_reference(name, tmp_path, cuda_device):
    import torch
    d, R, G = open_pair(tmp_path, name, cuda_device)
    rows, pcoeff = G.refresh_layout()
    assert pcoeff == R.scalar("PCoeff")
    assert np.array_equal(G.row_offsets(), R.get("rowoff").astype(np.int64))
    x0 = R.init_guess()
    d_x = torch.zeros(rows, dtype=torch.float64, device=cuda_device)
    G.init_guess(d_x)
    torch.cuda.synchronize()
    assert np.array_equal(d_x.cpu().numpy(), x0)
    labs = np.concatenate([G.get(f"{m}.label") for m in "mf"])
    assert (labs == 0).all(), "the assembly state is two-phase everywhere"

    t = d.dt
    rng = np.random.default_rng(13)
    xp = x0 * (1 + 1e-3 * rng.uniform(-1, 1, x0.shape))
    # residual
    f_ref = R.form_function(xp, t)
    d_x = torch.tensor(xp, device=cuda_device)
    d_f = torch.zeros(rows, dtype=torch.float64, device=cuda_device)
    d_s = torch.zeros_like(d_f)
    G.form_function(d_x, d_f, t)
    G.residual(d_f, d_s, t)
    torch.cuda.synchronize()
    f, scale = d_f.cpu().numpy(), d_s.cpu().numpy()
    bad = np.abs(f - f_ref) > 1e-10 * scale + 1e-300
    assert not bad.any(), (int(bad.sum()), rows, [(int(r), f[r], f_ref[r]) for r in np.nonzero(bad)[0][:8]])
    # Jacobian
    rr, rc, rv = R.form_jacobian(xp, t)
    Jr = np.zeros((rows, rows))
    np.add.at(Jr, (rr, rc), rv)
    Jb = G.alloc_jacobian(cuda_device)
    assert G.form_jacobian(d_x, Jb, t) == 0
    torch.cuda.synchronize()
    gr, gc, gv = G.jacobian_coo(Jb)
    Jg = np.zeros((rows, rows))
    np.add.at(Jg, (gr, gc), gv)
    row_max = np.maximum(np.abs(Jr).max(axis=1, keepdims=True), 1e-300)
    err = np.abs(Jg - Jr) / row_max
    bad = np.argwhere(~(err <= 1e-9))
    assert len(bad) == 0, (len(bad), [(int(r), int(c), Jg[r, c], Jr[r, c]) for r, c in bad[:8]])

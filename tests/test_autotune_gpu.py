"""The project's flash autotuner (osr_flash_autotune): it times its 48
candidate launch shapes on the caller's batch, keeps the fastest for the
batch's (component count, size bucket) and makes it current; results under
the tuned shape equal the default shape's to the flash bar (the shape only
schedules the same per-cell arithmetic); the tuned table survives a save /
load round trip and is used only when switched on."""
import os

import numpy as np
import pytest

import oracle
import osiris_b200 as osr
from osiris_b200 import workloads

pytestmark = pytest.mark.gpu


def test_autotune_picks_a_candidate_and_keeps_results(tmp_path, cuda_device):
    import torch
    tc, pc, acf, kij, eos = workloads.flash_fluid_srk6()
    f = osr.Fluid(tc, pc, acf, kij, eos)
    P, T, z = workloads.flash_cells(50_000, 6, seed=13)
    dev = cuda_device
    tP, tT, tz = (torch.from_numpy(a).to(dev) for a in (P, T, z))
    shape0, pair0 = osr.get_shape(), osr.get_pair_from()
    ref = {k: v.cpu().numpy() for k, v in osr.flash(f, tP, tT, tz, derivs=False).items()}
    try:
        best = osr.autotune(f, tP, tT, tz)
        assert best["candidates"] == 48 and best["ms"] > 0
        assert best["ss_batch"] in (24, 28) and best["park_after"] in (1, 2, 3)
        assert best["pair_from"] in (4, 5, 6, 12) and best["ctas_per_sm"] in (2, 3)
        assert osr.get_shape()[3] == best["park_after"] and osr.get_pair_from() == best["pair_from"]
        got = {k: v.cpu().numpy() for k, v in osr.flash(f, tP, tT, tz, derivs=False).items()}
        assert oracle.flash_parity(got, ref)["ok"]
        path = os.path.join(str(tmp_path), "tuned.txt")
        osr.tuning_save(path)
        line = open(path).read().split()
        assert [int(v) for v in line[:2]] == [6, 15]   # 50,000 cells: bucket floor(log2 n) = 15
        assert [int(v) for v in line[2:]] == [best["ss_batch"], best["tail_batch"], best["ctas_per_sm"],
                                              best["park_after"], best["pair_from"]]
        # restore the default knobs; the tuned shape applies only when switched on
        osr.set_shape(*shape0)
        osr.set_pair_from(pair0)
        osr.tuning_load(path)
        osr.use_tuned(True)
        got2 = {k: v.cpu().numpy() for k, v in osr.flash(f, tP, tT, tz, derivs=False).items()}
        assert oracle.flash_parity(got2, ref)["ok"]
        with open(path, "w") as fh:
            fh.write("6 15 99 32 3 2 6\n")
        with pytest.raises(osr.OsrError):
            osr.tuning_load(path)
    finally:
        osr.use_tuned(False)
        osr.set_shape(*shape0)
        osr.set_pair_from(pair0)

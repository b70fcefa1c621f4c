"""The time step's CUDA graph (osr_sim_set_graph): from the second pass on,
InitGuess2, FormFunction, FormJacobian, the whole linear solve,
x1 = x0 - dx, the acceptance test and the device-side branch (UpdateAll(x1,
true) + CreateBackups, or RestoreBackups + PJac) run as one graph launch
whose kernels read Dt, the time and PCoeff from device memory.  Two runs of the same deck, one through the graph
and one through direct launches, must take identical passes (accepted or
not, Dt, time, row count, solver iterations and reason, |dx|_1 / rows) and
hold bit-identical states after every pass, through rejections, phase
changes (a new graph per row layout) and the Dt clamps.  The graph must have
served the passes."""
import os

import numpy as np
import pytest

import osiris_b200 as osr
from osiris_b200 import deck

pytestmark = pytest.mark.gpu

CASES = {
    "config1_cdif0": lambda: deck.config_deck(cdif=0.0),
    "twophase_10MPa_rejections": lambda: dict(deck.config_deck(nx=6, ny=5, nz=3, cdif=0.0, ipress=1e7, seed=3),
                                              dt=2.0),
    "sample_12MPa": lambda: deck.sample_deck(),
    "all_well_types_9MPa": lambda: deck.all_wells_deck(),
    # layers of oil at 20 MPa over gas and two-phase fluid at 8 MPa: phase changes from the first passes
    "layered_states": lambda: dict(deck.config_deck(nx=3, ny=3, nz=9, ipress=[2e7 if k % 3 == 1 else 8e6
                                                                              for k in range(9)],
                                                    igc=[(0.5, 0.2, 0.3) if k % 3 != 0 else (0.9, 0.07, 0.03)
                                                         for k in range(9)],
                                                    wells=False, cdif=0.0), dt=0.05),
}
LAYOUT_CHANGES = {"layered_states"}
FIELDS = ("P", "sat", "x", "y", "label")


@pytest.mark.parametrize("name", list(CASES))
def test_graph_passes_equal_direct_launches(name, tmp_path, cuda_device):
    path = os.path.join(str(tmp_path), name + ".dat")
    deck.write_deck(path, CASES[name]())
    runs = []
    for graph in (True, False):
        G = osr.Grid(deck.parse_deck(path))
        G.initialize(cuda_device)
        sim = osr.Sim.from_deck(G)
        sim.set_graph(graph)
        runs.append((G, sim))
    accepted = passes = 0
    layouts = set()
    while accepted < 12 and passes < 40:
        passes += 1
        infos = [sim.step() for _, sim in runs]
        assert infos[0] == infos[1], (passes, infos)
        for f in FIELDS:
            for m in "mf":
                a, b = runs[0][0].get(f"{m}.{f}"), runs[1][0].get(f"{m}.{f}")
                assert np.array_equal(a, b, equal_nan=True), (passes, m, f)
        accepted += infos[0]["accepted"]
        layouts.add(infos[0]["rows"])
        if infos[0]["finished"]:
            break
    assert accepted > 0
    launches = runs[0][1].graph_launches()
    assert launches == passes - 1, (launches, passes)      # every pass after the first
    assert runs[0][1].graph_form() == 2                    # the whole pass, acceptance and UpdateAll included
    assert runs[1][1].graph_launches() == 0
    if name in LAYOUT_CHANGES:
        assert len(layouts) > 1, layouts
    print(f"{name}: {passes} passes, {accepted} accepted, {len(layouts)} row layouts, {launches} graph launches")

"""Decks and constructed one-phase states shared by the phase-appearance
and stability tests: both sides (the reference library and the device grid)
are opened on the same deck and given the same state."""
import os

import numpy as np

import oracle
import osiris_b200 as osr
from osiris_b200 import deck

G_, O_ = (0.9, 0.07, 0.03), (0.5, 0.2, 0.3)
_ST = {-1: (8e6, G_), 1: (2e7, O_), 0: (8e6, O_)}
_PAIRS = [(a, b) for a in (-1, 0, 1) for b in (-1, 0, 1)]

DECKS = {
    "state_pairs": lambda: deck.config_deck(nx=3, ny=3, nz=9, ipress=[_ST[a][0] for a, _ in _PAIRS],
                                            igc=[_ST[a][1] for a, _ in _PAIRS],
                                            fipress=[_ST[b][0] for _, b in _PAIRS],
                                            figc=[_ST[b][1] for _, b in _PAIRS], wells=False, cdif=0.0),
    "sample_6MPa": lambda: deck.sample_deck(ipress=6e6),
    "twophase_8MPa": lambda: deck.config_deck(nx=4, ny=4, nz=3, cdif=None, ipress=8e6, wells=False, seed=8),
}


def open_pair(tmp_path, name):
    path = os.path.join(str(tmp_path), name + ".dat")
    deck.write_deck(path, DECKS[name]())
    R = oracle.RefDeck(path)
    G = osr.Grid(deck.parse_deck(path))
    for mi, m in enumerate("mf"):
        G.set_state(mi, R.get(f"{m}.P")[1], R.get(f"{m}.sat"), R.get(f"{m}.x"), R.get(f"{m}.y"), R.get(f"{m}.z"),
                    R.get(f"{m}.label"), R.get(f"{m}.rho"))
    G.update_dependencies()
    return R, G


def construct_changes(R, G):
    """The same phase-change candidates on both sides (see the module doc)."""
    for mi, m in enumerate("mf"):
        lab = R.get(f"{m}.label").copy()
        sat = R.get(f"{m}.sat").copy()
        x, y, z = R.get(f"{m}.x").copy(), R.get(f"{m}.y").copy(), R.get(f"{m}.z").copy()
        two = np.nonzero(lab == 0)[0]
        for j, c in enumerate(two):
            kind = (j + mi) % 5
            if kind == 0:                      # oil-only with the feed as its composition
                lab[c] = 1
                x[:, c] = z[:, c]
            elif kind == 1:                    # gas-only with the feed as its composition
                lab[c] = -1
                y[:, c] = z[:, c]
            elif kind == 2:                    # vanished oil
                sat[1, c] = 0
                sat[2, c] = 1 - sat[0, c]
            elif kind == 3:                    # vanished gas
                sat[2, c] = 0
                sat[1, c] = 1 - sat[0, c]
        for name, v in (("label", lab), ("sat", sat), ("x", x), ("y", y)):
            R.set(f"{m}.{name}", v)
        G.set_state(mi, G.get(f"{m}.P")[1], sat, x, y, z, lab.astype(np.int8))
        R.set(f"{m}.P", G.get(f"{m}.P"))   # the phase pressures of the device's last property sweep

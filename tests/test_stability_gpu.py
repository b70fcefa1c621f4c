"""GPU parity of the saturation-pressure variants and the stability test that
the reference keeps without live call sites (Bubl_NR, Dew_NR, LowerDew_Succ,
critTest; compsim/Minor_NR.cpp:33-489, 2017-2308) against the reference's own
functions on the same matrix cells.

* Bubl_NR / Dew_NR on every one-phase cell whose device iteration stopped
  (status OK).  The reference iterates without a cap, so a cell the device
  stopped at its cap is not handed to it.  Pressure within 1e-9 relative and
  incipient composition within 1e-9, or both not finite.  Where the Newton
  converges only linearly (a dew point of an oil-like feed, ending on the
  1000 Pa pressure-step rule), the reference's own result moves by up to
  1e-6 relative when its input pressure moves by 1e-12 relative.  Such a
  cell is held to twice that spread instead: the reference is re-run at
  input pressures scaled by 1 +- 1e-12 and 1 +- 1e-11, and the spread of its
  results is the bar.
* LowerDew_Succ on every gas-only cell, under the same bar.
* critTest on every one-phase cell, on a state that holds oil-only cells of
  gas-like composition and gas-only cells of oil-like composition.  Labels
  must be identical; compositions and saturations within 1e-12.
"""
import numpy as np
import pytest

import oracle
from phase_cases import DECKS, construct_changes, open_pair

pytestmark = [pytest.mark.gpu, pytest.mark.timeout(600),
              pytest.mark.skipif(not oracle.ref_available(), reason="reference library missing")]


def _close(a, b, rel):
    if not (np.isfinite(a) and np.isfinite(b)):
        return not np.isfinite(a) and not np.isfinite(b)
    return abs(a - b) <= rel * abs(b)


def _reference_spread(R, kind, c, phase):
    """Spread of the reference's result (pressure, composition) over input
    pressures of cell c scaled by 1 +- 1e-12 and 1 +- 1e-11."""
    P = R.get("m.P").copy()
    ps, xs = [], []
    for eps in (0.0, 1e-12, -1e-12, 1e-11, -1e-11):
        P2 = P.copy()
        P2[phase, c] *= 1 + eps
        R.set("m.P", P2)
        p, x = R.sat_pressure_nr(kind, c)
        ps.append(p)
        xs.append(x)
    R.set("m.P", P)
    return float(np.ptp(ps)), float(np.ptp(np.asarray(xs), axis=0).max())


@pytest.mark.parametrize("name", list(DECKS))
@pytest.mark.parametrize("kind", ["bubble_nr", "dew_nr", "lower_dew"])
def test_saturation_pressure_nr_matches_reference(name, kind, tmp_path, cuda_device):
    import torch
    R, G = open_pair(tmp_path, name)
    construct_changes(R, G)
    p, xm, st, it = G.saturation_pressure_nr(0, kind, cuda_device)
    torch.cuda.synchronize()
    p, xm, st, it = p.cpu().numpy(), xm.cpu().numpy(), st.cpu().numpy(), it.cpu().numpy()
    lab = R.get("m.label")
    want = 1 if kind == "bubble_nr" else -1
    cells = np.nonzero(lab == want)[0]
    assert np.all(p[lab != want] == 0) and np.all(st[lab != want] == 0)
    checked = capped = spread_cells = 0
    K = G.SATP_KINDS[kind]
    for c in cells:
        if st[c] == 1:             # OSR_CELL_MAXIT: the reference would not stop either
            capped += 1
            continue
        pr, xr = R.sat_pressure_nr(K, int(c))
        checked += 1
        p_ok = _close(p[c], pr, 1e-9)
        x_ok = not (np.isfinite(pr) and pr != 1e100) or np.abs(xm[:, c] - xr).max() <= 1e-9
        if not (p_ok and x_ok):
            ps, xs = _reference_spread(R, K, int(c), 1 if kind == "bubble_nr" else 2)
            spread_cells += 1
            assert abs(p[c] - pr) <= 2 * ps + 1e-9 * abs(pr), (kind, int(c), p[c], pr, ps, int(it[c]))
            assert np.abs(xm[:, c] - xr).max() <= 2 * xs + 1e-9, (kind, int(c), xm[:, c], xr, xs)
    print(f"{name} {kind}: {checked} cells checked ({spread_cells} under the reference's spread), "
          f"{capped} stopped at the cap, steps {int(it[cells].max()) if len(cells) else 0} at most")
    if kind == "lower_dew":
        assert capped == 0
    assert checked >= capped


def _construct_crit(R, G):
    """Oil-only cells of a gas-like composition, gas-only cells of an oil-like
    composition and one-phase cells of the feed, in turn over the matrix."""
    lab = R.get("m.label").copy()
    sat = R.get("m.sat").copy()
    x, y, z = R.get("m.x").copy(), R.get("m.y").copy(), R.get("m.z").copy()
    nc = x.shape[0]
    gas_like = 0.02 ** np.arange(nc)
    gas_like /= gas_like.sum()
    oil_like = 4.0 ** np.arange(nc)
    oil_like /= oil_like.sum()
    for c in range(lab.shape[0]):
        kind = c % 4
        sw = sat[0, c]
        if kind in (0, 2):
            lab[c] = 1
            x[:, c] = gas_like if kind == 0 else z[:, c]
            sat[1, c], sat[2, c] = 1 - sw, 0
        else:
            lab[c] = -1
            y[:, c] = oil_like if kind == 1 else z[:, c]
            sat[1, c], sat[2, c] = 0, 1 - sw
    for nm, v in (("label", lab), ("sat", sat), ("x", x), ("y", y)):
        R.set(f"m.{nm}", v)
    G.set_state(0, G.get("m.P")[1], sat, x, y, z, lab.astype(np.int8))
    R.set("m.P", G.get("m.P"))


@pytest.mark.parametrize("name", list(DECKS))
def test_crit_test_matches_reference(name, tmp_path, cuda_device):
    import torch
    R, G = open_pair(tmp_path, name)
    _construct_crit(R, G)
    before = R.get("m.label").copy()
    L, changed = G.crit_test(0, cuda_device)
    torch.cuda.synchronize()
    for c in np.nonzero(before != 0)[0]:
        R.crit_test(int(c))
    lr, lg = R.get("m.label"), G.get("m.label")
    assert np.array_equal(lr, lg), np.nonzero(lr != lg)[0][:10]
    assert changed == int((lr != before).sum())
    assert changed > 0
    for k in ("x", "y", "sat"):
        assert np.abs(G.get(f"m.{k}") - R.get(f"m.{k}")).max() <= 1e-12, k
    L = L.cpu().numpy()
    assert np.all(L[before == 0] == -1) and np.all((L[before != 0] >= 0) & (L[before != 0] <= 1))
    print(f"{name}: {changed} of {int((before != 0).sum())} one-phase cells relabelled")

"""The reference's restart file (``test.rst``): WriteRST / ReadRST,
compsim/Do_Time_Step.cpp:179-294.

Layout (native little-endian, no header):

* oil-continuum pressures P[Nx+2][Ny+2][Nz+2][3] (water, oil, gas; x
  outermost, the phase innermost), the one-cell halo included: the reference
  zeroes the halo's six faces at start-up (Edge_Trans,
  compsim/Init_Calcs.cpp:262-300) and never writes its edges and corners,
  whose bytes in its files are whatever its allocator left there; this
  module writes zeros in the whole halo and ignores it when reading;
* the same for the fracture continuum;
* per matrix cell (x outermost, then y, then z): sat[3], then for every
  component x_i, y_i, then the phase label as one signed byte;
* the same per fracture cell;
* simTime (s), Dt (s), TSMCtrl (int32), SMethQ (the main loop's cumulative
  producer methane; the device run does not track it, so it is an argument).

The package's state arrays are [planes][cells] with cell = ix + nx (iy + ny
iz); this module converts between the two.
"""
from __future__ import annotations

import numpy as np


def _cell_record(nc: int) -> np.dtype:
    return np.dtype([("sat", "<f8", (3,)), ("xy", "<f8", (nc, 2)), ("label", "i1")], align=False)


def _trailer() -> np.dtype:
    return np.dtype([("sim_time", "<f8"), ("dt", "<f8"), ("tsm_ctrl", "<i4"), ("smethq", "<f8")], align=False)


def _to_xyz(a, nx, ny, nz):
    """[planes][cells] (x fastest) -> [nx][ny][nz][planes]."""
    a = np.asarray(a)
    planes = a.shape[0] if a.ndim == 2 else 1
    return a.reshape(planes, nz, ny, nx).transpose(3, 2, 1, 0)


def _from_xyz(a):
    """[nx][ny][nz][planes] -> [planes][cells] (x fastest)."""
    nx, ny, nz, planes = a.shape
    return np.ascontiguousarray(a.transpose(3, 2, 1, 0).reshape(planes, nx * ny * nz))


def write_rst_arrays(path: str, nx: int, ny: int, nz: int, nc: int, state: dict, sim_time: float, dt: float,
                     tsm_ctrl: int, smethq: float = 0.0) -> None:
    """Write a restart file from host arrays: state[m + "." + key] for m in
    "m", "f" and key in P [3][cells], sat [3][cells], x, y [nc][cells],
    label [cells]."""
    n = nx * ny * nz
    rec = _cell_record(nc)
    with open(path, "wb") as fh:
        for m in "mf":
            P = np.zeros((nx + 2, ny + 2, nz + 2, 3))
            P[1:-1, 1:-1, 1:-1] = _to_xyz(np.asarray(state[f"{m}.P"], np.float64).reshape(3, n), nx, ny, nz)
            fh.write(P.astype("<f8").tobytes())
        for m in "mf":
            r = np.zeros((nx, ny, nz), rec)
            r["sat"] = _to_xyz(np.asarray(state[f"{m}.sat"], np.float64).reshape(3, n), nx, ny, nz)
            r["xy"][..., 0] = _to_xyz(np.asarray(state[f"{m}.x"], np.float64).reshape(nc, n), nx, ny, nz)
            r["xy"][..., 1] = _to_xyz(np.asarray(state[f"{m}.y"], np.float64).reshape(nc, n), nx, ny, nz)
            r["label"] = _to_xyz(np.asarray(state[f"{m}.label"]).reshape(1, n), nx, ny, nz)[..., 0]
            fh.write(r.tobytes())
        t = np.zeros(1, _trailer())
        t["sim_time"], t["dt"], t["tsm_ctrl"], t["smethq"] = sim_time, dt, tsm_ctrl, smethq
        fh.write(t.tobytes())


def read_rst(path: str, nx: int, ny: int, nz: int, nc: int) -> dict:
    """Read a restart file into the package layout: m./f. + P, sat, x, y,
    label, and sim_time, dt, tsm_ctrl, smethq."""
    rec = _cell_record(nc)
    raw = open(path, "rb").read()
    halo = (nx + 2) * (ny + 2) * (nz + 2) * 3 * 8
    cells = nx * ny * nz * rec.itemsize
    if len(raw) != 2 * halo + 2 * cells + _trailer().itemsize:
        raise ValueError(f"{path}: {len(raw)} bytes, not a restart file of this grid and component count")
    out = {}
    off = 0
    for m in "mf":
        P = np.frombuffer(raw, "<f8", halo // 8, off).reshape(nx + 2, ny + 2, nz + 2, 3)
        out[f"{m}.P"] = _from_xyz(P[1:-1, 1:-1, 1:-1])
        off += halo
    for m in "mf":
        r = np.frombuffer(raw, rec, nx * ny * nz, off).reshape(nx, ny, nz)
        out[f"{m}.sat"] = _from_xyz(r["sat"])
        out[f"{m}.x"] = _from_xyz(r["xy"][..., 0])
        out[f"{m}.y"] = _from_xyz(r["xy"][..., 1])
        out[f"{m}.label"] = _from_xyz(r["label"][..., None].astype(np.int8))[0]
        off += cells
    t = np.frombuffer(raw, _trailer(), 1, off)[0]
    out.update(sim_time=float(t["sim_time"]), dt=float(t["dt"]), tsm_ctrl=int(t["tsm_ctrl"]),
               smethq=float(t["smethq"]))
    return out


def write_rst(path: str, grid, sim, smethq: float = 0.0) -> None:
    """Restart file of a device run (``osiris_b200.Grid`` + ``Sim``)."""
    state = {f"{m}.{k}": grid.get(f"{m}.{k}") for m in "mf" for k in ("P", "sat", "x", "y", "label")}
    t, dt = sim.time()
    write_rst_arrays(path, grid.deck.nx, grid.deck.ny, grid.deck.nz, grid.nc, state, t, dt, sim.marker_index(),
                     smethq)


def restore(grid, path: str):
    """Load a restart file into the device grid (the reference's ReadRST
    followed by UpdateDependencies(true), compsim/PrimeSim.cpp:84-85): the
    state, then phase control, PCoeff, layout and property sweeps.  The
    overall compositions and the densities stay as the grid holds them (the
    file carries neither; the reference keeps its start-up values).  Returns
    (sim_time, dt, tsm_ctrl, smethq) for ``Sim.restart``."""
    d = grid.deck
    r = read_rst(path, d.nx, d.ny, d.nz, grid.nc)
    for mi, m in enumerate("mf"):
        grid.set_state(mi, r[f"{m}.P"][1], r[f"{m}.sat"], r[f"{m}.x"], r[f"{m}.y"], grid.get(f"{m}.z"),
                       r[f"{m}.label"])
        grid.set_pressures(mi, r[f"{m}.P"])
    grid.phase_ctrl()
    grid.refresh_layout()
    grid.update_dependencies()
    return r["sim_time"], r["dt"], r["tsm_ctrl"], r["smethq"]

"""The restart file (osiris_b200/restart.py) against the reference's own
WriteRST (compsim/Do_Time_Step.cpp:179-234), CPU only: after three passes of
the reference's main loop, the file the package writes from the reference's
state is byte for byte the file WriteRST writes (except the pressure halo's
edges and corners, which the reference never writes), and reading
WriteRST's file gives back the reference's arrays and controls exactly."""
import os

import numpy as np
import pytest

import oracle
from oracle import steps
from osiris_b200 import deck, restart

needs_ref = pytest.mark.skipif(not oracle.ref_available(), reason="reference library missing")


@needs_ref
@pytest.mark.parametrize("spec", ["twophase_10MPa", "plain_oil"])
def test_restart_file_matches_reference_writer(spec, tmp_path):
    s = {"twophase_10MPa": lambda: deck.config_deck(nx=5, ny=4, nz=3, cdif=0.0, ipress=1e7, seed=3),
         "plain_oil": lambda: deck.config_deck(nx=4, ny=3, nz=2, cdif=None)}[spec]()
    path = os.path.join(str(tmp_path), "deck.dat")
    deck.write_deck(path, s)
    R = oracle.RefDeck(path)
    t = 0.0
    R.create_backups(t)
    for _ in range(3):
        t = steps.ref_pass(R, t)["sim_time"]
    ref_file = R.write_rst(str(tmp_path), t)
    state = {f"{m}.{k}": R.get(f"{m}.{k}") for m in "mf" for k in ("P", "sat", "x", "y", "label")}
    _, tsm = R.time_markers()
    mine = os.path.join(str(tmp_path), "mine.rst")
    restart.write_rst_arrays(mine, R.nx, R.ny, R.nz, R.nc, state, t, R.scalar("Dt"), tsm, R.scalar("SMethQ"))
    a, b = open(mine, "rb").read(), open(ref_file, "rb").read()
    assert len(a) == len(b)
    nh = (R.nx + 2) * (R.ny + 2) * (R.nz + 2) * 3
    # after the two pressure blocks: identical bytes
    assert a[2 * nh * 8:] == b[2 * nh * 8:]
    # pressure blocks: interior and halo faces identical (faces zero); the
    # halo's edges and corners are never written by the reference
    ix, iy, iz = np.meshgrid(np.arange(R.nx + 2), np.arange(R.ny + 2), np.arange(R.nz + 2), indexing="ij")
    on_halo = (ix == 0) | (ix == R.nx + 1), (iy == 0) | (iy == R.ny + 1), (iz == 0) | (iz == R.nz + 1)
    defined = (on_halo[0].astype(int) + on_halo[1] + on_halo[2]) <= 1
    for blk in range(2):
        Pa = np.frombuffer(a, "<f8", nh, blk * nh * 8).reshape(R.nx + 2, R.ny + 2, R.nz + 2, 3)
        Pb = np.frombuffer(b, "<f8", nh, blk * nh * 8).reshape(R.nx + 2, R.ny + 2, R.nz + 2, 3)
        assert np.array_equal(Pa[defined].view(np.int64), Pb[defined].view(np.int64)), blk
    r = restart.read_rst(ref_file, R.nx, R.ny, R.nz, R.nc)
    for k, v in state.items():
        assert np.array_equal(r[k], v), k
    assert (r["sim_time"], r["dt"], r["tsm_ctrl"]) == (t, R.scalar("Dt"), tsm)


def test_wrong_size_is_rejected(tmp_path):
    p = os.path.join(str(tmp_path), "x.rst")
    open(p, "wb").write(b"\0" * 100)
    with pytest.raises(ValueError):
        restart.read_rst(p, 2, 2, 2, 3)


_LISTING_CHILD = r"""
import ctypes, sys
# the reference's C++ output streams must bind to its own runtime: load it
# before numpy brings a second libstdc++ into the process
ctypes.CDLL(sys.argv[1])
import numpy as np
import oracle
from oracle import steps
R = oracle.RefDeck(sys.argv[2])
t = 0.0
R.create_backups(t)
for k in range(3):
    if k:
        t = steps.ref_pass(R, t)["sim_time"]
    R.print_all(sys.argv[3], t)
    np.savez(f"{sys.argv[4]}_{k}.npz", t=t, **{f"{m}.{q}": R.get(f"{m}.{q}") for m in "mf"
                                                for q in ("P", "sat", "x", "y")})
R.print_all(None, 0.0)
"""


@needs_ref
def test_state_listing_matches_reference_print_all(tmp_path):
    """The state listing from the reference's state is the reference's own
    PrintAll output character for character, over a start-up call and two
    calls after accepted passes on one stream (the reference runs in a child
    process that loads it before numpy, see _LISTING_CHILD)."""
    import subprocess
    import sys
    from osiris_b200 import output
    td = str(tmp_path)
    path = os.path.join(td, "deck.dat")
    spec = deck.config_deck(nx=4, ny=3, nz=2, cdif=0.0, ipress=1e7, seed=3)
    deck.write_deck(path, spec)
    ref_out = os.path.join(td, "ref.txt")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    env = dict(os.environ, PYTHONPATH=root + os.pathsep + os.environ.get("PYTHONPATH", ""))
    subprocess.run([sys.executable, "-c", _LISTING_CHILD, oracle.REF_LIB, path, ref_out, os.path.join(td, "st")],
                   check=True, env=env, stdout=subprocess.DEVNULL)
    d = deck.parse_deck(path)
    mine = output.StateListing(os.path.join(td, "mine.txt"))
    for k in range(3):
        z = np.load(os.path.join(td, f"st_{k}.npz"))
        mine.write(d.nx, d.ny, d.nz, d.nc, {q: z[q] for q in z.files if q != "t"}, float(z["t"]))
    mine.close()
    assert open(os.path.join(td, "mine.txt")).read() == open(ref_out).read()

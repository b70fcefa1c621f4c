"""The reference's state listing (PrintAll, compsim/ViewAssist.Cpp:39-88),
written by the main program at start-up and after every accepted step
(compsim/PrimeSim.cpp:89, 161), so that a device run can be compared with a
reference run line by line.

Per call: 80 dashes, the time in hours, a header (X Y Z P Sw So Sg, Xo[i],
Yg[i]), then "M" and one line per matrix cell (z outermost, x fastest): the
cell's indices, oil pressure, three saturations, the liquid then the vapour
composition, tab separated; then "F" and the same for the fracture.  Numbers
print as C++ streams print doubles: 20 significant digits (%.20g), except
the time of the first call on a stream, which precedes the stream's first
setprecision(20) and so prints with the default 6 (%g).
"""
from __future__ import annotations

import numpy as np


class StateListing:
    """One output stream of PrintAll calls."""

    def __init__(self, path: str):
        self.fh = open(path, "w")
        self.precise = False

    def write(self, nx: int, ny: int, nz: int, nc: int, state: dict, t: float) -> None:
        """state: m./f. + P [3][cells], sat [3][cells], x, y [nc][cells]."""
        out = ["-" * 80, "\n", ("%.20g" if self.precise else "%g") % (t / 3600)]
        out.append("\nX\tY\tZ\tP\t\t\tSw\t\t\tSo\t\t\tSg\t\t\t")
        out += [f"Xo[{i}]\t\t\t" for i in range(nc)]
        out += [f"Yg[{i}]\t\t\t" for i in range(nc)]
        for tag, m in (("\nM\n", "m"), ("\nF\n", "f")):
            out.append(tag)
            P = np.asarray(state[f"{m}.P"])[1]
            S, X, Y = (np.asarray(state[f"{m}.{k}"]) for k in ("sat", "x", "y"))
            c = 0
            for iz in range(nz):
                for iy in range(ny):
                    for ix in range(nx):
                        out.append("\n%d\t%d\t%d\t%.20g\t%.20g\t%.20g\t%.20g" % (ix, iy, iz, P[c], S[0, c], S[1, c],
                                                                             S[2, c]))
                        out += ["\t%.20g\t" % X[i, c] for i in range(nc)]
                        out += ["%.20g\t" % Y[i, c] for i in range(nc)]
                        c += 1
        out.append("\n\n\n")
        self.fh.write("".join(out))
        self.fh.flush()
        self.precise = True

    def write_grid(self, grid, t: float) -> None:
        """The current state of a device grid."""
        d = grid.deck
        state = {f"{m}.{k}": grid.get(f"{m}.{k}") for m in "mf" for k in ("P", "sat", "x", "y")}
        self.write(d.nx, d.ny, d.nz, grid.nc, state, t)

    def close(self):
        self.fh.close()

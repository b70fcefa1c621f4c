"""CPU restatement of one slab's part of the distributed linear solve
(osr_dksp_* of the C library), for testing the driver (osiris_b200.slabs.
solve_slabs) and its collectives between gloo ranks without a GPU.

The stages and scalar steps follow the device kernels (BiCGStab in PETSc's
left-preconditioned KSPBCGS arrangement with block-Jacobi, the dot products
over the owned rows, the vector updates over every local row), on a scipy
matrix in the slab's local row numbering.  Test infrastructure only."""
import numpy as np
import torch

RUNNING, CONV_RTOL, CONV_ATOL, DIV_ITS, DIV_DTOL, DIV_BREAKDOWN, DIV_NAN, FINISH_P = 0, 2, 3, -3, -4, -5, -9, -100


class CpuPart:
    def __init__(self, A, rowoff, owned_blocks, nx, ny, nz_local, has_lower, has_upper):
        self.A = A.tocsr()
        self.rowoff = np.asarray(rowoff)
        self.nx, self.ny, self.nz_local = nx, ny, nz_local
        self.has_lower, self.has_upper = has_lower, has_upper
        nb = len(self.rowoff) - 1
        b0, b1, b2, b3 = owned_blocks
        self.owned_rows = np.zeros(int(self.rowoff[-1]), bool)
        for lo_b, hi_b in ((b0, b1), (b2, b3)):
            self.owned_rows[self.rowoff[lo_b]:self.rowoff[hi_b]] = True
        self.inv = []
        dense = self.A.toarray()
        for b in range(nb):
            o0, o1 = self.rowoff[b], self.rowoff[b + 1]
            self.inv.append(np.linalg.inv(dense[o0:o1, o0:o1]))

    def _B(self, r):
        z = np.empty_like(r)
        for b, inv in enumerate(self.inv):
            o0, o1 = self.rowoff[b], self.rowoff[b + 1]
            z[o0:o1] = inv @ r[o0:o1]
        return z

    def _dot(self, a, b):
        m = self.owned_rows
        return float(np.dot(a[m], b[m]))

    def begin(self, b, rtol=1e-12, atol=1e-50, dtol=1e3, max_it=500):
        n = int(self.rowoff[-1])
        self.x = np.zeros(n)
        self.p = torch.zeros(n, dtype=torch.float64)
        self.s = torch.zeros(n, dtype=torch.float64)
        self.dots = torch.zeros(4, dtype=torch.float64)
        self.r = self._B(np.asarray(b, float))
        self.r0 = self.r.copy()
        self.v = np.zeros(n)
        self.t = np.zeros(n)
        self.w = np.zeros(n)
        self.sc = dict(rtol=rtol, atol=atol, dtol=dtol, max_it=max_it, reason=RUNNING, its=0, rnorm0=0.0,
                       rnorm=0.0, ttol=0.0, rho=0.0, rhoold=0.0, alpha=0.0, omega=0.0, omegaold=0.0, beta=0.0)
        self.dots[0] = self._dot(self.r, self.r)

    def _test(self, rn):
        s = self.sc
        if not np.isfinite(rn):
            s["reason"] = DIV_NAN
        elif rn <= s["ttol"]:
            s["reason"] = CONV_ATOL if rn < s["atol"] else CONV_RTOL
        elif s["its"] > 0 and s["dtol"] > 0 and rn >= s["dtol"] * s["rnorm0"]:
            s["reason"] = DIV_DTOL

    def stage(self, k):
        s, d = self.sc, self.dots.numpy()
        p, sv = self.p.numpy(), self.s.numpy()
        running = s["reason"] == RUNNING
        if k == 0:
            rn = np.sqrt(d[0])
            s.update(rnorm0=rn, rnorm=rn, ttol=max(s["rtol"] * rn, s["atol"]), its=0)
            self._test(rn)
            s.update(rho=d[0], rhoold=1.0, alpha=1.0, omegaold=1.0)
            s["beta"] = (s["rho"] / s["rhoold"]) * (s["alpha"] / s["omegaold"])
        elif k == 1 and running:
            p[:] = self.r + s["beta"] * p - (s["omegaold"] * s["beta"]) * self.v
        elif k == 2 and running:
            self.t = self.A @ p
            self.v = self._B(self.t)
            d[0] = self._dot(self.v, self.r0)
        elif k == 3 and running:
            d1 = d[0]
            if not np.isfinite(d1):
                s["reason"] = DIV_NAN
            elif d1 == 0.0:
                s["reason"] = DIV_BREAKDOWN
            else:
                s["alpha"] = s["rho"] / d1
            if s["reason"] == RUNNING:
                sv[:] = self.r - s["alpha"] * self.v
        elif k == 4 and running:
            self.w = self.A @ sv
            self.t = self._B(self.w)
            d[0], d[1], d[2] = self._dot(sv, self.t), self._dot(self.t, self.t), self._dot(sv, sv)
        elif k == 5 and running:
            d1, d2, ss = d[0], d[1], d[2]
            if d2 == 0.0:
                if ss != 0.0:
                    s["reason"] = DIV_BREAKDOWN
                else:
                    s.update(omega=0.0, rnorm=0.0, reason=FINISH_P)
                    s["its"] += 1
            else:
                s["omega"] = d1 / d2
            if s["reason"] == FINISH_P:
                self.x += s["alpha"] * p
            elif s["reason"] == RUNNING:
                self.x += s["alpha"] * p + s["omega"] * sv
                self.r = sv - s["omega"] * self.t
                d[0], d[1] = self._dot(self.r, self.r), self._dot(self.r, self.r0)
        elif k == 6:
            if s["reason"] == FINISH_P:
                s["reason"] = CONV_RTOL
            elif running:
                dp = np.sqrt(d[0])
                rho = s["rho"]
                s.update(rhoold=rho, omegaold=s["omega"], rnorm=dp)
                s["its"] += 1
                self._test(dp)
                if s["reason"] == RUNNING and rho == 0.0:
                    s["reason"] = DIV_BREAKDOWN
                if s["reason"] == RUNNING and s["its"] >= s["max_it"]:
                    s["reason"] = DIV_ITS
                s["rho"] = d[1]
                s["beta"] = (s["rho"] / s["rhoold"]) * (s["alpha"] / s["omegaold"])

    def info(self):
        s = self.sc
        return {"reason": s["reason"], "its": s["its"], "rnorm0": s["rnorm0"], "rnorm": s["rnorm"]}


class LocalComm:
    """The collectives of solve_slabs for slabs held in one process, in rank
    order: sums added slab by slab, ghost layers copied from the neighbours'
    owned layers."""

    def sum(self, parts, k):
        tot = parts[0].dots[:k].clone()
        for q in parts[1:]:
            tot += q.dots[:k]
        for q in parts:
            q.dots[:k] = tot

    def exchange(self, parts, name):
        from osiris_b200.slabs import layer_rows
        for lower, upper in zip(parts[:-1], parts[1:]):
            a, b = getattr(lower, name), getattr(upper, name)
            # upper's first owned layer -> lower's upper ghost; lower's last owned layer -> upper's lower ghost
            src_up = layer_rows(upper.rowoff, upper.nx, upper.ny, upper.nz_local, 1)
            dst_lo = layer_rows(lower.rowoff, lower.nx, lower.ny, lower.nz_local, lower.nz_local - 1)
            src_lo = layer_rows(lower.rowoff, lower.nx, lower.ny, lower.nz_local, lower.nz_local - 2)
            dst_up = layer_rows(upper.rowoff, upper.nx, upper.ny, upper.nz_local, 0)
            for (s0, s1), (d0, d1) in zip(src_up, dst_lo):
                a[d0:d1] = b[s0:s1]
            for (s0, s1), (d0, d1) in zip(src_lo, dst_up):
                b[d0:d1] = a[s0:s1]

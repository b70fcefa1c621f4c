"""CPU oracle for the flash hot path (test infrastructure only).

Two libraries sit behind this module:

* ``_ref/libosiris_ref.so`` -- the reference simulator compiled unmodified from
  its own C++ sources (``oracle/Makefile``), driven through the C entry points
  in ``oracle/ref_driver.cpp``.  It is only present where the reference sources
  were available at build time.
* ``_build/liboracle.so`` -- the plain-C restatement in ``oracle/flash_oracle.c``
  (each function cites the reference file:line it restates).

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` import this module, and only as the checker.  The CUDA library
never loads or calls it.

Array conventions match the CUDA library: per-cell scalars ``[n]``,
per-component fields ``[nc, n]``, derivative blocks ``[2, nc, nc, n]`` and
``[2, nc, n]`` with phase 0 = liquid, 1 = vapour.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_LIB = os.path.join(HERE, "_ref", "libosiris_ref.so")
ORACLE_LIB = os.path.join(HERE, "_build", "liboracle.so")
# the same restated source compiled with fused multiply-add contraction: it
# measures how sensitive the reference's algorithm is to rounding alone
ORACLE_FMA_LIB = os.path.join(HERE, "_build", "liboracle_fma.so")

_vp = ctypes.c_void_p


def _p(a):
    return None if a is None else a.ctypes.data_as(_vp)


class _Fluid(ctypes.Structure):
    _fields_ = [("nc", ctypes.c_int), ("eos", ctypes.c_int), ("tc", _vp), ("pc", _vp), ("acf", _vp),
                ("kij", _vp)]


_oracle = None
_oracle_fma = None
_ref = None


def oracle_lib(fma: bool = False):
    global _oracle, _oracle_fma
    if fma:
        if _oracle_fma is None:
            _oracle_fma = _load_oracle(ORACLE_FMA_LIB)
        return _oracle_fma
    if _oracle is None:
        _oracle = _load_oracle(ORACLE_LIB)
    return _oracle


def _load_oracle(path):
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} missing: run `make -C oracle oracle`")
    lib = ctypes.CDLL(path)
    lib.orc_solve_z.restype = ctypes.c_double
    lib.orc_solve_z.argtypes = [ctypes.c_double] * 3 + [ctypes.c_int]
    lib.orc_flash_batch.restype = ctypes.c_int
    lib.orc_flash_derivs_batch.restype = ctypes.c_int
    return lib


def ref_available() -> bool:
    return os.path.exists(REF_LIB)


def ref_lib():
    global _ref
    if _ref is None:
        if not ref_available():
            raise FileNotFoundError(f"{REF_LIB} missing: build with `make -C oracle ref`")
        lib = ctypes.CDLL(REF_LIB)
        lib.ref_flash_batch.restype = ctypes.c_int
        lib.ref_solve_z.restype = ctypes.c_double
        lib.ref_solve_z.argtypes = [ctypes.c_double] * 3 + [ctypes.c_int]
        lib.ref_eos_params.restype = ctypes.c_int
        _ref = lib
    return _ref


class Fluid:
    """Component table: critical temperature [K], critical pressure [Pa],
    acentric factor, symmetric kij with zero diagonal; eos 0 = PR, 1 = SRK."""

    def __init__(self, tc, pc, acf, kij, eos: int):
        self.tc = np.ascontiguousarray(tc, dtype=np.float64)
        self.pc = np.ascontiguousarray(pc, dtype=np.float64)
        self.acf = np.ascontiguousarray(acf, dtype=np.float64)
        self.kij = np.ascontiguousarray(kij, dtype=np.float64)
        self.nc = int(self.tc.shape[0])
        self.eos = int(eos)
        self._c = _Fluid(self.nc, self.eos, _p(self.tc), _p(self.pc), _p(self.acf), _p(self.kij))

    @property
    def cstruct(self):
        return ctypes.byref(self._c)


def flash_batch(fl: Fluid, P, T, z, fma: bool = False):
    """Restated flash (oracle/flash_oracle.c).  Returns a dict of arrays.
    fma=True runs the build with fused multiply-add contraction."""
    lib = oracle_lib(fma)
    P = np.ascontiguousarray(P, np.float64)
    T = np.ascontiguousarray(T, np.float64)
    z = np.ascontiguousarray(z, np.float64)
    n = P.shape[0]
    nc = fl.nc
    out = dict(label=np.zeros(n, np.int8), L=np.zeros(n), x=np.zeros((nc, n)), y=np.zeros((nc, n)),
               Zl=np.zeros(n), Zg=np.zeros(n), iters=np.zeros(n, np.int32), rr_iters=np.zeros(n, np.int32))
    rc = lib.orc_flash_batch(fl.cstruct, ctypes.c_long(n), _p(P), _p(T), _p(z), _p(out["label"]), _p(out["L"]),
                             _p(out["x"]), _p(out["y"]), _p(out["Zl"]), _p(out["Zg"]), _p(out["iters"]),
                             _p(out["rr_iters"]))
    if rc:
        raise RuntimeError(f"orc_flash_batch returned {rc}")
    return out


def flash_derivs(fl: Fluid, P, T, x, y, Zl, Zg):
    lib = oracle_lib()
    n = P.shape[0]
    nc = fl.nc
    dx = np.zeros((2, nc, nc, n))
    dp = np.zeros((2, nc, n))
    args = [np.ascontiguousarray(a, np.float64) for a in (P, T, x, y, Zl, Zg)]
    rc = lib.orc_flash_derivs_batch(fl.cstruct, ctypes.c_long(n), *[_p(a) for a in args], _p(dx), _p(dp))
    if rc:
        raise RuntimeError(f"orc_flash_derivs_batch returned {rc}")
    return dx, dp


def flash_polish(fl: Fluid, P, T, z, out: dict) -> int:
    """Two-phase cells of a flash result (dict of label, L, x, y, Zl, Zg;
    modified in place) solved to rounding by Newton's method on the
    equilibrium equations; returns the cells that did not settle."""
    lib = oracle_lib()
    n = P.shape[0]
    for k in ("L", "x", "y", "Zl", "Zg"):
        out[k] = np.ascontiguousarray(out[k], np.float64)
    lab = np.ascontiguousarray(out["label"], np.int8)
    return int(lib.orc_flash_polish(fl.cstruct, ctypes.c_long(n), _p(np.ascontiguousarray(P, np.float64)),
                                    _p(np.ascontiguousarray(T, np.float64)), _p(np.ascontiguousarray(z, np.float64)),
                                    _p(lab), _p(out["L"]), _p(out["x"]), _p(out["y"]), _p(out["Zl"]), _p(out["Zg"])))


def flash_adjoint(fl: Fluid, P, T, z, st: dict, xbar, ybar, Lbar):
    """Implicit-function adjoint of a flash result: (kij_bar [nc, nc],
    z_bar [nc, n], P_bar [n], singular cells)."""
    lib = oracle_lib()
    n, nc = P.shape[0], fl.nc
    kb = np.zeros(nc * nc)
    zb = np.zeros((nc, n))
    pb = np.zeros(n)
    args = [np.ascontiguousarray(v, np.float64) for v in (P, T, z)]
    lab = np.ascontiguousarray(st["label"], np.int8)
    fs = [np.ascontiguousarray(st[k], np.float64) for k in ("L", "x", "y", "Zl", "Zg")]
    bars = [np.ascontiguousarray(v, np.float64) for v in (xbar, ybar, Lbar)]
    bad = lib.orc_flash_adjoint(fl.cstruct, ctypes.c_long(n), *[_p(v) for v in args], _p(lab), *[_p(v) for v in fs],
                                *[_p(v) for v in bars], _p(kb), _p(zb), _p(pb))
    return kb.reshape(nc, nc), zb, pb, int(bad)


def fugacity(fl: Fluid, P: float, T: float, w, Z: float):
    """ln(phi), d ln(phi)/dw [nc, nc], d ln(phi)/dP for one phase."""
    lib = oracle_lib()
    nc = fl.nc
    w = np.ascontiguousarray(w, np.float64)
    lnphi = np.zeros(nc)
    dx = np.zeros((nc, nc))
    dp = np.zeros(nc)
    lib.orc_fugacity(fl.cstruct, ctypes.c_double(P), ctypes.c_double(T), _p(w), ctypes.c_double(Z), _p(lnphi),
                     _p(dx), _p(dp))
    return lnphi, dx, dp


def eos_params(fl: Fluid, T: float):
    lib = oracle_lib()
    a = np.zeros(fl.nc)
    b = np.zeros(fl.nc)
    lib.orc_eos_params(fl.cstruct, ctypes.c_double(T), _p(a), _p(b))
    return a, b


def solve_z(a1, a2, a3, gas: bool) -> float:
    return oracle_lib().orc_solve_z(a1, a2, a3, int(gas))


def ref_flash_batch(fl: Fluid, P, T, z):
    """The reference's own SuccFalsh over n cells (compsim/Init_Calcs.cpp:571)."""
    lib = ref_lib()
    P = np.ascontiguousarray(P, np.float64)
    T = np.ascontiguousarray(T, np.float64)
    z = np.ascontiguousarray(z, np.float64)
    n = P.shape[0]
    nc = fl.nc
    out = dict(label=np.zeros(n, np.int8), x=np.zeros((nc, n)), y=np.zeros((nc, n)), sat_o=np.zeros(n),
               sat_g=np.zeros(n), rho_o=np.zeros(n), rho_g=np.zeros(n))
    rc = lib.ref_flash_batch(nc, fl.eos, _p(fl.tc), _p(fl.pc), _p(fl.acf), _p(fl.kij), ctypes.c_long(n), _p(P),
                             _p(T), _p(z), _p(out["x"]), _p(out["y"]), _p(out["label"]), _p(out["sat_o"]),
                             _p(out["sat_g"]), _p(out["rho_o"]), _p(out["rho_g"]))
    if rc:
        raise RuntimeError(f"ref_flash_batch returned {rc}")
    return out


def ref_solve_z(a1, a2, a3, gas: bool) -> float:
    return ref_lib().ref_solve_z(a1, a2, a3, int(gas))


def ref_eos_params(fl: Fluid, T: float):
    lib = ref_lib()
    a = np.zeros(fl.nc)
    b = np.zeros(fl.nc)
    rc = lib.ref_eos_params(fl.nc, fl.eos, _p(fl.tc), _p(fl.pc), _p(fl.acf), ctypes.c_double(T), _p(a), _p(b))
    if rc:
        raise RuntimeError("ref_eos_params failed")
    return a, b


R_GAS = 8.3144621


def derived_sat_rho(fl_out, P, T):
    """Oil/gas volume fractions and molar densities from L and Z, as the
    reference's SuccFalsh forms them with zero water saturation
    (compsim/Init_Calcs.cpp:730-736)."""
    L, Zl, Zg = fl_out["L"], fl_out["Zl"], fl_out["Zg"]
    newD = Zl * L / (Zl * L + Zg * (1 - L))
    sat_o = newD * (1 - 0.0)
    sat_g = (1 - newD) * (1 - 0.0)
    rho_o = P / (Zl * R_GAS * T)
    rho_g = P / (Zg * R_GAS * T)
    return sat_o, sat_g, rho_o, rho_g


# ----------------------------------------------------------------------------- parity bar

FLASH_FIELDS = ("L", "x", "y", "Zl", "Zg")
RTOL = 1e-10          # the bar: relative error per value ...
ATOL = 1e-13          # ... with an absolute floor for trace mole fractions
WIDE_SCALE = 5e-8     # the bound every present-phase value must meet, relative to max(|v|, 1e-3)
MIN_TIGHT = 0.995     # fraction of cells whose present-phase values meet the 1e-10 bar
MIN_TIGHT_ABSENT = 0.99  # fraction of cells whose incipient-phase values meet the 1e-10 bar


def _present(field, label):
    """Cells where `field` belongs to a phase that exists (label +1 = liquid
    only, -1 = vapour only, 0 = both); the others carry the incipient phase."""
    if field in ("x", "Zl"):
        return label >= 0
    if field in ("y", "Zg"):
        return label <= 0
    return np.ones_like(label, dtype=bool)


def flash_parity(got, ref, fields=FLASH_FIELDS):
    """Compare a flash result with the oracle's.

    The reference's successive substitution stops on |L_k - L_{k-1}| <= 1e-14
    after a Rachford-Rice Newton truncated at step^2 <= 1e-8.  For a small set
    of cells the iterate then jitters at the 1e-11..1e-9 level from one
    substitution step to the next, so the value at which it stops depends on
    rounding alone: the same restated source compiled with fused multiply-add
    contraction moves those cells by as much (``flash_batch(fma=True)``).  In
    single-phase cells the absent phase's composition is an unconverged
    incipient-phase estimate, and its cubic can be degenerate (a double root
    at zero), where the reference's smallest-positive-root rule flips with
    rounding.  The bar is therefore:
      * phase labels identical in every cell;
      * present-phase values (L, and x/Zl or y/Zg of a phase that exists)
        within 1e-10 relative (+1e-13) in >= 99.5% of cells and within 5e-8
        of max(|v|, 1e-3) in every cell;
      * incipient-phase values within 1e-10 relative (+1e-13) in >= 99% of
        cells.
    Cells outside the 1e-10 bar are returned as the margin lists."""
    label = np.asarray(ref["label"])
    n = label.shape[0]
    labels_equal = bool(np.array_equal(np.asarray(got["label"]), label))
    loose = np.zeros(n, bool)
    loose_abs = np.zeros(n, bool)
    wide_ok = True
    max_scaled = 0.0
    for k in fields:
        a = np.asarray(got[k], dtype=np.float64)
        b = np.asarray(ref[k], dtype=np.float64)
        nan = np.isnan(a) & np.isnan(b)
        err = np.abs(a - b)
        tight = (err <= RTOL * np.abs(b) + ATOL) | nan
        scaled = np.where(nan, 0.0, err / np.maximum(np.abs(b), 1e-3))
        if tight.ndim > 1:
            tight = tight.all(axis=0)
            scaled = scaled.max(axis=0) if scaled.size else scaled.reshape(-1)
        pres = _present(k, label)
        wide_ok &= bool(np.all(scaled[pres] <= WIDE_SCALE))
        if pres.any():
            max_scaled = max(max_scaled, float(np.nanmax(scaled[pres])))
        loose |= ~tight & pres
        loose_abs |= ~tight & ~pres
    margin = np.nonzero(loose)[0]
    margin_abs = np.nonzero(loose_abs)[0]
    frac_tight = 1.0 - margin.size / max(n, 1)
    frac_tight_abs = 1.0 - margin_abs.size / max(n, 1)
    ok = labels_equal and wide_ok and frac_tight >= MIN_TIGHT and frac_tight_abs >= MIN_TIGHT_ABSENT
    return dict(ok=ok, labels_equal=labels_equal, wide_ok=wide_ok, frac_tight=frac_tight,
                frac_tight_incipient=frac_tight_abs, margin=margin, margin_incipient=margin_abs,
                max_scaled_err=max_scaled)


# ----------------------------------------------------------------------------- deck-driven reference

_FIELD_SHAPES = {"P": (3,), "sat": (3,), "x": ("nc",), "y": ("nc",), "z": ("nc",), "label": (), "rho": (2,),
                 "pc": (2,), "mu": (2,), "gam": (2,), "kr": (3,), "dkr": (5,), "dE": ("nc1", 2),
                 "pre": ("nc1",), "diff": ("nc", 2), "ift": (), "trans": (12, 3), "transS": (3, 3),
                 "wtran": (3,), "dwtran": (3,), "iftran": (3,), "por": (), "perm": (3,), "blockH": ()}


class RefDeck:
    """The reference simulator loaded from a deck (compsim/PrimeSim.cpp:35-85).
    One instance at a time: the reference keeps its state in globals."""

    def __init__(self, path: str):
        lib = ref_lib()
        lib.ref_deck_open.restype = ctypes.c_int
        lib.ref_get.restype = ctypes.c_long
        lib.ref_scalar.restype = ctypes.c_double
        lib.ref_form_jacobian.restype = ctypes.c_long
        lib.ref_set.restype = ctypes.c_long
        lib.ref_sat_pressure.restype = ctypes.c_double
        lib.ref_sat_pressure_nr.restype = ctypes.c_double
        lib.ref_crit_test.restype = ctypes.c_int
        rc = lib.ref_deck_open(path.encode())
        if rc:
            raise RuntimeError(f"reference could not open {path}")
        info = np.zeros(10, np.int32)
        lib.ref_deck_info(_p(info))
        self.nx, self.ny, self.nz, self.nc, self.pr, self.rows, self.nwells, self.nswt, self.nsgt, self.cdif = \
            (int(v) for v in info)
        self.cells = self.nx * self.ny * self.nz
        self.lib = lib

    def scalar(self, name: str) -> float:
        return float(self.lib.ref_scalar(name.encode()))

    def get(self, name: str) -> np.ndarray:
        key = name.split(".", 1)[-1]
        if name in ("gridDim",):
            n = self.nx + self.ny + self.nz
            shape = (n,)
        elif name == "fluid":
            shape = (self.nc, 15)
        elif name == "bic":
            shape = (self.nc, self.nc)
        elif name == "rowoff":
            shape = (2 * self.cells + 1,)
        else:
            dims = tuple(self.nc if d == "nc" else self.nc + 1 if d == "nc1" else d for d in _FIELD_SHAPES[key])
            shape = dims + (self.cells,)
        out = np.zeros(int(np.prod(shape)))
        w = self.lib.ref_get(name.encode(), _p(out))
        if w < 0:
            raise KeyError(name)
        return out.reshape(shape)

    def calc_re(self, well: int) -> float:
        self.lib.ref_calc_re.restype = ctypes.c_double
        return float(self.lib.ref_calc_re(int(well)))

    def set_well_condition(self, well: int, latched: bool):
        if self.lib.ref_set_well_condition(int(well), int(bool(latched))):
            raise IndexError(well)

    def init_guess(self) -> np.ndarray:
        self.rows = int(self.lib_info()[5])
        x = np.zeros(self.rows)
        self.lib.ref_init_guess(_p(x))
        return x

    def lib_info(self):
        info = np.zeros(10, np.int32)
        self.lib.ref_deck_info(_p(info))
        return info

    def set(self, name: str, values):
        """Overwrite a state array (m./f. + P, sat, x, y, z, label, rho) in
        the layout ``get`` returns."""
        v = np.ascontiguousarray(values, np.float64).ravel().copy()
        if self.lib.ref_set(name.encode(), _p(v)) < 0:
            raise KeyError(name)

    def sat_pressure(self, medium: int, cell: int):
        """(saturation pressure, incipient composition) of one cell as the
        reference's PhaseCtrl computes it."""
        xm = np.zeros(self.nc)
        p = self.lib.ref_sat_pressure(int(medium), ctypes.c_long(int(cell)), _p(xm))
        return float(p), xm

    def sat_pressure_nr(self, kind: int, cell: int):
        """(pressure, Xm) of matrix cell ``cell`` from Bubl_NR (kind 0),
        Dew_NR (1) or LowerDew_Succ (2).  Bubl_NR and Dew_NR have no
        iteration cap: call them only on cells whose restated iteration
        stopped."""
        xm = np.zeros(self.nc)
        p = self.lib.ref_sat_pressure_nr(int(kind), ctypes.c_long(int(cell)), _p(xm))
        return float(p), xm

    def crit_test(self, cell: int) -> int:
        """critTest on one-phase matrix cell ``cell``; its label afterwards."""
        return int(self.lib.ref_crit_test(ctypes.c_long(int(cell))))

    def phase_ctrl(self):
        self.lib.ref_phase_ctrl()

    def update_all(self, x, full: bool):
        x = np.ascontiguousarray(x, np.float64).copy()
        self.lib.ref_update_all(_p(x), int(full))
        self.rows = int(self.lib_info()[5])

    def override_fluid(self, deck):
        """Replace the component table with ``deck``'s (tc, pc, acf, mw, vc,
        zc, parachor, kij) and redo EOS_Init / Tr_Mu; the reference's deck
        keywords cannot carry arbitrary criticals."""
        a = [np.ascontiguousarray(getattr(deck, k), np.float64) for k in
             ("tc", "pc", "acf", "mw", "vc", "zc", "parachor")]
        kij = np.ascontiguousarray(deck.kij, np.float64).ravel()
        if self.lib.ref_override_fluid(int(self.nc), *(_p(v) for v in a), _p(kij)):
            raise ValueError("component count differs from the deck's")

    def relayout(self) -> int:
        """CalcPCoeff + PJac for labels set through ``set``; returns the row count."""
        self.lib.ref_relayout.restype = ctypes.c_long
        self.rows = int(self.lib.ref_relayout())
        return self.rows

    def time_rows(self, rows, x, which: int, t: float = 0.0) -> float:
        """Seconds the reference spends in IteratorFunction (which=0) or
        IteratorJacobian (which=1) over the given global rows, at the state
        of the last ``update_all``."""
        rows = np.ascontiguousarray(rows, np.int64)
        x = np.ascontiguousarray(x, np.float64).copy()
        f = np.zeros(self.rows)
        self.lib.ref_time_rows.restype = ctypes.c_double
        return float(self.lib.ref_time_rows(_p(rows), ctypes.c_long(len(rows)), _p(x), _p(f), ctypes.c_double(t),
                                            int(which)))

    def write_rst(self, directory: str, t: float) -> str:
        """The reference's WriteRST into directory/test.rst."""
        cwd = os.getcwd()
        try:
            os.chdir(directory)
            self.lib.ref_write_rst(ctypes.c_double(t))
        finally:
            os.chdir(cwd)
        return os.path.join(directory, "test.rst")

    def print_all(self, path, t: float):
        """The reference's PrintAll at time t appended to path (one stream
        kept open across calls); path None closes it."""
        self.lib.ref_print_all(None if path is None else path.encode(), ctypes.c_double(t))

    def create_backups(self, t: float):
        self.lib.ref_create_backups(ctypes.c_double(t))

    def time_step_ctrl(self, t: float, rejected: bool):
        """TimeStepCtrl after a pass: (flag, new time); Dt in scalar("Dt")."""
        tt = ctypes.c_double(t)
        flag = self.lib.ref_time_step_ctrl(ctypes.byref(tt), int(bool(rejected)))
        self.rows = int(self.lib_info()[5])
        return int(flag), tt.value

    def time_markers(self):
        out = np.zeros(2 * self.nwells + 1)
        ctrl = ctypes.c_int()
        k = self.lib.ref_time_markers(_p(out), ctypes.byref(ctrl))
        return out[:k], ctrl.value

    def form_function(self, x, t: float = 0.0) -> np.ndarray:
        x = np.ascontiguousarray(x, np.float64).copy()
        f = np.zeros(self.rows)
        self.lib.ref_form_function(_p(x), _p(f), ctypes.c_double(t))
        return f

    def form_jacobian(self, x, t: float = 0.0):
        x = np.ascontiguousarray(x, np.float64).copy()
        cap = self.rows * 10 * (2 * self.nc + 4)
        r = np.zeros(cap, np.int32)
        c = np.zeros(cap, np.int32)
        v = np.zeros(cap)
        n = self.lib.ref_form_jacobian(_p(x), ctypes.c_double(t), ctypes.c_long(cap), _p(r), _p(c), _p(v))
        if n < 0:
            raise RuntimeError("jacobian triplet buffer too small")
        return r[:n], c[:n], v[:n]

"""Reader and writer for the reference simulator's Data_Input deck format.

The format (compsim/Data_Input.cpp:13-1349, compsim/MIfstream.cpp:8-47) is a
stream of whitespace-separated words (printable ASCII 33..126).  Every
keyword is located by scanning the whole deck from its first word for an
exactly equal word, and its values are the words that follow.  Arrays are
given as ``CON v`` (constant), ``VAR v...`` (one value per cell, x fastest,
then y, then z), ``IVAR``/``KVAR`` (one value per i-column / k-layer) or, for
initial conditions in mode 0, ``n*v`` repeat groups (ECLStar,
compsim/Data_Input.cpp:1941-1975).  The reader keeps two of the reference's
quirks that change results: ``JVAR`` loops on an uninitialised counter in
the reference and is rejected here; pseudo-component critical temperatures
from the Cavett correlation are multiplied by the integer quotient 9/5 = 1
(compsim/Init_Calcs.cpp:531).

``Deck`` holds the parsed values as numpy arrays in the library's cell order
(index = i + nx*(j + ny*k)).  ``write_deck`` produces a deck from a plain dict.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

# Component library of the COMPNAME keyword (compsim/Data_Input.cpp:653-952):
# molecular weight [g/mol], Tc [K], Pc [Pa], Vc [cm3/mol], acentric factor,
# parachor, Zc.  Standard literature constants; parachor 0 where the
# reference gives none.
COMPONENT_LIBRARY = {
    "C1": (16.043, 190.56, 4599000, 98.6, 0.008, 74.05, 0.2862),
    "C2": (30.070, 305.32, 4872000, 145.5, 0.0995, 112.91, 0.2793),
    "C3": (44.096, 369.83, 4248000, 200, 0.1523, 154.03, 0.2763),
    "iC4": (58.123, 408.14, 3648000, 262.7, 0.1770, 185.32, 0.2824),
    "nC4": (58.123, 425.12, 3796000, 255, 0.2002, 193.90, 0.2739),
    "iC5": (72.150, 460.43, 3381000, 305.8, 0.2275, 229.37, 0.2701),
    "nC5": (72.150, 469.7, 3370000, 313, 0.2515, 236.00, 0.2701),
    "nC6": (86.177, 507.6, 3025000, 371, 0.3013, 276.71, 0.2659),
    "nC7": (100.204, 540.2, 2740000, 428, 0.3495, 318.44, 0.2611),
    "nC8": (114.231, 568.7, 2490000, 486, 0.3996, 359.33, 0.2559),
    "nC9": (128.258, 594.6, 2290000, 544, 0.4435, 399.57, 0.2520),
    "nC10": (142.285, 617.7, 2110000, 600, 0.4923, 440.69, 0.2465),
    "nC11": (156.312, 639, 1949000, 659, 0.5303, 482.00, 0.2419),
    "nC12": (170.338, 658, 1820000, 716, 0.5764, 522.26, 0.2382),
    "nC13": (184.365, 675, 1680000, 775, 0.6174, 536.77, 0.2320),
    "nC14": (198.392, 693, 1570000, 830, 0.6430, 606.05, 0.2262),
    "nC15": (212.419, 708, 1480000, 889, 0.6863, 647.43, 0.2235),
    "nC16": (226.446, 723, 1400000, 944, 0.7174, 688.50, 0.2199),
    "nC17": (240.473, 736, 1340000, 1000, 0.7697, 730.05, 0.2190),
    "nC18": (254.5, 747, 1270000, 1060, 0.8114, 771.95, 0.2168),
    "nC19": (268.527, 758, 1210000, 1120, 0.8522, 813.85, 0.2150),
    "nC20": (282.553, 768, 1160000, 1170, 0.9069, 853.67, 0.2126),
    "nC21": (296.580, 781.7, 1147000, 1198, 0.9220, 897.64, 0.2114),
    "nC22": (310.610, 791.8, 1101000, 1253, 0.9550, 939.55, 0.2095),
    "nC23": (324.630, 801.3, 1059000, 1307, 0.9890, 981.43, 0.2078),
    "nC24": (338.680, 810.4, 1019000, 1362, 1.0190, 1023.40, 0.2061),
    "CO2": (44.010, 304.19, 7382000, 94, 0.2276, 82.00, 0.2744),
    "O2": (31.999, 154.58, 5043000, 73.4, 0.0218, 0.0, 0.2880),
    "N2": (28.014, 126.1, 3394000, 90.1, 0.0403, 61.12, 0.2917),
    "H2S": (34.082, 373.53, 8963000, 98.5, 0.0827, 85.50, 0.2843),
    "SO2": (64.065, 430.75, 7884000, 122, 0.2451, 0.0, 0.2686),
    "H2": (2.016, 33.18, 1313000, 64.2, 0.2150, 0.0, 0.3053),
    "H2O": (18.015, 647.13, 22055000, 56, 0.3449, 0.0, 0.2294),
}

TIME_FACTOR = 3600.0  # deck times are hours (TIMECHFACT, compsim/Functions.h:243)
LN10 = 2.302585092994046
R_GAS = 8.3144621


class DeckError(ValueError):
    pass


def _num(w: str) -> float:
    """atof(): leading numeric prefix, 0 when none."""
    try:
        return float(w)
    except ValueError:
        j = 0
        while j < len(w) and (w[j].isdigit() or w[j] in "+-.eE"):
            j += 1
        for k in range(j, 0, -1):
            try:
                return float(w[:k])
            except ValueError:
                continue
        return 0.0


class _Words:
    def __init__(self, text: str):
        self.w = "".join(ch if 33 <= ord(ch) <= 126 else " " for ch in text).split()

    def find(self, kw: str):
        """Position after the first word equal to kw, or None."""
        try:
            return self.w.index(kw) + 1
        except ValueError:
            return None

    def need(self, kw: str) -> int:
        p = self.find(kw)
        if p is None:
            raise DeckError(f"No {kw} keyword in the deck")
        return p

    def take(self, p: int, n: int):
        if p + n > len(self.w):
            raise DeckError("deck ends inside a keyword's values")
        return self.w[p:p + n], p + n


@dataclass
class Deck:
    nx: int = 0
    ny: int = 0
    nz: int = 0
    pnc: int = 0
    unc: int = 0
    eos: int = 0                      # 0 PR, 1 SRK
    restemp: float = 0.0              # K
    wat_ro: float = 0.0
    wat_mu: float = 0.0
    di: np.ndarray = None
    dj: np.ndarray = None
    dk: np.ndarray = None
    tor: np.ndarray = None            # [cells]
    por: np.ndarray = None            # [cells]
    fpor: np.ndarray = None
    perm: np.ndarray = None           # [3, cells] mD
    fperm: np.ndarray = None
    cdif: float | None = None         # CDIF value, None when absent
    sigma: float = 1.0
    lf: float = 0.0
    re_f: float = 0.0
    refp: float = 0.0
    cpor: float = 0.0
    dcpor: float = 0.0
    mw: np.ndarray = None             # [nc]
    tc: np.ndarray = None
    pc: np.ndarray = None
    vc: np.ndarray = None             # cm3/mol as in the deck
    acf: np.ndarray = None
    parachor: np.ndarray = None
    zc: np.ndarray = None
    kij: np.ndarray = None            # [nc, nc]
    swt: np.ndarray = None            # [nswt, 4] Sw, krw, krow, Pcow
    sgt: np.ndarray = None            # [nsgt, 4] Sg, krg, krog, Pcgo
    initcond: int = 3
    p0: np.ndarray = None             # [cells] matrix oil pressure
    fp0: np.ndarray = None
    sw0: np.ndarray = None
    fsw0: np.ndarray = None
    z0: np.ndarray = None             # [nc, cells]
    fz0: np.ndarray = None
    wells_i: np.ndarray = None        # [nw, 5]: type, ix, iy, iz0, iz1 (0-based, as welli)
    wells_f: np.ndarray = None        # [nw, nc + 6] (as wellf, times in s)
    dt: float = 0.0                   # s
    total_time: float = 0.0           # s
    dtmax: float = 864000.0
    extra: dict = field(default_factory=dict)

    @property
    def nc(self) -> int:
        return self.pnc + self.unc

    @property
    def cells(self) -> int:
        return self.nx * self.ny * self.nz


def _grid_array(W: _Words, kw: str, nx, ny, nz, required=True, zero_floor=None):
    p = W.find(kw)
    if p is None:
        if required:
            raise DeckError(f"No {kw} keyword in the deck")
        return None
    (mode,), p = W.take(p, 1)
    n = nx * ny * nz
    if mode == "VAR":
        vals, _ = W.take(p, n)
        a = np.array([_num(v) for v in vals], dtype=np.float64)
        if zero_floor is not None:
            a[a == 0] = zero_floor
    elif mode == "CON":
        (v,), _ = W.take(p, 1)
        a = np.full(n, _num(v))
    elif mode == "IVAR":
        vals, _ = W.take(p, nx)
        col = np.array([_num(v) for v in vals])
        a = np.tile(col, ny * nz)
    elif mode == "KVAR":
        vals, _ = W.take(p, nz)
        lay = np.array([_num(v) for v in vals])
        a = np.repeat(lay, nx * ny)
    else:
        raise DeckError(f"Incorrect {kw} keyword format ({mode})")
    return a


def _dims(W: _Words, kw: str, count: int):
    p = W.need(kw)
    (mode,), p = W.take(p, 1)
    if mode == "VAR":
        vals, _ = W.take(p, count)
        return np.array([_num(v) for v in vals])
    if mode == "CON":
        (v,), _ = W.take(p, 1)
        return np.full(count, _num(v))
    raise DeckError(f"Incorrect {kw} keyword format")


def _ecl_stream(W: _Words, p: int, n: int):
    """n values from repeat groups 'k*v' or single values."""
    out = []
    while len(out) < n:
        (w,), p = W.take(p, 1)
        if "*" in w:
            k, v = w.split("*", 1)
            out += [_num(v)] * int(_num(k))
        else:
            out.append(_num(w))
    return np.array(out[:n])


def parse_deck(path: str) -> Deck:
    W = _Words(open(path).read())
    d = Deck()
    p = W.need("GRID")
    (a, b, c), _ = W.take(p, 3)
    d.nx, d.ny, d.nz = int(_num(a)), int(_num(b)), int(_num(c))
    p = W.need("NC")
    (a, b), _ = W.take(p, 2)
    d.pnc, d.unc = int(_num(a)), int(_num(b))
    nc, nx, ny, nz = d.nc, d.nx, d.ny, d.nz
    (v,), _ = W.take(W.need("RESTEMP"), 1)
    d.restemp = _num(v) + 273.15
    (a, b), _ = W.take(W.need("WATERPROPS"), 2)
    d.wat_ro, d.wat_mu = _num(a), _num(b)
    d.di = _dims(W, "DI", nx)
    d.dj = _dims(W, "DJ", ny)
    d.dk = _dims(W, "DK", nz)
    if W.find("TOR") is not None and W.w[W.find("TOR")] == "JVAR":
        raise DeckError("JVAR arrays are not supported (the reference's JVAR loop is malformed)")
    d.tor = _grid_array(W, "TOR", nx, ny, nz, required=False)
    if d.tor is None:
        d.tor = np.ones(nx * ny * nz)
    d.por = _grid_array(W, "POR", nx, ny, nz, zero_floor=1e-11)
    p = W.find("CDIF")
    d.cdif = None if p is None else _num(W.w[p])
    p = W.find("SIGMA")
    d.sigma = 1.0 if p is None else _num(W.w[p])
    p = W.find("DTMAX")
    d.dtmax = 864000.0 if p is None else _num(W.w[p])
    d.fpor = _grid_array(W, "FPOR", nx, ny, nz, zero_floor=1e-11)
    d.lf = _num(W.w[W.need("Lf")])
    d.re_f = _num(W.w[W.need("Re_f")])
    d.perm = np.stack([_grid_array(W, k, nx, ny, nz) for k in ("PERMI", "PERMJ", "PERMK")])
    d.fperm = np.stack([_grid_array(W, k, nx, ny, nz) for k in ("FPERMI", "FPERMJ", "FPERMK")])
    for key in ("REFP", "CPOR", "DCPOR"):
        p = W.find(key)
        setattr(d, key.lower(), 0.0 if p is None else _num(W.w[p]))
    (m,), _ = W.take(W.need("MODEL"), 1)
    if m not in ("PR", "SRK"):
        raise DeckError("Incorrect EOS keyword format")
    d.eos = 0 if m == "PR" else 1
    d.mw, d.tc, d.pc, d.vc, d.acf, d.parachor, d.zc = (np.zeros(nc) for _ in range(7))
    sg, tb = np.zeros(nc), np.zeros(nc)
    if d.unc:
        for key, arr in (("SG", sg), ("TB", tb), ("MW", d.mw), ("AC", d.acf), ("PCRIT", d.pc), ("TCRIT", d.tc),
                         ("VCRIT", d.vc), ("ZCRIT", d.zc)):
            p = W.find(key)
            if p is not None:
                vals, _ = W.take(p, d.unc)
                arr[d.pnc:] = [_num(v) for v in vals]
        # pseudo-component correlations, compsim/Init_Calcs.cpp:521-545
        for i in range(d.pnc, nc):
            Tb = tb[i] * 5 / 9 - 459.67
            API = 141.5 / sg[i] - 131.5
            Tc = (768.071 + 1.7134 * Tb - 1.0834e-3 * Tb * Tb + 3.889e-7 * Tb * Tb * Tb - 8.9213e-3 * Tb * API
                  + 5.3095e-6 * Tb * Tb * API + 3.2712e-8 * Tb * Tb * API * API)
            d.tc[i] = 1 * Tc  # the reference multiplies by the integer quotient 9/5 = 1
            Pc = (2.829 + 9.412e-4 * Tb - 3.0475e-6 * Tb * Tb + 1.5184e-9 * Tb * Tb * Tb - 2.0876e-5 * Tb * API
                  + 1.1048e-8 * Tb * Tb * API - 4.827e-8 * Tb * API * API + 1.395e-10 * Tb * Tb * API * API)
            d.pc[i] = 6897.549353301566 * math.exp(Pc * LN10)
            d.acf[i] = (3.0 / 7.0) * math.log(d.pc[i] / 101325) / (LN10 * (d.tc[i] / tb[i] - 1)) - 1
            Zc = 0.2901 - 0.0879 * d.acf[i]
            d.vc[i] = Zc * R_GAS * d.tc[i] / d.pc[i]
    p = W.need("COMPNAME")
    names, _ = W.take(p, d.pnc)
    for i, nm in enumerate(names):
        if nm not in COMPONENT_LIBRARY:
            raise DeckError(f"Unknown Component {nm}")
        d.mw[i], d.tc[i], d.pc[i], d.vc[i], d.acf[i], d.parachor[i], d.zc[i] = COMPONENT_LIBRARY[nm]
    d.extra["compnames"] = list(names)
    (n,), p = W.take(W.need("SWT"), 1)
    vals, _ = W.take(p, int(_num(n)) * 4)
    d.swt = np.array([_num(v) for v in vals]).reshape(-1, 4)
    (n,), p = W.take(W.need("SGT"), 1)
    vals, _ = W.take(p, int(_num(n)) * 4)
    d.sgt = np.array([_num(v) for v in vals]).reshape(-1, 4)
    # zero entries of the tables become RELPERM0 = 0, compsim/Data_Input.cpp:956-975
    d.kij = np.zeros((nc, nc))
    p = W.find("BIC")
    if p is not None:
        for i in range(1, nc):
            for j in range(i):
                (v,), p = W.take(p, 1)
                d.kij[i, j] = d.kij[j, i] = _num(v)
    (mode,), _ = W.take(W.need("INITCOND"), 1)
    d.initcond = int(_num(mode))
    n = nx * ny * nz
    if d.initcond == 0:
        d.p0 = _ecl_stream(W, W.need("IPRESS"), n)
        d.fp0 = _ecl_stream(W, W.need("FIPRESS"), n)
        d.sw0 = _ecl_stream(W, W.need("IWS"), n)
        d.fsw0 = _ecl_stream(W, W.need("FIWS"), n)
        d.z0 = _ecl_stream(W, W.need("IGC"), nc * n).reshape(nc, n)
        d.fz0 = _ecl_stream(W, W.need("FIGC"), nc * n).reshape(nc, n)
    elif d.initcond == 1:
        def layers(kw, per):
            vals, _ = W.take(W.need(kw), nz * per)
            return np.array([_num(v) for v in vals]).reshape(nz, per)
        d.p0 = np.repeat(layers("IPRESS", 1)[:, 0], nx * ny)
        d.fp0 = np.repeat(layers("FIPRESS", 1)[:, 0], nx * ny)
        d.sw0 = np.repeat(layers("IWS", 1)[:, 0], nx * ny)
        d.fsw0 = np.repeat(layers("FIWS", 1)[:, 0], nx * ny)
        d.z0 = np.repeat(layers("IGC", nc).T, nx * ny, axis=1)
        d.fz0 = np.repeat(layers("FIGC", nc).T, nx * ny, axis=1)
    elif d.initcond == 3:
        def one(kw, per=1):
            vals, _ = W.take(W.need(kw), per)
            return np.array([_num(v) for v in vals])
        d.p0 = np.full(n, one("IPRESS")[0])
        d.fp0 = np.full(n, one("FIPRESS")[0])
        d.sw0 = np.full(n, one("IWS")[0])
        d.fsw0 = np.full(n, one("FIWS")[0])
        d.z0 = np.repeat(one("IGC", nc)[:, None], n, axis=1)
        d.fz0 = np.repeat(one("FIGC", nc)[:, None], n, axis=1)
    else:
        raise DeckError(f"INITCOND {d.initcond} is not supported")
    (nw,), p = W.take(W.need("WELLS"), 1)
    nw = int(_num(nw))
    wi = np.zeros((nw, 5), dtype=np.int32)
    wf = np.zeros((nw, nc + 6))
    for w in range(nw):
        ints, p = W.take(p, 5)
        wi[w] = [int(_num(v)) - 1 for v in ints]
        wi[w, 0] += 1
        t = wi[w, 0]
        if t in (3, 8):
            cnt, tstart = nc + 6, nc + 3
        elif 0 <= t <= 7:
            cnt, tstart = 6, 3
        else:
            raise DeckError("Incorrect WELL keyword format")
        vals, p = W.take(p, cnt)
        for j, v in enumerate(vals):
            wf[w, j] = _num(v) * (TIME_FACTOR if j > tstart else 1.0)
    d.wells_i, d.wells_f = wi, wf
    d.dt = _num(W.w[W.need("DT")]) * TIME_FACTOR
    d.total_time = _num(W.w[W.need("TOTALT")]) * TIME_FACTOR
    return d


# ----------------------------------------------------------------------------- writer

TSTEPTOL = 1.0   # markers closer than this (s) merge (compsim/Functions.h:264)


def time_markers(d: Deck):
    """The run's time markers and first step length: every well's start and
    end time and the total time (compsim/Data_Input.cpp:1205-1344), sorted,
    with zero markers and markers closer than TSTEPTOL to the next one removed,
    and a first Dt cut to 1/2.1 of the first marker when it reaches it
    (ManageTSMarker, compsim/Init_Calcs.cpp:1133-1157).  Returns (markers,
    dt)."""
    nw = len(d.wells_i)
    m = []
    for w in range(nw):
        t = int(d.wells_i[w, 0])
        ts = d.nc + 3 if t in (3, 8) else 3
        m += [float(d.wells_f[w, ts + 1]), float(d.wells_f[w, ts + 2])]
    m.append(float(d.total_time))
    n = 2 * nw
    m.sort()
    j = 0
    for i in range(n):
        if abs(m[i - j] - m[i - j + 1]) < TSTEPTOL or not m[i - j]:
            for k in range(i - j, n - j):
                m[k] = m[k + 1]
            j += 1
    m = m[:n - j + 1]
    dt = d.dt if d.dt < m[0] else m[0] / 2.1
    return np.array(m), dt


def _fmt(v) -> str:
    return repr(float(v)) if not float(v).is_integer() else str(int(v)) if abs(v) < 1e15 else repr(float(v))


def write_deck(path: str, spec: dict) -> str:
    """Write a deck from a dict: keys follow the keywords (see config_deck)."""
    L = []
    nx, ny, nz = spec["grid"]
    L.append(f"GRID {nx} {ny} {nz}")
    for kw, key in (("DI", "di"), ("DJ", "dj"), ("DK", "dk")):
        v = np.atleast_1d(spec[key])
        L.append(f"{kw} CON {_fmt(v[0])}" if v.size == 1 else f"{kw} VAR " + " ".join(_fmt(x) for x in v))
    for kw, key in (("POR", "por"), ("FPOR", "fpor"), ("PERMI", "permi"), ("PERMJ", "permj"), ("PERMK", "permk"),
                    ("FPERMI", "fpermi"), ("FPERMJ", "fpermj"), ("FPERMK", "fpermk")):
        v = np.atleast_1d(spec[key])
        L.append(f"{kw} CON {_fmt(v[0])}" if v.size == 1 else f"{kw} VAR\n" + " ".join(_fmt(x) for x in v))
    L.append(f"Lf {_fmt(spec['lf'])}")
    L.append(f"Re_f {_fmt(spec['re_f'])}")
    L.append(f"MODEL {spec['model']}")
    L.append(f"NC {len(spec['comps'])} 0")
    L.append("COMPNAME " + " ".join(spec["comps"]))
    if spec.get("bic") is not None:
        k = np.asarray(spec["bic"])
        L.append("BIC " + " ".join(_fmt(k[i, j]) for i in range(1, k.shape[0]) for j in range(i)))
    for kw in ("SGT", "SWT"):
        t = np.asarray(spec[kw.lower()])
        L.append(f"{kw} {t.shape[0]}")
        L += [" ".join(_fmt(x) for x in row) for row in t]
    L.append(f"REFP {_fmt(spec.get('refp', 101325))}")
    L.append(f"CPOR {_fmt(spec.get('cpor', 0))}")
    L.append(f"DCPOR {_fmt(spec.get('dcpor', 0))}")
    wells = spec.get("wells", [])
    L.append(f"WELLS {len(wells)}")
    L += [" ".join(_fmt(x) for x in w) for w in wells]
    L.append(f"RESTEMP {_fmt(spec['restemp_c'])}")
    L.append(f"WATERPROPS {_fmt(spec.get('wat_ro', 1000))} {_fmt(spec.get('wat_mu', 1))}")
    L.append(f"DT {_fmt(spec.get('dt', 0.01))}")
    L.append(f"TOTALT {_fmt(spec.get('totalt', 17520))}")
    L.append(f"DTMAX {_fmt(spec.get('dtmax', 100))}")
    if spec.get("cdif") is not None:
        L.append(f"CDIF {_fmt(spec['cdif'])}")
    if np.ndim(spec["ipress"]) == 0:
        L.append("INITCOND 3")
        L.append(f"IPRESS {_fmt(spec['ipress'])}")
        L.append(f"IWS {_fmt(spec['iws'])}")
        L.append("IGC " + " ".join(_fmt(x) for x in spec["igc"]))
        L.append(f"FIPRESS {_fmt(spec['fipress'])}")
        L.append(f"FIWS {_fmt(spec['fiws'])}")
        L.append("FIGC " + " ".join(_fmt(x) for x in spec["figc"]))
    else:
        # one value (or composition row) per layer
        nz = spec["grid"][2]
        def lay(v, per):
            a = np.asarray(v, dtype=float).reshape(-1)
            return a if a.size == nz * per else np.tile(a, nz)
        L.append("INITCOND 1")
        L.append("IPRESS " + " ".join(_fmt(x) for x in lay(spec["ipress"], 1)))
        L.append("IWS " + " ".join(_fmt(x) for x in lay(spec["iws"], 1)))
        L.append("IGC " + " ".join(_fmt(x) for x in lay(spec["igc"], len(spec["comps"]))))
        L.append("FIPRESS " + " ".join(_fmt(x) for x in lay(spec["fipress"], 1)))
        L.append("FIWS " + " ".join(_fmt(x) for x in lay(spec["fiws"], 1)))
        L.append("FIGC " + " ".join(_fmt(x) for x in lay(spec["figc"], len(spec["comps"]))))
    text = "\n".join(L) + "\n"
    with open(path, "w") as fh:
        fh.write(text)
    return path


# Saturation tables of the reference's sample deck (compsim/test.dat:26-55):
# Sg, krg, krog, Pcgo and Sw, krw, krow, Pcow.
SAMPLE_SGT = [
    [0, 0, 1, 0], [0.031, 0.0131, 0.6702, 40667.85714], [0.063, 0.0173, 0.55, 51765.35714],
    [0.094, 0.0226, 0.4395, 62035.71429], [0.125, 0.0297, 0.3395, 72030.35714], [0.188, 0.0515, 0.1721, 94087.5],
    [0.298, 0.1399, 0.028, 256483.2143], [0.386, 0.3939, 0.002, 419085.7143], [0.438, 0.5456, 0, 1671517.857],
    [0.565, 0.6215, 0, 2566900], [0.684, 0.6784, 0, 3995100], [0.8, 1, 0, 26824242.86]]
SAMPLE_SWT = [
    [0.2, 0, 1, 1349897.143], [0.229, 0.0001, 0.7407, 656200], [0.255, 0.0003, 0.6829, 413571.4286],
    [0.308, 0.0012, 0.5722, 151642.8571], [0.334, 0.0023, 0.5194, 129585.7143], [0.412, 0.0102, 0.3715, 86850],
    [0.464, 0.0219, 0.1526, 58106.78571], [0.557, 0.0416, 0.0822, 30328.57143], [0.606, 0.0721, 0, 9098.571429],
    [0.647, 0.1448, 0, 0], [0.7, 0.178, 0, 0], [0.8, 0.2604, 0, 0], [1, 1, 0, 0]]


def config_deck(nx=10, ny=10, nz=3, seed=1, cdif=0.0, ipress=2e7, iws=0.2, restemp_c=86.85,
                comps=("C1", "nC4", "nC10"), igc=(0.5, 0.2, 0.3), bic=None, wells=True, fipress=None,
                figc=None) -> dict:
    """The small plain case: nx x ny x nz dual-porosity grid, matrix porosity
    0.20, fracture porosity 0.01, log-normal matrix permeability (median 10 mD,
    sigma_ln 0.5, seeded; the median is exp(mean of ln k)), fracture
    permeability, saturation tables, Lf, Re_f and block sizes of the
    reference's sample deck, PR, a gas injector (type 8) and a producer
    (type 0) at opposite corners spanning all layers.  cdif=None drops the
    CDIF keyword (diffusive matrix-fracture transfer on)."""
    rng = np.random.default_rng(seed)
    n = nx * ny * nz
    k = np.exp(np.log(10.0) + 0.5 * rng.standard_normal((3, n)))
    nc = len(comps)
    if bic is None:
        bic = np.zeros((nc, nc))
        if nc == 3:
            bic[0, 2] = bic[2, 0] = 0.04
    inj = [8, 1, 1, 1, nz, 50, 14000000, 0, 0.1] + [1] + [0] * (nc - 1) + [1, 17520]
    prod = [0, nx, ny, 1, nz, 7000000, 10, 0, 0.1, 1, 17520]
    return dict(grid=(nx, ny, nz), di=100, dj=100, dk=50, por=0.20, fpor=0.01, permi=k[0], permj=k[1], permk=k[2],
                fpermi=1000, fpermj=1000, fpermk=1000, lf=0.01, re_f=1000000, model="PR", comps=list(comps), bic=bic,
                sgt=SAMPLE_SGT, swt=SAMPLE_SWT, refp=101325, cpor=0, dcpor=0,
                wells=[inj, prod] if wells else [], restemp_c=restemp_c, wat_ro=1000, wat_mu=1, dt=0.01,
                totalt=17520, dtmax=100, cdif=cdif, ipress=ipress, iws=iws, igc=np.asarray(igc).tolist(),
                fipress=ipress if fipress is None else fipress, fiws=0,
                figc=np.asarray(igc if figc is None else figc).tolist())


def all_wells_deck(ipress=9e6, cdif=None) -> dict:
    """A 6 x 5 x 3 plain-case grid carrying one well of every type 0..8, at
    interior, edge and corner blocks (so every branch of the completion
    radius is used), two-phase at 9 MPa."""
    spec = config_deck(nx=6, ny=5, nz=3, cdif=cdif, ipress=ipress, seed=9)
    t = [1, 17520]
    spec["wells"] = [
        [0, 3, 3, 1, 2, 9.5e6, 1e-6, 0.5, 0.1] + t,       # constant Pwf production, interior, rate cap
        [1, 1, 3, 1, 3, 9.5e6, 1e-6, 0, 0.1] + t,         # constant Pwf gas production, edge x = 0
        [2, 6, 3, 2, 3, 9.5e6, 1e-6, 0, 0.1] + t,         # constant Pwf water injection, edge x = nx
        [3, 3, 1, 1, 3, 9.5e6, 1e-6, 0, 0.1, 0.9, 0.1, 0.0] + t,  # constant Pwf gas injection, edge y = 0
        [4, 3, 5, 1, 3, 0.5, 8e6, 0, 0.1] + t,            # constant oil rate, edge y = ny
        [5, 1, 5, 1, 3, 8e6, 0.5, 0, 0.1] + t,            # constant gas rate, corner (0, ny)
        [6, 6, 1, 1, 3, 0.5, 8e6, 0, 0.1] + t,            # constant total rate, corner (nx, 0)
        [7, 2, 2, 1, 3, 0.5, 9.5e6, 0, 0.1] + t,          # constant water injection rate, interior
        [8, 5, 4, 1, 3, 0.5, 9.5e6, 0, 0.1, 1, 0, 0] + t,  # constant gas injection rate, interior
    ]
    return spec


def sample_deck(ipress=12000000.0, iws=0.2, cdif=0.0) -> dict:
    """The reference's own sample deck (compsim/test.dat): 10 x 10 x 5,
    PR with C1 C2 nC5 nC10 nC15, initial pressure 12 MPa, feed
    (0, 0.1, 0.1, 0.3, 0.5), a gas injector (type 8) and a producer
    (type 0), CDIF 0."""
    spec = config_deck(nx=10, ny=10, nz=5, cdif=cdif, ipress=ipress, iws=iws, restemp_c=80,
                       comps=("C1", "C2", "nC5", "nC10", "nC15"), igc=(0, 0.1, 0.1, 0.3, 0.5),
                       bic=np.zeros((5, 5)))
    spec.update(permi=10, permj=10, permk=10, por=0.1932, fpor=0.02, fpermi=1000, fpermj=1000, fpermk=1000)
    spec["wells"] = [[8, 1, 1, 1, 5, 50, 14000000, 0, 0.1, 1, 0, 0, 0, 0, 1, 17520],
                     [0, 10, 10, 1, 1, 7000000, 10, 0, 0.1, 1, 17520]]
    return spec

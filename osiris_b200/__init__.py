"""osiris_b200: B200-native FP64 hot path of the Osiris reservoir simulator.

The compute lives in the CUDA library ``_lib/libosiris_b200.so`` (C ABI:
``include/osiris_b200.h``).  This module is a thin ctypes host mirror over
that ABI; PyTorch only supplies device memory and streams.  There is no CPU
fallback: every entry point raises if the library is missing or a call
fails.

Conventions (shared with the C ABI): per-cell scalars ``[n]``,
per-component fields ``[nc, n]``, fugacity derivative blocks
``[2, nc, nc, n]`` / ``[2, nc, n]`` with phase 0 = liquid, 1 = vapour; phase
labels +1 liquid only, -1 vapour only, 0 two-phase.
"""
from __future__ import annotations

import ctypes
import os
import re

import numpy as np

from .build import INCLUDE, LIB

__all__ = ["Fluid", "lib", "flash", "flash_host", "fugacity_derivs", "flash_adjoint", "flash_instances", "set_shape", "get_shape", "header_symbols", "OsrError",
           "FLASH_OUTPUTS"]

_vp = ctypes.c_void_p
_lib = None


class OsrError(RuntimeError):
    pass


class _CFluid(ctypes.Structure):
    _fields_ = [("nc", ctypes.c_int), ("eos", ctypes.c_int), ("tc", _vp), ("pc", _vp), ("acf", _vp),
                ("kij", _vp)]


class _CFlashOut(ctypes.Structure):
    _fields_ = [("label", _vp), ("L", _vp), ("x", _vp), ("y", _vp), ("Zl", _vp), ("Zg", _vp), ("iters", _vp),
                ("rr_iters", _vp), ("dlnphi_dx", _vp), ("dlnphi_dP", _vp)]


class KspOpts(ctypes.Structure):
    """osr_ksp_opts: RELTOL, ABSTOL, DIVTOL, MAXITERS and the host poll interval."""
    _fields_ = [("rtol", ctypes.c_double), ("atol", ctypes.c_double), ("dtol", ctypes.c_double),
                ("max_it", ctypes.c_int), ("check_every", ctypes.c_int)]


class KspInfo(ctypes.Structure):
    """osr_ksp_info: PETSc KSPConvergedReason, iterations, residual norms."""
    _fields_ = [("reason", ctypes.c_int), ("its", ctypes.c_int), ("rnorm0", ctypes.c_double),
                ("rnorm", ctypes.c_double)]


def ksp_opts(**kw) -> KspOpts:
    """The reference's KSP tolerances (osr_ksp_default_opts) with overrides."""
    o = KspOpts()
    lib().osr_ksp_default_opts(ctypes.byref(o))
    for k, v in kw.items():
        setattr(o, k, v)
    return o


class StepInfo(ctypes.Structure):
    """osr_step_info of one pass of the main loop."""
    _fields_ = [("sim_time", ctypes.c_double), ("dt", ctypes.c_double), ("accepted", ctypes.c_int),
                ("finished", ctypes.c_int), ("ksp_reason", ctypes.c_int), ("ksp_its", ctypes.c_int),
                ("vnorm", ctypes.c_double), ("rows", ctypes.c_long)]


R_GAS = 8.3144621   # RGAS, J/(mol K)

FLASH_OUTPUTS = ("label", "L", "x", "y", "Zl", "Zg", "iters", "rr_iters", "dlnphi_dx", "dlnphi_dP")


def header_signatures():
    """(return type, name, [parameter declarations]) of every function the
    public header declares."""
    out = []
    for h in sorted(os.listdir(INCLUDE)):
        if h.endswith(".h"):
            text = open(os.path.join(INCLUDE, h)).read()
            text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
            text = re.sub(r"//[^\n]*", "", text)
            for ret, name, params in re.findall(
                    r"^\s*((?:const\s+)?[A-Za-z_]\w*\s*\**)\s*(osr_[a-z0-9_]+)\s*\(([^;{]*?)\)\s*;", text, flags=re.M):
                ps = [p.strip() for p in params.split(",")]
                out.append((ret.strip(), name, [] if ps == ["void"] else ps))
    return out


def header_symbols():
    """Every function the public header declares."""
    return sorted({name for _, name, _ in header_signatures()})


_SCALARS = {"int": ctypes.c_int, "osr_status": ctypes.c_int, "long": ctypes.c_long, "double": ctypes.c_double}


def _ctype(decl: str):
    """ctypes type of one C declaration (a parameter or a return type).
    Every pointer is a full-width address; passing an address as a bare
    Python int without this would truncate it to a C int."""
    if "*" in decl:
        return ctypes.c_char_p if re.match(r"(const\s+)?char\s*\*\s*\w*$", decl) else ctypes.c_void_p
    if decl.strip() == "void":
        return None
    base = re.sub(r"\s+\w+$", "", decl.strip()) if len(decl.split()) > 1 else decl.strip()
    if base not in _SCALARS:
        raise OsrError(f"unmapped C type in header: {decl!r}")
    return _SCALARS[base]


def lib():
    """Load the CUDA library (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            raise OsrError(f"{LIB} is missing: run `python -m osiris_b200.build` (no CPU fallback exists)")
        L = ctypes.CDLL(LIB)
        for ret, name, params in header_signatures():
            fn = getattr(L, name)  # every declared entry point must resolve
            fn.restype = _ctype(ret)
            fn.argtypes = [_ctype(p) for p in params]
        _lib = L
    return _lib


def _check(rc: int, what: str):
    if rc != 0:
        L = lib()
        msg = L.osr_status_string(rc).decode()
        raise OsrError(f"{what}: status {rc} ({msg}), cuda error {L.osr_last_cuda_error()}")


class Fluid:
    """Component table: Tc [K], Pc [Pa], acentric factor, kij (symmetric, zero
    diagonal); eos 0 = Peng-Robinson, 1 = Soave-Redlich-Kwong."""

    def __init__(self, tc, pc, acf, kij, eos: int):
        self.tc = np.ascontiguousarray(tc, dtype=np.float64)
        self.pc = np.ascontiguousarray(pc, dtype=np.float64)
        self.acf = np.ascontiguousarray(acf, dtype=np.float64)
        self.kij = np.ascontiguousarray(kij, dtype=np.float64)
        self.nc = int(self.tc.shape[0])
        self.eos = int(eos)
        if self.kij.shape != (self.nc, self.nc):
            raise ValueError("kij must be [nc, nc]")
        self._c = _CFluid(self.nc, self.eos, self.tc.ctypes.data, self.pc.ctypes.data, self.acf.ctypes.data,
                          self.kij.ctypes.data)

    @property
    def cref(self):
        return ctypes.byref(self._c)


def _out_struct(outs: dict, ptr):
    return _CFlashOut(*[ptr(outs[k]) if outs.get(k) is not None else None for k in FLASH_OUTPUTS])


def alloc_flash_outputs(nc: int, n: int, derivs: bool, device, iters: bool = True):
    import torch
    f64 = dict(dtype=torch.float64, device=device)
    o = dict(label=torch.empty(n, dtype=torch.int8, device=device), L=torch.empty(n, **f64),
             x=torch.empty(nc, n, **f64), y=torch.empty(nc, n, **f64), Zl=torch.empty(n, **f64),
             Zg=torch.empty(n, **f64))
    if iters:
        o["iters"] = torch.empty(n, dtype=torch.int32, device=device)
        o["rr_iters"] = torch.empty(n, dtype=torch.int32, device=device)
    if derivs:
        o["dlnphi_dx"] = torch.empty(2, nc, nc, n, **f64)
        o["dlnphi_dP"] = torch.empty(2, nc, n, **f64)
    return o


def flash(fluid: Fluid, P, T, z, derivs: bool = True, form: str = "batched", out: dict | None = None,
          stream=None, iters: bool = True):
    """Flash cells held in device memory (torch CUDA float64 tensors P [n],
    T [n], z [nc, n]).  Returns (or fills) a dict of device tensors.
    Asynchronous on the current torch stream unless ``stream`` is given."""
    import torch
    n = int(P.shape[0])
    for t in (P, T, z):
        if not (t.is_cuda and t.dtype == torch.float64 and t.is_contiguous()):
            raise OsrError("P, T, z must be contiguous float64 CUDA tensors")
    if z.shape != (fluid.nc, n):
        raise OsrError("z must be [nc, n]")
    if out is None:
        out = alloc_flash_outputs(fluid.nc, n, derivs, P.device, iters)
    if stream is None:
        stream = torch.cuda.current_stream(P.device)
    co = _out_struct(out, lambda t: t.data_ptr())
    fn = {"batched": lib().osr_flash_batch, "plain": lib().osr_flash_batch_plain,
          "noalloc": lib().osr_flash_batch_noalloc}[form]
    # the library takes its scratch on the current device: make it the tensors'
    with torch.cuda.device(P.device):
        rc = fn(fluid.cref, _vp(P.data_ptr()), _vp(T.data_ptr()), _vp(z.data_ptr()), ctypes.c_long(n),
                ctypes.byref(co), _vp(stream.cuda_stream))
    _check(rc, f"osr_flash_batch ({form})")
    return out


def fugacity_derivs(fluid: Fluid, P, T, x, y, Zl, Zg, out: dict | None = None, stream=None):
    """d ln(phi)/d w and d ln(phi)/d P of both phases at given device states
    (``osr_fugacity_derivs``): P, T, Zl, Zg [n], x, y [nc, n] contiguous
    float64 CUDA tensors.  Returns (or fills) {"dlnphi_dx": [2, nc, nc, n],
    "dlnphi_dP": [2, nc, n]}."""
    import torch
    n, nc = int(P.shape[0]), fluid.nc
    for t in (P, T, x, y, Zl, Zg):
        if not (t.is_cuda and t.dtype == torch.float64 and t.is_contiguous()):
            raise OsrError("inputs must be contiguous float64 CUDA tensors")
    if x.shape != (nc, n) or y.shape != (nc, n):
        raise OsrError("x and y must be [nc, n]")
    if out is None:
        out = {"dlnphi_dx": torch.empty((2, nc, nc, n), dtype=torch.float64, device=P.device),
               "dlnphi_dP": torch.empty((2, nc, n), dtype=torch.float64, device=P.device)}
    if stream is None:
        stream = torch.cuda.current_stream(P.device)
    with torch.cuda.device(P.device):
        _check(lib().osr_fugacity_derivs(fluid.cref, *(_vp(t.data_ptr()) for t in (P, T, x, y, Zl, Zg)),
                                         ctypes.c_long(n), _vp(out["dlnphi_dx"].data_ptr()),
                                         _vp(out["dlnphi_dP"].data_ptr()), _vp(stream.cuda_stream)),
               "osr_fugacity_derivs")
    return out


def flash_adjoint(fluid: Fluid, P, T, z, state: dict, xbar, ybar, Lbar, want_z: bool = True, want_P: bool = True,
                  stream=None) -> dict:
    """Implicit-function adjoint of a flash result (osr_flash_adjoint):
    device tensors P, T [n], z [nc, n], the flash's outputs ``state`` and
    cotangents xbar, ybar [nc, n], Lbar [n].  Returns {"kij_bar": [nc, nc],
    "z_bar": [nc, n] | None, "P_bar": [n] | None, "singular": count}."""
    import torch
    n, nc = int(P.shape[0]), fluid.nc
    for t in (P, T, z, xbar, ybar, Lbar):
        if not (t.is_cuda and t.dtype == torch.float64 and t.is_contiguous()):
            raise OsrError("inputs and cotangents must be contiguous float64 CUDA tensors")
    dev = P.device
    kb = torch.empty((nc, nc), dtype=torch.float64, device=dev)
    zb = torch.empty((nc, n), dtype=torch.float64, device=dev) if want_z else None
    pb = torch.empty(n, dtype=torch.float64, device=dev) if want_P else None
    if stream is None:
        stream = torch.cuda.current_stream(dev)
    co = _out_struct(state, lambda t: t.data_ptr())
    sing = ctypes.c_long()
    with torch.cuda.device(dev):
        _check(lib().osr_flash_adjoint(fluid.cref, _vp(P.data_ptr()), _vp(T.data_ptr()), _vp(z.data_ptr()),
                                       ctypes.c_long(n), ctypes.byref(co), _vp(xbar.data_ptr()),
                                       _vp(ybar.data_ptr()), _vp(Lbar.data_ptr()), _vp(kb.data_ptr()),
                                       None if zb is None else _vp(zb.data_ptr()),
                                       None if pb is None else _vp(pb.data_ptr()), ctypes.byref(sing),
                                       _vp(stream.cuda_stream)), "osr_flash_adjoint")
    return {"kij_bar": kb, "z_bar": zb, "P_bar": pb, "singular": int(sing.value)}


CELL_STATUS = {0: "OK", 1: "MAXIT", 2: "NAN", 3: "NOROOT", 4: "RANGE"}


def flash_status(out: dict, nc: int, stream=None) -> dict:
    """Per-cell status of a device flash result (osr_flash_status): {"status":
    int8 [n] device tensor, "counts": {OK, MAXIT, NAN, NOROOT}, "first_bad":
    lowest non-OK cell or -1}."""
    import torch
    n = int(out["L"].shape[0])
    st = torch.empty(n, dtype=torch.int8, device=out["L"].device)
    counts = (ctypes.c_long * 4)()
    first = ctypes.c_long()
    if stream is None:
        stream = torch.cuda.current_stream(out["L"].device)
    co = _out_struct(out, lambda t: t.data_ptr())
    with torch.cuda.device(out["L"].device):
        _check(lib().osr_flash_status(ctypes.byref(co), int(nc), ctypes.c_long(n), _vp(st.data_ptr()), counts,
                                      ctypes.byref(first), _vp(stream.cuda_stream)), "osr_flash_status")
    return {"status": st, "counts": {CELL_STATUS[k]: int(counts[k]) for k in range(4)}, "first_bad": first.value}


def flash_host(fluid: Fluid, P, T, z, derivs: bool = True, out: dict | None = None, iters: bool = True):
    """End-to-end flash of host (numpy) arrays through osr_flash_batch_host.
    Inputs may be pinned torch CPU tensors or numpy arrays."""
    def host_ptr(a):
        if hasattr(a, "data_ptr"):
            return a.data_ptr()
        return a.ctypes.data
    n = int(P.shape[0])
    nc = fluid.nc
    if out is None:
        out = dict(label=np.empty(n, np.int8), L=np.empty(n), x=np.empty((nc, n)), y=np.empty((nc, n)),
                   Zl=np.empty(n), Zg=np.empty(n))
        if iters:
            out["iters"] = np.empty(n, np.int32)
            out["rr_iters"] = np.empty(n, np.int32)
        if derivs:
            out["dlnphi_dx"] = np.empty((2, nc, nc, n))
            out["dlnphi_dP"] = np.empty((2, nc, n))
    co = _out_struct(out, host_ptr)
    rc = lib().osr_flash_batch_host(fluid.cref, _vp(host_ptr(P)), _vp(host_ptr(T)), _vp(host_ptr(z)),
                                    ctypes.c_long(n), ctypes.byref(co), None)
    _check(rc, "osr_flash_batch_host")
    return out


def flash_passes() -> int:
    """Launches of the batched flash kernel per call with the current shape:
    park_after, doubling, ending at 500 substitution steps."""
    park = get_shape()[3]
    if park <= 0:
        return 1
    n, s = 0, park
    while s < 500 and n < 11:
        n += 1
        s *= 2
    return n + 1


def flash_instances(fluids, start, P, T, z, derivs: bool = True, out: dict | None = None, stream=None,
                    iters: bool = True):
    """Flash several instances of one component count in one batched call
    (``osr_flash_batch_instances``): ``fluids`` a list of Fluid, ``start``
    host int64 [len(fluids) + 1] cell offsets, P/T/z device tensors of all
    instances' cells.  Returns (or fills) the output dict."""
    import torch
    n = int(P.shape[0])
    nc = fluids[0].nc
    start = np.ascontiguousarray(start, dtype=np.int64)
    if start.shape != (len(fluids) + 1,):
        raise OsrError("start must have len(fluids) + 1 entries")
    arr = (_CFluid * len(fluids))(*[f._c for f in fluids])
    if out is None:
        out = alloc_flash_outputs(nc, n, derivs, P.device, iters)
    if stream is None:
        stream = torch.cuda.current_stream(P.device)
    co = _out_struct(out, lambda t: _vp(t.data_ptr()))
    _check(lib().osr_flash_batch_instances(arr, len(fluids), _vp(start.ctypes.data), _vp(P.data_ptr()),
                                           _vp(T.data_ptr()), _vp(z.data_ptr()), ctypes.c_long(n),
                                           ctypes.byref(co), _vp(stream.cuda_stream)), "osr_flash_batch_instances")
    return out


class _CFlashGroup(ctypes.Structure):
    _fields_ = [("fluids", _vp), ("n_inst", ctypes.c_int), ("inst_start", _vp), ("d_P", _vp), ("d_T", _vp),
                ("d_z", _vp), ("n", ctypes.c_long), ("out", _vp)]


class FlashPlan:
    """Instance groups of several component counts flashed as one CUDA graph
    (osr_flash_plan_*): ``groups`` a list of dicts with ``fluids`` (list of
    Fluid, one component count), ``start`` (host int64 cell offsets), device
    tensors ``P``, ``T``, ``z`` and an output dict ``out``.  ``run`` is one
    graph launch; refill the input tensors in place between runs."""

    def __init__(self, groups):
        self.groups = groups       # keeps the device tensors alive
        keep, cg = [], []
        for g in groups:
            fl = g["fluids"]
            arr = (_CFluid * len(fl))(*[f._c for f in fl])
            start = np.ascontiguousarray(g["start"], dtype=np.int64)
            co = _out_struct(g["out"], lambda t: _vp(t.data_ptr()))
            keep += [arr, start, co]
            cg.append(_CFlashGroup(ctypes.cast(arr, _vp), len(fl), _vp(start.ctypes.data), _vp(g["P"].data_ptr()),
                                   _vp(g["T"].data_ptr()), _vp(g["z"].data_ptr()), int(g["P"].shape[0]),
                                   ctypes.cast(ctypes.pointer(co), _vp)))
        garr = (_CFlashGroup * len(cg))(*cg)
        h = _vp()
        _check(lib().osr_flash_plan_create(garr, len(cg), ctypes.byref(h)), "osr_flash_plan_create")
        self._h = h

    def run(self, stream=None):
        import torch
        if stream is None:
            stream = torch.cuda.current_stream(self.groups[0]["P"].device)
        _check(lib().osr_flash_plan_run(self._h, _vp(stream.cuda_stream)), "osr_flash_plan_run")

    def run_persistent(self, stream=None):
        """The same step as one persistent cooperative kernel launch
        (osr_flash_plan_run_persistent)."""
        import torch
        if stream is None:
            stream = torch.cuda.current_stream(self.groups[0]["P"].device)
        _check(lib().osr_flash_plan_run_persistent(self._h, _vp(stream.cuda_stream)), "osr_flash_plan_run_persistent")

    def persistent_error(self, stream=None) -> int:
        import torch
        if stream is None:
            stream = torch.cuda.current_stream(self.groups[0]["P"].device)
        e = ctypes.c_int()
        _check(lib().osr_flash_plan_persistent_error(self._h, ctypes.byref(e), _vp(stream.cuda_stream)),
               "osr_flash_plan_persistent_error")
        return e.value

    def close(self):
        if getattr(self, "_h", None):
            lib().osr_flash_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def set_shape(ss_batch: int, tail_batch: int, ctas_per_sm: int, park_after: int):
    _check(lib().osr_flash_set_shape(int(ss_batch), int(tail_batch), int(ctas_per_sm), int(park_after)),
           "osr_flash_set_shape")


def set_pair_from(pass_index: int):
    """First pass of the batched flash in pair form (osr_flash_set_pair_from);
    12 = never."""
    _check(lib().osr_flash_set_pair_from(int(pass_index)), "osr_flash_set_pair_from")


def get_pair_from() -> int:
    return int(lib().osr_flash_get_pair_from())


class FlashTuning(ctypes.Structure):
    """osr_flash_tuning: the autotuner's winning launch shape."""
    _fields_ = [("ss_batch", ctypes.c_int), ("tail_batch", ctypes.c_int), ("ctas_per_sm", ctypes.c_int),
                ("park_after", ctypes.c_int), ("pair_from", ctypes.c_int), ("ms", ctypes.c_float),
                ("candidates", ctypes.c_int)]


def autotune(fluid: Fluid, P, T, z, out: dict | None = None, stream=None) -> dict:
    """Time every candidate launch shape of the batched flash on this batch
    (osr_flash_autotune); the winner becomes the current shape and the tuned
    shape of the batch's (component count, size bucket)."""
    import torch
    n = int(P.shape[0])
    if out is None:
        out = alloc_flash_outputs(fluid.nc, n, False, P.device)
    if stream is None:
        stream = torch.cuda.current_stream(P.device)
    co = _out_struct(out, lambda t: t.data_ptr())
    best = FlashTuning()
    with torch.cuda.device(P.device):
        _check(lib().osr_flash_autotune(fluid.cref, _vp(P.data_ptr()), _vp(T.data_ptr()), _vp(z.data_ptr()),
                                        ctypes.c_long(n), ctypes.byref(co), _vp(stream.cuda_stream),
                                        ctypes.byref(best)), "osr_flash_autotune")
    return {k: getattr(best, k) for k, _ in FlashTuning._fields_}


def use_tuned(on: bool):
    _check(lib().osr_flash_use_tuned(int(bool(on))), "osr_flash_use_tuned")


def tuning_save(path: str):
    _check(lib().osr_flash_tuning_save(path.encode()), "osr_flash_tuning_save")


def tuning_load(path: str):
    _check(lib().osr_flash_tuning_load(path.encode()), "osr_flash_tuning_load")


def set_group_from(pass_index: int):
    """First pass of the batched flash in group form (osr_flash_set_group_from);
    12 = never."""
    _check(lib().osr_flash_set_group_from(int(pass_index)), "osr_flash_set_group_from")


def get_group_from() -> int:
    return int(lib().osr_flash_get_group_from())


def get_shape():
    v = [ctypes.c_int() for _ in range(4)]
    _check(lib().osr_flash_get_shape(*[ctypes.byref(x) for x in v]), "osr_flash_get_shape")
    return tuple(x.value for x in v)


# ----------------------------------------------------------------------------- grid path

class _CModel(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int), ("nc", ctypes.c_int),
                ("eos", ctypes.c_int), ("restemp", ctypes.c_double), ("wat_ro", ctypes.c_double),
                ("wat_mu", ctypes.c_double), ("refp", ctypes.c_double), ("cpor", ctypes.c_double),
                ("dcpor", ctypes.c_double), ("lf", ctypes.c_double), ("re_f", ctypes.c_double),
                ("sigma", ctypes.c_double), ("has_cdif", ctypes.c_int), ("cdif", ctypes.c_double),
                ("di", _vp), ("dj", _vp), ("dk", _vp), ("por", _vp), ("fpor", _vp), ("perm", _vp), ("fperm", _vp),
                ("mw", _vp), ("tc", _vp), ("pc", _vp), ("vc", _vp), ("acf", _vp), ("parachor", _vp), ("zc", _vp),
                ("kij", _vp), ("nswt", ctypes.c_int), ("nsgt", ctypes.c_int), ("swt", _vp), ("sgt", _vp),
                ("nwells", ctypes.c_int), ("wells_i", _vp), ("wells_f", _vp), ("tor", _vp), ("dt", ctypes.c_double)]


def read_deck(path: str) -> dict:
    """The deck as the library's C++ reader parses it (osr_deck_open,
    osr_deck_model, osr_deck_initial_state, osr_deck_times): a dict of
    numpy copies keyed like ``deck.Deck``'s fields.  No device work."""
    L = lib()
    h = ctypes.c_void_p()
    rc = L.osr_deck_open(path.encode(), ctypes.byref(h))
    if rc:
        raise OsrError(f"osr_deck_open: {L.osr_deck_error().decode()}")
    try:
        m = _CModel()
        _check(L.osr_deck_model(h, ctypes.byref(m)), "osr_deck_model")
        n, nc = m.nx * m.ny * m.nz, m.nc

        def arr(ptr, count, ct=ctypes.c_double):
            if not ptr:
                return None
            return np.ctypeslib.as_array(ctypes.cast(ptr, ctypes.POINTER(ct)), shape=(count,)).copy()
        out = dict(nx=m.nx, ny=m.ny, nz=m.nz, nc=nc, eos=m.eos, restemp=m.restemp, wat_ro=m.wat_ro,
                   wat_mu=m.wat_mu, refp=m.refp, cpor=m.cpor, dcpor=m.dcpor, lf=m.lf, re_f=m.re_f, sigma=m.sigma,
                   cdif=m.cdif if m.has_cdif else None, di=arr(m.di, m.nx), dj=arr(m.dj, m.ny), dk=arr(m.dk, m.nz),
                   por=arr(m.por, n), fpor=arr(m.fpor, n), perm=arr(m.perm, 3 * n).reshape(3, n),
                   fperm=arr(m.fperm, 3 * n).reshape(3, n), tor=arr(m.tor, n), dt=m.dt,
                   swt=arr(m.swt, 4 * m.nswt).reshape(-1, 4), sgt=arr(m.sgt, 4 * m.nsgt).reshape(-1, 4),
                   kij=arr(m.kij, nc * nc).reshape(nc, nc))
        for k in ("mw", "tc", "pc", "vc", "acf", "parachor", "zc"):
            out[k] = arr(getattr(m, k), nc)
        nw = m.nwells
        out["wells_i"] = (arr(m.wells_i, 5 * nw, ctypes.c_int).reshape(nw, 5) if nw else np.zeros((0, 5), np.int32))
        out["wells_f"] = arr(m.wells_f, (nc + 6) * nw).reshape(nw, nc + 6) if nw else np.zeros((0, nc + 6))
        for med, (kp, ks, kz) in enumerate((("p0", "sw0", "z0"), ("fp0", "fsw0", "fz0"))):
            p0, sw0, z0 = (ctypes.c_void_p() for _ in range(3))
            _check(L.osr_deck_initial_state(h, med, ctypes.byref(p0), ctypes.byref(sw0), ctypes.byref(z0)),
                   "osr_deck_initial_state")
            out[kp], out[ks] = arr(p0.value, n), arr(sw0.value, n)
            out[kz] = arr(z0.value, nc * n).reshape(nc, n)
        dt, tt, dtmax, ic = ctypes.c_double(), ctypes.c_double(), ctypes.c_double(), ctypes.c_int()
        _check(L.osr_deck_times(h, ctypes.byref(dt), ctypes.byref(tt), ctypes.byref(dtmax), ctypes.byref(ic)),
               "osr_deck_times")
        out.update(total_time=tt.value, dtmax=dtmax.value, initcond=ic.value)
        return out
    finally:
        L.osr_deck_close(h)


class Grid:
    """A dual-porosity model on the device, built from a parsed deck
    (``osiris_b200.deck.parse_deck``)."""

    FIELD_PLANES = {"P": 3, "sat": 3, "x": "nc", "y": "nc", "z": "nc", "label": 1, "rho": 2, "pc": 2, "mu": 2,
                    "gam": 2, "kr": 3, "dkr": 5, "dE": "2nc1", "pre": "nc1", "diff": "2nc", "ift": 1, "trans": 36,
                    "transS": 9, "wtran": 3, "dwtran": 3, "por": 1, "perm": 3, "iftran": 3}

    def __init__(self, d):
        self.deck = d
        self.nc = d.nc
        self.cells = d.cells
        keep = dict(di=d.di, dj=d.dj, dk=d.dk, por=d.por, fpor=d.fpor, perm=d.perm, fperm=d.fperm, mw=d.mw, tc=d.tc,
                    pc=d.pc, vc=d.vc, acf=d.acf, parachor=d.parachor, zc=d.zc, kij=d.kij, swt=d.swt, sgt=d.sgt,
                    wells_f=d.wells_f, tor=d.tor)
        self._keep = {k: np.ascontiguousarray(v, dtype=np.float64) for k, v in keep.items()}
        self._keep["wells_i"] = np.ascontiguousarray(d.wells_i, dtype=np.int32)
        k = self._keep
        m = _CModel(d.nx, d.ny, d.nz, d.nc, d.eos, d.restemp, d.wat_ro, d.wat_mu, d.refp, d.cpor, d.dcpor, d.lf,
                    d.re_f, d.sigma, 0 if d.cdif is None else 1, 0.0 if d.cdif is None else d.cdif,
                    *[k[n].ctypes.data for n in ("di", "dj", "dk", "por", "fpor", "perm", "fperm", "mw", "tc", "pc",
                                                  "vc", "acf", "parachor", "zc", "kij")],
                    d.swt.shape[0], d.sgt.shape[0], k["swt"].ctypes.data, k["sgt"].ctypes.data,
                    d.wells_i.shape[0], k["wells_i"].ctypes.data, k["wells_f"].ctypes.data, k["tor"].ctypes.data,
                    d.dt)
        self._model = m
        h = ctypes.c_void_p()
        L = lib()
        _check(L.osr_grid_create(ctypes.byref(m), ctypes.byref(h)), "osr_grid_create")
        self._h = h

    @classmethod
    def create(cls, path: str, stream=None) -> "Grid":
        """osr_create: the deck read by the library's C++ reader and the
        start-up state formed on the current device in one C call."""
        from . import deck as _deck
        h = ctypes.c_void_p()
        L = lib()
        rc = L.osr_create(path.encode(), None if stream is None else _vp(stream), ctypes.byref(h))
        if rc == 7:
            raise OsrError(f"osr_create: {L.osr_deck_error().decode()}")
        _check(rc, "osr_create")
        g = cls.__new__(cls)
        g._h = h
        g.deck = _deck.parse_deck(path)
        g.nc, g.cells = g.deck.nc, g.deck.cells
        return g

    def close(self):
        if self._h:
            lib().osr_grid_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_state(self, medium: int, P_oil, sat, x, y, z, label, rho=None):
        arrs = [np.ascontiguousarray(a, np.float64) for a in (P_oil, sat, x, y, z)]
        lab = np.ascontiguousarray(label, np.int8)
        r = None if rho is None else np.ascontiguousarray(rho, np.float64)
        _check(lib().osr_grid_set_state(self._h, int(medium), *[a.ctypes.data for a in arrs], lab.ctypes.data,
                                        None if r is None else r.ctypes.data), "osr_grid_set_state")

    def initialize(self, device, stream=None):
        """The deck's initial state on the device, formed as the reference's
        start-up forms it: the INITCOND pressures, water saturations and feed
        compositions (compsim/Data_Input.cpp:1040-1181), a flash of every
        cell-medium (AllFlash, compsim/Init_Calcs.cpp:949-962; label, phase
        compositions, oil and gas saturations from the liquid volume fraction
        and densities from the Z factors as SuccFalsh sets them, :715-737),
        then UpdateDependencies(true) (compsim/PetscAUX.cpp:500-545): phase
        control, PCoeff, the row layout and the property sweeps."""
        import torch
        d = self.deck
        fl = Fluid(d.tc, d.pc, d.acf, d.kij, d.eos)
        for med, (p0, sw0, z0) in enumerate(((d.p0, d.sw0, d.z0), (d.fp0, d.fsw0, d.fz0))):
            P = torch.tensor(np.ascontiguousarray(p0, np.float64), device=device)
            T = torch.full_like(P, d.restemp)
            z = torch.tensor(np.ascontiguousarray(z0, np.float64), device=device)
            o = flash(fl, P, T, z, derivs=False)
            L, Zl, Zg = o["L"], o["Zl"], o["Zg"]
            sw = torch.tensor(np.ascontiguousarray(sw0, np.float64), device=device)
            liq = Zl * L / (Zl * L + Zg * (1 - L))
            sat = torch.stack([sw, liq * (1 - sw), (1 - liq) * (1 - sw)])
            rho = torch.stack([P / (Zl * R_GAS * T), P / (Zg * R_GAS * T)])
            self.set_state(med, p0, sat.cpu().numpy(), o["x"].cpu().numpy(), o["y"].cpu().numpy(), z0,
                           o["label"].cpu().numpy(), rho.cpu().numpy())
        self.phase_ctrl(stream)
        self.refresh_layout(stream)
        self.update_dependencies(stream)

    def set_pressures(self, medium: int, P):
        """All three phase pressures of one continuum, [3][cells]."""
        a = np.ascontiguousarray(P, np.float64)
        _check(lib().osr_grid_set_pressures(self._h, int(medium), a.ctypes.data), "osr_grid_set_pressures")

    def update_dependencies(self, stream=None):
        _check(lib().osr_grid_update_dependencies(self._h, None if stream is None else _vp(stream)),
               "osr_grid_update_dependencies")

    # -- residual path -------------------------------------------------------
    def refresh_layout(self, stream=None):
        """Row offsets of the current phase labels and PCoeff (PJac, CalcPCoeff)."""
        _check(lib().osr_grid_refresh_layout(self._h, None if stream is None else _vp(stream)),
               "osr_grid_refresh_layout")
        return self.layout()

    def layout(self):
        rows = ctypes.c_long()
        pc = ctypes.c_double()
        _check(lib().osr_grid_layout(self._h, ctypes.byref(rows), ctypes.byref(pc)), "osr_grid_layout")
        return rows.value, pc.value

    def row_offsets(self) -> np.ndarray:
        out = np.zeros(2 * self.cells + 1, np.int64)
        _check(lib().osr_grid_row_offsets(self._h, out.ctypes.data), "osr_grid_row_offsets")
        return out

    def set_controls(self, dt: float, pcoeff: float = 0.0):
        _check(lib().osr_grid_set_controls(self._h, ctypes.c_double(dt), ctypes.c_double(pcoeff)),
               "osr_grid_set_controls")

    def set_well_condition(self, well: int, latched: bool):
        _check(lib().osr_grid_set_well_condition(self._h, int(well), int(bool(latched))), "osr_grid_set_well_condition")

    def well_radius(self, well: int) -> float:
        v = ctypes.c_double()
        _check(lib().osr_grid_well_radius(self._h, int(well), ctypes.byref(v)), "osr_grid_well_radius")
        return v.value

    def init_guess(self, d_x, stream=None):
        """Write the unknown vector of the current state into device memory d_x (a CUDA tensor)."""
        _check(lib().osr_grid_init_guess(self._h, _vp(d_x.data_ptr()), None if stream is None else _vp(stream)),
               "osr_grid_init_guess")

    def well_sums(self, layer0: int, layer1: int, d_sums, stream=None):
        """Layer sums of the wells' rate split over layers [layer0, layer1)
        into d_sums [nwells, 2, 5] (osr_grid_well_sums)."""
        _check(lib().osr_grid_well_sums(self._h, int(layer0), int(layer1), _vp(d_sums.data_ptr()),
                                        None if stream is None else _vp(stream)), "osr_grid_well_sums")

    def set_well_sums(self, d_sums):
        """Take the wells' layer sums from d_sums (kept alive by the caller);
        None: the grid's own layers."""
        self._well_sums = d_sums
        _check(lib().osr_grid_set_well_sums(self._h, None if d_sums is None else _vp(d_sums.data_ptr())),
               "osr_grid_set_well_sums")

    def update_all(self, d_x, stream=None):
        _check(lib().osr_grid_update_all(self._h, _vp(d_x.data_ptr()), None if stream is None else _vp(stream)),
               "osr_grid_update_all")

    def residual(self, d_f, d_scale=None, sim_time: float = 0.0, stream=None):
        _check(lib().osr_grid_residual(self._h, _vp(d_f.data_ptr()),
                                       None if d_scale is None else _vp(d_scale.data_ptr()),
                                       ctypes.c_double(sim_time), None if stream is None else _vp(stream)),
               "osr_grid_residual")

    def residual_logk_vjp(self, d_lambda, d_gk, sim_time: float = 0.0, stream=None):
        """sum_r lambda_r dF_r/d ln k_c for every matrix cell c at the current
        state (osr_grid_residual_logk_vjp); d_lambda [rows], d_gk [cells]."""
        _check(lib().osr_grid_residual_logk_vjp(self._h, _vp(d_lambda.data_ptr()), _vp(d_gk.data_ptr()),
                                                ctypes.c_double(sim_time), None if stream is None else _vp(stream)),
               "osr_grid_residual_logk_vjp")

    def status(self):
        """(osr_cell_status code, first bad block or -1) of the current state
        (osr_grid_status)."""
        code, first = ctypes.c_int(), ctypes.c_long()
        _check(lib().osr_grid_status(self._h, ctypes.byref(code), ctypes.byref(first)), "osr_grid_status")
        return code.value, first.value

    def form_function(self, d_x, d_f, sim_time: float = 0.0, stream=None):
        _check(lib().osr_grid_form_function(self._h, _vp(d_x.data_ptr()), _vp(d_f.data_ptr()),
                                            ctypes.c_double(sim_time), None if stream is None else _vp(stream)),
               "osr_grid_form_function")

    # -- phase appearance ----------------------------------------------------
    def saturation_pressure(self, medium: int, device, stream=None):
        """(pressure [cells], incipient composition [nc, cells]) of every
        one-phase cell of one continuum (0 for two-phase cells, -1 where no
        saturation pressure is found), device tensors."""
        import torch
        p = torch.empty(self.cells, dtype=torch.float64, device=device)
        xm = torch.empty((self.nc, self.cells), dtype=torch.float64, device=device)
        _check(lib().osr_grid_saturation_pressure(self._h, int(medium), _vp(p.data_ptr()), _vp(xm.data_ptr()),
                                                  None if stream is None else _vp(stream)),
               "osr_grid_saturation_pressure")
        return p, xm

    SATP_KINDS = {"bubble_nr": 0, "dew_nr": 1, "lower_dew": 2}

    def saturation_pressure_nr(self, medium: int, kind: str, device, stream=None):
        """Bubl_NR ("bubble_nr", oil-only cells), Dew_NR ("dew_nr") or
        LowerDew_Succ ("lower_dew", gas-only cells) on one continuum:
        (pressure [cells], incipient composition [nc, cells], status [cells],
        steps [cells]) device tensors; 0 for cells of the other labels."""
        import torch
        p = torch.empty(self.cells, dtype=torch.float64, device=device)
        xm = torch.empty((self.nc, self.cells), dtype=torch.float64, device=device)
        st = torch.empty(self.cells, dtype=torch.int32, device=device)
        it = torch.empty(self.cells, dtype=torch.int32, device=device)
        _check(lib().osr_grid_saturation_pressure_nr(self._h, int(medium), self.SATP_KINDS[kind], _vp(p.data_ptr()),
                                                     _vp(xm.data_ptr()), _vp(st.data_ptr()), _vp(it.data_ptr()),
                                                     None if stream is None else _vp(stream)),
               "osr_grid_saturation_pressure_nr")
        return p, xm, st, it

    def crit_test(self, medium: int, device, stream=None):
        """critTest on every one-phase cell of one continuum (relabels the
        cells found in the other phase): (final L [cells] device tensor,
        number of relabelled cells)."""
        import torch
        L = torch.empty(self.cells, dtype=torch.float64, device=device)
        changed = torch.zeros(1, dtype=torch.int32, device=device)
        _check(lib().osr_grid_crit_test(self._h, int(medium), _vp(L.data_ptr()), _vp(changed.data_ptr()),
                                        None if stream is None else _vp(stream)), "osr_grid_crit_test")
        return L, int(changed.item())

    def phase_ctrl(self, stream=None):
        _check(lib().osr_grid_phase_ctrl(self._h, None if stream is None else _vp(stream)), "osr_grid_phase_ctrl")

    def write_listing(self, path: str, sim_time: float, first_call: bool):
        """Append the reference's state listing (PrintAll) through the C ABI."""
        _check(lib().osr_grid_write_listing(self._h, path.encode(), ctypes.c_double(sim_time), int(bool(first_call))),
               "osr_grid_write_listing")

    def update_all_full(self, d_x, stream=None):
        _check(lib().osr_grid_update_all_full(self._h, _vp(d_x.data_ptr()), None if stream is None else _vp(stream)),
               "osr_grid_update_all_full")

    # -- Jacobian path -------------------------------------------------------
    def jacobian_shape(self):
        """(block size, values per block row, shifted entries per block row)."""
        bs, ent, ovf = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        _check(lib().osr_grid_jacobian_shape(self._h, ctypes.byref(bs), ctypes.byref(ent), ctypes.byref(ovf)),
               "osr_grid_jacobian_shape")
        return bs.value, ent.value, ovf.value

    def block_columns(self) -> np.ndarray:
        out = np.zeros((2 * self.cells, 8), np.int64)
        _check(lib().osr_grid_block_columns(self._h, out.ctypes.data), "osr_grid_block_columns")
        return out

    def alloc_jacobian(self, device):
        """Device values of osr_grid_jacobian: float64 [chunks, entries, 32]
        (block row b at [b // 32, :, b % 32])."""
        import torch
        _, ent, _ = self.jacobian_shape()
        return torch.empty(((2 * self.cells + 31) // 32, ent, 32), dtype=torch.float64, device=device)

    def jacobian_pattern(self, device, stream=None):
        """Reference (row, column) of every value, int64 device tensors in the
        values' layout, -1 where the reference's matrix holds no entry."""
        import torch
        _, ent, _ = self.jacobian_shape()
        rows = torch.empty(((2 * self.cells + 31) // 32, ent, 32), dtype=torch.int64, device=device)
        cols = torch.empty_like(rows)
        _check(lib().osr_grid_jacobian_pattern(self._h, _vp(rows.data_ptr()), _vp(cols.data_ptr()),
                                               None if stream is None else _vp(stream)), "osr_grid_jacobian_pattern")
        return rows, cols

    def jacobian(self, vals, sim_time: float = 0.0, stream=None):
        return lib().osr_grid_jacobian(self._h, ctypes.c_double(sim_time), _vp(vals.data_ptr()),
                                       None if stream is None else _vp(stream))

    def form_jacobian(self, d_x, vals, sim_time: float = 0.0, stream=None):
        return lib().osr_grid_form_jacobian(self._h, _vp(d_x.data_ptr()), ctypes.c_double(sim_time),
                                            _vp(vals.data_ptr()), None if stream is None else _vp(stream))

    def jacobian_coo(self, vals):
        """(rows, cols, vals) host arrays in the reference's global numbering
        (the COO triplets a PETSc adapter hands to MatSetValuesCOO)."""
        import torch
        torch.cuda.synchronize(vals.device)
        rows, cols = self.jacobian_pattern(vals.device)
        torch.cuda.synchronize(vals.device)
        r, c, v = rows.cpu().numpy().ravel(), cols.cpu().numpy().ravel(), vals.cpu().numpy().ravel()
        keep = r >= 0
        return r[keep], c[keep], v[keep]

    # -- linear solve ----------------------------------------------------------
    def jacobian_apply(self, vals, d_x, d_y, stream=None):
        """d_y = J d_x on the compact Jacobian values (MatMult)."""
        _check(lib().osr_grid_jacobian_apply(self._h, _vp(vals.data_ptr()), _vp(d_x.data_ptr()),
                                             _vp(d_y.data_ptr()), None if stream is None else _vp(stream)),
               "osr_grid_jacobian_apply")

    def jacobian_apply_transpose(self, vals, d_lambda, d_y, stream=None):
        """d_y = J^T d_lambda (MatMultTranspose; the residual's product with
        an adjoint vector in the unknowns)."""
        _check(lib().osr_grid_jacobian_apply_transpose(self._h, _vp(vals.data_ptr()), _vp(d_lambda.data_ptr()),
                                                       _vp(d_y.data_ptr()), None if stream is None else _vp(stream)),
               "osr_grid_jacobian_apply_transpose")

    def ksp_solve(self, vals, d_rhs, d_sol, stream=None, **opts) -> dict:
        """Solve J d_sol = d_rhs (KSPBCGS + PCVPBJACOBI, zero initial guess);
        keyword overrides of the reference's tolerances: rtol, atol, dtol,
        max_it, check_every.  Returns reason, its, rnorm0, rnorm."""
        o = ksp_opts(**opts)
        info = KspInfo()
        _check(lib().osr_grid_ksp_solve(self._h, _vp(vals.data_ptr()), _vp(d_rhs.data_ptr()),
                                        _vp(d_sol.data_ptr()), ctypes.byref(o), ctypes.byref(info),
                                        None if stream is None else _vp(stream)), "osr_grid_ksp_solve")
        return {"reason": info.reason, "its": info.its, "rnorm0": info.rnorm0, "rnorm": info.rnorm}

    def ksp_solve_transpose(self, vals, d_rhs, d_sol, stream=None, **opts) -> dict:
        """Solve J^T d_sol = d_rhs (osr_grid_ksp_solve_transpose; the adjoint
        system of the Newton step)."""
        o = ksp_opts(**opts)
        info = KspInfo()
        _check(lib().osr_grid_ksp_solve_transpose(self._h, _vp(vals.data_ptr()), _vp(d_rhs.data_ptr()),
                                                  _vp(d_sol.data_ptr()), ctypes.byref(o), ctypes.byref(info),
                                                  None if stream is None else _vp(stream)),
               "osr_grid_ksp_solve_transpose")
        return {"reason": info.reason, "its": info.its, "rnorm0": info.rnorm0, "rnorm": info.rnorm}

    def get(self, name: str) -> np.ndarray:
        L = lib()
        n = L.osr_grid_field_size(self._h, name.encode())
        if n < 0:
            raise KeyError(name)
        out = np.zeros(n)
        _check(L.osr_grid_get(self._h, name.encode(), out.ctypes.data), "osr_grid_get")
        key = name.split(".", 1)[1]
        planes = self.FIELD_PLANES[key]
        nc = self.nc
        shape = {"nc": (nc,), "2nc1": (nc + 1, 2), "nc1": (nc + 1,), "2nc": (nc, 2)}.get(planes)
        if shape is None:
            shape = () if planes == 1 else ((12, 3) if key == "trans" else (3, 3) if key == "transS" else (planes,))
        return out.reshape(shape + (self.cells,))


class Sim:
    """A run of the reference's main loop on the device (osr_sim_*): one
    ``step()`` is SolveNonLinear + TimeStepCtrl.  Starts from the grid's
    current state; ``markers``/``dt`` as ``deck.time_markers`` gives them."""

    def __init__(self, grid: "Grid", markers, dt: float, max_dt: float):
        self.grid = grid   # the run uses the grid's device state
        m = np.ascontiguousarray(markers, np.float64)
        h = ctypes.c_void_p()
        _check(lib().osr_sim_create(grid._h, m.ctypes.data, len(m), ctypes.c_double(dt), ctypes.c_double(max_dt),
                                    ctypes.byref(h)), "osr_sim_create")
        self._h = h

    @classmethod
    def from_deck(cls, grid: "Grid"):
        from .deck import time_markers
        m, dt = time_markers(grid.deck)
        return cls(grid, m, dt, grid.deck.dtmax)

    def step(self, stream=None, **ksp) -> dict:
        o = ksp_opts(**ksp)
        info = StepInfo()
        _check(lib().osr_sim_step(self._h, ctypes.byref(o), ctypes.byref(info),
                                  None if stream is None else _vp(stream)), "osr_sim_step")
        return {k: getattr(info, k) for k, _ in StepInfo._fields_}

    def write_restart(self, path: str, smethq: float = 0.0):
        """The reference's restart file through the C ABI (osr_sim_write_restart)."""
        _check(lib().osr_sim_write_restart(self._h, path.encode(), ctypes.c_double(smethq)), "osr_sim_write_restart")

    def read_restart(self, path: str) -> float:
        """Load a restart file into the run's grid and clock (osr_sim_read_restart);
        returns SMethQ."""
        sm = ctypes.c_double()
        _check(lib().osr_sim_read_restart(self._h, path.encode(), ctypes.byref(sm)), "osr_sim_read_restart")
        return sm.value

    def set_graph(self, on: bool):
        """Run each pass's linearisation and solve as one CUDA graph (the
        default) or as direct launches (osr_sim_set_graph)."""
        _check(lib().osr_sim_set_graph(self._h, int(bool(on))), "osr_sim_set_graph")

    def graph_launches(self) -> int:
        n = ctypes.c_long()
        _check(lib().osr_sim_graph_launches(self._h, ctypes.byref(n)), "osr_sim_graph_launches")
        return n.value

    def graph_form(self) -> int:
        """0 no step graph, 1 linearisation and solve, 2 the whole pass."""
        f = ctypes.c_int()
        _check(lib().osr_sim_graph_form(self._h, ctypes.byref(f)), "osr_sim_graph_form")
        return f.value

    def marker_index(self) -> int:
        k = ctypes.c_int()
        _check(lib().osr_sim_marker_index(self._h, ctypes.byref(k)), "osr_sim_marker_index")
        return k.value

    def restart(self, sim_time: float, dt: float, tsm_ctrl: int):
        _check(lib().osr_sim_restart(self._h, ctypes.c_double(sim_time), ctypes.c_double(dt), int(tsm_ctrl)),
               "osr_sim_restart")

    def time(self):
        t, dt = ctypes.c_double(), ctypes.c_double()
        _check(lib().osr_sim_time(self._h, ctypes.byref(t), ctypes.byref(dt)), "osr_sim_time")
        return t.value, dt.value

    def close(self):
        if self._h:
            lib().osr_sim_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

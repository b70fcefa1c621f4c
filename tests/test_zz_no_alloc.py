"""GPU test of osr_flash_batch_noalloc, the flash entry point for callers that
cannot allocate device memory (their device memory belongs to another runtime
or allocator, or a no-allocation policy holds in their time-step loop).

It is called through the C ABI twice in a row on the same inputs, with fresh
outputs each time, and each result is checked against osr_flash_batch (the
allocating entry point) under the same bar as the other flash tests
(oracle.flash_parity; derivatives within 1e-10 of each block's largest
entry).  The second call also checks that the shared static scratch left by
the first call does not leak into the next one.  A batch beyond the static
scratch's size limit must be refused with OSR_ERR_SIZE.  This file is named
to be collected last."""
import ctypes

import numpy as np
import pytest

import oracle
import osiris_b200 as osr
from osiris_b200 import workloads

pytestmark = pytest.mark.gpu

OSR_ERR_SIZE = 5


def _inputs(n, seed):
    import torch
    tc, pc, acf, kij, eos = workloads.flash_fluid_srk6()
    fl = osr.Fluid(tc, pc, acf, kij, eos)
    P, T, z = workloads.flash_cells(n, 6, seed=seed)
    dev = torch.device("cuda:0")
    return fl, torch.from_numpy(P).to(dev), torch.from_numpy(T).to(dev), torch.from_numpy(z).to(dev)


def _host(out):
    return {k: v.cpu().numpy() for k, v in out.items()}


def _check_same(got, ref):
    r = oracle.flash_parity(got, ref)
    assert r["ok"], (r["frac_tight"], r["max_scaled_err"], r["margin"][:10])
    for key in ("dlnphi_dx", "dlnphi_dP"):
        a, b = got[key], ref[key]
        axes = tuple(range(1, a.ndim - 1))
        scale = np.abs(b).max(axis=axes, keepdims=True)
        scale = np.where(scale > 0, scale, 1.0)
        ok = np.isfinite(b).all(axis=tuple(range(a.ndim - 1)))
        err = (np.abs(a - b) / scale)[..., ok]
        assert err.size == 0 or err.max() <= 1e-10, (key, err.max())


def test_noalloc_matches_allocating_entry_point_twice(cuda_device):
    import torch
    fl, P, T, z = _inputs(200_000, seed=41)
    ref = _host(osr.flash(fl, P, T, z, derivs=True, form="batched"))
    torch.cuda.synchronize()
    for _ in range(2):
        out = osr.alloc_flash_outputs(6, int(P.shape[0]), True, P.device)
        torch.cuda.synchronize()
        taken = osr.lib().osr_pool_alloc_count()
        got = osr.flash(fl, P, T, z, derivs=True, form="noalloc", out=out)
        torch.cuda.synchronize()
        # the property in the entry point's name: the call took no block from
        # the library's device pools
        assert osr.lib().osr_pool_alloc_count() == taken
        _check_same(_host(got), ref)


def test_noalloc_second_call_on_different_cells(cuda_device):
    """A smaller, different batch right after a larger one: stale parked
    cells from the previous call must not be picked up."""
    import torch
    for n, seed in ((150_000, 43), (7_000, 44)):
        fl, P, T, z = _inputs(n, seed)
        ref = _host(osr.flash(fl, P, T, z, derivs=True, form="batched"))
        got = _host(osr.flash(fl, P, T, z, derivs=True, form="noalloc"))
        torch.cuda.synchronize()
        _check_same(got, ref)


def test_noalloc_rejects_batches_beyond_the_static_scratch(cuda_device):
    import torch
    fl, P, T, z = _inputs(16, seed=45)
    out = osr.alloc_flash_outputs(6, 16, True, P.device)
    co = osr._out_struct(out, lambda t: t.data_ptr())
    n_too_big = (64 << 20) // (48 + 16 * 6) + 1  # beyond n * (48 + 16 nc) + 4096 <= 64 MiB
    rc = osr.lib().osr_flash_batch_noalloc(fl.cref, ctypes.c_void_p(P.data_ptr()), ctypes.c_void_p(T.data_ptr()),
                                           ctypes.c_void_p(z.data_ptr()), ctypes.c_long(n_too_big),
                                           ctypes.byref(co), None)
    assert rc == OSR_ERR_SIZE
    torch.cuda.synchronize()

"""mlegs_idel2ln_static, the IDEL2LN entry point that allocates nothing.

Its elimination scratch is the library's fixed __device__ array instead of the
context's allocation.  Checked through the C ABI against mlegs_idel2ln on the
same inputs, on two calls in a row (the second call finds the first call's
contents in the shared array), within the banded-solve tolerance of the
parity tests; and an oversized grid must be rejected before any GPU work.
This file is collected last and also passes when run alone.
"""

import ctypes

import numpy as np
import pytest

from conftest import oracle_grid, random_fff, rel, small_cfg

pytestmark = pytest.mark.gpu

# The static path eliminates on the fly (solve_kernel); IDEL2LN substitutes
# with stored factors (solve_factored_kernel).  Same multipliers and order, but
# the compiler contracts different products into FMAs, so the two agree to a
# few ulps (2e-16 relative measured), not bit for bit.
SOLVE_TOL = 1e-13
MLEGS_ERR_ARG = 101


def _free_device_bytes():
    """cudaMemGetInfo's free bytes on device 0 (the device the tests use)."""
    rt = ctypes.CDLL("libcudart.so")
    free, total = ctypes.c_size_t(0), ctypes.c_size_t(0)
    assert rt.cudaSetDevice(0) == 0
    assert rt.cudaMemGetInfo(ctypes.byref(free), ctypes.byref(total)) == 0
    return free.value


def _solve_both(M, ctx, g, seed, pad):
    B = random_fff(g, seed, pad=pad)
    B.LN = 0.0
    b = ctx.field(M.FFF)
    b.upload(B.E, B.LN, M.FFF)
    a_ref = ctx.field(M.FFF)
    a_new = ctx.field(M.FFF)
    ctx.IDEL2LN(b, a_ref, pad)
    rc = ctx.lib.mlegs_idel2ln_static(ctx.c, b.h, a_new.h, pad)
    assert rc == 0, ctx.lib.mlegs_last_error(ctx.c)
    E_ref, ln_ref = a_ref.download()
    E_new, ln_new = a_new.download()
    assert a_new.space == M.FFF
    return E_ref, ln_ref, E_new, ln_new


@pytest.mark.parametrize("dims", [(32, 16, 16), (64, 32, 32)], ids=["32x16x16", "64x32x32"])
def test_static_scratch_matches_idel2ln(lib_built, dims):
    import mlegs_b200 as M
    cfg = small_cfg(*dims)
    g = oracle_grid(cfg)
    ctx = M.Context(cfg)
    try:
        for seed, pad in ((11, 0), (12, 3)):
            E_ref, ln_ref, E_new, ln_new = _solve_both(M, ctx, g, seed, pad)
            assert np.isfinite(E_new).all()
            assert rel(E_new, E_ref) < SOLVE_TOL
            assert abs(ln_new - ln_ref) <= SOLVE_TOL * max(1.0, abs(ln_ref))
    finally:
        ctx.close()


def test_static_scratch_allocates_nothing(lib_built):
    """After a first call (which looks the array up), further calls leave the
    device's free memory unchanged: no cudaMalloc behind the entry point."""
    import mlegs_b200 as M
    cfg = small_cfg(64, 32, 32)
    g = oracle_grid(cfg)
    ctx = M.Context(cfg)
    try:
        B = random_fff(g, 13)
        b = ctx.field(M.FFF)
        b.upload(B.E, 0.0, M.FFF)
        a = ctx.field(M.FFF)
        for pad in (0, 3):
            assert ctx.lib.mlegs_idel2ln_static(ctx.c, b.h, a.h, pad) == 0
        ctx.sync()
        before = _free_device_bytes()
        for pad in (0, 3, 0):
            assert ctx.lib.mlegs_idel2ln_static(ctx.c, b.h, a.h, pad) == 0
        ctx.sync()
        assert _free_device_bytes() == before
    finally:
        ctx.close()


def test_static_scratch_rejects_oversized_grid(lib_built):
    import mlegs_b200 as M
    # NRCHOPDIM * 4 * NTCHOPDIM * NXCHOPDIM = 206 * 4 * 85 * 169 doubles > 8,388,608
    cfg = small_cfg(256, 128, 256, nrchop=200, ntchop=85, nxchop=85)
    ctx = M.Context(cfg)
    try:
        b = ctx.field(M.FFF)
        a = ctx.field(M.FFF)
        rc = ctx.lib.mlegs_idel2ln_static(ctx.c, b.h, a.h, 0)
        assert rc == MLEGS_ERR_ARG
        msg = ctx.lib.mlegs_last_error(ctx.c)
        msg = msg.decode() if isinstance(msg, bytes) else str(msg)
        assert "static scratch" in msg and "bytes" in msg
    finally:
        ctx.close()

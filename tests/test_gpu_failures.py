"""Failure detection on the GPU without a GPU fault.

* A bounded wait inside the split-BF16 tensor-core GEMM is made to run out by
  giving the context a wait limit of a few SM cycles (mlegs_set_wait_limit):
  the kernel drains what it has in flight, frees its tensor memory and
  returns; the next mlegs_sync reports MLEGS_ERR_TIMEOUT once, and the same
  context then computes correct results again with the default limit.
* ANYNAN (mod_scalar3.f90:998-1045): a NaN uploaded from the host into a
  solver state field is reported as MLEGS_ERR_NONFINITE by mlegs_check_finite;
  an Inf likewise; clean fields pass.
"""

import numpy as np
import pytest

from conftest import oracle_grid, random_fff, rel, small_cfg

pytestmark = pytest.mark.gpu

MLEGS_ERR_NONFINITE = 103
MLEGS_ERR_TIMEOUT = 105


def test_split_wait_runs_out_and_context_recovers(lib_built):
    import mlegs_b200 as M
    from oracle import transforms as T
    cfg = small_cfg(64, 32, 32, adams=False)
    g = oracle_grid(cfg)
    ctx = M.Context(cfg, precision=M.PREC_SPLIT, split_slices=6)
    try:
        A = random_fff(g, 31)
        f = ctx.field(M.FFF)
        f.upload(A.E, 0.0, M.FFF)
        assert ctx.lib.mlegs_set_wait_limit(ctx.c, 2) == 0
        ctx.RTRAN(f, 1)
        with pytest.raises(M.MlegsError) as ei:
            ctx.sync()
        assert ei.value.code == MLEGS_ERR_TIMEOUT
        assert "timed out" in str(ei.value)
        ctx.sync()  # reported once
        # default limit again: the same context gives the oracle's result
        assert ctx.lib.mlegs_set_wait_limit(ctx.c, 0) == 0
        f.upload(A.E, 0.0, M.FFF)
        ctx.RTRAN(f, 1)
        ctx.sync()
        B = A.copy()
        T.rtran(g, B, 1)
        assert rel(f.download()[0], B.E) < 1e-12
        assert ctx.lib.mlegs_set_wait_limit(ctx.c, -1) == 101
    finally:
        ctx.close()


@pytest.mark.parametrize("bad", [np.nan, np.inf], ids=["nan", "inf"])
def test_check_finite_flags_uploaded_nonfinite(lib_built, bad):
    import mlegs_b200 as M
    cfg = small_cfg(32, 16, 16, adams=False)
    ctx = M.Context(cfg)
    try:
        fp, fc, fb = M.initial_state(ctx)
        ctx.initialize(fp, fc, fb)
        ctx.check_finite()
        E, ln = fb.download()
        E[3, 1, 2] = complex(bad, 0.0)
        fb.upload(E, ln, M.FFF)
        with pytest.raises(M.MlegsError) as ei:
            ctx.check_finite()
        assert ei.value.code == MLEGS_ERR_NONFINITE
        E[3, 1, 2] = 0.0
        fb.upload(E, ln, M.FFF)
        ctx.check_finite()
    finally:
        ctx.close()

"""The transform-only configuration: FFF -> PPP -> FFF at 256^3 per precision form.

NR = NTH = NX = 256 with 2/3 chops (NRCHOP 170, NTCHOP 170, NXCHOP 85); chi,
psi and b coefficient sets with amplitude exp(-(n + |m| + |k|) / 10)
(mlegs_b200.inputs.roundtrip_coefficients).  TOFP (RTRAN(+1), VERFFT(+1),
HORFFT(+1), mod_fft.f90:1371-1398) and TOFF (1342-1369) through the C ABI
against the FP64 oracle, for the FP64 tensor-path GEMMs and the split-BF16
forms with S = 4, 5, 6 slices.  The bound per form (max|d| / max|ref|) is the
form's precision: 2^-8S of each row's largest weight per GEMM, with margin.
"""

import numpy as np
import pytest

from conftest import rel

pytestmark = pytest.mark.gpu

FORMS = {"fp64": (0, 1e-12), "split4": (4, 1e-7), "split5": (5, 1e-9), "split6": (6, 1e-11)}


@pytest.fixture(scope="module")
def rt(lib_built):
    from mlegs_b200.inputs import CONFIGS, roundtrip_coefficients
    from oracle import transforms as T
    from oracle.grid import FFF, Grid
    cfg = CONFIGS["roundtrip_256"]
    g = Grid(cfg.nr, cfg.nth, cfg.nx, cfg.nrchop, cfg.ntchop, cfg.nxchop, cfg.ell, cfg.zlen)
    cases = []
    for i in range(3):
        c = roundtrip_coefficients(cfg, i)
        A = g.alloc(FFF)
        A.E = c.copy()
        T.tofp(g, A)
        ppp = A.E.copy()
        T.toff(g, A)
        cases.append((c, ppp, A.E.copy()))
    return cfg, cases


@pytest.mark.parametrize("form", list(FORMS))
def test_roundtrip_256(rt, form):
    import mlegs_b200 as M
    cfg, cases = rt
    S, tol = FORMS[form]
    ctx = M.Context(cfg, precision=M.PREC_SPLIT if S else M.PREC_FP64, split_slices=S)
    try:
        f = ctx.field(M.FFF)
        for c, ppp, fff in cases:
            f.upload(c, 0.0, M.FFF)
            ctx.TOFP(f)
            assert f.space == M.PPP
            assert rel(f.download()[0], ppp) < tol
            ctx.TOFF(f)
            E, ln = f.download()
            assert f.space == M.FFF and ln == 0.0
            assert rel(E, fff) < tol
            assert rel(E, c) < tol  # band-limited input: the round trip is the identity
        ms, by = ctx.kernel_time("roundtrip", reps=3)
        assert ms > 0 and by > 0
    finally:
        ctx.close()

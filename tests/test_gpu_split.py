"""Split-BF16 (Ozaki) tensor-core RTRAN(+1) against the FP64 oracle.

The slices carry 8 bits each (the first 9), so S slices resolve about 8S + 1
bits of each operand; levels 0..2 of the slice products accumulate exactly in
FP32, and the rest rounds near 2^-48 of the row x column scale.  Tolerances
(max |d| / max |ref| over the field) per S are stated below, with headroom
over the truncation bound 2^-(8S+1) * sqrt(K).
"""

import numpy as np
import pytest

from conftest import oracle_grid, random_fff, rel, small_cfg

pytestmark = pytest.mark.gpu

TOL = {3: 2e-6, 4: 1e-8, 5: 5e-11, 6: 5e-12}


def _ctx(M, cfg, S):
    return M.Context(cfg, precision=M.PREC_SPLIT, split_slices=S)


@pytest.mark.parametrize("S", [3, 4, 5, 6])
@pytest.mark.parametrize("dims", [(32, 16, 16), (64, 32, 32)], ids=["32x16x16", "64x32x32"])
@pytest.mark.parametrize("pad", [0, 3])
def test_split_rtran_forward_vs_oracle(lib_built, dims, S, pad):
    import mlegs_b200 as M
    from oracle import transforms as T
    cfg = small_cfg(*dims)
    g = oracle_grid(cfg)
    ctx = _ctx(M, cfg, S)
    try:
        A = random_fff(g, 7 + S, pad=pad)
        A.LN = 0.37
        f = ctx.field(M.FFF)
        f.upload(A.E, A.LN, M.FFF)
        ctx.RTRAN(f, 1, pad)
        ctx.sync()
        g.chopset(pad)
        T.rtran(g, A, 1)
        g.chopset(-pad)
        E, ln = f.download()
        err = rel(E, A.E)
        print("split S=%d %s pad=%d rel err %.3e" % (S, dims, pad, err))
        assert f.space == M.PFF and ln == 0.0
        assert np.isfinite(E).all()
        assert err < TOL[S]
    finally:
        ctx.close()


@pytest.mark.parametrize("S", [5, 6])
def test_split_rtran_matches_fp64_at_bench_grid(lib_built, S):
    """192x128x256 (NRCHOP 128): split vs the FP64 GPU kernel on the same field."""
    import mlegs_b200 as M
    cfg = M.CONFIGS["etd_192x128x256"]
    rng = np.random.default_rng(3)
    c64 = M.Context(cfg)
    cs = _ctx(M, cfg, S)
    try:
        shape = c64.shape(M.FFF)
        n = np.arange(shape[0])[:, None, None]
        E0 = (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)) * np.exp(-n / 12.0)
        out = []
        for ctx in (c64, cs):
            f = ctx.field(M.FFF)
            f.upload(E0, 0.25, M.FFF)
            ctx.CHOPDO(f, 3)
            ctx.RTRAN(f, 1, 3)
            ctx.sync()
            out.append(f.download()[0])
        err = rel(out[1], out[0])
        print("split S=%d 192x128x256 rel err vs FP64 GPU %.3e" % (S, err))
        assert err < TOL[S]
    finally:
        cs.close()
        c64.close()


@pytest.mark.parametrize("S", [3, 4, 5, 6])
@pytest.mark.parametrize("dims", [(32, 16, 16), (64, 32, 32)], ids=["32x16x16", "64x32x32"])
@pytest.mark.parametrize("pad", [0, 3])
def test_split_rtran_backward_vs_oracle(lib_built, dims, S, pad):
    import mlegs_b200 as M
    from oracle import transforms as T
    from oracle.grid import PFF
    cfg = small_cfg(*dims)
    g = oracle_grid(cfg)
    ctx = _ctx(M, cfg, S)
    try:
        rng = np.random.default_rng(30 + S)
        A = g.alloc(PFF)
        A.E[: g.NR] = rng.standard_normal(A.E[: g.NR].shape) + 1j * rng.standard_normal(A.E[: g.NR].shape)
        f = ctx.field(M.PFF)
        f.upload(A.E, 0.0, M.PFF)
        ctx.RTRAN(f, -1, pad)
        ctx.sync()
        g.chopset(pad)
        T.rtran(g, A, -1)
        g.chopset(-pad)
        E, _ = f.download()
        err = rel(E, A.E)
        print("split S=%d %s pad=%d RTRAN(-1) rel err %.3e" % (S, dims, pad, err))
        assert f.space == M.FFF and np.isfinite(E).all()
        assert err < TOL[S]
    finally:
        ctx.close()


@pytest.mark.parametrize("S", [5, 6])
@pytest.mark.parametrize("mode", ["ppp_ln0", "pff_none", "fff_psi"])
def test_split_project_vs_oracle(lib_built, S, mode):
    import mlegs_b200 as M
    from oracle import legops as L
    from oracle import transforms as T
    cfg = small_cfg(64, 32, 32)
    g = oracle_grid(cfg)
    ctx = _ctx(M, cfg, S)
    try:
        U = [random_fff(g, 20 + i, decay=4.0) for i in range(3)]
        if mode == "ppp_ln0":
            for u in U:
                T.tofp(g, u)
            ln = 0.0
        elif mode == "pff_none":
            for u in U:
                T.rtran(g, u, 1)
            ln = None
        else:
            ln = "psi"
        fs = []
        for u in U:
            f = ctx.field(u.space)
            f.upload(u.E, u.LN, u.space)
            fs.append(f)
        psi, chi = ctx.field(M.FFF), ctx.field(M.FFF)
        ctx.PROJECT(*fs, psi, chi, ln)
        ctx.sync()
        P, W = L.project(g, *U, ln)
        Ep, lnp = psi.download()
        Ec, _ = chi.download()
        e1, e2 = rel(Ep, P.E), rel(Ec, W.E)
        print("split S=%d PROJECT %s rel err psi %.3e chi %.3e" % (S, mode, e1, e2))
        assert e1 < 20 * TOL[S] and e2 < 20 * TOL[S]
        assert abs(lnp - P.LN) < 20 * TOL[S] * max(1.0, abs(P.LN))
    finally:
        ctx.close()


@pytest.mark.parametrize("S", [5, 6])
def test_split_ab2_config_100_steps(lib_built, S):
    """AB2-CN IVP at 64x32x32 on the split-BF16 GEMMs: 1 Richardson + 99 AB2
    steps against the FP64 oracle, <= 1e-9 relative per field."""
    import mlegs_b200 as M
    from test_gpu_parity import _run_pair
    cfg = M.CONFIGS["ab2_64x32x32"]
    out, ref = _run_pair(cfg, 99, graph=True, precision=M.PREC_SPLIT, split_slices=S)
    errs = [rel(E, R.E) for (E, _), R in zip(out, ref)]
    lns = [abs(ln - R.LN) / max(1.0, abs(R.LN)) for (_, ln), R in zip(out, ref)]
    print("split S=%d AB2 100 steps rel err psi %.3e chi %.3e b %.3e, LN %.3e %.3e" % (S, *errs, lns[0], lns[1]))
    assert max(errs) < 1e-9 and max(lns) < 1e-9


@pytest.mark.parametrize("S", [5, 6])
def test_split_etd_steps_vs_oracle(lib_built, S):
    import mlegs_b200 as M
    from test_gpu_parity import _run_pair
    cfg = small_cfg(64, 32, 32, adams=False)
    out, ref = _run_pair(cfg, 10, graph=True, precision=M.PREC_SPLIT, split_slices=S)
    errs = [rel(E, R.E) for (E, _), R in zip(out, ref)]
    print("split S=%d ETD 11 steps rel err psi %.3e chi %.3e b %.3e" % (S, *errs))
    # ETD re-projects the whole state through RTRAN(+1) and PROJECT every step,
    # so the per-GEMM slice error accumulates step by step (S=5: about 5e-10 a
    # step in chi, 5.3e-9 after these 11 steps; S=6: under 5e-11 a step)
    assert max(errs) < {5: 1e-8, 6: 5e-10}[S]

"""GPU parity at the headline grid and at every FFT instantiation, through the C ABI.

The step kernels are compiled per size: the theta transforms and products
(`theta5_kernel<N1, N2>`), HORFFT (`horfft5_kernel<N1, N2>`) and VERFFT
(`verfft4_kernel<N1, N2>`) are templates dispatched on NTH and NX.  These tests
run each dispatched form against the FP64 oracle:

* 192x128x256 (the ETD configuration the benchmark times, chops 128/85/85):
  the device Legendre table against the 50-digit golden values, RTRAN(+-1),
  VERFFT(+-1), HORFFT(+-1), TOFP/TOFF, PROJECT in its PFF and FFF forms,
  CALC_BOUSSI_NONLIN (`theta5<16,8>` in the nonlinear-term form),
  CALC_BOUSSI_FORCE, and the Richardson start-up plus two ETD2AB-CN steps,
  each in FP64 and with the split-BF16 (S = 6) tensor-core GEMMs;
* smaller NR at NTH / NX = 64, 128, 256, 512: the transforms, the two
  physical-stage forms and a start-up plus one ETD step.

Tolerances (max|d| / max|ref|): 1e-12 per operator (FP64 and split), 1e-11
for the projections and the nonlinear terms, 1e-10 for the banded solves and
whole steps.
"""

import os

import numpy as np
import pytest

from conftest import oracle_grid, oracle_physics, rel, small_cfg

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "legendre_golden.npz")
PRECS = ["fp64", "split6"]
# max|d| / max|ref| of PROJECT and CALC_BOUSSI_NONLIN: the split-BF16 form's
# per-row power-of-two scaling keeps 48 bits of each row's largest weight, and
# PROJECT's V and D weights (1/(n(n+1)(1-x^2)/w)) span many orders of magnitude
PROJ_TOL = {"fp64": 1e-11, "split6": 5e-11}


def _ctx(M, cfg, prec):
    if prec == "fp64":
        return M.Context(cfg)
    return M.Context(cfg, precision=M.PREC_SPLIT, split_slices=6)


def up(ctx, F):
    f = ctx.field(F.space)
    f.upload(F.E, F.LN, F.space)
    return f


@pytest.fixture(scope="module")
def head(lib_built):
    import mlegs_b200 as M
    from mlegs_b200.inputs import CONFIGS
    cfg = CONFIGS["etd_192x128x256"]
    g = oracle_grid(cfg)
    ctxs = {p: _ctx(M, cfg, p) for p in PRECS}
    yield M, ctxs, g, cfg
    for c in ctxs.values():
        c.close()


@pytest.fixture(scope="module")
def head_state(head):
    """The benchmark's initial state (q-vortex + seeded perturbation) in the oracle."""
    from mlegs_b200.inputs import perturbation_coefficients
    from oracle import layout
    M, ctxs, g, cfg = head
    cs = [perturbation_coefficients(cfg, i) for i in range(3)]
    return layout.initial_state(g, *cs)


def test_legendre_table_golden_192(head):
    """TFM%PF built on the device (FP64 recurrence) against the 50-digit
    LEG_TBL3 values at NR = 192 for m = 0, 42, 84 (NTCHOPDIM - 1)."""
    M, ctxs, g, cfg = head
    z = np.load(GOLDEN)
    assert int(z["c2_nr"]) == 192
    gold = z["c2_pf"]
    pf = ctxs["fp64"].legendre_table()
    assert pf.shape == (96, 135, 85) and gold.shape[:2] == pf.shape[:2]
    for j, m in enumerate(z["c2_ms"]):
        assert rel(pf[:, :, m], gold[:, :, j]) < 1e-12, m
        assert np.array_equal(pf[:, :, m] == 0.0, gold[:, :, j] == 0.0), m
    x, _, _ = ctxs["fp64"].grid()
    assert np.abs(x - z["c2_x"]).max() < 5e-15


@pytest.mark.parametrize("prec", PRECS)
@pytest.mark.parametrize("pad", [0, 3])
def test_rtran_headline(head, prec, pad):
    from conftest import random_fff
    from oracle import transforms as T
    from oracle.grid import PFF
    M, ctxs, g, cfg = head
    ctx = ctxs[prec]
    A = random_fff(g, 101, decay=12.0, pad=pad)
    A.LN = -0.45
    f = up(ctx, A)
    ctx.RTRAN(f, 1, pad)
    g.chopset(pad)
    T.rtran(g, A, 1)
    g.chopset(-pad)
    assert rel(f.download()[0], A.E) < 1e-12
    rng = np.random.default_rng(102)
    Bp = g.alloc(PFF)
    Bp.E[: g.NR] = rng.standard_normal(Bp.E[: g.NR].shape) + 1j * rng.standard_normal(Bp.E[: g.NR].shape)
    h = up(ctx, Bp)
    ctx.RTRAN(h, -1, pad)
    g.chopset(pad)
    T.rtran(g, Bp, -1)
    g.chopset(-pad)
    assert rel(h.download()[0], Bp.E) < 1e-12


def test_verfft_horfft_headline(head):
    """VERFFT(+-1) at NX = 256 (verfft4<16,16>) and HORFFT(+-1) at NTH = 128 (horfft5<16,8>)."""
    from oracle import transforms as T
    from oracle.grid import PFF, PFP
    M, ctxs, g, cfg = head
    ctx = ctxs["fp64"]
    rng = np.random.default_rng(103)
    A = g.alloc(PFF)
    A.E[: g.NR] = rng.standard_normal(A.E[: g.NR].shape) + 1j * rng.standard_normal(A.E[: g.NR].shape)
    f = up(ctx, A)
    ctx.VERFFT(f, 1)
    T.verfft(g, A, 1)
    assert f.space == M.PFP and rel(f.download()[0], A.E) < 1e-12
    ctx.VERFFT(f, -1)
    T.verfft(g, A, -1)
    assert f.space == M.PFF and rel(f.download()[0], A.E) < 1e-12
    P = g.alloc(PFP)
    sh = (g.NR, g.NTCHOPDIM, g.NX)
    P.E[: g.NR, : g.NTCHOPDIM, :] = rng.standard_normal(sh) + 1j * rng.standard_normal(sh)
    P.E[: g.NR, 0, :] = P.E[: g.NR, 0, :].real
    h = up(ctx, P)
    ctx.HORFFT(h, 1)
    T.horfft(g, P, 1)
    assert h.space == M.PPP and rel(h.download()[0], P.E) < 1e-12
    ctx.HORFFT(h, -1)
    T.horfft(g, P, -1)
    assert h.space == M.PFP and rel(h.download()[0], P.E) < 1e-12


@pytest.mark.parametrize("prec", PRECS)
@pytest.mark.parametrize("which", [0, 2], ids=["psi", "b"])
def test_tofp_toff_headline(head, head_state, prec, which):
    """TOFP then TOFF of the benchmark's psi (log term -0.5: RTRAN(+1) adds
    LN log(1-x) in physical space, which TOFF maps onto the spectrum) and b
    (LN = 0, band-limited: the round trip is the identity)."""
    from oracle import transforms as T
    M, ctxs, g, cfg = head
    ctx = ctxs[prec]
    B = head_state[which].copy()
    f = up(ctx, B)
    ctx.TOFP(f)
    T.tofp(g, B)
    assert f.space == M.PPP and rel(f.download()[0], B.E) < 1e-12
    ctx.TOFF(f)
    T.toff(g, B)
    E, ln = f.download()
    assert f.space == M.FFF and rel(E, B.E) < 1e-12 and ln == 0.0
    if head_state[which].LN == 0.0:
        assert rel(E, head_state[which].E) < 1e-12


def _velocity(g, P, C):
    from oracle import legops as L
    g.chopset(3)
    U = L.pc2vel(g, P, C)
    O = L.pc2vor(g, P, C)
    g.chopset(-3)
    return U, O


@pytest.mark.parametrize("prec", PRECS)
@pytest.mark.parametrize("form", ["pff", "fff_psi"])
def test_project_headline(head, head_state, prec, form):
    """PROJECT of PFF input with LN = 0 (the five fold products; legfold_dmma in
    FP64) and of FFF input with PSI%LN by reference (the steppers' form; the
    composite W.PF^T product projfff_dmma in FP64)."""
    from oracle import legops as L
    from oracle import transforms as T
    M, ctxs, g, cfg = head
    ctx = ctxs[prec]
    U, _ = _velocity(g, head_state[0], head_state[1])
    U = [u.copy() for u in U]
    for u in U:
        u.LN = 0.0
    if form == "pff":
        for u in U:
            T.rtran(g, u, 1)
        ln = 0.0
    else:
        ln = "psi"
    fs = [up(ctx, u) for u in U]
    psi, chi = ctx.field(M.FFF), ctx.field(M.FFF)
    ctx.PROJECT(*fs, psi, chi, ln)
    P, W = L.project(g, *[u.copy() for u in U], 0.0 if form == "pff" else "psi")
    Ep, lnp = psi.download()
    tol = PROJ_TOL[prec]
    assert rel(Ep, P.E) < tol
    assert rel(chi.download()[0], W.E) < tol
    assert abs(lnp - P.LN) < tol * max(1.0, abs(P.LN))


@pytest.fixture(scope="module")
def head_nonlin(head, head_state):
    """Inputs (velocity, vorticity) and the oracle's CALC_BOUSSI_NONLIN at 192x128x256."""
    from oracle import boussinesq as BQ
    M, ctxs, g, cfg = head
    P, C, B = head_state
    U, O = _velocity(g, P, C)
    ref = BQ.calc_boussi_nonlin(g, B.copy(), *[x.copy() for x in U], *[x.copy() for x in O])
    return U, O, ref


@pytest.mark.parametrize("prec", PRECS)
def test_boussi_nonlin_headline(head, head_state, head_nonlin, prec):
    """CALC_BOUSSI_NONLIN at 192x128x256: nine RTRAN(+1)/VERFFT(+1) pairs, the
    fused theta stage (theta5<16,8>: HORFFT(+1), VPRODSUB, VDOTPSUB,
    HORFFT(-1)), PROJECT, IDEL2, PC2VEL, TOFF."""
    M, ctxs, g, cfg = head
    ctx = ctxs[prec]
    U, O, (BN, NR_, NP_, NZ_) = head_nonlin
    fb = up(ctx, head_state[2])
    fu = [up(ctx, x) for x in U]
    fo = [up(ctx, x) for x in O]
    bn = ctx.field(M.FFF)
    ctx.CALC_BOUSSI_NONLIN(fb, *fu, bn, *fo)
    for f, R in zip(fo + [bn], (NR_, NP_, NZ_, BN)):
        E, ln = f.download()
        assert f.space == M.FFF
        assert rel(E, R.E) < PROJ_TOL[prec]
        assert abs(ln - R.LN) < PROJ_TOL[prec] * max(1.0, abs(R.LN))


def test_boussi_force_headline(head, head_state):
    """CALC_BOUSSI_FORCE (the AB2-CN right-hand side: theta5<16,8> with the
    Coriolis / buoyancy linear terms, 10 inverse transforms) at 192x128x256."""
    from oracle import boussinesq as BQ
    M, ctxs, g, cfg = head
    ctx = ctxs["fp64"]
    P, C, B = head_state
    fp, fc, fb = (up(ctx, x) for x in (P, C, B))
    outs = [ctx.field(M.FFF) for _ in range(3)]
    ctx.CALC_BOUSSI_FORCE(fp, fc, fb, *outs)
    ref = BQ.calc_boussi_force(g, oracle_physics(cfg), P.copy(), C.copy(), B.copy())
    for o, R in zip(outs, ref):
        E, ln = o.download()
        assert rel(E, R.E) < 1e-10  # CHIN comes out of the IDEL2LN banded solve
        assert abs(ln - R.LN) < 1e-10 * max(1.0, abs(R.LN))


@pytest.fixture(scope="module")
def head_oracle_steps(head, head_state):
    """Oracle Richardson start-up + 2 ETD2AB-CN steps from the benchmark state."""
    from oracle import boussinesq as BQ
    M, ctxs, g, cfg = head
    P, C, B = head_state
    s = BQ.Solver(g, oracle_physics(cfg), P.copy(), C.copy(), B.copy())
    s.initialize()
    s.step()
    s.step()
    return s


# whole steps: FP64 within the banded-solve tolerance; the split-BF16 path
# within the 1e-9 field bound the mixed-precision step is held to
STEP_TOL = {"fp64": 1e-10, "split6": 1e-9}


@pytest.mark.parametrize("prec", PRECS)
def test_etd_steps_headline(head, head_state, head_oracle_steps, prec):
    """The benchmark's step at its own size: Richardson start-up and two
    ETD2AB-CN steps (graph-replayed, as timed) against the oracle."""
    M, ctxs, g, cfg = head
    s = head_oracle_steps
    ctx = _ctx(M, cfg, prec)
    try:
        fp, fc, fb = (up(ctx, x) for x in head_state)
        ctx.initialize(fp, fc, fb)
        ctx.step(2, graph=True)
        ctx.check_finite()
        for f, R in ((fp, s.psi), (fc, s.chi), (fb, s.b)):
            E, ln = f.download()
            assert rel(E, R.E) < STEP_TOL[prec]
            assert abs(ln - R.LN) < STEP_TOL[prec] * max(1.0, abs(R.LN))
        t, n = ctx.time()
        assert n == 3 and abs(t - s.t) < 1e-12
    finally:
        ctx.close()


# ---------------------------------------------------------------- other sizes
# (NR, NTH, NX) -> theta5 / horfft5 <N1, N2> at NTH, verfft4 <N1, N2> at NX
GRIDS = [(32, 64, 128), (32, 256, 64), (16, 512, 512)]


@pytest.fixture(scope="module", params=GRIDS, ids=["%dx%dx%d" % x for x in GRIDS])
def other(request, lib_built):
    import mlegs_b200 as M
    cfg = small_cfg(*request.param, adams=False)
    g = oracle_grid(cfg)
    ctx = M.Context(cfg)
    yield M, ctx, g, cfg
    ctx.close()


def test_transforms_other_sizes(other):
    from conftest import random_fff
    from oracle import transforms as T
    M, ctx, g, cfg = other
    A = random_fff(g, 111)
    A.LN = 0.3
    f = up(ctx, A)
    B = A.copy()
    for IS, fn in ((1, "RTRAN"), (1, "VERFFT"), (1, "HORFFT")):
        getattr(ctx, fn)(f, IS)
        getattr(T, fn.lower())(g, B, IS)
        assert rel(f.download()[0], B.E) < 1e-12, fn
    for IS, fn in ((-1, "HORFFT"), (-1, "VERFFT"), (-1, "RTRAN")):
        getattr(ctx, fn)(f, IS)
        getattr(T, fn.lower())(g, B, IS)
        assert rel(f.download()[0], B.E) < 1e-12, fn


def test_physical_stage_other_sizes(other):
    """Both theta-stage forms: CALC_BOUSSI_FORCE (linear terms) and
    CALC_BOUSSI_NONLIN."""
    from mlegs_b200.inputs import perturbation_coefficients
    from oracle import boussinesq as BQ
    from oracle import layout
    M, ctx, g, cfg = other
    cs = [perturbation_coefficients(cfg, i) for i in range(3)]
    P, C, B = layout.initial_state(g, *cs)
    fp, fc, fb = (up(ctx, x) for x in (P, C, B))
    outs = [ctx.field(M.FFF) for _ in range(3)]
    ctx.CALC_BOUSSI_FORCE(fp, fc, fb, *outs)
    ref = BQ.calc_boussi_force(g, oracle_physics(cfg), P.copy(), C.copy(), B.copy())
    for o, R in zip(outs, ref):
        assert rel(o.download()[0], R.E) < 1e-11
    U, O = _velocity(g, P, C)
    fu = [up(ctx, x) for x in U]
    fo = [up(ctx, x) for x in O]
    bn = ctx.field(M.FFF)
    ctx.CALC_BOUSSI_NONLIN(fb, *fu, bn, *fo)
    BN, NR_, NP_, NZ_ = BQ.calc_boussi_nonlin(g, B.copy(), *[x.copy() for x in U], *[x.copy() for x in O])
    for f, R in zip(fo + [bn], (NR_, NP_, NZ_, BN)):
        assert rel(f.download()[0], R.E) < 1e-11


def test_etd_step_other_sizes(other):
    from mlegs_b200.inputs import perturbation_coefficients
    from oracle import boussinesq as BQ
    from oracle import layout
    M, ctx, g, cfg = other
    cs = [perturbation_coefficients(cfg, i) for i in range(3)]
    P, C, B = layout.initial_state(g, *cs)
    s = BQ.Solver(g, oracle_physics(cfg), P.copy(), C.copy(), B.copy())
    s.initialize()
    s.step()
    fp, fc, fb = (up(ctx, x) for x in (P, C, B))
    ctx.initialize(fp, fc, fb)
    ctx.step(1)
    for f, R in ((fp, s.psi), (fc, s.chi), (fb, s.b)):
        E, ln = f.download()
        assert rel(E, R.E) < 1e-10
        assert abs(ln - R.LN) < 1e-10 * max(1.0, abs(R.LN))

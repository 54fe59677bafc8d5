"""The device adjoint (include/mlegs_b200.h, MLEGS_T_* and the VJP entry
points; mlegs_b200/adjoint.py) on a B200.

1. Every transpose against the device's own forward operator by the
   dot-product identity <y, F(x)> = <F^T(y), x> (log terms included) on random
   inputs that fill every stored entry, chopped ones too.
2. The composite VJPs (CALC_BOUSSI_FORCE, one AB2-CN step, the Richardson
   start-up, the initial state, the objective's gradient) against the
   oracle's (oracle/adjoint.py) at small grids.
3. The whole gradient through torch.autograd (InitialState -> Startup ->
   checkpointed run_loop -> Objective) against the oracle's reverse
   accumulation, and at the gradient workload (96x64x64, 200 AB2-CN steps,
   checkpoints every 20) against central finite differences of the device's
   own forward on 32 random directions.
"""

import numpy as np
import pytest

from conftest import oracle_grid, oracle_physics, rel, small_cfg

pytestmark = pytest.mark.gpu

GRIDS = [(32, 16, 16), (48, 32, 32)]  # NTH and NX powers of two


@pytest.fixture(scope="module", params=GRIDS, ids=["%dx%dx%d" % d for d in GRIDS])
def env(request, lib_built):
    import mlegs_b200 as M
    cfg = small_cfg(*request.param, adams=True)
    ctx = M.Context(cfg)
    g = oracle_grid(cfg)
    yield M, ctx, g, cfg
    ctx.close()


def _dot(a, b):
    return float(np.sum(a.real * b.real + a.imag * b.imag))


def _rand(g, space, seed):
    from oracle.grid import Field
    rng = np.random.default_rng(seed)
    shape = g.shape(space)
    return Field(rng.standard_normal(shape) + 1j * rng.standard_normal(shape), space, float(rng.standard_normal()))


def _up(ctx, F):
    f = ctx.field(F.space)
    f.upload(F.E, F.LN, F.space)
    return f


def _down(f):
    return f.download()


def _check_identity(lhs, rhs, scale, tol):
    assert abs(lhs - rhs) <= tol * scale, (lhs, rhs, abs(lhs - rhs) / scale)


# ---------------------------------------------------------------- 1. transposes
def _spaces():
    from oracle.grid import FFF, PFF, PFP, PPP
    return FFF, PFF, PFP, PPP


@pytest.mark.parametrize("pad", [0, 3])
def test_transform_transposes(env, pad):
    """RTRAN(+-1), VERFFT(+-1), HORFFT(+-1), TOFP, TOFF."""
    M, ctx, g, cfg = env
    FFF, PFF, PFP, PPP = _spaces()
    cases = [  # name, forward, in space, out space, input LN used
        ("RTRAN+1", lambda f: ctx.RTRAN(f, 1, pad), FFF, PFF, True),
        ("RTRAN-1", lambda f: ctx.RTRAN(f, -1, pad), PFF, FFF, False),
        ("VERFFT+1", lambda f: ctx.VERFFT(f, 1), PFF, PFP, False),
        ("VERFFT-1", lambda f: ctx.VERFFT(f, -1), PFP, PFF, False),
        ("HORFFT+1", lambda f: ctx.HORFFT(f, 1), PFP, PPP, False),
        ("HORFFT-1", lambda f: ctx.HORFFT(f, -1), PPP, PFP, False),
        ("TOFP", lambda f: ctx.TOFP(f, pad), FFF, PPP, True),
        ("TOFF", lambda f: ctx.TOFF(f, pad), PPP, FFF, False),
    ]
    for i, (name, fwd, sin, sout, with_ln) in enumerate(cases):
        x = _rand(g, sin, 100 + i)
        if not with_ln:
            x.LN = 0.0
        y = _rand(g, sout, 200 + i)
        y.LN = 0.0
        fx = _up(ctx, x)
        fwd(fx)
        Fx, _ = _down(fx)
        xt = ctx.field(sin)
        ctx.TRANSPOSE(name, [_up(ctx, y)], [xt], pad)
        Xt, lt = _down(xt)
        lhs = _dot(y.E, Fx)
        rhs = _dot(Xt, x.E) + (lt * x.LN if with_ln else 0.0)
        scale = np.linalg.norm(y.E) * np.linalg.norm(Fx) + 1e-300
        _check_identity(lhs, rhs, scale, 1e-13)


@pytest.mark.parametrize("pad", [0, 3])
def test_operator_transposes(env, pad):
    """XXDX, MULXM, DELSQH, DEL2 (log-term rows), GRAD, PC2VEL, PC2VOR, IDELSQH."""
    M, ctx, g, cfg = env
    FFF = _spaces()[0]
    unary = [("XXDX", ctx.XXDX, True), ("MULXM", ctx.MULXM, False), ("DELSQH", ctx.DELSQH, True),
             ("DEL2", ctx.DEL2, True), ("IDELSQH", ctx.IDELSQH, False)]
    for i, (name, op, with_ln) in enumerate(unary):
        x = _rand(g, FFF, 300 + i)
        if not with_ln:
            x.LN = 0.0
        y = _rand(g, FFF, 400 + i)
        out = ctx.field(FFF)
        op(_up(ctx, x), out, pad)
        Fx, Fln = _down(out)
        xt = ctx.field(FFF)
        ctx.TRANSPOSE(name, [_up(ctx, y)], [xt], pad)
        Xt, lt = _down(xt)
        lhs = _dot(y.E, Fx) + y.LN * Fln
        rhs = _dot(Xt, x.E) + lt * x.LN
        scale = np.linalg.norm(y.E) * np.linalg.norm(Fx) + abs(y.LN * Fln) + 1e-300
        _check_identity(lhs, rhs, scale, 1e-13)
    # GRAD: one input (with LN), three outputs
    x = _rand(g, FFF, 500)
    ys = [_rand(g, FFF, 510 + q) for q in range(3)]
    outs = [ctx.field(FFF) for _ in range(3)]
    ctx.GRAD(_up(ctx, x), *outs, pad)
    Fx = [_down(o)[0] for o in outs]
    xt = ctx.field(FFF)
    ctx.TRANSPOSE("GRAD", [_up(ctx, y) for y in ys], [xt], pad)
    Xt, lt = _down(xt)
    lhs = sum(_dot(y.E, f) for y, f in zip(ys, Fx))
    rhs = _dot(Xt, x.E) + lt * x.LN
    scale = sum(np.linalg.norm(y.E) * np.linalg.norm(f) for y, f in zip(ys, Fx))
    _check_identity(lhs, rhs, scale, 1e-13)
    # PC2VEL, PC2VOR: two inputs (with LN), three outputs
    for name, op in (("PC2VEL", ctx.PC2VEL), ("PC2VOR", ctx.PC2VOR)):
        xs = [_rand(g, FFF, 600 + q) for q in range(2)]
        ys = [_rand(g, FFF, 610 + q) for q in range(3)]
        outs = [ctx.field(FFF) for _ in range(3)]
        op(_up(ctx, xs[0]), _up(ctx, xs[1]), *outs, pad)
        Fx = [_down(o)[0] for o in outs]
        xt = [ctx.field(FFF) for _ in range(2)]
        ctx.TRANSPOSE(name, [_up(ctx, y) for y in ys], xt, pad)
        Xt = [_down(f) for f in xt]
        lhs = sum(_dot(y.E, f) for y, f in zip(ys, Fx))
        rhs = sum(_dot(E, x.E) + l * x.LN for (E, l), x in zip(Xt, xs))
        scale = sum(np.linalg.norm(y.E) * np.linalg.norm(f) for y, f in zip(ys, Fx))
        _check_identity(lhs, rhs, scale, 1e-13)


def test_solve_and_project_transposes(env):
    """IDEL2LN, IHELM (with their log terms) and PROJECT of PPP inputs with LN = 0."""
    M, ctx, g, cfg = env
    FFF, PFF, PFP, PPP = _spaces()
    # IDEL2LN: B -> (A, A%LN); B%LN unused
    x = _rand(g, FFF, 700)
    x.LN = 0.0
    y = _rand(g, FFF, 701)
    out = ctx.field(FFF)
    ctx.IDEL2LN(_up(ctx, x), out)
    Fx, Fln = _down(out)
    xt = ctx.field(FFF)
    ctx.TRANSPOSE("IDEL2LN", [_up(ctx, y)], [xt])
    Xt, lt = _down(xt)
    assert lt == 0.0
    lhs = _dot(y.E, Fx) + y.LN * Fln
    _check_identity(lhs, _dot(Xt, x.E), np.linalg.norm(y.E) * np.linalg.norm(Fx) + abs(y.LN * Fln), 1e-12)
    # IHELM: (B, B%LN) -> (A, A%LN)
    for alp in (2 / cfg.nu / cfg.dt, 1 / (cfg.nu * cfg.dt)):
        x = _rand(g, FFF, 710)
        y = _rand(g, FFF, 711)
        out = ctx.field(FFF)
        ctx.IHELM(_up(ctx, x), out, alp)
        Fx, Fln = _down(out)
        xt = ctx.field(FFF)
        ctx.TRANSPOSE("IHELM", [_up(ctx, y)], [xt], 0, alp)
        Xt, lt = _down(xt)
        lhs = _dot(y.E, Fx) + y.LN * Fln
        rhs = _dot(Xt, x.E) + lt * x.LN
        _check_identity(lhs, rhs, np.linalg.norm(y.E) * np.linalg.norm(Fx) + abs(y.LN * Fln), 1e-12)
    # PROJECT(ROR, ROP, OZ, PSI, W, 0.0) of PPP inputs
    xs = [_rand(g, PPP, 720 + q) for q in range(3)]
    for x in xs:
        x.LN = 0.0
    ys = [_rand(g, FFF, 730 + q) for q in range(2)]
    fin = [_up(ctx, x) for x in xs]
    psi, w = ctx.field(FFF), ctx.field(FFF)
    ctx.PROJECT(*fin, psi, w, LN=0.0)
    Fp, lp = _down(psi)
    Fw, _ = _down(w)
    assert lp == 0.0
    xt = [ctx.field(PPP) for _ in range(3)]
    ctx.TRANSPOSE("PROJECT_PPP", [_up(ctx, y) for y in ys], xt)
    Xt = [_down(f)[0] for f in xt]
    lhs = _dot(ys[0].E, Fp) + _dot(ys[1].E, Fw)
    rhs = sum(_dot(X, x.E) for X, x in zip(Xt, xs))
    scale = np.linalg.norm(ys[0].E) * np.linalg.norm(Fp) + np.linalg.norm(ys[1].E) * np.linalg.norm(Fw)
    _check_identity(lhs, rhs, scale, 1e-12)


def test_transposes_match_oracle(env):
    """A few transposes value for value against oracle/adjoint.py."""
    from oracle import adjoint as AD
    M, ctx, g, cfg = env
    FFF, PFF, PFP, PPP = _spaces()
    y = _rand(g, PPP, 800)
    y.LN = 0.0
    xt = ctx.field(FFF)
    ctx.TRANSPOSE("TOFP", [_up(ctx, y)], [xt], 0)
    E, ln = _down(xt)
    ref = AD.tofp_T(g, y)
    assert rel(E, ref.E) < 1e-12 and abs(ln - ref.LN) <= 1e-12 * max(1.0, abs(ref.LN))
    y = _rand(g, FFF, 801)
    g.chopdo(y)
    xt = ctx.field(FFF)
    ctx.TRANSPOSE("IDEL2LN", [_up(ctx, y)], [xt])
    E, _ = _down(xt)
    assert rel(E, AD.idel2ln_T(g, y).E) < 1e-11
    alp = 2 / cfg.nu / cfg.dt
    ctx.TRANSPOSE("IHELM", [_up(ctx, y)], [xt], 0, alp)
    E, ln = _down(xt)
    ref = AD.ihelm_T(g, y, alp)
    assert rel(E, ref.E) < 1e-11 and abs(ln - ref.LN) <= 1e-11 * max(1.0, abs(ref.LN))


# ---------------------------------------------------------------- 2. composite VJPs
def _solver_state(M, cfg, g, steps=1):
    from oracle import boussinesq as BQ
    from oracle import layout
    from mlegs_b200.inputs import perturbation_coefficients
    ph = oracle_physics(cfg)
    P, C, B = layout.initial_state(g, *[perturbation_coefficients(cfg, i) for i in range(3)])
    s = BQ.Solver(g, ph, P, C, B)
    s.initialize()
    for _ in range(steps):
        s.step()
    return s, ph


def _rnd_fff(g, seed, ln=True):
    from oracle.grid import FFF
    F = _rand(g, FFF, seed)
    g.chopdo(F)
    if not ln:
        F.LN = 0.0
    return F


def test_force_vjp_matches_oracle(env):
    from oracle import adjoint as AD
    M, ctx, g, cfg = env
    s, ph = _solver_state(M, cfg, g)
    bars = [_rnd_fff(g, 900), _rnd_fff(g, 901), _rnd_fff(g, 902, ln=False)]
    ref = AD.boussi_force_vjp(g, ph, s.psi, s.chi, s.b, *bars)
    outs = [ctx.field() for _ in range(3)]
    ctx.CALC_BOUSSI_FORCE_VJP(_up(ctx, s.psi), _up(ctx, s.chi), _up(ctx, s.b), *[_up(ctx, b) for b in bars], *outs)
    for o, r in zip(outs, ref):
        E, ln = _down(o)
        assert rel(E, r.E) < 1e-10
        assert abs(ln - r.LN) <= 1e-10 * max(np.abs(r.E).max(), abs(r.LN))


def test_ab2_step_map_and_vjp_match_oracle(env):
    import copy
    from oracle import adjoint as AD
    M, ctx, g, cfg = env
    s, ph = _solver_state(M, cfg, g)
    keys = AD.AB2_STATE
    ins = [_up(ctx, getattr(s, k)) for k in keys]
    outs = [ctx.field() for _ in keys]
    ctx.AB2_STEP_MAP(ins, outs)
    s2 = copy.deepcopy(s)
    s2._step_ab_cn()
    for o, k in zip(outs, keys):
        E, ln = _down(o)
        r = getattr(s2, k)
        assert rel(E, r.E) < 1e-11, k
        assert abs(ln - r.LN) <= 1e-11 * max(1.0, abs(r.LN)), k
    lnk = ("psi", "chi", "n_psi", "n_chi")
    bars = {k: _rnd_fff(g, 950 + i, ln=k in lnk) for i, k in enumerate(keys)}
    ref = AD.ab_cn_step_vjp(s, bars)
    outs = [ctx.field() for _ in keys]
    ctx.AB2_STEP_VJP([_up(ctx, getattr(s, k)) for k in ("psi", "chi", "b")], [_up(ctx, bars[k]) for k in keys], outs)
    for o, k in zip(outs, keys):
        E, ln = _down(o)
        r = ref[k]
        assert rel(E, r.E) < 1e-10, k
        assert abs(ln - r.LN) <= 1e-10 * max(np.abs(r.E).max(), abs(r.LN)), k


def test_startup_map_and_vjp_match_oracle(env):
    import copy
    from oracle import adjoint as AD
    from oracle import boussinesq as BQ
    from oracle import layout
    from mlegs_b200.inputs import perturbation_coefficients
    M, ctx, g, cfg = env
    ph = oracle_physics(cfg)
    P, C, B = layout.initial_state(g, *[perturbation_coefficients(cfg, i) for i in range(3)])
    s0 = BQ.Solver(g, ph, P.copy(), C.copy(), B.copy())
    ins = [_up(ctx, F) for F in (P, C, B)]
    outs = [ctx.field() for _ in range(6)]
    ctx.AB2_STARTUP_MAP(ins, outs)
    s1 = copy.deepcopy(s0)
    s1.initialize()
    for o, k in zip(outs, AD.AB2_STATE):
        E, ln = _down(o)
        r = getattr(s1, k)
        assert rel(E, r.E) < 1e-11, k
        assert abs(ln - r.LN) <= 1e-11 * max(1.0, abs(r.LN)), k
    lnk = ("psi", "chi", "n_psi", "n_chi")
    bars = {k: _rnd_fff(g, 970 + i, ln=k in lnk) for i, k in enumerate(AD.AB2_STATE)}
    ref = AD.rich_fe_be_vjp(s0, bars)
    outs = [ctx.field() for _ in range(3)]
    ctx.AB2_STARTUP_VJP(ins, [_up(ctx, bars[k]) for k in AD.AB2_STATE], outs)
    for o, k in zip(outs, ("psi", "chi", "b")):
        E, ln = _down(o)
        r = ref[k]
        assert rel(E, r.E) < 1e-10, k
        assert abs(ln - r.LN) <= 1e-10 * max(np.abs(r.E).max(), abs(r.LN)), k


def test_objective_and_initial_state_transpose_match_oracle(env):
    from oracle import adjoint as AD
    M, ctx, g, cfg = env
    s, ph = _solver_state(M, cfg, g)
    J_ref = AD.energy_objective(g, s.psi, s.chi, s.b)
    G_ref = AD.energy_objective_grad(g, s.psi, s.chi, s.b)
    gs = [ctx.field() for _ in range(3)]
    J = ctx.ENERGY_OBJECTIVE(_up(ctx, s.psi), _up(ctx, s.chi), _up(ctx, s.b), *gs)
    assert abs(J - J_ref) <= 1e-11 * abs(J_ref)
    for o, r in zip(gs, G_ref):
        assert rel(_down(o)[0], r.E) < 1e-11
    bars = [_rnd_fff(g, 990), _rnd_fff(g, 991), _rnd_fff(g, 992, ln=False)]
    ref = AD.initial_state_T(g, *bars)
    outs = [ctx.field() for _ in range(3)]
    ctx.INITIAL_STATE_T([_up(ctx, b) for b in bars], outs)
    for o, r in zip(outs, ref):
        assert rel(_down(o)[0], r) < 1e-12


# ---------------------------------------------------------------- 3. the whole gradient
@pytest.mark.parametrize("dims", [(32, 16, 16), (48, 32, 32)], ids=["32x16x16", "48x32x32"])
def test_gradient_chain_matches_oracle(dims, lib_built):
    """torch.autograd through InitialState -> Startup -> run_loop -> Objective
    (two AB2-CN steps, checkpoints every step) against the oracle's reverse
    accumulation of the same maps."""
    import copy
    import mlegs_b200 as M
    from mlegs_b200.adjoint import DeviceAB2, dev_to_ref, gradient, ref_to_dev
    from mlegs_b200.checkpoint import LoopStats
    from mlegs_b200.inputs import perturbation_coefficients
    from oracle import adjoint as AD
    from oracle import boussinesq as BQ
    from oracle import layout
    from oracle.grid import FFF, Field
    cfg = small_cfg(*dims, adams=True)
    g = oracle_grid(cfg)
    ph = oracle_physics(cfg)
    cs = [perturbation_coefficients(cfg, i) for i in range(3)]
    n = 2
    P, C, B = layout.initial_state(g, *cs)
    s = BQ.Solver(g, ph, P.copy(), C.copy(), B.copy())
    s.initialize()
    traj = [s]
    for _ in range(n):
        s2 = copy.deepcopy(traj[-1])
        s2._step_ab_cn()
        traj.append(s2)
    J_ref = AD.energy_objective(g, *[getattr(traj[-1], k) for k in ("psi", "chi", "b")])
    keys = AD.AB2_STATE

    def objective_grad(st):
        gp, gc, gb = AD.energy_objective_grad(g, st["psi"], st["chi"], st["b"])
        bars = {k: Field(np.zeros(g.shape(FFF), dtype=np.complex128), FFF, 0.0) for k in keys}
        bars["psi"], bars["chi"], bars["b"] = gp, gc, gb
        return bars

    bars = AD.trajectory_grad(traj[0], n, objective_grad)
    x0_bar = AD.rich_fe_be_vjp(BQ.Solver(g, ph, P.copy(), C.copy(), B.copy()), bars)
    c_ref = AD.initial_state_T(g, x0_bar["psi"], x0_bar["chi"], x0_bar["b"])

    ctx = M.Context(cfg)
    try:
        solver = DeviceAB2(ctx)
        stats = LoopStats()
        J, grads = gradient(solver, [ref_to_dev(c) for c in cs], nsteps=n, every=1, stats=stats)
        assert stats.forward_steps == n and stats.vjp_steps == n
        assert abs(J - J_ref) <= 1e-10 * abs(J_ref)
        for gq, r in zip(grads, c_ref):
            assert rel(dev_to_ref(gq), r) < 1e-9
    finally:
        ctx.close()


def test_gradient_workload_matches_finite_differences(lib_built):
    """The gradient workload: 96x64x64, Re = 2000, start-up + 200 AB2-CN
    steps at dt = 1e-3, perturbation amplitude 1e-4, checkpoints every 20
    steps with recomputation; the device gradient against central finite
    differences of the device's own forward (the context's graph-captured
    solver) on 32 random directions, relative error <= 1e-6 each."""
    import torch
    import mlegs_b200 as M
    from mlegs_b200.adjoint import DeviceAB2, gradient, objective_of, ref_to_dev
    from mlegs_b200.checkpoint import LoopStats
    from mlegs_b200.inputs import CONFIGS, perturbation_coefficients
    cfg = CONFIGS["grad_96x64x64"]
    ctx = M.Context(cfg)
    try:
        solver = DeviceAB2(ctx)
        cs = [ref_to_dev(perturbation_coefficients(cfg, i)) for i in range(3)]
        stats = LoopStats()
        J, grads = gradient(solver, cs, nsteps=cfg.nsteps, every=20, stats=stats)
        assert stats.checkpoints == 10 and stats.recomputed_steps == 190 and stats.vjp_steps == 200
        J_fwd = objective_of(solver, cs, cfg.nsteps)
        assert abs(J_fwd - J) <= 1e-12 * abs(J)  # the step map and the solver's own steps agree
        rng = np.random.default_rng(2024)
        scale = max(float(c.abs().max()) for c in cs)
        h = 1e-5
        worst = 0.0
        for _ in range(32):
            d = [torch.from_numpy((rng.standard_normal(c.shape) + 1j * rng.standard_normal(c.shape)) * scale)
                 for c in cs]
            Jp = objective_of(solver, [c + h * e for c, e in zip(cs, d)], cfg.nsteps)
            Jm = objective_of(solver, [c - h * e for c, e in zip(cs, d)], cfg.nsteps)
            fd = (Jp - Jm) / (2 * h)
            an = sum(float((gq.cpu() * e.conj()).real.sum()) for gq, e in zip(grads, d))
            err = abs(fd - an) / abs(an)
            worst = max(worst, err)
            assert err <= 1e-6, (fd, an, err)
        print("gradient workload: J = %.6e, worst FD relative error over 32 directions %.2e" % (J, worst))
    finally:
        ctx.close()

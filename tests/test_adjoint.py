"""Adjoints of the transform and nonlinear-term maps (oracle/adjoint.py),
checked by the dot-product identity <y, F(x)> = <F^T(y), x> on random inputs
that fill every entry of each space (padding and chopped entries included,
so the projections are checked too), and the product adjoint by central
finite differences."""

import numpy as np
import pytest

from conftest import oracle_grid, small_cfg


def _rand(g, space, seed):
    from oracle.grid import Field
    rng = np.random.default_rng(seed)
    shape = g.shape(space)
    return Field(rng.standard_normal(shape) + 1j * rng.standard_normal(shape), space, float(rng.standard_normal()))


def _dot(a, b):
    return float(np.sum(a.real * b.real + a.imag * b.imag))


def _check(fwd, adj, x, y, with_ln=False):
    fx = fwd(x.copy())
    aty = adj(y)
    lhs = _dot(y.E, fx.E)
    rhs = _dot(aty.E, x.E) + (aty.LN * x.LN if with_ln else 0.0)
    assert abs(lhs - rhs) <= 1e-12 * max(1.0, abs(lhs))


@pytest.mark.parametrize("dims", [(32, 16, 16), (24, 12, 8)])
def test_transform_adjoints(dims):
    from oracle import adjoint as AD
    from oracle import transforms as T
    from oracle.grid import FFF, PFF, PFP, PPP
    g = oracle_grid(small_cfg(*dims))
    cases = [
        (lambda a: T.rtran(g, a, 1), lambda y: AD.rtran_T(g, y, 1), FFF, PFF, True),
        (lambda a: T.rtran(g, a, -1), lambda y: AD.rtran_T(g, y, -1), PFF, FFF, False),
        (lambda a: T.verfft(g, a, 1), lambda y: AD.verfft_T(g, y, 1), PFF, PFP, False),
        (lambda a: T.verfft(g, a, -1), lambda y: AD.verfft_T(g, y, -1), PFP, PFF, False),
        (lambda a: T.horfft(g, a, 1), lambda y: AD.horfft_T(g, y, 1), PFP, PPP, False),
        (lambda a: T.horfft(g, a, -1), lambda y: AD.horfft_T(g, y, -1), PPP, PFP, False),
        (lambda a: T.tofp(g, a), lambda y: AD.tofp_T(g, y), FFF, PPP, True),
        (lambda a: T.toff(g, a), lambda y: AD.toff_T(g, y), PPP, FFF, False),
    ]
    for i, (fwd, adj, sin, sout, ln) in enumerate(cases):
        x = _rand(g, sin, 10 + i)
        if not ln:
            x.LN = 0.0
        y = _rand(g, sout, 50 + i)
        y.LN = 0.0
        _check(fwd, adj, x, y, with_ln=ln)


def test_product_adjoint_matches_finite_differences():
    from oracle import adjoint as AD
    from oracle.grid import PPP
    from oracle.legops import vprodsub
    g = oracle_grid(small_cfg(24, 12, 8))
    U = [_rand(g, PPP, 100 + q) for q in range(3)]
    W = [_rand(g, PPP, 200 + q) for q in range(3)]
    Y = [_rand(g, PPP, 300 + q).E for q in range(3)]

    def J(Us, Ws):
        Wc = [w.copy() for w in Ws]
        vprodsub(g, *[u.copy() for u in Us], *Wc)
        sl = (slice(0, g.NR), slice(0, g.NTH), slice(None))
        return sum(_dot(Y[q][sl], Wc[q].E[sl]) for q in range(3))

    ub, wb = AD.vprodsub_T(g, [u.E for u in U], [w.E for w in W], Y)
    rng = np.random.default_rng(7)
    for _ in range(3):
        du = [_rand(g, PPP, int(rng.integers(1 << 30))) for _ in range(3)]
        dw = [_rand(g, PPP, int(rng.integers(1 << 30))) for _ in range(3)]
        h = 1e-6
        Up = [type(u)(u.E + h * d.E, PPP, 0.0) for u, d in zip(U, du)]
        Um = [type(u)(u.E - h * d.E, PPP, 0.0) for u, d in zip(U, du)]
        Wp = [type(w)(w.E + h * d.E, PPP, 0.0) for w, d in zip(W, dw)]
        Wm = [type(w)(w.E - h * d.E, PPP, 0.0) for w, d in zip(W, dw)]
        fd = (J(Up, Wp) - J(Um, Wm)) / (2 * h)
        an = sum(_dot(ub[q], du[q].E) + _dot(wb[q], dw[q].E) for q in range(3))
        assert abs(fd - an) <= 1e-6 * max(1.0, abs(an))


@pytest.mark.parametrize("dims", [(32, 16, 16), (24, 12, 8)])
def test_operator_adjoints(dims):
    """MULXM, XXDX, DELSQH, DEL2 (log-term rows included), GRAD, PC2VEL and
    PC2VOR against their transposes."""
    from oracle import adjoint as AD
    from oracle import legops as LO
    from oracle.grid import FFF
    g = oracle_grid(small_cfg(*dims))
    unary = [(LO.mulxm, AD.mulxm_T, False), (LO.xxdx, AD.xxdx_T, True),
             (LO.delsqh, AD.delsqh_T, True), (LO.del2, AD.del2_T, True)]
    for i, (f, ft, ln) in enumerate(unary):
        x = _rand(g, FFF, 400 + i)
        if not ln:
            x.LN = 0.0
        y = _rand(g, FFF, 500 + i)
        fx = f(g, x.copy())
        at = ft(g, y)
        lhs = _dot(y.E, fx.E)
        rhs = _dot(at.E, x.E) + at.LN * x.LN
        assert abs(lhs - rhs) <= 1e-12 * max(1.0, abs(lhs)), f.__name__
    # GRAD: one input, three outputs
    x = _rand(g, FFF, 600)
    ys = [_rand(g, FFF, 610 + q) for q in range(3)]
    outs = LO.grad(g, x.copy())
    at = AD.grad_T(g, *ys)
    lhs = sum(_dot(y.E, o.E) for y, o in zip(ys, outs))
    assert abs(lhs - (_dot(at.E, x.E) + at.LN * x.LN)) <= 1e-12 * max(1.0, abs(lhs))
    # PC2VEL / PC2VOR: two inputs, three outputs
    for f, ft, s0 in ((LO.pc2vel, AD.pc2vel_T, 700), (LO.pc2vor, AD.pc2vor_T, 800)):
        p, c = _rand(g, FFF, s0), _rand(g, FFF, s0 + 1)
        ys = [_rand(g, FFF, s0 + 10 + q) for q in range(3)]
        outs = f(g, p.copy(), c.copy())
        pb, cb = ft(g, *ys)
        lhs = sum(_dot(y.E, o.E) for y, o in zip(ys, outs))
        rhs = _dot(pb.E, p.E) + pb.LN * p.LN + _dot(cb.E, c.E) + cb.LN * c.LN
        assert abs(lhs - rhs) <= 1e-12 * max(1.0, abs(lhs)), f.__name__


def test_vdotpsub_and_project_adjoints():
    """VDOTPSUB (finite differences) and PROJECT of PFF inputs with the
    far-field fix (dot product)."""
    from oracle import adjoint as AD
    from oracle import legops as LO
    from oracle.grid import FFF, PFF, PPP
    g = oracle_grid(small_cfg(32, 16, 16))
    A = [_rand(g, PPP, 900 + q).E for q in range(3)]
    B = [_rand(g, PPP, 910 + q).E for q in range(3)]
    Y = _rand(g, PPP, 920).E
    sl = (slice(0, g.NR), slice(0, g.NTH), slice(None))

    def J(As, Bs):
        from oracle.grid import Field
        out = LO.vdotpsub(g, *[Field(a, PPP, 0.0) for a in As], *[Field(b, PPP, 0.0) for b in Bs])
        return _dot(Y[sl], out[sl])

    ab, bb = AD.vdotpsub_T(g, A, B, Y)
    rng = np.random.default_rng(3)
    da = [rng.standard_normal(A[0].shape) + 1j * rng.standard_normal(A[0].shape) for _ in range(3)]
    db = [rng.standard_normal(A[0].shape) + 1j * rng.standard_normal(A[0].shape) for _ in range(3)]
    h = 1e-6
    fd = (J([a + h * d for a, d in zip(A, da)], [b + h * d for b, d in zip(B, db)])
          - J([a - h * d for a, d in zip(A, da)], [b - h * d for b, d in zip(B, db)])) / (2 * h)
    an = sum(_dot(ab[q], da[q]) + _dot(bb[q], db[q]) for q in range(3))
    assert abs(fd - an) <= 1e-6 * max(1.0, abs(an))
    # PROJECT of PFF inputs: three inputs, two outputs
    xs = [_rand(g, PFF, 930 + q) for q in range(3)]
    for x in xs:
        x.LN = 0.0
        x.E[g.NR:] = 0.0          # PFF padding rows do not take part
    ys = [_rand(g, FFF, 940 + q) for q in range(2)]
    P, C = LO.project(g, *[x.copy() for x in xs])
    lhs = _dot(ys[0].E, P.E) + _dot(ys[1].E, C.E)
    bars = AD.project_T(g, *ys)
    rhs = sum(_dot(b.E, x.E) for b, x in zip(bars, xs))
    assert abs(lhs - rhs) <= 1e-12 * max(1.0, abs(lhs))


def test_idel2ln_adjoint():
    """IDEL2LN as B -> (A, A%LN) against its transpose (dot product, log term
    and far-field fix included)."""
    from oracle import adjoint as AD
    from oracle import legops as LO
    from oracle.grid import FFF
    g = oracle_grid(small_cfg(32, 16, 16))
    x = _rand(g, FFF, 960)
    x.LN = 0.0
    y = _rand(g, FFF, 961)
    A = LO.idel2ln(g, x.copy())
    lhs = _dot(y.E, A.E) + y.LN * A.LN
    bt = AD.idel2ln_T(g, y)
    rhs = _dot(bt.E, x.E)
    assert abs(lhs - rhs) <= 1e-10 * max(1.0, abs(lhs))


def test_idel2_and_vel2pln_adjoints():
    from oracle import adjoint as AD
    from oracle import legops as LO
    from oracle.grid import FFF, PFF
    g = oracle_grid(small_cfg(32, 16, 16))
    x = _rand(g, FFF, 970)
    x.LN = 0.0
    y = _rand(g, FFF, 971)
    y.LN = 0.0
    A = LO.idel2(g, x.copy())
    lhs = _dot(y.E, A.E)
    assert abs(lhs - _dot(AD.idel2_T(g, y).E, x.E)) <= 1e-10 * max(1.0, abs(lhs))
    # VEL2PLN with LN given: the update of RUP is linear in RUP
    r = _rand(g, PFF, 972)
    r.E[g.NR:] = 0.0
    yb = _rand(g, PFF, 973)
    yb.E[g.NR:] = 0.0
    rr = r.copy()
    P = g.alloc(FFF)
    LO.vel2pln(g, rr, P, 0.0)
    lhs = _dot(yb.E, rr.E)
    assert abs(lhs - _dot(AD.vel2pln_T(g, yb).E, r.E)) <= 1e-12 * max(1.0, abs(lhs))


def test_boussi_nonlin_vjp_matches_finite_differences():
    """The whole nonlinear term of the ETD step (GRAD, TOFP, VPRODSUB,
    VDOTPSUB, PROJECT with VEL2PLN, IDEL2, PC2VEL, TOFF) against central
    differences of the oracle's CALC_BOUSSI_NONLIN along random directions."""
    from oracle import adjoint as AD
    from oracle.boussinesq import calc_boussi_nonlin
    from oracle.grid import FFF
    g = oracle_grid(small_cfg(24, 12, 8, adams=False))

    def rnd(seed, ln=True):
        F = _rand(g, FFF, seed)
        g.chopdo(F)
        F.E *= 0.1
        if not ln:
            F.LN = 0.0
        return F

    X = [rnd(1000, ln=False)] + [rnd(1001 + q) for q in range(6)]
    Y = [rnd(1100 + q, ln=False) for q in range(4)]

    def J(Xs):
        outs = calc_boussi_nonlin(g, *[F.copy() for F in Xs])
        return sum(_dot(y.E, o.E) for y, o in zip(Y, outs))

    bars = AD.boussi_nonlin_vjp(g, *X, *Y)
    rng = np.random.default_rng(5)
    for _ in range(2):
        D = [rnd(int(rng.integers(1 << 30)), ln=(q > 0)) for q in range(7)]
        h = 1e-5

        def shift(s):
            out = []
            for x, d in zip(X, D):
                F = x.copy()
                F.E = x.E + s * h * d.E
                F.LN = x.LN + s * h * d.LN
                out.append(F)
            return out

        fd = (J(shift(1)) - J(shift(-1))) / (2 * h)
        an = sum(_dot(b.E, d.E) + b.LN * d.LN for b, d in zip(bars, D))
        assert abs(fd - an) <= 1e-6 * max(1.0, abs(an)), (fd, an)


def test_etd_step_vjp_matches_finite_differences():
    """One steady ETD2AB-CN step of the oracle (PC2VEL, PC2VOR, the nonlinear
    term, HYPERV3 filters, CALC_BOUSSI_ETDAB_SUB, PROJECT with the extracted
    log term, IDEL2LN, the history update) as a map of the whole state:
    its VJP against central differences along random directions."""
    import copy
    from oracle import adjoint as AD
    from oracle import boussinesq as BQ
    from oracle import layout
    from oracle.grid import FFF
    from conftest import oracle_physics
    from mlegs_b200.inputs import perturbation_coefficients
    cfg = small_cfg(24, 12, 8, adams=False, nup=0.3, kappap=0.3)
    g = oracle_grid(cfg)
    P, C, B = layout.initial_state(g, *[perturbation_coefficients(cfg, i) for i in range(3)])
    s = BQ.Solver(g, oracle_physics(cfg), P, C, B)
    s.initialize()
    s.step()
    keys = ("psi", "chi", "b") + AD.HISTORY

    def get(sv, k):
        return getattr(sv, k)

    def run(state):
        s2 = copy.deepcopy(s)
        for k in keys:
            setattr(s2, k, state[k].copy())
        s2._step_etdab_cn()
        return {k: get(s2, k) for k in keys}

    rng = np.random.default_rng(21)

    def rnd(ln):
        F = _rand(g, FFF, int(rng.integers(1 << 30)))
        g.chopdo(F)
        F.LN = F.LN if ln else 0.0
        return F

    Y = {k: rnd(k in ("psi", "chi")) for k in keys}
    x0 = {k: get(s, k).copy() for k in keys}

    def J(state):
        out = run(state)
        return sum(_dot(Y[k].E, out[k].E) + (Y[k].LN * out[k].LN if k in ("psi", "chi") else 0.0) for k in keys)

    bars = AD.etdab_cn_step_vjp(s, Y)
    scale = max(np.abs(x0[k].E).max() for k in keys)
    for _ in range(2):
        D = {k: rnd(k in ("psi", "chi")) for k in keys}
        h = 1e-6 * scale

        def shifted(sg):
            st = {}
            for k in keys:
                F = x0[k].copy()
                F.E = F.E + sg * h * D[k].E
                F.LN = F.LN + sg * h * D[k].LN
                st[k] = F
            return st

        fd = (J(shifted(1)) - J(shifted(-1))) / (2 * h)
        an = sum(_dot(bars[k].E, D[k].E) + (bars[k].LN * D[k].LN if k in ("psi", "chi") else 0.0) for k in keys)
        assert abs(fd - an) <= 1e-6 * max(1.0, abs(an)), (fd, an)


def test_trajectory_gradient_matches_finite_differences():
    """Gradient of J = 1/2 |b|^2 + 1/2 |psi|^2 + 1/2 psi%LN^2 after three ETD
    steps with respect to the whole initial state (reverse accumulation of
    the step VJPs) against central differences: <= 1e-6 relative."""
    import copy
    from oracle import adjoint as AD
    from oracle import boussinesq as BQ
    from oracle import layout
    from oracle.grid import FFF, Field
    from conftest import oracle_physics
    from mlegs_b200.inputs import perturbation_coefficients
    cfg = small_cfg(24, 12, 8, adams=False, nup=0.3, kappap=0.3)
    g = oracle_grid(cfg)
    P, C, B = layout.initial_state(g, *[perturbation_coefficients(cfg, i) for i in range(3)])
    s = BQ.Solver(g, oracle_physics(cfg), P, C, B)
    s.initialize()
    s.step()
    n = 3

    def objective(st):
        return 0.5 * (_dot(st["b"].E, st["b"].E) + _dot(st["psi"].E, st["psi"].E) + st["psi"].LN ** 2)

    def objective_grad(st):
        bars = {k: Field(np.zeros(g.shape(FFF), dtype=np.complex128), FFF, 0.0) for k in AD.STATE}
        bars["b"] = Field(st["b"].E.copy(), FFF, 0.0)
        bars["psi"] = Field(st["psi"].E.copy(), FFF, st["psi"].LN)
        return bars

    grad = AD.etd_trajectory_grad(s, n, objective_grad)

    def J(state):
        s2 = copy.deepcopy(s)
        for k in AD.STATE:
            setattr(s2, k, state[k].copy())
        for _ in range(n):
            s2._step_etdab_cn()
        return objective({k: getattr(s2, k) for k in AD.STATE})

    x0 = {k: getattr(s, k).copy() for k in AD.STATE}
    rng = np.random.default_rng(8)
    for _ in range(2):
        D = {}
        for k in AD.STATE:
            F = _rand(g, FFF, int(rng.integers(1 << 30)))
            g.chopdo(F)
            F.E *= np.abs(x0[k].E).max() + 1e-30
            F.LN = F.LN * abs(x0[k].LN) if k in ("psi", "chi") else 0.0
            D[k] = F
        h = 1e-6

        def shifted(sg):
            out = {}
            for k in AD.STATE:
                F = x0[k].copy()
                F.E = F.E + sg * h * D[k].E
                F.LN = F.LN + sg * h * D[k].LN
                out[k] = F
            return out

        fd = (J(shifted(1)) - J(shifted(-1))) / (2 * h)
        an = sum(_dot(grad[k].E, D[k].E) + (grad[k].LN * D[k].LN if k in ("psi", "chi") else 0.0)
                 for k in AD.STATE)
        assert abs(fd - an) <= 1e-6 * max(1e-12, abs(an)), (fd, an)


def test_ab2_step_vjp_matches_finite_differences():
    """One steady AB2-CN step (CALC_BOUSSI_FORCE with the linear terms, the
    AB2 update, VISC2 with IHELM for psi, chi and b) as a map of
    (psi, chi, b, n_psi, n_chi, n_b): its VJP against central differences."""
    import copy
    from oracle import adjoint as AD
    from oracle import boussinesq as BQ
    from oracle import layout
    from oracle.grid import FFF
    from conftest import oracle_physics
    from mlegs_b200.inputs import perturbation_coefficients
    cfg = small_cfg(24, 12, 8, adams=True)
    g = oracle_grid(cfg)
    P, C, B = layout.initial_state(g, *[perturbation_coefficients(cfg, i) for i in range(3)])
    s = BQ.Solver(g, oracle_physics(cfg), P, C, B)
    s.initialize()
    s.step()
    keys = AD.AB2_STATE
    lnk = ("psi", "chi", "n_psi", "n_chi")
    rng = np.random.default_rng(31)

    def rnd(ln):
        F = _rand(g, FFF, int(rng.integers(1 << 30)))
        g.chopdo(F)
        F.LN = F.LN if ln else 0.0
        return F

    Y = {k: rnd(k in lnk) for k in keys}
    x0 = {k: getattr(s, k).copy() for k in keys}

    def J(state):
        s2 = copy.deepcopy(s)
        for k in keys:
            setattr(s2, k, state[k].copy())
        s2._step_ab_cn()
        return sum(_dot(Y[k].E, getattr(s2, k).E) + (Y[k].LN * getattr(s2, k).LN if k in lnk else 0.0)
                   for k in keys)

    bars = AD.ab_cn_step_vjp(s, Y)
    for _ in range(2):
        D = {k: rnd(k in lnk) for k in keys}
        for k in keys:
            D[k].E *= np.abs(x0[k].E).max() + 1e-30
        h = 1e-6

        def shifted(sg):
            out = {}
            for k in keys:
                F = x0[k].copy()
                F.E = F.E + sg * h * D[k].E
                F.LN = F.LN + sg * h * D[k].LN
                out[k] = F
            return out

        fd = (J(shifted(1)) - J(shifted(-1))) / (2 * h)
        an = sum(_dot(bars[k].E, D[k].E) + (bars[k].LN * D[k].LN if k in lnk else 0.0) for k in keys)
        assert abs(fd - an) <= 1e-6 * max(1e-12, abs(an)), (fd, an)


def test_ab2_trajectory_gradient_matches_finite_differences():
    """The objective of the ETD test after three AB2-CN steps (the stepper of
    the gradient configuration), reverse accumulation against central
    differences."""
    import copy
    from oracle import adjoint as AD
    from oracle import boussinesq as BQ
    from oracle import layout
    from oracle.grid import FFF, Field
    from conftest import oracle_physics
    from mlegs_b200.inputs import perturbation_coefficients
    cfg = small_cfg(24, 12, 8, adams=True)
    g = oracle_grid(cfg)
    P, C, B = layout.initial_state(g, *[perturbation_coefficients(cfg, i) for i in range(3)])
    s = BQ.Solver(g, oracle_physics(cfg), P, C, B)
    s.initialize()
    n = 3
    keys = AD.AB2_STATE

    def objective(st):
        return 0.5 * (_dot(st["b"].E, st["b"].E) + _dot(st["psi"].E, st["psi"].E) + st["psi"].LN ** 2)

    def objective_grad(st):
        bars = {k: Field(np.zeros(g.shape(FFF), dtype=np.complex128), FFF, 0.0) for k in keys}
        bars["b"] = Field(st["b"].E.copy(), FFF, 0.0)
        bars["psi"] = Field(st["psi"].E.copy(), FFF, st["psi"].LN)
        return bars

    grad = AD.trajectory_grad(s, n, objective_grad)

    def J(state):
        s2 = copy.deepcopy(s)
        for k in keys:
            setattr(s2, k, state[k].copy())
        for _ in range(n):
            s2._step_ab_cn()
        return objective({k: getattr(s2, k) for k in keys})

    x0 = {k: getattr(s, k).copy() for k in keys}
    rng = np.random.default_rng(12)
    D = {}
    for k in keys:
        F = _rand(g, FFF, int(rng.integers(1 << 30)))
        g.chopdo(F)
        F.E *= np.abs(x0[k].E).max() + 1e-30
        F.LN = F.LN * abs(x0[k].LN) if k in ("psi", "chi", "n_psi", "n_chi") else 0.0
        D[k] = F
    h = 1e-6

    def shifted(sg):
        out = {}
        for k in keys:
            F = x0[k].copy()
            F.E = F.E + sg * h * D[k].E
            F.LN = F.LN + sg * h * D[k].LN
            out[k] = F
        return out

    fd = (J(shifted(1)) - J(shifted(-1))) / (2 * h)
    an = sum(_dot(grad[k].E, D[k].E) + grad[k].LN * D[k].LN for k in keys)
    assert abs(fd - an) <= 1e-6 * max(1e-12, abs(an)), (fd, an)


def test_energy_objective_gradient():
    """The gradient configuration's objective (fluctuation kinetic energy plus
    1/2 int b^2) and its gradient against central differences."""
    from oracle import adjoint as AD
    from oracle.grid import FFF
    g = oracle_grid(small_cfg(24, 12, 8))
    rng = np.random.default_rng(41)

    def rnd():
        F = _rand(g, FFF, int(rng.integers(1 << 30)))
        g.chopdo(F)
        return F

    x = [rnd(), rnd(), rnd()]
    x[2].LN = 0.0
    grads = AD.energy_objective_grad(g, *x)
    for _ in range(2):
        d = [rnd(), rnd(), rnd()]
        d[2].LN = 0.0
        h = 1e-6

        def J(sg):
            xs = []
            for a, b in zip(x, d):
                F = a.copy()
                F.E = a.E + sg * h * b.E
                F.LN = a.LN + sg * h * b.LN
                xs.append(F)
            return AD.energy_objective(g, *xs)

        fd = (J(1) - J(-1)) / (2 * h)
        an = sum(_dot(G.E, b.E) + G.LN * b.LN for G, b in zip(grads, d))
        assert abs(fd - an) <= 1e-6 * max(1.0, abs(an)), (fd, an)


def test_energy_objective_trajectory_gradient():
    """J = fluctuation KE + 1/2 int b^2 after three AB2-CN steps: reverse
    accumulation against central differences."""
    import copy
    from oracle import adjoint as AD
    from oracle import boussinesq as BQ
    from oracle import layout
    from oracle.grid import FFF, Field
    from conftest import oracle_physics
    from mlegs_b200.inputs import perturbation_coefficients
    cfg = small_cfg(24, 12, 8, adams=True)
    g = oracle_grid(cfg)
    P, C, B = layout.initial_state(g, *[perturbation_coefficients(cfg, i) for i in range(3)])
    s = BQ.Solver(g, oracle_physics(cfg), P, C, B)
    s.initialize()
    keys = AD.AB2_STATE
    n = 3

    def objective_grad(st):
        gp, gc, gb = AD.energy_objective_grad(g, st["psi"], st["chi"], st["b"])
        bars = {k: Field(np.zeros(g.shape(FFF), dtype=np.complex128), FFF, 0.0) for k in keys}
        bars["psi"], bars["chi"], bars["b"] = gp, gc, gb
        return bars

    grad = AD.trajectory_grad(s, n, objective_grad)

    def J(state):
        s2 = copy.deepcopy(s)
        for k in keys:
            setattr(s2, k, state[k].copy())
        for _ in range(n):
            s2._step_ab_cn()
        return AD.energy_objective(g, s2.psi, s2.chi, s2.b)

    x0 = {k: getattr(s, k).copy() for k in keys}
    rng = np.random.default_rng(77)
    D = {}
    for k in keys:
        F = _rand(g, FFF, int(rng.integers(1 << 30)))
        g.chopdo(F)
        F.E *= np.abs(x0[k].E).max() + 1e-30
        F.LN = F.LN * abs(x0[k].LN) if k in ("psi", "chi", "n_psi", "n_chi") else 0.0
        D[k] = F
    h = 1e-6

    def shifted(sg):
        out = {}
        for k in keys:
            F = x0[k].copy()
            F.E = F.E + sg * h * D[k].E
            F.LN = F.LN + sg * h * D[k].LN
            out[k] = F
        return out

    fd = (J(shifted(1)) - J(shifted(-1))) / (2 * h)
    an = sum(_dot(grad[k].E, D[k].E) + grad[k].LN * D[k].LN for k in keys)
    assert abs(fd - an) <= 1e-6 * max(1e-12, abs(an)), (fd, an)


def test_gradient_wrt_perturbation_coefficients():
    """The gradient configuration end to end in the oracle: J = fluctuation KE
    + 1/2 int b^2 after the Richardson start-up and two AB2-CN steps, with
    respect to the seeded perturbation coefficients (c_psi, c_chi, c_b),
    against central differences."""
    import copy
    from oracle import adjoint as AD
    from oracle import boussinesq as BQ
    from oracle import layout
    from oracle.grid import FFF, Field
    from conftest import oracle_physics
    from mlegs_b200.inputs import perturbation_coefficients
    cfg = small_cfg(24, 12, 8, adams=True)
    g = oracle_grid(cfg)
    ph = oracle_physics(cfg)
    cs = [perturbation_coefficients(cfg, i) for i in range(3)]
    n = 2

    def run(c):
        P, C, B = layout.initial_state(g, *c)
        s = BQ.Solver(g, ph, P, C, B)
        s.initialize()
        traj = [s]
        for _ in range(n):
            s2 = copy.deepcopy(traj[-1])
            s2._step_ab_cn()
            traj.append(s2)
        return P, C, B, traj

    def J(c):
        return AD.energy_objective(g, *[getattr(run(c)[3][-1], k) for k in ("psi", "chi", "b")])

    P, C, B, traj = run(cs)
    keys = AD.AB2_STATE

    def objective_grad(st):
        gp, gc, gb = AD.energy_objective_grad(g, st["psi"], st["chi"], st["b"])
        bars = {k: Field(np.zeros(g.shape(FFF), dtype=np.complex128), FFF, 0.0) for k in keys}
        bars["psi"], bars["chi"], bars["b"] = gp, gc, gb
        return bars

    bars = AD.trajectory_grad(traj[0], n, objective_grad)
    s0 = BQ.Solver(g, ph, P.copy(), C.copy(), B.copy())
    x0_bar = AD.rich_fe_be_vjp(s0, bars)
    c_bar = AD.initial_state_T(g, x0_bar["psi"], x0_bar["chi"], x0_bar["b"])
    rng = np.random.default_rng(99)
    for _ in range(2):
        d = [(rng.standard_normal(c.shape) + 1j * rng.standard_normal(c.shape)) * np.abs(c).max() for c in cs]
        h = 1e-6
        fd = (J([c + h * e for c, e in zip(cs, d)]) - J([c - h * e for c, e in zip(cs, d)])) / (2 * h)
        an = sum(_dot(cb, e) for cb, e in zip(c_bar, d))
        assert abs(fd - an) <= 1e-6 * max(1e-12, abs(an)), (fd, an)


def test_etd_startup_vjp_matches_finite_differences():
    """The ETD2AB-CN Richardson start-up (two half ETDFE steps against one full
    step, with the history it stores) as a map of (psi, chi, b): its VJP
    against central differences."""
    import copy
    from oracle import adjoint as AD
    from oracle import boussinesq as BQ
    from oracle import layout
    from oracle.grid import FFF
    from conftest import oracle_physics
    from mlegs_b200.inputs import perturbation_coefficients
    cfg = small_cfg(24, 12, 8, adams=False, nup=0.3, kappap=0.3)
    g = oracle_grid(cfg)
    P, C, B = layout.initial_state(g, *[perturbation_coefficients(cfg, i) for i in range(3)])
    s0 = BQ.Solver(g, oracle_physics(cfg), P, C, B)
    s0.etd_e, s0.etd_nl = BQ.calc_boussi_etd_op(cfg.bv0, cfg.omega, cfg.dt)   # as INITIALIZE sets them
    keys = AD.STATE
    ins = ("psi", "chi", "b")
    rng = np.random.default_rng(55)

    def rnd(ln):
        F = _rand(g, FFF, int(rng.integers(1 << 30)))
        g.chopdo(F)
        F.LN = F.LN if ln else 0.0
        return F

    Y = {k: rnd(k in ("psi", "chi")) for k in keys}

    def J(state):
        s2 = copy.deepcopy(s0)
        for k in ins:
            setattr(s2, k, state[k].copy())
        s2._rich_etdfe_be()
        return sum(_dot(Y[k].E, getattr(s2, k).E) + (Y[k].LN * getattr(s2, k).LN if k in ("psi", "chi") else 0.0)
                   for k in keys)

    bars = AD.rich_etdfe_be_vjp(s0, Y)
    x0 = {k: getattr(s0, k).copy() for k in ins}
    for _ in range(2):
        D = {k: rnd(k in ("psi", "chi")) for k in ins}
        for k in ins:
            D[k].E *= np.abs(x0[k].E).max()
        h = 1e-6

        def shifted(sg):
            out = {}
            for k in ins:
                F = x0[k].copy()
                F.E = F.E + sg * h * D[k].E
                F.LN = F.LN + sg * h * D[k].LN
                out[k] = F
            return out

        fd = (J(shifted(1)) - J(shifted(-1))) / (2 * h)
        an = sum(_dot(bars[k].E, D[k].E) + bars[k].LN * D[k].LN for k in ins)
        assert abs(fd - an) <= 1e-6 * max(1e-12, abs(an)), (fd, an)

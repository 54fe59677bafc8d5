"""Adaptive hyperviscosity (HYP3ADJ, mod_march.f90:2585-3182).

CPU: the host-side spectrum metrics and controller of the library (SPECURV,
SPESLOP, PDAJUST through the C ABI, no device) against the oracle's
restatement, with the reference's fallbacks, clamps and floors.
GPU: ENEMON, HYP3ADJ and ETD steps before and after the table update.
"""

import numpy as np
import pytest

from conftest import oracle_grid, oracle_physics, random_fff, rel, small_cfg


@pytest.fixture(scope="module")
def env(lib_built):
    import mlegs_b200 as M
    cfg = small_cfg(32, 16, 16)
    ctx = M.Context(cfg)
    yield M, ctx, oracle_grid(cfg), cfg
    ctx.close()


def up(ctx, F):
    f = ctx.field(F.space)
    f.upload(F.E, F.LN, F.space)
    return f


def _spectra():
    rng = np.random.default_rng(7)
    out = []
    for n in (3, 9, 12, 30, 61, 85):
        k = np.arange(1, n + 1, dtype=float)
        out.append(np.exp(rng.standard_normal(n) * 0.3) * k ** -3.0)            # power law
        out.append(np.exp(-0.3 * k + 0.2 * rng.standard_normal(n)))             # exponential
    tail = np.exp(-0.3 * np.arange(1, 41.0))
    tail[-6:] = 1e-30                                                          # below both floors
    out.append(tail)
    out.append(np.full(40, 1e-30))
    return out


def test_spectrum_metrics_match_oracle(lib_built):
    import mlegs_b200 as M
    from oracle import hyperadj as H
    for e in _spectra():
        for r in (0.25, 1.0 / 3.0, 0.5):
            assert abs(M.SPECURV(e, r) - H.specurv(e, r)) < 1e-12
            assert abs(M.SPESLOP(e, r) - H.speslop(e, r)) < 1e-12


def test_spectrum_metric_fallbacks(lib_built):
    """Too few points: SPECURV returns the target -0.05, SPESLOP -3; clamps hold."""
    import mlegs_b200 as M
    assert M.SPECURV(np.exp(-np.arange(1, 10.0)), 1.0 / 3.0) == -0.05
    assert M.SPESLOP(np.exp(-np.arange(1, 5.0)), 1.0 / 3.0) == -3.0
    floored = np.exp(-0.3 * np.arange(1, 41.0))
    floored[-6:] = 1e-30
    assert M.SPECURV(floored, 1.0 / 3.0) == -0.05      # more than 20 % of the range under the floor
    for e in _spectra():
        assert -10.0 <= M.SPECURV(e) <= 10.0 and -15.0 <= M.SPESLOP(e) <= 5.0


def test_pdajust_known_answers(lib_built):
    import mlegs_b200 as M
    from oracle import hyperadj as H
    cp = H.CURV_PARAMS
    # control = KP (c - p) + KD c + OFFSET = 0.05, times SCALE 0.8 -> x 1.04
    assert abs(M.PDAJUST(1.0, 0.0, 0.0, 0.5, cp) - 1.04) < 1e-15
    # both below the over-damping threshold: control = -(0.1 + 0.05 * 1) * 0.8
    assert abs(M.PDAJUST(1.0, -2.0, -3.0, 0.5, cp, -1.0) - 0.88) < 1e-15
    # clamps of SCALE * CONTROL to [-0.4, 1] and the floor at BASELINE
    assert abs(M.PDAJUST(1.0, 10.0, 0.0, 0.5, cp) - 2.0) < 1e-15
    assert abs(M.PDAJUST(1.0, -10.0, 0.0, 0.5, cp) - 0.6) < 1e-15
    assert M.PDAJUST(1.0, -10.0, 0.0, 0.9, cp) == 0.9
    rng = np.random.default_rng(3)
    for _ in range(200):
        c, cur, prev, base = rng.uniform(0.1, 3), rng.normal(0, 2), rng.normal(0, 2), rng.uniform(0, 1)
        thr = None if rng.uniform() < 0.5 else -1.0
        for prm in (H.CURV_PARAMS, H.SLOPE_PARAMS):
            assert abs(M.PDAJUST(c, cur, prev, base, prm, thr) - H.pdajust(c, cur, prev, base, prm, thr)) < 1e-14


def test_hyp3_controller_sequence_matches_oracle(lib_built):
    """The library's HYP3ADJ controller (host code) against the oracle over a
    sequence of calls with evolving history: spectra from shallow to steep
    power laws with noise, so the curvature, slope, over-damping and clamp
    branches all occur."""
    import mlegs_b200 as M
    from oracle import hyperadj as H
    rng = np.random.default_rng(11)
    state = np.array([-1.0, 0.0, 0.0, 0.0, 0.0])
    coef = np.array([0.3, 0.3, 0.3])
    nupb, hist, ref = -1.0, [0.0] * 4, [0.3, 0.3, 0.3]
    for step, p in enumerate((1.0, 2.5, 4.0, 6.0, 9.0, 3.0, 0.5, 12.0)):
        em = np.arange(1, 84, dtype=float) ** -p * np.exp(0.3 * rng.standard_normal(83))
        ek = np.arange(1, 86, dtype=float) ** -(p + 0.5) * np.exp(0.3 * rng.standard_normal(85))
        state, coef = M.HYP3_CONTROLLER(em, ek, state, coef)
        met = H.Hyp3Adj._metrics(em, ek)
        if nupb < 0.0:
            hist, nupb = list(met), H.BASELINE_NUP
        ref = H.Hyp3Adj._control(ref, met, hist, nupb)
        hist = list(met)
        assert np.abs(coef - np.array(ref)).max() < 1e-12 * max(1.0, np.abs(ref).max()), step
        assert np.abs(state[1:] - np.array(hist)).max() < 1e-12 and state[0] == nupb
        assert coef.min() >= nupb and coef[0] <= 2.0


def test_hyp3adj_controller_first_call():
    """First HYP3ADJ: the history takes the current metrics, NUPB = 0.8 and every
    coefficient ends at or above it, NUP_R at most 2."""
    from oracle import hyperadj as H
    from oracle.boussinesq import Hyperv3
    from oracle import layout
    from mlegs_b200.inputs import perturbation_coefficients
    cfg = small_cfg(32, 16, 16, adams=False, nup=0.3, kappap=0.3, p=4)
    g = oracle_grid(cfg)
    ph = oracle_physics(cfg)
    P, C, B = layout.initial_state(g, *[perturbation_coefficients(cfg, i) for i in range(3)])
    hyp = Hyperv3(g, ph)
    adj = H.Hyp3Adj()
    em, ek = adj.adjust(g, ph, hyp, P, C, B)
    assert em.shape == (g.NTCHOP,) and ek.shape == (g.NXCHOP,)
    assert adj.nupb == 0.8 and adj.kappapb == 0.8
    for coef in (hyp.nup, hyp.kappap):
        assert all(c >= 0.8 for c in coef) and coef[0] <= 2.0
    hv = hyp._set(g, ph, *hyp.nup)
    for a, b in zip(hv, hyp.hv):
        assert np.array_equal(a, b)


@pytest.mark.gpu
@pytest.mark.parametrize("pad", [0, 2])
def test_enemon(env, pad):
    from oracle import hyperadj as H
    M, ctx, g, cfg = env
    PSI, CHI = (random_fff(g, 80 + i, decay=4.0) for i in range(2))
    PSI.LN, CHI.LN = 0.3, -0.2
    em, ek = ctx.ENEMON(up(ctx, PSI), up(ctx, CHI), pad)
    g.chopset(pad)
    try:
        EM, EK = H.enemon(g, PSI, CHI)
    finally:
        g.chopset(-pad)
    assert rel(em, EM) < 1e-12 and rel(ek, EK) < 1e-12


@pytest.mark.gpu
@pytest.mark.parametrize("graph", [False, True], ids=["eager", "graph"])
def test_hyp3adj_steps(lib_built, graph):
    """ETD steps, HYP3ADJ (with B) on the device and in the oracle, then more
    steps: the coefficients agree and the steps (the captured graph included)
    use the rewritten HYPERV / HYPERD tables."""
    import mlegs_b200 as M
    from oracle import boussinesq as BQ
    from oracle import hyperadj as H
    from oracle import layout
    from mlegs_b200.inputs import perturbation_coefficients
    cfg = small_cfg(32, 16, 16, adams=False, nup=0.3, kappap=0.3, p=4)
    g = oracle_grid(cfg)
    ph = oracle_physics(cfg)
    P, C, B = layout.initial_state(g, *[perturbation_coefficients(cfg, i) for i in range(3)])
    s = BQ.Solver(g, ph, P, C, B)
    s.initialize()
    for _ in range(2):
        s.step()
    adj = H.Hyp3Adj()
    adj.adjust(g, ph, s.hyp, s.psi, s.chi, s.b)
    for _ in range(3):
        s.step()
    ctx = M.Context(cfg)
    fp, fc, fb = M.initial_state(ctx)
    ctx.initialize(fp, fc, fb)
    ctx.step(2, graph=graph)
    nup0, kap0 = ctx.hyp3_coeffs()
    assert nup0 == (0.3, 0.3, 0.3) and kap0 == (0.3, 0.3, 0.3)
    ctx.HYP3ADJ(fp, fc, fb)
    nup, kap = ctx.hyp3_coeffs()
    assert rel(np.array(nup), np.array(s.hyp.nup)) < 1e-12
    assert rel(np.array(kap), np.array(s.hyp.kappap)) < 1e-12
    ctx.step(3, graph=graph)
    out = [f.download() for f in (fp, fc, fb)]
    ctx.close()
    for (E, ln), R in zip(out, (s.psi, s.chi, s.b)):
        assert rel(E, R.E) < 1e-10
        assert abs(ln - R.LN) < 1e-10 * max(1.0, abs(R.LN))

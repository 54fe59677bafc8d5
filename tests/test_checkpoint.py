"""Checkpointed differentiation of the time loop (mlegs_b200/checkpoint.py):
the torch.autograd.Function's gradient against plain autograd through the
unrolled loop, against the oracle's full-trajectory reverse accumulation of
the AB2-CN and ETD2AB-CN step VJPs (mod_march.f90:609-661, 811-901), and its recomputation counts
for the gradient configuration's schedule (200 steps, a checkpoint every
20).  All on CPU."""

import copy

import numpy as np
import pytest
import torch

from conftest import oracle_grid, small_cfg
from mlegs_b200.checkpoint import LoopStats, run_loop


class ToyStepper:
    """A small bounded nonlinear map with a complex field and a real scalar,
    the layout of a field with its log term; its VJP comes from torch."""

    def __init__(self, seed=0):
        g = torch.Generator().manual_seed(seed)
        self.A = (torch.randn(6, 6, generator=g, dtype=torch.float64)
                  + 1j * torch.randn(6, 6, generator=g, dtype=torch.float64))
        self.A = self.A * (0.9 / torch.linalg.matrix_norm(self.A, ord=2))
        self.steps = 0

    def _f(self, z, ln):
        self.steps += 1
        a2 = z.real ** 2 + z.imag ** 2
        z2 = self.A @ z + 0.05 * z * a2 / (1 + a2) + 0.01 * ln
        ln2 = 0.9 * ln + 0.02 * torch.tanh((z.real ** 2).sum())
        return z2, ln2

    def step(self, state):
        return self._f(*state)

    def step_vjp(self, state, bars):
        with torch.enable_grad():
            x = tuple(t.detach().requires_grad_() for t in state)
            out = self._f(*x)
            self.steps -= 1
            gr = torch.autograd.grad(out, x, bars, allow_unused=True)
        return tuple(torch.zeros_like(t) if d is None else d for t, d in zip(state, gr))


def _toy_state(seed=1):
    g = torch.Generator().manual_seed(seed)
    z = (torch.randn(6, 3, generator=g, dtype=torch.float64)
         + 1j * torch.randn(6, 3, generator=g, dtype=torch.float64)) * 0.5
    return z, torch.tensor(0.3, dtype=torch.float64)


def _loss(z, ln):
    return 0.5 * (z.abs() ** 2).sum() + ln ** 2 + (z.imag[0] ** 3).sum()


@pytest.mark.parametrize("nsteps,every", [(7, 1), (7, 3), (7, 7), (7, 20), (12, 4)])
def test_checkpointed_gradient_equals_unrolled_autograd(nsteps, every):
    st = ToyStepper()
    z0, l0 = _toy_state()
    # Unrolled loop under autograd.
    z, l = z0.clone().requires_grad_(), l0.clone().requires_grad_()
    a, b = z, l
    for _ in range(nsteps):
        a, b = st._f(a, b)
    gz_ref, gl_ref = torch.autograd.grad(_loss(a, b), (z, l))
    # Checkpointed loop.
    z, l = z0.clone().requires_grad_(), l0.clone().requires_grad_()
    stats = LoopStats()
    a, b = run_loop(st, (z, l), nsteps, every=every, stats=stats)
    gz, gl = torch.autograd.grad(_loss(a, b), (z, l))
    torch.testing.assert_close(gz, gz_ref, rtol=1e-13, atol=1e-14)
    torch.testing.assert_close(gl, gl_ref, rtol=1e-13, atol=1e-14)
    nseg = -(-nsteps // every)
    assert stats.forward_steps == nsteps
    assert stats.checkpoints == nseg
    assert stats.recomputed_steps == nsteps - nseg
    assert stats.vjp_steps == nsteps


def test_gradient_configuration_schedule():
    """200 steps with a checkpoint every 20: 10 checkpoints, 190 steps
    recomputed, 200 VJPs, never more than 30 states held."""
    st = ToyStepper()
    z0, l0 = _toy_state()
    z, l = z0.clone().requires_grad_(), l0.clone().requires_grad_()
    stats = LoopStats()
    a, b = run_loop(st, (z, l), 200, every=20, store="cpu", stats=stats)
    (0.5 * (a.abs() ** 2).sum()).backward()
    assert (stats.checkpoints, stats.recomputed_steps, stats.vjp_steps) == (10, 190, 200)
    assert stats.peak_states <= 30
    assert z.grad is not None and torch.isfinite(z.grad.real).all()
    assert l.grad is not None


def test_unused_outputs_and_zero_steps():
    st = ToyStepper()
    z0, l0 = _toy_state()
    z, l = z0.clone().requires_grad_(), l0.clone().requires_grad_()
    a, _ = run_loop(st, (z, l), 4, every=2)
    (a.real.sum()).backward()          # the scalar output takes no part
    assert l.grad is not None
    z, l = z0.clone().requires_grad_(), l0.clone().requires_grad_()
    a, b = run_loop(st, (z, l), 0, every=2)
    (a.real.sum() + b).backward()
    torch.testing.assert_close(z.grad, torch.ones_like(z0))
    assert float(l.grad) == 1.0


def test_single_backward_pass():
    """A second backward through the same loop (retain_graph) is a clear
    error: the first one released the checkpoints."""
    st = ToyStepper()
    z0, l0 = _toy_state()
    z, l = z0.clone().requires_grad_(), l0.clone().requires_grad_()
    a, b = run_loop(st, (z, l), 5, every=2)
    loss = _loss(a, b)
    loss.backward(retain_graph=True)
    with pytest.raises(RuntimeError, match="single backward pass"):
        loss.backward()


def test_bad_arguments():
    st = ToyStepper()
    z0, l0 = _toy_state()
    with pytest.raises(ValueError):
        run_loop(st, (z0, l0), 3, every=0)
    with pytest.raises(ValueError):
        run_loop(st, (), 3)

    class Bad(ToyStepper):
        def step(self, state):
            return state[:1]
    with pytest.raises(ValueError):
        run_loop(Bad(), (z0, l0), 2, every=1)


class OracleStepper:
    """The oracle's steady step (AB2-CN or ETD2AB-CN, as s.ph.adams says) and
    its VJP on the state (psi, chi, b and the histories), each field as (E,
    LN) tensors; the solver `s` supplies the grid, physics and operators and
    is not changed."""

    def __init__(self, s):
        from oracle import adjoint as AD
        self.s, self.adams = s, s.ph.adams
        self.keys = AD.AB2_STATE if self.adams else AD.STATE

    def _solver(self, state):
        from oracle.grid import FFF, Field
        s2 = copy.deepcopy(self.s)
        for i, k in enumerate(self.keys):
            setattr(s2, k, Field(state[2 * i].numpy().copy(), FFF, float(state[2 * i + 1])))
        return s2

    def _tensors(self, fields):
        out = []
        for k in self.keys:
            out += [torch.from_numpy(np.array(fields[k].E)), torch.tensor(float(fields[k].LN), dtype=torch.float64)]
        return tuple(out)

    def step(self, state):
        s2 = self._solver(state)
        if self.adams:
            s2._step_ab_cn()
        else:
            s2._step_etdab_cn()
        return self._tensors({k: getattr(s2, k) for k in self.keys})

    def step_vjp(self, state, bars):
        from oracle import adjoint as AD
        from oracle.grid import FFF, Field
        s2 = self._solver(state)
        fb = {k: Field(bars[2 * i].numpy().copy(), FFF, float(bars[2 * i + 1])) for i, k in enumerate(self.keys)}
        vjp = AD.ab_cn_step_vjp if self.adams else AD.etdab_cn_step_vjp
        return self._tensors(vjp(s2, fb))


@pytest.mark.parametrize("adams", [True, False], ids=["ab2cn", "etdab2cn"])
def test_checkpointed_gradient_matches_oracle_trajectory(adams):
    """Five steady steps of the oracle stepper (AB2-CN, mod_march.f90:609-661,
    or ETD2AB-CN, 811-901), a checkpoint every 2: the gradient of
    1/2 (|b|^2 + |psi|^2 + LN_psi^2) with respect to the initial state equals
    the oracle's reverse accumulation over the stored trajectory."""
    from oracle import adjoint as AD
    from oracle import boussinesq as BQ
    from oracle import layout
    from oracle.grid import FFF, Field
    from conftest import oracle_physics
    from mlegs_b200.inputs import perturbation_coefficients
    cfg = small_cfg(24, 12, 8, adams=True) if adams else small_cfg(24, 12, 8, adams=False, nup=0.3, kappap=0.3)
    g = oracle_grid(cfg)
    P, C, B = layout.initial_state(g, *[perturbation_coefficients(cfg, i) for i in range(3)])
    s = BQ.Solver(g, oracle_physics(cfg), P, C, B)
    s.initialize()
    if not adams:
        s.step()                       # the ETD start-up fills the history
    stepper = OracleStepper(s)
    n, keys = 5, stepper.keys

    def objective_grad(st):
        bars = {k: Field(np.zeros(g.shape(FFF), dtype=np.complex128), FFF, 0.0) for k in keys}
        bars["b"] = Field(st["b"].E.copy(), FFF, 0.0)
        bars["psi"] = Field(st["psi"].E.copy(), FFF, st["psi"].LN)
        return bars

    ref = AD.trajectory_grad(s, n, objective_grad)

    x0 = tuple(t.requires_grad_() for t in stepper._tensors({k: getattr(s, k) for k in keys}))
    stats = LoopStats()
    out = run_loop(stepper, x0, n, every=2, stats=stats)
    ib, ip = 2 * keys.index("b"), 2 * keys.index("psi")
    loss = 0.5 * ((out[ib].abs() ** 2).sum() + (out[ip].abs() ** 2).sum() + out[ip + 1] ** 2)
    grads = torch.autograd.grad(loss, x0)
    assert (stats.checkpoints, stats.recomputed_steps) == (3, 2)
    for i, k in enumerate(keys):
        gE, gL = grads[2 * i].numpy(), float(grads[2 * i + 1])
        scale = max(1.0, float(np.abs(ref[k].E).max()))
        assert np.abs(gE - ref[k].E).max() <= 1e-13 * scale, k
        assert abs(gL - float(ref[k].LN)) <= 1e-13 * max(1.0, abs(float(ref[k].LN))), k


def test_gradient_configuration_through_checkpointed_loop_32_directions():
    """The gradient configuration's chain at a small grid: seeded perturbation
    coefficients -> initial state (IDELSQH and the far field) -> Richardson
    start-up (RICH_BOUSSI_FE_BE, mod_march.f90:535-606) -> four AB2-CN steps
    through run_loop with a checkpoint every 3 -> J = fluctuation KE +
    1/2 int b^2 (mod_boussinesq.f90:112-232 quadratures).  The gradient with
    respect to the coefficients against central differences on 32 random
    directions, bounded at 1e-9 relative in the worst direction.

    The start-up VJP is evaluated at the initial state itself: the oracle
    Solver advances the Field objects it is given in place (RICH_BOUSSI_FE_BE
    rebinds PSI%E to the forward-Euler predictor), so the linearisation point
    is copied before the start-up runs."""
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
    n = 4

    def started(c):
        P, C, B = layout.initial_state(g, *c)
        x0 = (P.copy(), C.copy(), B.copy())
        s = BQ.Solver(g, ph, P, C, B)
        s.initialize()
        return x0, s

    def J(c):
        s = started(c)[1]
        for _ in range(n):
            s._step_ab_cn()
        return AD.energy_objective(g, s.psi, s.chi, s.b)

    (P, C, B), s = started(cs)
    stepper = OracleStepper(s)
    keys = stepper.keys
    x0 = tuple(t.requires_grad_() for t in stepper._tensors({k: getattr(s, k) for k in keys}))
    out = run_loop(stepper, x0, n, every=3)
    fin = {k: Field(out[2 * i].detach().numpy().copy(), FFF, float(out[2 * i + 1].detach())) for i, k in enumerate(keys)}
    gp, gc, gb = AD.energy_objective_grad(g, fin["psi"], fin["chi"], fin["b"])
    seeds = {"psi": gp, "chi": gc, "b": gb}
    outs, grads = [], []
    for i, k in enumerate(keys):
        if k in seeds:
            outs += [out[2 * i], out[2 * i + 1]]
            grads += [torch.from_numpy(np.array(seeds[k].E)), torch.tensor(float(seeds[k].LN), dtype=torch.float64)]
    torch.autograd.backward(outs, grads)
    bars = {k: Field(x0[2 * i].grad.numpy().copy(), FFF, float(x0[2 * i + 1].grad)) for i, k in enumerate(keys)}
    s0 = BQ.Solver(g, ph, P.copy(), C.copy(), B.copy())
    x_bar = AD.rich_fe_be_vjp(s0, bars)
    c_bar = AD.initial_state_T(g, x_bar["psi"], x_bar["chi"], x_bar["b"])

    rng = np.random.default_rng(2024)
    # Central differences at h = 1e-5: truncation O(h^2) and rounding
    # O(eps / h) both stay near 1e-10 of J's directional derivative.
    h = 1e-5
    worst = 0.0
    for _ in range(32):
        d = [(rng.standard_normal(c.shape) + 1j * rng.standard_normal(c.shape)) * np.abs(c).max() for c in cs]
        fd = (J([c + h * e for c, e in zip(cs, d)]) - J([c - h * e for c, e in zip(cs, d)])) / (2 * h)
        an = sum(float(np.sum(cb.real * e.real + cb.imag * e.imag)) for cb, e in zip(c_bar, d))
        worst = max(worst, abs(fd - an) / max(1e-12, abs(an)))
    assert worst <= 1e-9, worst

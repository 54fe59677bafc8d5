"""Device gradient path of the AB2-CN solver behind torch.autograd.Function.

The reference has no adjoint.  This module differentiates the objective of
the gradient workload -- the fluctuation kinetic energy plus the buoyancy
variance of the state after a Richardson start-up (RICH_BOUSSI_FE_BE,
mod_march.f90:535-606) and `nsteps` steady AB2-CN steps (STEP_BOUSSI_AB_CN,
609-661, VISC%SW = 1) -- with respect to the seeded perturbation
coefficients of the initial state.  Every forward and reverse step runs in
the CUDA library (the step maps, the step and start-up VJPs, the objective
and its gradient, the initial state's transpose); torch only holds the
state between steps and orders the reverse pass:

    c -> InitialState -> Startup -> run_loop (checkpointed steps) -> Objective

State tensors are the device FFF layout [m][n][k] (complex128 CUDA tensors of
shape (NTCHOPDIM, NRCHOPDIM, NXCHOPDIM)) and one float64 tensor of the
fields' log terms LN.  A solver state is the 7-tuple (psi, chi, b, n_psi,
n_chi, n_b, ln[6]); cotangents follow torch's complex convention
dJ/dRe + i dJ/dIm, the real inner product the library's VJPs use.
"""

from __future__ import annotations

import numpy as np
import torch
from torch.autograd.function import once_differentiable

from . import FFF, MlegsError, qvortex
from .checkpoint import run_loop

__all__ = ["DeviceAB2", "InitialState", "Startup", "Objective", "ref_to_dev", "dev_to_ref", "gradient"]


def ref_to_dev(E):
    """Reference-layout FFF array E[n, m, k] -> device-layout tensor [m][n][k] (host)."""
    return torch.from_numpy(np.ascontiguousarray(np.asarray(E, dtype=np.complex128).transpose(1, 0, 2)))


def dev_to_ref(t):
    """Device-layout tensor [m][n][k] -> reference-layout array E[n, m, k] (host)."""
    return np.ascontiguousarray(t.detach().cpu().numpy().transpose(1, 0, 2))


class DeviceAB2:
    """The AB2-CN step of one context as a stepper for checkpoint.run_loop
    (step / step_vjp on the 7-tuple state), plus the start-up, the initial
    state and the objective.  FP64 contexts with AB2-CN and VISC%SW = 1."""

    def __init__(self, ctx):
        cfg = ctx.cfg
        if not cfg.adams or int(cfg.visc_sw) != 1:
            raise MlegsError(1, "DeviceAB2: AB2-CN contexts with VISC%SW = 1 only")
        self.ctx = ctx
        self.device = torch.device("cuda", getattr(ctx, "device", 0))
        self.shape = (ctx.NTCHOPDIM, ctx.NRCHOPDIM, ctx.NXCHOPDIM)
        mk = lambda n: [ctx.field(FFF) for _ in range(n)]
        self.f_in, self.f_out, self.f_bar, self.f_st = mk(6), mk(6), mk(6), mk(3)
        self._vortex = None

    # ------------------------------------------------------------ transfers
    # Tensors reach the context's fields and come back by device copies on the
    # context's stream, ordered against torch's current stream by events (no
    # host synchronisation): the context's stream waits for torch's work up to
    # the call (the outputs are allocated before that point), and torch's
    # stream waits for the results before the call returns.  Every tensor the
    # context's stream touched is referenced until then, so the caching
    # allocator can hand its memory out again only to torch-stream work that
    # is ordered after those copies.
    def _ext(self):
        if getattr(self, "_ext_stream", None) is None:
            self._ext_stream = torch.cuda.ExternalStream(self.ctx.stream(), device=self.device)
        return self._ext_stream

    def _prep(self, tensors, ln):
        ts = [t.detach().to(self.device, torch.complex128).contiguous() for t in tensors]
        for t in ts:
            if tuple(t.shape) != self.shape:
                raise ValueError("state tensor of shape %s, expected %s" % (tuple(t.shape), self.shape))
        lt = None if ln is None else ln.detach().to(self.device, torch.float64).contiguous()
        return ts, lt

    def _run(self, loads, outs_fields, call):
        """loads: [(fields, tensors, ln or None)]; call() runs on the context's
        stream; returns (tensors, ln) read from outs_fields."""
        ext = self._ext()
        cur = torch.cuda.current_stream(self.device)
        prepped = [(fs, *self._prep(ts, ln)) for fs, ts, ln in loads]
        outs = [torch.empty(self.shape, dtype=torch.complex128, device=self.device) for _ in outs_fields]
        lno = torch.empty(len(outs_fields), dtype=torch.float64, device=self.device)
        ev_in = torch.cuda.Event()
        ev_in.record(cur)
        ext.wait_event(ev_in)
        used = [lno] + outs
        for fields, ts, lt in prepped:
            for q, (f, t) in enumerate(zip(fields, ts)):
                lp = None if lt is None else lt.data_ptr() + 8 * q
                self.ctx.DEVICE_COPY(f, True, FFF, t.data_ptr(), lp)
            used += ts + ([] if lt is None else [lt])
        call()
        for q, f in enumerate(outs_fields):
            self.ctx.DEVICE_COPY(f, False, FFF, outs[q].data_ptr(), lno.data_ptr() + 8 * q)
        ev_out = torch.cuda.Event()
        ev_out.record(ext)
        cur.wait_event(ev_out)
        del used
        return outs, lno

    def _zeros_like_state(self, n):
        return ([torch.zeros(self.shape, dtype=torch.complex128, device=self.device) for _ in range(n)],
                torch.zeros(n, dtype=torch.float64, device=self.device))

    # ------------------------------------------------------------ stepper protocol
    def step(self, state):
        """One steady AB2-CN step of the 7-tuple state."""
        *fs, ln = state
        outs, lno = self._run([(self.f_in, fs, ln)], self.f_out,
                              lambda: self.ctx.AB2_STEP_MAP(self.f_in, self.f_out))
        return tuple(outs) + (lno,)

    def step_vjp(self, state, bars):
        """Cotangents of `state` given those of step(state)."""
        *fs, ln = state
        *bs, bln = bars
        outs, lno = self._run([(self.f_st, fs[:3], ln[:3]), (self.f_bar, bs, bln)], self.f_out,
                              lambda: self.ctx.AB2_STEP_VJP(self.f_st, self.f_bar, self.f_out))
        return tuple(outs) + (lno,)

    # ------------------------------------------------------------ the other maps
    def startup(self, x0):
        """RICH_BOUSSI_FE_BE of (psi, chi, b, ln[3]) -> the 7-tuple state."""
        *fs, ln = x0
        outs, lno = self._run([(self.f_st, fs, ln)], self.f_out,
                              lambda: self.ctx.AB2_STARTUP_MAP(self.f_st, self.f_out))
        return tuple(outs) + (lno,)

    def startup_vjp(self, x0, bars):
        *fs, ln = x0
        *bs, bln = bars
        outs, lno = self._run([(self.f_st, fs, ln), (self.f_bar, bs, bln)], self.f_out[:3],
                              lambda: self.ctx.AB2_STARTUP_VJP(self.f_st, self.f_bar, self.f_out[:3]))
        return tuple(outs) + (lno,)

    def vortex(self):
        if self._vortex is None:
            self._vortex = qvortex(self.ctx)
        return self._vortex

    def initial_state(self, coefs):
        """psi = vortex + IDELSQH(-c_psi), chi = vortex + IDELSQH(-c_chi) (each
        chopped), b = c_b chopped with its m = 0 far-field value removed (the
        construction of mlegs_b200.inputs); coefs in the device layout."""
        ctx = self.ctx
        c_psi, c_chi, c_b = coefs
        neg = [(-c_psi), (-c_chi)]
        vortex = self.vortex()

        def build():
            for q, vf in enumerate(vortex):
                tmp, out, F = self.f_in[3 + q], self.f_bar[q], self.f_out[q]
                ctx.CHOPDO(tmp)
                ctx.IDELSQH(tmp, out)
                ctx.COPY(F, vf)
                ctx.AXPBY(F, 1.0, out, 0.0, None, 1.0)
                ctx.CHOPDO(F)
            ctx.COPY(self.f_out[2], self.f_in[5])
            ctx.CHOPDO(self.f_out[2])
        outs, ln = self._run([(self.f_in[3:5], neg, None), (self.f_in[5:6], [c_b], None)], self.f_out[:3], build)
        # the CALCAT1 far-field value of b (m = 0, every k) removed, as the
        # reference's far-field fix writes it (mod_legops.f90:2540)
        n = int(ctx.cfg.nrchop)
        at1 = torch.sqrt((2 * torch.arange(n, dtype=torch.float64, device=self.device) + 1) / 2)
        b = outs[2]
        b[0, 0, :] -= (at1.to(torch.complex128) @ b[0, :n, :]) / at1[0]
        ln[2] = 0.0
        return outs[0], outs[1], b, ln

    def initial_state_T(self, bars):
        *bs, bln = bars
        outs, _ = self._run([(self.f_st, bs, bln)], self.f_out[:3],
                            lambda: self.ctx.INITIAL_STATE_T(self.f_st, self.f_out[:3]))
        return tuple(outs)

    def objective(self, psi, chi, b):
        """J and (gpsi, gchi, gb)."""
        res = {}

        def call():
            res["J"] = self.ctx.ENERGY_OBJECTIVE(self.f_st[0], self.f_st[1], self.f_st[2],
                                                 self.f_out[0], self.f_out[1], self.f_out[2])
        outs, _ = self._run([(self.f_st, [psi, chi, b], None)], self.f_out[:3], call)
        return res["J"], outs


class InitialState(torch.autograd.Function):
    """apply(solver, c_psi, c_chi, c_b) -> (psi, chi, b, ln[3])."""

    @staticmethod
    def forward(fctx, solver, c_psi, c_chi, c_b):
        fctx.solver = solver
        return solver.initial_state((c_psi, c_chi, c_b))

    @staticmethod
    @once_differentiable
    def backward(fctx, g_psi, g_chi, g_b, g_ln):
        solver = fctx.solver
        zs, zl = solver._zeros_like_state(3)
        gs = [g if g is not None else z for g, z in zip((g_psi, g_chi, g_b), zs)]
        gl = g_ln if g_ln is not None else zl
        return (None,) + solver.initial_state_T(tuple(gs) + (gl,))


class Startup(torch.autograd.Function):
    """apply(solver, psi, chi, b, ln[3]) -> (psi, chi, b, n_psi, n_chi, n_b, ln[6])."""

    @staticmethod
    def forward(fctx, solver, psi, chi, b, ln):
        fctx.solver = solver
        fctx.save_for_backward(psi, chi, b, ln)
        return solver.startup((psi, chi, b, ln))

    @staticmethod
    @once_differentiable
    def backward(fctx, *grads):
        solver = fctx.solver
        psi, chi, b, ln = fctx.saved_tensors
        zs, zl = solver._zeros_like_state(6)
        gs = [g if g is not None else z for g, z in zip(grads[:6], zs)]
        gl = grads[6] if grads[6] is not None else zl
        out = solver.startup_vjp((psi, chi, b, ln), tuple(gs) + (gl,))
        return (None,) + out


class Objective(torch.autograd.Function):
    """apply(solver, psi, chi, b) -> J (0-dimensional float64 tensor)."""

    @staticmethod
    def forward(fctx, solver, psi, chi, b):
        J, grads = solver.objective(psi, chi, b)
        fctx.grads = grads
        return torch.tensor(J, dtype=torch.float64, device=solver.device)

    @staticmethod
    @once_differentiable
    def backward(fctx, gJ):
        return (None,) + tuple(g * gJ for g in fctx.grads)


def gradient(solver, coefs, nsteps=200, every=20, stats=None):
    """J and dJ/dc after the start-up and `nsteps` AB2-CN steps, c = (c_psi,
    c_chi, c_b) in the device layout; the steady steps are checkpointed every
    `every` steps (10 checkpoints and 190 recomputed steps for 200)."""
    cs = [c.detach().to(solver.device, torch.complex128).clone().requires_grad_(True) for c in coefs]
    x0 = InitialState.apply(solver, *cs)
    st = Startup.apply(solver, *x0)
    final = run_loop(solver, st, nsteps, every=every, stats=stats)
    J = Objective.apply(solver, final[0], final[1], final[2])
    J.backward()
    solver.ctx.sync()  # the library's deferred error checks (no call above waits for the device)
    return float(J.item()), [c.grad for c in cs]


def objective_of(solver, coefs, nsteps, graph=True):
    """J alone, through the context's own solver (SOLVER_T's start-up and
    steps, graph-captured when `graph`): the forward of `gradient` without
    the tape, for finite differences."""
    ctx = solver.ctx
    if not hasattr(solver, "f_run"):
        solver.f_run = [ctx.field(FFF) for _ in range(3)]
    res = {}

    def call():
        ctx.initialize(*solver.f_run)
        ctx.step(nsteps, graph=graph)
        res["J"] = ctx.ENERGY_OBJECTIVE(*solver.f_run, *solver.f_out[:3])
    with torch.no_grad():
        psi, chi, b, ln = solver.initial_state(tuple(c.to(solver.device, torch.complex128) for c in coefs))
        solver._run([(solver.f_run, [psi, chi, b], ln)], [], call)
    return res["J"]

"""Checkpointed reverse-mode differentiation of a time loop, behind a
torch.autograd.Function.

The reference has no adjoint; this is the differentiation layer of the step
path: the gradient of an objective of the final state of `nsteps` steady
steps (STEP_BOUSSI_AB_CN, mod_march.f90:609-661, or STEP_BOUSSI_ETDAB_CN,
811-901) with respect to the initial state, taken by reverse accumulation of
one-step vector-Jacobian products.

Memory: the forward pass keeps the state only every `every` steps
(the checkpoints).  The backward pass walks the segments in reverse; for
each it recomputes the segment's states from its checkpoint, then applies
the step VJPs in reverse.  At most ceil(nsteps / every) checkpoints plus
`every` segment states are held at once, and nsteps - ceil(nsteps / every)
steps are recomputed (the checkpoint that opens a segment needs no step).

Cotangent convention: for a real objective J of complex arrays z = x + iy
the cotangent is dJ/dx + i dJ/dy, which is torch's convention for complex
gradients and the real inner product <a, b> = sum(Re a Re b + Im a Im b)
that the step VJPs are defined with; real tensors (the log terms LN) take
the plain derivative.

A stepper is any object with
    step(state)            -> next state (tuple of tensors, same layout)
    step_vjp(state, bars)  -> cotangents of `state`, given the cotangents
                              `bars` of step(state)
where `state` is a tuple of tensors.  step_vjp must not change `state`.
"""

from __future__ import annotations

import math
from dataclasses import dataclass

import torch
from torch.autograd.function import once_differentiable

__all__ = ["LoopStats", "CheckpointedLoop", "run_loop"]


@dataclass
class LoopStats:
    """Counters of one differentiated loop: steps taken forward, checkpoints
    kept, steps recomputed and step VJPs applied in the backward pass, and
    the largest number of states held at once (checkpoints + segment)."""
    forward_steps: int = 0
    checkpoints: int = 0
    recomputed_steps: int = 0
    vjp_steps: int = 0
    peak_states: int = 0


def _check_state(state, nstate, what):
    if not isinstance(state, (tuple, list)) or len(state) != nstate:
        raise ValueError(f"{what} returned {type(state).__name__} of length "
                         f"{len(state) if isinstance(state, (tuple, list)) else '?'}, "
                         f"expected a tuple of {nstate} tensors")
    return tuple(state)


def _stash(t, store):
    t = t.detach()
    if store is None or t.device == torch.device(store):
        return t.clone()
    return t.to(store, copy=True)


class CheckpointedLoop(torch.autograd.Function):
    """apply(stepper, nsteps, every, store, stats, *state) -> final state.

    `store` is the device checkpoints are kept on (None: beside the state;
    "cpu" moves them to host memory).  `stats` is a LoopStats filled in by
    the forward and backward passes, or None."""

    @staticmethod
    def forward(ctx, stepper, nsteps, every, store, stats, *state):
        nsteps, every = int(nsteps), int(every)
        if nsteps < 0:
            raise ValueError(f"nsteps = {nsteps} < 0")
        if every < 1:
            raise ValueError(f"checkpoint interval every = {every} < 1")
        n = len(state)
        cur = tuple(t.detach() for t in state)
        checkpoints = []
        for i in range(nsteps):
            if i % every == 0:
                checkpoints.append(tuple(_stash(t, store) for t in cur))
            cur = _check_state(stepper.step(cur), n, "step")
        ctx.stepper, ctx.nsteps, ctx.every, ctx.stats = stepper, nsteps, every, stats
        ctx.checkpoints = checkpoints
        ctx.devices = [t.device for t in state]
        if stats is not None:
            stats.forward_steps += nsteps
            stats.checkpoints += len(checkpoints)
        # Outputs must be tensors of their own, also for nsteps = 0.
        return tuple(t.clone() for t in cur)

    @staticmethod
    @once_differentiable
    def backward(ctx, *grads):
        stepper, nsteps, every, stats = ctx.stepper, ctx.nsteps, ctx.every, ctx.stats
        checkpoints = ctx.checkpoints
        if checkpoints is None:
            raise RuntimeError("run_loop supports a single backward pass: its checkpoints were "
                               "released by the previous one")
        n = len(grads)
        bars = tuple(grads)
        if nsteps > 0 and any(g is None for g in bars):
            # Zero cotangents take the shape of the final state's components,
            # which equal the checkpoints' shapes.
            ref = checkpoints[0]
            bars = tuple(g if g is not None else torch.zeros_like(r, device=d)
                         for g, r, d in zip(bars, ref, ctx.devices))
        nseg = len(checkpoints)
        for seg in range(nseg - 1, -1, -1):
            start = seg * every
            end = min(start + every, nsteps)
            states = [tuple(t.to(d) for t, d in zip(checkpoints[seg], ctx.devices))]
            for _ in range(start, end - 1):
                states.append(_check_state(stepper.step(states[-1]), n, "step"))
            if stats is not None:
                stats.recomputed_steps += end - 1 - start
                stats.peak_states = max(stats.peak_states, seg + 1 + len(states))
            for j in range(end - 1, start - 1, -1):
                bars = _check_state(stepper.step_vjp(states[j - start], bars), n, "step_vjp")
                if stats is not None:
                    stats.vjp_steps += 1
            checkpoints[seg] = None
            del states
        ctx.checkpoints = None
        return (None, None, None, None, None) + tuple(bars)


def run_loop(stepper, state, nsteps, every=20, store=None, stats=None):
    """Final state of `nsteps` steps of `stepper` from `state` (a tuple of
    tensors), differentiable with respect to `state` by checkpointed
    recomputation every `every` steps (20 in the gradient configuration:
    200 AB2-CN steps keep 10 checkpoints and recompute 190 steps)."""
    state = tuple(state)
    if not state:
        raise ValueError("empty state")
    if int(every) < 1:
        raise ValueError(f"checkpoint interval every = {every} < 1")
    if stats is not None and nsteps > 0:
        stats.peak_states = max(stats.peak_states, math.ceil(nsteps / every))
    return CheckpointedLoop.apply(stepper, nsteps, every, store, stats, *state)

"""Ensembles of AB2-CN runs of different grids with grouped launches.

Instances of different (NR, NTH, NX), Re and N (mlegs_b200.inputs.
ensemble_configs) stepped together by mlegs_ensemble_step: the grouped
persistent RTRAN(+1) / fold GEMMs and grouped banded solves run the
single-grid tile bodies, so every instance must match the same run on its
own context (FP64, same initial state) to rounding, and the FP64 oracle
(STEP_BOUSSI_AB_CN, mod_march.f90:609-661) within the banded-solve tolerance.
Eager steps and graph-replayed steps (after the autotuner's first pass) are
both covered.
"""

import numpy as np
import pytest

from conftest import oracle_grid, oracle_physics, rel

pytestmark = pytest.mark.gpu

SMALL = dict(nrs=(32, 48, 64), nths=(16, 32), nxs=(16, 32))


def _standalone(M, cfg, nsteps):
    ctx = M.Context(cfg)
    fs = M.initial_state(ctx, cfg)
    ctx.initialize(*fs)
    ctx.step(nsteps)
    out = [f.download() for f in fs]
    ctx.close()
    return out


def test_ensemble_matches_standalone_and_oracle(lib_built):
    import mlegs_b200 as M
    from mlegs_b200.inputs import ensemble_configs, perturbation_coefficients
    from oracle import boussinesq as BQ
    from oracle import layout
    cfgs = ensemble_configs(n=6, seed=7, **SMALL)
    assert len({(c.nr, c.nth, c.nx) for c in cfgs}) > 2
    ens = M.Ensemble(cfgs)
    try:
        states = []
        for ctx, cfg in zip(ens.contexts, cfgs):
            fs = M.initial_state(ctx, cfg)
            ctx.initialize(*fs)
            states.append(fs)
        ens.step(2, graph=False)
        ens.step(4, graph=True)
        ens.sync()
        got = [[f.download() for f in fs] for fs in states]
        for ctx in ens.contexts:
            t, n = ctx.time()
            assert n == 7
            ctx.check_finite()
        rows, ctas = ens.tuning()
        assert rows and all(r[3] in (16, 32) for r in rows)
        assert all(c in (2, 3, 4) for c in ctas)
    finally:
        ens.close()
    for cfg, g_out in zip(cfgs, got):
        ref = _standalone(M, cfg, 6)
        for (E, ln), (R, rl) in zip(g_out, ref):
            assert rel(E, R) < 1e-13, cfg.name
            assert abs(ln - rl) <= 1e-13 * max(1.0, abs(rl))
    for cfg, g_out in list(zip(cfgs, got))[:2]:
        g = oracle_grid(cfg)
        P, C, B = layout.initial_state(g, *[perturbation_coefficients(cfg, i) for i in range(3)])
        s = BQ.Solver(g, oracle_physics(cfg), P, C, B)
        s.initialize()
        for _ in range(6):
            s.step()
        for (E, ln), R in zip(g_out, (s.psi, s.chi, s.b)):
            assert rel(E, R.E) < 1e-10, cfg.name
            assert abs(ln - R.LN) < 1e-10 * max(1.0, abs(R.LN))


def test_ensemble_rejects_etd_instances(lib_built):
    import mlegs_b200 as M
    from mlegs_b200.inputs import ensemble_configs
    cfgs = ensemble_configs(n=2, seed=3, **SMALL)
    cfgs[1].adams = False
    ens = M.Ensemble(cfgs)
    try:
        for ctx, cfg in zip(ens.contexts, cfgs):
            ctx.initialize(*M.initial_state(ctx, cfg))
        with pytest.raises(M.MlegsError) as ei:
            ens.step(1)
        assert ei.value.code == 101
    finally:
        ens.close()

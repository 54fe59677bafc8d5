"""mlegs_run_host: time stepping with the state streamed through page-locked
host memory every step, the copies on their own streams (one field's upload
for the next step overlapping the next field's download).

Checked through the C ABI against the same steps made as separate calls
(mlegs_field_upload of psi, chi, b; mlegs_step_graph(1); mlegs_field_download
into the same buffers), bit for bit, for AB2-CN and ETD2AB-CN, and on its
argument and state errors.
"""

import ctypes

import numpy as np
import pytest

from conftest import small_cfg

pytestmark = pytest.mark.gpu

MLEGS_ERR_ARG, MLEGS_ERR_STATE = 101, 104  # include/mlegs_b200.h


def _pinned(shape):
    """A Fortran-ordered complex128 array in page-locked memory (and its owner)."""
    import torch
    buf = torch.empty(int(np.prod(shape)), dtype=torch.complex128, pin_memory=True)
    return np.ndarray(shape, dtype=np.complex128, buffer=buf.numpy(), order="F"), buf


def _state_on_host(M, ctx, fields):
    hosts, keep, lns = [], [], [0.0, 0.0, 0.0]
    for i, f in enumerate(fields):
        h, owner = _pinned(ctx.shape(M.FFF))
        _, lns[i] = f.download(out=h)
        hosts.append(h)
        keep.append(owner)
    return hosts, keep, lns


@pytest.mark.parametrize("adams", [True, False], ids=["ab2cn", "etd2ab"])
def test_run_host_matches_separate_calls(lib_built, adams):
    import mlegs_b200 as M
    cfg = small_cfg(32, 16, 16, adams=adams)
    res = []
    for mode in ("calls", "run_host"):
        ctx = M.Context(cfg)
        try:
            fs = M.initial_state(ctx)
            ctx.initialize(*fs)
            ctx.step(2, graph=(mode == "calls"))  # run_host captures its graph itself
            hosts, keep, lns = _state_on_host(M, ctx, fs)
            n0 = ctx.time()[1]
            if mode == "calls":
                for _ in range(3):
                    for i, f in enumerate(fs):
                        f.upload(hosts[i], lns[i], M.FFF)
                    ctx.step(1, graph=True)
                    for i, f in enumerate(fs):
                        _, lns[i] = f.download(out=hosts[i])
            else:
                assert ctx.run_host(hosts, lns, n=0) == lns  # set-up only
                lns = ctx.run_host(hosts, lns, n=3)
            # the device state is the last step's, as the host copies hold it
            for i, f in enumerate(fs):
                E, ln = f.download()
                assert f.space == M.FFF
                assert np.array_equal(E, hosts[i]) and ln == lns[i]
            assert ctx.time()[1] == n0 + 3
            res.append(([h.copy() for h in hosts], list(lns), ctx.time()))
        finally:
            ctx.close()
    (Ea, la, ta), (Eb, lb, tb) = res
    for a, b in zip(Ea, Eb):
        assert np.array_equal(a, b)
    assert la == lb
    assert ta == tb


def test_run_host_errors(lib_built):
    import mlegs_b200 as M
    ctx = M.Context(small_cfg(32, 16, 16))
    try:
        shape = ctx.shape(M.FFF)
        hosts = [np.zeros(shape, dtype=np.complex128, order="F") for _ in range(3)]
        with pytest.raises(M.MlegsError) as e:  # no solver state yet
            ctx.run_host(hosts, [0.0, 0.0, 0.0], n=1)
        assert e.value.code == MLEGS_ERR_STATE
        ptrs = (ctypes.c_void_p * 3)(*[h.ctypes.data for h in hosts])
        ln = (ctypes.c_double * 3)()
        assert ctx.lib.mlegs_run_host(ctx.c, -1, ctypes.cast(ptrs, ctypes.c_void_p), ln) == MLEGS_ERR_ARG
        assert ctx.lib.mlegs_run_host(ctx.c, 1, None, ln) == MLEGS_ERR_ARG
        ptrs[1] = None
        assert ctx.lib.mlegs_run_host(ctx.c, 1, ctypes.cast(ptrs, ctypes.c_void_p), ln) == MLEGS_ERR_ARG
        with pytest.raises(ValueError):
            ctx.run_host(hosts[:2], [0.0, 0.0], n=1)
    finally:
        ctx.close()

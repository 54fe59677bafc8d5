"""The single-kernel timing entry point (mlegs_kernel_time) for every kernel it
names, and the FP64 tensor-path ceiling kernel behind it.

mlegs_kernel_time launches one internal kernel on pool temporaries (3 warm-up
launches, then the timed ones) and reports the mean device time and the
algorithmic HBM bytes of one launch; for ``dmma_peak`` the second figure is
the FLOPs of a register-only FP64 MMA launch (4 CTAs x 8 warps per SM,
8 accumulators x 4,096 rounds of m8n8k4 per warp).
"""

import pytest

from conftest import small_cfg

pytestmark = pytest.mark.gpu

SPLIT_ONLY = {"split_b2p", "split_p2b"}
MLEGS_ERR_ARG, MLEGS_ERR_STATE = 101, 104  # include/mlegs_b200.h


def test_every_kernel_times():
    import mlegs_b200 as M
    ctx = M.Context(small_cfg(96, 64, 64), precision=M.PREC_FP64)
    try:
        for name in M.Context.KERNELS:
            if name in SPLIT_ONLY:
                with pytest.raises(M.MlegsError) as e:
                    ctx.kernel_time(name, reps=2)
                assert e.value.code == MLEGS_ERR_STATE
                continue
            try:
                ms, by = ctx.kernel_time(name, reps=2)
            except M.MlegsError as e:  # PROJECT of FFF inputs needs the tensor path
                assert name == "project_fff" and e.code == MLEGS_ERR_STATE
                continue
            assert ms > 0 and by > 0, name
    finally:
        ctx.close()
    ctx = M.Context(small_cfg(96, 64, 64), precision=M.PREC_SPLIT)
    try:
        for name in sorted(SPLIT_ONLY):
            ms, by = ctx.kernel_time(name, reps=2)
            assert ms > 0 and by > 0, name
    finally:
        ctx.close()


def test_dmma_peak():
    import torch
    import mlegs_b200 as M
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    ctx = M.Context(small_cfg(96, 64, 64), precision=M.PREC_FP64)
    try:
        ms, flops = ctx.kernel_time("dmma_peak", reps=3)
        assert flops == sms * 4 * 8 * 8 * 4096 * 512.0
        # 37.1 TFLOP/s measured on B200 at 1965 MHz; a loose floor for shared or capped clocks
        assert 10.0 < flops / ms / 1e9 < 60.0
    finally:
        ctx.close()
    # the kernel writes one double per thread: a grid whose field buffers hold fewer is refused
    ctx = M.Context(small_cfg(32, 16, 16), precision=M.PREC_FP64)
    try:
        with pytest.raises(M.MlegsError) as e:
            ctx.kernel_time("dmma_peak", reps=1)
        assert e.value.code == MLEGS_ERR_ARG
    finally:
        ctx.close()

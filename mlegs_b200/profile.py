"""Profiling driver: one or more eager steady-state steps of a configuration.

python -m mlegs_b200.profile [--config etd_192x128x256] [--steps 1] [--precision fp64|split]
python -m mlegs_b200.profile --kernel NAME [--reps 1]

Builds the seeded initial state on the device, fills the AB/ETD history with
the Richardson start-up, then runs --steps eager steps (no CUDA graph), so
that an external profiler sees each kernel launch of a steady step in order.
The launch count before the steps is printed so a profiler can skip it.

With --kernel, runs Context.kernel_time(NAME, reps) instead: 3 warm-up
launches of that one kernel, then --reps timed ones, on the configuration's
field sizes (for a single-kernel capture: skip 3, capture 1).  --kernel
dmma_peak times register-only FP64 MMAs and prints the tensor path's ceiling.
"""

import argparse
import os
import sys

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--config", default="etd_192x128x256")
    ap.add_argument("--steps", type=int, default=1)
    ap.add_argument("--precision", default="fp64", choices=["fp64", "split"])
    ap.add_argument("--kernel", default=None)
    ap.add_argument("--reps", type=int, default=1)
    a = ap.parse_args()
    import mlegs_b200 as M
    cfg = M.CONFIGS[a.config]
    ctx = M.Context(cfg, precision=M.PREC_FP64 if a.precision == "fp64" else M.PREC_SPLIT)
    if a.kernel:
        ms, nbytes = ctx.kernel_time(a.kernel, a.reps)
        if a.kernel == "dmma_peak":  # the figure is FLOPs: the FP64 tensor-path ceiling
            print("%s: %.1f us per launch, %.2f TFLOP/s" % (a.kernel, ms * 1e3, nbytes / ms / 1e9))
        else:
            print("%s: %.1f us per launch, %.1f GB/s algorithmic" % (a.kernel, ms * 1e3, nbytes / ms / 1e6))
        ctx.close()
        return
    psi, chi, b = M.initial_state(ctx)
    ctx.initialize(psi, chi, b)
    ctx.sync()
    n0 = ctx.launches()
    ctx.step(a.steps)
    ctx.sync()
    per_step = (ctx.launches() - n0) // max(a.steps, 1)
    ctx.check_finite()
    print("launches before steps: %d, per step: %d" % (n0, per_step))
    ctx.close()


if __name__ == "__main__":
    main()

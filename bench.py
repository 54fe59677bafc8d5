"""Benchmark: Boussinesq steps/s on one B200 (or N independent replicas).

python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                [--config etd_192x128x256] [--precision fp64|split] [--slices 6]

Workload: the ETD2AB-CN timestep at NR x NTH x NX = 192 x 128 x 256 (Re 5000,
hyperviscosity P=2 nu_p=kappa_p=1e-10, Omega 1, N 2, dt 5e-4) from a Gaussian
q-vortex plus a seeded spectral perturbation (mlegs_b200/inputs.py), one CUDA
graph replay per step.  Per-GPU work is fixed (replicas only, "weak").

`value` is the --precision path (default fp64: every GEMM on the FP64 tensor
path, mma.sync m8n8k4); "precision_comparison" times the other path beside it
(split: the Legendre GEMMs as split-BF16 slices on tcgen05, everything else
FP64) and reports the relative field error of the mixed path against the FP64
path after --error-steps steps from the same state, against the 1e-9 bound.
Every step touches several GB (100 MB physical fields), far above the 126 MB
L2, so no explicit L2 flush is needed between steps.

The error of both GPU paths against the FP64 oracle itself is measured too:
an oracle process (spawned before the first GPU call, so it runs on the host
cores while the GPU is timed) runs the Richardson start-up and --oracle-steps
- 1 steady steps from the same state; "precision_comparison" reports the
FP64 and the mixed GPU paths' field errors against it, and the mixed path's
error against the FP64 GPU path after --error-steps steps.

"ensemble" is the batched-run configuration: 64 AB2-CN runs of different
grids (NR 48..192, NTH 32..128, NX 32..256, Re 500..5000, N 0.5..4) stepped
50 times together with grouped launches (graph-replayed, after the
autotuner's pass), beside the same 64 runs one after another on their own
contexts, with each instance's field error against that FP64 run.

"transform_roundtrip" is the transform-only configuration: FFF -> PPP -> FFF
(TOFP, TOFF) at 256^3 with 2/3 chops, a batch of 8 fields, per precision
form (FP64 and split-BF16 S = 4, 5, 6): device time per round trip and the
relative error of PPP and of the returned FFF against the FP64 oracle for the
chi, psi and b coefficient sets (mlegs_b200.inputs.roundtrip_coefficients).

"gradient" is the gradient configuration: J = fluctuation KE + 1/2 int b^2
after the AB2-CN start-up and 200 steps at 96x64x64, differentiated with
respect to the perturbation coefficients through torch.autograd on the
device (step maps and VJPs of the library, checkpoints every 20 steps):
seconds per gradient beside the graph-replayed forward alone, and central
differences on two random directions.

--impl reference times the reference's path as restated on the CPU (the
numpy/scipy FP64 oracle under oracle/, all host cores): the reference itself
is Fortran 90 + MPI + FFTW + MKL and cannot be built in this image, so that
arm is a numpy restatement of the reference, not the Fortran solver.
"""

import argparse
import json
import os
import statistics
import subprocess
import tempfile
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Boussinesq steps/s 192x128x256: mixed-prec vs FP64 GPU at same error bound"
UNIT = "steps/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="etd_192x128x256")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "split"],
                    help="path timed for `value`; the other one is timed beside it")
    ap.add_argument("--slices", type=int, default=6, help="split-BF16 slices per operand (3..6)")
    ap.add_argument("--no-compare", action="store_true", help="skip the other path and the error check")
    ap.add_argument("--error-steps", type=int, default=100)
    ap.add_argument("--oracle-steps", type=int, default=10,
                    help="steps (start-up included) of the oracle trajectory the GPU paths are checked against")
    ap.add_argument("--no-roundtrip", action="store_true", help="skip the 256^3 transform round-trip leg")
    ap.add_argument("--no-ensemble", action="store_true", help="skip the 64-instance ensemble leg")
    ap.add_argument("--no-gradient", action="store_true", help="skip the adjoint gradient leg")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-steps", type=int, default=2)
    return ap.parse_args()


def dist_setup(n):
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime

        import torch.distributed as dist
        backend = "nccl"
        try:
            import torch
            if not torch.cuda.is_available():
                backend = "gloo"
            else:
                torch.cuda.set_device(local)
        except Exception:
            backend = "gloo"
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
    return ws, rank, local


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(ws, v):
    if ws == 1:
        return v
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([v], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


class Clocks:
    """nvidia-smi sampler running while the timed region runs."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        # the raw samples: MLEGS_CLOCKS_CSV, else the system temporary directory
        self.path = os.environ.get("MLEGS_CLOCKS_CSV") or os.path.join(tempfile.gettempdir(),
                                                                       "mlegs_clocks_bench.csv")
        os.makedirs(os.path.dirname(self.path), exist_ok=True)
        self.proc = None

    def __enter__(self):
        try:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "--query-gpu=" + self.Q, "--format=csv,noheader,nounits",
                                          "-i", str(self.index), "-lms", "200"], stdout=self.fh,
                                         stderr=subprocess.DEVNULL)
            time.sleep(0.5)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.3)
            self.proc.terminate()
            try:
                self.proc.wait(5)
            except Exception:
                self.proc.kill()
            self.fh.close()

    def summary(self):
        try:
            rows = [r.split(",") for r in open(self.path).read().strip().splitlines()]
        except Exception:
            return None
        rows = [[c.strip() for c in r] for r in rows if len(r) >= 9]
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        loaded = [v for v in sm if mx and v > 0.5 * max(mx)] or sm
        return {"sm_mhz": statistics.median(loaded) if loaded else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons, "samples": len(rows)}


def peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))), "measured"
    except Exception:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


def traffic_table():
    p = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        return json.load(open(p))
    except Exception:
        return {}


def legendre_flops(cfg, nxchopdim):
    """FP64 flops of one RTRAN-equivalent Legendre product with the parity fold
    (mod_fft.f90:1264-1336): 2 NR (sum over m < NTCHOP of NRCHOPS(m)) NXCHOPDIM,
    NRCHOPS(m) = NRCHOP - m (474 MFLOP at 192x128x256)."""
    snn = sum(max(0, cfg.nrchop - m) for m in range(cfg.ntchop))
    return 2.0 * cfg.nr * snn * nxchopdim


def oracle_steps(cfg, nsteps, warm=0):
    """Time steady-state oracle steps (zeroed AB/ETD history: same arithmetic)."""
    import numpy as np

    from mlegs_b200.inputs import perturbation_coefficients
    from oracle import boussinesq as BQ
    from oracle import layout
    from oracle.grid import Grid
    g = Grid(cfg.nr, cfg.nth, cfg.nx, cfg.nrchop, cfg.ntchop, cfg.nxchop, cfg.ell, cfg.zlen)
    ph = BQ.Physics(dt=cfg.dt, omega=cfg.omega, bv0=cfg.bv0, kappa=cfg.kappa, kappap=cfg.kappap,
                    adams=cfg.adams, visc_sw=cfg.visc_sw, nu=cfg.nu, nup=cfg.nup, p=cfg.p)
    P, C, B = layout.initial_state(g, *[perturbation_coefficients(cfg, i) for i in range(3)])
    s = BQ.Solver(g, ph, P, C, B)
    z = lambda: g.alloc(1)  # noqa: E731
    if cfg.adams:
        s.n_psi, s.n_chi, s.n_b = z(), z(), z()
    else:
        s.etd_e, s.etd_nl = BQ.calc_boussi_etd_op(cfg.bv0, cfg.omega, cfg.dt)
        s.n_b, s.r_n_r, s.r_n_p, s.n_z, s.r_pi_r, s.r_pi_p, s.pi_z = (z() for _ in range(7))
    for _ in range(warm):
        s.step()
    t0 = time.perf_counter()
    for _ in range(nsteps):
        s.step()
    dt = time.perf_counter() - t0
    assert np.isfinite(s.psi.E).all()
    return nsteps / dt


def oracle_trajectory(name, nsteps, threads):
    """Oracle (E, LN) of psi, chi, b after the Richardson start-up and nsteps - 1
    steady steps from the benchmark's initial state; runs in a child process
    on `threads` host threads.  Returns (states, seconds)."""
    for v in ("OMP_NUM_THREADS", "OPENBLAS_NUM_THREADS", "MKL_NUM_THREADS"):
        os.environ[v] = str(threads)
    from mlegs_b200.inputs import CONFIGS, perturbation_coefficients
    from oracle import boussinesq as BQ
    from oracle import layout
    from oracle import transforms
    from oracle.grid import Grid
    transforms.WORKERS = threads
    cfg = CONFIGS[name]
    t0 = time.perf_counter()
    g = Grid(cfg.nr, cfg.nth, cfg.nx, cfg.nrchop, cfg.ntchop, cfg.nxchop, cfg.ell, cfg.zlen)
    ph = BQ.Physics(dt=cfg.dt, omega=cfg.omega, bv0=cfg.bv0, kappa=cfg.kappa, kappap=cfg.kappap,
                    adams=cfg.adams, visc_sw=cfg.visc_sw, nu=cfg.nu, nup=cfg.nup, p=cfg.p)
    P, C, B = layout.initial_state(g, *[perturbation_coefficients(cfg, i) for i in range(3)])
    s = BQ.Solver(g, ph, P, C, B)
    s.initialize()
    for _ in range(nsteps - 1):
        s.step()
    return [(F.E, F.LN) for F in (s.psi, s.chi, s.b)], time.perf_counter() - t0


def start_oracle_trajectory(name, nsteps):
    """Start oracle_trajectory in a spawned process (before any GPU call)."""
    import multiprocessing as mp
    threads = max(1, (os.cpu_count() or 2) // 2)
    pool = mp.get_context("spawn").Pool(1)
    return pool, pool.apply_async(oracle_trajectory, (name, nsteps, threads))


def field_errors(got, ref):
    """max|d| / max|ref| per field and |d LN| / max(1, |LN|) per log term."""
    import numpy as np
    errs = {}
    for name, (E, ln), (R, rl) in zip(("psi", "chi", "b"), got, ref):
        errs[name] = float(np.abs(E - R).max() / np.abs(R).max())
        errs[name + "_ln"] = float(abs(ln - rl) / max(1.0, abs(rl)))
    return errs


def roundtrip_leg(local, reps=10, batch=8):
    """The transform-only configuration: FFF -> PPP -> FFF at 256^3 per precision form."""
    import numpy as np

    import mlegs_b200 as M
    from mlegs_b200.inputs import CONFIGS, roundtrip_coefficients
    from oracle import transforms as T
    from oracle.grid import FFF, Grid
    cfg = CONFIGS["roundtrip_256"]
    g = Grid(cfg.nr, cfg.nth, cfg.nx, cfg.nrchop, cfg.ntchop, cfg.nxchop, cfg.ell, cfg.zlen)
    names = ("chi", "psi", "b")
    coefs = [roundtrip_coefficients(cfg, i) for i in range(3)]
    refs = []
    for c in coefs:
        A = g.alloc(FFF)
        A.E = c.copy()
        T.tofp(g, A)
        ppp = A.E.copy()
        T.toff(g, A)
        refs.append((ppp, A.E.copy()))
    out = {"workload": cfg.name, "grid": [cfg.nr, cfg.nth, cfg.nx], "chops": [cfg.nrchop, cfg.ntchop, cfg.nxchop],
           "batch": batch, "reference": "FP64 oracle (numpy/scipy restatement of TOFP/TOFF)", "forms": {}}
    for form, prec, S in (("fp64", M.PREC_FP64, 0), ("split4", M.PREC_SPLIT, 4), ("split5", M.PREC_SPLIT, 5),
                          ("split6", M.PREC_SPLIT, 6)):
        try:
            ctx = M.Context(cfg, precision=prec, split_slices=S, device=local)
        except M.MlegsError as e:
            out["forms"][form] = {"unsupported": str(e)}
            continue
        try:
            ms, by = ctx.kernel_time("roundtrip", reps=reps)
            e_ppp, e_fff, e_id = {}, {}, {}
            f = ctx.field(M.FFF)
            for name, c, (ppp, fff) in zip(names, coefs, refs):
                f.upload(c, 0.0, M.FFF)
                ctx.TOFP(f)
                E, _ = f.download()
                e_ppp[name] = float(np.abs(E - ppp).max() / np.abs(ppp).max())
                ctx.TOFF(f)
                E, _ = f.download()
                e_fff[name] = float(np.abs(E - fff).max() / np.abs(fff).max())
                e_id[name] = float(np.abs(E - c).max() / np.abs(c).max())
            out["forms"][form] = {"ms_per_roundtrip": ms, "batch_ms": batch * ms,
                                  "roundtrips_per_s": 1000.0 / ms, "batches_per_s": 1000.0 / (batch * ms),
                                  "algorithmic_bytes_per_roundtrip": by, "achieved_gbs": by / (ms * 1e-3) / 1e9,
                                  "rel_err_ppp_vs_oracle": e_ppp, "rel_err_fff_vs_oracle": e_fff,
                                  "rel_err_fff_vs_input": e_id}
        finally:
            ctx.close()
    return out


def ensemble_leg(local, n=64, steps=50, warm=3):
    """The batched-run configuration: n AB2-CN instances of different grids
    (mlegs_b200.inputs.ensemble_configs) stepped together with grouped
    launches, graph-replayed; aggregate steps/s against the same instances
    run one after another on their own contexts (graph-replayed too), and
    each instance's field error against that standalone FP64 run."""
    import numpy as np
    import torch

    import mlegs_b200 as M
    from mlegs_b200.inputs import ensemble_configs
    cfgs = ensemble_configs(n)
    ens = M.Ensemble(cfgs, device=local)
    states = []
    for ctx, c in zip(ens.contexts, cfgs):
        fs = M.initial_state(ctx, c)
        ctx.initialize(*fs)
        states.append(fs)
    ens.step(warm, graph=True)  # eager step, autotuning, capture, replays
    ens.sync()
    st = torch.cuda.ExternalStream(ens.stream(), device=local)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    l0 = ens.launches()
    e0.record(st)
    ens.step(steps, graph=True)
    e1.record(st)
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    launches = ens.launches() - l0
    rows, ctas = ens.tuning()
    got = [[f.download() for f in fs] for fs in states]
    ens.close()
    # the same instances on their own contexts, one after another
    solo_ms, errs = 0.0, []
    for c, g_out in zip(cfgs, got):
        ctx = M.Context(c, device=local)
        fs = M.initial_state(ctx, c)
        ctx.initialize(*fs)
        ctx.step(warm, graph=True)
        ctx.sync()
        s = torch.cuda.ExternalStream(ctx.stream(), device=local)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(s)
        ctx.step(steps, graph=True)
        b.record(s)
        b.synchronize()
        solo_ms += a.elapsed_time(b)
        ref = [f.download() for f in fs]
        errs.append(max(float(np.abs(E - R).max() / np.abs(R).max()) for (E, _), (R, _) in zip(g_out, ref)))
        ctx.close()
    grids = sorted({(c.nr, c.nth, c.nx) for c in cfgs})
    return {"workload": "ensemble_%d_ab2" % n, "instances": n, "steps": steps, "distinct_grids": len(grids),
            "ms": ms, "aggregate_steps_per_s": n * steps / (ms * 1e-3), "gpu_launches": int(launches),
            "standalone_sequential_ms": solo_ms, "standalone_aggregate_steps_per_s": n * steps / (solo_ms * 1e-3),
            "speedup_vs_standalone": solo_ms / ms, "max_rel_error_vs_standalone_fp64": max(errs),
            "tuning": {"classes": [{"transform": "rtran+1" if r[0] == 0 else "fold", "NRH": r[1], "NRCHOP": r[2],
                                    "tile_columns": r[3]} for r in rows],
                       "ctas_per_sm": {"rtran+1": ctas[0], "fold": ctas[1]}}}


def gradient_leg(local, fd_directions=2):
    """The gradient configuration (grad_96x64x64): J = fluctuation KE + 1/2
    int b^2 after the AB2-CN start-up and 200 steps, differentiated with
    respect to the perturbation coefficients through torch.autograd (device
    step maps and VJPs, checkpoints every 20 steps).  Wall-clock seconds per
    gradient (host-driven calls, stream-ordered: the host waits only for J) beside the
    forward alone on the context's graph-replayed solver, and central
    differences on a few random directions."""
    import time

    import numpy as np
    import torch

    import mlegs_b200 as M
    from mlegs_b200.adjoint import DeviceAB2, gradient, objective_of, ref_to_dev
    from mlegs_b200.checkpoint import LoopStats
    from mlegs_b200.inputs import CONFIGS, perturbation_coefficients
    cfg = CONFIGS["grad_96x64x64"]
    ctx = M.Context(cfg, device=local)
    try:
        solver = DeviceAB2(ctx)
        cs = [ref_to_dev(perturbation_coefficients(cfg, i)) for i in range(3)]
        gradient(solver, cs, nsteps=4, every=2)  # set-up: factors, transposed tables, temporaries
        objective_of(solver, cs, cfg.nsteps)
        torch.cuda.synchronize(local)
        stats = LoopStats()
        l0 = ctx.launches()
        t0 = time.perf_counter()
        J, grads = gradient(solver, cs, nsteps=cfg.nsteps, every=20, stats=stats)
        torch.cuda.synchronize(local)
        t_grad = time.perf_counter() - t0
        launches = ctx.launches() - l0
        t0 = time.perf_counter()
        J_fwd = objective_of(solver, cs, cfg.nsteps)
        torch.cuda.synchronize(local)
        t_fwd = time.perf_counter() - t0
        rng = np.random.default_rng(7)
        scale = max(float(c.abs().max()) for c in cs)
        h, errs = 1e-5, []
        for _ in range(fd_directions):
            d = [torch.from_numpy((rng.standard_normal(c.shape) + 1j * rng.standard_normal(c.shape)) * scale)
                 for c in cs]
            fd = (objective_of(solver, [c + h * e for c, e in zip(cs, d)], cfg.nsteps)
                  - objective_of(solver, [c - h * e for c, e in zip(cs, d)], cfg.nsteps)) / (2 * h)
            an = sum(float((g.cpu() * e.conj()).real.sum()) for g, e in zip(grads, d))
            errs.append(abs(fd - an) / abs(an))
    finally:
        ctx.close()
    return {"workload": cfg.name, "grid": [cfg.nr, cfg.nth, cfg.nx], "steps": cfg.nsteps, "checkpoint_every": 20,
            "J": J, "J_forward_only": J_fwd, "seconds_per_gradient": t_grad,
            "seconds_forward_only_graph": t_fwd, "gradient_over_forward": t_grad / t_fwd,
            "checkpoints": stats.checkpoints, "recomputed_steps": stats.recomputed_steps,
            "vjp_steps": stats.vjp_steps, "peak_states": stats.peak_states, "gpu_launches": int(launches),
            "fd_directions": fd_directions, "fd_max_rel_error": max(errs),
            "timing": "wall clock around the gradient (host-driven calls, stream-ordered by events; one host wait for J)"}


def run_reference(args, cfg, ws, rank):
    if rank != 0:
        return
    cores = os.cpu_count()
    v = oracle_steps(cfg, args.steps, warm=args.warmup)
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 / v,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded q-vortex + spectral perturbation)",
            "config": {"workload": cfg.name, "grid": [cfg.nr, cfg.nth, cfg.nx],
                       "chops": [cfg.nrchop, cfg.ntchop, cfg.nxchop], "scheme": "ETD2AB-CN" if not cfg.adams else "AB2-CN",
                       "parallelism": "cpu threads"},
            "reference_kind": "numpy restatement of the reference (Fortran 90/MPI/FFTW solver unavailable: "
                              "not buildable in this image)",
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": "port",
                             "sample": "%d steady steps after %d warm-up, FP64 numpy/scipy restatement of the "
                                       "reference path (reference Fortran not buildable here)" % (args.steps, args.warmup)},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def _graph_steps(ctx, stream, steps):
    """Device time (ms) of `steps` graph-replayed steps on the library stream."""
    import torch
    ctx.sync()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    ctx.step(steps, graph=True)
    e1.record(stream)
    e1.synchronize()
    return e0.elapsed_time(e1)


def _state_after(M, cfg, prec, slices, nsteps, local):
    """(E, LN) of psi, chi, b after 1 Richardson + nsteps-1 graph steps."""
    ctx = M.Context(cfg, precision=prec, split_slices=slices, device=local)
    fs = M.initial_state(ctx)
    ctx.initialize(*fs)
    if nsteps > 1:
        ctx.step(nsteps - 1, graph=True)
    out = [f.download() for f in fs]
    ctx.close()
    return out


def run_ours(args, cfg, ws, rank, local):
    import numpy as np
    import torch

    import mlegs_b200 as M
    split = args.precision == "split"
    prec = M.PREC_SPLIT if split else M.PREC_FP64
    orc = None
    if not args.no_compare and rank == 0 and ws == 1:
        orc = start_oracle_trajectory(cfg.name, args.oracle_steps)  # before the first GPU call
    torch.cuda.set_device(local)
    ctx = M.Context(cfg, precision=prec, split_slices=args.slices if split else 0, device=local)
    psi, chi, b = M.initial_state(ctx)
    ctx.initialize(psi, chi, b)
    stream = torch.cuda.ExternalStream(ctx.stream(), device=local)
    ctx.step(max(args.warmup, 1), graph=True)  # first call captures the graph
    ctx.sync()

    vis = os.environ.get("CUDA_VISIBLE_DEVICES")
    smi_index = int(vis.split(",")[local]) if vis else local
    barrier(ws)
    ctx.reset_launches()
    with Clocks(smi_index) as clk:
        ms_total = _graph_steps(ctx, stream, args.steps)
    launches = ctx.launches()
    barrier(ws)
    ms_total = max_over_ranks(ws, ms_total)
    ms_step = ms_total / args.steps
    value = ws * args.steps / (ms_total / 1000.0)
    ctx.check_finite()

    # ---- e2e: per step, upload state from pinned host, one graph step, download.
    # The headline goes through mlegs_run_host (the copies on their own streams,
    # one field's upload overlapping the next field's download); the same steps
    # as separate upload / step / download calls are timed beside it.
    shape = ctx.shape(M.FFF)
    nbytes = int(np.prod(shape)) * 16
    hosts = []
    for f in (psi, chi, b):
        buf = torch.empty(int(np.prod(shape)), dtype=torch.complex128, pin_memory=True).numpy()
        arr = np.ndarray(shape, dtype=np.complex128, buffer=buf, order="F")
        hosts.append(arr)
    lns = [0.0, 0.0, 0.0]
    for i, f in enumerate((psi, chi, b)):
        _, lns[i] = f.download(out=hosts[i])
    lns = ctx.run_host(hosts, lns, n=1)  # sets up its streams and staging buffers

    def e2e_run(pipelined):
        barrier(ws)
        ctx.sync()
        e2 = torch.cuda.Event(enable_timing=True)
        e3 = torch.cuda.Event(enable_timing=True)
        t0 = time.perf_counter()
        e2.record(stream)
        lv = list(lns)
        if pipelined:
            lv = ctx.run_host(hosts, lv, n=args.steps)
        else:
            for _ in range(args.steps):
                for i, f in enumerate((psi, chi, b)):
                    f.upload(hosts[i], lv[i], M.FFF)
                ctx.step(1, graph=True)
                for i, f in enumerate((psi, chi, b)):
                    _, lv[i] = f.download(out=hosts[i])
        e3.record(stream)
        e3.synchronize()
        wall = time.perf_counter() - t0
        ms = max(e2.elapsed_time(e3), wall * 1000.0)
        barrier(ws)
        ms = max_over_ranks(ws, ms)
        lns[:] = lv
        return ws * args.steps / (ms / 1000.0)

    e2e_value = e2e_run(True)
    e2e_calls = e2e_run(False)

    # ---- roofline of the dominant kernel (live CUDA-event timing on the library stream)
    pk, pk_kind = peaks()
    kernels = {}
    for name in ctx.KERNELS:
        try:
            ms, by = ctx.kernel_time(name, reps=20)
        except M.MlegsError:
            continue  # tensor-core kernels exist only in split contexts
        if name == "dmma_peak":  # register-only FP64 MMAs: FLOPs, the tensor path's ceiling
            kernels[name] = {"ms": ms, "flops": by, "tflops": by / (ms * 1e-3) / 1e12}
        else:
            kernels[name] = {"ms": ms, "bytes": by, "gbs": by / (ms * 1e-3) / 1e9}
    # the Legendre GEMMs in useful FP64 flops against the FP64 tensor path's ceiling
    # (register-only m8n8k4 MMAs, timed above); PROJECT is five fold products
    ceil = kernels.get("dmma_peak", {}).get("tflops")
    if ceil and not split:
        fl = legendre_flops(cfg, ctx.NXCHOPDIM)
        for name, nprod in (("rtran_b2p", 1), ("rtran_p2b", 1), ("project", 5)):
            if name in kernels:
                tf = nprod * fl / (kernels[name]["ms"] * 1e-3) / 1e12
                kernels[name].update(fp64_flops=nprod * fl, tflops=tf, frac_of_fp64_ceiling=tf / ceil)
    dom = DOMINANT
    tr = traffic_table().get(cfg.name, {}).get(dom)
    ach = kernels[dom]["gbs"]
    roof = {"kernel": dom, "bound": "hbm", "achieved": ach, "peak": pk["hbm_gbs"], "unit": "GB/s",
            "frac": ach / pk["hbm_gbs"], "traffic": tr, "peak_source": pk_kind,
            "algorithmic_bytes_per_launch": kernels[dom]["bytes"], "ms_per_launch": kernels[dom]["ms"]}
    ctx.close()

    # ---- the other precision's step, and the error of the mixed path against FP64
    compare = None
    if not args.no_compare:
        other_split = not split
        c2 = M.Context(cfg, precision=M.PREC_SPLIT if other_split else M.PREC_FP64,
                       split_slices=args.slices if other_split else 0, device=local)
        fs = M.initial_state(c2)
        c2.initialize(*fs)
        s2 = torch.cuda.ExternalStream(c2.stream(), device=local)
        c2.step(max(args.warmup, 1), graph=True)
        ms2 = _graph_steps(c2, s2, args.steps)
        c2.close()
        barrier(ws)
        ms2 = max_over_ranks(ws, ms2)
        other_value = ws * args.steps / (ms2 / 1000.0)
        ref = _state_after(M, cfg, M.PREC_FP64, 0, args.error_steps, local)
        mix = _state_after(M, cfg, M.PREC_SPLIT, args.slices, args.error_steps, local)
        errs = field_errors(mix, ref)
        mixed_v, fp64_v = (other_value, value) if other_split else (value, other_value)
        compare = {"fp64_steps_per_s": fp64_v, "mixed_steps_per_s": mixed_v, "split_slices": args.slices,
                   "mixed_over_fp64": mixed_v / fp64_v, "error_steps": args.error_steps,
                   "mixed_rel_error_vs_fp64": errs, "error_bound": 1e-9,
                   "mixed_within_bound": max(errs.values()) <= 1e-9}
        if orc is not None:
            pool, job = orc
            orc_states, orc_s = job.get()
            pool.close()
            pool.join()
            n_o = args.oracle_steps
            fp_o = _state_after(M, cfg, M.PREC_FP64, 0, n_o, local)
            mx_o = _state_after(M, cfg, M.PREC_SPLIT, args.slices, n_o, local)
            e_fp, e_mx = field_errors(fp_o, orc_states), field_errors(mx_o, orc_states)
            compare.update({"oracle_steps": n_o, "oracle_seconds": orc_s,
                            "fp64_rel_error_vs_oracle": e_fp, "mixed_rel_error_vs_oracle": e_mx,
                            "comparand": "FP64 oracle (numpy restatement of the reference path) after %d steps "
                                         "(start-up included); the %d-step figures compare the mixed GPU path with "
                                         "the FP64 GPU path" % (n_o, args.error_steps)})
            orc = None

    if orc is not None:  # comparison skipped: do not leave the oracle process behind
        orc[0].terminate()
        orc[0].join()
    rtrip = None
    if rank == 0 and ws == 1 and not args.no_roundtrip:
        rtrip = roundtrip_leg(local)
    ensl = None
    if rank == 0 and ws == 1 and not args.no_ensemble:
        ensl = ensemble_leg(local)
    gradl = None
    if rank == 0 and ws == 1 and not args.no_gradient:
        gradl = gradient_leg(local)

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        v = oracle_steps(cfg, args.cpu_steps)
        cpu = {"value": v, "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
               "sample": "%d steady-state steps of the FP64 numpy/scipy oracle at %s (zeroed AB/ETD "
                         "history, same arithmetic as a steady step)" % (args.cpu_steps, cfg.name)}

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64" if not split else "bf16x%d-split/f32/f64" % args.slices,
                "data": "synthetic (seeded q-vortex + spectral perturbation)",
                "config": {"workload": cfg.name, "grid": [cfg.nr, cfg.nth, cfg.nx],
                           "chops": [cfg.nrchop, cfg.ntchop, cfg.nxchop],
                           "scheme": "ETD2AB-CN" if not cfg.adams else "AB2-CN", "dt": cfg.dt,
                           "precision": args.precision, "split_slices": args.slices if split else None,
                           "graph": True, "parallelism": "replicas x%d" % ws,
                           "l2": "inputs larger than L2 (several GB touched per step)"},
                "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": 3 * nbytes,
                        "d2h_bytes_per_step": 3 * nbytes, "api": "mlegs_run_host",
                        "separate_calls_value": e2e_calls},
                "gpu_launches": int(launches), "precision_comparison": compare,
                "roofline": roof, "kernels": kernels, "transform_roundtrip": rtrip, "ensemble": ensl,
                "gradient": gradl,
                "cpu_baseline": cpu,
                "clocks": clk.summary()}
        print(json.dumps(line), flush=True)


DOMINANT = "phys_nonlin"  # the fused physical kernel in the form the steady step runs


def main():
    args = parse()
    from mlegs_b200.inputs import CONFIGS
    cfg = CONFIGS[args.config]
    ws, rank, local = dist_setup(args.gpus)
    try:
        if args.impl == "reference":
            run_reference(args, cfg, ws, rank)
        else:
            run_ours(args, cfg, ws, rank, local)
    finally:
        if ws > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()

"""Benchmark of the BSSN RHS + RK4 step on B200.

    python bench.py [--gpus N --steps K --warmup W] [--impl b200|reference] [--n 128]

A step is one RK4 step (4 fused RHS+KO+stage launches, enforcement fused
into the last, 1 time-advance launch) of the 128^3-interior (+3 ghosts,
134^3 array, 462 MB state) q = 1/10 Brill-Lindquist workload on [-8,8]^3,
dt = 0.25 dx, KO sigma 0.1 (order 6). The metric is Mpoint-updates/s:
interior points x 4 RHS evaluations per step / time (the reference's unit,
3D/src/bssn3d/profile_regime.py:230). Inputs stay in HBM between steps and
are larger than L2 (126 MB).

For N > 1 (under torchrun) every rank evolves its own replica by default:
weak scaling, value = total work of all ranks / max-over-ranks time. With
``--split slab`` the one block is cut into N x-slabs instead
(``bssn3d_b200.slabs``: per stage, each rank's fused stage launch on its
slab, then its halo planes from the neighbours over NCCL): strong scaling,
value = the block's work / max-over-ranks time.

``--impl reference`` times the reference's own CPU algebra
(oracle/_ref/libdendro_ref.so, compiled from the reference's vendored
Dendro-GR CSE) with the oracle's restated stencils, KO, RK4 and enforcement
on all host threads, on a bounded sample of the same workload.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT / "integer-schemes_b200"))
sys.path.insert(0, str(ROOT))

import numpy as np  # noqa: E402

METRIC = "BSSN RHS Mpoint-updates/s (RK4 step, fused FP64)"
UNIT = "Mpoint-updates/s"
FLOPS_PER_POINT = 6714      # algorithmic FP64 flops per RHS point-update (oracle/count_flops.py): algebra 4,278 + derivatives 2,436
KO_FLOPS_PER_POINT = 936    # 24 fields x 3 axes x (7 taps: 7 mul + 6 add)
STAGE_BYTES = 960           # read Y, U, ACC; write ACC, Y_next (5 x 24 x 8 B)
# DRAM bytes per evaluated point of one stage launch, dram__bytes_read.sum +
# dram__bytes_write.sum from an ncu capture of the stage-1 kernel on the 102^3
# case, scaled to a launch by its points (the capture is named here)
TRAFFIC_BYTES_PER_POINT = 963
TRAFFIC_SOURCE = "ncu capture, profiles/stream_kernel_stage_102.md (963 B per evaluated point)"
LAST_STAGE_BYTES = 768      # read Y, U, ACC; write U_new


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--n", type=int, default=128, help="interior points per axis")
    ap.add_argument("--workload", default="bl128", choices=["bl128", "amr3", "amr4", "ozaki192"],
                    help="bl128: one uniform block (default, --n sets its size); amr3/amr4: the "
                         "600- and 2000-block Brill-Lindquist block lists; ozaki192: the RHS with "
                         "INT8 tensor-core derivatives on the 192^3 block, k = 5..8")
    ap.add_argument("--integrator", default="rk4", choices=["rk4", "rk4_2_1", "rk4_2_2"],
                    help="uniform workload: RK4 or a 2-step/3-stage MSRK integrator")
    ap.add_argument("--split", default="replicas", choices=["replicas", "slab"],
                    help="bl128 at N > 1: N independent replicas (weak scaling, the default) or the one "
                         "block cut into N x-slabs with a halo exchange per stage (strong scaling)")
    ap.add_argument("--ghosts", default="exchange", choices=["exchange", "evolve"],
                    help="block lists: refill ghosts from other blocks each stage, or evolve them")
    ap.add_argument("--track", type=int, default=0,
                    help="after timing, evolve this many more steps and record the constraint norms")
    ap.add_argument("--track-every", type=int, default=10)
    ap.add_argument("--blocks", type=int, default=0, help="amr3/amr4: block count instead of 600/2000 (small cases)")
    ap.add_argument("--fill-split", action="store_true",
                    help="amr3/amr4 with ghost exchange: also time each level's fill with its op list whole, "
                         "its copy boxes alone and its prolongation boxes alone (NVTX ranges 'fill L<level> "
                         "<part>' around each list's launches)")
    ap.add_argument("--ozaki-k", default="0",
                    help="ozaki192: one digit count instead of k = 5..8; amr3/amr4: evolve through the "
                         "Ozaki INT8 derivative path with this many digit planes (0 = float64 stencils, "
                         "auto = the smallest k whose rate stays within 1e-10 of float64 on this block list)")
    ap.add_argument("--ozaki-n", type=int, default=192, help="ozaki192: interior points per axis")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-fp64-peak", action="store_true")
    ap.add_argument("--no-stage-timing", action="store_true")
    ap.add_argument("--no-ozaki", action="store_true",
                    help="bl128: skip the Ozaki INT8 RHS measured beside the float64 one")
    ap.add_argument("--no-m4", action="store_true",
                    help="bl128: skip the reference's M4 CUDA RHS measured beside the fused one")
    return ap.parse_args()


def fill_split(evo, pool, Y, stream, dev, reps=10):
    """Per level: the fill's op list timed whole, its copy boxes alone and its
    prolongation boxes alone (each list uploaded through bssn_b200_fill_plan,
    one warm-up launch, then ``reps`` launches between CUDA events, each list
    inside the NVTX range 'fill L<level> <part>')."""
    import ctypes
    import torch
    from bssn3d_b200 import _lib
    from bssn3d_b200.ghosts import PROLONG, FillOp, W_MID
    lib = _lib.load()
    wmid = (ctypes.c_double * 6)(*W_MID)
    sp = stream.cuda_stream

    def upload(ops):
        arr = (FillOp * len(ops))(*ops)
        total = lib.bssn_b200_fill_plan(ctypes.addressof(arr), len(ops), int(pool.size))
        if total < 0:
            _lib.check(_lib.EINVAL)
        raw = bytes(memoryview(arr).cast("B"))
        return torch.frombuffer(bytearray(raw), dtype=torch.uint8).to(dev), len(ops), int(total)

    def timed(ops, name):
        dv, nops, npts = upload(ops)

        def run():
            _lib.check(lib.bssn_b200_fill(sp, Y.data_ptr(), dv.data_ptr(), nops, npts,
                                          ctypes.cast(wmid, ctypes.c_void_p)))
        torch.cuda.nvtx.range_push(name)
        run()
        torch.cuda.synchronize(dev)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(reps):
            run()
        b.record(stream)
        b.synchronize()
        torch.cuda.nvtx.range_pop()
        return round(a.elapsed_time(b) / reps, 4), npts

    out = []
    for lvl, ops in evo.plan.fill_lists:
        row = {"level": lvl, "ops": len(ops)}
        row["whole_ms"], row["points"] = timed(list(ops), f"fill L{lvl} whole")
        for part, keep in (("copy", lambda o: o.kind != PROLONG), ("prolong", lambda o: o.kind == PROLONG)):
            sel = [o for o in ops if keep(o)]
            if sel:
                row[f"{part}_ms"], row[f"{part}_points"] = timed(sel, f"fill L{lvl} {part}")
        out.append(row)
    return out


# ---------------------------------------------------------------- clocks
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []
        self._t = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except (FileNotFoundError, OSError):
            self.proc = None
            return
        self._t = threading.Thread(target=self._read, daemon=True)
        self._t.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self._t:
            self._t.join(timeout=2)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------- helpers
def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def cpu_threads():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def reference_step_sample(n_interior: int, planes: int = 8):
    """A bounded sample of the workload for the CPU reference: `planes`
    interior x-planes (+3 ghosts each side) of the full-size y-z cross section."""
    from bssn3d_b200 import initial_data as ID
    from bssn3d_b200.fused_rhs import pack_S
    grid, U, dt = ID.workload(1, n=n_interior)
    ng = grid.ng
    mid = U.shape[1] // 2
    Us = np.ascontiguousarray(U[:, mid - planes // 2 - ng: mid + planes // 2 + ng])
    S = pack_S(2.0, 0.06, dt, grid.dx, 0.6, 20.0, 0.0, (1, 1, 1, 1), (1, 0), grid.dy, grid.dz)
    interior = planes * n_interior * n_interior
    return Us, S, interior


def run_cpu_reference(U, S, steps, warmup, threads):
    """RK4 steps of evolve.py:125-137 with the reference's compiled algebra;
    the stage combinations run as multithreaded torch CPU operations on the
    same host threads as the OpenMP algebra."""
    import torch
    from oracle import oracle as O
    os.environ["OMP_NUM_THREADS"] = str(threads)
    torch.set_num_threads(threads)
    dt = float(S[2])
    g = (S[13], S[14], S[15])
    T = torch.from_numpy

    def rate(Y, tt):
        S2 = S.copy()
        S2[6] = tt
        r = T(O.ref_rhs(Y, S2, nthreads=threads))
        r.add_(T(O.ko(Y, *g, 0.1, 6)))
        return r

    def axpy(u, a, k):
        return torch.add(T(u), k, alpha=a).numpy()

    def step(U, t):
        k1 = rate(U, t)
        k2 = rate(axpy(U, 0.5 * dt, k1), t + 0.5 * dt)
        k3 = rate(axpy(U, 0.5 * dt, k2), t + 0.5 * dt)
        k4 = rate(axpy(U, dt, k3), t + dt)
        acc = k1.add_(k2, alpha=2.0).add_(k3, alpha=2.0).add_(k4)
        return O.enforce(axpy(U, dt / 6.0, acc))

    t = 0.0
    for _ in range(warmup):
        U = step(U, t)
        t += dt
    times = []
    for _ in range(steps):
        t0 = time.perf_counter()
        U = step(U, t)
        times.append(time.perf_counter() - t0)
        t += dt
    return times


def measure_fp64_peak(torch, dev):
    """cuBLAS DGEMM throughput on this GPU (TFLOP/s), the FP64 roofline denominator."""
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device=dev)
    b = torch.randn(n, n, dtype=torch.float64, device=dev)
    c = torch.empty_like(a)
    for _ in range(2):
        torch.matmul(a, b, out=c)
    torch.cuda.synchronize(dev)
    best = 0.0
    for _ in range(3):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b, out=c)
        e1.record()
        e1.synchronize()
        best = max(best, 2.0 * n ** 3 / (e0.elapsed_time(e1) * 1e-3) / 1e12)
    del a, b, c
    torch.cuda.empty_cache()
    return best


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return json.loads(p.read_text()), "measured"
        except ValueError:
            pass
    return {"hbm_gbs": 6650.0}, "fallback"


# ---------------------------------------------------------------- arms
def bench_reference(args):
    world, rank, _ = dist_env()
    if rank != 0:
        return
    threads = cpu_threads()
    U, S, interior = reference_step_sample(args.n)
    times = run_cpu_reference(U, S, args.steps, args.warmup, threads)
    t = sum(times)
    value = interior * 4 * args.steps / t / 1e6
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * t / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"Brill-Lindquist q=1/10, {args.n}^3 interior +3 ghosts on [-8,8]^3, "
                               f"RK4 step, KO sigma 0.1 order 6",
                   "sample": f"8 interior x-planes of the {args.n}^2 cross-section (+3 ghosts)"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "reference",
                         "sample": f"RK4 steps of an 8x{args.n}x{args.n}-interior slab: reference "
                                   f"Dendro-GR algebra (oracle/_ref) + restated stencils/KO/enforce"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def bench_b200(args):
    import torch
    world, rank, local = dist_env()
    if world > 1:
        import torch.distributed as dist
        torch.cuda.set_device(local)
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120),
                                device_id=torch.device(f"cuda:{local}"))
    dev = torch.device(f"cuda:{local}")
    torch.cuda.set_device(dev)

    from bssn3d_b200 import initial_data as ID
    from bssn3d_b200.evolve import BSSNEvolution
    from bssn3d_b200.state import BSSNState

    grid, U_host, dt = ID.workload(1, n=args.n)
    interior = grid.interior_points
    npts = int(np.prod(grid.shape))
    msrk = args.integrator != "rk4"
    nstage = 3 if msrk else 4
    evo = BSSNEvolution(grid, ko_sigma=0.1, bc="none", ko_order=6, integrator=args.integrator)
    U0 = torch.from_numpy(U_host).to(dev)
    S0 = evo._S(0.0, dt, dev)
    if msrk:
        # the RK4 start that keeps f(y_0), then the MSRK step captured as a graph
        KP = torch.empty_like(U0)
        U1 = U0.clone()
        evo._startup_inplace(U1, KP, S0)
        evo._advance_time(S0)
        graph, U_g, S_g, K_g = evo.capture_msrk(U1, S0, KP)
        args.no_stage_timing = True
        args.no_e2e = True
    else:
        graph, U_g, S_g = evo.capture(U0, S0)

    def barrier():
        if world > 1:
            import torch.distributed as dist
            dist.barrier()
        torch.cuda.synchronize(dev)

    for _ in range(args.warmup):
        graph.replay()
    barrier()
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)   # let the sampler come up before the timed region
    stream = torch.cuda.current_stream(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        graph.replay()
    e1.record(stream)
    barrier()
    clk = clocks.stop()
    ms = e0.elapsed_time(e1)
    if world > 1:
        import torch.distributed as dist
        t = torch.tensor([ms], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    finite = bool(torch.isfinite(U_g).all().item())
    tracked = None
    if args.track > 0:
        # a fresh run from t = 0 on its own captured step
        from bssn3d_b200.constraints import ConstraintSolver
        cs = ConstraintSolver(grid)
        S2 = evo._S(0.0, dt, dev)
        if msrk:
            K2, U2 = torch.empty_like(U0), U0.clone()
            evo._startup_inplace(U2, K2, S2)
            evo._advance_time(S2)
            g2, U2g, S2g, K2g = evo.capture_msrk(U2, S2, K2)   # the state after the RK4 start
        else:
            g2, U2g, S2g = evo.capture(U0, S2)

        def advance(k):
            for _ in range(k):
                g2.replay()
        offset = 1 if msrk else 0
        tracked = [[r[0] + offset] + r[1:]
                   for r in track_constraints(advance, lambda: cs.l2(U2g), args.track, args.track_every)]
        del g2

    # per-launch stage-kernel durations (roofline), on the launching stream
    stage_ms = []
    b = evo._buffers(U_g)
    for s in (range(4) if not args.no_stage_timing else []):
        Y = U_g if s == 0 else (b["Ya"] if s in (1, 3) else b["Yb"])
        Yn = {0: b["Ya"], 1: b["Yb"], 2: b["Ya"], 3: b["Yb"]}[s]   # stage 3 timed out of place
        durs = []
        for _ in range(3):
            a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a0.record(stream)
            evo._stage(s, U_g, Y, b["ACC"], Yn, S_g)
            a1.record(stream)
            a1.synchronize()
            durs.append(a0.elapsed_time(a1))
        stage_ms.append(statistics.median(durs))

    # end to end through the public API with host buffers: every step copies
    # its input state in from pinned host memory and its result out, the
    # copies of neighbouring steps overlapped with the step's compute
    e2e = None
    if not args.no_e2e:
        from bssn3d_b200.evolve import HostStepPipeline
        pipe = HostStepPipeline(evo, U_host.shape, dt, 0.0, dev)
        host_in = torch.from_numpy(U_host).pin_memory()
        host_out = torch.empty_like(host_in).pin_memory()
        pipe.run([host_in] * 3, [host_out] * 3)
        barrier()
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        f0.record(stream)
        pipe.run([host_in] * args.steps, [host_out] * args.steps)
        f1.record(stream)
        barrier()
        ems = f0.elapsed_time(f1)
        if world > 1:
            import torch.distributed as dist
            t = torch.tensor([ems], dtype=torch.float64, device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ems = float(t.item())
        nbytes = U_host.nbytes
        e2e = {"value": interior * 4 * args.steps * world / (ems * 1e-3) / 1e6, "unit": UNIT,
               "h2d_bytes_per_step": nbytes, "d2h_bytes_per_step": nbytes,
               "ms_per_step": ems / args.steps,
               "path": "evolve.HostStepPipeline: per step, pinned host state in, one RK4 step (C ABI "
                       "bssn_b200_rk4_stage, captured), result out; copies overlapped with the "
                       "neighbouring steps' compute"}
        del pipe
        # the host link alone, the ceiling of the end-to-end rate: one state in
        # and one state out at the same time, on two streams
        s_in, s_out = torch.cuda.Stream(dev), torch.cuda.Stream(dev)
        d_in = torch.empty(U_host.shape, dtype=torch.float64, device=dev)
        d_out = U_g.clone()

        def link_once():
            s_in.wait_stream(stream)
            s_out.wait_stream(stream)
            with torch.cuda.stream(s_in):
                d_in.copy_(host_in, non_blocking=True)
            with torch.cuda.stream(s_out):
                host_out.copy_(d_out, non_blocking=True)
            stream.wait_stream(s_in)
            stream.wait_stream(s_out)
        link_once()
        torch.cuda.synchronize(dev)
        l0, l1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        reps = 5
        l0.record(stream)
        for _ in range(reps):
            link_once()
        l1.record(stream)
        l1.synchronize()
        link_ms = l0.elapsed_time(l1) / reps
        dev_ms = ms / args.steps
        e2e["link"] = {"ms_per_state_each_way": link_ms, "gbs_each_way": nbytes / (link_ms * 1e-3) / 1e9,
                       "bound_value": interior * 4 * world / (max(link_ms, dev_ms) * 1e-3) / 1e6,
                       "what": "one state copied in (pinned host to device) and one out at the same time on "
                               "two streams; bound_value = the rate at max(link time, device step time)"}
        e2e["frac_of_bound"] = e2e["value"] / e2e["link"]["bound_value"]
        del d_in, d_out

    # the Ozaki INT8 half of the metric and the reference's M4 CUDA kernel, on
    # the same state (outside the timed region)
    ozaki = m4 = None
    if not args.no_ozaki and not msrk:
        k_leg = int(args.ozaki_k) if args.ozaki_k.isdigit() and int(args.ozaki_k) > 0 else 6
        ozaki = ozaki_leg(torch, dev, U0, grid, dt, k_leg, max(args.warmup, 3))
    if not args.no_m4 and not msrk:
        m4 = m4_leg(torch, dev, U0, grid, dt, max(args.warmup, 3))

    peaks, peak_kind = measured_peaks()
    fp64_peak = measure_fp64_peak(torch, dev) if (rank == 0 and not args.no_fp64_peak) else None

    value = interior * 4 * args.steps * world / (ms * 1e-3) / 1e6
    mean_stage = statistics.mean(stage_ms[:3]) if stage_ms else ms / args.steps / nstage
    # algorithmic bytes and flops of the interior point-updates a launch delivers
    # (the unit the metric credits); the kernel also evaluates the ghost points
    achieved_gbs = interior * STAGE_BYTES / (mean_stage * 1e-3) / 1e9
    flops = interior * (FLOPS_PER_POINT + KO_FLOPS_PER_POINT)
    achieved_tf = flops / (mean_stage * 1e-3) / 1e12
    roofline = {"bound": "hbm", "achieved": achieved_gbs, "peak": peaks.get("hbm_gbs"),
                "unit": "GB/s", "frac": achieved_gbs / peaks.get("hbm_gbs"),
                "traffic": TRAFFIC_BYTES_PER_POINT * npts, "peak_source": f"{peak_kind} hbm_gbs",
                "traffic_source": TRAFFIC_SOURCE,
                "kernel": "bssn::stream_kernel<3, MODE_STAGE, Shape<4,4,16>> (stages 0-2)",
                "bytes_per_point_update": STAGE_BYTES, "point_updates_per_launch": interior,
                "points_evaluated_per_launch": npts, "launch_ms": mean_stage}
    roofline_fp64 = {"bound": "fp64", "achieved": achieved_tf, "peak": fp64_peak,
                     "unit": "TFLOP/s", "frac": (achieved_tf / fp64_peak) if fp64_peak else None,
                     "peak_source": "cuBLAS DGEMM 8192^3 measured in this run",
                     "flops_per_point_update": FLOPS_PER_POINT + KO_FLOPS_PER_POINT}
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            threads = cpu_threads()
            Us, S, inter = reference_step_sample(args.n)
            times = run_cpu_reference(Us, S, 2, 1, threads)
            cpu = {"value": inter * 4 * len(times) / sum(times) / 1e6, "unit": UNIT,
                   "cores": threads, "kind": "reference",
                   "sample": f"2 RK4 steps of an 8x{args.n}x{args.n}-interior slab: reference "
                             f"Dendro-GR algebra (oracle/_ref) + restated stencils/KO/enforce"}
        except (FileNotFoundError, OSError) as exc:
            cpu = {"value": None, "unit": UNIT, "cores": 0, "kind": "reference",
                   "sample": f"unavailable: {exc}"}
    metric = METRIC
    if msrk:
        # a step advances the solution as far as an RK4 step: count it like one
        metric = f"BSSN RK4-equivalent Mpoint-updates/s ({args.integrator} MSRK step, fused FP64)"
    line = {
        "metric": metric, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": f"Brill-Lindquist q=1/10, {args.n}^3 interior +3 ghosts on [-8,8]^3, "
                               + (f"{args.integrator} MSRK step (3 fused RHS+KO+stage launches)" if msrk else
                                  "RK4 step (4 fused RHS+KO+stage launches)") + ", KO sigma 0.1 order 6",
                   "integrator": args.integrator,
                   "array": list(grid.shape), "state_bytes": int(U_host.nbytes),
                   "l2": "inputs larger than L2 (462 MB state)", "parallelism": f"replicas x{world}"},
        "clocks": clk, "gpu_launches": (nstage + 1) * args.steps, "finite": finite,
        "stage_ms": stage_ms, "roofline": roofline, "roofline_fp64": roofline_fp64,
        "e2e": e2e, "cpu_baseline": cpu, "ozaki": ozaki, "m4_reference": m4,
        "xla_reference": {"value": None, "unavailable": XLA_UNAVAILABLE},
    }
    if tracked is not None:
        line["constraints"] = tracked
    del graph
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


M4_LIB = ROOT / "baseline" / "_ref" / "m4" / "libm4_rhs.so"
XLA_UNAVAILABLE = ("unavailable on this box: the reference's XLA-verbatim path needs jax 0.9.2, which is "
                   "not installed on the B200 machine (import jax -> ModuleNotFoundError) and cannot be "
                   "installed offline")


def _timed_rhs(torch, dev, fn, reps: int) -> float:
    """ms per call: 3 warm-up calls, then the median of 5 batches of ``reps``
    calls, CUDA events on the current stream."""
    stream = torch.cuda.current_stream(dev)
    for _ in range(3):
        fn()
    torch.cuda.synchronize(dev)
    meds = []
    for _ in range(5):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(reps):
            fn()
        b.record(stream)
        b.synchronize()
        meds.append(a.elapsed_time(b) / reps)
    return statistics.median(meds)


def _bench_S(torch, dev, grid, dt):
    from bssn3d_b200.fused_rhs import device_scalars, pack_S
    return device_scalars(pack_S(2.0, 0.06, dt, grid.dx, 0.6, 20.0, 0.0, (1, 1, 1, 1), (1, 0),
                                 grid.dy, grid.dz), dev)


def m4_leg(torch, dev, U, grid, dt, reps: int):
    """The reference's own M4 fused CUDA RHS (3D/src/bssn3d/cuda/rhs_fused.cu,
    generated by its gen_fused.py and compiled for sm_100a by
    baseline/m4/build_m4.py) on the bench state, beside this project's fused
    RHS (bssn_b200_rhs) on the same state: ms per RHS, Mpoint-updates/s of
    interior points, and the per-field difference between the two outputs.
    The M4 kernel is 2.28x the reference's XLA-verbatim RHS on its own H100
    measurement (README.md:6-8), the closest GPU anchor of the reference that
    runs here."""
    import ctypes
    from bssn3d_b200.fused_rhs import rhs_tensor
    if not M4_LIB.exists():
        return {"value": None, "unavailable": f"{M4_LIB.relative_to(ROOT)} not built "
                                              "(python baseline/m4/build_m4.py where the reference tree is)"}
    lib = ctypes.CDLL(str(M4_LIB))
    lib.m4_rhs.argtypes = [ctypes.c_void_p] * 4 + [ctypes.c_int] * 4
    lib.m4_attributes.argtypes = [ctypes.POINTER(ctypes.c_int)] * 2
    S = _bench_S(torch, dev, grid, dt)
    _, Sx, Sy, Sz = U.shape
    out_m4 = torch.empty_like(U)
    stream = torch.cuda.current_stream(dev).cuda_stream

    def m4():
        rc = lib.m4_rhs(stream, U.data_ptr(), S.data_ptr(), out_m4.data_ptr(), Sx, Sy, Sz, 128)
        if rc != 0:
            raise RuntimeError(f"M4 launch failed: cudaError {rc}")
    out_b = torch.empty_like(U)
    m4_ms = _timed_rhs(torch, dev, m4, reps)
    b_ms = _timed_rhs(torch, dev, lambda: rhs_tensor(U, S, out_b), reps)
    num = (out_m4 - out_b).reshape(24, -1).abs().amax(dim=1)
    den = out_b.reshape(24, -1).abs().amax(dim=1).clamp_min(1e-300)
    err = torch.where(num == 0, torch.zeros_like(num), num / den)
    regs, local = ctypes.c_int(0), ctypes.c_int(0)
    lib.m4_attributes(ctypes.byref(regs), ctypes.byref(local))
    interior = grid.interior_points
    m4_rate = interior / (m4_ms * 1e-3) / 1e6
    b_rate = interior / (b_ms * 1e-3) / 1e6
    del out_m4, out_b
    torch.cuda.empty_cache()
    return {"value": m4_rate, "unit": UNIT, "ms_per_rhs": m4_ms, "registers": regs.value,
            "local_bytes_per_thread": local.value, "fused_value": b_rate, "fused_ms_per_rhs": b_ms,
            "fused_over_m4": m4_ms / b_ms, "max_field_diff_vs_fused": float(err.max()),
            "what": "one RHS of the bench state (no KO): the reference's M4 kernel "
                    "(baseline/_ref/m4/libm4_rhs.so, 1 thread per padded point, 128-thread blocks) "
                    "vs bssn_b200_rhs"}


def ozaki_leg(torch, dev, U, grid, dt, k: int, reps: int):
    """The RHS of the bench state through the Ozaki INT8 derivative path (k
    digit planes, tcgen05 kind::i8, float64 algebra) beside the fused float64
    RHS of the same state: time per RHS (CUDA events, median of 5 batches),
    Mpoint-updates/s of interior points, each field's max|oz - fp64| /
    max|fp64|, and bit-identity over 5 runs."""
    from bssn3d_b200.fused_rhs import rhs_tensor
    from bssn3d_b200.ozaki import OzakiDerivatives
    S = _bench_S(torch, dev, grid, dt)
    interior = grid.interior_points
    ref = rhs_tensor(U, S)
    out_fp = torch.empty_like(ref)
    fp_ms = _timed_rhs(torch, dev, lambda: rhs_tensor(U, S, out_fp), reps)
    oz = OzakiDerivatives(U.shape[1:], k, device=dev)
    oz_ms = _timed_rhs(torch, dev, lambda: oz.rhs(U, S), reps)
    got = oz.rhs(U, S)
    same = all(torch.equal(oz.rhs(U, S), got) for _ in range(4))
    oz.check()
    num = (got - ref).reshape(24, -1).abs().amax(dim=1)
    den = ref.reshape(24, -1).abs().amax(dim=1).clamp_min(1e-300)
    err = torch.where(num == 0, torch.zeros_like(num), num / den)
    del oz, got, ref, out_fp
    torch.cuda.empty_cache()
    fp_rate = interior / (fp_ms * 1e-3) / 1e6
    oz_rate = interior / (oz_ms * 1e-3) / 1e6
    return {"k": k, "value": oz_rate, "unit": UNIT, "ms_per_rhs": oz_ms,
            "fp64_value": fp_rate, "fp64_ms_per_rhs": fp_ms, "ratio_to_fp64": oz_rate / fp_rate,
            "max_field_err_vs_fp64": float(err.max()), "worst_field": int(err.argmax()),
            "per_field_err_vs_fp64": [float(x) for x in err.cpu()],
            "bit_identical_5_runs": same, "bar": 1e-10,
            "what": "one RHS of the bench state: Ozaki INT8 derivatives (bssn_b200_ozaki_derivatives) + "
                    "float64 algebra (bssn_b200_rhs_algebra) vs the fused float64 RHS (bssn_b200_rhs)"}


def track_constraints(advance, norms, total: int, every: int):
    """[[steps, H, M], ...]: the interior constraint norms at step 0 and after
    every ``every`` further steps, ``total`` steps in all."""
    out = [[0] + list(norms())]
    done = 0
    while done < total:
        k = min(every, total - done)
        advance(k)
        done += k
        out.append([done] + list(norms()))
    return out


def _oz_kind(f, axis):
    """Pass kind of field f along axis in the batched Ozaki bundle (ozaki.cu KINDS)."""
    d2 = f in (0, 1) or 3 <= f < 12
    return (0 if d2 else 1) if axis == 0 else ((2 if d2 else 3) if axis == 1 else 4)


def _pool_drift(pool, A, B):
    """Per field, over the interiors of all blocks: max |A - B| / max |B|."""
    import torch
    num = torch.zeros(24, dtype=torch.float64, device=A.device)
    den = torch.zeros(24, dtype=torch.float64, device=A.device)
    for i, b in enumerate(pool.blocks):
        o = int(pool.offsets[i])
        g = b.ng
        a = A[o:o + 24 * b.points].view((24,) + tuple(b.shape))[:, g:-g, g:-g, g:-g]
        r = B[o:o + 24 * b.points].view((24,) + tuple(b.shape))[:, g:-g, g:-g, g:-g]
        num = torch.maximum(num, (a - r).abs().amax(dim=(1, 2, 3)))
        den = torch.maximum(den, r.abs().amax(dim=(1, 2, 3)))
    return [float(x) for x in (num / den.clamp_min(1e-300)).cpu()]


def bench_amr(args):
    """A block-list workload: one persistent stage launch per RK4 stage over
    every block (plus the ghost fill per level with ghosts="exchange"), the
    step captured as a graph; value counts 4 point-updates per interior point
    per step. Replicas under torchrun."""
    import torch
    world, rank, local = dist_env()
    if world > 1:
        import torch.distributed as dist
        torch.cuda.set_device(local)
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120),
                                device_id=torch.device(f"cuda:{local}"))
    dev = torch.device(f"cuda:{local}")
    torch.cuda.set_device(dev)
    from bssn3d_b200 import amr

    index = int(args.workload[-1])
    blocks, punct, dt = amr.workload(index, count=args.blocks or None)
    pool = amr.BlockPool(blocks)
    U0 = torch.from_numpy(pool.initial_state(punct, seed=0)).to(dev)
    oz_k = int(args.ozaki_k) if args.ozaki_k.isdigit() else 0
    k_choice = None
    if args.ozaki_k == "auto":
        from bssn3d_b200.ozaki import choose_k
        chosen, k_errs = choose_k(pool, U0, dt, ghosts=args.ghosts, device=dev)
        oz_k = chosen or 8
        k_choice = {"chosen": chosen, "worst_field_err_by_k": {str(k): v for k, v in k_errs.items()},
                    "bar": 1e-10, "what": "RHS (first-stage accumulator, no KO) vs the float64 block path, per field "
                                                 "max|diff| / max|fp64| over the interiors"}
        torch.cuda.empty_cache()
    t_plan = time.time()
    if oz_k:
        from bssn3d_b200.ozaki import BatchedOzakiEvolution
        evo = BatchedOzakiEvolution(pool, k=oz_k, ko_sigma=0.1, ko_order=6, device=dev, ghosts=args.ghosts)
    else:
        evo = amr.BatchedEvolution(pool, ko_sigma=0.1, ko_order=6, variant=0, device=dev, ghosts=args.ghosts)
    t_plan = time.time() - t_plan
    tune = {} if oz_k else amr.autotune(evo, U0, dt)
    graph, U_g, S_g = evo.capture(U0, evo.scalars(0.0, dt))

    def barrier():
        if world > 1:
            import torch.distributed as dist
            dist.barrier()
        torch.cuda.synchronize(dev)

    for _ in range(args.warmup):
        graph.replay()
    barrier()
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    stream = torch.cuda.current_stream(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        graph.replay()
    e1.record(stream)
    barrier()
    clk = clocks.stop()
    ms = e0.elapsed_time(e1)
    if world > 1:
        import torch.distributed as dist
        t = torch.tensor([ms], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    finite = bool(torch.isfinite(U_g).all().item())
    interior = pool.interior_points
    value = interior * 4 * args.steps * world / (ms * 1e-3) / 1e6
    # where a stage's time goes, timed alone after the timed region (CUDA events)
    def ev_ms(fn, reps=5):
        fn()
        torch.cuda.synchronize(dev)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(reps):
            fn()
        b.record(stream)
        b.synchronize()
        return round(a.elapsed_time(b) / reps, 3)
    bufs = evo.buffers(U_g)
    Y_t = U_g.clone()
    breakdown = {"fill_ms_per_stage": ev_ms(lambda: evo.fill(Y_t)) if evo.dplan is not None else 0.0,
                 "stage_ms": ev_ms(lambda: evo.stage(1, U_g, Y_t, bufs["ACC"], bufs["Yb"], S_g))}
    if oz_k:
        breakdown["derivative_bundle_ms"] = ev_ms(lambda: evo.derivatives(Y_t, S_g))
    del Y_t
    if args.fill_split and evo.plan is not None:
        Y_s = U_g.clone()
        breakdown["fill_split"] = fill_split(evo, pool, Y_s, stream, dev)
        del Y_s
    fills = len(evo.dplan.fill) if evo.dplan is not None else 0
    ghost_counts = evo.plan.counts if evo.plan is not None else None
    variant = evo.variant
    per_stage = 1 + fills
    if oz_k:
        evo.check()
        # the bundle's passes with tiles, one stage launch
        per_stage = fills + 1 + sum(1 for f in range(24) for a in range(3)
                                    if evo.ntiles_kind[_oz_kind(f, a)] > 0) + 33
    del graph
    # the comparison point: the same step with one stage launch per block
    per_block = None
    if not oz_k:
        gpb, _, _ = evo.capture_per_block(U0, evo.scalars(0.0, dt))
        for _ in range(max(args.warmup, 1)):
            gpb.replay()
        torch.cuda.synchronize(dev)
        p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        p0.record(stream)
        for _ in range(args.steps):
            gpb.replay()
        p1.record(stream)
        p1.synchronize()
        pms = p0.elapsed_time(p1) / args.steps
        per_block = {"ms_per_step": pms, "value": interior * 4 / (pms * 1e-3) / 1e6, "unit": UNIT,
                     "stage_launches_per_step": 4 * len(evo.active),
                     "persistent_over_per_block": pms / (ms / args.steps),
                     "what": "the same captured step with one batched-stage launch per block (one-entry "
                             "block tables, same tile variant and fills) instead of one persistent launch"}
        del gpb
    tracked = tracked_fp64 = drift = None
    if args.track > 0:
        # a fresh run from t = 0 on its own captured step
        g2, U2g, S2g = evo.capture(U0, evo.scalars(0.0, dt))

        def advance(k):
            for _ in range(k):
                g2.replay()
        tracked = track_constraints(advance, lambda: evo.constraint_norms(U2g), args.track, args.track_every)
        del g2
        if oz_k:
            # the same run on the float64 stencils of the block path
            evo.check()
            U_oz = U2g.clone()
            del evo, U2g, U_g
            torch.cuda.empty_cache()
            fp = amr.BatchedEvolution(pool, ko_sigma=0.1, ko_order=6, variant=0, device=dev, ghosts=args.ghosts)
            g3, U3g, _ = fp.capture(U0, fp.scalars(0.0, dt))

            def advance_fp(k):
                for _ in range(k):
                    g3.replay()
            tracked_fp64 = track_constraints(advance_fp, lambda: fp.constraint_norms(U3g), args.track,
                                             args.track_every)
            del g3
            drift = _pool_drift(pool, U_oz, U3g)
    metric = METRIC.replace("RK4 step", "RK4 step over a block list")
    if oz_k:
        metric += f", Ozaki INT8 derivatives k={oz_k} + FP64 algebra"
    line = {
        "metric": metric, "value": value, "unit": UNIT,
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"{len(blocks)} Brill-Lindquist blocks, {len(set(b.level for b in blocks))} levels "
                               f"(amr.workload({index})), interiors 16^3/24^3/32^3 +3 ghosts",
                   "ghosts": args.ghosts, "interior_points": interior, "points": pool.points,
                   "state_bytes": int(pool.size * 8), "variant": None if oz_k else variant,
                   "block_order": None if oz_k else evo.order,
                   "autotune_ms": {f"{k[0]},{k[1]}": v for k, v in tune.items()},
                   "autotune": "tile variant x block order, one captured step each; fastest kept",
                   "plan_s": round(t_plan, 2), "parallelism": f"replicas x{world}"},
        "clocks": clk, "gpu_launches": (4 * per_stage + 1) * args.steps, "finite": finite,
        "ghost_points": ghost_counts, "breakdown": breakdown,
        "constraints": tracked, "roofline": None, "e2e": None, "cpu_baseline": None,
        "per_block_launches": per_block,
    }
    if oz_k:
        line["ozaki"] = {"k": oz_k, "k_choice": k_choice, "constraints_fp64": tracked_fp64,
                         "state_vs_fp64_after_track": drift}
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


def bench_ozaki(args):
    """RHS with Ozaki INT8 derivatives (k digit planes, tcgen05 kind::i8) and
    the float64 algebra on the 192^3 q=1/10 block, against the fused float64
    RHS of the same state: time per RHS, per-field normwise error, and
    bit-identity over 5 repeated runs, for k = 5..8. value = the smallest k
    whose worst field error is <= 1e-10."""
    import torch
    dev = torch.device("cuda:0")
    torch.cuda.set_device(dev)
    from bssn3d_b200 import initial_data as ID
    from bssn3d_b200.fused_rhs import device_scalars, pack_S, rhs_tensor
    from bssn3d_b200.ozaki import OzakiDerivatives
    grid, U_host, dt = ID.workload(2, n=args.ozaki_n)
    U = torch.from_numpy(U_host).to(dev)
    S = device_scalars(pack_S(2.0, 0.06, dt, grid.dx, 0.6, 20.0, 0.0, (1, 1, 1, 1), (1, 0),
                              grid.dy, grid.dz), dev)
    interior = grid.interior_points
    stream = torch.cuda.current_stream(dev)

    def timed(fn, reps):
        for _ in range(max(args.warmup, 1)):
            fn()
        torch.cuda.synchronize(dev)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(reps):
            fn()
        b.record(stream)
        b.synchronize()
        return a.elapsed_time(b) / reps

    ref = rhs_tensor(U, S)
    fp64_ms = timed(lambda: rhs_tensor(U, S), args.steps)
    den = ref.reshape(24, -1).abs().amax(dim=1)
    sweep = {}
    chosen = None
    one_k = int(args.ozaki_k) if args.ozaki_k.isdigit() else 0
    for k in ((one_k,) if one_k else (5, 6, 7, 8)):
        oz = OzakiDerivatives(U.shape[1:], k, device=dev)
        ms = timed(lambda: oz.rhs(U, S), args.steps)
        out = oz.rhs(U, S)
        oz.check()
        num = (out - ref).reshape(24, -1).abs().amax(dim=1)
        err = torch.where(num == 0, torch.zeros_like(num), num / den.clamp_min(1e-300))
        same = all(torch.equal(oz.rhs(U, S), out) for _ in range(4))
        sweep[str(k)] = {"ms_per_rhs": ms, "max_field_err": float(err.max()), "worst_field": int(err.argmax()),
                         "bit_identical_5_runs": same,
                         "mpoint_updates_per_s": interior / (ms * 1e-3) / 1e6}
        if chosen is None and float(err.max()) <= 1e-10:
            chosen = k
        del oz, out
        torch.cuda.empty_cache()
    k = chosen if chosen is not None else max(int(q) for q in sweep)
    line = {
        "metric": f"BSSN RHS Mpoint-updates/s (Ozaki INT8 derivatives k={k} + FP64 algebra)",
        "value": sweep[str(k)]["mpoint_updates_per_s"], "unit": UNIT, "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": sweep[str(k)]["ms_per_rhs"], "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "i8 digits, i32 accumulation, f64 algebra",
        "data": "synthetic",
        "config": {"workload": f"Brill-Lindquist q=1/10, {args.ozaki_n}^3 interior +3 ghosts on [-8,8]^3, one RHS",
                   "array": list(grid.shape), "k_chosen_for_1e-10": chosen},
        "fp64_fused": {"ms_per_rhs": fp64_ms, "mpoint_updates_per_s": interior / (fp64_ms * 1e-3) / 1e6},
        "sweep": sweep, "roofline": None, "e2e": None, "cpu_baseline": None,
    }
    print(json.dumps(line), flush=True)


def bench_slab(args):
    """The 128^3 block split into x-slabs, one per rank (strong scaling)."""
    import torch
    world, rank, local = dist_env()
    group = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=120),
                                device_id=torch.device(f"cuda:{local}"))
    dev = torch.device(f"cuda:{local}")
    torch.cuda.set_device(dev)
    from bssn3d_b200 import initial_data as ID
    from bssn3d_b200.slabs import SlabEvolution

    grid, U_host, dt = ID.workload(1, n=args.n)
    interior = grid.interior_points
    evo = SlabEvolution(grid, world=world, rank=rank, ko_sigma=0.1, ko_order=6, group=group)
    lay = evo.layout
    U = evo.local(torch.from_numpy(U_host)).to(dev)
    S = evo.scalars(0.0, dt, dev)

    def barrier():
        if world > 1:
            import torch.distributed as dist
            dist.barrier()
        torch.cuda.synchronize(dev)

    def max_over_ranks(ms):
        if world > 1:
            import torch.distributed as dist
            t = torch.tensor([ms], dtype=torch.float64, device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms = float(t.item())
        return ms

    for _ in range(args.warmup):
        evo.step_inplace(U, S)
        evo.advance_time(S)
    barrier()
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    stream = torch.cuda.current_stream(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        evo.step_inplace(U, S)
        evo.advance_time(S)
    e1.record(stream)
    barrier()
    clk = clocks.stop()
    ms = max_over_ranks(e0.elapsed_time(e1))
    finite = bool(torch.isfinite(evo.owned(U)).all().item())

    # end to end: every step copies the rank's slab in from pinned host memory
    # and its owned planes out
    e2e = None
    if not args.no_e2e:
        host_in = torch.from_numpy(U_host[:, lay.local_slice()].copy()).pin_memory()
        host_out = torch.empty_like(host_in[:, lay.owned_slice()]).pin_memory()
        Ue, Se = torch.empty_like(U), evo.scalars(0.0, dt, dev)

        def e2e_step():
            Ue.copy_(host_in, non_blocking=True)
            Se.copy_(S)
            evo.step_inplace(Ue, Se)
            host_out.copy_(evo.owned(Ue), non_blocking=True)
        for _ in range(args.warmup):
            e2e_step()
        barrier()
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        f0.record(stream)
        for _ in range(args.steps):
            e2e_step()
        f1.record(stream)
        barrier()
        ems = max_over_ranks(f0.elapsed_time(f1))
        nb = torch.tensor([host_in.numel() * 8, host_out.numel() * 8], dtype=torch.float64, device=dev)
        if world > 1:
            import torch.distributed as dist
            dist.all_reduce(nb)
        e2e = {"value": interior * 4 * args.steps / (ems * 1e-3) / 1e6, "unit": UNIT,
               "h2d_bytes_per_step": int(nb[0].item()), "d2h_bytes_per_step": int(nb[1].item()),
               "ms_per_step": ems / args.steps,
               "path": "bssn3d_b200.slabs.SlabEvolution: per step and rank, its slab in from pinned "
                       "host memory, one RK4 step with the halo exchanges, its owned planes out"}

    # per-launch stage time on this rank's slab (the owned interior points it delivers)
    b = evo.buffers(U)
    durs = []
    for _ in range(3):
        a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a0.record(stream)
        evo.stage_fn(1, U, b["Ya"], b["ACC"], b["Yb"], S)
        a1.record(stream)
        a1.synchronize()
        durs.append(a0.elapsed_time(a1))
    stage_ms = statistics.median(durs)
    ng = grid.ng
    owned_interior = max(min(lay.b, lay.Sx - ng) - max(lay.a, ng), 0) * grid.Ny * grid.Nz
    peaks, peak_kind = measured_peaks()
    achieved = owned_interior * STAGE_BYTES / (stage_ms * 1e-3) / 1e9
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peaks.get("hbm_gbs"), "unit": "GB/s",
                "frac": achieved / peaks.get("hbm_gbs"), "traffic": None,
                "peak_source": f"{peak_kind} hbm_gbs",
                "kernel": "bssn::stream_kernel<3, MODE_STAGE, Shape<4,4,16>> on rank 0's slab",
                "bytes_per_point_update": STAGE_BYTES, "point_updates_per_launch": owned_interior,
                "points_evaluated_per_launch": int(U[0].numel()), "launch_ms": stage_ms}
    value = interior * 4 * args.steps / (ms * 1e-3) / 1e6
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
        "scaling": "strong", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"Brill-Lindquist q=1/10, {args.n}^3 interior +3 ghosts on [-8,8]^3, "
                               f"RK4 step, KO sigma 0.1 order 6, split into {world} x-slabs",
                   "array": list(grid.shape), "slabs": lay.ranges, "halo_planes": lay.halo,
                   "exchange_bytes_per_stage_rank0": lay.exchange_bytes(grid.shape[1], grid.shape[2]),
                   "l2": "inputs larger than L2 (462 MB state)", "parallelism": f"slab x{world}"},
        "clocks": clk, "gpu_launches": 5 * args.steps, "finite": finite, "roofline": roofline,
        "e2e": e2e, "cpu_baseline": None,
    }
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        bench_reference(args)
    elif args.workload.startswith("amr"):
        bench_amr(args)
    elif args.workload == "ozaki192":
        bench_ozaki(args)
    elif args.split == "slab":
        bench_slab(args)
    else:
        bench_b200(args)


if __name__ == "__main__":
    main()

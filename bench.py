"""Benchmark: DGSEM right-hand-side throughput (DOF*RHS/s) on the
Navier-Stokes Taylor-Green vortex, 32^3 hex mesh, p=4 (4,096,000 LGL nodes x 5
conserved variables), Ranocha volume / HLL surface flux, BR1 viscous terms,
Ma=0.1, Re=1600, Pr=0.71, FP64.  One step = one right-hand side L(u) of the
whole mesh (RHSOperator::Mult).  DOF = solution nodes (E*N^d).

    python bench.py [--gpus N --steps K --warmup W] [--impl reference]

Prints one JSON line (rank 0): the headline FP64 figure, its end-to-end
figure through the C ABI with host buffers, the dominant kernel's roofline,
the FP32-mixed companion, the reference's CPU right-hand side on the same
workload, and (one GPU) compact results of the other configurations -- the
2-D isentropic vortex, the Sedov blast, the LTE Taylor-Green vortex and the
batched serving stream.  --impl reference times the reference's CPU
right-hand side (its own header kernels compiled here, all host threads) on
the full workload, one right-hand side per step.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = {"workload": "ns_tgv_32^3_p4", "mesh": [32, 32, 32], "order": 4, "dim": 3,
            "volume_flux": "ranocha", "surface_flux": "hll", "mach": 0.1, "reynolds": 1600,
            "Pr": 0.71, "noise": 1e-6}
METRIC = "DOF*RHS/s (solution nodes x right-hand-side evaluations per second)"
UNIT = "DOF*RHS/s"


def build_case(n=None, order=4):
    import theseus_b200 as T
    from theseus_b200 import cases
    n = n or WORKLOAD["mesh"]
    m = T.periodic_box(3, order, n, [0.0] * 3, [2 * np.pi] * 3)
    u = cases.taylor_green(m.coords, mach=WORKLOAD["mach"], noise=WORKLOAD["noise"], seed=0)
    return m, u


def physics():
    return dict(mu=1.0 / WORKLOAD["reynolds"], Pr=WORKLOAD["Pr"])


class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        try:
            for line in open(self.path):
                f = [x.strip() for x in line.split(",")]
                if len(f) < 9:
                    continue
                try:
                    sm.append(float(f[1]))
                    mx = float(f[2])
                except ValueError:
                    continue
                for nm, v in zip(names, f[5:9]):
                    if v.lower() == "active":
                        reasons.add(nm)
        except OSError:
            pass
        finally:
            if self.path:
                try:
                    os.unlink(self.path)
                except OSError:
                    pass
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def fp64_peak_tflops():
    """FP64 FMA throughput of this GPU (thx_measure_fp64_fma_peak: independent
    FMA chains on every SM, best of five CUDA-event-timed launches)."""
    import ctypes as C
    import torch
    import theseus_b200 as T
    lib = T.library()
    lib.thx_measure_fp64_fma_peak.argtypes = [C.c_int, C.c_int, C.POINTER(C.c_double), C.c_void_p]
    v = C.c_double()
    st = lib.thx_measure_fp64_fma_peak(2048, 5, C.byref(v), C.c_void_p(torch.cuda.current_stream().cuda_stream))
    return v.value / 1e12 if st == 0 else None


def bytes_per_phase(m, elem_size=8):
    """Algorithmic HBM bytes of each kernel for one RHS (geometry stored once):
    gradient: read u, write the physical viscous flux (dim x (neq-1) per node);
    face: read both traces of u and of the viscous flux, write F*;
    volume: read u, the viscous flux and F* once, write dudt."""
    nodes = m.num_nodes
    neq, dim = m.neq, m.dim
    nv = dim * (neq - 1)
    fpts = m.num_faces * m.nfp
    s = elem_size
    grad = nodes * (neq + nv) * s
    face = fpts * (2 * neq + 2 * nv + neq) * s
    vol = nodes * (2 * neq + nv) * s + fpts * neq * s
    return {"blend": nodes * neq * s, "grad": grad, "face": face, "volume": vol}


# Floating-point operations of one two-point volume flux as the kernels
# evaluate it from per-node primitives (rho, v, p and one auxiliary), counted
# from the source with +, -, x = 1, FMA = 2, divide / sqrt / log = 1; the log
# mean (y - x)/log(y/x) with its branch variable u is 11.  D = dimension.
#   Ranocha:       2 log means, p1 p2 / log mean, the kinetic-energy and
#                  pressure-work terms: 34 + 16 D
#   Chandrashekar: 2 log means, p_hat, h_hat: 33 + 15 D
#   Pirozzoli:     arithmetic means only: 10 + 12 D
PAIR_FLOPS = {"ranocha": lambda d: 34 + 16 * d, "chandrashekar": lambda d: 33 + 15 * d,
              "pirozzoli": lambda d: 10 + 12 * d}


def volume_flops(m, volume_flux, viscous):
    """Algorithmic flops of the volume kernel for one RHS: every symmetric pair
    once (PAIR_FLOPS) plus its D-hat-2 accumulation into both end nodes
    (2 nodes x neq FMAs); for Navier-Stokes the contravariant viscous flux
    (dim x dim metric products per flux row) and its D-hat divergence
    (N terms per direction) per node.  Returns (flops, pairs)."""
    dim, N, neq = m.dim, m.order + 1, m.neq
    pairs = m.num_elements * dim * N ** (dim - 1) * (N * (N - 1) // 2)
    per_pair = PAIR_FLOPS[volume_flux](dim) + 2 * 2 * neq
    per_node = (2 * dim * dim * (neq - 1) + 2 * dim * N * (neq - 1)) if viscous else 0
    return pairs * per_pair + m.num_nodes * per_node, pairs


# DRAM bytes per node of one launch, from ncu captures of the same kernels
# (dram__bytes_read.sum + dram__bytes_write.sum of one launch / nodes of the
# captured mesh: the NS Taylor-Green vortex at 20^3, p=4, FP64; the gradient
# phase is the entropy-variable kernel plus the gradient kernel).  A kernel's
# traffic grows with its node count, so the bench scales these to its own
# mesh.  Filled per (kernel, precision); absent: null.
TRAFFIC_PER_NODE = {
    # NS Taylor-Green 20^3 p=4 FP64 captures, 1,000,000 nodes
    ("volume_kernel", "fp64"): (160.683264e6 + 24.671488e6) / 1e6,
    ("grad_kernel", "fp64"): (40.011776e6 + 2.212608e6 + 83.475968e6 + 53.984e6) / 1e6,
    ("face_kernel", "fp64"): (139.248896e6 + 20.290816e6) / 1e6,
}


_CPU_FN = None


def cpu_rhs_fn():
    """The CPU right-hand side that stands for the reference: the reference's
    own point kernels compiled from its headers, OpenMP over elements and
    faces -- the fastest on this host of the optimised build (-O3, -march
    native or x86-64-v4, where this host can run it) and the parity build
    (oracle/_ref: -O2, separately rounded multiplies and adds), timed on a
    12^3 sample -- or, when neither was built, the oracle's restatement.
    Returns (rhs(mesh, cfg, u), kind, threads, build)."""
    global _CPU_FN
    if _CPU_FN is not None:
        return _CPU_FN
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    threads = O.max_threads()
    cands = []
    if O.ref_native() is not None:
        cands.append(((lambda om, cfg, u: O.ref_rhs(om, cfg, u, native=True)),
                      f"reference headers, {O.ref_native.build}, OpenMP"))
    if O.ref_available():
        try:
            O.ref()
            cands.append(((lambda om, cfg, u: O.ref_rhs(om, cfg, u)),
                          "reference headers, g++ -O2 -march=x86-64-v3 -ffp-contract=off, OpenMP"))
        except OSError:
            pass
    if not cands:
        _CPU_FN = ((lambda om, cfg, u: O.rhs(om, cfg, u, nthreads=threads)), "port", threads,
                   "oracle restatement, OpenMP")
        return _CPU_FN
    best = None
    if len(cands) > 1:
        om, cfg, u = cpu_case((12, 12, 12))
        for fn, build in cands:
            fn(om, cfg, u)
            t0 = time.perf_counter()
            for _ in range(3):
                fn(om, cfg, u)
            dt = time.perf_counter() - t0
            if best is None or dt < best[0]:
                best = (dt, fn, build)
    else:
        best = (0.0,) + cands[0]
    _CPU_FN = (best[1], "reference", threads, best[2] + " (fastest build on this host)")
    return _CPU_FN


def cpu_parity_rhs(om, cfg, u):
    """The reference's right-hand side from its parity build (separately
    rounded multiplies and adds, as the GPU's FP64 path) when built, else the
    oracle's; used to check this run's GPU rate, never timed."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    if O.ref_available():
        return O.ref_rhs(om, cfg, u), "reference parity build"
    return O.rhs(om, cfg, u, nthreads=O.max_threads()), "oracle"


def cpu_case(n=None):
    """The workload's mesh (the oracle's own box builder: nothing of the
    product library is loaded), its configuration and its state."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    from theseus_b200 import cases
    from theseus_b200._abi import make_config
    n = n or WORKLOAD["mesh"]
    om = O.box_mesh(3, WORKLOAD["order"], n, [0.0] * 3, [2 * np.pi] * 3)
    u = cases.taylor_green(om.coords, mach=WORKLOAD["mach"], noise=WORKLOAD["noise"], seed=0)
    cfg = make_config(flow="ns", volume_flux=WORKLOAD["volume_flux"],
                      surface_flux=WORKLOAD["surface_flux"], **physics())
    return om, cfg, u


def cpu_reference(budget_s=15.0, max_evals=20, keep_rate=False):
    """The CPU reference on the full workload, all host threads: one warm-up
    right-hand side, then evaluations until budget_s has passed (at most
    max_evals).  keep_rate: also return the last rate (for the parity check)."""
    fn, kind, threads, build = cpu_rhs_fn()
    om, cfg, u = cpu_case()
    du = fn(om, cfg, u)  # warm-up
    t0 = time.perf_counter()
    evals = 0
    while True:
        du = fn(om, cfg, u)
        evals += 1
        if time.perf_counter() - t0 > budget_s or evals >= max_evals:
            break
    dt = time.perf_counter() - t0
    nodes = om.num_elements * om.nd
    out = {"value": nodes * evals / dt, "unit": UNIT, "cores": threads, "kind": kind,
           "build": build,
           "sample": f"the full workload (TGV {om.shape[0]}^3 p={om.order}, {nodes} nodes): "
                     f"{evals} RHS evaluations in {dt:.1f} s"}
    return (out, du, u) if keep_rate else out


def run_reference(args):
    """--impl reference: the reference's CPU right-hand side on this host's
    cores, on the same workload (the full 32^3 mesh), each step one RHS."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    fn, kind, threads, build = cpu_rhs_fn()
    om, cfg, u = cpu_case()
    for _ in range(args.warmup):
        fn(om, cfg, u)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        fn(om, cfg, u)
    dt = time.perf_counter() - t0
    nodes = om.num_elements * om.nd
    value = nodes * args.steps / dt
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * dt / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "impl": "reference",
            "config": dict(WORKLOAD, parallelism="cpu threads"),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": kind,
                             "build": build,
                             "sample": f"the full workload ({nodes} nodes), one RHS per step"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def max_over_ranks(ms, dist=None, device=None):
    """The slowest rank's time: every rank contributes its own device-timed
    milliseconds (nccl: a CUDA tensor; gloo: a CPU tensor)."""
    if dist is None:
        return float(ms)
    import torch
    t = torch.tensor([float(ms)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_throughput(world, units_per_rank, steps, ms):
    """Whole-job throughput of `world` independent replicas, each processing
    units_per_rank units per step, timed as the slowest rank's ms."""
    return world * units_per_rank * steps / (ms * 1e-3)


def timed_rk3(op, u0, dt, steps, stream, repeats=2):
    """Device time (ms) of `steps` SSP-RK3 steps from u0, after a short warm-up
    run; the median of `repeats` runs, each from the same initial state.
    Returns (ms, final state of the last run)."""
    import torch
    y = u0.clone()
    op.rk3_steps(y, dt, 3)  # warm-up: graphs, caches, clocks
    times = []
    for _ in range(repeats):
        y.copy_(u0)
        torch.cuda.synchronize()
        ta, tb = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ta.record(stream)
        op.rk3_steps(y, dt, steps)
        tb.record(stream)
        torch.cuda.synchronize()
        times.append(ta.elapsed_time(tb))
    return float(statistics.median(times)), y


def field_errors(got, ref, groups):
    """Relative L2 per conserved field (rows grouped: density, momentum, energy)."""
    return [float(((got[g] - ref[g]).pow(2).sum() / ref[g].pow(2).sum()).sqrt()) for g in groups]


def run_ours(args):
    import torch
    import theseus_b200 as T
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist_
        import datetime
        dist_.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                 device_id=torch.device("cuda", local))
        dist = dist_
    if args.n != WORKLOAD["mesh"][0]:
        WORKLOAD["mesh"] = [args.n] * 3
        WORKLOAD["workload"] = f"ns_tgv_{args.n}^3_p4"
    m, u = build_case()
    prec = "fp32" if args.precision == "fp32" else "fp64"
    op = T.NSOperator(m, numerical_flux=WORKLOAD["volume_flux"], surface_flux=WORKLOAD["surface_flux"],
                      precision=prec, volume_staging=args.volume_staging, **physics())
    ud = torch.as_tensor(u, device="cuda").to(op.dtype).contiguous()
    du = torch.empty_like(ud)
    stream = torch.cuda.current_stream()

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()

    for _ in range(max(args.warmup, 3)):
        op.Mult(ud, du)
    barrier()
    with ClockSampler(local) as clk:
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0.record(stream)
        for _ in range(args.steps):
            op.Mult(ud, du)
        t1.record(stream)
        torch.cuda.synchronize()
    ms = t0.elapsed_time(t1)
    barrier()
    ms = max_over_ranks(ms, dist, "cuda")
    nodes = m.num_nodes
    value = replica_throughput(world, nodes, args.steps, ms)

    # end to end through the C ABI with host buffers (thx_rhs_host: each
    # step's FP64 state copied in from pinned host memory and its rate copied
    # back, the copies of neighbouring steps overlapping the kernels), timed
    # on the device from before the first copy-in to after the last copy-out
    hu = [torch.as_tensor(u, dtype=torch.float64).pin_memory() for _ in range(2)]
    hdu = [torch.empty_like(hu[0]).pin_memory() for _ in range(2)]
    op.mult_host([hu[i % 2] for i in range(3)], [hdu[i % 2] for i in range(3)])
    torch.cuda.synchronize()
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    op.mult_host([hu[i % 2] for i in range(args.steps)], [hdu[i % 2] for i in range(args.steps)])
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(e0.elapsed_time(e1), dist, "cuda")
    e2e = {"value": replica_throughput(world, nodes, args.steps, e2e_ms), "unit": UNIT,
           "h2d_bytes_per_step": hu[0].numel() * hu[0].element_size(),
           "d2h_bytes_per_step": hdu[0].numel() * hdu[0].element_size(), "overlap": "copy-in/compute/copy-out"}

    # per-kernel device times (CUDA events on the launching stream, one event
    # between consecutive kernels of a right-hand side) over as many
    # right-hand sides as the timed region, after it
    ud.copy_(torch.as_tensor(u).to(op.dtype))
    phases = np.zeros(4)
    nprof = max(3, args.steps)
    for _ in range(nprof):
        phases += np.array(op.profile(ud, du))
    phases /= nprof
    names = ["blend", "grad", "face", "volume"]
    es = 4 if prec == "fp32" else 8
    algo = bytes_per_phase(m, es)
    peak_hbm, peak_kind = peaks()
    fp64_tf = fp64_peak_tflops()
    vflops, pairs = volume_flops(m, WORKLOAD["volume_flux"], True)
    dom = int(np.argmax(phases))
    kname = names[dom] + "_kernel"
    traffic = TRAFFIC_PER_NODE.get((kname, prec))
    if names[dom] == "volume" and prec == "fp64" and fp64_tf:
        # the pair phase is FP64 arithmetic: roofline against the FP64 FMA peak
        achieved = vflops / (phases[dom] * 1e-3) / 1e12
        roofline = {"bound": "fp64", "kernel": kname, "achieved": achieved, "peak": fp64_tf,
                    "unit": "TFLOP/s", "frac": achieved / fp64_tf,
                    "peak_source": "measured (thx_measure_fp64_fma_peak, this run)",
                    "algorithmic_flops": vflops}
    else:
        achieved = algo[names[dom]] / (phases[dom] * 1e-3) / 1e9
        roofline = {"bound": "hbm", "kernel": kname, "achieved": achieved, "peak": peak_hbm,
                    "unit": "GB/s", "frac": achieved / peak_hbm, "peak_source": peak_kind}
    roofline["traffic"] = traffic * nodes if traffic else None
    roofline["traffic_source"] = ("ncu dram__bytes_read.sum + dram__bytes_write.sum of the same kernel "
                                  "on the 20^3 mesh, scaled by nodes") if traffic else None
    roofline["phase_ms"] = {k: float(v) for k, v in zip(names, phases)}
    roofline["algorithmic_bytes"] = {k: int(v) for k, v in algo.items()}
    roofline["hbm_frac"] = {k: (algo[k] / (phases[i] * 1e-3) / 1e9) / peak_hbm
                            for i, k in enumerate(names) if phases[i] > 0.01}
    roofline["volume_fp64"] = {"pairs": pairs, "pair_flops": PAIR_FLOPS[WORKLOAD["volume_flux"]](3),
                               "flops": vflops, "fp64_fma_peak_tflops": fp64_tf,
                               "pair_evals_per_s": pairs / (phases[3] * 1e-3),
                               # the algorithmic count takes a division or a log
                               # as one flop; the FP64 pipe also runs their
                               # iterations, so it is busier than frac says
                               "ncu_fp64_pipe_active": 0.483, "ncu_issue_active": 0.666,
                               "ncu_source": "ncu capture of this volume kernel on the 20^3 mesh "
                                             "(sm__pipe_fp64_cycles_active, smsp__issue_active)"}

    # the volume kernel with its element blocks' state staged by bulk copy
    # (cp.async.bulk into a double buffer, persistent CTAs) against the
    # default form, same state, per-kernel CUDA events
    extra = {}
    if prec == "fp64" and args.volume_staging == 0 and not args.no_mixed:
        alt = T.NSOperator(m, numerical_flux=WORKLOAD["volume_flux"],
                           surface_flux=WORKLOAD["surface_flux"], volume_staging=1, **physics())
        du_alt = torch.empty_like(du)
        ph_alt = np.mean([alt.profile(ud, du_alt) for _ in range(nprof)], axis=0)
        op.Mult(ud, du)
        extra["volume_staging_trial"] = {
            "volume_ms_loads": float(phases[3]), "volume_ms_bulk_copy": float(ph_alt[3]),
            "same_result": bool(torch.equal(du, du_alt)), "status": alt.read_status(),
            "kept": "loads" if phases[3] <= ph_alt[3] else "bulk_copy"}
        del alt, du_alt
    # FP32-mixed companion number and its error against FP64: RHS and the
    # final solution after a fixed-dt SSP-RK3 run from the same state
    if prec == "fp64" and not args.no_mixed:
        off = [1.0, 0.0, 0.0, 0.0, 1.0 / (1.4 * WORKLOAD["mach"] ** 2) / 0.4]
        op32 = T.NSOperator(m, numerical_flux=WORKLOAD["volume_flux"],
                            surface_flux=WORKLOAD["surface_flux"], precision="fp32",
                            state_offset=off, **physics())
        u64 = torch.as_tensor(u, device="cuda").contiguous()
        d32 = torch.empty_like(u64)
        for _ in range(3):
            op32.Mult(u64, d32)
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(args.steps):
            op32.Mult(u64, d32)
        b.record(stream)
        torch.cuda.synchronize()
        ms32 = a.elapsed_time(b)
        op.Mult(u64, du)
        ref = du.clone()
        err = ((d32 - ref).pow(2).sum(dim=(1, 2)) / ref.pow(2).sum(dim=(1, 2))).sqrt()
        # trajectories: fixed dt from CFL 0.5 at t=0, rk_steps SSP-RK3 steps
        # each, warmed up and timed twice (median)
        dt = op.estimate_dt(u64, 0.5)
        ms_rk64, ya = timed_rk3(op, u64, dt, args.rk_steps, stream)
        ms_rk32, yb = timed_rk3(op32, u64, dt, args.rk_steps, stream)
        serr = ((yb - ya).pow(2).sum(dim=(1, 2)) / ya.pow(2).sum(dim=(1, 2))).sqrt()
        ferr = field_errors(yb, ya, [[0], [1, 2, 3], [4]])
        ke0 = op.IntegralMeasures(u64)["ke"]
        ke64 = op.IntegralMeasures(ya)["ke"]
        ke32 = op.IntegralMeasures(yb)["ke"]
        ph32 = np.zeros(4)
        for _ in range(3):
            ph32 += np.array(op32.profile(u64, d32))
        ph32 /= 3
        extra["fp32_mixed"] = {
            "value": nodes * args.steps / (ms32 * 1e-3), "unit": UNIT,
            "speedup_vs_fp64": (ms / ms32) if ms32 > 0 else None,
            "rhs_rel_l2_vs_fp64": [float(x) for x in err.tolist()],
            "state_offset": off,
            "rk3": {"steps": args.rk_steps, "dt": dt, "timing": "median of 2 runs after a 3-step warm-up",
                    "fp64_dof_rhs_per_s": 3 * nodes * args.rk_steps / (ms_rk64 * 1e-3),
                    "fp32_mixed_dof_rhs_per_s": 3 * nodes * args.rk_steps / (ms_rk32 * 1e-3),
                    "speedup": ms_rk64 / ms_rk32,
                    "final_solution_rel_l2_vs_fp64": {
                        "density": ferr[0], "momentum": ferr[1], "energy": ferr[2],
                        "max": max(ferr),
                        "per_component": [float(x) for x in serr.tolist()]},
                    "kinetic_energy": {"t0": ke0, "fp64": ke64, "fp32_mixed": ke32,
                                       "rel_diff": abs(ke32 - ke64) / abs(ke64)}},
            "phase_ms": {k: float(v) for k, v in zip(["blend", "grad", "face", "volume"], ph32)}}
        del op32, ya, yb

    launches = args.steps * 3  # gradient, face and volume kernels per right-hand side
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64" if prec == "fp64" else "f32-mixed",
            "data": "synthetic",
            "config": dict(WORKLOAD, precision=prec, parallelism=f"replicas x{world}",
                           l2="working set (u 164 MB, viscous flux 393 MB, face fluxes 98 MB) "
                              "larger than the 126 MB L2",
                           kernel_layout=op.describe()),
            "e2e": e2e, "roofline": roofline, "clocks": clk.summary(),
            "gpu_launches": launches}
    line.update(extra)
    if rank == 0 and not args.skip_cpu and world == 1:
        # the reference's CPU right-hand side on the same (full) workload, and
        # this run's GPU rate against it
        cb, _, _ = cpu_reference(keep_rate=True)
        line["cpu_baseline"] = cb
        ud.copy_(torch.as_tensor(u))
        op.Mult(ud, du)
        got = du.cpu().numpy()
        om, cfg_, u_ = cpu_case()
        ref_du, ref_kind = cpu_parity_rhs(om, cfg_, u_)
        rel = np.sqrt(((got - ref_du) ** 2).reshape(5, -1).sum(1) / (ref_du ** 2).reshape(5, -1).sum(1))
        line["rhs_rel_l2_vs_cpu_reference_full_mesh"] = {"per_variable": [float(x) for x in rel],
                                                          "against": ref_kind}
    if world == 1 and not args.no_workloads:
        del op, ud, du
        torch.cuda.empty_cache()
        line["workloads"] = other_workloads(args)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


def other_workloads(args):
    """Compact results of the other configurations (each also available in
    full with --workload): the 2-D isentropic vortex, the Sedov blast, the LTE
    Taylor-Green vortex and the batched serving stream."""
    import torch
    out = {}
    for name, fn in (("vortex_2d", run_vortex), ("sedov", run_sedov), ("lte", run_lte),
                     ("serving", run_serving), ("batch", run_batch),
                     ("contraction_trial", run_trials)):
        try:
            full = fn(args)
            out[name] = compact(name, full)
        except Exception as exc:  # report, keep the headline line
            out[name] = {"error": f"{type(exc).__name__}: {exc}"[:400]}
        torch.cuda.empty_cache()
    return out


def compact(name, d):
    keep = {
        "vortex_2d": ["value", "unit", "config", "rk3", "fp32_mixed", "rhs_rel_l2_vs_oracle",
                      "final_rel_l2_vs_oracle", "entropy_residual", "cpu"],
        "sedov": ["value", "unit", "config", "fp32_speedup", "final_solution_rel_l2_fp32_vs_fp64",
                  "blending_agreement_t0", "rhs_rel_l2_vs_oracle_4cubed"],
        "lte": ["value", "unit", "config", "newton_recoveries_per_s", "lteec_pairs_per_s",
                "rhs_rel_l2_vs_oracle_3cubed", "rk3", "phase_ms"],
        "serving": ["value", "unit", "latency_s", "makespan_s", "dof_rhs_per_s", "one_at_a_time_fp64",
                    "speedup_vs_one_at_a_time", "final_solution_rel_l2_vs_fp64"],
        "contraction_trial": ["results"],
        "batch": ["value", "unit", "steps", "groups"],
    }[name]
    r = {k: d[k] for k in keep if k in d}
    if name == "sedov":
        for p in ("fp64", "fp32_mixed"):
            q = d[p]
            r[p] = {"dof_rhs_per_s": q["dof_rhs_per_s"], "blended_fraction": q["blended_fraction"],
                    "rk3_dof_rhs_per_s": q["rk3"]["dof_rhs_per_s"], "status": q["status"]}
    if name == "serving" and "final_solution_rel_l2_vs_fp64" in r:
        r["final_solution_rel_l2_vs_fp64"] = {k: v for k, v in r["final_solution_rel_l2_vs_fp64"].items()
                                              if k != "worst"}
    return r


def run_vortex(args):
    """2-D Euler isentropic vortex: periodic [-5, 5]^2, 32 x 32 quads, p=3
    (16,384 nodes, 4 conserved variables), Chandrashekar volume / Roe surface
    flux, no blending, rho = 1, u = (1, 1), p = 1 with a vortex of strength 5 at
    the origin, dt from CFL 0.5 at t = 0 (the oracle's estimate) held fixed,
    100 SSP-RK3 steps in FP64 and FP32-mixed.  Reports RHS throughput, the
    trajectories against the oracle's (all host threads), the entropy
    residual of the first right-hand side on both sides, and the reference's
    CPU right-hand side and the oracle's 100-step run timed on this host."""
    import torch
    import theseus_b200 as T
    from theseus_b200 import cases
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    steps = 100
    m = T.periodic_box(2, 3, (32, 32), [-5.0, -5.0], [5.0, 5.0])
    u = cases.isentropic_vortex(m.coords, strength=5.0)
    kw = dict(numerical_flux="chandrashekar", surface_flux="roe")
    cfg = T.make_config(flow="euler", volume_flux="chandrashekar", surface_flux="roe")
    om = O.Mesh(m.dim, m.order, m.jac, m.metric, m.face_elem, m.face_lface, m.face_normal,
                m.face_wminus, m.face_wplus)
    nth = O.max_threads()
    dt, _ = O.estimate_dt(om, cfg, u, 0.5)
    stream = torch.cuda.current_stream()
    op = T.EulerOperator(m, **kw)
    ud = torch.as_tensor(u, device="cuda").contiguous()
    du = torch.empty_like(ud)
    for _ in range(max(args.warmup, 3)):
        op.Mult(ud, du)
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for _ in range(args.steps):
        op.Mult(ud, du)
    b.record(stream)
    torch.cuda.synchronize()
    ms = a.elapsed_time(b) / args.steps
    gpu_du = du.cpu().numpy()
    ms_rk, y = timed_rk3(op, ud, dt, steps, stream)
    op32 = T.EulerOperator(m, precision="fp32", state_offset=[1.0, 1.0, 1.0, 3.5], **kw)
    ms_rk32, y32 = timed_rk3(op32, ud, dt, steps, stream)
    # oracle: first right-hand side, its entropy residual, the trajectory
    ref_du = O.rhs(om, cfg, u, nthreads=nth)
    t0 = time.perf_counter()
    ref_y = O.rk3_steps(om, cfg, u, dt, steps, nthreads=nth)
    port_s = time.perf_counter() - t0
    yg = y.cpu().numpy()
    rel = lambda g, r: [float(x) for x in np.sqrt(((g - r) ** 2).reshape(4, -1).sum(1) /
                                                  (r ** 2).reshape(4, -1).sum(1))]
    groups = [[0], [1, 2], [3]]
    y32g = y32.cpu().numpy()
    f32 = [float(np.sqrt(((y32g[g] - yg[g]) ** 2).sum() / (yg[g] ** 2).sum())) for g in groups]
    # the reference's CPU right-hand side on the same case
    fn, kind, threads, build = cpu_rhs_fn()
    fn(om, cfg, u)
    t0 = time.perf_counter()
    n_cpu = 0
    while time.perf_counter() - t0 < 2.0 and n_cpu < 200:
        fn(om, cfg, u)
        n_cpu += 1
    cpu_s = (time.perf_counter() - t0) / n_cpu
    return {"metric": "DOF*RHS/s (2-D Euler isentropic vortex)", "value": m.num_nodes / (ms * 1e-3),
            "unit": "DOF*RHS/s", "n_gpus": 1, "ms_per_step": ms, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "euler2d_vortex_32^2_p3", "nodes": m.num_nodes, "strength": 5.0,
                       "fluxes": {"volume": "chandrashekar", "surface": "roe"}, "blending": False,
                       "cfl": 0.5, "dt": dt, "steps": steps},
            "rk3": {"ms": ms_rk, "dof_rhs_per_s": 3 * steps * m.num_nodes / (ms_rk * 1e-3),
                    "timing": "median of 2 runs after a 3-step warm-up"},
            "fp32_mixed": {"rk3_ms": ms_rk32, "speedup": ms_rk / ms_rk32,
                           "final_solution_rel_l2_vs_fp64": dict(zip(("density", "momentum", "energy"),
                                                                     f32))},
            "rhs_rel_l2_vs_oracle": rel(gpu_du, ref_du),
            "final_rel_l2_vs_oracle": rel(yg, ref_y),
            "entropy_residual": {"gpu": O.entropy_residual(om, cfg, u, gpu_du),
                                 "oracle": O.entropy_residual(om, cfg, u, ref_du)},
            "cpu": {"rhs_dof_rhs_per_s": m.num_nodes / cpu_s, "kind": kind, "build": build,
                    "cores": threads, "oracle_100_steps_s": port_s, "oracle_threads": nth}}


def run_trials(args):
    """Tensor-core trial of the gradient's element-local derivative
    contraction (thx_trial_contraction) on the 32^3 p=4 mesh: SIMT FMA against
    mma.sync tiles -- FP64 m8n8k4, and FP32 m16n8k8 TF32 with one or three
    products -- device time per launch and the largest difference from the
    SIMT form relative to its largest value."""
    import ctypes as C
    import torch
    import theseus_b200 as T
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    lib = T.library()
    lib.thx_trial_contraction.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p,
                                          C.POINTER(C.c_double), C.c_void_p, C.c_int,
                                          C.POINTER(C.c_double), C.c_void_p]
    n, order = 32, 4
    ne, nd = n ** 3, (order + 1) ** 3
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    _, _, Dm, _, _ = O.operators(order)
    Dm = np.ascontiguousarray(Dm, np.float64)
    g = torch.Generator(device="cuda").manual_seed(0)
    fields = torch.rand((5, ne, nd), generator=g, dtype=torch.float64, device="cuda") * 2 - 1
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    out = {}
    for prec, name, dt, forms in ((T.PRECISION_FP64, "fp64", torch.float64, ("simt", "mma_m8n8k4_f64")),
                                  (T.PRECISION_FP32_MIXED, "fp32", torch.float32,
                                   ("simt", "mma_m16n8k8_tf32", "mma_m16n8k8_3xtf32"))):
        f = fields.to(dt).contiguous()
        res, ref = {}, None
        for form, fname in enumerate(forms):
            o = torch.empty((ne, nd), dtype=dt, device="cuda")
            ms = C.c_double()
            st = lib.thx_trial_contraction(3, order, ne, prec, form, C.c_void_p(f.data_ptr()),
                                           Dm.ctypes.data_as(C.POINTER(C.c_double)), C.c_void_p(o.data_ptr()),
                                           20, C.byref(ms), stream)
            if st != 0:
                res[fname] = {"status": st}
                continue
            torch.cuda.synchronize()
            if ref is None:
                ref = o.double()
            diff = float((o.double() - ref).abs().max() / ref.abs().max())
            res[fname] = {"ms": ms.value, "max_rel_diff_vs_simt": diff}
        out[name] = res
    return {"metric": "element-local derivative contraction: SIMT vs tensor-core tiles",
            "config": {"workload": "gradient_D_contraction_32^3_p4", "elements": ne, "fields": 5,
                       "directions": 3, "padding": "rows of S^T to 8 (FP64) / 16 (TF32), K=5 to 8, "
                                                    "N columns: 5 of 8 used"},
            "results": out}


def run_batch(args):
    """Batched kernels against one-case kernels, FP32-mixed: for each group
    kind (2-D vortex cases of p=2 Euler, p=3 Euler, p=3 Navier-Stokes, p=5
    Navier-Stokes), 64 equal cases of 32^2 quads (24^2 at p=5) advanced
    together through the batch engine, against one mesh of the same total
    size (256^2, 192^2 at p=5) through the one-case fused SSP-RK3 loop.  The
    engine's first batch tunes the group; the next three are timed from their
    last admission to their last completion (wall clock: the engine launches
    on its own streams) and the fastest counts; the one-case loop is timed by
    CUDA events.  Reports node-RHS/s of
    both and their ratio, with the group's tuned configuration."""
    import torch
    import theseus_b200 as T
    from theseus_b200 import cases
    from theseus_b200.serving import BatchEngine, Case
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    flux = dict(numerical_flux="chandrashekar", surface_flux="roe")
    steps, ncase = args.batch_steps, 64

    def vcase(order, n, viscous, seed):
        m = T.periodic_box(2, order, (n, n), [-5.0, -5.0], [5.0, 5.0])
        c = np.sqrt(1.4)
        v = 0.5 * c / np.sqrt(2.0)
        u0 = cases.isentropic_vortex(m.coords, strength=3.0, u_inf=(v, v))
        u0 = u0 * (1.0 + 1e-3 * np.random.default_rng(seed).uniform(-1, 1, u0.shape))
        dt = 0.4 * (10.0 / n) / ((2 * order + 1) * (np.sqrt(2) * v + c + 1.0))
        return Case(mesh=m, u0=u0, nsteps=steps, dt=dt, viscous=viscous, mu=0.01 if viscous else 0.0,
                    Pr=0.72, state_offset=(1.0, v, v, 1.0 / 0.4 + v * v, 0.0))

    groups = []
    for order, n, viscous in ((2, 32, False), (3, 32, False), (3, 32, True), (5, 24, True)):
        batch = [vcase(order, n, viscous, s) for s in range(ncase)]
        eng = BatchEngine(precision="fp32", steps_per_launch=10, **flux)
        walls = []
        for rep in range(4):  # the first batch tunes the group; best of the other three
            ids = [eng.admit(c) for c in batch]
            assert None not in ids
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            left = set(ids)
            while left:
                eng.advance()
                for cid in eng.poll():
                    left.discard(cid)
            if rep > 0:
                walls.append(time.perf_counter() - t0)
            for cid in ids:
                eng.fetch(cid, batch[0].u0.shape)
        wall = min(walls)
        tuned = eng.groups()
        eng.close()
        nodes = sum(c.mesh.num_nodes for c in batch)
        big = vcase(order, int(round(n * np.sqrt(ncase))), viscous, 0)
        op = (T.NSOperator if viscous else T.EulerOperator)(
            big.mesh, precision="fp32", mu=big.mu, Pr=big.Pr, state_offset=list(big.state_offset), **flux)
        u = torch.as_tensor(big.u0, device="cuda").contiguous()
        op.rk3_steps(u, big.dt, 5)
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        op.rk3_steps(u, big.dt, steps)
        b.record()
        torch.cuda.synchronize()
        one = 3 * steps * big.mesh.num_nodes / (a.elapsed_time(b) * 1e-3)
        del op, u
        batched = 3 * steps * nodes / wall
        groups.append({"order": order, "mesh": [n, n], "navier_stokes": viscous, "cases": ncase,
                       "batched_dof_rhs_per_s": batched, "one_case_dof_rhs_per_s": one,
                       "one_case_mesh": [int(round(n * np.sqrt(ncase)))] * 2,
                       "ratio": batched / one, "tuned": tuned[0] if tuned else None})
    return {"metric": "batched / one-case DOF*RHS/s (FP32-mixed, equal 2-D cases)",
            "value": float(np.mean([g["ratio"] for g in groups])), "unit": "ratio",
            "steps": steps, "groups": groups}


def run_serving(args):
    """Batched serving of the mixed 2-D stream: N cases (Poisson arrivals at
    2000/s) through the batch engine in FP32-mixed, against the same cases
    run one at a time on the plain FP64 path (a seeded sample of them), whose
    results also give each served case's final-solution error."""
    import torch
    import theseus_b200 as T
    from theseus_b200.serving import BatchEngine, SyntheticStream, serve
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    stream = SyntheticStream(args.cases, rate=2000.0, seed=0)
    reqs = [stream.case(i, lazy=True) for i in range(args.cases)]
    sample = set(range(0, args.cases, max(1, args.cases // args.sample)))
    flux = dict(numerical_flux="chandrashekar", surface_flux="roe")

    # one case at a time, plain FP64 (create, upload, steps, download, free)
    def one(c):
        op = (T.NSOperator if c.viscous else T.EulerOperator)(c.mesh, mu=c.mu, Pr=c.Pr, **flux)
        u = torch.as_tensor(c.state(), device="cuda").contiguous()
        op.rk3_steps(u, c.dt, c.nsteps)
        out = u.cpu().numpy()
        del op
        return out
    one(reqs[0])  # warm-up (library load, first kernels)
    ref = {}
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for i in sorted(sample):
        ref[i] = one(reqs[i])
    torch.cuda.synchronize()
    base_s = time.perf_counter() - t0
    base_rate = len(sample) / base_s
    for i in sample:
        reqs[i].u0 = None

    errs = []

    worst = []

    def keep(i, out):
        if i in ref:
            r = ref[i]
            groups = [[0], [1, 2], [3]]
            e = max(float(np.sqrt(((out[g] - r[g]) ** 2).sum() / (r[g] ** 2).sum())) for g in groups)
            errs.append(e)
            worst.append((e, {k: v for k, v in reqs[i].tag.items() if k != "arrival"}))

    eng = BatchEngine(precision="fp32", steps_per_launch=args.chunk, **flux)
    host = {}
    with ClockSampler(int(os.environ.get("LOCAL_RANK", "0"))) as clk:
        try:
            _, lat, makespan = serve(eng, reqs, on_result=keep, host=host, admitters=args.admitters)
        except Exception:
            free, total = torch.cuda.mem_get_info()
            print(json.dumps({"serving_failed": True, "engine": eng.stats(), "host_seconds": host,
                              "device_free_bytes": free, "device_total_bytes": total,
                              "budget_bytes": eng.hbm_budget}), file=sys.stderr, flush=True)
            raise
    st = eng.stats()
    tuned = eng.groups()
    eng.close()
    nodes = [r.mesh.num_nodes for r in reqs]
    line = {"metric": "solves/s (batched serving, FP32-mixed, 200 SSP-RK3 steps per case)",
            "value": args.cases / makespan, "unit": "solves/s", "n_gpus": 1,
            "higher_is_better": True, "dtype": "f32-mixed", "data": "synthetic",
            "config": {"workload": "serving_2d_mixed_stream", "cases": args.cases,
                       "arrival_rate_per_s": 2000.0, "sides": [8, 64], "orders": [2, 5],
                       "mach": [0.1, 2.0], "reynolds": [100, 1e4], "inviscid_fraction": 0.5,
                       "steps_per_case": 200, "steps_per_launch": args.chunk,
                       "admitters": args.admitters,
                       "mean_nodes_per_case": float(np.mean(nodes)), "fluxes": flux},
            "latency_s": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                          "max": float(lat.max())},
            "makespan_s": makespan,
            "dof_rhs_per_s": 3 * 200 * float(np.sum(nodes)) / makespan,
            "one_at_a_time_fp64": {"solves_per_s": base_rate, "sample_cases": len(sample),
                                   "seconds": base_s},
            "speedup_vs_one_at_a_time": (args.cases / makespan) / base_rate,
            "final_solution_rel_l2_vs_fp64": {"max": max(errs) if errs else None,
                                              "median": float(np.median(errs)) if errs else None,
                                              "cases": len(errs),
                                              "norm": "per conserved field (rho, momentum, E)",
                                              "worst": [dict(p, err=e) for e, p in
                                                        sorted(worst, key=lambda x: -x[0])[:3]]},
            "engine": st, "engine_groups": tuned, "host_seconds": host, "clocks": clk.summary()}
    return line


def run_lte(args):
    """LTE-gas Taylor-Green vortex: 24^3 hexes, p=4, LTEEC volume and face
    fluxes, a 256 x 512 synthetic Helmholtz table (ideal dissociating O2),
    rho = 0.01 kg/m^3, T = 3000 K, U0 = 300 m/s (Ma ~ 0.3), Navier-Stokes with the
    table's transport planes, FP64.  Reports RHS throughput, per-kernel times,
    Newton recoveries/s and LTEEC pair evaluations/s, the error of the GPU RHS
    against the FP64 oracle on a 3^3 sub-mesh, and a fixed-dt SSP-RK3 run."""
    import torch
    import theseus_b200 as T
    from theseus_b200 import cases
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    gas = dict(R=8.314462618 / 0.0319988, rho_d=1.5e5, theta_d=59500.0, mu0=1.9e-5, T0=273.15, Pr=0.71)
    tab = T.HelmholtzTable.ideal_dissociating_gas(256, 512, (-6.0, 1.0), (2.3, 4.3), **gas)
    n = args.lte_n
    m = T.periodic_box(3, 4, (n, n, n), [0.0] * 3, [2 * np.pi] * 3)
    u = cases.lte_taylor_green(m.coords)
    op = T.NSOperator(m, numerical_flux="lteec", surface_flux="lteec", gas=tab, Pr=0.71)
    ud = torch.as_tensor(u, device="cuda").contiguous()
    du = torch.empty_like(ud)
    for _ in range(max(args.warmup, 3)):
        op.Mult(ud, du)
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream()
    with ClockSampler(int(os.environ.get("LOCAL_RANK", "0"))) as clk:
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(args.steps):
            op.Mult(ud, du)
        b.record(stream)
        torch.cuda.synchronize()
    ms = a.elapsed_time(b) / args.steps
    ph = np.mean([op.profile(ud, du) for _ in range(3)], axis=0)
    status = op.read_status()
    N = 5
    pairs = m.num_elements * 3 * N * N * (N * (N - 1) // 2)
    # parity on a sub-mesh against the oracle (same table, same state formula)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    ms_ = T.periodic_box(3, 4, (3, 3, 3), [0.0] * 3, [2 * np.pi] * 3)
    us = cases.lte_taylor_green(ms_.coords)
    ops = T.NSOperator(ms_, numerical_flux="lteec", surface_flux="lteec", gas=tab, Pr=0.71)
    us_d = torch.as_tensor(us, device="cuda").contiguous()
    dus = torch.empty_like(us_d)
    ops.Mult(us_d, dus)
    om = O.Mesh(ms_.dim, ms_.order, ms_.jac, ms_.metric, ms_.face_elem, ms_.face_lface,
                ms_.face_normal, ms_.face_wminus, ms_.face_wplus)
    cfg = T.make_config(flow="ns", volume_flux="lteec", surface_flux="lteec", Pr=0.71)
    ot = O.LteTable(256, 512, (-6.0, 1.0), (2.3, 4.3))
    ref = O.rhs_lte(om, cfg, ot, us, nthreads=O.max_threads())
    got = dus.cpu().numpy()
    rel = np.sqrt(((got - ref) ** 2).reshape(5, -1).sum(1) / (ref ** 2).reshape(5, -1).sum(1))
    # SSP-RK3 trajectory at a fixed dt (acoustic CFL ~0.3 on the LGL spacing)
    h = 2 * np.pi / n / 16.0
    dt = 0.3 * h / (300.0 + 1100.0)
    rk_ms, y = timed_rk3(op, ud, dt, args.rk_steps, stream)
    rk_status = op.read_status()
    line = {"metric": "DOF*RHS/s (LTE Helmholtz gas, LTEEC)", "value": m.num_nodes / (ms * 1e-3),
            "unit": "DOF*RHS/s", "n_gpus": 1, "ms_per_step": ms, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"lte_tgv_{n}^3_p4", "table": [256, 512], "log_rho": [-6, 1],
                       "log_T": [2.3, 4.3], "rho": 0.01, "T": 3000.0, "U0": 300.0, "flow": "ns"},
            "phase_ms": {"recovery+indicator": ph[0], "gradient": ph[1], "face": ph[2], "volume": ph[3]},
            "newton_recoveries_per_s": m.num_nodes / (ph[0] * 1e-3) if ph[0] > 0 else None,
            "lteec_pairs_per_s": pairs / (ph[3] * 1e-3), "status": status,
            "rhs_rel_l2_vs_oracle_3cubed": [float(x) for x in rel],
            "rk3": {"steps": args.rk_steps, "dt": dt, "ms": rk_ms, "status": rk_status,
                    "dof_rhs_per_s": 3 * args.rk_steps * m.num_nodes / (rk_ms * 1e-3)},
            "clocks": clk.summary()}
    return line


def run_sedov(args):
    """Sedov-type blast: 64^3 hexes, p=3 (16.8 M nodes), Euler, Chandrashekar
    volume / LLF surface flux, Persson-Peraire indicator with subcell
    finite-volume (LLF) blending (alpha_max 0.5, alpha_min 0.001), rho = 1,
    p = 1e-5, energy 1.0 as a normalised Gaussian of width 0.05 on the periodic
    [-1, 1]^3.  FP64 and FP32-mixed RHS throughput, per-kernel times, the
    fraction of blended elements, the GPU RHS against the FP64 oracle on a
    4^3 sub-mesh, and a fixed-dt SSP-RK3 run (dt from CFL 0.5 at t = 0) in both
    precisions with the final-solution difference."""
    import torch
    import theseus_b200 as T
    from theseus_b200 import cases
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    n = args.sedov_n
    kw = dict(numerical_flux="chandrashekar", surface_flux="llf", fv_flux="llf", blending=True,
              alpha_max=0.5, alpha_min=0.001)
    m = T.periodic_box(3, 3, (n, n, n), [-1.0] * 3, [1.0] * 3)
    u = cases.sedov(m.coords, width=0.05)
    stream = torch.cuda.current_stream()
    out = {}
    for prec in ("fp64", "fp32"):
        op = T.EulerOperator(m, precision=prec, **kw)
        ud = torch.as_tensor(u, device="cuda").contiguous()
        du = torch.empty_like(ud)
        for _ in range(max(args.warmup, 3)):
            op.Mult(ud, du)
        torch.cuda.synchronize()
        with ClockSampler(int(os.environ.get("LOCAL_RANK", "0"))) as clk:
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            for _ in range(args.steps):
                op.Mult(ud, du)
            b.record(stream)
            torch.cuda.synchronize()
        ms = a.elapsed_time(b) / args.steps
        ph = np.mean([op.profile(ud, du) for _ in range(3)], axis=0)
        alpha, _ = op.blending_coefficients()
        dt = op.estimate_dt(ud, 0.5) if prec == "fp64" else out["fp64"]["rk3"]["dt"]
        rk_ms, y = timed_rk3(op, ud, dt, args.sedov_steps, stream)
        out[prec] = {"dof_rhs_per_s": m.num_nodes / (ms * 1e-3), "ms_per_rhs": ms,
                     "phase_ms": {"indicator": ph[0], "face": ph[2], "volume+fv": ph[3]},
                     "blended_fraction": float((alpha > 0).float().mean().item()),
                     "_alpha": alpha.cpu().numpy(),
                     "status": op.read_status(), "clocks": clk.summary(),
                     "rk3": {"steps": args.sedov_steps, "dt": dt, "ms": rk_ms,
                             "dof_rhs_per_s": 3 * args.sedov_steps * m.num_nodes / (rk_ms * 1e-3)},
                     "_final": y.cpu().numpy()}
        del op, ud, du, y
        torch.cuda.empty_cache()
    r64, r32 = out["fp64"].pop("_final"), out["fp32"].pop("_final")
    a64, a32 = out["fp64"].pop("_alpha"), out["fp32"].pop("_alpha")
    agreement = {"same_blended_set": float(np.mean((a64 > 0) == (a32 > 0))),
                 "max_abs_alpha_diff": float(np.abs(a64 - a32).max())}
    groups = [[0], [1, 2, 3], [4]]
    fin = {name: float(np.sqrt(((r32[g] - r64[g]) ** 2).sum() / (r64[g] ** 2).sum()))
           for name, g in zip(("density", "momentum", "energy"), groups)}
    # parity on a sub-mesh against the oracle (same state formula)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    ms_ = T.periodic_box(3, 3, (4, 4, 4), [-1.0] * 3, [1.0] * 3)
    us = cases.sedov(ms_.coords, width=0.05)
    ops = T.EulerOperator(ms_, **kw)
    us_d = torch.as_tensor(us, device="cuda").contiguous()
    dus = torch.empty_like(us_d)
    ops.Mult(us_d, dus)
    om = O.Mesh(ms_.dim, ms_.order, ms_.jac, ms_.metric, ms_.face_elem, ms_.face_lface,
                ms_.face_normal, ms_.face_wminus, ms_.face_wplus)
    cfg = T.make_config(flow="euler", volume_flux="chandrashekar", surface_flux="llf", fv_flux="llf",
                        blending=True, alpha_max=0.5, alpha_min=0.001)
    ref, _, _ = O.rhs(om, cfg, us, nthreads=O.max_threads(), want_alpha=True)
    got = dus.cpu().numpy()
    num = np.sqrt(((got - ref) ** 2).reshape(5, -1).sum(1))
    den = np.sqrt((ref ** 2).reshape(5, -1).sum(1))
    rel = np.where(den > 0, num / np.where(den > 0, den, 1.0), num)  # absolute where ref is 0
    line = {"metric": "DOF*RHS/s (Euler, Persson-Peraire + subcell FV blending)",
            "value": out["fp64"]["dof_rhs_per_s"], "unit": "DOF*RHS/s", "n_gpus": 1,
            "ms_per_step": out["fp64"]["ms_per_rhs"], "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"sedov_{n}^3_p3", "nodes": m.num_nodes, "rho": 1.0, "p": 1e-5,
                       "energy": 1.0, "width": 0.05, "fluxes": {"volume": "chandrashekar",
                                                                "surface": "llf", "fv": "llf"},
                       "alpha_max": 0.5, "alpha_min": 0.001, "cfl": 0.5},
            "fp64": out["fp64"], "fp32_mixed": out["fp32"],
            "fp32_speedup": out["fp32"]["dof_rhs_per_s"] / out["fp64"]["dof_rhs_per_s"],
            "final_solution_rel_l2_fp32_vs_fp64": dict(fin, max=max(fin.values())),
            "blending_agreement_t0": agreement,
            "rhs_rel_l2_vs_oracle_4cubed": [float(x) for x in rel],
            "rhs_vs_oracle_note": "absolute L2 for fields whose oracle rate is zero (mass at rest)"}
    return line


def run_setup(args):
    """Mesh set-up on the device: a 64^3 hexahedral box at p=3 (262,144 cells,
    16.8 M nodes) from its cells -- the face table built by the library on
    the host (thx_cell_faces), the geometric factors (Jacobian, adjugate
    metric, node coordinates, face normals and lift weights) computed by the
    device kernels (thx_cell_geometry) -- against the library's host box
    builder (thx_box_geometry) for the same mesh, with the largest relative
    difference of the factors."""
    import torch
    import theseus_b200 as T
    from theseus_b200.cells import cell_faces, cell_geometry
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    n, order, dim = args.setup_n, 3, 3
    h = 1.0 / n
    ijk = np.stack(np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij"), -1).reshape(-1, 3)[:, ::-1]
    off = np.array([[(v >> d) & 1 for d in range(3)] for v in range(8)])
    cell = ijk[:, None, :] + off[None, :, :]                      # (ne, 8, 3) lattice corners
    corners = cell * h
    ids = ((cell % n) * np.array([1, n, n * n])).sum(-1).astype(np.int64)
    t0 = time.perf_counter()
    fe, fl, be, bl = cell_faces(dim, ids)
    faces_s = time.perf_counter() - t0
    geo = cell_geometry(dim, order, corners, fe, fl, be, bl)     # warm-up (module load, allocation)
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    import ctypes as C
    from theseus_b200.cells import _lib as cells_lib
    lib = cells_lib()
    cd = torch.as_tensor(corners.astype(np.float64), device="cuda").contiguous()
    fed, fld = (torch.as_tensor(x, device="cuda").contiguous() for x in (fe, fl))
    ptr = lambda t: C.c_void_p(t.data_ptr()) if t is not None and t.numel() else None
    a.record(stream)
    for _ in range(args.steps):
        lib.thx_cell_geometry(dim, order, len(ids), ptr(cd), len(fe), ptr(fed), ptr(fld), 0, None, None,
                              ptr(geo["jac"]), ptr(geo["metric"]), ptr(geo["face_normal"]), ptr(geo["face_wminus"]),
                              ptr(geo["face_wplus"]), None, None, ptr(geo["coords"]), C.c_void_p(stream.cuda_stream))
    b.record(stream)
    torch.cuda.synchronize()
    dev_ms = a.elapsed_time(b) / args.steps
    t0 = time.perf_counter()
    ref = T.periodic_box(dim, order, (n, n, n), [0.0] * 3, [1.0] * 3)
    host_s = time.perf_counter() - t0
    jac, met = geo["jac"].cpu().numpy(), geo["metric"].cpu().numpy()
    diff = max(float(np.abs(jac - ref.jac).max() / np.abs(ref.jac).max()),
               float(np.abs(met - ref.metric).max() / np.abs(ref.metric).max()))
    nodes, nfp = len(ids) * (order + 1) ** 3, (order + 1) ** 2
    written = nodes * 8 * (1 + 9 + 3) + len(fe) * nfp * 8 * (3 + 2)
    read = len(ids) * 8 * 3 * 8 + len(fe) * 16 + len(fe) * nfp * (2 * 8 + 3 * 8)
    gbs = (read + written) / (dev_ms * 1e-3) / 1e9
    peak, src = peaks()
    line = {"metric": "mesh set-up time (geometric factors on the device)", "value": dev_ms, "unit": "ms",
            "higher_is_better": False, "n_gpus": 1, "steps": args.steps, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"setup_box_{n}^3_p{order}", "cells": len(ids), "nodes": nodes,
                       "faces": len(fe)},
            "face_table_host_s": faces_s, "host_box_builder_s": host_s,
            "speedup_vs_host_builder": host_s / (dev_ms * 1e-3),
            "max_rel_diff_vs_host_builder": diff,
            "roofline": {"bound": "hbm", "achieved": gbs, "peak": peak, "unit": "GB/s", "frac": gbs / peak,
                         "peak_source": src, "algorithmic_bytes": read + written}}
    return line


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="fp64", choices=["fp64", "fp32"])
    ap.add_argument("--skip-cpu", action="store_true")
    ap.add_argument("--no-mixed", action="store_true")
    ap.add_argument("--n", type=int, default=32, help="elements per direction (profiling cases)")
    ap.add_argument("--rk-steps", type=int, default=200, help="SSP-RK3 steps of the precision comparison")
    ap.add_argument("--workload", default="rhs",
                    choices=["rhs", "serving", "lte", "sedov", "setup", "vortex", "trials", "batch"],
                    help="rhs: the headline RHS throughput (with compact results of vortex, "
                         "sedov, lte and serving unless --no-workloads); serving: the batched "
                         "case stream; lte: the LTE-gas Taylor-Green vortex; sedov: the blended "
                         "blast; setup: mesh set-up on the device; vortex: the 2-D isentropic vortex; "
                         "trials: the tensor-core trial of the gradient's derivative contraction; "
                         "batch: batched against one-case kernels on equal 2-D cases")
    ap.add_argument("--volume-staging", type=int, default=0, choices=[0, 1],
                    help="rhs: 1 stages each element block's state by bulk copy (TMA) in the "
                         "volume kernel")
    ap.add_argument("--no-workloads", action="store_true",
                    help="rhs: skip the other configurations")
    ap.add_argument("--sedov-n", type=int, default=64, help="sedov: elements per direction")
    ap.add_argument("--sedov-steps", type=int, default=300, help="sedov: SSP-RK3 steps")
    ap.add_argument("--lte-n", type=int, default=24, help="lte: elements per direction")
    ap.add_argument("--setup-n", type=int, default=64, help="setup: cells per direction")
    ap.add_argument("--cases", type=int, default=4096, help="serving: cases in the stream")
    ap.add_argument("--sample", type=int, default=256, help="serving: cases also run one at a time")
    ap.add_argument("--chunk", type=int, default=10, help="serving: SSP-RK3 steps per graph launch")
    ap.add_argument("--batch-steps", type=int, default=1000, help="batch: SSP-RK3 steps per case")
    ap.add_argument("--admitters", type=int, default=1,
                    help="serving: host threads setting up arriving cases (1: strict arrival order)")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "rhs":
        run_ours(args)
    else:
        fn = {"serving": run_serving, "lte": run_lte, "sedov": run_sedov, "setup": run_setup,
              "vortex": run_vortex, "trials": run_trials, "batch": run_batch}[args.workload]
        print(json.dumps(fn(args)), flush=True)


if __name__ == "__main__":
    main()

#!/usr/bin/env python
"""Benchmark of the projection engine on its headline workload.

Workload (one step): fan-beam forward projection followed by the matched
backprojection of a 2048 x 2048 float32 ellipse phantom; 1440 views over
[0, 2 pi), 2048 detectors of unit pitch at the isocentre, source 8192 px from
the isocentre.  Unit: Gray-px/s = 1e9 ray-pixel updates per second, an update
being one nonzero entry of the projection operator visited (counted exactly on
the device; forward and backward counts summed).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 runs N independent replicas (the engine is single-GPU; slices shard
with no collective), one process per GPU: without torchrun's environment the
script starts torchrun itself.  value = all ranks' updates / the slowest rank's
time.  --impl reference times the reference's own CPU projector (prj/cpuPrj.c
compiled unchanged into oracle/_ref) on the host cores, on the same workload
and the same number of steps.
"""
import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "fwd+adjoint Gray-px/s & BHC grad-iter/s vs plain path, 1 B200, rel err≤1e-5"
WORKLOAD = dict(workload="fan-beam fwd+backprojection 2048^2, 1440 views/[0,2pi), 2048 bins, "
                         "d=8192 px, float32 ellipse phantom",
                n=2048, prjWidth=2048, np=1440, prjFull=1440, dSize=1.0, effectiveRate=1.0, d=8192.0)
L2_FLUSH_BYTES = 512 << 20   # > 126 MB L2
# polychromatic (BHC) gradient iteration on the same geometry: two-material
# phantom (0 / 2.7 / 7.8 g/cm^3), J = 30 b1 coefficients on kappa log-spaced over
# [1e-2, 1e2] cm^2/g, Poisson counts at I0 = 1e5 per ray, 2 cm field of view
BHC = dict(J=30, I0=1e5, fov_cm=2.0)
# the double-precision masked parallel operator (mParPrj) measured beside
PARPRJ = dict(n=512, prjWidth=727, np=360)
# the polychromatic model's own configuration: fan 1024^2, 720 views over
# [0, 2 pi), 1024 detectors, source 2048 px from the isocentre
BHC_WORKLOAD = dict(n=1024, prjWidth=1024, np=720, prjFull=720, dSize=1.0, effectiveRate=1.0, d=2048.0)
# the projector alone on each configuration's geometry (--legs geometries):
# (n, prjWidth, np, prjFull, dSize, effectiveRate, d)
GEOMETRIES = {
    "par256 (config 1)": (256, 363, 180, 360, 1.0, 1.0, 0.0),
    "fan512 d=2048 (config 2)": (512, 1024, 360, 360, 1.0, 1.0, 2048.0),
    "fan512 d=1024": (512, 512, 360, 360, 1.0, 1.0, 1024.0),
    "fan1024 d=2048 (config 3)": (1024, 1024, 720, 720, 1.0, 1.0, 2048.0),
    "par2048": (2048, 2048, 1440, 1440, 1.0, 1.0, 0.0),
    "fan2048 d=8192 (config 5, headline)": (2048, 2048, 1440, 1440, 1.0, 1.0, 8192.0),
}


def run_config(world):
    """The `config` of both arms' lines, identical by construction: the
    workload, how the timed steps treat the GPU's L2, and the process layout."""
    return dict(WORKLOAD, l2="GPU arm: 512 MiB written between timed steps (L2 flushed); "
                             "reference arm: the same steps on the host cores",
                parallelism="replicas" if world > 1 else "single GPU")


def geometry_tuple(w):
    return (w["n"], w["prjWidth"], w["np"], w["prjFull"], w["dSize"], w["effectiveRate"], w["d"])


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock / throttle-reason samples for one GPU while running."""
    FIELDS = ("uuid,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, uuid):
        self.uuid = uuid
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "--query-gpu=" + self.FIELDS, "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 8 or (self.uuid and self.uuid not in parts[0]):
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[4:8]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def max_over_ranks(v, pg, device):
    """The largest of the ranks' values of v (every rank gets it); v itself
    when there is no process group."""
    if pg is None:
        return float(v)
    import torch
    t = torch.tensor([float(v)], dtype=torch.float64, device=device)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def replica_value(world, updates_per_rank, t_max_ms):
    """Whole-job throughput of `world` independent replicas in Gray-px/s: all
    ranks' updates over the slowest rank's time."""
    return world * updates_per_rank / (t_max_ms * 1e-3) / 1e9


def init_dist():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def cpu_reference_run(steps, warmup, w=None):
    """The reference's own prj/cpuPrj.c (oracle/_ref) -- or, where it was not
    compiled, the oracle's FP32 port -- on workload w (default: the headline
    workload itself): each step is one forward and one backward pass over the
    same phantom as the GPU arm.  Returns (updates/s, median seconds per step,
    info)."""
    import types

    import oracle
    from oracle import ref
    from imgrecsrc_b200 import phantom
    g = types.SimpleNamespace(**(w or WORKLOAD))
    x = phantom.ellipse_phantom(g.n, seed=1)
    nnz = oracle.forward_nnz(g) + oracle.backward_nnz(g)
    ncores = os.cpu_count() or 1
    if ref.available("libref_prj32"):
        kind, cores = "reference", min(64, ncores)   # cpuPrj.c runs 64 pthreads

        def step():
            s = ref.forward(g, x, prec=32)
            ref.backward(g, s, prec=32)
    else:
        kind, cores = "port", ncores

        def step():
            s = oracle.forward(g, x, prec=32, threads=ncores)
            oracle.backward(g, s, prec=32, threads=ncores)
    for _ in range(warmup):
        step()
    times = []
    for _ in range(steps):
        t0 = time.perf_counter()
        step()
        times.append(time.perf_counter() - t0)
    t = statistics.median(times)
    sample = ("fan %d^2, %d views/[0,2pi), %d bins, d=%g px (the headline workload itself): one "
              "forward + one backward pass per step, %d timed after %d warm-up; %d nonzero updates "
              "per step; host has %d cores" % (g.n, g.np, g.prjWidth, g.d, steps, warmup, nnz, ncores))
    return nnz / t / 1e9, t, dict(kind=kind, cores=cores, sample=sample)


def reference_arm(args):
    """The reference's CPU projector on the same workload, metric and step
    counts as the GPU arm (one full forward + backward pass per step, about
    6 s each on a 16-core host).  Under torchrun rank 0 alone runs it."""
    world, rank, _ = init_dist()
    if world != args.gpus:
        raise SystemExit("bench.py: %d ranks started for --gpus %d" % (world, args.gpus))
    if rank != 0:
        return
    steps, warmup = max(1, args.steps), max(3, args.warmup)
    v, t, info = cpu_reference_run(steps, warmup)
    line = {"metric": METRIC, "value": v, "unit": "Gray-px/s", "n_gpus": args.gpus,
            "steps": steps, "warmup": warmup, "ms_per_step": t * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded ellipse phantom)",
            "impl": "reference", "config": run_config(world),
            "cpu_baseline": dict(value=v, unit="Gray-px/s", **info),
            "e2e": {"value": v, "unit": "Gray-px/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def cpu_parprj_run():
    """The reference's own prj/parPrj.c (oracle/_ref) on the host cores, on the
    masked parallel operator workload of extras_leg: (forward s, backward s)."""
    import numpy as np

    from oracle import ref
    if not ref.available("libref_parprj"):
        return None
    n, W, nang = PARPRJ["n"], PARPRJ["prjWidth"], PARPRJ["np"]
    r = np.arange(n) - (n - 1) / 2
    mask = np.flatnonzero(((r[:, None] ** 2 + r[None, :] ** 2) <= (0.48 * n) ** 2).ravel(order="F"))
    conf = dict(bw=1.0, nc=n, nr=n, prjWidth=W, theta=np.arange(nang) * 180.0 / nang)
    x = np.random.default_rng(5).random(mask.size)
    t0 = time.perf_counter()
    y = ref.par_forward(x, mask, conf)
    t1 = time.perf_counter()
    ref.par_backward(y, mask, conf)
    t2 = time.perf_counter()
    return t1 - t0, t2 - t1


def our_arm(args):
    import numpy as np
    import torch

    world, rank, local = init_dist()
    if world != args.gpus:
        raise SystemExit("bench.py: %d ranks started for --gpus %d" % (world, args.gpus))
    torch.cuda.set_device(local)
    pg = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
        pg = dist
    import imgrecsrc_b200 as ct
    from imgrecsrc_b200 import phantom

    g = ct.Geometry(*geometry_tuple(WORKLOAD))
    pr = ct.Projector(g, device=local)
    nnz_f, nnz_b = pr.count_updates()
    x = torch.from_numpy(phantom.ellipse_phantom(g.n, seed=1)).cuda()
    sino = torch.empty(g.np, g.prjWidth, device="cuda")
    back = torch.empty(g.n, g.n, device="cuda")
    flush = torch.empty(L2_FLUSH_BYTES // 4, device="cuda")
    stream = torch.cuda.current_stream()

    def step():
        pr.forward(x, out=sino)
        pr.backward(sino, out=back)

    for _ in range(max(3, args.warmup)):
        flush.zero_()
        step()
    torch.cuda.synchronize()

    uuid = None
    try:
        uuid = str(torch.cuda.get_device_properties(local).uuid)
    except Exception:
        pass
    clocks = ClockSampler(uuid)
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    clocks.start()
    time.sleep(0.3)
    ev = [[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in range(args.steps)]
    for i in range(args.steps):
        flush.zero_()                     # L2 flushed between timed steps (outside the events)
        ev[i][0].record(stream)
        pr.forward(x, out=sino)
        ev[i][1].record(stream)
        pr.backward(sino, out=back)
        ev[i][2].record(stream)
    torch.cuda.synchronize()
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    clk = clocks.stop()
    t_fwd = [ev[i][0].elapsed_time(ev[i][1]) for i in range(args.steps)]
    t_bwd = [ev[i][1].elapsed_time(ev[i][2]) for i in range(args.steps)]
    t_step = sum(a + b for a, b in zip(t_fwd, t_bwd)) / args.steps   # ms
    t_max = max_over_ranks(t_step, pg, "cuda")
    value = replica_value(world, nnz_f + nnz_b, t_max)

    # roofline of the dominant kernel: 4 B per update + the compulsory image and
    # sinogram streams; duration from the CUDA events around its launch
    fwd_ms, bwd_ms = statistics.mean(t_fwd), statistics.mean(t_bwd)
    compulsory = 4 * (g.n * g.n + g.np * g.prjWidth)
    if bwd_ms >= fwd_ms:
        kname, kms, kbytes = "k_backward_tiled<fan>", bwd_ms, 4 * nnz_b + compulsory
    else:
        kname, kms, kbytes = "k_quad + k_forward<fan>", fwd_ms, 4 * nnz_f + compulsory + 12 * g.n * g.n
    peak, peak_kind = peaks()
    achieved = kbytes / (kms * 1e-3) / 1e9
    prof = profiled_kernels().get("k_backward_tiled<fan>" if bwd_ms >= fwd_ms else "k_forward<fan>", {})
    traffic = prof.get("dram_bytes_per_launch")
    issue = issue_roof(prof, kname, kms, clk.get("sm_mhz"), nnz_b if bwd_ms >= fwd_ms else nnz_f)
    shared = shared_roof(prof, kname, kms, clk.get("sm_mhz"))

    bhc_line = batch_line = extras_line = loop_line = None
    if args.legs in ("all", "bhc"):
        # BHC gradient iterations on the polychromatic model's own configuration
        # (fan 1024^2, 720 views, 1024 bins, J = 20) and on the 2048^2 geometry
        g3 = ct.Geometry(*geometry_tuple(BHC_WORKLOAD))
        pr3 = ct.Projector(g3, device=local)
        bhc_line = {"fan_1024": bhc_leg(ct, g3, pr3, flush, stream, max(3, args.steps // 2), 20,
                                        "fan 1024^2, 720 views/[0,2pi), 1024 bins, d=2048 px"),
                    "fan_2048": bhc_leg(ct, g, pr, flush, stream, max(3, args.steps // 2), BHC["J"],
                                        "fan 2048^2, 1440 views, 2048 bins, d=8192 px")}
        pr3.close()
    if args.legs == "all":
        batch_line = batch_leg(ct, flush, stream, max(3, args.steps // 2))
        extras_line = extras_leg(ct, g, pr, flush, stream, max(3, args.steps // 2))
        if args.loop_iters > 0:
            if args.loop_geometry == "1024":
                gl = ct.Geometry(*geometry_tuple(BHC_WORKLOAD))
                prl = ct.Projector(gl, device=local)
                loop_line = loop_leg(ct, gl, prl, args.loop_iters)
                prl.close()
            else:
                loop_line = loop_leg(ct, g, pr, args.loop_iters)

    # end to end through the reference-facing C ABI: setup() once, then per
    # step gpuPrj(FWD) and gpuPrj(BWD) on pinned host buffers (every call
    # copies its input to the device and its result back, as the reference does)
    os.environ["CTPRJ_DEVICE"] = str(local)
    L = ct.lib()
    L.setup(*geometry_tuple(WORKLOAD))
    h_img = torch.from_numpy(phantom.ellipse_phantom(g.n, seed=1)).pin_memory()
    h_sino = torch.empty(g.np, g.prjWidth).pin_memory()
    h_back = torch.empty(g.n, g.n).pin_memory()
    for _ in range(2):
        ct.check(L.gpuPrj(ctypes.c_void_p(h_img.data_ptr()), ctypes.c_void_p(h_sino.data_ptr()), bytes([ct.FWD_BIT])))
        ct.check(L.gpuPrj(ctypes.c_void_p(h_back.data_ptr()), ctypes.c_void_p(h_sino.data_ptr()), bytes([ct.BWD_BIT])))
    e2e_times = []
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ct.check(L.gpuPrj(ctypes.c_void_p(h_img.data_ptr()), ctypes.c_void_p(h_sino.data_ptr()), bytes([ct.FWD_BIT])))
        ct.check(L.gpuPrj(ctypes.c_void_p(h_back.data_ptr()), ctypes.c_void_p(h_sino.data_ptr()), bytes([ct.BWD_BIT])))
        e2e_times.append(time.perf_counter() - t0)
    e2e_t = max_over_ranks(statistics.mean(e2e_times), pg, "cuda")
    e2e_val = replica_value(world, nnz_f + nnz_b, e2e_t * 1e3)
    img_b, sino_b = 4 * g.n * g.n, 4 * g.np * g.prjWidth
    # the same calls on pageable host buffers (the reference gateway's malloc'd
    # arrays, prj/mPrj.c:70-73), for the record
    p_img = np.ascontiguousarray(h_img.numpy().copy())
    p_sino = np.empty((g.np, g.prjWidth), np.float32)
    p_back = np.empty((g.n, g.n), np.float32)
    pageable_times = []
    for it in range(2 + min(args.steps, 5)):
        flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ct.check(L.gpuPrj(ctypes.c_void_p(p_img.ctypes.data), ctypes.c_void_p(p_sino.ctypes.data), bytes([ct.FWD_BIT])))
        ct.check(L.gpuPrj(ctypes.c_void_p(p_back.ctypes.data), ctypes.c_void_p(p_sino.ctypes.data), bytes([ct.BWD_BIT])))
        if it >= 2:
            pageable_times.append(time.perf_counter() - t0)
    pageable_t = max_over_ranks(statistics.mean(pageable_times), pg, "cuda")

    line = {
        "metric": METRIC, "value": value, "unit": "Gray-px/s", "n_gpus": world,
        "steps": args.steps, "warmup": max(3, args.warmup), "ms_per_step": t_max,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded ellipse phantom)",
        "config": run_config(world),
        "updates_per_step": {"forward": nnz_f, "backward": nnz_b},
        "pass_ms": {"forward": fwd_ms, "backward": bwd_ms},
        "roofline": {"bound": "hbm", "kernel": kname, "achieved": achieved, "peak": peak,
                     "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": traffic,
                     "bytes_per_launch": kbytes, "bytes_rule": "4 B per nonzero update + image + sinogram"},
        "e2e": {"value": e2e_val, "unit": "Gray-px/s", "h2d_bytes_per_step": img_b + sino_b,
                "d2h_bytes_per_step": sino_b + img_b, "api": "setup()/gpuPrj() C ABI, pinned host buffers",
                "ms_per_step": e2e_t * 1e3, "pageable_ms_per_step": pageable_t * 1e3},
        "gpu_launches": 3 * args.steps,
        "clocks": clk,
    }
    line["roofline"]["issue"] = issue
    if shared:
        line["roofline"]["shared"] = shared
    if rank == 0 and world == 1 and not args.no_cpu:
        # the reference's cpuPrj.c on the headline workload itself: 1 warm-up
        # and 3 timed passes (about 25 s on a 16-core host)
        v, t, info = cpu_reference_run(3, 1)
        line["cpu_baseline"] = dict(value=v, unit="Gray-px/s", **info)
        par = cpu_parprj_run()
        if par:
            line["cpu_baseline"]["parprj"] = {"kind": "reference", "forward_ms": par[0] * 1e3,
                                              "backward_ms": par[1] * 1e3,
                                              "threads": 32}   # parPrj.c runs 32 pthreads
    # the secondary legs in full, then (last, so that a tail of the output
    # keeps it) a compact summary of every leg's headline figures
    line.update({k: v for k, v in (("bhc", bhc_line), ("batch", batch_line), ("bhc_loop", loop_line),
                                   ("extras", extras_line)) if v is not None})
    line["summary"] = summary(line)
    if pg:
        pg.barrier()
        pg.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


def summary(line):
    """Headline figures of every leg in one short object (rounded)."""
    def r(v, k=4):
        return None if v is None else float("%.*g" % (k, v))
    c = line["pass_ms"]
    out = {"fwd_ms": r(c["forward"]), "bwd_ms": r(c["backward"]), "gray_px_s": r(line["value"]),
           "e2e_gray_px_s": r(line["e2e"]["value"]),
           "issue_frac": r((line["roofline"].get("issue") or {}).get("frac"), 3)}
    if line["roofline"].get("shared"):
        out["shared_frac"] = r(line["roofline"]["shared"]["frac"], 3)
    if "cpu_baseline" in line:
        out["cpu_gray_px_s"] = r(line["cpu_baseline"]["value"])
    for key, b in (line.get("bhc") or {}).items():
        out["bhc_" + key] = {"fused_grad_iter_per_s": r(b["fused_grad_iter_per_s"]),
                             "plain_grad_iter_per_s": r(b["plain_grad_iter_per_s"]),
                             "speedup_vs_plain": r(b["speedup_vs_plain"], 3),
                             "speedup_vs_plain_min": r(b["speedup_vs_plain_min"], 3)}
    bt = line.get("batch")
    if bt:
        out["batch"] = {"batched_ms": r(bt["batched_ms"]), "per_slice_ms": r(bt["per_slice_ms"]),
                        "speedup": r(bt["speedup"], 3)}
    lp = line.get("bhc_loop")
    if lp:
        out["loop"] = {k: r(lp[k]["iter_per_s"]) for k in lp if isinstance(lp[k], dict) and "iter_per_s" in lp[k]}
        out["loop"]["pg_speedup_fused_vs_unfused"] = r(lp["pg_speedup_fused_vs_unfused"], 3)
        out["loop"]["pg_final_cost"] = r(lp["pg_fused"]["final_cost"], 9)
    ex = line.get("extras")
    if ex:
        out["extras"] = {"fbp_ms": r(ex["fbp_ms"]), "tv_us_per_it": r(ex["tv_denoise"]["us_per_iteration"]),
                         "wvlt_us_per_it": r(ex["wvlt_admm"]["us_per_iteration"]),
                         "parprj_fwd_ms": r(ex["parprj"]["forward_ms"]),
                         "parprj_bwd_ms": r(ex["parprj"]["backward_ms"])}
    return out


def bhc_leg(ct, g, pr, flush, stream, steps, J, workload):
    """BHC gradient iterations per second: the fused forward (projection with
    the spline epilogue) + adjoint, against the plain FP32 projector path in
    the reference's call structure (bhc/beamhardenSpline.m:382-447: Phi(alpha),
    unfused polyIout + poissLAlpha terms, Phit; then Phi(alpha) again, the
    materialised rays x J basis matrix and A^T (1 - m/Ir) of poissLI) and
    against a minimal plain path (one projection, unfused terms, same adjoint).
    Each iteration yields f (FP64), df/dx and df/dIe."""
    import torch

    from imgrecsrc_b200 import bhc, phantom
    I0 = BHC["I0"]
    Ts = BHC["fov_cm"] / g.n
    x = torch.from_numpy(phantom.two_material_phantom(g.n, seed=2)).cuda()
    nodes = bhc.kappa_nodes(J)
    Ie = torch.from_numpy(phantom.spectrum_bump(J, seed=2)).cuda()
    model = bhc.BHCModel(pr, nodes, Ts)
    sino = pr.forward(x)
    A = model.basis(sino)
    BL = (A @ Ie).reshape(g.np, g.prjWidth)
    gen = torch.Generator(device="cuda").manual_seed(7)
    imea = (torch.poisson(I0 * BL, generator=gen) / I0).float().contiguous()
    del A, BL

    def fused():
        model.forward(x, Ie, imea, save=True)
        return model.backward()

    def plain_ref():
        s1 = pr.forward(x)
        model.terms(s1, Ie, imea, save=True)
        gx, _ = model.backward(grad_Ie=False)
        s2 = pr.forward(x)
        Am = model.basis(s2)
        gI = Am.t() @ (1 - imea.double().ravel() / (Am @ Ie))
        return gx, gI

    def plain_min():
        s1 = pr.forward(x)
        model.terms(s1, Ie, imea, save=True)
        return model.backward()

    out = {"workload": "%s; two-material phantom; J=%d b1 spectrum on [1e-2,1e2] cm^2/g; "
                       "Poisson counts I0=1e5; Ts=%g cm" % (workload, J, Ts),
           "iteration": "f (FP64) + df/dx + df/dIe"}
    for name, fn in (("fused", fused), ("plain", plain_ref), ("plain_min", plain_min)):
        for _ in range(2):
            fn()
        torch.cuda.synchronize()
        ms = 0.0
        for _ in range(steps):
            flush.zero_()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            fn()
            e1.record(stream)
            torch.cuda.synchronize()
            ms += e0.elapsed_time(e1)
        ms /= steps
        out[name + "_ms"] = ms
        out[name + "_grad_iter_per_s"] = 1e3 / ms
    out["speedup_vs_plain"] = out["plain_ms"] / out["fused_ms"]
    out["speedup_vs_plain_min"] = out["plain_min_ms"] / out["fused_ms"]
    out["fused_launches_per_iter"] = 6
    model.close()
    return out


def loop_leg(ct, g, pr, iters):
    """The alternating BHC reconstruction on geometry g (J = 30, Poisson counts at
    I0 = 1e5): `iters` iterations of a projected-gradient density step
    (npg/PG.m with the projection on x >= 0, majorisation line search) and an
    FP64 non-negative spectrum step (Newton with an active-set QP on Ie >= 0),
    on the fused path and on the plain FP32 unfused path, then the same with
    the reference's default accelerated density step (npg/NPG.m), and NPG with
    the isotropic TV proximal map (opt.proximal = 'tviso') and with the
    reference's default regulariser ('wvltADMM': Haar wavelet, 6 levels), both
    at its default weight u = 1e-3; iterations
    per second, likelihood evaluations, spectrum time, and how far apart the
    fused and unfused results are."""
    import torch

    from imgrecsrc_b200 import bhc, phantom
    J, I0 = BHC["J"], BHC["I0"]
    Ts = BHC["fov_cm"] / g.n
    x_true = torch.from_numpy(phantom.two_material_phantom(g.n, seed=2)).cuda()
    nodes = bhc.kappa_nodes(J)
    I_true = torch.from_numpy(phantom.spectrum_bump(J, seed=2)).cuda()
    model = bhc.BHCModel(pr, nodes, Ts)
    A = model.basis(pr.forward(x_true))
    BL = (A @ I_true).reshape(g.np, g.prjWidth)
    gen = torch.Generator(device="cuda").manual_seed(7)
    imea = (torch.poisson(I0 * BL, generator=gen) / I0).float().contiguous()
    del A, BL
    out = {"workload": "fan %d^2, %d views, %d bins, d=%g; J=30; I0=1e5; start x=1 g/cm^3, "
                       "Ie uniform; %d iterations of density step + spectrum step (<= 2 Newton steps)"
                       % (g.n, g.np, g.prjWidth, g.d, iters)}
    res = {}
    for name, method, unfused, prox in (("pg_fused", "pg", False, "nonneg"), ("pg_unfused", "pg", True, "nonneg"),
                                        ("npg_fused", "npg", False, "nonneg"),
                                        ("npg_tviso_fused", "npg", False, "tviso"),
                                        ("npg_wvlt_fused", "npg", False, "wvltADMM")):
        x = torch.full((g.n, g.n), 1.0, device="cuda")
        Ie = torch.full((J,), 1.0 / J, dtype=torch.float64, device="cuda")
        st = model.reconstruct(x, Ie, imea, iterations=iters, x_step=1e-3, unfused=unfused, method=method,
                               proximal=prox, u=1e-3)
        res[name] = (x, Ie)
        out[name] = {"iter_per_s": st["iterations"] / (st["ms"] * 1e-3), "ms": st["ms"],
                     "first_cost": st["cost"][0] if st["cost"] else None, "final_cost": st["final_cost"],
                     "evaluations": st["evaluations"], "ms_per_evaluation": st["ms"] / max(st["evaluations"], 1),
                     "ms_spectrum": st["ms_spectrum"], "newton_steps": st["newton_steps"],
                     "restarts": st["restarts"], "tv_inner_iterations": st["inner_iterations"],
                     "rel_err_vs_truth_x": (torch.linalg.norm((x - x_true).double())
                                            / torch.linalg.norm(x_true.double())).item()}
    out["pg_speedup_fused_vs_unfused"] = out["pg_fused"]["iter_per_s"] / out["pg_unfused"]["iter_per_s"]
    (xf, If), (xu, Iu) = res["pg_fused"], res["pg_unfused"]
    out["pg_fused_vs_unfused_rel_x"] = (torch.linalg.norm((xf - xu).double()) / torch.linalg.norm(xu.double())).item()
    out["pg_fused_vs_unfused_rel_Ie"] = (torch.linalg.norm(If - Iu) / torch.linalg.norm(Iu)).item()
    model.close()
    return out


def batch_leg(ct, flush, stream, steps):
    """64 slices of mixed geometry (n in {128..1024}, 90..720 views, half
    parallel, half fan): forward + backprojection of every slice, as one tuned,
    graph-captured persistent launch per direction, against a loop of per-slice
    ctprj_forward / ctprj_backward calls on the same stream."""
    import numpy as np
    import torch

    from imgrecsrc_b200 import batch, phantom
    geoms = batch.cfg4_geometries(64, seed=0)
    rng = np.random.default_rng(3)
    imgs = [torch.from_numpy(phantom.ellipse_phantom(g.n, seed=i)).cuda() for i, g in enumerate(geoms)]
    sinos = [torch.empty(g.np, g.prjWidth, device="cuda") for g in geoms]
    bimgs = [torch.empty(g.n, g.n, device="cuda") for g in geoms]
    projs = [ct.Projector(g) for g in geoms]
    updates = 0
    for p in projs:
        f, bw = p.count_updates()
        updates += f + bw
    b = batch.Batch(geoms)
    b.bind(imgs, sinos, sinos, bimgs)
    cfg = b.autotune(None)
    b.capture()

    def batched():
        b.forward()
        b.backward()

    def looped():
        for p, x, y, z in zip(projs, imgs, sinos, bimgs):
            p.forward(x, out=y)
            p.backward(y, out=z)

    out = {"workload": "64 seeded slices: n in {128,256,384,512,768,1024}, views in {90,180,360,720} "
                       "(fan 90 -> 92), half parallel [0,pi) / half fan [0,2pi) d=4n, prjWidth=ceil(1.42n)",
           "updates_per_step": updates, "tuned": cfg}
    for name, fn in (("batched", batched), ("per_slice", looped)):
        for _ in range(2):
            fn()
        torch.cuda.synchronize()
        ms = 0.0
        for _ in range(steps):
            flush.zero_()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            fn()
            e1.record(stream)
            torch.cuda.synchronize()
            ms += e0.elapsed_time(e1)
        ms /= steps
        out[name + "_ms"] = ms
        out[name + "_gray_px_per_s"] = updates / (ms * 1e-3) / 1e9
    out["speedup"] = out["per_slice_ms"] / out["batched_ms"]
    out["batched_launches_per_step"] = 5   # 2 counter resets, quad image, forward, backward
    b.close()
    for p in projs:
        p.close()
    return out


def extras_leg(ct, g, pr, flush, stream, steps):
    """FBP on the headline geometry, and the double-precision masked parallel
    operator of mParPrj (prj/parPrj.c) on device buffers: 512^2 image, a disc
    mask, 360 angles over [0, 180) degrees, 727 detectors; and the TV proximal
    map of the density step (100 FGP iterations on the headline image size)."""
    import ctypes

    import numpy as np
    import torch

    def timed(fn):
        for _ in range(2):
            fn()
        torch.cuda.synchronize()
        ms = 0.0
        for _ in range(steps):
            flush.zero_()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            fn()
            e1.record(stream)
            torch.cuda.synchronize()
            ms += e0.elapsed_time(e1)
        return ms / steps

    out = {}
    y = torch.randn(g.np, g.prjWidth, device="cuda", generator=torch.Generator(device="cuda").manual_seed(5))
    img = torch.empty(g.n, g.n, device="cuda")
    out["fbp_ms"] = timed(lambda: pr.fbp(y, out=img))
    n, W, nang = PARPRJ["n"], PARPRJ["prjWidth"], PARPRJ["np"]
    r = np.arange(n) - (n - 1) / 2
    mask = np.flatnonzero(((r[:, None] ** 2 + r[None, :] ** 2) <= (0.48 * n) ** 2).ravel(order="F"))
    theta = np.ascontiguousarray(np.arange(nang) * 180.0 / nang)
    conf = ct._lib.ParDevConf(1.0, n, n, nang, W)
    d_mask = torch.from_numpy(mask.astype(np.float64)).cuda()
    d_x = torch.rand(mask.size, dtype=torch.float64, device="cuda")
    d_y = torch.zeros(nang * W, dtype=torch.float64, device="cuda")
    d_b = torch.zeros(mask.size, dtype=torch.float64, device="cuda")
    L = ct.lib()
    hs = ctypes.c_void_p(stream.cuda_stream)
    vp = lambda t: ctypes.c_void_p(t.data_ptr())

    def fwd():
        d_y.zero_()
        ct.check(L.ctprj_par_forward(ctypes.byref(conf), theta.ctypes.data, vp(d_mask), mask.size,
                                     vp(d_x), vp(d_y), hs))

    def bwd():
        d_b.zero_()
        ct.check(L.ctprj_par_backward(ctypes.byref(conf), theta.ctypes.data, vp(d_mask), mask.size,
                                      vp(d_y), vp(d_b), hs))
    # the TV proximal map (FGP) on the headline image size, 100 iterations (epsilon = 0)
    xo = torch.rand(g.n, g.n, device="cuda", generator=torch.Generator(device="cuda").manual_seed(9))
    xd = torch.empty_like(xo)
    itn = ctypes.c_int(0)
    tv_iters = 100

    def tv_run(iters):
        ct.check(L.ctprj_tv_denoise(vp(xo), g.n, g.n, 0.05, 0.0, float("inf"), 0, iters, 0.0, vp(xd),
                                    ctypes.byref(itn), hs))
    tv_ms = timed(lambda: tv_run(tv_iters))
    tv_ms20 = timed(lambda: tv_run(20))
    # per iteration: the marginal time of 80 more iterations (the call's setup,
    # a workspace allocation and the start, excluded).  Algorithmic bytes per
    # iteration: the fused iteration reads Xobs, D_old, P1, P2, P1_prev,
    # P2_prev and writes D, P1_new, P2_new (36 B/pixel)
    us_it = 1e3 * (tv_ms - tv_ms20) / (tv_iters - 20)
    out["tv_denoise"] = {"workload": "isotropic TV FGP on %d^2, lambda 0.05, %d iterations" % (g.n, tv_iters),
                         "ms": tv_ms, "ms_20_iterations": tv_ms20, "us_per_iteration": us_it,
                         "algorithmic_GBps": 36.0 * g.n * g.n / (us_it * 1e-6) / 1e9}
    # the wavelet ADMM proximal map (npg/admm.m, Haar, 6 levels) on the headline
    # image size: marginal time of 80 more iterations (relativeTol = 0), by the
    # fused per-tile iteration (one launch: s, nu and a in, s and nu out, 20 B
    # per pixel) and, for comparison, by the level-by-level passes
    # (CTPRJ_WVLT_KERNEL=levels: 13 launches, about 41 B per pixel)
    from imgrecsrc_b200 import wavelet as wvm
    haar = np.ascontiguousarray(wvm.daubcqf(2))
    wa = torch.rand(g.n, g.n, device="cuda", generator=torch.Generator(device="cuda").manual_seed(11)) - 0.3
    wo = torch.empty_like(wa)

    def admm_run(iters):
        ct.check(L.ctprj_wvlt_admm(vp(wa), g.n, g.n, haar.ctypes.data, 2, 6, 0.05, 0.0, iters, None, vp(wo),
                                   ctypes.byref(itn), hs))

    def admm_us():
        t100, t20 = timed(lambda: admm_run(100)), timed(lambda: admm_run(20))
        return t100, 1e3 * (t100 - t20) / 80
    wv_ms, wv_us = admm_us()
    os.environ["CTPRJ_WVLT_KERNEL"] = "levels"
    try:
        wl_ms, wl_us = admm_us()
    finally:
        del os.environ["CTPRJ_WVLT_KERNEL"]
    out["wvlt_admm"] = {"workload": "wavelet ADMM (Haar, 6 levels, u 0.05) on %d^2, 101 iterations" % g.n,
                        "ms": wv_ms, "us_per_iteration": wv_us,
                        "algorithmic_GBps": 20.0 * g.n * g.n / (wv_us * 1e-6) / 1e9,
                        "launches_per_iteration": 1,
                        "level_passes": {"ms": wl_ms, "us_per_iteration": wl_us, "launches_per_iteration": 13,
                                         "algorithmic_GBps": (8 + 4 + 4 + 4 + 16 + 2 * (4.0 / 3.0) * 4)
                                         * g.n * g.n / (wl_us * 1e-6) / 1e9}}
    out["parprj"] = {"workload": "FP64 masked parallel operator (mParPrj): %d^2 image, disc mask of %d "
                                 "pixels, %d angles over [0,180) deg, %d detectors" % (n, mask.size, nang, W),
                     "forward_ms": timed(fwd), "backward_ms": timed(bwd)}
    return out


# Per-launch counters of the projection kernels from the committed ncu summary
# (profiles/projector_counters.json): dram__bytes_read.sum +
# dram__bytes_write.sum and smsp__inst_executed.sum per launch.
def profiled_kernels():
    """Counters per launch of each profiled kernel, or {} when the summary is
    absent."""
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "profiles", "projector_counters.json")
    try:
        with open(path) as f:
            return json.load(f)["kernels"]
    except (OSError, KeyError, ValueError):
        return {}


SMS, SCHEDULERS = 148, 4


def issue_roof(prof, kname, kms, sm_mhz, updates):
    """The roof that binds the projection kernels: warp-instruction issue.  The
    kernel's warp instructions per launch (ncu smsp__inst_executed.sum) over the
    issue slots of its CUDA-event duration at the sampled SM clock
    (148 SMs x 4 schedulers x 1 instruction per cycle)."""
    inst = prof.get("warp_inst_per_launch")
    if not inst or not sm_mhz:
        return None
    slots = kms * 1e-3 * SMS * SCHEDULERS * sm_mhz * 1e6
    return {"kernel": kname, "warp_inst_per_launch": inst, "issue_slots_per_launch": slots,
            "frac": inst / slots, "sm_mhz": sm_mhz,
            "thread_inst_per_update": 32.0 * inst / updates,
            "source": "profiles/projector_counters.json (ncu smsp__inst_executed.sum)"}


def geometries_arm(args):
    """Forward, backprojection and FBP (ramp filter + weighted backprojection)
    times per geometry (CUDA events around each launch on the launching stream,
    the 512 MiB L2 flush before each; median of --steps launches after
    --warmup), one GPU."""
    import torch
    import imgrecsrc_b200 as ct
    torch.cuda.set_device(0)
    stream = torch.cuda.current_stream()
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")
    gen = torch.Generator(device="cuda").manual_seed(0)
    out = {}
    for name, t in GEOMETRIES.items():
        g = ct.Geometry(*t)
        pr = ct.Projector(g)
        x = torch.rand(g.n, g.n, device="cuda", generator=gen)
        y = torch.rand(g.np, g.prjWidth, device="cuda", generator=gen)
        s = torch.empty(g.np, g.prjWidth, device="cuda")
        b = torch.empty(g.n, g.n, device="cuda")
        res = {}
        for kind in ("fwd_ms", "bwd_ms", "fbp_ms"):
            ts = []
            for it in range(max(3, args.warmup) + args.steps):
                flush.zero_()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                if kind == "fwd_ms":
                    pr.forward(x, out=s)
                elif kind == "bwd_ms":
                    pr.backward(y, out=b)
                else:
                    pr.fbp(y, out=b)
                e1.record(stream)
                torch.cuda.synchronize()
                if it >= max(3, args.warmup):
                    ts.append(e0.elapsed_time(e1))
            res[kind] = round(statistics.median(ts), 4)
        out[name] = res
        pr.close()
    print(json.dumps({"geometries": out, "steps": args.steps, "warmup": max(3, args.warmup),
                      "timing": "CUDA events per launch, L2 flushed before each, median"}), flush=True)


def shared_roof(prof, kname, kms, sm_mhz):
    """The shared-memory roof of the staged backprojection: its shared-memory
    wavefronts per launch (ncu l1tex__data_pipe_lsu_wavefronts_mem_shared.sum)
    over the wavefront slots of its CUDA-event duration at the sampled SM clock
    (148 SMs x 1 wavefront per cycle)."""
    wf = prof.get("shared_wavefronts_per_launch")
    if not wf or not sm_mhz:
        return None
    slots = kms * 1e-3 * SMS * sm_mhz * 1e6
    return {"kernel": kname, "wavefronts_per_launch": wf, "wavefront_slots_per_launch": slots,
            "frac": wf / slots, "sm_mhz": sm_mhz,
            "source": "profiles/projector_counters.json (ncu l1tex__data_pipe_lsu_wavefronts_mem_shared.sum)"}


def relaunch(args, argv):
    """--gpus N > 1 without torchrun's environment: start N ranks of this
    script under torch.distributed.run on this node (rendezvous on
    127.0.0.1) and return their exit status."""
    import socket
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        port = so.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1",
           "--nproc-per-node=%d" % args.gpus, "--master-addr=127.0.0.1",
           "--master-port=%d" % port, os.path.abspath(__file__)] + argv
    return subprocess.run(cmd).returncode


def selftest_arm(args):
    """The multi-rank plumbing without a GPU (gloo): each rank times a small
    host computation in place of the projection step, and rank 0 prints the
    bench line with the same world check, MAX-over-ranks time and replica
    aggregation as the GPU arm."""
    import datetime

    import numpy as np
    import torch.distributed as dist

    world, rank, _ = init_dist()
    if world != args.gpus:
        raise SystemExit("bench.py: %d ranks started for --gpus %d" % (world, args.gpus))
    pg = None
    if world > 1:
        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
        pg = dist
    a = np.random.default_rng(rank).random((256, 256), dtype=np.float32)
    for _ in range(max(3, args.warmup)):
        a @ a
    if pg:
        pg.barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        a @ a
    t_ms = (time.perf_counter() - t0) * 1e3 / args.steps
    t_max = max_over_ranks(t_ms, pg, "cpu")
    updates = 2 * 256 ** 3
    line = {"metric": "selftest host matmul (not a projector measurement)",
            "value": replica_value(world, updates, t_max), "unit": "Gflop/s", "n_gpus": world,
            "steps": args.steps, "warmup": max(3, args.warmup), "ms_per_step": t_max,
            "rank_ms": t_ms}
    if pg:
        pg.barrier()
        pg.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the cpu_baseline leg")
    ap.add_argument("--loop-iters", type=int, default=50,
                    help="alternating BHC iterations of the reconstruction leg (0: skip)")
    ap.add_argument("--loop-geometry", default="2048", choices=["2048", "1024"],
                    help="reconstruction leg on the 2048^2 workload (config 5) or on the "
                         "1024^2 configuration of the polychromatic model (smaller, for profiling)")
    ap.add_argument("--legs", default="all", choices=["all", "projector", "bhc", "geometries"],
                    help="projector: the headline step and its end-to-end run only (for profiling); "
                         "bhc: the same plus the BHC gradient-iteration legs; "
                         "geometries: forward, backprojection and FBP times on each configuration's geometry")
    ap.add_argument("--selftest", action="store_true", help=argparse.SUPPRESS)
    args = ap.parse_args()
    if args.gpus < 1:
        ap.error("--gpus must be >= 1")
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        sys.exit(relaunch(args, sys.argv[1:]))
    if args.selftest:
        selftest_arm(args)
    elif args.legs == "geometries":
        geometries_arm(args)
    elif args.impl == "reference":
        reference_arm(args)
    else:
        our_arm(args)


if __name__ == "__main__":
    main()

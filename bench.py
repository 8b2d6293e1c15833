"""Benchmark of the CUDA cloth solver (one JSON line on rank 0).

Headline workload (the default, a step = one simulated frame of the whole batch):
  c4  64 batched grid cloths of side U{64..512} (6,641,977 vertices), k = 1e3 N/m,
      k_b = 1e-2, 0.1 kg area-lumped each, two corners pinned, a random wind force
      per instance per frame, h = 1/60 s. The warm-start network is trained first on
      60 recorded plain frames of the batch (seeds 0..59; 150k Adam steps).
      Two forms, each iterated to the SAME fixed relative residual
      r = ||grad G(x)|| / ||grad G(y)|| <= --tol (1e-4) with an iteration cap
      (--cap 200), converged instances skipped; residual probes on the extrapolated
      schedule (--probe-policy 1: the first two after 10 and 20 iterations
      (--check-every), then after half the iterations the residual's contraction
      predicts are still needed, or at the cap when it stalls):
        learned  predict, the network's guess (potential fallback per instance), VBD;
        plain    predict, VBD (the reference's method, batched).
      Both run from the same frame-start state each frame (held-out wind seeds
      10010+); the plain frame's end state starts the next frame.

  value  frames/s of the learned form, device-timed (CUDA events around each whole
         frame, host probes included), with the plain form's frames/s, the speed-up
         and p50 / p99 beside it; the working set (1.4 GB) is far larger than L2.
  tolerance  whether 1e-4 is reached under the cap (fraction of instance-frames),
         and a sweep over tolerances 0.5 .. 1e-4: iterations to each tolerance from
         FP64 residual traces of both forms, and timed frames to each tolerance.
  e2e    the learned frame through the public C ABI with host arrays: every frame
         uploads (x, v) from pinned host memory and reads them back (wall clock).
  roofline  vbd_sweep_list_kernel, the colour sweep of these frames: algorithmic
         bytes per launch (40 V + 12 E + 56 B per iteration, shared by colour) over
         its per-launch time, measured in this run as 50 listed iterations timed with
         CUDA events (predict, update and two probes included, so a lower bound),
         against the measured HBM copy bandwidth.
  cpu_baseline  the CPU oracle (a C++ restatement of the reference's CPU VBD; the
         reference itself does not build here) iterating the same plain form to the
         same tolerance and cap on a sample (instance 0, 55,696 of 6,641,977
         vertices), with all host cores, scaled to the batch by vertex count.
  gpu_launches  library kernels launched in the timed region (ats_kernel_launches:
         direct launches plus the kernel nodes of graph replays).
  extras (N = 1)  c1 (one 512^2 cloth, plain VBD, 50 iterations, L2-resident) frames/s
         and sweep roofline; the same cloth under XPBD.

--impl reference: the CPU oracle alone on this workload's plain form (the same tol /
cap / probes), each step one frame of the sample, scaled to the batch; the median of
the steps with all host cores, and a 1-core median of 5 frames beside it.

Other workloads (--workload): c1 (512^2 cloth, plain VBD, fixed 50 iterations), c2
(256 batched cloths, plain VBD, fixed 50 iterations), c3 (one 128^2 cloth with wind,
the c4 protocol). Each prints its own metric name.

Multi-GPU: c4's instances are independent, so N ranks split them by balanced
bin-packing (no collective on the data path, "strong" scaling: the batch is fixed);
each rank trains its own network on its own instances; frame times are the max over
ranks. c1 runs N replicas ("weak").
"""
import argparse
import json
import os
import platform
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "frames/s to 1e-4 residual: batched+learned VBD vs plain CUDA VBD, 1 B200"
UNIT = "frames/s"
WORKLOADS = {
    "c4": "c4: 64 batched grid cloths, side U{{64..512}}, wind per instance; batched+learned vs plain batched VBD, "
          "both iterated to a relative residual of {tol:g} (cap {cap} iterations, probes from every {check})",
    "c3": "c3: 128x128 grid cloth, wind per frame; learned vs plain VBD, both iterated to a relative residual of "
          "{tol:g} (cap {cap} iterations, probes from every {check})",
    "c1": "c1: 512x512 grid cloth, plain VBD, 50 iterations x 4 colours per frame",
    "c2": "c2: 256 batched grid cloths, side U{16..256}, plain VBD, 50 iterations per frame",
}
METRICS = {"c1": "frames/s, plain VBD, 50 iterations, 512x512 cloth",
           "c2": "frames/s, plain batched VBD, 50 iterations, 256 cloths",
           "c3": "frames/s to {tol:g} residual: learned VBD vs plain CUDA VBD, 128x128 cloth"}
SWEEP_TOLS = [0.5, 0.3, 0.2, 1e-1, 1e-2, 1e-3, 1e-4]


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--workload", default="c4", choices=["c1", "c2", "c3", "c4"])
    p.add_argument("--tol", type=float, default=1e-4)
    p.add_argument("--cap", type=int, default=200)
    p.add_argument("--check-every", type=int, default=10)
    p.add_argument("--probe-policy", type=int, default=1, choices=[0, 1],
                   help="residual probes: 0 every check-every iterations, 1 extrapolated from the contraction")
    p.add_argument("--train-steps", type=int, default=150000)
    p.add_argument("--instances", type=int, default=0, help="only the first N instances (a small case for profiling)")
    p.add_argument("--record-frames", type=int, default=30, help="recorded frames per trajectory (c4)")
    p.add_argument("--sweep-cap", type=int, default=400, help="iterations of the residual traces")
    p.add_argument("--trace-out", default="", help="write the full residual traces (JSON) here")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-extras", action="store_true")
    p.add_argument("--list-sweep", type=int, default=-1, choices=[-1, 0, 1, 2],
                   help="sweep of the residual-driven frames: -1 the autotuner's choice, 0 plain, 1 pipelined, "
                        "2 streamed")
    p.add_argument("--l2-persisting", type=int, default=-1, choices=[-1, 0, 1],
                   help="list sweeps keep the positions persisting in L2: -1 the autotuner's choice, 0 off, 1 on")
    p.add_argument("--tpv", type=int, default=0)
    p.add_argument("--block", type=int, default=0)
    return p.parse_args()


def dist_env():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("LOCAL_RANK", "0"))


def alg_bytes_per_iter(nv, ne, nb):
    return 40 * nv + 12 * ne + 56 * nb


def cpu_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return platform.processor() or "unknown"


def hbm_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        try:
            return float(json.load(open(path))["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs)"
        except Exception:
            pass
    return 6650.0, "fallback"


class ClockSampler:
    """SM clock and throttle reasons polled through NVML during the timed region."""

    REASONS = {0x4: "sw_power_cap", 0x8: "hw_slowdown", 0x20: "sw_thermal_slowdown", 0x40: "hw_thermal_slowdown",
               0x80: "hw_power_brake_slowdown"}

    def __init__(self, torch_device):
        self.dev = torch_device
        self.samples = []
        self.reasons = set()
        self.stop_flag = False
        self.handle = None
        self.max_mhz = None
        self.t = None

    def start(self):
        try:
            import pynvml
            import torch
            pynvml.nvmlInit()
            pr = torch.cuda.get_device_properties(self.dev)
            bus = "%08X:%02X:%02X.0" % (pr.pci_domain_id, pr.pci_bus_id, pr.pci_device_id)
            self.handle = pynvml.nvmlDeviceGetHandleByPciBusId(bus)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self.handle, pynvml.NVML_CLOCK_SM)
            self.nvml = pynvml
        except Exception as e:  # no NVML: say so in the line
            self.error = str(e)
            return
        self.t = threading.Thread(target=self._poll, daemon=True)
        self.t.start()

    def _poll(self):
        nv = self.nvml
        while not self.stop_flag:
            try:
                self.samples.append(nv.nvmlDeviceGetClockInfo(self.handle, nv.NVML_CLOCK_SM))
                mask = nv.nvmlDeviceGetCurrentClocksEventReasons(self.handle)
                for bit, name in self.REASONS.items():
                    if mask & bit:
                        self.reasons.add(name)
            except Exception:
                pass
            time.sleep(0.005)

    def stop(self):
        self.stop_flag = True
        if self.handle is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "note": getattr(self, "error", "no NVML")}
        if self.t:
            self.t.join(timeout=2)
        return {"sm_mhz": float(np.median(self.samples)) if self.samples else None, "sm_max_mhz": self.max_mhz,
                "reasons": sorted(self.reasons), "samples": len(self.samples)}


# ---------------------------------------------------------------- CPU legs (oracle)
def c4_cpu_sample():
    """Instance 0 of c4 (236 x 236) and the batch's total vertex count."""
    from libatssim_b200 import configs
    insts, prm = configs.c4()
    return insts[0], prm, sum(i.num_verts for i in insts)


def cpu_to_tolerance_frames(threads, frames, tol, cap, check_every, policy, approach=2):
    """Seconds per frame of the oracle's plain VBD frame iterated to `tol` (cap
    iterations, probes every check_every) on the c4 sample, after `approach` plain
    50-iteration frames from rest; winds as instance 0 of the GPU run's frames."""
    from libatssim_b200 import configs
    from oracle import ats_oracle
    ats_oracle.build()
    inst, prm, _ = c4_cpu_sample()
    s = ats_oracle.Scene(inst.positions, inst.faces, inst.mass, inst.fixed, dt=prm["implicit_dt"], substeps=1,
                         iterations=prm["iterations"], k_stretch=inst.k_stretch, k_bend=inst.k_bend,
                         damping=prm["damping"], threads=threads)
    total = float(inst.mass.sum())
    for f in range(approach):
        s.set_gravity(configs.wind_accel(np.random.RandomState(10000 + f), total))
        s.frame()
    times, iters, res = [], [], []
    for f in range(frames):
        s.set_gravity(configs.wind_accel(np.random.RandomState(10010 + f), total))
        t = time.perf_counter()
        it, r = s.frame_to_residual(tol, check_every=check_every, max_iterations=cap, policy=policy)
        times.append(time.perf_counter() - t)
        iters.append(it)
        res.append(r)
    s.close()
    return np.array(times), np.array(iters), np.array(res)


def cpu_plain_fixed_frames(threads, frames, workload):
    """Seconds per frame of the oracle's plain VBD frame (the handle's full iteration
    count) on c1's cloth or on a c2 sample instance; returns (times, vertices of the
    sample, vertices of the workload)."""
    from libatssim_b200 import configs
    from oracle import ats_oracle
    ats_oracle.build()
    insts, prm = configs.c1() if workload == "c1" else configs.c2()
    inst = insts[0]
    s = ats_oracle.Scene(inst.positions, inst.faces, inst.mass, inst.fixed, dt=prm["implicit_dt"], substeps=1,
                         iterations=prm["iterations"], k_stretch=inst.k_stretch, k_bend=inst.k_bend,
                         damping=prm["damping"], threads=threads)
    s.frame()
    times = []
    for _ in range(frames):
        t = time.perf_counter()
        s.frame()
        times.append(time.perf_counter() - t)
    s.close()
    return np.array(times), inst.num_verts, sum(i.num_verts for i in insts)


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    wl = args.workload
    if wl in ("c4", "c3"):
        if wl == "c3":
            print(json.dumps({"impl": "reference", "unavailable": "c3 reference arm not provided; use c4"}))
            return
        t_all, it_all, r_all = cpu_to_tolerance_frames(threads, args.warmup + args.steps, args.tol, args.cap,
                                                       args.check_every, args.probe_policy)
        t_all = t_all[args.warmup:]
        t_one, _, _ = cpu_to_tolerance_frames(1, 5, args.tol, args.cap, args.check_every, args.probe_policy)
        inst, _, total_v = c4_cpu_sample()
        scale = total_v / inst.num_verts
        per_frame = float(np.median(t_all)) * scale
        one = float(np.median(t_one)) * scale
        sample = (f"one frame of c4 instance 0 ({inst.num_verts} of {total_v} vertices) per step, plain VBD to "
                  f"{args.tol:g} (cap {args.cap}, probe policy {args.probe_policy}, check every {args.check_every}), "
                  f"scaled by vertex count; "
                  f"reached tol in {float(np.mean(r_all <= args.tol)):.2f} of frames, mean iterations "
                  f"{float(np.mean(it_all)):.0f}")
        config = {"workload": WORKLOADS["c4"].format(tol=args.tol, cap=args.cap, check=args.check_every),
                  "vertices": total_v, "tol": args.tol, "cap": args.cap, "check_every": args.check_every,
                  "probe_policy": args.probe_policy}
        metric = METRIC
    else:
        t_all, nv_s, nv_t = cpu_plain_fixed_frames(threads, args.warmup + args.steps, wl)
        t_all = t_all[args.warmup:]
        t_one, _, _ = cpu_plain_fixed_frames(1, 5, wl)
        scale = nv_t / nv_s
        per_frame = float(np.median(t_all)) * scale
        one = float(np.median(t_one)) * scale
        sample = (f"full frames of 50 iterations of {'the cloth' if wl == 'c1' else 'c2 instance 0'}"
                  + (f", scaled by vertex count ({nv_s} of {nv_t})" if scale != 1 else ""))
        config = {"workload": WORKLOADS[wl], "vertices": nv_t, "iterations": 50}
        metric = METRICS[wl]
    fps = 1.0 / per_frame
    out = {"impl": "reference", "metric": metric, "value": fps, "unit": UNIT, "n_gpus": args.gpus,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": per_frame * 1e3, "higher_is_better": True,
           "scaling": "strong" if wl == "c4" else "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
           "config": config,
           "cpu_baseline": {"value": fps, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample,
                            "statistic": f"median of {args.steps} steps", "cpu_model": cpu_model(),
                            "nproc": os.cpu_count(),
                            "one_core": {"value": 1.0 / one, "unit": UNIT, "cores": 1, "statistic": "median of 5"}},
           "e2e": {"value": fps, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


# ---------------------------------------------------------------- GPU arm
def init_dist(world, local):
    import torch
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))


def maxrank(v):
    from libatssim_b200 import sharding
    return float(sharding.allreduce_stats([float(v)], op="max")[0])


# DRAM traffic over algorithmic bytes of the list sweeps, per launch, from ncu captures
# of the full c4 batch (1 lane per vertex, 64 threads per block): dram__bytes_read.sum +
# dram__bytes_write.sum, one pass, 3 launches, --cache-control none (warm caches, as in
# the bench; ncu's default flushes them before every launch) --clock-control none.
# Plain sweep: 32-instance case, cold caches, scaled (216.9 of 214.0 MB).
SWEEP_TRAFFIC = {
    "vbd_sweep_stream_kernel<1> (positions persisting in L2)": (0.894, "ncu, full c4 batch, warm caches: "
                                                                        "360.2 MB a launch"),
    "vbd_sweep_stream_kernel<1>": (0.889, "ncu, full c4 batch, warm caches: 357.9 MB a launch"),
    "vbd_sweep_list_kernel<1>": (1.013, "ncu, 32-instance c4 case, cold caches, scaled by algorithmic bytes"),
}


def sweep_roofline(cloth, stream, reps=3, iters=50):
    """Per-launch time of vbd_sweep_list_kernel: `iters` listed iterations over every
    instance (a to-residual frame with tol 0 and one probe at the cap), CUDA-event
    timed; predict, update and the probes are inside, so this bounds the sweep from
    above. Returns (ms per launch, frame ms, algorithmic bytes per launch)."""
    import torch
    info = cloth.info
    x0, v0 = cloth.state(stream=stream)
    ms = []
    for _ in range(reps):
        cloth.set_state(x0, v0, stream=stream)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        cloth.frame_to_residual(0.0, check_every=iters, max_iterations=iters, stream=stream)
        e1.record(stream)
        torch.cuda.synchronize()
        ms.append(e0.elapsed_time(e1))
    cloth.set_state(x0, v0, stream=stream)
    frame_ms = float(np.median(ms))
    per_launch = frame_ms / (iters * info.num_vertex_colors)
    bytes_launch = alg_bytes_per_iter(info.num_verts, info.num_edges, info.num_bending_edges) / info.num_vertex_colors
    return per_launch, frame_ms, bytes_launch


def plain_extras(stream, peak):
    """c1 (one 512^2 cloth, L2-resident): plain VBD CUDA-graph frames and XPBD frames,
    each L2-flushed between frames, device-timed; the sweep per launch from a graph
    frame of 50 iterations."""
    import torch

    import libatssim_b200 as ats
    from libatssim_b200 import configs
    insts, prm = configs.c1()
    cloth = ats.Cloth(insts, **prm)
    cloth.autotune(iterations=20, stream=stream)
    info = cloth.info
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda")

    def timed(solver, frames):
        for _ in range(3):
            cloth.frame(solver, stream=stream, graph=True)
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(frames)]
        torch.cuda.synchronize()
        for i in range(frames):
            flush.fill_(i & 0xFF)
            ev[i][0].record(stream)
            cloth.frame(solver, stream=stream, graph=True)
            ev[i][1].record(stream)
        torch.cuda.synchronize()
        return np.array([a.elapsed_time(b) for a, b in ev])

    chosen = {"vbd": info.vbd_form, "xpbd": info.xpbd_form}
    forms = ["a launch per colour", "persistent"]
    # both forms of each solver, timed; the autotuner's choice is the reported rate
    vbd_ms, xpbd_ms = {}, {}
    for form in (0, 1):
        cloth.set_sweep_form(form, ats.SOLVER_VBD)
        vbd_ms[form] = timed(ats.SOLVER_VBD, 200)
        cloth.set_sweep_form(form, ats.SOLVER_XPBD)
        xpbd_ms[form] = timed(ats.SOLVER_XPBD, 50)
    launches = 50 * info.num_vertex_colors
    v_ms = vbd_ms[chosen["vbd"]]
    per_launch_upper = float(np.median(vbd_ms[0])) / launches  # predict and update inside: an upper bound
    bytes_launch = alg_bytes_per_iter(info.num_verts, info.num_edges, info.num_bending_edges) / info.num_vertex_colors
    x_ms = xpbd_ms[chosen["xpbd"]]
    xpbd_bytes = (28 * info.num_verts + 20 * info.num_edges + 64 * info.num_bending_edges) * 50
    out = {"workload": WORKLOADS["c1"], "frames_per_s": 1e3 / float(np.mean(v_ms)),
           "ms_per_frame_p50": float(np.median(v_ms)), "frames_timed": int(len(v_ms)),
           "vbd_form": forms[chosen["vbd"]],
           "vbd_ms_per_frame_p50_by_form": {forms[f]: float(np.median(vbd_ms[f])) for f in (0, 1)},
           "sweep": {"kernel": f"vbd_sweep_kernel<{info.threads_per_vertex}>",
                     "us_per_launch_upper_bound": per_launch_upper * 1e3,
                     "achieved_gbs_lower_bound": bytes_launch / (per_launch_upper * 1e-3) / 1e9,
                     "frac_of_measured_hbm": bytes_launch / (per_launch_upper * 1e-3) / 1e9 / peak,
                     "note": "a launch per colour; the 64 MB working set is L2-resident inside a frame: an L2 "
                             "figure, not HBM"},
           "xpbd": {"frames_per_s": 1e3 / float(np.mean(x_ms)), "ms_per_frame_p50": float(np.median(x_ms)),
                    "form": forms[chosen["xpbd"]],
                    "ms_per_frame_p50_by_form": {forms[f]: float(np.median(xpbd_ms[f])) for f in (0, 1)},
                    "achieved_gbs": xpbd_bytes / (float(np.median(x_ms)) * 1e-3) / 1e9,
                    "frac_of_measured_hbm": xpbd_bytes / (float(np.median(x_ms)) * 1e-3) / 1e9 / peak}}
    cloth.close()
    del flush
    return out


def run_learned(args):
    """c4 (or c3): learned and plain forms to the same fixed tolerance."""
    import torch
    rank, world, local = dist_env()
    init_dist(world, local)
    import libatssim_b200 as ats
    from libatssim_b200 import build, configs, learned, sharding
    build.build()
    wl = args.workload
    if wl == "c4":
        all_insts, prm = configs.c4()
        traj, frames = 2, args.record_frames
    else:
        all_insts, prm = configs.c3()
        traj, frames = 20, 100
    if args.instances:
        all_insts = all_insts[:args.instances]
    insts = all_insts
    if world > 1:
        insts, _ = sharding.shard(all_insts, args.cap)
    rec_iters = prm["iterations"]
    stream = torch.cuda.current_stream()
    t0 = time.perf_counter()
    cloth = ats.Cloth(insts, threads_per_vertex=args.tpv, block_size=args.block, **prm)
    t_create = time.perf_counter() - t0
    # the autotuned shape unless one is given (--tpv / --block, for shape sweeps)
    tuned = cloth.autotune(iterations=20, stream=stream) if not (args.tpv or args.block) else (args.tpv, args.block)
    cloth.set_probe_policy(args.probe_policy)
    if args.list_sweep >= 0:
        cloth.set_list_sweep(args.list_sweep)
    if args.l2_persisting >= 0:
        cloth.set_l2_persisting(args.l2_persisting)
    info = cloth.info
    nv = info.num_verts
    # training data: plain frames of this rank's instances
    ds = ats.Dataset(traj * frames * nv)
    t0 = time.perf_counter()
    learned.record(cloth, insts, ds, traj, frames, rec_iters, seed0=0)
    torch.cuda.synchronize()
    t_record = time.perf_counter() - t0
    model, loss, t_train = learned.train(ds, steps=args.train_steps)
    ds.close()

    # the measured frames: a moving cloth, held-out winds
    learned.approach(cloth, insts, 10, seed0=10000, stream=stream)
    clocks = ClockSampler(local)
    launches = {}

    def on_timed(start):
        # the timed frames are bracketed by a barrier and a device synchronisation
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()
        if start:
            clocks.start()
            launches["a"] = ats.kernel_launches()
        else:
            launches["b"] = ats.kernel_launches()

    res = learned.fixed_tolerance_frames(cloth, insts, model, args.tol, args.cap, args.check_every, args.steps,
                                         args.warmup, seed0=10010, stream=stream, on_timed=on_timed)
    clk = clocks.stop()
    lm, pm = res["learned_ms"], res["plain_ms"]
    learned_ms = maxrank(np.mean(lm))
    plain_ms = maxrank(np.mean(pm))
    reached_l = float(np.mean(res["learned_res"] <= args.tol))
    reached_p = float(np.mean(res["plain_res"] <= args.tol))
    vw = np.array([i.num_verts for i in insts], dtype=np.float64)
    its_l = float(np.sum(res["learned_iters"] * vw) / (vw.sum() * len(lm)))
    its_p = float(np.sum(res["plain_iters"] * vw) / (vw.sum() * len(pm)))

    # sweep roofline in this run (listed sweep over all instances)
    per_launch, rf_frame_ms, bytes_launch = sweep_roofline(cloth, stream)
    sweep_kernel = (("vbd_sweep_list_kernel", "vbd_sweep_pipe_kernel", "vbd_sweep_stream_kernel")[info.list_form]
                    + f"<{info.threads_per_vertex}>"
                    + (" (positions persisting in L2)" if info.l2_persisting else ""))
    peak, peak_src = hbm_peak()
    achieved = bytes_launch / (per_launch * 1e-3) / 1e9
    sweeps_per_learned_frame = float(np.mean(res["learned_iters"].max(axis=1))) * info.num_vertex_colors

    # end to end through the C ABI with host arrays
    x_h = torch.empty((nv, 3), dtype=torch.float32, pin_memory=True).numpy()
    v_h = torch.empty((nv, 3), dtype=torch.float32, pin_memory=True).numpy()
    cloth.state_into(x_h, v_h, stream=stream)
    masses = [float(i.mass.sum()) for i in insts]
    e2e_frames = 5
    for f in range(e2e_frames + 1):
        if f == 1:
            if world > 1:
                torch.distributed.barrier()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
        cloth.set_accel(learned.wind_table(np.random.RandomState(20000 + f), masses), stream=stream)
        cloth.set_state(x_h, v_h, stream=stream)
        cloth.frame_warm_to_residual(model, args.tol, check_every=args.check_every, max_iterations=args.cap,
                                     stream=stream)
        cloth.state_into(x_h, v_h, stream=stream)
    torch.cuda.synchronize()
    e2e_s = maxrank((time.perf_counter() - t0) / e2e_frames)
    state_bytes = 2 * 3 * 4 * nv

    sweep, trace, timed_tols = None, None, None
    if world == 1 and args.sweep_cap > 0:
        points = sorted(set([0, 1, 2, 3, 5, 7, 10, 15, 20, 30, 40, 50, 70, 100, 150, 200, 300, 400, 600, 800, 1000,
                             1500, 2000, 3000, 4000, 5000]) | {args.sweep_cap})
        points = [p for p in points if p <= args.sweep_cap]
        sweep, trace = learned.tolerance_sweep(cloth, insts, model, SWEEP_TOLS, points, 2, seed0=30000,
                                               stream=stream)
        timed_tols = [learned.timed_to_tolerance(cloth, insts, model, t, args.cap, args.check_every, 2,
                                                 seed0=40000 + 10 * k, stream=stream)
                      for k, t in enumerate(SWEEP_TOLS[:-1])]
        if args.trace_out:
            os.makedirs(os.path.dirname(os.path.abspath(args.trace_out)), exist_ok=True)
            json.dump({"workload": wl, "sweep": sweep, "trace": trace, "timed": timed_tols},
                      open(args.trace_out, "w"), indent=1)

    extras = None
    if world == 1 and not args.no_extras:
        extras = plain_extras(stream, peak)

    out = None
    if rank == 0:
        value = 1e3 / learned_ms
        plain_fps = 1e3 / plain_ms
        tol_s = f"{args.tol:g}"
        out = {"metric": METRIC if wl == "c4" else METRICS["c3"].format(tol=args.tol), "value": value, "unit": UNIT,
               "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": learned_ms,
               "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
               "dtype": "f32 (MLP bf16 / fp32 accumulate; residuals fp64)", "data": "synthetic",
               "config": {"workload": WORKLOADS[wl].format(tol=args.tol, cap=args.cap, check=args.check_every),
                          "instances": len(all_insts), "vertices": sum(i.num_verts for i in all_insts),
                          "recorded_frames": traj * frames,
                          "tol": args.tol, "cap": args.cap, "check_every": args.check_every,
                          "probe_policy": ["fixed", "extrapolated"][args.probe_policy],
                          "parallelism": f"instance-shards{world}", "create_s": t_create,
                          "threads_per_vertex": info.threads_per_vertex, "block_size": info.block_size,
                          "autotuned": list(tuned),
                          "l2": "inputs larger than L2 (1.4 GB working set per frame); no flush"},
               "headline": {"form": "learned (batched + learned warm start)", "learned_fps": value,
                            "plain_fps": plain_fps, "speedup_vs_plain": plain_ms / learned_ms,
                            "target_speedup": 2.0, "pass_2x": bool(plain_ms / learned_ms >= 2.0 and
                                                                   reached_l >= 1.0),
                            "learned_ms_p50": float(np.percentile(lm, 50)),
                            "learned_ms_p99": float(np.percentile(lm, 99)),
                            "plain_ms_p50": float(np.percentile(pm, 50)),
                            "plain_ms_p99": float(np.percentile(pm, 99)),
                            "reached_tol_fraction": {"learned": reached_l, "plain": reached_p},
                            "iterations_vertex_weighted": {"learned": its_l, "plain": its_p},
                            "residual_at_stop_median": {"learned": float(np.median(res["learned_res"])),
                                                        "plain": float(np.median(res["plain_res"]))},
                            "guess_kept_fraction": float(res["used"].mean()),
                            "verdict": (f"{tol_s} reached by {reached_l:.0%} (learned) / {reached_p:.0%} (plain) "
                                        f"of instance-frames within {args.cap} iterations; speed-up "
                                        f"{plain_ms / learned_ms:.2f}x against the 2x target")},
               "tolerance_sweep": sweep, "timed_to_tolerance": timed_tols,
               "e2e": {"value": 1.0 / e2e_s, "unit": UNIT, "h2d_bytes_per_step": state_bytes,
                       "d2h_bytes_per_step": state_bytes,
                       "path": "ats_set_state from pinned host, ats_frame_warm_to_residual, ats_get_state to pinned "
                               "host; wall clock"},
               "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                            "frac": achieved / peak,
                            "traffic": (SWEEP_TRAFFIC[sweep_kernel][0] * bytes_launch
                                        if sweep_kernel in SWEEP_TRAFFIC else None),
                            "traffic_source": ("not captured in this run (DRAM bytes read + written per launch, as "
                                               "a ratio to the algorithmic bytes): " + SWEEP_TRAFFIC[sweep_kernel][1]
                                               if sweep_kernel in SWEEP_TRAFFIC else "no capture of this kernel"),
                            "kernel": sweep_kernel,
                            "us_per_launch_upper_bound": per_launch * 1e3, "alg_bytes_per_launch": bytes_launch,
                            "layout_bytes_per_launch": info.sweep_layout_bytes / info.num_vertex_colors,
                            "layout_note": "bytes the streamed sweep must move in this layout (merged per-vertex "
                                           "stencil, no per-vertex material record); achieved and frac use the "
                                           "algorithmic bytes",
                            "timing": "50 listed iterations over all instances, CUDA events, predict/update/2 probes "
                                      "included", "peak_source": peak_src,
                            "sweeps_per_learned_frame": sweeps_per_learned_frame,
                            "sweep_share_of_learned_frame_upper": sweeps_per_learned_frame * per_launch / learned_ms},
               "gpu_launches": int(launches.get("b", 0) - launches.get("a", 0)),
               "clocks": clk,
               "train": {"samples": traj * frames * nv, "record_s": t_record, "train_s": t_train,
                         "steps": args.train_steps, "final_loss_normalised": loss}}
        if extras is not None:
            out["extras"] = extras
    if rank == 0 and world == 1 and not args.no_cpu_baseline and wl == "c4":
        threads = os.cpu_count() or 1
        t_cpu, it_cpu, r_cpu = cpu_to_tolerance_frames(threads, 3, args.tol, args.cap, args.check_every,
                                                       args.probe_policy)
        inst0, _, total_v = c4_cpu_sample()
        per_frame = float(np.median(t_cpu)) * total_v / inst0.num_verts
        out["cpu_baseline"] = {"value": 1.0 / per_frame, "unit": UNIT, "cores": threads, "kind": "port",
                               "sample": f"c4 instance 0 ({inst0.num_verts} of {total_v} vertices), 3 frames of plain "
                                         f"VBD to {args.tol:g} (cap {args.cap}; mean iterations "
                                         f"{float(np.mean(it_cpu)):.0f}), median, scaled by vertex count",
                               "cpu_model": cpu_model(), "nproc": os.cpu_count()}
    if out is not None:
        print(json.dumps(out), flush=True)
    model.close()
    cloth.close()
    if world > 1:
        torch.distributed.destroy_process_group()


def run_plain(args):
    """c1 / c2: plain VBD, fixed 50 iterations, CUDA-graph frames."""
    import torch
    rank, world, local = dist_env()
    init_dist(world, local)
    import libatssim_b200 as ats
    from libatssim_b200 import build, configs, sharding
    build.build()
    insts, prm = configs.c1() if args.workload == "c1" else configs.c2()
    sharded = args.workload == "c2" and world > 1
    if sharded:
        insts, _ = sharding.shard(insts, prm["iterations"])
    cloth = ats.Cloth(insts, threads_per_vertex=args.tpv, block_size=args.block, **prm)
    stream = torch.cuda.current_stream()
    if not args.tpv and not args.block:
        cloth.autotune(iterations=20, stream=stream)
    info = cloth.info
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda")
    for _ in range(args.warmup):
        cloth.frame(stream=stream, graph=True)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    clocks = ClockSampler(local)
    clocks.start()
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    l0 = ats.kernel_launches()
    for i in range(args.steps):
        flush.fill_(i & 0xFF)
        ev[i][0].record(stream)
        cloth.frame(stream=stream, graph=True)
        ev[i][1].record(stream)
    torch.cuda.synchronize()
    l1 = ats.kernel_launches()
    clk = clocks.stop()
    ms = np.array([a.elapsed_time(b) for a, b in ev])
    ms_step = maxrank(np.mean(ms))
    value = (1 if sharded else world) * 1e3 / ms_step
    peak, peak_src = hbm_peak()
    bytes_launch = alg_bytes_per_iter(info.num_verts, info.num_edges, info.num_bending_edges) / info.num_vertex_colors
    per_launch = ms_step / (prm["iterations"] * info.num_vertex_colors)
    achieved = bytes_launch / (per_launch * 1e-3) / 1e9
    x_h = torch.empty((info.num_verts, 3), dtype=torch.float32, pin_memory=True).numpy()
    v_h = torch.empty((info.num_verts, 3), dtype=torch.float32, pin_memory=True).numpy()
    cloth.state_into(x_h, v_h, stream=stream)
    n_e2e = 20
    for f in range(n_e2e + 1):
        if f == 1:
            if world > 1:
                torch.distributed.barrier()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
        cloth.set_state(x_h, v_h, stream=stream)
        cloth.frame(stream=stream, graph=True)
        cloth.state_into(x_h, v_h, stream=stream)
    e2e_s = maxrank((time.perf_counter() - t0) / n_e2e)
    state_bytes = 2 * 3 * 4 * info.num_verts
    out = None
    if rank == 0:
        out = {"metric": METRICS[args.workload], "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
               "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True,
               "scaling": "strong" if sharded else "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
               "config": {"workload": WORKLOADS[args.workload], "instances": info.num_instances,
                          "vertices": info.num_verts, "iterations": prm["iterations"],
                          "threads_per_vertex": info.threads_per_vertex, "block_size": info.block_size,
                          "parallelism": f"instance-shards{world}" if sharded else f"replicas{world}",
                          "l2": "flushed between frames (256 MiB write, outside the event pairs)"},
               "e2e": {"value": (1 if sharded else world) / e2e_s, "unit": UNIT, "h2d_bytes_per_step": state_bytes,
                       "d2h_bytes_per_step": state_bytes},
               "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                            "frac": achieved / peak, "traffic": None,
                            "kernel": f"vbd_sweep_kernel<{info.threads_per_vertex}>",
                            "us_per_launch_upper_bound": per_launch * 1e3, "alg_bytes_per_launch": bytes_launch,
                            "timing": "whole graph frame over its sweep launches (predict and update included)",
                            "peak_source": peak_src},
               "gpu_launches": int(l1 - l0), "clocks": clk}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        t_cpu, nv_s, nv_t = cpu_plain_fixed_frames(threads, 3, args.workload)
        per_frame = float(np.median(t_cpu)) * nv_t / nv_s
        out["cpu_baseline"] = {"value": 1.0 / per_frame, "unit": UNIT, "cores": threads, "kind": "port",
                               "sample": "3 full frames (50 iterations), median"
                                         + (f", instance 0 scaled by vertex count" if nv_t != nv_s else ""),
                               "cpu_model": cpu_model(), "nproc": os.cpu_count()}
    if out is not None:
        print(json.dumps(out), flush=True)
    cloth.close()
    if world > 1:
        torch.distributed.destroy_process_group()


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    elif args.workload in ("c3", "c4"):
        run_learned(args)
    else:
        run_plain(args)


if __name__ == "__main__":
    main()

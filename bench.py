"""Benchmark of the CUDA cloth solver (one JSON line on rank 0).

Workload (a step = one simulated frame): a 512 x 512-vertex grid cloth
(262,144 vertices, 784,385 edges, 782,341 bending edges), k = 1e3 N/m,
k_b = 1e-2, 0.1 kg area-lumped, two top corners pinned, h = 1/60 s,
plain Vertex Block Descent with 50 iterations x 4 colours per frame, FP32.

  value  frames/s with the state resident in HBM, device-timed (CUDA events on
         the launching stream, one event pair per frame, L2 flushed between frames
         outside the event pairs), summed over ranks.
  e2e    frames/s through the public C ABI with host arrays: every frame uploads
         the state (x, v) from pinned host memory, runs the frame and reads (x, v)
         back into it (wall clock around the calls, which synchronise).
  roofline  the colour-sweep kernel: algorithmic bytes per launch
         (40 V + 12 E + 56 B per iteration, shared by colour) over its mean
         CUDA-event duration, against the measured HBM copy bandwidth.
  cpu_baseline  the CPU oracle (a C++ restatement of the reference's CPU VBD,
         the reference itself does not build here) on a bounded sample of the
         same workload, rank 0 only.
  xpbd   the same cloth solved by XPBD instead (CUDA-graph frames of 50 x
         (stretch + bending colours) projections): frames/s and bandwidth.

--impl reference times that CPU implementation alone on this workload with all
host threads (each step = 10 of the frame's 50 iterations, scaled to frames/s).

Other workloads (--workload):
  c2  256 batched cloths of side U{16..256} with random materials and pins, plain
      VBD, one launch per colour over all instances; the same keys as c1.
  c3  a 128 x 128 cloth with a random wind per frame, 200 iterations; c4 64 batched
      cloths of side U{64..512} with wind, 50 iterations. Both record plain frames,
      train the warm-start network on the GPU and compare, on held-out frames,
      plain VBD with learned-guess frames that stop at each instance's plain
      residual (libatssim_b200/learned.py describes the protocol).

Multi-GPU: the single cloth does not partition (a graph split would need a halo
exchange per colour), so N > 1 runs N independent replicas ("weak" scaling); c2
shards its instances over the ranks ("strong" scaling). Timing is the max over
ranks.
"""
import argparse
import json
import os
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "frames/s to 1e-4 residual: batched+learned VBD vs plain CUDA VBD, 1 B200"
UNIT = "frames/s"
WORKLOAD = "c1: 512x512 grid cloth, plain VBD, 50 iterations x 4 colours per frame"
WORKLOAD_C2 = "c2: 256 batched grid cloths, side U{16..256}, plain VBD, 50 iterations per frame"
ITERS = 50
REF_SAMPLE_ITERS = 10


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--tpv", type=int, default=0)
    p.add_argument("--block", type=int, default=0)
    p.add_argument("--workload", default="c1", choices=["c1", "c2", "c3", "c4"],
                   help="c1: 512x512 cloth (the headline); c2: 256 batched instances; c3: learned warm start on a "
                        "128x128 cloth; c4: 64 batched instances with the learned warm start")
    return p.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def alg_bytes_per_iter(nv, ne, nb):
    return 40 * nv + 12 * ne + 56 * nb


class ClockSampler:
    """SM clock and throttle reasons polled through NVML during the timed region
    (nvidia-smi's 200 ms period is longer than the region itself)."""

    REASONS = {0x4: "sw_power_cap", 0x8: "hw_slowdown", 0x20: "sw_thermal_slowdown", 0x40: "hw_thermal_slowdown",
               0x80: "hw_power_brake_slowdown"}

    def __init__(self, torch_device):
        self.dev = torch_device
        self.samples = []
        self.reasons = set()
        self.stop_flag = False
        self.handle = None
        self.max_mhz = None

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
        except Exception as e:  # no NVML: report it
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
            time.sleep(0.002)

    def stop(self):
        self.stop_flag = True
        if self.handle is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "note": getattr(self, "error", "no NVML")}
        self.t.join(timeout=2)
        return {"sm_mhz": float(np.median(self.samples)) if self.samples else None, "sm_max_mhz": self.max_mhz,
                "reasons": sorted(self.reasons), "samples": len(self.samples)}


def cpu_port_sample(threads, iters):
    """Times the CPU oracle on one frame of `iters` iterations of the workload."""
    from libatssim_b200 import configs
    from oracle import ats_oracle
    ats_oracle.build()
    insts, prm = configs.c1()
    inst = insts[0]
    s = ats_oracle.Scene(inst.positions, inst.faces, inst.mass, inst.fixed, dt=prm["implicit_dt"],
                         substeps=1, iterations=iters, k_stretch=inst.k_stretch, k_bend=inst.k_bend,
                         damping=prm["damping"], threads=threads)
    return s


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    s = cpu_port_sample(threads, REF_SAMPLE_ITERS)
    for _ in range(args.warmup):
        s.frame()
    t = time.perf_counter()
    for _ in range(args.steps):
        s.frame()
    dt = time.perf_counter() - t
    per_frame = dt / args.steps * (ITERS / REF_SAMPLE_ITERS)
    fps = 1.0 / per_frame
    out = {"impl": "reference", "metric": METRIC, "value": fps, "unit": UNIT, "n_gpus": args.gpus,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": per_frame * 1e3, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
           "config": {"workload": WORKLOAD, "vertices": 262144, "iterations": ITERS, "frames": args.steps},
           "cpu_baseline": {"value": fps, "unit": UNIT, "cores": threads, "kind": "port",
                            "sample": f"{REF_SAMPLE_ITERS} of {ITERS} iterations per frame, scaled; "
                                      "C++ restatement of examples/example2_async_iter.cpp VBD"},
           "e2e": {"value": fps, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


def profile_traffic(alg_bytes, workload):
    """DRAM bytes per sweep launch from the committed ncu summary of this workload's
    sweep, else the c1 one (cold and warm-in-frame) scaled to a launch of `alg_bytes`
    algorithmic bytes (traffic grows with the vertices swept)."""
    own = os.path.join(ROOT, "profiles", f"vbd_sweep_{workload}_ncu.json")
    if workload != "c1" and os.path.exists(own):
        try:
            d = json.load(open(own))
            return d["dram_bytes_per_launch"], None, "ncu capture of this workload's sweep (cold caches)"
        except Exception:
            pass
    p = os.path.join(ROOT, "profiles", "vbd_sweep_c1_ncu.json")
    if not os.path.exists(p):
        return None, None, None
    try:
        d = json.load(open(p))
        scale = alg_bytes / d["alg_bytes_per_launch"]
        src = "ncu capture of this launch" if abs(scale - 1.0) < 1e-9 else \
            "ncu capture of the c1 sweep (512^2), scaled by algorithmic bytes"
        return d["dram_bytes_per_launch"] * scale, d["dram_bytes_per_launch_warm"] * scale, src
    except Exception:
        return None, None, None


def run_ours(args):
    import torch
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    import libatssim_b200 as ats
    from libatssim_b200 import build, configs
    build.build()
    from libatssim_b200 import sharding
    insts, prm = configs.c1() if args.workload == "c1" else configs.c2()
    sharded = args.workload == "c2" and world > 1
    if sharded:
        insts, _ = sharding.shard(insts, prm["iterations"])  # this rank's instances, no data-path collective
    t_create = time.perf_counter()
    cloth = ats.Cloth(insts, threads_per_vertex=args.tpv, block_size=args.block, **prm)
    t_create = time.perf_counter() - t_create
    stream = torch.cuda.current_stream()
    tuned = None
    if not args.tpv and not args.block:
        tuned = cloth.autotune(iterations=20, stream=stream)
    info = cloth.info
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda")

    def barrier():
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()

    # warm-up (also captures the frame graph)
    for _ in range(args.warmup):
        cloth.frame(stream=stream, graph=True)
    torch.cuda.synchronize()

    # --- device-timed frames, L2 flushed between frames outside the event pairs
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    clocks = ClockSampler(local)
    clocks.start()
    barrier()
    for i in range(args.steps):
        flush.fill_(i & 0xFF)
        starts[i].record(stream)
        cloth.frame(stream=stream, graph=True)
        ends[i].record(stream)
    barrier()
    clk = clocks.stop()
    ms = sum(s.elapsed_time(e) for s, e in zip(starts, ends))
    ms = float(sharding.allreduce_stats([ms], op="max")[0])  # max over ranks
    ms_per_step = ms / args.steps
    # replicas: every rank advances a whole cloth per step; sharded c2: all ranks
    # together advance the 256 instances once per step
    value = (1 if sharded else world) * 1e3 / ms_per_step

    # --- residual reached after the frame's iterations (reported, not timed)
    x_end, v_end = cloth.state()
    cloth.predict(stream=stream)
    r0 = cloth.residual(stream=stream)[0]
    for _ in range(ITERS):
        for c in range(info.num_vertex_colors):
            cloth.vbd_color_sweep(c, stream=stream)
    r1 = cloth.residual(stream=stream)[0]
    cloth.set_state(x_end, v_end, stream=stream)

    # --- per-launch sweep duration: CUDA events around ITERS back-to-back iterations
    # (ITERS x colours sweep launches, chained by programmatic dependent launch as in
    # the frame), L2 flushed before each repetition as between timed frames
    reps = []
    for rep in range(3):
        flush.fill_(rep)
        cloth.predict(stream=stream)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        cloth.vbd_iterations(ITERS, stream=stream)
        e1.record(stream)
        cloth.update_velocity(stream=stream)
        reps.append((e0, e1))
    torch.cuda.synchronize()
    mean_sweep_ms = float(np.mean([a.elapsed_time(b) for a, b in reps])) / (ITERS * info.num_vertex_colors)
    bytes_iter = alg_bytes_per_iter(info.num_verts, info.num_edges, info.num_bending_edges)
    bytes_launch = bytes_iter / info.num_vertex_colors
    achieved = bytes_launch / (mean_sweep_ms * 1e-3) / 1e9
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(peaks_path):
        peak = float(json.load(open(peaks_path))["hbm_gbs"])
        peak_src = "measured"
    else:
        peak, peak_src = 6650.0, "fallback"

    # --- XPBD at the same scale (the reference's other solver): CUDA-graph frames of
    # predict, lambda reset, ITERS x (stretch colours + bending colours) projections and
    # update, L2 flushed between frames; algorithmic bytes 28 V + 20 E + 64 B per iteration
    x_keep, v_keep = cloth.state()
    for _ in range(2):
        cloth.frame(ats.SOLVER_XPBD, stream=stream, graph=True)
    xpbd_ms = []
    for i in range(max(3, min(args.steps, 10))):
        flush.fill_(i & 0xFF)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        cloth.frame(ats.SOLVER_XPBD, stream=stream, graph=True)
        e1.record(stream)
        torch.cuda.synchronize()
        xpbd_ms.append(e0.elapsed_time(e1))
    xpbd_frame_ms = float(sharding.allreduce_stats([float(np.median(xpbd_ms))], op="max")[0])
    xpbd_bytes = (28 * info.num_verts + 20 * info.num_edges + 64 * info.num_bending_edges) * ITERS
    cloth.set_state(x_keep, v_keep, stream=stream)
    xpbd = {"frames_per_s": (1 if sharded else world) * 1e3 / xpbd_frame_ms, "ms_per_frame": xpbd_frame_ms,
            "launches_per_frame": 3 + ITERS * (info.num_stretch_colors + info.num_bending_colors),
            "achieved_gbs": xpbd_bytes / (xpbd_frame_ms * 1e-3) / 1e9,
            "note": "whole-frame algorithmic bytes (28V+20E+64B per iteration) over the device-timed frame"}

    # --- end to end through the public API with host arrays: every frame uploads the
    # state (x, v) from pinned host memory, runs the frame and reads (x, v) back into it
    x_h = torch.empty((info.num_verts, 3), dtype=torch.float32, pin_memory=True).numpy()
    v_h = torch.empty((info.num_verts, 3), dtype=torch.float32, pin_memory=True).numpy()
    cloth.state_into(x_h, v_h, stream=stream)
    e2e_steps = max(3, min(args.steps, 10))
    for _ in range(2):  # warm-up of the host path
        cloth.set_state(x_h, v_h, stream=stream)
        cloth.frame(stream=stream, graph=True)
        cloth.state_into(x_h, v_h, stream=stream)
    barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        cloth.set_state(x_h, v_h, stream=stream)
        cloth.frame(stream=stream, graph=True)
        cloth.state_into(x_h, v_h, stream=stream)
    barrier()
    e2e_s = (time.perf_counter() - t0) / e2e_steps
    e2e_s = float(sharding.allreduce_stats([e2e_s], op="max")[0])
    state_bytes = 2 * 3 * 4 * info.num_verts

    traffic = profile_traffic(bytes_launch, args.workload)
    out = None
    if rank == 0:
        out = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
               "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
               "scaling": "strong" if sharded else "weak",
               "vs_baseline": None, "dtype": "f32", "data": "synthetic",
               "config": {"workload": WORKLOAD if args.workload == "c1" else WORKLOAD_C2,
                          "instances": info.num_instances, "create_s": t_create, "vertices": info.num_verts, "edges": info.num_edges,
                          "bending_edges": info.num_bending_edges, "colors": info.num_vertex_colors,
                          "iterations": ITERS, "threads_per_vertex": info.threads_per_vertex,
                          "block_size": info.block_size, "autotuned": tuned is not None,
                          "parallelism": f"instance-shards{world}" if sharded else f"replicas{world}",
                          "l2": "flushed between frames (256 MiB write, outside the event pairs)"},
               "residual": {"relative_after_frame": float(r1 / r0), "definition":
                            "||grad G(x)|| / ||grad G(y)||, FP64, free vertices"},
               "e2e": {"value": (1 if sharded else world) / e2e_s, "unit": UNIT, "h2d_bytes_per_step": state_bytes,
                       "d2h_bytes_per_step": state_bytes},
               "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                            "frac": achieved / peak, "traffic": traffic[0], "traffic_warm_in_frame": traffic[1],
                            "traffic_source": traffic[2],
                            "kernel": f"vbd_sweep_kernel<{info.threads_per_vertex}>", "mean_launch_us": mean_sweep_ms * 1e3,
                            "alg_bytes_per_launch": bytes_launch, "peak_source": peak_src},
               "gpu_launches": args.steps * (2 + ITERS * info.num_vertex_colors),
               "clocks": clk,
               "xpbd": dict(xpbd, frac_of_peak=xpbd["achieved_gbs"] / peak)}
    if rank == 0 and world == 1 and not args.no_cpu_baseline and args.workload == "c1":
        threads = os.cpu_count() or 1
        s = cpu_port_sample(threads, REF_SAMPLE_ITERS)
        s.frame()
        t = time.perf_counter()
        n = 2
        for _ in range(n):
            s.frame()
        per_frame = (time.perf_counter() - t) / n * (ITERS / REF_SAMPLE_ITERS)
        out["cpu_baseline"] = {"value": 1.0 / per_frame, "unit": UNIT, "cores": threads, "kind": "port",
                               "sample": f"{n} frames of {REF_SAMPLE_ITERS}/{ITERS} iterations, scaled"}
    if out is not None:
        print(json.dumps(out), flush=True)
    cloth.close()
    if world > 1:
        torch.distributed.destroy_process_group()


def run_learned(args):
    """c3 / c4: plain VBD against the learned warm start, frames/s to the plain
    solver's own residual (libatssim_b200/learned.py describes the protocol)."""
    import torch
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    import libatssim_b200 as ats
    from libatssim_b200 import build, configs, learned
    build.build()
    if args.workload == "c3":
        insts, prm = configs.c3()
        trajectories, frames, eval_traj, eval_frames, skip = 20, 100, 2, 40, 15
        desc = "c3: 128x128 cloth, wind per frame, 200 iterations; MLP trained on 2000 plain frames (seeds 0-1999)"
    else:
        insts, prm = configs.c4()
        trajectories, frames, eval_traj, eval_frames, skip = 2, 30, 1, 30, 10
        desc = ("c4: 64 batched cloths, side U{64..512}, wind per instance, 50 iterations; shared MLP trained on "
                "60 plain frames of the batch")
    iters = prm["iterations"]
    cloth = ats.Cloth(insts, **prm)
    cloth.autotune(iterations=20)
    nv = cloth.info.num_verts
    ds = ats.Dataset(trajectories * frames * nv)
    t = time.perf_counter()
    learned.record(cloth, insts, ds, trajectories, frames, iters, seed0=0)
    torch.cuda.synchronize()
    t_record = time.perf_counter() - t
    model, loss, t_train = learned.train(ds)
    ds.close()
    # probes every 5 iterations, the first one at the previous frame's count minus 3
    # (c3) or at the 75th percentile of the previous frame's counts (c4)
    check_every, schedule = (5, "prev") if args.workload == "c3" else (5, 75)
    clocks = ClockSampler(local)
    clocks.start()
    res = learned.evaluate(cloth, insts, model, iters, seed0=10000, trajectories=eval_traj, frames=eval_frames,
                           skip=skip, check_every=check_every, schedule=schedule, lead=3)
    per_instance = learned.plain_per_instance_ms(insts, prm) if args.workload == "c4" else None
    sm = learned.summary(res, iters, per_instance)
    clk = clocks.stop()
    sm["check_every"] = check_every
    sm["probe_schedule"] = ("first at the previous frame's count - 3, then every 5" if schedule == "prev" else
                            "first at the 75th percentile of the previous frame's counts, then every 5")
    # fixed budget: the most iterations any to-residual frame needed,
    # measured on fresh frames (seed0 20000) as a CUDA graph
    budget = int(min(iters, 5 * np.ceil(np.max(res["learned_iters"]) / 5.0)))
    fx = learned.evaluate_fixed(cloth, insts, model, budget, iters, seed0=20000, trajectories=eval_traj,
                                frames=eval_frames, skip=skip)
    fx["speedup_vs_plain"] = fx["learned_fixed_fps"] / sm["plain_fps"]
    if per_instance is not None:
        fx["speedup_vs_unbatched"] = fx["learned_fixed_fps"] * per_instance / 1e3
    sm["fixed_budget"] = fx
    # the fixed-budget graph counts only when every instance of every evaluated frame
    # reached the plain residual; the residual-driven frames always do
    best = sm["learned_fps"]
    if fx["reached_plain_residual_fraction"] >= 1.0:
        best = max(best, fx["learned_fixed_fps"])
    sm["headline_arm"] = "fixed_budget" if best != sm["learned_fps"] else "to_residual"
    out = {"metric": METRIC, "value": best, "unit": UNIT, "n_gpus": 1, "steps": sm["frames"],
           "warmup": skip, "ms_per_step": 1e3 / best, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f32 (MLP bf16 / fp32 accumulate)", "data": "synthetic",
           "config": {"workload": desc, "instances": cloth.info.num_instances, "vertices": nv,
                      "iterations": iters, "threads_per_vertex": cloth.info.threads_per_vertex},
           "clocks": clk,
           "target": "each instance's relative residual after the plain solver's iteration budget "
                     "(a 1e-4 residual is not reached by plain VBD on these cloths within thousands of iterations)",
           "learned_vs_plain": sm, "train": {"samples": trajectories * frames * nv, "record_s": t_record,
                                             "train_s": t_train, "final_loss_normalised": loss}}
    if rank == 0:
        print(json.dumps(out), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    elif args.workload in ("c3", "c4"):
        run_learned(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()

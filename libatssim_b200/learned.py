"""Training and evaluation protocol of the learned warm start (configurations c3, c4).

Everything runs through the C ABI; this module only sequences the calls.

  record   frames of the plain solver with a random wind per frame (per instance):
           predict -> ats_record_frame_begin -> `iters` VBD iterations ->
           ats_record_frame_end -> update, trajectories restarted from rest.
  train    normalisation from the data, then Adam on batches drawn from it.
  evaluate on held-out wind seeds, from the same frame-start states:
           plain    the CUDA-graph frame (predict, `iters` iterations, update) is timed;
                    its per-instance residual r_plain = ||grad G(x)|| / ||grad G(y)||
                    (the same sweeps replayed untimed) is the target;
           learned  predict, learned guess (potential fallback per instance), then
                    iterations until each instance reaches its r_plain, at most `iters`;
                    converged instances are skipped. Probes every `check_every`, the
                    first one (schedule) at the instance's previous-frame count minus
                    `lead` ("prev") or at a percentile of all previous-frame counts
                    (a number), or at check_every (None).
           Frame times are CUDA-event times of each whole frame (host checks included).
"""
import time

import numpy as np

from . import Dataset, MLP, configs


def wind_table(rng, masses):
    return np.stack([configs.wind_accel(rng, m) for m in masses]).astype(np.float32)


def record(cloth, insts, dataset, trajectories, frames, iters, seed0):
    masses = [float(i.mass.sum()) for i in insts]
    x_rest = np.concatenate([i.positions for i in insts])
    for t in range(trajectories):
        cloth.set_state(x_rest, np.zeros_like(x_rest))
        for f in range(frames):
            cloth.set_accel(wind_table(np.random.RandomState(seed0 + t * frames + f), masses))
            cloth.predict()
            cloth.record_begin()
            cloth.vbd_iterations(iters)
            cloth.record_end(dataset)
            cloth.update_velocity()


def train(dataset, steps=150000, batch=32768, lr=2e-3, seed=0):
    """Normalisation from the data, then Adam: half the steps at lr, a quarter at lr/3,
    a quarter at lr/10. Returns (model, mean loss of the last steps, seconds)."""
    m = MLP(seed=seed)
    m.fit_normalization(dataset)
    t = time.perf_counter()
    m.train(dataset, steps=steps // 2, batch=batch, lr=lr, seed=seed)
    m.train(dataset, steps=steps // 4, batch=batch, lr=lr / 3, seed=seed + 1)
    loss = m.train(dataset, steps=steps - steps // 2 - steps // 4, batch=batch, lr=lr / 10, seed=seed + 2)
    return m, loss, time.perf_counter() - t


def evaluate(cloth, insts, model, iters, seed0, trajectories=2, frames=40, skip=15, check_every=5, schedule=None,
             lead=2, stream=None):
    """Per evaluated frame: plain and learned frame times, iterations, residuals,
    and the FP64 incremental potential reached by both."""
    import torch
    masses = [float(i.mass.sum()) for i in insts]
    x_rest = np.concatenate([i.positions for i in insts])
    st = stream if stream is not None else torch.cuda.current_stream()
    out = {"plain_ms": [], "learned_ms": [], "learned_iters": [], "used": [], "g_plain": [], "g_learned": [],
           "r_plain": [], "r_learned": []}
    prev = None  # iterations of the previous learned frame, per instance
    for t in range(trajectories):
        cloth.set_state(x_rest, np.zeros_like(x_rest))
        for f in range(frames):
            cloth.set_accel(wind_table(np.random.RandomState(seed0 + t * frames + f), masses))
            if f >= skip:
                x0, v0 = cloth.state()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                # plain: the CUDA-graph frame (predict, iters x colours, update)
                torch.cuda.synchronize()
                e0.record(st)
                cloth.frame(graph=True, stream=st)
                e1.record(st)
                torch.cuda.synchronize()
                out["plain_ms"].append(e0.elapsed_time(e1))
                # its per-instance residual (the same sweeps, replayed untimed)
                cloth.set_state(x0, v0)
                _, r_plain = cloth.frame_to_residual(0.0, check_every=iters, max_iterations=iters, stream=st)
                out["r_plain"].append(r_plain)
                out["g_plain"].append(final_potential(cloth, x0, v0))
                # learned: guess, then iterations until every instance reaches r_plain
                torch.cuda.synchronize()
                e0.record(st)
                first = None
                if prev is not None and schedule == "prev":
                    first = np.maximum(1, prev - lead)
                elif prev is not None and schedule is not None:
                    first = np.full(len(prev), max(1, int(np.percentile(prev, schedule))), dtype=np.int32)
                torch.cuda.nvtx.range_push("learned_frame")  # lets a profiler select these kernels
                its, r_l, used = cloth.frame_warm_to_residual(model, r_plain, check_every=check_every,
                                                              max_iterations=iters, first_check=first, stream=st)
                torch.cuda.nvtx.range_pop()
                prev = its.copy()
                e1.record(st)
                torch.cuda.synchronize()
                out["learned_ms"].append(e0.elapsed_time(e1))
                out["learned_iters"].append(its)
                out["used"].append(used)
                out["r_learned"].append(r_l)
                out["g_learned"].append(final_potential(cloth, x0, v0))
            cloth.frame(graph=True)
    return {k: np.array(v) for k, v in out.items()}


def evaluate_fixed(cloth, insts, model, budget, iters, seed0, trajectories=2, frames=40, skip=15, stream=None):
    """The learned frame with a fixed iteration budget, replayed as a CUDA graph:
    per evaluated frame its time and, per instance, whether it reached the residual of
    the plain frame (plain `iters` iterations from the same start)."""
    import torch
    masses = [float(i.mass.sum()) for i in insts]
    x_rest = np.concatenate([i.positions for i in insts])
    st = stream if stream is not None else torch.cuda.current_stream()
    ms, reached, ratio = [], [], []
    # capture the graph before timing (a replay after capture is what a frame costs)
    cloth.set_state(x_rest, np.zeros_like(x_rest))
    cloth.frame_warm(model, fallback=True, iterations=budget, graph=True, stream=st)
    torch.cuda.synchronize()
    for t in range(trajectories):
        cloth.set_state(x_rest, np.zeros_like(x_rest))
        for f in range(frames):
            cloth.set_accel(wind_table(np.random.RandomState(seed0 + t * frames + f), masses))
            if f >= skip:
                x0, v0 = cloth.state()
                _, r_plain = cloth.frame_to_residual(0.0, check_every=iters, max_iterations=iters, stream=st)
                cloth.set_state(x0, v0)
                cloth.predict(stream=st)
                r0 = cloth.residual(stream=st)
                cloth.warm_start(model, fallback=True, stream=st)
                cloth.vbd_iterations(budget, stream=st)
                r_l = cloth.residual(stream=st) / r0
                reached.append(r_l <= r_plain * (1 + 1e-9))
                ratio.append(r_l / r_plain)
                cloth.set_state(x0, v0)
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                torch.cuda.synchronize()
                e0.record(st)
                cloth.frame_warm(model, fallback=True, iterations=budget, graph=True, stream=st)
                e1.record(st)
                torch.cuda.synchronize()
                ms.append(e0.elapsed_time(e1))
                cloth.set_state(x0, v0)
            cloth.frame(graph=True)
    return {"budget": int(budget), "learned_fixed_fps": float(1e3 / np.mean(ms)),
            "learned_fixed_ms_p50": float(np.percentile(ms, 50)), "learned_fixed_ms_p99": float(np.percentile(ms, 99)),
            "reached_plain_residual_fraction": float(np.mean(np.concatenate(reached))),
            "residual_ratio_median": float(np.median(np.concatenate(ratio)))}


def plain_per_instance_ms(insts, prm, frames=10, warmup=3, seed0=10000, stream=None):
    """The unbatched plain form: one handle per instance, every instance advanced one
    frame (CUDA-graph replay) per step, all on one stream; mean ms per step."""
    import torch

    from . import Cloth
    st = stream if stream is not None else torch.cuda.current_stream()
    handles = [Cloth([i], **prm) for i in insts]
    for h in handles:
        h.autotune(iterations=10)
    rng_masses = [float(i.mass.sum()) for i in insts]
    for f in range(warmup):
        for h in handles:
            h.frame(graph=True, stream=st)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    for f in range(frames):
        acc = wind_table(np.random.RandomState(seed0 + f), rng_masses)
        for k, h in enumerate(handles):
            h.set_accel(acc[k:k + 1], stream=st)
            h.frame(graph=True, stream=st)
    e1.record(st)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / frames
    for h in handles:
        h.close()
    return ms


def final_potential(cloth, x0, v0):
    """FP64 incremental potential of the frame just finished (its end state is the new
    frame start) against its own frame start (x0, v0); leaves the handle at (x0, v0)."""
    x_end, _ = cloth.state()
    cloth.set_state(x0, v0)
    cloth.set_positions(x_end)
    e = float(cloth.energy().sum())
    cloth.set_state(x0, v0)
    return e


def summary(res, iters, per_instance_ms=None):
    plain = res["plain_ms"]
    learned = res["learned_ms"]
    it = res["learned_iters"].astype(np.float64)
    extra = {}
    if per_instance_ms is not None:
        extra = {"plain_unbatched_fps": float(1e3 / per_instance_ms),
                 "speedup_vs_unbatched": float(per_instance_ms / np.mean(learned))}
    return {**extra,
        "frames": int(len(plain)),
        "plain_fps": float(1e3 / np.mean(plain)),
        "learned_fps": float(1e3 / np.mean(learned)),
        "speedup": float(np.mean(plain) / np.mean(learned)),
        "plain_ms_p50": float(np.percentile(plain, 50)),
        "plain_ms_p99": float(np.percentile(plain, 99)),
        "learned_ms_p50": float(np.percentile(learned, 50)),
        "learned_ms_p99": float(np.percentile(learned, 99)),
        "iterations_plain": int(iters),
        "iterations_learned_mean": float(it.mean()),
        "iterations_learned_p50": float(np.median(it)),
        "guess_kept_fraction": float(res["used"].mean()),
        "residual_plain_median": float(np.median(res["r_plain"])),
        "residual_learned_median": float(np.median(res["r_learned"])),
        "potential_rel_diff_median": float(np.median((res["g_learned"] - res["g_plain"]) / np.abs(res["g_plain"]))),
    }

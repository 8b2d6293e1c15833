"""Training and evaluation protocol of the learned warm start (configurations c3, c4).

Everything runs through the C ABI; this module only sequences the calls.

  record   frames of the plain solver with a random wind per frame (per instance):
           predict -> ats_record_frame_begin -> `iters` VBD iterations ->
           ats_record_frame_end -> update, trajectories restarted from rest.
  train    normalisation from the data, then Adam on batches drawn from it.
  fixed_tolerance_frames
           the comparison at one fixed relative residual `tol` with an iteration
           cap, on held-out wind seeds. Per frame, from the same start state:
             learned  predict, the network's guess (per-instance potential fallback),
                      then VBD iterations until each instance's residual
                      ||grad G(x)|| / ||grad G(y)|| <= tol or `cap` iterations;
             plain    predict, then VBD iterations to the same tol / cap.
           Both probe every `check_every` iterations (and at the cap) and skip the
           instances that have stopped. The plain frame's end state starts the next
           frame, so the trajectory is the plain form's. Frame times are CUDA events
           around each whole frame, host checks included.
  residual_traces / tolerance_sweep
           the relative residual of every instance at fixed iteration counts for
           both forms from the same start (untimed, FP64), and from it the iterations
           each form needs to reach each tolerance.
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



def approach(cloth, insts, frames, seed0, stream=None):
    """From rest, `frames` plain CUDA-graph frames with a seeded wind per frame (the
    cloth is moving when the measured frames begin)."""
    masses = [float(i.mass.sum()) for i in insts]
    x_rest = np.concatenate([i.positions for i in insts])
    cloth.set_state(x_rest, np.zeros_like(x_rest))
    for f in range(frames):
        cloth.set_accel(wind_table(np.random.RandomState(seed0 + f), masses), stream=stream)
        cloth.frame(graph=True, stream=stream)


def fixed_tolerance_frames(cloth, insts, model, tol, cap, check_every, frames, warmup, seed0, stream=None,
                           on_timed=None):
    """The learned and the plain frame to the same relative residual `tol` (at most
    `cap` iterations) from the same start, `warmup` untimed then `frames` timed frames
    with winds seeded seed0, seed0 + 1, ... Returns per-frame times (ms), and per frame
    and instance the iterations, relative residuals and whether the guess was kept.
    on_timed(True/False) brackets the timed frames (e.g. a clock sampler)."""
    import torch
    st = stream if stream is not None else torch.cuda.current_stream()
    masses = [float(i.mass.sum()) for i in insts]
    out = {k: [] for k in ("learned_ms", "plain_ms", "learned_iters", "plain_iters", "learned_res", "plain_res",
                           "used")}
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    for f in range(warmup + frames):
        timed = f >= warmup
        if timed and f == warmup and on_timed:
            on_timed(True)
        cloth.set_accel(wind_table(np.random.RandomState(seed0 + f), masses), stream=st)
        x0, v0 = cloth.state(stream=st)
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_push("learned_frame")  # lets a profiler select these kernels
        ev[0].record(st)
        it_l, r_l, used = cloth.frame_warm_to_residual(model, tol, check_every=check_every, max_iterations=cap,
                                                       stream=st)
        ev[1].record(st)
        torch.cuda.nvtx.range_pop()
        cloth.set_state(x0, v0, stream=st)
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_push("plain_frame")
        ev[2].record(st)
        it_p, r_p = cloth.frame_to_residual(tol, check_every=check_every, max_iterations=cap, stream=st)
        ev[3].record(st)
        torch.cuda.nvtx.range_pop()
        torch.cuda.synchronize()
        if timed:
            out["learned_ms"].append(ev[0].elapsed_time(ev[1]))
            out["plain_ms"].append(ev[2].elapsed_time(ev[3]))
            out["learned_iters"].append(it_l)
            out["plain_iters"].append(it_p)
            out["learned_res"].append(r_l)
            out["plain_res"].append(r_p)
            out["used"].append(used)
    if on_timed:
        on_timed(False)
    return {k: np.array(v) for k, v in out.items()}


def residual_traces(cloth, model, points, stream=None):
    """From the current frame-start state: predict, then (plain) VBD iterations with
    the FP64 relative residual of every instance after each count in `points`, and the
    same from the learned guess. Returns (plain, learned), arrays (len(points), ninst);
    the frame-start state is restored."""
    x0, v0 = cloth.state(stream=stream)
    traces = []
    for warm in (False, True):
        cloth.set_state(x0, v0, stream=stream)
        cloth.predict(stream=stream)
        r0 = cloth.residual(stream=stream)
        if warm:
            cloth.warm_start(model, fallback=True, stream=stream)
        done = 0
        rows = []
        for k in points:
            if k > done:
                cloth.vbd_iterations(k - done, stream=stream)
                done = k
            rows.append(np.where(r0 > 0, cloth.residual(stream=stream) / np.where(r0 > 0, r0, 1.0), 0.0))
        traces.append(np.array(rows))
    cloth.set_state(x0, v0, stream=stream)
    return traces[0], traces[1]


def iterations_to(trace, points, tol):
    """Per instance the first count in `points` at which the trace is <= tol (-1: never)."""
    hit = trace <= tol
    first = np.argmax(hit, axis=0)
    return np.where(hit.any(axis=0), np.asarray(points)[first], -1)


def tolerance_sweep(cloth, insts, model, tols, points, frames, seed0, stream=None):
    """Residual traces of both forms over `frames` held-out frames (the trajectory
    advanced by plain CUDA-graph frames between them), and per tolerance the
    iterations each form needs (vertex-weighted over instance-frames that reached it
    within max(points), and the fraction that did)."""
    masses = [float(i.mass.sum()) for i in insts]
    nv = np.array([i.num_verts for i in insts], dtype=np.float64)
    plain, learned = [], []
    for f in range(frames):
        cloth.set_accel(wind_table(np.random.RandomState(seed0 + f), masses), stream=stream)
        p, l = residual_traces(cloth, model, points, stream=stream)
        plain.append(p)
        learned.append(l)
        cloth.frame(graph=True, stream=stream)
    plain = np.concatenate(plain, axis=1)  # (points, frames * ninst)
    learned = np.concatenate(learned, axis=1)
    w = np.tile(nv, frames)
    rows = []
    for tol in tols:
        row = {"tol": tol}
        for name, tr in (("plain", plain), ("learned", learned)):
            it = iterations_to(tr, points, tol)
            ok = it >= 0
            row[name + "_reached_fraction"] = float(ok.mean())
            row[name + "_iterations_vertex_weighted"] = (float(np.sum(it[ok] * w[ok]) / np.sum(w[ok]))
                                                         if ok.any() else None)
            row[name + "_iterations_p50"] = float(np.median(it[ok])) if ok.any() else None
        rows.append(row)
    trace = {"points": list(map(int, points)),
             "plain_median": np.median(plain, axis=1).tolist(), "learned_median": np.median(learned, axis=1).tolist(),
             "plain_max": np.max(plain, axis=1).tolist(), "learned_max": np.max(learned, axis=1).tolist(),
             "plain_min": np.min(plain, axis=1).tolist(), "learned_min": np.min(learned, axis=1).tolist()}
    return rows, trace


def timed_to_tolerance(cloth, insts, model, tol, cap, check_every, frames, seed0, stream=None):
    """Mean frame time (ms) of both forms to `tol` (cap iterations) over `frames`
    held-out frames from the same starts, and the fraction of instance-frames that
    reached tol; the trajectory is advanced by the plain frame."""
    res = fixed_tolerance_frames(cloth, insts, model, tol, cap, check_every, frames, 0, seed0, stream=stream)
    return {"tol": tol, "plain_ms": float(np.mean(res["plain_ms"])), "learned_ms": float(np.mean(res["learned_ms"])),
            "speedup": float(np.mean(res["plain_ms"]) / np.mean(res["learned_ms"])),
            "plain_reached_fraction": float(np.mean(res["plain_res"] <= tol)),
            "learned_reached_fraction": float(np.mean(res["learned_res"] <= tol))}

"""Multi-GPU layout of the batched workloads: one process per GPU.

Batched instances are independent during a frame, so they are partitioned across
ranks with no collective on the data path; each rank builds its own handle (and its
own frame graph) over its share. What crosses GPUs:
  * per-frame FP64 statistics (residual norms, energies, counts), one all-reduce;
  * during data-parallel training of the warm-start MLP, the averaged gradient of
    the 10,115 parameters per step.
torch.distributed carries both (NCCL across GPUs, gloo on CPU); without an
initialised process group every function here is the single-rank identity.
"""
import numpy as np


def _dist():
    try:
        import torch.distributed as dist
        if dist.is_available() and dist.is_initialized():
            return dist
    except Exception:
        pass
    return None


def rank_world():
    d = _dist()
    return (d.get_rank(), d.get_world_size()) if d else (0, 1)


def partition(costs, world):
    """Greedy balanced bin-packing: instances by decreasing cost, each to the rank
    with the least load so far (ties to the lower rank). Returns per-rank lists of
    instance indices in increasing order."""
    costs = np.asarray(costs, dtype=np.float64)
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    load = [0.0] * world
    out = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda q: (load[q], q))
        out[r].append(i)
        load[r] += costs[i]
    return [sorted(x) for x in out]


def shard(instances, iterations, rank=None, world=None):
    """This rank's instances (cost = vertices x iterations)."""
    if rank is None:
        rank, world = rank_world()
    parts = partition([inst.num_verts * iterations for inst in instances], world)
    return [instances[i] for i in parts[rank]], parts[rank]


def _device():
    d = _dist()
    if d and d.get_backend() == "nccl":
        import torch
        return torch.device("cuda", torch.cuda.current_device())
    return None


def allreduce_stats(values, op="sum"):
    """FP64 all-reduce of a small statistics vector (sum or max)."""
    d = _dist()
    v = np.asarray(values, dtype=np.float64)
    if not d:
        return v
    import torch
    t = torch.from_numpy(v.copy())
    dev = _device()
    if dev is not None:
        t = t.to(dev)
    d.all_reduce(t, op=d.ReduceOp.SUM if op == "sum" else d.ReduceOp.MAX)
    return t.cpu().numpy()


def global_residual(local_norms):
    """||grad G|| over all ranks' instances from each rank's per-instance norms."""
    return float(np.sqrt(allreduce_stats([float(np.sum(np.square(local_norms)))])[0]))


def data_parallel_train(mlp, dataset, steps, batch=4096, lr=1e-3, seed=0):
    """Each rank draws its own batches; gradients are averaged over ranks before every
    Adam step, so every rank holds the same parameters. Returns the last mean loss."""
    rank, world = rank_world()
    loss = 0.0
    for s in range(steps):
        l, g = mlp.batch_gradient(dataset, batch=batch, seed=seed * 1_000_003 + s * world + rank)
        red = allreduce_stats(np.concatenate([g.astype(np.float64), [l]]))
        mlp.apply_gradient((red[:-1] / world).astype(np.float32), lr=lr)
        loss = red[-1] / world
    return float(loss)

"""Sweeps of independent nozzle instances sharded over GPUs (one process per
GPU): instances are assigned to ranks balanced by cell count, each rank
advances its share as a batch on its own GPU, and the per-instance results
(iterations, normpl, fmi, fme, Fd, Cd) are gathered on every rank in the
sweep's order.  The instances never exchange data while they run; the only
collectives are the result gather and the max-over-ranks of the timings.
"""
import time


def shard_indices(sizes, world):
    """Longest-processing-time assignment: instances in decreasing size, each
    to the rank with the least total so far (ties: lowest rank).  Returns one
    sorted index list per rank."""
    load = [0] * world
    parts = [[] for _ in range(world)]
    for i in sorted(range(len(sizes)), key=lambda k: (-sizes[k], k)):
        r = min(range(world), key=lambda q: (load[q], q))
        parts[r].append(i)
        load[r] += sizes[i]
    return [sorted(p) for p in parts]


def gather_results(local, n, group=None):
    """local: {instance index: tuple of floats} of this rank; returns the list
    of all n tuples in index order (every rank gets it)."""
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized():
        return [local[i] for i in range(n)]
    world = dist.get_world_size(group)
    parts = [None] * world
    dist.all_gather_object(parts, local, group=group)
    merged = {}
    for p in parts:
        merged.update(p)
    if sorted(merged) != list(range(n)):
        raise RuntimeError("sweep: gathered results do not cover every instance exactly once")
    return [merged[i] for i in range(n)]


def run_shard(cases, indices, device, iters, graph=True, timings=None, tune=0):
    """Advances the cases at `indices` as one batch on `device`: `iters` outer
    iterations each (or, with iters <= 0, each to its stopping iteration, at
    most 100000).  Returns ({index: (it, normpl, fmi, fme, Fd, Cd)}, seconds).
    With a dict `timings`, also records the batch set-up time in
    timings["setup_s"] (grids, metrics and initial fields of every instance).
    With tune > 0 (and graph), the batch's MSI schedule is first autotuned on
    the batch's own next iterations (m2d_batch_autotune, `tune` timed
    iterations per candidate; the schedules give the same iterates), and
    timings["schedule"] records the choice and the candidates' times."""
    import torch

    from .simplec import Batch
    if not indices:
        if timings is not None:
            timings["setup_s"] = 0.0
        return {}, 0.0
    torch.cuda.synchronize(device)
    t_setup = time.perf_counter()
    b = Batch([cases[i] for i in indices], device=device)
    torch.cuda.synchronize(device)
    if timings is not None:
        timings["setup_s"] = time.perf_counter() - t_setup
    if graph:
        for s in b.instances:
            s.set_graph(True)
        if tune > 0:
            chosen, ms = b.autotune(tune)
            if timings is not None:
                timings["schedule"] = {"chosen": chosen, "ms_per_batch_iteration": ms,
                                       "tuning_iterations": (1 + tune) * len(ms)}
    torch.cuda.synchronize(device)
    t0 = time.perf_counter()
    if iters > 0:
        reps = b.iterate(iters)
    else:
        reps = [s.run(100000) for s in b.instances]
    torch.cuda.synchronize(device)
    secs = time.perf_counter() - t0
    out = {}
    for i, s, r in zip(indices, b.instances, reps):
        fmi, fme, Fd, Cd, _ = s.integrals()
        out[i] = (float(r.it), float(r.normpl), float(fmi), float(fme), float(Fd), float(Cd))
    b.close()
    return out, secs

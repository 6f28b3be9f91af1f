"""Multi-GPU analyzer sharding: configurations are independent, so each rank
measures a contiguous block of them on its own GPU (no exchange during the
solves) and the per-configuration outputs are all-gathered at the end, after
which every rank holds the ensemble and rank 0 runs the host reductions
(domain_wall/analyze_configs.cpp:78-227) exactly as on one GPU.

Works with any torch.distributed backend: NCCL between GPUs (CUDA tensors),
gloo on the host (the multi-process CPU tests)."""
import numpy as np


def partition(nconf, world, rank):
    """[start, stop) of this rank's configurations: contiguous, sizes differing
    by at most one, earlier ranks taking the remainder."""
    if nconf < 0 or world < 1 or not 0 <= rank < world:
        raise ValueError("partition: bad nconf / world / rank")
    base, rem = divmod(nconf, world)
    start = rank * base + min(rank, rem)
    return start, start + base + (1 if rank < rem else 0)


def gather_outputs(local, nconf, world, rank, device=None):
    """All-gather {name: array [n_local, ...]} into {name: array [nconf, ...]}
    in configuration order. Blocks are padded to the largest shard for the
    collective and trimmed afterwards."""
    sizes = [partition(nconf, world, r)[1] - partition(nconf, world, r)[0] for r in range(world)]
    if world == 1:
        # one rank holds the whole ensemble: no collective (and no process group) needed
        for name in local:
            if np.shape(local[name])[0] != nconf:
                raise ValueError(f"gather_outputs: {name} has {np.shape(local[name])[0]} rows, "
                                 f"rank owns {nconf}")
        return {name: np.asarray(local[name]) for name in sorted(local)}
    import torch
    import torch.distributed as dist
    cap = max(sizes) if sizes else 0
    out = {}
    for name in sorted(local):
        a = np.asarray(local[name])
        if a.shape[0] != sizes[rank]:
            raise ValueError(f"gather_outputs: {name} has {a.shape[0]} rows, rank owns {sizes[rank]}")
        tail = a.shape[1:]
        cplx = np.iscomplexobj(a)
        real = a.view(np.float64).reshape((a.shape[0],) + tail + ((2,) if cplx else ())) if cplx \
            else a.astype(np.float64)
        buf = np.zeros((cap,) + real.shape[1:], np.float64)
        buf[:real.shape[0]] = real
        t = torch.from_numpy(buf)
        if device is not None:
            t = t.to(device)
        parts = [torch.empty_like(t) for _ in range(world)]
        dist.all_gather(parts, t)
        rows = [p.cpu().numpy()[:sizes[r]] for r, p in enumerate(parts)]
        full = np.concatenate(rows, axis=0) if rows else np.zeros((0,) + real.shape[1:])
        if cplx:
            full = np.ascontiguousarray(full).view(np.complex128).reshape((nconf,) + tail)
        out[name] = full
    return out


def sharded_measure(measure, thetas, world, rank, device=None):
    """Run measure(thetas_block) -> {name: [n_block, ...]} on this rank's block
    and gather the ensemble on every rank."""
    thetas = np.asarray(thetas)
    nconf = thetas.shape[0]
    a, b = partition(nconf, world, rank)
    local = measure(thetas[a:b])
    return gather_outputs(local, nconf, world, rank, device)

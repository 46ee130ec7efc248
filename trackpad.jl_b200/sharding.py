"""Data-parallel tracking over several GPUs, one process per GPU.

Particles are independent, and so are lattice variants, so the tracking path
shards without any exchange: each rank tracks a contiguous range of the
particles (one lattice) or a set of whole variants (a batch), on its own GPU.
The only collective is the adjoint's: the loss and its gradient over the
union of the ranks' particles need the sums of the per-rank terms, one
all-reduce of (3 + number of parameters) doubles per gradient.

  particle_shard(n, rank, world)      contiguous [start, stop) of rank's particles
  variant_shard(costs, world)         variants per rank, balanced by cost (longest first)
  combine_adjoint(terms, all_reduce)  global loss and gradient from per-rank terms
  distributed_ringpass_(...)          ringpass! of one coordinate matrix split over the ranks,
                                      each rank tracking its shard, the results gathered back
  distributed_ringpass_adjoint(...)   the adjoint on this rank's shard, combined over the group

Launch one process per GPU (torchrun); the collective runs on whatever
process group the caller passes (NCCL for GPU tensors, gloo on CPU).
"""
import numpy as np


def particle_shard(n, rank, world):
    """[start, stop) of the particles of `rank` out of `world`: contiguous,
    sizes differing by at most one."""
    if world <= 0 or not 0 <= rank < world:
        raise ValueError("need 0 <= rank < world")
    base, extra = divmod(int(n), int(world))
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def variant_shard(costs, world):
    """Assign variants to ranks: longest-processing-time first, each to the
    rank with the least work so far.  costs[v] is the work of variant v (e.g.
    elements x particles).  Returns one sorted list of variant indices per rank;
    the assignment is deterministic, so every rank computes the same one."""
    costs = [float(c) for c in costs]
    order = sorted(range(len(costs)), key=lambda v: (-costs[v], v))
    load = [0.0] * int(world)
    out = [[] for _ in range(int(world))]
    for v in order:
        r = min(range(int(world)), key=lambda k: (load[k], k))
        out[r].append(v)
        load[r] += costs[v]
    return [sorted(x) for x in out]


def local_terms(loss, grad, survivors, alive0, lost_weight):
    """The additive terms of one rank's result: (sum of q over its survivors,
    survivors, alive at start, survivors x gradient), with
    loss = sum_q / survivors + lost_weight * (alive0 - survivors) / alive0."""
    grad = np.asarray(grad, dtype=np.float64)
    if survivors > 0:
        frac = (alive0 - survivors) / alive0 if alive0 > 0 else 0.0
        qsum = (loss - lost_weight * frac) * survivors
    else:
        qsum = 0.0
    return np.concatenate([[qsum, float(survivors), float(alive0)], grad * float(survivors)])


def combine_adjoint(terms, all_reduce, lost_weight):
    """Global (loss, grad) from this rank's `local_terms` vector.  `all_reduce`
    sums a float64 numpy vector over the ranks in place or returns the sum."""
    v = np.array(terms, dtype=np.float64)
    r = all_reduce(v)
    if r is not None:
        v = np.asarray(r, dtype=np.float64)
    qsum, surv, alive = v[0], v[1], v[2]
    frac = (alive - surv) / alive if alive > 0 else 0.0
    loss = (qsum / surv if surv > 0 else 0.0) + lost_weight * frac
    grad = v[3:] / surv if surv > 0 else np.zeros_like(v[3:])
    return float(loss), grad


def torch_all_reduce(group=None, device=None):
    """A sum all-reduce over a torch.distributed group (NCCL or gloo)."""
    import torch
    import torch.distributed as dist

    def reduce(v):
        t = torch.from_numpy(np.ascontiguousarray(v))
        if device is not None:
            t = t.to(device)
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
        return t.cpu().numpy()

    return reduce


def distributed_ringpass_adjoint(coords0, lat, beam, lost0, nturns, params, *, sigma, lost_weight=1e3,
                                 group=None, device=None, **kw):
    """Loss and gradient over the particles of every rank of `group`: each rank
    passes its own shard (`particle_shard`), runs the adjoint on its GPU, and
    one all-reduce of (3 + len(params)) doubles combines the results."""
    from . import tracking
    loss, grad = tracking.ringpass_adjoint(coords0, lat, beam, lost0, nturns, params, sigma=sigma,
                                           lost_weight=lost_weight, **kw)
    st = tracking.last_stats()
    terms = local_terms(loss, grad, st["survivors"], st["particles"], lost_weight)
    return combine_adjoint(terms, torch_all_reduce(group, _collective_device(group, device)), lost_weight)


def _collective_device(group, device):
    """Where a collective's tensors live: the given device, else the current
    GPU for NCCL (which takes CUDA tensors only), else the host (gloo)."""
    import torch.distributed as dist
    if device is not None:
        return device
    if dist.get_backend(group) == "nccl":
        import torch
        return torch.device("cuda", torch.cuda.current_device())
    return None


def torch_all_gather(group=None, device=None):
    """Gather one numpy array per rank (same dtype and trailing shape, leading
    sizes may differ) over a torch.distributed group: every rank gets the
    list of all ranks' arrays in rank order.  Arrays are padded to the largest
    leading size for the collective (all_gather wants equal sizes)."""
    import torch
    import torch.distributed as dist

    def gather(a):
        a = np.ascontiguousarray(a)
        world = dist.get_world_size(group)
        n = torch.tensor([a.shape[0]], dtype=torch.int64, device=device)
        sizes = [torch.zeros_like(n) for _ in range(world)]
        dist.all_gather(sizes, n, group=group)
        sizes = [int(x.item()) for x in sizes]
        m = max(sizes) if sizes else 0
        buf = np.zeros((m,) + a.shape[1:], dtype=a.dtype)
        buf[:a.shape[0]] = a
        t = torch.from_numpy(buf)
        if device is not None:
            t = t.to(device)
        outs = [torch.empty_like(t) for _ in range(world)]
        dist.all_gather(outs, t, group=group)
        return [o.cpu().numpy()[:k] for o, k in zip(outs, sizes)]

    return gather


def shard_and_gather(coords, lost_flags, rank, world, track_shard, gather, lost_turn=None, lost_elem=None):
    """Split the N x 6 host matrix `coords` (and its per-particle arrays) into
    `world` contiguous particle shards, let `track_shard(c, lost, lt, le)`
    update this rank's shard in place (c is an (n_r, 6) column-major copy),
    then gather every rank's shard back into the full arrays, in place, on
    every rank.  Returns this rank's (start, stop)."""
    n = coords.shape[0]
    lo, hi = particle_shard(n, rank, world)
    c = np.asfortranarray(coords[lo:hi])
    lf = np.ascontiguousarray(lost_flags[lo:hi])
    lt = None if lost_turn is None else np.ascontiguousarray(lost_turn[lo:hi])
    le = None if lost_elem is None else np.ascontiguousarray(lost_elem[lo:hi])
    track_shard(c, lf, lt, le)
    # one gather of a packed row per particle: 6 coordinates, flag, turn, element
    packed = np.empty((hi - lo, 9), dtype=np.float64)
    packed[:, :6] = c
    packed[:, 6] = lf
    packed[:, 7] = -1 if lt is None else lt
    packed[:, 8] = -1 if le is None else le
    parts = gather(packed)
    full = np.concatenate(parts, axis=0) if parts else packed
    if full.shape[0] != n:
        raise RuntimeError(f"gathered {full.shape[0]} particles, expected {n}")
    coords[...] = full[:, :6]
    lost_flags[...] = full[:, 6].astype(np.int64)
    if lost_turn is not None:
        lost_turn[...] = full[:, 7].astype(np.int32)
    if lost_elem is not None:
        lost_elem[...] = full[:, 8].astype(np.int32)
    return lo, hi


def distributed_ringpass_(coords, lat, beam, lost_flags, nturns, *, group=None, device=None, lost_turn=None,
                          lost_elem=None, **kw):
    """ringpass!(coords, lat, beam, lost_flags, nturns) with the particles
    split over the ranks of `group`: every rank passes the same N x 6 host
    matrix, tracks its contiguous shard (`particle_shard`) on its own GPU (the
    current device), and the shards are gathered back so that every rank ends
    with the whole result, as a single-process call would give.  No collective
    runs on the tracking path; the gather is one all-gather of 9 doubles per
    particle (coordinates, flag, turn and element of loss), on `device` when
    the group's backend is NCCL.  Keywords are those of tracking.ringpass_."""
    import torch.distributed as dist

    from . import tracking
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    coll_dev = _collective_device(group, device)

    def track(c, lf, lt, le):
        if c.shape[0]:
            tracking.ringpass_(c, lat, beam, lf, nturns, lost_turn=lt, lost_elem=le, **kw)

    return shard_and_gather(coords, lost_flags, rank, world, track, torch_all_gather(group, coll_dev),
                            lost_turn=lost_turn, lost_elem=lost_elem)

"""Multi-GPU plumbing: one process per GPU, points sharded by walker.

Points (walkers x electrons) are independent, so the forward evaluation needs
no exchange: each rank evaluates its own walkers with a full copy of the
basis and MO coefficients (a few MB).  The adjoint has one exchange step: the
coefficient and nuclear gradients are sums over all points, so each rank's
partial sums are all-reduced (torch.distributed, NCCL on GPUs).  The point
gradients stay with the rank that owns the points.

Timing across ranks is the maximum over ranks of each rank's device time.
"""
import torch


def shard(n, rank, world):
    """Contiguous block of range(n) owned by `rank` of `world`: (start, stop)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank outside the world")
    base, extra = divmod(n, world)
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def _dist():
    import torch.distributed as dist
    return dist if dist.is_available() and dist.is_initialized() else None


def max_over_ranks(value, device=None):
    """Maximum of a float over the ranks of the default process group (the value itself without one)."""
    dist = _dist()
    if dist is None:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks_(tensor):
    """In-place sum over the ranks of the default process group; returns the tensor."""
    dist = _dist()
    if dist is not None:
        dist.all_reduce(tensor, op=dist.ReduceOp.SUM)
    return tensor


def sharded_adjoint(walk_num, elec_num, rank, world, local_adjoint):
    """Gradients of L = sum W * mo_vgl with the walkers sharded over the ranks.

    local_adjoint(w0, w1) returns (grad_coef, grad_nucl, grad_coord) for the
    points of walkers [w0, w1) as tensors (grad_coord [3][points] of those
    walkers).  The coefficient and nuclear gradients are summed over the
    ranks (one all-reduce each); the point gradients are returned for the
    local walkers only, with the local walker range.
    """
    w0, w1 = shard(walk_num, rank, world)
    gc, gn, gr = local_adjoint(w0, w1)
    sum_over_ranks_(gc)
    sum_over_ranks_(gn)
    return gc, gn, gr, (w0, w1)

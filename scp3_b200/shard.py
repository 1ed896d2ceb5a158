"""Sample-range sharding of the Hamiltonian build over ranks (one per GPU).

Samples are independent and the Gray-code addressing reaches any Sobol index
directly, so rank r takes its own contiguous index range and accumulates a
private matrix; the one exchange is the sum of the ranks' matrices at read-out
(an all-reduce of the dense FP64 matrix), where SCP3 would otherwise sum one
process's blocks (SCP3.cpp:187-232)."""

RANK_STRIDE = 1 << 40   # weak scaling: rank r starts 2^40 points after rank r-1


def sample_range(rank, world, index0, n, scaling="weak"):
    """(first Sobol index, count) of rank `rank`.

    weak:   every rank takes n samples, rank r from index0 + r * 2^40.
    strong: the n samples from index0 are cut into `world` contiguous pieces,
            the first n % world ranks taking one more."""
    if not 0 <= rank < world:
        raise ValueError("rank out of range")
    if scaling == "weak":
        return index0 + rank * RANK_STRIDE, n
    if scaling == "strong":
        base, extra = divmod(n, world)
        start = index0 + rank * base + min(rank, extra)
        return start, base + (1 if rank < extra else 0)
    raise ValueError("scaling is 'weak' or 'strong'")


def reduce_matrix(M, group=None):
    """Sum a dense matrix (torch tensor) over the ranks of `group`, in place."""
    import torch.distributed as dist
    if dist.is_initialized() and dist.get_world_size(group) > 1:
        dist.all_reduce(M, op=dist.ReduceOp.SUM, group=group)
    return M

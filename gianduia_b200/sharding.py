"""Sample-pass sharding across ranks (one process per GPU).

Paths are independent, so N ranks render disjoint pass ranges of the same image and the
films -- per pixel sums of wL, w and wL^2 -- add up: rank r renders passes
[first + r * spp, first + (r + 1) * spp), and one sum-reduce of the films to rank 0 is the
only exchange (weak scaling: every rank does the work of one full render)."""


def pass_range(rank, world, spp, first=0):
    """Passes [begin, end) that `rank` of `world` renders when each rank renders `spp`."""
    if world <= 0 or not (0 <= rank < world):
        raise ValueError("rank %r outside a world of %r" % (rank, world))
    if spp <= 0:
        raise ValueError("spp must be positive")
    begin = first + rank * spp
    return begin, begin + spp


def reduce_film(film, dist, dst=0):
    """Sums the ranks' films (float32 [H, W, 7]) into rank `dst` with one collective.
    `film` is a torch tensor on the rank's device (NCCL) or on the CPU (gloo)."""
    dist.reduce(film, dst=dst, op=dist.ReduceOp.SUM)
    return film

"""Sample-pass sharding across ranks (one process per GPU).

Paths are independent, so N ranks render disjoint pass ranges of the same image and the
films -- per pixel sums of wL, w and wL^2 -- add up: rank r renders passes
[first + r * spp, first + (r + 1) * spp), and one sum-reduce of the films to rank 0 is the
only exchange (weak scaling: every rank does the work of one full render).

The exact film (gnd_gpu_render_fixed) keeps sum wL and sum w as 64-bit integers in units
of 2^-24: reduced as int64 (two's complement addition is the modulo-2^64 sum) they equal
one render of all the passes bit for bit, whatever the number of ranks."""
import numpy as np


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


def reduce_fixed_film(fsum, fsq, dist, dst=0):
    """Sums the ranks' exact films into rank `dst`: fsum (int64 torch tensor [H, W, 4], the
    uint64 sums viewed as int64) and fsq (float32 [H, W, 3]), on the rank's device (NCCL)
    or on the CPU (gloo). Two collectives, the same on every rank."""
    dist.reduce(fsum, dst=dst, op=dist.ReduceOp.SUM)
    dist.reduce(fsq, dst=dst, op=dist.ReduceOp.SUM)
    return fsum, fsq


def as_int64(fsum):
    """A uint64 numpy film viewed as int64 (same bits), for the collectives."""
    return np.ascontiguousarray(fsum).view(np.int64)


def as_uint64(fsum):
    """The inverse of as_int64."""
    return np.ascontiguousarray(fsum).view(np.uint64)

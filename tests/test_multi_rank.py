"""The N > 1 path of the bench on CPU: two gloo ranks each render their pass range of
the Cornell box with the oracle and reduce the films to rank 0; the sum equals one
render of all passes (film sums are additive; float sums are compared within 1e-5)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from gianduia_b200 import scenes
from gianduia_b200.sharding import pass_range


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, xml, spp, out_dir):
    import torch
    import torch.distributed as dist
    from oracle import pyoracle as O
    from gianduia_b200.sharding import pass_range, reduce_film
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        sc = O.Scene.load(xml)
        s0, s1 = pass_range(rank, world, spp)
        film, _, _ = sc.render(s0, s1, nthreads=2)
        t = torch.from_numpy(film)
        reduce_film(t, dist)
        if rank == 0:
            np.save(os.path.join(out_dir, "reduced.npy"), t.numpy())
    finally:
        dist.destroy_process_group()


def test_pass_range():
    assert pass_range(0, 2, 8) == (0, 8)
    assert pass_range(1, 2, 8) == (8, 16)
    assert pass_range(3, 4, 16, first=5) == (53, 69)
    with pytest.raises(ValueError):
        pass_range(2, 2, 8)
    with pytest.raises(ValueError):
        pass_range(0, 1, 0)


def test_two_gloo_ranks_sum_to_one_render(tmp_path):
    from oracle import pyoracle as O
    xml = scenes.cornell(str(tmp_path / "c"), width=24, height=24, spp=2, max_depth=4)
    spp = 2
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, xml, spp, str(tmp_path))) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    reduced = np.load(tmp_path / "reduced.npy")
    whole, _, _ = O.Scene.load(xml).render(0, 2 * spp, nthreads=2)
    np.testing.assert_allclose(reduced, whole, rtol=1e-5, atol=1e-6)

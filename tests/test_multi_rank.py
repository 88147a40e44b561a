"""The N > 1 path of the bench on CPU: two gloo ranks each render their pass range of
the Cornell box with the oracle and reduce the films to rank 0; the sum equals one
render of all passes. Float films are compared within 1e-5; the exact films (fixed-point
sum wL and sum w, reduced as int64) must equal the single render bit for bit."""
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


def _rank_main_fixed(rank, world, port, xml, spp, out_dir):
    import torch
    import torch.distributed as dist
    from oracle import pyoracle as O
    from gianduia_b200.sharding import as_int64, pass_range, reduce_fixed_film
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        sc = O.Scene.load(xml)
        s0, s1 = pass_range(rank, world, spp)
        fsum, fsq, _, _ = sc.render_fixed(s0, s1, nthreads=2)
        ts, tq = torch.from_numpy(as_int64(fsum)), torch.from_numpy(fsq)
        reduce_fixed_film(ts, tq, dist)
        if rank == 0:
            np.save(os.path.join(out_dir, "fixed_sum.npy"), ts.numpy())
            np.save(os.path.join(out_dir, "fixed_sq.npy"), tq.numpy())
    finally:
        dist.destroy_process_group()


def _run_ranks(target, world, xml, spp, out_dir):
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=target, args=(r, world, port, xml, spp, out_dir)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0


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


def test_fixed_point_films_reduce_exactly(tmp_path):
    """Exact films of two gloo ranks (passes [0, 3) and [3, 6)) reduced as int64 equal one
    render of passes [0, 6) bit for bit; sum wL^2 (float) agrees to rounding. The scene
    uses the default Gaussian filter, so samples reach up to 16 pixels."""
    from oracle import pyoracle as O
    from gianduia_b200.sharding import as_uint64
    xml = scenes.cornell(str(tmp_path / "c"), width=20, height=16, spp=3, max_depth=4, filter="gaussian")
    _run_ranks(_rank_main_fixed, 2, xml, 3, str(tmp_path))
    reduced = as_uint64(np.load(tmp_path / "fixed_sum.npy"))
    whole, wq, _, _ = O.Scene.load(xml).render_fixed(0, 6, nthreads=3)
    assert reduced.dtype == np.uint64 and np.array_equal(reduced, whole)
    assert int(whole[..., 3].min()) > 0
    np.testing.assert_allclose(np.load(tmp_path / "fixed_sq.npy"), wq, rtol=1e-5, atol=1e-6)
    # the fixed-point film resolves to the float film's image
    film, _, _ = O.Scene.load(xml).render(0, 6, nthreads=3)
    img_f = whole[..., :3].astype(np.float64) / whole[..., 3:4].astype(np.float64)
    img = film[..., :3] / film[..., 3:4]
    np.testing.assert_allclose(img_f, img, rtol=1e-4, atol=1e-5)

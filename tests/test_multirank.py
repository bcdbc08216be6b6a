"""The multi-GPU host logic on CPU ranks (gloo, world size 2): each rank renders disjoint frames of the spline (no
collective on the data path), the job's time is the slowest rank's and its rays every rank's; and two ranks rendering
their frames with the oracle give the images one rank gives for the same frames."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

import bench


def free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def test_frames_are_disjoint_across_ranks():
    for world in (1, 2, 4, 8):
        timed = [bench.rank_frames(r, world, 5, 20)[1] for r in range(world)]
        flat = [f for t in timed for f in t]
        assert len(flat) == len(set(flat)) == 20 * world
        assert all(len(t) == 20 for t in timed)


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import oracle
        from threert_b200 import prep, scenes
        from threert_b200.gpu import frame_of
        d = scenes.city(n_objects=30, width=24, height=16, seed=5, extent=40.0, n_emitters=20, box_segments=1,
                        sphere_slices=6, sphere_stacks=5, sky_size=(32, 16), sky="gradient")
        P = prep.prepare(d)
        _, frames = bench.rank_frames(rank, world, 1, 2, frames=8)
        O = oracle.Oracle(P)
        imgs, rays = {}, 0
        for f in frames:
            cam = scenes.city_camera(f, 8, 5, 24, 16, 40.0)
            acc, st = O.render(prep.set_camera(P.params, cam), 2, threads=1)
            imgs[f] = frame_of(acc, 24, 16, 2).color
            rays += st["closest_rays"] + st["shadow_rays"]
        ms, e2e, total = bench.reduce_over_ranks(dist, 10.0 + rank, 20.0 - rank, float(rays))
        gathered = [None] * world
        dist.all_gather_object(gathered, (imgs, rays))
        if rank == 0:
            out.put((ms, e2e, total, gathered))
    finally:
        dist.destroy_process_group()


def test_two_ranks_render_the_frames_one_rank_renders():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    try:
        ms, e2e, total, gathered = q.get(timeout=240)
    finally:
        for p in procs:
            p.join(timeout=60)
    assert all(p.exitcode == 0 for p in procs)
    assert ms == 11.0 and e2e == 20.0  # the slowest rank's times
    assert total == sum(r for _, r in gathered)
    frames0, frames1 = set(gathered[0][0]), set(gathered[1][0])
    assert not frames0 & frames1
    # One rank rendering the same frames gets the same images: a frame's pixels do not depend on the rank.
    import oracle
    from threert_b200 import prep, scenes
    from threert_b200.gpu import frame_of
    d = scenes.city(n_objects=30, width=24, height=16, seed=5, extent=40.0, n_emitters=20, box_segments=1,
                    sphere_slices=6, sphere_stacks=5, sky_size=(32, 16), sky="gradient")
    P = prep.prepare(d)
    O = oracle.Oracle(P)
    for imgs, _ in gathered:
        for f, img in imgs.items():
            cam = scenes.city_camera(f, 8, 5, 24, 16, 40.0)
            acc, _ = O.render(prep.set_camera(P.params, cam), 2, threads=1)
            assert np.array_equal(frame_of(acc, 24, 16, 2).color, img)


def test_sample_ranges_cover_the_samples_once():
    from threert_b200.split import sample_range
    for world in (1, 2, 3, 4, 8):
        for spp in (0, 1, 5, 16, 64, 67):
            r = [sample_range(k, world, spp) for k in range(world)]
            got = [s for first, n in r for s in range(first, first + n)]
            assert got == list(range(spp)), (world, spp, r)
    with pytest.raises(ValueError):
        sample_range(2, 2, 4)


def _split_rank(rank, world, port, out):
    """A rank of the sample-range split: its samples of one frame through the oracle (this rank's stand-in for the
    device's render, which renders the same samples), its accum summed into rank 0's by gloo."""
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import torch
        import oracle
        from threert_b200 import prep, scenes
        from threert_b200.split import reduce_accum, sample_range
        P = prep.prepare(scenes.cornell(24, 16))
        first, k = sample_range(rank, world, 6)
        acc, _ = oracle.Oracle(P).render(P.params, k, first_sample=first, threads=1)
        t = reduce_accum(dist, torch.from_numpy(acc.reshape(-1).copy()))
        if rank == 0:
            out.put(t.numpy())
    finally:
        dist.destroy_process_group()


def test_an_image_split_by_sample_ranges_sums_to_the_one_rank_image():
    """Two ranks render samples [0, 3) and [3, 6) of the same frame; their accums summed on rank 0 are the one-rank
    render of samples [0, 6), up to the order of the sums (the sample counts exactly)."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=_split_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    try:
        got = q.get(timeout=240)
    finally:
        for p in procs:
            p.join(timeout=60)
    assert all(p.exitcode == 0 for p in procs)
    import oracle
    from threert_b200 import prep, scenes
    P = prep.prepare(scenes.cornell(24, 16))
    want, _ = oracle.Oracle(P).render(P.params, 6, threads=1)
    got = got.reshape(want.shape)
    assert np.array_equal(got[:, 3], want[:, 3]) and (want[:, 3] == 6).all()  # sample counts
    assert np.allclose(got, want, rtol=1e-5, atol=1e-6)

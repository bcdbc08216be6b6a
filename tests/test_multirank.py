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

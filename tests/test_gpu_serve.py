"""The serving loop on the device (trt_server_*): requests of different scenes, image sizes, sample counts and
depths batched into shared waves must give each request the accum it gets rendered alone, bit for bit; the server's
ray counts must be the sum of the requests'; what cannot be served is refused at submission."""
import numpy as np
import pytest

from threert_b200 import RenderError, prep, scenes
from threert_b200.prep import params_with
from threert_b200.serve import Request, Server, run_stream

from util import small_city, small_crowd

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def resident(gpu):
    Ps = [prep.prepare(scenes.cornell(48, 48)), prep.prepare(small_city()), prep.prepare(small_crowd(n=60).desc)]
    S = [gpu.upload(P) for P in Ps]
    yield Ps, S
    for s in S:
        s.close()


def the_mix(Ps, seed=3):
    rng = np.random.default_rng(seed)
    sizes = [(16, 16), (40, 24), (64, 36), (48, 48), (33, 17)]
    reqs = []
    for i in range(14):
        k = i % len(Ps)
        w, h = sizes[int(rng.integers(len(sizes)))]
        reqs.append(Request(k, params_with(Ps[k].params, width=w, height=h), int(rng.choice([1, 3, 8]))))
    return reqs


@pytest.mark.parametrize("launch_mode", [0, 1])  # steps replayed from CUDA graphs; launched one by one
@pytest.mark.parametrize("wave_slots", [16384, 1 << 20])  # small: requests spread over steps; large: one step
def test_each_result_is_the_same_alone_and_in_the_mix(gpu, resident, wave_slots, launch_mode):
    Ps, S = resident
    reqs = the_mix(Ps)
    srv = Server(gpu, wave_slots=wave_slots, max_active=8, launch_mode=launch_mode)
    try:
        before = srv.stats()
        res = run_stream(srv, S, reqs, rate=0.0)  # all at once: they share waves
        after = srv.stats()
    finally:
        srv.close()
    assert res["failed"] == 0
    rays = 0
    for r in reqs:
        alone, st = S[r.scene].render_raw(r.params, r.spp)
        assert np.array_equal(r.accum, alone), (r.scene, r.params[16], r.params[17], r.spp)
        rays += st.closest_rays + st.shadow_rays
    assert after["closest_rays"] + after["shadow_rays"] - before["closest_rays"] - before["shadow_rays"] == rays
    if wave_slots == 1 << 20:
        assert res["steps"] < len(reqs)  # several requests a step
    else:
        assert max(r.done["steps"] for r in reqs) > 1  # a request's samples over several steps


def test_requests_that_arrive_during_a_run_join_it(gpu, resident):
    Ps, S = resident
    reqs = the_mix(Ps, seed=5)
    srv = Server(gpu, wave_slots=16384, max_active=4)
    try:
        res = run_stream(srv, S, reqs, rate=400.0)
    finally:
        srv.close()
    assert res["failed"] == 0 and res["requests"] == len(reqs)
    for r in reqs:
        assert np.array_equal(r.accum, S[r.scene].render_raw(r.params, r.spp)[0])


def test_scheduled_arrivals_wait_for_their_time(gpu, resident):
    """trt_server_submit_at: requests handed over at once with arrival times 40 ms apart are started no earlier than
    their arrival (their submit_ms), in arrival order, and give the accum each gets alone."""
    Ps, S = resident
    reqs = the_mix(Ps, seed=9)[:6]
    srv = Server(gpu, wave_slots=16384, max_active=4)
    try:
        t = srv.clock() + 20.0
        at = [t + 40.0 * i for i in range(len(reqs))]
        for r, a in zip(reqs[::-1], at[::-1]):  # handed over last-first: the arrival times set the order
            srv.submit(S[r.scene], r, at_ms=a)
        done = []
        while len(done) < len(reqs):
            done += srv.poll(wait_ms=50)
    finally:
        srv.close()
    for r, a in zip(reqs, at):
        assert r.done["status"] == 0 and r.done["submit_ms"] == a
        assert r.done["start_ms"] >= a, (r.done["start_ms"], a)
        assert np.array_equal(r.accum, S[r.scene].render_raw(r.params, r.spp)[0])
    starts = [r.done["start_ms"] for r in reqs]
    assert starts == sorted(starts)


def test_what_cannot_be_served_is_refused(gpu, resident):
    Ps, S = resident
    srv = Server(gpu, wave_slots=4096)
    try:
        with pytest.raises(RenderError):  # the image needs more path slots than a step holds
            srv.submit(S[0], Request(0, params_with(Ps[0].params, width=128, height=128), 1))
        bad = Ps[0].params.copy()
        bad[124] = 0xFFFFFFF  # a table section past the tables
        with pytest.raises(RenderError):
            srv.submit(S[0], Request(0, bad, 1))
    finally:
        srv.close()


def test_denoised_requests_are_the_denoise_of_their_render_alone(gpu, resident):
    """The serving mix's denoiser (configs: on for spp <= 4): a request submitted for its denoised image gets what the
    learned denoiser makes of the same request rendered alone with its depth guide, bit for bit, beside requests that
    are not denoised; what the network cannot take is refused."""
    from threert_b200 import unet
    from threert_b200 import _native as N
    Ps, S = resident
    net = unet.UNet(0, max_batch=1, max_h=64, max_w=64)
    net.set_params(unet.init_params(11))
    sizes = [(16, 16), (40, 24), (64, 32), (48, 48)]
    reqs = []
    for i in range(10):
        k = i % len(Ps)
        w, h = sizes[i % len(sizes)]
        spp = [1, 2, 4, 8][i % 4]
        reqs.append(Request(k, params_with(Ps[k].params, width=w, height=h), spp, denoise=spp <= 4))
    srv = Server(gpu, wave_slots=16384, max_active=8, denoiser=net)
    try:
        res = run_stream(srv, S, reqs, rate=0.0)
        with pytest.raises(RenderError):  # more samples than the server denoises
            srv.submit(S[0], Request(0, params_with(Ps[0].params, width=16, height=16), 8, denoise=True))
        with pytest.raises(RenderError):  # not a multiple of 8
            srv.submit(S[0], Request(0, params_with(Ps[0].params, width=20, height=16), 1, denoise=True))
    finally:
        srv.close()
    assert res["failed"] == 0
    for r in reqs:
        w, h = int(r.params[16]), int(r.params[17])
        if r.denoise:
            S[r.scene].render_raw(r.params, r.spp, flags=N.TRT_RENDER_DEPTH, read=False)
            alone, _ = net.denoise(S[r.scene])
            assert r.accum is None and np.array_equal(r.rgb.reshape(h, w, 3), alone), (r.scene, w, h, r.spp)
        else:
            assert np.array_equal(r.accum, S[r.scene].render_raw(r.params, r.spp)[0])
    net.close()


def test_a_720p_frame_rendered_in_two_half_waves_is_the_servers_one_wave(gpu, resident):
    """trt_render runs a wave of 2^19 paths or more as two half-waves (each with its first pixel index); the server
    renders the same request in one wave. Both give the same accum, bit for bit: a path's pixel, sample and random
    numbers do not depend on which half-wave it is in."""
    Ps, S = resident
    params = params_with(Ps[1].params, width=1280, height=720)
    alone, _ = S[1].render_raw(params, 1)  # 921,600 paths: two half-waves
    srv = Server(gpu, wave_slots=1 << 21)
    try:
        r = Request(1, params, 1)
        res = run_stream(srv, S, [r], rate=0.0)
    finally:
        srv.close()
    assert res["failed"] == 0
    assert np.array_equal(r.accum, alone)

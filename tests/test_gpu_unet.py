"""The learned denoiser's network on the device against its CPU oracle (oracle/unet_ref.py, itself pinned by finite
differences): outputs and every layer's gradients within bf16's rounding; training fits a batch; inference on a
scene's accum on the device equals the host-side feature path."""
import numpy as np
import pytest

from oracle import unet_ref as R
from threert_b200 import prep, unet
from threert_b200 import _native as N

from util import small_city

pytestmark = pytest.mark.gpu


def bf16(a):
    """Round to bfloat16 (nearest even), as the device stores weights and inputs."""
    u = np.asarray(a, np.float32).view(np.uint32).astype(np.uint64)
    u = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return u.astype(np.uint32).view(np.float32)


def case(seed=3, b=2, h=16, w=16):
    rng = np.random.default_rng(seed)
    p = unet.init_params(seed)
    o = 0
    for cin, cout in unet.LAYERS:
        o += 9 * cin * unet.r64(cout)
        p[o:o + cout] = rng.normal(0, 0.05, cout)
        o += unet.r64(cout)
    feats = rng.normal(0, 1, (b, h, w, unet.N_FEAT)).astype(np.float32)
    tgt = rng.normal(0, 1, (b, h, w, 3)).astype(np.float32)
    return p, feats, tgt


@pytest.fixture(scope="module")
def net():
    n = unet.UNet(0, max_batch=4, max_h=64, max_w=80)
    yield n
    n.close()


def test_forward_matches_the_oracle(net):
    p, feats, _ = case()
    net.set_params(p)
    got, ms = net.forward(feats)
    want, _ = R.forward(R.unpack(bf16(p).astype(np.float64)), bf16(feats).astype(np.float64))
    err = np.linalg.norm(got - want) / np.linalg.norm(want)
    assert err < 0.03, err
    assert ms > 0


def test_forward_matches_the_oracle_rounding_as_the_device_does(net):
    """With the oracle's activations stored as bf16 where the device stores them (each hidden layer's output, each
    pooling's), what is left between the two is the f32 accumulation against float64, and the bf16 roundings it tips
    the other way: 1e-2 relative over the image (measured 4.3e-3), and no output off by more than 2 % of the output's
    scale (measured 5.1e-3)."""
    for seed, (b, h, w) in ((3, (2, 16, 16)), (11, (1, 40, 72))):
        p, feats, _ = case(seed=seed, b=b, h=h, w=w)
        net.set_params(p)
        got, _ = net.forward(feats)
        want, _ = R.forward(R.unpack(bf16(p).astype(np.float64)), bf16(feats).astype(np.float64), act=R.bf16_round)
        err = np.linalg.norm(got - want) / np.linalg.norm(want)
        worst = np.abs(got - want).max() / np.abs(want).max()
        print(f"forward {b}x{h}x{w}: relative error {err:.2e}, worst output {worst:.2e}")
        assert err < 1e-2 and worst < 0.02, (err, worst)


def test_forward_on_ragged_tiles_matches_the_oracle(net):
    # 72 x 40: tiles of 8 x 16 pixels at the top level (the last row of tiles half outside the image), 4 x 32,
    # 2 x 64, then 1 x 128 over a 9 x 5 level
    p, feats, _ = case(seed=4, b=1, h=40, w=72)
    net.set_params(p)
    got, _ = net.forward(feats)
    want, _ = R.forward(R.unpack(bf16(p).astype(np.float64)), bf16(feats).astype(np.float64))
    err = np.linalg.norm(got - want) / np.linalg.norm(want)
    assert err < 0.03, err


def test_forward_on_wide_rows_matches_the_oracle():
    # 256 x 24: tiles of 128 x 1 pixels at the two widest levels (a tile a row, its halo rows above and below read by
    # the shifted TMA boxes), 64 x 2 and 32 x 4 below
    wide = unet.UNet(0, max_batch=1, max_h=24, max_w=256)
    p, feats, _ = case(seed=6, b=1, h=24, w=256)
    wide.set_params(p)
    got, _ = wide.forward(feats)
    want, _ = R.forward(R.unpack(bf16(p).astype(np.float64)), bf16(feats).astype(np.float64))
    err = np.linalg.norm(got - want) / np.linalg.norm(want)
    assert err < 0.03, err
    wide.close()


def test_halo_row_tiles_match_the_oracle():
    """Images at least 128 wide: a layer of one output tile whose weights fit in shared memory (up to four 32-channel
    blocks at 64 outputs, two at 128) runs the halo kernel on every level at least 128 wide, a row tile of 128 pixels
    read once a block with its halo and the nine taps as shifted descriptors into it: at 256 the full-resolution
    layers (one and three blocks) and the second level's 32 -> 64 and 64 -> 64; at 512 also the third level's
    64 -> 96 (two blocks, 128 outputs); at 1000 the last tile of each row is ragged on three levels (104, 116 and 122
    of its 128 pixels inside the image). The
    forward as tight as the 2-D tiles' (activations rounded to bf16 where the device stores them), and every layer's
    gradient, whose input gradient runs the same kernel with the flipped weights."""
    wide = unet.UNet(0, max_batch=1, max_h=24, max_w=1000)
    try:
        for seed, h, w in ((12, 16, 1000), (13, 24, 256), (14, 16, 512)):
            p, feats, tgt = case(seed=seed, b=1, h=h, w=w)
            wide.set_params(p)
            got, _ = wide.forward(feats)
            want, _ = R.forward(R.unpack(bf16(p).astype(np.float64)), bf16(feats).astype(np.float64), act=R.bf16_round)
            err = np.linalg.norm(got - want) / np.linalg.norm(want)
            worst = np.abs(got - want).max() / np.abs(want).max()
            print(f"halo forward 1x{h}x{w}: relative error {err:.2e}, worst output {worst:.2e}")
            assert err < 1e-2 and worst < 0.02, (w, err, worst)
            loss, g, _ = wide.step(feats, tgt, update=False, grads=True)
            ref_loss, G, _ = R.loss_and_grads(R.unpack(bf16(p).astype(np.float64)), bf16(feats).astype(np.float64), tgt)
            assert abs(loss / ref_loss - 1) < 0.02
            gp = R.unpack(g.astype(np.float64))
            for name in R.NAMES:
                for k in range(2):
                    a, b = gp[name][k].ravel(), G[name][k].ravel()
                    cos = a @ b / (np.linalg.norm(a) * np.linalg.norm(b) + 1e-30)
                    ratio = np.linalg.norm(a) / (np.linalg.norm(b) + 1e-30)
                    assert cos > 0.98 and abs(ratio - 1) < 0.1, (w, name, k, cos, ratio)
    finally:
        wide.close()


@pytest.mark.parametrize("b,h,w", [(2, 16, 16), (4, 64, 64)])
def test_every_layers_gradient_matches_the_oracle(net, b, h, w):
    # 2 x 16 x 16: a 128-pixel tile a CTA; 4 x 64 x 64: the weight gradient's CTAs take runs of two to six tiles at
    # the two top levels (the accumulator summed over stages, the pipeline's stages reused)
    p, feats, tgt = case(seed=5, b=b, h=h, w=w)
    net.set_params(p)
    loss, g, _ = net.step(feats, tgt, update=False, grads=True)
    ref_loss, G, _ = R.loss_and_grads(R.unpack(bf16(p).astype(np.float64)), bf16(feats).astype(np.float64), tgt)
    assert abs(loss / ref_loss - 1) < 0.02
    gp = R.unpack(g.astype(np.float64))
    for name in R.NAMES:
        for k in range(2):  # weights, bias
            a, b = gp[name][k].ravel(), G[name][k].ravel()
            cos = a @ b / (np.linalg.norm(a) * np.linalg.norm(b) + 1e-30)
            ratio = np.linalg.norm(a) / (np.linalg.norm(b) + 1e-30)
            assert cos > 0.98 and abs(ratio - 1) < 0.1, (name, k, cos, ratio)
    # the padding's gradients are zero
    flat = R.pack(gp, g)
    assert np.allclose(g[flat == 0], 0.0)


def test_gradients_are_the_same_every_step(net):
    # the weight gradient's CTA partials are summed in a fixed order: no dependence on the CTAs' timing
    p, feats, tgt = case(seed=10, b=4, h=64, w=64)
    net.set_params(p)
    _, g1, _ = net.step(feats, tgt, update=False, grads=True)
    _, g2, _ = net.step(feats, tgt, update=False, grads=True)
    assert np.array_equal(g1, g2)


def test_training_fits_a_batch(net):
    p, feats, _ = case(seed=7, b=4, h=32, w=32)
    rng = np.random.default_rng(8)
    tgt = (0.5 * feats[..., 0:3] + 0.3 * rng.normal(0, 1, feats[..., 0:3].shape)).astype(np.float32)
    net.set_params(p)
    first, _, _ = net.step(feats, tgt, lr=1e-3)
    for _ in range(150):
        last, _, _ = net.step(feats, tgt, lr=1e-3)
    assert last < 0.6 * first, (first, last)


def test_inference_on_the_device_is_the_host_path(gpu, net):
    P = prep.prepare(small_city(width=64, height=32))
    S = gpu.upload(P)
    acc, _ = S.render_raw(P.params, 2, flags=N.TRT_RENDER_DEPTH)
    p, _, _ = case(seed=9)
    net.set_params(p)
    got, ms = net.denoise(S)
    f, s = unet.features(acc, 64, 32)
    pred, _ = net.forward(f[None])
    want = unet.radiance(pred[0], s)
    assert ms > 0
    assert np.linalg.norm(got - want) / np.linalg.norm(want) < 0.02
    S.close()


@pytest.mark.parametrize("h,w", [(64, 64), (32, 256)])  # the first layer on 2-D tiles; on halo row tiles
def test_a_withheld_copy_ends_the_forward_with_an_error_and_the_network_stays_usable(h, w):
    """The convolution's pipeline waits are bounded (about a second): a copy that never lands (one activation stage
    withheld by trt_unet_hold_next_load) ends its wait, the call reports it (TRT_ECUDA, "gave up") instead of hanging,
    and the next forward on the same network gives the same output as before."""
    from threert_b200 import RenderError
    n = unet.UNet(0, max_batch=1, max_h=h, max_w=w)
    try:
        n.set_params(unet.init_params(3))
        f = np.random.default_rng(9).normal(0, 1, (1, h, w, unet.N_FEAT)).astype(np.float32)
        want, _ = n.forward(f)
        n.hold_next_load()
        with pytest.raises(RenderError, match="gave up"):
            n.forward(f)
        got, _ = n.forward(f)
        assert np.array_equal(got, want)
    finally:
        n.close()

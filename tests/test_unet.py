"""The learned warm start's network: the CPU restatement (oracle/unet_ref.py)
checked against finite differences, and the CUDA tensor-core forward and
backward passes checked against it."""
import numpy as np
import pytest

from bevy_eulerian_fluid_b200 import _capi as capi
from oracle import unet_ref


def _random_case(seed, n=32, head_scale=0.05, nx=None):
    nx = n if nx is None else nx
    rng = np.random.default_rng(seed)
    params = []
    for ci, co, relu in unet_ref.SPEC:
        std = np.sqrt(2.0 / (9 * ci)) if relu else head_scale
        params.append(rng.normal(0, std, 9 * ci * co))
        params.append(rng.normal(0, 0.05, co))
    params = np.concatenate(params).astype(np.float32)
    feats = np.zeros((n, nx, 16), np.float32)
    feats[:, :, :5] = rng.normal(0, 1, (n, nx, 5))
    target = rng.normal(0, 0.1, (n, nx)).astype(np.float32)
    mask = (rng.random((n, nx)) < 0.7).astype(np.uint8)
    return params, feats, target, mask


def test_oracle_backward_matches_finite_differences():
    params, feats, target, mask = _random_case(1, n=16)
    params = params.astype(np.float64)
    net = unet_ref.Net(params, rounding=False)
    net.forward(feats.astype(np.float64))
    _, g = net.backward(target, mask)
    rng = np.random.default_rng(2)
    off = 0
    for ci, co, _ in unet_ref.SPEC:  # one random direction within each layer's parameters
        n = 9 * ci * co + co
        v = np.zeros_like(params)
        v[off:off + n] = rng.normal(0, 1, n)
        off += n
        eps = 1e-6
        lp = unet_ref.Net(params + eps * v, rounding=False)
        lp.forward(feats.astype(np.float64))
        lm = unet_ref.Net(params - eps * v, rounding=False)
        lm.forward(feats.astype(np.float64))
        fp, _ = lp.backward(target, mask)
        fm, _ = lm.backward(target, mask)
        fd = (fp - fm) / (2 * eps)
        assert fd == pytest.approx(float(g @ v), rel=1e-5, abs=1e-10)


def test_oracle_bf16_rounding():
    x = np.array([1.0, 1.00390625, 1.005859375, -3.14159, 0.0], np.float32)
    r = unet_ref.bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0  # a tie rounds to even
    assert r[2] == np.float32(1.0078125)
    assert abs(r[3] - (-3.140625)) < 1e-6 and r[4] == 0.0


def _rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / max(1e-30, np.linalg.norm(b)))


@pytest.mark.gpu
def test_unet_forward_matches_oracle(gpu_api):
    params, feats, target, mask = _random_case(3)
    net = capi.UNet(gpu_api, 64, 64, seed=5)
    net.set_params(params)
    assert np.array_equal(net.get_params(), params)
    pred = net.forward(feats)
    ref = unet_ref.Net(params).forward(feats)
    assert _rel(pred, ref) < 2e-3  # 1.6e-4 measured


@pytest.mark.gpu
def test_unet_wide_rows_match_oracle(gpu_api):
    """At 128 x 512, forward and backward: the 512-wide level runs the row-tile
    convolution with two stretches per CTA and the weight ring (512 tiles),
    the 256- and 128-wide ones with resident weights, or the ring where nine
    tiles do not fit (128 -> 64 channels), and the 64-wide one the multistage
    kernel; all agree with the oracle."""
    params, feats, target, mask = _random_case(6, n=128, nx=512)
    net = capi.UNet(gpu_api, 512, 128, seed=5)
    net.set_params(params)
    ref = unet_ref.Net(params)
    assert _rel(net.forward(feats), ref.forward(feats)) < 1e-2  # 3.1e-3 measured
    loss, g = net.gradients(feats, target, mask)
    rloss, rg = ref.backward(target, mask)
    assert loss == pytest.approx(rloss, rel=1e-4)  # 6.9e-6 measured
    cos = float(g.astype(np.float64) @ rg / (np.linalg.norm(g) * np.linalg.norm(rg)))
    assert cos > 0.9999 and _rel(g, rg) < 5e-3, (cos, _rel(g, rg))  # 1 - 7e-8 and 7.6e-4 measured


@pytest.mark.gpu
def test_unet_forward_512_matches_oracle(gpu_api):
    """At 512 x 512 the row-tile convolution covers two stretches per CTA and
    streams its weights through the ring at the 512- and 256-wide levels
    (1024 and 256 CTAs), and keeps them resident at the 128-wide one (128
    tiles); the forward agrees with the oracle."""
    params, feats, _, _ = _random_case(8, n=512)
    net = capi.UNet(gpu_api, 512, 512, seed=5)
    net.set_params(params)
    assert _rel(net.forward(feats), unet_ref.Net(params).forward(feats)) < 1e-2


@pytest.mark.gpu
@pytest.mark.parametrize("seed", [4, 9, 11])
def test_unet_gradients_match_oracle(gpu_api, seed):
    """Every layer's weight and bias gradients agree with the oracle's: cosine
    similarity above 0.998 and relative L2 error below 6 %.  (The tensor cores
    accumulate in another order than the CPU; near-zero pre-activations then
    flip a ReLU or a bf16 rounding now and then, and the flip propagates to the
    deep layers' gradients -- by up to a few percent, as it does between two
    CPU accumulation orders.  Many cases agree to 1e-4.)"""
    params, feats, target, mask = _random_case(seed)
    net = capi.UNet(gpu_api, 64, 64)
    net.set_params(params)
    loss, g = net.gradients(feats, target, mask)
    ref = unet_ref.Net(params)
    ref.forward(feats)
    rloss, rg = ref.backward(target, mask)
    assert loss == pytest.approx(rloss, rel=2e-3)  # at most 2.6e-4 measured
    off = 0
    for i, (ci, co, _) in enumerate(unet_ref.SPEC):
        nw = 9 * ci * co
        for name, n in (("w", nw), ("b", co)):
            seg, rseg = g[off:off + n].astype(np.float64), rg[off:off + n]
            off += n
            cos = float(seg @ rseg / max(1e-300, np.linalg.norm(seg) * np.linalg.norm(rseg)))
            assert cos > 0.998 and _rel(seg, rseg) < 6e-2, (i, name, cos, _rel(seg, rseg))


@pytest.mark.gpu
def test_unet_training_reduces_loss(gpu_api):
    """Adam on the GPU fits a fixed sample recorded from a simulation."""
    from bevy_eulerian_fluid_b200 import scenes
    sc = scenes.coupled(64, tolerance=1e-5, n_per_shape=1)
    sim = sc.make(gpu_api)
    net = capi.UNet(gpu_api, 64, 64, seed=7)
    net.attach(sim, warm_start=False, record=True)
    sim.step(sc.dt)
    sim.step(sc.dt)
    losses = [net.train_step(1e-3) for _ in range(60)]
    assert losses[-1] < 0.5 * losses[0]


@pytest.mark.gpu
def test_learned_warm_start_gain(gpu_api):
    """What the trained network gains: after a short training on C2-style
    scenes (seeds 1-8, 256^2), the initial relative residual of the benchmark
    scene's solves falls clearly below that of the previous-pressure start,
    and every solve still reaches the tolerance.  (The iteration counts of
    RBGS barely move: they are set by the slowest, long-wavelength error
    modes, which a 4-level network's receptive field does not reach.)"""
    from bevy_eulerian_fluid_b200 import learned, scenes
    net, log = learned.train(gpu_api, size=256, seeds=tuple(range(1, 9)), steps=100, lr=1e-3)
    out = learned.compare(gpu_api, net, scenes.coupled(256), warmup=5, steps=4)
    r_l = np.mean([x[1] for x in out["learned"]])
    r_p = np.mean([x[1] for x in out["plain"]])
    assert r_l < 0.8 * r_p, (r_l, r_p)
    assert all(x[3] for x in out["learned"] + out["plain"])


@pytest.mark.gpu
def test_pretrained_warm_start_saves_iterations(gpu_api):
    """What the trained network gains, in iterations: the committed network (run on the grid coarsened 8x,
    trained offline on seeds other than the benchmark's) warm-starts the benchmark scene coupled_512.  From the
    same states, the warm-started RBGS solves reach the same 1e-5 in at least a third fewer iterations in total
    than solves started from the previous pressure, and every one converges."""
    from bevy_eulerian_fluid_b200 import learned, scenes
    net = learned.load_weights(gpu_api, 512, 512)
    assert net is not None, "the pretrained weights file is missing"
    out = learned.compare(gpu_api, net, scenes.coupled(512), warmup=5, steps=3)
    it_l = sum(x[0] for x in out["learned"])
    it_p = sum(x[0] for x in out["plain"])
    assert all(x[3] for x in out["learned"] + out["plain"])
    assert it_l < 0.67 * it_p, (it_l, it_p)
    net.close()


@pytest.mark.gpu
def test_prediction_judged_against_fp64_solve(gpu_api):
    """The warm start's error stated against an FP64 CPU solve of the same Poisson system (a sparse direct solve
    of the operator of residual.wgsl:33-54): the start iterate is closer to that solution than the previous
    pressure, and supplies most of the correction's block means (the part the sweeps remove slowest)."""
    from bevy_eulerian_fluid_b200 import learned, scenes
    net = learned.load_weights(gpu_api, 512, 512)
    pe = learned.prediction_error(gpu_api, net, scenes.coupled(512), warmup=5)
    assert pe["relative_error_start"] < pe["relative_error_previous"], pe
    assert pe["captured_block_means"] > 0.5, pe
    net.close()


def test_canvas_forward_equals_per_image_forwards():
    """The batch's canvas (efl_canvas_pack's layout, 8-pixel gaps): a forward over the canvas whose convolutions
    write zeros at the gap pixels (all but the head) gives, inside each rectangle, each image's own forward --
    here with the CPU restatement, so the gap rule itself is checked (the GPU test compares the batched
    simulations with their own steps)."""
    rng = np.random.default_rng(12)
    params, _, _, _ = _random_case(2, n=16)
    sizes = [(16, 16), (32, 16), (16, 32), (48, 32), (24, 8)]  # (w, h), multiples of 8
    org, W, H = capi.canvas_pack(capi.load(), sizes)
    masks = []
    for lvl in range(4):
        m = np.zeros((H >> lvl, W >> lvl), bool)
        for (x, y), (w, h) in zip(org, sizes):
            m[y >> lvl:(y + h) >> lvl, x >> lvl:(x + w) >> lvl] = True
        masks.append(m)

    class CanvasNet(unet_ref.Net):
        def _c(self, i, x):
            y = super()._c(i, x)
            if i == len(unet_ref.SPEC) - 1:
                return y
            lvl = int(round(np.log2(H / y.shape[0])))
            return y * masks[lvl][:, :, None]

    feats = np.zeros((H, W, 16), np.float32)
    single = []
    for (x, y), (w, h) in zip(org, sizes):
        f = np.zeros((h, w, 16), np.float32)
        f[:, :, :5] = rng.normal(0, 1, (h, w, 5))
        feats[y:y + h, x:x + w] = f
        single.append(unet_ref.Net(params).forward(f))
    out = CanvasNet(params).forward(feats)
    for (x, y), (w, h), ref in zip(org, sizes, single):
        np.testing.assert_allclose(out[y:y + h, x:x + w], ref, rtol=1e-6, atol=1e-9)

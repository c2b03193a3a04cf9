"""The learned proposal's device kernels against the CPU oracle (oracle/mlp_ref.py):
the tcgen05 GEMM over tile-edge shapes, the network forward, the gradients of one
training step, the Adam update, a training run, and the patch features against a
numpy restatement from the residual planes and projections."""
import numpy as np
import pytest

from oracle import mlp_ref as R
from pyopenlpt_b200 import _ffi, synth
from tests import _scenes

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = _ffi.Context(0)
    yield c
    c.close()


def _bf(rng, shape, s=1.0):
    return R.bf16(rng.normal(0, s, shape).astype(np.float32))


@pytest.mark.parametrize("M,N,K", [(1, 16, 16), (127, 256, 64), (128, 128, 64), (300, 300, 100),
                                   (1000, 256, 493), (19000, 256, 64), (256, 512, 2048)])
def test_gemm_matches_numpy(ctx, M, N, K):
    rng = np.random.default_rng(M * 7 + N * 3 + K)
    a, b = _bf(rng, (M, K)), _bf(rng, (N, K))
    bias = rng.normal(0, 1, N).astype(np.float32)
    got = ctx.bf16_gemm(R.bf16_bits(a), R.bf16_bits(b), bias)
    a64, b64 = a.astype(np.float64), b.astype(np.float64)
    want = a64 @ b64.T + bias
    bound = np.abs(a64) @ np.abs(b64).T + np.abs(bias)  # f32 accumulation-order bound
    assert np.all(np.abs(got - want) <= 1e-5 * bound + 1e-6)
    if M == 300:
        g = ctx.bf16_gemm(R.bf16_bits(a), R.bf16_bits(b), bias, gelu=True)
        assert np.allclose(g, R.gelu(want), rtol=1e-4, atol=1e-4)


def _features(rng, n):
    x = np.zeros((n, R.IN), np.float32)
    x[:, :484] = np.clip(rng.normal(0.2, 0.3, (n, 484)), 0, None)
    x[:, 484:492] = rng.uniform(-0.5, 0.5, (n, 8))
    x[:, 492] = 1.0
    return x


def _targets(rng, n):
    t = rng.normal(0, 1, (n, 4)).astype(np.float32)
    t[:, 3] = (rng.random(n) < 0.3).astype(np.float32)
    return t


def test_forward_matches_oracle(ctx):
    rng = np.random.default_rng(1)
    flat = R.init(3)
    flat[R.N_PARAMS - 4:] = [0.1, -0.2, 0.3, -0.5]
    ctx.mlp_set_params(flat)
    x = _features(rng, 1000)
    got = ctx.mlp_forward(x)
    want, _ = R.forward(flat, x)
    d = np.abs(got - want)
    print("forward |diff| max", d.max(), "mean", d.mean(), "output scale", np.abs(want).max())
    assert d.max() < 3e-2 and d.mean() < 3e-3


def test_gradients_match_oracle(ctx):
    rng = np.random.default_rng(2)
    flat = R.init(4)
    ctx.mlp_set_params(flat)
    x, t = _features(rng, 700), _targets(rng, 700)
    loss, g = ctx.mlp_train_step(x, t, lr=0.0, ghost_weight=0.7, update=False, want_grad=True)
    loss_ref, g_ref = R.backward(flat, x, t, 0.7)
    assert abs(loss - loss_ref) <= 2e-3 * abs(loss_ref)
    off = 0
    for name, shp in R.SHAPES:
        k = int(np.prod(shp))
        a, b = g[off:off + k], g_ref[off:off + k]
        rel = np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-12)
        print(f"grad {name}: rel err {rel:.2e}")
        assert rel < 2e-2, name
        off += k
    # parameters untouched without update
    assert np.array_equal(ctx.mlp_get_params(), flat)


def test_adam_update_matches_oracle(ctx):
    rng = np.random.default_rng(5)
    flat = R.init(6)
    ctx.mlp_set_params(flat)
    x, t = _features(rng, 256), _targets(rng, 256)
    _, g = ctx.mlp_train_step(x, t, lr=1e-3, update=True, want_grad=True)
    want, _, _ = R.adam(flat.astype(np.float64), g.astype(np.float64), 0.0, 0.0, 1, 1e-3)
    got = ctx.mlp_get_params()
    assert np.abs(got - want).max() < 1e-6


def test_training_fits_a_smooth_target(ctx):
    """The forward + backward + Adam loop learns a fixed smooth map of the inputs."""
    rng = np.random.default_rng(7)
    ctx.mlp_init(11)
    P = rng.normal(0, 1, (R.IN, 3)).astype(np.float32) / np.sqrt(R.IN)
    xs = _features(rng, 8192)
    ts = np.zeros((len(xs), 4), np.float32)
    ts[:, :3] = np.tanh(xs @ P * 3)
    ts[:, 3] = (xs[:, 484] > 0.2).astype(np.float32)
    first = ctx.mlp_train_step(xs[:1024], ts[:1024], lr=0.0, update=False)
    for it in range(300):
        i = (it % 8) * 1024
        ctx.mlp_train_step(xs[i:i + 1024], ts[i:i + 1024], lr=2e-3)
    last = ctx.mlp_train_step(xs[:1024], ts[:1024], lr=0.0, update=False)
    print("loss", first, "->", last)
    assert last < 0.35 * first


def _round_half_away(v):
    return np.where(v >= 0, np.floor(v + 0.5), -np.floor(-v + 0.5))


def _roi(H, W, cx, cy, r):
    # Shake::calROIBound restated (empty rect -> None)
    if cx <= 0 or cy <= 0 or cx >= W or cy >= H:
        return None
    w = int(_round_half_away(2 * r))
    cmin = int(_round_half_away(cx - (w - 1) / 2.0))
    rmin = int(_round_half_away(cy - (w - 1) / 2.0))
    cmax, rmax = cmin + w, rmin + w
    return max(rmin, 0), min(rmax, H), max(cmin, 0), min(cmax, W)


@pytest.mark.parametrize("kind", ["small", "poly"])
def test_features_match_restatement(ctx, kind):
    """4 pinhole cameras with a uniform OTF, and 6 polynomial cameras with a 5x5x5 OTF."""
    sc = _scenes.scene(kind)
    s = _scenes.settings(kind)
    g = _scenes.gpu_context(sc)
    n_c = sc.n_cam
    base, one = 121 * n_c, 121 * n_c + 2 * n_c
    try:
        g.upload_images(sc.images)
        rng = np.random.default_rng(3)
        xyz = sc.xyz[:300] + rng.normal(0, 0.03 if kind == "small" else 0.01, (300, 3))
        g.upload_objects(xyz)
        sp = _ffi.shake_params(s, precision=0)
        feats = g.mlp_features(sp)
        objs = g.objects()
        H, W = sc.images[0].shape
        res = [g.residual_image(c, (H, W), np.float32) for c in range(sc.n_cam)]
        otf = [g.otf_param(c, xyz) for c in range(sc.n_cam)]
        want = np.zeros_like(feats)
        for o in range(len(xyz)):
            for c in range(sc.n_cam):
                u, v = objs["uv"][o, c]
                q = otf[c][o].astype(np.float32)
                ru, rv = _round_half_away(u), _round_half_away(v)
                pr = _roi(H, W, u, v, s.radius_obj)
                for t in range(121):
                    row, col = int(rv) + t // 11 - 5, int(ru) + t % 11 - 5
                    val = np.float32(0)
                    if 0 <= row < H and 0 <= col < W:
                        val = res[c][row, col]
                        if pr and pr[0] <= row < pr[1] and pr[2] <= col < pr[3]:
                            dx, dy = np.float32(col - u), np.float32(row - v)
                            xx, yy = dx * q[3] + dy * q[4], -dx * q[4] + dy * q[3]
                            p = q[0] * np.exp(-(q[1] * xx * xx + q[2] * yy * yy))
                            val = val + max(p, np.float32(0))
                        val = val / max(q[0], np.float32(1e-6)) if val > 0 else np.float32(0)
                    want[o, c * 121 + t] = val
                want[o, base + 2 * c] = u - ru
                want[o, base + 1 + 2 * c] = v - rv
            want[o, one] = 1.0
        assert feats.shape == (len(xyz), one + 1)
        d = np.abs(feats - want)
        print(f"{kind} features |diff| max", d.max())
        assert d.max() < 1e-4
        assert feats[:, :base].max() > 0.5  # the particles are in the patches
    finally:
        g.close()


def test_resident_dataset_training(ctx):
    """olpt_mlp_train: the dataset copied once, mini-batches sampled on the device."""
    rng = np.random.default_rng(8)
    ctx.mlp_init(12)
    P = rng.normal(0, 1, (R.IN, 3)).astype(np.float32) / np.sqrt(R.IN)
    xs = _features(rng, 20000)
    ts = np.zeros((len(xs), 4), np.float32)
    ts[:, :3] = np.tanh(xs @ P * 3)
    ts[:, 3] = (xs[:, 484] > 0.2).astype(np.float32)
    losses = ctx.mlp_train(xs, ts, steps=400, batch=2048, lr=2e-3, seed=3)
    assert len(losses) == 400 and np.all(np.isfinite(losses))
    first = ctx.mlp_train_step(xs[:2048], ts[:2048], lr=0.0, update=False)
    print("resident-dataset training: loss", losses[0], "->", np.mean(losses[-20:]), "eval", first)
    assert np.mean(losses[-20:]) < 0.35 * losses[0]


def test_six_camera_network_matches_oracle():
    """The network of a 6-camera rig (n_in = 739, padded to 768): forward and the
    gradients of one training step against the oracle."""
    sc = _scenes.scene("poly")
    g = _scenes.gpu_context(sc)
    try:
        n_in, n_params = g.mlp_dims()
        assert (n_in, n_params) == (R.n_in(6), 256 * R.n_in(6) + 256 * 3 + 2 * 256 * 256 + 4 * 256 + 4)
        rng = np.random.default_rng(21)
        flat = R.init(9, n_in)
        g.mlp_set_params(flat)
        x = np.zeros((900, n_in), np.float32)
        x[:, :726] = np.clip(rng.normal(0.2, 0.3, (900, 726)), 0, None)
        x[:, 726:738] = rng.uniform(-0.5, 0.5, (900, 12))
        x[:, 738] = 1.0
        got = g.mlp_forward(x)
        want, _ = R.forward(flat, x)
        d = np.abs(got - want)
        print("6-camera forward |diff| max", d.max(), "mean", d.mean())
        assert d.max() < 3e-2 and d.mean() < 3e-3
        t = _targets(rng, 900)
        loss, gr = g.mlp_train_step(x, t, lr=0.0, update=False, want_grad=True)
        loss_ref, g_ref = R.backward(flat, x, t, 1.0)
        assert abs(loss - loss_ref) <= 2e-3 * abs(loss_ref)
        off = 0
        for name, shp in R.shapes(n_in):
            k = int(np.prod(shp))
            a, b = gr[off:off + k], g_ref[off:off + k]
            rel = np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-12)
            print(f"6-camera grad {name}: rel err {rel:.2e}")
            assert rel < 2e-2, name
            off += k
    finally:
        g.close()

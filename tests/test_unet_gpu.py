"""The learned warm start's BF16 U-Net on the GPU against its float64 torch-CPU
oracle (oracle/unet.py), through the C-ABI.

Tolerances (relative L2): with random weights, the forward pass within 1e-2 of
the oracle that rounds to BF16 where the network stores BF16, the loss within
1e-2 and every layer's weight gradient within 1e-1 (FP32-versus-FP64
accumulation moves values across BF16 rounding boundaries, and 18 layers
amplify those flips); with integer weights and data, where every sum is exact
(test_gradients_exact_arithmetic), the forward within 1e-6 and every layer's
weight and bias gradient within 1e-5."""
import numpy as np
import pytest

from oracle import unet as U

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx(pkg):
    c = pkg.Context(0)
    yield c
    c.close()


def rel(a, b):
    return float(np.linalg.norm(np.ravel(a) - np.ravel(b)) / np.linalg.norm(np.ravel(b)))


def data(B, H, W, seed):
    rng = np.random.default_rng(seed)
    x = rng.standard_normal((B, 2, H * W)).astype(np.float32)
    t = (0.5 * x + 0.1 * rng.standard_normal(x.shape)).astype(np.float32)
    return x, t


def test_param_count_and_roundtrip(pkg, ctx):
    net = pkg.UNet(ctx, 1, 16, 16, seed=3)
    try:
        assert net.num_params() == U.n_params()
        p = net.get_params()
        q = p.copy()
        q[::7] += 0.25
        net.set_params(q)
        assert np.array_equal(net.get_params(), q)
    finally:
        net.close()


def test_forward_matches_oracle(pkg, ctx):
    B, H, W = 2, 32, 48
    net = pkg.UNet(ctx, B, H, W, seed=11)
    p = net.get_params()
    x, _ = data(B, H, W, 1)
    y = net.forward(x, np.zeros_like(x))
    want, _ = U.forward(p, x, H, W, emulate_bf16=True)
    exact, _ = U.forward(p, x, H, W, emulate_bf16=False)
    net.close()
    e, e64 = rel(y, want.detach().numpy()), rel(y, exact.detach().numpy())
    print(f"forward vs BF16-emulating oracle {e:.2e}, vs float64 oracle {e64:.2e}")
    assert e < 1e-2


def test_gradients_match_oracle(pkg, ctx):
    B, H, W = 2, 32, 32
    net = pkg.UNet(ctx, B, H, W, seed=12)
    p = net.get_params()
    x, t = data(B, H, W, 2)
    loss, g = net.gradients(x, t)
    loss_o, g_o = U.loss_and_grads(p, x, t, H, W, emulate_bf16=True)
    assert abs(loss - loss_o) / loss_o < 1e-2
    worst, errs = 0.0, []
    for i, (a, b) in enumerate(U.layer_slices()):
        ref = g_o[a:b]
        if i == 0:  # only the two real input channels of the first layer carry gradient
            ref = ref.reshape(32, 9, 16)[:, :, :2]
            got = g[a:b].reshape(32, 9, 16)[:, :, :2]
        elif i == len(U.CFG) - 1:  # only outputs 0 and 1 of the last layer
            ref = ref.reshape(16, 32)[:2]
            got = g[a:b].reshape(16, 32)[:2]
        else:
            got = g[a:b]
        e = rel(got, ref)
        worst = max(worst, e)
        errs.append(e)
    net.close()
    print(f"loss {loss:.6f} vs {loss_o:.6f}; layer weight-gradient errors "
          + " ".join(f"{e:.1e}" for e in errs))
    assert worst < 1e-1


def exact_params(seed):
    """Weights in {-1, 0, +1} (each tap non-zero with probability ~2 / fan-in,
    so activations neither die out nor grow past 2^24), biases in {-1, 0, 1}."""
    rng = np.random.default_rng(seed)
    parts = []
    for i, (ci, co, k, _) in enumerate(U.CFG):
        fan = k * k * (2 if i == 0 else ci)
        q = min(1.0, 2.5 / fan)
        w = rng.choice([-1.0, 0.0, 1.0], size=co * k * k * ci, p=[q / 2, 1 - q, q / 2])
        parts += [w, rng.integers(-1, 2, co).astype(np.float64)]
    return np.concatenate(parts).astype(np.float32)


def test_gradients_exact_arithmetic(pkg, ctx):
    """A gradient check without rounding noise: integer weights, inputs and
    targets and a power-of-two pixel count make every FP32 sum of the forward
    and backward passes exact, so the GPU and the BF16-emulating float64
    oracle round identical values to BF16 at identical points (activations,
    output gradients) and break pooling ties alike (first maximum).  Any
    difference is then an error of the kernels: forward within 1e-6, every
    layer's weight and bias gradient within 1e-5 (FP32 rounding of the final
    weight-gradient sums only)."""
    B, H, W = 2, 32, 32
    rng = np.random.default_rng(5)
    x = rng.integers(-4, 5, (B, 2, H * W)).astype(np.float32)
    t = rng.integers(-4, 5, (B, 2, H * W)).astype(np.float32)
    p = exact_params(17)
    net = pkg.UNet(ctx, B, H, W, seed=1)
    try:
        net.set_params(p)
        y = net.forward(x, np.zeros_like(x))
        loss, g = net.gradients(x, t)
    finally:
        net.close()
    want, _ = U.forward(p, x, H, W, emulate_bf16=True)
    loss_o, g_o = U.loss_and_grads(p, x, t, H, W, emulate_bf16=True)
    ef = rel(y, want.detach().numpy())
    errs = []
    for i, (a, b) in enumerate(U.layer_slices()):
        ci, co, k, _ = U.CFG[i]
        wa, wb, ba, bb = a, b, b, b + co
        got_w, ref_w = g[wa:wb], g_o[wa:wb]
        if i == 0:  # the two real input channels
            got_w = got_w.reshape(co, k * k, ci)[:, :, :2]
            ref_w = ref_w.reshape(co, k * k, ci)[:, :, :2]
        got_b, ref_b = g[ba:bb], g_o[ba:bb]
        if i == len(U.CFG) - 1:  # outputs 0 and 1 of the last layer
            got_w, ref_w = got_w.reshape(co, ci)[:2], ref_w.reshape(co, ci)[:2]
            got_b, ref_b = got_b[:2], ref_b[:2]
        ew = rel(got_w, ref_w) if np.linalg.norm(ref_w) > 0 else float(np.abs(got_w).max())
        eb = rel(got_b, ref_b) if np.linalg.norm(ref_b) > 0 else float(np.abs(got_b).max())
        errs.append(max(ew, eb))
    print(f"exact arithmetic: forward {ef:.1e}, loss {loss:.6f} vs {loss_o:.6f}, layer "
          f"gradient errors " + " ".join(f"{e:.1e}" for e in errs))
    assert np.abs(y).max() < 2 ** 20  # the exactness premise
    assert ef < 1e-6
    assert abs(loss - loss_o) <= 1e-6 * loss_o
    assert max(errs) < 1e-5


def test_training_reduces_loss(pkg, ctx):
    B, H, W = 4, 32, 32
    net = pkg.UNet(ctx, B, H, W, seed=13)
    x, t = data(B, H, W, 3)
    try:
        losses = [net.train_step(x, t, 2e-3) for _ in range(80)]
    finally:
        net.close()
    print(f"loss {losses[0]:.4f} -> {losses[-1]:.4f}")
    assert losses[-1] < 0.2 * losses[0]


def test_row_strip_convolutions(pkg, ctx, monkeypatch):
    """16 x 256 images: the 3x3 layers with <= 64 channels at widths 256 and 128
    run the row-strip kernel (halo strips, taps as shifted shared-memory views).
    Forward within 1e-2 of the BF16-emulating oracle; forward and gradients
    equal to the 8 x 16 patch kernel's up to FP32 summation order."""
    B, H, W = 1, 16, 256
    x, t = data(B, H, W, 9)
    res = {}
    for name, env in (("strip", "1"), ("patch", "0")):
        monkeypatch.setenv("IMP_UNET_STRIP", env)
        net = pkg.UNet(ctx, B, H, W, seed=31)
        try:
            p = net.get_params()
            y = net.forward(x, np.zeros_like(x))
            loss, g = net.gradients(x, t)
        finally:
            net.close()
        res[name] = (y, loss, g)
    want, _ = U.forward(p, x, H, W, emulate_bf16=True)
    e = rel(res["strip"][0], want.detach().numpy())
    es, eg = rel(res["strip"][0], res["patch"][0]), rel(res["strip"][2], res["patch"][2])
    print(f"strip vs oracle {e:.2e}; strip vs patch: forward {es:.2e}, gradients {eg:.2e}")
    assert e < 1e-2
    assert es < 1e-5
    assert abs(res["strip"][1] - res["patch"][1]) / res["patch"][1] < 1e-4
    assert eg < 1e-3


def test_tensor_memory_and_wmma_kernels_agree(pkg, ctx, monkeypatch):
    """The tcgen05 convolution (accumulator in tensor memory) and the WMMA one
    give the same forward pass and gradients up to FP32 summation order."""
    B, H, W = 2, 32, 32
    x, t = data(B, H, W, 5)
    nets = {}
    for name, env in (("tc", "0"), ("wmma", "1")):
        monkeypatch.setenv("IMP_UNET_WMMA", env)
        net = pkg.UNet(ctx, B, H, W, seed=21)
        try:
            y = net.forward(x, np.zeros_like(x))
            loss, g = net.gradients(x, t)
        finally:
            net.close()
        nets[name] = (y, loss, g)
    (y1, l1, g1), (y2, l2, g2) = nets["tc"], nets["wmma"]
    print(f"tc vs wmma: forward {rel(y1, y2):.2e}, gradients {rel(g1, g2):.2e}")
    assert rel(y1, y2) < 1e-2
    assert abs(l1 - l2) / l2 < 1e-3
    assert rel(g1, g2) < 5e-2

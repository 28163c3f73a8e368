"""What the trained network gains over plain CG, at a small scale that trains
in seconds: 64x64 images, 4 coils, an 8 x 512 spiral, 320 training phantoms
with 50-iteration CG labels (regularized CG: lambda = 1e-3 lambda_max).  The network's starting image must be much closer
to the converged solution than zero, and CG from it must need fewer updates to
reach NRMSE 1e-3 against the converged solution than CG from zero.  Plus the
warm-start CG entry
point itself against the FP64 oracle's CG."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx(pkg):
    c = pkg.Context(0)
    yield c
    c.close()


@pytest.fixture(scope="module")
def prob(pkg, ctx):
    from impatient_mri_b200 import learn
    return learn.ToepProblem(pkg, ctx, n=64, C=4, n_il=8, n_s=512, seed=21)


def test_warm_cg_matches_oracle(pkg, ctx, prob):
    """CG from a nonzero start to a residual tolerance, against the oracle's CG
    started from the same image (same operator: the GPU's Q)."""
    import torch
    from oracle import toeplitz as T
    from impatient_mri_b200 import synth
    rng = np.random.default_rng(4)
    n, N = prob.n, prob.N
    img = synth.to_voxel_order(synth.ellipse_phantom((n, n), 8, rng))
    xt = torch.as_tensor(np.stack([img.real, img.imag]).astype(np.float32)).cuda()
    b = prob.aha(xt, torch.zeros_like(xt))
    x0 = (0.5 * xt).contiguous()
    x = x0.clone()
    it = prob.cg(b, x, 1e-2, 200)
    assert 0 < it < 200
    Q = (prob.qr + 1j * prob.qi).cpu().numpy().astype(np.complex128).reshape(1, 2 * n, 2 * n)
    sens = (prob.sr + 1j * prob.si).cpu().numpy().reshape(prob.C, n, n)
    bc = (b[0] + 1j * b[1]).cpu().numpy().astype(np.complex128).reshape(n, n)
    Qf = T.qf_from_q(Q)
    A = lambda v: (T.aha(v, Qf, sens, np.zeros((n, n)), 0.0, 0.0)
                   + T.dhwd(v, np.ones((n, n)), prob.lam))
    xo = (x0[0] + 1j * x0[1]).cpu().numpy().astype(np.complex128).reshape(n, n)
    r = bc - A(xo)
    p, rr = r.copy(), np.vdot(r, r).real
    for _ in range(it):
        q = A(p)
        a = rr / np.vdot(p, q).real
        xo, r = xo + a * p, r - a * q
        rr2 = np.vdot(r, r).real
        p, rr = r + (rr2 / rr) * p, rr2
    got = (x[0] + 1j * x[1]).cpu().numpy().reshape(n, n)
    err = np.linalg.norm(got - xo) / np.linalg.norm(xo)
    print(f"warm CG ({it} updates) vs oracle CG: {err:.2e}")
    assert err < 1e-4


def test_cg_after_a_tolerance_stop_starts_clean(pkg, ctx, prob):
    """A CG call that stopped on its tolerance leaves the device stop flag set;
    the next call must not inherit it (its first A^H A would be skipped)."""
    import torch
    from impatient_mri_b200 import learn, synth
    rng = np.random.default_rng(6)
    img = synth.to_voxel_order(synth.ellipse_phantom((prob.n, prob.n), 8, rng))
    xt = torch.as_tensor(np.stack([img.real, img.imag]).astype(np.float32)).cuda()
    b = prob.aha(xt, torch.zeros_like(xt))
    zero = torch.zeros_like(b)
    a = learn._cg_k(prob, b, zero, 10)
    x = zero.clone()
    assert prob.cg(b, x, 1e-3, 200) < 200  # stops on the tolerance
    c = learn._cg_k(prob, b, zero, 10)
    assert torch.equal(a, c)


def test_network_warm_start_saves_iterations(pkg, ctx, prob):
    import torch
    from impatient_mri_b200 import learn
    b, lab, _ = prob.make_pairs(328, seed=5)
    x, y, kappa = learn.normalise(b[:320], lab[:320])
    net = pkg.UNet(ctx, 8, 64, 64, seed=7)
    net1 = pkg.UNet(ctx, 1, 64, 64, seed=7)
    try:
        losses = learn.train(net, x, y, epochs=60, lr=2e-3)
        net1.set_params(net.get_params())
        res = learn.evaluate(prob, net1, kappa, b[320:328], target=1e-3, kmax=300)
    finally:
        net.close()
        net1.close()
    it_z = np.mean([r["zero_iters"] for r in res])
    it_w = np.mean([r["warm_iters"] for r in res])
    x0 = np.mean([r["x0_nrmse"] for r in res])
    it_tz = np.mean([r["zero_iters_tol"] for r in res])
    it_tw = np.mean([r["warm_iters_tol"] for r in res])
    print(f"train loss {losses[0]:.4f} -> {losses[-1]:.4f}; start NRMSE {x0:.3f}; "
          f"CG updates to NRMSE 1e-3: zero {it_z:.1f}, warm {it_w:.1f}; "
          f"to relative residual 1e-4: zero {it_tz:.1f}, warm {it_tw:.1f}")
    assert losses[-1] < 0.5 * losses[0]
    assert x0 < 0.3
    assert it_w < it_z

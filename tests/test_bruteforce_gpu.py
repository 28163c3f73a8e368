"""Brute-force CG on the GPU against the reference's FP64 recon (golden
vectors) and the FP64 oracle.  Tolerance: 1e-4 relative L2 on the final
image after the same iteration count and semantics (cg_num-1 updates)."""
import numpy as np
import pytest

import oracle
from conftest import golden

pytestmark = pytest.mark.gpu
TOL_IMG = 1e-4


@pytest.fixture(scope="module")
def ctx(pkg):
    c = pkg.Context(0)
    yield c
    c.close()


@pytest.fixture(scope="module", autouse=True)
def built():
    oracle.build(ref=False)


def test_bf_2d_tv_matches_reference_fp64(pkg, ctx):
    from gpu_util import gpu_recon
    c = golden("bf_2d")
    x = gpu_recon(pkg, ctx, c, cg_num=int(c["cg_num"]), lam=float(c["lam"]), tv=True,
                  tv_num=int(c["tv_num"]), eps=1e-7)
    err = oracle.rel_l2(x, c["x64"])
    err32 = oracle.rel_l2(c["x32"], c["x64"])
    print(f"GPU vs reference FP64: {err:.2e}; reference FP32 vs FP64: {err32:.2e}")
    assert err < TOL_IMG


def test_bf_2d_long_tv_no_worse_than_reference_fp32(pkg, ctx):
    """A long TV run amplifies rounding-level perturbations of the CG step by
    1e5 or more (tests/golden/gen_golden.py), so the gate is the reference's
    own FP32 build: the GPU image must be as close to the FP64 image as the
    reference's FP32 image is."""
    from gpu_util import gpu_recon
    c = golden("bf_2d_tv_long")
    x = gpu_recon(pkg, ctx, c, cg_num=int(c["cg_num"]), lam=float(c["lam"]), tv=True,
                  tv_num=int(c["tv_num"]), eps=1e-7)
    err = oracle.rel_l2(x, c["x64"])
    err32 = oracle.rel_l2(c["x32"], c["x64"])
    print(f"long TV: GPU vs reference FP64 {err:.2e}; reference FP32 vs FP64 {err32:.2e}")
    assert err < max(2.0 * err32, TOL_IMG)


def test_bf2d_64_timed_config_no_worse_than_reference_fp32(pkg, ctx):
    """The 2-D one-coil configuration that bench.py times (64x64, 4 x 1024
    spiral, field map, cg_num 8, TV lambda 1e-3 with 10 passes), on the same
    inputs (tests/golden/bf2d_64_timed.npz): a chaotic run (10 reweighting
    passes), so the gate is the reference's own FP32 build against its FP64
    build, as in the long-TV test above."""
    from gpu_util import gpu_recon
    c = golden("bf2d_64_timed")
    x = gpu_recon(pkg, ctx, c, cg_num=int(c["cg_num"]), lam=float(c["lam"]), tv=True,
                  tv_num=int(c["tv_num"]), eps=1e-6)
    err = oracle.rel_l2(x, c["x64"])
    err32 = oracle.rel_l2(c["x32"], c["x64"])
    print(f"timed 2-D configuration: GPU vs reference FP64 {err:.2e}; reference FP32 vs "
          f"FP64 {err32:.2e}")
    assert err < max(2.0 * err32, TOL_IMG)


def test_bf_2d_sense_matches_reference_fp64(pkg, ctx):
    from gpu_util import gpu_recon
    c = golden("bf_2d_c3")
    x = gpu_recon(pkg, ctx, c, cg_num=int(c["cg_num"]), lam=float(c["lam"]), tv=False, eps=1e-7)
    assert oracle.rel_l2(x, c["x64"]) < TOL_IMG


def test_bf_2d_24_coils_tensor_core_against_oracle(pkg, ctx, synth):
    """Twenty-four coils: the single-slice solver plans one coil group of 32 on
    the tensor-core NUDFT (its autotuner times only tensor-core launch shapes
    for such a group); FD-regularized CG within 1e-4 of the FP64 oracle."""
    from gpu_util import gpu_recon
    rng = np.random.default_rng(37)
    n, C = 24, 24
    ix, iy, iz = synth.grid_positions(n, n, 1)
    sens = np.stack([synth.to_voxel_order(m) for m in synth.coil_maps((n, n), C, rng)])
    kx, ky, t = synth.spiral(5, 256, n / 2, rng)
    img = synth.to_voxel_order(synth.ellipse_phantom((n, n), 5, rng))
    fm = synth.to_voxel_order(synth.field_map((n, n), rng)).astype(np.float32)
    c = dict(kx=kx, ky=ky, kz=np.zeros_like(kx), t=t, ix=ix, iy=iy, iz=iz, fm=fm,
             sens=sens.astype(np.complex64), dims=(n, n, 1), opts=dict(use_z=0))
    c["kdata"] = synth.add_noise(oracle.ft(img, c, use_z=0), 40.0, rng).astype(np.complex64)
    x = gpu_recon(pkg, ctx, c, cg_num=6, lam=1e-2, tv=False)
    ref = oracle.bf_cg(c, cg_num=6, lam=1e-2, tv=False, use_z=0)
    assert oracle.rel_l2(x, ref) < TOL_IMG


def small_3d(synth, seed=31):
    rng = np.random.default_rng(seed)
    ny = nx = 24
    nz = 8
    kx2, ky2, t2 = synth.spiral(4, 128, 12.0, rng)
    kz = np.repeat(np.arange(-4, 4, dtype=np.float32), kx2.size)
    case = dict(kx=np.tile(kx2, 8), ky=np.tile(ky2, 8), kz=kz, t=np.tile(t2, 8))
    ix, iy, iz = synth.grid_positions(ny, nx, nz)
    img = synth.ellipse_phantom((ny, nx, nz), 5, rng)
    case.update(ix=ix, iy=iy, iz=iz, fm=synth.field_map((ny, nx, nz), rng).ravel(),
                sens=synth.coil_maps((ny, nx, nz), 4, rng).reshape(4, -1), dims=(nx, ny, nz),
                opts=dict(use_z=1, cg_num=6))
    y = oracle.ft(img.ravel(), case, use_z=1)
    case["kdata"] = synth.add_noise(y, 40.0, rng).astype(np.complex64)
    return case


def test_bf_3d_tv_matches_oracle(pkg, ctx, synth):
    from gpu_util import gpu_recon
    c = small_3d(synth)
    x = gpu_recon(pkg, ctx, c, cg_num=3, lam=1e-2, tv=True, tv_num=2, eps=1e-6, use_z=1,
                  dims=c["dims"])
    ref = oracle.bf_cg(c, cg_num=3, lam=1e-2, tv=True, tv_num=2, eps=1e-6, use_z=1)
    assert oracle.rel_l2(x, ref) < TOL_IMG


def test_batch_3d_tv_matches_oracle(pkg, ctx, synth):
    """Batched multi-slice with the true 3-D phase and 3-D TV: two 24x24x8
    slices with their own stacks of spirals, the second one shorter (uneven
    M), each within 1e-4 of the FP64 oracle."""
    cases = [small_3d(synth, seed=41), small_3d(synth, seed=42)]
    keep = cases[1]["kx"].size - 640  # drop the last 640 samples of slice 1
    c1 = cases[1]
    C = np.asarray(c1["sens"]).size // c1["ix"].size
    kd1 = np.asarray(c1["kdata"]).reshape(C, -1)[:, :keep]
    cases[1] = dict(c1, kx=c1["kx"][:keep], ky=c1["ky"][:keep], kz=c1["kz"][:keep],
                    t=c1["t"][:keep], kdata=kd1)
    f32 = lambda a: np.ascontiguousarray(a, np.float32)
    N = cases[0]["ix"].size
    k_off = np.cumsum([0] + [c["kx"].size for c in cases])
    cat = lambda k: f32(np.concatenate([np.ravel(c[k]) for c in cases]))
    kd = np.concatenate([np.asarray(c["kdata"]).ravel() for c in cases])
    sens = np.asarray(cases[0]["sens"]).reshape(C, N)
    xr, xi = np.zeros(2 * N, np.float32), np.zeros(2 * N, np.float32)
    opts = pkg.bf_options(cg_num=3, fd_penalizer=1e-2, tv=True, tv_num=2, use_z=1,
                          dims=cases[0]["dims"])
    pkg.bruteForceBatch(ctx, opts, xr, xi, f32(kd.real), f32(kd.imag), cat("kx"), cat("ky"),
                        cat("kz"), cat("t"), k_off, cases[0]["ix"], cases[0]["iy"],
                        cases[0]["iz"], cat("fm"), f32(sens.real), f32(sens.imag), N, C)
    for s, c in enumerate(cases):
        got = xr[s * N:(s + 1) * N] + 1j * xi[s * N:(s + 1) * N].astype(np.float64)
        # the batch shares slice 0's coil maps; the oracle solves the same model
        ref = oracle.bf_cg(dict(c, sens=cases[0]["sens"]), cg_num=3, lam=1e-2, tv=True,
                           tv_num=2, eps=1e-6, use_z=1)
        assert oracle.rel_l2(got, ref) < TOL_IMG, s


def test_expired_wait_is_reported_and_context_stays_usable(pkg):
    """Failure path of the bounded device-side waits, without a GPU fault: a
    kernel waits on an mbarrier nothing arrives on, gives up after 1000 rounds,
    records the timeout and returns; the call reports IMP_ERR_TIMEOUT and the
    same context then reconstructs within 1e-4 of the FP64 oracle."""
    from gpu_util import gpu_recon
    with pkg.Context(0) as c0:
        with pytest.raises(pkg.ImpError) as e:
            c0.check_wait_expiry(1000)
        assert e.value.status == 7 and "wait" in str(e.value)
        c = golden("bf_2d_c3")
        x = gpu_recon(pkg, c0, c, cg_num=3, lam=1e-2, tv=False)
    ref = oracle.bf_cg(c, cg_num=3, lam=1e-2, tv=False, eps=1e-6, use_z=0)
    assert oracle.rel_l2(x, ref) < TOL_IMG


def test_host_and_device_pointers_agree(pkg, ctx):
    from gpu_util import gpu_recon
    c = golden("bf_2d_c3")
    a = gpu_recon(pkg, ctx, c, cg_num=4, lam=1e-2, tv=True, tv_num=2, host_ptrs=True)
    b = gpu_recon(pkg, ctx, c, cg_num=4, lam=1e-2, tv=True, tv_num=2, host_ptrs=False)
    assert np.array_equal(a, b)


def test_context_reuse_matches_fresh_context(pkg, ctx, synth):
    """A context keeps its solver between calls of the same size; a second
    geometry of that size must give what a fresh context gives."""
    from gpu_util import gpu_recon
    c = golden("bf_2d")
    rng = np.random.default_rng(9)
    kx, ky, t = synth.spiral(4, 1024, 32.0, rng)
    c2 = dict(c, kx=kx, ky=ky, t=t, fm=(c["fm"] * 0.3).astype(np.float32))
    gpu_recon(pkg, ctx, c, cg_num=3, lam=1e-2, tv=True, tv_num=2)
    a = gpu_recon(pkg, ctx, c2, cg_num=3, lam=1e-2, tv=True, tv_num=2)
    with pkg.Context(0) as fresh:
        b = gpu_recon(pkg, fresh, c2, cg_num=3, lam=1e-2, tv=True, tv_num=2)
    assert np.array_equal(a, b)


def test_multi_slice_equals_slice_by_slice(pkg, ctx):
    from gpu_util import gpu_recon
    c = golden("bf_2d_c3")
    rng = np.random.default_rng(2)
    kd2 = c["kdata"] * (0.5 + 0.1j) + 0.01 * rng.standard_normal(c["kdata"].shape)
    fm2 = (c["fm"] * -0.7).astype(np.float32)
    both = dict(c, kdata=np.concatenate([c["kdata"].ravel(), kd2.ravel()]),
                fm=np.concatenate([c["fm"], fm2]))
    x = gpu_recon(pkg, ctx, both, cg_num=5, lam=1e-2, tv=True, tv_num=2)
    a = gpu_recon(pkg, ctx, c, cg_num=5, lam=1e-2, tv=True, tv_num=2)
    b = gpu_recon(pkg, ctx, dict(c, kdata=kd2, fm=fm2), cg_num=5, lam=1e-2, tv=True, tv_num=2)
    N = c["ix"].size
    assert np.array_equal(x[:N], a) and np.array_equal(x[N:], b)


def _mgpu_case(n_slices):
    c = golden("bf_2d_c3")
    rng = np.random.default_rng(3)
    kds, fms = [], []
    for s in range(n_slices):
        kds.append(c["kdata"] * (0.4 + 0.15 * s + 0.1j)
                   + 0.01 * rng.standard_normal(c["kdata"].shape))
        fms.append((c["fm"] * (1.0 - 0.3 * s)).astype(np.float32))
    return c, np.concatenate([k.ravel() for k in kds]), np.concatenate(fms)


def _mgpu_args(c, kd, fm, n_slices):
    f32 = lambda a: np.ascontiguousarray(a, np.float32)
    N, M = c["ix"].size, c["kx"].size
    C = np.asarray(c["sens"]).size // N
    s = np.asarray(c["sens"]).reshape(C, N)
    xr, xi = np.zeros(n_slices * N, np.float32), np.zeros(n_slices * N, np.float32)
    args = (xr, xi, f32(kd.real), f32(kd.imag), f32(c["kx"]), f32(c["ky"]), f32(c["kz"]),
            f32(c["ix"]), f32(c["iy"]), f32(c["iz"]), f32(fm), f32(c["t"]), f32(s.real),
            f32(s.imag), M, N, C, n_slices)
    return args, xr, xi


def test_mgpu_work_queue_matches_one_context(pkg, ctx):
    """-mgpu work queue: three worker threads, each with its own context on GPU
    0, claim five slices; every slice equals the multi-slice call on one
    context to 1e-5 (the contexts tune their launch shapes independently)."""
    S = 5
    c, kd, fm = _mgpu_case(S)
    opts = pkg.bf_options(cg_num=5, fd_penalizer=1e-2, tv=True, tv_num=2)
    args, xr, xi = _mgpu_args(c, kd, fm, S)
    pkg.bruteForceMgpu(opts, *args, devices=[0, 0, 0])
    got = xr + 1j * xi.astype(np.float64)
    args1, yr, yi = _mgpu_args(c, kd, fm, S)
    pkg.bruteForceGpu(ctx, opts, *args1)
    ref = yr + 1j * yi.astype(np.float64)
    N = c["ix"].size
    for s in range(S):
        assert oracle.rel_l2(got[s * N:(s + 1) * N], ref[s * N:(s + 1) * N]) < 1e-5, s


def test_mgpu_reports_a_failing_worker(pkg):
    """A worker whose device does not exist stops the queue; the call returns
    its error (status and message) in the caller's thread."""
    c, kd, fm = _mgpu_case(3)
    opts = pkg.bf_options(cg_num=3)
    args, _, _ = _mgpu_args(c, kd, fm, 3)
    with pytest.raises(pkg.ImpError) as e:
        pkg.bruteForceMgpu(opts, *args, devices=[0, 4096])
    assert e.value.status == 1 and "4096" in str(e.value)


def test_warm_start_from_idata(pkg, ctx):
    """idata is the initial estimate (bruteForceCpu starts from *idata)."""
    from gpu_util import gpu_recon
    c = golden("bf_2d_c3")
    x0 = oracle.bf_cg(c, cg_num=3, lam=1e-2, tv=False, eps=1e-6, use_z=0).astype(np.complex64)
    x = gpu_recon(pkg, ctx, c, x0=x0, cg_num=3, lam=1e-2, tv=False)
    ref = oracle.bf_cg(c, x0=x0, cg_num=3, lam=1e-2, tv=False, eps=1e-6, use_z=0)
    assert oracle.rel_l2(x, ref) < TOL_IMG


def test_cli_end_to_end(pkg, tmp_path):
    """mriSolver on a 0.2-format directory writes output_gpu_{r,i}.dat ("%f")."""
    from impatient_mri_b200 import io
    c = golden("bf_2d")
    io.write_dataset(tmp_path / "in", "0.2", kx=c["kx"], ky=c["ky"], kz=c["kz"], t=c["t"],
                     ix=c["ix"], iy=c["iy"], iz=c["iz"], fm=c["fm"], kdata=c["kdata"],
                     sensi=c["sens"], dims=(64, 64, 1))
    rc = pkg.mriSolver("-idir", str(tmp_path / "in"), "-odir", str(tmp_path / "out"),
                       "-cg_num", "3", "-fdp", "0.01", "-tv_num", "2")
    assert rc == 0
    xr = np.loadtxt(tmp_path / "out" / "output_gpu_r.dat")
    xi = np.loadtxt(tmp_path / "out" / "output_gpu_i.dat")
    ref = oracle.bf_cg(c, cg_num=3, lam=1e-2, tv=True, tv_num=2, eps=1e-6, use_z=0)
    # "%f" keeps 6 decimals
    assert np.max(np.abs(xr + 1j * xi - ref)) < 1e-5 + 1e-4 * np.max(np.abs(ref))


def test_cli_mgpu_matches_single_gpu(pkg, tmp_path):
    """mriSolver -mgpu (slices over every visible GPU) writes the images of the
    single-GPU run on a two-slice 0.2-format directory."""
    from impatient_mri_b200 import io
    c, kd, fm = _mgpu_case(2)
    N = c["ix"].size
    n = int(round(np.sqrt(N)))
    io.write_dataset(tmp_path / "in", "0.2", kx=c["kx"], ky=c["ky"], kz=c["kz"], t=c["t"],
                     ix=c["ix"], iy=c["iy"], iz=c["iz"], fm=fm, kdata=kd, sensi=c["sens"],
                     dims=(n, n, 1), num_coil=np.asarray(c["sens"]).size // N, num_slices=2)
    outs = []
    for extra in ([], ["-mgpu"]):
        od = tmp_path / ("out_m" if extra else "out_1")
        rc = pkg.mriSolver("-idir", str(tmp_path / "in"), "-odir", str(od), "-cg_num", "3",
                           "-fdp", "0.01", *extra)
        assert rc == 0
        outs.append(np.loadtxt(od / "output_gpu_r.dat") + 1j * np.loadtxt(od / "output_gpu_i.dat"))
    assert outs[0].size == 2 * c["ix"].size
    assert np.max(np.abs(outs[0] - outs[1])) <= 2e-6 + 1e-5 * np.max(np.abs(outs[0]))


def test_batch_with_uneven_trajectories(pkg, ctx, synth, monkeypatch):
    """imp_bruteforce_batch: slices with their own spirals of different lengths
    and their own field maps, solved in lockstep by one batched solver; each
    slice matches the single-slice call on its own trajectory to 1e-5 (the
    batched launches split the FP32 partial sums and the FP64 block partials
    differently) and stays within 1e-4 of the FP64 oracle.  The single-slice
    calls take the default launch shape (no autotuning), so that both solves
    run the same NUDFT kernel: TV reweighting amplifies the 1e-7-level
    difference between the tensor-core and CUDA-core kernels about a
    hundredfold."""
    from gpu_util import gpu_recon
    monkeypatch.setenv("IMP_AUTOTUNE", "0")
    rng = np.random.default_rng(17)
    n, C = 32, 2
    ix, iy, iz = synth.grid_positions(n, n, 1)
    sens = np.stack([synth.to_voxel_order(m) for m in synth.coil_maps((n, n), C, rng)])
    cases = []
    for il in (3, 5, 4):
        kx, ky, t = synth.spiral(il, 256, n / 2, rng)
        img = synth.to_voxel_order(synth.ellipse_phantom((n, n), 6, rng))
        fm = synth.to_voxel_order(synth.field_map((n, n), rng)).astype(np.float32)
        c = dict(kx=kx, ky=ky, kz=np.zeros_like(kx), t=t, ix=ix, iy=iy, iz=iz, fm=fm,
                 sens=sens.astype(np.complex64), dims=(n, n, 1), opts=dict(use_z=0))
        c["kdata"] = synth.add_noise(oracle.ft(img, c, use_z=0), 40.0, rng).astype(np.complex64)
        cases.append(c)
    f32 = lambda a: np.ascontiguousarray(a, np.float32)
    k_off = np.cumsum([0] + [c["kx"].size for c in cases])
    cat = lambda k: f32(np.concatenate([c[k] for c in cases]))
    kd = np.concatenate([np.asarray(c["kdata"]).ravel() for c in cases])
    N = n * n
    xr = np.zeros(3 * N, np.float32)
    xi = np.zeros(3 * N, np.float32)
    opts = pkg.bf_options(cg_num=4, fd_penalizer=1e-2, tv=True, tv_num=2)
    pkg.bruteForceBatch(ctx, opts, xr, xi, f32(kd.real), f32(kd.imag), cat("kx"), cat("ky"),
                        cat("kz"), cat("t"), k_off, ix, iy, iz, cat("fm"), f32(sens.real),
                        f32(sens.imag), N, C)
    for s, c in enumerate(cases):
        got = xr[s * N:(s + 1) * N] + 1j * xi[s * N:(s + 1) * N].astype(np.float64)
        single = gpu_recon(pkg, ctx, c, cg_num=4, lam=1e-2, tv=True, tv_num=2)
        ref = oracle.bf_cg(c, cg_num=4, lam=1e-2, tv=True, tv_num=2, eps=1e-6, use_z=0)
        assert oracle.rel_l2(got, single) < 1e-5
        assert oracle.rel_l2(got, ref) < TOL_IMG


def test_batch_tensor_core_coil_group(pkg, ctx, synth):
    """Twenty coils: the plan takes one coil group of 32 (12 zero coil slots) on
    the tensor-core NUDFT, whose batched launches skip the blocks past a shorter
    slice's range and split the accumulator drain by coils; three slices of
    768, 1792 and 512 samples, each within 1e-4 of the FP64 oracle."""
    rng = np.random.default_rng(31)
    n, C = 24, 20
    ix, iy, iz = synth.grid_positions(n, n, 1)
    sens = np.stack([synth.to_voxel_order(m) for m in synth.coil_maps((n, n), C, rng)])
    cases = []
    for il in (3, 7, 2):
        kx, ky, t = synth.spiral(il, 256, n / 2, rng)
        img = synth.to_voxel_order(synth.ellipse_phantom((n, n), 5, rng))
        fm = synth.to_voxel_order(synth.field_map((n, n), rng)).astype(np.float32)
        c = dict(kx=kx, ky=ky, kz=np.zeros_like(kx), t=t, ix=ix, iy=iy, iz=iz, fm=fm,
                 sens=sens.astype(np.complex64), dims=(n, n, 1), opts=dict(use_z=0))
        c["kdata"] = synth.add_noise(oracle.ft(img, c, use_z=0), 40.0, rng).astype(np.complex64)
        cases.append(c)
    f32 = lambda a: np.ascontiguousarray(a, np.float32)
    k_off = np.cumsum([0] + [c["kx"].size for c in cases])
    cat = lambda k: f32(np.concatenate([c[k] for c in cases]))
    kd = np.concatenate([np.asarray(c["kdata"]).ravel() for c in cases])
    N, S = n * n, len(cases)
    xr = np.zeros(S * N, np.float32)
    xi = np.zeros(S * N, np.float32)
    pkg.bruteForceBatch(ctx, pkg.bf_options(cg_num=5), xr, xi, f32(kd.real), f32(kd.imag),
                        cat("kx"), cat("ky"), cat("kz"), cat("t"), k_off, ix, iy, iz, cat("fm"),
                        f32(sens.real), f32(sens.imag), N, C)
    for s, c in enumerate(cases):
        got = xr[s * N:(s + 1) * N] + 1j * xi[s * N:(s + 1) * N].astype(np.float64)
        ref = oracle.bf_cg(c, cg_num=5, tv=False, tv_num=1, eps=1e-6, use_z=0)
        assert oracle.rel_l2(got, ref) < TOL_IMG, s


def test_batch_many_slices_against_oracle(pkg, ctx, synth):
    """Seven slices whose sample counts pad to 1, 2 and 3 blocks of 1024, eight
    coils (one coil group of 8), plain CG: every slice within 1e-4 of the FP64
    oracle, and the launch count is that of one lockstep solve (independent of
    the number of slices)."""
    rng = np.random.default_rng(29)
    n, C = 24, 8
    ix, iy, iz = synth.grid_positions(n, n, 1)
    sens = np.stack([synth.to_voxel_order(m) for m in synth.coil_maps((n, n), C, rng)])
    cases = []
    for il in (2, 9, 4, 11, 3, 6, 1):
        kx, ky, t = synth.spiral(il, 256, n / 2, rng)
        img = synth.to_voxel_order(synth.ellipse_phantom((n, n), 5, rng))
        fm = synth.to_voxel_order(synth.field_map((n, n), rng)).astype(np.float32)
        c = dict(kx=kx, ky=ky, kz=np.zeros_like(kx), t=t, ix=ix, iy=iy, iz=iz, fm=fm,
                 sens=sens.astype(np.complex64), dims=(n, n, 1), opts=dict(use_z=0))
        c["kdata"] = synth.add_noise(oracle.ft(img, c, use_z=0), 40.0, rng).astype(np.complex64)
        cases.append(c)
    f32 = lambda a: np.ascontiguousarray(a, np.float32)
    k_off = np.cumsum([0] + [c["kx"].size for c in cases])
    cat = lambda k: f32(np.concatenate([c[k] for c in cases]))
    kd = np.concatenate([np.asarray(c["kdata"]).ravel() for c in cases])
    N, S = n * n, len(cases)
    launches = []
    for n_sl in (S, 2):
        xr = np.zeros(n_sl * N, np.float32)
        xi = np.zeros(n_sl * N, np.float32)
        opts = pkg.bf_options(cg_num=6)
        kk = k_off[:n_sl + 1]
        pkg.bruteForceBatch(ctx, opts, xr, xi, f32(kd.real[:C * kk[-1]]),
                            f32(kd.imag[:C * kk[-1]]), cat("kx")[:kk[-1]], cat("ky")[:kk[-1]],
                            cat("kz")[:kk[-1]], cat("t")[:kk[-1]], kk, ix, iy, iz,
                            cat("fm")[:n_sl * N], f32(sens.real), f32(sens.imag), N, C)
        launches.append(ctx.launch_count())
        if n_sl == S:
            for s, c in enumerate(cases):
                got = xr[s * N:(s + 1) * N] + 1j * xi[s * N:(s + 1) * N].astype(np.float64)
                ref = oracle.bf_cg(c, cg_num=6, tv=False, tv_num=1, eps=1e-6, use_z=0)
                assert oracle.rel_l2(got, ref) < TOL_IMG, s
    assert launches[0] == launches[1]


def test_batch_tuned_shapes_are_cached(pkg, ctx, synth, monkeypatch, tmp_path):
    """The batched solver tunes its launch shape per batched problem (both
    directions, timed over the whole batch) and caches it as "b1" lines; a
    second solve of the same problem reads the cache and gives the same image
    bit for bit; every slice stays within 1e-4 of the FP64 oracle."""
    cache = tmp_path / "tune.txt"
    monkeypatch.setenv("IMP_TUNE_CACHE", str(cache))
    monkeypatch.delenv("IMP_AUTOTUNE", raising=False)
    rng = np.random.default_rng(41)
    n, C = 24, 4
    ix, iy, iz = synth.grid_positions(n, n, 1)
    sens = np.stack([synth.to_voxel_order(m) for m in synth.coil_maps((n, n), C, rng)])
    cases = []
    for il in (5, 3, 8, 2, 6):
        kx, ky, t = synth.spiral(il, 256, n / 2, rng)
        img = synth.to_voxel_order(synth.ellipse_phantom((n, n), 5, rng))
        fm = synth.to_voxel_order(synth.field_map((n, n), rng)).astype(np.float32)
        c = dict(kx=kx, ky=ky, kz=np.zeros_like(kx), t=t, ix=ix, iy=iy, iz=iz, fm=fm,
                 sens=sens.astype(np.complex64), dims=(n, n, 1), opts=dict(use_z=0))
        c["kdata"] = synth.add_noise(oracle.ft(img, c, use_z=0), 40.0, rng).astype(np.complex64)
        cases.append(c)
    f32 = lambda a: np.ascontiguousarray(a, np.float32)
    k_off = np.cumsum([0] + [c["kx"].size for c in cases])
    cat = lambda k: f32(np.concatenate([c[k] for c in cases]))
    kd = np.concatenate([np.asarray(c["kdata"]).ravel() for c in cases])
    N, S = n * n, len(cases)
    images = []
    for _ in range(2):
        xr = np.zeros(S * N, np.float32)
        xi = np.zeros(S * N, np.float32)
        pkg.bruteForceBatch(ctx, pkg.bf_options(cg_num=6), xr, xi, f32(kd.real), f32(kd.imag),
                            cat("kx"), cat("ky"), cat("kz"), cat("t"), k_off, ix, iy, iz,
                            cat("fm"), f32(sens.real), f32(sens.imag), N, C)
        images.append(xr + 1j * xi.astype(np.float64))
    lines = [ln.split() for ln in cache.read_text().splitlines() if ln.startswith("b1 ")]
    assert sorted(int(ln[1]) for ln in lines) == [0, 1]  # one line per direction, written once
    assert all(int(ln[5]) == S for ln in lines)
    assert np.array_equal(images[0], images[1])
    for s, c in enumerate(cases):
        got = images[0][s * N:(s + 1) * N]
        ref = oracle.bf_cg(c, cg_num=6, tv=False, tv_num=1, eps=1e-6, use_z=0)
        assert oracle.rel_l2(got, ref) < TOL_IMG, s

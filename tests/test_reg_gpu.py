"""-reg (roughness regularization with a sparse matrix C) on the GPU through
the C-ABI: lambda C^T W C replaces lambda D^H W D in the brute-force and
Toeplitz CG (bruteForce/bruteForceCpu.cpp:306-380, toeplitz/recon.cu:
1543-1673).  Against the reference's own FP64 bruteForceCpu -reg result
(tests/golden/bf_2d_reg.npz, a generic C) at 1e-4, the FP64 Toeplitz oracle
with the same C at 1e-4 (recon) and 1e-5 (one application), and the GPU's own
-fd run when C is the periodic difference matrix (1e-5)."""
import numpy as np
import pytest

import oracle
from conftest import golden
from oracle import toeplitz as T

pytestmark = pytest.mark.gpu
TOL_IMG, TOL_OP = 1e-4, 1e-5


@pytest.fixture(scope="module")
def ctx(pkg):
    c = pkg.Context(0)
    yield c
    c.close()


def sparse_of(pkg, c):
    return pkg.Sparse.from_coo(int(c["C_rows"]), int(c["C_cols"]), c["C_I"], c["C_J"], c["C_V"])


def bf(pkg, ctx, c, opts):
    M, N = c["kx"].size, c["ix"].size
    s = np.asarray(c["sens"]).reshape(-1, N)
    f = lambda a: np.ascontiguousarray(a, np.float32)
    kd = np.asarray(c["kdata"]).ravel()
    xr, xi = np.zeros(N, np.float32), np.zeros(N, np.float32)
    pkg.bruteForceGpu(ctx, opts, xr, xi, f(kd.real), f(kd.imag), f(c["kx"]), f(c["ky"]),
                      f(c["kz"]), f(c["ix"]), f(c["iy"]), f(c["iz"]), f(c["fm"]), f(c["t"]),
                      f(s.real), f(s.imag), M, N, s.shape[0], 1)
    return xr + 1j * xi.astype(np.float64)


def test_bf_reg_matches_reference_fp64(pkg, ctx):
    c = golden("bf_2d_reg")
    opts = pkg.bf_options(cg_num=int(c["cg_num"]), fd_penalizer=float(c["lam"]), tv=True,
                          tv_num=int(c["tv_num"]), tv_eps=1e-6, reg=sparse_of(pkg, c))
    x = bf(pkg, ctx, c, opts)
    err, err32 = oracle.rel_l2(x, c["x64"]), oracle.rel_l2(c["x32"], c["x64"])
    print(f"-reg brute force: GPU vs reference FP64 {err:.2e}; reference FP32 {err32:.2e}")
    assert err < TOL_IMG


def test_bf_reg_with_difference_matrix_equals_fd(pkg, ctx, synth):
    """C = the periodic difference matrix: the -reg recon is the -fd recon."""
    c = golden("bf_2d")
    R, N, I, J, V = synth.fd_matrix((64, 64))
    kw = dict(cg_num=3, fd_penalizer=1e-2, tv=True, tv_num=2, tv_eps=1e-6)
    a = bf(pkg, ctx, c, pkg.bf_options(**kw, reg=pkg.Sparse.from_coo(R, N, I, J, V)))
    b = bf(pkg, ctx, c, pkg.bf_options(**kw))
    print(f"-reg (difference matrix) vs -fd: {oracle.rel_l2(a, b):.2e}")
    assert oracle.rel_l2(a, b) < TOL_OP
    assert oracle.rel_l2(b, c["x64"]) < TOL_IMG


def toep_case(dims, C, L, seed):
    rng = np.random.default_rng(seed)
    nx, ny, nz = dims
    N, M = nx * ny * nz, 64
    G = 4 * nx * ny * (1 if nz == 1 else 2 * nz)
    return dict(dims=dims, L=L, t=np.sort(rng.uniform(0.0, 0.01, M)).astype(np.float32),
                fm=rng.uniform(-200.0, 200.0, N).astype(np.float32),
                sens=(rng.standard_normal((C, N)) + 1j * rng.standard_normal((C, N))).astype(
                    np.complex64),
                Q=(rng.standard_normal((L + 1, G)) + 1j * rng.standard_normal((L + 1, G))).astype(
                    np.complex64),
                p=(rng.standard_normal(N) + 1j * rng.standard_normal(N)).astype(np.complex64),
                rng=rng)


def generic_matrix(synth, shape, rng):
    R, N, I, J, V = synth.fd_matrix(shape)
    return R, N, I, J, V * rng.uniform(0.5, 1.5, V.size)


@pytest.mark.parametrize("dims", [(32, 32, 1), (16, 16, 8)])
def test_toeplitz_apply_reg_matches_oracle(pkg, ctx, synth, dims):
    c = toep_case(dims, 2, 1, 5 + dims[2])
    nx, ny, nz = dims
    shape = (nx, ny) if nz == 1 else (ny, nx, nz)
    reg = generic_matrix(synth, shape, c["rng"])
    f = lambda a: np.ascontiguousarray(a, np.float32)
    N = nx * ny * nz
    s = c["sens"]
    o = pkg.toeplitz_options(cg_num=1, fd_penalizer=0.05, ntime_segs=c["L"],
                             reg=pkg.Sparse.from_coo(*reg))
    outr, outi = np.zeros(N, np.float32), np.zeros(N, np.float32)
    pkg.toeplitz_apply(ctx, o, outr, outi, f(c["p"].real), f(c["p"].imag), f(c["Q"].real.ravel()),
                       f(c["Q"].imag.ravel()), f(c["t"]), 64, f(c["fm"]), f(s.real), f(s.imag), 2,
                       nx, ny, nz)
    got = outr + 1j * outi.astype(np.float64)
    tau, t0 = T.time_segments(c["t"], c["L"])
    q_shape = tuple(2 * n if n > 1 else 1 for n in shape)
    Qf = T.qf_from_q(np.asarray(c["Q"], np.complex128).reshape(c["L"] + 1, *q_shape))
    p = np.asarray(c["p"]).reshape(shape)
    want = (T.aha(p, Qf, np.asarray(s, np.complex128).reshape(2, *shape),
                  np.asarray(c["fm"], np.float64).reshape(shape), tau, t0)
            + T.reg_penalty(p, reg, np.ones(shape), 0.05)).ravel()
    err = oracle.rel_l2(got, want)
    print(f"apply with -reg {dims}: {err:.2e}")
    assert err < TOL_OP


def test_toeplitz_recon_reg_matches_oracle(pkg, ctx, synth):
    """Toeplitz CG with TV reweighting and -reg from the reference's own Q and
    F^H d (tests/golden/toep_2d_tv.npz) against the FP64 oracle's CG."""
    from test_toeplitz_gpu import gpu_recon, opts_of
    from test_toeplitz_oracle import load
    c = load("toep_2d_tv")
    nx, ny, nz = (int(v) for v in c["dims"])
    reg = generic_matrix(synth, (nx, ny), np.random.default_rng(9))
    o = opts_of(pkg, c)
    o2 = pkg.toeplitz_options(cg_num=o.cg_num, fd_penalizer=o.fd_penalizer, tv=bool(o.enable_tv),
                              tv_num=o.tv_num, ntime_segs=o.ntime_segs, gridOS_Q=o.gridOS_Q,
                              gridOS_FH=o.gridOS_FH, reg=pkg.Sparse.from_coo(*reg))
    x = gpu_recon(pkg, ctx, o2, c, c["Q"], c["fhd"])
    shape = (nx, ny)
    N = nx * ny
    Q = np.asarray(c["Q"], np.complex128).reshape(int(c["L"]) + 1, 2 * nx, 2 * ny)
    want = T.toeplitz_cg(np.asarray(c["fhd"], np.complex128).reshape(shape), Q,
                         np.asarray(c["sens"], np.complex128).reshape(-1, N), c["fm"], c["t"],
                         int(c["L"]), int(c["cg"]), lam=float(c["fdp"]), tv=int(c["tv_num"]) > 0,
                         tv_num=max(int(c["tv_num"]), 1), reg=reg)
    err = oracle.rel_l2(x, want.ravel())
    print(f"Toeplitz CG with -reg vs FP64 oracle: {err:.2e}")
    assert err < TOL_IMG


def test_reg_argument_checks(pkg, ctx, synth):
    c = golden("bf_2d_reg")
    R, N, I, J, V = synth.fd_matrix((16, 16))  # the wrong image size
    opts = pkg.bf_options(cg_num=2, fd_penalizer=1e-2, reg=pkg.Sparse.from_coo(R, N, I, J, V))
    with pytest.raises(pkg.ImpError, match="INVALID_ARG.*-reg matrix"):
        bf(pkg, ctx, c, opts)


def test_cli_reg(pkg, tmp_path, synth):
    """mriSolver -reg reads idir/c.rmtx: its image equals the in-process call's."""
    from impatient_mri_b200 import io
    c = golden("bf_2d_reg")
    n = 32
    io.write_dataset(tmp_path / "in", "0.2", kx=c["kx"], ky=c["ky"], kz=c["kz"], t=c["t"],
                     ix=c["ix"], iy=c["iy"], iz=c["iz"], fm=c["fm"], kdata=c["kdata"],
                     sensi=c["sens"], dims=(n, n, 1), num_coil=2)
    io.write_mtx(tmp_path / "in" / "c.rmtx", int(c["C_rows"]), int(c["C_cols"]), c["C_I"],
                 c["C_J"], c["C_V"])
    rc = pkg.mriSolver("-idir", str(tmp_path / "in"), "-odir", str(tmp_path / "out"), "-reg",
                       "-fdp", str(float(c["lam"])), "-cg_num", str(int(c["cg_num"])),
                       "-tv_num", str(int(c["tv_num"])))
    assert rc == 0
    xr = np.loadtxt(tmp_path / "out" / "output_gpu_r.dat")
    xi = np.loadtxt(tmp_path / "out" / "output_gpu_i.dat")
    ref = c["x64"]
    assert np.max(np.abs(xr + 1j * xi - ref)) < 1e-5 + 1e-4 * np.max(np.abs(ref))

"""Toeplitz path on the GPU, called through the C-ABI, against the reference's
own outputs (tests/golden/toep_2d_*.npz, made by its GPU program) and the
FP64 oracle (oracle/toeplitz.py).

Tolerances (relative L2): Q, F^H d and one A^H A application 1e-5; the final
image 1e-4 after the same CG iteration count (cg_num updates, reconBest)."""
import os
import subprocess
import sys

import numpy as np
import pytest

import oracle
from oracle import toeplitz as T
from test_toeplitz_oracle import load, rel

pytestmark = pytest.mark.gpu
TOL_OP = 1e-5
TOL_IMG = 1e-4

f32 = lambda a: np.ascontiguousarray(a, np.float32)


@pytest.fixture(scope="module")
def ctx(pkg):
    c = pkg.Context(0)
    yield c
    c.close()


def opts_of(pkg, c):
    return pkg.toeplitz_options(cg_num=c["cg"], fd_penalizer=c["fdp"], tv=c["tv_num"] > 0,
                                tv_num=max(c["tv_num"], 1), ntime_segs=c["L"],
                                gridOS_Q=c["os_q"], gridOS_FH=c["os_fh"])


def grid_elems(dims):
    nx, ny, nz = dims
    return 4 * nx * ny * (1 if nz == 1 else 2 * nz)


def gpu_q(pkg, ctx, o, c):
    nx, ny, nz = c["dims"]
    G = grid_elems(c["dims"])
    qr = np.zeros((c["L"] + 1) * G, np.float32)
    qi = np.zeros_like(qr)
    pkg.toeplitz_q(ctx, o, qr, qi, f32(c["kx"]), f32(c["ky"]), f32(c["kz"]), f32(c["t"]),
                   c["kx"].size, nx, ny, nz)
    return (qr + 1j * qi.astype(np.float64)).reshape(c["L"] + 1, G)


def gpu_fhd(pkg, ctx, o, c):
    nx, ny, nz = c["dims"]
    N = nx * ny * nz
    kd = np.asarray(c["kdata"]).reshape(-1)
    s = np.asarray(c["sens"]).reshape(-1)
    fr = np.zeros(N, np.float32)
    fi = np.zeros(N, np.float32)
    C = np.asarray(c["sens"]).reshape(-1, N).shape[0]
    pkg.toeplitz_fhd(ctx, o, fr, fi, f32(kd.real), f32(kd.imag), f32(c["kx"]), f32(c["ky"]),
                     f32(c["kz"]), f32(c["t"]), f32(c["fm"]), f32(s.real), f32(s.imag),
                     c["kx"].size, C, nx, ny, nz)
    return fr + 1j * fi.astype(np.float64)


def gpu_recon(pkg, ctx, o, c, Q, fhd, device=False):
    nx, ny, nz = c["dims"]
    N = nx * ny * nz
    s = np.asarray(c["sens"]).reshape(-1, N)
    Q = np.asarray(Q).reshape(-1)
    fhd = np.asarray(fhd).reshape(-1)
    args = [f32(fhd.real), f32(fhd.imag), f32(Q.real), f32(Q.imag), f32(c["t"])]
    tail = [f32(c["fm"]), f32(s.real), f32(s.imag)]
    xr = np.zeros(N, np.float32)
    xi = np.zeros(N, np.float32)
    if device:
        from gpu_util import dev, host
        args = [dev(a) for a in args]
        tail = [dev(a) for a in tail]
        xr, xi = dev(xr), dev(xi)
    pkg.toeplitz_recon(ctx, o, xr, xi, *args, c["kx"].size, *tail, s.shape[0], nx, ny, nz)
    if device:
        return host(xr) + 1j * host(xi)
    return xr + 1j * xi.astype(np.float64)


def gpu_apply(pkg, ctx, o, c, Q, p):
    nx, ny, nz = c["dims"]
    N = nx * ny * nz
    s = np.asarray(c["sens"]).reshape(-1, N)
    Q = np.asarray(Q).reshape(-1)
    p = np.asarray(p).reshape(-1)
    outr = np.zeros(N, np.float32)
    outi = np.zeros(N, np.float32)
    pkg.toeplitz_apply(ctx, o, outr, outi, f32(p.real), f32(p.imag), f32(Q.real), f32(Q.imag),
                       f32(c["t"]), c["kx"].size, f32(c["fm"]), f32(s.real), f32(s.imag),
                       s.shape[0], nx, ny, nz)
    return outr + 1j * outi.astype(np.float64)


def image_shape(dims):
    nx, ny, nz = dims
    return (nx, ny) if nz == 1 else (ny, nx, nz)


def oracle_apply(c, Q, p, lam):
    shape = image_shape(c["dims"])
    N = int(np.prod(shape))
    tau, t0 = T.time_segments(c["t"], c["L"])
    q_shape = tuple(2 * n if n > 1 else 1 for n in shape)
    Qf = T.qf_from_q(np.asarray(Q, np.complex128).reshape(c["L"] + 1, *q_shape))
    sens = np.asarray(c["sens"], np.complex128).reshape(-1, *shape)
    fm = np.asarray(c["fm"], np.float64).reshape(shape)
    p = np.asarray(p).reshape(shape)
    out = T.aha(p, Qf, sens, fm, tau, t0)
    if lam is not None:
        out = out + T.dhwd(p, np.ones(shape), lam)
    return out.reshape(N)


# ------------------------------------------------------------- 2-D vs the reference

@pytest.mark.parametrize("name", ["toep_2d_fd", "toep_2d_tv"])
def test_q_2d_matches_reference(pkg, ctx, name):
    c = load(name)
    err = rel(gpu_q(pkg, ctx, opts_of(pkg, c), c), c["Q"])
    print(f"{name}: Q vs reference {err:.2e}")
    assert err < TOL_OP


@pytest.mark.parametrize("name", ["toep_2d_fd", "toep_2d_tv"])
def test_fhd_2d_matches_reference(pkg, ctx, name):
    c = load(name)
    err = rel(gpu_fhd(pkg, ctx, opts_of(pkg, c), c), c["fhd"])
    print(f"{name}: F^H d vs reference {err:.2e}")
    assert err < TOL_OP


@pytest.mark.parametrize("name", ["toep_2d_fd", "toep_2d_tv"])
def test_recon_2d_matches_reference(pkg, ctx, name):
    """CG from the reference's own Q and F^H d, then the whole chain from the
    GPU's Q and F^H d: both within 1e-4 of the reference's out.file."""
    c = load(name)
    o = opts_of(pkg, c)
    x = gpu_recon(pkg, ctx, o, c, c["Q"], c["fhd"])
    err = rel(x, c["out"])
    q = gpu_q(pkg, ctx, o, c)
    f = gpu_fhd(pkg, ctx, o, c)
    err_chain = rel(gpu_recon(pkg, ctx, o, c, q, f), c["out"])
    print(f"{name}: recon vs reference {err:.2e}, whole chain {err_chain:.2e}")
    assert err < TOL_IMG
    assert err_chain < TOL_IMG


def test_apply_2d_matches_oracle(pkg, ctx):
    c = load("toep_2d_fd")
    rng = np.random.default_rng(3)
    N = c["ix"].size
    p = (rng.standard_normal(N) + 1j * rng.standard_normal(N)).astype(np.complex64)
    got = gpu_apply(pkg, ctx, opts_of(pkg, c), c, c["Q"], p)
    want = oracle_apply(c, c["Q"], p, c["fdp"])
    assert rel(got, want) < TOL_OP


@pytest.mark.parametrize("dims,C,L", [((32, 64, 16), 2, 2), ((128, 64, 1), 3, 1),
                                      ((8, 4, 2), 1, 0), ((24, 40, 1), 2, 2),
                                      ((12, 8, 6), 2, 1)])
def test_apply_sizes_match_oracle(pkg, ctx, dims, C, L):
    """One A^H A (+ lambda D^H D) application with random Q, field map and
    sensitivities.  Power-of-two sizes run the pruned FFT engine (one- and
    two-pass line transforms, 2-D and 3-D); other even sizes run the
    zero-padded cuFFT chain."""
    rng = np.random.default_rng(sum(dims) + 7 * C + L)
    nx, ny, nz = dims
    N, M, G = nx * ny * nz, 64, grid_elems(dims)
    c = dict(dims=dims, L=L, cg=1, fdp=1e-2, tv_num=0, os_q=2.0, os_fh=1.5,
             t=np.sort(rng.uniform(0.0, 0.01, M)).astype(np.float32),
             kx=np.zeros(M, np.float32),
             fm=rng.uniform(-300.0, 300.0, N).astype(np.float32),
             sens=(rng.standard_normal((C, N)) + 1j * rng.standard_normal((C, N))).astype(
                 np.complex64))
    if C == 1:  # one coil: unit sensitivities (toeplitz/computeFH.cmem.cu:305-310)
        c["sens"] = np.ones((1, N), np.complex64)
    Q = (rng.standard_normal((L + 1, G)) + 1j * rng.standard_normal((L + 1, G))).astype(
        np.complex64)
    p = (rng.standard_normal(N) + 1j * rng.standard_normal(N)).astype(np.complex64)
    got = gpu_apply(pkg, ctx, opts_of(pkg, c), c, Q, p)
    err = rel(got, oracle_apply(c, Q, p, c["fdp"]))
    print(f"apply {dims} C={C} L={L}: {err:.2e}")
    assert err < TOL_OP


@pytest.mark.parametrize("dims", [(256, 256, 32), (512, 512, 1)])
def test_apply_production_sizes_match_oracle(pkg, ctx, dims):
    """One A^H A (+ lambda D^H D) application at the sizes the benchmarks run:
    the 3-D 256x256x32 image (two-pass n = 256 line transforms, s = 256 on the
    slow axis) and the 2-D 512x512 image (two-pass n = 512), both on the
    plane kernels instantiated on compile-time geometry, against the FP64
    oracle with random Q, field map and sensitivities (2 coils, 2 segments)."""
    rng = np.random.default_rng(sum(dims) + 101)
    nx, ny, nz = dims
    C, L, M = 2, 1, 64
    N, G = nx * ny * nz, grid_elems(dims)
    c = dict(dims=dims, L=L, cg=1, fdp=1e-2, tv_num=0, os_q=2.0, os_fh=1.5,
             t=np.sort(rng.uniform(0.0, 0.01, M)).astype(np.float32),
             kx=np.zeros(M, np.float32),
             fm=rng.uniform(-300.0, 300.0, N).astype(np.float32),
             sens=(rng.standard_normal((C, N)) + 1j * rng.standard_normal((C, N))).astype(
                 np.complex64))
    Q = (rng.standard_normal((L + 1, G)) + 1j * rng.standard_normal((L + 1, G))).astype(
        np.complex64)
    p = (rng.standard_normal(N) + 1j * rng.standard_normal(N)).astype(np.complex64)
    got = gpu_apply(pkg, ctx, opts_of(pkg, c), c, Q, p)
    err = rel(got, oracle_apply(c, Q, p, c["fdp"]))
    print(f"apply {dims} C={C} L={L}: {err:.2e} vs the FP64 oracle")
    assert err < TOL_OP


@pytest.mark.parametrize("dims", [(256, 256, 32), (512, 512, 1)])
def test_apply_many_coils_per_block_match_oracle(pkg, ctx, dims):
    """Sixteen coils at the benchmark sizes: the inverse plane kernel's cluster of
    8 blocks gives each block two coils (register partial sums over both, the
    next quadrant's copies across the coil boundary), and in 3-D each slow-axis
    block loops over all 16 coils with the next coil's columns copied in ahead;
    one application against the FP64 oracle (2 segments)."""
    rng = np.random.default_rng(sum(dims) + 303)
    nx, ny, nz = dims
    C, L, M = 16, 1, 64
    N, G = nx * ny * nz, grid_elems(dims)
    c = dict(dims=dims, L=L, cg=1, fdp=1e-2, tv_num=0, os_q=2.0, os_fh=1.5,
             t=np.sort(rng.uniform(0.0, 0.01, M)).astype(np.float32),
             kx=np.zeros(M, np.float32),
             fm=rng.uniform(-300.0, 300.0, N).astype(np.float32),
             sens=(rng.standard_normal((C, N)) + 1j * rng.standard_normal((C, N))).astype(
                 np.complex64))
    Q = (rng.standard_normal((L + 1, G)) + 1j * rng.standard_normal((L + 1, G))).astype(
        np.complex64)
    p = (rng.standard_normal(N) + 1j * rng.standard_normal(N)).astype(np.complex64)
    got = gpu_apply(pkg, ctx, opts_of(pkg, c), c, Q, p)
    err = rel(got, oracle_apply(c, Q, p, c["fdp"]))
    print(f"apply {dims} C={C} L={L}: {err:.2e} vs the FP64 oracle")
    assert err < TOL_OP


@pytest.mark.parametrize("dims", [(256, 256, 32), (512, 512, 1)])
def test_specialised_plane_kernels_match_generic(pkg, monkeypatch, dims):
    """The plane kernels instantiated on compile-time geometry (3-D 256x256x32
    and 2-D 512x512 images) give the A^H A application of the generic
    runtime-geometry kernels (which the oracle tests above cover)."""
    rng = np.random.default_rng(sum(dims))
    nx, ny, nz = dims
    C, L, M = 2, 1, 64
    N, G = nx * ny * nz, grid_elems(dims)
    c = dict(dims=dims, L=L, cg=1, fdp=1e-2, tv_num=0, os_q=2.0, os_fh=1.5,
             t=np.sort(rng.uniform(0.0, 0.01, M)).astype(np.float32),
             kx=np.zeros(M, np.float32),
             fm=rng.uniform(-300.0, 300.0, N).astype(np.float32),
             sens=(rng.standard_normal((C, N)) + 1j * rng.standard_normal((C, N))).astype(
                 np.complex64))
    Q = (rng.standard_normal((L + 1, G)) + 1j * rng.standard_normal((L + 1, G))).astype(
        np.complex64)
    p = (rng.standard_normal(N) + 1j * rng.standard_normal(N)).astype(np.complex64)
    out = {}
    for name, env in (("specialised", "0"), ("generic", "1")):
        monkeypatch.setenv("IMP_TOEP_GENERIC", env)
        with pkg.Context(0) as c0:  # the choice is made when the context plans
            out[name] = gpu_apply(pkg, c0, opts_of(pkg, c), c, Q, p)
    err = rel(out["specialised"], out["generic"])
    print(f"apply {dims}: specialised vs generic {err:.2e}")
    assert err < 1e-6


@pytest.mark.parametrize("dims", [(32, 32, 8), (64, 64, 1)])
def test_padded_chain_matches_pruned_engine(pkg, monkeypatch, dims):
    """The zero-padded chain (pad, forward grid FFT of the 2N grid, x Qf_l,
    inverse, crop; the path of image sizes that are not powers of two, forced
    here by IMP_TOEP_PADDED=1) and the pruned parity-split engine give the same
    A^H A application on a power-of-two image: two independent
    implementations of the F^H F glue (3 coils, 3 segments, field map)."""
    rng = np.random.default_rng(sum(dims) + 7)
    nx, ny, nz = dims
    C, L, M = 3, 2, 64
    N, G = nx * ny * nz, grid_elems(dims)
    c = dict(dims=dims, L=L, cg=1, fdp=1e-2, tv_num=0, os_q=2.0, os_fh=1.5,
             t=np.sort(rng.uniform(0.0, 0.01, M)).astype(np.float32),
             kx=np.zeros(M, np.float32),
             fm=rng.uniform(-300.0, 300.0, N).astype(np.float32),
             sens=(rng.standard_normal((C, N)) + 1j * rng.standard_normal((C, N))).astype(
                 np.complex64))
    Q = (rng.standard_normal((L + 1, G)) + 1j * rng.standard_normal((L + 1, G))).astype(
        np.complex64)
    p = (rng.standard_normal(N) + 1j * rng.standard_normal(N)).astype(np.complex64)
    out = {}
    for name, env in (("pruned", "0"), ("padded", "1")):
        monkeypatch.setenv("IMP_TOEP_PADDED", env)
        with pkg.Context(0) as c0:  # the choice is made when the context plans
            out[name] = gpu_apply(pkg, c0, opts_of(pkg, c), c, Q, p)
    err = rel(out["pruned"], out["padded"])
    print(f"apply {dims}: padded chain vs pruned engine {err:.2e}")
    assert err < 1e-5
    assert rel(out["padded"], oracle_apply(c, Q, p, c["fdp"])) < TOL_OP


def test_device_and_host_pointers_agree(pkg, ctx):
    c = load("toep_2d_tv")
    o = opts_of(pkg, c)
    a = gpu_recon(pkg, ctx, o, c, c["Q"], c["fhd"], device=False)
    b = gpu_recon(pkg, ctx, o, c, c["Q"], c["fhd"], device=True)
    assert rel(a, b) < 1e-6


# ------------------------------------------------------------- 3-D vs the FP64 oracle

@pytest.fixture(scope="module")
def case3d(synth):
    c = synth.make_case("toep3d_256x256x32", small=True,
                        forward=lambda x, s, cs: oracle.ft(x, cs, use_z=1, sens=s))
    c.update(L=4, os_q=2.0, os_fh=1.5, cg=6, fdp=1e-3, tv_num=2)
    c["Q_oracle"] = T.compute_q(c["kx"], c["ky"], c["kz"], c["t"], c["dims"], c["L"],
                                c["os_q"]).reshape(c["L"] + 1, -1)
    c["fhd_oracle"] = T.compute_fhd(c["kx"], c["ky"], c["kz"], c["t"], c["dims"], c["L"],
                                    c["os_fh"], c["kdata"], c["sens"], c["fm"]).reshape(-1)
    return c


def test_q_3d_matches_oracle(pkg, ctx, case3d):
    c = case3d
    err = rel(gpu_q(pkg, ctx, opts_of(pkg, c), c), c["Q_oracle"])
    print(f"3-D Q vs oracle {err:.2e}")
    assert err < TOL_OP


def test_fhd_3d_matches_oracle(pkg, ctx, case3d):
    c = case3d
    err = rel(gpu_fhd(pkg, ctx, opts_of(pkg, c), c), c["fhd_oracle"])
    print(f"3-D F^H d vs oracle {err:.2e}")
    assert err < TOL_OP


def test_apply_3d_matches_oracle(pkg, ctx, case3d):
    c = case3d
    rng = np.random.default_rng(4)
    N = c["ix"].size
    p = (rng.standard_normal(N) + 1j * rng.standard_normal(N)).astype(np.complex64)
    got = gpu_apply(pkg, ctx, opts_of(pkg, c), c, c["Q_oracle"], p)
    assert rel(got, oracle_apply(c, c["Q_oracle"], p, c["fdp"])) < TOL_OP


def test_recon_3d_tv_matches_oracle(pkg, ctx, case3d):
    c = case3d
    shape = image_shape(c["dims"])
    x64 = T.toeplitz_cg(c["fhd_oracle"].reshape(shape),
                        c["Q_oracle"].reshape(c["L"] + 1, *(2 * n for n in shape)),
                        c["sens"], c["fm"], c["t"], c["L"], c["cg"], lam=c["fdp"], tv=True,
                        tv_num=c["tv_num"])
    x = gpu_recon(pkg, ctx, opts_of(pkg, c), c, c["Q_oracle"], c["fhd_oracle"])
    err = rel(x, x64)
    print(f"3-D TV recon vs oracle {err:.2e}")
    assert err < TOL_IMG


# ------------------------------------------------------------- directory level and CLI

def write_case(pkg, c, d):
    from impatient_mri_b200 import io
    io.write_dataset(d, "0.2", kx=c["kx"], ky=c["ky"], kz=c["kz"], t=c["t"], ix=c["ix"],
                     iy=c["iy"], iz=c["iz"], fm=c["fm"], kdata=c["kdata"], sensi=c["sens"],
                     dims=tuple(c["dims"]), num_coil=c["sens"].shape[0])


def read_pairs(fn, n):
    a = np.fromfile(fn, np.float32).reshape(-1, 2, n)
    return (a[:, 0] + 1j * a[:, 1].astype(np.float64)).squeeze()


def test_dir_writes_reference_files_and_reuses_q(pkg, tmp_path):
    c = load("toep_2d_fd")
    o = opts_of(pkg, c)
    N, G = c["ix"].size, grid_elems(c["dims"])
    write_case(pkg, c, tmp_path)
    pkg.toeplitz(str(tmp_path), o, writeQ=True)
    assert (tmp_path / "Q_stone.file").stat().st_size == (c["L"] + 1) * G * 8
    assert rel(read_pairs(tmp_path / "Q_stone.file", G), c["Q"]) < TOL_OP
    assert rel(read_pairs(tmp_path / "FhD.file", N), c["fhd"]) < TOL_OP
    out1 = read_pairs(tmp_path / "out.file", N)
    assert rel(out1, c["out"]) < TOL_IMG
    os.remove(tmp_path / "out.file")
    pkg.toeplitz(str(tmp_path), o, reuseQ=True)
    assert rel(read_pairs(tmp_path / "out.file", N), out1) < 1e-5
    # a Q file of the wrong size is refused (-ntime_segs changed)
    bad = opts_of(pkg, dict(c, L=c["L"] + 1))
    with pytest.raises(pkg.ImpError) as e:
        pkg.toeplitz(str(tmp_path), bad, reuseQ=True)
    assert e.value.status == 4  # IMP_ERR_FORMAT


def test_dir_direct_q_and_fhd_match_exact_sums(pkg, tmp_path):
    """-toeplitzDirect: Q_l = sum_k h_l(t_k) exp(+i 2 pi k.r) on the 2N grid
    (non-cumulative in l) and the exact adjoint F^H d with field map."""
    c = load("toep_2d_fd")
    o = opts_of(pkg, c)
    N, G, n, L = c["ix"].size, grid_elems(c["dims"]), c["dims"][0], c["L"]
    write_case(pkg, c, tmp_path)
    pkg.toeplitz(str(tmp_path), o, direct=True, writeQ=True)
    x = np.arange(-n, n) / n
    X, Y = np.meshgrid(x, x, indexing="ij")
    ph = np.exp(2j * np.pi * (np.outer(X.ravel(), c["kx"].astype(np.float64))
                              + np.outer(Y.ravel(), c["ky"].astype(np.float64))))
    tau, t0 = T.time_segments(c["t"], L)
    Qd = np.stack([ph @ T.hanning(c["t"], tau, l, t0) for l in range(L + 1)])
    assert rel(read_pairs(tmp_path / "Q_stone.file", G), Qd) < TOL_OP
    case = dict(c, opts=dict(use_z=0))
    want = oracle.ift(np.asarray(c["kdata"]), case, use_z=0, sens=c["sens"])
    assert rel(read_pairs(tmp_path / "FhD.file", N), want) < TOL_OP
    # CG from the direct Q and F^H d: the oracle's CG on the exact sums
    x64 = T.toeplitz_cg(want.reshape(n, n), Qd.reshape(L + 1, 2 * n, 2 * n), c["sens"],
                        c["fm"], c["t"], L, c["cg"], lam=c["fdp"])
    assert rel(read_pairs(tmp_path / "out.file", N), x64) < TOL_IMG


def test_cli_toeplitz_gridding(pkg, tmp_path):
    c = load("toep_2d_tv")
    write_case(pkg, c, tmp_path)
    exe = os.path.join(os.path.dirname(pkg.__file__), "bin", "mriSolver")
    r = subprocess.run([exe, "-idir", str(tmp_path), "-toeplitzGridding",
                        *[str(f) for f in c["flags"]]], capture_output=True, text=True,
                       timeout=300)
    print(r.stdout[-2000:], r.stderr[-2000:], file=sys.stderr)
    assert r.returncode == 0
    assert rel(read_pairs(tmp_path / "out.file", c["ix"].size), c["out"]) < TOL_IMG

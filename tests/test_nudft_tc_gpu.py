"""The tensor-core NUDFT kernel (TF32 tcgen05 MMA, A operand written into
tensor memory; nudft_tc.cu) against the CUDA-core kernel (IMP_NUDFT_TC=0) and
the FP64 oracle, through the operator C-ABI (parallelFtGpu / parallelIftGpu,
kernels/parImagingGpu.cu:92-152 in the reference).  Tolerance: 1e-5 relative
L2 per apply, the operator bar of the CUDA-core kernel."""
import os

import numpy as np
import pytest

import oracle
from test_nudft_gpu import case_nd

pytestmark = pytest.mark.gpu
TOL_OP = 1e-5


@pytest.fixture(scope="module")
def ctx(pkg):
    c = pkg.Context(0)
    yield c
    c.close()


@pytest.fixture(scope="module", autouse=True)
def built(tmp_path_factory):
    oracle.build(ref=False)
    old = {k: os.environ.get(k) for k in ("IMP_TUNE_CACHE", "IMP_NUDFT_TC", "IMP_AUTOTUNE")}
    # no tuned launch shapes (file or in-process): the default shape decides
    # which kernel runs
    os.environ["IMP_TUNE_CACHE"] = str(tmp_path_factory.mktemp("tune") / "none.txt")
    os.environ["IMP_AUTOTUNE"] = "0"
    yield
    for k, v in old.items():
        if v is None:
            os.environ.pop(k, None)
        else:
            os.environ[k] = v


def both(fn):
    """fn() with the tensor-core kernel, then with the CUDA-core kernel."""
    os.environ["IMP_NUDFT_TC"] = "1"
    a = fn()
    os.environ["IMP_NUDFT_TC"] = "0"
    try:
        b = fn()
    finally:
        os.environ["IMP_NUDFT_TC"] = "1"
    return a, b


def check(a, b, ref):
    assert oracle.rel_l2(a, ref) < TOL_OP
    assert oracle.rel_l2(a, b) < TOL_OP
    # different arithmetic: equal bits would mean one kernel ran twice
    assert not np.array_equal(a, b)


@pytest.mark.parametrize("C", [1, 2, 3, 4, 8, 9, 16, 20, 32, 40])
def test_coil_groups_2d(pkg, ctx, synth, C):
    """Coil groups of 1, 2, 4, 8 (both kernels), 16 and 32 (tensor-core kernel
    only; with IMP_NUDFT_TC=0 the plan takes groups of 8)."""
    from gpu_util import gpu_ft, gpu_ift
    c = case_nd(synth, 32, 32, 1, C, 1000, seed=40 + C)
    rng = np.random.default_rng(C)
    x = rng.standard_normal(1024) + 1j * rng.standard_normal(1024)
    d = rng.standard_normal((C, 1000)) + 1j * rng.standard_normal((C, 1000))
    a, b = both(lambda: gpu_ft(pkg, ctx, c, x))
    check(a, b, oracle.ft(x, c, use_z=0))
    a, b = both(lambda: gpu_ift(pkg, ctx, c, d))
    check(a, b, oracle.ift(d, c, use_z=0))


@pytest.mark.parametrize("C", [1, 4, 32])
def test_3d_with_field_map(pkg, ctx, synth, C):
    from gpu_util import gpu_ft, gpu_ift
    c = case_nd(synth, 16, 16, 8, C, 3000, seed=50 + C)
    rng = np.random.default_rng(C)
    N = c["ix"].size
    x = rng.standard_normal(N) + 1j * rng.standard_normal(N)
    d = rng.standard_normal((C, 3000)) + 1j * rng.standard_normal((C, 3000))
    a, b = both(lambda: gpu_ft(pkg, ctx, c, x, use_z=1))
    check(a, b, oracle.ft(x, c, use_z=1))
    a, b = both(lambda: gpu_ift(pkg, ctx, c, d, use_z=1))
    check(a, b, oracle.ift(d, c, use_z=1))


@pytest.mark.parametrize("M,N", [(1, 1), (7, 5), (1025, 3), (3, 2049)])
def test_ragged_sizes(pkg, ctx, M, N):
    from gpu_util import gpu_ft, gpu_ift
    rng = np.random.default_rng(M * 17 + N)
    c = dict(kx=rng.uniform(-16, 16, M).astype(np.float32),
             ky=rng.uniform(-16, 16, M).astype(np.float32),
             kz=np.zeros(M, np.float32), t=rng.uniform(0, 0.01, M).astype(np.float32),
             ix=rng.uniform(-0.5, 0.5, N).astype(np.float32),
             iy=rng.uniform(-0.5, 0.5, N).astype(np.float32), iz=np.zeros(N, np.float32),
             fm=rng.uniform(-300, 300, N).astype(np.float32), sens=np.ones((1, N), np.complex64),
             opts=dict(use_z=0))
    x = rng.standard_normal(N) + 1j * rng.standard_normal(N)
    d = rng.standard_normal(M) + 1j * rng.standard_normal(M)
    a, _ = both(lambda: gpu_ft(pkg, ctx, c, x))
    assert oracle.rel_l2(a, oracle.ft(x, c, use_z=0)) < TOL_OP
    a, _ = both(lambda: gpu_ift(pkg, ctx, c, d))
    assert oracle.rel_l2(a, oracle.ift(d, c, use_z=0)) < TOL_OP


def test_large_dynamic_range(pkg, ctx, synth):
    """k-space values over twelve decades: the TF32 head/tail split of the
    data keeps the relative error of every product near 2^-21."""
    from gpu_util import gpu_ift
    c = case_nd(synth, 32, 32, 1, 4, 2000, seed=61)
    rng = np.random.default_rng(61)
    mag = 10.0 ** rng.uniform(-6, 6, (4, 2000))
    d = mag * (rng.standard_normal((4, 2000)) + 1j * rng.standard_normal((4, 2000)))
    a, b = both(lambda: gpu_ift(pkg, ctx, c, d))
    check(a, b, oracle.ift(d, c, use_z=0))


def test_full_size_3d_against_cuda_cores(pkg, ctx, synth):
    """At the benchmark size (64x64x16, 4 coils, M = 65536) both kernels agree
    and a 64-sample spot check matches the FP64 oracle."""
    from gpu_util import gpu_ft, gpu_ift
    case = synth.make_case("bf3d_64x64x16")
    rng = np.random.default_rng(8)
    N, M, C = case["N"], case["M"], case["num_coil"]
    x = rng.standard_normal(N) + 1j * rng.standard_normal(N)
    y = rng.standard_normal((C, M)) + 1j * rng.standard_normal((C, M))
    a, b = both(lambda: gpu_ft(pkg, ctx, case, x, use_z=1))
    assert oracle.rel_l2(a, b) < TOL_OP and not np.array_equal(a, b)
    sel = rng.choice(M, 64, replace=False)
    sub = dict(case, kx=case["kx"][sel], ky=case["ky"][sel], kz=case["kz"][sel],
               t=case["t"][sel])
    assert oracle.rel_l2(a[:, sel], oracle.ft(x, sub, use_z=1)) < TOL_OP
    a, b = both(lambda: gpu_ift(pkg, ctx, case, y, use_z=1))
    assert oracle.rel_l2(a, b) < TOL_OP and not np.array_equal(a, b)

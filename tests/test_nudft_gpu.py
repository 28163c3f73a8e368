"""Parity of the sm_100a NUDFT tile engine (through the C-ABI) with the FP64
oracle and the reference's FP64 golden vectors.  Tolerance: 1e-5 relative L2
per operator apply."""
import numpy as np
import pytest

import oracle
from conftest import golden

pytestmark = pytest.mark.gpu
TOL_OP = 1e-5


@pytest.fixture(scope="module")
def ctx(pkg):
    c = pkg.Context(0)
    yield c
    c.close()


@pytest.fixture(scope="module", autouse=True)
def built():
    oracle.build(ref=False)


def case_nd(synth, ny, nx, nz, C, M, seed, fm=True):
    rng = np.random.default_rng(seed)
    n_il = 4
    kx, ky, t = synth.spiral(n_il, max(M // n_il, 1), nx / 2, rng)
    kx, ky, t = kx[:M], ky[:M], t[:M]
    kz = rng.integers(-nz // 2, max(nz // 2, 1), size=kx.size).astype(np.float32) if nz > 1 \
        else np.zeros_like(kx)
    ix, iy, iz = synth.grid_positions(ny, nx, nz)
    shape = (ny, nx, nz) if nz > 1 else (ny, nx)
    f = synth.field_map(shape, rng).ravel() if fm else np.zeros(ix.size, np.float32)
    if C == 1:
        sens = np.ones((1, ix.size), np.complex64)
    else:
        sens = synth.coil_maps(shape, C, rng).reshape(C, -1)
    return dict(kx=kx, ky=ky, kz=kz, t=t, ix=ix, iy=iy, iz=iz, fm=f.astype(np.float32),
                sens=sens, dims=(nx, ny, nz), opts=dict(use_z=int(nz > 1)))


@pytest.mark.parametrize("name", ["ops_2d", "ops_2d_c3"])
def test_ops_match_reference_fp64_golden(pkg, ctx, name):
    from gpu_util import gpu_ft, gpu_ift
    c = golden(name)
    assert oracle.rel_l2(gpu_ft(pkg, ctx, c, c["x"]), c["ft64"]) < TOL_OP
    assert oracle.rel_l2(gpu_ift(pkg, ctx, c, c["d"]), c["ift64"]) < TOL_OP


@pytest.mark.parametrize("C", [1, 2, 3, 4, 5, 8, 9])
def test_coil_groups_2d(pkg, ctx, synth, C):
    from gpu_util import gpu_ft, gpu_ift
    c = case_nd(synth, 32, 32, 1, C, 1000, seed=C)
    rng = np.random.default_rng(C)
    x = rng.standard_normal(1024) + 1j * rng.standard_normal(1024)
    d = rng.standard_normal((C, 1000)) + 1j * rng.standard_normal((C, 1000))
    assert oracle.rel_l2(gpu_ft(pkg, ctx, c, x), oracle.ft(x, c, use_z=0)) < TOL_OP
    assert oracle.rel_l2(gpu_ift(pkg, ctx, c, d), oracle.ift(d, c, use_z=0)) < TOL_OP


@pytest.mark.parametrize("C", [1, 4])
def test_3d_phase_with_z(pkg, ctx, synth, C):
    from gpu_util import gpu_ft, gpu_ift
    c = case_nd(synth, 16, 16, 8, C, 3000, seed=10 + C)
    rng = np.random.default_rng(C)
    N = c["ix"].size
    x = rng.standard_normal(N) + 1j * rng.standard_normal(N)
    d = rng.standard_normal((C, 3000)) + 1j * rng.standard_normal((C, 3000))
    assert oracle.rel_l2(gpu_ft(pkg, ctx, c, x, use_z=1), oracle.ft(x, c, use_z=1)) < TOL_OP
    assert oracle.rel_l2(gpu_ift(pkg, ctx, c, d, use_z=1), oracle.ift(d, c, use_z=1)) < TOL_OP


@pytest.mark.parametrize("M,N", [(1, 1), (7, 5), (1025, 3), (3, 2049)])
def test_ragged_sizes(pkg, ctx, M, N):
    rng = np.random.default_rng(M * 31 + N)
    c = dict(kx=rng.uniform(-16, 16, M).astype(np.float32),
             ky=rng.uniform(-16, 16, M).astype(np.float32),
             kz=np.zeros(M, np.float32), t=rng.uniform(0, 0.01, M).astype(np.float32),
             ix=rng.uniform(-0.5, 0.5, N).astype(np.float32),
             iy=rng.uniform(-0.5, 0.5, N).astype(np.float32), iz=np.zeros(N, np.float32),
             fm=rng.uniform(-300, 300, N).astype(np.float32), sens=np.ones((1, N), np.complex64),
             opts=dict(use_z=0))
    from gpu_util import gpu_ft, gpu_ift
    x = rng.standard_normal(N) + 1j * rng.standard_normal(N)
    d = rng.standard_normal(M) + 1j * rng.standard_normal(M)
    assert oracle.rel_l2(gpu_ft(pkg, ctx, c, x), oracle.ft(x, c, use_z=0)) < TOL_OP
    assert oracle.rel_l2(gpu_ift(pkg, ctx, c, d), oracle.ift(d, c, use_z=0)) < TOL_OP


def test_no_field_map_pointer(pkg, ctx, synth):
    from gpu_util import gpu_ft
    c = case_nd(synth, 32, 32, 1, 1, 512, seed=3)
    x = np.random.default_rng(0).standard_normal(1024) + 0j
    c0 = dict(c, fm=np.zeros_like(c["fm"]))
    assert oracle.rel_l2(gpu_ft(pkg, ctx, c, x, fm=False), oracle.ft(x, c0, use_z=0)) < TOL_OP


def test_out_of_range_coordinates_are_reported(pkg, ctx, synth):
    from gpu_util import gpu_ft
    c = case_nd(synth, 16, 16, 1, 1, 64, seed=4)
    c["kx"] = c["kx"].copy()
    c["kx"][3] = 1e6
    with pytest.raises(pkg.ImpError) as e:
        gpu_ft(pkg, ctx, c, np.ones(256, np.complex64))
    assert e.value.status == 5


def test_deterministic(pkg, ctx, synth):
    from gpu_util import gpu_ft
    c = case_nd(synth, 32, 32, 1, 4, 2000, seed=5)
    x = np.random.default_rng(1).standard_normal(1024) + 0j
    a = gpu_ft(pkg, ctx, c, x)
    b = gpu_ft(pkg, ctx, c, x)
    assert np.array_equal(a, b)


def test_full_size_3d_adjoint_and_linearity(pkg, ctx, synth):
    """At the benchmark size (64x64x16, 4 coils, M = 65536): adjoint identity
    <F x, y> = <x, F^H y> and linearity, which hold independent of size."""
    from gpu_util import gpu_ft, gpu_ift
    case = synth.make_case("bf3d_64x64x16")
    rng = np.random.default_rng(7)
    N, M, C = case["N"], case["M"], case["num_coil"]
    x = rng.standard_normal(N) + 1j * rng.standard_normal(N)
    x2 = rng.standard_normal(N) + 1j * rng.standard_normal(N)
    y = rng.standard_normal((C, M)) + 1j * rng.standard_normal((C, M))
    Fx = gpu_ft(pkg, ctx, case, x, use_z=1)
    Fhy = gpu_ift(pkg, ctx, case, y, use_z=1)
    lhs, rhs = np.vdot(y, Fx), np.vdot(Fhy, x)
    assert abs(lhs - rhs) / abs(lhs) < 1e-5
    Fx2 = gpu_ft(pkg, ctx, case, x2, use_z=1)
    Fs = gpu_ft(pkg, ctx, case, 0.5 * x - 2.0 * x2, use_z=1)
    assert oracle.rel_l2(Fs, 0.5 * Fx - 2.0 * Fx2) < 1e-5
    # spot check of 64 samples against the FP64 oracle at full N
    sel = rng.choice(M, 64, replace=False)
    sub = dict(case, kx=case["kx"][sel], ky=case["ky"][sel], kz=case["kz"][sel],
               t=case["t"][sel])
    assert oracle.rel_l2(Fx[:, sel], oracle.ft(x, sub, use_z=1)) < TOL_OP

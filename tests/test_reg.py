"""-reg (roughness regularization with a sparse matrix) on the CPU: the
Matrix Market I/O of c.rmtx, the roughness-matrix generator (restating
matlab_utils/create_sparse_matrix) against the FP64 oracle's finite-difference
stencil, and -- where the reference's CPU build is present -- the reference's
own bruteForceCpu with -reg against its -fd run and the committed fixture."""
import numpy as np
import pytest

import oracle
from conftest import golden
from oracle import toeplitz as T


def dense(R, N, I, J, V):
    C = np.zeros((R, N))
    np.add.at(C, (np.asarray(I), np.asarray(J)), np.asarray(V))
    return C


@pytest.mark.parametrize("shape", [(16, 12), (8, 6, 5), (32, 32)])
def test_fd_matrix_equals_the_stencil(synth, shape):
    """C^T W C x of the generated matrix = D^H W D x of the periodic stencil
    (DHWD2dCpu / DHWD3dGpu_toeplitz semantics) to FP64 rounding."""
    R, N, I, J, V = synth.fd_matrix(shape)
    assert N == np.prod(shape) and R == len(shape) * N
    rng = np.random.default_rng(len(shape))
    x = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    w = rng.uniform(0.5, 2.0, shape)
    got = T.reg_penalty(x, (R, N, I, J, V), w, 0.7)
    want = T.dhwd(x, w, 0.7)
    assert np.abs(got - want).max() < 1e-12 * np.abs(want).max()
    C = dense(R, N, I, J, V)
    assert np.allclose((C.T @ (np.tile(w.ravel(), len(shape)) * (C @ x.ravel()))).reshape(shape)
                       * 0.7, want)


def test_mtx_round_trip(tmp_path, pkg):
    from impatient_mri_b200 import io as mio
    rng = np.random.default_rng(0)
    I = rng.integers(0, 40, 100)
    J = rng.integers(0, 20, 100)
    V = rng.standard_normal(100)
    fn = tmp_path / "c.rmtx"
    mio.write_mtx(fn, 40, 20, I, J, V)
    assert fn.read_text().startswith("%%MatrixMarket matrix coordinate real general\n40 20 100\n")
    rows, cols, I2, J2, V2 = mio.read_mtx(fn)
    assert (rows, cols) == (40, 20)
    assert np.array_equal(I, I2) and np.array_equal(J, J2) and np.array_equal(V, V2)


def test_reg_fixture_shape():
    c = golden("bf_2d_reg")
    N = c["ix"].size
    assert int(c["C_cols"]) == N and int(c["C_rows"]) == 2 * N
    assert np.all(c["C_I"] < 2 * N) and np.all(c["C_J"] < N)


@pytest.mark.skipif(not oracle.ref_available("bf64"), reason="reference CPU build absent")
def test_reference_reg_equals_reference_fd(synth):
    """The reference's bruteForceCpu with -reg and the generated difference
    matrix gives exactly its -fd result (with TV reweighting): the generator
    restates the matrix the reference's own scripts make."""
    import sys
    from pathlib import Path
    sys.path.insert(0, str(Path(__file__).parent / "golden"))
    from gen_golden import small_case
    case, _ = small_case(32, 1, 4, 256, 31)
    R = synth.fd_matrix((32, 32))
    a = oracle.ref_bf_cg_reg(case, R, kind="bf64", cg_num=5, lam=1e-2, tv=True, tv_num=2)
    b = oracle.ref_bf_cg(case, kind="bf64", cg_num=5, lam=1e-2, tv=True, tv_num=2)
    assert oracle.rel_l2(a, b) < 1e-13


@pytest.mark.skipif(not oracle.ref_available("bf64"), reason="reference CPU build absent")
def test_reg_fixture_reproduced_by_reference():
    c = golden("bf_2d_reg")
    reg = (int(c["C_rows"]), int(c["C_cols"]), c["C_I"], c["C_J"], c["C_V"])
    x = oracle.ref_bf_cg_reg(c, reg, kind="bf64", cg_num=int(c["cg_num"]), lam=float(c["lam"]),
                             tv=True, tv_num=int(c["tv_num"]))
    assert oracle.rel_l2(x, c["x64"]) < 1e-13

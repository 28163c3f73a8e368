"""The Toeplitz oracle (oracle/toeplitz.py) pinned to the reference's own
Toeplitz outputs, and host-side checks of the Toeplitz C-ABI (no GPU).

The golden files hold the reference GPU program's Q_stone.file, FhD.file and
out.file for two seeded 2-D cases (tests/golden/gen_toeplitz_golden.py)."""
import ctypes

import numpy as np
import pytest

from conftest import GOLDEN
from oracle import toeplitz as T

TOL_OP = 1e-5   # operator outputs against the reference's FP32 GPU program
TOL_IMG = 1e-4  # final image


def load(name):
    z = np.load(GOLDEN / f"{name}.npz")
    c = {k: z[k] for k in z.files}
    f = [str(x) for x in c["flags"]]
    val = lambda k, d=None: f[f.index(k) + 1] if k in f else d
    c["L"] = int(float(val("-ntime_segs")))
    c["os_q"] = float(val("-gridOS_Q"))
    c["os_fh"] = float(val("-gridOS_FH"))
    c["cg"] = int(val("-cg_num"))
    c["fdp"] = float(val("-fdp"))
    c["tv_num"] = int(val("-tv_num", 0))
    c["dims"] = tuple(int(v) for v in c["dims"])
    return c


def rel(a, b):
    return float(np.linalg.norm(np.ravel(a) - np.ravel(b)) / np.linalg.norm(np.ravel(b)))


@pytest.mark.parametrize("name", ["toep_2d_fd", "toep_2d_tv"])
def test_oracle_q_matches_reference(name):
    c = load(name)
    Q = T.compute_q(c["kx"], c["ky"], c["kz"], c["t"], c["dims"], c["L"], c["os_q"])
    assert rel(Q.reshape(c["L"] + 1, -1), c["Q"]) < TOL_OP


@pytest.mark.parametrize("name", ["toep_2d_fd", "toep_2d_tv"])
def test_oracle_fhd_matches_reference(name):
    c = load(name)
    fhd = T.compute_fhd(c["kx"], c["ky"], c["kz"], c["t"], c["dims"], c["L"], c["os_fh"],
                        c["kdata"], c["sens"], c["fm"])
    assert rel(fhd, c["fhd"]) < TOL_OP


@pytest.mark.parametrize("name", ["toep_2d_fd", "toep_2d_tv"])
def test_oracle_cg_matches_reference(name):
    """CG from the reference's own Q and F^H d: cg_num updates, reconBest,
    x carried across TV passes."""
    c = load(name)
    n = c["dims"][0]
    fhd = c["fhd"].astype(np.complex128).reshape(n, n)
    Q = c["Q"].astype(np.complex128).reshape(c["L"] + 1, 2 * n, 2 * n)
    x = T.toeplitz_cg(fhd, Q, c["sens"], c["fm"], c["t"], c["L"], c["cg"], lam=c["fdp"],
                      tv=c["tv_num"] > 0, tv_num=max(c["tv_num"], 1))
    assert rel(x, c["out"]) < TOL_OP * 5


def test_gridded_q_equals_direct_q_at_os2():
    """Known answer: Q_l(r) = sum_k h_l(t_k) exp(+i 2 pi k.r) on the 2N grid;
    KB gridding at oversampling 2 reproduces it to about 1e-5."""
    c = load("toep_2d_fd")
    n, L = c["dims"][0], c["L"]
    Qg = T.compute_q(c["kx"], c["ky"], c["kz"], c["t"], c["dims"], L, 2.0).reshape(L + 1, -1)
    x = np.arange(-n, n) / n
    X, Y = np.meshgrid(x, x, indexing="ij")
    ph = np.exp(2j * np.pi * (np.outer(X.ravel(), c["kx"]) + np.outer(Y.ravel(), c["ky"])))
    tau, t0 = T.time_segments(c["t"], L)
    for l in range(L + 1):
        assert rel(Qg[l], ph @ T.hanning(c["t"], tau, l, t0)) < 5e-5


def test_fhf_is_the_normal_operator_without_field_map():
    """With one coil, no field map and one segment, A^H A p from Q equals the
    direct F^H F p (exact NUDFT pair) when Q is the direct one."""
    rng = np.random.default_rng(5)
    n, M = 8, 40
    kx = rng.uniform(-n / 2, n / 2, M)
    ky = rng.uniform(-n / 2, n / 2, M)
    ax = (np.arange(n) - n // 2) / n
    X, Y = np.meshgrid(ax, ax, indexing="ij")
    F = np.exp(-2j * np.pi * (np.outer(kx, X.ravel()) + np.outer(ky, Y.ravel())))
    x2 = np.arange(-n, n) / n
    X2, Y2 = np.meshgrid(x2, x2, indexing="ij")
    Q = (np.exp(2j * np.pi * (np.outer(X2.ravel(), kx) + np.outer(Y2.ravel(), ky)))
         @ np.ones(M)).reshape(1, 2 * n, 2 * n)
    p = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    got = T.aha(p, T.qf_from_q(Q), np.ones((1, n, n)), np.zeros((n, n)), 0.0, 0.0)
    want = (F.conj().T @ (F @ p.ravel())).reshape(n, n)
    assert rel(got, want) < 1e-12


# ---------------------------------------------------------------- C-ABI host side

def test_toeplitz_options_default(pkg):
    o = pkg.toeplitz_options()
    ref = pkg.ToepOptions()
    pkg.lib().imp_toeplitz_options_default(ctypes.byref(ref))
    assert (ref.cg_num, ref.tv_num, ref.enable_fd, ref.enable_tv) == (8, 10, 0, 0)
    assert ref.ntime_segs == 12.0 and ref.gridOS_Q == 1.125 and ref.gridOS_FH == 1.5
    assert abs(ref.tv_eps - 1e-6) < 1e-12
    assert o.cg_num == 8


@pytest.mark.parametrize("dims,osq,osf,msg", [
    ((31, 32, 1), 1.125, 1.5, "even"),
    ((32, 32, 1), 0.5, 1.5, "oversampling"),
    ((32, 32, 1), 1.125, 2.5, "oversampling"),
    ((0, 32, 1), 1.125, 1.5, "> 0"),
])
def test_toeplitz_q_rejects_bad_arguments_before_touching_a_gpu(pkg, dims, osq, osf, msg):
    """Argument checks run before any device work, so a NULL context is never
    dereferenced here."""
    o = pkg.toeplitz_options(gridOS_Q=osq, gridOS_FH=osf)
    a = np.zeros(16, np.float32)
    L = pkg.lib()
    st = L.imp_toeplitz_q(None, ctypes.byref(o), a.ctypes.data, a.ctypes.data, a.ctypes.data,
                          a.ctypes.data, a.ctypes.data, a.ctypes.data, 16, *dims)
    assert st == 1  # IMP_ERR_INVALID_ARG
    assert msg in L.imp_last_error().decode()

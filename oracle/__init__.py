"""TEST INFRASTRUCTURE ONLY: the CPU oracle of the reconstruction path.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline and
reference legs may import this package, and only as the checker.

Three layers:
  * ``ref``     -- the reference's own CPU brute-force code (bruteForceCpu,
                  parallelFtCpu, parallelIftCpu, DHWD2dCpu) compiled from the
                  reference sources by ``build_ref.sh`` into ``_ref/``; FP64
                  (pinning), FP32 and FP32+OpenMP builds.
  * ``orc``     -- liboracle.so, the FP64 C restatement in oracle.c (adds the
                  3-D phase and 3-D TV the reference brute force lacks).
  * ``toeplitz`` (oracle/toeplitz.py) -- numpy FP64 restatement of the
                  Toeplitz path, which has no CPU code in the reference.
"""
from __future__ import annotations

import ctypes
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REF_DIR = HERE / "_ref"
_P = ctypes.POINTER(ctypes.c_double)


def build(ref: bool = True) -> None:
    """Builds liboracle.so, and the reference CPU libraries when the reference
    sources are present (build_ref.sh skips otherwise)."""
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    if ref:
        subprocess.run(["bash", str(HERE / "build_ref.sh")], check=True,
                       stdout=subprocess.DEVNULL)


def _d(a):
    a = np.ascontiguousarray(a, dtype=np.float64)
    return a, a.ctypes.data_as(_P)


class _Lib:
    def __init__(self, path: Path):
        if not path.exists():
            raise FileNotFoundError(f"{path} not built (python -c 'import oracle; oracle.build()')")
        self.path = path
        self.L = ctypes.CDLL(str(path))


_orc = None
_refs: dict = {}


def orc() -> ctypes.CDLL:
    global _orc
    if _orc is None:
        _orc = _Lib(HERE / "liboracle.so").L
    return _orc


def ref_available(kind: str = "bf64") -> bool:
    return (REF_DIR / f"libref_{kind}.so").exists()


def ref(kind: str = "bf64") -> ctypes.CDLL:
    """kind: bf64 (FP64 pinning build), bf32, bf32_omp."""
    if kind not in _refs:
        L = _Lib(REF_DIR / f"libref_{kind}.so").L
        L.ref_bf_recon_dir.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_int,
                                       ctypes.c_double, ctypes.c_int, ctypes.c_int, _P, _P,
                                       ctypes.c_int]
        L.ref_dir_dims.argtypes = [ctypes.c_char_p] + [ctypes.POINTER(ctypes.c_int)] * 4
        L.ref_dhwd2d.argtypes = [_P] * 5 + [ctypes.c_int, ctypes.c_int, ctypes.c_double]
        _refs[kind] = L
    return _refs[kind]


def _traj(case):
    return [_d(case[k]) for k in ("kx", "ky", "kz", "t", "ix", "iy", "iz")]


def _sens(sens, C, N):
    s = np.asarray(sens).reshape(C, N)
    return _d(s.real.ravel()), _d(s.imag.ravel())


# ---------------------------------------------------------------- oracle.c --

def ft(x, case, use_z=None, sens=None):
    """FP64 y[c][k] = sum_r S_c x e^{-i theta}  (oracle.c orc_ft)."""
    use_z = case["opts"]["use_z"] if use_z is None else use_z
    M, N = case["kx"].size, case["ix"].size
    s = case["sens"] if sens is None else sens
    C = np.asarray(s).size // N
    (kx, pkx), (ky, pky), (kz, pkz), (t, pt), (ix, pix), (iy, piy), (iz, piz) = _traj(case)
    fm, pfm = _d(case["fm"])
    (sr, psr), (si, psi) = _sens(s, C, N)
    xr, pxr = _d(np.real(x))
    xi, pxi = _d(np.imag(x))
    out_r = np.zeros(C * M)
    out_i = np.zeros(C * M)
    orc().orc_ft(out_r.ctypes.data_as(_P), out_i.ctypes.data_as(_P), pxr, pxi, pkx, pky, pkz, pt,
                 pix, piy, piz, pfm, psr, psi, M, N, C, int(use_z))
    return (out_r + 1j * out_i).reshape(C, M)


def ift(d, case, use_z=None, sens=None):
    """FP64 x[r] = sum_c conj(S_c) sum_k d_c e^{+i theta}  (oracle.c orc_ift)."""
    use_z = case["opts"]["use_z"] if use_z is None else use_z
    M, N = case["kx"].size, case["ix"].size
    s = case["sens"] if sens is None else sens
    C = np.asarray(s).size // N
    (kx, pkx), (ky, pky), (kz, pkz), (t, pt), (ix, pix), (iy, piy), (iz, piz) = _traj(case)
    fm, pfm = _d(case["fm"])
    (sr, psr), (si, psi) = _sens(s, C, N)
    d = np.asarray(d).reshape(C * M)
    dr, pdr = _d(d.real)
    di, pdi = _d(d.imag)
    out_r = np.zeros(N)
    out_i = np.zeros(N)
    orc().orc_ift(out_r.ctypes.data_as(_P), out_i.ctypes.data_as(_P), pdr, pdi, pkx, pky, pkz,
                  pt, pix, piy, piz, pfm, psr, psi, M, N, C, int(use_z))
    return out_r + 1j * out_i


def tv_grid(case):
    nx, ny, nz = case["dims"]
    if case["opts"].get("use_z", 0) and nz > 1:
        return (ny, nx, nz)
    n = int(round(np.sqrt(case["ix"].size)))
    return (n, n, 1)


def dhwd(p, w, grid, lam):
    p = np.asarray(p)
    pr, ppr = _d(p.real)
    pi, ppi = _d(p.imag)
    ww, pw = _d(w)
    sr = np.zeros(p.size)
    si = np.zeros(p.size)
    orc().orc_dhwd(sr.ctypes.data_as(_P), si.ctypes.data_as(_P), ppr, ppi, pw, *grid,
                   ctypes.c_double(lam))
    return sr + 1j * si


def tv_weight(x, grid, eps):
    x = np.asarray(x)
    xr, pxr = _d(x.real)
    xi, pxi = _d(x.imag)
    w = np.zeros(x.size)
    orc().orc_tv_weight(w.ctypes.data_as(_P), pxr, pxi, *grid, ctypes.c_double(eps))
    return w


def bf_cg(case, x0=None, kdata=None, cg_num=None, lam=None, tv=None, tv_num=None, eps=1e-6,
          use_z=None):
    """FP64 brute-force CG (oracle.c orc_bf_cg, bruteForceCpu.cpp:121-528)."""
    o = case["opts"]
    use_z = o["use_z"] if use_z is None else use_z
    cg_num = o["cg_num"] if cg_num is None else cg_num
    lam = o.get("fd_penalizer") if lam is None else lam
    tv = o.get("tv", False) if tv is None else tv
    tv_num = o.get("tv_num", 1) if tv_num is None else tv_num
    M, N = case["kx"].size, case["ix"].size
    C = case["sens"].size // N
    (kx, pkx), (ky, pky), (kz, pkz), (t, pt), (ix, pix), (iy, piy), (iz, piz) = _traj(case)
    fm, pfm = _d(case["fm"])
    (sr, psr), (si, psi) = _sens(case["sens"], C, N)
    y = (case["kdata"] if kdata is None else kdata).reshape(C * M)
    yr, pyr = _d(y.real)
    yi, pyi = _d(y.imag)
    x0 = np.zeros(N, np.complex128) if x0 is None else np.asarray(x0, np.complex128)
    xr = np.ascontiguousarray(x0.real.copy())
    xi = np.ascontiguousarray(x0.imag.copy())
    grid = tv_grid(dict(case, opts=dict(o, use_z=use_z)))
    orc().orc_bf_cg(xr.ctypes.data_as(_P), xi.ctypes.data_as(_P), pyr, pyi, pkx, pky, pkz, pt,
                    pix, piy, piz, pfm, psr, psi, M, N, C, int(use_z), *grid, int(cg_num),
                    1 if lam is not None else 0, ctypes.c_double(lam or 0.0), 1 if tv else 0,
                    int(tv_num if tv else 1), ctypes.c_double(eps))
    return xr + 1j * xi


# ------------------------------------------------------- reference builds --

def ref_parallel_ft(x, case, kind="bf64"):
    L = ref(kind)
    M, N = case["kx"].size, case["ix"].size
    C = case["sens"].size // N
    (kx, pkx), (ky, pky), (kz, pkz), (t, pt), (ix, pix), (iy, piy), (iz, piz) = _traj(case)
    fm, pfm = _d(case["fm"])
    (sr, psr), (si, psi) = _sens(case["sens"], C, N)
    xr, pxr = _d(np.real(x))
    xi, pxi = _d(np.imag(x))
    out_r = np.zeros(C * M)
    out_i = np.zeros(C * M)
    L.ref_parallel_ft(out_r.ctypes.data_as(_P), out_i.ctypes.data_as(_P), pxr, pxi, pkx, pky,
                      pkz, pix, piy, piz, pfm, pt, M, N, psr, psi, C)
    return (out_r + 1j * out_i).reshape(C, M)


def ref_parallel_ift(d, case, kind="bf64"):
    L = ref(kind)
    M, N = case["kx"].size, case["ix"].size
    C = case["sens"].size // N
    (kx, pkx), (ky, pky), (kz, pkz), (t, pt), (ix, pix), (iy, piy), (iz, piz) = _traj(case)
    fm, pfm = _d(case["fm"])
    (sr, psr), (si, psi) = _sens(case["sens"], C, N)
    d = np.asarray(d).reshape(C * M)
    dr, pdr = _d(d.real)
    di, pdi = _d(d.imag)
    out_r = np.zeros(N)
    out_i = np.zeros(N)
    L.ref_parallel_ift(out_r.ctypes.data_as(_P), out_i.ctypes.data_as(_P), pdr, pdi, pkx, pky,
                       pkz, pix, piy, piz, pfm, pt, M, N, psr, psi, C)
    return out_r + 1j * out_i


def ref_bf_cg(case, x0=None, kind="bf64", cg_num=None, lam=None, tv=None, tv_num=None):
    L = ref(kind)
    o = case["opts"]
    cg_num = o["cg_num"] if cg_num is None else cg_num
    lam = o.get("fd_penalizer") if lam is None else lam
    tv = o.get("tv", False) if tv is None else tv
    tv_num = o.get("tv_num", 1) if tv_num is None else tv_num
    M, N = case["kx"].size, case["ix"].size
    C = case["sens"].size // N
    (kx, pkx), (ky, pky), (kz, pkz), (t, pt), (ix, pix), (iy, piy), (iz, piz) = _traj(case)
    fm, pfm = _d(case["fm"])
    (sr, psr), (si, psi) = _sens(case["sens"], C, N)
    y = case["kdata"].reshape(C * M)
    yr, pyr = _d(y.real)
    yi, pyi = _d(y.imag)
    x0 = np.zeros(N, np.complex128) if x0 is None else np.asarray(x0, np.complex128)
    xr = np.ascontiguousarray(x0.real.copy())
    xi = np.ascontiguousarray(x0.imag.copy())
    L.ref_bf_cg(xr.ctypes.data_as(_P), xi.ctypes.data_as(_P), pyr, pyi, pkx, pky, pkz, pix, piy,
                piz, pfm, pt, M, N, psr, psi, C, int(cg_num), 1 if lam is not None else 0,
                ctypes.c_double(lam or 0.0), 1 if tv else 0, int(tv_num if tv else 1))
    return xr + 1j * xi


def ref_bf_cg_reg(case, reg, kind="bf64", cg_num=None, lam=0.0, tv=False, tv_num=1):
    """The reference's bruteForceCpu with -reg: reg = (rows, cols, I, J, V),
    0-based coordinates of the roughness matrix C."""
    L = ref(kind)
    rows, cols, I, J, V = reg
    o = case["opts"]
    cg_num = o["cg_num"] if cg_num is None else cg_num
    M, N = case["kx"].size, case["ix"].size
    C = case["sens"].size // N
    (kx, pkx), (ky, pky), (kz, pkz), (t, pt), (ix, pix), (iy, piy), (iz, piz) = _traj(case)
    fm, pfm = _d(case["fm"])
    (sr, psr), (si, psi) = _sens(case["sens"], C, N)
    y = case["kdata"].reshape(C * M)
    yr, pyr = _d(y.real)
    yi, pyi = _d(y.imag)
    xr = np.zeros(N)
    xi = np.zeros(N)
    Ii = np.ascontiguousarray(I, np.int32)
    Jj = np.ascontiguousarray(J, np.int32)
    Vv, pv = _d(V)
    IP = ctypes.POINTER(ctypes.c_int)
    L.ref_bf_cg_reg(xr.ctypes.data_as(_P), xi.ctypes.data_as(_P), pyr, pyi, pkx, pky, pkz, pix,
                    piy, piz, pfm, pt, M, N, psr, psi, C, int(cg_num), ctypes.c_double(lam),
                    1 if tv else 0, int(tv_num if tv else 1), int(rows), int(cols), int(Ii.size),
                    Ii.ctypes.data_as(IP), Jj.ctypes.data_as(IP), pv)
    return xr + 1j * xi


def ref_recon_dir(idir, cg_num, lam=None, tv=False, tv_num=10, kind="bf64"):
    L = ref(kind)
    nk, ni, nc, ns = (ctypes.c_int() for _ in range(4))
    L.ref_dir_dims(str(idir).encode(), *(ctypes.byref(v) for v in (nk, ni, nc, ns)))
    n = ni.value * ns.value
    out_r = np.zeros(n)
    out_i = np.zeros(n)
    L.ref_bf_recon_dir(str(idir).encode(), int(cg_num), 1 if lam is not None else 0,
                       float(lam or 0.0), 1 if tv else 0, int(tv_num), out_r.ctypes.data_as(_P),
                       out_i.ctypes.data_as(_P), n)
    return out_r + 1j * out_i


def rel_l2(a, b) -> float:
    a = np.asarray(a, np.complex128).ravel()
    b = np.asarray(b, np.complex128).ravel()
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))

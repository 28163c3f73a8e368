"""Python binding of the IMPATIENT MRI B200 C-ABI (include/impatient_b200.h).

The product is the sm_100a shared library ``libimpatient_b200.so`` and the
``bin/mriSolver`` executable next to this file.  This module loads the library
with ctypes and exposes the reference's operator and recon entry points under
their reference names, on torch CUDA tensors (device pointers) or numpy
arrays (host pointers).  There is no CPU fallback: if the library is missing
or no GPU is visible, the calls raise.

Names mirror the reference:
    ftGpu / iftGpu                  kernels/ftGpu.cu:198, :653
    parallelFtGpu / parallelIftGpu  kernels/parImagingGpu.cu:92, :119
    bruteForceGpu                   bruteForce/bruteForceGpu.cuh:72-86
    bruteForce                      main_mri.cuh:110-118 (directory level)
    mriSolver                       main.cpp:103 (command line)
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

import numpy as np

PKG_DIR = Path(__file__).resolve().parent
LIB_PATH = PKG_DIR / "libimpatient_b200.so"
MRISOLVER = PKG_DIR / "bin" / "mriSolver"

IMP_OK = 0
STATUS_NAMES = {
    0: "IMP_OK", 1: "IMP_ERR_INVALID_ARG", 2: "IMP_ERR_CUDA", 3: "IMP_ERR_IO",
    4: "IMP_ERR_FORMAT", 5: "IMP_ERR_RANGE", 6: "IMP_ERR_NOMEM", 7: "IMP_ERR_TIMEOUT",
    8: "IMP_ERR_UNSUPPORTED",
}

# Every symbol include/impatient_b200.h declares (checked by the CPU tests).
EXPORTED = [
    "imp_abi_version", "imp_status_string", "imp_last_error",
    "imp_context_create", "imp_context_destroy", "imp_context_synchronize",
    "imp_context_launch_count", "imp_context_profile", "imp_context_profile_read",
    "imp_check_wait_expiry",
    "imp_ft", "imp_ift", "imp_parallel_ft", "imp_parallel_ift", "imp_parallel_ift_noalloc",
    "imp_bf_options_default", "imp_bruteforce_recon", "imp_bruteforce_dir",
    "imp_bruteforce_batch", "imp_bruteforce_mgpu",
    "imp_dataset_info", "imp_mrisolver_main", "imp_measure_alu_peaks",
    "imp_toeplitz_options_default", "imp_toeplitz_q", "imp_toeplitz_fhd", "imp_toeplitz_recon",
    "imp_grid_fft",
    "imp_toeplitz_apply", "imp_toeplitz_dir", "imp_toeplitz_cg",
    "imp_unet_create", "imp_unet_destroy", "imp_unet_num_params", "imp_unet_get_params",
    "imp_unet_set_params", "imp_unet_forward", "imp_unet_gradients", "imp_unet_train_step",
]


class ImpError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


class Sparse(ctypes.Structure):
    """imp_sparse: a real COO matrix (0-based) in host memory; keeps its arrays."""
    _fields_ = [
        ("rows", ctypes.c_int), ("cols", ctypes.c_int), ("nnz", ctypes.c_int),
        ("row", ctypes.POINTER(ctypes.c_int)), ("col", ctypes.POINTER(ctypes.c_int)),
        ("val", ctypes.POINTER(ctypes.c_float)),
    ]

    @classmethod
    def from_coo(cls, rows, cols, I, J, V):
        I = np.ascontiguousarray(I, np.int32)
        J = np.ascontiguousarray(J, np.int32)
        V = np.ascontiguousarray(V, np.float32)
        m = cls(int(rows), int(cols), int(I.size),
                I.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                J.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                V.ctypes.data_as(ctypes.POINTER(ctypes.c_float)))
        m._keep = (I, J, V)
        return m


class BfOptions(ctypes.Structure):
    _fields_ = [
        ("cg_num", ctypes.c_int), ("enable_fd", ctypes.c_int),
        ("fd_penalizer", ctypes.c_float), ("enable_tv", ctypes.c_int),
        ("tv_num", ctypes.c_int), ("tv_eps", ctypes.c_float), ("use_z", ctypes.c_int),
        ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
        ("reg", ctypes.POINTER(Sparse)),
    ]


class ToepOptions(ctypes.Structure):
    _fields_ = [
        ("cg_num", ctypes.c_int), ("enable_fd", ctypes.c_int),
        ("fd_penalizer", ctypes.c_float), ("enable_tv", ctypes.c_int),
        ("tv_num", ctypes.c_int), ("tv_eps", ctypes.c_float), ("ntime_segs", ctypes.c_float),
        ("gridOS_Q", ctypes.c_float), ("gridOS_FH", ctypes.c_float),
        ("reg", ctypes.POINTER(Sparse)),
    ]


_lib = None


def lib() -> ctypes.CDLL:
    """Loads the shared library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `python impatient-mri_b200/build.py`")
        L = ctypes.CDLL(str(LIB_PATH))
        vp, ip, fp = ctypes.c_void_p, ctypes.c_int, ctypes.c_float
        L.imp_last_error.restype = ctypes.c_char_p
        L.imp_status_string.restype = ctypes.c_char_p
        L.imp_status_string.argtypes = [ip]
        L.imp_context_create.argtypes = [ip, ctypes.POINTER(vp)]
        L.imp_context_destroy.argtypes = [vp]
        L.imp_context_synchronize.argtypes = [vp]
        L.imp_context_launch_count.argtypes = [vp]
        L.imp_check_wait_expiry.argtypes = [vp, ip]
        L.imp_context_launch_count.restype = ctypes.c_long
        L.imp_context_profile.argtypes = [vp, ip]
        L.imp_context_profile_read.argtypes = [vp, ip, ctypes.POINTER(ctypes.c_double),
                                               ctypes.POINTER(ctypes.c_long)]
        op = [vp] + [vp] * 4 + [vp] * 8 + [ip, ip]
        L.imp_ft.argtypes = op + [ip]
        L.imp_ift.argtypes = op + [ip]
        L.imp_parallel_ft.argtypes = op + [vp, vp, ip, ip]
        L.imp_parallel_ift.argtypes = op + [vp, vp, ip, ip]
        L.imp_parallel_ift_noalloc.argtypes = [vp] * 12 + [ip, ip, vp, vp, ip, ip, vp]
        L.imp_bf_options_default.argtypes = [ctypes.POINTER(BfOptions)]
        L.imp_bruteforce_recon.argtypes = ([vp, ctypes.POINTER(BfOptions)] + [vp] * 14
                                           + [ip, ip, ip, ip])
        L.imp_bruteforce_batch.argtypes = ([vp, ctypes.POINTER(BfOptions)] + [vp] * 8
                                           + [ctypes.POINTER(ip)] + [vp] * 6 + [ip, ip, ip])
        L.imp_bruteforce_mgpu.argtypes = ([ctypes.POINTER(BfOptions)] + [vp] * 14
                                          + [ip, ip, ip, ip, ctypes.POINTER(ip), ip])
        L.imp_bruteforce_dir.argtypes = [ctypes.c_char_p, ctypes.c_char_p,
                                         ctypes.POINTER(BfOptions), ip]
        L.imp_dataset_info.argtypes = [ctypes.c_char_p] + [ctypes.POINTER(ctypes.c_int)] * 7
        L.imp_mrisolver_main.argtypes = [ip, ctypes.POINTER(ctypes.c_char_p)]
        L.imp_measure_alu_peaks.argtypes = [ip, ctypes.POINTER(ctypes.c_double),
                                            ctypes.POINTER(ctypes.c_double)]
        TO = ctypes.POINTER(ToepOptions)
        L.imp_toeplitz_options_default.argtypes = [TO]
        L.imp_toeplitz_q.argtypes = [vp, TO] + [vp] * 6 + [ip] * 4
        L.imp_toeplitz_fhd.argtypes = [vp, TO] + [vp] * 11 + [ip] * 5
        L.imp_toeplitz_recon.argtypes = [vp, TO] + [vp] * 7 + [ip] + [vp] * 3 + [ip] * 4
        L.imp_toeplitz_apply.argtypes = [vp, TO] + [vp] * 7 + [ip] + [vp] * 3 + [ip] * 4
        L.imp_grid_fft.argtypes = [vp, vp, vp, ip, ip, ip, ip, ip]
        L.imp_toeplitz_dir.argtypes = [ctypes.c_char_p, TO, ip, ip, ip, ctypes.c_char_p, ip]
        L.imp_toeplitz_cg.argtypes = ([vp, TO] + [vp] * 7 + [ip] + [vp] * 3 + [ip] * 4
                                      + [ctypes.c_double, ip, ctypes.POINTER(ip)])
        L.imp_unet_create.argtypes = [vp, ip, ip, ip, ctypes.c_ulonglong, ctypes.POINTER(vp)]
        L.imp_unet_destroy.argtypes = [vp]
        L.imp_unet_destroy.restype = None
        L.imp_unet_num_params.argtypes = [vp]
        L.imp_unet_num_params.restype = ctypes.c_long
        L.imp_unet_get_params.argtypes = [vp, vp]
        L.imp_unet_set_params.argtypes = [vp, vp]
        L.imp_unet_forward.argtypes = [vp, vp, vp]
        L.imp_unet_gradients.argtypes = [vp, vp, vp, vp, ctypes.POINTER(fp)]
        L.imp_unet_train_step.argtypes = [vp, vp, vp, fp, ctypes.POINTER(fp)]
        _lib = L
    return _lib


def _check(status: int) -> None:
    if status != IMP_OK:
        raise ImpError(status, lib().imp_last_error().decode())


class Context:
    """An imp_context: one CUDA stream and the device work memory."""

    def __init__(self, device: int = 0):
        self._h = ctypes.c_void_p()
        _check(lib().imp_context_create(device, ctypes.byref(self._h)))
        self.device = device

    @property
    def handle(self):
        return self._h

    def launch_count(self) -> int:
        return int(lib().imp_context_launch_count(self._h))

    def check_wait_expiry(self, polls: int = 1000) -> None:
        """Runs a kernel whose bounded wait runs out; raises ImpError
        (IMP_ERR_TIMEOUT) as every expired wait does."""
        _check(lib().imp_check_wait_expiry(self._h, polls))

    def synchronize(self) -> None:
        _check(lib().imp_context_synchronize(self._h))

    def profile(self, enable: bool) -> None:
        """Per-launch NUDFT kernel timing of recon calls (disables graphs)."""
        _check(lib().imp_context_profile(self._h, int(enable)))

    def profile_read(self):
        """{'forward': (total_ms, launches), 'adjoint': (total_ms, launches)}"""
        out = {}
        for i, name in enumerate(("forward", "adjoint")):
            ms, n = ctypes.c_double(), ctypes.c_long()
            _check(lib().imp_context_profile_read(self._h, i, ctypes.byref(ms), ctypes.byref(n)))
            out[name] = (ms.value, n.value)
        return out

    def close(self) -> None:
        if self._h:
            lib().imp_context_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _ptr(a):
    """Device (torch CUDA tensor) or host (numpy / CPU tensor) float32 pointer."""
    if a is None:
        return None
    if hasattr(a, "data_ptr"):
        if a.dtype.__str__() != "torch.float32" or not a.is_contiguous():
            raise TypeError("tensors must be contiguous float32")
        return ctypes.c_void_p(a.data_ptr())
    if isinstance(a, np.ndarray):
        if a.dtype != np.float32 or not a.flags.c_contiguous:
            raise TypeError("arrays must be C-contiguous float32")
        return ctypes.c_void_p(a.ctypes.data)
    raise TypeError(f"unsupported array type {type(a)}")


def ftGpu(ctx, kdata_r, kdata_i, idata_r, idata_i, kx, ky, kz, ix, iy, iz, fm, t,
          num_k, num_i, use_z=0):
    _check(lib().imp_ft(ctx.handle, *map(_ptr, (kdata_r, kdata_i, idata_r, idata_i, kx, ky, kz,
                                                ix, iy, iz, fm, t)), num_k, num_i, use_z))


def iftGpu(ctx, idata_r, idata_i, kdata_r, kdata_i, kx, ky, kz, ix, iy, iz, fm, t,
           num_k, num_i, use_z=0):
    _check(lib().imp_ift(ctx.handle, *map(_ptr, (idata_r, idata_i, kdata_r, kdata_i, kx, ky, kz,
                                                 ix, iy, iz, fm, t)), num_k, num_i, use_z))


def parallelFtGpu(ctx, kdata_r, kdata_i, idata_r, idata_i, kx, ky, kz, ix, iy, iz, fm, t,
                  num_k, num_i, sensi_r, sensi_i, num_coil, use_z=0):
    _check(lib().imp_parallel_ft(ctx.handle, *map(_ptr, (kdata_r, kdata_i, idata_r, idata_i,
                                                         kx, ky, kz, ix, iy, iz, fm, t)),
                                 num_k, num_i, _ptr(sensi_r), _ptr(sensi_i), num_coil, use_z))


def parallelIftGpu(ctx, idata_r, idata_i, kdata_r, kdata_i, kx, ky, kz, ix, iy, iz, fm, t,
                   num_k, num_i, sensi_r, sensi_i, num_coil, use_z=0):
    _check(lib().imp_parallel_ift(ctx.handle, *map(_ptr, (idata_r, idata_i, kdata_r, kdata_i,
                                                          kx, ky, kz, ix, iy, iz, fm, t)),
                                  num_k, num_i, _ptr(sensi_r), _ptr(sensi_i), num_coil, use_z))


def bf_options(cg_num=8, fd_penalizer=None, tv=False, tv_num=10, tv_eps=1e-6, use_z=0,
               dims=None, reg=None) -> BfOptions:
    """Options of the brute-force recon; fd_penalizer enables the FD term
    (as -fdp does, main.cpp:306-316).  dims = (nx, ny, nz) sets the TV grid.
    reg: a Sparse roughness matrix C (-reg): lambda C^T W C replaces the FD
    term, lambda = fd_penalizer (0 when None, as the reference's default)."""
    o = BfOptions()
    lib().imp_bf_options_default(ctypes.byref(o))
    o.cg_num = cg_num
    o.enable_fd = 1 if fd_penalizer is not None else 0
    o.fd_penalizer = float(fd_penalizer or 0.0)
    o.enable_tv = 1 if tv else 0
    o.tv_num = tv_num
    o.tv_eps = float(tv_eps)
    o.use_z = int(use_z)
    if dims is not None:
        o.nx, o.ny, o.nz = (int(d) for d in dims)
    if reg is not None:
        o.reg = ctypes.pointer(reg)
        o._keep_reg = reg
    return o


def bruteForceGpu(ctx, opts: BfOptions, idata_r, idata_i, kdata_r, kdata_i, kx, ky, kz, ix, iy,
                  iz, fm, t, sensi_r, sensi_i, num_k, num_i, num_coil, num_slices=1):
    """In-place brute-force CG: idata_* hold the initial estimate and receive the image."""
    _check(lib().imp_bruteforce_recon(
        ctx.handle, ctypes.byref(opts), *map(_ptr, (idata_r, idata_i, kdata_r, kdata_i, kx, ky,
                                                    kz, ix, iy, iz, fm, t, sensi_r, sensi_i)),
        num_k, num_i, num_coil, num_slices))


def bruteForceBatch(ctx, opts: BfOptions, idata_r, idata_i, kdata_r, kdata_i, kx, ky, kz, t,
                    k_off, ix, iy, iz, fm, sensi_r, sensi_i, num_i, num_coil):
    """Slices with their own trajectories: k_off (num_slices+1 offsets into the
    concatenated kx/ky/kz/t); kdata slice-major, coil-major within a slice;
    idata/fm [slice][num_i].  idata_* hold the initial estimates and receive
    the images."""
    off = (ctypes.c_int * len(k_off))(*[int(v) for v in k_off])
    _check(lib().imp_bruteforce_batch(
        ctx.handle, ctypes.byref(opts), *map(_ptr, (idata_r, idata_i, kdata_r, kdata_i, kx, ky,
                                                    kz, t)),
        off, *map(_ptr, (ix, iy, iz, fm, sensi_r, sensi_i)), num_i, num_coil, len(k_off) - 1))


def bruteForceMgpu(opts: BfOptions, idata_r, idata_i, kdata_r, kdata_i, kx, ky, kz, ix, iy,
                   iz, fm, t, sensi_r, sensi_i, num_k, num_i, num_coil, num_slices,
                   devices=None) -> None:
    """-mgpu: the slices of bruteForceGpu spread over GPUs, one worker thread
    and context per entry of `devices` (None: every visible GPU).  Host
    arrays; idata_* receive the images."""
    dev = None
    n = 0
    if devices is not None:
        dev = (ctypes.c_int * len(devices))(*[int(d) for d in devices])
        n = len(devices)
    _check(lib().imp_bruteforce_mgpu(
        ctypes.byref(opts), *map(_ptr, (idata_r, idata_i, kdata_r, kdata_i, kx, ky, kz, ix, iy,
                                        iz, fm, t, sensi_r, sensi_i)),
        num_k, num_i, num_coil, num_slices, dev, n))


def bruteForce(idir: str, odir: str, opts: BfOptions, gpu_id: int = 0) -> None:
    _check(lib().imp_bruteforce_dir(os.fsencode(idir), os.fsencode(odir), ctypes.byref(opts),
                                    gpu_id))


def dataset_info(idir: str) -> dict:
    """Sizes of an input directory as the reference reader sees them (no GPU)."""
    v = [ctypes.c_int(0) for _ in range(7)]
    _check(lib().imp_dataset_info(os.fsencode(idir), *(ctypes.byref(x) for x in v)))
    keys = ("num_k", "num_i", "num_coil", "num_slices", "nx", "ny", "nz")
    return {k: x.value for k, x in zip(keys, v)}


def measure_alu_peaks(device: int = 0):
    """(FP32 FMA TFLOP/s, SFU sine G ops/s) measured on `device`."""
    f, s = ctypes.c_double(), ctypes.c_double()
    _check(lib().imp_measure_alu_peaks(device, ctypes.byref(f), ctypes.byref(s)))
    return f.value, s.value


def toeplitz_options(cg_num=8, fd_penalizer=None, tv=False, tv_num=10, tv_eps=1e-6,
                     ntime_segs=12.0, gridOS_Q=1.125, gridOS_FH=1.5, reg=None) -> ToepOptions:
    """Options of the Toeplitz recon; fd_penalizer enables the FD term, reg
    (a Sparse roughness matrix, -reg) replaces it by lambda C^T W C."""
    o = ToepOptions()
    lib().imp_toeplitz_options_default(ctypes.byref(o))
    o.cg_num = cg_num
    o.enable_fd = 1 if fd_penalizer is not None else 0
    o.fd_penalizer = float(fd_penalizer or 0.0)
    o.enable_tv = 1 if tv else 0
    o.tv_num = tv_num
    o.tv_eps = float(tv_eps)
    o.ntime_segs = float(ntime_segs)
    o.gridOS_Q = float(gridOS_Q)
    o.gridOS_FH = float(gridOS_FH)
    if reg is not None:
        o.reg = ctypes.pointer(reg)
        o._keep_reg = reg
    return o


def toeplitz_q(ctx, opts: ToepOptions, q_r, q_i, kx, ky, kz, t, num_k, nx, ny, nz=1):
    """Q_l for l = 0..L into q_r/q_i ((L+1) x 2N-grid floats each)."""
    _check(lib().imp_toeplitz_q(ctx.handle, ctypes.byref(opts),
                                *map(_ptr, (q_r, q_i, kx, ky, kz, t)), num_k, nx, ny, nz))


def toeplitz_fhd(ctx, opts: ToepOptions, fhd_r, fhd_i, kdata_r, kdata_i, kx, ky, kz, t, fm,
                 sensi_r, sensi_i, num_k, num_coil, nx, ny, nz=1):
    _check(lib().imp_toeplitz_fhd(
        ctx.handle, ctypes.byref(opts), *map(_ptr, (fhd_r, fhd_i, kdata_r, kdata_i, kx, ky, kz,
                                                    t, fm, sensi_r, sensi_i)),
        num_k, num_coil, nx, ny, nz))


def toeplitz_recon(ctx, opts: ToepOptions, x_r, x_i, fhd_r, fhd_i, q_r, q_i, t, num_k, fm,
                   sensi_r, sensi_i, num_coil, nx, ny, nz=1):
    _check(lib().imp_toeplitz_recon(
        ctx.handle, ctypes.byref(opts), *map(_ptr, (x_r, x_i, fhd_r, fhd_i, q_r, q_i, t)),
        num_k, _ptr(fm), _ptr(sensi_r), _ptr(sensi_i), num_coil, nx, ny, nz))


def toeplitz_apply(ctx, opts: ToepOptions, out_r, out_i, p_r, p_i, q_r, q_i, t, num_k, fm,
                   sensi_r, sensi_i, num_coil, nx, ny, nz=1):
    _check(lib().imp_toeplitz_apply(
        ctx.handle, ctypes.byref(opts), *map(_ptr, (out_r, out_i, p_r, p_i, q_r, q_i, t)),
        num_k, _ptr(fm), _ptr(sensi_r), _ptr(sensi_i), num_coil, nx, ny, nz))


def toeplitz(idir: str, opts: ToepOptions, direct=False, gpu_id=0, reuseQ=False, Qdir=None,
             writeQ=False) -> None:
    """Directory-level Toeplitz recon: writes idir/FhD.file, idir/out.file
    (and idir/Q_stone.file with writeQ)."""
    _check(lib().imp_toeplitz_dir(os.fsencode(idir), ctypes.byref(opts), int(direct), gpu_id,
                                  int(reuseQ), os.fsencode(Qdir) if Qdir else None,
                                  int(writeQ)))


def grid_fft(ctx, data_r, data_i, n0, n1, n2, batch=1, inverse=False):
    """In-place unnormalised complex FFT of `batch` n0 x n1 x n2 grids (n2
    fastest), split re/im float32 arrays (host numpy or CUDA tensors)."""
    _check(lib().imp_grid_fft(ctx.handle, _ptr(data_r), _ptr(data_i), int(n0), int(n1), int(n2),
                              int(batch), 1 if inverse else 0))


def toeplitz_cg(ctx, opts: ToepOptions, x_r, x_i, fhd_r, fhd_i, q_r, q_i, t, num_k, fm,
                sensi_r, sensi_i, num_coil, nx, ny, nz=1, tol=1e-4, max_iter=100) -> int:
    """CG from the image in x_r/x_i (overwritten with the result) to relative
    residual tol; returns the number of CG updates."""
    it = ctypes.c_int(0)
    _check(lib().imp_toeplitz_cg(
        ctx.handle, ctypes.byref(opts), *map(_ptr, (x_r, x_i, fhd_r, fhd_i, q_r, q_i, t)),
        num_k, _ptr(fm), _ptr(sensi_r), _ptr(sensi_i), num_coil, nx, ny, nz,
        float(tol), int(max_iter), ctypes.byref(it)))
    return it.value


class UNet:
    """The BF16 U-Net of the learned warm start (images [batch][2][H*W] float32)."""

    def __init__(self, ctx, batch: int, height: int, width: int, seed: int = 0):
        self._h = ctypes.c_void_p()
        self.ctx = ctx
        _check(lib().imp_unet_create(ctx.handle, batch, height, width, seed,
                                     ctypes.byref(self._h)))
        self.batch, self.height, self.width = batch, height, width

    def num_params(self) -> int:
        return int(lib().imp_unet_num_params(self._h))

    def get_params(self, out=None):
        out = np.zeros(self.num_params(), np.float32) if out is None else out
        _check(lib().imp_unet_get_params(self._h, _ptr(out)))
        return out

    def set_params(self, p):
        _check(lib().imp_unet_set_params(self._h, _ptr(p)))

    def forward(self, x, y):
        _check(lib().imp_unet_forward(self._h, _ptr(x), _ptr(y)))
        return y

    def gradients(self, x, target, grads=None):
        grads = np.zeros(self.num_params(), np.float32) if grads is None else grads
        loss = ctypes.c_float()
        _check(lib().imp_unet_gradients(self._h, _ptr(x), _ptr(target), _ptr(grads),
                                        ctypes.byref(loss)))
        return float(loss.value), grads

    def train_step(self, x, target, lr: float) -> float:
        loss = ctypes.c_float()
        _check(lib().imp_unet_train_step(self._h, _ptr(x), _ptr(target), float(lr),
                                         ctypes.byref(loss)))
        return float(loss.value)

    def close(self):
        if self._h:
            lib().imp_unet_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def mriSolver(*args: str) -> int:
    """Runs the mriSolver command line in-process; returns its exit code."""
    argv = [b"mriSolver"] + [os.fsencode(a) for a in args]
    arr = (ctypes.c_char_p * (len(argv) + 1))(*argv, None)
    return int(lib().imp_mrisolver_main(len(argv), arr))

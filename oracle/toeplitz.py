"""TEST INFRASTRUCTURE ONLY -- FP64 numpy restatement of the reference's
Toeplitz path (gridded Q and F^H d, FFT-based F^H F with time segmentation and
SENSE, Toeplitz CG with the best-residual iterate).  The reference has no CPU
code for this path; each function cites the reference lines it follows.

Conventions kept from the reference:
* single-precision parameter arithmetic (the oversampling rounding, beta and
  the grid sizes are computed in float32 exactly as the reference does);
* the grid of cell X covers shifted coordinate k' = OS (k + imageSize/2)
  (toeplitz/GPU_kernels.cu:78-86), cells outside [0, gridSize) do not exist;
* Kaiser-Bessel weight I0(beta sqrt(1 - (2d/W)^2)) / W for d = |k' - X| / OS
  <= W/2, W = 4, with I0 from the Abramowitz-Stegun 9.8.1-9.8.2 polynomial
  (toeplitz/GPU_kernels.cu:22-45, 270-300);
* Hanning time interpolators h_l(t) = 0.5 + 0.5 cos(pi (t - tau l - t0)/tau)
  for |t - tau l - t0| < tau (toeplitz/GPU_kernels.cu:49-65);
* inverse FFT unnormalised, half-rotation shifts (all sizes even), crop of the
  centre, deapodisation by the closed-form KB transform and 1/OS^d
  (toeplitz/gridding_utils.cu:60-205).
Reference quirk not reproduced: bins holding more than 128 samples are
gridded on the CPU with beta = 18.5547 and a wrong time index
(toeplitz/CPU_kernels.cpp:356,385); here every sample uses the GPU formula.
Axis order: images and grids are arrays [x, y] in 2-D (x slow, y fast) and
[y, x, z] in 3-D (z fastest), the reference's voxel order.
"""
from __future__ import annotations

import numpy as np

try:  # the same FP64 pocketfft transforms as numpy's, on all host threads
    import scipy.fft as _sfft

    def _fftn(a, axes=None):
        return _sfft.fftn(a, axes=axes, workers=-1)

    def _ifftn(a, axes=None):
        return _sfft.ifftn(a, axes=axes, workers=-1)
except ImportError:  # pragma: no cover
    _fftn = np.fft.fftn
    _ifftn = np.fft.ifftn

F32 = np.float32
PI32 = F32(3.1415926535897932384626433832795029)
KW = 4.0


def rounded_os(os: float, n_img: tuple) -> float:
    """gridOS rounding of computeQ.cmem.cu:439-446 / computeFH.cmem.cu:505-512:
    2-D -> even grid along x, 3-D -> grid along z divisible by four."""
    os = F32(os)
    if n_img[2] == 1:
        return float(F32(2.0) * F32(np.ceil(F32(os * F32(n_img[0])) / F32(2.0))) / F32(n_img[0]))
    return float(F32(4.0) * F32(np.ceil(F32(os * F32(n_img[2])) / F32(4.0))) / F32(n_img[2]))


def beatty_beta(os: float) -> float:
    """Beatty's beta, computeQ.cmem.cu:460-463 (float32)."""
    os = F32(os)
    w = F32(KW)
    v = F32((os - F32(0.5)) * (os - F32(0.5)) * (w * w * F32(4.0)) / (os * os) - F32(0.8))
    return float(PI32 * F32(np.sqrt(v)))


def grid_size(os: float, n_img: tuple) -> tuple:
    """computeQ.cmem.cu:476-486: xy even, z = ceil(OS nz) (or 1)."""
    os = F32(os)
    gx = int(np.ceil(F32(os * F32(n_img[0]))))
    gy = int(np.ceil(F32(os * F32(n_img[1]))))
    gx += gx % 2
    gy += gy % 2
    gz = 1 if n_img[2] == 1 else int(np.ceil(F32(os * F32(n_img[2]))))
    return gx, gy, gz


def bessi0(x):
    """Modified Bessel I0 by the Abramowitz-Stegun 9.8.1-9.8.2 polynomials."""
    x = np.abs(np.asarray(x, np.float64))
    out = np.empty_like(x)
    s = x < 3.75
    y = (x[s] / 3.75) ** 2
    out[s] = 1.0 + y * (3.5156229 + y * (3.0899424 + y * (1.2067492 + y * (
        0.2659732 + y * (0.360768e-1 + y * 0.45813e-2)))))
    ax = x[~s]
    y = 3.75 / ax
    out[~s] = (np.exp(ax) / np.sqrt(ax)) * (0.39894228 + y * (0.1328592e-1 + y * (
        0.225319e-2 + y * (-0.157565e-2 + y * (0.916281e-2 + y * (-0.2057706e-1 + y * (
            0.2635537e-1 + y * (-0.1647633e-1 + y * 0.392377e-2))))))))
    return out


def kb_weight(d, beta):
    """KB weight for distance d (image-grid units), 0 outside |d| <= W/2."""
    d = np.abs(d)
    arg = 1.0 - (4.0 / (KW * KW)) * d * d
    w = np.where(arg >= 0.0, bessi0(beta * np.sqrt(np.clip(arg, 0.0, None))) / KW, 0.0)
    return np.where(d <= KW / 2, w, 0.0)


def hanning(t, tau, l, t0):
    x = np.asarray(t, np.float64) - tau * l - t0
    return np.where(np.abs(x) < tau, 0.5 + 0.5 * np.cos(np.pi * x / tau), 0.0)


def kb_transform(u, beta):
    """Closed-form KB transform shape used for deapodisation
    (gridding_utils.cu:60-110)."""
    e = (np.pi * KW * u) ** 2 - beta * beta
    out = np.empty_like(e)
    pos = e >= 0
    sp = np.sqrt(e[pos])
    out[pos] = np.where(sp > 0, np.sin(sp) / np.where(sp > 0, sp, 1.0), 1.0)
    sn = np.sqrt(-e[~pos])
    out[~pos] = np.sinh(sn) / sn
    return out


def grid_samples(kx, ky, kz, data, weights, n_img, os, beta):
    """Scatter form of gridding_GPU_2D/3D: grid[X,Y,Z] = sum_s w_x w_y w_z
    data_s weights_s, shifted coordinates k' = OS (k + n_img/2)."""
    gs = grid_size(os, n_img)
    grid = np.zeros(gs, np.complex128)
    osd = float(F32(os))
    coords = [osd * (np.asarray(k, np.float64) + n / 2.0) for k, n in zip((kx, ky, kz), n_img)]
    val = np.asarray(data, np.complex128) * np.asarray(weights, np.float64)
    keep = val != 0
    coords = [c[keep] for c in coords]
    val = val[keep]
    reach = int(np.ceil(KW / 2 * osd)) + 1
    ndim = 2 if n_img[2] == 1 else 3
    axes_w = []
    axes_i = []
    for a in range(ndim):
        base = np.floor(coords[a]).astype(np.int64)
        ws, ids = [], []
        for o in range(-reach, reach + 1):
            idx = base + o
            w = kb_weight((coords[a] - idx) / osd, beta)
            w = np.where((idx >= 0) & (idx < gs[a]), w, 0.0)
            ws.append(w)
            ids.append(np.clip(idx, 0, gs[a] - 1))
        axes_w.append(ws)
        axes_i.append(ids)
    if ndim == 2:
        for wx, ix in zip(axes_w[0], axes_i[0]):
            for wy, iy in zip(axes_w[1], axes_i[1]):
                w = wx * wy
                m = w != 0
                np.add.at(grid[:, :, 0], (ix[m], iy[m]), w[m] * val[m])
    else:
        for wx, ix in zip(axes_w[0], axes_i[0]):
            for wy, iy in zip(axes_w[1], axes_i[1]):
                wxy = wx * wy
                for wz, iz in zip(axes_w[2], axes_i[2]):
                    w = wxy * wz
                    m = w != 0
                    np.add.at(grid, (ix[m], iy[m], iz[m]), w[m] * val[m])
    return grid


def grid_to_image(grid, n_img, os, beta):
    """ifftshift -> unnormalised inverse FFT -> fftshift -> crop centre ->
    deapodise / OS^d, then to the reference's voxel order."""
    gs = grid.shape
    ndim = 2 if n_img[2] == 1 else 3
    g = grid[:, :, 0] if ndim == 2 else grid
    img = np.fft.fftshift(_ifftn(np.fft.ifftshift(g)) * g.size)
    sl = tuple(slice(gs[a] // 2 - n_img[a] // 2, gs[a] // 2 - n_img[a] // 2 + n_img[a])
               for a in range(ndim))
    img = img[sl]
    osd = float(F32(os))
    kern = 1.0
    for a in range(ndim):
        u = (np.arange(n_img[a]) - n_img[a] / 2.0) / n_img[a]
        shape = [1] * ndim
        shape[a] = n_img[a]
        kern = kern * kb_transform(u, beta).reshape(shape)
    img = img / kern / osd ** ndim
    if ndim == 3:
        img = np.transpose(img, (1, 0, 2))  # (x, y, z) -> (y, x, z)
    return img


def time_segments(t, L):
    t = np.asarray(t, np.float32)
    tau = float(F32(t[-1] - t[0]) / F32(L)) if L > 0 else float(t[-1] - t[0])
    return tau, float(t[0])


def compute_q(kx, ky, kz, t, dims, L, os_q):
    """Q_l on the 2N grid, l = 0..L (computeQ.cmem.cu:401-754, 826-1028).
    dims = (Nx, Ny, Nz).  Returns complex array [L+1, ...] in voxel order."""
    Nx, Ny, Nz = dims
    n_q = (2 * Nx, 2 * Ny, 1 if Nz == 1 else 2 * Nz)
    os = rounded_os(os_q, n_q)
    beta = beatty_beta(os)  # Q: beta after rounding (computeQ.cmem.cu:460)
    tau, t0 = time_segments(t, L)
    out = []
    for l in range(L + 1):
        h = hanning(t, tau, l, t0)
        g = grid_samples(2.0 * np.asarray(kx, np.float64), 2.0 * np.asarray(ky, np.float64),
                         2.0 * np.asarray(kz, np.float64), np.ones(len(kx)), h, n_q, os, beta)
        out.append(grid_to_image(g, n_q, os, beta))
    return np.stack(out)


def compute_fhd(kx, ky, kz, t, dims, L, os_fh, kdata, sens, fm):
    """Gridded F^H d with time segmentation and SENSE
    (computeFH.cmem.cu:469-802, 1034-1129).  kdata [C][M], sens [C][N], fm [N];
    returns the image in voxel order ([x, y] 2-D, [y, x, z] 3-D)."""
    Nx, Ny, Nz = dims
    n_i = (Nx, Ny, Nz)
    beta = beatty_beta(os_fh)  # F^H d: beta before rounding (computeFH.cmem.cu:497)
    os = rounded_os(os_fh, n_i)
    tau, t0 = time_segments(t, L)
    shape = (Nx, Ny) if Nz == 1 else (Ny, Nx, Nz)
    fm = np.asarray(fm, np.float64).reshape(shape)
    C = np.asarray(kdata).shape[0]
    out = np.zeros(shape, np.complex128)
    for c in range(C):
        acc = np.zeros(shape, np.complex128)
        for l in range(L + 1):
            h = hanning(t, tau, l, t0)
            g = grid_samples(kx, ky, kz, np.asarray(kdata)[c], h, n_i, os, beta)
            acc += grid_to_image(g, n_i, os, beta) * np.exp(1j * fm * (tau * l + t0))
        out += np.conj(np.asarray(sens)[c].reshape(shape)) * acc
    return out


def qf_from_q(Q):
    """Qf_l = FFT(ifftshift(Q_l)) on the 2N grid (recon.cu:1939-1964);
    grids in FFT axis order ([x, y] 2-D, [x, y, z] 3-D)."""
    out = []
    for q in Q:
        g = q if q.ndim == 2 else np.transpose(q, (1, 0, 2))
        out.append(_fftn(np.fft.ifftshift(g)))
    return np.stack(out)


def fhf(image, qf):
    """recon.cu:1113-1202: pad into the 2N grid, shift, FFT, x Qf, inverse FFT
    (unnormalised), shift back, crop, scale 1/G."""
    img = image if image.ndim == 2 else np.transpose(image, (1, 0, 2))
    n = img.shape
    big = np.zeros(qf.shape, np.complex128)
    sl = tuple(slice(s - s // 2, s - s // 2 + s) for s in n)
    big[sl] = img
    f = _fftn(np.fft.ifftshift(big)) * qf
    r = np.fft.fftshift(_ifftn(f) * f.size)[sl] / qf.size
    return r if image.ndim == 2 else np.transpose(r, (1, 0, 2))


def aha(p, Qf, sens, fm, tau, t0):
    """parCudaAhA / CudaAhA (recon.cu:1370-1465)."""
    out = np.zeros_like(p, dtype=np.complex128)
    for s in sens:
        s = s.reshape(p.shape)
        acc = np.zeros_like(out)
        for l in range(len(Qf)):
            ph = np.exp(-1j * fm * (tau * l + t0))
            acc += np.conj(ph) * fhf(s * p * ph, Qf[l])
        out += np.conj(s) * acc
    return out


def aha_coils(p, Qf, sens, fm, tau, t0):
    """aha() with the coils batched into one FFT call per segment (the same
    FP64 arithmetic, for many coils at large sizes).  p: image in voxel
    order; sens [C, *p.shape]; Qf [L+1, *grid] in FFT axis order."""
    tr = p.ndim == 3
    img_t = (lambda a: np.transpose(a, (0, 2, 1, 3))) if tr else (lambda a: a)
    sens = np.asarray(sens).reshape(len(sens), *p.shape)
    n = p.shape if not tr else (p.shape[1], p.shape[0], p.shape[2])
    gshape = Qf.shape[1:]
    sl = (slice(None),) + tuple(slice(m - m // 2, m - m // 2 + m) for m in n)
    axes = tuple(range(1, len(gshape) + 1))
    out = np.zeros(p.shape, np.complex128)
    for l in range(len(Qf)):
        ph = np.exp(-1j * np.asarray(fm, np.float64).reshape(p.shape) * (tau * l + t0))
        big = np.zeros((len(sens),) + gshape, np.complex128)
        big[sl] = img_t(sens * (p * ph))
        f = _fftn(np.fft.ifftshift(big, axes=axes), axes=axes)
        f *= Qf[l]
        r = np.fft.fftshift(_ifftn(f, axes=axes), axes=axes)[sl] * (f[0].size / Qf[l].size)
        out += np.conj(ph) * np.sum(np.conj(sens) * img_t(r), axis=0)
    return out


def tv_grid_shape(dims):
    Nx, Ny, Nz = dims
    return (Nx, Ny, 1) if Nz == 1 else (Ny, Nx, Nz)


def dhwd(p, w, lam):
    """lambda D^H W D p, periodic forward differences on every axis of size > 1
    (DHWD{2,3}dGpu_toeplitz.cu)."""
    s = np.zeros_like(p, dtype=np.complex128)
    for ax in range(p.ndim):
        if p.shape[ax] == 1:
            continue
        t = w * (p - np.roll(p, -1, axis=ax))
        s += t - np.roll(t, 1, axis=ax)
    return lam * s


def reg_penalty(v, reg, w, lam):
    """lambda C^T (W (C v)) for -reg (toeplitz/recon.cu:1543-1673): reg =
    (rows, cols, I, J, V) 0-based coordinates of the real roughness matrix C,
    W = w applied to every block of N rows."""
    rows, cols, I, J, V = reg
    x = np.asarray(v).ravel()
    y = np.zeros(rows, np.complex128)
    np.add.at(y, np.asarray(I), np.asarray(V, np.float64) * x[np.asarray(J)])
    y *= np.tile(np.asarray(w, np.float64).ravel(), rows // x.size)
    out = np.zeros(x.size, np.complex128)
    np.add.at(out, np.asarray(J), np.asarray(V, np.float64) * y[np.asarray(I)])
    return lam * out.reshape(np.shape(v))


def tv_weight(x, eps):
    s = np.zeros(x.shape)
    for ax in range(x.ndim):
        if x.shape[ax] == 1:
            continue
        s += np.abs(x - np.roll(x, -1, axis=ax)) ** 2
    return 0.5 / np.sqrt(s + eps)


def toeplitz_cg(fhd, Q, sens, fm, t, L, cg_num, lam=None, tv=False, tv_num=1, eps=1e-6,
                tol=1e-16, reg=None):
    """toeplitz_recon (recon.cu:1724-2191): CG on (A^H A + lambda D^H W D) x =
    F^H d from x = 0, x carried over TV passes, best-residual iterate
    returned; with reg (the -reg roughness matrix) lambda C^T W C replaces the
    finite-difference term.  Images in voxel order."""
    tau, t0 = time_segments(t, L)
    shape = fhd.shape
    fm = np.asarray(fm, np.float64).reshape(shape)
    sens = np.asarray(sens).reshape(len(sens), *shape)
    Qf = qf_from_q(Q)
    x = np.zeros(shape, np.complex128)
    best = x.copy()
    norm_fhd = np.vdot(fhd, fhd).real
    w = np.ones(shape)

    def A(v):
        out = aha(v, Qf, sens, fm, tau, t0)
        if reg is not None:  # -reg takes precedence over -fd
            out = out + reg_penalty(v, reg, w, lam or 0.0)
        elif lam is not None:
            out = out + dhwd(v, w, lam)
        return out

    for tv_i in range(tv_num if tv else 1):
        if tv_i != 0:
            w = tv_weight(x, eps)
        r = fhd - A(x)
        beta2 = res_best = np.vdot(r, r).real
        p = r.copy()
        for _ in range(cg_num):
            q = A(p)
            beta = beta2
            alpha = beta / np.vdot(p, q).real
            x = x + alpha * p
            r = r - alpha * q
            beta2 = np.vdot(r, r).real
            p = r + (beta2 / beta) * p
            if beta2 < res_best:
                res_best = beta2
                best = x.copy()
            if np.sqrt(beta2 / norm_fhd) < tol:
                break
    return best

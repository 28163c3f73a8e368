"""Seeded synthetic inputs with the shapes of the benchmark configurations.

No public dataset is involved: trajectories, phantoms, coil maps and field
maps are generated from a seed.  Conventions follow the reference inputs:
k in cycles/FOV, positions in FOV units on the grid (i - n/2)/n, field map in
rad/s with forward phase exp(-i(2 pi k.r + fm t)), 2-D voxel order x-slow /
y-fast, 3-D order (y, x, z) with z fastest.
"""
from __future__ import annotations

import numpy as np

TWO_PI = 2.0 * np.pi


def grid_positions(ny: int, nx: int, nz: int = 1):
    """(ix, iy, iz) float32 for the reference voxel order.  2-D (nz == 1) is
    x-slow / y-fast; 3-D is (y, x, z) with z fastest."""
    ax = lambda n: ((np.arange(n) - n // 2) / n).astype(np.float64)
    if nz == 1:
        X, Y = np.meshgrid(ax(nx), ax(ny), indexing="ij")
        Z = np.zeros_like(X)
    else:
        Y, X, Z = np.meshgrid(ax(ny), ax(nx), ax(nz), indexing="ij")
    return (X.ravel().astype(np.float32), Y.ravel().astype(np.float32),
            Z.ravel().astype(np.float32))


def spiral(n_interleaves: int, n_samples: int, kmax: float, rng, density_power: float = 1.5,
           turns: float | None = None, t_read: float = 0.010):
    """Variable-density Archimedean-type spiral: radius grows as (s)^density_power
    (denser near the centre), interleaves rotated evenly; t uniform over the
    readout window [0, t_read) for each interleave."""
    s = np.arange(n_samples) / n_samples
    if turns is None:
        turns = max(kmax / n_interleaves, 1.0)
    r = kmax * s ** density_power
    phase0 = rng.uniform(0, TWO_PI)
    kx, ky = [], []
    for i in range(n_interleaves):
        th = TWO_PI * turns * s + TWO_PI * i / n_interleaves + phase0
        kx.append(r * np.cos(th))
        ky.append(r * np.sin(th))
    kx = np.clip(np.concatenate(kx), -kmax, np.nextafter(kmax, 0))
    ky = np.clip(np.concatenate(ky), -kmax, np.nextafter(kmax, 0))
    t = np.tile(s * t_read, n_interleaves)
    return kx.astype(np.float32), ky.astype(np.float32), t.astype(np.float32)


def ellipse_phantom(shape, n_ellipses: int, rng, smooth_phase: bool = True):
    """Complex phantom on the (y, x[, z]) grid: sum of random ellipses
    (ellipsoids in 3-D) with intensities U(0.1, 1) and a smooth global phase."""
    coords = np.meshgrid(*[(np.arange(n) - n // 2) / n for n in shape], indexing="ij")
    img = np.zeros(shape)
    for _ in range(n_ellipses):
        c = rng.uniform(-0.25, 0.25, len(shape))
        a = rng.uniform(0.05, 0.3, len(shape))
        th = rng.uniform(0, np.pi)
        u = coords[0] - c[0]
        v = coords[1] - c[1]
        ur = u * np.cos(th) + v * np.sin(th)
        vr = -u * np.sin(th) + v * np.cos(th)
        q = (ur / a[0]) ** 2 + (vr / a[1]) ** 2
        if len(shape) == 3:
            q = q + ((coords[2] - c[2]) / max(a[2], 0.2)) ** 2
        img[q <= 1.0] += rng.uniform(0.1, 1.0)
    phase = np.zeros(shape)
    if smooth_phase:
        for ci in coords:
            phase += rng.uniform(-1.0, 1.0) * ci
        phase += rng.uniform(-0.5, 0.5) * sum(ci ** 2 for ci in coords) * 4
    return img * np.exp(1j * np.pi * phase)


def field_map(shape, rng, max_hz: float = 50.0):
    """Smooth quadratic + Gaussian bump, scaled to |omega| <= 2 pi max_hz rad/s."""
    coords = np.meshgrid(*[(np.arange(n) - n // 2) / n for n in shape], indexing="ij")
    quad = sum(rng.uniform(-1, 1) * c ** 2 for c in coords) + sum(
        rng.uniform(-0.5, 0.5) * c for c in coords)
    c0 = rng.uniform(-0.2, 0.2, len(shape))
    bump = np.exp(-sum((c - m) ** 2 for c, m in zip(coords, c0)) / (2 * 0.1 ** 2))
    f = quad + rng.uniform(0.5, 1.0) * bump
    f = f / max(np.abs(f).max(), 1e-12)
    return (TWO_PI * max_hz * f).astype(np.float32)


def coil_maps(shape, n_coils: int, rng, sigma: float = 0.4, ring: bool = False):
    """Complex Gaussian-bump coil sensitivities placed around the FOV (on a
    ring when `ring`), each with a linear phase, normalised to unit
    root-sum-of-squares."""
    coords = np.meshgrid(*[(np.arange(n) - n // 2) / n for n in shape], indexing="ij")
    maps = []
    for c in range(n_coils):
        ang = TWO_PI * c / n_coils + (0.0 if ring else rng.uniform(-0.2, 0.2))
        rad = 0.5
        centre = [rad * np.cos(ang), rad * np.sin(ang)] + [0.0] * (len(shape) - 2)
        g = np.exp(-sum((x - m) ** 2 for x, m in zip(coords, centre)) / (2 * sigma ** 2))
        lin = sum(rng.uniform(-1.0, 1.0) * x for x in coords)
        maps.append(g * np.exp(1j * np.pi * lin))
    maps = np.stack(maps)
    rss = np.sqrt((np.abs(maps) ** 2).sum(0))
    return (maps / rss).astype(np.complex64)


def to_voxel_order(vol):
    """(y, x) -> x-slow / y-fast for 2-D; (y, x, z) stays row-major in 3-D."""
    vol = np.asarray(vol)
    if vol.ndim == 2:
        return vol.T.ravel()
    return vol.ravel()


def add_noise(y, snr_db: float, rng):
    """Complex Gaussian noise at the given SNR (signal power over the sampled k-data)."""
    p = np.mean(np.abs(y) ** 2)
    sigma = np.sqrt(p / 10 ** (snr_db / 10) / 2)
    return y + sigma * (rng.standard_normal(y.shape) + 1j * rng.standard_normal(y.shape))


def make_case(name: str, seed: int | None = None, forward=None, small: bool = False):
    """Inputs of one benchmark configuration (without k-space data if
    `forward` is None).  forward(x, sens, case) -> complex [C][M] FP64/FP32 data.

    names: "bf2d_64"        64x64, 1 coil, 4 x 1024 spiral, 8 CG, TV 1e-3
           "bf3d_64x64x16"  64x64x16, 4 coils, 16 kz x 4 x 1024 stack of spirals
           "toep3d_256x256x32"  256x256x32, 4 coils, 32 kz x 16 x 4096 (Toeplitz)
    `small` shrinks the sample count for fast tests (same recipe)."""
    seed = {"bf2d_64": 1001, "bf3d_64x64x16": 1002,
            "toep3d_256x256x32": 1003}.get(name, 1000) if seed is None else seed
    rng = np.random.default_rng(seed)
    if name == "bf2d_64":
        ny = nx = 64
        nz = 1
        n_il, n_s = (4, 256) if small else (4, 1024)
        kx, ky, t = spiral(n_il, n_s, 32.0, rng)
        kz = np.zeros_like(kx)
        C = 1
        img = ellipse_phantom((ny, nx), 8, rng)
        fm = field_map((ny, nx), rng)
        sens = np.ones((1, ny * nx), np.complex64)
        x_true = to_voxel_order(img)
        fm_v = to_voxel_order(fm)
        dims = (nx, ny, 1)
        opts = dict(cg_num=8, fd_penalizer=1e-3, tv=True, tv_num=10, use_z=0)
    elif name == "bf3d_64x64x16":
        ny = nx = 64
        nz = 16
        n_part, n_il, n_s = (16, 4, 64) if small else (16, 4, 1024)
        kx2, ky2, t2 = spiral(n_il, n_s, 32.0, rng)
        kz_levels = np.arange(-nz // 2, nz // 2, dtype=np.float32)[:n_part]
        kx = np.tile(kx2, n_part)
        ky = np.tile(ky2, n_part)
        kz = np.repeat(kz_levels, kx2.size).astype(np.float32)
        t = np.tile(t2, n_part)
        C = 4
        img = ellipse_phantom((ny, nx, nz), 8, rng)
        fm = field_map((ny, nx, nz), rng)
        sens = coil_maps((ny, nx, nz), C, rng).reshape(C, -1)
        x_true = img.ravel()
        fm_v = fm.ravel()
        dims = (nx, ny, nz)
        opts = dict(cg_num=16, fd_penalizer=1e-3, tv=True, tv_num=10, use_z=1)
    elif name == "toep3d_256x256x32":
        # 256x256x32, 4 coils, 32 kz partitions x 16 interleaves x 4096
        # (small: 16x16x8, 2 coils, 8 x 2 x 128)
        ny, nx, nz = (16, 16, 8) if small else (256, 256, 32)
        n_part, n_il, n_s = (8, 2, 128) if small else (32, 16, 4096)
        kx2, ky2, t2 = spiral(n_il, n_s, nx / 2 - 0.05, rng)
        kz_levels = np.arange(-nz // 2, nz // 2, dtype=np.float32)[:n_part]
        kx = np.tile(kx2, n_part)
        ky = np.tile(ky2, n_part)
        kz = np.repeat(kz_levels, kx2.size).astype(np.float32)
        t = np.tile(t2, n_part)
        C = 2 if small else 4
        img = ellipse_phantom((ny, nx, nz), 8, rng)
        fm = field_map((ny, nx, nz), rng)
        sens = coil_maps((ny, nx, nz), C, rng).reshape(C, -1)
        x_true = img.ravel()
        fm_v = fm.ravel()
        dims = (nx, ny, nz)
        opts = dict(cg_num=20, fd_penalizer=1e-3, tv=True, tv_num=10, use_z=1, ntime_segs=8,
                    gridOS_Q=2.0, gridOS_FH=1.5)
    else:
        raise ValueError(name)
    ix, iy, iz = grid_positions(ny, nx, nz)
    case = dict(name=name, seed=seed, kx=kx, ky=ky, kz=kz, t=t, ix=ix, iy=iy, iz=iz,
                fm=fm_v.astype(np.float32), sens=np.asarray(sens, np.complex64),
                x_true=x_true.astype(np.complex64), dims=dims, num_coil=C, M=kx.size,
                N=ix.size, opts=opts)
    if forward is not None:
        y = forward(case["x_true"], case["sens"], case)
        case["kdata"] = add_noise(np.asarray(y), 40.0, rng).astype(np.complex64)
    return case


def fd_matrix(shape):
    """Roughness matrix C for -reg: periodic first-order differences
    (C x)_k = x_i - x_{i+1 (mod n)} along each axis of length > 2, one block of
    N = prod(shape) rows per axis, stacked; coordinate form (rows, cols, I, J,
    V), 0-based.  Restates matlab_utils/create_sparse_matrix/
    createDWithPeriodicBoundary.m (2-D) and createDWithPeriodicBoundary3D.m
    (3-D) for IMPATIENT's row-major voxel order, as that directory's README
    prescribes: 2-D images [x][y] (y fastest) give the y block then the x
    block; 3-D images [y][x][z] (z fastest) give the z, x and y blocks.
    `shape` is the image in voxel order: (nx, ny) or (ny, nx, nz)."""
    shape = tuple(int(n) for n in shape)
    N = int(np.prod(shape))
    idx = np.arange(N).reshape(shape)
    Is, Js, Vs = [], [], []
    row0 = 0
    for ax in reversed(range(len(shape))):  # fastest axis first
        if shape[ax] <= 2:
            continue
        nxt = np.roll(idx, -1, axis=ax)
        # MATLAB's spdiags order within a block: the column-major (fastest axis
        # first) ordering of the rows, which is also the voxel index here
        r = row0 + idx.ravel()
        Is += [r, r]
        Js += [idx.ravel(), nxt.ravel()]
        Vs += [np.ones(N), -np.ones(N)]
        row0 += N
    I = np.concatenate(Is)
    J = np.concatenate(Js)
    V = np.concatenate(Vs)
    order = np.lexsort((I, J))  # column-major entry order, as mmwrite writes a sparse matrix
    return row0, N, I[order], J[order], V[order]

"""Helpers shared by the GPU tests."""
import numpy as np
import torch


def dev(a):
    return torch.as_tensor(np.ascontiguousarray(a, np.float32)).cuda()


def host(t):
    return t.detach().cpu().numpy().astype(np.float64)


def gpu_ft(pkg, ctx, case, x, use_z=0, fm=True):
    M, N = case["kx"].size, case["ix"].size
    s = np.asarray(case["sens"]).reshape(-1, N)
    C = s.shape[0]
    yr = torch.zeros(C * M, device="cuda")
    yi = torch.zeros(C * M, device="cuda")
    pkg.parallelFtGpu(ctx, yr, yi, dev(np.real(x)), dev(np.imag(x)), dev(case["kx"]),
                      dev(case["ky"]), dev(case["kz"]), dev(case["ix"]), dev(case["iy"]),
                      dev(case["iz"]), dev(case["fm"]) if fm else None, dev(case["t"]), M, N,
                      dev(s.real), dev(s.imag), C, use_z)
    return (host(yr) + 1j * host(yi)).reshape(C, M)


def gpu_ift(pkg, ctx, case, d, use_z=0, fm=True):
    M, N = case["kx"].size, case["ix"].size
    s = np.asarray(case["sens"]).reshape(-1, N)
    C = s.shape[0]
    d = np.asarray(d).reshape(C * M)
    xr = torch.zeros(N, device="cuda")
    xi = torch.zeros(N, device="cuda")
    pkg.parallelIftGpu(ctx, xr, xi, dev(d.real), dev(d.imag), dev(case["kx"]), dev(case["ky"]),
                       dev(case["kz"]), dev(case["ix"]), dev(case["iy"]), dev(case["iz"]),
                       dev(case["fm"]) if fm else None, dev(case["t"]), M, N, dev(s.real),
                       dev(s.imag), C, use_z)
    return host(xr) + 1j * host(xi)


def gpu_recon(pkg, ctx, case, x0=None, *, cg_num, lam, tv, tv_num=1, eps=1e-6, use_z=0,
              dims=None, host_ptrs=True):
    M, N = case["kx"].size, case["ix"].size
    s = np.asarray(case["sens"]).reshape(-1, N)
    C = s.shape[0]
    S = np.asarray(case["kdata"]).size // (C * M)
    x0 = np.zeros(S * N, np.complex64) if x0 is None else x0
    f = lambda a: np.ascontiguousarray(a, np.float32)
    conv = f if host_ptrs else dev
    xr, xi = conv(np.real(x0)), conv(np.imag(x0))
    kd = np.asarray(case["kdata"]).ravel()
    opts = pkg.bf_options(cg_num=cg_num, fd_penalizer=lam, tv=tv, tv_num=tv_num, tv_eps=eps,
                          use_z=use_z, dims=dims)
    pkg.bruteForceGpu(ctx, opts, xr, xi, conv(kd.real), conv(kd.imag), conv(case["kx"]),
                      conv(case["ky"]), conv(case["kz"]), conv(case["ix"]), conv(case["iy"]),
                      conv(case["iz"]), conv(case["fm"]), conv(case["t"]), conv(s.real),
                      conv(s.imag), M, N, C, S)
    if host_ptrs:
        return xr.astype(np.float64) + 1j * xi.astype(np.float64)
    return host(xr) + 1j * host(xi)

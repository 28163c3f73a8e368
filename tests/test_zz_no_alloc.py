"""The allocation-free adjoint (imp_parallel_ift_noalloc) against the regular
one (imp_parallel_ift), called through the C-ABI.

The variant exists for callers that cannot call cudaMalloc (a host that owns
all device memory through its own allocator, or a fixed memory budget): it
works in a static device array instead.  Because every call shares that array
and it keeps the previous call's contents, the test makes two calls in a row
on different inputs.  This file is collected last so that a run stopping at
its first failure has run every other test already.
"""
import ctypes

import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu
TOL_OP = 1e-5


def _inputs(synth, n, nz, C, M, seed):
    rng = np.random.default_rng(seed)
    kx, ky, t = synth.spiral(4, M // 4, n / 2, rng)
    kz = (rng.integers(-nz // 2, max(nz // 2, 1), kx.size).astype(np.float32) if nz > 1
          else np.zeros_like(kx))
    ix, iy, iz = synth.grid_positions(n, n, nz)
    shape = (n, n, nz) if nz > 1 else (n, n)
    fm = synth.field_map(shape, rng).ravel()
    sens = (synth.coil_maps(shape, C, rng).reshape(C, -1) if C > 1
            else np.ones((1, ix.size), np.complex64))
    d = (rng.standard_normal((C, kx.size)) + 1j * rng.standard_normal((C, kx.size))).ravel()
    return dict(kx=kx, ky=ky, kz=kz, t=t, ix=ix, iy=iy, iz=iz, fm=fm, sens=sens, d=d,
                M=kx.size, N=ix.size, C=C, use_z=int(nz > 1))


def _noalloc(pkg, c):
    import torch
    from gpu_util import dev, host
    N = c["N"]
    xr = torch.zeros(N, device="cuda")
    xi = torch.zeros(N, device="cuda")
    s = c["sens"]
    args = [dev(c["d"].real), dev(c["d"].imag)] + [dev(c[k]) for k in
                                                  ("kx", "ky", "kz", "ix", "iy", "iz", "fm", "t")]
    sr, si = dev(s.real), dev(s.imag)
    p = lambda a: ctypes.c_void_p(a.data_ptr())
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    st = pkg.lib().imp_parallel_ift_noalloc(p(xr), p(xi), *map(p, args), c["M"], N, p(sr), p(si),
                                            c["C"], c["use_z"], stream)
    assert st == 0, pkg.lib().imp_last_error()
    return host(xr) + 1j * host(xi)


def _regular(pkg, c):
    from gpu_util import gpu_ift
    case = dict(c)
    with pkg.Context(0) as ctx:
        return gpu_ift(pkg, ctx, case, c["d"].reshape(c["C"], -1), use_z=c["use_z"])


def test_noalloc_adjoint_matches_regular_twice(pkg, synth):
    cases = [_inputs(synth, 32, 8, 4, 4096, seed=1), _inputs(synth, 48, 1, 3, 2000, seed=2)]
    for c in cases:  # two calls in a row: the second must not see the first's contents
        a = _noalloc(pkg, c)
        b = _regular(pkg, c)
        assert oracle.rel_l2(a, b) < TOL_OP


def test_noalloc_adjoint_tensor_core_coil_group(pkg, synth):
    """Twenty coils: one coil group of 32 on the tensor-core kernel inside the
    static array, against the regular adjoint and the FP64 oracle."""
    c = _inputs(synth, 32, 1, 20, 2048, seed=3)
    a = _noalloc(pkg, c)
    b = _regular(pkg, c)
    assert oracle.rel_l2(a, b) < TOL_OP
    case = dict(c)
    ref = oracle.ift(c["d"].reshape(c["C"], -1), case, use_z=0)
    assert oracle.rel_l2(a, ref) < TOL_OP


def test_noalloc_rejects_sizes_beyond_the_scratch(pkg, synth):
    import torch
    M, N = 1 << 20, 1 << 20
    z = torch.zeros(max(M, N), device="cuda")
    p = ctypes.c_void_p(z.data_ptr())
    st = pkg.lib().imp_parallel_ift_noalloc(p, p, p, p, p, p, p, p, p, p, None, p, M, N, None,
                                            None, 1, 0, None)
    assert st == 1

// Total-variation stencil shared by the brute-force and Toeplitz solvers.
//
// Periodic forward differences (D p)_i = p_i - p_{i+1} along every axis of
// size > 1 of a row-major (n0, n1, n2) grid (n2 fastest), their adjoint
// (D^H t)_i = t_i - t_{i-1}, and the reweighting W = 0.5 / sqrt(sum |D x|^2 + eps):
// kernels/Dhori2dCpu.cpp:84-126, kernels/Dverti2dCpu.cpp:84-124,
// kernels/DHWD2dCpu.cpp:94-270, kernels/multiplyCpu.cpp:84-110,
// toeplitz/DHWD3dGpu_toeplitz.cu:170-580, toeplitz/multiplyGpu_toeplitz.cu:153-172.
#pragma once
#include <cuda_runtime.h>

namespace imp {

struct Grid3 {
    int n0, n1, n2;
};

// lambda-free D^H W D p at voxel i: sum over axes of
//   w_i (p_i - p_{i+1}) - w_{i-1} (p_{i-1} - p_i)     (periodic)
// (kernels/DHWD2dCpu.cpp:94-270, toeplitz/DHWD3dGpu_toeplitz.cu:170-580)
__device__ __forceinline__ float2 dhwd_at(const float2 *__restrict__ p,
                                          const float *__restrict__ w, int i, Grid3 gd) {
    const int c = i % gd.n2;
    const int b = (i / gd.n2) % gd.n1;
    const int a = i / (gd.n2 * gd.n1);
    const float2 pi = p[i];
    const float wi = w[i];
    float2 acc = make_float2(0.f, 0.f);
    const int coord[3] = {a, b, c};
    const int n[3] = {gd.n0, gd.n1, gd.n2};
    const int st[3] = {gd.n1 * gd.n2, gd.n2, 1};
#pragma unroll
    for (int ax = 0; ax < 3; ++ax) {
        if (n[ax] == 1) continue;
        const int in = coord[ax] == n[ax] - 1 ? i - (n[ax] - 1) * st[ax] : i + st[ax];
        const int ip = coord[ax] == 0 ? i + (n[ax] - 1) * st[ax] : i - st[ax];
        const float2 pn = p[in], pp = p[ip];
        const float wp = w[ip];
        const float tir = wi * (pi.x - pn.x), tii = wi * (pi.y - pn.y);
        const float tpr = wp * (pp.x - pi.x), tpi = wp * (pp.y - pi.y);
        acc.x += tir - tpr;
        acc.y += tii - tpi;
    }
    return acc;
}


// w = 0.5 / sqrt(sum_axes |D_a x|^2 + eps) for the N voxels of x.
cudaError_t tv_weight(float *w, const float2 *x, int N, Grid3 gd, float eps, cudaStream_t st);

}  // namespace imp

// Toeplitz reconstruction path on B200.
//
//   Q_l   = deapod(crop(IFFT(KB-grid_{2k}(h_l(t)))))          toeplitz/computeQ.cmem.cu:401-754
//   F^H d = sum_c conj(S_c) sum_l e^{+i w (tau l + t0)}
//             deapod(crop(IFFT(KB-grid_k(h_l(t) d_c))))      toeplitz/computeFH.cmem.cu:469-1129
//   A^H A p = sum_c conj(S_c) sum_l e^{+i w tau_l}
//             crop(IFFT(Qf_l . FFT(pad(e^{-i w tau_l} S_c p)))) / G   toeplitz/recon.cu:1113-1465
//   CG on (A^H A + lambda D^H W D) x = F^H d from x = 0, best-residual
//   iterate returned                                          toeplitz/recon.cu:1724-2191
//
// B200 design (not a translation of the reference kernels):
// * gridding is a scatter of each sample's separable KB footprint with vector
//   float2 atomics straight into the ifftshifted position of the FFT buffer,
//   one warp per sample (the lanes on contiguous cells), for the (at most two)
//   time segments whose Hanning window covers the sample -- no CPU binning, no
//   overflow path, no host round trips; the inverse transform is cropped to the
//   cells the post kernels read;
// * every shift / crop / deapodisation / phase / SENSE step is an index map
//   fused into the kernels around the FFTs; the FFTs are this library's own
//   (the pruned F^H F engine of toep_fft.cu for power-of-two images, the
//   mixed-radix grid transform of grid_fft.cu for the gridding grids, Qf_l
//   and the zero-padded chain of other sizes, all coils batched in one
//   transform);
// * Qf_l, sensitivities and phase factors stay resident in HBM; one CG
//   iteration (FFT chain + FP64 CG scalars, best-iterate tracking and the
//   tolerance stop all on the device) is captured once as a CUDA graph.
#include "../../include/impatient_b200.h"
#include "common.cuh"
#include "io.h"
#include "toeplitz.cuh"
#include "tv.cuh"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstddef>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <string>
#include <sys/stat.h>
#include <vector>

namespace imp {

namespace {

constexpr float kPiF = 3.1415926535897932384626433832795029f;
constexpr float kKW = 4.0f;  // kernel width
constexpr int kVB = 256;
constexpr int kTBlocks = 296;
constexpr int kMaxTaps = 12;

enum { T_PQ = 0, T_RR = 1, T_NORM = 2, T_SCAL = 3 };
// scalars (after the three partial slabs): beta2[2], resBest, normFhd, cur, done
struct TScal {
    double beta2[2];
    double res_best;
    double norm_fhd;
    int cur;
    int done;
    double tol;   // stop when sqrt(|r|^2 / |F^H d|^2) < tol
    int iters;    // CG updates performed since the solve started
    unsigned arrive;  // k_t_dir blocks done with this update (the last one finishes it)
};

__device__ __forceinline__ TScal *scal(double *dots) {
    return reinterpret_cast<TScal *>(dots + T_SCAL * kTBlocks);
}

// Modified Bessel I0 (Abramowitz & Stegun 9.8.1, 9.8.2).
__device__ __forceinline__ float bessi0f(float x) {
    const float ax = fabsf(x);
    if (ax < 3.75f) {
        float y = x / 3.75f;
        y *= y;
        return 1.0f + y * (3.5156229f + y * (3.0899424f + y * (1.2067492f + y * (0.2659732f +
                                         y * (0.360768e-1f + y * 0.45813e-2f)))));
    }
    const float y = 3.75f / ax;
    return (expf(ax) * rsqrtf(ax)) *
           (0.39894228f + y * (0.1328592e-1f + y * (0.225319e-2f + y * (-0.157565e-2f + y * (
                                0.916281e-2f + y * (-0.2057706e-1f + y * (0.2635537e-1f + y * (
                                                       -0.1647633e-1f + y * 0.392377e-2f))))))));
}

// KB weight at distance d (image-grid units): toeplitz/GPU_kernels.cu:270-300.
__device__ __forceinline__ float kb_weight(float d, float beta) {
    if (d > 0.5f * kKW) return 0.f;
    const float a = 1.0f - (4.0f / (kKW * kKW)) * d * d;
    if (!(a >= 0.f)) return 0.f;
    return bessi0f(beta * sqrtf(a)) * (1.0f / kKW);
}

__device__ __forceinline__ float hanning(float t, float tau, int l, float t0) {
    const float x = t - tau * (float)l - t0;
    return fabsf(x) < tau ? 0.5f + 0.5f * cosf(kPiF * x / tau) : 0.f;
}

// KB transform shape for deapodisation: toeplitz/gridding_utils.cu:60-110.
__device__ __forceinline__ float kb_transform(float u, float beta) {
    const float e = kPiF * kPiF * kKW * kKW * u * u - beta * beta;
    if (e > 0.f) {
        const float s = sqrtf(e);
        return sinf(s) / s;
    }
    if (e < 0.f) {
        const float s = sqrtf(-e);
        return sinhf(s) / s;
    }
    return 1.f;
}

// Scatter gridding of one time segment, one warp per sample: each sample's
// separable KB footprint is added into the ifftshifted position (X + gs/2) mod
// gs of every cell X it covers (ready for the inverse FFT).  The lanes take the
// cells of the footprint's two fastest-varying axes (z and y in 3-D, y and x in 2-D; up to
// 9 x 9 at OS 2), so one atomic instruction of the warp updates a few
// contiguous runs of the grid instead of 32 scattered cells, and the outer
// axis is looped.  The per-axis KB weights are computed once per sample into
// shared memory.
constexpr int kGridWarps = 8;

__global__ void __launch_bounds__(kGridWarps * 32)
    k_grid_w(float2 *grid, const float *kx, const float *ky, const float *kz, const float *t,
             const float *dr, const float *di, int M, GridSpec g, float tau, float t0, int l) {
    __shared__ float wsh[kGridWarps][3][kMaxTaps];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    float(&ws)[3][kMaxTaps] = wsh[wid];
    const float inv_os = 1.0f / g.os;
    // loop axis A, lane axes B (slower) and Cc (faster)
    const int A = g.is3d ? 0 : 2, B = g.is3d ? 1 : 0, Cc = g.is3d ? 2 : 1;
    for (int s = blockIdx.x * kGridWarps + wid; s < M; s += gridDim.x * kGridWarps) {
        const float h = hanning(__ldg(&t[s]), tau, l, t0);
        if (h == 0.f) continue;  // warp-uniform: every lane reads the same sample
        float vr = h, vi = 0.f;
        if (dr) {
            vr = h * __ldg(&dr[s]);
            vi = h * (di ? __ldg(&di[s]) : 0.f);
            if (vr == 0.f && vi == 0.f) continue;
        }
        const float k3[3] = {__ldg(&kx[s]), __ldg(&ky[s]), g.is3d ? __ldg(&kz[s]) : 0.f};
        int lo[3], cnt[3];
        float cc[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            if (a == 2 && !g.is3d) {
                lo[2] = 0;
                cnt[2] = 1;
                cc[2] = 0.f;
                continue;
            }
            const float c = g.os * (g.kscale * k3[a] + 0.5f * (float)g.img[a]);
            const float r = 0.5f * kKW * g.os;
            int a0 = (int)ceilf(c - r), a1 = (int)floorf(c + r);
            a0 = max(a0, 0);
            a1 = min(a1, g.gs[a] - 1);
            a1 = min(a1, a0 + kMaxTaps - 1);
            lo[a] = a0;
            cnt[a] = max(a1 - a0 + 1, 0);
            cc[a] = c;
        }
        for (int q = lane; q < 3 * kMaxTaps; q += 32) {
            const int a = q / kMaxTaps, j = q - a * kMaxTaps;
            if (j < cnt[a])
                ws[a][j] = (a == 2 && !g.is3d)
                               ? 1.f
                               : kb_weight(fabsf(cc[a] - (float)(lo[a] + j)) * inv_os, g.beta);
        }
        __syncwarp();
        // Shifted index lo + j + gs / 2 of a covered cell is below 2 gs: it wraps
        // at most once (one conditional subtraction, no division per cell).  The
        // loop axis steps by a fixed stride and wraps once.
        const int nbc = cnt[B] * cnt[Cc];
        int a0 = g.is3d ? lo[A] + g.gs[A] / 2 : 0;
        if (a0 >= g.gs[A]) a0 -= g.gs[A];
        const size_t astride = g.is3d ? (size_t)g.gs[1] * g.gs[2] : 0;
        const size_t awrap = astride * g.gs[A];
        const int rowlen = g.is3d ? g.gs[2] : g.gs[1];  // stride of axis B
        for (int p = lane; p < nbc; p += 32) {
            const int jb = p / cnt[Cc], jc = p - jb * cnt[Cc];
            const float wbc = ws[B][jb] * ws[Cc][jc];
            if (wbc == 0.f) continue;
            int ib = lo[B] + jb + g.gs[B] / 2;
            if (ib >= g.gs[B]) ib -= g.gs[B];
            int ic = lo[Cc] + jc + g.gs[Cc] / 2;
            if (ic >= g.gs[Cc]) ic -= g.gs[Cc];
            size_t cell = (size_t)a0 * astride + (size_t)ib * rowlen + ic;
            int ia = a0;
            for (int ja = 0; ja < cnt[A]; ++ja) {
                const float ww = wbc * ws[A][ja];
                if (ww != 0.f) atomicAdd(&grid[cell], make_float2(ww * vr, ww * vi));
                cell += astride;
                if (++ia == g.gs[A]) {
                    ia = 0;
                    cell -= awrap;
                }
            }
        }
        __syncwarp();  // the next sample overwrites ws
    }
}

struct NV {
    int v[3];
};

// Voxel coordinates (x, y, z) of a voxel-order index (2-D [x][y], 3-D [y][x][z]).
__device__ __forceinline__ void vox_xyz(size_t q, const int nv[3], bool is3d, int &x, int &y,
                                        int &z) {
    if (!is3d) {
        x = (int)(q / nv[1]);
        y = (int)(q % nv[1]);
        z = 0;
    } else {
        z = (int)(q % nv[2]);
        x = (int)((q / nv[2]) % nv[1]);
        y = (int)(q / ((size_t)nv[2] * nv[1]));
    }
}

// Value of image voxel (x, y, z) of a gridding problem after the inverse FFT:
// fftshift, crop of the centre and deapodisation.
__device__ __forceinline__ float2 grid_image_value(const float2 *A, const GridSpec &g, int x,
                                                   int y, int z) {
    const int c[3] = {x, y, z};
    size_t idx = 0;
    float kern = 1.f;
    for (int a = 0; a < 3; ++a) {
        const int off = g.gs[a] / 2 - g.img[a] / 2;
        const int j = (c[a] + off + g.gs[a] / 2) % g.gs[a];
        idx = idx * g.gs[a] + j;
        if (a < 2 || g.is3d)
            kern *= kb_transform(((float)c[a] - 0.5f * (float)g.img[a]) / (float)g.img[a], g.beta);
    }
    const float osd = g.is3d ? g.os * g.os * g.os : g.os * g.os;
    const float s = 1.0f / (kern * osd);
    const float2 v = A[idx];
    return make_float2(v.x * s, v.y * s);
}

// Q_l from the inverse-FFT'd grid: optional export in the reference layout and
// the ifftshifted copy that feeds Qf_l = FFT(ifftshift(Q_l)).
__global__ void k_q_post(const float2 *A, GridSpec g, NV n2, float2 *fftbuf, float *qr,
                         float *qi, size_t G2) {
    // n2: the 2N grid in voxel axis order
    const int nv[3] = {n2.v[0], n2.v[1], n2.v[2]};
    for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < G2;
         q += (size_t)gridDim.x * blockDim.x) {
        int x, y, z;
        vox_xyz(q, nv, g.is3d, x, y, z);
        const float2 v = grid_image_value(A, g, x, y, z);
        if (qr) {
            qr[q] = v.x;
            qi[q] = v.y;
        }
        // ifftshift in voxel axis order
        size_t o;
        if (!g.is3d)
            o = (size_t)((x + nv[0] / 2) % nv[0]) * nv[1] + (y + nv[1] / 2) % nv[1];
        else
            o = ((size_t)((y + nv[0] / 2) % nv[0]) * nv[1] + (x + nv[1] / 2) % nv[1]) * nv[2] +
                (z + nv[2] / 2) % nv[2];
        fftbuf[o] = v;
    }
}

// Q_l given in the reference layout -> ifftshifted FFT input.
__global__ void k_q_shift(const float *qr, const float *qi, NV n2, bool is3d, float2 *fftbuf,
                          size_t G2) {
    const int nv[3] = {n2.v[0], n2.v[1], n2.v[2]};
    for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < G2;
         q += (size_t)gridDim.x * blockDim.x) {
        int x, y, z;
        vox_xyz(q, nv, is3d, x, y, z);
        size_t o;
        if (!is3d)
            o = (size_t)((x + nv[0] / 2) % nv[0]) * nv[1] + (y + nv[1] / 2) % nv[1];
        else
            o = ((size_t)((y + nv[0] / 2) % nv[0]) * nv[1] + (x + nv[1] / 2) % nv[1]) * nv[2] +
                (z + nv[2] / 2) % nv[2];
        fftbuf[o] = make_float2(qr[q], qi[q]);
    }
}

// F^H d accumulation of one (coil, segment): acc += conj(S_c) e^{+i w tau_l} image.
__global__ void k_fh_post(const float2 *A, GridSpec g, NV nv3, size_t N,
                          const float2 *sens_c, const float2 *eph_l, float2 *acc) {
    const int nv[3] = {nv3.v[0], nv3.v[1], nv3.v[2]};
    for (size_t r = blockIdx.x * (size_t)blockDim.x + threadIdx.x; r < N;
         r += (size_t)gridDim.x * blockDim.x) {
        int x, y, z;
        vox_xyz(r, nv, g.is3d, x, y, z);
        const float2 v = grid_image_value(A, g, x, y, z);
        const float2 e = eph_l[r];  // exp(-i w tau_l)
        const float2 ve = cmulc(e, v);
        const float2 s = sens_c ? sens_c[r] : make_float2(1.f, 0.f);
        const float2 u = cmulc(s, ve);
        float2 a = acc[r];
        a.x += u.x;
        a.y += u.y;
        acc[r] = a;
    }
}

__global__ void k_eph(float2 *eph, const float *fm, size_t N, int L1, float tau, float t0) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < (size_t)L1 * N;
         i += (size_t)gridDim.x * blockDim.x) {
        const int l = (int)(i / N);
        const size_t r = i % N;
        const double arg = -(double)(fm ? fm[r] : 0.f) * ((double)tau * l + (double)t0);
        double s, c;
        sincos(arg, &s, &c);
        eph[i] = make_float2((float)c, (float)s);
    }
}

__global__ void k_pack_sens_c(float2 *sens, const float *sr, const float *si, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x)
        sens[i] = sr ? make_float2(sr[i], si ? si[i] : 0.f) : make_float2(1.f, 0.f);
}

// FFT-buffer index of image voxel q in the zero-padded, ifftshifted 2N grid:
// per axis (q + N/2 + N) mod 2N (recon.cu:325-421 and the half-rotation shifts).
__device__ __forceinline__ size_t pad_index(size_t q, const int nv[3], bool is3d) {
    int x, y, z;
    vox_xyz(q, nv, is3d, x, y, z);
    if (!is3d) {
        const int ox = (x + nv[0] / 2 + nv[0]) % (2 * nv[0]);
        const int oy = (y + nv[1] / 2 + nv[1]) % (2 * nv[1]);
        return (size_t)ox * (2 * nv[1]) + oy;
    }
    const int oy = (y + nv[0] / 2 + nv[0]) % (2 * nv[0]);
    const int ox = (x + nv[1] / 2 + nv[1]) % (2 * nv[1]);
    const int oz = (z + nv[2] / 2 + nv[2]) % (2 * nv[2]);
    return ((size_t)oy * (2 * nv[1]) + ox) * (2 * nv[2]) + oz;
}

// pad[c][o(q)] = S_c[q] p[q] exp(-i w tau_l)[q]
__global__ void k_pad(float2 *pad, const float2 *p, const float2 *sens, const float2 *eph_l,
                      NV nv, bool is3d, size_t N, size_t G2, int C, const double *dots) {
    if (dots && scal(const_cast<double *>(dots))->done) return;
    for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < N;
         q += (size_t)gridDim.x * blockDim.x) {
        const size_t o = pad_index(q, nv.v, is3d);
        const float2 pe = cmul(p[q], eph_l[q]);
        for (int c = 0; c < C; ++c) pad[(size_t)c * G2 + o] = cmul(sens[(size_t)c * N + q], pe);
    }
}

__global__ void k_mulq(float2 *big, const float2 *qf, size_t G2, int C, const double *dots) {
    if (dots && scal(const_cast<double *>(dots))->done) return;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < (size_t)C * G2;
         i += (size_t)gridDim.x * blockDim.x)
        big[i] = cmul(big[i], qf[i % G2]);
}

// acc[q] (+)= conj(exp(-i w tau_l)) sum_c conj(S_c) big[c][o(q)] / G2
__global__ void k_crop_acc(float2 *acc, const float2 *big, const float2 *sens,
                           const float2 *eph_l, NV nv, bool is3d, size_t N, size_t G2, int C,
                           int first, float scale, const double *dots) {
    if (dots && scal(const_cast<double *>(dots))->done) return;
    for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < N;
         q += (size_t)gridDim.x * blockDim.x) {
        const size_t o = pad_index(q, nv.v, is3d);
        float2 s = make_float2(0.f, 0.f);
        for (int c = 0; c < C; ++c) {
            const float2 u = cmulc(sens[(size_t)c * N + q], big[(size_t)c * G2 + o]);
            s.x += u.x;
            s.y += u.y;
        }
        float2 v = cmulc(eph_l[q], s);
        v.x *= scale;
        v.y *= scale;
        if (!first) {
            const float2 a = acc[q];
            v.x += a.x;
            v.y += a.y;
        }
        acc[q] = v;
    }
}

// q += lambda D^H W D p (pen 1) or lambda C^T W C p (pen 2, y = W C p formed
// beforehand); partial Re<p, q>
__global__ void __launch_bounds__(kVB) k_t_tvdot(float2 *__restrict__ q,
                                                 const float2 *__restrict__ p,
                                                 const float *__restrict__ w, int N, Grid3 gd,
                                                 int pen, float lambda, RegView reg,
                                                 double *dots) {
    __shared__ double sh[33];
    if (scal(dots)->done) return;
    double loc = 0.0;
#pragma unroll 4
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < N; r += gridDim.x * blockDim.x) {
        float2 v = q[r];
        if (pen) {
            const float2 t = pen == 2 ? reg_ct_at(reg, r) : dhwd_at(p, w, r, gd);
            v.x += lambda * t.x;
            v.y += lambda * t.y;
            q[r] = v;
        }
        const float2 pv = p[r];
        loc += (double)pv.x * v.x + (double)pv.y * v.y;
    }
    const double b = block_sum(loc, sh);
    if (threadIdx.x == 0) dots[T_PQ * kTBlocks + blockIdx.x] = b;
}

// alpha = beta2 / Re<p,q>; x += alpha p; r -= alpha q; partial |r|^2
__global__ void __launch_bounds__(kVB) k_t_update(float2 *__restrict__ x, float2 *__restrict__ r,
                                                  const float2 *__restrict__ p,
                                                  const float2 *__restrict__ q, int N,
                                                  double *dots) {
    __shared__ double sh[33];
    TScal *S = scal(dots);
    if (S->done) return;
    const double pq = sum_partials(dots + T_PQ * kTBlocks, kTBlocks, sh);
    const float alpha = (float)(S->beta2[S->cur] / pq);
    double loc = 0.0;
#pragma unroll 4
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
        const float2 pv = p[i], qv = q[i];
        float2 xv = x[i], rv = r[i];
        xv.x += alpha * pv.x;
        xv.y += alpha * pv.y;
        rv.x -= alpha * qv.x;
        rv.y -= alpha * qv.y;
        x[i] = xv;
        r[i] = rv;
        loc += (double)rv.x * rv.x + (double)rv.y * rv.y;
    }
    const double b = block_sum(loc, sh);
    if (threadIdx.x == 0) dots[T_RR * kTBlocks + blockIdx.x] = b;
}

// p = r + (beta2_new / beta2) p; best-residual tracking.  The last block to
// finish (arrival counter) closes the update: best residual, beta2 swap,
// iteration count and the stopping test (recon.cu:2107-2112).  Every block
// has read the scalars it uses before it arrives, so the update of the
// scalars cannot race with those reads.
__global__ void __launch_bounds__(kVB) k_t_dir(float2 *__restrict__ p,
                                               const float2 *__restrict__ r,
                                               const float2 *__restrict__ x,
                                               float2 *__restrict__ best, int N, double *dots) {
    __shared__ double sh[33];
    TScal *S = scal(dots);
    if (S->done) return;
    const double bnew = sum_partials(dots + T_RR * kTBlocks, kTBlocks, sh);
    const int cur = S->cur;
    const double bold = S->beta2[cur];
    const float ratio = (float)(bnew / bold);
    const bool better = bnew < S->res_best;
#pragma unroll 4
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
        const float2 rv = r[i], pv = p[i];
        p[i] = make_float2(rv.x + ratio * pv.x, rv.y + ratio * pv.y);
        if (better) best[i] = x[i];
    }
    __syncthreads();  // the block's reads of the scalars are done
    if (threadIdx.x == 0) {
        __threadfence();
        if (atomicAdd(&S->arrive, 1u) == gridDim.x - 1) {
            __threadfence();
            S->beta2[cur ^ 1] = bnew;
            if (bnew < S->res_best) S->res_best = bnew;
            S->cur = cur ^ 1;
            S->iters += 1;
            if (sqrt(bnew / S->norm_fhd) < S->tol) S->done = 1;
            S->arrive = 0;
        }
    }
}

__global__ void k_t_setup(double *dots, double tol) {
    TScal *S = scal(dots);
    S->tol = tol;
    S->iters = 0;
    S->arrive = 0;
}

// TV-pass start: r = fhd - q; p = r; partial |r|^2
__global__ void __launch_bounds__(kVB) k_t_init(float2 *r, float2 *p, const float2 *fhd,
                                                const float2 *q, int N, double *dots) {
    __shared__ double sh[33];
    double loc = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
        const float2 f = fhd[i], qv = q[i];
        const float2 rv = make_float2(f.x - qv.x, f.y - qv.y);
        r[i] = rv;
        p[i] = rv;
        loc += (double)rv.x * rv.x + (double)rv.y * rv.y;
    }
    const double b = block_sum(loc, sh);
    if (threadIdx.x == 0) dots[T_RR * kTBlocks + blockIdx.x] = b;
}

__global__ void __launch_bounds__(kVB) k_t_init_finish(double *dots) {
    __shared__ double sh[33];
    const double rr = sum_partials(dots + T_RR * kTBlocks, kTBlocks, sh);
    if (threadIdx.x == 0) {
        TScal *S = scal(dots);
        S->cur = 0;
        S->beta2[0] = rr;
        S->res_best = rr;
        S->done = 0;
    }
}

__global__ void __launch_bounds__(kVB) k_t_norm(const float2 *f, int N, double *dots) {
    __shared__ double sh[33];
    double loc = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
        const float2 v = f[i];
        loc += (double)v.x * v.x + (double)v.y * v.y;
    }
    const double b = block_sum(loc, sh);
    if (threadIdx.x == 0) dots[T_NORM * kTBlocks + blockIdx.x] = b;
}

__global__ void __launch_bounds__(kVB) k_t_norm_finish(double *dots) {
    __shared__ double sh[33];
    const double n = sum_partials(dots + T_NORM * kTBlocks, kTBlocks, sh);
    if (threadIdx.x == 0) scal(dots)->norm_fhd = n;
}

__global__ void k_soa2c(float2 *o, const float *r, const float *i, size_t n) {
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n;
         k += (size_t)gridDim.x * blockDim.x)
        o[k] = make_float2(r[k], i[k]);
}

__global__ void k_c2soa(float *r, float *i, const float2 *o, size_t n) {
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n;
         k += (size_t)gridDim.x * blockDim.x) {
        r[k] = o[k].x;
        i[k] = o[k].y;
    }
}

__global__ void k_fillf(float *w, float v, size_t n) {
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n;
         k += (size_t)gridDim.x * blockDim.x)
        w[k] = v;
}

int gridn(size_t n) {
    return (int)std::min<size_t>(std::max<size_t>((n + kVB - 1) / kVB, 1), 148 * 16);
}

float beatty_beta(float os) {
    const float v = (os - 0.5f) * (os - 0.5f) * (kKW * kKW * 4.0f) / (os * os) - 0.8f;
    return kPiF * std::sqrt(v);
}

}  // namespace

// The output crop the post kernels read after the inverse transform of a
// gridding grid, as half-lengths per FFT axis (grid_image_value: along each
// axis the image's img/2 cells on either side of index 0).
struct Crop {
    int v[3];
};
static Crop crop_of(const GridSpec &g) {
    if (g.is3d) return Crop{{g.img[0] / 2, g.img[1] / 2, g.img[2] / 2}};
    return Crop{{0, g.img[0] / 2, g.img[1] / 2}};
}

// Blocks of the warp-per-sample gridding: resident blocks of 8 warps on every
// SM a few times over (grid-stride over the samples).
static unsigned grid_blocks() { return 148u * 8u; }

GridSpec grid_spec(const int img[3], float os, bool beta_after_rounding, float kscale) {
    GridSpec g;
    for (int a = 0; a < 3; ++a) g.img[a] = img[a];
    g.is3d = img[2] > 1;
    const float beta_before = beatty_beta(os);
    float osr;
    if (!g.is3d)
        osr = 2.0f * std::ceil((os * (float)img[0]) / 2.0f) / (float)img[0];
    else
        osr = 4.0f * std::ceil((os * (float)img[2]) / 4.0f) / (float)img[2];
    g.os = osr;
    g.beta = beta_after_rounding ? beatty_beta(osr) : beta_before;
    g.gs[0] = (int)std::ceil(osr * (float)img[0]);
    g.gs[1] = (int)std::ceil(osr * (float)img[1]);
    if (g.gs[0] % 2) g.gs[0] += 1;
    if (g.gs[1] % 2) g.gs[1] += 1;
    g.gs[2] = g.is3d ? (int)std::ceil(osr * (float)img[2]) : 1;
    g.kscale = kscale;
    return g;
}

#define T_TRY(x)                                \
    do {                                        \
        cudaError_t e_ = (x);                   \
        if (e_ != cudaSuccess) return e_;       \
    } while (0)

ToepSolver::~ToepSolver() { release(); }

void ToepSolver::release() {
    if (g_iter_) cudaGraphExecDestroy(g_iter_);
    g_iter_ = nullptr;
    for (GridFft *f : {&gf2_, &gf1_, &gfq_, &gff_}) {
        grid_fft_destroy(f);
        *f = GridFft();
    }
    reg_.release();
    void *bufs[] = {sens_, eph_, fm_, qf_, big_, x_, r_, p_, q_, best_, fhd_, w_, dots_,
                    t_, grid_, qf2_, b1_, tw_};
    for (void *b : bufs)
        if (b) cudaFree(b);
    sens_ = eph_ = qf_ = big_ = x_ = r_ = p_ = q_ = best_ = fhd_ = grid_ = nullptr;
    qf2_ = b1_ = tw_ = nullptr;
    fast_ = false;
    fm_ = w_ = t_ = nullptr;
    dots_ = nullptr;
    grid_cells_ = 0;
}

cudaError_t ToepSolver::setup(const ToepConfig &cfg, const float *t, const float *fm,
                              const float *sensi_r, const float *sensi_i, unsigned *dev_err,
                              cudaStream_t st) {
    // Same sizes and stream: keep buffers, FFT plans and (same CG terms) the
    // captured iteration graph; only the per-call inputs are refreshed.
    const bool same_shape = dots_ && st == st_ && cfg.nx == cfg_.nx && cfg.ny == cfg_.ny &&
                            cfg.nz == cfg_.nz && cfg.C == cfg_.C && cfg.M == cfg_.M &&
                            (int)cfg.ntime_segs == L_;
    if (same_shape) {
        if (g_iter_ && (cfg.fd != cfg_.fd || cfg.lambda != cfg_.lambda ||
                        cfg.use_graphs != cfg_.use_graphs)) {
            cudaGraphExecDestroy(g_iter_);
            g_iter_ = nullptr;
        }
        cfg_ = cfg;
        err_ = dev_err;
        float tb[2] = {0.f, 0.f};
        T_TRY(cudaMemcpyAsync(&tb[0], t, sizeof(float), cudaMemcpyDeviceToHost, st));
        T_TRY(cudaMemcpyAsync(&tb[1], t + cfg.M - 1, sizeof(float), cudaMemcpyDeviceToHost, st));
        T_TRY(cudaStreamSynchronize(st));
        tau_ = cfg.ntime_segs > 0.f ? (tb[1] - tb[0]) / cfg.ntime_segs : (tb[1] - tb[0]);
        t0_ = tb[0];
        const int L1 = L_ + 1, C = cfg.C;
        T_TRY(cudaMemcpyAsync(t_, t, sizeof(float) * cfg.M, cudaMemcpyDeviceToDevice, st));
        k_pack_sens_c<<<gridn((size_t)C * N_), kVB, 0, st>>>(sens_, sensi_r, sensi_i,
                                                            (size_t)C * N_);
        k_eph<<<gridn((size_t)L1 * N_), kVB, 0, st>>>(eph_, fm, N_, L1, tau_, t0_);
        launches_ = 2;
        T_TRY(cudaGetLastError());
        return set_reg();
    }
    release();
    cfg_ = cfg;
    st_ = st;
    err_ = dev_err;
    L_ = (int)cfg.ntime_segs;
    const bool is3d = cfg.nz > 1;
    N_ = (size_t)cfg.nx * cfg.ny * cfg.nz;
    if (!is3d) {
        nv[0] = cfg.nx;
        nv[1] = cfg.ny;
        nv[2] = 1;
        n2[0] = 2 * cfg.nx;
        n2[1] = 2 * cfg.ny;
        n2[2] = 1;
    } else {
        nv[0] = cfg.ny;
        nv[1] = cfg.nx;
        nv[2] = cfg.nz;
        n2[0] = 2 * cfg.ny;
        n2[1] = 2 * cfg.nx;
        n2[2] = 2 * cfg.nz;
    }
    G2_ = (size_t)n2[0] * n2[1] * n2[2];
    // tau = (t[M-1] - t[0]) / L (toeplitz/computeFH.cmem.cu:1227-1229)
    float tb[2] = {0.f, 0.f};
    T_TRY(cudaMemcpyAsync(&tb[0], t, sizeof(float), cudaMemcpyDeviceToHost, st));
    T_TRY(cudaMemcpyAsync(&tb[1], t + cfg.M - 1, sizeof(float), cudaMemcpyDeviceToHost, st));
    T_TRY(cudaStreamSynchronize(st));
    tau_ = cfg.ntime_segs > 0.f ? (tb[1] - tb[0]) / cfg.ntime_segs : (tb[1] - tb[0]);
    t0_ = tb[0];
    const int L1 = L_ + 1, C = cfg.C;
    T_TRY(cudaMalloc(&t_, sizeof(float) * cfg.M));
    T_TRY(cudaMemcpyAsync(t_, t, sizeof(float) * cfg.M, cudaMemcpyDeviceToDevice, st));
    T_TRY(cudaMalloc(&sens_, sizeof(float2) * C * N_));
    T_TRY(cudaMalloc(&eph_, sizeof(float2) * L1 * N_));
    // The pruned FFT engine needs power-of-two image sizes; other sizes (and
    // IMP_TOEP_PADDED=1) use the zero-padded chain on the grid transform.
    const char *force_padded = std::getenv("IMP_TOEP_PADDED");
    fast_ = !(force_padded && force_padded[0] == '1') &&
            toep_fft_plan(nv[0], is3d ? nv[1] : 1, is3d ? nv[2] : nv[1], C, &fp_);
    if (fast_) {
        T_TRY(cudaMalloc(&qf_, sizeof(float2) * G2_));  // one segment, before permutation
        T_TRY(cudaMalloc(&qf2_, sizeof(float2) * L1 * G2_));
        T_TRY(cudaMalloc(&b1_, sizeof(float2) * fp_.b1_elems()));
        T_TRY(toep_fft_twiddles(&tw_));
    } else {
        T_TRY(cudaMalloc(&qf_, sizeof(float2) * L1 * G2_));
        T_TRY(cudaMalloc(&big_, sizeof(float2) * C * G2_));
    }
    for (float2 **b : {&x_, &r_, &p_, &q_, &best_, &fhd_}) T_TRY(cudaMalloc(b, sizeof(float2) * N_));
    T_TRY(cudaMalloc(&w_, sizeof(float) * N_));
    T_TRY(cudaMalloc(&dots_, sizeof(double) * (T_SCAL * kTBlocks + 8)));
    T_TRY(cudaMemsetAsync(dots_, 0, sizeof(double) * (T_SCAL * kTBlocks + 8), st));
    k_pack_sens_c<<<gridn((size_t)C * N_), kVB, 0, st>>>(sens_, sensi_r, sensi_i, (size_t)C * N_);
    k_eph<<<gridn((size_t)L1 * N_), kVB, 0, st>>>(eph_, fm, N_, L1, tau_, t0_);
    T_TRY(cudaGetLastError());
    // the 2N grid: batched over the coils for the zero-padded chain, single
    // for Qf_l (2-D grids are [n2[0]][n2[1]], 3-D [n2[0]][n2[1]][n2[2]])
    const int d0 = is3d ? n2[0] : 1, d1 = is3d ? n2[1] : n2[0], d2 = is3d ? n2[2] : n2[1];
    if (!fast_) T_TRY(grid_fft_create(&gf2_, d0, d1, d2, C));
    T_TRY(grid_fft_create(&gf1_, d0, d1, d2, 1));
    launches_ = 2;
    return set_reg();
}

cudaError_t ToepSolver::ensure_grid_plan(const GridSpec &g, GridFft *plan) {
    const int d0 = g.is3d ? g.gs[0] : 1, d1 = g.is3d ? g.gs[1] : g.gs[0];
    const int d2 = g.is3d ? g.gs[2] : g.gs[1];
    if (plan->tw[0] || plan->tw[1] || plan->tw[2]) {
        if (plan->n[0] == d0 && plan->n[1] == d1 && plan->n[2] == d2) return cudaSuccess;
    }
    T_TRY(grid_fft_create(plan, d0, d1, d2, 1));
    if (g.cells() > grid_cells_) {
        if (grid_) cudaFree(grid_);
        grid_ = nullptr;
        T_TRY(cudaMalloc(&grid_, sizeof(float2) * g.cells()));
        grid_cells_ = g.cells();
    }
    return cudaSuccess;
}

cudaError_t ToepSolver::compute_q(const float *kx, const float *ky, const float *kz,
                                  float *q_out_r, float *q_out_i) {
    const bool is3d = cfg_.nz > 1;
    const int img[3] = {2 * cfg_.nx, 2 * cfg_.ny, is3d ? 2 * cfg_.nz : 1};
    const GridSpec g = grid_spec(img, cfg_.os_q, true, 2.0f);
    T_TRY(ensure_grid_plan(g, &gfq_));
    const NV n2d{{n2[0], n2[1], n2[2]}};
    for (int l = 0; l <= L_; ++l) {
        T_TRY(cudaMemsetAsync(grid_, 0, sizeof(float2) * g.cells(), st_));
        k_grid_w<<<grid_blocks(), kGridWarps * 32, 0, st_>>>(grid_, kx, ky, kz, t_, nullptr,
                                                             nullptr, cfg_.M, g, tau_, t0_, l);
        T_TRY(cudaGetLastError());
        T_TRY(grid_fft_exec_cropped(gfq_, grid_, true, crop_of(g).v, st_));
        float2 *qf_l = fast_ ? qf_ : qf_ + (size_t)l * G2_;
        k_q_post<<<gridn(G2_), kVB, 0, st_>>>(grid_, g, n2d, qf_l,
                                             q_out_r ? q_out_r + (size_t)l * G2_ : nullptr,
                                             q_out_i ? q_out_i + (size_t)l * G2_ : nullptr, G2_);
        T_TRY(cudaGetLastError());
        T_TRY(grid_fft_exec(gf1_, qf_l, false, st_));
        launches_ += 2 + gfq_.passes() + gf1_.passes();
        if (fast_) {
            T_TRY(toep_fft_qf(fp_, qf2_ + (size_t)l * G2_, qf_l, 1.0f / (float)G2_, st_));
            ++launches_;
        }
    }
    return cudaStreamSynchronize(st_);
}

cudaError_t ToepSolver::load_q(const float *q_r, const float *q_i) {
    const NV n2d{{n2[0], n2[1], n2[2]}};
    for (int l = 0; l <= L_; ++l) {
        float2 *qf_l = fast_ ? qf_ : qf_ + (size_t)l * G2_;
        k_q_shift<<<gridn(G2_), kVB, 0, st_>>>(q_r + (size_t)l * G2_, q_i + (size_t)l * G2_, n2d,
                                              cfg_.nz > 1, qf_l, G2_);
        T_TRY(cudaGetLastError());
        T_TRY(grid_fft_exec(gf1_, qf_l, false, st_));
        launches_ += 1 + gf1_.passes();
        if (fast_) {
            T_TRY(toep_fft_qf(fp_, qf2_ + (size_t)l * G2_, qf_l, 1.0f / (float)G2_, st_));
            ++launches_;
        }
    }
    return cudaStreamSynchronize(st_);
}

cudaError_t ToepSolver::compute_fhd(const float *kx, const float *ky, const float *kz,
                                    const float *kd_r, const float *kd_i, float *fhd_r,
                                    float *fhd_i) {
    const bool is3d = cfg_.nz > 1;
    const int img[3] = {cfg_.nx, cfg_.ny, cfg_.nz};
    const GridSpec g = grid_spec(img, cfg_.os_fh, false, 1.0f);
    T_TRY(ensure_grid_plan(g, &gff_));
    const NV nvd{{nv[0], nv[1], nv[2]}};
    (void)is3d;
    T_TRY(cudaMemsetAsync(fhd_, 0, sizeof(float2) * N_, st_));
    for (int c = 0; c < cfg_.C; ++c)
        for (int l = 0; l <= L_; ++l) {
            T_TRY(cudaMemsetAsync(grid_, 0, sizeof(float2) * g.cells(), st_));
            k_grid_w<<<grid_blocks(), kGridWarps * 32, 0, st_>>>(
                grid_, kx, ky, kz, t_, kd_r + (size_t)c * cfg_.M, kd_i + (size_t)c * cfg_.M,
                cfg_.M, g, tau_, t0_, l);
            T_TRY(cudaGetLastError());
            T_TRY(grid_fft_exec_cropped(gff_, grid_, true, crop_of(g).v, st_));
            k_fh_post<<<gridn(N_), kVB, 0, st_>>>(grid_, g, nvd, N_, sens_ + (size_t)c * N_,
                                                 eph_ + (size_t)l * N_, fhd_);
            T_TRY(cudaGetLastError());
            launches_ += 2 + gff_.passes();
        }
    if (fhd_r) {
        k_c2soa<<<gridn(N_), kVB, 0, st_>>>(fhd_r, fhd_i, fhd_, N_);
        T_TRY(cudaGetLastError());
        ++launches_;
    }
    return cudaStreamSynchronize(st_);
}

// q = A^H A p over all segments and coils (no TV term)
cudaError_t ToepSolver::apply_aha(const float2 *p, float2 *q) {
    const bool is3d = cfg_.nz > 1;
    NV nvv{{nv[0], nv[1], nv[2]}};
    const int C = cfg_.C;
    const float scale = 1.0f / (float)G2_;
    const double *dots = dots_;
    if (fast_) {
        const int *done = reinterpret_cast<const int *>(
            reinterpret_cast<const char *>(dots_ + T_SCAL * kTBlocks) + offsetof(TScal, done));
        for (int l = 0; l <= L_; ++l)
            T_TRY(toep_fft_apply_l(fp_, q, p, sens_, eph_ + (size_t)l * N_, b1_,
                                   qf2_ + (size_t)l * G2_, l == 0 ? 1 : 0, done, tw_, err_,
                                   st_));
        return cudaSuccess;
    }
    for (int l = 0; l <= L_; ++l) {
        const float2 *eph_l = eph_ + (size_t)l * N_;
        T_TRY(cudaMemsetAsync(big_, 0, sizeof(float2) * C * G2_, st_));
        k_pad<<<gridn(N_), kVB, 0, st_>>>(big_, p, sens_, eph_l, nvv, is3d, N_, G2_, C, dots);
        T_TRY(cudaGetLastError());
        T_TRY(grid_fft_exec(gf2_, big_, false, st_));
        k_mulq<<<gridn((size_t)C * G2_), kVB, 0, st_>>>(big_, qf_ + (size_t)l * G2_, G2_, C, dots);
        T_TRY(cudaGetLastError());
        T_TRY(grid_fft_exec(gf2_, big_, true, st_));
        k_crop_acc<<<gridn(N_), kVB, 0, st_>>>(q, big_, sens_, eph_l, nvv, is3d, N_, G2_, C,
                                              l == 0 ? 1 : 0, scale, dots);
        T_TRY(cudaGetLastError());
    }
    return cudaSuccess;
}

const int *ToepSolver::done_flag() const {
    return reinterpret_cast<const int *>(
        reinterpret_cast<const char *>(dots_ + T_SCAL * kTBlocks) + offsetof(TScal, done));
}

// -reg takes precedence over -fd (toeplitz/recon.cu:1543-1680)
cudaError_t ToepSolver::penalty_dot(float2 *q, const float2 *p) {
    const Grid3 gd{nv[0], nv[1], nv[2]};
    const int pen = reg_.on() ? 2 : cfg_.fd ? 1 : 0;
    if (pen == 2) {
        T_TRY(reg_.apply_cw(p, w_, done_flag(), st_));
        ++launches_;
    }
    k_t_tvdot<<<kTBlocks, kVB, 0, st_>>>(q, p, w_, (int)N_, gd, pen, cfg_.lambda, reg_.view(),
                                        dots_);
    return cudaGetLastError();
}

cudaError_t ToepSolver::set_reg() {
    if (!cfg_.reg) {
        if (reg_.on()) {
            reg_.release();
            if (g_iter_) cudaGraphExecDestroy(g_iter_);
            g_iter_ = nullptr;
        }
        return cudaSuccess;
    }
    const bool was_on = reg_.on();
    bool moved = false;
    T_TRY(reg_.set(*cfg_.reg, (int)N_, st_, &moved));
    if ((moved || !was_on) && g_iter_) {
        cudaGraphExecDestroy(g_iter_);
        g_iter_ = nullptr;
    }
    return cudaSuccess;
}

cudaError_t ToepSolver::cg_iteration() {
    const Grid3 gd{nv[0], nv[1], nv[2]};
    T_TRY(apply_aha(p_, q_));
    T_TRY(penalty_dot(q_, p_));
    k_t_update<<<kTBlocks, kVB, 0, st_>>>(x_, r_, p_, q_, (int)N_, dots_);
    k_t_dir<<<kTBlocks, kVB, 0, st_>>>(p_, r_, x_, best_, (int)N_, dots_);
    return cudaGetLastError();
}

static cudaError_t capture_graph(cudaStream_t st, cudaGraphExec_t *exec,
                                 cudaError_t (ToepSolver::*fn)(), ToepSolver *self) {
    T_TRY(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    cudaError_t body = (self->*fn)();
    cudaGraph_t graph = nullptr;
    cudaError_t end = cudaStreamEndCapture(st, &graph);
    if (body != cudaSuccess) {
        if (graph) cudaGraphDestroy(graph);
        return body;
    }
    if (end != cudaSuccess) return end;
    cudaError_t inst = cudaGraphInstantiate(exec, graph, 0);
    cudaGraphDestroy(graph);
    return inst;
}

cudaError_t ToepSolver::solve(const float *fhd_r, const float *fhd_i, float *x_r, float *x_i) {
    const Grid3 gd{nv[0], nv[1], nv[2]};
    const int N = (int)N_;
    if (fhd_r) {
        k_soa2c<<<gridn(N_), kVB, 0, st_>>>(fhd_, fhd_r, fhd_i, N_);
        T_TRY(cudaGetLastError());
    }
    T_TRY(cudaMemsetAsync(x_, 0, sizeof(float2) * N_, st_));
    T_TRY(cudaMemsetAsync(best_, 0, sizeof(float2) * N_, st_));
    k_fillf<<<gridn(N_), kVB, 0, st_>>>(w_, 1.f, N_);
    k_t_norm<<<kTBlocks, kVB, 0, st_>>>(fhd_, N, dots_);
    k_t_norm_finish<<<1, kVB, 0, st_>>>(dots_);
    k_t_setup<<<1, 1, 0, st_>>>(dots_, 1.0e-16);  // recon.cu:2112
    T_TRY(cudaGetLastError());
    launches_ += 5;
    const int iter_launches = 3 * (L_ + 1) + 3 + (reg_.on() ? 1 : 0);  // one CG iteration
    if (cfg_.use_graphs && !g_iter_) T_TRY(capture_graph(st_, &g_iter_, &ToepSolver::cg_iteration, this));
    for (int tv_i = 0; tv_i < std::max(cfg_.tv ? cfg_.tv_num : 1, 1); ++tv_i) {
        if (tv_i != 0) {
            T_TRY(tv_weight(w_, x_, N, gd, cfg_.tv_eps, st_));
            ++launches_;
        }
        // r = F^H d - A x; p = r; beta2 = resBest = |r|^2   (recon.cu:2036-2057)
        T_TRY(cudaMemsetAsync(reinterpret_cast<char *>(dots_ + T_SCAL * kTBlocks) +
                                  offsetof(TScal, done),
                              0, sizeof(int), st_));
        T_TRY(apply_aha(x_, q_));
        T_TRY(penalty_dot(q_, x_));
        k_t_init<<<kTBlocks, kVB, 0, st_>>>(r_, p_, fhd_, q_, N, dots_);
        k_t_init_finish<<<1, kVB, 0, st_>>>(dots_);
        T_TRY(cudaGetLastError());
        launches_ += 3 * (L_ + 1) + 3;
        for (int it = 0; it < cfg_.cg_num; ++it) {
            if (g_iter_)
                T_TRY(cudaGraphLaunch(g_iter_, st_));
            else
                T_TRY(cg_iteration());
            launches_ += iter_launches;
        }
        if (!cfg_.tv) break;
    }
    k_c2soa<<<gridn(N_), kVB, 0, st_>>>(x_r, x_i, best_, N_);
    T_TRY(cudaGetLastError());
    ++launches_;
    return cudaSuccess;
}

cudaError_t ToepSolver::solve_from(const float *fhd_r, const float *fhd_i, float *x_r,
                                   float *x_i, double tol, int max_iter, int *iters) {
    const Grid3 gd{nv[0], nv[1], nv[2]};
    const int N = (int)N_;
    if (fhd_r) k_soa2c<<<gridn(N_), kVB, 0, st_>>>(fhd_, fhd_r, fhd_i, N_);
    k_soa2c<<<gridn(N_), kVB, 0, st_>>>(x_, x_r, x_i, N_);
    T_TRY(cudaMemcpyAsync(best_, x_, sizeof(float2) * N_, cudaMemcpyDeviceToDevice, st_));
    k_fillf<<<gridn(N_), kVB, 0, st_>>>(w_, 1.f, N_);
    k_t_norm<<<kTBlocks, kVB, 0, st_>>>(fhd_, N, dots_);
    k_t_norm_finish<<<1, kVB, 0, st_>>>(dots_);
    k_t_setup<<<1, 1, 0, st_>>>(dots_, tol);
    T_TRY(cudaGetLastError());
    launches_ += 6;
    if (cfg_.use_graphs && !g_iter_) T_TRY(capture_graph(st_, &g_iter_, &ToepSolver::cg_iteration, this));
    // The kernels return at once while `done` is set (a previous solve may have
    // stopped on its tolerance): clear it before the first A^H A.
    T_TRY(cudaMemsetAsync(reinterpret_cast<char *>(dots_ + T_SCAL * kTBlocks) +
                              offsetof(TScal, done),
                          0, sizeof(int), st_));
    // r = F^H d - A x0; p = r
    T_TRY(apply_aha(x_, q_));
    T_TRY(penalty_dot(q_, x_));
    k_t_init<<<kTBlocks, kVB, 0, st_>>>(r_, p_, fhd_, q_, N, dots_);
    k_t_init_finish<<<1, kVB, 0, st_>>>(dots_);
    T_TRY(cudaGetLastError());
    launches_ += 3 * (L_ + 1) + 3;
    const int iter_launches = 3 * (L_ + 1) + 3 + (reg_.on() ? 1 : 0);
    const TScal *S = reinterpret_cast<const TScal *>(dots_ + T_SCAL * kTBlocks);
    int it = 0;
    while (it < max_iter) {
        const int chunk = std::min(4, max_iter - it);
        for (int k = 0; k < chunk; ++k) {
            if (g_iter_)
                T_TRY(cudaGraphLaunch(g_iter_, st_));
            else
                T_TRY(cg_iteration());
            launches_ += iter_launches;
        }
        it += chunk;
        int done = 0;
        T_TRY(cudaMemcpyAsync(&done, &S->done, sizeof(int), cudaMemcpyDeviceToHost, st_));
        T_TRY(cudaStreamSynchronize(st_));
        if (done) break;
    }
    if (iters) {
        T_TRY(cudaMemcpyAsync(iters, &S->iters, sizeof(int), cudaMemcpyDeviceToHost, st_));
        T_TRY(cudaStreamSynchronize(st_));
    }
    k_c2soa<<<gridn(N_), kVB, 0, st_>>>(x_r, x_i, best_, N_);
    ++launches_;
    return cudaGetLastError();
}

cudaError_t ToepSolver::apply(const float *p_r, const float *p_i, float *q_r, float *q_i) {
    k_soa2c<<<gridn(N_), kVB, 0, st_>>>(p_, p_r, p_i, N_);
    T_TRY(cudaMemsetAsync(dots_ + T_SCAL * kTBlocks, 0, sizeof(TScal), st_));
    T_TRY(apply_aha(p_, q_));
    if (cfg_.fd || reg_.on()) {
        k_fillf<<<gridn(N_), kVB, 0, st_>>>(w_, 1.f, N_);
        T_TRY(penalty_dot(q_, p_));
    }
    k_c2soa<<<gridn(N_), kVB, 0, st_>>>(q_r, q_i, q_, N_);
    return cudaGetLastError();
}

}  // namespace imp

// ============================================================================
// C-ABI of the Toeplitz path
// ============================================================================
#include "context.h"
#include "nudft.cuh"

using imp::DevKeep;
using imp::fail;

namespace {

imp_status toep_args(const imp_toeplitz_options *o, int nx, int ny, int nz, int num_k) {
    if (!o) return fail(IMP_ERR_INVALID_ARG, "null options");
    if (nx <= 0 || ny <= 0 || nz <= 0 || num_k <= 0)
        return fail(IMP_ERR_INVALID_ARG, "nx, ny, nz and num_k must be > 0");
    if (nx % 2 || ny % 2 || (nz > 1 && nz % 2))
        return fail(IMP_ERR_INVALID_ARG, "image sizes must be even (half-rotation shifts)");
    if (o->ntime_segs < 0.f) return fail(IMP_ERR_INVALID_ARG, "ntime_segs must be >= 0");
    if (o->gridOS_Q < 1.f || o->gridOS_Q > 2.f || o->gridOS_FH < 1.f || o->gridOS_FH > 2.f)
        return fail(IMP_ERR_INVALID_ARG, "gridding oversampling factor should be in [1.0,2.0]");
    if (o->cg_num <= 0) return fail(IMP_ERR_INVALID_ARG, "cg_num must be > 0");
    if (o->reg) {
        const char *why = imp::sparse_reg_check(*o->reg, nx * ny * nz);
        if (why[0]) return fail(IMP_ERR_INVALID_ARG, std::string("-reg matrix: ") + why);
    }
    return IMP_OK;
}

imp::ToepConfig toep_cfg(const imp_toeplitz_options *o, int nx, int ny, int nz, int C, int M) {
    imp::ToepConfig c;
    c.nx = nx;
    c.ny = ny;
    c.nz = nz;
    c.C = C;
    c.M = M;
    c.ntime_segs = o->ntime_segs;
    c.os_q = o->gridOS_Q;
    c.os_fh = o->gridOS_FH;
    c.cg_num = o->cg_num;
    c.fd = o->enable_fd != 0;
    c.lambda = o->fd_penalizer;
    c.tv = o->enable_tv != 0;
    c.tv_num = o->enable_tv ? o->tv_num : 1;
    c.tv_eps = o->tv_eps;
    c.reg = o->reg;
    return c;
}

// The same configuration without the CG's penalty terms (Q and F^H d).
imp::ToepConfig toep_cfg_nopen(const imp_toeplitz_options *o, int nx, int ny, int nz, int C,
                               int M) {
    imp::ToepConfig c = toep_cfg(o, nx, ny, nz, C, M);
    c.reg = nullptr;
    return c;
}

imp::ToepSolver &solver_of(imp_context *ctx) {
    if (!ctx->tp) ctx->tp.reset(new imp::ToepSolver());
    return *ctx->tp;
}

// Q is coil-free: it gets its own solver, so that alternating Q and
// F^H d / CG calls (one coil versus num_coil) keep both set up instead of
// rebuilding buffers and FFT plans on every call.
imp::ToepSolver &solver_q_of(imp_context *ctx) {
    if (!ctx->tp_q) ctx->tp_q.reset(new imp::ToepSolver());
    return *ctx->tp_q;
}

imp_status copy_out(imp_context *ctx, float *dst, const float *src, size_t n) {
    IMP_CUDA(cudaMemcpyAsync(dst, src, n * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream),
             "output D2H");
    return IMP_OK;
}

}  // namespace

extern "C" {

void imp_toeplitz_options_default(imp_toeplitz_options *o) {
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->cg_num = 8;
    o->tv_num = 10;
    o->tv_eps = 1e-6f;
    o->ntime_segs = 12.f;
    o->gridOS_Q = 1.125f;
    o->gridOS_FH = 1.5f;
}

imp_status imp_toeplitz_q(imp_context *ctx, const imp_toeplitz_options *opt, float *q_r,
                          float *q_i, const float *kx, const float *ky, const float *kz,
                          const float *t, int num_k, int nx, int ny, int nz) {
    imp_status s = toep_args(opt, nx, ny, nz, num_k);
    if (s != IMP_OK) return s;
    if (!q_r || !q_i || !kx || !ky || !t || (nz > 1 && !kz))
        return fail(IMP_ERR_INVALID_ARG, "null array argument");
    if ((s = imp::begin(ctx)) != IMP_OK) return s;
    imp::stage_reset(ctx);
    DevKeep keep;
    const float *dkx, *dky, *dkz = nullptr, *dt;
    if ((s = imp::to_device_staged(ctx, kx, num_k, &dkx, nullptr)) ||
        (s = imp::to_device_staged(ctx, ky, num_k, &dky, nullptr)) ||
        (s = imp::to_device_staged(ctx, kz, nz > 1 ? num_k : 0, &dkz, nullptr)) ||
        (s = imp::to_device_staged(ctx, t, num_k, &dt, nullptr)))
        return s;
    imp::ToepSolver &ts = solver_q_of(ctx);
    IMP_CUDA(ts.setup(toep_cfg_nopen(opt, nx, ny, nz, 1, num_k), dt, nullptr, nullptr, nullptr,
                      ctx->dev_err, ctx->stream),
             "toeplitz setup");
    const size_t nq = (size_t)ts.segments() * ts.q_elems();
    float *dqr, *dqi;
    bool hr, hi;
    if ((s = imp::out_device_staged(ctx, q_r, nq, &dqr, &hr)) ||
        (s = imp::out_device_staged(ctx, q_i, nq, &dqi, &hi)))
        return s;
    IMP_CUDA(ts.compute_q(dkx, dky, dkz, dqr, dqi), "Q gridding");
    if (hr && (s = copy_out(ctx, q_r, dqr, nq))) return s;
    if (hi && (s = copy_out(ctx, q_i, dqi, nq))) return s;
    s = imp::finish(ctx);
    ctx->launches = ts.launches();
    return s;
}

imp_status imp_toeplitz_fhd(imp_context *ctx, const imp_toeplitz_options *opt, float *fhd_r,
                            float *fhd_i, const float *kdata_r, const float *kdata_i,
                            const float *kx, const float *ky, const float *kz, const float *t,
                            const float *fm, const float *sensi_r, const float *sensi_i,
                            int num_k, int num_coil, int nx, int ny, int nz) {
    imp_status s = toep_args(opt, nx, ny, nz, num_k);
    if (s != IMP_OK) return s;
    if (!fhd_r || !fhd_i || !kdata_r || !kdata_i || !kx || !ky || !t || (nz > 1 && !kz))
        return fail(IMP_ERR_INVALID_ARG, "null array argument");
    if (num_coil <= 0 || (num_coil > 1 && (!sensi_r || !sensi_i)))
        return fail(IMP_ERR_INVALID_ARG, "num_coil > 0 and sensi for num_coil > 1");
    if ((s = imp::begin(ctx)) != IMP_OK) return s;
    imp::stage_reset(ctx);
    const size_t N = (size_t)nx * ny * nz, M = num_k, C = num_coil;
    DevKeep keep;
    const float *dkx, *dky, *dkz = nullptr, *dt, *dfm = nullptr, *dsr = nullptr, *dsi = nullptr,
                      *dkr, *dki;
    if ((s = imp::to_device_staged(ctx, kx, M, &dkx, nullptr)) ||
        (s = imp::to_device_staged(ctx, ky, M, &dky, nullptr)) ||
        (s = imp::to_device_staged(ctx, kz, nz > 1 ? M : 0, &dkz, nullptr)) ||
        (s = imp::to_device_staged(ctx, t, M, &dt, nullptr)) ||
        (s = imp::to_device_staged(ctx, fm, N, &dfm, nullptr)) ||
        (s = imp::to_device_staged(ctx, num_coil > 1 ? sensi_r : nullptr, C * N, &dsr, nullptr)) ||
        (s = imp::to_device_staged(ctx, num_coil > 1 ? sensi_i : nullptr, C * N, &dsi, nullptr)) ||
        (s = imp::to_device_staged(ctx, kdata_r, C * M, &dkr, nullptr)) ||
        (s = imp::to_device_staged(ctx, kdata_i, C * M, &dki, nullptr)))
        return s;
    imp::ToepSolver &ts = solver_of(ctx);
    IMP_CUDA(ts.setup(toep_cfg_nopen(opt, nx, ny, nz, num_coil, num_k), dt, dfm, dsr, dsi,
                      ctx->dev_err, ctx->stream),
             "toeplitz setup");
    float *dfr, *dfi;
    bool hr, hi;
    if ((s = imp::out_device_staged(ctx, fhd_r, N, &dfr, &hr)) ||
        (s = imp::out_device_staged(ctx, fhd_i, N, &dfi, &hi)))
        return s;
    IMP_CUDA(ts.compute_fhd(dkx, dky, dkz, dkr, dki, dfr, dfi), "F^H d gridding");
    if (hr && (s = copy_out(ctx, fhd_r, dfr, N))) return s;
    if (hi && (s = copy_out(ctx, fhd_i, dfi, N))) return s;
    s = imp::finish(ctx);
    ctx->launches = ts.launches();
    return s;
}

static imp_status toeplitz_common(imp_context *ctx, const imp_toeplitz_options *opt,
                                  const float *q_r, const float *q_i, const float *t, int num_k,
                                  const float *fm, const float *sensi_r, const float *sensi_i,
                                  int num_coil, int nx, int ny, int nz, DevKeep &keep,
                                  imp::ToepSolver **out) {
    imp_status s = toep_args(opt, nx, ny, nz, num_k);
    if (s != IMP_OK) return s;
    if (!q_r || !q_i || !t) return fail(IMP_ERR_INVALID_ARG, "null array argument");
    if (num_coil <= 0 || (num_coil > 1 && (!sensi_r || !sensi_i)))
        return fail(IMP_ERR_INVALID_ARG, "num_coil > 0 and sensi for num_coil > 1");
    if ((s = imp::begin(ctx)) != IMP_OK) return s;
    imp::stage_reset(ctx);
    const size_t N = (size_t)nx * ny * nz, C = num_coil;
    const float *dt, *dfm = nullptr, *dsr = nullptr, *dsi = nullptr, *dqr, *dqi;
    if ((s = imp::to_device_staged(ctx, t, num_k, &dt, nullptr)) ||
        (s = imp::to_device_staged(ctx, fm, N, &dfm, nullptr)) ||
        (s = imp::to_device_staged(ctx, num_coil > 1 ? sensi_r : nullptr, C * N, &dsr, nullptr)) ||
        (s = imp::to_device_staged(ctx, num_coil > 1 ? sensi_i : nullptr, C * N, &dsi, nullptr)))
        return s;
    imp::ToepSolver &ts = solver_of(ctx);
    IMP_CUDA(ts.setup(toep_cfg(opt, nx, ny, nz, num_coil, num_k), dt, dfm, dsr, dsi,
                      ctx->dev_err, ctx->stream),
             "toeplitz setup");
    const size_t nq = (size_t)ts.segments() * ts.q_elems();
    if ((s = imp::to_device_staged(ctx, q_r, nq, &dqr, nullptr)) ||
        (s = imp::to_device_staged(ctx, q_i, nq, &dqi, nullptr)))
        return s;
    IMP_CUDA(ts.load_q(dqr, dqi), "Qf");
    *out = &ts;
    return IMP_OK;
}

imp_status imp_toeplitz_recon(imp_context *ctx, const imp_toeplitz_options *opt, float *x_r,
                              float *x_i, const float *fhd_r, const float *fhd_i,
                              const float *q_r, const float *q_i, const float *t, int num_k,
                              const float *fm, const float *sensi_r, const float *sensi_i,
                              int num_coil, int nx, int ny, int nz) {
    if (!x_r || !x_i || !fhd_r || !fhd_i) return fail(IMP_ERR_INVALID_ARG, "null array argument");
    DevKeep keep;
    imp::ToepSolver *ts = nullptr;
    imp_status s = toeplitz_common(ctx, opt, q_r, q_i, t, num_k, fm, sensi_r, sensi_i, num_coil,
                                   nx, ny, nz, keep, &ts);
    if (s != IMP_OK) return s;
    const size_t N = (size_t)nx * ny * nz;
    const float *dfr, *dfi;
    float *dxr, *dxi;
    bool hr, hi;
    if ((s = imp::to_device_staged(ctx, fhd_r, N, &dfr, nullptr)) ||
        (s = imp::to_device_staged(ctx, fhd_i, N, &dfi, nullptr)) ||
        (s = imp::out_device_staged(ctx, x_r, N, &dxr, &hr)) ||
        (s = imp::out_device_staged(ctx, x_i, N, &dxi, &hi)))
        return s;
    IMP_CUDA(ts->solve(dfr, dfi, dxr, dxi), "toeplitz CG");
    if (hr && (s = copy_out(ctx, x_r, dxr, N))) return s;
    if (hi && (s = copy_out(ctx, x_i, dxi, N))) return s;
    s = imp::finish(ctx);
    ctx->launches = ts->launches();
    return s;
}

imp_status imp_toeplitz_cg(imp_context *ctx, const imp_toeplitz_options *opt, float *x_r,
                           float *x_i, const float *fhd_r, const float *fhd_i, const float *q_r,
                           const float *q_i, const float *t, int num_k, const float *fm,
                           const float *sensi_r, const float *sensi_i, int num_coil, int nx,
                           int ny, int nz, double tol, int max_iter, int *iterations) {
    if (!x_r || !x_i || !fhd_r || !fhd_i) return fail(IMP_ERR_INVALID_ARG, "null array argument");
    if (max_iter < 0 || !(tol >= 0.0)) return fail(IMP_ERR_INVALID_ARG, "max_iter >= 0, tol >= 0");
    imp_toeplitz_options o = *opt;
    o.enable_tv = 0;  // one CG run, no reweighting passes
    DevKeep keep;
    imp::ToepSolver *ts = nullptr;
    imp_status s = toeplitz_common(ctx, &o, q_r, q_i, t, num_k, fm, sensi_r, sensi_i, num_coil,
                                   nx, ny, nz, keep, &ts);
    if (s != IMP_OK) return s;
    const size_t N = (size_t)nx * ny * nz;
    const float *dfr, *dfi, *dx0r, *dx0i;
    float *dxr, *dxi;
    bool hr, hi;
    if ((s = imp::to_device_staged(ctx, fhd_r, N, &dfr, nullptr)) ||
        (s = imp::to_device_staged(ctx, fhd_i, N, &dfi, nullptr)) ||
        (s = imp::to_device_staged(ctx, x_r, N, &dx0r, nullptr)) ||
        (s = imp::to_device_staged(ctx, x_i, N, &dx0i, nullptr)) ||
        (s = imp::out_device_staged(ctx, x_r, N, &dxr, &hr)) ||
        (s = imp::out_device_staged(ctx, x_i, N, &dxi, &hi)))
        return s;
    if (hr) IMP_CUDA(cudaMemcpyAsync(dxr, dx0r, N * 4, cudaMemcpyDeviceToDevice, ctx->stream), "x0");
    if (hi) IMP_CUDA(cudaMemcpyAsync(dxi, dx0i, N * 4, cudaMemcpyDeviceToDevice, ctx->stream), "x0");
    int it = 0;
    IMP_CUDA(ts->solve_from(dfr, dfi, dxr, dxi, tol, max_iter, &it), "toeplitz warm CG");
    if (iterations) *iterations = it;
    if (hr && (s = copy_out(ctx, x_r, dxr, N))) return s;
    if (hi && (s = copy_out(ctx, x_i, dxi, N))) return s;
    s = imp::finish(ctx);
    ctx->launches = ts->launches();
    return s;
}

imp_status imp_grid_fft(imp_context *ctx, float *data_r, float *data_i, int n0, int n1, int n2,
                        int batch, int inverse) {
    if (!data_r || !data_i) return fail(IMP_ERR_INVALID_ARG, "null array argument");
    if (n0 < 1 || n1 < 1 || n2 < 1 || batch < 1)
        return fail(IMP_ERR_INVALID_ARG, "grid sizes and batch must be >= 1");
    const size_t n = (size_t)batch * n0 * n1 * n2;
    if (n > ((size_t)1 << 31)) return fail(IMP_ERR_INVALID_ARG, "grid larger than 2^31 points");
    imp_status s = imp::begin(ctx);
    if (s != IMP_OK) return s;
    imp::GridFft f;
    const cudaError_t pe = imp::grid_fft_create(&f, n0, n1, n2, batch);
    if (pe == cudaErrorInvalidValue)
        return fail(IMP_ERR_UNSUPPORTED, "grid FFT: an axis is longer than 4096 points or has "
                                         "a prime factor above 255");
    IMP_CUDA(pe, "grid FFT plan");
    std::unique_ptr<imp::GridFft, void (*)(imp::GridFft *)> guard(&f, imp::grid_fft_destroy);
    DevKeep keep;
    const float *dr, *di;
    float *odr, *odi;
    bool hr, hi;
    if ((s = imp::to_device(ctx, data_r, n, keep, &dr, nullptr)) ||
        (s = imp::to_device(ctx, data_i, n, keep, &di, nullptr)) ||
        (s = imp::out_device(ctx, data_r, n, keep, &odr, &hr)) ||
        (s = imp::out_device(ctx, data_i, n, keep, &odi, &hi)))
        return s;
    void *buf = nullptr;
    IMP_CUDA(cudaMalloc(&buf, n * sizeof(float2)), "grid FFT buffer");
    keep.emplace_back(buf, [](void *q) { cudaFree(q); });
    float2 *b = (float2 *)buf;
    const cudaStream_t st = ctx->stream;
    imp::k_soa2c<<<imp::gridn(n), imp::kVB, 0, st>>>(b, dr, di, n);
    IMP_CUDA(cudaGetLastError(), "grid FFT pack");
    IMP_CUDA(imp::grid_fft_exec(f, b, inverse != 0, st), "grid FFT");
    imp::k_c2soa<<<imp::gridn(n), imp::kVB, 0, st>>>(odr, odi, b, n);
    IMP_CUDA(cudaGetLastError(), "grid FFT unpack");
    if (hr && (s = copy_out(ctx, data_r, odr, n))) return s;
    if (hi && (s = copy_out(ctx, data_i, odi, n))) return s;
    s = imp::finish(ctx);
    ctx->launches = 2 + f.passes();
    return s;
}

imp_status imp_toeplitz_apply(imp_context *ctx, const imp_toeplitz_options *opt, float *q_out_r,
                              float *q_out_i, const float *p_r, const float *p_i,
                              const float *q_r, const float *q_i, const float *t, int num_k,
                              const float *fm, const float *sensi_r, const float *sensi_i,
                              int num_coil, int nx, int ny, int nz) {
    if (!q_out_r || !q_out_i || !p_r || !p_i)
        return fail(IMP_ERR_INVALID_ARG, "null array argument");
    DevKeep keep;
    imp::ToepSolver *ts = nullptr;
    imp_status s = toeplitz_common(ctx, opt, q_r, q_i, t, num_k, fm, sensi_r, sensi_i, num_coil,
                                   nx, ny, nz, keep, &ts);
    if (s != IMP_OK) return s;
    const size_t N = (size_t)nx * ny * nz;
    const float *dpr, *dpi;
    float *dor, *doi;
    bool hr, hi;
    if ((s = imp::to_device_staged(ctx, p_r, N, &dpr, nullptr)) ||
        (s = imp::to_device_staged(ctx, p_i, N, &dpi, nullptr)) ||
        (s = imp::out_device_staged(ctx, q_out_r, N, &dor, &hr)) ||
        (s = imp::out_device_staged(ctx, q_out_i, N, &doi, &hi)))
        return s;
    IMP_CUDA(ts->apply(dpr, dpi, dor, doi), "toeplitz apply");
    if (hr && (s = copy_out(ctx, q_out_r, dor, N))) return s;
    if (hi && (s = copy_out(ctx, q_out_i, doi, N))) return s;
    s = imp::finish(ctx);
    ctx->launches = ts->launches();
    return s;
}

}  // extern "C"

// BF16 U-Net for the learned CG warm start (see unet.cuh).
//
// Convolutions are implicit GEMMs on the tensor cores (BF16 operands, FP32
// accumulation): forward and data-gradient share one kernel (the data
// gradient is the forward conv of the masked output gradient with flipped,
// transposed weights); the weight gradient is a split-K GEMM over pixels.
// The convolution runs on tcgen05 (TMA-fed stages, accumulator in tensor
// memory); a WMMA kernel with cp.async double buffering is kept as the
// alternative selected by IMP_UNET_WMMA=1.
#include "common.cuh"
#include "unet.cuh"

#include <cuda.h>
#include <cudaTypedefs.h>
#include <mma.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <random>
#include <vector>

#define U_TRY(x)                              \
    do {                                      \
        cudaError_t e_ = (x);                 \
        if (e_ != cudaSuccess) return e_;     \
    } while (0)

namespace imp {

using bf16 = __nv_bfloat16;
using namespace nvcuda;

// Arguments of one convolution launch (forward or data gradient).
struct ConvArgs {
    const bf16 *x;
    int ldx, xoff;          // input channel stride and offset
    const bf16 *w;          // [cout][ks*ks*cin]
    const float *bias;      // [cout] or null
    bf16 *y;                // BF16 output or null
    int ldy, yoff;
    float *yf;              // FP32 output or null
    int ldyf, yfoff, accumulate;
    int B, H, W, cin, cout, ks, relu;
    int up2;                // BF16 output written to the 2 x 2 block of an image of size 2H x 2W
};

namespace {

constexpr int kCT = 128;  // threads of the GEMM kernels (4 warps, 2 x 2)

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem, bool valid) {
    const unsigned s = smem_u32(smem);
    const int sz = valid ? 16 : 0;
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(sz)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
    asm volatile("cp.async.commit_group;\n" ::: "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}



// out[p][co] = act(bias + sum_{tap, ci} in[p + shift(tap)][ci] w[co][tap][ci]),
// zero padding; 64 pixels x 64 output channels per block.
template <int BK>
__global__ void __launch_bounds__(kCT) k_conv_fwd(ConvArgs a) {
    constexpr int LDA = BK + 8;
    constexpr int STAGE = 64 * LDA;
    constexpr int SMEM_AB = 2 * 2 * STAGE * (int)sizeof(bf16);
    constexpr int SMEM_C = 64 * 68 * (int)sizeof(float);
    __shared__ __align__(128) unsigned char sraw[SMEM_AB > SMEM_C ? SMEM_AB : SMEM_C];
    bf16 *As = reinterpret_cast<bf16 *>(sraw);
    bf16 *Bs = As + 2 * STAGE;
    const int P = a.B * a.H * a.W;
    const int m0 = blockIdx.x * 64, n0 = blockIdx.y * 64;
    const int K = a.ks * a.ks * a.cin;
    const int nk = K / BK;
    const int half = a.ks / 2;
    auto load = [&](int kt, int stage) {
        const int k0 = kt * BK;
        const int tap = k0 / a.cin, c0 = k0 % a.cin;
        const int dy = tap / a.ks - half, dx = tap % a.ks - half;
        constexpr int CPR = BK / 8;
        for (int id = threadIdx.x; id < 64 * CPR; id += kCT) {
            const int m = id / CPR, j = id % CPR;
            const int p = m0 + m;
            bool valid = p < P;
            const bf16 *src = a.x;
            if (valid) {
                const int xx = p % a.W, yy = (p / a.W) % a.H;
                const int ys = yy + dy, xs = xx + dx;
                valid = ys >= 0 && ys < a.H && xs >= 0 && xs < a.W;
                if (valid)
                    src = a.x + (size_t)(p + dy * a.W + dx) * a.ldx + a.xoff + c0 + j * 8;
            }
            cp_async16(As + stage * STAGE + m * LDA + j * 8, src, valid);
        }
        for (int id = threadIdx.x; id < 64 * CPR; id += kCT) {
            const int n = id / CPR, j = id % CPR;
            const int co = n0 + n;
            const bool valid = co < a.cout;
            const bf16 *src = valid ? a.w + (size_t)co * K + k0 + j * 8 : a.w;
            cp_async16(Bs + stage * STAGE + n * LDA + j * 8, src, valid);
        }
        cp_async_commit();
    };
    const int warp = threadIdx.x >> 5, wm = warp >> 1, wn = warp & 1;
    wmma::fragment<wmma::accumulator, 16, 16, 16, float> acc[2][2];
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 2; ++j) wmma::fill_fragment(acc[i][j], 0.f);
    load(0, 0);
    for (int kt = 0; kt < nk; ++kt) {
        if (kt + 1 < nk) {
            load(kt + 1, (kt + 1) & 1);
            cp_async_wait<1>();
        } else {
            cp_async_wait<0>();
        }
        __syncthreads();
        const bf16 *as = As + (kt & 1) * STAGE;
        const bf16 *bs = Bs + (kt & 1) * STAGE;
#pragma unroll
        for (int kk = 0; kk < BK / 16; ++kk) {
            wmma::fragment<wmma::matrix_a, 16, 16, 16, bf16, wmma::row_major> fa[2];
            wmma::fragment<wmma::matrix_b, 16, 16, 16, bf16, wmma::col_major> fb[2];
#pragma unroll
            for (int i = 0; i < 2; ++i)
                wmma::load_matrix_sync(fa[i], as + (wm * 32 + i * 16) * LDA + kk * 16, LDA);
#pragma unroll
            for (int j = 0; j < 2; ++j)
                wmma::load_matrix_sync(fb[j], bs + (wn * 32 + j * 16) * LDA + kk * 16, LDA);
#pragma unroll
            for (int i = 0; i < 2; ++i)
#pragma unroll
                for (int j = 0; j < 2; ++j) wmma::mma_sync(acc[i][j], fa[i], fb[j], acc[i][j]);
        }
        __syncthreads();
    }
    float *Cs = reinterpret_cast<float *>(sraw);
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 2; ++j)
            wmma::store_matrix_sync(Cs + (wm * 32 + i * 16) * 68 + wn * 32 + j * 16, acc[i][j], 68,
                                    wmma::mem_row_major);
    __syncthreads();
    for (int idx = threadIdx.x; idx < 64 * 64; idx += kCT) {
        const int m = idx >> 6, n = idx & 63;
        const int p = m0 + m, co = n0 + n;
        if (p >= P || co >= a.cout) continue;
        float v = Cs[m * 68 + n];
        if (a.bias) v += a.bias[co];
        if (a.relu) v = fmaxf(v, 0.f);
        if (a.y) a.y[(size_t)p * a.ldy + a.yoff + co] = __float2bfloat16(v);
        if (a.yf) {
            float *d = a.yf + (size_t)p * a.ldyf + a.yfoff + co;
            *d = a.accumulate ? *d + v : v;
        }
    }
}

struct WgArgs {
    const bf16 *dz;   // [P][cout]
    const bf16 *x;    // input, channel stride ldx, offset xoff
    int ldx, xoff;
    float *dw;        // [cout][ks*ks*cin] (accumulated with atomics)
    int B, H, W, cin, cout, ks, splits;
};

// dw[co][tap][ci] += sum_p dz[p][co] x[p + shift(tap)][ci]; block = 64 x 64
// (co, ci) for one tap and one pixel range; 32 pixels per k-step.
__global__ void __launch_bounds__(kCT) k_wgrad(WgArgs a) {
    constexpr int LD = 72;
    constexpr int STAGE = 32 * LD;
    constexpr int SMEM_AB = 2 * 2 * STAGE * (int)sizeof(bf16);
    constexpr int SMEM_C = 64 * 68 * (int)sizeof(float);
    __shared__ __align__(128) unsigned char sraw[SMEM_AB > SMEM_C ? SMEM_AB : SMEM_C];
    bf16 *As = reinterpret_cast<bf16 *>(sraw);
    bf16 *Bs = As + 2 * STAGE;
    const int P = a.B * a.H * a.W;
    const int taps = a.ks * a.ks;
    const int tap = blockIdx.z % taps, split = blockIdx.z / taps;
    const int co0 = blockIdx.x * 64, ci0 = blockIdx.y * 64;
    const int half = a.ks / 2;
    const int dy = tap / a.ks - half, dx = tap % a.ks - half;
    const int chunk = ((P + a.splits - 1) / a.splits + 31) / 32 * 32;
    const int p0 = split * chunk, p1 = min(P, p0 + chunk);
    if (p0 >= p1) return;
    const int nk = (p1 - p0 + 31) / 32;
    auto load = [&](int kt, int stage) {
        for (int id = threadIdx.x; id < 32 * 8; id += kCT) {
            const int r = id >> 3, j = id & 7;
            const int p = p0 + kt * 32 + r;
            const bool pv = p < p1;
            const bool av = pv && co0 + j * 8 < a.cout;
            cp_async16(As + stage * STAGE + r * LD + j * 8,
                       av ? a.dz + (size_t)p * a.cout + co0 + j * 8 : a.dz, av);
            bool bv = pv && ci0 + j * 8 < a.cin;
            const bf16 *src = a.x;
            if (bv) {
                const int xx = p % a.W, yy = (p / a.W) % a.H;
                const int ys = yy + dy, xs = xx + dx;
                bv = ys >= 0 && ys < a.H && xs >= 0 && xs < a.W;
                if (bv) src = a.x + (size_t)(p + dy * a.W + dx) * a.ldx + a.xoff + ci0 + j * 8;
            }
            cp_async16(Bs + stage * STAGE + r * LD + j * 8, src, bv);
        }
        cp_async_commit();
    };
    const int warp = threadIdx.x >> 5, wm = warp >> 1, wn = warp & 1;
    wmma::fragment<wmma::accumulator, 16, 16, 16, float> acc[2][2];
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 2; ++j) wmma::fill_fragment(acc[i][j], 0.f);
    load(0, 0);
    for (int kt = 0; kt < nk; ++kt) {
        if (kt + 1 < nk) {
            load(kt + 1, (kt + 1) & 1);
            cp_async_wait<1>();
        } else {
            cp_async_wait<0>();
        }
        __syncthreads();
        const bf16 *as = As + (kt & 1) * STAGE;
        const bf16 *bs = Bs + (kt & 1) * STAGE;
#pragma unroll
        for (int kk = 0; kk < 2; ++kk) {
            wmma::fragment<wmma::matrix_a, 16, 16, 16, bf16, wmma::col_major> fa[2];
            wmma::fragment<wmma::matrix_b, 16, 16, 16, bf16, wmma::row_major> fb[2];
#pragma unroll
            for (int i = 0; i < 2; ++i)
                wmma::load_matrix_sync(fa[i], as + kk * 16 * LD + wm * 32 + i * 16, LD);
#pragma unroll
            for (int j = 0; j < 2; ++j)
                wmma::load_matrix_sync(fb[j], bs + kk * 16 * LD + wn * 32 + j * 16, LD);
#pragma unroll
            for (int i = 0; i < 2; ++i)
#pragma unroll
                for (int j = 0; j < 2; ++j) wmma::mma_sync(acc[i][j], fa[i], fb[j], acc[i][j]);
        }
        __syncthreads();
    }
    float *Cs = reinterpret_cast<float *>(sraw);
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 2; ++j)
            wmma::store_matrix_sync(Cs + (wm * 32 + i * 16) * 68 + wn * 32 + j * 16, acc[i][j], 68,
                                    wmma::mem_row_major);
    __syncthreads();
    const int K = taps * a.cin;
    for (int idx = threadIdx.x; idx < 64 * 64; idx += kCT) {
        const int m = idx >> 6, n = idx & 63;
        const int co = co0 + m, ci = ci0 + n;
        if (co >= a.cout || ci >= a.cin) continue;
        atomicAdd(&a.dw[(size_t)co * K + tap * a.cin + ci], Cs[m * 68 + n]);
    }
}

// Eight BF16 <-> FP32 values as one 16-byte vector.
__device__ __forceinline__ void bf16x8_to_f32(const uint4 &q, float *f) {
    const __nv_bfloat162 *h = reinterpret_cast<const __nv_bfloat162 *>(&q);
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const float2 t = __bfloat1622float2(h[j]);
        f[2 * j] = t.x;
        f[2 * j + 1] = t.y;
    }
}
__device__ __forceinline__ uint4 f32_to_bf16x8(const float *f) {
    uint32_t w[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const __nv_bfloat162 h = __floats2bfloat162_rn(f[2 * j], f[2 * j + 1]);
        w[j] = ((uint32_t)__bfloat16_as_ushort(h.y) << 16) | __bfloat16_as_ushort(h.x);
    }
    return make_uint4(w[0], w[1], w[2], w[3]);
}

// db[co] += sum_p dz[p][co].  Thread = 8 channels x a pixel lane (cout / 8
// divides the block); lanes are summed in shared memory, then one atomic per
// channel and block.
__global__ void k_bgrad(float *db, const bf16 *dz, int P, int cout) {
    __shared__ float acc[256];
    const int groups = cout >> 3, lanes = blockDim.x / groups;
    const int cg = threadIdx.x % groups, pl = threadIdx.x / groups;
    for (int c = threadIdx.x; c < cout; c += blockDim.x) acc[c] = 0.f;
    __syncthreads();
    float s[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    for (int p = blockIdx.x * lanes + pl; p < P; p += gridDim.x * lanes) {
        float f[8];
        bf16x8_to_f32(*reinterpret_cast<const uint4 *>(dz + (size_t)p * cout + cg * 8), f);
#pragma unroll
        for (int j = 0; j < 8; ++j) s[j] += f[j];
    }
#pragma unroll
    for (int j = 0; j < 8; ++j) atomicAdd(&acc[cg * 8 + j], s[j]);
    __syncthreads();
    for (int c = threadIdx.x; c < cout; c += blockDim.x) atomicAdd(&db[c], acc[c]);
}

// dz[p][co] = g[p][goff + co] * (relu ? (y[p][yoff + co] > 0) : 1), as BF16;
// 8 channels per thread (cout, ldg, goff, ldy, yoff multiples of 8).
__global__ void k_dz(bf16 *dz, const float *g, int ldg, int goff, const bf16 *y, int ldy, int yoff,
                     int P, int cout, int relu) {
    const int groups = cout >> 3;
    const size_t n = (size_t)P * groups;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x) {
        const size_t p = i / groups;
        const int c = (int)(i - p * groups) * 8;
        const float4 *gp = reinterpret_cast<const float4 *>(g + p * ldg + goff + c);
        const float4 g0 = gp[0], g1 = gp[1];
        float v[8] = {g0.x, g0.y, g0.z, g0.w, g1.x, g1.y, g1.z, g1.w};
        if (relu) {
            float yv[8];
            bf16x8_to_f32(*reinterpret_cast<const uint4 *>(y + p * ldy + yoff + c), yv);
#pragma unroll
            for (int j = 0; j < 8; ++j)
                if (!(yv[j] > 0.f)) v[j] = 0.f;
        }
        *reinterpret_cast<uint4 *>(dz + p * cout + c) = f32_to_bf16x8(v);
    }
}

// wt[ci][taps - 1 - t][co] = w[co][t][ci]
__global__ void k_wtrans(bf16 *wt, const bf16 *w, int cin, int cout, int taps) {
    const size_t n = (size_t)cin * cout * taps;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x) {
        const int ci = (int)(i % cin);
        const size_t r = i / cin;
        const int t = (int)(r % taps);
        const int co = (int)(r / taps);
        wt[((size_t)ci * taps + (taps - 1 - t)) * cout + co] = w[i];
    }
}

// 2x2 max pooling; idx = argmax position (dy * 2 + dx), the first of equal
// maxima.  8 channels per thread (C, ldi, ioff multiples of 8).
__global__ void k_pool_fwd(bf16 *out, unsigned char *idx, const bf16 *in, int ldi, int ioff, int B,
                           int H, int W, int C) {
    const int Ho = H / 2, Wo = W / 2, G = C >> 3;
    const size_t n = (size_t)B * Ho * Wo * G;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x) {
        const int c = (int)(i % G) * 8;
        const size_t q = i / G;
        const int xo = (int)(q % Wo), yo = (int)((q / Wo) % Ho), b = (int)(q / ((size_t)Wo * Ho));
        float best[8];
        uint32_t bi[2] = {0u, 0u};
#pragma unroll
        for (int j = 0; j < 8; ++j) best[j] = -INFINITY;
#pragma unroll
        for (int d = 0; d < 4; ++d) {
            const size_t p = ((size_t)b * H + 2 * yo + (d >> 1)) * W + 2 * xo + (d & 1);
            float v[8];
            bf16x8_to_f32(*reinterpret_cast<const uint4 *>(in + p * ldi + ioff + c), v);
#pragma unroll
            for (int j = 0; j < 8; ++j)
                if (v[j] > best[j]) {
                    best[j] = v[j];
                    bi[j >> 2] = (bi[j >> 2] & ~(0xffu << (8 * (j & 3)))) | ((uint32_t)d << (8 * (j & 3)));
                }
        }
        *reinterpret_cast<uint4 *>(out + q * C + c) = f32_to_bf16x8(best);
        *reinterpret_cast<uint2 *>(idx + q * C + c) = make_uint2(bi[0], bi[1]);
    }
}

// gin[argmax pixel][goff + c] += gout[q][c]; 4 channels per thread.
__global__ void k_pool_bwd(float *gin, int ldg, int goff, const float *gout,
                           const unsigned char *idx, int B, int H, int W, int C) {
    const int Ho = H / 2, Wo = W / 2, G = C >> 2;
    const size_t n = (size_t)B * Ho * Wo * G;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x) {
        const int c = (int)(i % G) * 4;
        const size_t q = i / G;
        const int xo = (int)(q % Wo), yo = (int)((q / Wo) % Ho), b = (int)(q / ((size_t)Wo * Ho));
        const float4 g4 = *reinterpret_cast<const float4 *>(gout + q * C + c);
        const uint32_t id = *reinterpret_cast<const uint32_t *>(idx + q * C + c);
        const float gv[4] = {g4.x, g4.y, g4.z, g4.w};
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int d = (int)((id >> (8 * j)) & 3u);
            const size_t p = ((size_t)b * H + 2 * yo + (d >> 1)) * W + 2 * xo + (d & 1);
            gin[p * ldg + goff + c + j] += gv[j];
        }
    }
}

// nearest x2: out[b][y][x][off + c] = in[b][y/2][x/2][c]  (H, W: output size);
// 8 channels per thread.
__global__ void k_up_fwd(bf16 *out, int ldo, int ooff, const bf16 *in, int B, int H, int W,
                         int C) {
    const int G = C >> 3;
    const size_t n = (size_t)B * H * W * G;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x) {
        const int c = (int)(i % G) * 8;
        const size_t p = i / G;
        const int x = (int)(p % W), y = (int)((p / W) % H), b = (int)(p / ((size_t)W * H));
        const size_t pi = ((size_t)b * (H / 2) + y / 2) * (W / 2) + x / 2;
        *reinterpret_cast<uint4 *>(out + p * ldo + ooff + c) =
            *reinterpret_cast<const uint4 *>(in + pi * C + c);
    }
}

// gin[b][i][j][c] += sum of the 2 x 2 block of gout[..][goff + c]  (H, W: input
// size); 4 channels per thread.
__global__ void k_up_bwd(float *gin, const float *gout, int ldg, int goff, int B, int H, int W,
                         int C) {
    const int G = C >> 2;
    const size_t n = (size_t)B * H * W * G;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x) {
        const int c = (int)(i % G) * 4;
        const size_t p = i / G;
        const int x = (int)(p % W), y = (int)((p / W) % H), b = (int)(p / ((size_t)W * H));
        float4 s = *reinterpret_cast<const float4 *>(gin + p * C + c);
#pragma unroll
        for (int d = 0; d < 4; ++d) {
            const size_t po = ((size_t)b * 2 * H + 2 * y + (d >> 1)) * (2 * W) + 2 * x + (d & 1);
            const float4 v = *reinterpret_cast<const float4 *>(gout + po * ldg + goff + c);
            s.x += v.x;
            s.y += v.y;
            s.z += v.z;
            s.w += v.w;
        }
        *reinterpret_cast<float4 *>(gin + p * C + c) = s;
    }
}

// x [B][2][HW] -> X0 [P][16] (channels 2..15 zero); one pixel per thread.
__global__ void k_pack(bf16 *x0, const float *x, int B, int HW) {
    const size_t n = (size_t)B * HW;
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < n;
         p += (size_t)gridDim.x * blockDim.x) {
        const size_t b = p / HW, r = p % HW;
        const float f[8] = {x[(b * 2) * HW + r], x[(b * 2 + 1) * HW + r], 0.f, 0.f, 0.f, 0.f,
                            0.f, 0.f};
        uint4 *o = reinterpret_cast<uint4 *>(x0 + p * 16);
        o[0] = f32_to_bf16x8(f);
        o[1] = make_uint4(0u, 0u, 0u, 0u);
    }
}

__global__ void k_unpack(float *y, const float *outf, int B, int HW) {
    const size_t n = (size_t)B * 2 * HW;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x) {
        const size_t r = i % HW, bc = i / HW;
        const size_t b = bc / 2, c = bc % 2;
        y[i] = outf[(b * HW + r) * 16 + c];
    }
}

// gout[p][c] = 2 (out - t) / n for c < 2; per-block partial sums of (out - t)^2
__global__ void k_loss(float *gout, double *part, const float *outf, const float *t, int B,
                       int HW) {
    __shared__ double sh[33];
    const size_t n = (size_t)B * 2 * HW;
    const float sc = 2.0f / (float)n;
    double loc = 0.0;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x) {
        const size_t r = i % HW, bc = i / HW;
        const size_t b = bc / 2, c = bc % 2;
        const size_t o = (b * HW + r) * 16 + c;
        const float d = outf[o] - t[i];
        gout[o] = sc * d;
        loc += (double)d * d;
    }
    const double s = block_sum(loc, sh);
    if (threadIdx.x == 0) part[blockIdx.x] = s;
}

__global__ void k_adam(float *p, float *m, float *v, const float *g, size_t n, float lr,
                       float b1c, float b2c) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = 0.9f * m[i] + 0.1f * gi;
        const float vi = 0.999f * v[i] + 0.001f * gi * gi;
        m[i] = mi;
        v[i] = vi;
        p[i] -= lr * (mi / b1c) / (sqrtf(vi / b2c) + 1e-8f);
    }
}

__global__ void k_to_bf16(bf16 *o, const float *s, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x)
        o[i] = __float2bfloat16(s[i]);
}

// ---------------------------------------------------------------------------
// tcgen05 implicit-GEMM convolution (sm_100a).  One block computes a patch of
// 8 x 16 pixels of one image (M = 128 GEMM rows) times NT output channels
// (N), K = taps x input channels in chunks of CK channels.  Per K step the
// TMA warp loads the patch shifted by the tap, {CK, 16, 8, 1} of the NHWC
// activations (coordinates outside the image read zeros: the convolution's
// padding), and the {CK, NT} slice of the weights into one of S stages; the
// MMA warp issues CK/16 tcgen05.mma into the FP32 accumulator in tensor
// memory and releases the stage through tcgen05.commit; the four epilogue
// warps read the accumulator with tcgen05.ld and store BF16 / FP32 rows with
// bias and ReLU fused.  Every mbarrier wait is bounded.
// Both operands are K-major with the TMA swizzle whose span is one row of the
// tile (CK * 2 bytes: 32, 64 or 128 B), i.e. 8-row atoms of CK * 16 bytes,
// which is the UMMA canonical K-major swizzled layout (leading byte offset
// unused = 1, stride byte offset = one atom).
// ---------------------------------------------------------------------------
constexpr int kTcM = 128;
constexpr int kTcThreads = 192;  // warps 0-3 epilogue, warp 4 TMA, warp 5 MMA
constexpr int kTileX = 16, kTileY = 8;

// Shared-memory matrix descriptor (version 1): start address, leading byte
// offset lbo, stride byte offset sbo, swizzle layout code (2 = 128 B,
// 4 = 64 B, 6 = 32 B).  K-major swizzled operands: lbo unused (16 B), sbo =
// one 8-row atom.  MN-major swizzled operands: lbo = distance between atom
// columns along M / N, sbo = distance between 8-row groups along K.
__device__ __forceinline__ uint64_t umma_desc(unsigned saddr, unsigned lbo, unsigned sbo,
                                              unsigned layout) {
    uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;
    d |= (uint64_t)layout << 61;
    return d;
}
__device__ __forceinline__ uint64_t umma_desc_sw(unsigned saddr, unsigned sbo, unsigned layout) {
    return umma_desc(saddr, 16, sbo, layout);
}

// Swizzle layout code of a tile whose rows hold c BF16 channels (c * 2 bytes).
__host__ __device__ constexpr unsigned sw_layout(int c) {
    return c == 64 ? 2u : (c == 32 ? 4u : 6u);
}

__device__ __forceinline__ void tma_load_4d(void *dst, const CUtensorMap *tm, int c0, int c1,
                                            int c2, int c3, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(tm)), "r"(c0), "r"(c1), "r"(c2), "r"(c3),
        "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ void mbar_arrive_local(uint64_t *bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *tm, int c0, int c1,
                                            uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3}], [%4];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(tm)), "r"(c0), "r"(c1), "r"(smem_u32(bar))
        : "memory");
}

// Instruction descriptor: BF16 x BF16 -> F32, A and B K-major, M x N.
__host__ __device__ constexpr uint32_t umma_idesc_bf16(int M, int N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) |
           ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void tc_fence_after() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_before() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}

__device__ __forceinline__ bool mbar_wait_tc(uint64_t *bar, unsigned parity) {
    for (unsigned it = 0; it < (1u << 22); ++it)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

// Pipeline depth for a stage of `stage` bytes: about 96 KB of stages, so two
// persistent blocks share an SM.
__host__ __device__ constexpr int tc_stages(int stage) {
    return (96 * 1024) / stage < 2 ? 2 : ((96 * 1024) / stage > 12 ? 12 : (96 * 1024) / stage);
}

// Output tile t of a convolution: N tile fastest (blocks working on one pixel
// patch at the same time share its loads in L2), then x, y, image.
struct TcTile {
    int x0, y0, b, n0;
};
__device__ __forceinline__ TcTile tc_tile(int t, int n_nt, int tiles_x, int tiles_y, int NT) {
    TcTile r;
    r.n0 = (t % n_nt) * NT;
    t /= n_nt;
    r.x0 = (t % tiles_x) * kTileX;
    t /= tiles_x;
    r.y0 = (t % tiles_y) * kTileY;
    r.b = t / tiles_y;
    return r;
}

// Epilogue of one tile for accumulator row r (pixel r of the 8 x 16 patch):
// NT columns from tensor memory at tacc, + bias, ReLU, then 16 channels per
// vector group to the BF16 output (at the pixel, or with up2 at the 2 x 2
// block of the pixel in an image of twice the size: nearest up-sampling)
// and / or the FP32 output (optionally accumulated).
// STRIP: the tile is 128 consecutive pixels of one image row (x0 .. x0+127
// of row y0) instead of an 8 x 16 patch.
template <int NT, bool STRIP = false>
__device__ __forceinline__ void conv_tc_store(const ConvArgs &a, const TcTile &T, uint32_t tacc,
                                              int r) {
    const int xx = STRIP ? T.x0 + r : T.x0 + (r & (kTileX - 1));
    const int yy = STRIP ? T.y0 : T.y0 + r / kTileX;
    const bool valid = xx < a.W && yy < a.H;
    const size_t p = ((size_t)T.b * a.H + yy) * a.W + xx;
#pragma unroll 1
    for (int c0 = 0; c0 < NT; c0 += 16) {
        uint32_t v[16];
        __syncwarp();
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,"
            "%12,%13,%14,%15}, [%16];"
            : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]),
              "=r"(v[6]), "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]),
              "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
            : "r"(tacc + (uint32_t)c0));
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        const int co = T.n0 + c0;
        if (!valid || co >= a.cout) continue;
        float f[16];
#pragma unroll
        for (int j = 0; j < 16; ++j) {
            f[j] = __uint_as_float(v[j]);
            if (a.bias) f[j] += a.bias[co + j];
            if (a.relu) f[j] = fmaxf(f[j], 0.f);
        }
        if (a.y) {
            uint32_t qw[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const __nv_bfloat162 h = __floats2bfloat162_rn(f[2 * j], f[2 * j + 1]);
                qw[j] = ((uint32_t)__bfloat16_as_ushort(h.y) << 16) | __bfloat16_as_ushort(h.x);
            }
            const uint4 q[2] = {make_uint4(qw[0], qw[1], qw[2], qw[3]),
                                make_uint4(qw[4], qw[5], qw[6], qw[7])};
            if (a.up2) {
                const size_t W2 = 2 * (size_t)a.W;
                const size_t p0 = ((size_t)T.b * 2 * a.H + 2 * yy) * W2 + 2 * xx;
#pragma unroll
                for (int d = 0; d < 4; ++d) {
                    uint4 *o = reinterpret_cast<uint4 *>(
                        a.y + (p0 + (d >> 1) * W2 + (d & 1)) * a.ldy + a.yoff + co);
                    o[0] = q[0];
                    o[1] = q[1];
                }
            } else {
                uint4 *o = reinterpret_cast<uint4 *>(a.y + p * a.ldy + a.yoff + co);
                o[0] = q[0];
                o[1] = q[1];
            }
        }
        if (a.yf) {
            float4 *d = reinterpret_cast<float4 *>(a.yf + p * a.ldyf + a.yfoff + co);
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                float4 o = make_float4(f[4 * j], f[4 * j + 1], f[4 * j + 2], f[4 * j + 3]);
                if (a.accumulate) {
                    const float4 g = d[j];
                    o.x += g.x;
                    o.y += g.y;
                    o.z += g.z;
                    o.w += g.w;
                }
                d[j] = o;
            }
        }
    }
}

// Persistent: block i handles tiles i, i + gridDim.x, ...; the TMA warp runs
// ahead across tile boundaries, the accumulator is double-buffered in tensor
// memory so the epilogue of one tile overlaps the MMAs of the next.
template <int CK, int NT>
__global__ void __launch_bounds__(kTcThreads) k_conv_tc(const __grid_constant__ CUtensorMap tmx,
                                                         const __grid_constant__ CUtensorMap tmw,
                                                         ConvArgs a, int tiles_x, int tiles_y,
                                                         unsigned *err) {
    constexpr int A_BYTES = kTcM * CK * 2;
    constexpr int B_REAL = NT * CK * 2;
    constexpr int B_BYTES = (B_REAL + 1023) / 1024 * 1024;
    constexpr int STAGE = A_BYTES + B_BYTES;
    constexpr int S = tc_stages(STAGE);
    constexpr int ACOLS = NT < 32 ? 32 : NT;  // columns of one accumulator
    constexpr int TCOLS = 2 * ACOLS;
    constexpr uint32_t IDESC = umma_idesc_bf16(kTcM, NT);
    constexpr unsigned LAYOUT = CK == 64 ? 2u : (CK == 32 ? 4u : 6u);
    constexpr unsigned SBO = 8 * CK * 2;
    extern __shared__ unsigned char smraw[];
    __shared__ __align__(8) uint64_t full[S], empty[S], acc_full[2], acc_empty[2];
    __shared__ uint32_t tmem_sh;
    // Stage tiles start on 1024-byte boundaries (the swizzle pattern's period).
    unsigned char *sm = smraw + ((1024u - (smem_u32(smraw) & 1023u)) & 1023u);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int n_nt = (a.cout + NT - 1) / NT;
    const int n_tiles = n_nt * tiles_x * tiles_y * a.B;
    const int cpt = a.cin / CK;  // channel chunks per tap
    const int nk = a.ks * a.ks * cpt;
    const int half = a.ks / 2;
    if (warp == 5) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(&tmem_sh)),
                     "r"(TCOLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (threadIdx.x == 0) {
        for (int s = 0; s < S; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        for (int i = 0; i < 2; ++i) {
            mbar_init(&acc_full[i], 1);
            mbar_init(&acc_empty[i], 4);  // one arrival per epilogue warp
        }
        fence_mbar_init();
    }
    if (warp == 4 && lane == 0) {
        asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&tmx)) : "memory");
        asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&tmw)) : "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_sh;

    if (warp == 4) {
        if (lane == 0) {  // TMA producer
            bool ok = true;
            int g = 0;  // K steps issued by this block so far
            for (int t = blockIdx.x; t < n_tiles; t += gridDim.x) {
                const TcTile T = tc_tile(t, n_nt, tiles_x, tiles_y, NT);
                for (int k = 0; k < nk; ++k, ++g) {
                    const int s = g % S;
                    const unsigned u = (unsigned)(g / S);
                    if (g >= S && !mbar_wait_tc(&empty[s], (u - 1) & 1)) ok = false;
                    const int tap = k / cpt, c0 = (k - tap * cpt) * CK;
                    const int dy = tap / a.ks - half, dx = tap % a.ks - half;
                    unsigned char *sa = sm + s * STAGE;
                    mbar_arrive_expect_tx(&full[s], A_BYTES + B_REAL);
                    tma_load_4d(sa, &tmx, c0, T.x0 + dx, T.y0 + dy, T.b, &full[s]);
                    tma_load_2d(sa + A_BYTES, &tmw, tap * a.cin + c0, T.n0, &full[s]);
                }
            }
            if (!ok && err) atomicOr(err, DEV_ERR_TIMEOUT);
        }
        __syncwarp();
    } else if (warp == 5) {
        if (lane == 0) {  // MMA issuer
            bool ok = true;
            int g = 0, it = 0;
            for (int t = blockIdx.x; t < n_tiles; t += gridDim.x, ++it) {
                const int ab = it & 1;
                const unsigned au = (unsigned)(it >> 1);
                // the epilogue has drained this accumulator's previous tile
                if (it >= 2 && !mbar_wait_tc(&acc_empty[ab], (au - 1) & 1)) ok = false;
                tc_fence_after();
                const uint32_t dacc = tmem + (uint32_t)(ab * ACOLS);
                for (int k = 0; k < nk; ++k, ++g) {
                    const int s = g % S;
                    const unsigned u = (unsigned)(g / S);
                    if (!mbar_wait_tc(&full[s], u & 1)) ok = false;
                    tc_fence_after();
                    const unsigned sa = smem_u32(sm + s * STAGE);
                    const unsigned sb = sa + A_BYTES;
#pragma unroll
                    for (int kk = 0; kk < CK / 16; ++kk) {
                        const uint64_t da = umma_desc_sw(sa + kk * 32, SBO, LAYOUT);
                        const uint64_t db = umma_desc_sw(sb + kk * 32, SBO, LAYOUT);
                        const uint32_t acc = (k > 0 || kk > 0) ? 1u : 0u;
                        asm volatile(
                            "{\n\t.reg .pred p;\n\t"
                            "setp.ne.b32 p, %4, 0;\n\t"
                            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(
                                dacc),
                            "l"(da), "l"(db), "r"(IDESC), "r"(acc)
                            : "memory");
                    }
                    asm volatile(
                        "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 "
                        "[%0];" ::"r"(smem_u32(&empty[s]))
                        : "memory");
                }
                asm volatile(
                    "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 "
                    "[%0];" ::"r"(smem_u32(&acc_full[ab]))
                    : "memory");
            }
            if (!ok && err) atomicOr(err, DEV_ERR_TIMEOUT);
        }
        __syncwarp();
    } else {  // epilogue: warp w reads accumulator lanes (rows) 32w .. 32w + 31
        int it = 0;
        for (int t = blockIdx.x; t < n_tiles; t += gridDim.x, ++it) {
            const TcTile T = tc_tile(t, n_nt, tiles_x, tiles_y, NT);
            const int ab = it & 1;
            const unsigned au = (unsigned)(it >> 1);
            if (!mbar_wait_tc(&acc_full[ab], au & 1)) {
                if (err && lane == 0) atomicOr(err, DEV_ERR_TIMEOUT);
                mbar_wait_tc(&acc_full[ab], au & 1);  // once more, bounded
            }
            tc_fence_after();
            conv_tc_store<NT>(a, T,
                              tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(ab * ACOLS),
                              warp * 32 + lane);
            // this warp's rows of the accumulator are stored: release it
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive_local(&acc_empty[ab]);
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 5)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                     "r"(TCOLS)
                     : "memory");
}

// cuTensorMapEncodeTiled from the driver, looked up once through the runtime
// (no link-time dependency on libcuda).
PFN_cuTensorMapEncodeTiled_v12000 tmap_encoder() {
    static const PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) !=
                cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            p = nullptr;
        return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }();
    return fn;
}

template <int CK, int NT>
cudaError_t launch_conv_tc(const ConvArgs &a, unsigned *err, cudaStream_t st) {
    constexpr int STAGE = kTcM * CK * 2 + (NT * CK * 2 + 1023) / 1024 * 1024;
    constexpr int SMEM = tc_stages(STAGE) * STAGE + 1024;
    const auto enc = tmap_encoder();
    if (!enc) return cudaErrorNotSupported;
    cudaError_t e = cudaFuncSetAttribute(k_conv_tc<CK, NT>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM);
    if (e != cudaSuccess) return e;
    const CUtensorMapSwizzle swz = CK == 64 ? CU_TENSOR_MAP_SWIZZLE_128B
                                   : CK == 32 ? CU_TENSOR_MAP_SWIZZLE_64B
                                              : CU_TENSOR_MAP_SWIZZLE_32B;
    // Activations: {channel, x, y, image} of the channel slice [xoff, xoff + cin).
    CUtensorMap tmx, tmw;
    const cuuint64_t xd[4] = {(cuuint64_t)a.cin, (cuuint64_t)a.W, (cuuint64_t)a.H,
                              (cuuint64_t)a.B};
    const cuuint64_t xs[3] = {(cuuint64_t)a.ldx * 2, (cuuint64_t)a.ldx * 2 * a.W,
                              (cuuint64_t)a.ldx * 2 * a.W * a.H};
    const cuuint32_t xb[4] = {(cuuint32_t)CK, kTileX, kTileY, 1};
    const cuuint32_t one[4] = {1, 1, 1, 1};
    if (enc(&tmx, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, (void *)(a.x + a.xoff), xd, xs, xb, one,
            CU_TENSOR_MAP_INTERLEAVE_NONE, swz, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
        return cudaErrorInvalidValue;
    // Weights: {k, output channel}, k = tap * cin + input channel.
    const int K = a.ks * a.ks * a.cin;
    const cuuint64_t wd[2] = {(cuuint64_t)K, (cuuint64_t)a.cout};
    const cuuint64_t ws[1] = {(cuuint64_t)K * 2};
    const cuuint32_t wb[2] = {(cuuint32_t)CK, (cuuint32_t)NT};
    if (enc(&tmw, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, (void *)a.w, wd, ws, wb, one,
            CU_TENSOR_MAP_INTERLEAVE_NONE, swz, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
        return cudaErrorInvalidValue;
    const int tiles_x = (a.W + kTileX - 1) / kTileX, tiles_y = (a.H + kTileY - 1) / kTileY;
    const long long n_tiles = (long long)tiles_x * tiles_y * a.B * ((a.cout + NT - 1) / NT);
    if (n_tiles > 0x7fffffffLL) return cudaErrorInvalidValue;
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        return cudaErrorInvalidDevice;
    const int grid = (int)std::min<long long>(n_tiles, 2LL * sms);  // two blocks per SM
    k_conv_tc<CK, NT><<<grid, kTcThreads, SMEM, st>>>(tmx, tmw, a, tiles_x, tiles_y, err);
    return cudaGetLastError();
}

template <int CK>
cudaError_t conv_tc_n(const ConvArgs &a, unsigned *err, cudaStream_t st) {
    if (a.cout <= 16) return launch_conv_tc<CK, 16>(a, err, st);
    if (a.cout <= 32) return launch_conv_tc<CK, 32>(a, err, st);
    if (a.cout <= 64) return launch_conv_tc<CK, 64>(a, err, st);
    return launch_conv_tc<CK, 128>(a, err, st);
}

// The tensor-memory path for a convolution: channel counts multiples of 16,
// channel strides and offsets multiples of 16 (16-byte aligned TMA rows and
// vector stores).
bool conv_args_ok(const ConvArgs &a) {
    return !(a.cin % 16 || a.cout % 16 || a.ldx % 16 || a.xoff % 16 || a.xoff + a.cin > a.ldx ||
             (a.y && (a.ldy % 16 || a.yoff % 16 || a.yoff + a.cout > a.ldy)) ||
             (a.yf && (a.ldyf % 16 || a.yfoff % 16 || a.yfoff + a.cout > a.ldyf)) ||
             (a.ks != 1 && a.ks != 3) || a.B < 1 || a.H < 1 || a.W < 1 || (a.up2 && !a.y));
}

cudaError_t conv_tc(const ConvArgs &a, int, unsigned *err, cudaStream_t st) {
    if (!conv_args_ok(a)) return cudaErrorInvalidValue;
    if (a.cin % 64 == 0) return conv_tc_n<64>(a, err, st);
    if (a.cin % 32 == 0) return conv_tc_n<32>(a, err, st);
    return conv_tc_n<16>(a, err, st);
}

// ---------------------------------------------------------------------------
// Weight gradient on tcgen05:
//   dw[co][m] += sum_p x[p + shift(tap)][ci] * dz[p][co],  m = tap * cin + ci.
// GEMM rows = m (128 per block, as 128 / CA regions of CA channels of one tap),
// columns = output channels (NT per block, NT / CB regions of CB channels),
// K = pixels, one 8 x 16 patch per K step.  Both operands arrive as TMA boxes
// {CA | CB channels, 16, 8, 1} of the NHWC tensors: pixel-major rows with the
// channels contiguous, i.e. MN-major UMMA operands, one region per swizzle
// atom column (leading byte offset = region size, stride byte offset = 8
// pixel rows; a K = 16 MMA spans two 8-row groups).  The blocks of one
// (row tile, column tile) split the patches between them and add their
// accumulators to dw with FP32 atomics (coalesced along m).
// ---------------------------------------------------------------------------
__host__ __device__ constexpr int wg_stages(int stage) {
    return (200 * 1024) / stage < 2 ? 2 : ((200 * 1024) / stage > 6 ? 6 : (200 * 1024) / stage);
}

template <int CA, int NT>
__global__ void __launch_bounds__(kTcThreads) k_wgrad_tc(const __grid_constant__ CUtensorMap tmx,
                                                          const __grid_constant__ CUtensorMap tmz,
                                                          WgArgs a, int tiles_x, int tiles_y,
                                                          int n_mt, int n_nt, int per,
                                                          unsigned *err) {
    constexpr int CB = NT < 64 ? NT : 64;
    constexpr int RA = kTcM / CA, RB = NT / CB;
    constexpr int REGA = kTcM * CA * 2, REGB = kTcM * CB * 2;  // one box: 128 pixel rows
    constexpr int A_BYTES = RA * REGA, B_BYTES = RB * REGB;
    constexpr int STAGE = A_BYTES + B_BYTES;
    constexpr int S = wg_stages(STAGE);
    constexpr int TCOLS = NT < 32 ? 32 : NT;
    constexpr uint32_t IDESC = umma_idesc_bf16(kTcM, NT) | (1u << 15) | (1u << 16);  // MN-major
    constexpr unsigned SBOA = 8 * CA * 2, SBOB = 8 * CB * 2;
    extern __shared__ unsigned char smraw[];
    __shared__ __align__(8) uint64_t full[S], empty[S], done;
    __shared__ uint32_t tmem_sh;
    unsigned char *sm = smraw + ((1024u - (smem_u32(smraw) & 1023u)) & 1023u);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int u = blockIdx.x;
    const int m0 = (u % n_mt) * kTcM, n0 = ((u / n_mt) % n_nt) * NT;
    const int q0 = (u / (n_mt * n_nt)) * per;
    const int M = a.ks * a.ks * a.cin;
    const int nk = min(per, tiles_x * tiles_y * a.B - q0);  // >= 1 by the host's split
    const int ra = min(RA, (M - m0) / CA);                   // regions holding rows < M
    const int half = a.ks / 2;
    if (warp == 5) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(&tmem_sh)),
                     "r"(TCOLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (threadIdx.x == 0) {
        for (int s = 0; s < S; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        mbar_init(&done, 1);
        fence_mbar_init();
    }
    if (warp == 4 && lane == 0) {
        asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&tmx)) : "memory");
        asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&tmz)) : "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_sh;

    if (warp == 4) {
        if (lane == 0) {  // TMA producer
            bool ok = true;
            for (int k = 0; k < nk; ++k) {
                const int s = k % S;
                const unsigned su = (unsigned)(k / S);
                if (k >= S && !mbar_wait_tc(&empty[s], (su - 1) & 1)) ok = false;
                int q = q0 + k;
                const int x0 = (q % tiles_x) * kTileX;
                q /= tiles_x;
                const int y0 = (q % tiles_y) * kTileY, b = q / tiles_y;
                unsigned char *sa = sm + s * STAGE;
                mbar_arrive_expect_tx(&full[s], (unsigned)(ra * REGA + B_BYTES));
                for (int j = 0; j < ra; ++j) {
                    const int m = m0 + j * CA;
                    const int tap = m / a.cin, c = m - tap * a.cin;
                    tma_load_4d(sa + j * REGA, &tmx, c, x0 + tap % a.ks - half,
                                y0 + tap / a.ks - half, b, &full[s]);
                }
                for (int j = 0; j < RB; ++j)
                    tma_load_4d(sa + A_BYTES + j * REGB, &tmz, n0 + j * CB, x0, y0, b, &full[s]);
            }
            if (!ok && err) atomicOr(err, DEV_ERR_TIMEOUT);
        }
        __syncwarp();
    } else if (warp == 5) {
        if (lane == 0) {  // MMA issuer
            bool ok = true;
            for (int k = 0; k < nk; ++k) {
                const int s = k % S;
                if (!mbar_wait_tc(&full[s], (unsigned)(k / S) & 1)) ok = false;
                tc_fence_after();
                const unsigned sa = smem_u32(sm + s * STAGE);
                const unsigned sb = sa + A_BYTES;
#pragma unroll
                for (int kk = 0; kk < kTcM / 16; ++kk) {  // 16 pixel rows per MMA
                    const uint64_t da = umma_desc(sa + kk * 2 * SBOA, REGA, SBOA, sw_layout(CA));
                    const uint64_t db = umma_desc(sb + kk * 2 * SBOB, REGB, SBOB, sw_layout(CB));
                    const uint32_t acc = (k > 0 || kk > 0) ? 1u : 0u;
                    asm volatile(
                        "{\n\t.reg .pred p;\n\t"
                        "setp.ne.b32 p, %4, 0;\n\t"
                        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(
                            tmem),
                        "l"(da), "l"(db), "r"(IDESC), "r"(acc)
                        : "memory");
                }
                asm volatile(
                    "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 "
                    "[%0];" ::"r"(smem_u32(&empty[s]))
                    : "memory");
            }
            asm volatile(
                "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                    smem_u32(&done))
                : "memory");
            if (!ok && err) atomicOr(err, DEV_ERR_TIMEOUT);
        }
        __syncwarp();
    } else {  // epilogue: accumulator row r = GEMM row m0 + r
        if (!mbar_wait_tc(&done, 0)) {
            if (err && lane == 0) atomicOr(err, DEV_ERR_TIMEOUT);
            mbar_wait_tc(&done, 0);  // once more, bounded
        }
        tc_fence_after();
        const int m = m0 + warp * 32 + lane;
#pragma unroll 1
        for (int c0 = 0; c0 < NT; c0 += 16) {
            uint32_t v[16];
            __syncwarp();
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,"
                "%12,%13,%14,%15}, [%16];"
                : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]),
                  "=r"(v[6]), "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]),
                  "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
                : "r"(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (m < M) {
#pragma unroll
                for (int j = 0; j < 16; ++j)
                    atomicAdd(&a.dw[(size_t)(n0 + c0 + j) * M + m], __uint_as_float(v[j]));
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 5)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                     "r"(TCOLS)
                     : "memory");
}

// Tensor map of a BF16 NHWC tensor's channel slice [0, C) (channel stride ld
// elements) with boxes of {bc channels, bx, by, 1}, swizzle span bc * 2 bytes.
cudaError_t encode_nhwc(CUtensorMap *tm, const bf16 *base, int C, int ld, int W, int H, int B,
                        int bc, CUtensorMapL2promotion l2, int bx = kTileX, int by = kTileY) {
    const auto enc = tmap_encoder();
    if (!enc) return cudaErrorNotSupported;
    const cuuint64_t d[4] = {(cuuint64_t)C, (cuuint64_t)W, (cuuint64_t)H, (cuuint64_t)B};
    const cuuint64_t s[3] = {(cuuint64_t)ld * 2, (cuuint64_t)ld * 2 * W,
                             (cuuint64_t)ld * 2 * W * H};
    const cuuint32_t box[4] = {(cuuint32_t)bc, (cuuint32_t)bx, (cuuint32_t)by, 1};
    const cuuint32_t one[4] = {1, 1, 1, 1};
    const CUtensorMapSwizzle swz = bc == 64   ? CU_TENSOR_MAP_SWIZZLE_128B
                                   : bc == 32 ? CU_TENSOR_MAP_SWIZZLE_64B
                                              : CU_TENSOR_MAP_SWIZZLE_32B;
    if (enc(tm, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, (void *)base, d, s, box, one,
            CU_TENSOR_MAP_INTERLEAVE_NONE, swz, l2, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) !=
        CUDA_SUCCESS)
        return cudaErrorInvalidValue;
    return cudaSuccess;
}

template <int CA, int NT>
cudaError_t launch_wgrad_tc(const WgArgs &a, unsigned *err, cudaStream_t st) {
    constexpr int CB = NT < 64 ? NT : 64;
    constexpr int STAGE = kTcM * kTcM * 2 + NT * kTcM * 2;
    constexpr int SMEM = wg_stages(STAGE) * STAGE + 1024;
    U_TRY(cudaFuncSetAttribute(k_wgrad_tc<CA, NT>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM));
    CUtensorMap tmx, tmz;
    U_TRY(encode_nhwc(&tmx, a.x + a.xoff, a.cin, a.ldx, a.W, a.H, a.B, CA,
                            CU_TENSOR_MAP_L2_PROMOTION_L2_128B));
    U_TRY(encode_nhwc(&tmz, a.dz, a.cout, a.cout, a.W, a.H, a.B, CB,
                            CU_TENSOR_MAP_L2_PROMOTION_L2_128B));
    int dev = 0, sms = 148;
    U_TRY(cudaGetDevice(&dev));
    U_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const int tiles_x = (a.W + kTileX - 1) / kTileX, tiles_y = (a.H + kTileY - 1) / kTileY;
    const long long n_patch = (long long)tiles_x * tiles_y * a.B;
    const int n_mt = (a.ks * a.ks * a.cin + kTcM - 1) / kTcM, n_nt = a.cout / NT;
    if (n_patch > 0x7fffffffLL) return cudaErrorInvalidValue;
    // one full wave of resident blocks (no tail wave); every block gets at
    // least one patch
    int per_sm = 1;
    U_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_wgrad_tc<CA, NT>, kTcThreads,
                                                        SMEM));
    const long long wave = (long long)sms * std::max(per_sm, 1);
    const long long want = std::max(1LL, wave / (n_mt * n_nt));
    const int per = (int)((n_patch + want - 1) / want);
    const int splits = (int)((n_patch + per - 1) / per);
    k_wgrad_tc<CA, NT><<<n_mt * n_nt * splits, kTcThreads, SMEM, st>>>(
        tmx, tmz, a, tiles_x, tiles_y, n_mt, n_nt, per, err);
    return cudaGetLastError();
}

template <int CA>
cudaError_t wgrad_tc_n(const WgArgs &a, unsigned *err, cudaStream_t st) {
    if (a.cout == 16) return launch_wgrad_tc<CA, 16>(a, err, st);
    if (a.cout == 32) return launch_wgrad_tc<CA, 32>(a, err, st);
    if (a.cout == 64) return launch_wgrad_tc<CA, 64>(a, err, st);
    return launch_wgrad_tc<CA, 128>(a, err, st);
}

// The tensor-memory weight gradient (accumulates into a.dw): cin and cout
// multiples of 16, cout 16, 32, 64 or a multiple of 128.
cudaError_t wgrad_tc(const WgArgs &a, unsigned *err, cudaStream_t st) {
    if (a.cin % 16 || a.ldx % 16 || a.xoff % 16 || a.xoff + a.cin > a.ldx ||
        !(a.cout == 16 || a.cout == 32 || a.cout == 64 || a.cout % 128 == 0) ||
        (a.ks != 1 && a.ks != 3) || a.B < 1 || a.H < 1 || a.W < 1)
        return cudaErrorInvalidValue;
    if (a.cin % 64 == 0) return wgrad_tc_n<64>(a, err, st);
    if (a.cin % 32 == 0) return wgrad_tc_n<32>(a, err, st);
    return wgrad_tc_n<16>(a, err, st);
}

// ---------------------------------------------------------------------------
// Strip variant of the 3x3 convolution, for images whose width is a multiple
// of 128 and at most 64 input and 64 output channels (CK = cin, NT = cout):
// the tile is 128 consecutive pixels of one image row.  Per tile the TMA warp
// loads the three halo strips {cin, 130, 1, 1} of rows y-1, y, y+1 (pixels
// x0-1 .. x0+128, zeros outside the image) into one stage, and the MMA warp
// issues the nine taps as MMAs on views of those strips that start 0, 1 or 2
// rows in.  The swizzle is a function of the absolute shared-memory address,
// so a view starting at any row of a strip written by TMA is a valid K-major
// operand (descriptor base offset 0; checked on the hardware for the 128-
// and 64-byte swizzles at every row shift 0 .. 7).  The nine taps' weights
// stay resident in shared memory for the block's lifetime.  Per tile this
// moves 3 x 130 TMA rows instead of 9 x (128 + NT); TMA issue (about one row
// per three clocks per SM) bounds the patch variant on these layers.
// ---------------------------------------------------------------------------
constexpr int kStripW = 128, kStripRows = kStripW + 2;

__host__ __device__ constexpr int strip_region(int ck) {  // one halo strip, 1024-aligned
    return (kStripRows * ck * 2 + 1023) / 1024 * 1024;
}
__host__ __device__ constexpr int strip_wtap(int ck, int nt) {  // one tap's weights
    return (nt * ck * 2 + 1023) / 1024 * 1024;
}
__host__ __device__ constexpr int strip_stages(int ck, int nt) {  // ~200 KB in all
    return (200 * 1024 - 9 * strip_wtap(ck, nt)) / (3 * strip_region(ck)) < 2
               ? 2
               : ((200 * 1024 - 9 * strip_wtap(ck, nt)) / (3 * strip_region(ck)) > 6
                      ? 6
                      : (200 * 1024 - 9 * strip_wtap(ck, nt)) / (3 * strip_region(ck)));
}
__host__ __device__ constexpr int strip_smem(int ck, int nt) {
    return 9 * strip_wtap(ck, nt) + strip_stages(ck, nt) * 3 * strip_region(ck) + 1024;
}

template <int CK, int NT>
__global__ void __launch_bounds__(kTcThreads) k_conv_strip(const __grid_constant__ CUtensorMap tmx,
                                                            const __grid_constant__ CUtensorMap tmw,
                                                            ConvArgs a, int strips_x,
                                                            unsigned *err) {
    constexpr int REG = strip_region(CK);
    constexpr int STAGE = 3 * REG;
    constexpr int WTAP = strip_wtap(CK, NT);
    constexpr int S = strip_stages(CK, NT);
    constexpr int ACOLS = NT < 32 ? 32 : NT;
    constexpr int TCOLS = 2 * ACOLS;
    constexpr uint32_t IDESC = umma_idesc_bf16(kTcM, NT);
    constexpr unsigned LAYOUT = sw_layout(CK);
    constexpr unsigned SBO = 8 * CK * 2;
    constexpr unsigned ROWB = CK * 2;  // bytes of one pixel row of a strip
    extern __shared__ unsigned char smraw[];
    __shared__ __align__(8) uint64_t full[S], empty[S], acc_full[2], acc_empty[2], wbar;
    __shared__ uint32_t tmem_sh;
    unsigned char *sm = smraw + ((1024u - (smem_u32(smraw) & 1023u)) & 1023u);
    unsigned char *sw = sm;                 // weights [tap][WTAP]
    unsigned char *sst = sm + 9 * WTAP;     // stages [S][dy][REG]
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int n_tiles = strips_x * a.H * a.B;
    auto tile_of = [&](int t) {
        TcTile T;
        T.x0 = (t % strips_x) * kStripW;
        t /= strips_x;
        T.y0 = t % a.H;
        T.b = t / a.H;
        T.n0 = 0;
        return T;
    };
    if (warp == 5) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(&tmem_sh)),
                     "r"(TCOLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (threadIdx.x == 0) {
        for (int s = 0; s < S; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        for (int i = 0; i < 2; ++i) {
            mbar_init(&acc_full[i], 1);
            mbar_init(&acc_empty[i], 4);
        }
        mbar_init(&wbar, 1);
        fence_mbar_init();
    }
    if (warp == 4 && lane == 0) {
        asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&tmx)) : "memory");
        asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&tmw)) : "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_sh;

    if (warp == 4) {
        if (lane == 0) {  // TMA producer: the weights once, then three strips per tile
            bool ok = true;
            mbar_arrive_expect_tx(&wbar, 9u * NT * CK * 2);
            for (int tap = 0; tap < 9; ++tap)
                tma_load_2d(sw + tap * WTAP, &tmw, tap * a.cin, 0, &wbar);
            int g = 0;
            for (int t = blockIdx.x; t < n_tiles; t += gridDim.x, ++g) {
                const TcTile T = tile_of(t);
                const int s = g % S;
                const unsigned u = (unsigned)(g / S);
                if (g >= S && !mbar_wait_tc(&empty[s], (u - 1) & 1)) ok = false;
                unsigned char *st = sst + s * STAGE;
                mbar_arrive_expect_tx(&full[s], 3u * kStripRows * CK * 2);
                for (int d = 0; d < 3; ++d)
                    tma_load_4d(st + d * REG, &tmx, 0, T.x0 - 1, T.y0 + d - 1, T.b, &full[s]);
            }
            if (!ok && err) atomicOr(err, DEV_ERR_TIMEOUT);
        }
        __syncwarp();
    } else if (warp == 5) {
        if (lane == 0) {  // MMA issuer: nine taps per tile
            bool ok = mbar_wait_tc(&wbar, 0);
            int it = 0;
            for (int t = blockIdx.x; t < n_tiles; t += gridDim.x, ++it) {
                const int ab = it & 1;
                const unsigned au = (unsigned)(it >> 1);
                if (it >= 2 && !mbar_wait_tc(&acc_empty[ab], (au - 1) & 1)) ok = false;
                const int s = it % S;
                if (!mbar_wait_tc(&full[s], (unsigned)(it / S) & 1)) ok = false;
                tc_fence_after();
                const uint32_t dacc = tmem + (uint32_t)(ab * ACOLS);
                const unsigned st = smem_u32(sst + s * STAGE);
                const unsigned sb = smem_u32(sw);
#pragma unroll
                for (int tap = 0; tap < 9; ++tap) {
                    // output pixel i reads strip (tap / 3) at row i + tap % 3
                    const unsigned av = st + (tap / 3) * REG + (tap % 3) * ROWB;
                    const unsigned bv = sb + tap * WTAP;
#pragma unroll
                    for (int kk = 0; kk < CK / 16; ++kk) {
                        const uint64_t da = umma_desc_sw(av + kk * 32, SBO, LAYOUT);
                        const uint64_t db = umma_desc_sw(bv + kk * 32, SBO, LAYOUT);
                        const uint32_t acc = (tap > 0 || kk > 0) ? 1u : 0u;
                        asm volatile(
                            "{\n\t.reg .pred p;\n\t"
                            "setp.ne.b32 p, %4, 0;\n\t"
                            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(
                                dacc),
                            "l"(da), "l"(db), "r"(IDESC), "r"(acc)
                            : "memory");
                    }
                }
                asm volatile(
                    "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 "
                    "[%0];" ::"r"(smem_u32(&empty[s]))
                    : "memory");
                asm volatile(
                    "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 "
                    "[%0];" ::"r"(smem_u32(&acc_full[ab]))
                    : "memory");
            }
            if (!ok && err) atomicOr(err, DEV_ERR_TIMEOUT);
        }
        __syncwarp();
    } else {  // epilogue
        int it = 0;
        for (int t = blockIdx.x; t < n_tiles; t += gridDim.x, ++it) {
            const TcTile T = tile_of(t);
            const int ab = it & 1;
            const unsigned au = (unsigned)(it >> 1);
            if (!mbar_wait_tc(&acc_full[ab], au & 1)) {
                if (err && lane == 0) atomicOr(err, DEV_ERR_TIMEOUT);
                mbar_wait_tc(&acc_full[ab], au & 1);  // once more, bounded
            }
            tc_fence_after();
            conv_tc_store<NT, true>(
                a, T, tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(ab * ACOLS),
                warp * 32 + lane);
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive_local(&acc_empty[ab]);
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 5)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                     "r"(TCOLS)
                     : "memory");
}

template <int CK, int NT>
cudaError_t launch_conv_strip(const ConvArgs &a, unsigned *err, cudaStream_t st) {
    constexpr int SMEM = strip_smem(CK, NT);
    static_assert(SMEM <= 227 * 1024, "strip stages exceed shared memory");
    U_TRY(cudaFuncSetAttribute(k_conv_strip<CK, NT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               SMEM));
    CUtensorMap tmx, tmw;
    U_TRY(encode_nhwc(&tmx, a.x + a.xoff, a.cin, a.ldx, a.W, a.H, a.B, CK,
                      CU_TENSOR_MAP_L2_PROMOTION_L2_128B, kStripRows, 1));
    const auto enc = tmap_encoder();
    if (!enc) return cudaErrorNotSupported;
    const int K = 9 * a.cin;
    const cuuint64_t wd[2] = {(cuuint64_t)K, (cuuint64_t)a.cout};
    const cuuint64_t ws[1] = {(cuuint64_t)K * 2};
    const cuuint32_t wb[2] = {(cuuint32_t)CK, (cuuint32_t)NT};
    const cuuint32_t one[2] = {1, 1};
    const CUtensorMapSwizzle swz = CK == 64   ? CU_TENSOR_MAP_SWIZZLE_128B
                                   : CK == 32 ? CU_TENSOR_MAP_SWIZZLE_64B
                                              : CU_TENSOR_MAP_SWIZZLE_32B;
    if (enc(&tmw, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, (void *)a.w, wd, ws, wb, one,
            CU_TENSOR_MAP_INTERLEAVE_NONE, swz, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
        return cudaErrorInvalidValue;
    int dev = 0, sms = 148, per_sm = 1;
    U_TRY(cudaGetDevice(&dev));
    U_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    U_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_conv_strip<CK, NT>,
                                                        kTcThreads, SMEM));
    const int strips_x = a.W / kStripW;
    const long long n_tiles = (long long)strips_x * a.H * a.B;
    if (n_tiles > 0x7fffffffLL) return cudaErrorInvalidValue;
    const int grid = (int)std::min<long long>(n_tiles, (long long)sms * std::max(per_sm, 1));
    k_conv_strip<CK, NT><<<grid, kTcThreads, SMEM, st>>>(tmx, tmw, a, strips_x, err);
    return cudaGetLastError();
}

template <int CK>
cudaError_t conv_strip_n(const ConvArgs &a, unsigned *err, cudaStream_t st) {
    if (a.cout == 16) return launch_conv_strip<CK, 16>(a, err, st);
    if (a.cout == 32) return launch_conv_strip<CK, 32>(a, err, st);
    return launch_conv_strip<CK, 64>(a, err, st);
}

bool conv_strip_fits(const ConvArgs &a) {
    return a.ks == 3 && !a.up2 && a.W % kStripW == 0 &&
           (a.cin == 16 || a.cin == 32 || a.cin == 64) &&
           (a.cout == 16 || a.cout == 32 || a.cout == 64);
}

cudaError_t conv_strip(const ConvArgs &a, unsigned *err, cudaStream_t st) {
    if (!conv_args_ok(a) || !conv_strip_fits(a)) return cudaErrorInvalidValue;
    if (a.cin == 64) return conv_strip_n<64>(a, err, st);
    if (a.cin == 32) return conv_strip_n<32>(a, err, st);
    return conv_strip_n<16>(a, err, st);
}

int gridn_u(size_t n) { return (int)std::min<size_t>((n + 255) / 256, 148 * 32); }

constexpr int kLossBlocks = 296;

}  // namespace

UNet::~UNet() { release(); }

void UNet::release() {
    for (void *p : {(void *)master_, (void *)grad_, (void *)m_, (void *)v_, (void *)wb_,
                    (void *)wt_, (void *)dz_, (void *)pidx_, (void *)scratch_, (void *)outg_})
        if (p) cudaFree(p);
    master_ = grad_ = m_ = v_ = outg_ = nullptr;
    scratch_ = nullptr;
    wb_ = wt_ = dz_ = nullptr;
    pidx_ = nullptr;
    for (Act &a : acts_) {
        if (a.v) cudaFree(a.v);
        if (a.g) cudaFree(a.g);
    }
    acts_.clear();
    layers_.clear();
}

// Activation indices.
enum {
    A_X0, A_E1A, A_D1, A_P1, A_E2A, A_D2, A_P2, A_E3A, A_D3, A_P3, A_M1, A_M2, A_T3, A_F3A,
    A_F3B, A_T2, A_F2A, A_F2B, A_T1, A_F1A, A_F1B, A_OUT, A_COUNT
};

cudaError_t UNet::setup(int batch, int H, int W, unsigned long long seed, cudaStream_t st,
                        unsigned *err) {
    release();
    st_ = st;
    err_ = err;
    const char *wm = std::getenv("IMP_UNET_WMMA");
    use_tc_ = !(wm && wm[0] == '1');
    const char *ws = std::getenv("IMP_UNET_STRIP");
    use_strip_ = !(ws && ws[0] == '0');
    B_ = batch;
    H_ = H;
    W_ = W;
    step_ = 0;
    const int cfg[18][4] = {  // cin, cout, ks, relu
        {16, 32, 3, 1},   {32, 32, 3, 1},   {32, 64, 3, 1},   {64, 64, 3, 1},
        {64, 128, 3, 1},  {128, 128, 3, 1}, {128, 256, 3, 1}, {256, 256, 3, 1},
        {256, 128, 1, 0}, {256, 128, 3, 1}, {128, 128, 3, 1}, {128, 64, 1, 0},
        {128, 64, 3, 1},  {64, 64, 3, 1},   {64, 32, 1, 0},   {64, 32, 3, 1},
        {32, 32, 3, 1},   {32, 16, 1, 0}};
    size_t off = 0;
    for (auto &c : cfg) {
        ConvLayer L;
        L.cin = c[0];
        L.cout = c[1];
        L.ks = c[2];
        L.relu = c[3] != 0;
        L.w_off = off;
        off += L.wsize();
        L.b_off = off;
        off += L.cout;
        layers_.push_back(L);
    }
    n_params_ = off;
    // He initialisation (seeded, host); the zero input channels 2..15 of the
    // first layer and the unused outputs 2..15 of the last stay zero.
    std::vector<float> h(n_params_, 0.f);
    std::mt19937_64 rng(seed);
    for (size_t li = 0; li < layers_.size(); ++li) {
        const ConvLayer &L = layers_[li];
        const int cin_eff = li == 0 ? 2 : L.cin;
        const double sd = std::sqrt((L.relu ? 2.0 : 1.0) / (L.ks * L.ks * cin_eff));
        std::normal_distribution<double> nd(0.0, sd);
        const int taps = L.ks * L.ks;
        for (int co = 0; co < L.cout; ++co) {
            if (li + 1 == layers_.size() && co >= 2) continue;
            for (int t = 0; t < taps; ++t)
                for (int ci = 0; ci < cin_eff; ++ci)
                    h[L.w_off + ((size_t)co * taps + t) * L.cin + ci] = (float)nd(rng);
        }
    }
    const size_t pb = n_params_ * sizeof(float);
    U_TRY(cudaMalloc(&master_, pb));
    U_TRY(cudaMalloc(&grad_, pb));
    U_TRY(cudaMalloc(&m_, pb));
    U_TRY(cudaMalloc(&v_, pb));
    U_TRY(cudaMalloc(&wb_, n_params_ * sizeof(bf16)));
    U_TRY(cudaMalloc(&wt_, n_params_ * sizeof(bf16)));
    U_TRY(cudaMemcpy(master_, h.data(), pb, cudaMemcpyHostToDevice));
    U_TRY(cudaMemsetAsync(m_, 0, pb, st));
    U_TRY(cudaMemsetAsync(v_, 0, pb, st));
    // activations
    const int Hs[4] = {H, H / 2, H / 4, H / 8}, Ws[4] = {W, W / 2, W / 4, W / 8};
    const int shape[A_COUNT][2] = {  // level, channels
        {0, 16}, {0, 32}, {0, 64}, {1, 32}, {1, 64}, {1, 128}, {2, 64}, {2, 128},
        {2, 256}, {3, 128}, {3, 256}, {3, 256}, {3, 128}, {2, 128}, {2, 128}, {2, 64},
        {1, 64}, {1, 64}, {1, 32}, {0, 32}, {0, 32}, {0, 16}};
    acts_.resize(A_COUNT);
    size_t max_dz = 0;
    for (int i = 0; i < A_COUNT; ++i) {
        Act &a = acts_[i];
        a.H = Hs[shape[i][0]];
        a.W = Ws[shape[i][0]];
        a.C = shape[i][1];
        const size_t n = (size_t)B_ * a.H * a.W * a.C;
        U_TRY(cudaMalloc(&a.v, n * sizeof(bf16)));
        U_TRY(cudaMalloc(&a.g, n * sizeof(float)));
        max_dz = std::max(max_dz, n);
    }
    U_TRY(cudaMalloc(&dz_, max_dz * sizeof(bf16)));
    size_t pidx = 0;
    const int pool_src[3] = {A_P1, A_P2, A_P3};
    for (int l = 0; l < 3; ++l) {
        const Act &a = acts_[pool_src[l]];
        pidx_off_[l] = pidx;
        pidx += (size_t)B_ * a.H * a.W * a.C;
    }
    U_TRY(cudaMalloc(&pidx_, pidx));
    U_TRY(cudaMalloc(&scratch_, kLossBlocks * sizeof(double)));
    U_TRY(cudaMalloc(&outg_, (size_t)B_ * H_ * W_ * 16 * sizeof(float)));
    return sync_weights();
}

cudaError_t UNet::sync_weights() {
    k_to_bf16<<<gridn_u(n_params_), 256, 0, st_>>>(wb_, master_, n_params_);
    ++launches_;
    for (const ConvLayer &L : layers_) {
        k_wtrans<<<gridn_u(L.wsize()), 256, 0, st_>>>(wt_ + L.w_off, wb_ + L.w_off, L.cin, L.cout,
                                                      L.ks * L.ks);
        ++launches_;
    }
    return cudaGetLastError();
}

cudaError_t UNet::conv_fwd(int li, const Act &in, int in_off, Act &out, int out_off, bool up2) {
    const ConvLayer &L = layers_[li];
    ConvArgs a{};
    a.up2 = up2 ? 1 : 0;
    a.x = in.v;
    a.ldx = in.C;
    a.xoff = in_off;
    a.w = wb_ + L.w_off;
    a.bias = master_ + L.b_off;
    a.B = B_;
    a.H = in.H;
    a.W = in.W;
    a.cin = L.cin;
    a.cout = L.cout;
    a.ks = L.ks;
    a.relu = L.relu ? 1 : 0;
    if (&out == &acts_[A_OUT]) {
        a.yf = out.g;  // the FP32 network output lives in OUT's gradient-sized buffer
        a.ldyf = out.C;
        a.yfoff = 0;
        a.y = nullptr;
    } else {
        a.y = out.v;
        a.ldy = out.C;
        a.yoff = out_off;
    }
    const int P = B_ * in.H * in.W;
    return run_conv(a, P);
}

// Tensor-memory (tcgen05) kernels unless IMP_UNET_WMMA=1 selects the WMMA
// one: the strip variant where it applies (IMP_UNET_STRIP=0 turns it off),
// else the 8 x 16 patch variant.
cudaError_t UNet::run_conv(const ConvArgs &a, int P) {
    ++launches_;
    if (use_tc_) {
        if (use_strip_ && conv_strip_fits(a)) return conv_strip(a, err_, st_);
        return conv_tc(a, P, err_, st_);
    }
    const dim3 grid((P + 63) / 64, (a.cout + 63) / 64);
    if (a.cin % 32 == 0)
        k_conv_fwd<32><<<grid, kCT, 0, st_>>>(a);
    else
        k_conv_fwd<16><<<grid, kCT, 0, st_>>>(a);
    return cudaGetLastError();
}

// Gradients of layer li whose output is out[..][out_off, +cout) with gradient
// out.g: weights, bias, and (when in.g is set and li > 0) the input gradient
// in.g[..][in_off, +cin) += ...
cudaError_t UNet::conv_bwd(int li, Act &in, int in_off, Act &out, int out_off) {
    const ConvLayer &L = layers_[li];
    const int P = B_ * in.H * in.W;
    const bool is_out = &out == &acts_[A_OUT];
    k_dz<<<gridn_u((size_t)P * L.cout / 8), 256, 0, st_>>>(
        dz_, is_out ? outg_ : out.g, out.C, is_out ? 0 : out_off, out.v, out.C,
        out_off, P, L.cout, L.relu ? 1 : 0);
    WgArgs w{};
    w.dz = dz_;
    w.x = in.v;
    w.ldx = in.C;
    w.xoff = in_off;
    w.dw = grad_ + L.w_off;
    w.B = B_;
    w.H = in.H;
    w.W = in.W;
    w.cin = L.cin;
    w.cout = L.cout;
    w.ks = L.ks;
    if (use_tc_) {
        U_TRY(wgrad_tc(w, err_, st_));
    } else {
        const int base = ((L.cout + 63) / 64) * ((L.cin + 63) / 64) * L.ks * L.ks;
        w.splits = std::max(1, std::min((P + 31) / 32, 148 * 8 / base));
        k_wgrad<<<dim3((L.cout + 63) / 64, (L.cin + 63) / 64, L.ks * L.ks * w.splits), kCT, 0,
                   st_>>>(w);
    }
    const int lanes = 256 / (L.cout / 8);  // pixel lanes of a k_bgrad block
    k_bgrad<<<std::min((P + lanes - 1) / lanes, 148 * 4), 256, 0, st_>>>(grad_ + L.b_off, dz_, P,
                                                                         L.cout);
    launches_ += 3;
    if (li > 0 && in.g) {
        ConvArgs a{};
        a.x = dz_;
        a.ldx = L.cout;
        a.xoff = 0;
        a.w = wt_ + L.w_off;
        a.bias = nullptr;
        a.y = nullptr;
        a.yf = in.g;
        a.ldyf = in.C;
        a.yfoff = in_off;
        a.accumulate = 1;
        a.B = B_;
        a.H = in.H;
        a.W = in.W;
        a.cin = L.cout;
        a.cout = L.cin;
        a.ks = L.ks;
        a.relu = 0;
        cudaError_t e = run_conv(a, P);
        if (e != cudaSuccess) return e;
    }
    return cudaGetLastError();
}

cudaError_t UNet::pack_input(const float *x) {
    k_pack<<<gridn_u((size_t)B_ * H_ * W_), 256, 0, st_>>>(acts_[A_X0].v, x, B_, H_ * W_);
    ++launches_;
    return cudaGetLastError();
}

cudaError_t UNet::run_forward() {
    auto &A = acts_;
    auto pool = [&](int src, int lvl, int dst) {
        const Act &s = A[src];
        Act &d = A[dst];
        k_pool_fwd<<<gridn_u((size_t)B_ * d.H * d.W * d.C / 8), 256, 0, st_>>>(
            d.v, pidx_ + pidx_off_[lvl], s.v, s.C, 0, B_, s.H, s.W, d.C);
        ++launches_;
    };
    auto up = [&](int src, int dst, int off) {
        const Act &s = A[src];
        Act &d = A[dst];
        k_up_fwd<<<gridn_u((size_t)B_ * d.H * d.W * s.C / 8), 256, 0, st_>>>(d.v, d.C, off, s.v, B_,
                                                                       d.H, d.W, s.C);
        ++launches_;
    };
    U_TRY(conv_fwd(0, A[A_X0], 0, A[A_E1A], 0));
    U_TRY(conv_fwd(1, A[A_E1A], 0, A[A_D1], 0));
    pool(A_D1, 0, A_P1);
    U_TRY(conv_fwd(2, A[A_P1], 0, A[A_E2A], 0));
    U_TRY(conv_fwd(3, A[A_E2A], 0, A[A_D2], 0));
    pool(A_D2, 1, A_P2);
    U_TRY(conv_fwd(4, A[A_P2], 0, A[A_E3A], 0));
    U_TRY(conv_fwd(5, A[A_E3A], 0, A[A_D3], 0));
    pool(A_D3, 2, A_P3);
    U_TRY(conv_fwd(6, A[A_P3], 0, A[A_M1], 0));
    U_TRY(conv_fwd(7, A[A_M1], 0, A[A_M2], 0));
    // 1x1 conv then nearest x2 up-sampling into the upper channels of the skip
    // buffer: fused into the tensor-memory kernel's epilogue (the backward pass
    // needs only the up-sampled copy; these layers have no ReLU to mask).
    auto conv_up = [&](int li, int src, int t, int dst, int off) -> cudaError_t {
        if (use_tc_) return conv_fwd(li, A[src], 0, A[dst], off, true);
        U_TRY(conv_fwd(li, A[src], 0, A[t], 0));
        up(t, dst, off);
        return cudaSuccess;
    };
    U_TRY(conv_up(8, A_M2, A_T3, A_D3, 128));
    U_TRY(conv_fwd(9, A[A_D3], 0, A[A_F3A], 0));
    U_TRY(conv_fwd(10, A[A_F3A], 0, A[A_F3B], 0));
    U_TRY(conv_up(11, A_F3B, A_T2, A_D2, 64));
    U_TRY(conv_fwd(12, A[A_D2], 0, A[A_F2A], 0));
    U_TRY(conv_fwd(13, A[A_F2A], 0, A[A_F2B], 0));
    U_TRY(conv_up(14, A_F2B, A_T1, A_D1, 32));
    U_TRY(conv_fwd(15, A[A_D1], 0, A[A_F1A], 0));
    U_TRY(conv_fwd(16, A[A_F1A], 0, A[A_F1B], 0));
    U_TRY(conv_fwd(17, A[A_F1B], 0, A[A_OUT], 0));
    return cudaGetLastError();
}

cudaError_t UNet::forward(const float *x, float *y) {
    U_TRY(pack_input(x));
    U_TRY(run_forward());
    k_unpack<<<gridn_u((size_t)B_ * 2 * H_ * W_), 256, 0, st_>>>(y, acts_[A_OUT].g, B_, H_ * W_);
    ++launches_;
    return cudaGetLastError();
}

cudaError_t UNet::train_step(const float *x, const float *target, float lr, float *loss) {
    U_TRY(gradients(x, target, loss));
    ++step_;
    const float b1c = 1.0f - std::pow(0.9f, (float)step_);
    const float b2c = 1.0f - std::pow(0.999f, (float)step_);
    k_adam<<<gridn_u(n_params_), 256, 0, st_>>>(master_, m_, v_, grad_, n_params_, lr, b1c, b2c);
    ++launches_;
    return sync_weights();
}

cudaError_t UNet::gradients(const float *x, const float *target, float *loss) {
    auto &A = acts_;
    U_TRY(pack_input(x));
    U_TRY(run_forward());
    // loss and its gradient (the FP32 output sits in OUT.g; its gradient in out_grad)
    float *og = outg_;
    U_TRY(cudaMemsetAsync(og, 0, (size_t)B_ * H_ * W_ * 16 * sizeof(float), st_));
    k_loss<<<kLossBlocks, 256, 0, st_>>>(og, scratch_, A[A_OUT].g, target, B_, H_ * W_);
    ++launches_;
    for (int i = 0; i < A_COUNT; ++i)
        if (i != A_OUT)
            U_TRY(cudaMemsetAsync(A[i].g, 0, (size_t)B_ * A[i].H * A[i].W * A[i].C * sizeof(float),
                                  st_));
    U_TRY(cudaMemsetAsync(grad_, 0, n_params_ * sizeof(float), st_));
    auto pool_bwd = [&](int dst, int lvl, int src) {  // gradient of pool(dst) -> dst.g
        Act &d = A[dst];
        const Act &s = A[src];
        k_pool_bwd<<<gridn_u((size_t)B_ * s.H * s.W * s.C / 4), 256, 0, st_>>>(
            d.g, d.C, 0, s.g, pidx_ + pidx_off_[lvl], B_, d.H, d.W, s.C);
        ++launches_;
    };
    auto up_bwd = [&](int src, int dst, int off) {  // d(up(src) -> dst[off]) -> src.g
        Act &s = A[src];
        const Act &d = A[dst];
        k_up_bwd<<<gridn_u((size_t)B_ * s.H * s.W * s.C / 4), 256, 0, st_>>>(s.g, d.g, d.C, off, B_,
                                                                        s.H, s.W, s.C);
        ++launches_;
    };
    U_TRY(conv_bwd(17, A[A_F1B], 0, A[A_OUT], 0));
    U_TRY(conv_bwd(16, A[A_F1A], 0, A[A_F1B], 0));
    U_TRY(conv_bwd(15, A[A_D1], 0, A[A_F1A], 0));
    up_bwd(A_T1, A_D1, 32);
    U_TRY(conv_bwd(14, A[A_F2B], 0, A[A_T1], 0));
    U_TRY(conv_bwd(13, A[A_F2A], 0, A[A_F2B], 0));
    U_TRY(conv_bwd(12, A[A_D2], 0, A[A_F2A], 0));
    up_bwd(A_T2, A_D2, 64);
    U_TRY(conv_bwd(11, A[A_F3B], 0, A[A_T2], 0));
    U_TRY(conv_bwd(10, A[A_F3A], 0, A[A_F3B], 0));
    U_TRY(conv_bwd(9, A[A_D3], 0, A[A_F3A], 0));
    up_bwd(A_T3, A_D3, 128);
    U_TRY(conv_bwd(8, A[A_M2], 0, A[A_T3], 0));
    U_TRY(conv_bwd(7, A[A_M1], 0, A[A_M2], 0));
    U_TRY(conv_bwd(6, A[A_P3], 0, A[A_M1], 0));
    pool_bwd(A_D3, 2, A_P3);
    U_TRY(conv_bwd(5, A[A_E3A], 0, A[A_D3], 0));
    U_TRY(conv_bwd(4, A[A_P2], 0, A[A_E3A], 0));
    pool_bwd(A_D2, 1, A_P2);
    U_TRY(conv_bwd(3, A[A_E2A], 0, A[A_D2], 0));
    U_TRY(conv_bwd(2, A[A_P1], 0, A[A_E2A], 0));
    pool_bwd(A_D1, 0, A_P1);
    U_TRY(conv_bwd(1, A[A_E1A], 0, A[A_D1], 0));
    U_TRY(conv_bwd(0, A[A_X0], 0, A[A_E1A], 0));
    if (loss) {
        double part[kLossBlocks];
        U_TRY(cudaMemcpyAsync(part, scratch_, sizeof(part), cudaMemcpyDeviceToHost, st_));
        U_TRY(cudaStreamSynchronize(st_));
        double s = 0.0;
        for (double p : part) s += p;
        *loss = (float)(s / ((double)B_ * 2 * H_ * W_));
    }
    return cudaGetLastError();
}

}  // namespace imp

// ============================================================================
// C-ABI of the learned warm start (no counterpart in the reference)
// ============================================================================
#include "context.h"

struct imp_unet {
    imp_context *ctx = nullptr;
    imp::UNet net;
};

using imp::DevKeep;
using imp::fail;

namespace {

imp_status unet_io(imp_unet *u, const float *x, size_t nx, DevKeep &keep, const float **dx) {
    return imp::to_device(u->ctx, x, nx, keep, dx, nullptr);
}

}  // namespace

extern "C" {

imp_status imp_unet_create(imp_context *ctx, int batch, int height, int width,
                           unsigned long long seed, imp_unet **out) {
    if (!out) return fail(IMP_ERR_INVALID_ARG, "null output pointer");
    *out = nullptr;
    if (batch < 1 || height < 8 || width < 8 || height % 8 || width % 8)
        return fail(IMP_ERR_INVALID_ARG, "batch >= 1 and height, width multiples of 8 required");
    imp_status s = imp::begin(ctx);
    if (s != IMP_OK) return s;
    imp_unet *u = new imp_unet();
    u->ctx = ctx;
    cudaError_t e = u->net.setup(batch, height, width, seed, ctx->stream, ctx->dev_err);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) {
        delete u;
        return imp::from_cuda(e, "unet setup");
    }
    *out = u;
    return IMP_OK;
}

// Frees the network's device memory (cudaFree synchronizes the device); does
// not touch the context, which may already be destroyed.
void imp_unet_destroy(imp_unet *u) { delete u; }

long imp_unet_num_params(const imp_unet *u) { return u ? (long)u->net.n_params() : 0; }

imp_status imp_unet_get_params(imp_unet *u, float *out) {
    if (!u || !out) return fail(IMP_ERR_INVALID_ARG, "null argument");
    imp_status s = imp::begin(u->ctx);
    if (s != IMP_OK) return s;
    IMP_CUDA(cudaMemcpyAsync(out, u->net.params(), u->net.n_params() * sizeof(float),
                             cudaMemcpyDefault, u->ctx->stream),
             "unet params D2H");
    return imp::finish(u->ctx);
}

imp_status imp_unet_set_params(imp_unet *u, const float *in) {
    if (!u || !in) return fail(IMP_ERR_INVALID_ARG, "null argument");
    imp_status s = imp::begin(u->ctx);
    if (s != IMP_OK) return s;
    IMP_CUDA(cudaMemcpyAsync(u->net.params(), in, u->net.n_params() * sizeof(float),
                             cudaMemcpyDefault, u->ctx->stream),
             "unet params H2D");
    IMP_CUDA(u->net.sync_weights(), "unet weights");
    return imp::finish(u->ctx);
}

imp_status imp_unet_forward(imp_unet *u, const float *x, float *y) {
    if (!u || !x || !y) return fail(IMP_ERR_INVALID_ARG, "null argument");
    imp_status s = imp::begin(u->ctx);
    if (s != IMP_OK) return s;
    const size_t n = (size_t)u->net.batch() * 2 * u->net.height() * u->net.width();
    DevKeep keep;
    const float *dx;
    float *dy;
    bool yh;
    if ((s = unet_io(u, x, n, keep, &dx)) || (s = imp::out_device(u->ctx, y, n, keep, &dy, &yh)))
        return s;
    IMP_CUDA(u->net.forward(dx, dy), "unet forward");
    if (yh)
        IMP_CUDA(cudaMemcpyAsync(y, dy, n * sizeof(float), cudaMemcpyDeviceToHost,
                                 u->ctx->stream),
                 "unet output D2H");
    s = imp::finish(u->ctx);
    u->ctx->launches = u->net.launches();
    return s;
}

imp_status imp_unet_gradients(imp_unet *u, const float *x, const float *target, float *grads,
                              float *loss) {
    if (!u || !x || !target || !grads) return fail(IMP_ERR_INVALID_ARG, "null argument");
    imp_status s = imp::begin(u->ctx);
    if (s != IMP_OK) return s;
    const size_t n = (size_t)u->net.batch() * 2 * u->net.height() * u->net.width();
    DevKeep keep;
    const float *dx, *dt;
    if ((s = unet_io(u, x, n, keep, &dx)) || (s = unet_io(u, target, n, keep, &dt))) return s;
    float l = 0.f;
    IMP_CUDA(u->net.gradients(dx, dt, &l), "unet gradients");
    IMP_CUDA(cudaMemcpyAsync(grads, u->net.grads(), u->net.n_params() * sizeof(float),
                             cudaMemcpyDefault, u->ctx->stream),
             "unet gradients D2H");
    if (loss) *loss = l;
    return imp::finish(u->ctx);
}

imp_status imp_unet_train_step(imp_unet *u, const float *x, const float *target, float lr,
                               float *loss) {
    if (!u || !x || !target) return fail(IMP_ERR_INVALID_ARG, "null argument");
    if (!(lr > 0.f)) return fail(IMP_ERR_INVALID_ARG, "learning rate must be > 0");
    imp_status s = imp::begin(u->ctx);
    if (s != IMP_OK) return s;
    const size_t n = (size_t)u->net.batch() * 2 * u->net.height() * u->net.width();
    DevKeep keep;
    const float *dx, *dt;
    if ((s = unet_io(u, x, n, keep, &dx)) || (s = unet_io(u, target, n, keep, &dt))) return s;
    float l = 0.f;
    IMP_CUDA(u->net.train_step(dx, dt, lr, &l), "unet train step");
    if (loss) *loss = l;
    s = imp::finish(u->ctx);
    u->ctx->launches = u->net.launches();
    return s;
}

}  // extern "C"

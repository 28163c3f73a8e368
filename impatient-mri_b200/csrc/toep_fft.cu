// Pruned, fused FFT engine for the Toeplitz F^H F (see toep_fft.cuh).
//
// Line transforms of length n <= 32 run in one register pass; longer ones as
// n = R1 * R2 (R1, R2 <= 32) in two passes over shared memory:
//   pass 1 ("stride"):  for each j1, an R2-point DFT over j2 of x[j1 + R1 j2],
//                       times w_n^{j1 k2}, stored back at j1 + R1 k2;
//   pass 2 ("contig"):  for each k2, an R1-point DFT over the slots
//                       k1 + R1 k2, which then hold X[k2 + R2 k1].
// The inverse runs the two passes in the opposite order (contig with the
// conjugate twiddle after the DFT, then stride) and returns natural order, so
// the forward's permuted "slot" order never has to be undone in memory.
#include "common.cuh"
#include "toep_fft.cuh"

#include <cooperative_groups.h>

#include <algorithm>
#include <type_traits>
#include <cstdlib>
#include <cmath>
#include <vector>

namespace imp {

namespace cg = cooperative_groups;

namespace {

constexpr int kTwN = 2048;      // twiddle table: exp(-2 pi i j / kTwN)
constexpr int kPlaneThreads = 512;

__host__ __device__ constexpr int ilog2c(int n) { return n <= 1 ? 0 : 1 + ilog2c(n >> 1); }

__host__ __device__ constexpr int rev_bits(int i, int bits) {
    int r = 0;
    for (int b = 0; b < bits; ++b) r |= ((i >> b) & 1) << (bits - 1 - b);
    return r;
}

// n = R1 * R2 with R1 = 1 for n <= 32, else R1 = 2^floor(log2(n) / 2).
__host__ __device__ constexpr int split_r1(int n) { return n <= 32 ? 1 : 1 << (ilog2c(n) / 2); }

constexpr int kTwLg = 11;      // log2(kTwN)

// Slot of natural frequency k after a forward transform of length n = r1 r2
// (lr2 = log2 r2).
__device__ __forceinline__ int slot_of(int k, int r1, int lr2) {
    return (k >> lr2) + r1 * (k & ((1 << lr2) - 1));
}

// w_n^e (conjugated when inv), n = 2^lg <= kTwN.
__device__ __forceinline__ float2 wn(const float2 *__restrict__ tw, int e, int lg, bool inv) {
    float2 w = tw[(e & ((1 << lg) - 1)) << (kTwLg - lg)];  // global or shared table
    if (inv) w.y = -w.y;
    return w;
}

__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }

// cos / sin of a compile-time angle (radians, |x| <= 2 pi) by Taylor series,
// evaluated by the compiler; used for the butterfly constants of the register
// DFTs so that they become immediates.
__host__ __device__ constexpr double taylor_sin(double x) {
    double term = x, sum = x;
    for (int k = 1; k < 30; ++k) {
        term *= -x * x / ((2.0 * k) * (2.0 * k + 1.0));
        sum += term;
    }
    return sum;
}
__host__ __device__ constexpr double taylor_cos(double x) {
    double term = 1.0, sum = 1.0;
    for (int k = 1; k < 30; ++k) {
        term *= -x * x / ((2.0 * k - 1.0) * (2.0 * k));
        sum += term;
    }
    return sum;
}

// Butterflies of twiddle index K in the stage of half-width HALF, then the
// rest of the network (radix-2 DIT on bit-reversed registers).
template <int R, int HALF, int K, bool INV>
__device__ __forceinline__ void dit_stage(float2 (&v)[R]) {
    if constexpr (HALF < R) {
        if constexpr (K < HALF) {
            // w = exp(-+ 2 pi i K / (2 HALF))
            constexpr double ang = -3.14159265358979323846264338327950288 * K / HALF;
            constexpr float wc = (float)taylor_cos(ang);
            constexpr float ws = (float)(INV ? -taylor_sin(ang) : taylor_sin(ang));
#pragma unroll
            for (int i = 0; i < R; i += 2 * HALF) {
                const float2 a = v[i + K];
                float2 b = v[i + K + HALF];
                if constexpr (K == 0) {
                } else if constexpr (2 * K == HALF) {  // -i (forward) / +i (inverse)
                    b = INV ? make_float2(-b.y, b.x) : make_float2(b.y, -b.x);
                } else {
                    b = make_float2(b.x * wc - b.y * ws, b.x * ws + b.y * wc);
                }
                v[i + K] = make_float2(a.x + b.x, a.y + b.y);
                v[i + K + HALF] = make_float2(a.x - b.x, a.y - b.y);
            }
            dit_stage<R, HALF, K + 1, INV>(v);
        } else {
            dit_stage<R, 2 * HALF, 0, INV>(v);
        }
    }
}

// In-register DFT of R points, natural order in and out (radix-2 DIT; the
// bit reversal is a compile-time register renaming).
template <int R, bool INV>
__device__ __forceinline__ void dft(float2 (&v)[R], const float2 *__restrict__) {
    constexpr int LG = ilog2c(R);
#pragma unroll
    for (int i = 0; i < R; ++i) {
        const int j = rev_bits(i, LG);
        if (j > i) {
            const float2 t = v[i];
            v[i] = v[j];
            v[j] = t;
        }
    }
    dit_stage<R, 1, 0, INV>(v);
}

// A set of 2^nl_lg lines in shared memory: line l starts at
// (l >> lpb_lg) * bstride + (l & (2^lpb_lg - 1)) * lstride; element e of a
// line is at start + e * es.
// sk = 1: the line is stored skewed, r2 groups of r1 elements each followed by
// one pad element (element x at x + x / r1), so that reading the forward
// transform's permuted slots in natural frequency order (slot stride r1)
// does not put a half-warp on one shared-memory bank.
struct Lines {
    int nl_lg, lpb_lg, lstride, bstride, es;
    int sk = 0;
};

__device__ __forceinline__ int line_base(const Lines &L, int l) {
    return (l >> L.lpb_lg) * L.bstride + (l & ((1 << L.lpb_lg) - 1)) * L.lstride;
}

// Stride pass: R = R2-point DFTs over j2 for every (line, j1); optional
// twiddle w_n^{+-j1 k2} after the DFT.
template <int R, bool INV>
__device__ __forceinline__ void pass_stride(float2 *buf, const Lines L, int r1, int lgn,
                                            bool twiddle, const float2 *__restrict__ tw) {
    const int items = r1 << L.nl_lg;
    for (int it = threadIdx.x; it < items; it += blockDim.x) {
        const int l = it & ((1 << L.nl_lg) - 1), j1 = it >> L.nl_lg;
        float2 *b = buf + line_base(L, l) + j1 * L.es;
        const int st = (r1 + L.sk) * L.es;
        float2 v[R];
#pragma unroll
        for (int q = 0; q < R; ++q) v[q] = b[q * st];
        dft<R, INV>(v, tw);
        if (twiddle && j1 != 0) {
#pragma unroll
            for (int q = 1; q < R; ++q) v[q] = cmul(v[q], wn(tw, j1 * q, lgn, INV));
        }
#pragma unroll
        for (int q = 0; q < R; ++q) b[q * st] = v[q];
    }
}

// Contiguous-slot pass: R = R1-point DFTs over k1 for every (line, k2); the
// inverse multiplies output j1 by w_n^{-j1 k2}.
template <int R, bool INV>
__device__ __forceinline__ void pass_contig(float2 *buf, const Lines L, int r2, int lgn,
                                            const float2 *__restrict__ tw) {
    const int items = r2 << L.nl_lg;
    for (int it = threadIdx.x; it < items; it += blockDim.x) {
        const int l = it & ((1 << L.nl_lg) - 1), k2 = it >> L.nl_lg;
        float2 *b = buf + line_base(L, l) + (R + L.sk) * k2 * L.es;
        float2 v[R];
#pragma unroll
        for (int q = 0; q < R; ++q) v[q] = b[q * L.es];
        dft<R, INV>(v, tw);
        if (INV && k2 != 0) {
#pragma unroll
            for (int q = 1; q < R; ++q) v[q] = cmul(v[q], wn(tw, q * k2, lgn, true));
        }
#pragma unroll
        for (int q = 0; q < R; ++q) b[q * L.es] = v[q];
    }
}

template <bool INV>
__device__ __forceinline__ void run_stride(float2 *buf, const Lines L, int r1, int r2, int lgn,
                                           bool twiddle, const float2 *__restrict__ tw) {
    switch (r2) {
        case 1: break;
        case 2: pass_stride<2, INV>(buf, L, r1, lgn, twiddle, tw); break;
        case 4: pass_stride<4, INV>(buf, L, r1, lgn, twiddle, tw); break;
        case 8: pass_stride<8, INV>(buf, L, r1, lgn, twiddle, tw); break;
        case 16: pass_stride<16, INV>(buf, L, r1, lgn, twiddle, tw); break;
        default: pass_stride<32, INV>(buf, L, r1, lgn, twiddle, tw); break;
    }
}

template <bool INV>
__device__ __forceinline__ void run_contig(float2 *buf, const Lines L, int r1, int r2, int lgn,
                                           const float2 *__restrict__ tw) {
    switch (r1) {
        case 1: break;
        case 2: pass_contig<2, INV>(buf, L, r2, lgn, tw); break;
        case 4: pass_contig<4, INV>(buf, L, r2, lgn, tw); break;
        case 8: pass_contig<8, INV>(buf, L, r2, lgn, tw); break;
        case 16: pass_contig<16, INV>(buf, L, r2, lgn, tw); break;
        default: pass_contig<32, INV>(buf, L, r2, lgn, tw); break;
    }
}

struct PlaneGeo {
    int ns, nm, nf, qm, ps, rs, ncol, C;
    int r1m, r2m, r1f, r2f;
    int lnm, lnf, lplane, lr2m, lr2f, lps;  // log2 of nm, nf, nm*nf, r2m, r2f, ps
    int sk;                                 // rows along f stored skewed (2-D, nf > 32)
};

// The same geometry with the plane sizes as compile-time constants (the slow
// size and the coil count stay runtime): the plane kernels instantiated on it
// fold their per-element index arithmetic into immediates.
template <int NM, int NF, int PS>
struct PlaneGeoC {
    static constexpr int r1m = split_r1(NM), r2m = NM / r1m;
    static constexpr int r1f = split_r1(NF), r2f = NF / r1f;
    static constexpr int sk = (NM == 1 && r1f > 1) ? 1 : 0;
    static constexpr int nm = NM, nf = NF, ps = PS, qm = NM > 1 ? 2 : 1;
    static constexpr int rs = NF + sk * r2f + 1;
    static constexpr int ncol = qm * 2 * NM * NF;
    static constexpr int lnm = ilog2c(NM), lnf = ilog2c(NF), lplane = lnm + lnf;
    static constexpr int lr2m = ilog2c(r2m), lr2f = ilog2c(r2f), lps = ilog2c(PS);
    int ns, C;
};

// The compile-time-geometry kernels keep the twiddle table in shared memory
// (kTwN float2 after their regions); the generic ones read it through the
// read-only global path.

// Shared-memory offset of element x of a row along f (skewed rows: x + x / r1f).
template <class Geo>
__device__ __forceinline__ int fphys(const Geo &g, int x) {
    return g.sk ? x + (x >> (g.lnf - g.lr2f)) : x;
}

// Bounded mbarrier wait (about 2^22 polls); false when it ran out.
__device__ __forceinline__ bool wait_bounded(uint64_t *bar, unsigned parity) {
    for (unsigned it = 0; it < (1u << 22); ++it)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

// Asynchronous global -> shared copies (cp.async: 8 bytes L1-allocating, 16
// bytes L2 only), their commit and the wait for all but the N most recent
// groups of this thread.
__device__ __forceinline__ void cp_async8(float2 *dst, const float2 *src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(smem_u32(dst)), "l"(src)
                 : "memory");
}
__device__ __forceinline__ void cp_async16(float2 *dst, const float2 *src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(smem_u32(dst)), "l"(src)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// Forward plane transform of coil c = blockIdx.y for the s-planes
// [blockIdx.x * ps, +ps) (runtime geometry).  The padded input S_c e_l x is
// formed once in shared memory (U); each (am, af) parity quadrant is then
// twiddled into the work plane P, transformed, and written to
// b1[c][s][am][af][km][kf] in natural frequency order.
template <int VPT, class Geo = PlaneGeo>
__global__ void __launch_bounds__(kPlaneThreads) k_fwd_plane(
    float2 *__restrict__ b1, const float2 *__restrict__ x, const float2 *__restrict__ sens,
    const float2 *__restrict__ eph_l, Geo g, const float2 *__restrict__ tw_g,
    const int *__restrict__ done) {
    extern __shared__ float2 smem[];
    if (done && *done) return;
    const float2 *tw = tw_g;
    const int plane = 1 << g.lplane;
    const int s0 = blockIdx.x * g.ps, c = blockIdx.y;
    const int ecta = g.ps << g.lplane;
    const size_t N = (size_t)g.ns << g.lplane;
    const size_t vbase = (size_t)s0 << g.lplane;
    const int pstride = g.nm * g.rs;
    float2 *P = smem;
    float2 *U = smem + (size_t)g.ps * pstride;
    const Lines rows{g.lps + g.lnm, g.lps + g.lnm, g.rs, 0, 1, g.sk};
    const Lines cols{g.lps + g.lnf, g.lnf, 1, pstride, g.rs};
    const float2 *sc = sens + (size_t)c * N + vbase;
    const float2 *ec = eph_l + vbase;
    const float2 *xc = x + vbase;
#pragma unroll
    for (int i = 0; i < VPT; ++i) {
        const int e = threadIdx.x + i * kPlaneThreads;
        if (e < ecta) U[e] = cmul(cmul(__ldg(&sc[e]), __ldg(&ec[e])), __ldg(&xc[e]));
    }
    for (int am = 0; am < g.qm; ++am)
        for (int af = 0; af < 2; ++af) {
            __syncthreads();
#pragma unroll
            for (int i = 0; i < VPT; ++i) {
                const int e = threadIdx.x + i * kPlaneThreads;
                if (e < ecta) {
                    const int pp = e >> g.lplane, r = e & (plane - 1);
                    const int m = r >> g.lnf, f = r & (g.nf - 1);
                    float2 val = U[e];
                    if (am) val = cmul(val, wn(tw, m, g.lnm + 1, false));
                    if (af) val = cmul(val, wn(tw, f, g.lnf + 1, false));
                    P[pp * pstride + m * g.rs + fphys(g, f)] = val;
                }
            }
            __syncthreads();
            run_stride<false>(P, rows, g.r1f, g.r2f, g.lnf, true, tw);
            __syncthreads();
            if (g.r1f > 1) {
                run_contig<false>(P, rows, g.r1f, g.r2f, g.lnf, tw);
                __syncthreads();
            }
            if (g.nm > 1) {
                run_stride<false>(P, cols, g.r1m, g.r2m, g.lnm, true, tw);
                __syncthreads();
                if (g.r1m > 1) {
                    run_contig<false>(P, cols, g.r1m, g.r2m, g.lnm, tw);
                    __syncthreads();
                }
            }
            float2 *dst = b1 + ((size_t)c * g.ns + s0) * g.ncol + ((size_t)(am * 2 + af) << g.lplane);
#pragma unroll
            for (int i = 0; i < VPT; ++i) {
                const int e = threadIdx.x + i * kPlaneThreads;
                if (e < ecta) {
                    const int pp = e >> g.lplane, r = e & (plane - 1);
                    const int km = r >> g.lnf, kf = r & (g.nf - 1);
                    const int sm = g.nm > 1 ? slot_of(km, g.r1m, g.lr2m) : 0;
                    dst[(size_t)pp * g.ncol + r] =
                        P[pp * pstride + sm * g.rs + fphys(g, slot_of(kf, g.r1f, g.lr2f))];
                }
            }
        }
}

// Forward plane transform on a compile-time geometry, both f-parity quadrants
// of an m-parity at once: the work planes P0 (af = 0) and P1 (af = 1) lie back
// to back and their lines form one set, so each line pass has twice the items
// (the one-pass rows of 32 and the stride pass of the rows of 512 otherwise
// keep only half of the block's threads busy) and half as many barriers.  The
// padded input S_c e_l x is kept in shared memory (U) only when both
// m-parities read it (3-D); 2-D blocks form it on the fly.
template <class Geo>
__global__ void __launch_bounds__(kPlaneThreads) k_fwd_pair(
    float2 *__restrict__ b1, const float2 *__restrict__ x, const float2 *__restrict__ sens,
    const float2 *__restrict__ eph_l, Geo g, const float2 *__restrict__ tw_g,
    const int *__restrict__ done) {
    constexpr int plane = 1 << Geo::lplane, ecta = Geo::ps * plane;
    constexpr int VPT = ecta / kPlaneThreads;
    constexpr int pstride = Geo::nm * Geo::rs, par = Geo::ps * pstride;
    constexpr bool kU = Geo::qm == 2;
    static_assert(ecta % kPlaneThreads == 0, "whole elements per thread");
    extern __shared__ float2 smem[];
    if (done && *done) return;
    float2 *P = smem;                     // [af][ps][nm][rs]
    float2 *U = smem + 2 * par;           // [ps][plane], kU only
    float2 *tw = U + (kU ? ecta : 0);     // twiddle table
    for (int i = threadIdx.x; i < kTwN; i += kPlaneThreads) tw[i] = __ldg(&tw_g[i]);
    const int s0 = blockIdx.x * Geo::ps, c = blockIdx.y;
    const size_t N = (size_t)g.ns << Geo::lplane;
    const size_t vbase = (size_t)s0 << Geo::lplane;
    const Lines rows{Geo::lps + Geo::lnm + 1, Geo::lps + Geo::lnm + 1, Geo::rs, 0, 1, Geo::sk};
    const Lines cols{Geo::lps + Geo::lnf + 1, Geo::lnf, 1, pstride, Geo::rs};
    const float2 *sc = sens + (size_t)c * N + vbase;
    const float2 *ec = eph_l + vbase;
    const float2 *xc = x + vbase;
    if constexpr (kU) {
#pragma unroll
        for (int i = 0; i < VPT; ++i) {
            const int e = threadIdx.x + i * kPlaneThreads;  // read back by this thread only
            U[e] = cmul(cmul(__ldg(&sc[e]), __ldg(&ec[e])), __ldg(&xc[e]));
        }
    }
    // f = e mod nf is the same for all of a thread's elements (nf divides the
    // block size): one f-parity twiddle per thread, read once.
    static_assert(kPlaneThreads % Geo::nf == 0, "f fixed per thread");
    const int fth = threadIdx.x & (Geo::nf - 1);
    float2 wf = make_float2(1.f, 0.f);
    for (int am = 0; am < Geo::qm; ++am) {
        __syncthreads();  // twiddle table loaded / previous outputs read
        if (am == 0) wf = wn(tw, fth, Geo::lnf + 1, false);
#pragma unroll
        for (int i = 0; i < VPT; ++i) {
            const int e = threadIdx.x + i * kPlaneThreads;
            const int pp = e >> Geo::lplane, r = e & (plane - 1);
            const int m = r >> Geo::lnf;
            float2 val;
            if constexpr (kU) val = U[e];
            else val = cmul(cmul(__ldg(&sc[e]), __ldg(&ec[e])), __ldg(&xc[e]));
            if (am) val = cmul(val, wn(tw, m, Geo::lnm + 1, false));
            const int o = pp * pstride + m * Geo::rs + fphys(g, fth);
            P[o] = val;
            P[par + o] = cmul(val, wf);
        }
        __syncthreads();
        run_stride<false>(P, rows, Geo::r1f, Geo::r2f, Geo::lnf, true, tw);
        __syncthreads();
        if constexpr (Geo::r1f > 1) {
            run_contig<false>(P, rows, Geo::r1f, Geo::r2f, Geo::lnf, tw);
            __syncthreads();
        }
        if constexpr (Geo::nm > 1) {
            run_stride<false>(P, cols, Geo::r1m, Geo::r2m, Geo::lnm, true, tw);
            __syncthreads();
            if constexpr (Geo::r1m > 1) {
                run_contig<false>(P, cols, Geo::r1m, Geo::r2m, Geo::lnm, tw);
                __syncthreads();
            }
        }
        float2 *dst = b1 + ((size_t)c * g.ns + s0) * Geo::ncol + ((size_t)(am * 2) << Geo::lplane);
#pragma unroll
        for (int i = 0; i < VPT; ++i) {
            const int e = threadIdx.x + i * kPlaneThreads;
            const int pp = e >> Geo::lplane, r = e & (plane - 1);
            const int km = r >> Geo::lnf, kf = r & (Geo::nf - 1);
            const int sm = Geo::nm > 1 ? slot_of(km, Geo::r1m, Geo::lr2m) : 0;
            const int o = pp * pstride + sm * Geo::rs + fphys(g, slot_of(kf, Geo::r1f, Geo::lr2f));
            float2 *d = dst + (size_t)pp * Geo::ncol + r;
            d[0] = P[o];
            d[plane] = P[par + o];
        }
    }
}

// Inverse plane transform for the s-planes [blockIdx.x * ps, +ps).  The
// blockDim.y-wide cluster (cluster rank = blockIdx.y) splits the coils: block
// r takes coils r, r + csize, ...  Each parity quadrant of b1 is brought into
// the staging buffer St by bulk copies (cp.async.bulk on an mbarrier, the next
// quadrant's copy overlapping this quadrant's transform), scattered into the
// work plane P in slot order, inverse-transformed, twiddled, multiplied by
// conj(S_c) and added to the block's partial sum Y.  The cluster then adds the
// csize partial sums over distributed shared memory (block r reduces its
// 1/csize share of the plane), applies conj(e_l) and writes (first) or
// accumulates q.  A copy that does not complete within the bounded wait sets
// DEV_ERR_TIMEOUT in *err and ends the block's work early.
template <int VPT, class Geo = PlaneGeo>
__global__ void __launch_bounds__(kPlaneThreads) k_inv_plane(
    float2 *__restrict__ q, const float2 *__restrict__ b1, const float2 *__restrict__ sens,
    const float2 *__restrict__ eph_l, Geo g, int first, const float2 *__restrict__ tw_g,
    const int *__restrict__ done, unsigned *err) {
    extern __shared__ __align__(16) float2 smem[];
    __shared__ __align__(8) uint64_t bar;
    cg::cluster_group cluster = cg::this_cluster();
    const int plane = 1 << g.lplane;
    const int ecta = g.ps << g.lplane;
    const int pstride = g.nm * g.rs;
    float2 *St = smem;                                // staging, natural order [ps][plane]
    float2 *Y = smem + ecta;                          // partial coil sum, natural order
    float2 *P = smem + 2 * (size_t)ecta;              // FFT work plane(s), padded rows
    const bool skip = done && *done;
    const int rank = blockIdx.y, csize = gridDim.y;
    const int s0 = blockIdx.x * g.ps;
    const float2 *tw = tw_g;
    if (!skip) {
        const size_t N = (size_t)g.ns << g.lplane;
        const size_t vbase = (size_t)s0 << g.lplane;
        const Lines rows{g.lps + g.lnm, g.lps + g.lnm, g.rs, 0, 1, g.sk};
        const Lines cols{g.lps + g.lnf, g.lnf, 1, pstride, g.rs};
        const int nquad = g.qm * 2;
        const int my_coils = (g.C - rank + csize - 1) / csize;
        const int nq = my_coils * nquad;
        auto src_of = [&](int qi) {
            const int c = rank + (qi / nquad) * csize, quad = qi % nquad;
            return b1 + ((size_t)c * g.ns + s0) * g.ncol + ((size_t)quad << g.lplane);
        };
        auto issue = [&](int qi) {
            const float2 *src = src_of(qi);
            mbar_arrive_expect_tx(&bar, (unsigned)(ecta * sizeof(float2)));
            for (int pp = 0; pp < g.ps; ++pp)
                bulk_g2s(St + (size_t)pp * plane, src + (size_t)pp * g.ncol,
                         (unsigned)(plane * sizeof(float2)), &bar);
        };
        if (threadIdx.x == 0) {
            mbar_init(&bar, 1);
            fence_mbar_init();
        }
        for (int e = threadIdx.x; e < ecta; e += kPlaneThreads) Y[e] = make_float2(0.f, 0.f);
        __syncthreads();
        if (threadIdx.x == 0 && nq > 0) issue(0);
        unsigned phase = 0;
        for (int qi = 0; qi < nq; ++qi) {
            const bool ok = wait_bounded(&bar, phase);
            phase ^= 1u;
            if (__syncthreads_or(!ok)) {
                if (threadIdx.x == 0) {
                    if (err) atomicOr(err, DEV_ERR_TIMEOUT);
                    wait_bounded(&bar, phase ^ 1u);  // the copy still in flight, bounded
                }
                break;
            }
            const int c = rank + (qi / nquad) * csize, quad = qi % nquad;
            const int am = quad >> 1, af = quad & 1;
#pragma unroll
            for (int i = 0; i < VPT; ++i) {
                const int e = threadIdx.x + i * kPlaneThreads;
                if (e < ecta) {
                    const int pp = e >> g.lplane, r = e & (plane - 1);
                    const int km = r >> g.lnf, kf = r & (g.nf - 1);
                    const int sm = g.nm > 1 ? slot_of(km, g.r1m, g.lr2m) : 0;
                    P[pp * pstride + sm * g.rs + fphys(g, slot_of(kf, g.r1f, g.lr2f))] = St[e];
                }
            }
            __syncthreads();
            if (threadIdx.x == 0 && qi + 1 < nq) {
                fence_proxy_async_smem();  // St reads done before the next async write
                issue(qi + 1);
            }
            if (g.nm > 1) {
                if (g.r1m > 1) {
                    run_contig<true>(P, cols, g.r1m, g.r2m, g.lnm, tw);
                    __syncthreads();
                }
                run_stride<true>(P, cols, g.r1m, g.r2m, g.lnm, false, tw);
                __syncthreads();
            }
            if (g.r1f > 1) {
                run_contig<true>(P, rows, g.r1f, g.r2f, g.lnf, tw);
                __syncthreads();
            }
            run_stride<true>(P, rows, g.r1f, g.r2f, g.lnf, false, tw);
            __syncthreads();
            const float2 *sc = sens + (size_t)c * N + vbase;
#pragma unroll
            for (int i = 0; i < VPT; ++i) {
                const int e = threadIdx.x + i * kPlaneThreads;
                if (e < ecta) {
                    const int pp = e >> g.lplane, r = e & (plane - 1);
                    const int m = r >> g.lnf, f = r & (g.nf - 1);
                    float2 val = P[pp * pstride + m * g.rs + fphys(g, f)];
                    if (am) val = cmul(val, wn(tw, m, g.lnm + 1, true));
                    if (af) val = cmul(val, wn(tw, f, g.lnf + 1, true));
                    Y[e] = cadd(Y[e], cmulc(__ldg(&sc[e]), val));
                }
            }
        }
    }
    cluster.sync();
    if (!skip) {
        const size_t vbase = (size_t)s0 << g.lplane;
        const int share = (ecta + csize - 1) / csize;
        const int e0 = rank * share, e1 = min(ecta, e0 + share);
        for (int e = e0 + threadIdx.x; e < e1; e += kPlaneThreads) {
            float2 sum = make_float2(0.f, 0.f);
            for (int r = 0; r < csize; ++r) sum = cadd(sum, cluster.map_shared_rank(Y, r)[e]);
            const size_t v = vbase + e;
            float2 out = cmulc(eph_l[v], sum);
            if (!first) out = cadd(out, q[v]);
            q[v] = out;
        }
    }
    cluster.sync();  // no block leaves while another still reads its Y
}

// Inverse plane transform on a compile-time geometry (same work split and
// result as k_inv_plane).  Each parity quadrant of b1 is copied straight into
// a work plane in slot order by per-thread 8-byte cp.async copies (coalesced:
// a warp reads 32 consecutive spectrum values), two work planes alternating so
// that the next quadrant's copies land while this one is transformed; no
// staging buffer and no scatter pass.  Each thread keeps the partial coil sum
// of its own elements in registers; after the last quadrant the sums go to
// shared memory (over the work planes) for the cluster's coil reduction.
// ONE_COIL (every block has exactly one coil: C <= cluster size): the quadrants
// are summed first and conj(S_c) applied once at the end, one sensitivity read
// per element instead of one per quadrant.
template <class Geo, bool ONE_COIL = false>
__global__ void __launch_bounds__(kPlaneThreads) k_inv_async(
    float2 *__restrict__ q, const float2 *__restrict__ b1, const float2 *__restrict__ sens,
    const float2 *__restrict__ eph_l, Geo g, int first, const float2 *__restrict__ tw_g,
    const int *__restrict__ done) {
    constexpr int plane = 1 << Geo::lplane, ecta = Geo::ps * plane;
    constexpr int VPT = ecta / kPlaneThreads;
    constexpr int pstride = Geo::nm * Geo::rs, buf = Geo::ps * pstride;
    constexpr int nquad = Geo::qm * 2;
    static_assert(ecta % kPlaneThreads == 0 && ecta <= 2 * buf, "plane split / partial sums");
    extern __shared__ __align__(16) float2 smem[];
    cg::cluster_group cluster = cg::this_cluster();
    float2 *tw = smem + 2 * buf;
    float2 *Y = smem;  // partial coil sums, after the last transform
    static_assert(kPlaneThreads % Geo::nf == 0, "f fixed per thread");
    const bool skip = done && *done;
    const int rank = blockIdx.y, csize = gridDim.y;
    const int s0 = blockIdx.x * Geo::ps;
    const size_t N = (size_t)g.ns << Geo::lplane;
    const size_t vbase = (size_t)s0 << Geo::lplane;
    const int fth = threadIdx.x & (Geo::nf - 1);  // f of every element of this thread
    float2 y[VPT];
#pragma unroll
    for (int i = 0; i < VPT; ++i) y[i] = make_float2(0.f, 0.f);
    if (!skip) {
        for (int i = threadIdx.x; i < kTwN; i += kPlaneThreads) tw[i] = __ldg(&tw_g[i]);
        const Lines rows{Geo::lps + Geo::lnm, Geo::lps + Geo::lnm, Geo::rs, 0, 1, Geo::sk};
        const Lines cols{Geo::lps + Geo::lnf, Geo::lnf, 1, pstride, Geo::rs};
        const int my_coils = (g.C - rank + csize - 1) / csize;
        const int nq = my_coils * nquad;
        auto issue = [&](int qi) {
            const int c = rank + (qi / nquad) * csize, quad = qi % nquad;
            const float2 *src = b1 + ((size_t)c * g.ns + s0) * Geo::ncol + ((size_t)quad << Geo::lplane);
            float2 *P = smem + (qi & 1) * buf;
#pragma unroll
            for (int i = 0; i < VPT; ++i) {
                const int e = threadIdx.x + i * kPlaneThreads;
                const int pp = e >> Geo::lplane, r = e & (plane - 1);
                const int km = r >> Geo::lnf, kf = r & (Geo::nf - 1);
                const int sm = Geo::nm > 1 ? slot_of(km, Geo::r1m, Geo::lr2m) : 0;
                cp_async8(P + pp * pstride + sm * Geo::rs + fphys(g, slot_of(kf, Geo::r1f, Geo::lr2f)),
                          src + (size_t)pp * Geo::ncol + r);
            }
            cp_async_commit();
        };
        if (nq > 0) issue(0);
        for (int qi = 0; qi < nq; ++qi) {
            __syncthreads();  // every thread is done with the plane the next copy overwrites
            if (qi + 1 < nq) {
                issue(qi + 1);
                cp_async_wait<1>();
            } else {
                cp_async_wait<0>();
            }
            __syncthreads();  // quadrant qi (and the twiddle table) visible to all threads
            float2 *P = smem + (qi & 1) * buf;
            const int c = rank + (qi / nquad) * csize, quad = qi % nquad;
            const int am = quad >> 1, af = quad & 1;
            if constexpr (Geo::nm > 1) {
                if constexpr (Geo::r1m > 1) {
                    run_contig<true>(P, cols, Geo::r1m, Geo::r2m, Geo::lnm, tw);
                    __syncthreads();
                }
                run_stride<true>(P, cols, Geo::r1m, Geo::r2m, Geo::lnm, false, tw);
                __syncthreads();
            }
            if constexpr (Geo::r1f > 1) {
                run_contig<true>(P, rows, Geo::r1f, Geo::r2f, Geo::lnf, tw);
                __syncthreads();
            }
            run_stride<true>(P, rows, Geo::r1f, Geo::r2f, Geo::lnf, false, tw);
            __syncthreads();
            const float2 *sc = sens + (size_t)c * N + vbase;
            const float2 wf = wn(tw, fth, Geo::lnf + 1, true);
#pragma unroll
            for (int i = 0; i < VPT; ++i) {
                const int e = threadIdx.x + i * kPlaneThreads;
                const int pp = e >> Geo::lplane, r = e & (plane - 1);
                const int m = r >> Geo::lnf;
                float2 val = P[pp * pstride + m * Geo::rs + fphys(g, fth)];
                if (am) val = cmul(val, wn(tw, m, Geo::lnm + 1, true));
                if (af) val = cmul(val, wf);
                if constexpr (ONE_COIL) y[i] = cadd(y[i], val);
                else y[i] = cadd(y[i], cmulc(__ldg(&sc[e]), val));
            }
        }
        if constexpr (ONE_COIL) {
            if (nq > 0) {
                const float2 *sc = sens + (size_t)rank * N + vbase;
#pragma unroll
                for (int i = 0; i < VPT; ++i)
                    y[i] = cmulc(__ldg(&sc[threadIdx.x + i * kPlaneThreads]), y[i]);
            }
        }
        __syncthreads();  // the work planes become the partial-sum array
#pragma unroll
        for (int i = 0; i < VPT; ++i) Y[threadIdx.x + i * kPlaneThreads] = y[i];
    }
    cluster.sync();
    if (!skip) {
        const int share = (ecta + csize - 1) / csize;
        const int e0 = rank * share, e1 = min(ecta, e0 + share);
        for (int e = e0 + threadIdx.x; e < e1; e += kPlaneThreads) {
            float2 sum = make_float2(0.f, 0.f);
            for (int r = 0; r < csize; ++r) sum = cadd(sum, cluster.map_shared_rank(Y, r)[e]);
            const size_t v = vbase + e;
            float2 out = cmulc(eph_l[v], sum);
            if (!first) out = cadd(out, q[v]);
            q[v] = out;
        }
    }
    cluster.sync();  // no block leaves while another still reads its Y
}

template <class Geo>
constexpr size_t inv_async_smem() {  // k_inv_async: two work planes, twiddle table
    return ((size_t)2 * Geo::ps * Geo::nm * Geo::rs + kTwN) * sizeof(float2);
}

// Slow axis for the spectrum columns [blockIdx.x * W, +W) of every coil:
// per s-parity a, forward FFT along s of x[s] w_2ns^{a s}, x Qf_l (parity a),
// inverse FFT, times w_2ns^{-a s}; the two parities are summed and written
// back in place.  Both parities run at once as 2W tile columns (column a W + w
// holds parity a of spectrum column w): blockDim = 2 W R1, and in the stride
// passes thread (a, j1, w) with a the top bit of the thread index, so that a
// warp works on one parity.  The parity factor w_2ns^{a (j1 + R1 q)} splits
// into w_2ns^{a j1}, which commutes with the R2-point DFT and joins the
// inter-pass twiddle (w_2ns^{j1 (2 k2 + a)}), and w_{2 R2}^{a q}, a
// compile-time constant.  Tile element (row, col) is stored at
// row 2W + (col ^ ((row & 1) W)), so that the two rows of a half-warp fall
// on different bank halves.
// TWS: the twiddle table sits in shared memory after the tile (else it is read
// through the read-only global path; the 2-D 512-row instantiation, whose two
// blocks per SM keep more L1 that way, measures faster so).  STAGE (blocks that
// loop over several coils): the block's Qf_l columns are copied into shared
// memory once (cp.async) and read from there by every coil, and the next
// coil's input columns are copied in while the current coil is transformed.
constexpr int kSlowThreads = 256;

// w_{2R}^{q} (conjugated when INV), q < R, as compile-time constants.
template <int R, bool INV>
struct HalfTw {
    float c[R], s[R];
    constexpr HalfTw() : c(), s() {
        for (int q = 0; q < R; ++q) {
            const double ang = -3.14159265358979323846264338327950288 * q / R;
            c[q] = (float)taylor_cos(ang);
            s[q] = (float)(INV ? -taylor_sin(ang) : taylor_sin(ang));
        }
    }
};

template <int NS, int W>
struct SlowStage {  // shared-memory layout of the STAGE kernels (float2 offsets)
    static constexpr int tile = 2 * NS * W;           // E [NS][2W]
    static constexpr int qpar = NS * W + 8;           // Qs parity stride (8: other bank half)
    static constexpr int qs = tile + kTwN;            // Qs [2][NS][W] (+pad)
    static constexpr int xs = qs + 2 * qpar;          // Xs [NS][W]
    static constexpr int total = xs + NS * W;
};

// WC, NCOLC > 0: the block's column count W and the spectrum's column count
// ncol as compile-time constants (the runtime arguments are then ignored).
template <int NS, int WC = 0, int NCOLC = 0, bool STAGE = false, bool TWS = true>
__global__ void __launch_bounds__(kSlowThreads, 2) k_slow(
    float2 *__restrict__ b1, const float2 *__restrict__ qf2, int C, int ncol_rt, int W_rt,
    const float2 *__restrict__ tw_g, const int *__restrict__ done) {
    constexpr int R1 = split_r1(NS), R2 = NS / R1;
    constexpr int LNS = ilog2c(NS);
    static_assert(!STAGE || (WC > 0 && WC % 2 == 0 && NCOLC > 0 && TWS), "staged tiles: 16-byte rows");
    const int W = WC > 0 ? WC : W_rt;
    const int ncol = NCOLC > 0 ? NCOLC : ncol_rt;
    extern __shared__ __align__(16) float2 E[];       // [NS][2W], twiddle table, staging
    if (done && *done) return;
    const float2 *tw = tw_g;
    if constexpr (TWS) {
        float2 *tws = E + 2 * NS * W;
        for (int i = threadIdx.x; i < kTwN; i += blockDim.x) tws[i] = __ldg(&tw_g[i]);
        tw = tws;
    }
    const int col0 = blockIdx.x * W;
    const int lw = WC > 0 ? ilog2c(WC) : __ffs(W) - 1;
    const int W2 = 2 * W, lw2 = lw + 1;
    const int half = W * R1;                  // threads per parity in the stride passes
    const int a = threadIdx.x >= half ? 1 : 0;
    const int rem = threadIdx.x - a * half;
    const int w = rem & (W - 1), j1 = rem >> lw;
    const int cw2 = a * W + w;                // tile column
    auto ei = [&](int row, int col) { return row * W2 + (col ^ ((row & 1) << lw)); };
    const size_t per_coil = (size_t)NS * ncol;
    float2 *Qs = nullptr, *Xs = nullptr;
    if constexpr (STAGE) {
        Qs = E + SlowStage<NS, WC>::qs;
        Xs = E + SlowStage<NS, WC>::xs;
    }
    // STAGE: rows of W float2 as W / 2 16-byte pieces
    auto stage_x = [&](int c) {
        const float2 *src = b1 + (size_t)c * per_coil + col0;
        for (int i = threadIdx.x; i < NS * (W / 2); i += blockDim.x) {
            const int row = i / (W / 2), pc = 2 * (i % (W / 2));
            cp_async16(Xs + row * W + pc, src + (size_t)row * ncol + pc);
        }
        cp_async_commit();
    };
    if constexpr (STAGE) {
        for (int i = threadIdx.x; i < 2 * NS * (W / 2); i += blockDim.x) {
            const int row = i / (W / 2), pc = 2 * (i % (W / 2));
            const int aa = row / NS, k = row % NS;
            cp_async16(Qs + aa * SlowStage<NS, WC>::qpar + k * W + pc,
                       qf2 + (size_t)row * ncol + col0 + pc);
        }
        stage_x(blockIdx.y);  // one group: Qf columns and the first coil's input
    }
    for (int c = blockIdx.y; c < C; c += gridDim.y) {
        float2 *bc = b1 + (size_t)c * per_coil + col0;
        if constexpr (STAGE) cp_async_wait<0>();
        __syncthreads();  // twiddle table / staged tiles visible; previous coil's tile reads done
        {   // stride pass, forward (both parities read the same column)
            float2 v[R2];
#pragma unroll
            for (int q = 0; q < R2; ++q) {
                const int s = j1 + R1 * q;
                if constexpr (STAGE) v[q] = Xs[s * W + w];
                else v[q] = bc[(size_t)s * ncol + w];
            }
            if (a) {
                constexpr HalfTw<R2, false> hw{};
#pragma unroll
                for (int q = 1; q < R2; ++q) v[q] = cmul(v[q], make_float2(hw.c[q], hw.s[q]));
            }
            dft<R2, false>(v, tw);
            if (a) {
#pragma unroll
                for (int q = 0; q < R2; ++q) v[q] = cmul(v[q], wn(tw, j1 * (2 * q + 1), LNS + 1, false));
            } else if (j1 != 0) {
#pragma unroll
                for (int q = 1; q < R2; ++q) v[q] = cmul(v[q], wn(tw, j1 * q, LNS, false));
            }
#pragma unroll
            for (int q = 0; q < R2; ++q) E[ei(j1 + R1 * q, cw2)] = v[q];
        }
        __syncthreads();
        if constexpr (STAGE) {
            if (c + (int)gridDim.y < C) stage_x(c + gridDim.y);  // lands during this coil's work
        }
        // contiguous pass: forward, x Qf_l of the column's parity, inverse
        for (int it = threadIdx.x; it < W2 * R2; it += blockDim.x) {
            const int cw = it & (W2 - 1), k2 = it >> lw2;
            const int aa = cw >> lw, ww = cw & (W - 1);
            float2 z[R1];
#pragma unroll
            for (int k1 = 0; k1 < R1; ++k1) z[k1] = E[ei(k1 + R1 * k2, cw)];
            dft<R1, false>(z, tw);
#pragma unroll
            for (int k1 = 0; k1 < R1; ++k1) {
                const int k = k2 + R2 * k1;
                float2 qv;
                if constexpr (STAGE) qv = Qs[aa * SlowStage<NS, WC>::qpar + k * W + ww];
                else qv = __ldg(&qf2[(size_t)(aa * NS + k) * ncol + col0 + ww]);
                z[k1] = cmul(z[k1], qv);
            }
            dft<R1, true>(z, tw);
            if (k2 != 0 || aa) {  // w_2ns^{-j (2 k2 + aa)}: with the parity's j1 factor
#pragma unroll
                for (int j = 1; j < R1; ++j)
                    z[j] = cmul(z[j], wn(tw, j * (2 * k2 + aa), LNS + 1, true));
            }
#pragma unroll
            for (int j = 0; j < R1; ++j) E[ei(j + R1 * k2, cw)] = z[j];
        }
        __syncthreads();
        {   // stride pass, inverse, the constant part of the parity twiddle
            float2 v[R2];
#pragma unroll
            for (int q = 0; q < R2; ++q) v[q] = E[ei(j1 + R1 * q, cw2)];
            dft<R2, true>(v, tw);
            if (a) {
                constexpr HalfTw<R2, true> hw{};
#pragma unroll
                for (int q = 1; q < R2; ++q) v[q] = cmul(v[q], make_float2(hw.c[q], hw.s[q]));
            }
#pragma unroll
            for (int q = 0; q < R2; ++q) E[ei(j1 + R1 * q, cw2)] = v[q];
        }
        __syncthreads();
        // parity sum, written back in place (W consecutive columns per row)
        for (int it = threadIdx.x; it < NS * W; it += blockDim.x) {
            const int sidx = it >> lw, ww = it & (W - 1);
            bc[(size_t)sidx * ncol + ww] = cadd(E[ei(sidx, ww)], E[ei(sidx, W + ww)]);
        }
    }
}

template <int NS, int WC = 0, int NCOLC = 0, bool STAGE = false, bool TWS = true>
size_t slow_smem(int W) {  // dynamic shared memory of k_slow
    if constexpr (STAGE) return (size_t)SlowStage<NS, WC>::total * sizeof(float2);
    return ((size_t)2 * NS * W + (TWS ? kTwN : 0)) * sizeof(float2);
}

__global__ void k_qf_perm(float2 *__restrict__ qf2, const float2 *__restrict__ qf, int ns, int nm,
                          int nf, int qm, int ncol, float scale) {
    const int nmf = qm == 2 ? 2 * nm : 1;
    const size_t total = (size_t)2 * ns * nmf * 2 * nf;
    for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < total;
         idx += (size_t)gridDim.x * blockDim.x) {
        const int kfn = (int)(idx % (2 * nf));
        const size_t t = idx / (2 * nf);
        const int kmn = (int)(t % nmf);
        const int ksn = (int)(t / nmf);
        const int as = ksn & 1, ks = ksn >> 1, af = kfn & 1, kf = kfn >> 1;
        const int am = qm == 2 ? (kmn & 1) : 0, km = qm == 2 ? (kmn >> 1) : 0;
        const int col = ((am * 2 + af) * nm + km) * nf + kf;
        const float2 v = qf[idx];
        qf2[(size_t)(as * ns + ks) * ncol + col] = make_float2(v.x * scale, v.y * scale);
    }
}

bool pow2(int n) { return n >= 1 && (n & (n - 1)) == 0; }

template <class Geo>
constexpr size_t pair_smem() {  // k_fwd_pair: P0, P1, U (3-D), twiddle table
    return ((size_t)2 * Geo::ps * Geo::nm * Geo::rs + (Geo::qm == 2 ? (size_t)Geo::ps << Geo::lplane : 0) +
            kTwN) * sizeof(float2);
}

template <int VPT, class Geo = PlaneGeo>
cudaError_t set_plane_smem(size_t fwd_bytes, size_t inv_bytes) {
    cudaError_t e;
    if constexpr (std::is_same<Geo, PlaneGeo>::value)
        e = cudaFuncSetAttribute(k_fwd_plane<VPT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)fwd_bytes);
    else
        e = cudaFuncSetAttribute(k_fwd_pair<Geo>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)pair_smem<Geo>());
    if (e != cudaSuccess) return e;
    if constexpr (std::is_same<Geo, PlaneGeo>::value)
        return cudaFuncSetAttribute(k_inv_plane<VPT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)inv_bytes);
    else {
        cudaError_t e2 = cudaFuncSetAttribute(k_inv_async<Geo>,
                                              cudaFuncAttributeMaxDynamicSharedMemorySize,
                                              (int)inv_async_smem<Geo>());
        if (e2 != cudaSuccess) return e2;
        return cudaFuncSetAttribute(k_inv_async<Geo, true>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)inv_async_smem<Geo>());
    }
}

// Plane geometries with compile-time instantiations: 3-D 256 x 256 x 32 images
// (planes of 256 x 32, one per block) and 2-D 512 x 512 images (rows of 512,
// 16 per block).  Others run the generic (runtime-geometry) kernels.
using GeoC3d = PlaneGeoC<256, 32, 1>;
using GeoC2d = PlaneGeoC<1, 512, 16>;
static_assert(pair_smem<GeoC3d>() <= 227 * 1024 && pair_smem<GeoC2d>() <= 227 * 1024 &&
                  inv_async_smem<GeoC3d>() <= 227 * 1024 && inv_async_smem<GeoC2d>() <= 227 * 1024,
              "shared memory of the compile-time-geometry plane kernels");
// IMP_TOEP_GENERIC=1 keeps the generic kernels (the tests compare both).
int spec_kind(const ToepFftPlan &p) {
    const char *gen = std::getenv("IMP_TOEP_GENERIC");
    if (gen && gen[0] == '1') return 0;
    if (p.vpt == 16 && p.nm == 256 && p.nf == 32 && p.ps == 1) return 1;
    if (p.vpt == 16 && p.nm == 1 && p.nf == 512 && p.ps == 16) return 2;
    return 0;
}
template <class G>
G geo_c(const ToepFftPlan &p) {
    G g;
    g.ns = p.ns;
    g.C = p.C;
    return g;
}

template <int NS, int WC = 0, int NCOLC = 0, bool STAGE = false, bool TWS = true>
cudaError_t set_slow_smem(int W) {
    return cudaFuncSetAttribute(k_slow<NS, WC, NCOLC, STAGE, TWS>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)slow_smem<NS, WC, NCOLC, STAGE, TWS>(W));
}

// Slow-axis instantiations with compile-time block and spectrum widths for the
// two specialised geometries (only when the plan's W and ncol are the ones
// compiled in).
int slow_spec(const ToepFftPlan &p) {
    if (p.spec == 1 && p.ns == 256 && p.W == 8 && p.ncol == 32768) return 1;
    if (p.spec == 2 && p.ns == 512 && p.W == 8 && p.ncol == 1024) return 2;
    return 0;
}

PlaneGeo geo_of(const ToepFftPlan &p) {
    PlaneGeo g;
    g.ns = p.ns;
    g.nm = p.nm;
    g.nf = p.nf;
    g.qm = p.qm;
    g.ps = p.ps;
    g.rs = p.rs;
    g.ncol = p.ncol;
    g.C = p.C;
    g.r1m = split_r1(p.nm);
    g.r2m = p.nm / g.r1m;
    g.r1f = split_r1(p.nf);
    g.r2f = p.nf / g.r1f;
    g.lnm = ilog2c(p.nm);
    g.lnf = ilog2c(p.nf);
    g.lplane = g.lnm + g.lnf;
    g.lr2m = ilog2c(g.r2m);
    g.lr2f = ilog2c(g.r2f);
    g.lps = ilog2c(p.ps);
    g.sk = p.sk;
    return g;
}

}  // namespace

bool toep_fft_plan(int ns, int nm, int nf, int C, ToepFftPlan *plan) {
    if (!pow2(ns) || !pow2(nm) || !pow2(nf) || ns < 2 || nf < 2 || ns > 1024 || nf > 1024 ||
        nm > 1024 || (size_t)nm * nf > 16384 || C < 1)
        return false;
    ToepFftPlan p;
    p.ns = ns;
    p.nm = nm;
    p.nf = nf;
    p.qm = nm > 1 ? 2 : 1;
    p.C = C;
    const int plane = nm * nf;
    p.ps = std::max(1, std::min(ns, 8192 / plane));
    p.sk = (nm == 1 && split_r1(nf) > 1) ? 1 : 0;
    p.rs = nf + p.sk * (nf / split_r1(nf)) + 1;
    const int ecta = p.ps * plane;
    p.vpt = std::max(1, ecta / kPlaneThreads);
    p.ncol = p.qm * 2 * plane;
    const int r1 = split_r1(ns);
    p.W = std::max(1, std::min(p.ncol, std::min(4096 / ns, kSlowThreads / (2 * r1))));
    p.smem_plane = (size_t)p.ps * nm * p.rs * sizeof(float2) + (size_t)ecta * sizeof(float2);
    p.smem_inv = p.smem_plane + (size_t)ecta * sizeof(float2);
    p.smem_slow = ((size_t)2 * ns * p.W + kTwN) * sizeof(float2);
    constexpr size_t kMaxSmem = 227 * 1024 - 64;  // room for the static mbarrier
    if (p.smem_inv > kMaxSmem || p.smem_slow > kMaxSmem) return false;
    for (int cs = std::min(C, 8); cs >= 1; --cs)
        if (C % cs == 0) {
            p.csize = cs;
            break;
        }
    cudaError_t e;
    switch (p.vpt) {
        case 1: e = set_plane_smem<1>(p.smem_plane, p.smem_inv); break;
        case 2: e = set_plane_smem<2>(p.smem_plane, p.smem_inv); break;
        case 4: e = set_plane_smem<4>(p.smem_plane, p.smem_inv); break;
        case 8: e = set_plane_smem<8>(p.smem_plane, p.smem_inv); break;
        case 16: e = set_plane_smem<16>(p.smem_plane, p.smem_inv); break;
        case 32: e = set_plane_smem<32>(p.smem_plane, p.smem_inv); break;
        default: return false;
    }
    if (e != cudaSuccess) return false;
    p.spec = spec_kind(p);
    if (p.spec == 1) e = set_plane_smem<16, GeoC3d>(0, 0);
    if (p.spec == 2) e = set_plane_smem<16, GeoC2d>(0, 0);
    if (e != cudaSuccess) return false;
    switch (ns) {
        case 2: e = set_slow_smem<2>(p.W); break;
        case 4: e = set_slow_smem<4>(p.W); break;
        case 8: e = set_slow_smem<8>(p.W); break;
        case 16: e = set_slow_smem<16>(p.W); break;
        case 32: e = set_slow_smem<32>(p.W); break;
        case 64: e = set_slow_smem<64>(p.W); break;
        case 128: e = set_slow_smem<128>(p.W); break;
        case 256: e = set_slow_smem<256>(p.W); break;
        case 512: e = set_slow_smem<512>(p.W); break;
        default: e = set_slow_smem<1024>(p.W); break;
    }
    if (e != cudaSuccess) return false;
    if (slow_spec(p) == 1) {
        e = set_slow_smem<256, 8, 32768>(p.W);
        if (e == cudaSuccess) e = set_slow_smem<256, 8, 32768, true>(p.W);
    }
    if (slow_spec(p) == 2) e = set_slow_smem<512, 8, 1024, false, false>(p.W);
    if (e != cudaSuccess) return false;
    *plan = p;
    return true;
}

cudaError_t toep_fft_twiddles(float2 **tw) {
    std::vector<float2> h(kTwN);
    for (int j = 0; j < kTwN; ++j) {
        const double a = -2.0 * 3.14159265358979323846264338327950288 * j / kTwN;
        h[j] = make_float2((float)std::cos(a), (float)std::sin(a));
    }
    cudaError_t e = cudaMalloc(tw, sizeof(float2) * kTwN);
    if (e != cudaSuccess) return e;
    return cudaMemcpy(*tw, h.data(), sizeof(float2) * kTwN, cudaMemcpyHostToDevice);
}

cudaError_t toep_fft_qf(const ToepFftPlan &p, float2 *qf2_l, const float2 *qf_l, float scale,
                        cudaStream_t st) {
    const size_t total = (size_t)2 * p.ns * p.ncol;
    const int blocks = (int)std::min<size_t>((total + 255) / 256, 148 * 16);
    k_qf_perm<<<blocks, 256, 0, st>>>(qf2_l, qf_l, p.ns, p.nm, p.nf, p.qm, p.ncol, scale);
    return cudaGetLastError();
}

cudaError_t toep_fft_apply_l(const ToepFftPlan &p, float2 *q, const float2 *x,
                             const float2 *sens, const float2 *eph_l, float2 *b1,
                             const float2 *qf2_l, int first, const int *done, const float2 *tw,
                             unsigned *err, cudaStream_t st) {
    const PlaneGeo g = geo_of(p);
    const dim3 ga(p.ns / p.ps, p.C);
    const int spec = p.spec;
#define IMP_PLANE_CASE(V)                                                                   \
    case V:                                                                                 \
        k_fwd_plane<V><<<ga, kPlaneThreads, p.smem_plane, st>>>(b1, x, sens, eph_l, g, tw,  \
                                                                done);                      \
        break;
    if (spec == 1) {
        k_fwd_pair<GeoC3d><<<ga, kPlaneThreads, pair_smem<GeoC3d>(), st>>>(
            b1, x, sens, eph_l, geo_c<GeoC3d>(p), tw, done);
    } else if (spec == 2) {
        k_fwd_pair<GeoC2d><<<ga, kPlaneThreads, pair_smem<GeoC2d>(), st>>>(
            b1, x, sens, eph_l, geo_c<GeoC2d>(p), tw, done);
    } else {
        switch (p.vpt) {
            IMP_PLANE_CASE(1)
            IMP_PLANE_CASE(2)
            IMP_PLANE_CASE(4)
            IMP_PLANE_CASE(8)
            IMP_PLANE_CASE(16)
            IMP_PLANE_CASE(32)
            default: return cudaErrorInvalidValue;
        }
    }
#undef IMP_PLANE_CASE
    const int r1 = split_r1(p.ns);
    const int cols = p.ncol / p.W;
    // Coils: one block row each when Qf_l of the segment (read by every coil)
    // stays in L2 anyway (2-D 512x512: 8 MB), which fills the SMs with blocks;
    // otherwise (3-D 256x256x32: 134 MB) each block loops over its coils so that
    // Qf_l is read from DRAM once and reused from cache by the later coils.
    const size_t qf_bytes = (size_t)2 * p.ns * p.ncol * sizeof(float2);
    const int rows_y = qf_bytes <= (size_t(64) << 20)
                           ? p.C
                           : std::max(1, std::min(p.C, (2 * 148 + cols - 1) / cols));
    const dim3 blocks(cols, rows_y);
    const int threads = 2 * p.W * r1;
#define IMP_SLOW_CASE(NSV)                                                                 \
    case NSV:                                                                              \
        k_slow<NSV><<<blocks, threads, p.smem_slow, st>>>(b1, qf2_l, p.C, p.ncol, p.W, tw, \
                                                          done);                           \
        break;
    const int sspec = slow_spec(p);
    if (sspec == 1 && rows_y < p.C)
        k_slow<256, 8, 32768, true><<<blocks, threads, slow_smem<256, 8, 32768, true>(p.W), st>>>(
            b1, qf2_l, p.C, p.ncol, p.W, tw, done);
    else if (sspec == 1)
        k_slow<256, 8, 32768><<<blocks, threads, p.smem_slow, st>>>(b1, qf2_l, p.C, p.ncol, p.W,
                                                                   tw, done);
    else if (sspec == 2)
        k_slow<512, 8, 1024, false, false>
            <<<blocks, threads, slow_smem<512, 8, 1024, false, false>(p.W), st>>>(
                b1, qf2_l, p.C, p.ncol, p.W, tw, done);
    else switch (p.ns) {
        IMP_SLOW_CASE(2)
        IMP_SLOW_CASE(4)
        IMP_SLOW_CASE(8)
        IMP_SLOW_CASE(16)
        IMP_SLOW_CASE(32)
        IMP_SLOW_CASE(64)
        IMP_SLOW_CASE(128)
        IMP_SLOW_CASE(256)
        IMP_SLOW_CASE(512)
        IMP_SLOW_CASE(1024)
        default: return cudaErrorInvalidValue;
    }
#undef IMP_SLOW_CASE
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(p.ns / p.ps, p.csize);
    cfg.blockDim = dim3(kPlaneThreads);
    cfg.dynamicSmemBytes = spec == 1   ? inv_async_smem<GeoC3d>()
                           : spec == 2 ? inv_async_smem<GeoC2d>()
                                       : p.smem_inv;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = 1;
    attr[0].val.clusterDim.y = p.csize;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaError_t e;
    const bool one_coil = p.C == p.csize;  // cluster rank r takes coil r only
    if (spec == 1 && one_coil)
        e = cudaLaunchKernelEx(&cfg, k_inv_async<GeoC3d, true>, q, b1, sens, eph_l,
                               geo_c<GeoC3d>(p), first, tw, done);
    else if (spec == 1)
        e = cudaLaunchKernelEx(&cfg, k_inv_async<GeoC3d>, q, b1, sens, eph_l, geo_c<GeoC3d>(p),
                               first, tw, done);
    else if (spec == 2 && one_coil)
        e = cudaLaunchKernelEx(&cfg, k_inv_async<GeoC2d, true>, q, b1, sens, eph_l,
                               geo_c<GeoC2d>(p), first, tw, done);
    else if (spec == 2)
        e = cudaLaunchKernelEx(&cfg, k_inv_async<GeoC2d>, q, b1, sens, eph_l, geo_c<GeoC2d>(p),
                               first, tw, done);
    else switch (p.vpt) {
        case 1: e = cudaLaunchKernelEx(&cfg, k_inv_plane<1>, q, b1, sens, eph_l, g, first, tw, done, err); break;
        case 2: e = cudaLaunchKernelEx(&cfg, k_inv_plane<2>, q, b1, sens, eph_l, g, first, tw, done, err); break;
        case 4: e = cudaLaunchKernelEx(&cfg, k_inv_plane<4>, q, b1, sens, eph_l, g, first, tw, done, err); break;
        case 8: e = cudaLaunchKernelEx(&cfg, k_inv_plane<8>, q, b1, sens, eph_l, g, first, tw, done, err); break;
        case 16: e = cudaLaunchKernelEx(&cfg, k_inv_plane<16>, q, b1, sens, eph_l, g, first, tw, done, err); break;
        case 32: e = cudaLaunchKernelEx(&cfg, k_inv_plane<32>, q, b1, sens, eph_l, g, first, tw, done, err); break;
        default: return cudaErrorInvalidValue;
    }
    if (e != cudaSuccess) return e;
    return cudaGetLastError();
}

}  // namespace imp

// NUDFT tile engine on the tensor cores: the per-coil complex multiply-add of
// every (sample, voxel) pair runs as a TF32 tcgen05 MMA whose A operand is
// written by the CUDA cores straight into tensor memory.
//
// Same operator, inputs and partial-sum layout as k_nudft (nudft.cu), which
// replaces ftGpuKernel / iftGpuKernel (kernels/ftGpu.cu:306-604, 756-1013) and
// the coil loop of parallelFtGpu / parallelIftGpu (kernels/parImagingGpu.cu:92-152).
//
// Per CTA: PT accumulator tiles of 128 "ours" rows (tensor-memory lane = row);
// PT = 2 for coil groups of up to 16, 1 for 32 (N = NN columns: 16 up to 4
// coils, else 4 per coil, i.e. 32, 64 or 128).
// For every "theirs" element j the CUDA cores compute the exact fixed-point
// phase and e = (cos, sin) of the angle once per row, split each component
// into a TF32 head and tail (v = hi + lo, hi = v rounded to TF32) and store
//     A[row][4j .. 4j+3] = (cos_hi, sin_hi, cos_lo, sin_lo)
// into tensor memory.  The "theirs" data d_c (per coil) is expanded chunk by
// chunk (16 elements) by the same producer threads into the B operand (shared
// memory, K-major, 128-byte swizzle), with
// rows n of the N = NN accumulator columns
//     n = 2c     (re, head):  ( dx_hi,  dy_hi,  dx_hi,  dy_hi)
//     n = 2c + 1 (im, head):  ( dy_hi, -dx_hi,  dy_hi, -dx_hi)
//     n = H + 2c     (re, tail): ( dx_lo,  dy_lo, 0, 0)
//     n = H + 2c + 1 (im, tail): ( dy_lo, -dx_lo, 0, 0)        (H = NN / 2)
// so that the head columns gather hi*hi + lo*hi and the tail columns hi*lo of
// re = dx cos + dy sin, im = dy cos - dx sin (the k_nudft products); the
// missing lo*lo term is below 2^-22 relative.  Every 64 "theirs" elements
// the accumulator is moved into FP32 registers (double-buffered in tensor
// memory), which bounds the MMA's own accumulation error.
//
// Warp roles (4 H + 2 warps; H = 2):
//   warps 0 .. 4H-1   A producers: warp w writes lanes 32 (w % 4) .. +31 for
//                     the "theirs" share w / 4 (of H) of every chunk and
//                     expands its share of the chunk's B; with PT = 2 group g
//                     drains the accumulators of row tile g, with PT = 1 group
//                     g drains the head and tail columns of coils
//                     [g CG / 2, (g + 1) CG / 2) (the adjoint's coil sum then
//                     completes across the groups in shared memory); all write
//                     the partial sums
//   warp 4H           bulk loads of the "theirs" tiles
//   warp 4H + 1       tensor-memory allocation and the MMA issue (lane 0)
// Every mbarrier wait is bounded; on expiry DEV_ERR_TIMEOUT is raised and the
// kernel runs to its end.
#include "nudft.cuh"
#include "common.cuh"

#include <atomic>

namespace imp {

namespace {

constexpr double kMagicTc = 1572864.0 + 0.5 + 5.9604644775390625e-08;
constexpr float kTwoPiTc = 6.28318530717958647692f;
constexpr float kThreePiTc = 9.42477796076937971538f;

// v rounded to TF32 (nearest, ties away from zero) for finite v: the low 13
// mantissa bits cleared after adding half of their range.
__device__ __forceinline__ uint32_t tf32_rna(float v) {
    return (__float_as_uint(v) + 0x1000u) & 0xFFFFE000u;
}

// Bounded wait: at most 2^20 tries, SLEEP ns apart (the loader and MMA warps
// back off so that their polling takes few issue slots from the producers;
// the producers, about four times slower per chunk than the MMAs, leave the
// MMA warp that much slack).
// After one expiry (ok == false) the thread stops waiting, so a broken
// pipeline ends the launch after one timeout per thread.
template <unsigned SLEEP = 0>
__device__ __forceinline__ void tc_wait(uint64_t *bar, unsigned parity, bool &ok) {
    if (!ok) return;
    for (unsigned it = 0; it < (1u << 20); ++it) {
        if (mbar_try_wait(bar, parity)) return;
        if (SLEEP) __nanosleep(SLEEP);
    }
    ok = false;
}

__device__ __forceinline__ void tc_arrive(uint64_t *bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ void tc_commit(uint64_t *bar) {
    asm volatile(
        "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
            smem_u32(bar))
        : "memory");
}

// K-major, 128-byte swizzle, version 1; sbo = one 8-row group (1024 B).
__device__ __forceinline__ uint64_t tc_bdesc(unsigned saddr) {
    uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)1 << 16;
    d |= (uint64_t)(1024 >> 4) << 32;
    d |= (uint64_t)1 << 46;
    d |= (uint64_t)2 << 61;
    return d;
}

// TF32 x TF32 -> F32, A (tensor memory) and B K-major, M = 128.
__host__ __device__ constexpr uint32_t tc_idesc(int N) {
    return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(N >> 3) << 17) | (8u << 24);
}

__device__ __forceinline__ void tc_st32(uint32_t taddr, const uint32_t *v) {
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x32.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,"
        "%13,%14,%15,%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31,%32};" ::"r"(
            taddr),
        "r"(v[0]), "r"(v[1]), "r"(v[2]), "r"(v[3]), "r"(v[4]), "r"(v[5]), "r"(v[6]), "r"(v[7]),
        "r"(v[8]), "r"(v[9]), "r"(v[10]), "r"(v[11]), "r"(v[12]), "r"(v[13]), "r"(v[14]),
        "r"(v[15]), "r"(v[16]), "r"(v[17]), "r"(v[18]), "r"(v[19]), "r"(v[20]), "r"(v[21]),
        "r"(v[22]), "r"(v[23]), "r"(v[24]), "r"(v[25]), "r"(v[26]), "r"(v[27]), "r"(v[28]),
        "r"(v[29]), "r"(v[30]), "r"(v[31])
        : "memory");
}

__device__ __forceinline__ void tc_ld16(uint32_t taddr, float (&f)[16]) {
    uint32_t v[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,"
        "%14,%15}, [%16];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
          "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]),
          "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) f[i] = __uint_as_float(v[i]);
}

__device__ __forceinline__ void tc_fence_before_sync() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after_sync() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// Compile-time shape of one instantiation.
template <int CG, int PT, int H>
struct TcShape {
    static constexpr int NN = CG <= 4 ? 16 : 4 * CG;  // accumulator columns
    static constexpr int HALF = NN / 2;               // tail columns start here
    static constexpr int CSLOT = HALF / 2;            // coil slots (CG, or 4 when CG < 4)
    static constexpr int KC = 16;                     // "theirs" per chunk
    static constexpr int JPW = KC / H;                // "theirs" per producer warp per chunk
    static constexpr int CHUNKS = kTile / KC;         // chunks per "theirs" tile
    static constexpr int ACOLS = 4 * KC;              // A columns per row tile per chunk
    // A (and B) chunk buffers (three, where tensor memory holds them, measured
    // the same on the 64-slice 384x384 32-coil batch: 98.2 s against 98.5 s)
    static constexpr int NB = 2;
    static constexpr int NBB = NB;                    // B chunk buffers (paired with A's)
    static constexpr int DCOLS = 2 * PT * NN;         // two accumulator sets
    static constexpr int USED = DCOLS + NB * PT * ACOLS;
    static constexpr int TMEM = USED <= 32 ? 32 : USED <= 64 ? 64 : USED <= 128 ? 128
                                : USED <= 256 ? 256 : 512;
    static constexpr int ATOM = NN * 128;             // one 32-K atom of B
    static constexpr int BCHUNK = 2 * ATOM;           // B of one chunk (64 K values)
    static constexpr int WARPS = 4 * H + 2;
    static constexpr int THREADS = 32 * WARPS;
    static constexpr int PROD = 4 * H;
    static constexpr int SCOLS = 4 * JPW;             // A columns per producer store
    // Accumulator drain: with PT == H each producer group g drains row tile g
    // (all NN columns); with PT == 1 and H == 2 group g drains the coils
    // [g CG / 2, (g + 1) CG / 2) of the single row tile (head and tail
    // columns), and the adjoint's coil sum is completed across the groups.
    static constexpr bool CSPLIT = PT == 1;
    static constexpr int DCOL_N = CSPLIT ? CG : NN;   // columns drained per range
    static constexpr int NACC = CSPLIT ? 2 * CG : NN; // accumulators per producer thread
    static_assert(USED <= 512, "tensor memory");
    static_assert(SCOLS == 32, "one 32-column store per row tile and chunk");
    static_assert(PT == H || (PT == 1 && H == 2 && CG >= 16), "drain assignment");
    static_assert(ACOLS == 64, "a chunk spans two 32-K atoms of B");
    static_assert(NN <= 256, "one MMA covers all accumulator columns");
    // "theirs" data rows in shared memory: CG float2 per element, padded by 16
    // bytes from 8 coils up (one bulk copy per element), so that the B expansion's
    // reads of 16 consecutive elements of one coil spread over the banks
    static constexpr bool PADDAT = CG >= 8;
    static constexpr int DROWF = PADDAT ? CG + 2 : CG;  // float2 per row
    // dynamic shared memory: B ring (1024-aligned) | geo[2] | dat[2] | red[128]
    static constexpr size_t SMEM = 1024 + NBB * (size_t)BCHUNK + 2 * kTile * sizeof(double4) +
                                   2 * (size_t)kTile * DROWF * sizeof(float2) +
                                   128 * sizeof(float2);
};

template <int CG, int PT, int H, bool USEZ, bool ADJ, bool BATCH>
__global__ void __launch_bounds__(TcShape<CG, PT, H>::THREADS, 1)
    k_nudft_tc(const double4 *__restrict__ ours, const double4 *__restrict__ theirs,
               const float2 *__restrict__ tdata, const float2 *__restrict__ sens,
               float2 *__restrict__ out, int n_ours_pad, int n_theirs_pad, int per_split,
               unsigned *err, const NuSlice *__restrict__ sl, int n_groups) {
    using S = TcShape<CG, PT, H>;
    extern __shared__ unsigned char smraw[];
    __shared__ __align__(8) uint64_t full[2], tempty[2];
    __shared__ __align__(8) uint64_t afull[S::NB], aempty[S::NB], dfull[2], ddone[2];
    __shared__ uint32_t tmem_sh;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    int g = blockIdx.z;
    if constexpr (BATCH) {
        const int s = blockIdx.z / n_groups;
        g = blockIdx.z - s * n_groups;
        const NuSlice d = sl[s];
        if (blockIdx.x * (128 * PT) >= d.n_ours) return;  // whole block: before any barrier
        ours += d.ours;
        theirs += d.theirs;
        tdata += d.tdata;
        out += d.out;
        n_ours_pad = d.n_ours;
        n_theirs_pad = d.n_theirs;
        per_split = d.per_split;
    }
    const int split = blockIdx.y;
    const int t0 = split * per_split;
    const int ntiles = per_split / kTile;
    const double4 *gsrc = theirs + t0;
    const float2 *dsrc = tdata + ((size_t)g * n_theirs_pad + t0) * CG;
    constexpr unsigned kGeoBytes = kTile * sizeof(double4);
    constexpr unsigned kDatBytes = kTile * CG * sizeof(float2);

    unsigned char *sm = smraw + ((1024u - (smem_u32(smraw) & 1023u)) & 1023u);
    unsigned char *s_b = sm;                                          // [NBB][BCHUNK]
    unsigned char *s_rest = sm + S::NBB * S::BCHUNK;
    double4 *s_geo = reinterpret_cast<double4 *>(s_rest);             // [2][kTile]
    float2 *s_dat = reinterpret_cast<float2 *>(s_rest + 2 * kGeoBytes);  // [2][kTile][DROWF]
    constexpr unsigned kDatSmem = kTile * S::DROWF * sizeof(float2);  // one tile's rows
    float2 *s_red = reinterpret_cast<float2 *>(s_rest + 2 * kGeoBytes + 2 * kDatSmem);  // [128]

    if (warp == S::PROD + 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(&tmem_sh)),
                     "r"(S::TMEM)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (threadIdx.x == 0) {
        for (int i = 0; i < 2; ++i) {
            mbar_init(&full[i], 1);
            mbar_init(&tempty[i], S::PROD);
            mbar_init(&dfull[i], 1);
            mbar_init(&ddone[i], S::PROD);
        }
        for (int i = 0; i < S::NB; ++i) {
            mbar_init(&afull[i], S::PROD);
            mbar_init(&aempty[i], 1);
        }
        fence_mbar_init();
    }
    tc_fence_before_sync();
    __syncthreads();
    tc_fence_after_sync();
    const uint32_t tmem = tmem_sh;
    bool ok = true;

    if (warp < S::PROD) {
        // ------------------------------ A producers ------------------------------
        const int quad = warp & 3, grp = warp >> 2;
        const int row = quad * 32 + lane;
        const int e0 = blockIdx.x * (128 * PT) + row;
        double ox[PT], oy[PT], oz[PT], ow[PT];
#pragma unroll
        for (int p = 0; p < PT; ++p) {
            const double4 q = ours[e0 + p * 128];
            ox[p] = q.x;
            oy[p] = q.y;
            oz[p] = q.z;
            ow[p] = q.w;
        }
        // drained row tile and accumulator column ranges of this producer group
        const int dtile = S::CSPLIT ? 0 : grp;
        const int head0 = S::CSPLIT ? grp * CG : 0;          // first head column
        const int tail0 = S::CSPLIT ? S::HALF + grp * CG : 0;  // first tail column (CSPLIT)
        const bool drains = dtile < PT;
        float acc[S::NACC];
#pragma unroll
        for (int n = 0; n < S::NACC; ++n) acc[n] = 0.f;
        const uint32_t tlane = tmem + ((uint32_t)(quad * 32) << 16);
        // B operand of one chunk from its KC "theirs" data records (all producer
        // threads; items (sample jc, coil slot cc), 16 consecutive threads take
        // the 16 samples of one coil: conflict-free 16-byte stores).  A thread's
        // items and their offsets are the same in every chunk: computed once.
        const int ptid = warp * 32 + lane;
        constexpr int NITEM = S::KC * S::CSLOT;
        constexpr int NIT = (NITEM + S::PROD * 32 - 1) / (S::PROD * 32);
        int it_dat[NIT];       // float2 index of the item's datum in a chunk's rows (-1: none)
        unsigned it_off[NIT][4];  // byte offsets of its four B rows in a chunk buffer
#pragma unroll
        for (int i = 0; i < NIT; ++i) {
            const int it = ptid + i * S::PROD * 32;
            const int jc = it & (S::KC - 1), cc = it / S::KC;
            const unsigned chunk = (unsigned)(jc & 7);
            const unsigned atom = (unsigned)(jc >> 3) * S::ATOM;
            const int rows[4] = {2 * cc, 2 * cc + 1, S::HALF + 2 * cc, S::HALF + 2 * cc + 1};
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                const unsigned n = (unsigned)rows[r];
                it_off[i][r] = atom + (n >> 3) * 1024 + (n & 7) * 128 + ((chunk ^ (n & 7)) << 4);
            }
            it_dat[i] = (it < NITEM && cc < CG) ? jc * S::DROWF + cc : (it < NITEM ? -2 : -1);
        }
        auto expand_b = [&](unsigned char *bt, const float2 *dat) {
#pragma unroll
            for (int i = 0; i < NIT; ++i) {
                if (it_dat[i] == -1) continue;  // no item for this thread
                float xh = 0.f, yh = 0.f, xl = 0.f, yl = 0.f;
                if (it_dat[i] >= 0) {  // -2: a padding coil slot (zero rows)
                    const float2 d = dat[it_dat[i]];
                    xh = __uint_as_float(tf32_rna(d.x));
                    yh = __uint_as_float(tf32_rna(d.y));
                    xl = __uint_as_float(tf32_rna(d.x - xh));  // tail rounded, not truncated
                    yl = __uint_as_float(tf32_rna(d.y - yh));
                }
                *reinterpret_cast<float4 *>(bt + it_off[i][0]) = make_float4(xh, yh, xh, yh);
                *reinterpret_cast<float4 *>(bt + it_off[i][1]) = make_float4(yh, -xh, yh, -xh);
                *reinterpret_cast<float4 *>(bt + it_off[i][2]) = make_float4(xl, yl, 0.f, 0.f);
                *reinterpret_cast<float4 *>(bt + it_off[i][3]) = make_float4(yl, -xl, 0.f, 0.f);
            }
        };
        auto drain = [&](int t) {  // accumulators of tile t into acc
            const int b = t & 1;
            tc_wait<20>(&dfull[b], (unsigned)(t >> 1) & 1, ok);
            tc_fence_after_sync();
            if (drains) {
                const uint32_t dcol = tlane + (uint32_t)((b * PT + dtile) * S::NN);
#pragma unroll
                for (int r = 0; r < (S::CSPLIT ? 2 : 1); ++r)
#pragma unroll
                    for (int n0 = 0; n0 < S::DCOL_N; n0 += 16) {
                        float f[16];
                        tc_ld16(dcol + (uint32_t)((r ? tail0 : head0) + n0), f);
#pragma unroll
                        for (int n = 0; n < 16; ++n) acc[r * S::DCOL_N + n0 + n] += f[n];
                    }
            }
            tc_fence_before_sync();
            __syncwarp();
            if (lane == 0) tc_arrive(&ddone[b]);
        };
        int ci = 0;  // chunk counter
        for (int t = 0; t < ntiles; ++t) {
            const int s = t & 1;
            if (t >= 2) drain(t - 2);
            tc_wait<20>(&full[s], (unsigned)(t >> 1) & 1, ok);
            const double4 *geo = s_geo + s * kTile;
#pragma unroll 1
            for (int c = 0; c < S::CHUNKS; ++c, ++ci) {
                const int ab = ci % S::NB;
                // A buffer ab and B buffer ab are free once chunk ci - NB's MMAs are done
                if (ci >= S::NB) tc_wait<20>(&aempty[ab], (unsigned)(ci / S::NB - 1) & 1, ok);
                tc_fence_after_sync();
                expand_b(s_b + ab * S::BCHUNK, s_dat + (s * kTile + c * S::KC) * S::DROWF);
                uint32_t v[PT][S::SCOLS];
#pragma unroll
                for (int jj = 0; jj < S::JPW; ++jj) {
                    const double4 q = geo[c * S::KC + grp * S::JPW + jj];
#pragma unroll
                    for (int p = 0; p < PT; ++p) {
                        double a = fma(ox[p], q.x, kMagicTc);
                        a = fma(oy[p], q.y, a);
                        if (USEZ) a = fma(oz[p], q.z, a);
                        a = fma(ow[p], q.w, a);
                        const unsigned P = (unsigned)__double2loint(a);
                        const float f1 = __uint_as_float(__funnelshift_r(P, 0x7Fu, 9));
                        const float ang = ADJ ? fmaf(f1, -kTwoPiTc, kThreePiTc)
                                              : fmaf(f1, kTwoPiTc, -kThreePiTc);
                        float sn, cs;
                        __sincosf(ang, &sn, &cs);
                        const uint32_t ch = tf32_rna(cs), sh = tf32_rna(sn);
                        v[p][4 * jj + 0] = ch;
                        v[p][4 * jj + 1] = sh;
                        v[p][4 * jj + 2] = __float_as_uint(cs - __uint_as_float(ch));
                        v[p][4 * jj + 3] = __float_as_uint(sn - __uint_as_float(sh));
                    }
                }
#pragma unroll
                for (int p = 0; p < PT; ++p) {
                    const uint32_t ta =
                        tlane + (uint32_t)(S::DCOLS + (ab * PT + p) * S::ACOLS + grp * S::SCOLS);
                    tc_st32(ta, v[p]);
                }
                asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
                fence_proxy_async_smem();  // this thread's B stores, for the MMA
                tc_fence_before_sync();
                __syncwarp();
                if (lane == 0) tc_arrive(&afull[ab]);
            }
            __syncwarp();
            if (lane == 0) tc_arrive(&tempty[s]);
        }
        for (int t = ntiles >= 2 ? ntiles - 2 : 0; t < ntiles; ++t) drain(t);

        // ------------------------------ partial sums -----------------------------
        const int G = BATCH ? n_groups : (int)gridDim.z;
        const int e = blockIdx.x * (128 * PT) + dtile * 128 + row;
        constexpr int NC = S::CSPLIT ? CG / 2 : CG;  // coils in this thread's accumulators
        const int c0 = S::CSPLIT ? grp * NC : 0;     // first of them
        const int hoff = S::CSPLIT ? S::DCOL_N : S::HALF;  // tail offset inside acc
        if (!ADJ) {
            if (drains) {
                float2 *o = out + ((size_t)(split * G + g) * n_ours_pad + e) * CG + c0;
#pragma unroll
                for (int c = 0; c < NC; ++c)
                    o[c] = make_float2(acc[2 * c] + acc[hoff + 2 * c],
                                       acc[2 * c + 1] + acc[hoff + 2 * c + 1]);
            }
        } else {
            float zr = 0.f, zi = 0.f;
            if (drains) {
                const float2 *sv = sens + ((size_t)g * n_ours_pad + e) * CG + c0;
#pragma unroll
                for (int c = 0; c < NC; ++c) {
                    const float re = acc[2 * c] + acc[hoff + 2 * c];
                    const float im = acc[2 * c + 1] + acc[hoff + 2 * c + 1];
                    const float2 w = sv[c];
                    zr += w.x * re + w.y * im;
                    zi += w.x * im - w.y * re;
                }
            }
            if constexpr (S::CSPLIT) {
                // coil sum across the two producer groups (producer warps only)
                if (grp == 1) s_red[row] = make_float2(zr, zi);
                asm volatile("bar.sync 1, %0;" ::"n"(S::PROD * 32) : "memory");
                if (grp == 0) {
                    const float2 o1 = s_red[row];
                    out[(size_t)(split * G + g) * n_ours_pad + e] =
                        make_float2(zr + o1.x, zi + o1.y);
                }
            } else if (drains) {
                out[(size_t)(split * G + g) * n_ours_pad + e] = make_float2(zr, zi);
            }
        }
    } else if (warp == S::PROD) {
        // ------------------------------ bulk loads ------------------------------
        if (lane == 0)
            for (int t = 0; t < ntiles; ++t) {
                const int s = t & 1;
                if (t >= 2) tc_wait<32>(&tempty[s], (unsigned)((t - 2) >> 1) & 1, ok);
                fence_proxy_async_smem();
                mbar_arrive_expect_tx(&full[s], kGeoBytes + kDatBytes);
                bulk_g2s(s_geo + s * kTile, gsrc + (size_t)t * kTile, kGeoBytes, &full[s]);
                if constexpr (S::PADDAT) {
                    for (int j = 0; j < kTile; ++j)  // CG * 8 bytes: a multiple of 16
                        bulk_g2s(s_dat + (s * kTile + j) * S::DROWF,
                                 dsrc + ((size_t)t * kTile + j) * CG, CG * sizeof(float2),
                                 &full[s]);
                } else {
                    bulk_g2s(s_dat + s * kTile * CG, dsrc + (size_t)t * kTile * CG, kDatBytes,
                             &full[s]);
                }
            }
        __syncwarp();
    } else {
        // ------------------------------- MMA issue -------------------------------
        if (lane == 0) {
            constexpr uint32_t IDESC = tc_idesc(S::NN);
            const unsigned sb0 = smem_u32(s_b);
            int ci = 0;
            for (int t = 0; t < ntiles; ++t) {
                const int s = t & 1;
                if (t >= 2) tc_wait<128>(&ddone[s], (unsigned)((t - 2) >> 1) & 1, ok);
                for (int c = 0; c < S::CHUNKS; ++c, ++ci) {
                    const int ab = ci % S::NB;
                    tc_wait<128>(&afull[ab], (unsigned)(ci / S::NB) & 1, ok);
                    tc_fence_after_sync();
                    // the chunk's B: atoms 0, 1 of buffer ab (S::ACOLS = 64 K values)
                    const uint64_t bd = tc_bdesc(sb0 + ab * S::BCHUNK);
                    const uint32_t dbase = tmem + (uint32_t)(s * PT * S::NN);
                    const uint32_t abase = tmem + (uint32_t)(S::DCOLS + ab * PT * S::ACOLS);
                    const uint32_t first = c > 0 ? 1u : 0u;
#pragma unroll
                    for (int p = 0; p < PT; ++p)
#pragma unroll
                        for (int kk = 0; kk < S::ACOLS / 8; ++kk) {
                            // descriptor start field += byte offset / 16 (no carry: < 256 KB)
                            const uint64_t bdk =
                                bd + (uint64_t)((((kk >> 2) * S::ATOM) + (kk & 3) * 32) >> 4);
                            asm volatile(
                                "{\n\t.reg .pred p;\n\t"
                                "setp.ne.b32 p, %4, 0;\n\t"
                                "tcgen05.mma.cta_group::1.kind::tf32 [%0], [%1], %2, %3, p;\n\t}\n" ::
                                    "r"(dbase + (uint32_t)(p * S::NN)),
                                "r"(abase + (uint32_t)(p * S::ACOLS + kk * 8)), "l"(bdk),
                                "r"(IDESC), "r"(kk > 0 ? 1u : first)
                                : "memory");
                        }
                    tc_commit(&aempty[ab]);
                }
                tc_commit(&dfull[s]);
            }
        }
        __syncwarp();
    }
    if (!ok && err) atomicOr(err, DEV_ERR_TIMEOUT);
    tc_fence_before_sync();
    __syncthreads();
    if (warp == S::PROD + 1)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                     "r"(S::TMEM)
                     : "memory");
}

template <int CG, int PT, int H, bool USEZ, bool ADJ, bool BATCH>
cudaError_t launch_tc(dim3 grid, const double4 *ours, const double4 *theirs, const float2 *tdata,
                      const float2 *sens, float2 *out, int n_ours, int n_theirs, int per_split,
                      unsigned *err, const NuSlice *sl, int G, cudaStream_t st) {
    using S = TcShape<CG, PT, H>;
    auto k = k_nudft_tc<CG, PT, H, USEZ, ADJ, BATCH>;
    // the shared-memory limit is set once per instantiation and device (-mgpu
    // workers drive several devices from several threads)
    static std::atomic<unsigned long long> attr_set{0};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    const unsigned long long bit = dev < 64 ? 1ull << dev : 0ull;
    if (!bit || !(attr_set.load(std::memory_order_acquire) & bit)) {
        e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)S::SMEM);
        if (e != cudaSuccess) return e;
        attr_set.fetch_or(bit, std::memory_order_acq_rel);
    }
    k<<<grid, S::THREADS, S::SMEM, st>>>(ours, theirs, tdata, sens, out, n_ours, n_theirs,
                                         per_split, err, sl, G);
    return cudaGetLastError();
}

template <int CG, bool ADJ, bool BATCH>
cudaError_t launch_tc_z(const NuPlan &p, dim3 grid, const double4 *ours, const double4 *theirs,
                        const float2 *tdata, float2 *out, int n_ours, int n_theirs,
                        int per_split, unsigned *err, const NuSlice *sl, cudaStream_t st) {
    constexpr int PT = CG >= 32 ? 1 : 2, H = 2;
    if (p.use_z)
        return launch_tc<CG, PT, H, true, ADJ, BATCH>(grid, ours, theirs, tdata, p.sens, out,
                                                      n_ours, n_theirs, per_split, err, sl, p.G,
                                                      st);
    return launch_tc<CG, PT, H, false, ADJ, BATCH>(grid, ours, theirs, tdata, p.sens, out,
                                                   n_ours, n_theirs, per_split, err, sl, p.G, st);
}

template <bool ADJ, bool BATCH>
cudaError_t launch_tc_cg(const NuPlan &p, dim3 grid, const double4 *ours, const double4 *theirs,
                         const float2 *tdata, float2 *out, int n_ours, int n_theirs,
                         int per_split, unsigned *err, const NuSlice *sl, cudaStream_t st) {
    switch (p.CG) {
        case 1:
            return launch_tc_z<1, ADJ, BATCH>(p, grid, ours, theirs, tdata, out, n_ours,
                                              n_theirs, per_split, err, sl, st);
        case 2:
            return launch_tc_z<2, ADJ, BATCH>(p, grid, ours, theirs, tdata, out, n_ours,
                                              n_theirs, per_split, err, sl, st);
        case 4:
            return launch_tc_z<4, ADJ, BATCH>(p, grid, ours, theirs, tdata, out, n_ours,
                                              n_theirs, per_split, err, sl, st);
        case 8:
            return launch_tc_z<8, ADJ, BATCH>(p, grid, ours, theirs, tdata, out, n_ours,
                                              n_theirs, per_split, err, sl, st);
        case 16:
            return launch_tc_z<16, ADJ, BATCH>(p, grid, ours, theirs, tdata, out, n_ours,
                                               n_theirs, per_split, err, sl, st);
        case 32:
            return launch_tc_z<32, ADJ, BATCH>(p, grid, ours, theirs, tdata, out, n_ours,
                                               n_theirs, per_split, err, sl, st);
        default:
            return cudaErrorInvalidConfiguration;
    }
}

}  // namespace

bool nu_tc_supported(int CG) {
    return CG == 1 || CG == 2 || CG == 4 || CG == 8 || CG == 16 || CG == 32;
}

int nu_tc_rows(int CG) { return CG >= 32 ? 128 : 256; }

cudaError_t nu_partials_tc(const NuPlan &p, const NuLaunch &l, bool adj, const float2 *tdata,
                           float2 *out, unsigned *err, cudaStream_t st) {
    const int n_ours = adj ? p.Npad : p.Mpad;
    const int n_theirs = adj ? p.Mpad : p.Npad;
    const int rows = nu_tc_rows(p.CG);
    if (!nu_split_ok(n_theirs, l.split) || n_ours % rows) return cudaErrorInvalidConfiguration;
    const dim3 grid(n_ours / rows, l.split, p.G);
    const double4 *ours = adj ? p.vgeo : p.kgeo;
    const double4 *theirs = adj ? p.kgeo : p.vgeo;
    const int per_split = n_theirs / l.split;
    return adj ? launch_tc_cg<true, false>(p, grid, ours, theirs, tdata, out, n_ours, n_theirs,
                                           per_split, err, nullptr, st)
               : launch_tc_cg<false, false>(p, grid, ours, theirs, tdata, out, n_ours, n_theirs,
                                            per_split, err, nullptr, st);
}

cudaError_t nu_partials_tc_batch(const NuPlan &p, const NuLaunch &l, bool adj, int S,
                                 int max_ours, const NuSlice *d_slices, const double4 *ours,
                                 const double4 *theirs, const float2 *tdata, float2 *out,
                                 unsigned *err, cudaStream_t st) {
    const int rows = nu_tc_rows(p.CG);
    if ((long long)S * p.G > 65535 || max_ours % rows) return cudaErrorInvalidConfiguration;
    const dim3 grid(max_ours / rows, l.split, S * p.G);
    return adj ? launch_tc_cg<true, true>(p, grid, ours, theirs, tdata, out, 0, 0, 0, err,
                                          d_slices, st)
               : launch_tc_cg<false, true>(p, grid, ours, theirs, tdata, out, 0, 0, 0, err,
                                           d_slices, st);
}

}  // namespace imp

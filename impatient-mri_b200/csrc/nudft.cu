// NUDFT tile engine: exact-phase brute-force F / F^H with field map and SENSE
// coils sharing one sin/cos per (sample, voxel) pair.
//
// Replaces ftGpuKernel / iftGpuKernel (kernels/ftGpu.cu:306-604, 756-1013),
// the coil loop of parallelFtGpu / parallelIftGpu (kernels/parImagingGpu.cu:92-152)
// and the direct F^H d kernel ComputeFH_GPU_BF (toeplitz/computeFH.cmem.cu:155-200).
//
// Work decomposition ("ours" / "theirs"):
//   F   : ours = samples (one thread holds PT samples in registers),
//         theirs = voxels, streamed through shared memory in tiles of kTile
//   F^H : ours = voxels, theirs = samples
// The phase is the 4-term dot product ours.(x,y,z,w) . theirs.(x,y,z,w) in
// turns, so one kernel template serves both directions.  Tiles of "theirs"
// (geometry + per-coil data) are moved by cp.async.bulk onto an mbarrier,
// double buffered.  The per-coil complex multiply-add of two "ours" rows runs
// as packed FP32x2 FMAs (sm_100 FFMA2), element by element the scalar fmaf
// sequence.  The "theirs" range is split across blockIdx.y; each split
// writes deterministic partial sums that a small kernel adds up.
#include "nudft.cuh"
#include "common.cuh"

#include <algorithm>
#include <cstdlib>

namespace imp {

namespace {

// 1.5*2^20 keeps every accumulated phase in the binade [2^20, 2^21), where the
// double's ulp is 2^-32 turn.  +0.5 turn recentres the angle to [-pi, pi) and
// +2^-24 turn rounds (instead of truncating) to the 23 bits kept in FP32.
constexpr double kMagic = 1572864.0 + 0.5 + 5.9604644775390625e-08;
constexpr float kTwoPiF = 6.28318530717958647692f;
constexpr float kThreePiF = 9.42477796076937971538f;

// BATCH: blockIdx.z = slice * G + coil group; the slice's offsets and padded
// sizes come from sl[slice] (blocks past the slice's "ours" range exit).
template <int CG, int PT, bool USEZ, bool ADJ, int OCC, bool BATCH>
__global__ void __launch_bounds__(kNT, OCC)
    k_nudft(const double4 *__restrict__ ours, const double4 *__restrict__ theirs,
            const float2 *__restrict__ tdata, const float2 *__restrict__ sens,
            float2 *__restrict__ out, int n_ours_pad, int n_theirs_pad, int per_split,
            unsigned *err, const NuSlice *__restrict__ sl, int n_groups) {
    __shared__ __align__(128) double4 s_geo[2][kTile];
    __shared__ __align__(128) float2 s_dat[2][kTile * CG];
    __shared__ __align__(8) uint64_t s_bar[2];

    const int tid = threadIdx.x;
    int g = blockIdx.z;
    if constexpr (BATCH) {
        const int s = blockIdx.z / n_groups;
        g = blockIdx.z - s * n_groups;
        const NuSlice d = sl[s];
        if (blockIdx.x * (kNT * PT) >= d.n_ours) return;  // whole block: before any barrier
        ours += d.ours;
        theirs += d.theirs;
        tdata += d.tdata;
        out += d.out;
        n_ours_pad = d.n_ours;
        n_theirs_pad = d.n_theirs;
        per_split = d.per_split;
    }
    const int split = blockIdx.y;
    const int e0 = blockIdx.x * (kNT * PT) + tid;

    double ox[PT], oy[PT], oz[PT], ow[PT];
#pragma unroll
    for (int j = 0; j < PT; ++j) {
        const double4 q = ours[e0 + j * kNT];
        ox[j] = q.x;
        oy[j] = q.y;
        oz[j] = q.z;
        ow[j] = q.w;
    }

    const int t0 = split * per_split;
    const double4 *gsrc = theirs + t0;
    const float2 *dsrc = tdata + ((size_t)g * n_theirs_pad + t0) * CG;
    const int ntiles = per_split / kTile;
    constexpr unsigned kGeoBytes = kTile * sizeof(double4);
    constexpr unsigned kDatBytes = kTile * CG * sizeof(float2);

    if (tid == 0) {
        mbar_init(&s_bar[0], 1);
        mbar_init(&s_bar[1], 1);
        fence_mbar_init();
    }
    __syncthreads();
    if (tid == 0) {
        mbar_arrive_expect_tx(&s_bar[0], kGeoBytes + kDatBytes);
        bulk_g2s(s_geo[0], gsrc, kGeoBytes, &s_bar[0]);
        bulk_g2s(s_dat[0], dsrc, kDatBytes, &s_bar[0]);
    }

    float ar[PT][CG], ai[PT][CG];
#pragma unroll
    for (int j = 0; j < PT; ++j)
#pragma unroll
        for (int c = 0; c < CG; ++c) ar[j][c] = ai[j][c] = 0.f;

    for (int t = 0; t < ntiles; ++t) {
        const int b = t & 1;
        if (tid == 0 && t + 1 < ntiles) {
            // buffer b^1 was released by the __syncthreads() closing tile t-1
            fence_proxy_async_smem();
            mbar_arrive_expect_tx(&s_bar[b ^ 1], kGeoBytes + kDatBytes);
            bulk_g2s(s_geo[b ^ 1], gsrc + (size_t)(t + 1) * kTile, kGeoBytes, &s_bar[b ^ 1]);
            bulk_g2s(s_dat[b ^ 1], dsrc + (size_t)(t + 1) * kTile * CG, kDatBytes, &s_bar[b ^ 1]);
        }
        mbar_wait_bounded(&s_bar[b], (t >> 1) & 1, err);

        // per-tile partial sums keep the FP32 accumulation error small.  Rows
        // 2m and 2m + 1 share one packed FP32x2 FMA (sm_100 FFMA2: two FMAs per
        // instruction, each rounded as fmaf), so every element is computed
        //     tr = fma(dx, cs, fma(dy, sn, tr)),  ti = fma(dy, cs, fma(dx, -sn, ti))
        // in the order of the scalar form, with half the multiply-add instructions.
        static_assert(PT % 2 == 0, "rows are packed in pairs");
        constexpr int PP = PT / 2;
        float2 tr[PP][CG], ti[PP][CG];
#pragma unroll
        for (int m = 0; m < PP; ++m)
#pragma unroll
            for (int c = 0; c < CG; ++c) tr[m][c] = ti[m][c] = make_float2(0.f, 0.f);

#pragma unroll 2
        for (int v = 0; v < kTile; ++v) {
            const double4 q = s_geo[b][v];
            float2 dx2[CG], dy2[CG];  // the datum broadcast to both rows of a pair
#pragma unroll
            for (int c = 0; c < CG; ++c) {
                const float2 d = s_dat[b][v * CG + c];
                dx2[c] = make_float2(d.x, d.x);
                dy2[c] = make_float2(d.y, d.y);
            }
            float cs[PT], sn[PT];
#pragma unroll
            for (int j = 0; j < PT; ++j) {
                double acc = fma(ox[j], q.x, kMagic);
                acc = fma(oy[j], q.y, acc);
                if (USEZ) acc = fma(oz[j], q.z, acc);
                acc = fma(ow[j], q.w, acc);
                const unsigned P = (unsigned)__double2loint(acc);
                const float f1 = __uint_as_float(__funnelshift_r(P, 0x7Fu, 9));
                const float ang =
                    ADJ ? fmaf(f1, -kTwoPiF, kThreePiF) : fmaf(f1, kTwoPiF, -kThreePiF);
                __sincosf(ang, &sn[j], &cs[j]);
            }
#pragma unroll
            for (int m = 0; m < PP; ++m) {
                const float2 c2 = make_float2(cs[2 * m], cs[2 * m + 1]);
                const float2 s2 = make_float2(sn[2 * m], sn[2 * m + 1]);
                const float2 ns2 = make_float2(-sn[2 * m], -sn[2 * m + 1]);
#pragma unroll
                for (int c = 0; c < CG; ++c) {
                    tr[m][c] = __ffma2_rn(dx2[c], c2, __ffma2_rn(dy2[c], s2, tr[m][c]));
                    ti[m][c] = __ffma2_rn(dy2[c], c2, __ffma2_rn(dx2[c], ns2, ti[m][c]));
                }
            }
        }
#pragma unroll
        for (int m = 0; m < PP; ++m)
#pragma unroll
            for (int c = 0; c < CG; ++c) {
                ar[2 * m][c] += tr[m][c].x;
                ar[2 * m + 1][c] += tr[m][c].y;
                ai[2 * m][c] += ti[m][c].x;
                ai[2 * m + 1][c] += ti[m][c].y;
            }
        __syncthreads();
    }

    const int G = BATCH ? n_groups : (int)gridDim.z;
    if (!ADJ) {
        float2 *o = out + ((size_t)(split * G + g) * n_ours_pad) * CG;
#pragma unroll
        for (int j = 0; j < PT; ++j) {
            const int e = e0 + j * kNT;
#pragma unroll
            for (int c = 0; c < CG; ++c) o[(size_t)e * CG + c] = make_float2(ar[j][c], ai[j][c]);
        }
    } else {
        float2 *o = out + (size_t)(split * G + g) * n_ours_pad;
        const float2 *s = sens + (size_t)g * n_ours_pad * CG;
#pragma unroll
        for (int j = 0; j < PT; ++j) {
            const int e = e0 + j * kNT;
            float zr = 0.f, zi = 0.f;
#pragma unroll
            for (int c = 0; c < CG; ++c) {
                const float2 sv = s[(size_t)e * CG + c];
                zr += sv.x * ar[j][c] + sv.y * ai[j][c];
                zi += sv.x * ai[j][c] - sv.y * ar[j][c];
            }
            o[e] = make_float2(zr, zi);
        }
    }
}

// ------------------------------ packing ------------------------------------

__global__ void k_pack_kgeo(double4 *kgeo, const float *kx, const float *ky, const float *kz,
                            const float *t, int M, int Mpad, int use_z, unsigned *err) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= Mpad) return;
    double4 q = make_double4(0.0, 0.0, 0.0, 0.0);
    if (i < M) {
        q.x = (double)kx[i];
        q.y = (double)ky[i];
        q.z = use_z ? (double)kz[i] : 0.0;
        q.w = (double)t[i];
        // keeps |phase| < 2^19 turns: |k| <= 2^15 cycles/FOV, |t| <= 16 s
        if (!(fabs(q.x) <= 32768.0 && fabs(q.y) <= 32768.0 && fabs(q.z) <= 32768.0 &&
              fabs(q.w) <= 16.0))
            atomicOr(err, DEV_ERR_RANGE);
    }
    kgeo[i] = q;
}

__global__ void k_pack_vgeo(double4 *vgeo, const float *ix, const float *iy, const float *iz,
                            const float *fm, int N, int Npad, int use_z, unsigned *err) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= Npad) return;
    double4 q = make_double4(0.0, 0.0, 0.0, 0.0);
    if (i < N) {
        q.x = (double)ix[i];
        q.y = (double)iy[i];
        q.z = use_z ? (double)iz[i] : 0.0;
        q.w = fm ? (double)fm[i] / kTwoPi : 0.0;
        // |r| <= 2 FOV, |omega / 2pi| <= 8192 Hz
        if (!(fabs(q.x) <= 2.0 && fabs(q.y) <= 2.0 && fabs(q.z) <= 2.0 && fabs(q.w) <= 8192.0))
            atomicOr(err, DEV_ERR_RANGE);
    }
    vgeo[i] = q;
}

__global__ void k_set_fm(double4 *vgeo, const float *fm, int N, int Npad, unsigned *err) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= Npad) return;
    const double f = (i < N && fm) ? (double)fm[i] / kTwoPi : 0.0;
    if (!(fabs(f) <= 8192.0)) atomicOr(err, DEV_ERR_RANGE);
    vgeo[i].w = f;
}

__global__ void k_pack_sens(float2 *sens, const float *sr, const float *si, int N, int Npad,
                            int C, int CG, int G) {
    const size_t n = (size_t)G * Npad * CG;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x) {
        const int cg = (int)(i % CG);
        const size_t gr = i / CG;
        const int r = (int)(gr % Npad);
        const int g = (int)(gr / Npad);
        const int c = g * CG + cg;
        float2 v = make_float2(0.f, 0.f);
        if (c < C && r < N) {
            if (sr)
                v = make_float2(sr[(size_t)c * N + r], si ? si[(size_t)c * N + r] : 0.f);
            else
                v = make_float2(1.f, 0.f);
        }
        sens[i] = v;
    }
}

__global__ void k_pack_image(float2 *xs, const float2 *x, const float2 *sens, int Npad, int CG,
                             int G) {
    const size_t n = (size_t)G * Npad * CG;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x) {
        const int r = (int)((i / CG) % Npad);
        xs[i] = cmul(sens[i], x[r]);
    }
}

__global__ void k_pack_image_soa(float2 *xs, const float *xr, const float *xi,
                                 const float2 *sens, int N, int Npad, int CG, int G) {
    const size_t n = (size_t)G * Npad * CG;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x) {
        const int r = (int)((i / CG) % Npad);
        const float2 x = r < N ? make_float2(xr[r], xi[r]) : make_float2(0.f, 0.f);
        xs[i] = cmul(sens[i], x);
    }
}

__global__ void k_pack_kdata(float2 *packed, const float *dr, const float *di, int M, int Mpad,
                             int C, int CG, int G) {
    const size_t n = (size_t)G * Mpad * CG;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x) {
        const int cg = (int)(i % CG);
        const size_t gk = i / CG;
        const int k = (int)(gk % Mpad);
        const int c = (int)(gk / Mpad) * CG + cg;
        packed[i] = (c < C && k < M) ? make_float2(dr[(size_t)c * M + k], di[(size_t)c * M + k])
                                     : make_float2(0.f, 0.f);
    }
}

__global__ void k_fwd_finish_soa(float *yr, float *yi, const float2 *part, int M, int Mpad,
                                 int C, int CG, int G, int S) {
    const size_t n = (size_t)C * M;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x) {
        const int c = (int)(i / M), k = (int)(i % M);
        const int g = c / CG, cg = c % CG;
        float sr = 0.f, si = 0.f;
        for (int s = 0; s < S; ++s) {
            const float2 v = part[(((size_t)s * G + g) * Mpad + k) * CG + cg];
            sr += v.x;
            si += v.y;
        }
        yr[i] = sr;
        yi[i] = si;
    }
}

__global__ void k_adj_finish_soa(float *xr, float *xi, const float2 *part, int N, int Npad,
                                 int SG) {
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < N; r += gridDim.x * blockDim.x) {
        float sr = 0.f, si = 0.f;
        for (int s = 0; s < SG; ++s) {
            const float2 v = part[(size_t)s * Npad + r];
            sr += v.x;
            si += v.y;
        }
        xr[r] = sr;
        xi[r] = si;
    }
}

inline int grid_for(size_t n, int bs = 256) {
    size_t b = (n + bs - 1) / bs;
    return (int)std::min<size_t>(std::max<size_t>(b, 1), 148 * 16);
}

// ------------------------------ dispatch -----------------------------------

template <int CG, int PT, bool ADJ, int OCC>
cudaError_t launch_cg_pt(const NuPlan &p, int split, const double4 *ours, const double4 *theirs,
                         const float2 *tdata, float2 *out, unsigned *err, cudaStream_t st) {
    const int n_ours = ADJ ? p.Npad : p.Mpad;
    const int n_theirs = ADJ ? p.Mpad : p.Npad;
    if (!nu_split_ok(n_theirs, split)) return cudaErrorInvalidConfiguration;
    const int per_split = n_theirs / split;
    dim3 grid(n_ours / (kNT * PT), split, p.G);
    if (p.use_z)
        k_nudft<CG, PT, true, ADJ, OCC, false><<<grid, kNT, 0, st>>>(
            ours, theirs, tdata, p.sens, out, n_ours, n_theirs, per_split, err, nullptr, p.G);
    else
        k_nudft<CG, PT, false, ADJ, OCC, false><<<grid, kNT, 0, st>>>(
            ours, theirs, tdata, p.sens, out, n_ours, n_theirs, per_split, err, nullptr, p.G);
    return cudaGetLastError();
}

// Batched: S slices sharing N, C and the sensitivities; `max_ours` is the
// largest padded "ours" count of a slice.
template <int CG, int PT, bool ADJ, int OCC>
cudaError_t launch_cg_pt_batch(const NuPlan &p, int split, int S, int max_ours,
                               const NuSlice *sl, const double4 *ours, const double4 *theirs,
                               const float2 *tdata, float2 *out, unsigned *err,
                               cudaStream_t st) {
    if ((long long)S * p.G > 65535 || max_ours % (kNT * PT)) return cudaErrorInvalidConfiguration;
    dim3 grid(max_ours / (kNT * PT), split, S * p.G);
    if (p.use_z)
        k_nudft<CG, PT, true, ADJ, OCC, true><<<grid, kNT, 0, st>>>(
            ours, theirs, tdata, p.sens, out, 0, 0, 0, err, sl, p.G);
    else
        k_nudft<CG, PT, false, ADJ, OCC, true><<<grid, kNT, 0, st>>>(
            ours, theirs, tdata, p.sens, out, 0, 0, 0, err, sl, p.G);
    return cudaGetLastError();
}

template <bool ADJ>
cudaError_t launch_nudft_batch(const NuPlan &p, const NuLaunch &l, int S, int max_ours,
                               const NuSlice *sl, const double4 *ours, const double4 *theirs,
                               const float2 *tdata, float2 *out, unsigned *err,
                               cudaStream_t st) {
    if (l.tc)
        return nu_partials_tc_batch(p, l, ADJ, S, max_ours, sl, ours, theirs, tdata, out, err,
                                    st);
#define IMP_CASE(CGV, PTV)                                                                     \
    if (p.CG == CGV && l.pt == PTV) {                                                          \
        if (l.occ == 6)                                                                        \
            return launch_cg_pt_batch<CGV, PTV, ADJ, 6>(p, l.split, S, max_ours, sl, ours,     \
                                                        theirs, tdata, out, err, st);          \
        return launch_cg_pt_batch<CGV, PTV, ADJ, 4>(p, l.split, S, max_ours, sl, ours, theirs, \
                                                    tdata, out, err, st);                      \
    }
    IMP_CASE(1, 4)
    IMP_CASE(1, 8)
    IMP_CASE(2, 4)
    IMP_CASE(4, 2)
    IMP_CASE(4, 4)
    IMP_CASE(8, 2)
#undef IMP_CASE
    return cudaErrorInvalidConfiguration;
}

template <bool ADJ>
cudaError_t launch_nudft(const NuPlan &p, const NuLaunch &l, const float2 *tdata, float2 *out,
                         unsigned *err, cudaStream_t st) {
    if (l.tc) return nu_partials_tc(p, l, ADJ, tdata, out, err, st);
    const double4 *ours = ADJ ? p.vgeo : p.kgeo;
    const double4 *theirs = ADJ ? p.kgeo : p.vgeo;
#define IMP_CASE(CGV, PTV)                                                                   \
    if (p.CG == CGV && l.pt == PTV) {                                                        \
        if (l.occ == 6)                                                                      \
            return launch_cg_pt<CGV, PTV, ADJ, 6>(p, l.split, ours, theirs, tdata, out, err, \
                                                  st);                                       \
        return launch_cg_pt<CGV, PTV, ADJ, 4>(p, l.split, ours, theirs, tdata, out, err, st); \
    }
    IMP_CASE(1, 4)
    IMP_CASE(1, 8)
    IMP_CASE(2, 4)
    IMP_CASE(4, 2)
    IMP_CASE(4, 4)
    IMP_CASE(8, 2)
#undef IMP_CASE
    return cudaErrorInvalidConfiguration;
}

}  // namespace

bool nu_split_ok(int n_theirs, int split) {
    return split >= 1 && n_theirs % split == 0 && (n_theirs / split) % kTile == 0 &&
           n_theirs / split >= kTile;
}

bool nu_tc_enabled() {
    const char *e = std::getenv("IMP_NUDFT_TC");
    return !(e && e[0] == '0');
}

bool nu_tc_forced() {
    const char *e = std::getenv("IMP_NUDFT_TC");
    return e && e[0] == '1';
}

bool nu_shape_supported(int CG, int pt) {
    return (CG == 1 && (pt == 4 || pt == 8)) || (CG == 2 && pt == 4) ||
           (CG == 4 && (pt == 2 || pt == 4)) || (CG == 8 && pt == 2);
}

// Coils per group.  Above 8 coils the tensor-core kernel takes groups of 16
// or 32 (one phase per pair for all of them); IMP_NUDFT_TC=0 keeps groups of
// at most 8 for the CUDA-core kernel.
static int choose_cg(int C) {
    if (C <= 1) return 1;
    if (C <= 2) return 2;
    if (C <= 4) return 4;
    if (C <= 8 || !nu_tc_enabled()) return 8;
    return C <= 16 ? 16 : 32;
}

static int round_up(int a, int b) { return (a + b - 1) / b * b; }

NuLaunch nu_default_launch(const NuPlan &p, bool adj) {
    NuLaunch l;
    l.pt = p.CG >= 8 ? 2 : 4;
    const int n_ours = adj ? p.Npad : p.Mpad;
    const int n_theirs = adj ? p.Mpad : p.Npad;
    const bool simt = nu_shape_supported(p.CG, p.CG >= 8 ? 2 : 4);
    if ((nu_tc_forced() || !simt) && nu_tc_supported(p.CG) && n_ours % nu_tc_rows(p.CG) == 0) {
        // one block per SM: about eight waves of blocks, whole tiles per split
        l.tc = 1;
        const long blocks = (long)(n_ours / nu_tc_rows(p.CG)) * p.G;
        int split = 1;
        while (blocks * split < 148L * 8 && split < 64 && nu_split_ok(n_theirs, split * 2) &&
               n_theirs / (split * 2) >= 4 * kTile)
            split *= 2;
        l.split = split;
        return l;
    }
    const long blocks = (long)(n_ours / (kNT * l.pt)) * p.G;
    const long target = 148L * 4 * 2;  // two waves at four blocks per SM
    int split = 1;
    while (blocks * split < target && split < 64 && nu_split_ok(n_theirs, split * 2) &&
           n_theirs / (split * 2) >= 4 * kTile)
        split *= 2;
    l.split = split;
    return l;
}

static cudaError_t pack_geometry(NuPlan &p, const float *kx, const float *ky, const float *kz,
                                 const float *t, const float *ix, const float *iy,
                                 const float *iz, const float *fm, const float *sensi_r,
                                 const float *sensi_i, unsigned *dev_err, cudaStream_t st) {
    k_pack_kgeo<<<(p.Mpad + 255) / 256, 256, 0, st>>>(p.kgeo, kx, ky, kz, t, p.M, p.Mpad,
                                                       p.use_z ? 1 : 0, dev_err);
    k_pack_vgeo<<<(p.Npad + 255) / 256, 256, 0, st>>>(p.vgeo, ix, iy, iz, fm, p.N, p.Npad,
                                                       p.use_z ? 1 : 0, dev_err);
    k_pack_sens<<<grid_for((size_t)p.G * p.Npad * p.CG), 256, 0, st>>>(
        p.sens, sensi_r, sensi_i, p.N, p.Npad, p.C, p.CG, p.G);
    return cudaGetLastError();
}

cudaError_t nu_plan_create(NuPlan &p, const float *kx, const float *ky, const float *kz,
                           const float *t, const float *ix, const float *iy, const float *iz,
                           const float *fm, const float *sensi_r, const float *sensi_i, int M,
                           int N, int C, bool use_z, unsigned *dev_err, cudaStream_t st) {
    nu_plan_destroy(p);
    p.M = M;
    p.N = N;
    p.C = C;
    p.CG = choose_cg(C);
    p.G = (C + p.CG - 1) / p.CG;
    p.Mpad = round_up(std::max(M, 1), kPadM);
    p.Npad = round_up(std::max(N, 1), kPadM);
    p.use_z = use_z;
    cudaError_t e;
    if ((e = cudaMalloc(&p.kgeo, sizeof(double4) * p.Mpad)) != cudaSuccess) return e;
    if ((e = cudaMalloc(&p.vgeo, sizeof(double4) * p.Npad)) != cudaSuccess) return e;
    if ((e = cudaMalloc(&p.sens, sizeof(float2) * (size_t)p.G * p.Npad * p.CG)) != cudaSuccess)
        return e;
    p.fwd = nu_default_launch(p, false);
    p.adj = nu_default_launch(p, true);
    return pack_geometry(p, kx, ky, kz, t, ix, iy, iz, fm, sensi_r, sensi_i, dev_err, st);
}

cudaError_t nu_plan_repack(NuPlan &p, const float *kx, const float *ky, const float *kz,
                           const float *t, const float *ix, const float *iy, const float *iz,
                           const float *sensi_r, const float *sensi_i, unsigned *dev_err,
                           cudaStream_t st) {
    return pack_geometry(p, kx, ky, kz, t, ix, iy, iz, nullptr, sensi_r, sensi_i, dev_err, st);
}

cudaError_t nu_plan_set_fm(NuPlan &p, const float *fm, unsigned *dev_err, cudaStream_t st) {
    k_set_fm<<<(p.Npad + 255) / 256, 256, 0, st>>>(p.vgeo, fm, p.N, p.Npad, dev_err);
    return cudaGetLastError();
}

void nu_plan_dims(NuPlan &p, int M, int N, int C, bool use_z) {
    p.M = M;
    p.N = N;
    p.C = C;
    p.CG = choose_cg(C);
    p.G = (C + p.CG - 1) / p.CG;
    p.Mpad = round_up(std::max(M, 1), kPadM);
    p.Npad = round_up(std::max(N, 1), kPadM);
    p.use_z = use_z;
}

cudaError_t nu_plan_place(NuPlan &p, double4 *kgeo, double4 *vgeo, float2 *sens,
                          const float *kx, const float *ky, const float *kz, const float *t,
                          const float *ix, const float *iy, const float *iz, const float *fm,
                          const float *sensi_r, const float *sensi_i, unsigned *dev_err,
                          cudaStream_t st) {
    p.kgeo = kgeo;
    p.vgeo = vgeo;
    p.sens = sens;
    p.fwd = nu_default_launch(p, false);
    p.adj = nu_default_launch(p, true);
    return pack_geometry(p, kx, ky, kz, t, ix, iy, iz, fm, sensi_r, sensi_i, dev_err, st);
}

void nu_plan_destroy(NuPlan &p) {
    if (p.kgeo) cudaFree(p.kgeo);
    if (p.vgeo) cudaFree(p.vgeo);
    if (p.sens) cudaFree(p.sens);
    p.kgeo = nullptr;
    p.vgeo = nullptr;
    p.sens = nullptr;
}

size_t nu_fwd_partial_bytes(const NuPlan &p, const NuLaunch &l) {
    return sizeof(float2) * (size_t)l.split * p.G * p.Mpad * p.CG;
}
size_t nu_adj_partial_bytes(const NuPlan &p, const NuLaunch &l) {
    return sizeof(float2) * (size_t)l.split * p.G * p.Npad;
}

cudaError_t nu_pack_image(const NuPlan &p, const float2 *x, float2 *xs, cudaStream_t st) {
    k_pack_image<<<grid_for((size_t)p.G * p.Npad * p.CG), 256, 0, st>>>(xs, x, p.sens, p.Npad,
                                                                       p.CG, p.G);
    return cudaGetLastError();
}

cudaError_t nu_pack_image_soa(const NuPlan &p, const float *xr, const float *xi, float2 *xs,
                              cudaStream_t st) {
    k_pack_image_soa<<<grid_for((size_t)p.G * p.Npad * p.CG), 256, 0, st>>>(
        xs, xr, xi, p.sens, p.N, p.Npad, p.CG, p.G);
    return cudaGetLastError();
}

cudaError_t nu_forward_partials(const NuPlan &p, const NuLaunch &l, const float2 *xs,
                                float2 *part, unsigned *dev_err, cudaStream_t st) {
    return launch_nudft<false>(p, l, xs, part, dev_err, st);
}

cudaError_t nu_adjoint_partials(const NuPlan &p, const NuLaunch &l, const float2 *data,
                                float2 *part, unsigned *dev_err, cudaStream_t st) {
    return launch_nudft<true>(p, l, data, part, dev_err, st);
}

cudaError_t nu_partials_batch(const NuPlan &p, const NuLaunch &l, bool adj, int S, int max_ours,
                              const NuSlice *d_slices, const double4 *ours,
                              const double4 *theirs, const float2 *tdata, float2 *part,
                              unsigned *dev_err, cudaStream_t st) {
    if (S < 1 || !d_slices) return cudaErrorInvalidValue;
    return adj ? launch_nudft_batch<true>(p, l, S, max_ours, d_slices, ours, theirs, tdata, part,
                                          dev_err, st)
               : launch_nudft_batch<false>(p, l, S, max_ours, d_slices, ours, theirs, tdata,
                                           part, dev_err, st);
}

cudaError_t nu_pack_kdata(const NuPlan &p, const float *dr, const float *di, float2 *packed,
                          cudaStream_t st) {
    k_pack_kdata<<<grid_for((size_t)p.G * p.Mpad * p.CG), 256, 0, st>>>(
        packed, dr, di, p.M, p.Mpad, p.C, p.CG, p.G);
    return cudaGetLastError();
}

cudaError_t nu_forward_finish_soa(const NuPlan &p, const NuLaunch &l, const float2 *part,
                                  float *yr, float *yi, cudaStream_t st) {
    k_fwd_finish_soa<<<grid_for((size_t)p.C * p.M), 256, 0, st>>>(yr, yi, part, p.M, p.Mpad,
                                                                   p.C, p.CG, p.G, l.split);
    return cudaGetLastError();
}

cudaError_t nu_adjoint_finish_soa(const NuPlan &p, const NuLaunch &l, const float2 *part,
                                  float *xr, float *xi, cudaStream_t st) {
    k_adj_finish_soa<<<grid_for((size_t)p.N), 256, 0, st>>>(xr, xi, part, p.N, p.Npad,
                                                            l.split * p.G);
    return cudaGetLastError();
}

}  // namespace imp

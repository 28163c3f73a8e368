// Batched multi-slice brute-force CG: S slices with their own trajectories
// (uneven sample counts), field maps and k-space data, one image grid and one
// set of coil maps, solved in lockstep.
//
// The iteration is the single-slice one of bruteforce.cu (bruteForceGpu /
// bruteForceCpu, bruteForce/bruteForceGpu.cu:431-760), run for every slice at
// once: each NUDFT apply is one launch of the tile engine over all slices
// (grid z = slice x coil group, offsets from a device table), each vector step
// one launch with blockIdx.y = slice, and each slice has its own FP64 CG
// scalars (its blocks' partial sums, summed by the consumer in fixed order).
// This replaces the reference's per-slice loop (main_mri.cu:875-895).
//
// Layouts (koff = the slice's offset in padded samples, sum of the earlier
// slices' Mpad):
//   kgeo [sum Mpad]            vgeo [S][Npad]          sens [G][Npad][CG] (shared)
//   y, af, q, rpk: slice at G*CG*koff, [G][Mpad][CG]
//   pf: slice at split_f*G*CG*koff, [split_f][G][Mpad][CG]
//   xs [S][G][Npad][CG]        pa [S][split_a][G][Npad]
//   x, g, d, w [S][Npad]       dots [S][5][kb]
#include "bruteforce.cuh"
#include "common.cuh"
#include "tv.cuh"

#include <algorithm>

namespace imp {

namespace {

enum { DOT_GG = 0, DOT_DG = 1, DOT_QQ = 2, DOT_SD = 3, DOT_OLD = 4 };
constexpr int kVB = 256;

struct BbSlice {
    long long koff;  // padded sample offset
    int M, Mpad;
    long long kraw;  // unpadded sample offset (k_off)
};

__device__ __forceinline__ bool k_valid(size_t i, int M, int Mpad, int C, int CG) {
    const int k = (int)((i / CG) % Mpad);
    const int c = (int)(i / ((size_t)CG * Mpad)) * CG + (int)(i % CG);
    return k < M && c < C;
}

// slice s's partial-sum row for product `which`
__device__ __forceinline__ double *dots_at(double *dots, int kb, int which) {
    return dots + ((size_t)blockIdx.y * 5 + which) * kb;
}

__global__ void k_bb_fill(float *w, float v, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x)
        w[i] = v;
}

// x [S][Npad] interleaved <- SoA [S][N]
__global__ void k_bb_soa_to_c2(float2 *x, const float *xr, const float *xi, int N, int Npad) {
    const int s = blockIdx.y;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < Npad; i += gridDim.x * blockDim.x)
        x[(size_t)s * Npad + i] = i < N ? make_float2(xr[(size_t)s * N + i], xi[(size_t)s * N + i])
                                        : make_float2(0.f, 0.f);
}

__global__ void k_bb_c2_to_soa(float *xr, float *xi, const float2 *x, int N, int Npad) {
    const int s = blockIdx.y;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
        const float2 v = x[(size_t)s * Npad + i];
        xr[(size_t)s * N + i] = v.x;
        xi[(size_t)s * N + i] = v.y;
    }
}

// k-space SoA (slice s: [C][M_s] at C * kraw) -> packed [G][Mpad][CG] at G*CG*koff
__global__ void k_bb_pack_kdata(float2 *packed, const float *dr, const float *di,
                                const BbSlice *sl, int C, int CG, int G) {
    const BbSlice d = sl[blockIdx.y];
    const size_t n = (size_t)G * d.Mpad * CG;
    float2 *o = packed + (size_t)d.koff * G * CG;
    const float *r = dr + (size_t)d.kraw * C, *im = di + (size_t)d.kraw * C;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x) {
        const int cg = (int)(i % CG);
        const size_t gk = i / CG;
        const int k = (int)(gk % d.Mpad);
        const int c = (int)(gk / d.Mpad) * CG + cg;
        o[i] = (c < C && k < d.M) ? make_float2(r[(size_t)c * d.M + k], im[(size_t)c * d.M + k])
                                  : make_float2(0.f, 0.f);
    }
}

// xs[s][g][r][cg] = S[g][r][cg] x[s][r]
__global__ void k_bb_pack_image(float2 *xs, const float2 *x, const float2 *sens, int Npad, int CG,
                                int G) {
    const int s = blockIdx.y;
    const size_t n = (size_t)G * Npad * CG;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x) {
        const int r = (int)((i / CG) % Npad);
        xs[(size_t)s * n + i] = cmul(sens[i], x[(size_t)s * Npad + r]);
    }
}

__global__ void k_bb_tv_weight(float *w, const float2 *x, int N, int Npad, Grid3 gd, float eps) {
    const int s = blockIdx.y;
    const float2 *xs = x + (size_t)s * Npad;
    float *ws = w + (size_t)s * Npad;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
        const int c = i % gd.n2;
        const int b = (i / gd.n2) % gd.n1;
        const int a = i / (gd.n2 * gd.n1);
        const float2 xi = xs[i];
        const int coord[3] = {a, b, c};
        const int n[3] = {gd.n0, gd.n1, gd.n2};
        const int st[3] = {gd.n1 * gd.n2, gd.n2, 1};
        float acc = 0.f;
#pragma unroll
        for (int ax = 0; ax < 3; ++ax) {
            if (n[ax] == 1) continue;
            const int in = coord[ax] == n[ax] - 1 ? i - (n[ax] - 1) * st[ax] : i + st[ax];
            const float2 xn = xs[in];
            const float dr = xi.x - xn.x, di = xi.y - xn.y;
            acc += dr * dr + di * di;
        }
        ws[i] = 0.5f / sqrtf(acc + eps);
    }
}

// Af = sum of forward partials (padding masked); rpk = y - Af
__global__ void __launch_bounds__(kVB) k_bb_init(float2 *af, float2 *rpk, const float2 *y,
                                                 const float2 *pf, int SF, const BbSlice *sl,
                                                 int C, int CG, int G) {
    const BbSlice d = sl[blockIdx.y];
    const size_t n = (size_t)G * d.Mpad * CG;
    const size_t base = (size_t)d.koff * G * CG;
    const float2 *p = pf + (size_t)SF * base;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x) {
        float2 v = make_float2(0.f, 0.f);
        if (k_valid(i, d.M, d.Mpad, C, CG))
            for (int s = 0; s < SF; ++s) {
                const float2 u = p[(size_t)s * n + i];
                v.x += u.x;
                v.y += u.y;
            }
        af[base + i] = v;
        const float2 yy = y[base + i];
        rpk[base + i] = make_float2(yy.x - v.x, yy.y - v.y);
    }
}

// g = sum adjoint partials - lambda D^H W D x ; partial <g,g>
__global__ void __launch_bounds__(kVB) k_bb_grad(float2 *g, const float2 *pa, int SG, int N,
                                                 int Npad, const float2 *x, const float *w,
                                                 Grid3 gd, int fd, float lambda, double *dots,
                                                 int kb) {
    __shared__ double sh[33];
    const size_t o = (size_t)blockIdx.y * Npad;
    const float2 *ps = pa + (size_t)blockIdx.y * SG * Npad;
    double loc = 0.0;
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < Npad; r += gridDim.x * blockDim.x) {
        float2 v = make_float2(0.f, 0.f);
        if (r < N) {
            for (int s = 0; s < SG; ++s) {
                const float2 u = ps[(size_t)s * Npad + r];
                v.x += u.x;
                v.y += u.y;
            }
            if (fd) {
                const float2 t = dhwd_at(x + o, w + o, r, gd);
                v.x -= lambda * t.x;
                v.y -= lambda * t.y;
            }
        }
        g[o + r] = v;
        loc += (double)v.x * v.x + (double)v.y * v.y;
    }
    const double b = block_sum(loc, sh);
    if (threadIdx.x == 0) dots_at(dots, kb, DOT_GG)[blockIdx.x] = b;
}

// d = g + gamma d ; xs = S d ; partial <d,g>
__global__ void __launch_bounds__(kVB) k_bb_dir(float2 *d, float2 *xs, const float2 *g,
                                                const float2 *sens, int Npad, int CG, int G,
                                                double *dots, int kb) {
    __shared__ double sh[33];
    const double newin = sum_partials(dots_at(dots, kb, DOT_GG), kb, sh);
    const double oldin = dots_at(dots, kb, DOT_OLD)[0];
    const float gam = oldin == 0.0 ? 0.f : (float)(newin / oldin);
    const size_t o = (size_t)blockIdx.y * Npad;
    float2 *xss = xs + (size_t)blockIdx.y * G * Npad * CG;
    double loc = 0.0;
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < Npad; r += gridDim.x * blockDim.x) {
        const float2 gv = g[o + r], dv = d[o + r];
        const float2 dn = make_float2(gv.x + gam * dv.x, gv.y + gam * dv.y);
        d[o + r] = dn;
        loc += (double)dn.x * gv.x + (double)dn.y * gv.y;
        for (int gg = 0; gg < G; ++gg)
            for (int c = 0; c < CG; ++c) {
                const size_t e = ((size_t)gg * Npad + r) * CG + c;
                xss[e] = cmul(sens[e], dn);
            }
    }
    const double b = block_sum(loc, sh);
    if (threadIdx.x == 0) dots_at(dots, kb, DOT_DG)[blockIdx.x] = b;
}

// q = sum forward partials (masked) ; partial |q|^2
__global__ void __launch_bounds__(kVB) k_bb_q(float2 *q, const float2 *pf, int SF,
                                              const BbSlice *sl, int C, int CG, int G,
                                              double *dots, int kb) {
    __shared__ double sh[33];
    const BbSlice d = sl[blockIdx.y];
    const size_t n = (size_t)G * d.Mpad * CG;
    const size_t base = (size_t)d.koff * G * CG;
    const float2 *p = pf + (size_t)SF * base;
    double loc = 0.0;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x) {
        float2 v = make_float2(0.f, 0.f);
        if (k_valid(i, d.M, d.Mpad, C, CG))
            for (int s = 0; s < SF; ++s) {
                const float2 u = p[(size_t)s * n + i];
                v.x += u.x;
                v.y += u.y;
            }
        q[base + i] = v;
        loc += (double)v.x * v.x + (double)v.y * v.y;
    }
    const double b = block_sum(loc, sh);
    if (threadIdx.x == 0) dots_at(dots, kb, DOT_QQ)[blockIdx.x] = b;
}

// partial Re<lambda D^H W D d, d>
__global__ void __launch_bounds__(kVB) k_bb_tvdot(const float2 *d, const float *w, int N,
                                                  int Npad, Grid3 gd, float lambda, double *dots,
                                                  int kb) {
    __shared__ double sh[33];
    const size_t o = (size_t)blockIdx.y * Npad;
    double loc = 0.0;
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < N; r += gridDim.x * blockDim.x) {
        const float2 t = dhwd_at(d + o, w + o, r, gd);
        const float2 dv = d[o + r];
        loc += (double)(lambda * t.x) * dv.x + (double)(lambda * t.y) * dv.y;
    }
    const double b = block_sum(loc, sh);
    if (threadIdx.x == 0) dots_at(dots, kb, DOT_SD)[blockIdx.x] = b;
}

// alpha ; Af += alpha q ; rpk = y - Af ; x += alpha d ; <g,g>_old = <g,g>
__global__ void __launch_bounds__(kVB) k_bb_update(float2 *af, float2 *rpk, const float2 *y,
                                                   const float2 *q, float2 *x, const float2 *d,
                                                   const BbSlice *sl, int CG, int G, int Npad,
                                                   double *dots, int kb) {
    __shared__ double sh[33];
    const double dg = sum_partials(dots_at(dots, kb, DOT_DG), kb, sh);
    const double qq = sum_partials(dots_at(dots, kb, DOT_QQ), kb, sh);
    const double sd = sum_partials(dots_at(dots, kb, DOT_SD), kb, sh);
    const float alpha = (float)(dg / (qq + sd));
    const BbSlice ds = sl[blockIdx.y];
    const size_t n = (size_t)G * ds.Mpad * CG;
    const size_t base = (size_t)ds.koff * G * CG;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x) {
        const float2 qv = q[base + i];
        float2 a = af[base + i];
        a.x += alpha * qv.x;
        a.y += alpha * qv.y;
        af[base + i] = a;
        const float2 yy = y[base + i];
        rpk[base + i] = make_float2(yy.x - a.x, yy.y - a.y);
    }
    const size_t o = (size_t)blockIdx.y * Npad;
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < Npad; r += gridDim.x * blockDim.x) {
        const float2 dv = d[o + r];
        float2 xv = x[o + r];
        xv.x += alpha * dv.x;
        xv.y += alpha * dv.y;
        x[o + r] = xv;
    }
    if (blockIdx.x == 0) {
        const double gg = sum_partials(dots_at(dots, kb, DOT_GG), kb, sh);
        if (threadIdx.x == 0) dots_at(dots, kb, DOT_OLD)[0] = gg;
    }
}

template <typename T>
cudaError_t dalloc(T **p, size_t count) {
    return cudaMalloc((void **)p, sizeof(T) * std::max<size_t>(count, 1));
}

// Split of the "theirs" range: about two waves of four blocks per SM, and
// whole tiles for every slice's range (`ranges`).
int batch_split(long long blocks, const std::vector<int> &ranges, bool tc) {
    // two waves at four blocks per SM; the tensor-core kernel runs one block
    // per SM and gets about eight waves
    const long long target = tc ? 148LL * 8 : 148LL * 4 * 2;
    int split = 1;
    auto ok = [&](int sp) {
        for (int r : ranges)
            if (!nu_split_ok(r, sp) || r / sp < 4 * kTile) return false;
        return true;
    };
    while (blocks * split < target && split < 64 && ok(split * 2)) split *= 2;
    return split;
}

}  // namespace

#define BB_TRY(x)                               \
    do {                                        \
        cudaError_t e_ = (x);                   \
        if (e_ != cudaSuccess) return e_;       \
    } while (0)

BfBatch::~BfBatch() { release(); }

void BfBatch::release() {
    if (g_iter_) cudaGraphExecDestroy(g_iter_);
    if (g_init_) cudaGraphExecDestroy(g_init_);
    g_iter_ = g_init_ = nullptr;
    void *bufs[] = {kgeo_, vgeo_, sens_, tab_fwd_, tab_adj_, tab_vec_, y_, af_, q_, rpk_, xs_,
                    x_,    g_,    d_,    w_,       pf_,      pa_,      dots_};
    for (void *b : bufs)
        if (b) cudaFree(b);
    kgeo_ = vgeo_ = nullptr;
    sens_ = y_ = af_ = q_ = rpk_ = xs_ = x_ = g_ = d_ = pf_ = pa_ = nullptr;
    tab_fwd_ = tab_adj_ = nullptr;
    tab_vec_ = nullptr;
    w_ = nullptr;
    dots_ = nullptr;
    plan_.kgeo = plan_.vgeo = nullptr;  // views of the buffers above
    plan_.sens = nullptr;
    S_ = 0;
}

cudaError_t BfBatch::setup(const BfConfig &cfg, int S, const int *k_off, const float *kx,
                           const float *ky, const float *kz, const float *t, const float *ix,
                           const float *iy, const float *iz, const float *fm,
                           const float *sensi_r, const float *sensi_i, unsigned *dev_err,
                           cudaStream_t st) {
    if (S < 1 || !k_off) return cudaErrorInvalidValue;
    release();
    cfg_ = cfg;
    st_ = st;
    err_ = dev_err;
    S_ = S;
    k_off_.assign(k_off, k_off + S + 1);
    m_.resize(S);
    mpad_.resize(S);
    koff_pad_.resize(S + 1);
    koff_pad_[0] = 0;
    max_mpad_ = 0;
    for (int s = 0; s < S; ++s) {
        m_[s] = k_off[s + 1] - k_off[s];
        if (m_[s] < 1) return cudaErrorInvalidValue;
        NuPlan ps;
        nu_plan_dims(ps, m_[s], cfg.N, cfg.C, cfg.use_z);
        mpad_[s] = ps.Mpad;
        koff_pad_[s + 1] = koff_pad_[s] + ps.Mpad;
        max_mpad_ = std::max(max_mpad_, ps.Mpad);
    }
    mpad_total_ = koff_pad_[S];
    nu_plan_dims(plan_, max_mpad_, cfg.N, cfg.C, cfg.use_z);
    const int G = plan_.G, CG = plan_.CG, Npad = plan_.Npad;
    if ((long long)S * G > 65535) return cudaErrorInvalidValue;
    BB_TRY(dalloc(&kgeo_, (size_t)mpad_total_));
    BB_TRY(dalloc(&vgeo_, (size_t)S * Npad));
    BB_TRY(dalloc(&sens_, (size_t)G * Npad * CG));
    // geometry of every slice, placed at its offsets (the shared sensitivities
    // are packed with each slice: same values)
    for (int s = 0; s < S; ++s) {
        NuPlan ps;
        nu_plan_dims(ps, m_[s], cfg.N, cfg.C, cfg.use_z);
        const size_t o = (size_t)k_off[s];
        BB_TRY(nu_plan_place(ps, kgeo_ + koff_pad_[s], vgeo_ + (size_t)s * Npad, sens_, kx + o,
                             ky + o, kz ? kz + o : nullptr, t + o, ix, iy, iz,
                             fm ? fm + (size_t)s * cfg.N : nullptr, sensi_r, sensi_i, dev_err,
                             st));
    }
    plan_.kgeo = kgeo_;
    plan_.vgeo = vgeo_;
    plan_.sens = sens_;
    // one launch shape for every slice: the heuristic, replaced by the batch's
    // tuned shape (tune_shapes) when tuning is on
    fwd_ = nu_default_launch(plan_, false);
    adj_ = nu_default_launch(plan_, true);
    const int fwd_rows = fwd_.tc ? nu_tc_rows(CG) : kNT * fwd_.pt;
    const int adj_rows = adj_.tc ? nu_tc_rows(CG) : kNT * adj_.pt;
    fwd_.split = batch_split((long long)(mpad_total_ / fwd_rows) * G, std::vector<int>{Npad},
                             fwd_.tc != 0);
    adj_.split = batch_split((long long)(Npad / adj_rows) * G * S, mpad_, adj_.tc != 0);
    std::vector<BbSlice> tv(S);
    for (int s = 0; s < S; ++s) tv[s] = BbSlice{koff_pad_[s], m_[s], mpad_[s], (long long)k_off[s]};
    BB_TRY(dalloc(&tab_fwd_, S));
    BB_TRY(dalloc(&tab_adj_, S));
    BB_TRY(cudaMalloc(&tab_vec_, sizeof(BbSlice) * S));
    BB_TRY(cudaMemcpyAsync(tab_vec_, tv.data(), sizeof(BbSlice) * S, cudaMemcpyHostToDevice, st));
    const size_t nk = (size_t)mpad_total_ * G * CG;
    BB_TRY(dalloc(&y_, nk));
    BB_TRY(dalloc(&af_, nk));
    BB_TRY(dalloc(&q_, nk));
    BB_TRY(dalloc(&rpk_, nk));
    BB_TRY(dalloc(&xs_, (size_t)S * G * Npad * CG));
    BB_TRY(dalloc(&x_, (size_t)S * Npad));
    BB_TRY(dalloc(&g_, (size_t)S * Npad));
    BB_TRY(dalloc(&d_, (size_t)S * Npad));
    BB_TRY(dalloc(&w_, (size_t)S * Npad));
    BB_TRY(tune_shapes(false));
    BB_TRY(tune_shapes(true));
    BB_TRY(set_table(false, fwd_.split));
    BB_TRY(set_table(true, adj_.split));
    BB_TRY(dalloc(&pf_, nk * fwd_.split));
    BB_TRY(dalloc(&pa_, (size_t)S * adj_.split * G * Npad));
    kb_ = std::max(2, std::min(kDotBlocks, (kDotBlocks + S - 1) / S));
    BB_TRY(dalloc(&dots_, (size_t)S * 5 * kb_));
    BB_TRY(cudaMemsetAsync(dots_, 0, sizeof(double) * S * 5 * kb_, st));
    return cudaStreamSynchronize(st);
}

// Per-slice table of one direction for a given split (see NuSlice).
cudaError_t BfBatch::set_table(bool adj, int split) {
    const int S = S_, G = plan_.G, CG = plan_.CG, Npad = plan_.Npad;
    std::vector<NuSlice> tab(S);
    for (int s = 0; s < S; ++s) {
        const long long ko = koff_pad_[s];
        tab[s] = adj ? NuSlice{(long long)s * Npad, ko, (long long)G * CG * ko,
                               (long long)s * split * G * Npad, Npad, mpad_[s], mpad_[s] / split}
                     : NuSlice{ko, (long long)s * Npad, (long long)s * G * Npad * CG,
                               (long long)split * G * CG * ko, mpad_[s], Npad, Npad / split};
    }
    BB_TRY(cudaMemcpyAsync(adj ? tab_adj_ : tab_fwd_, tab.data(), sizeof(NuSlice) * S,
                           cudaMemcpyHostToDevice, st_));
    return cudaStreamSynchronize(st_);  // `tab` ends with this call
}

// Launch shape of one direction for the whole batch: a cached result for this
// batched problem, else (tuning on) every candidate -- within the heuristic's
// kernel family, splits from half to four times the heuristic's that cut every
// slice into whole tiles and keep the partial sums within twice the
// heuristic's (at least 1 GB); for the CUDA-core kernel also every supported
// pt and both register budgets -- timed once over the whole batch with CUDA
// events on the batch's stream (inputs zeroed; the timing does not depend on
// the values), the fastest kept and cached.
cudaError_t BfBatch::tune_shapes(bool adj) {
    NuLaunch &l = adj ? adj_ : fwd_;
    const int G = plan_.G, CG = plan_.CG, Npad = plan_.Npad;
    const NuBatchKey key{adj ? 1 : 0, CG, G, plan_.use_z ? 1 : 0, S_, Npad, max_mpad_,
                         mpad_total_, l.tc};
    NuLaunch cached;
    if (nu_batch_lookup(key, &cached)) {
        l = cached;
        return cudaSuccess;
    }
    if (!nu_tuning_enabled()) return cudaSuccess;
    const std::vector<int> ranges = adj ? mpad_ : std::vector<int>{Npad};
    auto split_ok = [&](int sp) {
        for (int r : ranges)
            if (!nu_split_ok(r, sp) || r / sp < 2 * kTile) return false;
        return true;
    };
    const size_t per_split = adj ? (size_t)S_ * G * Npad : (size_t)mpad_total_ * G * CG;
    const size_t cap = std::max(2 * per_split * l.split, (size_t(1) << 30) / sizeof(float2));
    std::vector<NuLaunch> cands;
    std::vector<int> pts, occs;
    if (l.tc) {
        pts = {l.pt};
        occs = {l.occ};
    } else {
        for (int pt : {2, 4, 8})
            if (nu_shape_supported(CG, pt)) pts.push_back(pt);
        occs = {4, 6};
    }
    int max_split = 0;
    for (int pt : pts)
        for (int occ : occs)
            for (int sp = std::max(1, l.split / 2); sp <= std::min(64, 4 * l.split); sp *= 2) {
                if (!split_ok(sp) || per_split * sp > cap) continue;
                NuLaunch c = l;
                c.pt = pt;
                c.occ = occ;
                c.split = sp;
                cands.push_back(c);
                max_split = std::max(max_split, sp);
            }
    if (cands.size() < 2) {
        nu_batch_store(key, l, 0.0);
        return cudaSuccess;
    }
    float2 *part = nullptr;
    BB_TRY(dalloc(&part, per_split * max_split));
    const float2 *in = adj ? rpk_ : xs_;
    const size_t in_elems = adj ? (size_t)mpad_total_ * G * CG : (size_t)S_ * G * Npad * CG;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaError_t e = cudaMemsetAsync(const_cast<float2 *>(in), 0, sizeof(float2) * in_elems, st_);
    if (e == cudaSuccess) e = cudaEventCreate(&e0);
    if (e == cudaSuccess) e = cudaEventCreate(&e1);
    const int max_ours = adj ? Npad : max_mpad_;
    auto run = [&](const NuLaunch &c) {
        return adj ? nu_partials_batch(plan_, c, true, S_, max_ours, tab_adj_, vgeo_, kgeo_, in,
                                       part, err_, st_)
                   : nu_partials_batch(plan_, c, false, S_, max_ours, tab_fwd_, kgeo_, vgeo_, in,
                                       part, err_, st_);
    };
    float best = 1e30f;
    NuLaunch best_l = l;
    int table_split = -1;
    for (size_t i = 0; i < cands.size() && e == cudaSuccess; ++i) {
        const NuLaunch &c = cands[i];
        if (c.split != table_split) {
            e = set_table(adj, c.split);
            table_split = c.split;
            if (e != cudaSuccess) break;
        }
        if (i == 0 && (e = run(c)) != cudaSuccess) break;  // first use: module and caches warm
        cudaEventRecord(e0, st_);
        if ((e = run(c)) != cudaSuccess) break;
        cudaEventRecord(e1, st_);
        if ((e = cudaEventSynchronize(e1)) != cudaSuccess) break;
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (ms < best) {
            best = ms;
            best_l = c;
        }
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaFree(part);
    if (e != cudaSuccess) return e;
    l = best_l;
    nu_batch_store(key, l, best);
    return cudaSuccess;
}

cudaError_t BfBatch::run_init() {
    const int G = plan_.G, CG = plan_.CG, Npad = plan_.Npad;
    const BbSlice *tv = static_cast<const BbSlice *>(tab_vec_);
    k_bb_pack_image<<<dim3(kb_, S_), kVB, 0, st_>>>(xs_, x_, sens_, Npad, CG, G);
    BB_TRY(cudaGetLastError());
    BB_TRY(nu_partials_batch(plan_, fwd_, false, S_, max_mpad_, tab_fwd_, kgeo_, vgeo_, xs_, pf_,
                             err_, st_));
    k_bb_init<<<dim3(kb_, S_), kVB, 0, st_>>>(af_, rpk_, y_, pf_, fwd_.split, tv, plan_.C, CG, G);
    BB_TRY(cudaGetLastError());
    BB_TRY(cudaMemsetAsync(d_, 0, sizeof(float2) * S_ * Npad, st_));
    BB_TRY(cudaMemsetAsync(dots_, 0, sizeof(double) * S_ * 5 * kb_, st_));
    per_init_launches_ = 3;
    return cudaSuccess;
}

cudaError_t BfBatch::run_iteration() {
    const int G = plan_.G, CG = plan_.CG, Npad = plan_.Npad;
    const Grid3 gd{cfg_.n0, cfg_.n1, cfg_.n2};
    const BbSlice *tv = static_cast<const BbSlice *>(tab_vec_);
    const dim3 grid(kb_, S_);
    BB_TRY(nu_partials_batch(plan_, adj_, true, S_, Npad, tab_adj_, vgeo_, kgeo_, rpk_, pa_, err_,
                             st_));
    k_bb_grad<<<grid, kVB, 0, st_>>>(g_, pa_, adj_.split * G, plan_.N, Npad, x_, w_, gd,
                                     cfg_.fd ? 1 : 0, cfg_.lambda, dots_, kb_);
    BB_TRY(cudaGetLastError());
    k_bb_dir<<<grid, kVB, 0, st_>>>(d_, xs_, g_, sens_, Npad, CG, G, dots_, kb_);
    BB_TRY(cudaGetLastError());
    BB_TRY(nu_partials_batch(plan_, fwd_, false, S_, max_mpad_, tab_fwd_, kgeo_, vgeo_, xs_, pf_,
                             err_, st_));
    k_bb_q<<<grid, kVB, 0, st_>>>(q_, pf_, fwd_.split, tv, plan_.C, CG, G, dots_, kb_);
    BB_TRY(cudaGetLastError());
    int n = 5;
    if (cfg_.fd) {
        k_bb_tvdot<<<grid, kVB, 0, st_>>>(d_, w_, plan_.N, Npad, gd, cfg_.lambda, dots_, kb_);
        BB_TRY(cudaGetLastError());
        ++n;
    }
    k_bb_update<<<grid, kVB, 0, st_>>>(af_, rpk_, y_, q_, x_, d_, tv, CG, G, Npad, dots_, kb_);
    BB_TRY(cudaGetLastError());
    per_iter_launches_ = n + 1;
    return cudaSuccess;
}

static cudaError_t capture_bb(cudaStream_t st, cudaGraphExec_t *exec,
                              cudaError_t (BfBatch::*fn)(), BfBatch *self) {
    BB_TRY(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
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

cudaError_t BfBatch::solve(const float *kd_r, const float *kd_i, float *x_r, float *x_i) {
    if (S_ < 1) return cudaErrorInvalidValue;
    launches_ = 0;
    const int N = plan_.N, Npad = plan_.Npad;
    const Grid3 gd{cfg_.n0, cfg_.n1, cfg_.n2};
    const BbSlice *tv = static_cast<const BbSlice *>(tab_vec_);
    k_bb_pack_kdata<<<dim3(kb_, S_), kVB, 0, st_>>>(y_, kd_r, kd_i, tv, plan_.C, plan_.CG,
                                                    plan_.G);
    BB_TRY(cudaGetLastError());
    k_bb_soa_to_c2<<<dim3(kb_, S_), kVB, 0, st_>>>(x_, x_r, x_i, N, Npad);
    BB_TRY(cudaGetLastError());
    launches_ += 2;
    if (cfg_.use_graphs && !g_iter_) {
        BB_TRY(capture_bb(st_, &g_init_, &BfBatch::run_init, this));
        BB_TRY(capture_bb(st_, &g_iter_, &BfBatch::run_iteration, this));
    }
    for (int tv_i = 0; tv_i < std::max(cfg_.tv_num, 1); ++tv_i) {
        if (tv_i == 0)
            k_bb_fill<<<kDotBlocks, kVB, 0, st_>>>(w_, 1.f, (size_t)S_ * Npad);
        else if (cfg_.fd)
            k_bb_tv_weight<<<dim3(kb_, S_), kVB, 0, st_>>>(w_, x_, N, Npad, gd, cfg_.tv_eps);
        BB_TRY(cudaGetLastError());
        ++launches_;
        if (g_init_) {
            BB_TRY(cudaGraphLaunch(g_init_, st_));
        } else {
            BB_TRY(run_init());
        }
        launches_ += per_init_launches_;
        for (int it = 1; it < cfg_.cg_num; ++it) {
            if (g_iter_) {
                BB_TRY(cudaGraphLaunch(g_iter_, st_));
            } else {
                BB_TRY(run_iteration());
            }
            launches_ += per_iter_launches_;
        }
        if (!cfg_.tv) break;
    }
    k_bb_c2_to_soa<<<dim3(kb_, S_), kVB, 0, st_>>>(x_r, x_i, x_, N, Npad);
    BB_TRY(cudaGetLastError());
    ++launches_;
    return cudaSuccess;
}

}  // namespace imp

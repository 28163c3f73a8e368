// Brute-force CG reconstruction on the NUDFT tile engine.
//
// Same iteration as bruteForceGpu / bruteForceCpu
// (bruteForce/bruteForceGpu.cu:431-760, bruteForce/bruteForceCpu.cpp:246-478):
//
//   for tv_i < tv_num:                       W = 1 on the first pass, then
//       W = 0.5 / sqrt(sum_axes |D_a x|^2 + eps)        (multiplyCpu.cpp:84-110)
//       Af = A x
//       repeat cg_num-1 times:
//           g   = A^H (y - Af) - lambda D^H W D x
//           gam = <g,g> / <g,g>_old      (0 on the first update)
//           d   = g + gam d
//           q   = A d
//           alp = Re<d,g> / (|q|^2 + Re<lambda D^H W D d, d>)
//           Af += alp q ;  x += alp d
//
// A = F with SENSE coils.  The CG inner products, gamma and alpha are FP64
// and never leave the GPU: every kernel that needs a scalar sums the FP64
// per-block partials of its producer itself (deterministic order).  One CG
// update is seven launches, captured once into a CUDA graph and replayed.
#include "bruteforce.cuh"
#include "common.cuh"
#include "tv.cuh"

#include <algorithm>

namespace imp {

namespace {

enum { DOT_GG = 0, DOT_DG = 1, DOT_QQ = 2, DOT_SD = 3, DOT_OLD = 4 };
constexpr int kVB = 256;  // threads per vector-kernel block

__global__ void k_tv_weight(float *w, const float2 *x, int N, Grid3 gd, float eps) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
        const int c = i % gd.n2;
        const int b = (i / gd.n2) % gd.n1;
        const int a = i / (gd.n2 * gd.n1);
        const float2 xi = x[i];
        const int coord[3] = {a, b, c};
        const int n[3] = {gd.n0, gd.n1, gd.n2};
        const int st[3] = {gd.n1 * gd.n2, gd.n2, 1};
        float s = 0.f;
#pragma unroll
        for (int ax = 0; ax < 3; ++ax) {
            if (n[ax] == 1) continue;
            const int in = coord[ax] == n[ax] - 1 ? i - (n[ax] - 1) * st[ax] : i + st[ax];
            const float2 xn = x[in];
            const float dr = xi.x - xn.x, di = xi.y - xn.y;
            s += dr * dr + di * di;
        }
        w[i] = 0.5f / sqrtf(s + eps);
    }
}

__global__ void k_fill(float *w, float v, int n) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        w[i] = v;
}

__global__ void k_soa_to_c2(float2 *x, const float *xr, const float *xi, int N, int Npad) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < Npad; i += gridDim.x * blockDim.x)
        x[i] = i < N ? make_float2(xr[i], xi[i]) : make_float2(0.f, 0.f);
}

__global__ void k_c2_to_soa(float *xr, float *xi, const float2 *x, int N) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
        const float2 v = x[i];
        xr[i] = v.x;
        xi[i] = v.y;
    }
}

struct KLayout {
    int M, Mpad, C, CG, G;
    __host__ __device__ size_t n() const { return (size_t)G * Mpad * CG; }
    __device__ bool valid(size_t i) const {
        const int k = (int)((i / CG) % Mpad);
        const int c = (int)(i / ((size_t)CG * Mpad)) * CG + (int)(i % CG);
        return k < M && c < C;
    }
};

// Af = sum of forward partials (padding masked); rpk = y - Af
__global__ void k_bf_init(float2 *af, float2 *rpk, const float2 *y, const float2 *pf, int S,
                          KLayout L) {
    const size_t n = L.n();
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x) {
        float2 v = make_float2(0.f, 0.f);
        if (L.valid(i))
            for (int s = 0; s < S; ++s) {
                const float2 u = pf[(size_t)s * n + i];
                v.x += u.x;
                v.y += u.y;
            }
        af[i] = v;
        const float2 yy = y[i];
        rpk[i] = make_float2(yy.x - v.x, yy.y - v.y);
    }
}

// Penalty term of the gradient and of the step length: 0 none, 1 the
// finite-difference stencil lambda D^H W D, 2 the sparse roughness matrix
// lambda C^T W C (with y = W C v formed beforehand).
enum { PEN_NONE = 0, PEN_FD = 1, PEN_REG = 2 };

// g = sum adjoint partials - lambda (D^H W D | C^T W C) x ; partial <g,g>
__global__ void __launch_bounds__(kVB) k_bf_grad(float2 *g, const float2 *pa, int SG, int N,
                                                 int Npad, const float2 *x, const float *w,
                                                 Grid3 gd, int pen, float lambda, RegView reg,
                                                 double *dots) {
    __shared__ double sh[33];
    double loc = 0.0;
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < Npad; r += gridDim.x * blockDim.x) {
        float2 v = make_float2(0.f, 0.f);
        if (r < N) {
            for (int s = 0; s < SG; ++s) {
                const float2 u = pa[(size_t)s * Npad + r];
                v.x += u.x;
                v.y += u.y;
            }
            if (pen) {
                const float2 t = pen == PEN_REG ? reg_ct_at(reg, r) : dhwd_at(x, w, r, gd);
                v.x -= lambda * t.x;
                v.y -= lambda * t.y;
            }
        }
        g[r] = v;
        loc += (double)v.x * v.x + (double)v.y * v.y;
    }
    const double b = block_sum(loc, sh);
    if (threadIdx.x == 0) dots[DOT_GG * kDotBlocks + blockIdx.x] = b;
}

// d = g + gamma d ; xs = S d ; partial <d,g>
__global__ void __launch_bounds__(kVB) k_bf_dir(float2 *d, float2 *xs, const float2 *g,
                                                const float2 *sens, int Npad, int CG, int G,
                                                double *dots) {
    __shared__ double sh[33];
    const double newin = sum_partials(dots + DOT_GG * kDotBlocks, kDotBlocks, sh);
    const double oldin = dots[DOT_OLD * kDotBlocks];
    const float gam = oldin == 0.0 ? 0.f : (float)(newin / oldin);
    double loc = 0.0;
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < Npad; r += gridDim.x * blockDim.x) {
        const float2 gv = g[r], dv = d[r];
        const float2 dn = make_float2(gv.x + gam * dv.x, gv.y + gam * dv.y);
        d[r] = dn;
        loc += (double)dn.x * gv.x + (double)dn.y * gv.y;
        for (int gg = 0; gg < G; ++gg)
            for (int c = 0; c < CG; ++c) {
                const size_t o = ((size_t)gg * Npad + r) * CG + c;
                xs[o] = cmul(sens[o], dn);
            }
    }
    const double b = block_sum(loc, sh);
    if (threadIdx.x == 0) dots[DOT_DG * kDotBlocks + blockIdx.x] = b;
}

// q = sum forward partials (masked) ; partial |q|^2
__global__ void __launch_bounds__(kVB) k_bf_q(float2 *q, const float2 *pf, int S, KLayout L,
                                              double *dots) {
    __shared__ double sh[33];
    const size_t n = L.n();
    double loc = 0.0;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x) {
        float2 v = make_float2(0.f, 0.f);
        if (L.valid(i))
            for (int s = 0; s < S; ++s) {
                const float2 u = pf[(size_t)s * n + i];
                v.x += u.x;
                v.y += u.y;
            }
        q[i] = v;
        loc += (double)v.x * v.x + (double)v.y * v.y;
    }
    const double b = block_sum(loc, sh);
    if (threadIdx.x == 0) dots[DOT_QQ * kDotBlocks + blockIdx.x] = b;
}

// partial Re<lambda (D^H W D | C^T W C) d, d>
__global__ void __launch_bounds__(kVB) k_bf_tvdot(const float2 *d, const float *w, int N,
                                                  Grid3 gd, int pen, float lambda, RegView reg,
                                                  double *dots) {
    __shared__ double sh[33];
    double loc = 0.0;
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < N; r += gridDim.x * blockDim.x) {
        const float2 t = pen == PEN_REG ? reg_ct_at(reg, r) : dhwd_at(d, w, r, gd);
        const float2 dv = d[r];
        loc += (double)(lambda * t.x) * dv.x + (double)(lambda * t.y) * dv.y;
    }
    const double b = block_sum(loc, sh);
    if (threadIdx.x == 0) dots[DOT_SD * kDotBlocks + blockIdx.x] = b;
}

// alpha ; Af += alpha q ; rpk = y - Af ; x += alpha d ; <g,g>_old = <g,g>
__global__ void __launch_bounds__(kVB) k_bf_update(float2 *af, float2 *rpk, const float2 *y,
                                                   const float2 *q, float2 *x, const float2 *d,
                                                   KLayout L, int Npad, double *dots) {
    __shared__ double sh[33];
    const double dg = sum_partials(dots + DOT_DG * kDotBlocks, kDotBlocks, sh);
    const double qq = sum_partials(dots + DOT_QQ * kDotBlocks, kDotBlocks, sh);
    const double sd = sum_partials(dots + DOT_SD * kDotBlocks, kDotBlocks, sh);
    const float alpha = (float)(dg / (qq + sd));
    const size_t n = L.n();
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x) {
        const float2 qv = q[i];
        float2 a = af[i];
        a.x += alpha * qv.x;
        a.y += alpha * qv.y;
        af[i] = a;
        const float2 yy = y[i];
        rpk[i] = make_float2(yy.x - a.x, yy.y - a.y);
    }
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < Npad; r += gridDim.x * blockDim.x) {
        const float2 dv = d[r];
        float2 xv = x[r];
        xv.x += alpha * dv.x;
        xv.y += alpha * dv.y;
        x[r] = xv;
    }
    if (blockIdx.x == 0) {
        const double gg = sum_partials(dots + DOT_GG * kDotBlocks, kDotBlocks, sh);
        if (threadIdx.x == 0) dots[DOT_OLD * kDotBlocks] = gg;
    }
}

template <typename T>
cudaError_t dalloc(T **p, size_t count) {
    return cudaMalloc((void **)p, sizeof(T) * std::max<size_t>(count, 1));
}

}  // namespace

cudaError_t tv_weight(float *w, const float2 *x, int N, Grid3 gd, float eps, cudaStream_t st) {
    k_tv_weight<<<kDotBlocks, kVB, 0, st>>>(w, x, N, gd, eps);
    return cudaGetLastError();
}

#define IMP_TRY(x)                              \
    do {                                        \
        cudaError_t e_ = (x);                   \
        if (e_ != cudaSuccess) return e_;       \
    } while (0)

BfSolver::~BfSolver() {
    release();
    for (cudaEvent_t e : prof_ev_) cudaEventDestroy(e);
}

// Records one timing event (pairs of marks bracket one launch of `kind`).
cudaError_t BfSolver::prof_mark(int kind) {
    if (!prof_on_) return cudaSuccess;
    if (prof_used_ == prof_ev_.size()) {
        cudaEvent_t e;
        IMP_TRY(cudaEventCreate(&e));
        prof_ev_.push_back(e);
        prof_kind_.push_back(kind);
    }
    prof_kind_[prof_used_] = kind;
    IMP_TRY(cudaEventRecord(prof_ev_[prof_used_], st_));
    ++prof_used_;
    return cudaSuccess;
}

cudaError_t BfSolver::profile_collect(double ms[2], long count[2]) {
    for (size_t i = 0; i + 1 < prof_used_; i += 2) {
        float t = 0.f;
        IMP_TRY(cudaEventElapsedTime(&t, prof_ev_[i], prof_ev_[i + 1]));
        ms[prof_kind_[i]] += t;
        count[prof_kind_[i]] += 1;
    }
    prof_used_ = 0;
    return cudaSuccess;
}

void BfSolver::release() {
    if (g_iter_) cudaGraphExecDestroy(g_iter_);
    if (g_init_) cudaGraphExecDestroy(g_init_);
    g_iter_ = g_init_ = nullptr;
    reg_.release();
    void *bufs[] = {y_, af_, q_, rpk_, xs_, x_, g_, d_, w_, pf_, pa_, dots_};
    for (void *b : bufs)
        if (b) cudaFree(b);
    y_ = af_ = q_ = rpk_ = xs_ = x_ = g_ = d_ = nullptr;
    w_ = nullptr;
    pf_ = pa_ = nullptr;
    dots_ = nullptr;
    nu_plan_destroy(plan_);
}

cudaError_t BfSolver::setup(const BfConfig &cfg, const float *kx, const float *ky,
                            const float *kz, const float *t, const float *ix, const float *iy,
                            const float *iz, const float *sensi_r, const float *sensi_i,
                            unsigned *dev_err, cudaStream_t st) {
    const bool same_shape = plan_.kgeo && st == st_ && dev_err == err_ && cfg.M == cfg_.M &&
                            cfg.N == cfg_.N && cfg.C == cfg_.C && cfg.use_z == cfg_.use_z &&
                            cfg.n0 == cfg_.n0 && cfg.n1 == cfg_.n1 && cfg.n2 == cfg_.n2 &&
                            cfg.autotune == cfg_.autotune;
    if (same_shape) {
        // keep buffers, tuned launch shapes and (if the captured scalars match) the graphs
        bool stale = cfg.fd != cfg_.fd || cfg.lambda != cfg_.lambda;
        cfg_ = cfg;
        bool moved = false;
        IMP_TRY(set_reg(&moved));
        if (stale || moved) {
            if (g_iter_) cudaGraphExecDestroy(g_iter_);
            if (g_init_) cudaGraphExecDestroy(g_init_);
            g_iter_ = g_init_ = nullptr;
        }
        return nu_plan_repack(plan_, kx, ky, kz, t, ix, iy, iz, sensi_r, sensi_i, dev_err, st);
    }
    release();
    cfg_ = cfg;
    st_ = st;
    err_ = dev_err;
    // field map is set per slice in solve()
    IMP_TRY(nu_plan_create(plan_, kx, ky, kz, t, ix, iy, iz, nullptr, sensi_r, sensi_i, cfg.M,
                           cfg.N, cfg.C, cfg.use_z, dev_err, st));
    const size_t nk = (size_t)plan_.G * plan_.Mpad * plan_.CG;
    const size_t nxs = (size_t)plan_.G * plan_.Npad * plan_.CG;
    IMP_TRY(dalloc(&y_, nk));
    IMP_TRY(dalloc(&af_, nk));
    IMP_TRY(dalloc(&q_, nk));
    IMP_TRY(dalloc(&rpk_, nk));
    IMP_TRY(dalloc(&xs_, nxs));
    IMP_TRY(dalloc(&x_, plan_.Npad));
    IMP_TRY(dalloc(&g_, plan_.Npad));
    IMP_TRY(dalloc(&d_, plan_.Npad));
    IMP_TRY(dalloc(&w_, plan_.Npad));
    // partial-sum scratch sized for every shape the autotuner may pick
    size_t pf_bytes = nu_fwd_partial_bytes(plan_, plan_.fwd);
    size_t pa_bytes = nu_adj_partial_bytes(plan_, plan_.adj);
    if (cfg.autotune) {
        pf_bytes = std::max(pf_bytes, nu_tune_partial_bytes(plan_, false));
        pa_bytes = std::max(pa_bytes, nu_tune_partial_bytes(plan_, true));
    }
    IMP_TRY(cudaMalloc(&pf_, pf_bytes));
    IMP_TRY(cudaMalloc(&pa_, pa_bytes));
    if (cfg.autotune) {
        IMP_TRY(cudaMemsetAsync(xs_, 0, sizeof(float2) * nxs, st_));
        IMP_TRY(cudaMemsetAsync(rpk_, 0, sizeof(float2) * nk, st_));
        IMP_TRY(nu_autotune(plan_, false, xs_, pf_, pf_bytes, err_, st_, &plan_.fwd));
        IMP_TRY(nu_autotune(plan_, true, rpk_, pa_, pa_bytes, err_, st_, &plan_.adj));
    }
    IMP_TRY(dalloc(&dots_, (size_t)5 * kDotBlocks));
    IMP_TRY(cudaMemsetAsync(dots_, 0, sizeof(double) * 5 * kDotBlocks, st_));
    bool moved = false;
    IMP_TRY(set_reg(&moved));
    return cudaGetLastError();
}

// Uploads (or drops) the -reg matrix of cfg_; *graphs_stale when the penalty
// kernels' arguments changed (matrix switched on or off, or its buffers moved).
cudaError_t BfSolver::set_reg(bool *graphs_stale) {
    *graphs_stale = false;
    if (!cfg_.reg) {
        if (reg_.on()) {
            reg_.release();
            *graphs_stale = true;
        }
        return cudaSuccess;
    }
    const bool was_on = reg_.on();
    bool moved = false;
    IMP_TRY(reg_.set(*cfg_.reg, cfg_.N, st_, &moved));
    *graphs_stale = moved || !was_on;
    return cudaSuccess;
}

cudaError_t BfSolver::run_init() {
    const Grid3 gd{cfg_.n0, cfg_.n1, cfg_.n2};
    (void)gd;
    KLayout L{plan_.M, plan_.Mpad, plan_.C, plan_.CG, plan_.G};
    IMP_TRY(nu_pack_image(plan_, x_, xs_, st_));
    IMP_TRY(prof_mark(0));
    IMP_TRY(nu_forward_partials(plan_, plan_.fwd, xs_, pf_, err_, st_));
    IMP_TRY(prof_mark(0));
    k_bf_init<<<kDotBlocks, kVB, 0, st_>>>(af_, rpk_, y_, pf_, plan_.fwd.split, L);
    IMP_TRY(cudaGetLastError());
    IMP_TRY(cudaMemsetAsync(d_, 0, sizeof(float2) * plan_.Npad, st_));
    IMP_TRY(cudaMemsetAsync(dots_ + DOT_OLD * kDotBlocks, 0, sizeof(double), st_));
    per_init_launches_ = 3;
    return cudaSuccess;
}

cudaError_t BfSolver::run_iteration() {
    const Grid3 gd{cfg_.n0, cfg_.n1, cfg_.n2};
    KLayout L{plan_.M, plan_.Mpad, plan_.C, plan_.CG, plan_.G};
    IMP_TRY(prof_mark(1));
    IMP_TRY(nu_adjoint_partials(plan_, plan_.adj, rpk_, pa_, err_, st_));
    IMP_TRY(prof_mark(1));
    // -reg takes precedence over -fd (bruteForce/bruteForceCpu.cpp:306-325)
    const int pen = reg_.on() ? PEN_REG : cfg_.fd ? PEN_FD : PEN_NONE;
    int n = 5;
    if (pen == PEN_REG) {  // y = W C x
        IMP_TRY(reg_.apply_cw(x_, w_, nullptr, st_));
        ++n;
    }
    k_bf_grad<<<kDotBlocks, kVB, 0, st_>>>(g_, pa_, plan_.adj.split * plan_.G, plan_.N,
                                           plan_.Npad, x_, w_, gd, pen, cfg_.lambda, reg_.view(),
                                           dots_);
    IMP_TRY(cudaGetLastError());
    k_bf_dir<<<kDotBlocks, kVB, 0, st_>>>(d_, xs_, g_, plan_.sens, plan_.Npad, plan_.CG, plan_.G,
                                          dots_);
    IMP_TRY(cudaGetLastError());
    IMP_TRY(prof_mark(0));
    IMP_TRY(nu_forward_partials(plan_, plan_.fwd, xs_, pf_, err_, st_));
    IMP_TRY(prof_mark(0));
    k_bf_q<<<kDotBlocks, kVB, 0, st_>>>(q_, pf_, plan_.fwd.split, L, dots_);
    IMP_TRY(cudaGetLastError());
    if (pen == PEN_REG) {  // y = W C d
        IMP_TRY(reg_.apply_cw(d_, w_, nullptr, st_));
        ++n;
    }
    if (pen) {
        k_bf_tvdot<<<kDotBlocks, kVB, 0, st_>>>(d_, w_, plan_.N, gd, pen, cfg_.lambda,
                                                reg_.view(), dots_);
        IMP_TRY(cudaGetLastError());
        ++n;
    }
    k_bf_update<<<kDotBlocks, kVB, 0, st_>>>(af_, rpk_, y_, q_, x_, d_, L, plan_.Npad, dots_);
    IMP_TRY(cudaGetLastError());
    per_iter_launches_ = n + 1;
    return cudaSuccess;
}

static cudaError_t capture(cudaStream_t st, cudaGraphExec_t *exec,
                           cudaError_t (BfSolver::*fn)(), BfSolver *self) {
    IMP_TRY(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
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

cudaError_t BfSolver::solve(const float *fm, const float *kd_r, const float *kd_i, float *x_r,
                            float *x_i) {
    launches_ = 0;
    const Grid3 gd{cfg_.n0, cfg_.n1, cfg_.n2};
    const int N = plan_.N, Npad = plan_.Npad;
    IMP_TRY(nu_plan_set_fm(plan_, fm, err_, st_));
    IMP_TRY(nu_pack_kdata(plan_, kd_r, kd_i, y_, st_));
    k_soa_to_c2<<<kDotBlocks, kVB, 0, st_>>>(x_, x_r, x_i, N, Npad);
    IMP_TRY(cudaGetLastError());
    launches_ += 3;
    if (cfg_.use_graphs && !prof_on_ && !g_iter_) {
        IMP_TRY(capture(st_, &g_init_, &BfSolver::run_init, this));
        IMP_TRY(capture(st_, &g_iter_, &BfSolver::run_iteration, this));
    }
    for (int tv_i = 0; tv_i < std::max(cfg_.tv_num, 1); ++tv_i) {
        if (tv_i == 0)
            k_fill<<<kDotBlocks, kVB, 0, st_>>>(w_, 1.f, Npad);
        else if (cfg_.fd || reg_.on())
            k_tv_weight<<<kDotBlocks, kVB, 0, st_>>>(w_, x_, N, gd, cfg_.tv_eps);
        IMP_TRY(cudaGetLastError());
        ++launches_;
        if (g_init_ && !prof_on_) {
            IMP_TRY(cudaGraphLaunch(g_init_, st_));
        } else {
            IMP_TRY(run_init());
        }
        launches_ += per_init_launches_;
        for (int it = 1; it < cfg_.cg_num; ++it) {
            if (g_iter_ && !prof_on_) {
                IMP_TRY(cudaGraphLaunch(g_iter_, st_));
            } else {
                IMP_TRY(run_iteration());
            }
            launches_ += per_iter_launches_;
        }
        if (!cfg_.tv) break;
    }
    k_c2_to_soa<<<kDotBlocks, kVB, 0, st_>>>(x_r, x_i, x_, N);
    IMP_TRY(cudaGetLastError());
    ++launches_;
    return cudaSuccess;
}

}  // namespace imp

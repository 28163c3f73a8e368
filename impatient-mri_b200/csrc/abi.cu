// C-ABI entry points (include/impatient_b200.h) and the mriSolver CLI.
#include "../../include/impatient_b200.h"
#include "bruteforce.cuh"
#include "common.cuh"
#include "context.h"
#include "io.h"
#include "nudft.cuh"
#include "toeplitz.cuh"

#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

imp_context::~imp_context() = default;

namespace imp {

namespace {
thread_local std::string g_last_error;
}  // namespace

imp_status fail(imp_status s, const std::string &msg) {
    g_last_error = msg;
    return s;
}

imp_status from_cuda(cudaError_t e, const char *what) {
    if (e == cudaSuccess) return IMP_OK;
    const imp_status s = e == cudaErrorMemoryAllocation ? IMP_ERR_NOMEM : IMP_ERR_CUDA;
    return fail(s, std::string(what) + ": " + cudaGetErrorString(e));
}

// Makes `ctx` current and clears its device error word.
imp_status begin(imp_context *ctx) {
    if (!ctx) return fail(IMP_ERR_INVALID_ARG, "null context");
    IMP_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
    // a call that failed part-way may have left work queued that reads the
    // staging arena this call is about to refill
    IMP_CUDA(cudaStreamSynchronize(ctx->stream), "stream synchronize");
    IMP_CUDA(cudaMemsetAsync(ctx->dev_err, 0, sizeof(unsigned), ctx->stream), "clear error word");
    ctx->launches = 0;
    return IMP_OK;
}

// Synchronizes and turns device error bits into a status.
imp_status finish(imp_context *ctx) {
    unsigned h = 0;
    IMP_CUDA(cudaMemcpyAsync(&h, ctx->dev_err, sizeof(unsigned), cudaMemcpyDeviceToHost,
                             ctx->stream),
             "read error word");
    IMP_CUDA(cudaStreamSynchronize(ctx->stream), "stream synchronize");
    if (h & imp::DEV_ERR_RANGE)
        return fail(IMP_ERR_RANGE,
                    "input outside the fixed-point phase range (|k| <= 32768 cycles/FOV, "
                    "|r| <= 2 FOV, |t| <= 16 s, |fm| <= 2 pi 8192 rad/s)");
    if (h & imp::DEV_ERR_TIMEOUT)
        return fail(IMP_ERR_TIMEOUT, "a bounded device-side wait expired");
    return IMP_OK;
}

namespace {
// One block whose bounded wait on an mbarrier that nothing ever arrives on
// runs out after `polls` rounds: it records DEV_ERR_TIMEOUT and returns.
__global__ void k_wait_expiry(unsigned *err, unsigned polls) {
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        fence_mbar_init();
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        bool done = false;
        for (unsigned it = 0; it < polls && !done; ++it) done = mbar_try_wait(&bar, 0);
        if (!done) atomicOr(err, DEV_ERR_TIMEOUT);
    }
}
}  // namespace

}  // namespace imp

using imp::begin;
using imp::fail;
using imp::finish;
using imp::from_cuda;

namespace {

imp_status scratch(imp_context *ctx, size_t bytes, void **p) {
    if (bytes > ctx->scratch_bytes) {
        if (ctx->scratch) cudaFree(ctx->scratch);
        ctx->scratch = nullptr;
        ctx->scratch_bytes = 0;
        IMP_CUDA(cudaMalloc(&ctx->scratch, bytes), "scratch allocation");
        ctx->scratch_bytes = bytes;
    }
    *p = ctx->scratch;
    return IMP_OK;
}

struct PlanGuard {
    imp::NuPlan p;
    ~PlanGuard() { imp::nu_plan_destroy(p); }
};

size_t align256(size_t b) { return (b + 255) / 256 * 256; }

imp_status check_op_args(const void *out_r, const void *out_i, const void *in_r,
                         const void *in_i, const void *kx, const void *ky, const void *ix,
                         const void *iy, const void *t, int num_k, int num_i, int use_z,
                         const void *kz, const void *iz) {
    if (!out_r || !out_i || !in_r || !in_i || !kx || !ky || !ix || !iy || !t)
        return fail(IMP_ERR_INVALID_ARG, "null array argument");
    if (use_z && (!kz || !iz)) return fail(IMP_ERR_INVALID_ARG, "use_z needs kz and iz");
    if (num_k <= 0 || num_i <= 0) return fail(IMP_ERR_INVALID_ARG, "num_k and num_i must be > 0");
    if (num_k > (1 << 30) || num_i > (1 << 30))
        return fail(IMP_ERR_INVALID_ARG, "num_k / num_i above 2^30");
    return IMP_OK;
}

imp_status run_forward(imp_context *ctx, float *yr, float *yi, const float *xr, const float *xi,
                       const float *kx, const float *ky, const float *kz, const float *ix,
                       const float *iy, const float *iz, const float *fm, const float *t,
                       int M, int N, const float *sr, const float *si, int C, int use_z) {
    imp_status s = check_op_args(yr, yi, xr, xi, kx, ky, ix, iy, t, M, N, use_z, kz, iz);
    if (s != IMP_OK) return s;
    if (C <= 0) return fail(IMP_ERR_INVALID_ARG, "num_coil must be > 0");
    if (C > 1 && (!sr || !si)) return fail(IMP_ERR_INVALID_ARG, "sensi needed for num_coil > 1");
    if ((s = begin(ctx)) != IMP_OK) return s;
    PlanGuard g;
    IMP_CUDA(imp::nu_plan_create(g.p, kx, ky, kz, t, ix, iy, iz, fm, sr, si, M, N, C,
                                 use_z != 0, ctx->dev_err, ctx->stream),
             "plan");
    imp::nu_tuned_lookup(g.p, false, &g.p.fwd);
    const size_t xs_b = align256(sizeof(float2) * (size_t)g.p.G * g.p.Npad * g.p.CG);
    const size_t pf_b = align256(imp::nu_fwd_partial_bytes(g.p, g.p.fwd));
    void *w = nullptr;
    if ((s = scratch(ctx, xs_b + pf_b, &w)) != IMP_OK) return s;
    float2 *xs = (float2 *)w;
    float2 *pf = (float2 *)((char *)w + xs_b);
    IMP_CUDA(imp::nu_pack_image_soa(g.p, xr, xi, xs, ctx->stream), "pack image");
    IMP_CUDA(imp::nu_forward_partials(g.p, g.p.fwd, xs, pf, ctx->dev_err, ctx->stream), "F");
    IMP_CUDA(imp::nu_forward_finish_soa(g.p, g.p.fwd, pf, yr, yi, ctx->stream), "F finish");
    ctx->launches = 6;
    return finish(ctx);
}

imp_status run_adjoint(imp_context *ctx, float *xr, float *xi, const float *dr, const float *di,
                       const float *kx, const float *ky, const float *kz, const float *ix,
                       const float *iy, const float *iz, const float *fm, const float *t,
                       int M, int N, const float *sr, const float *si, int C, int use_z) {
    imp_status s = check_op_args(xr, xi, dr, di, kx, ky, ix, iy, t, M, N, use_z, kz, iz);
    if (s != IMP_OK) return s;
    if (C <= 0) return fail(IMP_ERR_INVALID_ARG, "num_coil must be > 0");
    if (C > 1 && (!sr || !si)) return fail(IMP_ERR_INVALID_ARG, "sensi needed for num_coil > 1");
    if ((s = begin(ctx)) != IMP_OK) return s;
    PlanGuard g;
    IMP_CUDA(imp::nu_plan_create(g.p, kx, ky, kz, t, ix, iy, iz, fm, sr, si, M, N, C,
                                 use_z != 0, ctx->dev_err, ctx->stream),
             "plan");
    imp::nu_tuned_lookup(g.p, true, &g.p.adj);
    const size_t dp_b = align256(sizeof(float2) * (size_t)g.p.G * g.p.Mpad * g.p.CG);
    const size_t pa_b = align256(imp::nu_adj_partial_bytes(g.p, g.p.adj));
    void *w = nullptr;
    if ((s = scratch(ctx, dp_b + pa_b, &w)) != IMP_OK) return s;
    float2 *dp = (float2 *)w;
    float2 *pa = (float2 *)((char *)w + dp_b);
    IMP_CUDA(imp::nu_pack_kdata(g.p, dr, di, dp, ctx->stream), "pack kdata");
    IMP_CUDA(imp::nu_adjoint_partials(g.p, g.p.adj, dp, pa, ctx->dev_err, ctx->stream), "F^H");
    IMP_CUDA(imp::nu_adjoint_finish_soa(g.p, g.p.adj, pa, xr, xi, ctx->stream), "F^H finish");
    ctx->launches = 6;
    return finish(ctx);
}

// Host or device pointer -> device pointer (copies host data into `keep`).
}  // namespace

namespace imp {

static bool is_device_ptr(const void *p) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

imp_status to_device(imp_context *ctx, const float *p, size_t n, DevKeep &keep,
                     const float **out, bool *was_host) {
    *out = p;
    if (was_host) *was_host = false;
    if (!p || n == 0) return IMP_OK;
    if (is_device_ptr(p)) return IMP_OK;
    void *d = nullptr;
    IMP_CUDA(cudaMalloc(&d, n * sizeof(float)), "input staging");
    keep.emplace_back(d, [](void *q) { cudaFree(q); });
    IMP_CUDA(cudaMemcpyAsync(d, p, n * sizeof(float), cudaMemcpyHostToDevice, ctx->stream),
             "input H2D");
    *out = (const float *)d;
    if (was_host) *was_host = true;
    return IMP_OK;
}

void stage_reset(imp_context *ctx) {
    ctx->stage_chunk = 0;
    ctx->stage_off = 0;
}

static imp_status stage_alloc(imp_context *ctx, size_t bytes, void **out) {
    bytes = (bytes + 255) & ~(size_t)255;
    while (ctx->stage_chunk < ctx->stage.size()) {
        const auto &c = ctx->stage[ctx->stage_chunk];
        if (ctx->stage_off + bytes <= c.second) {
            *out = (char *)c.first + ctx->stage_off;
            ctx->stage_off += bytes;
            return IMP_OK;
        }
        ++ctx->stage_chunk;
        ctx->stage_off = 0;
    }
    const size_t cap = std::max(bytes, (size_t)64 << 20);
    void *d = nullptr;
    IMP_CUDA(cudaMalloc(&d, cap), "staging arena");
    ctx->stage.emplace_back(d, cap);
    ctx->stage_chunk = ctx->stage.size() - 1;
    ctx->stage_off = bytes;
    *out = d;
    return IMP_OK;
}

imp_status to_device_staged(imp_context *ctx, const float *p, size_t n, const float **out,
                            bool *was_host) {
    *out = p;
    if (was_host) *was_host = false;
    if (!p || n == 0) return IMP_OK;
    if (is_device_ptr(p)) return IMP_OK;
    void *d = nullptr;
    imp_status s = stage_alloc(ctx, n * sizeof(float), &d);
    if (s != IMP_OK) return s;
    IMP_CUDA(cudaMemcpyAsync(d, p, n * sizeof(float), cudaMemcpyHostToDevice, ctx->stream),
             "input H2D");
    *out = (const float *)d;
    if (was_host) *was_host = true;
    return IMP_OK;
}

imp_status out_device_staged(imp_context *ctx, float *p, size_t n, float **out, bool *was_host) {
    *out = p;
    *was_host = false;
    if (!p || n == 0) return IMP_OK;
    if (is_device_ptr(p)) return IMP_OK;
    void *d = nullptr;
    imp_status s = stage_alloc(ctx, n * sizeof(float), &d);
    if (s != IMP_OK) return s;
    *out = (float *)d;
    *was_host = true;
    return IMP_OK;
}

imp_status out_device(imp_context *ctx, float *p, size_t n, DevKeep &keep, float **out,
                      bool *was_host) {
    (void)ctx;
    *out = p;
    *was_host = false;
    if (!p || n == 0) return IMP_OK;
    if (is_device_ptr(p)) return IMP_OK;
    void *d = nullptr;
    IMP_CUDA(cudaMalloc(&d, n * sizeof(float)), "output staging");
    keep.emplace_back(d, [](void *q) { cudaFree(q); });
    *out = (float *)d;
    *was_host = true;
    return IMP_OK;
}

}  // namespace imp

using imp::stage_reset;
using imp::to_device;
using imp::to_device_staged;

extern "C" {

int imp_abi_version(void) { return 100; }

const char *imp_status_string(imp_status s) {
    switch (s) {
        case IMP_OK: return "ok";
        case IMP_ERR_INVALID_ARG: return "invalid argument";
        case IMP_ERR_CUDA: return "CUDA error";
        case IMP_ERR_IO: return "I/O error";
        case IMP_ERR_FORMAT: return "malformed input file";
        case IMP_ERR_RANGE: return "input out of range";
        case IMP_ERR_NOMEM: return "out of device memory";
        case IMP_ERR_TIMEOUT: return "device wait timed out";
        case IMP_ERR_UNSUPPORTED: return "unsupported option";
        default: return "unknown status";
    }
}

const char *imp_last_error(void) { return imp::g_last_error.c_str(); }

imp_status imp_context_create(int device, imp_context **out) {
    if (!out) return fail(IMP_ERR_INVALID_ARG, "null output pointer");
    *out = nullptr;
    int n = 0;
    IMP_CUDA(cudaGetDeviceCount(&n), "cudaGetDeviceCount");
    if (device < 0 || device >= n)
        return fail(IMP_ERR_INVALID_ARG, "device " + std::to_string(device) + " not present (" +
                                             std::to_string(n) + " visible)");
    IMP_CUDA(cudaSetDevice(device), "cudaSetDevice");
    std::unique_ptr<imp_context> c(new imp_context());
    c->device = device;
    // a blocking stream: it orders after work queued on the legacy default stream
    IMP_CUDA(cudaStreamCreateWithFlags(&c->stream, cudaStreamDefault), "stream");
    IMP_CUDA(cudaMalloc(&c->dev_err, sizeof(unsigned)), "error word");
    IMP_CUDA(cudaMemset(c->dev_err, 0, sizeof(unsigned)), "error word");
    *out = c.release();
    return IMP_OK;
}

imp_status imp_context_destroy(imp_context *ctx) {
    if (!ctx) return IMP_OK;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    ctx->bf.reset();
    ctx->bb.reset();
    ctx->tp.reset();
    ctx->tp_q.reset();
    for (auto &c : ctx->stage) cudaFree(c.first);
    ctx->stage.clear();
    if (ctx->scratch) cudaFree(ctx->scratch);
    if (ctx->dev_err) cudaFree(ctx->dev_err);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
    return IMP_OK;
}

imp_status imp_context_synchronize(imp_context *ctx) {
    if (!ctx) return fail(IMP_ERR_INVALID_ARG, "null context");
    IMP_CUDA(cudaStreamSynchronize(ctx->stream), "stream synchronize");
    return IMP_OK;
}

long imp_context_launch_count(const imp_context *ctx) { return ctx ? ctx->launches : 0; }

imp_status imp_ft(imp_context *ctx, float *kdata_r, float *kdata_i, const float *idata_r,
                  const float *idata_i, const float *kx, const float *ky, const float *kz,
                  const float *ix, const float *iy, const float *iz, const float *fm,
                  const float *t, int num_k, int num_i, int use_z) {
    return run_forward(ctx, kdata_r, kdata_i, idata_r, idata_i, kx, ky, kz, ix, iy, iz, fm, t,
                       num_k, num_i, nullptr, nullptr, 1, use_z);
}

imp_status imp_ift(imp_context *ctx, float *idata_r, float *idata_i, const float *kdata_r,
                   const float *kdata_i, const float *kx, const float *ky, const float *kz,
                   const float *ix, const float *iy, const float *iz, const float *fm,
                   const float *t, int num_k, int num_i, int use_z) {
    return run_adjoint(ctx, idata_r, idata_i, kdata_r, kdata_i, kx, ky, kz, ix, iy, iz, fm, t,
                       num_k, num_i, nullptr, nullptr, 1, use_z);
}

imp_status imp_parallel_ft(imp_context *ctx, float *kdata_r, float *kdata_i,
                           const float *idata_r, const float *idata_i, const float *kx,
                           const float *ky, const float *kz, const float *ix, const float *iy,
                           const float *iz, const float *fm, const float *t, int num_k,
                           int num_i, const float *sensi_r, const float *sensi_i, int num_coil,
                           int use_z) {
    return run_forward(ctx, kdata_r, kdata_i, idata_r, idata_i, kx, ky, kz, ix, iy, iz, fm, t,
                       num_k, num_i, sensi_r, sensi_i, num_coil, use_z);
}

imp_status imp_parallel_ift(imp_context *ctx, float *idata_r, float *idata_i,
                            const float *kdata_r, const float *kdata_i, const float *kx,
                            const float *ky, const float *kz, const float *ix, const float *iy,
                            const float *iz, const float *fm, const float *t, int num_k,
                            int num_i, const float *sensi_r, const float *sensi_i,
                            int num_coil, int use_z) {
    return run_adjoint(ctx, idata_r, idata_i, kdata_r, kdata_i, kx, ky, kz, ix, iy, iz, fm, t,
                       num_k, num_i, sensi_r, sensi_i, num_coil, use_z);
}

void imp_bf_options_default(imp_bf_options *opt) {
    if (!opt) return;
    std::memset(opt, 0, sizeof(*opt));
    opt->cg_num = 8;
    opt->tv_num = 10;
    opt->tv_eps = 1e-6f;
}

// BfConfig of one brute-force problem from the C options (TV grid as the
// reference: sqrt(N) x sqrt(N) unless nx, ny, nz are given).
static imp_status bf_config(const imp_bf_options *opt, int num_k, int num_i, int num_coil,
                     imp::BfConfig *cfg) {
    cfg->M = num_k;
    cfg->N = num_i;
    cfg->C = num_coil;
    cfg->use_z = opt->use_z != 0;
    cfg->cg_num = opt->cg_num;
    cfg->fd = opt->enable_fd != 0;
    cfg->lambda = opt->fd_penalizer;
    cfg->tv = opt->enable_tv != 0;
    cfg->tv_num = opt->enable_tv ? opt->tv_num : 1;
    cfg->tv_eps = opt->tv_eps;
    cfg->reg = nullptr;
    if (opt->reg) {
        const char *why = imp::sparse_reg_check(*opt->reg, num_i);
        if (why[0]) return fail(IMP_ERR_INVALID_ARG, std::string("-reg matrix: ") + why);
        cfg->reg = opt->reg;
    }
    if (opt->nx == 0 && opt->ny == 0 && opt->nz == 0) {
        // the reference's 2-D TV grid of side sqrt(N) (bruteForceGpu.cu:446-451)
        const int side = (int)std::lround(std::sqrt((double)num_i));
        if ((cfg->fd || cfg->tv) && side * side != num_i)
            return fail(IMP_ERR_INVALID_ARG, "TV on a sqrt(N) x sqrt(N) grid needs square N");
        cfg->n0 = side;
        cfg->n1 = side;
        cfg->n2 = 1;
        if (side * side != num_i) {
            cfg->n0 = num_i;
            cfg->n1 = 1;
        }
    } else {
        if (opt->nx <= 0 || opt->ny <= 0 || opt->nz <= 0 ||
            (long)opt->nx * opt->ny * opt->nz != num_i)
            return fail(IMP_ERR_INVALID_ARG, "nx*ny*nz must equal num_i");
        cfg->n0 = opt->ny;  // (y, x, z) with z fastest
        cfg->n1 = opt->nx;
        cfg->n2 = opt->nz;
    }
    return IMP_OK;
}

imp_status imp_bruteforce_recon(imp_context *ctx, const imp_bf_options *opt, float *idata_r,
                                float *idata_i, const float *kdata_r, const float *kdata_i,
                                const float *kx, const float *ky, const float *kz,
                                const float *ix, const float *iy, const float *iz,
                                const float *fm, const float *t, const float *sensi_r,
                                const float *sensi_i, int num_k, int num_i, int num_coil,
                                int num_slices) {
    if (!opt) return fail(IMP_ERR_INVALID_ARG, "null options");
    imp_status s = check_op_args(idata_r, idata_i, kdata_r, kdata_i, kx, ky, ix, iy, t, num_k,
                                 num_i, opt->use_z, kz, iz);
    if (s != IMP_OK) return s;
    if (num_coil <= 0 || num_slices <= 0)
        return fail(IMP_ERR_INVALID_ARG, "num_coil and num_slices must be > 0");
    if (num_coil > 1 && (!sensi_r || !sensi_i))
        return fail(IMP_ERR_INVALID_ARG, "sensi needed for num_coil > 1");
    if (opt->cg_num <= 0) return fail(IMP_ERR_INVALID_ARG, "cg_num must be > 0");
    if (opt->enable_tv && opt->tv_num <= 0) return fail(IMP_ERR_INVALID_ARG, "tv_num must be > 0");
    imp::BfConfig cfg;
    if ((s = bf_config(opt, num_k, num_i, num_coil, &cfg)) != IMP_OK) return s;
    if ((s = begin(ctx)) != IMP_OK) return s;
    const size_t M = num_k, N = num_i, C = num_coil, S = num_slices;
    const float *d_kx, *d_ky, *d_kz = nullptr, *d_ix, *d_iy, *d_iz = nullptr, *d_t, *d_fm = nullptr;
    const float *d_sr = nullptr, *d_si = nullptr, *d_kr, *d_ki, *d_xr0, *d_xi0;
    bool x_host = false, dummy;
    stage_reset(ctx);
    if ((s = to_device_staged(ctx, kx, M, &d_kx, &dummy)) ||
        (s = to_device_staged(ctx, ky, M, &d_ky, &dummy)) ||
        (s = to_device_staged(ctx, kz, M, &d_kz, &dummy)) ||
        (s = to_device_staged(ctx, t, M, &d_t, &dummy)) ||
        (s = to_device_staged(ctx, ix, N, &d_ix, &dummy)) ||
        (s = to_device_staged(ctx, iy, N, &d_iy, &dummy)) ||
        (s = to_device_staged(ctx, iz, N, &d_iz, &dummy)) ||
        (s = to_device_staged(ctx, fm, S * N, &d_fm, &dummy)) ||
        (s = to_device_staged(ctx, sensi_r, C * N, &d_sr, &dummy)) ||
        (s = to_device_staged(ctx, sensi_i, C * N, &d_si, &dummy)) ||
        (s = to_device_staged(ctx, kdata_r, S * C * M, &d_kr, &dummy)) ||
        (s = to_device_staged(ctx, kdata_i, S * C * M, &d_ki, &dummy)) ||
        (s = to_device_staged(ctx, idata_r, S * N, &d_xr0, &x_host)) ||
        (s = to_device_staged(ctx, idata_i, S * N, &d_xi0, &dummy)))
        return s;
    float *d_xr = const_cast<float *>(d_xr0), *d_xi = const_cast<float *>(d_xi0);
    if (num_coil == 1) {
        d_sr = nullptr;  // one coil: unit sensitivity (kernels/structures.cpp:710-716)
        d_si = nullptr;
    }
    // the context keeps one solver: buffers, tuned shapes and CUDA graphs are
    // reused by later calls of the same problem size
    if (!ctx->bf) ctx->bf.reset(new imp::BfSolver());
    imp::BfSolver &solver = *ctx->bf;
    IMP_CUDA(solver.setup(cfg, d_kx, d_ky, d_kz, d_t, d_ix, d_iy, d_iz, d_sr, d_si, ctx->dev_err,
                          ctx->stream),
             "brute-force setup");
    solver.set_profiling(ctx->prof_on);
    long launches = 4;
    for (int sl = 0; sl < num_slices; ++sl) {
        IMP_CUDA(solver.solve(d_fm ? d_fm + (size_t)sl * N : nullptr, d_kr + (size_t)sl * C * M,
                              d_ki + (size_t)sl * C * M, d_xr + (size_t)sl * N,
                              d_xi + (size_t)sl * N),
                 "brute-force solve");
        launches += solver.launches();
    }
    if (x_host) {
        IMP_CUDA(cudaMemcpyAsync(idata_r, d_xr, S * N * sizeof(float), cudaMemcpyDeviceToHost,
                                 ctx->stream),
                 "output D2H");
        IMP_CUDA(cudaMemcpyAsync(idata_i, d_xi, S * N * sizeof(float), cudaMemcpyDeviceToHost,
                                 ctx->stream),
                 "output D2H");
    }
    s = finish(ctx);
    ctx->launches = launches;
    if (s == IMP_OK && ctx->prof_on)
        IMP_CUDA(solver.profile_collect(ctx->prof_ms, ctx->prof_count), "profile collect");
    return s;
}

imp_status imp_bruteforce_batch(imp_context *ctx, const imp_bf_options *opt, float *idata_r,
                                float *idata_i, const float *kdata_r, const float *kdata_i,
                                const float *kx, const float *ky, const float *kz,
                                const float *t, const int *k_off, const float *ix,
                                const float *iy, const float *iz, const float *fm,
                                const float *sensi_r, const float *sensi_i, int num_i,
                                int num_coil, int num_slices) {
    if (!opt || !k_off) return fail(IMP_ERR_INVALID_ARG, "null options or offsets");
    if (num_slices <= 0 || num_coil <= 0 || num_i <= 0)
        return fail(IMP_ERR_INVALID_ARG, "num_slices, num_coil and num_i must be > 0");
    if (k_off[0] != 0) return fail(IMP_ERR_INVALID_ARG, "k_off[0] must be 0");
    for (int sl = 0; sl < num_slices; ++sl)
        if (k_off[sl + 1] <= k_off[sl])
            return fail(IMP_ERR_INVALID_ARG, "every slice needs at least one sample");
    const size_t Mt = (size_t)k_off[num_slices];
    imp_status s = check_op_args(idata_r, idata_i, kdata_r, kdata_i, kx, ky, ix, iy, t,
                                 (int)std::min<size_t>(Mt, INT32_MAX), num_i, opt->use_z, kz, iz);
    if (s != IMP_OK) return s;
    if (num_coil > 1 && (!sensi_r || !sensi_i))
        return fail(IMP_ERR_INVALID_ARG, "sensi needed for num_coil > 1");
    if (opt->cg_num <= 0) return fail(IMP_ERR_INVALID_ARG, "cg_num must be > 0");
    if (opt->enable_tv && opt->tv_num <= 0) return fail(IMP_ERR_INVALID_ARG, "tv_num must be > 0");
    if ((s = begin(ctx)) != IMP_OK) return s;
    const size_t N = num_i, C = num_coil, S = num_slices;
    const float *d_kx, *d_ky, *d_kz = nullptr, *d_ix, *d_iy, *d_iz = nullptr, *d_t, *d_fm = nullptr;
    const float *d_sr = nullptr, *d_si = nullptr, *d_kr, *d_ki, *d_xr0, *d_xi0;
    bool x_host = false, dummy;
    stage_reset(ctx);
    if ((s = to_device_staged(ctx, kx, Mt, &d_kx, &dummy)) ||
        (s = to_device_staged(ctx, ky, Mt, &d_ky, &dummy)) ||
        (s = to_device_staged(ctx, kz, Mt, &d_kz, &dummy)) ||
        (s = to_device_staged(ctx, t, Mt, &d_t, &dummy)) ||
        (s = to_device_staged(ctx, ix, N, &d_ix, &dummy)) ||
        (s = to_device_staged(ctx, iy, N, &d_iy, &dummy)) ||
        (s = to_device_staged(ctx, iz, N, &d_iz, &dummy)) ||
        (s = to_device_staged(ctx, fm, S * N, &d_fm, &dummy)) ||
        (s = to_device_staged(ctx, sensi_r, C * N, &d_sr, &dummy)) ||
        (s = to_device_staged(ctx, sensi_i, C * N, &d_si, &dummy)) ||
        (s = to_device_staged(ctx, kdata_r, C * Mt, &d_kr, &dummy)) ||
        (s = to_device_staged(ctx, kdata_i, C * Mt, &d_ki, &dummy)) ||
        (s = to_device_staged(ctx, idata_r, S * N, &d_xr0, &x_host)) ||
        (s = to_device_staged(ctx, idata_i, S * N, &d_xi0, &dummy)))
        return s;
    float *d_xr = const_cast<float *>(d_xr0), *d_xi = const_cast<float *>(d_xi0);
    if (num_coil == 1) {
        d_sr = nullptr;  // one coil: unit sensitivity (kernels/structures.cpp:710-716)
        d_si = nullptr;
    }
    // all slices in lockstep: every CG step is one launch over all slices
    imp::BfConfig cfg;
    if ((s = bf_config(opt, k_off[1] - k_off[0], num_i, num_coil, &cfg)) != IMP_OK) return s;
    if (cfg.reg)
        return fail(IMP_ERR_UNSUPPORTED, "-reg is not available in the batched multi-slice "
                                         "solver; reconstruct the slices with "
                                         "imp_bruteforce_recon");
    if (!ctx->bb) ctx->bb.reset(new imp::BfBatch());
    IMP_CUDA(ctx->bb->setup(cfg, num_slices, k_off, d_kx, d_ky, d_kz, d_t, d_ix, d_iy, d_iz, d_fm,
                            d_sr, d_si, ctx->dev_err, ctx->stream),
             "batched brute-force setup");
    IMP_CUDA(ctx->bb->solve(d_kr, d_ki, d_xr, d_xi), "batched brute-force solve");
    const long launches = ctx->bb->launches();
    if (x_host) {
        IMP_CUDA(cudaMemcpyAsync(idata_r, d_xr, S * N * sizeof(float), cudaMemcpyDeviceToHost,
                                 ctx->stream),
                 "output D2H");
        IMP_CUDA(cudaMemcpyAsync(idata_i, d_xi, S * N * sizeof(float), cudaMemcpyDeviceToHost,
                                 ctx->stream),
                 "output D2H");
    }
    s = finish(ctx);
    ctx->launches = launches;
    return s;
}

imp_status imp_check_wait_expiry(imp_context *ctx, int polls) {
    if (!ctx || polls <= 0) return fail(IMP_ERR_INVALID_ARG, "null context or polls <= 0");
    imp_status s = begin(ctx);
    if (s != IMP_OK) return s;
    imp::k_wait_expiry<<<1, 32, 0, ctx->stream>>>(ctx->dev_err, (unsigned)polls);
    IMP_CUDA(cudaGetLastError(), "wait-expiry kernel");
    ctx->launches = 1;
    return finish(ctx);  // IMP_ERR_TIMEOUT, read from the device error word
}

imp_status imp_context_profile(imp_context *ctx, int enable) {
    if (!ctx) return fail(IMP_ERR_INVALID_ARG, "null context");
    ctx->prof_on = enable != 0;
    ctx->prof_ms[0] = ctx->prof_ms[1] = 0.0;
    ctx->prof_count[0] = ctx->prof_count[1] = 0;
    return IMP_OK;
}

imp_status imp_context_profile_read(const imp_context *ctx, int which, double *total_ms,
                                    long *count) {
    if (!ctx || which < 0 || which > 1 || !total_ms || !count)
        return fail(IMP_ERR_INVALID_ARG, "bad profile query");
    *total_ms = ctx->prof_ms[which];
    *count = ctx->prof_count[which];
    return IMP_OK;
}

}  // extern "C"

// Internal interface of the brute-force CG solver on the NUDFT tile engine.
#pragma once
#include <cuda_runtime.h>
#include <vector>
#include "nudft.cuh"
#include "sparse_reg.cuh"

namespace imp {

struct BfConfig {
    int M = 0, N = 0, C = 1;
    int n0 = 0, n1 = 0, n2 = 1;  // TV grid (row-major, n2 fastest); n0*n1*n2 == N
    bool use_z = false;
    int cg_num = 8;              // the reference performs cg_num-1 updates
    bool fd = false;             // finite-difference (TV) regularizer on
    float lambda = 0.f;          // fd_penalizer
    bool tv = false;             // TV reweighting outer loop
    int tv_num = 1;
    float tv_eps = 1e-6f;        // MRI_SMOOTH_FACTOR (FP32 build)
    bool use_graphs = true;
    bool autotune = true;        // time launch shapes once per problem shape
    const imp_sparse *reg = nullptr;  // -reg roughness matrix (host COO), null = off
};

class BfSolver {
public:
    BfSolver() = default;
    ~BfSolver();
    BfSolver(const BfSolver &) = delete;
    BfSolver &operator=(const BfSolver &) = delete;

    // Geometry shared by every slice (device SoA pointers, float32).
    cudaError_t setup(const BfConfig &cfg, const float *kx, const float *ky, const float *kz,
                      const float *t, const float *ix, const float *iy, const float *iz,
                      const float *sensi_r, const float *sensi_i, unsigned *dev_err,
                      cudaStream_t st);
    // One slice: fm [N], kdata [C][M] SoA, x [N] SoA in/out (initial estimate -> result).
    cudaError_t solve(const float *fm, const float *kd_r, const float *kd_i, float *x_r,
                      float *x_i);

    // Launch counts of the most recent solve (kernels of this library).
    long launches() const { return launches_; }
    NuPlan &plan() { return plan_; }
    void release();

    // Kernel timing: when on, graphs are not used and every NUDFT launch is
    // bracketed by CUDA events on the launching stream.
    void set_profiling(bool on) { prof_on_ = on; }
    // After the stream is synchronized: summed milliseconds and launch counts
    // of the forward (index 0) and adjoint (index 1) NUDFT kernels since the
    // last collect.
    cudaError_t profile_collect(double ms[2], long count[2]);

private:
    cudaError_t run_iteration();
    cudaError_t run_init();
    cudaError_t prof_mark(int kind);

    bool prof_on_ = false;
    std::vector<cudaEvent_t> prof_ev_;
    std::vector<int> prof_kind_;
    size_t prof_used_ = 0;

    cudaError_t set_reg(bool *graphs_stale);

    BfConfig cfg_;
    NuPlan plan_;
    SparseReg reg_;           // -reg: C and C^T on the device
    cudaStream_t st_ = nullptr;
    unsigned *err_ = nullptr;
    float2 *y_ = nullptr, *af_ = nullptr, *q_ = nullptr, *rpk_ = nullptr, *xs_ = nullptr;
    float2 *x_ = nullptr, *g_ = nullptr, *d_ = nullptr;
    float *w_ = nullptr;
    float2 *pf_ = nullptr, *pa_ = nullptr;
    double *dots_ = nullptr;  // [4][kDotBlocks] gg, dg, qq, sd; then oldin
    cudaGraphExec_t g_iter_ = nullptr, g_init_ = nullptr;
    long launches_ = 0;
    int per_iter_launches_ = 0, per_init_launches_ = 0;
};

constexpr int kDotBlocks = 296;  // 2 x 148 SMs, grid-stride

// S independent slices sharing the image grid, the coil maps and the options,
// each with its own trajectory (uneven sample counts), field map and data,
// solved in lockstep (every slice runs the same cg_num / tv_num): each CG step
// is ONE launch over all slices -- the batched NUDFT (blockIdx.z = slice x
// coil group, per-slice offsets from a device table) or a vector kernel with
// blockIdx.y = slice -- and every slice keeps its own FP64 scalars.  The
// initialisation and the CG update are captured once as CUDA graphs.
class BfBatch {
public:
    BfBatch() = default;
    ~BfBatch();
    BfBatch(const BfBatch &) = delete;
    BfBatch &operator=(const BfBatch &) = delete;

    // cfg.M is ignored.  Slice s owns samples k_off[s] .. k_off[s+1]-1 (host
    // array) of the device SoA trajectory arrays; fm: [S][N] (or null).
    cudaError_t setup(const BfConfig &cfg, int S, const int *k_off, const float *kx,
                      const float *ky, const float *kz, const float *t, const float *ix,
                      const float *iy, const float *iz, const float *fm, const float *sensi_r,
                      const float *sensi_i, unsigned *dev_err, cudaStream_t st);
    // kdata: slice s's [C][M_s] block at C * k_off[s]; x: [S][N] SoA in/out.
    cudaError_t solve(const float *kd_r, const float *kd_i, float *x_r, float *x_i);

    long launches() const { return launches_; }
    int slices() const { return S_; }
    void release();

private:
    cudaError_t run_init();
    cudaError_t run_iteration();
    cudaError_t set_table(bool adj, int split);
    cudaError_t tune_shapes(bool adj);

    BfConfig cfg_;
    NuPlan plan_;          // C, CG, G, Npad, use_z and the shared sensitivities
    NuLaunch fwd_, adj_;   // one launch shape for all slices
    int S_ = 0, kb_ = 1;   // slices; vector-kernel blocks per slice
    int max_mpad_ = 0;
    long long mpad_total_ = 0;  // sum of the slices' padded sample counts
    std::vector<int> k_off_, m_, mpad_;
    std::vector<long long> koff_pad_;
    cudaStream_t st_ = nullptr;
    unsigned *err_ = nullptr;
    double4 *kgeo_ = nullptr, *vgeo_ = nullptr;
    float2 *sens_ = nullptr;
    NuSlice *tab_fwd_ = nullptr, *tab_adj_ = nullptr;
    void *tab_vec_ = nullptr;  // per-slice (padded offset, M, Mpad) of the vector kernels
    float2 *y_ = nullptr, *af_ = nullptr, *q_ = nullptr, *rpk_ = nullptr, *xs_ = nullptr;
    float2 *x_ = nullptr, *g_ = nullptr, *d_ = nullptr;
    float *w_ = nullptr;
    float2 *pf_ = nullptr, *pa_ = nullptr;
    double *dots_ = nullptr;  // [S][5][kb_]
    cudaGraphExec_t g_iter_ = nullptr, g_init_ = nullptr;
    long launches_ = 0;
    int per_iter_launches_ = 0, per_init_launches_ = 0;
};

}  // namespace imp

// Internal interface of the brute-force CG solver on the NUDFT tile engine.
#pragma once
#include <cuda_runtime.h>
#include <vector>
#include "nudft.cuh"

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

    BfConfig cfg_;
    NuPlan plan_;
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

}  // namespace imp

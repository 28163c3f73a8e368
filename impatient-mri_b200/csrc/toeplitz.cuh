// Internal interface of the Toeplitz path: Kaiser-Bessel gridding of Q and
// F^H d, the FFT-based F^H F with time segmentation and SENSE, and the
// Toeplitz CG (toeplitz/computeQ.cmem.cu, toeplitz/computeFH.cmem.cu,
// toeplitz/recon.cu).
#pragma once
#include <cuda_runtime.h>
#include <vector>

#include "grid_fft.cuh"
#include "sparse_reg.cuh"
#include "toep_fft.cuh"

namespace imp {

// One gridding problem: image size and grid size in gridding axis order
// (x, y, z), oversampling and KB shape (toeplitz/computeQ.cmem.cu:439-486).
struct GridSpec {
    int img[3] = {1, 1, 1};
    int gs[3] = {1, 1, 1};
    float os = 1.f;
    float beta = 0.f;
    float kscale = 1.f;  // 2 for Q (samples at 2k), 1 for F^H d
    bool is3d = false;
    size_t cells() const { return (size_t)gs[0] * gs[1] * gs[2]; }
};

// Q: beta after the oversampling rounding; F^H d: before (as the reference).
GridSpec grid_spec(const int img_xyz[3], float os_requested, bool beta_after_rounding,
                   float kscale);

struct ToepConfig {
    int nx = 0, ny = 0, nz = 1;  // image; nz == 1 is 2-D
    int C = 1;                   // coils
    int M = 0;                   // samples per coil
    float ntime_segs = 0.f;      // L: segments l = 0..(int)L
    float os_q = 1.125f, os_fh = 1.5f;
    int cg_num = 8;
    bool fd = false;
    float lambda = 0.f;
    bool tv = false;
    int tv_num = 1;
    float tv_eps = 1e-6f;
    bool use_graphs = true;
    const imp_sparse *reg = nullptr;  // -reg roughness matrix (host COO), null = off
};

class ToepSolver {
public:
    ToepSolver() = default;
    ~ToepSolver();
    ToepSolver(const ToepSolver &) = delete;
    ToepSolver &operator=(const ToepSolver &) = delete;

    // Sizes and per-voxel inputs (device pointers, float32 SoA).
    // fm: [N] rad/s (may be null); sensi: [C][N] (null with C == 1); t: [M].
    cudaError_t setup(const ToepConfig &cfg, const float *t, const float *fm,
                      const float *sensi_r, const float *sensi_i, unsigned *dev_err,
                      cudaStream_t st);
    // Q_l by gridding (kx, ky, kz device [M]); q_out (optional, device) gets
    // Q in the reference layout [(L+1)][2N grid] as split re/im.
    cudaError_t compute_q(const float *kx, const float *ky, const float *kz, float *q_out_r,
                          float *q_out_i);
    // Q_l given (reference layout, split re/im, device).
    cudaError_t load_q(const float *q_r, const float *q_i);
    // F^H d by gridding with time segmentation and SENSE; kdata [C][M].
    cudaError_t compute_fhd(const float *kx, const float *ky, const float *kz,
                            const float *kd_r, const float *kd_i, float *fhd_r, float *fhd_i);
    // Toeplitz CG from x = 0; fhd (device SoA [N]); result = best-residual iterate.
    cudaError_t solve(const float *fhd_r, const float *fhd_i, float *x_r, float *x_i);
    // CG from x (device SoA, in: x0, out: minimum-residual iterate) until
    // sqrt(|r|^2/|F^H d|^2) < tol or max_iter updates; no TV passes.
    cudaError_t solve_from(const float *fhd_r, const float *fhd_i, float *x_r, float *x_i,
                           double tol, int max_iter, int *iters);
    // One application of A^H A (+ lambda D^H W D with W = 1) for tests.
    cudaError_t apply(const float *p_r, const float *p_i, float *q_r, float *q_i);

    long launches() const { return launches_; }
    int segments() const { return L_ + 1; }
    size_t q_elems() const { return G2_; }
    size_t voxels() const { return N_; }
    void release();

private:
    cudaError_t apply_aha(const float2 *p, float2 *q);  // q = A^H A p (no TV term)
    // q += lambda (D^H W D | C^T W C) p (when a penalty is on); partial Re<p, q>
    cudaError_t penalty_dot(float2 *q, const float2 *p);
    const int *done_flag() const;
    cudaError_t set_reg();
    cudaError_t cg_iteration();
    cudaError_t ensure_grid_plan(const GridSpec &g, GridFft *plan);

    ToepConfig cfg_;
    SparseReg reg_;            // -reg: C and C^T on the device
    cudaStream_t st_ = nullptr;
    unsigned *err_ = nullptr;
    int L_ = 0;
    float tau_ = 0.f, t0_ = 0.f;
    size_t N_ = 0, G2_ = 0;
    int n2[3] = {1, 1, 1};   // 2N grid in FFT / voxel axis order
    int nv[3] = {1, 1, 1};   // image in voxel axis order
    // resident state
    float2 *sens_ = nullptr;   // [C][N]
    float2 *eph_ = nullptr;    // [(L+1)][N] exp(-i fm (tau l + t0))
    float *fm_ = nullptr;      // [N]
    float2 *qf_ = nullptr;     // [(L+1)][G2] (one segment of scratch with the engine)
    float2 *big_ = nullptr;    // [C][G2] zero-padded chain (sizes the engine does not take)
    float2 *x_ = nullptr, *r_ = nullptr, *p_ = nullptr, *q_ = nullptr, *best_ = nullptr;
    float2 *fhd_ = nullptr;
    float *w_ = nullptr;
    double *dots_ = nullptr;   // block partials + scalars
    float *t_ = nullptr;       // copy of t [M]
    GridFft gf2_;              // 2N grid, batch C (zero-padded chain)
    GridFft gf1_;              // 2N grid, one transform (Qf_l)
    GridFft gfq_, gff_;        // gridding grids of Q and F^H d
    float2 *grid_ = nullptr;   // gridding scratch
    size_t grid_cells_ = 0;
    cudaGraphExec_t g_iter_ = nullptr;
    long launches_ = 0;
    // pruned FFT engine (power-of-two sizes); the zero-padded chain otherwise
    bool fast_ = false;
    ToepFftPlan fp_;
    float2 *qf2_ = nullptr;    // [(L+1)][G2] Qf_l in parity-major order, scaled 1/G2
    float2 *b1_ = nullptr;     // [C][half spectrum] engine scratch
    float2 *tw_ = nullptr;     // twiddle table
};

}  // namespace imp

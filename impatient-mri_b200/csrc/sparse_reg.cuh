// Roughness regularization with a sparse matrix (-reg): the penalty term
//   lambda C^T (W (C x))
// of the reference's brute-force and Toeplitz CG (bruteForce/bruteForceCpu.cpp:
// 306-380, toeplitz/recon.cu:1543-1673), C real with rows = B * N (B blocks of
// N rows, one per difference direction) and N columns, W the per-voxel TV
// weight applied to every block (row k weighted by w[k mod N]).
//
// Both C and C^T are kept on the device in CSR form (built once on the host
// from the coordinate form).  One kernel forms y = W (C x) over the B N rows;
// the consumers (the CG's gradient and step-length kernels) evaluate
// (C^T y)_r for their own voxel r with reg_ct_at, fused as the finite-
// difference stencil is.
#pragma once
#include "../../include/impatient_b200.h"

#include <cuda_runtime.h>
#include <vector>

namespace imp {

// What a kernel needs to evaluate (C^T y)_r.
struct RegView {
    const int *ptr = nullptr;    // [N + 1] CSR of C^T
    const int *col = nullptr;    // [nnz]
    const float *val = nullptr;  // [nnz]
    const float2 *y = nullptr;   // [rows] W (C x)
};

__device__ __forceinline__ float2 reg_ct_at(const RegView &v, int r) {
    float2 acc = make_float2(0.f, 0.f);
    for (int k = v.ptr[r]; k < v.ptr[r + 1]; ++k) {
        const float c = v.val[k];
        const float2 y = v.y[v.col[k]];
        acc.x = fmaf(c, y.x, acc.x);
        acc.y = fmaf(c, y.y, acc.y);
    }
    return acc;
}

class SparseReg {
public:
    ~SparseReg() { release(); }
    // Uploads C (rows = B * n, cols = n) and its transpose.  Keeps the device
    // buffers when the sizes match the previous matrix (so captured graphs
    // that read them stay valid); `reallocated` reports whether they moved.
    cudaError_t set(const imp_sparse &c, int n, cudaStream_t st, bool *reallocated);
    // y = W (C x) (w = nullptr: W = 1); returns at once when *done != 0.
    cudaError_t apply_cw(const float2 *x, const float *w, const int *done, cudaStream_t st);
    RegView view() const { return RegView{t_ptr_, t_col_, t_val_, y_}; }
    bool on() const { return rows_ > 0; }
    void release();

private:
    int rows_ = 0, n_ = 0, nnz_ = 0;
    int *c_ptr_ = nullptr, *c_col_ = nullptr;
    float *c_val_ = nullptr;
    int *t_ptr_ = nullptr, *t_col_ = nullptr;
    float *t_val_ = nullptr;
    float2 *y_ = nullptr;
    std::vector<int> hbuf_i_;
    std::vector<float> hbuf_f_;
};

// Checks a matrix for -reg against an image of n voxels: rows a positive
// multiple of n, cols == n, every index in range.  Returns an empty string
// when it is usable, else the reason.
const char *sparse_reg_check(const imp_sparse &c, int n);

}  // namespace imp

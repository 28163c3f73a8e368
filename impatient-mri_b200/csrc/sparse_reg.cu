// Sparse roughness regularization (see sparse_reg.cuh).
#include "sparse_reg.cuh"

#include <algorithm>
#include <cstring>

namespace imp {

namespace {

constexpr int kRegThreads = 256;

// y[k] = w[k mod n] sum_j C[k][j] x[j]   (one thread per row of C)
__global__ void k_reg_cw(float2 *__restrict__ y, const int *__restrict__ ptr,
                         const int *__restrict__ col, const float *__restrict__ val,
                         const float2 *__restrict__ x, const float *__restrict__ w, int rows, int n,
                         const int *__restrict__ done) {
    if (done && *done) return;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < rows; k += gridDim.x * blockDim.x) {
        float2 acc = make_float2(0.f, 0.f);
        for (int e = ptr[k]; e < ptr[k + 1]; ++e) {
            const float c = val[e];
            const float2 v = x[col[e]];
            acc.x = fmaf(c, v.x, acc.x);
            acc.y = fmaf(c, v.y, acc.y);
        }
        const float s = w ? w[k % n] : 1.f;
        y[k] = make_float2(acc.x * s, acc.y * s);
    }
}

// CSR of a coordinate matrix with `nr` rows; entries of a row keep their
// order in the coordinate list (the reference's COO loops add in list order).
void coo_to_csr(int nr, int nnz, const int *ri, const int *ci, const float *v, int *ptr, int *col,
                float *val) {
    std::fill(ptr, ptr + nr + 1, 0);
    for (int e = 0; e < nnz; ++e) ++ptr[ri[e] + 1];
    for (int r = 0; r < nr; ++r) ptr[r + 1] += ptr[r];
    std::vector<int> fill(ptr, ptr + nr);
    for (int e = 0; e < nnz; ++e) {
        const int d = fill[ri[e]]++;
        col[d] = ci[e];
        val[d] = v[e];
    }
}

}  // namespace

const char *sparse_reg_check(const imp_sparse &c, int n) {
    if (n <= 0) return "empty image";
    if (c.nnz < 0 || (c.nnz > 0 && (!c.row || !c.col || !c.val)))
        return "null index or value array";
    if (c.cols != n) return "matrix columns differ from the number of voxels";
    if (c.rows <= 0 || c.rows % n) return "matrix rows are not a positive multiple of the voxels";
    for (int e = 0; e < c.nnz; ++e)
        if (c.row[e] < 0 || c.row[e] >= c.rows || c.col[e] < 0 || c.col[e] >= c.cols)
            return "matrix index out of range";
    return "";
}

void SparseReg::release() {
    for (void *p : {(void *)c_ptr_, (void *)c_col_, (void *)c_val_, (void *)t_ptr_,
                    (void *)t_col_, (void *)t_val_, (void *)y_})
        if (p) cudaFree(p);
    c_ptr_ = c_col_ = t_ptr_ = t_col_ = nullptr;
    c_val_ = t_val_ = nullptr;
    y_ = nullptr;
    rows_ = n_ = nnz_ = 0;
}

cudaError_t SparseReg::set(const imp_sparse &c, int n, cudaStream_t st, bool *reallocated) {
    const bool same = rows_ == c.rows && n_ == n && nnz_ == c.nnz && y_;
    *reallocated = !same;
    if (!same) {
        release();
        const size_t nz = (size_t)std::max(c.nnz, 1);
        cudaError_t e;
        if ((e = cudaMalloc(&c_ptr_, sizeof(int) * (c.rows + 1))) ||
            (e = cudaMalloc(&c_col_, sizeof(int) * nz)) ||
            (e = cudaMalloc(&c_val_, sizeof(float) * nz)) ||
            (e = cudaMalloc(&t_ptr_, sizeof(int) * (n + 1))) ||
            (e = cudaMalloc(&t_col_, sizeof(int) * nz)) ||
            (e = cudaMalloc(&t_val_, sizeof(float) * nz)) ||
            (e = cudaMalloc(&y_, sizeof(float2) * c.rows))) {
            release();
            return e;
        }
        rows_ = c.rows;
        n_ = n;
        nnz_ = c.nnz;
    }
    // host staging: [c_ptr | c_col | t_ptr | t_col] and [c_val | t_val]
    const size_t nz = (size_t)c.nnz;
    hbuf_i_.assign((size_t)(c.rows + 1) + nz + (size_t)(n + 1) + nz, 0);
    hbuf_f_.assign(2 * nz, 0.f);
    int *cp = hbuf_i_.data(), *cc = cp + c.rows + 1, *tp = cc + nz, *tc = tp + n + 1;
    float *cv = hbuf_f_.data(), *tv = cv + nz;
    coo_to_csr(c.rows, c.nnz, c.row, c.col, c.val, cp, cc, cv);
    coo_to_csr(n, c.nnz, c.col, c.row, c.val, tp, tc, tv);
    cudaError_t e;
    if ((e = cudaMemcpyAsync(c_ptr_, cp, sizeof(int) * (c.rows + 1), cudaMemcpyHostToDevice, st)) ||
        (e = cudaMemcpyAsync(t_ptr_, tp, sizeof(int) * (n + 1), cudaMemcpyHostToDevice, st)))
        return e;
    if (nz) {
        if ((e = cudaMemcpyAsync(c_col_, cc, sizeof(int) * nz, cudaMemcpyHostToDevice, st)) ||
            (e = cudaMemcpyAsync(c_val_, cv, sizeof(float) * nz, cudaMemcpyHostToDevice, st)) ||
            (e = cudaMemcpyAsync(t_col_, tc, sizeof(int) * nz, cudaMemcpyHostToDevice, st)) ||
            (e = cudaMemcpyAsync(t_val_, tv, sizeof(float) * nz, cudaMemcpyHostToDevice, st)))
            return e;
    }
    // the host staging buffers must outlive the copies
    return cudaStreamSynchronize(st);
}

cudaError_t SparseReg::apply_cw(const float2 *x, const float *w, const int *done,
                                cudaStream_t st) {
    const int blocks = std::max(1, std::min((rows_ + kRegThreads - 1) / kRegThreads, 148 * 8));
    k_reg_cw<<<blocks, kRegThreads, 0, st>>>(y_, c_ptr_, c_col_, c_val_, x, w, rows_, n_, done);
    return cudaGetLastError();
}

}  // namespace imp

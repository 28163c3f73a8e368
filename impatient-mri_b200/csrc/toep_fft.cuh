// Pruned, fused FFT engine for the Toeplitz F^H F (one time segment, all coils).
//
// F^H F_l p = crop(IFFT(Qf_l . FFT(zeropad(S_c e_l p)))) / G on the 2N grid
// (toeplitz/recon.cu:1113-1202, 1370-1465).  The zero padding is never
// stored: along an axis of image length n, a 2n-point FFT whose input is zero
// on [n, 2n) splits by output parity a into two n-point FFTs,
//     X[2k + a] = FFT_n(x[j] w_2n^{a j})[k],
// and the inverse restricted to outputs [0, n) is
//     y[j] = sum_a w_2n^{-a j} IFFT_n(Y[2k + a])[j].
// Every transform here is an n-point FFT on image-sized data; the spectrum is
// kept in parity-major order and Qf_l is permuted (and scaled by 1/G) to match.
//
// Axes (voxel order): slow s, middle m, fast f.  3-D [y][x][z]: s = y, m = x,
// f = z.  2-D [x][y]: s = x, m absent (length 1, not doubled), f = y.
// Three kernels per segment:
//   k_fwd_plane  per s-plane (and coil): pad + parity twiddles + 2-D FFT (m, f)
//   k_slow       per spectrum column: FFT along s, x Qf_l, inverse along s
//   k_inv_plane  per s-plane: inverse 2-D FFT, parity recombination, coil sum
//                with conj(S_c), conj(e_l), accumulation over segments
#pragma once
#include <cuda_runtime.h>
#include <cstddef>

namespace imp {

struct ToepFftPlan {
    int ns = 0, nm = 1, nf = 0;  // image lengths along s, m, f (powers of two)
    int qm = 1;                  // m parities (2 in 3-D, 1 in 2-D)
    int C = 1;                   // coils
    int ps = 1;                  // s-planes per plane-kernel block
    int sk = 0;                  // 2-D rows of nf > 32 stored skewed (one pad per r1 slots)
    int rs = 0;                  // padded shared-memory row stride (nf + sk nf / r1 + 1)
    int vpt = 1;                 // image elements per thread in the plane kernels
    int ncol = 0;                // spectrum columns per s: qm * 2 * nm * nf
    int W = 1;                   // columns per k_slow block
    int csize = 1;               // k_inv_plane cluster width (coil split), divides C, <= 8
    int spec = 0;                // plane kernels with compile-time geometry (0 = generic)
    size_t smem_plane = 0, smem_inv = 0, smem_slow = 0;
    size_t b1_elems() const { return (size_t)C * ns * ncol; }
};

// Fills `plan` and returns true when the engine supports the sizes (powers of
// two, every length <= 1024, nm * nf <= 16384); sets the kernels' shared memory
// limits.  ns, nm, nf: image lengths in voxel axis order (nm = 1 for 2-D).
bool toep_fft_plan(int ns, int nm, int nf, int C, ToepFftPlan *plan);

// exp(-2 pi i j / 2048), j < 2048, as a device table (caller frees).
cudaError_t toep_fft_twiddles(float2 **tw);

// Qf_l in the natural 2N-grid voxel order -> parity-major order, times scale.
cudaError_t toep_fft_qf(const ToepFftPlan &p, float2 *qf2_l, const float2 *qf_l, float scale,
                        cudaStream_t st);

// q (=, first != 0; += otherwise) conj(e_l) sum_c conj(S_c) F^H F_l(S_c e_l p).
// b1: scratch of plan.b1_elems() complex values.  done: optional device flag;
// when it is non-zero the kernels return at once (converged CG).  err: device
// error word (DEV_ERR_TIMEOUT when a bounded wait on a bulk copy ran out).
cudaError_t toep_fft_apply_l(const ToepFftPlan &p, float2 *q, const float2 *x,
                             const float2 *sens, const float2 *eph_l, float2 *b1,
                             const float2 *qf2_l, int first, const int *done, const float2 *tw,
                             unsigned *err, cudaStream_t st);

}  // namespace imp

// Multi-dimensional complex FFT of the Toeplitz path's grids (the gridding
// grids of Q and F^H d, the 2N grid of Qf_l = FFT(Q_l), and the zero-padded
// F^H F chain of sizes the pruned engine does not take).  The reference
// calls cuFFT C2C at these places (toeplitz/computeQ.cmem.cu:623,
// toeplitz/computeFH.cmem.cu:679, toeplitz/recon.cu:1161,1177,1959); this is
// a hand-written replacement with the same conventions: forward
// X[k] = sum_j x[j] e^{-2 pi i jk/n}, inverse with e^{+...}, unnormalised,
// in place on a row-major [batch][n0][n1][n2] array (n2 fastest).
//
// One kernel launch per axis of length > 1: each block loads a tile of whole
// lines into shared memory (consecutive lines for the contiguous axis,
// consecutive columns for a strided one, so the global accesses coalesce),
// runs the mixed-radix Stockham stages between two shared buffers, and
// writes the lines back.  Butterflies of radix 2, 3, 4, 5, 7, 8 and 16 are
// register DFTs with compile-time constants; any other prime factor runs a
// per-output loop over its R inputs.  Axes up to 4096 points.
#pragma once
#include <cuda_runtime.h>

namespace imp {

struct GridFft {
    int n[3] = {1, 1, 1};  // axis lengths, n[2] fastest (2-D: n[0] = 1)
    int batch = 1;
    float2 *tw[3] = {nullptr, nullptr, nullptr};  // exp(-2 pi i j / n[a]), j < n[a]
    int nfac[3] = {0, 0, 0};
    unsigned char fac[3][24] = {};                // radix sequence per axis
    int cw[3] = {1, 1, 1};                        // lines per block
    int rs[3] = {1, 1, 1};                        // shared tile row stride (elements)
    size_t smem[3] = {0, 0, 0};
    size_t elems() const { return (size_t)batch * n[0] * n[1] * n[2]; }
    int passes() const { return (n[0] > 1) + (n[1] > 1) + (n[2] > 1); }  // kernel launches
};

constexpr int kGridFftMaxN = 4096;

// Plans a transform of `batch` grids of n0 x n1 x n2 (n2 fastest; pass n0 = 1
// for 2-D, n0 = n1 = 1 for 1-D).  Allocates the twiddle tables (device
// memory, freed by grid_fft_destroy).  cudaErrorInvalidValue when an axis
// exceeds kGridFftMaxN.
cudaError_t grid_fft_create(GridFft *f, int n0, int n1, int n2, int batch);
void grid_fft_destroy(GridFft *f);

// In-place unnormalised transform of `data` (f.elems() complex values).
cudaError_t grid_fft_exec(const GridFft &f, float2 *data, bool inverse, cudaStream_t st);

// The same transform when only a crop of the output is read afterwards: along
// axis a, outputs j < keep_half[a] and j >= n[a] - keep_half[a] (0: all).  Each
// axis pass (fastest first) transforms only the lines whose faster coordinates
// are kept and stores only its kept outputs; everything else of `data` is left
// undefined.
cudaError_t grid_fft_exec_cropped(const GridFft &f, float2 *data, bool inverse,
                                  const int keep_half[3], cudaStream_t st);

}  // namespace imp

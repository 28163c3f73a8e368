// Internal host-side interface of the NUDFT tile engine.
//
// The engine evaluates, for every (sample k, voxel r) pair,
//     theta = 2 pi (kx x + ky y + kz z) + omega_r t_k
// (the exponent of kernels/ftCpu.cpp:158-160, with the z term of
// toeplitz/computeFH.cmem.cu:185-188 when use_z is set) and
//     F   : y_c[k] += S_c[r] x[r] e^{-i theta}        (kernels/ftGpu.cu:306-604)
//     F^H : x[r]   += conj(S_c[r]) d_c[k] e^{+i theta} (kernels/ftGpu.cu:756-1013)
//
// Phase arithmetic: the four products are accumulated in FP64 on top of the
// constant 1.5*2^20 turns, so that the low 32 bits of the double's mantissa
// are the phase modulo one turn in units of 2^-32 turn (an exact fixed-point
// reduction; no FP32 rounding of large arguments).  The top 23 of those bits
// become an FP32 angle in [-pi, pi) for the hardware sin/cos.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

namespace imp {

constexpr int kNT = 128;     // threads per NUDFT block
constexpr int kTile = 64;    // "theirs" elements per shared-memory tile
constexpr int kPadM = 1024;  // sample / voxel counts are padded to this

struct NuLaunch {
    int pt = 4;     // "ours" elements per thread
    int split = 1;  // partitions of the "theirs" range (partial sums)
    int occ = 4;    // blocks per SM the register budget is sized for (4 or 6)
    int tc = 0;     // 1: tensor-core kernel (nudft_tc.cu; pt and occ unused)
};

struct NuPlan {
    int M = 0, N = 0, C = 0;     // samples, voxels, coils
    int CG = 1, G = 1;           // coils per group, groups (CG * G >= C)
    int Mpad = 0, Npad = 0;
    bool use_z = false;
    double4 *kgeo = nullptr;     // [Mpad]  (kx, ky, kz, t)        turns / s
    double4 *vgeo = nullptr;     // [Npad]  (x, y, z, omega/2pi)   FOV / Hz
    float2 *sens = nullptr;      // [G][Npad][CG] coil sensitivities (zero padded)
    NuLaunch fwd, adj;
};

// Creates geometry and packed sensitivities from device SoA inputs.
// sensi_r/sensi_i may be null (unit sensitivity, C must be 1).
cudaError_t nu_plan_create(NuPlan &p, const float *kx, const float *ky, const float *kz,
                           const float *t, const float *ix, const float *iy, const float *iz,
                           const float *fm, const float *sensi_r, const float *sensi_i, int M,
                           int N, int C, bool use_z, unsigned *dev_err, cudaStream_t st);
// Re-packs geometry and sensitivities of the same sizes into an existing plan.
cudaError_t nu_plan_repack(NuPlan &p, const float *kx, const float *ky, const float *kz,
                           const float *t, const float *ix, const float *iy, const float *iz,
                           const float *sensi_r, const float *sensi_i, unsigned *dev_err,
                           cudaStream_t st);
// Sizes of a plan (M, N, C, CG, G, Mpad, Npad, use_z) without any memory.
void nu_plan_dims(NuPlan &p, int M, int N, int C, bool use_z);
// Packs geometry into caller-provided device memory (kgeo [Mpad], vgeo
// [Npad], sens [G][Npad][CG]) of a plan sized by nu_plan_dims.  Nothing is
// allocated; such a plan must not be passed to nu_plan_destroy.
cudaError_t nu_plan_place(NuPlan &p, double4 *kgeo, double4 *vgeo, float2 *sens,
                          const float *kx, const float *ky, const float *kz, const float *t,
                          const float *ix, const float *iy, const float *iz, const float *fm,
                          const float *sensi_r, const float *sensi_i, unsigned *dev_err,
                          cudaStream_t st);
// Replaces only the field map (per-slice) of an existing plan.
cudaError_t nu_plan_set_fm(NuPlan &p, const float *fm, unsigned *dev_err, cudaStream_t st);
void nu_plan_destroy(NuPlan &p);

// Heuristic launch shape (replaced by the autotuner when enabled).
NuLaunch nu_default_launch(const NuPlan &p, bool adj);

// Scratch bytes for the partial sums of one apply.
size_t nu_fwd_partial_bytes(const NuPlan &p, const NuLaunch &l);
size_t nu_adj_partial_bytes(const NuPlan &p, const NuLaunch &l);

// xs[g][r][cg] = S[g][r][cg] * x[r]   (x interleaved complex, [Npad])
cudaError_t nu_pack_image(const NuPlan &p, const float2 *x, float2 *xs, cudaStream_t st);
// Same from SoA x (operator API).
cudaError_t nu_pack_image_soa(const NuPlan &p, const float *xr, const float *xi, float2 *xs,
                              cudaStream_t st);

// Forward partials: part[split][g][Mpad][CG].
cudaError_t nu_forward_partials(const NuPlan &p, const NuLaunch &l, const float2 *xs,
                                float2 *part, unsigned *dev_err, cudaStream_t st);
// Adjoint partials (after conj(S) and the in-group coil sum): part[split][g][Npad].
// `data` is [G][Mpad][CG].
cudaError_t nu_adjoint_partials(const NuPlan &p, const NuLaunch &l, const float2 *data,
                                float2 *part, unsigned *dev_err, cudaStream_t st);

// One slice of a batched launch: element offsets into the concatenated
// "ours" / "theirs" geometry (double4), the "theirs" data and the partial
// sums (float2), and the slice's padded sizes.
struct NuSlice {
    long long ours, theirs, tdata, out;
    int n_ours, n_theirs, per_split;
};

// Partials of S slices in one launch (grid: max_ours / (kNT * pt) x split x
// S * G); `p` supplies C, CG, G, use_z and the shared sensitivities, `l` the
// launch shape (its split must cut every slice's "theirs" range into whole
// tiles).  Per-slice layouts are those of nu_forward_partials /
// nu_adjoint_partials at the slice's offsets.
cudaError_t nu_partials_batch(const NuPlan &p, const NuLaunch &l, bool adj, int S, int max_ours,
                              const NuSlice *d_slices, const double4 *ours,
                              const double4 *theirs, const float2 *tdata, float2 *part,
                              unsigned *dev_err, cudaStream_t st);

// k-space SoA [C][M] <-> packed [G][Mpad][CG]
cudaError_t nu_pack_kdata(const NuPlan &p, const float *dr, const float *di, float2 *packed,
                          cudaStream_t st);
// Sum forward partials and write SoA [C][M] (operator API).
cudaError_t nu_forward_finish_soa(const NuPlan &p, const NuLaunch &l, const float2 *part,
                                  float *yr, float *yi, cudaStream_t st);
// Sum adjoint partials and write SoA [N].
cudaError_t nu_adjoint_finish_soa(const NuPlan &p, const NuLaunch &l, const float2 *part,
                                  float *xr, float *xi, cudaStream_t st);

// Launch shapes the kernel set covers.
bool nu_shape_supported(int CG, int pt);
// True when `split` partitions n_theirs into whole shared-memory tiles.
bool nu_split_ok(int n_theirs, int split);

// Tensor-core kernel (nudft_tc.cu): same partial-sum layouts as
// nu_forward_partials / nu_adjoint_partials / nu_partials_batch; coil groups
// of 1, 2, 4, 8, 16 or 32.  It is an autotuner candidate unless
// IMP_NUDFT_TC=0 (nu_tc_enabled), the default launch shape when
// IMP_NUDFT_TC=1 (nu_tc_forced), and the only kernel for coil groups of 16
// and 32 (plans of more than 8 coils, unless IMP_NUDFT_TC=0).
bool nu_tc_supported(int CG);
bool nu_tc_enabled();
bool nu_tc_forced();
// "ours" rows per block of the tensor-core kernel for coil groups of CG.
int nu_tc_rows(int CG);
cudaError_t nu_partials_tc(const NuPlan &p, const NuLaunch &l, bool adj, const float2 *tdata,
                           float2 *out, unsigned *dev_err, cudaStream_t st);
cudaError_t nu_partials_tc_batch(const NuPlan &p, const NuLaunch &l, bool adj, int S,
                                 int max_ours, const NuSlice *d_slices, const double4 *ours,
                                 const double4 *theirs, const float2 *tdata, float2 *out,
                                 unsigned *dev_err, cudaStream_t st);

// Autotuner (tune.cu): times every supported (pt, occ, split) of one direction
// and the tensor-core kernel's splits
// on the live buffers `tdata` / `part` (part_bytes of scratch) and returns the
// fastest.  Results are cached per problem shape in memory and in a text file
// ($IMP_TUNE_CACHE, default ~/.cache/impatient_b200/nudft_tune.txt).
cudaError_t nu_autotune(const NuPlan &p, bool adj, const float2 *tdata, float2 *part,
                        size_t part_bytes, unsigned *dev_err, cudaStream_t st, NuLaunch *out);
// Cached result for this shape, if any (no timing).
bool nu_tuned_lookup(const NuPlan &p, bool adj, NuLaunch *out);
// Largest partial-sum scratch any tuning candidate needs.
size_t nu_tune_partial_bytes(const NuPlan &p, bool adj);

// Batched launches (one shape for all slices): the launch shape within the
// kernel family of the plan (tensor-core: split; CUDA-core: pt, occupancy and
// split) is tuned per batched problem -- direction, coil grouping, slice count
// and padded sizes -- by timing the whole batch, and cached beside the
// single-slice shapes (lines "b1 ...").
struct NuBatchKey {
    int adj, CG, G, use_z, S, Npad, max_mpad;
    long long mpad_total;
    int tc;
};
bool nu_tuning_enabled();
bool nu_batch_lookup(const NuBatchKey &k, NuLaunch *out);
void nu_batch_store(const NuBatchKey &k, const NuLaunch &l, double ms);

}  // namespace imp

/*
 * impatient_b200.h -- C-ABI of the B200 (sm_100a) rebuild of the IMPATIENT MRI
 * iterative non-Cartesian reconstruction path (mriSolver).
 *
 * Conventions
 *   - Plain pointers and sizes only.  Complex vectors are split real/imag
 *     float32 arrays (the reference's SoA layout).  Coil-indexed arrays are
 *     coil-major: sensi[c*num_i + r], kdata[c*num_k + k].
 *   - Every entry point returns an imp_status (0 = IMP_OK) and never exits the
 *     process; imp_last_error() gives a message for the calling thread.
 *   - An imp_context owns one CUDA stream and the device work memory; use one
 *     context per thread.  Operator-level calls take DEVICE pointers and are
 *     synchronous.  Recon-level calls accept host or device pointers.
 *   - The reference's interfaces that each entry point replaces are cited as
 *     path:line within the reference project.
 */
#ifndef IMPATIENT_B200_H
#define IMPATIENT_B200_H

#ifdef __cplusplus
extern "C" {
#endif

typedef int imp_status;

#define IMP_OK 0
#define IMP_ERR_INVALID_ARG 1  /* bad size, null pointer, inconsistent flags      */
#define IMP_ERR_CUDA 2         /* a CUDA runtime call failed                       */
#define IMP_ERR_IO 3           /* file missing / unreadable / unwritable           */
#define IMP_ERR_FORMAT 4       /* malformed 0.2 / 1.0 input file                   */
#define IMP_ERR_RANGE 5        /* coordinate outside the fixed-point phase range   */
#define IMP_ERR_NOMEM 6        /* device allocation failed                         */
#define IMP_ERR_TIMEOUT 7      /* a bounded device-side wait expired               */
#define IMP_ERR_UNSUPPORTED 8  /* option the library does not implement            */

/* Version of this ABI (major*100 + minor). */
int imp_abi_version(void);
const char *imp_status_string(imp_status s);
/* Message of the last failing call on this thread ("" if none). */
const char *imp_last_error(void);

typedef struct imp_context imp_context;

/* Creates a context on CUDA device `device` with its own stream (a blocking
 * stream: it orders after work queued on the legacy default stream). */
imp_status imp_context_create(int device, imp_context **ctx);
imp_status imp_context_destroy(imp_context *ctx);
/* Blocks until all work of the context's stream is done. */
imp_status imp_context_synchronize(imp_context *ctx);
/* Number of this library's kernels launched by the most recent call. */
long imp_context_launch_count(const imp_context *ctx);

/* Kernel timing of recon calls (no reference counterpart; replaces the
 * reference's cutil timer singleton, kernels/structures.h:206-601).  While
 * enabled, recon calls run without CUDA graphs and bracket every NUDFT launch
 * with CUDA events on the launching stream; enabling resets the totals. */
imp_status imp_context_profile(imp_context *ctx, int enable);
/* which: 0 = forward NUDFT kernel, 1 = adjoint NUDFT kernel. */
imp_status imp_context_profile_read(const imp_context *ctx, int which, double *total_ms,
                                    long *count);

/* Runs one kernel whose bounded mbarrier wait runs out (a barrier nothing
 * arrives on, `polls` try_wait rounds): the failure path of every bounded
 * wait in the library's kernels.  Returns IMP_ERR_TIMEOUT with its message;
 * the kernel ends normally and the context stays usable.  No reference
 * counterpart (the reference's kernels have no device-side waits). */
imp_status imp_check_wait_expiry(imp_context *ctx, int polls);

/* Measures the FP32 FMA rate (TFLOP/s, 2 flops per FMA) and the SFU sine rate
 * (G ops/s) of `device` with two short throughput kernels: the denominators
 * of the NUDFT roofline.  No reference counterpart. */
imp_status imp_measure_alu_peaks(int device, double *fp32_tflops, double *sfu_gops);

/* ------------------------------------------------------------------------
 * Operator level: NUDFT with field map (DEVICE pointers, synchronous).
 * theta(k,r) = 2 pi (kx[k] ix[r] + ky[k] iy[r] + use_z*kz[k] iz[r]) + fm[r] t[k]
 * use_z = 0 reproduces the reference, whose NUDFT drops z
 * (kernels/ftGpu.cu:325-328); use_z = 1 is the 3-D formula of
 * toeplitz/computeFH.cmem.cu:185-188.  fm may be NULL (no field map).
 * ---------------------------------------------------------------------- */

/* kdata[k] = sum_r idata[r] exp(-i theta)
 * replaces ftGpu(), kernels/ftGpu.cu:198 / kernels/gpuPrototypes.cuh:154 */
imp_status imp_ft(imp_context *ctx, float *kdata_r, float *kdata_i, const float *idata_r,
                  const float *idata_i, const float *kx, const float *ky, const float *kz,
                  const float *ix, const float *iy, const float *iz, const float *fm,
                  const float *t, int num_k, int num_i, int use_z);

/* idata[r] = sum_k kdata[k] exp(+i theta)
 * replaces iftGpu(), kernels/ftGpu.cu:653 / kernels/gpuPrototypes.cuh:162 */
imp_status imp_ift(imp_context *ctx, float *idata_r, float *idata_i, const float *kdata_r,
                   const float *kdata_i, const float *kx, const float *ky, const float *kz,
                   const float *ix, const float *iy, const float *iz, const float *fm,
                   const float *t, int num_k, int num_i, int use_z);

/* kdata[c*num_k + k] = sum_r sensi[c*num_i + r] idata[r] exp(-i theta)
 * replaces parallelFtGpu(), kernels/parImagingGpu.cu:92 */
imp_status imp_parallel_ft(imp_context *ctx, float *kdata_r, float *kdata_i,
                           const float *idata_r, const float *idata_i, const float *kx,
                           const float *ky, const float *kz, const float *ix, const float *iy,
                           const float *iz, const float *fm, const float *t, int num_k,
                           int num_i, const float *sensi_r, const float *sensi_i, int num_coil,
                           int use_z);

/* idata[r] = sum_c conj(sensi[c*num_i + r]) sum_k kdata[c*num_k + k] exp(+i theta)
 * replaces parallelIftGpu(), kernels/parImagingGpu.cu:119 */
imp_status imp_parallel_ift(imp_context *ctx, float *idata_r, float *idata_i,
                            const float *kdata_r, const float *kdata_i, const float *kx,
                            const float *ky, const float *kz, const float *ix, const float *iy,
                            const float *iz, const float *fm, const float *t, int num_k,
                            int num_i, const float *sensi_r, const float *sensi_i,
                            int num_coil, int use_z);

/* The same adjoint as imp_parallel_ift, for callers that cannot allocate
 * device memory -- for example a reconstruction host that reserves all device
 * memory through its own allocator at start-up or runs under a fixed memory
 * budget.  No counterpart in the reference.
 *   - Allocates nothing and needs no context: all work memory (packed
 *     geometry, sensitivities and k-space data, partial sums) is one static
 *     device array of 32 MiB that every GPU loading this library holds until
 *     the process exits.  Sizes whose work memory does not fit are rejected
 *     with IMP_ERR_INVALID_ARG.  About 40 bytes per voxel and 40 bytes per
 *     sample per group of up to 8 coils are needed, plus partial sums.
 *   - Runs on `stream` (a cudaStream_t; NULL is the legacy default stream) of
 *     the current device, synchronizes that stream and returns when the
 *     result is in idata; a failing call also drains its own queued work
 *     before it returns.  imp_last_error() describes a failure.
 *   - The first call on a device looks up the device address of the array
 *     with that device current; make that first call before any stream
 *     capture.  The address is kept for the process: do not call this after
 *     a cudaDeviceReset.
 *   - Every call shares the array: calls that overlap on the GPU race. */
imp_status imp_parallel_ift_noalloc(float *idata_r, float *idata_i, const float *kdata_r,
                                    const float *kdata_i, const float *kx, const float *ky,
                                    const float *kz, const float *ix, const float *iy,
                                    const float *iz, const float *fm, const float *t,
                                    int num_k, int num_i, const float *sensi_r,
                                    const float *sensi_i, int num_coil, int use_z,
                                    void *stream);

/* ------------------------------------------------------------------------
 * Recon level: brute-force CG (host or device pointers).
 * ---------------------------------------------------------------------- */
/* Real sparse matrix in coordinate form, 0-based (the reference's CooMatrix,
 * kernels/structures.h:927-990, read from c.rmtx by readMtxFile,
 * kernels/mmio.cpp:668-830).  For -reg it is the roughness matrix C:
 * rows = B * num_i (B blocks of num_i rows, one per difference direction),
 * cols = num_i. */
typedef struct imp_sparse {
    int rows, cols, nnz;
    const int *row;      /* [nnz] row indices (host memory) */
    const int *col;      /* [nnz] column indices (host memory) */
    const float *val;    /* [nnz] values (host memory) */
} imp_sparse;

typedef struct imp_bf_options {
    int cg_num;          /* CG iteration number; cg_num-1 updates are made  */
    int enable_fd;       /* finite-difference regularizer (-fd / -fdp)      */
    float fd_penalizer;  /* lambda (-fdp)                                   */
    int enable_tv;       /* TV reweighting outer loop (-tv)                 */
    int tv_num;          /* TV iterations (-tv_num)                         */
    float tv_eps;        /* TV smoothing, reference FP32 value 1e-6         */
    int use_z;           /* 0: reference 2-D semantics, 1: true 3-D         */
    int nx, ny, nz;      /* TV grid.  0,0,0 = reference sqrt(N) x sqrt(N)   */
    const imp_sparse *reg;  /* -reg: roughness matrix C; NULL = off.  When set,
                             * lambda C^T W C replaces lambda D^H W D (the
                             * reference gives -reg precedence over -fd,
                             * bruteForce/bruteForceCpu.cpp:306-380) */
} imp_bf_options;

/* Fills `opt` with the reference defaults (main.cpp:96-101). */
void imp_bf_options_default(imp_bf_options *opt);

/* Brute-force CG recon of one or more slices.  idata (num_slices*num_i) is the
 * initial estimate on entry and the image on return; kdata is
 * [slice][coil][num_k]; fm is [slice][num_i]; trajectories, t and sensi are
 * shared by all slices, as in the reference's slice loop.
 * replaces bruteForceGpu(), bruteForce/bruteForceGpu.cuh:72-86 (called per
 * slice from bruteForce(), main_mri.cu:875-895) */
imp_status imp_bruteforce_recon(imp_context *ctx, const imp_bf_options *opt, float *idata_r,
                                float *idata_i, const float *kdata_r, const float *kdata_i,
                                const float *kx, const float *ky, const float *kz,
                                const float *ix, const float *iy, const float *iz,
                                const float *fm, const float *t, const float *sensi_r,
                                const float *sensi_i, int num_k, int num_i, int num_coil,
                                int num_slices);

/* The slices of imp_bruteforce_recon spread over several GPUs: one host
 * thread per worker, each with its own context on devices[w] (devices null:
 * GPUs 0 .. num_workers-1; num_workers <= 0: every visible GPU), takes the
 * next unclaimed slice and reconstructs it; images land in disjoint slices of
 * idata.  Host arrays, same layouts as imp_bruteforce_recon.  The first failure
 * stops further slices and is returned.
 * replaces the -mgpu path: bruteForceMgpu / its pthread work queue,
 * bruteForce/bruteForceMgpu.cu:81-128, main_mri.cu:770-834 */
imp_status imp_bruteforce_mgpu(const imp_bf_options *opt, float *idata_r, float *idata_i,
                               const float *kdata_r, const float *kdata_i, const float *kx,
                               const float *ky, const float *kz, const float *ix,
                               const float *iy, const float *iz, const float *fm,
                               const float *t, const float *sensi_r, const float *sensi_i,
                               int num_k, int num_i, int num_coil, int num_slices,
                               const int *devices, int num_workers);

/* Brute-force CG recon of num_slices slices that share the image grid
 * (ix, iy, iz: num_i) and the coil maps but each have their own trajectory and
 * sample count (uneven M), k-space data and field map -- the multi-slice loop
 * of main_mri.cu:875-895 generalised to per-slice trajectories.  Slice s owns
 * samples k_off[s] .. k_off[s+1]-1 of kx, ky, kz, t (k_off: host array of
 * num_slices+1 offsets, k_off[0] = 0); its data are
 * kdata[num_coil*k_off[s] + c*(k_off[s+1]-k_off[s]) + k]; fm and idata are
 * [slice][num_i].  All slices are solved in lockstep: every CG step is one
 * kernel launch over all slices (uneven sample counts included), each slice
 * with its own FP64 CG scalars; the CG update is a CUDA graph. */
imp_status imp_bruteforce_batch(imp_context *ctx, const imp_bf_options *opt, float *idata_r,
                                float *idata_i, const float *kdata_r, const float *kdata_i,
                                const float *kx, const float *ky, const float *kz,
                                const float *t, const int *k_off, const float *ix,
                                const float *iy, const float *iz, const float *fm,
                                const float *sensi_r, const float *sensi_i, int num_i,
                                int num_coil, int num_slices);

/* Directory-level drop-in of bruteForce(idir, odir, ...) (main_mri.cuh:110-118,
 * main_mri.cu:652-1025): reads idir in the 0.2 or 1.0 format
 * (kernels/structures.cpp:569-1162), reconstructs every slice and writes
 * odir/output_gpu_r.dat and odir/output_gpu_i.dat as "%f\n" text
 * (kernels/structures.cpp:1165-1175).  gpu_id < 0 is the -mgpu mode: the
 * slices are spread over every visible GPU (imp_bruteforce_mgpu). */
imp_status imp_bruteforce_dir(const char *idir, const char *odir, const imp_bf_options *opt,
                              int gpu_id);

/* Reads the sizes of an input directory with the reference's reader rules
 * (loadInputData, kernels/structures.cpp:569-780) without touching a GPU.
 * Any output pointer may be NULL. */
imp_status imp_dataset_info(const char *idir, int *num_k, int *num_i, int *num_coil,
                            int *num_slices, int *nx, int *ny, int *nz);

/* ---- Toeplitz path ------------------------------------------------------
 * Image layout: 2-D [x][y] (y fastest), 3-D [y][x][z] (z fastest), the
 * voxel order of the reference's ix/iy/iz files.  Q is stored as in
 * Q_stone.file: for each segment l = 0..(int)ntime_segs one block of
 * (2nx)(2ny)(2nz or 1) values on the 2N grid, split into re and im arrays.
 * Every array argument may be a host or a device pointer. */

typedef struct imp_toeplitz_options {
    int cg_num;          /* CG iterations (-cg_num) */
    int enable_fd;       /* finite-difference regularization (-fd / -fdp) */
    float fd_penalizer;  /* lambda (-fdp) */
    int enable_tv;       /* TV reweighting passes (-tv) */
    int tv_num;          /* TV passes (-tv_num) */
    float tv_eps;        /* TV smoothing epsilon (1e-6 in the reference) */
    float ntime_segs;    /* L (-ntime_segs); segments l = 0..(int)L */
    float gridOS_Q;      /* oversampling of the Q gridding (-gridOS_Q) */
    float gridOS_FH;     /* oversampling of the F^H d gridding (-gridOS_FH) */
    const imp_sparse *reg;  /* -reg: roughness matrix C (NULL = off); lambda
                             * C^T W C replaces lambda D^H W D in A^H A
                             * (toeplitz/recon.cu:1543-1673) */
} imp_toeplitz_options;

/* Defaults of main.cpp:103-444 for the Toeplitz flags. */
void imp_toeplitz_options_default(imp_toeplitz_options *opt);

/* Q_l, l = 0..L, by Kaiser-Bessel gridding of h_l(t) at 2k on the
 * oversampled 2N grid, FFT and deapodization.
 * replaces computeQ_GPU_Grid(), toeplitz/computeQ.cmem.cu:402-756
 * (driven by computeQ_GPU, toeplitz/computeQ.cmem.cu:757-1028).
 * q_r/q_i: (L+1) * (2nx)(2ny)(2nz or 1) floats each. */
imp_status imp_toeplitz_q(imp_context *ctx, const imp_toeplitz_options *opt, float *q_r,
                          float *q_i, const float *kx, const float *ky, const float *kz,
                          const float *t, int num_k, int nx, int ny, int nz);

/* F^H d with time segmentation and SENSE by gridding.
 * replaces computeFH_GPU_Grid(), toeplitz/computeFH.cmem.cu:470-805
 * (driven by computeFH_GPU, toeplitz/computeFH.cmem.cu:1188-1409).
 * kdata, sensi: [coil][...]; fm may be NULL (zero field map). */
imp_status imp_toeplitz_fhd(imp_context *ctx, const imp_toeplitz_options *opt, float *fhd_r,
                            float *fhd_i, const float *kdata_r, const float *kdata_i,
                            const float *kx, const float *ky, const float *kz, const float *t,
                            const float *fm, const float *sensi_r, const float *sensi_i,
                            int num_k, int num_coil, int nx, int ny, int nz);

/* Toeplitz CG (with optional FD regularization and TV passes) from x = 0;
 * x receives the iterate with the smallest residual.
 * replaces toeplitz_recon(), toeplitz/recon.cu:1724-2191. */
imp_status imp_toeplitz_recon(imp_context *ctx, const imp_toeplitz_options *opt, float *x_r,
                              float *x_i, const float *fhd_r, const float *fhd_i,
                              const float *q_r, const float *q_i, const float *t, int num_k,
                              const float *fm, const float *sensi_r, const float *sensi_i,
                              int num_coil, int nx, int ny, int nz);

/* In-place complex FFT of `batch` grids of n0 x n1 x n2 points (row-major, n2
 * fastest; n0 = 1 for 2-D, n0 = n1 = 1 for 1-D), split re/im, host or device
 * pointers: forward X[k] = sum_j x[j] e^{-2 pi i jk/n} per axis (inverse != 0:
 * e^{+...}), unnormalised.  The transform the Toeplitz path runs on its
 * gridding grids and on the 2N grid; replaces the cuFFT C2C calls at
 * toeplitz/recon.cu:1161,1177,1959, toeplitz/computeQ.cmem.cu:623 and
 * toeplitz/computeFH.cmem.cu:679.  Axes up to 4096 points whose prime factors
 * are <= 255 (IMP_ERR_UNSUPPORTED otherwise). */
imp_status imp_grid_fft(imp_context *ctx, float *data_r, float *data_i, int n0, int n1, int n2,
                        int batch, int inverse);

/* One application of A^H A p (+ lambda D^H D p when enable_fd), the operator
 * inside each Toeplitz CG iteration (toeplitz/recon.cu:598-840 with
 * DHWD at W = 1).  For tests and custom solvers. */
imp_status imp_toeplitz_apply(imp_context *ctx, const imp_toeplitz_options *opt, float *out_r,
                              float *out_i, const float *p_r, const float *p_i,
                              const float *q_r, const float *q_i, const float *t, int num_k,
                              const float *fm, const float *sensi_r, const float *sensi_i,
                              int num_coil, int nx, int ny, int nz);

/* Toeplitz CG started from the image in x (the warm start) and stopped when
 * sqrt(|r|^2 / |F^H d|^2) < tol (the residual test of toeplitz/recon.cu:2112)
 * or after max_iter updates; x receives the minimum-residual iterate and
 * *iterations (optional) the updates performed.  FD regularization as in opt;
 * no TV passes.  No counterpart in the reference (which always starts from
 * zero, toeplitz/recon.cu:1871): it is the CG half of the learned warm start. */
imp_status imp_toeplitz_cg(imp_context *ctx, const imp_toeplitz_options *opt, float *x_r,
                           float *x_i, const float *fhd_r, const float *fhd_i, const float *q_r,
                           const float *q_i, const float *t, int num_k, const float *fm,
                           const float *sensi_r, const float *sensi_i, int num_coil, int nx,
                           int ny, int nz, double tol, int max_iter, int *iterations);

/* ---- Learned warm start: BF16 U-Net (no counterpart in the reference) ----
 * 2 channels (re, im) in and out, 4 levels of 32-256 channels, 3x3 convs with
 * ReLU, max-pool down, nearest x2 + 1x1 conv up, skip concatenation; BF16
 * weights and activations with FP32 accumulation on the tensor cores, FP32
 * master weights and Adam.  Images are [batch][2][height*width] float32,
 * height and width multiples of 8; pointers may be host or device. */
typedef struct imp_unet imp_unet;

imp_status imp_unet_create(imp_context *ctx, int batch, int height, int width,
                           unsigned long long seed, imp_unet **out);
void imp_unet_destroy(imp_unet *net);
long imp_unet_num_params(const imp_unet *net);
/* FP32 parameters, per layer weights [cout][ky][kx][cin] then bias [cout]. */
imp_status imp_unet_get_params(imp_unet *net, float *params);
imp_status imp_unet_set_params(imp_unet *net, const float *params);
imp_status imp_unet_forward(imp_unet *net, const float *x, float *y);
/* Gradients (same layout as the parameters) of the mean squared error between
 * forward(x) and target, without an update; *loss (optional) gets the error. */
imp_status imp_unet_gradients(imp_unet *net, const float *x, const float *target, float *grads,
                              float *loss);
/* One Adam step (lr) on the mean squared error between forward(x) and target;
 * *loss (optional) receives that error before the step. */
imp_status imp_unet_train_step(imp_unet *net, const float *x, const float *target, float lr,
                               float *loss);

/* Directory-level drop-in of toeplitz(idir, ...) (main_mri.cuh:97-108,
 * main_mri.cu:207-630): Q by gridding, by direct evaluation (direct != 0)
 * or read from Qdir/Q_stone.file (reuseQ != 0; Qdir NULL = idir), F^H d,
 * Toeplitz CG; writes idir/Q_stone.file (writeQ != 0), idir/FhD.file and
 * idir/out.file as raw float32 [re x N][im x N]. */
imp_status imp_toeplitz_dir(const char *idir, const imp_toeplitz_options *opt, int direct,
                            int gpu_id, int reuseQ, const char *Qdir, int writeQ);

/* The mriSolver command line (main.cpp:103-444) as a library call: same
 * flags, defaults and exit codes (0 ok, 1 error). */
int imp_mrisolver_main(int argc, char **argv);

#ifdef __cplusplus
}
#endif

#endif /* IMPATIENT_B200_H */

/*
 * TEST INFRASTRUCTURE ONLY -- the FP64 CPU oracle for the brute-force path.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load
 * this library, and only as the checker.  The product never links it.
 *
 * It restates, in double precision, the reference's brute-force algorithm:
 *   orc_ft      kernels/ftCpu.cpp:110-172 + kernels/parImagingCpu.cpp:84-108
 *               y_c[k] = sum_r S_c[r] x[r] exp(-i(2 pi k.r + fm[r] t[k]))
 *   orc_ift     kernels/ftCpu.cpp:185-277 + kernels/parImagingCpu.cpp:119-147
 *               x[r]   = sum_c conj(S_c[r]) sum_k d_c[k] exp(+i(2 pi k.r + fm[r] t[k]))
 *   orc_tv_weight kernels/multiplyCpu.cpp:84-110 (2-D) and
 *               toeplitz/multiplyGpu_toeplitz.cu:153-172 (3-D):
 *               w = 0.5 / sqrt(sum_axes |D_a x|^2 + eps)
 *   orc_dhwd    kernels/DHWD2dCpu.cpp:94-270 (2-D) and
 *               toeplitz/DHWD3dGpu_toeplitz.cu:170-580 (3-D):
 *               s = lambda * sum_axes D_a^H W D_a p, with (D p)_i = p_i - p_{i+1}
 *               and (D^H t)_i = t_i - t_{i-1}, periodic.
 *   orc_bf_cg   bruteForce/bruteForceCpu.cpp:121-528 (TV outer loop, cg_num-1
 *               Fletcher-Reeves updates tracking Af, alpha with the FD term).
 *
 * Phase convention: use_z = 0 drops the z term, as the reference's FP64 CPU
 * build (DATATRAJ_NO_Z_DIM, kernels/structures.h:121-125) and its GPU kernel
 * (kernels/ftGpu.cu:325-328) do; use_z = 1 adds 2 pi kz[k] z[r] per pair, the
 * 3-D formula of toeplitz/computeFH.cmem.cu:185-188.
 *
 * The image grid for TV is (n0, n1, n2), row-major with n2 fastest.  The
 * reference 2-D case is (sqrt N, sqrt N, 1): n0 is the "column" index that
 * Dhori2dCpu differences (stride num_row) and n1 the "row" index of
 * Dverti2dCpu (stride 1); an axis of size 1 contributes nothing.
 *
 * Parity pinning: tests compare every function here against the reference's
 * own FP64 CPU build (oracle/_ref/libref_bf64.so, built by build_ref.sh from
 * the reference sources) on the shipped datasets and on seeded inputs.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define TWO_PI 6.283185307179586476925286766559

static void ft_one(double *out_r, double *out_i, const double *xs_r, const double *xs_i,
                   const double *kx, const double *ky, const double *kz, const double *t,
                   const double *ix, const double *iy, const double *iz, const double *fm,
                   int M, int N, int use_z) {
    #pragma omp parallel for schedule(static)
    for (int k = 0; k < M; ++k) {
        double sr = 0.0, si = 0.0;
        const double a = kx[k] * TWO_PI, b = ky[k] * TWO_PI, c = use_z ? kz[k] * TWO_PI : 0.0;
        const double tk = t[k];
        for (int r = 0; r < N; ++r) {
            double e = (a * ix[r] + b * iy[r] + c * iz[r]) + fm[r] * tk;
            double s, co;
            s = sin(e); co = cos(e);
            sr += co * xs_r[r] + s * xs_i[r];
            si += -s * xs_r[r] + co * xs_i[r];
        }
        out_r[k] = sr;
        out_i[k] = si;
    }
}

void orc_ft(double *out_r, double *out_i, const double *x_r, const double *x_i,
            const double *kx, const double *ky, const double *kz, const double *t,
            const double *ix, const double *iy, const double *iz, const double *fm,
            const double *s_r, const double *s_i, int M, int N, int C, int use_z) {
    double *xs_r = (double *)malloc(sizeof(double) * (size_t)N);
    double *xs_i = (double *)malloc(sizeof(double) * (size_t)N);
    for (int c = 0; c < C; ++c) {
        const double *sr = s_r + (size_t)c * N, *si = s_i + (size_t)c * N;
        for (int r = 0; r < N; ++r) {
            xs_r[r] = sr[r] * x_r[r] - si[r] * x_i[r];
            xs_i[r] = sr[r] * x_i[r] + si[r] * x_r[r];
        }
        ft_one(out_r + (size_t)c * M, out_i + (size_t)c * M, xs_r, xs_i, kx, ky, kz, t, ix, iy,
               iz, fm, M, N, use_z);
    }
    free(xs_r);
    free(xs_i);
}

void orc_ift(double *out_r, double *out_i, const double *d_r, const double *d_i,
             const double *kx, const double *ky, const double *kz, const double *t,
             const double *ix, const double *iy, const double *iz, const double *fm,
             const double *s_r, const double *s_i, int M, int N, int C, int use_z) {
    #pragma omp parallel for schedule(static)
    for (int r = 0; r < N; ++r) {
        const double a = ix[r] * TWO_PI, b = iy[r] * TWO_PI, cz = use_z ? iz[r] * TWO_PI : 0.0;
        const double f = fm[r];
        double acc_r = 0.0, acc_i = 0.0;
        for (int c = 0; c < C; ++c) {
            const double *dr = d_r + (size_t)c * M, *di = d_i + (size_t)c * M;
            double sr = 0.0, si = 0.0;
            for (int k = 0; k < M; ++k) {
                double e = (kx[k] * a + ky[k] * b + kz[k] * cz) + f * t[k];
                double s = sin(e), co = cos(e);
                sr += co * dr[k] - s * di[k];
                si += s * dr[k] + co * di[k];
            }
            const double pr = s_r[(size_t)c * N + r], pi = s_i[(size_t)c * N + r];
            acc_r += pr * sr + pi * si;
            acc_i += pr * si - pi * sr;
        }
        out_r[r] = acc_r;
        out_i[r] = acc_i;
    }
}

/* forward difference along one axis: p[i] - p[i+1], periodic */
static inline size_t nxt(size_t idx, int coord, int n, size_t stride) {
    return (coord == n - 1) ? idx - (size_t)(n - 1) * stride : idx + stride;
}
static inline size_t prv(size_t idx, int coord, int n, size_t stride) {
    return (coord == 0) ? idx + (size_t)(n - 1) * stride : idx - stride;
}

void orc_tv_weight(double *w, const double *x_r, const double *x_i, int n0, int n1, int n2,
                   double eps) {
    const size_t s0 = (size_t)n1 * n2, s1 = (size_t)n2, s2 = 1;
    #pragma omp parallel for schedule(static)
    for (int a = 0; a < n0; ++a)
        for (int b = 0; b < n1; ++b)
            for (int c = 0; c < n2; ++c) {
                size_t i = a * s0 + b * s1 + c * s2;
                double acc = 0.0;
                size_t j;
                j = nxt(i, a, n0, s0);
                acc += (x_r[i] - x_r[j]) * (x_r[i] - x_r[j]) + (x_i[i] - x_i[j]) * (x_i[i] - x_i[j]);
                j = nxt(i, b, n1, s1);
                acc += (x_r[i] - x_r[j]) * (x_r[i] - x_r[j]) + (x_i[i] - x_i[j]) * (x_i[i] - x_i[j]);
                j = nxt(i, c, n2, s2);
                acc += (x_r[i] - x_r[j]) * (x_r[i] - x_r[j]) + (x_i[i] - x_i[j]) * (x_i[i] - x_i[j]);
                w[i] = 0.5 / sqrt(acc + eps);
            }
}

void orc_dhwd(double *s_r, double *s_i, const double *p_r, const double *p_i, const double *w,
              int n0, int n1, int n2, double lam) {
    const size_t s0 = (size_t)n1 * n2, s1 = (size_t)n2, s2 = 1;
    #pragma omp parallel for schedule(static)
    for (int a = 0; a < n0; ++a)
        for (int b = 0; b < n1; ++b)
            for (int c = 0; c < n2; ++c) {
                size_t i = a * s0 + b * s1 + c * s2;
                double ar = 0.0, ai = 0.0;
                int coord[3] = {a, b, c};
                int n[3] = {n0, n1, n2};
                size_t st[3] = {s0, s1, s2};
                for (int ax = 0; ax < 3; ++ax) {
                    if (n[ax] == 1) continue;
                    size_t ip = prv(i, coord[ax], n[ax], st[ax]);
                    size_t in = nxt(i, coord[ax], n[ax], st[ax]);
                    size_t ipn = i; /* next of prev is i */
                    /* t_i = w_i (p_i - p_{i+1}); t_{i-1} = w_{i-1} (p_{i-1} - p_i) */
                    double ti_r = w[i] * (p_r[i] - p_r[in]), ti_i = w[i] * (p_i[i] - p_i[in]);
                    double tp_r = w[ip] * (p_r[ip] - p_r[ipn]), tp_i = w[ip] * (p_i[ip] - p_i[ipn]);
                    ar += ti_r - tp_r;
                    ai += ti_i - tp_i;
                }
                s_r[i] = lam * ar;
                s_i[i] = lam * ai;
            }
}

static double dotre(const double *ar, const double *ai, const double *br, const double *bi,
                    size_t n) {
    double s = 0.0;
    for (size_t i = 0; i < n; ++i) s += ar[i] * br[i] + ai[i] * bi[i];
    return s;
}

/* Brute-force CG, bruteForce/bruteForceCpu.cpp:121-528, in FP64.
 * x (in/out, N) starts from the initial estimate. y is [C][M]. */
void orc_bf_cg(double *x_r, double *x_i, const double *y_r, const double *y_i,
               const double *kx, const double *ky, const double *kz, const double *t,
               const double *ix, const double *iy, const double *iz, const double *fm,
               const double *s_r, const double *s_i, int M, int N, int C, int use_z,
               int n0, int n1, int n2, int cg_num, int fd, double lam, int tv, int tv_num,
               double eps) {
    const size_t CM = (size_t)C * M;
    double *Af_r = calloc(CM, 8), *Af_i = calloc(CM, 8);
    double *q_r = calloc(CM, 8), *q_i = calloc(CM, 8);
    double *r_r = calloc(CM, 8), *r_i = calloc(CM, 8);
    double *g_r = calloc(N, 8), *g_i = calloc(N, 8);
    double *gt_r = calloc(N, 8), *gt_i = calloc(N, 8);
    double *d_r = calloc(N, 8), *d_i = calloc(N, 8);
    double *s_fr = calloc(N, 8), *s_fi = calloc(N, 8);
    double *w = calloc(N, 8);
    for (int tvi = 0; tvi < tv_num; ++tvi) {
        if (tvi == 0) for (int i = 0; i < N; ++i) w[i] = 1.0;
        if (tv && fd && tvi != 0) orc_tv_weight(w, x_r, x_i, n0, n1, n2, eps);
        orc_ft(Af_r, Af_i, x_r, x_i, kx, ky, kz, t, ix, iy, iz, fm, s_r, s_i, M, N, C, use_z);
        double oldin = 0.0;
        for (int it = 1; it < cg_num; ++it) {
            for (size_t j = 0; j < CM; ++j) { r_r[j] = y_r[j] - Af_r[j]; r_i[j] = y_i[j] - Af_i[j]; }
            orc_ift(gt_r, gt_i, r_r, r_i, kx, ky, kz, t, ix, iy, iz, fm, s_r, s_i, M, N, C, use_z);
            if (fd) {
                orc_dhwd(s_fr, s_fi, x_r, x_i, w, n0, n1, n2, lam);
                for (int i = 0; i < N; ++i) { g_r[i] = gt_r[i] - s_fr[i]; g_i[i] = gt_i[i] - s_fi[i]; }
            } else {
                memcpy(g_r, gt_r, 8 * (size_t)N); memcpy(g_i, gt_i, 8 * (size_t)N);
            }
            double newin = dotre(g_r, g_i, g_r, g_i, N);
            if (it == 1) {
                memcpy(d_r, g_r, 8 * (size_t)N); memcpy(d_i, g_i, 8 * (size_t)N);
            } else {
                double gamma = (oldin == 0.0) ? 0.0 : newin / oldin;
                for (int i = 0; i < N; ++i) { d_r[i] = g_r[i] + gamma * d_r[i]; d_i[i] = g_i[i] + gamma * d_i[i]; }
            }
            oldin = newin;
            orc_ft(q_r, q_i, d_r, d_i, kx, ky, kz, t, ix, iy, iz, fm, s_r, s_i, M, N, C, use_z);
            double ctcd = 0.0;
            if (fd) {
                orc_dhwd(s_fr, s_fi, d_r, d_i, w, n0, n1, n2, lam);
                ctcd = dotre(s_fr, s_fi, d_r, d_i, N);
            }
            double dg = dotre(d_r, d_i, g_r, g_i, N);
            double qq = dotre(q_r, q_i, q_r, q_i, CM);
            double alpha = dg / (qq + ctcd);
            for (size_t j = 0; j < CM; ++j) { Af_r[j] += alpha * q_r[j]; Af_i[j] += alpha * q_i[j]; }
            for (int i = 0; i < N; ++i) { x_r[i] += alpha * d_r[i]; x_i[i] += alpha * d_i[i]; }
        }
        if (!tv) break;
    }
    free(Af_r); free(Af_i); free(q_r); free(q_i); free(r_r); free(r_i);
    free(g_r); free(g_i); free(gt_r); free(gt_i); free(d_r); free(d_i);
    free(s_fr); free(s_fi); free(w);
}

// Test infrastructure only: a C-ABI shim around the reference's own CPU
// brute-force path, compiled from the reference sources by build_ref.sh into
// oracle/_ref/.  Nothing in the product links or loads this file; tests and
// bench.py's reference / cpu_baseline legs load the built .so as the checker.
//
// Wrapped reference entry points:
//   loadInputData            kernels/structures.cpp:569
//   bruteForceCpu            bruteForce/bruteForceCpu.cpp:121
//   parallelFtCpu            kernels/parImagingCpu.cpp:84
//   parallelIftCpu           kernels/parImagingCpu.cpp:119
//   DHWD2dCpu                kernels/DHWD2dCpu.cpp:94
//
// FLOAT_T is float or double depending on ENABLE_DOUBLE_PRECISION; the shim
// always speaks double at its boundary and converts.
#include <cstring>
#include <cstdlib>
#include <string>
#include <vector>

#include <cutil.h>
#include <tools.h>
#include <structures.h>
#include <bruteForceCpu.h>
#include <parImagingCpu.h>
#include <DHWD2dCpu.h>

namespace {

std::vector<FLOAT_T> to_ft(const double *p, int n) {
    std::vector<FLOAT_T> v(n);
    for (int i = 0; i < n; ++i) v[i] = (FLOAT_T)p[i];
    return v;
}

void fill_traj(DataTraj *tr, const double *x, const double *y, const double *z, int n) {
    for (int i = 0; i < n; ++i) {
        tr[i].x = (FLOAT_T)x[i];
        tr[i].y = (FLOAT_T)y[i];
#if !DATATRAJ_NO_Z_DIM
        // the reference loader stores only kz[0] / iz[0] (structures.cpp:744-758)
        tr[i].z = (FLOAT_T)z[0];
#endif
    }
}

bool g_timer_init = false;
void ensure_timer() {
    if (!g_timer_init) { initMriTimer(); g_timer_init = true; }
}

}  // namespace

extern "C" {

int ref_is_double(void) {
#ifdef ENABLE_DOUBLE_PRECISION
    return 1;
#else
    return 0;
#endif
}

int ref_smooth_factor_is(double *eps) { *eps = (double)MRI_SMOOTH_FACTOR; return 0; }

// Loads `idir` with the reference reader and reports its sizes.
int ref_dir_dims(const char *idir, int *num_k, int *num_i, int *num_coil, int *num_slices) {
    ensure_timer();
    FLOAT_T version; int ns, nk, ni, nc, Nx = 0, Ny = 0, Nz = 1;
    DataTrajArray ktraj, itraj;
    TArray<FLOAT_T> kr, ki, ir, ii, sr, si, fm, t;
    CooMatrix c;
    loadInputData(std::string(idir), version, ns, nk, ni, nc, ktraj, itraj, kr, ki, ir, ii,
                  sr, si, fm, t, c, false, Nx, Ny, Nz);
    *num_k = nk; *num_i = ni; *num_coil = nc; *num_slices = ns;
    return 0;
}

// Runs the reference brute-force recon of every slice in `idir` (the CPU branch
// of bruteForce(), main_mri.cu:925-948).  out_r/out_i receive num_slices*num_i.
int ref_bf_recon_dir(const char *idir, int cg_num, int fd, double fdp, int tv, int tv_num,
                     double *out_r, double *out_i, int out_len) {
    ensure_timer();
    FLOAT_T version; int ns, nk, ni, nc, Nx = 0, Ny = 0, Nz = 1;
    DataTrajArray ktraj, itraj;
    TArray<FLOAT_T> kr, ki, ir, ii, sr, si, fm, t;
    CooMatrix c;
    loadInputData(std::string(idir), version, ns, nk, ni, nc, ktraj, itraj, kr, ki, ir, ii,
                  sr, si, fm, t, c, false, Nx, Ny, Nz);
    if (out_len < ns * ni) return -1;
    for (int s = 0; s < ns; ++s) {
        FLOAT_T *xr = ir.array + s * ni, *xi = ii.array + s * ni;
        bruteForceCpu(&xr, &xi, kr.array + s * nk, ki.array + s * nk, ktraj.array, itraj.array,
                      fm.array + s * ni, t.array, &c, cg_num, nk, ni, false, fd != 0,
                      (FLOAT_T)fdp, tv != 0, tv_num, sr.array, si.array, nc);
    }
    for (int i = 0; i < ns * ni; ++i) { out_r[i] = ir.array[i]; out_i[i] = ii.array[i]; }
    return 0;
}

// SENSE forward NUDFT: out[c*num_k + k] (parImagingCpu.cpp:84).
void ref_parallel_ft(double *out_r, double *out_i, const double *x_r, const double *x_i,
                     const double *kx, const double *ky, const double *kz,
                     const double *ix, const double *iy, const double *iz,
                     const double *fm, const double *t, int num_k, int num_i,
                     const double *s_r, const double *s_i, int num_coil) {
    ensure_timer();
    std::vector<DataTraj> kt(num_k), it(num_i);
    fill_traj(kt.data(), kx, ky, kz, num_k);
    fill_traj(it.data(), ix, iy, iz, num_i);
    auto xr = to_ft(x_r, num_i), xi = to_ft(x_i, num_i), f = to_ft(fm, num_i), tt = to_ft(t, num_k);
    auto sr = to_ft(s_r, num_i * num_coil), si = to_ft(s_i, num_i * num_coil);
    std::vector<FLOAT_T> o_r(num_k * num_coil), o_i(num_k * num_coil);
    parallelFtCpu(o_r.data(), o_i.data(), xr.data(), xi.data(), kt.data(), it.data(), f.data(),
                  tt.data(), num_k, num_i, sr.data(), si.data(), num_coil);
    for (int i = 0; i < num_k * num_coil; ++i) { out_r[i] = o_r[i]; out_i[i] = o_i[i]; }
}

// SENSE adjoint NUDFT with coil combination (parImagingCpu.cpp:119).
void ref_parallel_ift(double *out_r, double *out_i, const double *d_r, const double *d_i,
                      const double *kx, const double *ky, const double *kz,
                      const double *ix, const double *iy, const double *iz,
                      const double *fm, const double *t, int num_k, int num_i,
                      const double *s_r, const double *s_i, int num_coil) {
    ensure_timer();
    std::vector<DataTraj> kt(num_k), it(num_i);
    fill_traj(kt.data(), kx, ky, kz, num_k);
    fill_traj(it.data(), ix, iy, iz, num_i);
    auto dr = to_ft(d_r, num_k * num_coil), di = to_ft(d_i, num_k * num_coil);
    auto f = to_ft(fm, num_i), tt = to_ft(t, num_k);
    auto sr = to_ft(s_r, num_i * num_coil), si = to_ft(s_i, num_i * num_coil);
    std::vector<FLOAT_T> o_r(num_i), o_i(num_i);
    parallelIftCpu(o_r.data(), o_i.data(), dr.data(), di.data(), kt.data(), it.data(), f.data(),
                   tt.data(), num_k, num_i, sr.data(), si.data(), num_coil);
    for (int i = 0; i < num_i; ++i) { out_r[i] = o_r[i]; out_i[i] = o_i[i]; }
}

// lambda * D^H W D p on a num_row x num_col periodic grid (DHWD2dCpu.cpp:94).
void ref_dhwd2d(double *s_r, double *s_i, const double *p_r, const double *p_i, const double *w,
                int num_row, int num_col, double lambda) {
    ensure_timer();
    int n = num_row * num_col;
    auto pr = to_ft(p_r, n), pi = to_ft(p_i, n), ww = to_ft(w, n);
    std::vector<FLOAT_T> o_r(n), o_i(n);
    DHWD2dCpu(o_r.data(), o_i.data(), pr.data(), pi.data(), ww.data(), num_row, num_col,
              (FLOAT_T)lambda);
    for (int i = 0; i < n; ++i) { s_r[i] = o_r[i]; s_i[i] = o_i[i]; }
}

// Brute-force CG from in-memory arrays; x is the initial estimate and the result.
void ref_bf_cg(double *x_r, double *x_i, const double *kd_r, const double *kd_i,
               const double *kx, const double *ky, const double *kz,
               const double *ix, const double *iy, const double *iz,
               const double *fm, const double *t, int num_k, int num_i,
               const double *s_r, const double *s_i, int num_coil,
               int cg_num, int fd, double fdp, int tv, int tv_num) {
    ensure_timer();
    std::vector<DataTraj> kt(num_k), it(num_i);
    fill_traj(kt.data(), kx, ky, kz, num_k);
    fill_traj(it.data(), ix, iy, iz, num_i);
    auto xr = to_ft(x_r, num_i), xi = to_ft(x_i, num_i);
    auto kr = to_ft(kd_r, num_k * num_coil), ki = to_ft(kd_i, num_k * num_coil);
    auto f = to_ft(fm, num_i), tt = to_ft(t, num_k);
    auto sr = to_ft(s_r, num_i * num_coil), si = to_ft(s_i, num_i * num_coil);
    CooMatrix c;
    FLOAT_T *pxr = xr.data(), *pxi = xi.data();
    bruteForceCpu(&pxr, &pxi, kr.data(), ki.data(), kt.data(), it.data(), f.data(), tt.data(), &c,
                  cg_num, num_k, num_i, false, fd != 0, (FLOAT_T)fdp, tv != 0, tv_num,
                  sr.data(), si.data(), num_coil);
    for (int i = 0; i < num_i; ++i) { x_r[i] = xr[i]; x_i[i] = xi[i]; }
}

// The same with -reg: the roughness matrix C (COO, 0-based) replaces the
// finite-difference term (bruteForceCpu.cpp:306-380).
void ref_bf_cg_reg(double *x_r, double *x_i, const double *kd_r, const double *kd_i,
                   const double *kx, const double *ky, const double *kz,
                   const double *ix, const double *iy, const double *iz,
                   const double *fm, const double *t, int num_k, int num_i,
                   const double *s_r, const double *s_i, int num_coil,
                   int cg_num, double fdp, int tv, int tv_num,
                   int c_rows, int c_cols, int c_nnz, const int *c_i, const int *c_j,
                   const double *c_v) {
    ensure_timer();
    std::vector<DataTraj> kt(num_k), it(num_i);
    fill_traj(kt.data(), kx, ky, kz, num_k);
    fill_traj(it.data(), ix, iy, iz, num_i);
    auto xr = to_ft(x_r, num_i), xi = to_ft(x_i, num_i);
    auto kr = to_ft(kd_r, num_k * num_coil), ki = to_ft(kd_i, num_k * num_coil);
    auto f = to_ft(fm, num_i), tt = to_ft(t, num_k);
    auto sr = to_ft(s_r, num_i * num_coil), si = to_ft(s_i, num_i * num_coil);
    auto cv = to_ft(c_v, c_nnz);
    CooMatrix c(c_rows, c_cols, c_nnz, c_i, c_j, cv.data());
    FLOAT_T *pxr = xr.data(), *pxi = xi.data();
    bruteForceCpu(&pxr, &pxi, kr.data(), ki.data(), kt.data(), it.data(), f.data(), tt.data(), &c,
                  cg_num, num_k, num_i, true, false, (FLOAT_T)fdp, tv != 0, tv_num,
                  sr.data(), si.data(), num_coil);
    for (int i = 0; i < num_i; ++i) { x_r[i] = xr[i]; x_i[i] = xi[i]; }
}

}  // extern "C"

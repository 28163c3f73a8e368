// Directory-level drop-in of the reference's toeplitz() driver
// (main_mri.cuh:97-108, main_mri.cu:207-630): reads an mriSolver input
// directory, computes Q (gridded, direct, or reused from Q_stone.file) and
// F^H d, runs the Toeplitz CG, and writes Q_stone.file (-writeQ), FhD.file and
// out.file into the input directory as the reference does.
//
// File formats (byte-compatible with the reference):
//   Q_stone.file  for l = 0..L: Re(Q_l) float32 x G, Im(Q_l) float32 x G
//                 (toeplitz/computeQ.cmem.cu:280-300, read back by
//                 matrix_t::read_pack, toeplitz/utils.cpp:168-214)
//   FhD.file      Re(F^H d) float32 x N, Im x N   (computeFH.cmem.cu:314-321)
//   out.file      Re(x) float32 x N, Im x N       (recon.cu:2150-2165)
#include "../../include/impatient_b200.h"
#include "context.h"
#include "io.h"

#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <sys/stat.h>
#include <vector>

namespace {

int read_q_file(const std::string &fn, size_t per_seg, int segs, std::vector<float> &qr,
                std::vector<float> &qi) {
    struct stat sb;
    if (stat(fn.c_str(), &sb) != 0) {
        std::fprintf(stderr, "Error: bad directory path that contains the Q file (%s)\n", fn.c_str());
        return IMP_ERR_IO;
    }
    if ((size_t)sb.st_size != per_seg * segs * 2 * sizeof(float)) {
        std::fprintf(stderr, "Error: incorrect Q file size\n");
        return IMP_ERR_FORMAT;
    }
    FILE *f = std::fopen(fn.c_str(), "rb");
    if (!f) return IMP_ERR_IO;
    qr.resize(per_seg * segs);
    qi.resize(per_seg * segs);
    bool ok = true;
    for (int l = 0; l < segs && ok; ++l) {
        ok = std::fread(qr.data() + l * per_seg, 4, per_seg, f) == per_seg &&
             std::fread(qi.data() + l * per_seg, 4, per_seg, f) == per_seg;
    }
    std::fclose(f);
    return ok ? IMP_OK : IMP_ERR_FORMAT;
}

int write_pairs(const std::string &fn, const std::vector<float> &re, const std::vector<float> &im,
                size_t per_seg, int segs) {
    FILE *f = std::fopen(fn.c_str(), "wb");
    if (!f) {
        std::fprintf(stderr, "Error: cannot write %s\n", fn.c_str());
        return IMP_ERR_IO;
    }
    bool ok = true;
    for (int l = 0; l < segs && ok; ++l)
        ok = std::fwrite(re.data() + l * per_seg, 4, per_seg, f) == per_seg &&
             std::fwrite(im.data() + l * per_seg, 4, per_seg, f) == per_seg;
    std::fclose(f);
    return ok ? IMP_OK : IMP_ERR_IO;
}

float hanning_host(float t, float tau, int l, float t0) {
    const float x = t - tau * (float)l - t0;
    return std::fabs(x) < tau ? 0.5f + 0.5f * std::cos(3.1415926535897932f * x / tau) : 0.f;
}

// Direct Q_l = sum_k h_l(t_k) exp(+i 2 pi k.r) on the 2N grid through the
// NUDFT engine (non-cumulative over l; the reference's direct Q accumulates
// across segments, toeplitz/computeQ.cmem.cu:190,911-964, which is not kept).
int direct_q(imp_context *ctx, const imp::Dataset &ds, int Nx, int Ny, int Nz, int L, float tau,
             float t0, std::vector<float> &qr, std::vector<float> &qi) {
    const bool is3d = Nz > 1;
    std::vector<float> px, py, pz;
    if (!is3d) {
        for (int x = -Nx; x < Nx; ++x)
            for (int y = -Ny; y < Ny; ++y) {
                px.push_back((float)x / Nx);
                py.push_back((float)y / Ny);
                pz.push_back(0.f);
            }
    } else {
        for (int y = -Ny; y < Ny; ++y)
            for (int x = -Nx; x < Nx; ++x)
                for (int z = -Nz; z < Nz; ++z) {
                    px.push_back((float)x / Nx);
                    py.push_back((float)y / Ny);
                    pz.push_back((float)z / Nz);
                }
    }
    const size_t G = px.size(), M = ds.num_k;
    qr.assign(G * (L + 1), 0.f);
    qi.assign(G * (L + 1), 0.f);
    std::vector<float> h(M), zero(M, 0.f);
    for (int l = 0; l <= L; ++l) {
        for (size_t k = 0; k < M; ++k) h[k] = hanning_host(ds.t[k], tau, l, t0);
        // the operator entry points take device pointers
        float *d[9];
        const std::vector<float> *src[9] = {&h, &zero, &ds.kx, &ds.ky, &ds.kz, &px, &py, &pz, &ds.t};
        for (int i = 0; i < 9; ++i) {
            if (cudaMalloc(&d[i], src[i]->size() * 4) != cudaSuccess) return IMP_ERR_NOMEM;
            cudaMemcpy(d[i], src[i]->data(), src[i]->size() * 4, cudaMemcpyHostToDevice);
        }
        float *outr, *outi;
        cudaMalloc(&outr, G * 4);
        cudaMalloc(&outi, G * 4);
        imp_status s = imp_ift(ctx, outr, outi, d[0], d[1], d[2], d[3], d[4], d[5], d[6], d[7],
                               nullptr, d[8], (int)M, (int)G, is3d ? 1 : 0);
        if (s == IMP_OK) {
            cudaMemcpy(qr.data() + l * G, outr, G * 4, cudaMemcpyDeviceToHost);
            cudaMemcpy(qi.data() + l * G, outi, G * 4, cudaMemcpyDeviceToHost);
        }
        for (int i = 0; i < 9; ++i) cudaFree(d[i]);
        cudaFree(outr);
        cudaFree(outi);
        if (s != IMP_OK) return s;
    }
    return IMP_OK;
}

// Direct F^H d: exact adjoint NUDFT with field map and SENSE (ComputeFH_GPU_BF,
// toeplitz/computeFH.cmem.cu:155-200).
int direct_fhd(imp_context *ctx, const imp::Dataset &ds, bool is3d, std::vector<float> &fr,
               std::vector<float> &fi) {
    const size_t N = ds.num_i, M = ds.num_k, C = ds.num_coil;
    const std::vector<float> *src[11] = {&ds.kdata_r, &ds.kdata_i, &ds.kx,      &ds.ky,
                                         &ds.kz,      &ds.ix,      &ds.iy,      &ds.iz,
                                         &ds.fm,      &ds.t,       &ds.sensi_r};
    const size_t cnt[11] = {C * M, C * M, M, M, M, N, N, N, N, M, C * N};
    float *d[12];
    for (int i = 0; i < 11; ++i) {
        if (cudaMalloc(&d[i], cnt[i] * 4) != cudaSuccess) return IMP_ERR_NOMEM;
        cudaMemcpy(d[i], src[i]->data(), cnt[i] * 4, cudaMemcpyHostToDevice);
    }
    cudaMalloc(&d[11], C * N * 4);
    cudaMemcpy(d[11], ds.sensi_i.data(), C * N * 4, cudaMemcpyHostToDevice);
    float *outr, *outi;
    cudaMalloc(&outr, N * 4);
    cudaMalloc(&outi, N * 4);
    imp_status s = imp_parallel_ift(ctx, outr, outi, d[0], d[1], d[2], d[3], d[4], d[5], d[6],
                                    d[7], d[8], d[9], (int)M, (int)N, d[10], d[11], (int)C,
                                    is3d ? 1 : 0);
    fr.resize(N);
    fi.resize(N);
    if (s == IMP_OK) {
        cudaMemcpy(fr.data(), outr, N * 4, cudaMemcpyDeviceToHost);
        cudaMemcpy(fi.data(), outi, N * 4, cudaMemcpyDeviceToHost);
    }
    for (float *p : d) cudaFree(p);
    cudaFree(outr);
    cudaFree(outi);
    return s;
}

}  // namespace

extern "C" imp_status imp_toeplitz_dir(const char *idir, const imp_toeplitz_options *opt,
                                       int direct, int gpu_id, int reuseQ, const char *Qdir,
                                       int writeQ) {
    if (!idir || !opt) return IMP_ERR_INVALID_ARG;
    imp::Dataset ds;
    std::string err;
    int st = imp::load_input_dir(idir, ds, err);
    if (st != IMP_OK) {
        std::fprintf(stderr, "Error: %s\n", err.c_str());
        return st;
    }
    // image size as the reference derives it (main_mri.cu:300-312)
    const int Nz = ds.version >= 1.0f ? std::max(ds.nz, 1) : 1;
    const int Ny = (int)std::sqrt((double)(ds.num_i / Nz));
    const int Nx = Ny;
    if ((long)Nx * Ny * Nz != ds.num_i) {
        std::fprintf(stderr, "Error: the Toeplitz path needs a square (Ny = Nx) image\n");
        return IMP_ERR_INVALID_ARG;
    }
    if (ds.num_slices != 1)
        std::fprintf(stderr, "mriSolver: Toeplitz path reconstructs the first slice only\n");
    const int L = (int)opt->ntime_segs;
    const float tau = opt->ntime_segs > 0.f ? (ds.t[ds.num_k - 1] - ds.t[0]) / opt->ntime_segs
                                            : (ds.t[ds.num_k - 1] - ds.t[0]);
    const float t0 = ds.t[0];
    std::printf("  Recon method           : Toeplitz with %s for Q and FHD (B200)\n",
                direct ? "direct evaluation" : "gridding");
    std::printf("  Image data size (yxz)  : (%d,%d,%d)\n", Ny, Nx, Nz);
    std::printf("  Number of coils        : %d\n", ds.num_coil);
    std::printf("  K-space data size/coil : %d\n", ds.num_k);
    std::printf("  Number of CG iterations: %d\n", opt->cg_num);
    std::printf("  Number of time segments: %f\n", opt->ntime_segs);
    imp_context *ctx = nullptr;
    if ((st = imp_context_create(gpu_id, &ctx)) != IMP_OK) {
        std::fprintf(stderr, "Error: %s\n", imp_last_error());
        return st;
    }
    const size_t G = (size_t)(2 * Nx) * (2 * Ny) * (Nz == 1 ? 1 : 2 * Nz);
    const size_t N = ds.num_i;
    std::vector<float> qr, qi, fr(N), fi(N), xr(N), xi(N);
    const std::string dir(idir);
    const float *kz = ds.kz.data();
    const float *fm = ds.fm.data();
    const float *sr = ds.sensi_r.data(), *si = ds.sensi_i.data();
    // Q of the gridding path stays in device memory between steps 1 and 3
    // (a host copy only for -writeQ); the other paths produce it on the host.
    float *dq = nullptr;
    const float *q_r = nullptr, *q_i = nullptr;
    using clk = std::chrono::steady_clock;
    auto ms_since = [](clk::time_point a) {
        return std::chrono::duration<double, std::milli>(clk::now() - a).count();
    };
    do {
        std::printf("======== Step 1. Compute Q matrices: Q[%d] ========\n", L + 1);
        const auto tq = clk::now();
        if (reuseQ) {
            std::string qdir = Qdir ? Qdir : dir;
            std::printf("  Re-using the Q at %s/Q_stone.file\n", qdir.c_str());
            if ((st = read_q_file(qdir + "/Q_stone.file", G, L + 1, qr, qi)) != IMP_OK) break;
        } else if (direct) {
            if ((st = direct_q(ctx, ds, Nx, Ny, Nz, L, tau, t0, qr, qi)) != IMP_OK) break;
        } else {
            const size_t nq = G * (L + 1);
            if (cudaSetDevice(gpu_id) != cudaSuccess ||
                cudaMalloc(&dq, 2 * nq * sizeof(float)) != cudaSuccess) {
                std::fprintf(stderr, "Error: no device memory for Q (%zu bytes)\n",
                             2 * nq * sizeof(float));
                st = IMP_ERR_NOMEM;
                break;
            }
            if ((st = imp_toeplitz_q(ctx, opt, dq, dq + nq, ds.kx.data(), ds.ky.data(), kz,
                                     ds.t.data(), ds.num_k, Nx, Ny, Nz)) != IMP_OK)
                break;
            q_r = dq;
            q_i = dq + nq;
            if (writeQ) {
                qr.resize(nq);
                qi.resize(nq);
                if (cudaMemcpy(qr.data(), q_r, nq * sizeof(float), cudaMemcpyDeviceToHost) !=
                        cudaSuccess ||
                    cudaMemcpy(qi.data(), q_i, nq * sizeof(float), cudaMemcpyDeviceToHost) !=
                        cudaSuccess) {
                    std::fprintf(stderr, "Error: Q device-to-host copy failed\n");
                    st = IMP_ERR_CUDA;
                    break;
                }
            }
        }
        if (!q_r) {
            q_r = qr.data();
            q_i = qi.data();
        }
        std::printf("  GPU: Q Kernel Time: %f (ms)\n", ms_since(tq));
        if (writeQ && !reuseQ &&
            (st = write_pairs(dir + "/Q_stone.file", qr, qi, G, L + 1)) != IMP_OK)
            break;
        std::printf("======== Step 2. Compute FH ========\n");
        const auto tf = clk::now();
        if (direct) {
            if ((st = direct_fhd(ctx, ds, Nz > 1, fr, fi)) != IMP_OK) break;
        } else if ((st = imp_toeplitz_fhd(ctx, opt, fr.data(), fi.data(), ds.kdata_r.data(),
                                          ds.kdata_i.data(), ds.kx.data(), ds.ky.data(), kz,
                                          ds.t.data(), fm, sr, si, ds.num_k, ds.num_coil, Nx,
                                          Ny, Nz)) != IMP_OK)
            break;
        std::printf("  GPU: F^H(d) Kernel Time: %f (ms)\n", ms_since(tf));
        if ((st = write_pairs(dir + "/FhD.file", fr, fi, N, 1)) != IMP_OK) break;
        std::printf("======== Step 3. Toeplitz CG ========\n");
        const auto tc = clk::now();
        if ((st = imp_toeplitz_recon(ctx, opt, xr.data(), xi.data(), fr.data(), fi.data(), q_r,
                                     q_i, ds.t.data(), ds.num_k, fm, sr, si, ds.num_coil, Nx,
                                     Ny, Nz)) != IMP_OK)
            break;
        std::printf("  GPU: CG Execution Time: %f (ms)\n", ms_since(tc));
        if ((st = write_pairs(dir + "/out.file", xr, xi, N, 1)) != IMP_OK) break;
        std::printf("  GPU: Exporting results to %s/out.file\n", idir);
    } while (false);
    if (st != IMP_OK && st != IMP_ERR_IO && st != IMP_ERR_FORMAT)
        std::fprintf(stderr, "Error: %s\n", imp_last_error());
    if (dq) cudaFree(dq);
    imp_context_destroy(ctx);
    return st;
}

extern "C" imp_status imp_toeplitz_dir_cli(const char *idir, const char *odir, int cg_num,
                                           int enable_fd, float fdp, int enable_tv, int tv_num,
                                           int direct, float gridOS_Q, float gridOS_FH,
                                           float ntime_segs, int gpu_id, int reuseQ,
                                           const char *Qpath, int writeQ,
                                           const imp_sparse *reg) {
    (void)odir;  // the reference writes the Toeplitz outputs into the input directory
    imp_toeplitz_options o;
    imp_toeplitz_options_default(&o);
    o.reg = reg;
    o.cg_num = cg_num;
    o.enable_fd = enable_fd;
    o.fd_penalizer = fdp;
    o.enable_tv = enable_tv;
    o.tv_num = tv_num;
    o.ntime_segs = ntime_segs;
    o.gridOS_Q = gridOS_Q;
    o.gridOS_FH = gridOS_FH;
    return imp_toeplitz_dir(idir, &o, direct, gpu_id, reuseQ, Qpath, writeQ);
}

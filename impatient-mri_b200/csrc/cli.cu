// mriSolver command line (flags, defaults and messages of main.cpp:96-444)
// and the directory-level drop-in of bruteForce() (main_mri.cu:652-1025).
#include "../../include/impatient_b200.h"
#include "context.h"
#include "io.h"

#include <cuda_runtime.h>

#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

namespace {

void usage(FILE *f) {
    std::fprintf(f,
                 "Usage: mriSolver -idir <input dir> [options]\n"
                 "  -odir <dir>            output directory (default <idir>/output)\n"
                 "  -cg_num <n>            CG iteration number (default 8)\n"
                 "  -fd / -fdp <lambda>    finite-difference regularization weight\n"
                 "  -tv, -tv_num <n>       total-variation reweighting (default 10)\n"
                 "  -tv_update             as -tv (per-pass output dumps not written)\n"
                 "  -toeplitzGridding      Toeplitz CG, Q and F^H d by gridding\n"
                 "  -toeplitzDirect        Toeplitz CG, Q and F^H d by direct NUDFT\n"
                 "  -ntime_segs <L>        time segments (Toeplitz, default 12)\n"
                 "  -gridOS_Q <os>         gridding oversampling for Q, [1,2] (default 1.125)\n"
                 "  -gridOS_FH <os>        gridding oversampling for F^H d, [1,2] (default 1.5)\n"
                 "  -reuseQ <dir>, -writeQ reuse / write Q_stone.file (Toeplitz)\n"
                 "  -gpu_id <id>           CUDA device (default 0)\n"
                 "  -bf3d                  brute force with the true 3-D phase and 3-D TV\n"
                 "  -mgpu                  slices spread over every visible GPU (brute force)\n"
                 "  -reg                   roughness regularization with the sparse matrix idir/c.rmtx\n"
                 "  -cpu, -nogpu           not provided by this build\n");
}

}  // namespace

// Work queue of the -mgpu path (bruteForceMgpu, bruteForce/bruteForceMgpu.cu:82,
// started per GPU at main_mri.cu:900; the reference splits the slices into
// contiguous blocks per GPU, main_mri.cu:776-834).  Here every worker thread
// owns one context on its device and claims slices from a shared counter, so
// uneven slices balance; each slice is one imp_bruteforce_recon call on the
// slice's views of the host arrays.
extern "C" imp_status imp_bruteforce_mgpu(const imp_bf_options *opt, float *idata_r,
                                          float *idata_i, const float *kdata_r,
                                          const float *kdata_i, const float *kx,
                                          const float *ky, const float *kz, const float *ix,
                                          const float *iy, const float *iz, const float *fm,
                                          const float *t, const float *sensi_r,
                                          const float *sensi_i, int num_k, int num_i,
                                          int num_coil, int num_slices, const int *devices,
                                          int num_workers) {
    if (!opt || !idata_r || !idata_i || !kdata_r || !kdata_i || num_slices <= 0 ||
        num_k <= 0 || num_i <= 0 || num_coil <= 0)
        return IMP_ERR_INVALID_ARG;
    if (num_workers <= 0) {
        int n = 0;
        if (cudaGetDeviceCount(&n) != cudaSuccess || n <= 0)
            return imp::fail(IMP_ERR_CUDA, "no CUDA device for -mgpu");
        num_workers = n;
    }
    num_workers = std::min(num_workers, num_slices);
    const size_t N = (size_t)num_i, KC = (size_t)num_k * num_coil;
    std::atomic<int> next{0};
    std::atomic<int> failed{IMP_OK};
    std::mutex mu;
    std::string first_msg;
    auto worker = [&](int w) {
        const int dev = devices ? devices[w] : w;
        imp_context *ctx = nullptr;
        imp_status s = imp_context_create(dev, &ctx);
        while (s == IMP_OK && failed.load() == IMP_OK) {
            const int sl = next.fetch_add(1);
            if (sl >= num_slices) break;
            s = imp_bruteforce_recon(ctx, opt, idata_r + sl * N, idata_i + sl * N,
                                     kdata_r + sl * KC, kdata_i + sl * KC, kx, ky, kz, ix, iy,
                                     iz, fm ? fm + sl * N : nullptr, t, sensi_r, sensi_i, num_k,
                                     num_i, num_coil, 1);
        }
        if (s != IMP_OK) {
            std::lock_guard<std::mutex> lk(mu);
            int expect = IMP_OK;
            if (failed.compare_exchange_strong(expect, s))
                first_msg = "GPU " + std::to_string(dev) + ": " + imp_last_error();
        }
        imp_context_destroy(ctx);
    };
    std::vector<std::thread> pool;
    for (int w = 0; w < num_workers; ++w) pool.emplace_back(worker, w);
    for (std::thread &th : pool) th.join();
    const int s = failed.load();
    return s == IMP_OK ? IMP_OK : imp::fail((imp_status)s, first_msg);  // message in this thread
}

extern "C" imp_status imp_bruteforce_dir(const char *idir, const char *odir,
                                         const imp_bf_options *opt, int gpu_id) {
    if (!idir || !odir || !opt) return IMP_ERR_INVALID_ARG;
    imp::Dataset ds;
    std::string err;
    int st = imp::load_input_dir(idir, ds, err);
    if (st != IMP_OK) {
        std::fprintf(stderr, "Error: %s\n", err.c_str());
        return st;
    }
    imp_bf_options o = *opt;
    if (o.use_z) {
        if (ds.nx <= 0 || ds.ny <= 0 || ds.nz <= 0 || (long)ds.nx * ds.ny * ds.nz != ds.num_i) {
            std::fprintf(stderr, "Error: -bf3d needs x/y/zDimension headers matching the image\n");
            return IMP_ERR_INVALID_ARG;
        }
        o.nx = ds.nx;
        o.ny = ds.ny;
        o.nz = ds.nz;
    }
    std::printf("  Recon method           : Brute Force (B200)\n");
    std::printf("  Input folder           : %s\n", idir);
    std::printf("  Output folder          : %s\n", odir);
    std::printf("  Number of coils        : %d\n", ds.num_coil);
    std::printf("  Number of slices       : %d\n", ds.num_slices);
    std::printf("  Image data size        : %d\n", ds.num_i);
    std::printf("  K-space data size      : %d\n", ds.num_k);
    std::printf("  Number of CG iterations: %d\n", o.cg_num);
    if (o.enable_fd) std::printf("  FD penalizer value     : %f\n", o.fd_penalizer);
    if (o.enable_tv) std::printf("  Number of TV iterations: %d\n", o.tv_num);
    if (gpu_id < 0) {  // -mgpu
        int n = 0;
        if (cudaGetDeviceCount(&n) != cudaSuccess) n = 0;
        std::printf("  Number of online GPUs  : %d\n", n);
        st = imp_bruteforce_mgpu(&o, ds.idata_r.data(), ds.idata_i.data(), ds.kdata_r.data(),
                                 ds.kdata_i.data(), ds.kx.data(), ds.ky.data(), ds.kz.data(),
                                 ds.ix.data(), ds.iy.data(), ds.iz.data(), ds.fm.data(),
                                 ds.t.data(), ds.sensi_r.data(), ds.sensi_i.data(), ds.num_k,
                                 ds.num_i, ds.num_coil, ds.num_slices, nullptr, 0);
    } else {
        imp_context *ctx = nullptr;
        st = imp_context_create(gpu_id, &ctx);
        if (st != IMP_OK) {
            std::fprintf(stderr, "Error: %s\n", imp_last_error());
            return st;
        }
        st = imp_bruteforce_recon(ctx, &o, ds.idata_r.data(), ds.idata_i.data(),
                                  ds.kdata_r.data(), ds.kdata_i.data(), ds.kx.data(),
                                  ds.ky.data(), ds.kz.data(), ds.ix.data(), ds.iy.data(),
                                  ds.iz.data(), ds.fm.data(), ds.t.data(), ds.sensi_r.data(),
                                  ds.sensi_i.data(), ds.num_k, ds.num_i, ds.num_coil,
                                  ds.num_slices);
        imp_context_destroy(ctx);
    }
    if (st != IMP_OK) {
        std::fprintf(stderr, "Error: %s\n", imp_last_error());
        return st;
    }
    if ((st = imp::make_dirs(odir, err)) != IMP_OK ||
        (st = imp::export_text(std::string(odir) + "/output_gpu_r.dat", ds.idata_r.data(),
                               (size_t)ds.num_slices * ds.num_i, err)) != IMP_OK ||
        (st = imp::export_text(std::string(odir) + "/output_gpu_i.dat", ds.idata_i.data(),
                               (size_t)ds.num_slices * ds.num_i, err)) != IMP_OK) {
        std::fprintf(stderr, "Error: %s\n", err.c_str());
        return st;
    }
    return IMP_OK;
}

extern "C" imp_status imp_dataset_info(const char *idir, int *num_k, int *num_i, int *num_coil,
                                       int *num_slices, int *nx, int *ny, int *nz) {
    if (!idir) return IMP_ERR_INVALID_ARG;
    imp::Dataset ds;
    std::string err;
    const int st = imp::load_input_dir(idir, ds, err);
    if (st != IMP_OK) {
        std::fprintf(stderr, "Error: %s\n", err.c_str());
        return st;
    }
    if (num_k) *num_k = ds.num_k;
    if (num_i) *num_i = ds.num_i;
    if (num_coil) *num_coil = ds.num_coil;
    if (num_slices) *num_slices = ds.num_slices;
    if (nx) *nx = ds.nx;
    if (ny) *ny = ds.ny;
    if (nz) *nz = ds.nz;
    return IMP_OK;
}

// Declared in the Toeplitz translation unit.
extern "C" imp_status imp_toeplitz_dir_cli(const char *idir, const char *odir, int cg_num,
                                           int enable_fd, float fdp, int enable_tv, int tv_num,
                                           int direct, float gridOS_Q, float gridOS_FH,
                                           float ntime_segs, int gpu_id, int reuseQ,
                                           const char *Qpath, int writeQ,
                                           const imp_sparse *reg);

extern "C" int imp_mrisolver_main(int argc, char **argv) {
    std::string idir, odir;
    bool have_idir = false, have_odir = false;
    int cg_num = 8, tv_num = 10, gpu_id = 0;
    bool nogpu = false, mgpu = false, cpu = false, reg = false, fd = false, tv = false;
    bool tgrid = false, tdirect = false, reuseQ = false, writeQ = false, bf3d = false;
    float fdp = 0.f, ntime = 12.f, osQ = 1.125f, osFH = 1.5f;
    std::string Qloc;
    bool fdp_given = false;

    if (argc > 1) {
        std::printf("mriSolver: Command options: ");
        for (int i = 1; i < argc; ++i) std::printf("%s ", argv[i]);
        std::printf("\n");
    }
    auto value = [&](int &i) -> const char * {
        ++i;
        if (i < argc && argv[i] && argv[i][0] != '-') return argv[i];
        return nullptr;
    };
    for (int i = 1; i < argc; ++i) {
        const char *a = argv[i];
        const char *v;
        if (!std::strcmp(a, "-idir")) {
            if (!(v = value(i))) { std::fprintf(stderr, "\nError: Missing input directory name.\n"); return 1; }
            idir = v;
            have_idir = true;
        } else if (!std::strcmp(a, "-odir")) {
            if (!(v = value(i))) { std::fprintf(stderr, "\nError: Missing output directory name.\n"); return 1; }
            odir = v;
            have_odir = true;
        } else if (!std::strcmp(a, "-gpu_id")) {
            if (!(v = value(i)) || std::atoi(v) < 0) { std::fprintf(stderr, "\nError: invalid GPU device ID.\n"); return 1; }
            gpu_id = std::atoi(v);
        } else if (!std::strcmp(a, "-cg_num")) {
            if (!(v = value(i)) || std::atoi(v) == 0) { std::fprintf(stderr, "\nError: Zero or wrong CG iteration number format.\n"); return 1; }
            cg_num = std::atoi(v);
        } else if (!std::strcmp(a, "-nogpu")) {
            nogpu = true;
        } else if (!std::strcmp(a, "-mgpu")) {
            mgpu = true;
        } else if (!std::strcmp(a, "-cpu")) {
            cpu = true;
        } else if (!std::strcmp(a, "-reg")) {
            reg = true;
        } else if (!std::strcmp(a, "-fd")) {
            fd = true;
        } else if (!std::strcmp(a, "-bf3d")) {
            bf3d = true;
        } else if (!std::strcmp(a, "-toeplitzGridding")) {
            tgrid = true;
            tdirect = false;
            nogpu = mgpu = cpu = false;
        } else if (!std::strcmp(a, "-toeplitzDirect")) {
            tdirect = true;
            tgrid = false;
            nogpu = mgpu = cpu = false;
        } else if (!std::strcmp(a, "-reuseQ")) {
            if (!(tgrid || tdirect) || !(v = value(i))) {
                std::fprintf(stderr, "\nError: -reuseQ flag requires toeplitz strategy to turn on.\n");
                return 1;
            }
            reuseQ = true;
            Qloc = v;
        } else if (!std::strcmp(a, "-writeQ")) {
            writeQ = true;
        } else if (!std::strcmp(a, "-ntime_segs")) {
            if (!(tgrid || tdirect) || !(v = value(i))) {
                std::fprintf(stderr, "\nError:-toeplitz flag is not found or invalid number of time segments.\n");
                return 1;
            }
            ntime = (float)std::atof(v);
            if (ntime < 1.f) {
                std::fprintf(stderr, "\nError: number of time segments has to be a natural number in floating format.\n");
                return 1;
            }
        } else if (!std::strcmp(a, "-gridOS_Q") || !std::strcmp(a, "-gridOS_FH")) {
            const bool q = !std::strcmp(a, "-gridOS_Q");
            if (!tgrid || !(v = value(i))) {
                std::fprintf(stderr, "\nError:-toeplitzGridding flag is not found or invalid gridding OS factor.\n");
                return 1;
            }
            const float os = (float)std::atof(v);
            if (os < 1.f || os > 2.f) {
                std::fprintf(stderr, "\nError: gridding oversampling factor should be in [1.0,2.0].\n");
                return 1;
            }
            (q ? osQ : osFH) = os;
        } else if (!std::strcmp(a, "-fdp")) {
            if (!(v = value(i))) { std::fprintf(stderr, "\nError: Missing finite difference penalty.\n"); return 1; }
            fd = true;
            fdp = (float)std::atof(v);
            fdp_given = true;
        } else if (!std::strcmp(a, "-tv")) {
            tv = true;
        } else if (!std::strcmp(a, "-tv_num")) {
            if (!(v = value(i)) || std::atoi(v) == 0) { std::fprintf(stderr, "\nError: Zero or wrong TV iteration number format.\n"); return 1; }
            tv = true;
            tv_num = std::atoi(v);
        } else if (!std::strcmp(a, "-tv_update")) {
            tv = true;
        } else if (!std::strcmp(a, "-version")) {
            std::printf("mriSolver (IMPATIENT MRI B200 rebuild), ABI %d\n", imp_abi_version());
            return 1;
        } else if (!std::strcmp(a, "-help")) {
            usage(stderr);
            return 1;
        } else {
            std::fprintf(stderr, "\nError: Unknown option \"%s\"\n", a);
            usage(stderr);
            return 1;
        }
    }
    if (argc == 1) {
        usage(stderr);
        return 1;
    }
    if (!have_idir) {
        std::fprintf(stderr, "\nError: Missing input directory name.\n");
        return 1;
    }
    if (!have_odir) {
        odir = idir + "/output";
        std::fprintf(stderr, "mriSolver: Using default output directory name \"%s\".\n", odir.c_str());
    }
    if ((fd || tv) && !fdp_given) {
        std::fprintf(stderr, "\n Error: Regularization enabled, but no weight parameter specified. Hint: -fdp [lambda].\n");
        return 1;
    }
    // -reg: the roughness matrix C from idir/c.rmtx (kernels/structures.cpp:722-735);
    // it takes precedence over -fd, which the reference only warns about
    // (main.cpp:374-381)
    imp::SparseCoo rc;
    imp_sparse rs{};
    if (reg) {
        if (fd) std::printf("mriSolver: Error: Roughness regularization and finite difference are exclusive.\n");
        std::printf("mriSolver: Enable roughness regularization.\n");
        std::string err;
        if (imp::read_mtx(idir + "/c.rmtx", rc, err) != IMP_OK) {
            std::fprintf(stderr, "\nError: %s\n", err.c_str());
            return 1;
        }
        rs.rows = rc.rows;
        rs.cols = rc.cols;
        rs.nnz = (int)rc.val.size();
        rs.row = rc.row.data();
        rs.col = rc.col.data();
        rs.val = rc.val.data();
    }
    if (nogpu || cpu) {
        std::fprintf(stderr, "\nError: -cpu / -nogpu: this build has no CPU reconstruction path.\n");
        return 1;
    }
    if (mgpu && (tgrid || tdirect))
        std::printf("mriSolver: -mgpu applies to the brute-force path; Toeplitz runs on GPU %d.\n",
                    gpu_id);
    imp_status st;
    if (tgrid || tdirect) {
        st = imp_toeplitz_dir_cli(idir.c_str(), odir.c_str(), cg_num, fd, fdp, tv, tv_num,
                                  tdirect ? 1 : 0, osQ, osFH, ntime, gpu_id, reuseQ ? 1 : 0,
                                  Qloc.c_str(), writeQ ? 1 : 0, reg ? &rs : nullptr);
    } else {
        imp_bf_options o;
        imp_bf_options_default(&o);
        o.cg_num = cg_num;
        o.enable_fd = fd;
        o.fd_penalizer = fdp;
        o.enable_tv = tv;
        o.tv_num = tv_num;
        o.use_z = bf3d;
        o.reg = reg ? &rs : nullptr;
        st = imp_bruteforce_dir(idir.c_str(), odir.c_str(), &o, mgpu ? -1 : gpu_id);
    }
    if (st != IMP_OK) {
        std::fprintf(stderr, "Error: Failed to execute the mriSolver.\n");
        return 1;
    }
    return 0;
}

// Allocation-free variant of the SENSE adjoint NUDFT (imp_parallel_ift).
//
// Some callers cannot call cudaMalloc: a reconstruction host that reserves all
// device memory through its own allocator when it starts, or runs under a fixed
// device-memory budget, must not have a library allocate behind its back.  This
// entry point needs no context and allocates nothing: the work memory of the
// adjoint -- packed trajectory and voxel geometry, packed coil sensitivities,
// packed k-space data and the per-split partial sums -- lives in one file-scope
// device array of kNoAllocBytes (32 MiB), which every GPU that loads this
// library holds until the process exits.  The caller passes the inputs and the
// output only.
//
// Host code cannot use the array's name as a device address (in host code it
// names a host-side stand-in), so the address is looked up with
// cudaGetSymbolAddress once per device, with that device current, on the first
// call made on that device, and kept for the life of the process (a
// cudaDeviceReset ends the context that address belongs to, so this entry
// point must not be used after one).  Every call shares the array and it keeps
// the previous call's contents: the error word is cleared at the start of each
// call and every other region is fully rewritten before it is read.  Calls
// that overlap on the GPU (from two streams or two host threads) race on the
// array.  Every return, failures included, comes after the stream has drained
// the call's own work, so a failed call leaves nothing queued on the array.
// Failures set the message that imp_last_error() returns, as every other entry
// point does.
#include "../../include/impatient_b200.h"
#include "common.cuh"
#include "context.h"
#include "nudft.cuh"

#include <string>

#include <cstdio>
#include <mutex>

namespace {
constexpr size_t kNoAllocBytes = size_t(32) << 20;
constexpr size_t kAlign = 256;
}  // namespace

// The work memory of every call, on every GPU that loads the library.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

namespace {

std::mutex g_mu;
void *g_addr[256] = {};  // device address of g_noalloc_scratch per device ordinal

size_t up(size_t b) { return (b + kAlign - 1) / kAlign * kAlign; }

// Sets up (once per device, with that device current) the device address of
// the scratch array.
imp_status scratch_address(int device, unsigned char **out) {
    if (device < 0 || device >= 256)
        return imp::fail(IMP_ERR_INVALID_ARG, "imp_parallel_ift_noalloc: device ordinal " +
                                                  std::to_string(device) + " out of range");
    std::lock_guard<std::mutex> g(g_mu);
    if (!g_addr[device]) {
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            cudaGetLastError();
            return imp::fail(IMP_ERR_CUDA,
                             std::string("imp_parallel_ift_noalloc: cudaGetSymbolAddress: ") +
                                 cudaGetErrorString(e));
        }
        g_addr[device] = p;
    }
    *out = (unsigned char *)g_addr[device];
    return IMP_OK;
}

}  // namespace

extern "C" imp_status imp_parallel_ift_noalloc(
    float *idata_r, float *idata_i, const float *kdata_r, const float *kdata_i, const float *kx,
    const float *ky, const float *kz, const float *ix, const float *iy, const float *iz,
    const float *fm, const float *t, int num_k, int num_i, const float *sensi_r,
    const float *sensi_i, int num_coil, int use_z, void *stream) {
    const char *who = "imp_parallel_ift_noalloc: ";
    if (!idata_r || !idata_i || !kdata_r || !kdata_i || !kx || !ky || !ix || !iy || !t)
        return imp::fail(IMP_ERR_INVALID_ARG, std::string(who) + "null data pointer");
    if (use_z && (!kz || !iz))
        return imp::fail(IMP_ERR_INVALID_ARG, std::string(who) + "use_z needs kz and iz");
    if (num_k <= 0 || num_i <= 0 || num_coil <= 0 || num_k > (1 << 30) || num_i > (1 << 30))
        return imp::fail(IMP_ERR_INVALID_ARG, std::string(who) + "bad num_k / num_i / num_coil");
    if (num_coil > 1 && (!sensi_r || !sensi_i))
        return imp::fail(IMP_ERR_INVALID_ARG, std::string(who) + "num_coil > 1 needs sensi");
    cudaStream_t st = (cudaStream_t)stream;
    int device = 0;
    {
        const cudaError_t e = cudaGetDevice(&device);
        if (e != cudaSuccess) return imp::from_cuda(e, "imp_parallel_ift_noalloc: cudaGetDevice");
    }

    imp::NuPlan p;
    imp::nu_plan_dims(p, num_k, num_i, num_coil, use_z != 0);
    // carve: error word | kgeo | vgeo | sens | packed k-data | partial sums
    const size_t b_err = up(sizeof(unsigned));
    const size_t b_kgeo = up(sizeof(double4) * (size_t)p.Mpad);
    const size_t b_vgeo = up(sizeof(double4) * (size_t)p.Npad);
    const size_t b_sens = up(sizeof(float2) * (size_t)p.G * p.Npad * p.CG);
    const size_t b_data = up(sizeof(float2) * (size_t)p.G * p.Mpad * p.CG);
    const size_t fixed = b_err + b_kgeo + b_vgeo + b_sens + b_data;
    imp::NuLaunch l = imp::nu_default_launch(p, true);
    imp::nu_tuned_lookup(p, true, &l);
    // the partial sums must fit what is left: fewer splits if needed
    while (fixed + up(imp::nu_adj_partial_bytes(p, l)) > kNoAllocBytes && l.split > 1) l.split /= 2;
    if (fixed + up(imp::nu_adj_partial_bytes(p, l)) > kNoAllocBytes) {
        char msg[256];
        std::snprintf(msg, sizeof msg,
                      "imp_parallel_ift_noalloc: num_k=%d num_i=%d num_coil=%d needs %zu bytes "
                      "of work memory; the static scratch holds %zu",
                      num_k, num_i, num_coil, fixed + up(imp::nu_adj_partial_bytes(p, l)),
                      kNoAllocBytes);
        std::fprintf(stderr, "%s\n", msg);
        return imp::fail(IMP_ERR_INVALID_ARG, msg);
    }
    unsigned char *base = nullptr;
    imp_status s = scratch_address(device, &base);
    if (s != IMP_OK) return s;
    unsigned *err = (unsigned *)base;
    double4 *kgeo = (double4 *)(base + b_err);
    double4 *vgeo = (double4 *)(base + b_err + b_kgeo);
    float2 *sens = (float2 *)(base + b_err + b_kgeo + b_vgeo);
    float2 *data = (float2 *)(base + b_err + b_kgeo + b_vgeo + b_sens);
    float2 *part = (float2 *)(base + fixed);

    // On a failed launch, wait for whatever of this call is already queued
    // before returning, so that no kernel of it still writes the shared array.
    auto failed = [&](cudaError_t e, const char *what) {
        cudaStreamSynchronize(st);
        cudaGetLastError();
        return imp::from_cuda(e, (std::string(who) + what).c_str());
    };
    cudaError_t e = cudaMemsetAsync(err, 0, sizeof(unsigned), st);
    if (e != cudaSuccess) return failed(e, "clear error word");
    if ((e = imp::nu_plan_place(p, kgeo, vgeo, sens, kx, ky, kz, t, ix, iy, iz, fm, sensi_r,
                                sensi_i, err, st)) != cudaSuccess)
        return failed(e, "geometry");
    if ((e = imp::nu_pack_kdata(p, kdata_r, kdata_i, data, st)) != cudaSuccess)
        return failed(e, "pack k-space data");
    if ((e = imp::nu_adjoint_partials(p, l, data, part, err, st)) != cudaSuccess)
        return failed(e, "adjoint");
    if ((e = imp::nu_adjoint_finish_soa(p, l, part, idata_r, idata_i, st)) != cudaSuccess)
        return failed(e, "adjoint sum");
    unsigned h = 0;
    if ((e = cudaMemcpyAsync(&h, err, sizeof(unsigned), cudaMemcpyDeviceToHost, st)) !=
        cudaSuccess)
        return failed(e, "read error word");
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return failed(e, "stream synchronize");
    if (h & imp::DEV_ERR_RANGE)
        return imp::fail(IMP_ERR_RANGE,
                         std::string(who) + "input outside the fixed-point phase range "
                                            "(|k| <= 32768 cycles/FOV, |r| <= 2 FOV, |t| <= 16 s, "
                                            "|fm| <= 2 pi 8192 rad/s)");
    if (h & imp::DEV_ERR_TIMEOUT)
        return imp::fail(IMP_ERR_TIMEOUT, std::string(who) + "a bounded wait on a bulk copy "
                                                             "ran out");
    return IMP_OK;
}

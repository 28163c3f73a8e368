// The imp_context behind the C-ABI and the helpers every entry point shares.
#pragma once
#include "../../include/impatient_b200.h"

#include <cuda_runtime.h>
#include <map>
#include <memory>
#include <string>
#include <vector>

namespace imp {
class BfSolver;
class BfBatch;
class ToepSolver;
}  // namespace imp

struct imp_context {
    int device = 0;
    cudaStream_t stream = nullptr;
    unsigned *dev_err = nullptr;  // device error word (imp::DEV_ERR_*)
    long launches = 0;
    void *scratch = nullptr;      // grow-only work memory of the operator calls
    size_t scratch_bytes = 0;
    bool prof_on = false;         // per-launch NUDFT timing (imp_context_profile)
    double prof_ms[2] = {0.0, 0.0};
    long prof_count[2] = {0, 0};
    std::unique_ptr<imp::BfSolver> bf;    // brute-force solver reused across calls
    std::unique_ptr<imp::BfBatch> bb;     // batched multi-slice solver
    std::unique_ptr<imp::ToepSolver> tp;  // Toeplitz solver reused across calls
    std::unique_ptr<imp::ToepSolver> tp_q;  // Toeplitz Q gridding (one coil)
    // Grow-only staging arena for the host inputs / outputs of the brute-force
    // entry points (which call no other entry point): chunks are kept across
    // calls, so repeated calls of one size allocate nothing.
    std::vector<std::pair<void *, size_t>> stage;
    size_t stage_chunk = 0, stage_off = 0;
    ~imp_context();
};

namespace imp {

using DevKeep = std::vector<std::unique_ptr<void, void (*)(void *)>>;

// Records `msg` as this thread's last error and returns `s`.
imp_status fail(imp_status s, const std::string &msg);
// cudaSuccess -> IMP_OK, else IMP_ERR_NOMEM / IMP_ERR_CUDA with a message.
imp_status from_cuda(cudaError_t e, const char *what);
// Makes ctx current and clears its device error word.
imp_status begin(imp_context *ctx);
// Synchronizes the context's stream and turns device error bits into a status.
imp_status finish(imp_context *ctx);
// Host or device pointer -> device pointer (host data is staged into `keep`).
imp_status to_device(imp_context *ctx, const float *p, size_t n, DevKeep &keep,
                     const float **out, bool *was_host);
// A writable device buffer for an output that may live in host memory.
imp_status out_device(imp_context *ctx, float *p, size_t n, DevKeep &keep, float **out,
                      bool *was_host);
// to_device through the context's staging arena (no allocation once the arena
// has grown to the call's size); stage_reset starts a call's arena use.
void stage_reset(imp_context *ctx);
imp_status to_device_staged(imp_context *ctx, const float *p, size_t n, const float **out,
                            bool *was_host);
imp_status out_device_staged(imp_context *ctx, float *p, size_t n, float **out, bool *was_host);

}  // namespace imp

#define IMP_CUDA(call, what)                                      \
    do {                                                          \
        imp_status s_ = ::imp::from_cuda((call), what);           \
        if (s_ != IMP_OK) return s_;                              \
    } while (0)

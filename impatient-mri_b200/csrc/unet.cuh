// BF16 U-Net for the learned CG warm start (no counterpart in the reference).
//
// Architecture (2-D, NHWC activations in BF16, FP32 accumulation, FP32 master
// weights with Adam):
//   enc1  conv3x3 16->32, conv3x3 32->32            (input: 2 channels + 14 zero)
//   enc2  maxpool2, conv3x3 32->64, conv3x3 64->64
//   enc3  maxpool2, conv3x3 64->128, conv3x3 128->128
//   mid   maxpool2, conv3x3 128->256, conv3x3 256->256
//   dec3  conv1x1 256->128, nearest x2 into concat [enc3 | up] (256), conv3x3 256->128, 128->128
//   dec2  conv1x1 128->64, x2, concat (128), conv3x3 128->64, 64->64
//   dec1  conv1x1 64->32, x2, concat (64), conv3x3 64->32, 32->32
//   out   conv1x1 32->16 (channels 0, 1 used), no activation
// Every conv3x3 is followed by ReLU; the 1x1 convs are linear.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <cstddef>
#include <vector>

namespace imp {

struct ConvArgs;

struct ConvLayer {
    int cin = 0, cout = 0, ks = 3;
    bool relu = true;
    size_t w_off = 0, b_off = 0;  // offsets into the parameter arrays (floats)
    size_t wsize() const { return (size_t)cout * ks * ks * cin; }
};

class UNet {
public:
    UNet() = default;
    ~UNet();
    UNet(const UNet &) = delete;
    UNet &operator=(const UNet &) = delete;

    // Batch, image size (H, W multiples of 8), seed for the He initialisation.
    cudaError_t setup(int batch, int H, int W, unsigned long long seed, cudaStream_t st,
                      unsigned *err);
    // x: [B][2][H*W] FP32 (channel-major per image), y: same; the network
    // output for channels 0 and 1.
    cudaError_t forward(const float *x, float *y);
    // Loss (mean squared error, host, optional) and parameter gradients of the
    // MSE between forward(x) and target, left in grads().
    cudaError_t gradients(const float *x, const float *target, float *loss);
    // One Adam step on the MSE between forward(x) and target; loss (optional,
    // host) receives the mean squared error.
    cudaError_t train_step(const float *x, const float *target, float lr, float *loss);
    const float *grads() const { return grad_; }

    size_t n_params() const { return n_params_; }
    // FP32 master parameters (device pointer), layout: per layer weights
    // [cout][ks][ks][cin] then bias [cout].
    float *params() { return master_; }
    cudaError_t sync_weights();  // master -> BF16 copies after an external write
    const std::vector<ConvLayer> &layers() const { return layers_; }
    long launches() const { return launches_; }
    int batch() const { return B_; }
    int height() const { return H_; }
    int width() const { return W_; }
    void release();

private:
    struct Act {  // one activation tensor (BF16) and its gradient (FP32)
        int H = 0, W = 0, C = 0;
        __nv_bfloat16 *v = nullptr;
        float *g = nullptr;
    };
    // up2: out has twice in's size and receives the nearest x2 up-sampled output
    cudaError_t conv_fwd(int li, const Act &in, int in_off, Act &out, int out_off,
                         bool up2 = false);
    cudaError_t conv_bwd(int li, Act &in, int in_off, Act &out, int out_off);
    cudaError_t pack_input(const float *x);
    cudaError_t run_conv(const ConvArgs &a, int P);
    cudaError_t run_forward();

    cudaStream_t st_ = nullptr;
    int B_ = 0, H_ = 0, W_ = 0;
    std::vector<ConvLayer> layers_;
    size_t n_params_ = 0;
    float *master_ = nullptr, *grad_ = nullptr, *m_ = nullptr, *v_ = nullptr;
    __nv_bfloat16 *wb_ = nullptr;   // BF16 weights [cout][k]
    __nv_bfloat16 *wt_ = nullptr;   // BF16 flipped/transposed weights [cin][k'] (data grad)
    __nv_bfloat16 *dz_ = nullptr;   // BF16 masked output gradient scratch
    unsigned char *pidx_ = nullptr; // max-pool argmax scratch (3 levels)
    size_t pidx_off_[3] = {0, 0, 0};
    double *scratch_ = nullptr;     // loss partials
    float *outg_ = nullptr;         // gradient of the FP32 network output [P][16]
    std::vector<Act> acts_;
    int step_ = 0;
    long launches_ = 0;
    unsigned *err_ = nullptr;  // device error word (bounded-wait timeouts)
    bool use_tc_ = true;       // tcgen05 convolutions (else WMMA)
    bool use_strip_ = true;    // row-strip variant for the layers it fits
};

}  // namespace imp

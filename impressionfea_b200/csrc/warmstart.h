// warmstart.h — the learned warm start's network (per-node MLP 16 -> 128 -> 128 -> 128 -> 3, GELU), trained and
// evaluated on the B200 tensor cores (mlp.cu). The 3D stepper (solver3d.cu) records training samples into it and
// asks it for each increment's initial velocity guess.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "runtime.cuh"

namespace ifea {
namespace wsm {

constexpr int NIN = 16, HID = 128, NOUT = 3;
// flat FP32 parameter layout: W1 [HID][NIN], b1, W2 [HID][HID], b2, W3 [HID][HID], b3, W4 [NOUT][HID], b4
constexpr int OFF_W1 = 0, OFF_B1 = OFF_W1 + HID * NIN, OFF_W2 = OFF_B1 + HID, OFF_B2 = OFF_W2 + HID * HID,
              OFF_W3 = OFF_B2 + HID, OFF_B3 = OFF_W3 + HID * HID, OFF_W4 = OFF_B3 + HID, OFF_B4 = OFF_W4 + NOUT * HID,
              NPAR = OFF_B4 + NOUT;
constexpr int NNORM = 2 * NIN + 2 * NOUT;  // input mean, input std, output mean, output std
constexpr int BMAX = 8192;                 // largest training batch (a multiple of 128)

}  // namespace wsm

class WarmStartNet {
  public:
    explicit WarmStartNet(uint64_t seed);
    ~WarmStartNet();
    std::string error;

    void get_params(float *host) const;
    void set_params(const float *host);
    void get_norm(float *host) const;
    void set_norm(const float *host);
    // training set (raw features and raw targets, FP32), appended on the device
    void add_samples_device(const float *d_x, const float *d_t, int64_t n, cudaStream_t s);
    void add_samples_host(const float *x, const float *t, int64_t n);
    void clear_samples() { count_ = 0; }
    int64_t samples() const { return count_; }
    void fit_normalisation();
    // y = network(normalised x), de-normalised; d_x raw [n][16] on the device, d_y [n][3]
    void infer_device(const float *d_x, int64_t n, float *d_y, cudaStream_t s);
    void infer_host(const float *x, int64_t n, float *y);
    // gradients of the mean squared error (normalised targets) at the current parameters, for n rows (a multiple
    // of 128, at most BMAX) of host data; grad_host gets NPAR values
    float gradients_host(const float *x, const float *t, int64_t n, float *grad_host);
    // Adam over random batches of the training set; returns the mean loss of the last tenth of the steps
    float train(int steps, int batch, float lr, uint64_t seed);
    double train_ms = 0;

  private:
    void publish(cudaStream_t s);
    void forward(int B, bool train, cudaStream_t s);
    float backward_and_step(int B, bool apply, float lr, cudaStream_t s);
    void ensure_batch(int B);

    cudaStream_t st_ = nullptr;
    int adam_t_ = 0;
    DBuf<float> par_, grad_, m_, v_, norm_;
    DBuf<__nv_bfloat16> w1_, w2_, w3_, w2t_, w3t_;
    // batch workspace
    int bcap_ = 0;
    DBuf<__nv_bfloat16> xb_, xbt_, h1_, h2_, h3_, h1t_, h2t_, dz1_, dz2_, dz3_, dz1t_, dz2t_, dz3t_;
    DBuf<float> tb_, z1_, z2_, z3_, y_, part_, hpart_, loss_;
    DBuf<int32_t> idx_;
    // training set
    DBuf<float> dx_, dt_;
    int64_t count_ = 0, cap_ = 0;
    std::vector<float> norm_host_;
    HostPinned<float> hloss_;
};

}  // namespace ifea

// The C ABI's handle (include/ifea_gpu.h).
struct ifea_mlp {
    ifea::WarmStartNet *net = nullptr;
    std::string err;
};

// Learned radial surrogate: a small MLP r -> R_nl(r) for every (l, n) of the
// calculator's radial basis, trained on the GPU on exact (analytic GTO)
// radial integrals, evaluated with BF16 weights on the tensor cores.
//
//   x = 2 r / r_c - 1
//   h1 = silu(w1 x + b1)                  [H]
//   h2 = silu(W2 h1 + b2)                 [H]
//   y  = W3 h2 + b3                       [O = (lmax + 1) nmax], normalised outputs
//   R_o(r) = s_o y_o, dR_o/dr by forward-mode differentiation of the same net
//
// Training updates FP32 master weights with Adam; the output layer is then
// refitted by least squares (values and r-derivatives).  The tensor-core
// inference reads W2 and W3 as sums of three BF16 matrices (hi + mid + lo).
#pragma once

#include <cstdint>
#include <vector>

#include "engine.hpp"

namespace fb200 {

class RadialSurrogate {
  public:
    RadialSurrogate(Engine& engine, int hidden, uint64_t seed);
    ~RadialSurrogate();
    RadialSurrogate(const RadialSurrogate&) = delete;

    int hidden() const { return H_; }
    int n_outputs() const { return O_; }
    int64_t n_params() const { return n_params_; }
    int64_t n_samples() const { return n_samples_; }

    // exact radial integrals of `n` r uniform in [0, r_c] (training set)
    void make_dataset(int64_t n, uint64_t seed, cudaStream_t stream);
    // `steps` Adam steps on random minibatches of `batch` samples, replayed
    // from a captured CUDA graph; returns the loss of the last step
    double train(int64_t steps, int64_t batch, double lr, cudaStream_t stream);
    // weight lambda of the derivative term of the training loss
    void set_derivative_weight(double lambda) {
        if (!(lambda >= 0.0 && lambda < 1e6)) throw invalid_parameter("the derivative weight must be >= 0");
        deriv_weight_ = lambda;
    }
    double derivative_weight() const { return deriv_weight_; }
    // loss and gradient w.r.t. the master parameters on the first `n`
    // samples of the training set (host copy of the gradient)
    double loss_and_gradient(int64_t n, std::vector<float>& gradient, cudaStream_t stream);
    std::vector<float> parameters(cudaStream_t stream) const;
    void set_parameters(const std::vector<float>& p, cudaStream_t stream);
    std::vector<float> scales() const { return scale_; }
    std::vector<float> dataset_r(cudaStream_t stream) const;

    // R_o(r) and dR_o/dr for `n` distances (device), written at
    // values[i * ld + o] / derivs[i * ld + o]; on the tensor cores
    // (tcgen05, BF16 operands, FP32 accumulation) or with CUDA cores
    // (or, on the CUDA cores with `bf16_weights`, with W2 and W3 rounded to
    // one BF16 each: the single-BF16 control)
    void evaluate(const double* r, int64_t n, float* values, float* derivs, int64_t ld, bool tensor_cores,
                  cudaStream_t stream, bool check = true, bool bf16_weights = false);
    // least-squares refit of the output layer (W3, b3) on the whole training
    // set, values and lambda-weighted r-derivatives (FP64 normal equations)
    void fit_output_layer(double lambda, cudaStream_t stream);
    // the same outputs from the calculator's own radial integral (FP64 spline,
    // or the exact analytic integral), rounded to FP32
    void evaluate_reference(const double* r, int64_t n, float* values, float* derivs, int64_t ld, bool analytic,
                            cudaStream_t stream);
    int out_pad() const { return out_pad_; }
    const Engine* engine() const { return &engine_; }

  private:
    void batch_step(int64_t batch, bool sample, cudaStream_t stream, double lr);

    Engine& engine_;
    int H_ = 64, O_ = 0;
    int64_t n_params_ = 0;
    double rc_ = 0.0;
    int device_ = -1;
    std::vector<float> scale_;
    float* d_scale_ = nullptr;
    float* d_master_ = nullptr;  // FP32 parameters
    float* d_grad_ = nullptr;
    float* d_m_ = nullptr;
    float* d_v_ = nullptr;
    int64_t* d_step_ = nullptr;  // Adam step counter (device, so that a graph can replay steps)
    float* d_loss_ = nullptr;
    // training set
    int64_t n_samples_ = 0;
    float* d_r_ = nullptr;       // [n]
    float* d_t_ = nullptr;       // [n][O] normalised targets
    float* d_dt_ = nullptr;      // [n][O] their r-derivatives (same normalisation)
    // minibatch activations, their x-derivatives and deltas (per sample)
    struct Batch {
        float *x = nullptr, *h1 = nullptr, *dh1 = nullptr, *dz1 = nullptr, *gw1 = nullptr, *h2 = nullptr,
              *dh2 = nullptr, *dz2 = nullptr, *ddz2 = nullptr, *dy = nullptr, *df = nullptr, *partial = nullptr,
              *loss_part = nullptr;
    };
    void ensure_batch(int64_t batch);
    int64_t batch_cap_ = 0;
    Batch bufs_;
    double deriv_weight_ = 0.1;
    // BF16 weights in the tensor-core operand layout, hi / mid / lo parts
    void* d_w2_bf16_ = nullptr;
    void* d_w3_bf16_ = nullptr;
    int out_pad_ = 0;
    // captured training step
    cudaGraph_t graph_ = nullptr;
    cudaGraphExec_t graph_exec_ = nullptr;
    int64_t graph_steps_ = 0;
    double graph_lr_ = 0.0;
    double graph_deriv_weight_ = -1.0;
    uint64_t seed_ = 0;
    std::vector<void*> buffers_;
};

}  // namespace fb200

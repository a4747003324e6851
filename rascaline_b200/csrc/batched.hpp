// Batched form: thousands of small non-periodic systems (molecules) through one
// persistent kernel launch, replayed from a captured CUDA graph, FP32
// arithmetic, with the energy gradient of a linear model (or of any dL/dP)
// by the adjoint of the power spectrum.
#pragma once

#include <map>
#include <memory>
#include <tuple>
#include <vector>

#include "engine.hpp"

namespace fb200 {

struct BatchArgs {
    int lmax, nmax, n_species, n_keys, K, n_props;
    int64_t n_atoms;
    int64_t n_systems;
    double rc2;
    const double* positions;     // [n_atoms][3] device
    const int32_t* species;      // [n_atoms] species index
    const int32_t* atom_system;  // [n_atoms]
    const int64_t* atom_offset;  // [n_systems + 1]
    const int64_t* h_offset;     // [n_systems] first direction slot of each system (n^2 slots)
    const int32_t* order;        // [n_atoms] centres in work order (largest systems first)
    int32_t* queue;              // work counter, zero at launch
    unsigned int* barrier;       // grid barrier [count, generation], zero at launch
    int32_t* status;             // bit 0: radial integral failed, bit 1: barrier timed out
    DeviceRadial exact;
    DenseTables<float> tab;
    CutoffParams cut;
    const float* weights;        // [S][n_keys][n_props] dE/dP of a linear model per centre species, or null
    const float* grad_values;    // [n_atoms][n_keys][n_props] dL/dP, or null
    float* values;               // [n_atoms][n_keys][n_props] output, or null
    float* h;                    // [sum n^2][3] scratch: dL/dr_ab seen from centre a
    float* atom_energy;          // [n_atoms] scratch
    float* atom_strain;          // [n_atoms][9] scratch
    float* grad_positions;       // [n_atoms][3] output dL/dr, or null
    float* energies;             // [n_systems] output (linear model), or null
    float* grad_strain;          // [n_systems][9] output dL/dstrain, or null
};

// launch parameters chosen by the autotuner
struct BatchConfig {
    int warps = 8;        // warps per CTA, one centre per warp
    int chunk = 32;       // neighbour directions staged per warp in the forward pass
    int layout = 1;       // 0: lane per (l, m, n) coefficient; 1: lane per (l, m), n in registers
    int ctas_per_sm = 1;  // resident CTAs per SM of the persistent grid
    // 0: the persistent kernel above; 1: the dense pipeline of the adjoint
    // form (several launches with host synchronisation, no graph), faster on
    // large batches
    int pipeline = 0;
};

class BatchPlan {
  public:
    BatchPlan(Engine& engine, const std::vector<int64_t>& sizes, const std::vector<int32_t>& types,
              const std::vector<int32_t>& species);
    ~BatchPlan();
    BatchPlan(const BatchPlan&) = delete;

    // one replay of the captured graph on `stream`
    void run(const double* positions, const float* weights, const float* grad_values, float* values,
             float* grad_positions, float* energies, float* grad_strain, cudaStream_t stream);
    // time every candidate configuration on these buffers, keep the fastest;
    // returns its time in ms
    double tune(const double* positions, const float* weights, const float* grad_values, float* values,
                float* grad_positions, float* energies, float* grad_strain, cudaStream_t stream);
    int32_t status(cudaStream_t stream);

    int64_t n_atoms() const { return n_atoms_; }
    int64_t n_systems() const { return (int64_t)sizes_.size(); }
    int n_species() const { return (int)species_.size(); }
    int n_keys() const { return n_keys_; }
    int n_props() const { return n_props_; }
    const std::vector<int32_t>& species() const { return species_; }
    BatchConfig config;

  private:
    using Key = std::tuple<const void*, const void*, const void*, void*, void*, void*, void*, int, int, int, int>;
    struct Graph {
        cudaGraph_t graph = nullptr;
        cudaGraphExec_t exec = nullptr;
    };
    struct Shape {
        void* fn = nullptr;
        size_t smem = 0;
        int threads = 0, blocks = 0, per_sm = 0;
    };
    BatchArgs args(const double* positions, const float* weights, const float* grad_values, float* values,
                   float* grad_positions, float* energies, float* grad_strain) const;
    void run_dense(const double* positions, const float* weights, const float* grad_values, float* values,
                   float* grad_positions, float* energies, float* grad_strain, cudaStream_t stream);
    std::vector<HostSystem> systems_;   // types and zero cells, for the dense pipeline
    float* d_values_scratch_ = nullptr;  // dense pipeline without a values output
    float* d_grad_scratch_ = nullptr;    // dense pipeline without a positions output
    Shape shape(const BatchArgs& a, const BatchConfig& c) const;
    void enqueue(const BatchArgs& a, const Shape& sh, bool cooperative, cudaStream_t stream);
    Graph& graph_for(const Key& key, const BatchArgs& a, const BatchConfig& c);
    bool cooperative_ = true;

    Engine& engine_;
    int device_ = -1;
    int64_t n_atoms_ = 0;
    int n_keys_ = 0, n_props_ = 0;
    std::vector<int64_t> sizes_;
    std::vector<int32_t> species_;
    std::vector<void*> buffers_;
    int32_t* d_species_ = nullptr;
    int32_t* d_atom_system_ = nullptr;
    int64_t* d_atom_offset_ = nullptr;
    int64_t* d_h_offset_ = nullptr;
    int32_t* d_order_ = nullptr;
    int32_t* d_control_ = nullptr;  // queue, barrier (2), status
    float* d_h_ = nullptr;
    float* d_atom_energy_ = nullptr;
    float* d_atom_strain_ = nullptr;
    cudaStream_t capture_stream_ = nullptr;
    std::map<Key, Graph> graphs_;
};

}  // namespace fb200

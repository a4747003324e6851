// Dense power spectrum with an adjoint backward pass.
//
// The forward pass writes the power spectrum of every atom as one dense row
// [species pair (a <= b)][l, n1, n2] (zero for species pairs absent around the
// atom) in FP64 or FP32, and keeps what the backward pass needs: the pairs,
// the direction segments and the spherical expansion coefficients.  The
// backward pass contracts dL/dP into dL/dpositions, dL/dcell and the strain
// derivative without materialising any per-pair gradient block; the
// per-pair Y_lm, R_nl and their derivatives are recomputed.
#pragma once

#include <memory>
#include <vector>

#include "engine.hpp"

namespace fb200 {

class RadialSurrogate;

template <typename T>
struct DenseArgs {
    int lmax, nmax, n_species, n_keys, K;
    // forward: compute the pair features with their derivatives (layout with
    // gradients); backward: `features` already holds them
    bool gradient_features = false;
    int64_t n_atoms, n_props, n_systems;
    FeatureLayout layout;
    DevicePairs pairs;
    const int32_t* atom_species;  // [n_atoms]
    const int64_t* seg_offset;    // [n_atoms * S + 1]
    const int32_t* dir_code;      // [2 n_pairs]
    const int64_t* pair_start;    // [n_atoms + 1] pairs of each first atom
    const int64_t* atom_offset;   // [n_systems + 1]
    DeviceRadial exact;
    DenseTables<T> tab;
    CutoffParams cut;
    T* features;          // [n_pairs][layout.stride]
    T* coef;              // [n_atoms][S][K]
    T* values;            // [n_atoms][n_keys][n_props]
    const T* grad_values; // same layout
    // when set, the dL/dP row of centre c is grad_values[grad_species[c]]:
    // one row per species (the weights of a linear model)
    const int32_t* grad_species = nullptr;
    T* grad_coef;         // [n_atoms][S][K]
    T* pair_grad;         // [n_pairs][3] dL/dr_ij
    T* grad_positions;    // [n_atoms][3]
    T* atom_partial;      // [n_atoms][18] strain then cell sums over the atom's own pairs
    T* grad_strain;       // [n_systems][9] or null
    T* grad_cell;         // [n_systems][9] or null
    int32_t* status;
    // FP32 only: R_nl and dR_nl/dr from the learned radial surrogate instead
    // of the spline
    RadialSurrogate* surrogate = nullptr;
    // when set, events recorded on the stream between the phases: [0] before
    // the pair features, [1] after them, [2] after the expansion, [3] after
    // the contraction (forward); [4] before dL/dc, [5] after it, [6] after the
    // pair adjoint, [7] after the reductions (backward)
    cudaEvent_t* marks = nullptr;
};

// write the surrogate's R_nl(r) (and dR/dr when `derivs`) of every pair into
// the feature records
void surrogate_fill(RadialSurrogate* surrogate, const double* distance, int64_t n, float* values, float* derivs,
                    int64_t ld, cudaStream_t stream);

// State of one forward pass, owned by the caller until the backward pass
struct DenseState {
    Engine* engine = nullptr;
    int device = -1;
    int precision = 64;
    cudaStream_t stream = nullptr;
    int64_t n_atoms = 0, n_pairs = 0, n_systems = 0, n_props = 0;
    int n_species = 0, n_keys = 0, K = 0;
    std::vector<int32_t> species_types;
    std::vector<int64_t> atom_offset;
    DevicePairs pairs;
    int64_t* pair_start = nullptr;
    int32_t* atom_species = nullptr;
    int64_t* seg_offset = nullptr;
    int32_t* dir_code = nullptr;
    int64_t* d_atom_offset = nullptr;
    void* coef = nullptr;
    // pair features with their derivatives, computed by the forward pass when
    // the caller announced a backward pass that recomputes them otherwise
    // (FP32 with the learned radial surrogate); the backward reads them
    void* features_grad = nullptr;

    DenseState() = default;
    DenseState(const DenseState&) = delete;
    ~DenseState();
    void* alloc(size_t bytes);

  private:
    std::vector<void*> allocations_;
};

// FP32 contractions on the tensor cores (dense_mma.cu): the power spectrum
// P_l = X_l^T X_l and dL/dc; supported when S nmax <= 128 and 2 lmax + 1 <= 32
bool dense_mma_supported(const DenseArgs<float>& a);
void launch_dense_contraction_mma(const DenseArgs<float>& a, cudaStream_t stream);
void launch_dense_grad_coef_mma(const DenseArgs<float>& a, cudaStream_t stream);
// angular channels per round of the tensor-core kernels (1 to 4)
extern int dense_mma_channels_per_round;
// whether the FP32 contractions use the tensor cores (default) or the CUDA
// cores; FEATOMIC_B200_DENSE_MMA=0 in the environment selects the CUDA cores
bool dense_mma_enabled();
void set_dense_mma_enabled(bool enabled);

template <typename T>
void launch_dense_forward(const DenseArgs<T>& a, int64_t n_pairs, cudaStream_t stream);
// the adjoint; with coef_grad_given, a.grad_coef already holds dL/dc (the
// spherical expansion's own backward pass) and dL/dP is not read
template <typename T>
void launch_dense_backward(const DenseArgs<T>& a, int64_t n_pairs, cudaStream_t stream, bool coef_grad_given = false);
// forward-mode derivative along (tangent_positions [atoms][3], tangent_cell
// [systems][9] or null): pair_tangent [pairs][K] scratch, tangent_coef
// [atoms][S][K] and, when not null, tangent_values [atoms][keys][props]
template <typename T>
void launch_dense_jvp(const DenseArgs<T>& a, int64_t n_pairs, const T* tangent_positions, const T* tangent_cell,
                      T* pair_tangent, T* tangent_coef, T* tangent_values, cudaStream_t stream);
void launch_dense_directions(const DevicePairs& pairs, const int32_t* atom_species, int n_species, int64_t n_atoms,
                             int32_t* dir_code, int64_t* seg_offset, DeviceArena& arena, cudaStream_t stream);

}  // namespace fb200

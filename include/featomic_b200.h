/* featomic-b200: B200-native SOAP spherical expansion / power spectrum behind
 * featomic's C ABI.
 *
 * Every `featomic_*` entry point keeps the name, signature, status codes and
 * ownership rules of featomic's C API (featomic/include/featomic.h, implemented
 * in featomic/src/c_api/*.rs); the comment above each one cites the interface
 * it replaces.  metatensor is not available, so the TensorMap returned by
 * `featomic_calculator_compute` is this library's own minimal
 * `mts_tensormap_t`, read through the `mts_*` accessors below (names and
 * signatures follow metatensor's C API where one exists) and the
 * `featomic_b200_block_values` accessor.
 *
 * Supported calculators: "spherical_expansion", "spherical_expansion_by_pair",
 * "soap_power_spectrum"
 * (Gaussian density with GTO or Dirac density with Tabulated radial bases,
 * TensorProduct or Explicit basis, ShiftedCosine or Step smoothing, optional
 * Willatt2018 radial scaling) and
 * "soap_radial_spectrum" (featomic/src/calculators/soap/radial_spectrum.rs:
 * the same density and GTO radial basis, l = 0 only, keys
 * (center_type, neighbor_type), no components).
 */
#ifndef FEATOMIC_B200_H
#define FEATOMIC_B200_H

#include <stdbool.h>
#include <stdint.h>

/* featomic.h status codes */
#define FEATOMIC_SUCCESS 0
#define FEATOMIC_INVALID_PARAMETER_ERROR 1
#define FEATOMIC_JSON_ERROR 2
#define FEATOMIC_UTF8_ERROR 3
#define FEATOMIC_SYSTEM_ERROR 128
#define FEATOMIC_BUFFER_SIZE_ERROR 254
#define FEATOMIC_INTERNAL_ERROR 255

#define FEATOMIC_LOG_LEVEL_ERROR 1
#define FEATOMIC_LOG_LEVEL_WARN 2
#define FEATOMIC_LOG_LEVEL_INFO 3
#define FEATOMIC_LOG_LEVEL_DEBUG 4
#define FEATOMIC_LOG_LEVEL_TRACE 5

#ifdef __cplusplus
extern "C" {
#endif

typedef int32_t featomic_status_t;
typedef int32_t mts_status_t;
typedef struct featomic_calculator_t featomic_calculator_t;
typedef struct mts_tensormap_t mts_tensormap_t;
typedef struct mts_block_t mts_block_t;
typedef void (*featomic_logging_callback_t)(int32_t level, const char* message);

/* metatensor's mts_labels_t layout (metatensor.h): names, row-major int32
 * values, `size` dimensions and `count` entries.  Labels handed out by this
 * library are borrowed views into the TensorMap. */
typedef struct mts_labels_t {
    const void* internal_ptr_;
    const char* const* names;
    const int32_t* values;
    uintptr_t size;
    uintptr_t count;
} mts_labels_t;

/* featomic.h:114-120, same layout as featomic's Rust `Pair` */
typedef struct featomic_pair_t {
    uintptr_t first;
    uintptr_t second;
    double distance;
    double vector[3];
    int32_t cell_shift_indices[3];
} featomic_pair_t;

/* featomic.h:167-175 */
typedef struct featomic_system_t {
    void* user_data;
    featomic_status_t (*size)(const void* user_data, uintptr_t* size);
    featomic_status_t (*types)(const void* user_data, const int32_t** types);
    featomic_status_t (*positions)(const void* user_data, const double** positions);
    featomic_status_t (*cell)(const void* user_data, double* cell);
    featomic_status_t (*compute_neighbors)(void* user_data, double cutoff);
    featomic_status_t (*pairs)(const void* user_data, const featomic_pair_t** pairs, uintptr_t* count);
    featomic_status_t (*pairs_containing)(const void* user_data, uintptr_t atom, const featomic_pair_t** pairs,
                                          uintptr_t* count);
} featomic_system_t;

/* featomic.h:245-251 */
typedef struct featomic_labels_selection_t {
    const mts_labels_t* subset;
    const mts_tensormap_t* predefined;
} featomic_labels_selection_t;

/* featomic.h:270-277 */
typedef struct featomic_calculation_options_t {
    const char* const* gradients;
    uintptr_t gradients_count;
    bool use_native_system;
    featomic_labels_selection_t selected_samples;
    featomic_labels_selection_t selected_properties;
    const mts_labels_t* selected_keys;
} featomic_calculation_options_t;

/* ---- featomic C API -------------------------------------------------------- */

/* featomic/src/c_api/status.rs:110-131 */
const char* featomic_last_error(void);

/* featomic/src/c_api/logging.rs:51 */
featomic_status_t featomic_set_logging_callback(featomic_logging_callback_t callback);

/* featomic/src/c_api/calculator.rs:54-84 */
featomic_calculator_t* featomic_calculator(const char* name, const char* parameters);

/* featomic/src/c_api/calculator.rs:95-105 */
featomic_status_t featomic_calculator_free(featomic_calculator_t* calculator);

/* featomic/src/c_api/calculator.rs:118-133 */
featomic_status_t featomic_calculator_name(const featomic_calculator_t* calculator, char* name, uintptr_t bufflen);

/* featomic/src/c_api/calculator.rs:146-161 */
featomic_status_t featomic_calculator_parameters(const featomic_calculator_t* calculator, char* parameters,
                                                 uintptr_t bufflen);

/* featomic/src/c_api/calculator.rs:175-190 */
featomic_status_t featomic_calculator_cutoffs(const featomic_calculator_t* calculator, const double** cutoffs,
                                              uintptr_t* cutoffs_count);

/* featomic/src/c_api/calculator.rs:392-461.  The returned TensorMap lives in
 * host memory and is owned by the caller (free with mts_tensormap_free). */
featomic_status_t featomic_calculator_compute(featomic_calculator_t* calculator, mts_tensormap_t** descriptor,
                                              featomic_system_t* systems, uintptr_t systems_count,
                                              featomic_calculation_options_t options);

/* featomic/src/c_api/profiling.rs:17-91 */
featomic_status_t featomic_profiling_clear(void);
featomic_status_t featomic_profiling_enable(bool enabled);
featomic_status_t featomic_profiling_get(const char* format, char* buffer, uintptr_t bufflen);

/* ---- minimal metatensor accessors (metatensor/include/metatensor.h) --------- */

/* mts_tensormap_free */
mts_status_t mts_tensormap_free(mts_tensormap_t* tensor);
/* A TensorMap holding labels only, the predefined samples / properties of a
 * selection (featomic's LabelsSelection::Predefined, calculator.rs:38-44):
 * block k has the key keys[k], the samples samples[k] and the properties
 * properties[k] (a NULL array gives every block the single entry
 * ("_" = 0)), no components, zero values.  Built with metatensor's own
 * mts_block / mts_tensormap in featomic; this library keeps its TensorMaps
 * opaque, so this stands in for those two calls.  Free with
 * mts_tensormap_free. */
featomic_status_t featomic_b200_labels_tensormap(const mts_labels_t* keys, const mts_labels_t* samples,
                                                 const mts_labels_t* properties, mts_tensormap_t** tensor);
/* mts_tensormap_keys: borrowed view */
mts_status_t mts_tensormap_keys(const mts_tensormap_t* tensor, mts_labels_t* keys);
/* mts_tensormap_block_by_id */
mts_status_t mts_tensormap_block_by_id(mts_tensormap_t* tensor, mts_block_t** block, uintptr_t index);
/* mts_block_labels: axis 0 = samples, 1..n = components, n+1 = properties */
mts_status_t mts_block_labels(const mts_block_t* block, uintptr_t axis, mts_labels_t* labels);
/* mts_block_gradient: NULL-free lookup, INVALID_PARAMETER if absent */
mts_status_t mts_block_gradient(mts_block_t* block, const char* parameter, mts_block_t** gradient);
/* mts_block_gradients_list */
mts_status_t mts_block_gradients_list(const mts_block_t* block, const char* const** parameters, uintptr_t* count);
/* mts_labels_free: no-op for the borrowed views handed out here */
mts_status_t mts_labels_free(mts_labels_t* labels);

/* ---- featomic-b200 extensions (no counterpart in featomic) ------------------- */

/* Data of a block: a contiguous row-major float64 array of `shape`.  When the
 * TensorMap lives on the GPU (featomic_b200_calculator_compute_device) `data`
 * is a device pointer and `*on_device` is 1. */
featomic_status_t featomic_b200_block_values(const mts_block_t* block, double** data, const uintptr_t** shape,
                                             uintptr_t* shape_count, int32_t* on_device);

/* Systems whose positions are already resident on the current CUDA device:
 * atoms of all systems concatenated, `positions` a device pointer to
 * [total atoms][3] float64; `types`, `cells` ([n_systems][9]) and
 * `system_sizes` stay on the host. */
typedef struct featomic_b200_device_systems_t {
    uintptr_t n_systems;
    const uintptr_t* system_sizes;
    const int32_t* types;
    const double* cells;
    const double* positions;
} featomic_b200_device_systems_t;

/* Same calculation as featomic_calculator_compute, with device-resident
 * positions and a TensorMap whose values stay in GPU memory, enqueued on
 * `stream` (a cudaStream_t, NULL for the legacy default stream). */
featomic_status_t featomic_b200_calculator_compute_device(featomic_calculator_t* calculator,
                                                          mts_tensormap_t** descriptor,
                                                          const featomic_b200_device_systems_t* systems,
                                                          featomic_calculation_options_t options, void* stream);

/* Half neighbour list of one system computed by the GPU cell list (the list
 * featomic builds in featomic/src/systems/neighbors.rs:349-403), ordered by
 * (first, second, cell shift).  `positions` [n_atoms][3] and `cell` [9] are
 * host arrays.  Writes at most `capacity` pairs and always sets `*count`;
 * returns FEATOMIC_BUFFER_SIZE_ERROR when `capacity` < `*count`. */
featomic_status_t featomic_b200_neighbor_list(const double* positions, uintptr_t n_atoms, const double* cell,
                                              double cutoff, featomic_pair_t* pairs, uintptr_t capacity,
                                              uintptr_t* count);

/* The same half neighbour list (same pairs, same order, same bits as
 * featomic_b200_neighbor_list) computed without allocating any device memory.
 * No counterpart in featomic.
 *
 * For callers that cannot allocate device memory while they run: an
 * application whose own allocator owns the whole device memory budget (a
 * molecular-dynamics engine with a fixed pool, or torch's caching allocator
 * holding the free memory), where a cudaMalloc would fail or fragment the
 * pool, and time steps that must not pay for cudaMalloc / cudaFree, whose
 * cudaFree waits for the whole device.  All working tables live in one fixed
 * array of about 3.7 MB in this library's device memory, one copy per device.
 *
 * `positions` ([n_atoms][3] float64) and `pairs` (`capacity` entries) are
 * device memory of the current CUDA device, owned by the caller; `cell` [9] is
 * a host array.  Work is enqueued on `stream` (a cudaStream_t, NULL for the
 * legacy default stream); the call waits for `stream` once, to learn the
 * number of pairs, which it stores in `*count`.  The pairs are written
 * asynchronously and are ready when `stream` reaches the end of the call.
 *
 * Limits: at most 65536 atoms, 100000 cells (featomic's own cap) and 2048
 * pairs per atom in the half list; beyond them the call returns
 * FEATOMIC_INVALID_PARAMETER_ERROR with a message naming the limit and writes
 * nothing.  When `capacity` < `*count` it returns FEATOMIC_BUFFER_SIZE_ERROR
 * and writes no pair (query the size with capacity 0).  Nothing has to be
 * zeroed by the caller: the call clears its own counters.
 *
 * The first call on each device does a one-time set-up (it looks up the
 * address of that device's scratch array with the device current); make that
 * first call before any stream capture begins.  Calls on the same device share
 * the scratch array, so calls that overlap race: make them one after another
 * (one host thread at a time) on the same stream, or synchronize the stream of
 * the previous call before starting a call on another stream. */
featomic_status_t featomic_b200_neighbor_list_noalloc(const double* positions, uintptr_t n_atoms, const double* cell,
                                                      double cutoff, featomic_pair_t* pairs, uintptr_t capacity,
                                                      uintptr_t* count, void* stream);

/* ---- dense power spectrum with an adjoint backward pass ---------------------
 *
 * The power spectrum of every atom as one dense row, computed in FP64
 * (precision 64, same values as featomic_calculator_compute) or with FP32
 * arithmetic (precision 32), plus a backward pass that turns dL/dvalues into
 * dL/dpositions, dL/dcell and dL/dstrain without materialising the gradient
 * blocks.  This replaces the explicit-gradient autograd of featomic-torch
 * (featomic-torch/src/autograd.cpp:237-317 PositionsGrad, :429-503 CellGrad).
 *
 * Layout of `values` (device memory, float64 or float32):
 *   [atom][species pair (a, b), a <= b][l, n1, n2]
 * with the species pairs of the sorted species list in row-major upper
 * triangle order, n_keys = S (S + 1) / 2, and the properties in featomic's
 * (l, n_1, n_2) order, n_properties = (max_angular + 1) (max_radial + 1)^2.
 * Rows of species pairs absent around an atom are zero; featomic's block
 * (center_type, neighbor_1_type, neighbor_2_type) holds the rows of the atoms of
 * center_type that have both neighbour types (the atom itself counts). */
typedef struct featomic_b200_dense_t featomic_b200_dense_t;

/* Forward pass.  `species` (n_species sorted or not, NULL for the types of the
 * systems) fixes the species list; every atom's type must be in it.
 * `values_count` must be n_atoms x n_keys x n_properties.  The returned state
 * keeps what the backward pass needs; free it with featomic_b200_dense_free,
 * before the calculator.  Work is enqueued on `stream` (the neighbour list
 * waits for it once). */
featomic_status_t featomic_b200_power_spectrum_dense(featomic_calculator_t* calculator,
                                                     const featomic_b200_device_systems_t* systems,
                                                     const int32_t* species, uintptr_t n_species, int32_t precision,
                                                     void* values, uintptr_t values_count,
                                                     featomic_b200_dense_t** state, void* stream);

/* Sizes of a forward pass: atoms, species, species pairs, properties, pairs */
featomic_status_t featomic_b200_dense_shape(const featomic_b200_dense_t* state, uintptr_t* n_atoms,
                                            uintptr_t* n_species, uintptr_t* n_keys, uintptr_t* n_properties,
                                            uintptr_t* n_pairs);

/* Host copies of the species list ([n_species]) and of the number of
 * neighbour directions of each species around every atom
 * ([n_atoms][n_species], may be NULL); waits for the forward pass. */
featomic_status_t featomic_b200_dense_species(const featomic_b200_dense_t* state, int32_t* species,
                                              int32_t* neighbor_counts);

/* Backward pass: `grad_values` has the layout of `values`; writes
 * dL/dpositions [n_atoms][3] and, when not NULL, dL/dstrain and dL/dcell
 * [n_systems][3][3] (strain: sum over pairs of r_ij[x] dL/dr_ij[y]; cell:
 * dL/dH[abc][xyz] with the cell vectors as rows), all device memory of the
 * forward precision.  May be called more than once per state. */
featomic_status_t featomic_b200_power_spectrum_dense_backward(featomic_b200_dense_t* state, const void* grad_values,
                                                              void* grad_positions, void* grad_strain,
                                                              void* grad_cell, void* stream);

featomic_status_t featomic_b200_dense_free(featomic_b200_dense_t* state);

/* The spherical expansion of every atom as one dense row per neighbour
 * species, [atom][species][(l, m), n] with (l, m) = l^2 + l + m over
 * l <= max_angular and n over max_radial + 1 (zero for species absent around
 * the atom), for a spherical_expansion calculator, in FP64 or FP32 arithmetic.
 * featomic's block (o3_lambda = l, center_type, neighbor_type) holds the rows
 * [atom][neighbor species][l^2 .. l^2 + 2l][n] of the atoms of center_type
 * that have neighbour type (the atom itself counts).  `values_count` must be
 * n_atoms x n_species x (max_angular + 1)^2 (max_radial + 1).  The state is
 * the one of featomic_b200_power_spectrum_dense (free it with
 * featomic_b200_dense_free).  Replaces the explicit-gradient autograd of
 * featomic-torch's SphericalExpansion (featomic-torch/src/autograd.cpp). */
featomic_status_t featomic_b200_spherical_expansion_dense(featomic_calculator_t* calculator,
                                                          const featomic_b200_device_systems_t* systems,
                                                          const int32_t* species, uintptr_t n_species,
                                                          int32_t precision, void* values, uintptr_t values_count,
                                                          featomic_b200_dense_t** state, void* stream);

/* Backward pass of featomic_b200_spherical_expansion_dense: dL/dcoefficients
 * in the layout of its `values` to dL/dpositions, dL/dstrain and dL/dcell (as
 * featomic_b200_power_spectrum_dense_backward). */
featomic_status_t featomic_b200_spherical_expansion_dense_backward(featomic_b200_dense_t* state,
                                                                   const void* grad_coefficients, void* grad_positions,
                                                                   void* grad_strain, void* grad_cell, void* stream);

/* Forward-mode derivative of a dense forward pass along a displacement of
 * the positions (`tangent_positions` [n_atoms][3]) and of the cells
 * (`tangent_cell` [n_systems][3][3], rows = cell vectors, NULL for none;
 * positions are held fixed when the cell moves, as in featomic's cell
 * gradient): the tangent of the expansion coefficients (`tangent_coefficients`,
 * layout of featomic_b200_spherical_expansion_dense) and/or of the power
 * spectrum (`tangent_values`, layout of featomic_b200_power_spectrum_dense),
 * device buffers of the forward precision, either may be NULL.  This is the
 * derivative of the backward pass's output with respect to its input dL/dX,
 * i.e. what the double backward of featomic-torch's PositionsGrad / CellGrad
 * computes (featomic-torch/src/autograd.cpp:318-426). */
featomic_status_t featomic_b200_dense_jvp(featomic_b200_dense_t* state, const void* tangent_positions,
                                          const void* tangent_cell, void* tangent_coefficients, void* tangent_values,
                                          void* stream);

/* Engine of the FP32 per-centre contractions of the dense forms (the power
 * spectrum P_l = X_l^T X_l and the adjoint dL/dc): `tensor_cores` = 1 (the
 * default) runs them on the tcgen05 tensor cores with TF32 hi + lo operands
 * and FP32 accumulation, 0 on the CUDA cores; the value of the environment
 * variable FEATOMIC_B200_DENSE_MMA ("0" or "1") is the initial setting.
 * Process-wide; FP64 always uses the CUDA cores.  `channels_per_round`
 * (1 to 4, or 0 to keep the current value) is the number of angular channels
 * of one tensor-core round; FEATOMIC_B200_MMA_CHANNELS gives its initial
 * value.  No counterpart in featomic. */
featomic_status_t featomic_b200_set_contraction_engine(int32_t tensor_cores, int32_t channels_per_round);

/* Kernels of the FP64 spherical expansion (featomic_calculator_compute and
 * featomic_b200_calculator_compute_device): `fused` = 1 (the default) builds
 * every pair's cutoff, Y_lm and R_nl in shared memory inside the expansion
 * kernel (max_angular <= 8 with splined radial integrals), 0 writes them to a
 * per-pair record in device memory first and reads them back.  Both give
 * identical results.  The environment variable FEATOMIC_B200_FUSED_SE ("0" or
 * "1") is the initial setting.  Process-wide.  No counterpart in featomic. */
featomic_status_t featomic_b200_set_expansion_engine(int32_t fused);

/* ---- batched form: many molecules in one persistent launch ------------------
 *
 * Non-periodic systems (molecules) of up to 4096 atoms each, computed with
 * FP32 arithmetic by one persistent, cooperative kernel launch replayed from a
 * captured CUDA graph.  Per atom it produces the dense power spectrum row (the
 * layout of featomic_b200_power_spectrum_dense), and for a loss L the
 * gradient dL/dpositions through the adjoint, without gradient blocks.  L is
 * either a linear model E = sum_atoms weights[species] . P (`weights`, float32
 * [n_species][n_keys][n_properties]) or any loss with dL/dP given per atom
 * (`grad_values`, float32 [n_atoms][n_keys][n_properties]).  Limits:
 * max_angular <= 8, max_radial <= 15, at most 8 species.  No counterpart in
 * featomic. */
typedef struct featomic_b200_batch_t featomic_b200_batch_t;

/* Plan a batch: system sizes and atomic types (host); `species` (NULL for
 * the types present) fixes the species list.  The plan keeps its own device
 * tables and the captured graphs. */
featomic_status_t featomic_b200_batch_create(featomic_calculator_t* calculator, uintptr_t n_systems,
                                             const uintptr_t* system_sizes, const int32_t* types,
                                             const int32_t* species, uintptr_t n_species,
                                             featomic_b200_batch_t** batch);

featomic_status_t featomic_b200_batch_shape(const featomic_b200_batch_t* batch, uintptr_t* n_atoms,
                                            uintptr_t* n_systems, uintptr_t* n_species, uintptr_t* n_keys,
                                            uintptr_t* n_properties);

/* One replay on `stream`.  `positions` is device float64 [n_atoms][3]; every
 * output is a device float32 buffer or NULL: `values` [n_atoms][n_keys]
 * [n_properties], `grad_positions` dL/dr [n_atoms][3], `energies` (linear
 * model) [n_systems], `grad_strain` dL/dstrain [n_systems][3][3].  Give at
 * most one of `weights` and `grad_values`; with neither only the values are
 * computed.  The first run with a new set of buffers captures a graph. */
featomic_status_t featomic_b200_batch_run(featomic_b200_batch_t* batch, const double* positions,
                                          const float* weights, const float* grad_values, float* values,
                                          float* grad_positions, float* energies, float* grad_strain,
                                          void* stream);

/* Time every launch configuration on these buffers and keep the fastest;
 * `best_ms` receives its time per run. */
featomic_status_t featomic_b200_batch_tune(featomic_b200_batch_t* batch, const double* positions,
                                           const float* weights, const float* grad_values, float* values,
                                           float* grad_positions, float* energies, float* grad_strain,
                                           void* stream, double* best_ms);

/* The launch configuration: [warps per CTA, directions staged per warp,
 * coefficient layout (0: lane per (l, m, n), 1: lane per (l, m)), CTAs per
 * SM, pipeline (0: the persistent kernel replayed from a CUDA graph; 1: the
 * dense pipeline of featomic_b200_power_spectrum_dense and its backward,
 * several launches with host synchronisation)].  The tuner times both. */
featomic_status_t featomic_b200_batch_config(const featomic_b200_batch_t* batch, int32_t* config);
featomic_status_t featomic_b200_batch_set_config(featomic_b200_batch_t* batch, const int32_t* config);

/* Error bits of the last run (waits for `stream`): 1 the radial integral
 * failed, 2 the grid barrier timed out. */
featomic_status_t featomic_b200_batch_status(featomic_b200_batch_t* batch, void* stream, int32_t* status);

featomic_status_t featomic_b200_batch_free(featomic_b200_batch_t* batch);

/* ---- learned radial surrogate -------------------------------------------------
 *
 * A small MLP r -> R_nl(r), 1 -> 64 -> 64 -> (max_angular + 1) (max_radial + 1)
 * with SiLU activations, trained on the GPU by this library's own kernels on
 * exact (analytic GTO) radial integrals of the calculator (Adam, then a
 * least-squares refit of the output layer), evaluated on the tensor cores
 * with BF16 operands (weights and activations each stored as three BF16
 * parts) and FP32 accumulation.  Attached to a
 * calculator it replaces the spline in the FP32 dense power spectrum and its
 * adjoint.  featomic's radial basis does not depend on the atomic species, so
 * one network serves every species pair.  No counterpart in featomic. */
typedef struct featomic_b200_surrogate_t featomic_b200_surrogate_t;

featomic_status_t featomic_b200_surrogate_create(featomic_calculator_t* calculator, int32_t hidden, uint64_t seed,
                                                 featomic_b200_surrogate_t** surrogate);
/* number of outputs, of parameters and of training samples */
featomic_status_t featomic_b200_surrogate_shape(const featomic_b200_surrogate_t* surrogate, uintptr_t* n_outputs,
                                                uintptr_t* n_parameters, uintptr_t* n_samples);
/* training set: `n_samples` distances uniform in [0, cutoff] and their exact
 * radial integrals, computed on the GPU */
featomic_status_t featomic_b200_surrogate_dataset(featomic_b200_surrogate_t* surrogate, uintptr_t n_samples,
                                                  uint64_t seed, void* stream);
/* weight lambda of the derivative term of the training loss (default 0.1) */
featomic_status_t featomic_b200_surrogate_set_derivative_weight(featomic_b200_surrogate_t* surrogate,
                                                                double derivative_weight);
/* `steps` Adam steps on random minibatches (one captured CUDA graph per step);
 * `loss` receives the loss of the last minibatch: the mean squared error of
 * the normalised outputs plus lambda times that of their derivatives with
 * respect to x = 2 r / cutoff - 1 */
featomic_status_t featomic_b200_surrogate_train(featomic_b200_surrogate_t* surrogate, uintptr_t steps,
                                                uintptr_t batch, double learning_rate, double* loss, void* stream);
/* Least-squares refit of the output layer (the last linear layer, W3 and
 * b3) over the whole training set: minimises the squared error of the
 * normalised outputs plus `derivative_weight` times that of their
 * r-derivatives, through FP64 normal equations solved on the GPU (Cholesky).
 * Call after featomic_b200_surrogate_train. */
featomic_status_t featomic_b200_surrogate_fit_output_layer(featomic_b200_surrogate_t* surrogate,
                                                           double derivative_weight, void* stream);
/* loss and gradient (host, n_parameters) on the first `n` training samples */
featomic_status_t featomic_b200_surrogate_gradient(featomic_b200_surrogate_t* surrogate, uintptr_t n,
                                                   float* gradient, double* loss, void* stream);
/* host copy of the FP32 parameters (w1, b1, W2, b2, W3, b3), of the output
 * scales and of the training distances; `set` != 0 writes the parameters */
featomic_status_t featomic_b200_surrogate_parameters(featomic_b200_surrogate_t* surrogate, float* parameters,
                                                     uintptr_t count, int32_t set, void* stream);
featomic_status_t featomic_b200_surrogate_scales(const featomic_b200_surrogate_t* surrogate, float* scales,
                                                 uintptr_t count);
featomic_status_t featomic_b200_surrogate_samples(const featomic_b200_surrogate_t* surrogate, float* r,
                                                  uintptr_t count, void* stream);
/* R_o(r) and dR_o/dr (o = l (max_radial + 1) + n) for `n` device distances,
 * written to device float32 rows of stride `ld`; `method` 0: tensor cores
 * (W2, W3 and the activations as sums of three BF16 parts), 1: CUDA cores
 * (same network, FP32 weights), 2: the calculator's FP64 spline, 3: the exact
 * analytic integral, 4: CUDA cores with W2 and W3 rounded to one BF16 each
 * (the single-BF16 control of the error) */
featomic_status_t featomic_b200_surrogate_evaluate(featomic_b200_surrogate_t* surrogate, const double* r,
                                                   uintptr_t n, float* values, float* derivs, uintptr_t ld,
                                                   int32_t method, void* stream);
/* use `surrogate` (NULL: the spline) for the radial integral of this
 * calculator's FP32 dense power spectrum and adjoint; the calculator only
 * holds it weakly and falls back to the spline once it is freed */
featomic_status_t featomic_b200_calculator_set_surrogate(featomic_calculator_t* calculator,
                                                         featomic_b200_surrogate_t* surrogate);
/* a surrogate can be freed before or after its calculator, but not used
 * after its calculator is freed */
featomic_status_t featomic_b200_surrogate_free(featomic_b200_surrogate_t* surrogate);

/* Radial integral R_nl(r) and dR_nl/dr of this calculator, as the kernels see
 * it (the Hermite spline of featomic/src/calculators/soap/radial_integral/
 * spline.rs, or the analytic GTO integral of radial_integral/gto.rs when
 * spline_accuracy is null), evaluated on the host for `n_r` distances:
 * values / gradients are [n_r][max_angular + 1][max_radial + 1].
 * `knots`, when not NULL, receives the number of spline knots of each angular
 * channel ([max_angular + 1], 0 for the analytic integral). */
featomic_status_t featomic_b200_radial_integral(const featomic_calculator_t* calculator, const double* r,
                                                uintptr_t n_r, double* values, double* gradients, int32_t* knots);

/* Device times (ms, CUDA events on the caller's stream) of the phases of the
 * last dense forward and backward passes of this calculator
 * (featomic_b200_power_spectrum_dense, ..._spherical_expansion_dense and
 * their backward passes, the batched form's dense pipeline): [0] pair
 * features, [1] expansion, [2] contraction, [3] dL/dc, [4] pair adjoint,
 * [5] reductions; `count` entries at most are written.  Waits for the last
 * backward pass; concurrent passes of one calculator overwrite each other's
 * times.  No counterpart in featomic. */
featomic_status_t featomic_b200_dense_timings(const featomic_calculator_t* calculator, double* times,
                                             uintptr_t count);

/* Per-phase device time (ms) of the last compute call of this calculator:
 * [neighbours, host metadata, pair features, expansion, contraction,
 *  device->host transfer, total wall, power-spectrum values kernel,
 *  power-spectrum positions-gradient kernel, strain / cell kernels,
 *  host metadata built before the contraction kernels launch, host labels
 *  written while they run] */
featomic_status_t featomic_b200_calculator_timings(const featomic_calculator_t* calculator, double* times,
                                                   uintptr_t count);

/* ---- Clebsch-Gordan tensor products -------------------------------------
 * The numerical core of featomic's Python clebsch_gordan module
 * (python/featomic/featomic/clebsch_gordan/_coefficients.py): real CG
 * coefficients and the coupling of two equivariant blocks.  No counterpart in
 * featomic's C API (featomic does these in Python / torch). */

/* Real Clebsch-Gordan coefficients coupling l1 and l2 to lambda, written as a
 * dense [2 l1 + 1][2 l2 + 1][2 lambda + 1] array (`count` must be that size);
 * the values of _coefficients.py:_build_dense_cg_coeff_dict (:137-224).
 * Host computation, no device needed. */
featomic_status_t featomic_b200_cg_coefficients(int32_t l1, int32_t l2, int32_t lambda, double* coefficients,
                                                uintptr_t count);

/* One block product: output[s][mu][p * n_second + q] =
 *   sum_{m1, m2} C[m1][m2][mu] first[s][m1][p] second[s][m2][q]
 * (_coefficients.py:_cg_tensor_product_dense, :677-709).  All three arrays are
 * device memory, contiguous, of the precision given to
 * featomic_b200_cg_product. */
typedef struct featomic_b200_cg_task_t {
    const void* first;   /* [n_samples][2 l1 + 1][n_first] */
    const void* second;  /* [n_samples][2 l2 + 1][n_second] */
    void* output;        /* [n_samples][2 lambda + 1][n_first * n_second] */
    int64_t n_samples;
    int32_t l1;
    int32_t l2;
    int32_t lambda;
    int32_t n_first;
    int32_t n_second;
    /* elements between consecutive (sample, mu) rows of `output`; 0 means
     * n_first * n_second (a dense block).  A larger stride writes the
     * product into columns of a wider block. */
    int64_t output_stride;
} featomic_b200_cg_task_t;

/* Run `n_tasks` block products in one launch on `stream` (NULL = the legacy
 * default stream); precision 32 (float) or 64 (double).  Returns once the
 * products are queued; the tasks array may be freed on return. */
featomic_status_t featomic_b200_cg_product(const featomic_b200_cg_task_t* tasks, uintptr_t n_tasks,
                                           int32_t precision, void* stream);

/* One coupling of two spherical axes (_coefficients.py:387-545, cg_couple):
 * output[o][mu][i] = sum_{m1, m2} C[m1][m2][mu] input[o][m1][m2][i], all
 * device memory, contiguous. */
typedef struct featomic_b200_cg_couple_task_t {
    const void* input;  /* [n_outer][2 l1 + 1][2 l2 + 1][n_inner] */
    void* output;       /* [n_outer][2 lambda + 1][n_inner] */
    int64_t n_outer;
    int64_t n_inner;
    int32_t l1;
    int32_t l2;
    int32_t lambda;
} featomic_b200_cg_couple_task_t;

/* Run `n_tasks` couplings in one launch on `stream`, precision 32 or 64. */
featomic_status_t featomic_b200_cg_couple(const featomic_b200_cg_couple_task_t* tasks, uintptr_t n_tasks,
                                          int32_t precision, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* FEATOMIC_B200_H */

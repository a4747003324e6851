// Device-side data structures and launchers of the B200 SOAP engine.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "host.hpp"

#define CUDA_CHECK(expr)                                                                         \
    do {                                                                                         \
        cudaError_t err__ = (expr);                                                              \
        if (err__ != cudaSuccess) {                                                              \
            throw ::fb200::internal_error(std::string("CUDA error: ") + cudaGetErrorString(err__) + \
                                          " at " + __FILE__ + ":" + std::to_string(__LINE__));   \
        }                                                                                        \
    } while (0)

namespace fb200 {

// Named, growing device buffers reused across calls of one calculator.
class DeviceArena {
  public:
    DeviceArena() = default;
    DeviceArena(const DeviceArena&) = delete;
    ~DeviceArena();

    void* alloc_bytes(const std::string& name, size_t bytes);
    template <typename T>
    T* alloc(const std::string& name, int64_t count) {
        return static_cast<T*>(alloc_bytes(name, sizeof(T) * (size_t)(count > 0 ? count : 1)));
    }
    // out[i] = sum_{k<i} in[k]
    void exclusive_scan(const int32_t* in, int32_t* out, int64_t n, cudaStream_t stream);
    void exclusive_scan(const int64_t* in, int64_t* out, int64_t n, cudaStream_t stream);
    size_t bytes_reserved() const;
    void release();

  private:
    struct Buffer {
        void* ptr = nullptr;
        size_t bytes = 0;
    };
    std::map<std::string, Buffer> buffers_;
};

// Cell-list parameters of one system
struct NlSystem {
    int64_t atom_offset;
    int64_t cell_offset;
    int32_t n_atoms;
    int32_t infinite;
    int32_t n_cells[3];
    int32_t n_search[3];
    double cutoff2;
    double H[9];
    double inv[9];
};

NlSystem make_nl_system(const double* cell, double cutoff, int64_t atom_offset, int64_t n_atoms, int64_t cell_offset);

// Half neighbour list on the device (global atom indices), structure of arrays
struct DevicePairs {
    int32_t* first = nullptr;
    int32_t* second = nullptr;
    double* distance = nullptr;
    double* vector = nullptr;  // [count][3]
    int32_t* shift = nullptr;  // [count][3]
    int64_t count = 0;
};

class NeighborBuilder {
  public:
    DevicePairs pairs;
    // [n_atoms + 1] first pair of every atom (pairs are sorted by first atom)
    const int64_t* pair_start = nullptr;
    int64_t build(const std::vector<NlSystem>& systems, const std::vector<int32_t>& atom_system,
                  const double* d_positions, int64_t n_atoms, DeviceArena& arena, cudaStream_t stream);
};

// ---------------------------------------------------------------------------
// Spherical expansion (kernel b)
// ---------------------------------------------------------------------------
struct DeviceRadial {
    int lmax, nmax;
    int splined;
    const int32_t* knot_offset;
    const int32_t* knot_count;
    const double* positions;
    const double* values;
    const double* derivs;
    double c, width2;
    const double* bn;
    const double* ortho;
};

// recursion coefficients of the spherical harmonics, in the arithmetic type T
template <typename T>
struct DeviceYlmT {
    int lmax;
    const T *A, *B, *sq_plus, *sq_minus, *sq_2l1, *sq_half, *sq_ll1, *inv_ll;
};
using DeviceYlm = DeviceYlmT<double>;

// spline tables with values / derivatives in T (knot positions in FP64)
template <typename T>
struct DeviceSplineT {
    int lmax, nmax, splined;
    const int32_t* knot_offset;
    const int32_t* knot_count;
    const double* positions;
    const T* values;
    const T* derivs;
};

// device tables of the dense kernels in one arithmetic type
template <typename T>
struct DenseTables {
    DeviceYlmT<T> ylm;
    DeviceSplineT<T> spline;
    const T* self_contribution = nullptr;
};

struct CutoffParams {
    double rc, width;
    int smoothing;
    int scaling;
    double scale, rate, exponent;
};

// layout of the per-pair feature record (doubles)
struct FeatureLayout {
    int lmax, nmax, L2, with_grad;
    int off_y, off_dy, off_r, off_dr, stride;
    static FeatureLayout make(int lmax, int nmax, bool grad) {
        FeatureLayout f;
        f.lmax = lmax;
        f.nmax = nmax;
        f.L2 = (lmax + 1) * (lmax + 1);
        f.with_grad = grad ? 1 : 0;
        f.off_y = 16;
        f.off_dy = f.off_y + f.L2;
        f.off_r = f.off_dy + (grad ? 3 * f.L2 : 0);
        f.off_dr = f.off_r + (lmax + 1) * nmax;
        int end = f.off_dr + (grad ? (lmax + 1) * nmax : 0);
        f.stride = (end + 3) / 4 * 4;
        return f;
    }
};

struct SeArgs {
    FeatureLayout layout;
    int64_t n_centres;
    int n_species;
    const int32_t* centre_species;  // [n_centres]
    const int64_t* seg_offset;      // [n_centres * S + 1]
    const int32_t* dir_code;        // (pair << 1) | inverse
    const double* features;         // [pairs][stride]
    const double* self_contribution;
    int do_positions, do_strain, do_cell;
    // outputs
    double* coef;       // [c][S][L2][nmax]
    double* pair_grad;  // [pair][3][L2][nmax]
    double* self_grad;  // [c][S][3][L2][nmax]
    double* strain;     // [c][S][3][3][L2][nmax]
    double* cellg;      // [c][S][3][3][L2][nmax]
};

void launch_pair_features(const DevicePairs& pairs, const DeviceRadial& radial, const DeviceYlm& ylm,
                          const CutoffParams& cut, const FeatureLayout& layout, double* features, int32_t* status,
                          cudaStream_t stream);
void launch_se_accumulate(const SeArgs& args, cudaStream_t stream);
// pair_features + se_accumulate in one kernel (the pair terms built in shared
// memory, args.features unused), for lmax <= 8 and splined radial
// integrals; bit-identical results
bool se_fused_supported(const FeatureLayout& layout, const DeviceRadial& radial);
void launch_se_fused(const SeArgs& args, const DevicePairs& pairs, const DeviceRadial& radial, const DeviceYlm& ylm,
                     const CutoffParams& cut, cudaStream_t stream);
// whether the drop-in's spherical expansion uses the fused kernel (default)
// or the two-kernel path; FEATOMIC_B200_FUSED_SE=0 selects the two kernels
bool se_fused_enabled();
void set_se_fused_enabled(bool enabled);

// ---------------------------------------------------------------------------
// Power spectrum (kernel c)
// ---------------------------------------------------------------------------
struct PsKeySlot {
    int32_t block;
    int32_t sample;
    int32_t a;  // species index of neighbor_1_type
    int32_t b;  // species index of neighbor_2_type
};

struct PsEntry {
    int32_t atom;     // global atom index of the neighbour (or the centre)
    int32_t species;
    int32_t d0, d1;   // direction range in the (centre, species) segment
};

struct PsArgs {
    int lmax, nmax, n_species;
    int64_t n_centres;
    int64_t n_props;
    const double* coef;
    const double* pair_grad;
    const double* self_grad;
    const double* strain;
    const double* cellg;
    const int32_t* dir_code;
    const int64_t* slot_offset;     // [n_centres + 1]
    const PsKeySlot* slots;
    const int64_t* entry_offset;    // [n_centres + 1]
    const PsEntry* entries;
    // per entry: [S] number of earlier neighbours of each species in the
    // centre's list, then [S] = 1 if the centre itself comes earlier
    const int32_t* entry_cum;
    const int64_t* slot_row;        // first positions-gradient row of each slot
    const int64_t* off_values;      // per block, offsets into `out` (doubles)
    const int64_t* off_positions;
    const int64_t* off_strain;
    const int64_t* off_cell;
    double* out;
};

// timing events of launch_power_spectrum (each may be null)
struct PsEvents {
    cudaEvent_t after_values = nullptr;       // side stream
    cudaEvent_t after_strain_cell = nullptr;  // side stream
    cudaEvent_t before_positions = nullptr;   // caller's stream
    cudaEvent_t after_positions = nullptr;    // caller's stream
};

// positions rows on `stream`; values, strain and cell rows beside it on a
// second stream of the device; `stream` waits for both before later work
void launch_power_spectrum(const PsArgs& args, bool positions, bool strain, bool cell, cudaStream_t stream,
                           const PsEvents& events);

// The power-spectrum kernels' neighbourhood tables built on the device from
// the sorted directions: for every centre its unique neighbours (and itself)
// by atom index, with the per-species prefix counts, the number of unique
// neighbours of each species and the species present around it.  The merge
// of the host's build_neighborhoods, one thread per centre, so the tables
// are identical to the host's.
struct DeviceNeighborhoods {
    int64_t* entry_offset = nullptr;   // [n_atoms + 1]
    PsEntry* entries = nullptr;        // [entry_offset[n_atoms]]
    int32_t* entry_cum = nullptr;      // [entries][S + 1]
    int32_t* species_count = nullptr;  // [n_atoms * S]
    uint8_t* species_mask = nullptr;   // [n_atoms * S]
};
// When `host_count` / `host_mask` are given, the species counts and masks are
// copied to them right after the counting kernel and `counted` is recorded
// there, before the scan and the fill.
DeviceNeighborhoods launch_neighborhoods(const DevicePairs& pairs, const int32_t* atom_species, const int32_t* dir_code,
                                         const int64_t* seg_offset, int n_species, int64_t n_atoms, DeviceArena& arena,
                                         cudaStream_t stream, int32_t* host_count = nullptr,
                                         uint8_t* host_mask = nullptr, cudaEvent_t counted = nullptr);

// Spherical expansion output scatter (spherical_expansion calculator)
struct SeOutArgs {
    int lmax, nmax, n_species;
    const double* coef;
    const double* pair_grad;
    const double* self_grad;
    const double* strain;
    const double* cellg;
    const int32_t* dir_code;
    // one entry per (block, sample)
    int64_t n_rows;
    const int32_t* row_centre;   // global centre
    const int32_t* row_block;    // block index
    const int32_t* row_sample;   // sample index in the block
    // one entry per gradient row
    int64_t n_grad_rows;
    const int32_t* grad_block;
    const int64_t* grad_row;     // row index in the block
    const int32_t* grad_centre;
    const int32_t* grad_atom;    // neighbour (== centre for self rows)
    const int32_t* grad_d0;      // direction range
    const int32_t* grad_d1;
    const int32_t* block_l;
    const int32_t* block_species;
    const int64_t* off_values;
    const int64_t* off_positions;
    const int64_t* off_strain;
    const int64_t* off_cell;
    double* out;
};

void launch_se_output(const SeOutArgs& args, bool positions, bool strain, bool cell, cudaStream_t stream);

// spherical_expansion_by_pair output: every direction's pair contribution
// scattered into its rows (tables from plan_by_pair)
struct ByPairArgs {
    FeatureLayout layout;
    int64_t n_dirs;                  // 2 x pairs
    DevicePairs pairs;
    const double* features;          // drop-in pair records
    const int32_t* dir_block0;       // [n_dirs]
    const int64_t* dir_row0;         // [n_dirs]
    const int64_t* dir_row1;         // [n_dirs]
    const int64_t* dir_grow;         // [n_dirs]
    const int64_t *off_values, *off_positions, *off_strain, *off_cell;  // per block
    int64_t n_self;
    const int32_t* self_block;       // [n_self]
    const int64_t* self_row;         // [n_self]
    const double* self_contribution; // [nmax]
    double* out;                     // zero-filled before the launch
};

void launch_by_pair(const ByPairArgs& args, bool positions, bool strain, bool cell, cudaStream_t stream);

}  // namespace fb200

namespace fb200 {

struct DenseState;
struct Neighborhoods;
template <typename T>
struct DenseArgs;
class RadialSurrogate;

struct PhaseTimes {
    double neighbors = 0, metadata = 0, features = 0, expansion = 0, contraction = 0, transfer = 0, total = 0;
    // kernels of the contraction phase
    double ps_values = 0, ps_positions = 0, ps_strain_cell = 0;
    // host metadata split: built before the contraction kernels can launch,
    // and the output labels written while they run
    double metadata_before_launch = 0, labels = 0;
};

// One calculator's GPU state: constant tables on the device, the workspace
// arena, and the compute pipeline.
class Engine {
  public:
    static constexpr int OUTPUT_EXPANSION = 0, OUTPUT_POWER_SPECTRUM = 1, OUTPUT_BY_PAIR = 2;

    explicit Engine(const Hypers& h);
    ~Engine();

    // kind: OUTPUT_EXPANSION, OUTPUT_POWER_SPECTRUM or OUTPUT_BY_PAIR
    std::unique_ptr<TensorMap> compute(int kind, std::vector<HostSystem>& systems, const GradientOptions& g,
                                       bool device_output, const double* d_positions, cudaStream_t stream);

    const RadialTables& radial() const { return radial_; }
    const PhaseTimes& last_times() const { return times_; }
    int device() const { return device_; }

    // dense power spectrum with its adjoint (dense.hpp); `species` empty means
    // the sorted atomic types of the systems; `values` is a device buffer of
    // n_atoms x n_keys x n_properties elements of the precision (32 / 64)
    // `expansion`: `values` receives the spherical expansion coefficients
    // [n_atoms][n_species][(lmax + 1)^2 nmax] instead, with no contraction
    std::unique_ptr<DenseState> forward_dense(int precision, std::vector<HostSystem>& systems,
                                              const double* d_positions, const std::vector<int32_t>& species,
                                              void* values, int64_t values_count, cudaStream_t stream,
                                              bool expansion = false, bool backward_follows = false);
    // dL/dpositions [n_atoms][3], and when not null dL/dstrain and dL/dcell
    // [n_systems][3][3], all device buffers of the forward precision
    // `by_species`: grad_values holds one dL/dP row per species (the weights
    // of a linear model) instead of one per atom
    // `coefficients`: grad_values is dL/dc [n_atoms][n_species][K] of the
    // spherical expansion instead of dL/dP
    void backward_dense(DenseState& state, const void* grad_values, void* grad_positions, void* grad_strain,
                        void* grad_cell, cudaStream_t stream, bool by_species = false, bool coefficients = false);
    // forward-mode derivative along a displacement of the positions
    // ([n_atoms][3]) and cells ([n_systems][3][3] or null): the tangent of the
    // coefficients (when `tangent_coef` is not null) and of the power spectrum
    // (when `tangent_values` is not null), device buffers of the forward
    // precision
    void jvp_dense(DenseState& state, const void* tangent_positions, const void* tangent_cell, void* tangent_coef,
                   void* tangent_values, cudaStream_t stream);
    // device times (ms) of the phases of the last dense forward and backward
    // passes: pair features, expansion, contraction, dL/dc, pair adjoint,
    // reductions (waits for the last backward pass; 0 for a phase not run)
    std::vector<double> dense_times();

    // device tables for the kernels of the batched form (uploaded on first use)
    const DenseTables<float>& dense_tables_f() {
        upload_tables();
        return dense_f_;
    }
    const DeviceRadial& device_radial() {
        upload_tables();
        return d_radial_;
    }
    const Hypers& hypers() const { return h_; }
    // radial integral of the FP32 dense forms from a learned surrogate (empty:
    // the spline); held weakly, so that a freed surrogate falls back to the
    // spline
    void set_surrogate(const std::shared_ptr<RadialSurrogate>& s) { surrogate_ = s; }

  private:
    // events between the phases of the dense forms (dense_times), created on
    // first use on the engine's device
    cudaEvent_t dense_marks_[8] = {};
    bool dense_marks_ready_ = false;
    cudaEvent_t* dense_marks();
    void upload_tables();
    template <typename T>
    void dense_args(const DenseState& st, bool grad, DenseArgs<T>& a);
    DenseTables<double> dense_d_{};
    DenseTables<float> dense_f_{};
    std::weak_ptr<RadialSurrogate> surrogate_;
    RadialSurrogate* active_surrogate_ = nullptr;  // held during one forward / backward pass
    Hypers h_;
    RadialTables radial_;
    YlmTables ylm_;
    DeviceArena arena_;
    NeighborBuilder nl_;
    int device_ = -1;
    bool tables_ready_ = false;
    DeviceRadial d_radial_{};
    DeviceYlm d_ylm_{};
    double* d_self_ = nullptr;
    std::vector<void*> table_buffers_;
    PhaseTimes times_;
    // host neighbourhood tables of the power spectrum (labels), kept between
    // calls for their storage, and a pinned buffer their device copy comes
    // back through
    std::unique_ptr<Neighborhoods> nh_;
    void* staging_ = nullptr;
    size_t staging_bytes_ = 0;
    void* staging(size_t bytes);
};

}  // namespace fb200

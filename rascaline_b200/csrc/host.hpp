// Host-side data model of the B200 SOAP engine: hyper-parameters, radial
// spline tables, systems, labels / TensorMap, and the engine entry points.
#pragma once

#include <cstdint>
#include <functional>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "json.hpp"

struct featomic_pair_t;

namespace fb200 {

// featomic status codes, featomic/include/featomic.h
constexpr int32_t STATUS_SUCCESS = 0;
constexpr int32_t STATUS_INVALID_PARAMETER = 1;
constexpr int32_t STATUS_JSON_ERROR = 2;
constexpr int32_t STATUS_UTF8_ERROR = 3;
constexpr int32_t STATUS_SYSTEM_ERROR = 128;
constexpr int32_t STATUS_BUFFER_SIZE_ERROR = 254;
constexpr int32_t STATUS_INTERNAL_ERROR = 255;

struct Error : std::runtime_error {
    int32_t status;
    Error(int32_t s, const std::string& m) : std::runtime_error(m), status(s) {}
};

inline Error invalid_parameter(const std::string& m) { return Error(STATUS_INVALID_PARAMETER, m); }
inline Error internal_error(const std::string& m) { return Error(STATUS_INTERNAL_ERROR, m); }

// ---------------------------------------------------------------------------
// SOAP hyper-parameters (featomic's SphericalExpansionParameters /
// PowerSpectrumParameters, spherical_expansion_pair.rs:37-45,
// power_spectrum.rs:35-43)
// ---------------------------------------------------------------------------
// A user-given spline of the radial integral (featomic's `Tabulated` radial
// basis, basis/radial/tabulated.rs): control points sorted by position, each
// with `size` values and derivatives
struct TabulatedSpline {
    int size = 0;
    std::vector<double> positions;  // [points]
    std::vector<double> values;     // [points][size]
    std::vector<double> derivs;     // [points][size]
};

struct Hypers {
    double cutoff = 0.0;
    int smoothing = 0;  // 0 ShiftedCosine, 1 Step
    double smoothing_width = 0.0;
    double density_width = 0.0;
    double center_atom_weight = 1.0;
    bool scaling = false;
    double scaling_scale = 0.0, scaling_rate = 0.0, scaling_exponent = 0.0;
    int max_angular = 0;
    int max_radial = 0;
    bool splined = true;
    double spline_accuracy = 1e-8;
    // Explicit basis (basis/mod.rs:95-116): number of radial functions of each
    // angular channel l = 0..max_angular, 0 for a channel absent from the
    // basis; max_radial + 1 is the largest.  Empty for TensorProduct.
    std::vector<int> radial_sizes;
    bool explicit_basis() const { return !radial_sizes.empty(); }
    // Tabulated radial basis: the spline of each angular channel (empty for
    // GTO; an absent Explicit channel has size 0)
    std::vector<TabulatedSpline> tabulated;
    bool tabulated_basis() const { return !tabulated.empty(); }

    int nmax() const { return max_radial + 1; }
    int lm_count() const { return (max_angular + 1) * (max_angular + 1); }
};

// parse + validate; `deny_unknown_top` mirrors serde's deny_unknown_fields on
// the top-level struct (spherical expansion: yes, power spectrum and radial
// spectrum: no).  `radial_spectrum_basis` reads featomic's
// RadialSpectrumBasis {radial, spline_accuracy} (radial_spectrum.rs:44-57)
// instead of a SphericalExpansionBasis, with max_angular = 0.
Hypers parse_hypers(const std::string& json, bool deny_unknown_top, bool radial_spectrum_basis = false);

// LODE spherical expansion (featomic/src/calculators/lode/
// spherical_expansion.rs:30-58): smeared power-law density, GTO radial basis
// of an explicit radius, k-space cutoff (default 1.2 pi / smearing)
struct LodeHypers {
    double smearing = 0.0;
    int exponent = 0;
    double center_atom_weight = 1.0;
    double k_cutoff = 0.0;
    int max_angular = 0;
    int max_radial = 0;
    double radius = 0.0;
    bool splined = true;
    double spline_accuracy = 1e-8;
    int nmax() const { return max_radial + 1; }
};

LodeHypers parse_lode_hypers(const std::string& json);

// GTO radial basis (shared/basis/radial/gto.rs:44-80): Gaussian widths
// radius max(sqrt(n), 1) / size and the orthonormalisation matrix O,
// row-major, orthonormal functions R_k = sum_n O[k][n] raw_n
std::vector<double> gto_basis_widths(int size, double radius);
std::vector<double> gto_basis_orthonormalization(int size, double radius);

// Adaptive Hermite spline knots of a function R -> R^n on [0, stop]: 11
// uniform points, then every interval midpoint until the mean absolute or the
// mean relative interpolation error over the first `checked` outputs at the
// midpoints drops below `accuracy` (featomic/src/math/splines.rs:79-193, at
// most 10 000 points).  `eval(x, values, derivatives)` fills n outputs.
void build_spline_knots(const std::function<void(double, double*, double*)>& eval, double stop, int n, int checked,
                        double accuracy, std::vector<double>& positions, std::vector<double>& values,
                        std::vector<double>& derivatives);

// ---------------------------------------------------------------------------
// Radial integral tables (one Hermite spline per angular channel, knots chosen
// adaptively like featomic/src/math/splines.rs:79-193)
// ---------------------------------------------------------------------------
struct RadialTables {
    int lmax = 0, nmax = 0;
    bool splined = true;
    // spline: for each l, knots [offset[l], offset[l] + count[l])
    std::vector<int32_t> knot_offset, knot_count;
    std::vector<double> positions;      // [total knots]
    std::vector<double> values, derivs; // [total knots][nmax], orthonormalised
    // analytic mode
    double c = 0.0, width2 = 0.0;
    std::vector<double> bn;             // [nmax]
    std::vector<double> ortho;          // [nmax][nmax], R[k] = sum_n raw[n] ortho[k][n]
    // self contribution I_n^{l=0}(0) * w * f(0) * Y00 (spherical_expansion_pair.rs:222-252)
    std::vector<double> self_contribution;  // [nmax]
};

RadialTables build_radial_tables(const Hypers& h);

// orthonormalised radial integral on the host (knot construction, tests)
void radial_integral_host(const RadialTables& t, int l, double r, double* values, double* grads);

// ---------------------------------------------------------------------------
// Spherical harmonics constant tables (featomic/src/math/spherical_harmonics.rs:203-301)
// ---------------------------------------------------------------------------
struct YlmTables {
    int lmax = 0;
    std::vector<double> A, B;          // [(l+1)(l+2)/2], index m + l(l+1)/2
    std::vector<double> sq_plus, sq_minus;  // sqrt((l+m)(l-m+1)), sqrt((l-m)(l+m+1))
    std::vector<double> sq_2l1, sq_half, sq_ll1, inv_ll;  // per l
};

YlmTables build_ylm_tables(int lmax);

// ---------------------------------------------------------------------------
// Systems
// ---------------------------------------------------------------------------
struct Pair {
    uint64_t first;
    uint64_t second;
    double distance;
    double vector[3];
    int32_t shift[3];
};

struct HostSystem {
    int64_t n_atoms = 0;
    std::vector<int32_t> types;
    std::vector<double> positions;  // n x 3
    double cell[9] = {0};
    bool has_pairs = false;         // pairs supplied by the caller's neighbour list
    std::vector<Pair> pairs;
};

// ---------------------------------------------------------------------------
// Labels / blocks / TensorMap (metatensor layout, minimal)
// ---------------------------------------------------------------------------
struct Labels {
    std::vector<std::string> names;
    std::vector<int32_t> values;  // count x names.size()
    size_t count() const { return names.empty() ? 0 : values.size() / names.size(); }
};

struct Block {
    Labels samples;
    std::vector<Labels> components;
    Labels properties;
    std::vector<size_t> shape;
    double* data = nullptr;  // host or device pointer, owned by the TensorMap's buffer
    std::vector<std::pair<std::string, std::unique_ptr<Block>>> gradients;
    size_t size() const {
        size_t s = 1;
        for (auto d : shape) s *= d;
        return s;
    }
};

struct TensorMap {
    Labels keys;
    std::vector<std::unique_ptr<Block>> blocks;
    bool on_device = false;
    int device = 0;
    std::shared_ptr<void> storage;  // owns the data of every block
};

// ---------------------------------------------------------------------------
// Engine
// ---------------------------------------------------------------------------
struct GradientOptions {
    bool positions = false, strain = false, cell = false;
    bool any() const { return positions || strain || cell; }
};

class Engine;
class LodeEngine;

struct CalculatorImpl {
    std::string name;        // registry name
    std::string pretty_name; // CalculatorBase::name
    std::string parameters;  // JSON as given
    Hypers hypers;
    std::vector<double> cutoffs;
    std::unique_ptr<Engine> engine;      // SOAP calculators
    std::unique_ptr<LodeEngine> lode;    // lode_spherical_expansion
    bool power_spectrum = false;
    bool radial_spectrum = false;  // spherical expansion l = 0, keys (center_type, neighbor_type)
    bool by_pair = false;          // spherical_expansion_by_pair
    ~CalculatorImpl();
};

std::unique_ptr<CalculatorImpl> create_calculator(const std::string& name, const std::string& json);

// Full calculation.  Systems are on the host; `positions_device` optionally
// points to the concatenated positions already resident on the GPU (then the
// host positions are not uploaded).  Output on the host unless
// `device_output`.
std::unique_ptr<TensorMap> compute(CalculatorImpl& calc, std::vector<HostSystem>& systems,
                                   const GradientOptions& grads, bool device_output,
                                   const double* positions_device, void* stream);

// Samples / properties / keys selections (featomic's CalculationOptions,
// calculator.rs:20-158), applied to the output of a full calculation (on the
// host, or on the device with a gather kernel)
struct Selection {
    const Labels* keys = nullptr;
    const Labels* samples = nullptr;
    const Labels* properties = nullptr;
    const TensorMap* samples_predefined = nullptr;
    const TensorMap* properties_predefined = nullptr;
    int max_angular = 0;  // for the components of keys the systems do not produce
    // predefined samples the full calculation does not produce (a centre of
    // the key's center_type without neighbours of a key's neighbour type)
    // get zero rows; their positions gradient samples need the atomic types
    // and the atoms within the cutoff of an atom (any order, repeats allowed)
    const std::vector<HostSystem>* systems = nullptr;
    std::function<std::vector<int32_t>(int64_t system, int64_t atom)> neighbors;
    bool any() const { return keys || samples || properties || samples_predefined || properties_predefined; }
};

std::unique_ptr<TensorMap> apply_selection(std::unique_ptr<TensorMap> full, const Selection& selection);

// dst[r][m][p] = src[rows[r]][m][props[p]] on the device (rows[r] < 0: zero
// row), src rows of `inner` x `src_props` doubles; index arrays on the device
void launch_gather_rows(const double* src, const int64_t* rows, int64_t n_rows, int64_t inner, int64_t src_props,
                        const int64_t* props, int64_t n_props, double* dst);

// run kernel (a) on one system given on the host, return the pairs
std::vector<Pair> neighbor_list(const double* positions, int64_t n_atoms, const double* cell, double cutoff);

// kernel (a) on one system whose positions are on the current device, pairs
// written to the caller's device buffer, with no device allocation
void neighbor_list_noalloc(const double* positions, int64_t n_atoms, const double* cell, double cutoff,
                           featomic_pair_t* pairs, int64_t capacity, uintptr_t* count, void* stream);

// last-call timings (ms) for the profiling API
std::string profiling_report(const std::string& format);
void profiling_enable(bool enable);
void profiling_clear();

}  // namespace fb200

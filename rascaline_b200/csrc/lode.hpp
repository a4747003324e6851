// LODE spherical expansion (featomic/src/calculators/lode/): long-range
// expansion of a smeared power-law density around every atom, computed in
// reciprocal space from the k-vectors of the periodic cell.
#pragma once

#include <cuda_runtime.h>

#include <memory>
#include <vector>

#include "engine.hpp"
#include "host.hpp"

namespace fb200 {

// ---- host math (lode/radial_integral/gto.rs, lode/spherical_expansion.rs) --

// exponential integrals E1(x) (x > 0) and Ei(x)
double exp1(double x);
double expi(double x);
// Gauss series of 2F1(1, b; c; z) for 0 <= z < 1
double hyp2f1_one(double b, double c, double z);

// k-vectors of compute_k_vectors (math/k_vectors.rs:19-87): one of each +-k
// pair inside the k_cutoff ball, norms and unit directions
struct KVectors {
    std::vector<double> norm;       // [K]
    std::vector<double> direction;  // [K][3]
    size_t count() const { return norm.size(); }
};
KVectors compute_k_vectors(const double cell[9], double k_cutoff);

// Host tables of one LODE calculator: widths and orthonormalisation of the
// GTO basis, the radial integral splines over [0, k_cutoff] (or none for the
// analytic integral), the central-atom contribution and the k = 0 term
struct LodeTables {
    LodeHypers h;
    std::vector<double> widths, ortho;
    // spline of channel l: knots [knot_offset[l], knot_offset[l] + knot_count[l])
    std::vector<int32_t> knot_offset, knot_count;
    std::vector<double> positions, values, derivs;  // [knots], [knots][nmax] x 2
    std::vector<double> center;                     // [nmax] <n 0 0> of the central atom
    std::vector<double> k0;                         // [nmax] k = 0 term (without 4 pi / V)
    // orthonormalised radial integral of channel l at |k| (and d/dk)
    void radial(int l, double k, double* values, double* grads) const;
    // Fourier transform of the density at |k|
    double density_fourier(double k) const;
};

LodeTables build_lode_tables(const LodeHypers& h);

// ---- the calculator -----------------------------------------------------------

class LodeEngine {
  public:
    explicit LodeEngine(const LodeHypers& h);
    ~LodeEngine();

    // values and (optionally) positions gradients of every system, keys
    // (o3_lambda, o3_sigma, center_type, neighbor_type)
    std::unique_ptr<TensorMap> compute(const std::vector<HostSystem>& systems, const GradientOptions& g,
                                       bool device_output, const double* d_positions, cudaStream_t stream);
    const PhaseTimes& last_times() const { return times_; }
    const LodeTables& tables() const { return tables_; }

  private:
    void upload_tables();
    LodeTables tables_;
    YlmTables ylm_;
    DeviceYlm d_ylm_{};
    std::vector<void*> table_buffers_;
    bool tables_ready_ = false;
    int device_ = -1;
    DeviceArena arena_;
    PhaseTimes times_;
};

}  // namespace fb200

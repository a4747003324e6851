// Calculator set-up on the host: hyper-parameter parsing / validation, the GTO
// radial basis orthonormalisation, the adaptive Hermite spline tables of the
// radial integral, and the constant tables of the spherical harmonics.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <sstream>

#include "host.hpp"
#include "soap_math.cuh"

namespace fb200 {

using json::Value;

// ---------------------------------------------------------------------------
// JSON -> Hypers, with serde's accept / reject rules:
// deny_unknown_fields on Cutoff, Smoothing, DensityScaling, the basis and the
// radial basis (featomic/src/calculators/soap/cutoff.rs:4-29,
// calculators/shared/density.rs:4-75, calculators/shared/basis/mod.rs:11-59,
// calculators/shared/basis/radial/mod.rs:9-37).  Type errors are JSON errors
// (FEATOMIC_JSON_ERROR), semantic errors are invalid parameters.
// ---------------------------------------------------------------------------
namespace {

Error json_error(const std::string& m) { return Error(STATUS_JSON_ERROR, m); }

const Value& field(const Value& obj, const char* name, const char* context) {
    const Value* v = obj.get(name);
    if (!v) throw json_error(std::string("missing field `") + name + "` in " + context);
    return *v;
}

void deny_unknown(const Value& obj, std::initializer_list<const char*> allowed, const char* context) {
    for (auto& kv : obj.object) {
        bool ok = false;
        for (auto a : allowed)
            if (kv.first == a) ok = true;
        if (!ok) {
            std::string list;
            for (auto a : allowed) list += std::string(list.empty() ? "" : ", ") + "`" + a + "`";
            throw json_error("unknown field `" + kv.first + "` in " + context + ", expected one of " + list);
        }
    }
}

const Value& object(const Value& v, const char* context) {
    if (v.kind != Value::Object)
        throw json_error(std::string("invalid type: ") + v.kind_name() + ", expected " + context);
    return v;
}

double as_f64(const Value& v, const char* name) {
    if (v.kind != Value::Number) throw json_error(std::string("invalid type: ") + v.kind_name() + " for `" + name + "`, expected f64");
    return v.number;
}

int64_t as_usize(const Value& v, const char* name) {
    if (v.kind != Value::Number || !v.is_integer)
        throw json_error(std::string("invalid type: ") + v.kind_name() + " for `" + name + "`, expected usize");
    if (v.integer < 0) throw json_error(std::string("invalid value: integer `") + std::to_string(v.integer) + "` for `" + name + "`, expected usize");
    return v.integer;
}

std::string tag(const Value& v, const char* context) {
    const Value* t = v.get("type");
    if (!t) throw json_error(std::string("missing field `type` in ") + context);
    if (t->kind != Value::String) throw json_error(std::string("invalid type for `type` in ") + context);
    return t->string;
}

// Tabulated radial basis: {"type": "Tabulated", "points": [{"position",
// "values", "derivatives"}, ...]} with the checks of
// basis/radial/tabulated.rs:174-210, points sorted by position
TabulatedSpline parse_tabulated(const Value& radial) {
    deny_unknown(radial, {"type", "points"}, "Tabulated");
    const Value& points = field(radial, "points", "Tabulated");
    if (points.kind != Value::Array) throw json_error(std::string("invalid type: ") + points.kind_name() + ", expected a sequence");
    if (points.array.size() < 2)
        throw invalid_parameter("we need at least two points to define a 'Tabulated' radial basis");
    struct Point {
        double position;
        std::vector<double> values, derivs;
    };
    std::vector<Point> list;
    size_t size = 0;
    for (size_t k = 0; k < points.array.size(); k++) {
        const Value& p = object(points.array[k], "struct SplinePoint");
        deny_unknown(p, {"position", "values", "derivatives"}, "SplinePoint");
        Point q;
        q.position = as_f64(field(p, "position", "SplinePoint"), "position");
        for (const char* name : {"values", "derivatives"}) {
            const Value& arr = field(p, name, "SplinePoint");
            if (arr.kind != Value::Array) throw json_error(std::string("invalid type: ") + arr.kind_name() + ", expected a sequence");
            auto& dst = std::string(name) == "values" ? q.values : q.derivs;
            for (auto& x : arr.array) dst.push_back(as_f64(x, name));
        }
        if (k == 0) size = q.values.size();
        if (!std::isfinite(q.position)) {
            std::ostringstream m;
            m << "expected all points 'position' in 'Tabulated' radial basis to be finite numbers, got " << q.position;
            throw invalid_parameter(m.str());
        }
        if (q.values.size() != size)
            throw invalid_parameter("expected all points 'values' in 'Tabulated' radial basis to have the same size, got " +
                                    std::to_string(q.values.size()) + " and " + std::to_string(size));
        if (q.derivs.size() != size)
            throw invalid_parameter("expected all points 'derivatives' in 'Tabulated' radial basis to have the same size, got " +
                                    std::to_string(q.derivs.size()) + " and " + std::to_string(size));
        list.push_back(std::move(q));
    }
    if (size == 0) throw invalid_parameter("a 'Tabulated' radial basis needs at least one function");
    std::stable_sort(list.begin(), list.end(), [](const Point& a, const Point& b) { return a.position < b.position; });
    TabulatedSpline t;
    t.size = (int)size;
    for (auto& q : list) {
        t.positions.push_back(q.position);
        t.values.insert(t.values.end(), q.values.begin(), q.values.end());
        t.derivs.insert(t.derivs.end(), q.derivs.begin(), q.derivs.end());
    }
    return t;
}

}  // namespace

Hypers parse_hypers(const std::string& text, bool deny_unknown_top, bool radial_spectrum_basis) {
    Value root;
    try {
        root = json::parse(text);
    } catch (json::ParseError& e) {
        throw json_error(e.what());
    }
    object(root, "struct parameters");
    if (deny_unknown_top) deny_unknown(root, {"cutoff", "density", "basis"}, "parameters");
    Hypers h;

    // cutoff
    const Value& cutoff = object(field(root, "cutoff", "parameters"), "struct Cutoff");
    deny_unknown(cutoff, {"radius", "smoothing"}, "Cutoff");
    h.cutoff = as_f64(field(cutoff, "radius", "Cutoff"), "radius");
    const Value& smoothing = object(field(cutoff, "smoothing", "Cutoff"), "internally tagged enum Smoothing");
    std::string st = tag(smoothing, "Smoothing");
    if (st == "ShiftedCosine") {
        deny_unknown(smoothing, {"type", "width"}, "ShiftedCosine");
        h.smoothing = 0;
        h.smoothing_width = as_f64(field(smoothing, "width", "ShiftedCosine"), "width");
    } else if (st == "Step") {
        deny_unknown(smoothing, {"type"}, "Step");
        h.smoothing = 1;
    } else {
        throw json_error("unknown variant `" + st + "`, expected `ShiftedCosine` or `Step`");
    }

    // density: DensityKind is flattened, so unknown fields are not rejected
    const Value& density = object(field(root, "density", "parameters"), "struct Density");
    std::string dt = tag(density, "Density");
    bool gaussian = false;
    if (dt == "Gaussian") {
        gaussian = true;
        h.density_width = as_f64(field(density, "width", "Gaussian"), "width");
    } else if (dt == "DiracDelta") {
    } else if (dt == "SmearedPowerLaw") {
        as_f64(field(density, "smearing", "SmearedPowerLaw"), "smearing");
        as_usize(field(density, "exponent", "SmearedPowerLaw"), "exponent");
    } else {
        throw json_error("unknown variant `" + dt + "`, expected one of `DiracDelta`, `Gaussian`, `SmearedPowerLaw`");
    }
    if (const Value* cw = density.get("center_atom_weight")) h.center_atom_weight = as_f64(*cw, "center_atom_weight");
    if (const Value* sc = density.get("scaling")) {
        if (sc->kind != Value::Null) {
            object(*sc, "internally tagged enum DensityScaling");
            std::string t = tag(*sc, "DensityScaling");
            if (t != "Willatt2018") throw json_error("unknown variant `" + t + "`, expected `Willatt2018`");
            deny_unknown(*sc, {"type", "scale", "rate", "exponent"}, "Willatt2018");
            h.scaling = true;
            h.scaling_scale = as_f64(field(*sc, "scale", "Willatt2018"), "scale");
            h.scaling_rate = as_f64(field(*sc, "rate", "Willatt2018"), "rate");
            h.scaling_exponent = as_f64(field(*sc, "exponent", "Willatt2018"), "exponent");
        }
    }

    // basis
    const char* basis_name = radial_spectrum_basis ? "RadialSpectrumBasis" : "TensorProduct";
    const Value* basis_ptr = nullptr;
    if (radial_spectrum_basis) {
        // one radial basis, l = 0 only (radial_spectrum.rs:44-57, :79-91)
        basis_ptr = &object(field(root, "basis", "parameters"), "struct RadialSpectrumBasis");
        deny_unknown(*basis_ptr, {"radial", "spline_accuracy"}, "RadialSpectrumBasis");
        h.max_angular = 0;
    } else {
        basis_ptr = &object(field(root, "basis", "parameters"), "internally tagged enum SphericalExpansionBasis");
        std::string bt = tag(*basis_ptr, "SphericalExpansionBasis");
        if (bt == "Explicit") {
            // one radial basis per angular channel (basis/mod.rs:60-116)
            deny_unknown(*basis_ptr, {"type", "by_angular", "spline_accuracy"}, "ExplicitBasis");
            const Value& by = object(field(*basis_ptr, "by_angular", "ExplicitBasis"), "a map");
            if (by.object.empty()) throw invalid_parameter("the Explicit basis needs at least one angular channel");
            std::map<int, int> sizes;
            std::map<int, TabulatedSpline> tabulated;
            for (auto& kv : by.object) {
                char* end = nullptr;
                const long l = std::strtol(kv.first.c_str(), &end, 10);
                if (kv.first.empty() || *end != '\0' || l < 0 || kv.first[0] == '-' || kv.first[0] == '+')
                    throw json_error("invalid digit found in string `" + kv.first + "` for the by_angular keys");
                const Value& radial = object(kv.second, "internally tagged enum SoapRadialBasis");
                const std::string rt = tag(radial, "SoapRadialBasis");
                if (rt == "Tabulated") {
                    tabulated[(int)l] = parse_tabulated(radial);
                    sizes[(int)l] = tabulated[(int)l].size;
                    continue;
                }
                if (rt != "Gto") throw json_error("unknown variant `" + rt + "`, expected `Gto` or `Tabulated`");
                deny_unknown(radial, {"type", "max_radial", "radius"}, "Gto");
                if (const Value* rr = radial.get("radius"))
                    if (rr->kind != Value::Null && as_f64(*rr, "radius") != h.cutoff)
                        throw internal_error("GTO radius must be the same as the cutoff radius in SOAP, or should not provided");
                sizes[(int)l] = (int)as_usize(field(radial, "max_radial", "Gto"), "max_radial") + 1;
            }
            h.max_angular = sizes.rbegin()->first;
            if (h.max_angular > 24) throw invalid_parameter("max_angular larger than 24 is not supported by featomic-b200");
            h.radial_sizes.assign(h.max_angular + 1, 0);
            int largest = 0;
            for (auto& kv : sizes) {
                h.radial_sizes[kv.first] = kv.second;
                largest = std::max(largest, kv.second);
            }
            h.max_radial = largest - 1;
            if (!tabulated.empty()) {
                // one kind of radial basis for every channel: Gto needs a
                // Gaussian density, Tabulated a Dirac one
                if (tabulated.size() != sizes.size())
                    throw invalid_parameter("this combination of basis and density is not supported in SOAP");
                h.tabulated.assign(h.max_angular + 1, TabulatedSpline());
                for (auto& kv : tabulated) h.tabulated[kv.first] = kv.second;
            }
            if (const Value* sa = basis_ptr->get("spline_accuracy")) {
                if (sa->kind == Value::Null && tabulated.empty()) {
                    throw invalid_parameter("the Explicit basis needs a splined radial integral in featomic-b200 "
                                            "(spline_accuracy can not be null)");
                }
                if (sa->kind == Value::Null) goto validate;
                h.spline_accuracy = as_f64(*sa, "spline_accuracy");
            }
            goto validate;
        } else if (bt != "TensorProduct") {
            throw json_error("unknown variant `" + bt + "`, expected `TensorProduct` or `Explicit`");
        }
        deny_unknown(*basis_ptr, {"type", "max_angular", "radial", "spline_accuracy"}, "TensorProduct");
        h.max_angular = (int)as_usize(field(*basis_ptr, "max_angular", "TensorProduct"), "max_angular");
    }
    {
    const Value& basis = *basis_ptr;
    const Value& radial = object(field(basis, "radial", basis_name), "internally tagged enum SoapRadialBasis");
    std::string rt = tag(radial, "SoapRadialBasis");
    if (rt == "Tabulated") {
        // the same user spline for every angular channel
        const TabulatedSpline t = parse_tabulated(radial);
        h.max_radial = t.size - 1;
        h.tabulated.assign(h.max_angular + 1, t);
        goto accuracy;
    } else if (rt != "Gto") {
        throw json_error("unknown variant `" + rt + "`, expected `Gto` or `Tabulated`");
    }
    deny_unknown(radial, {"type", "max_radial", "radius"}, "Gto");
    h.max_radial = (int)as_usize(field(radial, "max_radial", "Gto"), "max_radial");
    if (const Value* rr = radial.get("radius")) {
        if (rr->kind != Value::Null) {
            double radius = as_f64(*rr, "radius");
            if (radius != h.cutoff)
                throw internal_error("GTO radius must be the same as the cutoff radius in SOAP, or should not provided");
        }
    }
accuracy:
    if (const Value* sa = basis.get("spline_accuracy")) {
        if (sa->kind == Value::Null) {
            h.splined = false;
        } else {
            h.spline_accuracy = as_f64(*sa, "spline_accuracy");
        }
    }

    }
validate:
    // a Tabulated basis is its own spline
    if (h.tabulated_basis()) h.splined = true;
    // validation: cutoff.rs:32-45, density.rs:79-105, radial_integral/mod.rs:78-123
    if (h.smoothing == 0 && (h.smoothing_width <= 0.0 || !std::isfinite(h.smoothing_width))) {
        std::ostringstream m;
        m << "expected positive width for shifted cosine cutoff function, got " << h.smoothing_width;
        throw invalid_parameter(m.str());
    }
    if (h.scaling) {
        if (h.scaling_scale <= 0.0) throw invalid_parameter("expected positive scale for Willatt2018 radial scaling function");
        if (h.scaling_rate <= 0.0) throw invalid_parameter("expected positive rate for Willatt2018 radial scaling function");
        if (h.scaling_exponent <= 0.0) throw invalid_parameter("expected positive exponent for Willatt2018 radial scaling function");
    }
    // radial_integral/mod.rs:86-113: Gaussian density with GTO, Dirac density
    // with Tabulated
    if (h.tabulated_basis() ? dt != "DiracDelta" : !gaussian)
        throw invalid_parameter("this combination of basis and density is not supported in SOAP");
    if (gaussian && !(h.density_width > 1e-16 && std::isfinite(h.density_width)))
        throw invalid_parameter("expected positive and finite Gaussian width");
    if (!(h.cutoff > 0.0 && std::isfinite(h.cutoff))) throw invalid_parameter("cutoff must be positive and finite");
    if (h.splined && h.spline_accuracy < 0.0) {
        std::ostringstream m;
        m << "got invalid accuracy in spline (" << h.spline_accuracy << "), it must be positive";
        throw invalid_parameter(m.str());
    }
    if (h.max_angular > 24) throw invalid_parameter("max_angular larger than 24 is not supported by featomic-b200");
    if (h.max_radial > 63) throw invalid_parameter("max_radial larger than 63 is not supported by featomic-b200");
    return h;
}

// ---------------------------------------------------------------------------
// GTO radial basis: widths sigma_n = rc max(sqrt n, 1) / n_max and the
// orthonormalisation S^{-1/2} diag(norm) of the analytic overlap
// (featomic/src/calculators/shared/basis/radial/gto.rs:17-75).
// ---------------------------------------------------------------------------
namespace {

// Eigen-decomposition of a real symmetric matrix: Householder reduction to
// tridiagonal form followed by the implicit QL algorithm (EISPACK tred2 /
// tql2, Bowdler, Martin, Reinsch and Wilkinson, Handbook for Automatic
// Computation vol. II), eigenvalues sorted in increasing order.  featomic
// uses this algorithm (featomic/src/math/eigen.rs:23-244); the overlap matrix
// is ill-conditioned, so S^{-1/2} depends on the solver at 5e-11 (8 radial
// functions) to 2e-8 (12) and the same solver is needed to agree with
// featomic.  `v` is row-major n x n: the input matrix on entry, the
// eigenvectors (columns) on exit.
void symmetric_eigen(std::vector<double>& v, int n, std::vector<double>& d) {
    auto V = [&](int i, int j) -> double& { return v[(size_t)i * n + j]; };
    std::vector<double> e(n, 0.0);
    d.assign(n, 0.0);
    for (int j = 0; j < n; j++) d[j] = V(n - 1, j);
    for (int i = n - 1; i > 0; i--) {
        double scale = 0.0, h = 0.0;
        for (int k = 0; k < i; k++) scale += std::fabs(d[k]);
        if (scale == 0.0) {
            e[i] = d[i - 1];
            for (int j = 0; j < i; j++) {
                d[j] = V(i - 1, j);
                V(i, j) = 0.0;
                V(j, i) = 0.0;
            }
        } else {
            for (int k = 0; k < i; k++) {
                d[k] /= scale;
                h += d[k] * d[k];
            }
            double f = d[i - 1];
            double g = std::sqrt(h);
            if (f > 0) g = -g;
            e[i] = scale * g;
            h -= f * g;
            d[i - 1] = f - g;
            for (int j = 0; j < i; j++) e[j] = 0.0;
            for (int j = 0; j < i; j++) {
                f = d[j];
                V(j, i) = f;
                g = e[j] + V(j, j) * f;
                for (int k = j + 1; k <= i - 1; k++) {
                    g += V(k, j) * d[k];
                    e[k] += V(k, j) * f;
                }
                e[j] = g;
            }
            f = 0.0;
            for (int j = 0; j < i; j++) {
                e[j] /= h;
                f += e[j] * d[j];
            }
            double hh = f / (h + h);
            for (int j = 0; j < i; j++) e[j] -= hh * d[j];
            for (int j = 0; j < i; j++) {
                f = d[j];
                g = e[j];
                for (int k = j; k <= i - 1; k++) V(k, j) -= (f * e[k] + g * d[k]);
                d[j] = V(i - 1, j);
                V(i, j) = 0.0;
            }
        }
        d[i] = h;
    }
    for (int i = 0; i < n - 1; i++) {
        V(n - 1, i) = V(i, i);
        V(i, i) = 1.0;
        double h = d[i + 1];
        if (h != 0.0) {
            for (int k = 0; k <= i; k++) d[k] = V(k, i + 1) / h;
            for (int j = 0; j <= i; j++) {
                double g = 0.0;
                for (int k = 0; k <= i; k++) g += V(k, i + 1) * V(k, j);
                for (int k = 0; k <= i; k++) V(k, j) -= g * d[k];
            }
        }
        for (int k = 0; k <= i; k++) V(k, i + 1) = 0.0;
    }
    for (int j = 0; j < n; j++) {
        d[j] = V(n - 1, j);
        V(n - 1, j) = 0.0;
    }
    V(n - 1, n - 1) = 1.0;
    e[0] = 0.0;

    // implicit QL
    for (int i = 1; i < n; i++) e[i - 1] = e[i];
    e[n - 1] = 0.0;
    double f = 0.0, tst1 = 0.0;
    for (int l = 0; l < n; l++) {
        tst1 = std::max(tst1, std::fabs(d[l]) + std::fabs(e[l]));
        int m = l;
        while (m < n) {
            if (std::fabs(e[m]) <= soap::DBL_EPS * tst1) break;
            m++;
        }
        if (m > l) {
            for (int iter = 0; iter < 10000; iter++) {
                double g = d[l];
                double p = (d[l + 1] - g) / (2.0 * e[l]);
                double r = std::hypot(p, 1.0);
                if (p < 0) r = -r;
                d[l] = e[l] / (p + r);
                d[l + 1] = e[l] * (p + r);
                double dl1 = d[l + 1];
                double h = g - d[l];
                for (int i = l + 2; i < n; i++) d[i] -= h;
                f += h;
                p = d[m];
                double c = 1.0, c2 = c, c3 = c;
                double el1 = e[l + 1];
                double s = 0.0, s2 = 0.0;
                for (int i = m - 1; i >= l; i--) {
                    c3 = c2;
                    c2 = c;
                    s2 = s;
                    g = c * e[i];
                    h = c * p;
                    r = std::hypot(p, e[i]);
                    e[i + 1] = s * r;
                    s = e[i] / r;
                    c = p / r;
                    p = c * d[i] - s * g;
                    d[i + 1] = h + s * (c * g + s * d[i]);
                    for (int k = 0; k < n; k++) {
                        h = V(k, i + 1);
                        V(k, i + 1) = s * V(k, i) + c * h;
                        V(k, i) = c * V(k, i) - s * h;
                    }
                }
                p = -s * s2 * c3 * el1 * e[l] / dl1;
                e[l] = s * p;
                d[l] = c * p;
                if (std::fabs(e[l]) <= soap::DBL_EPS * tst1) break;
            }
        }
        d[l] += f;
        e[l] = 0.0;
    }
    // selection sort of the eigenvalues (and their vectors), increasing
    for (int i = 0; i < n - 1; i++) {
        int k = i;
        double p = d[i];
        for (int j = i + 1; j < n; j++) {
            if (d[j] < p) {
                k = j;
                p = d[j];
            }
        }
        if (k != i) {
            d[k] = d[i];
            d[i] = p;
            for (int j = 0; j < n; j++) std::swap(V(j, i), V(j, k));
        }
    }
}

std::vector<double> gto_widths(int size, double radius) {
    std::vector<double> w(size);
    for (int n = 0; n < size; n++) w[n] = radius * std::max(std::sqrt((double)n), 1.0) / (double)size;
    return w;
}

std::vector<double> gto_orthonormalization(int size, double radius) {
    auto w = gto_widths(size, radius);
    std::vector<double> S((size_t)size * size);
    for (int n1 = 0; n1 < size; n1++) {
        double s1 = w[n1], s1sq = s1 * s1;
        for (int n2 = n1; n2 < size; n2++) {
            double s2 = w[n2], s2sq = s2 * s2;
            double e = 0.5 * (3.0 + (double)n1 + (double)n2);
            double v = std::pow(0.5 / s1sq + 0.5 / s2sq, -e) / (soap::powi(s1, n1) * soap::powi(s2, n2)) * soap::gamma_fn(e) /
                       (std::pow(s1 * s2, 1.5) * std::sqrt(soap::gamma_fn((double)n1 + 1.5) * soap::gamma_fn((double)n2 + 1.5)));
            S[(size_t)n2 * size + n1] = v;
            S[(size_t)n1 * size + n2] = v;
        }
    }
    std::vector<double> evals;
    symmetric_eigen(S, size, evals);
    for (int n = 0; n < size; n++) {
        if (evals[n] <= soap::DBL_EPS) {
            throw internal_error("radial overlap matrix is singular, try with a lower max_radial (current value is " +
                                 std::to_string(size - 1) + ")");
        }
        evals[n] = 1.0 / std::sqrt(evals[n]);
    }
    // (V diag(1/sqrt(lambda))) V^T diag(norm)
    std::vector<double> vd((size_t)size * size), M((size_t)size * size, 0.0);
    for (int i = 0; i < size; i++)
        for (int j = 0; j < size; j++) vd[(size_t)i * size + j] = S[(size_t)i * size + j] * evals[j];
    for (int i = 0; i < size; i++) {
        for (int j = 0; j < size; j++) {
            double s = 0.0;
            for (int k = 0; k < size; k++) s += vd[(size_t)i * size + k] * S[(size_t)j * size + k];
            double norm = std::sqrt(2.0 / (soap::powi(w[j], 2 * j + 3) * soap::gamma_fn((double)j + 1.5)));
            M[(size_t)i * size + j] = s * norm;
        }
    }
    return M;
}

}  // namespace

std::vector<double> gto_basis_widths(int size, double radius) { return gto_widths(size, radius); }
std::vector<double> gto_basis_orthonormalization(int size, double radius) { return gto_orthonormalization(size, radius); }

void radial_integral_host(const RadialTables& t, int l, double r, double* values, double* grads) {
    int N = t.nmax;
    if (t.splined) {
        const double* pos = &t.positions[t.knot_offset[l]];
        int count = t.knot_count[l];
        int k = soap::spline_interval(pos, count, r);
        auto w = soap::hermite_weights(pos[k], pos[k + 1], r);
        const double* pv = &t.values[((size_t)t.knot_offset[l] + k) * N];
        const double* pd = &t.derivs[((size_t)t.knot_offset[l] + k) * N];
        for (int n = 0; n < N; n++) {
            values[n] = soap::hermite_value(w, pv[n], pd[n], pv[N + n], pd[N + n]);
            if (grads) grads[n] = soap::hermite_derivative(w, pv[n], pd[n], pv[N + n], pd[N + n]);
        }
        return;
    }
    std::vector<double> v(N), g(N);
    if (!soap::gto_radial_raw(l, N, r, t.c, t.width2, t.bn.data(), v.data(), grads ? g.data() : nullptr)) {
        throw internal_error("Failed to compute radial integral with GTO basis. Try increasing decreasing the `cutoff`, "
                             "or increasing the Gaussian's `width`.");
    }
    for (int k = 0; k < N; k++) {
        double s = 0.0, sg = 0.0;
        for (int n = 0; n < N; n++) {
            s += v[n] * t.ortho[(size_t)k * N + n];
            if (grads) sg += g[n] * t.ortho[(size_t)k * N + n];
        }
        values[k] = s;
        if (grads) grads[k] = sg;
    }
}

// featomic/src/calculators/lode/spherical_expansion.rs:30-58 and :180-224
// (validation); LodeRadialBasis::Gto of shared/basis/radial/mod.rs:55-68
LodeHypers parse_lode_hypers(const std::string& text) {
    Value root;
    try {
        root = json::parse(text);
    } catch (json::ParseError& e) {
        throw json_error(e.what());
    }
    object(root, "struct LodeSphericalExpansionParameters");
    LodeHypers h;
    const Value& density = object(field(root, "density", "parameters"), "struct Density");
    std::string dt = tag(density, "Density");
    if (dt != "SmearedPowerLaw") {
        if (dt != "Gaussian" && dt != "DiracDelta")
            throw json_error("unknown variant `" + dt + "`, expected one of `DiracDelta`, `Gaussian`, `SmearedPowerLaw`");
        throw invalid_parameter("only SmearedPowerLaw density can be used with LODE");
    }
    h.smearing = as_f64(field(density, "smearing", "SmearedPowerLaw"), "smearing");
    h.exponent = (int)as_usize(field(density, "exponent", "SmearedPowerLaw"), "exponent");
    if (const Value* cw = density.get("center_atom_weight")) h.center_atom_weight = as_f64(*cw, "center_atom_weight");
    if (const Value* sc = density.get("scaling"))
        if (sc->kind != Value::Null) throw invalid_parameter("LODE does not support custom density scaling");
    if (h.exponent >= 10) throw invalid_parameter("LODE is only implemented for potential_exponent < 10");
    h.k_cutoff = 1.2 * M_PI / h.smearing;
    if (const Value* kc = root.get("k_cutoff"))
        if (kc->kind != Value::Null) h.k_cutoff = as_f64(*kc, "k_cutoff");

    const Value& basis = object(field(root, "basis", "parameters"), "internally tagged enum SphericalExpansionBasis");
    std::string bt = tag(basis, "SphericalExpansionBasis");
    if (bt == "Explicit") throw invalid_parameter("the Explicit basis is not supported by featomic-b200's LODE");
    if (bt != "TensorProduct") throw json_error("unknown variant `" + bt + "`, expected `TensorProduct` or `Explicit`");
    deny_unknown(basis, {"type", "max_angular", "radial", "spline_accuracy"}, "TensorProduct");
    h.max_angular = (int)as_usize(field(basis, "max_angular", "TensorProduct"), "max_angular");
    const Value& radial = object(field(basis, "radial", "TensorProduct"), "internally tagged enum LodeRadialBasis");
    std::string rt = tag(radial, "LodeRadialBasis");
    if (rt == "Tabulated") throw invalid_parameter("the Tabulated radial basis is not supported by featomic-b200's LODE");
    if (rt != "Gto") throw json_error("unknown variant `" + rt + "`, expected `Gto` or `Tabulated`");
    deny_unknown(radial, {"type", "max_radial", "radius"}, "Gto");
    h.max_radial = (int)as_usize(field(radial, "max_radial", "Gto"), "max_radial");
    h.radius = as_f64(field(radial, "radius", "Gto"), "radius");
    if (const Value* sa = basis.get("spline_accuracy")) {
        if (sa->kind == Value::Null) h.splined = false;
        else h.spline_accuracy = as_f64(*sa, "spline_accuracy");
    }
    // gto.rs:27-57 (LODE)
    if (h.radius < 1e-16) throw invalid_parameter("radius of GTO radial basis can not be negative");
    if (!std::isfinite(h.radius)) throw invalid_parameter("radius of GTO radial basis can not be infinite/NaN");
    if (h.splined && h.spline_accuracy < 0.0) {
        std::ostringstream m;
        m << "got invalid accuracy in spline (" << h.spline_accuracy << "), it must be positive";
        throw invalid_parameter(m.str());
    }
    if (h.max_angular > 16) throw invalid_parameter("featomic-b200's LODE supports max_angular <= 16");
    if (h.nmax() > 64) throw invalid_parameter("featomic-b200's LODE supports max_radial < 64");
    return h;
}

void build_spline_knots(const std::function<void(double, double*, double*)>& eval, double stop, int N, int NL,
                        double accuracy, std::vector<double>& pos, std::vector<double>& val, std::vector<double>& der) {
    pos.clear();
    val.clear();
    der.clear();
    std::vector<double> v(N), d(N);
    const int initial = 11;
    double step = (stop - 0.0) / (double)(initial - 1);
    for (int k = 0; k < initial - 1; k++) {
        double x = 0.0 + (double)k * step;
        eval(x, v.data(), d.data());
        pos.push_back(x);
        val.insert(val.end(), v.begin(), v.end());
        der.insert(der.end(), d.begin(), d.end());
    }
    eval(stop, v.data(), d.data());
    pos.push_back(stop);
    val.insert(val.end(), v.begin(), v.end());
    der.insert(der.end(), d.begin(), d.end());

    while (true) {
        double mean_abs = 0.0, mean_rel = 0.0;
        size_t count = 0;
        std::vector<double> mid_pos, mid_val, mid_der;
        for (size_t k = 0; k + 1 < pos.size(); k++) {
            double x = (pos[k] + pos[k + 1]) / 2.0;
            eval(x, v.data(), d.data());
            auto w = soap::hermite_weights(pos[k], pos[k + 1], x);
            for (int n = 0; n < NL; n++) {
                double s = soap::hermite_value(w, val[k * N + n], der[k * N + n], val[(k + 1) * N + n], der[(k + 1) * N + n]);
                mean_abs += std::fabs(s - v[n]);
                mean_rel += std::fabs((s - v[n]) / v[n]);
                count++;
            }
            mid_pos.push_back(x);
            mid_val.insert(mid_val.end(), v.begin(), v.end());
            mid_der.insert(mid_der.end(), d.begin(), d.end());
        }
        if (count == 0) break;  // an angular channel absent from an Explicit basis
        mean_abs /= (double)count;
        mean_rel /= (double)count;
        if (mean_abs < accuracy || mean_rel < accuracy) break;
        if (pos.size() + mid_pos.size() > 10000) {
            std::ostringstream m;
            m << "failed to reach requested accuracy (" << accuracy
              << ") in spline interpolation, mean absolute error is " << mean_abs
              << " and mean relative error is " << mean_rel;
            throw internal_error(m.str());
        }
        std::vector<double> p2, v2, d2;
        for (size_t k = 0; k < pos.size(); k++) {
            p2.push_back(pos[k]);
            v2.insert(v2.end(), val.begin() + k * N, val.begin() + (k + 1) * N);
            d2.insert(d2.end(), der.begin() + k * N, der.begin() + (k + 1) * N);
            if (k < mid_pos.size()) {
                p2.push_back(mid_pos[k]);
                v2.insert(v2.end(), mid_val.begin() + k * N, mid_val.begin() + (k + 1) * N);
                d2.insert(d2.end(), mid_der.begin() + k * N, mid_der.begin() + (k + 1) * N);
            }
        }
        pos.swap(p2);
        val.swap(v2);
        der.swap(d2);
    }
}

// Adaptive knots: 11 uniform points on [0, rc], then every interval midpoint
// is added until the mean absolute or the mean relative interpolation error
// at the midpoints drops below the accuracy (featomic/src/math/splines.rs:79-193,
// limit of 10 000 points).
RadialTables build_radial_tables(const Hypers& h) {
    RadialTables t;
    t.lmax = h.max_angular;
    t.nmax = h.nmax();
    t.splined = false;  // evaluate analytically while building the knots
    // (the analytic GTO parameters are not used with a Tabulated basis)
    t.c = h.tabulated_basis() ? 0.0 : 1.0 / (2.0 * h.density_width * h.density_width);
    t.width2 = h.density_width * h.density_width;
    for (double s : gto_widths(t.nmax, h.cutoff)) t.bn.push_back(1.0 / (2.0 * s * s));
    t.ortho = gto_orthonormalization(t.nmax, h.cutoff);
    int N = t.nmax;

    std::vector<double> all_pos, all_val, all_der;
    std::vector<int32_t> offsets, counts;
    if (h.tabulated_basis()) {
        // the user's control points, each channel padded with zero functions
        // to N (radial_integral/spline.rs from_tabulated)
        for (int l = 0; l <= h.max_angular; l++) {
            const TabulatedSpline& ts = h.tabulated[l];
            offsets.push_back((int32_t)all_pos.size());
            if (ts.size == 0) {
                all_pos.insert(all_pos.end(), {0.0, h.cutoff});
                all_val.insert(all_val.end(), 2 * (size_t)N, 0.0);
                all_der.insert(all_der.end(), 2 * (size_t)N, 0.0);
                counts.push_back(2);
                continue;
            }
            counts.push_back((int32_t)ts.positions.size());
            for (size_t k = 0; k < ts.positions.size(); k++) {
                all_pos.push_back(ts.positions[k]);
                for (int n = 0; n < N; n++) {
                    all_val.push_back(n < ts.size ? ts.values[k * ts.size + n] : 0.0);
                    all_der.push_back(n < ts.size ? ts.derivs[k * ts.size + n] : 0.0);
                }
            }
        }
        t.knot_offset = offsets;
        t.knot_count = counts;
        t.positions = all_pos;
        t.values = all_val;
        t.derivs = all_der;
        t.splined = true;
    } else if (h.splined) {
        for (int l = 0; l <= h.max_angular; l++) {
            std::vector<double> pos, val, der;
            // Explicit basis: channel l has its own GTO basis of radial_sizes[l]
            // functions (its own widths and orthonormalisation), evaluated and
            // splined with those functions only, then padded with zeros to N
            RadialTables tl;
            int NL = N;
            if (h.explicit_basis()) {
                NL = h.radial_sizes[l];
                tl = t;
                tl.nmax = NL;
                tl.bn.clear();
                for (double sw : gto_widths(std::max(NL, 1), h.cutoff)) tl.bn.push_back(1.0 / (2.0 * sw * sw));
                tl.ortho = gto_orthonormalization(std::max(NL, 1), h.cutoff);
            }
            auto eval = [&](double x, std::vector<double>& v, std::vector<double>& d) {
                v.assign(N, 0.0);
                d.assign(N, 0.0);
                if (!h.explicit_basis()) {
                    radial_integral_host(t, l, x, v.data(), d.data());
                } else if (NL > 0) {
                    radial_integral_host(tl, l, x, v.data(), d.data());
                }
            };
            std::vector<double> v, d;
            build_spline_knots([&](double x, double* vv, double* dd) {
                eval(x, v, d);
                std::copy(v.begin(), v.end(), vv);
                std::copy(d.begin(), d.end(), dd);
            }, h.cutoff, N, NL, h.spline_accuracy, pos, val, der);
            offsets.push_back((int32_t)all_pos.size());
            counts.push_back((int32_t)pos.size());
            all_pos.insert(all_pos.end(), pos.begin(), pos.end());
            all_val.insert(all_val.end(), val.begin(), val.end());
            all_der.insert(all_der.end(), der.begin(), der.end());
        }
        t.knot_offset = offsets;
        t.knot_count = counts;
        t.positions = all_pos;
        t.values = all_val;
        t.derivs = all_der;
        t.splined = true;
    }

    // self contribution: centre weight * f(0) * Y00(z) * I_n^{l=0}(0)
    std::vector<double> r0(N);
    radial_integral_host(t, 0, 0.0, r0.data(), nullptr);
    double f0, df0;
    soap::cutoff_function(h.smoothing, h.cutoff, h.smoothing_width, 0.0, &f0, &df0);
    double scale = 1.0;
    if (h.scaling) {
        double ds;
        soap::willatt2018(h.scaling_scale, h.scaling_rate, h.scaling_exponent, 0.0, &scale, &ds);
    }
    const double y00 = 0.3989422804014327 / 1.4142135623730951;  // P_0^0 / sqrt(2)
    double factor = h.center_atom_weight * (scale * f0) * y00;
    t.self_contribution.resize(N);
    for (int n = 0; n < N; n++) t.self_contribution[n] = factor * r0[n];
    return t;
}

// Constant factors of the Legendre recursion and of the derivative factors,
// featomic/src/math/spherical_harmonics.rs:203-301 (same expressions, hoisted
// out of the per-pair evaluation).
YlmTables build_ylm_tables(int lmax) {
    YlmTables t;
    t.lmax = lmax;
    size_t n = (size_t)(lmax + 1) * (lmax + 2) / 2;
    t.A.assign(n, 0.0);
    t.B.assign(n, 0.0);
    t.sq_plus.assign(n, 0.0);
    t.sq_minus.assign(n, 0.0);
    t.sq_2l1.assign(lmax + 1, 0.0);
    t.sq_half.assign(lmax + 1, 0.0);
    t.sq_ll1.assign(lmax + 1, 0.0);
    t.inv_ll.assign(lmax + 1, 0.0);
    auto li = [](int l, int m) { return (size_t)(m + l * (l + 1) / 2); };
    for (int l = 2; l <= lmax; l++) {
        double ls = (double)(l * l), lm1s = (double)((l - 1) * (l - 1));
        for (int m = 0; m < l - 1; m++) {
            double ms = (double)(m * m);
            t.A[li(l, m)] = std::sqrt((4.0 * ls - 1.0) / (ls - ms));
            t.B[li(l, m)] = -std::sqrt((lm1s - ms) / (4.0 * lm1s - 1.0));
        }
    }
    for (int l = 0; l <= lmax; l++) {
        t.sq_2l1[l] = std::sqrt(2.0 * (double)l + 1.0);
        t.sq_half[l] = l > 0 ? std::sqrt(1.0 + 0.5 / (double)l) : 0.0;
        t.sq_ll1[l] = std::sqrt(0.5 * (double)(l * (l + 1)));
        t.inv_ll[l] = l > 0 ? -1.0 / (double)(l * l + l) : 0.0;
        for (int m = 0; m <= l; m++) {
            t.sq_plus[li(l, m)] = std::sqrt((double)((l + m) * (l - m + 1)));
            t.sq_minus[li(l, m)] = std::sqrt((double)((l - m) * (l + m + 1)));
        }
    }
    return t;
}

}  // namespace fb200

// Calculator facade: registry, construction from JSON and dispatch to the
// engine (featomic/src/calculator.rs:243-526, registry :574-588): spherical
// expansion, spherical expansion by pair, SOAP power spectrum, SOAP radial
// spectrum and the LODE spherical expansion.
#include "engine.hpp"
#include "host.hpp"
#include "lode.hpp"

namespace fb200 {

CalculatorImpl::~CalculatorImpl() = default;

std::unique_ptr<CalculatorImpl> create_calculator(const std::string& name, const std::string& json) {
    auto c = std::make_unique<CalculatorImpl>();
    c->name = name;
    c->parameters = json;
    if (name == "spherical_expansion") {
        c->pretty_name = "spherical expansion";
        c->hypers = parse_hypers(json, /*deny_unknown_top=*/true);
        c->power_spectrum = false;
    } else if (name == "soap_power_spectrum") {
        c->pretty_name = "SOAP power spectrum";
        c->hypers = parse_hypers(json, /*deny_unknown_top=*/false);
        c->power_spectrum = true;
    } else if (name == "soap_radial_spectrum") {
        c->pretty_name = "radial spectrum";
        c->hypers = parse_hypers(json, /*deny_unknown_top=*/false, /*radial_spectrum_basis=*/true);
        c->power_spectrum = false;
        c->radial_spectrum = true;
    } else if (name == "spherical_expansion_by_pair") {
        c->pretty_name = "spherical expansion by pair";
        c->hypers = parse_hypers(json, /*deny_unknown_top=*/true);
        c->power_spectrum = false;
        c->by_pair = true;
    } else if (name == "lode_spherical_expansion") {
        // no cutoff: every atom of the periodic system is a neighbour
        c->pretty_name = "lode spherical expansion";
        LodeHypers lh = parse_lode_hypers(json);
        c->hypers.max_angular = lh.max_angular;
        c->hypers.max_radial = lh.max_radial;
        c->lode = std::make_unique<LodeEngine>(lh);
        return c;
    } else if (name == "atomic_composition" || name == "dummy_calculator" || name == "neighbor_list" ||
               name == "sorted_distances") {
        throw invalid_parameter("calculator '" + name + "' is not implemented by featomic-b200");
    } else {
        throw invalid_parameter("unknown calculator with name '" + name + "'");
    }
    c->cutoffs = {c->hypers.cutoff};
    c->engine = std::make_unique<Engine>(c->hypers);
    return c;
}

namespace {

// The radial spectrum is the l = 0 spherical expansion with its keys
// (o3_lambda = 0, o3_sigma = 1, center_type, neighbor_type) reduced to
// (center_type, neighbor_type) and the single o3_mu component dropped
// (radial_spectrum.rs:102-130, :237-323).  The data layout is the same, so
// only the metadata changes: values [samples, n], positions gradients
// [rows, xyz, n], strain [samples, xyz_2, xyz_1, n], cell [samples, xyz, abc, n].
void drop_mu_component(Block& b) {
    if (b.components.empty() || b.components.back().names != std::vector<std::string>{"o3_mu"})
        throw internal_error("radial spectrum: expected an o3_mu component");
    b.components.pop_back();
    b.shape.erase(b.shape.end() - 2);
}

void to_radial_spectrum(TensorMap& tm) {
    Labels keys;
    keys.names = {"center_type", "neighbor_type"};
    const size_t width = tm.keys.names.size();
    for (size_t k = 0; k < tm.keys.count(); k++) {
        if (tm.keys.values[k * width] != 0) throw internal_error("radial spectrum: expected o3_lambda = 0 only");
        keys.values.push_back(tm.keys.values[k * width + 2]);
        keys.values.push_back(tm.keys.values[k * width + 3]);
    }
    tm.keys = std::move(keys);
    for (auto& b : tm.blocks) {
        drop_mu_component(*b);
        for (auto& g : b->gradients) drop_mu_component(*g.second);
    }
}

// Explicit basis (basis/mod.rs:95-116): the engine runs every channel with
// max_radial + 1 functions, the channels with fewer padded with zero
// functions; the output keeps the angular channels of the basis (keys with
// their o3_lambda) and, per channel, its own radial functions (properties n,
// or (l, n_1, n_2) of the power spectrum, power_spectrum.rs:512-523).
std::unique_ptr<TensorMap> explicit_basis_output(std::unique_ptr<TensorMap> tm, const Hypers& h) {
    if (!tm || tm->blocks.empty()) return tm;
    const auto& size = h.radial_sizes;
    size_t lc = 0;
    while (lc < tm->keys.names.size() && tm->keys.names[lc] != "o3_lambda") lc++;
    const bool has_lambda = lc < tm->keys.names.size();
    const size_t kw = tm->keys.names.size();
    Labels keys;
    keys.names = tm->keys.names;
    TensorMap props;
    for (size_t k = 0; k < tm->keys.count(); k++) {
        const Block& src = *tm->blocks[k];
        auto blk = std::make_unique<Block>();
        blk->properties.names = src.properties.names;
        const size_t pw = src.properties.names.size();
        if (has_lambda) {
            const int l = tm->keys.values[k * kw + lc];
            if (size[l] == 0) continue;  // channel absent from the basis
            for (int n = 0; n < size[l]; n++) blk->properties.values.push_back(n);
        } else if (pw == 3) {
            for (size_t r = 0; r < src.properties.count(); r++) {
                const int32_t* p = &src.properties.values[3 * r];
                if (p[1] < size[p[0]] && p[2] < size[p[0]]) blk->properties.values.insert(blk->properties.values.end(), p, p + 3);
            }
        } else {
            // l = 0 only (radial spectrum)
            for (int n = 0; n < size[0]; n++) blk->properties.values.push_back(n);
        }
        keys.values.insert(keys.values.end(), tm->keys.values.begin() + k * kw, tm->keys.values.begin() + (k + 1) * kw);
        props.blocks.push_back(std::move(blk));
    }
    props.keys = keys;
    Selection sel;
    sel.keys = &keys;
    sel.properties_predefined = &props;
    sel.max_angular = h.max_angular;
    return apply_selection(std::move(tm), sel);
}

}  // namespace

std::unique_ptr<TensorMap> compute(CalculatorImpl& calc, std::vector<HostSystem>& systems, const GradientOptions& grads,
                                   bool device_output, const double* positions_device, void* stream) {
    if (calc.lode) return calc.lode->compute(systems, grads, device_output, positions_device, (cudaStream_t)stream);
    if (calc.hypers.explicit_basis() && device_output)
        throw invalid_parameter("the Explicit basis is supported with host output (featomic_calculator_compute) only");
    const int kind = calc.power_spectrum ? Engine::OUTPUT_POWER_SPECTRUM
                     : calc.by_pair      ? Engine::OUTPUT_BY_PAIR
                                         : Engine::OUTPUT_EXPANSION;
    auto tm = calc.engine->compute(kind, systems, grads, device_output, positions_device, (cudaStream_t)stream);
    if (calc.radial_spectrum && tm) to_radial_spectrum(*tm);
    if (calc.hypers.explicit_basis()) tm = explicit_basis_output(std::move(tm), calc.hypers);
    return tm;
}

}  // namespace fb200

// Calculator facade: registry, construction from JSON and dispatch to the
// engine (featomic/src/calculator.rs:243-526, registry :574-588).
#include "engine.hpp"
#include "host.hpp"

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
    } else if (name == "spherical_expansion_by_pair" || name == "soap_radial_spectrum" ||
               name == "lode_spherical_expansion" || name == "atomic_composition" || name == "dummy_calculator" ||
               name == "neighbor_list" || name == "sorted_distances") {
        throw invalid_parameter("calculator '" + name + "' is not implemented by featomic-b200");
    } else {
        throw invalid_parameter("unknown calculator with name '" + name + "'");
    }
    c->cutoffs = {c->hypers.cutoff};
    c->engine = std::make_unique<Engine>(c->hypers);
    return c;
}

std::unique_ptr<TensorMap> compute(CalculatorImpl& calc, std::vector<HostSystem>& systems, const GradientOptions& grads,
                                   bool device_output, const double* positions_device, void* stream) {
    return calc.engine->compute(calc.power_spectrum, systems, grads, device_output, positions_device,
                                (cudaStream_t)stream);
}

}  // namespace fb200

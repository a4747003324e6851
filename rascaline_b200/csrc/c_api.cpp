// featomic's C ABI on top of the B200 engine (see include/featomic_b200.h).
//
// Errors follow featomic/src/c_api/status.rs: every entry point catches
// exceptions, stores the message in a thread-local buffer read by
// featomic_last_error(), and returns the status code of the error kind.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <sstream>

#include "../../include/featomic_b200.h"
#include "batched.hpp"
#include "clebsch_gordan.hpp"
#include "dense.hpp"
#include "engine.hpp"
#include "host.hpp"
#include "lode.hpp"
#include "surrogate.hpp"

using namespace fb200;

struct featomic_calculator_t {
    std::unique_ptr<CalculatorImpl> impl;
};

struct mts_block_t {
    Block* block;
    bool on_device = false;
    std::vector<std::unique_ptr<mts_block_t>> gradient_handles;
    std::vector<const char*> gradient_names;
    // name pointer storage for labels
    std::vector<std::vector<const char*>> name_ptrs;
    std::vector<uintptr_t> shape;
};

struct mts_tensormap_t {
    std::unique_ptr<TensorMap> tm;
    std::vector<std::unique_ptr<mts_block_t>> handles;
    std::vector<const char*> key_names;
};

namespace {

thread_local std::string LAST_ERROR;

std::mutex LOG_MUTEX;
featomic_logging_callback_t LOG_CALLBACK = nullptr;

void log_message(int32_t level, const std::string& msg) {
    std::lock_guard<std::mutex> lock(LOG_MUTEX);
    if (LOG_CALLBACK) LOG_CALLBACK(level, ("featomic_b200 -- " + msg).c_str());
}

template <typename F>
featomic_status_t guarded(F&& f) {
    try {
        f();
        return FEATOMIC_SUCCESS;
    } catch (Error& e) {
        LAST_ERROR = e.what();
        return e.status;
    } catch (std::bad_alloc&) {
        LAST_ERROR = "out of memory";
        return FEATOMIC_INTERNAL_ERROR;
    } catch (std::exception& e) {
        LAST_ERROR = std::string("internal error: ") + e.what();
        return FEATOMIC_INTERNAL_ERROR;
    } catch (...) {
        LAST_ERROR = "internal error: unknown exception";
        return FEATOMIC_INTERNAL_ERROR;
    }
}

#define CHECK_POINTER(p)                                                                                   \
    do {                                                                                                   \
        if ((p) == nullptr)                                                                                \
            throw invalid_parameter(std::string("got invalid NULL pointer for ") + #p + " at " + __FILE__ + \
                                    ":" + std::to_string(__LINE__));                                       \
    } while (0)

void copy_str(const std::string& s, char* buffer, uintptr_t len) {
    if (s.size() + 1 > len) {
        throw Error(FEATOMIC_BUFFER_SIZE_ERROR, "string buffer is not big enough: got space for " + std::to_string(len) +
                                                    " characters, but we need " + std::to_string(s.size() + 1));
    }
    std::memcpy(buffer, s.c_str(), s.size() + 1);
}

void check_system_status(featomic_status_t status, const char* what) {
    if (status == FEATOMIC_SUCCESS) return;
    std::string msg = std::string("error in C system callback `") + what + "`";
    if (status < 0) throw Error(status, msg);
    throw Error(FEATOMIC_SYSTEM_ERROR, msg);
}

struct Profile {
    std::mutex mutex;
    bool enabled = false;
    std::map<std::string, std::pair<double, int64_t>> spans;  // name -> (total ms, calls)
    void add(const std::string& name, double ms) {
        if (!enabled) return;
        auto& s = spans[name];
        s.first += ms;
        s.second++;
    }
};

Profile& profile() {
    static Profile p;
    return p;
}

void record_profile(const PhaseTimes& t) {
    Profile& p = profile();
    std::lock_guard<std::mutex> lock(p.mutex);
    p.add("Calculator::compute", t.total);
    p.add("NeighborsList", t.neighbors);
    p.add("Calculator::prepare", t.metadata);
    p.add("SphericalExpansion::pair_features", t.features);
    p.add("SphericalExpansion::compute", t.expansion);
    p.add("SoapPowerSpectrum::compute", t.contraction);
    p.add("TensorMap::to_host", t.transfer);
}

GradientOptions parse_options(const featomic_calculation_options_t& options) {
    GradientOptions g;
    if (options.gradients_count > 0) CHECK_POINTER(options.gradients);
    for (uintptr_t k = 0; k < options.gradients_count; k++) {
        CHECK_POINTER(options.gradients[k]);
        std::string p = options.gradients[k];
        if (p == "positions") g.positions = true;
        else if (p == "strain") g.strain = true;
        else if (p == "cell") g.cell = true;
        else
            throw invalid_parameter("unexpected gradient \"" + p +
                                    "\", should be one of \"positions\", \"cell\", or \"strain\"");
    }
    if (g.cell && std::getenv("FEATOMIC_NO_WARN_CELL_GRADIENTS") == nullptr) {
        log_message(FEATOMIC_LOG_LEVEL_WARN,
                    "The meaning of \"cell\" gradients has changed recently, you likely want \"strain\" gradients "
                    "instead. Please review the documentation carefully.");
    }
    return g;
}

Labels labels_from_c(const mts_labels_t* c, const char* what) {
    Labels out;
    if (c->size > 0) CHECK_POINTER(c->names);
    if (c->count > 0 && c->size > 0) CHECK_POINTER(c->values);
    for (uintptr_t k = 0; k < c->size; k++) {
        if (!c->names[k]) throw invalid_parameter(std::string("NULL name in ") + what + " selection");
        out.names.push_back(c->names[k]);
    }
    out.values.assign(c->values, c->values + c->size * c->count);
    return out;
}

// The atoms within the cutoff of an atom, for the gradient samples of
// predefined samples the full calculation does not produce: the systems' own
// pairs, or the neighbour list kernel on positions from the host or (device
// entry point) copied from the device; one list per system, built on first use
struct NeighborCache {
    const std::vector<HostSystem>* systems = nullptr;
    double cutoff = 0.0;
    const double* device_positions = nullptr;  // concatenated positions on the device
    std::map<int64_t, std::vector<std::vector<int32_t>>> lists;

    std::vector<int32_t> operator()(int64_t system, int64_t atom) {
        auto it = lists.find(system);
        if (it == lists.end()) {
            const HostSystem& s = (*systems)[system];
            std::vector<std::vector<int32_t>> around(s.n_atoms);
            std::vector<Pair> pairs;
            if (s.has_pairs) {
                pairs = s.pairs;
            } else if (device_positions) {
                int64_t off = 0;
                for (int64_t k = 0; k < system; k++) off += (*systems)[k].n_atoms;
                std::vector<double> positions(3 * s.n_atoms);
                if (s.n_atoms &&
                    cudaMemcpy(positions.data(), device_positions + 3 * off, sizeof(double) * 3 * s.n_atoms,
                               cudaMemcpyDeviceToHost) != cudaSuccess) {
                    cudaGetLastError();
                    throw internal_error("could not read the positions back from the device");
                }
                pairs = neighbor_list(positions.data(), s.n_atoms, s.cell, cutoff);
            } else {
                pairs = neighbor_list(s.positions.data(), s.n_atoms, s.cell, cutoff);
            }
            for (auto& p : pairs) {
                around[p.first].push_back((int32_t)p.second);
                around[p.second].push_back((int32_t)p.first);
            }
            it = lists.emplace(system, std::move(around)).first;
        }
        return it->second[atom];
    }
};

// featomic's selections in C form (featomic.h:245-277) -> owned labels
struct SelectionStorage {
    Labels keys, samples, properties;
    Selection selection;
    std::shared_ptr<NeighborCache> neighbors = std::make_shared<NeighborCache>();
};

void parse_selections(const featomic_calculation_options_t& options, int max_angular, SelectionStorage& st,
                      const std::vector<HostSystem>& systems, double cutoff, const double* device_positions = nullptr) {
    st.selection.max_angular = max_angular;
    st.neighbors->systems = &systems;
    st.neighbors->cutoff = cutoff;
    st.neighbors->device_positions = device_positions;
    st.selection.systems = cutoff > 0.0 ? &systems : nullptr;  // no neighbour rule without a cutoff
    auto cache = st.neighbors;
    st.selection.neighbors = [cache](int64_t system, int64_t atom) { return (*cache)(system, atom); };
    if (options.selected_keys) {
        st.keys = labels_from_c(options.selected_keys, "keys");
        st.selection.keys = &st.keys;
    }
    const featomic_labels_selection_t* which[2] = {&options.selected_samples, &options.selected_properties};
    for (int k = 0; k < 2; k++) {
        const featomic_labels_selection_t& s = *which[k];
        const char* kind = k == 0 ? "samples" : "properties";
        if (s.subset && s.predefined)
            throw invalid_parameter(std::string("can not have both a subset and a predefined ") + kind + " selection");
        if (s.subset) {
            Labels& dst = k == 0 ? st.samples : st.properties;
            dst = labels_from_c(s.subset, kind);
            (k == 0 ? st.selection.samples : st.selection.properties) = &dst;
        }
        if (s.predefined) (k == 0 ? st.selection.samples_predefined : st.selection.properties_predefined) = s.predefined->tm.get();
    }
}

const PhaseTimes& last_times(const CalculatorImpl& c) {
    return c.lode ? c.lode->last_times() : c.engine->last_times();
}

// the SOAP engine behind an entry point that only SOAP calculators have
Engine& soap_engine(const featomic_calculator_t* calculator) {
    if (!calculator->impl->engine)
        throw invalid_parameter("this function needs a SOAP calculator (spherical expansion, power spectrum or "
                                "radial spectrum), not " + calculator->impl->name);
    return *calculator->impl->engine;
}

mts_tensormap_t* wrap(std::unique_ptr<TensorMap> tm) {
    auto* out = new mts_tensormap_t;
    out->tm = std::move(tm);
    for (auto& n : out->tm->keys.names) out->key_names.push_back(n.c_str());
    for (auto& b : out->tm->blocks) {
        auto h = std::make_unique<mts_block_t>();
        h->block = b.get();
        h->on_device = out->tm->on_device;
        for (auto& g : b->gradients) {
            auto gh = std::make_unique<mts_block_t>();
            gh->block = g.second.get();
            gh->on_device = out->tm->on_device;
            h->gradient_names.push_back(g.first.c_str());
            h->gradient_handles.push_back(std::move(gh));
        }
        out->handles.push_back(std::move(h));
    }
    return out;
}

void fill_labels(const Labels& l, std::vector<const char*>& names, mts_labels_t* out) {
    names.clear();
    for (auto& n : l.names) names.push_back(n.c_str());
    out->internal_ptr_ = nullptr;
    out->names = names.data();
    out->values = l.values.data();
    out->size = l.names.size();
    out->count = l.count();
}

void warn_close_pairs(const std::vector<HostSystem>& systems) {
    for (auto& s : systems)
        for (auto& p : s.pairs)
            if (p.distance * p.distance < 1e-3)
                log_message(FEATOMIC_LOG_LEVEL_WARN, "atoms " + std::to_string(p.first) + " and " + std::to_string(p.second) +
                                                         " are very close to one another (" + std::to_string(p.distance) + " A)");
}

}  // namespace

extern "C" {

const char* featomic_last_error(void) { return LAST_ERROR.c_str(); }

featomic_status_t featomic_set_logging_callback(featomic_logging_callback_t callback) {
    return guarded([&] {
        std::lock_guard<std::mutex> lock(LOG_MUTEX);
        LOG_CALLBACK = callback;
    });
}

featomic_calculator_t* featomic_calculator(const char* name, const char* parameters) {
    featomic_calculator_t* out = nullptr;
    featomic_status_t status = guarded([&] {
        CHECK_POINTER(name);
        CHECK_POINTER(parameters);
        auto impl = create_calculator(name, parameters);
        out = new featomic_calculator_t{std::move(impl)};
    });
    if (status != FEATOMIC_SUCCESS) return nullptr;
    return out;
}

featomic_status_t featomic_calculator_free(featomic_calculator_t* calculator) {
    return guarded([&] { delete calculator; });
}

featomic_status_t featomic_calculator_name(const featomic_calculator_t* calculator, char* name, uintptr_t bufflen) {
    return guarded([&] {
        CHECK_POINTER(calculator);
        CHECK_POINTER(name);
        copy_str(calculator->impl->pretty_name, name, bufflen);
    });
}

featomic_status_t featomic_calculator_parameters(const featomic_calculator_t* calculator, char* parameters,
                                                 uintptr_t bufflen) {
    return guarded([&] {
        CHECK_POINTER(calculator);
        CHECK_POINTER(parameters);
        copy_str(calculator->impl->parameters, parameters, bufflen);
    });
}

featomic_status_t featomic_calculator_cutoffs(const featomic_calculator_t* calculator, const double** cutoffs,
                                              uintptr_t* cutoffs_count) {
    return guarded([&] {
        CHECK_POINTER(calculator);
        CHECK_POINTER(cutoffs);
        CHECK_POINTER(cutoffs_count);
        *cutoffs = calculator->impl->cutoffs.data();
        *cutoffs_count = calculator->impl->cutoffs.size();
    });
}

featomic_status_t featomic_calculator_compute(featomic_calculator_t* calculator, mts_tensormap_t** descriptor,
                                              featomic_system_t* systems, uintptr_t systems_count,
                                              featomic_calculation_options_t options) {
    return guarded([&] {
        if (systems_count == 0) {
            log_message(FEATOMIC_LOG_LEVEL_WARN, "0 systems given to featomic_calculator_compute, nothing to do");
            return;
        }
        CHECK_POINTER(calculator);
        CHECK_POINTER(descriptor);
        CHECK_POINTER(systems);
        GradientOptions g = parse_options(options);
        double cutoff = calculator->impl->hypers.cutoff;
        std::vector<HostSystem> host(systems_count);
        for (uintptr_t s = 0; s < systems_count; s++) {
            featomic_system_t& sys = systems[s];
            HostSystem& h = host[s];
            if (!sys.size || !sys.types || !sys.positions || !sys.cell)
                throw invalid_parameter("system callbacks (size, types, positions, cell) can not be NULL");
            uintptr_t n = 0;
            check_system_status(sys.size(sys.user_data, &n), "size");
            h.n_atoms = (int64_t)n;
            const int32_t* types = nullptr;
            const double* positions = nullptr;
            check_system_status(sys.types(sys.user_data, &types), "types");
            check_system_status(sys.positions(sys.user_data, &positions), "positions");
            check_system_status(sys.cell(sys.user_data, h.cell), "cell");
            if (n > 0 && (!types || !positions)) throw Error(FEATOMIC_SYSTEM_ERROR, "system returned NULL types or positions");
            h.types.assign(types, types + n);
            h.positions.assign(positions, positions + 3 * n);
            for (double x : h.positions)
                if (!std::isfinite(x)) throw invalid_parameter("atomic positions must be finite");
            if (!options.use_native_system && !calculator->impl->lode) {
                // the caller's own neighbour list (featomic/src/c_api/system.rs:248-320);
                // the LODE calculator has no cutoff and asks for none
                if (!sys.compute_neighbors || !sys.pairs)
                    throw invalid_parameter("system callbacks `compute_neighbors` and `pairs` are required when use_native_system is false");
                check_system_status(sys.compute_neighbors(sys.user_data, cutoff), "compute_neighbors");
                const featomic_pair_t* pairs = nullptr;
                uintptr_t count = 0;
                check_system_status(sys.pairs(sys.user_data, &pairs, &count), "pairs");
                h.has_pairs = true;
                h.pairs.resize(count);
                for (uintptr_t k = 0; k < count; k++) {
                    h.pairs[k].first = pairs[k].first;
                    h.pairs[k].second = pairs[k].second;
                    h.pairs[k].distance = pairs[k].distance;
                    for (int x = 0; x < 3; x++) {
                        h.pairs[k].vector[x] = pairs[k].vector[x];
                        h.pairs[k].shift[x] = pairs[k].cell_shift_indices[x];
                    }
                }
            }
        }
        SelectionStorage selection;
        parse_selections(options, calculator->impl->hypers.max_angular, selection, host,
                         calculator->impl->hypers.cutoff);
        warn_close_pairs(host);
        auto tm = compute(*calculator->impl, host, g, false, nullptr, nullptr);
        record_profile(last_times(*calculator->impl));
        *descriptor = wrap(apply_selection(std::move(tm), selection.selection));
    });
}

featomic_status_t featomic_b200_calculator_compute_device(featomic_calculator_t* calculator,
                                                          mts_tensormap_t** descriptor,
                                                          const featomic_b200_device_systems_t* systems,
                                                          featomic_calculation_options_t options, void* stream) {
    return guarded([&] {
        CHECK_POINTER(calculator);
        CHECK_POINTER(descriptor);
        CHECK_POINTER(systems);
        GradientOptions g = parse_options(options);
        if (systems->n_systems == 0) {
            log_message(FEATOMIC_LOG_LEVEL_WARN, "0 systems given to featomic_b200_calculator_compute_device, nothing to do");
            return;
        }
        CHECK_POINTER(systems->system_sizes);
        CHECK_POINTER(systems->cells);
        std::vector<HostSystem> host(systems->n_systems);
        int64_t off = 0;
        for (uintptr_t s = 0; s < systems->n_systems; s++) {
            host[s].n_atoms = (int64_t)systems->system_sizes[s];
            if (host[s].n_atoms > 0) CHECK_POINTER(systems->types);
            host[s].types.assign(systems->types + off, systems->types + off + host[s].n_atoms);
            std::memcpy(host[s].cell, systems->cells + 9 * s, 9 * sizeof(double));
            off += host[s].n_atoms;
        }
        if (off > 0) {
            CHECK_POINTER(systems->positions);
            cudaPointerAttributes attr;
            if (cudaPointerGetAttributes(&attr, systems->positions) != cudaSuccess || attr.type != cudaMemoryTypeDevice) {
                cudaGetLastError();
                throw invalid_parameter("featomic_b200_calculator_compute_device expects device positions");
            }
        }
        SelectionStorage selection;
        parse_selections(options, calculator->impl->hypers.max_angular, selection, host,
                         calculator->impl->hypers.cutoff, systems->positions);
        auto tm = compute(*calculator->impl, host, g, true, systems->positions, (cudaStream_t)stream);
        record_profile(last_times(*calculator->impl));
        if (selection.selection.any()) CUDA_CHECK(cudaStreamSynchronize((cudaStream_t)stream));
        *descriptor = wrap(apply_selection(std::move(tm), selection.selection));
    });
}

struct featomic_b200_dense_t {
    std::unique_ptr<fb200::DenseState> state;
};

namespace {

std::vector<HostSystem> device_systems(const featomic_b200_device_systems_t* systems) {
    std::vector<HostSystem> host(systems->n_systems);
    if (systems->n_systems == 0) return host;
    CHECK_POINTER(systems->system_sizes);
    CHECK_POINTER(systems->cells);
    int64_t off = 0;
    for (uintptr_t s = 0; s < systems->n_systems; s++) {
        host[s].n_atoms = (int64_t)systems->system_sizes[s];
        if (host[s].n_atoms > 0) CHECK_POINTER(systems->types);
        host[s].types.assign(systems->types + off, systems->types + off + host[s].n_atoms);
        std::memcpy(host[s].cell, systems->cells + 9 * s, 9 * sizeof(double));
        off += host[s].n_atoms;
    }
    if (off > 0) {
        CHECK_POINTER(systems->positions);
        cudaPointerAttributes attr;
        if (cudaPointerGetAttributes(&attr, systems->positions) != cudaSuccess || attr.type != cudaMemoryTypeDevice) {
            cudaGetLastError();
            throw invalid_parameter("expected device positions");
        }
    }
    return host;
}

}  // namespace

featomic_status_t featomic_b200_power_spectrum_dense(featomic_calculator_t* calculator,
                                                     const featomic_b200_device_systems_t* systems,
                                                     const int32_t* species, uintptr_t n_species, int32_t precision,
                                                     void* values, uintptr_t values_count,
                                                     featomic_b200_dense_t** state, void* stream) {
    return guarded([&] {
        CHECK_POINTER(calculator);
        CHECK_POINTER(systems);
        CHECK_POINTER(state);
        *state = nullptr;
        if (!calculator->impl->power_spectrum)
            throw invalid_parameter("featomic_b200_power_spectrum_dense needs a soap_power_spectrum calculator");
        if (calculator->impl->hypers.explicit_basis())
            throw invalid_parameter("the dense power spectrum does not support the Explicit basis");
        std::vector<HostSystem> host = device_systems(systems);
        std::vector<int32_t> sp;
        if (n_species > 0) {
            CHECK_POINTER(species);
            sp.assign(species, species + n_species);
        }
        auto result = std::make_unique<featomic_b200_dense_t>();
        result->state = soap_engine(calculator).forward_dense(precision, host, systems->positions, sp, values,
                                                                (int64_t)values_count, (cudaStream_t)stream);
        *state = result.release();
    });
}

featomic_status_t featomic_b200_spherical_expansion_dense(featomic_calculator_t* calculator,
                                                          const featomic_b200_device_systems_t* systems,
                                                          const int32_t* species, uintptr_t n_species,
                                                          int32_t precision, void* values, uintptr_t values_count,
                                                          featomic_b200_dense_t** state, void* stream) {
    return guarded([&] {
        CHECK_POINTER(calculator);
        CHECK_POINTER(systems);
        CHECK_POINTER(state);
        *state = nullptr;
        const auto& impl = *calculator->impl;
        if (impl.power_spectrum || impl.radial_spectrum || impl.by_pair)
            throw invalid_parameter("featomic_b200_spherical_expansion_dense needs a spherical_expansion calculator");
        if (impl.hypers.explicit_basis())
            throw invalid_parameter("the dense spherical expansion does not support the Explicit basis");
        std::vector<HostSystem> host = device_systems(systems);
        std::vector<int32_t> sp;
        if (n_species > 0) {
            CHECK_POINTER(species);
            sp.assign(species, species + n_species);
        }
        auto result = std::make_unique<featomic_b200_dense_t>();
        result->state = impl.engine->forward_dense(precision, host, systems->positions, sp, values, (int64_t)values_count,
                                                   (cudaStream_t)stream, /*expansion=*/true);
        *state = result.release();
    });
}

featomic_status_t featomic_b200_dense_shape(const featomic_b200_dense_t* state, uintptr_t* n_atoms,
                                            uintptr_t* n_species, uintptr_t* n_keys, uintptr_t* n_properties,
                                            uintptr_t* n_pairs) {
    return guarded([&] {
        CHECK_POINTER(state);
        const DenseState& st = *state->state;
        if (n_atoms) *n_atoms = (uintptr_t)st.n_atoms;
        if (n_species) *n_species = (uintptr_t)st.n_species;
        if (n_keys) *n_keys = (uintptr_t)st.n_keys;
        if (n_properties) *n_properties = (uintptr_t)st.n_props;
        if (n_pairs) *n_pairs = (uintptr_t)st.n_pairs;
    });
}

featomic_status_t featomic_b200_dense_species(const featomic_b200_dense_t* state, int32_t* species,
                                              int32_t* neighbor_counts) {
    return guarded([&] {
        CHECK_POINTER(state);
        const DenseState& st = *state->state;
        if (species) std::copy(st.species_types.begin(), st.species_types.end(), species);
        if (neighbor_counts && st.n_atoms > 0) {
            const int64_t n = st.n_atoms * st.n_species + 1;
            std::vector<int64_t> seg(n);
            CUDA_CHECK(cudaMemcpyAsync(seg.data(), st.seg_offset, sizeof(int64_t) * n, cudaMemcpyDeviceToHost, st.stream));
            CUDA_CHECK(cudaStreamSynchronize(st.stream));
            for (int64_t k = 0; k + 1 < n; k++) neighbor_counts[k] = (int32_t)(seg[k + 1] - seg[k]);
        }
    });
}

featomic_status_t featomic_b200_power_spectrum_dense_backward(featomic_b200_dense_t* state, const void* grad_values,
                                                              void* grad_positions, void* grad_strain,
                                                              void* grad_cell, void* stream) {
    return guarded([&] {
        CHECK_POINTER(state);
        DenseState& st = *state->state;
        st.engine->backward_dense(st, grad_values, grad_positions, grad_strain, grad_cell, (cudaStream_t)stream);
    });
}

featomic_status_t featomic_b200_spherical_expansion_dense_backward(featomic_b200_dense_t* state,
                                                                   const void* grad_coefficients, void* grad_positions,
                                                                   void* grad_strain, void* grad_cell, void* stream) {
    return guarded([&] {
        CHECK_POINTER(state);
        DenseState& st = *state->state;
        if (st.n_atoms > 0) CHECK_POINTER(grad_coefficients);
        st.engine->backward_dense(st, grad_coefficients, grad_positions, grad_strain, grad_cell, (cudaStream_t)stream,
                                  /*by_species=*/false, /*coefficients=*/true);
    });
}

featomic_status_t featomic_b200_dense_jvp(featomic_b200_dense_t* state, const void* tangent_positions,
                                          const void* tangent_cell, void* tangent_coefficients, void* tangent_values,
                                          void* stream) {
    return guarded([&] {
        CHECK_POINTER(state);
        DenseState& st = *state->state;
        if (!tangent_coefficients && !tangent_values)
            throw invalid_parameter("one of tangent_coefficients and tangent_values must not be NULL");
        st.engine->jvp_dense(st, tangent_positions, tangent_cell, tangent_coefficients, tangent_values,
                             (cudaStream_t)stream);
    });
}

featomic_status_t featomic_b200_dense_free(featomic_b200_dense_t* state) {
    return guarded([&] { delete state; });
}

featomic_status_t featomic_b200_set_contraction_engine(int32_t tensor_cores, int32_t channels_per_round) {
    return guarded([&] {
        if (tensor_cores != 0 && tensor_cores != 1) throw fb200::invalid_parameter("tensor_cores must be 0 or 1");
        if (channels_per_round < 0 || channels_per_round > 4)
            throw fb200::invalid_parameter("channels_per_round must be between 1 and 4 (0 keeps the current value)");
        fb200::set_dense_mma_enabled(tensor_cores == 1);
        if (channels_per_round > 0) fb200::dense_mma_channels_per_round = channels_per_round;
    });
}

featomic_status_t featomic_b200_labels_tensormap(const mts_labels_t* keys, const mts_labels_t* samples,
                                                 const mts_labels_t* properties, mts_tensormap_t** tensor) {
    return guarded([&] {
        CHECK_POINTER(keys);
        CHECK_POINTER(tensor);
        auto tm = std::make_unique<TensorMap>();
        tm->keys = labels_from_c(keys, "keys");
        const size_t n = tm->keys.count();
        Labels single;
        single.names = {"_"};
        single.values = {0};
        std::vector<Block*> blocks;
        size_t total = 0;
        for (size_t k = 0; k < n; k++) {
            auto b = std::make_unique<Block>();
            b->samples = samples ? labels_from_c(samples + k, "samples") : single;
            b->properties = properties ? labels_from_c(properties + k, "properties") : single;
            b->shape = {b->samples.count(), b->properties.count()};
            total += b->size();
            blocks.push_back(b.get());
            tm->blocks.push_back(std::move(b));
        }
        auto* zeros = static_cast<double*>(std::calloc(std::max<size_t>(1, total), sizeof(double)));
        if (!zeros) throw std::bad_alloc();
        tm->storage = std::shared_ptr<void>(zeros, std::free);
        size_t off = 0;
        for (Block* b : blocks) {
            b->data = zeros + off;
            off += b->size();
        }
        *tensor = wrap(std::move(tm));
    });
}

featomic_status_t featomic_b200_set_expansion_engine(int32_t fused) {
    return guarded([&] {
        if (fused != 0 && fused != 1) throw fb200::invalid_parameter("fused must be 0 or 1");
        fb200::set_se_fused_enabled(fused == 1);
    });
}

struct featomic_b200_batch_t {
    std::unique_ptr<fb200::BatchPlan> plan;
};

featomic_status_t featomic_b200_batch_create(featomic_calculator_t* calculator, uintptr_t n_systems,
                                             const uintptr_t* system_sizes, const int32_t* types,
                                             const int32_t* species, uintptr_t n_species,
                                             featomic_b200_batch_t** batch) {
    return guarded([&] {
        CHECK_POINTER(calculator);
        CHECK_POINTER(batch);
        *batch = nullptr;
        if (!calculator->impl->power_spectrum)
            throw invalid_parameter("featomic_b200_batch_create needs a soap_power_spectrum calculator");
        if (calculator->impl->hypers.explicit_basis())
            throw invalid_parameter("the batched form does not support the Explicit basis");
        if (n_systems > 0) CHECK_POINTER(system_sizes);
        std::vector<int64_t> sizes(n_systems);
        int64_t total = 0;
        for (uintptr_t s = 0; s < n_systems; s++) total += (int64_t)(sizes[s] = (int64_t)system_sizes[s]);
        if (total > 0) CHECK_POINTER(types);
        std::vector<int32_t> t(types, types + total), sp;
        if (n_species > 0) {
            CHECK_POINTER(species);
            sp.assign(species, species + n_species);
        }
        auto result = std::make_unique<featomic_b200_batch_t>();
        result->plan = std::make_unique<BatchPlan>(soap_engine(calculator), sizes, t, sp);
        *batch = result.release();
    });
}

featomic_status_t featomic_b200_batch_shape(const featomic_b200_batch_t* batch, uintptr_t* n_atoms,
                                            uintptr_t* n_systems, uintptr_t* n_species, uintptr_t* n_keys,
                                            uintptr_t* n_properties) {
    return guarded([&] {
        CHECK_POINTER(batch);
        const BatchPlan& p = *batch->plan;
        if (n_atoms) *n_atoms = (uintptr_t)p.n_atoms();
        if (n_systems) *n_systems = (uintptr_t)p.n_systems();
        if (n_species) *n_species = (uintptr_t)p.n_species();
        if (n_keys) *n_keys = (uintptr_t)p.n_keys();
        if (n_properties) *n_properties = (uintptr_t)p.n_props();
    });
}

featomic_status_t featomic_b200_batch_run(featomic_b200_batch_t* batch, const double* positions,
                                          const float* weights, const float* grad_values, float* values,
                                          float* grad_positions, float* energies, float* grad_strain,
                                          void* stream) {
    return guarded([&] {
        CHECK_POINTER(batch);
        batch->plan->run(positions, weights, grad_values, values, grad_positions, energies, grad_strain,
                         (cudaStream_t)stream);
    });
}

featomic_status_t featomic_b200_batch_tune(featomic_b200_batch_t* batch, const double* positions,
                                           const float* weights, const float* grad_values, float* values,
                                           float* grad_positions, float* energies, float* grad_strain,
                                           void* stream, double* best_ms) {
    return guarded([&] {
        CHECK_POINTER(batch);
        const double ms = batch->plan->tune(positions, weights, grad_values, values, grad_positions, energies,
                                            grad_strain, (cudaStream_t)stream);
        if (best_ms) *best_ms = ms;
    });
}

featomic_status_t featomic_b200_batch_config(const featomic_b200_batch_t* batch, int32_t* config) {
    return guarded([&] {
        CHECK_POINTER(batch);
        CHECK_POINTER(config);
        const BatchConfig& c = batch->plan->config;
        config[0] = c.warps;
        config[1] = c.chunk;
        config[2] = c.layout;
        config[3] = c.ctas_per_sm;
        config[4] = c.pipeline;
    });
}

featomic_status_t featomic_b200_batch_set_config(featomic_b200_batch_t* batch, const int32_t* config) {
    return guarded([&] {
        CHECK_POINTER(batch);
        CHECK_POINTER(config);
        if ((config[0] != 4 && config[0] != 8) || (config[1] != 16 && config[1] != 32) ||
            (config[2] != 0 && config[2] != 1) || config[3] < 1 || config[3] > 8 || (config[4] != 0 && config[4] != 1))
            throw invalid_parameter("invalid batch configuration");
        batch->plan->config = BatchConfig{config[0], config[1], config[2], config[3], config[4]};
    });
}

featomic_status_t featomic_b200_batch_status(featomic_b200_batch_t* batch, void* stream, int32_t* status) {
    return guarded([&] {
        CHECK_POINTER(batch);
        CHECK_POINTER(status);
        *status = batch->plan->status((cudaStream_t)stream);
    });
}

featomic_status_t featomic_b200_batch_free(featomic_b200_batch_t* batch) {
    return guarded([&] { delete batch; });
}

struct featomic_b200_surrogate_t {
    std::shared_ptr<fb200::RadialSurrogate> impl;
};

featomic_status_t featomic_b200_surrogate_create(featomic_calculator_t* calculator, int32_t hidden, uint64_t seed,
                                                 featomic_b200_surrogate_t** surrogate) {
    return guarded([&] {
        CHECK_POINTER(calculator);
        CHECK_POINTER(surrogate);
        *surrogate = nullptr;
        auto result = std::make_unique<featomic_b200_surrogate_t>();
        if (calculator->impl->hypers.explicit_basis() || calculator->impl->hypers.tabulated_basis())
            throw invalid_parameter("the learned radial surrogate needs a GTO TensorProduct basis");
        result->impl = std::make_shared<RadialSurrogate>(soap_engine(calculator), hidden, seed);
        *surrogate = result.release();
    });
}

featomic_status_t featomic_b200_surrogate_shape(const featomic_b200_surrogate_t* surrogate, uintptr_t* n_outputs,
                                                uintptr_t* n_parameters, uintptr_t* n_samples) {
    return guarded([&] {
        CHECK_POINTER(surrogate);
        if (n_outputs) *n_outputs = (uintptr_t)surrogate->impl->n_outputs();
        if (n_parameters) *n_parameters = (uintptr_t)surrogate->impl->n_params();
        if (n_samples) *n_samples = (uintptr_t)surrogate->impl->n_samples();
    });
}

featomic_status_t featomic_b200_surrogate_dataset(featomic_b200_surrogate_t* surrogate, uintptr_t n_samples,
                                                  uint64_t seed, void* stream) {
    return guarded([&] {
        CHECK_POINTER(surrogate);
        surrogate->impl->make_dataset((int64_t)n_samples, seed, (cudaStream_t)stream);
    });
}

featomic_status_t featomic_b200_surrogate_train(featomic_b200_surrogate_t* surrogate, uintptr_t steps,
                                                uintptr_t batch, double learning_rate, double* loss, void* stream) {
    return guarded([&] {
        CHECK_POINTER(surrogate);
        if (!(learning_rate > 0.0 && std::isfinite(learning_rate)))
            throw invalid_parameter("the learning rate must be positive");
        const double l = surrogate->impl->train((int64_t)steps, (int64_t)batch, learning_rate, (cudaStream_t)stream);
        if (loss) *loss = l;
    });
}

featomic_status_t featomic_b200_surrogate_set_derivative_weight(featomic_b200_surrogate_t* surrogate,
                                                                double derivative_weight) {
    return guarded([&] {
        CHECK_POINTER(surrogate);
        surrogate->impl->set_derivative_weight(derivative_weight);
    });
}

featomic_status_t featomic_b200_surrogate_fit_output_layer(featomic_b200_surrogate_t* surrogate,
                                                           double derivative_weight, void* stream) {
    return guarded([&] {
        CHECK_POINTER(surrogate);
        surrogate->impl->fit_output_layer(derivative_weight, (cudaStream_t)stream);
    });
}

featomic_status_t featomic_b200_surrogate_gradient(featomic_b200_surrogate_t* surrogate, uintptr_t n,
                                                   float* gradient, double* loss, void* stream) {
    return guarded([&] {
        CHECK_POINTER(surrogate);
        CHECK_POINTER(gradient);
        std::vector<float> g;
        const double l = surrogate->impl->loss_and_gradient((int64_t)n, g, (cudaStream_t)stream);
        std::copy(g.begin(), g.end(), gradient);
        if (loss) *loss = l;
    });
}

featomic_status_t featomic_b200_surrogate_parameters(featomic_b200_surrogate_t* surrogate, float* parameters,
                                                     uintptr_t count, int32_t set, void* stream) {
    return guarded([&] {
        CHECK_POINTER(surrogate);
        CHECK_POINTER(parameters);
        if ((int64_t)count != surrogate->impl->n_params())
            throw invalid_parameter("expected " + std::to_string(surrogate->impl->n_params()) + " parameters");
        if (set) {
            surrogate->impl->set_parameters(std::vector<float>(parameters, parameters + count), (cudaStream_t)stream);
        } else {
            const std::vector<float> p = surrogate->impl->parameters((cudaStream_t)stream);
            std::copy(p.begin(), p.end(), parameters);
        }
    });
}

featomic_status_t featomic_b200_surrogate_scales(const featomic_b200_surrogate_t* surrogate, float* scales,
                                                 uintptr_t count) {
    return guarded([&] {
        CHECK_POINTER(surrogate);
        CHECK_POINTER(scales);
        const std::vector<float> s = surrogate->impl->scales();
        if (count != s.size()) throw invalid_parameter("expected " + std::to_string(s.size()) + " scales");
        std::copy(s.begin(), s.end(), scales);
    });
}

featomic_status_t featomic_b200_surrogate_samples(const featomic_b200_surrogate_t* surrogate, float* r,
                                                  uintptr_t count, void* stream) {
    return guarded([&] {
        CHECK_POINTER(surrogate);
        CHECK_POINTER(r);
        const std::vector<float> s = surrogate->impl->dataset_r((cudaStream_t)stream);
        if (count != s.size()) throw invalid_parameter("expected " + std::to_string(s.size()) + " samples");
        std::copy(s.begin(), s.end(), r);
    });
}

featomic_status_t featomic_b200_surrogate_evaluate(featomic_b200_surrogate_t* surrogate, const double* r,
                                                   uintptr_t n, float* values, float* derivs, uintptr_t ld,
                                                   int32_t method, void* stream) {
    return guarded([&] {
        CHECK_POINTER(surrogate);
        if (n == 0) return;
        CHECK_POINTER(r);
        CHECK_POINTER(values);
        cudaStream_t s = (cudaStream_t)stream;
        switch (method) {
            case 0: surrogate->impl->evaluate(r, (int64_t)n, values, derivs, (int64_t)ld, true, s); break;
            case 1: surrogate->impl->evaluate(r, (int64_t)n, values, derivs, (int64_t)ld, false, s); break;
            case 2: surrogate->impl->evaluate_reference(r, (int64_t)n, values, derivs, (int64_t)ld, false, s); break;
            case 3: surrogate->impl->evaluate_reference(r, (int64_t)n, values, derivs, (int64_t)ld, true, s); break;
            case 4: surrogate->impl->evaluate(r, (int64_t)n, values, derivs, (int64_t)ld, false, s, true, true); break;
            default: throw invalid_parameter("method must be 0, 1, 2, 3 or 4");
        }
    });
}

featomic_status_t featomic_b200_calculator_set_surrogate(featomic_calculator_t* calculator,
                                                         featomic_b200_surrogate_t* surrogate) {
    return guarded([&] {
        CHECK_POINTER(calculator);
        if (surrogate && surrogate->impl->engine() != &soap_engine(calculator))
            throw invalid_parameter("the surrogate was trained for another calculator");
        soap_engine(calculator).set_surrogate(surrogate ? surrogate->impl : nullptr);
    });
}

featomic_status_t featomic_b200_surrogate_free(featomic_b200_surrogate_t* surrogate) {
    return guarded([&] { delete surrogate; });
}

featomic_status_t featomic_b200_neighbor_list(const double* positions, uintptr_t n_atoms, const double* cell,
                                              double cutoff, featomic_pair_t* pairs, uintptr_t capacity,
                                              uintptr_t* count) {
    return guarded([&] {
        CHECK_POINTER(cell);
        CHECK_POINTER(count);
        if (n_atoms > 0) CHECK_POINTER(positions);
        if (!(cutoff > 0.0 && std::isfinite(cutoff))) throw invalid_parameter("cutoff must be positive and finite");
        std::vector<Pair> out = neighbor_list(positions, (int64_t)n_atoms, cell, cutoff);
        *count = out.size();
        if (capacity < out.size()) {
            throw Error(FEATOMIC_BUFFER_SIZE_ERROR, "pair buffer is too small: got space for " + std::to_string(capacity) +
                                                        " pairs, need " + std::to_string(out.size()));
        }
        if (!out.empty()) CHECK_POINTER(pairs);
        for (size_t k = 0; k < out.size(); k++) {
            pairs[k].first = out[k].first;
            pairs[k].second = out[k].second;
            pairs[k].distance = out[k].distance;
            for (int x = 0; x < 3; x++) {
                pairs[k].vector[x] = out[k].vector[x];
                pairs[k].cell_shift_indices[x] = out[k].shift[x];
            }
        }
    });
}

featomic_status_t featomic_b200_neighbor_list_noalloc(const double* positions, uintptr_t n_atoms, const double* cell,
                                                      double cutoff, featomic_pair_t* pairs, uintptr_t capacity,
                                                      uintptr_t* count, void* stream) {
    return guarded([&] {
        CHECK_POINTER(cell);
        CHECK_POINTER(count);
        if (n_atoms > 0) CHECK_POINTER(positions);
        if (!(cutoff > 0.0 && std::isfinite(cutoff))) throw invalid_parameter("cutoff must be positive and finite");
        const int64_t cap = capacity > (uintptr_t)INT64_MAX ? INT64_MAX : (int64_t)capacity;
        neighbor_list_noalloc(positions, (int64_t)std::min<uintptr_t>(n_atoms, (uintptr_t)INT64_MAX), cell, cutoff,
                              pairs, cap, count, stream);
    });
}

featomic_status_t featomic_b200_radial_integral(const featomic_calculator_t* calculator, const double* r,
                                                uintptr_t n_r, double* values, double* gradients, int32_t* knots) {
    return guarded([&] {
        CHECK_POINTER(calculator);
        const RadialTables& t = soap_engine(calculator).radial();
        if (n_r > 0) {
            CHECK_POINTER(r);
            CHECK_POINTER(values);
        }
        size_t per = (size_t)(t.lmax + 1) * t.nmax;
        for (uintptr_t k = 0; k < n_r; k++) {
            if (!(r[k] >= 0.0 && r[k] <= calculator->impl->hypers.cutoff))
                throw invalid_parameter("distances must be in [0, cutoff]");
            for (int l = 0; l <= t.lmax; l++)
                radial_integral_host(t, l, r[k], values + k * per + (size_t)l * t.nmax,
                                     gradients ? gradients + k * per + (size_t)l * t.nmax : nullptr);
        }
        if (knots)
            for (int l = 0; l <= t.lmax; l++) knots[l] = t.splined ? t.knot_count[l] : 0;
    });
}

featomic_status_t featomic_b200_dense_timings(const featomic_calculator_t* calculator, double* times,
                                             uintptr_t count) {
    return guarded([&] {
        CHECK_POINTER(calculator);
        CHECK_POINTER(times);
        const std::vector<double> t = soap_engine(calculator).dense_times();
        for (uintptr_t k = 0; k < count && k < t.size(); k++) times[k] = t[k];
    });
}

featomic_status_t featomic_b200_calculator_timings(const featomic_calculator_t* calculator, double* times,
                                                   uintptr_t count) {
    return guarded([&] {
        CHECK_POINTER(calculator);
        CHECK_POINTER(times);
        const PhaseTimes& t = last_times(*calculator->impl);
        double all[12] = {t.neighbors,    t.metadata,       t.features,
                          t.expansion,    t.contraction,    t.transfer,
                          t.total,        t.ps_values,      t.ps_positions,
                          t.ps_strain_cell, t.metadata_before_launch, t.labels};
        for (uintptr_t k = 0; k < count && k < 12; k++) times[k] = all[k];
    });
}

featomic_status_t featomic_profiling_clear(void) {
    return guarded([&] {
        std::lock_guard<std::mutex> lock(profile().mutex);
        profile().spans.clear();
    });
}

featomic_status_t featomic_profiling_enable(bool enabled) {
    return guarded([&] {
        std::lock_guard<std::mutex> lock(profile().mutex);
        profile().enabled = enabled;
    });
}

featomic_status_t featomic_profiling_get(const char* format, char* buffer, uintptr_t bufflen) {
    return guarded([&] {
        CHECK_POINTER(format);
        std::string f = format;
        std::ostringstream out;
        std::lock_guard<std::mutex> lock(profile().mutex);
        if (f == "json") {
            out << "{";
            bool first = true;
            for (auto& kv : profile().spans) {
                out << (first ? "" : ",") << "\"" << kv.first << "\":{\"total_ms\":" << kv.second.first
                    << ",\"calls\":" << kv.second.second << "}";
                first = false;
            }
            out << "}";
        } else if (f == "table" || f == "short_table") {
            out << "| span | calls | total (ms) | mean (ms) |\n|---|---|---|---|\n";
            for (auto& kv : profile().spans)
                out << "| " << kv.first << " | " << kv.second.second << " | " << kv.second.first << " | "
                    << kv.second.first / (double)std::max<int64_t>(1, kv.second.second) << " |\n";
        } else {
            throw invalid_parameter("invalid data format in featomic_profiling_get: " + f +
                                    ", expected 'table', 'short_table' or 'json'");
        }
        copy_str(out.str(), buffer, bufflen);
    });
}

// ---- minimal metatensor accessors -------------------------------------------

mts_status_t mts_tensormap_free(mts_tensormap_t* tensor) {
    return guarded([&] { delete tensor; });
}

mts_status_t mts_tensormap_keys(const mts_tensormap_t* tensor, mts_labels_t* keys) {
    return guarded([&] {
        CHECK_POINTER(tensor);
        CHECK_POINTER(keys);
        keys->internal_ptr_ = nullptr;
        keys->names = tensor->key_names.data();
        keys->values = tensor->tm->keys.values.data();
        keys->size = tensor->tm->keys.names.size();
        keys->count = tensor->tm->keys.count();
    });
}

mts_status_t mts_tensormap_block_by_id(mts_tensormap_t* tensor, mts_block_t** block, uintptr_t index) {
    return guarded([&] {
        CHECK_POINTER(tensor);
        CHECK_POINTER(block);
        if (index >= tensor->handles.size())
            throw invalid_parameter("block index out of bounds: we have " + std::to_string(tensor->handles.size()) +
                                    " blocks but the index is " + std::to_string(index));
        *block = tensor->handles[index].get();
    });
}

mts_status_t mts_block_labels(const mts_block_t* block, uintptr_t axis, mts_labels_t* labels) {
    return guarded([&] {
        CHECK_POINTER(block);
        CHECK_POINTER(labels);
        auto* b = const_cast<mts_block_t*>(block);
        const Block& blk = *b->block;
        size_t n_axes = blk.components.size() + 2;
        if (axis >= n_axes) throw invalid_parameter("axis out of bounds for this block");
        const Labels* l;
        if (axis == 0) l = &blk.samples;
        else if (axis == n_axes - 1) l = &blk.properties;
        else l = &blk.components[axis - 1];
        b->name_ptrs.emplace_back();
        fill_labels(*l, b->name_ptrs.back(), labels);
    });
}

mts_status_t mts_block_gradient(mts_block_t* block, const char* parameter, mts_block_t** gradient) {
    return guarded([&] {
        CHECK_POINTER(block);
        CHECK_POINTER(parameter);
        CHECK_POINTER(gradient);
        for (size_t k = 0; k < block->gradient_names.size(); k++) {
            if (std::strcmp(block->gradient_names[k], parameter) == 0) {
                *gradient = block->gradient_handles[k].get();
                return;
            }
        }
        throw invalid_parameter(std::string("can not find gradients with respect to '") + parameter + "' in this block");
    });
}

mts_status_t mts_block_gradients_list(const mts_block_t* block, const char* const** parameters, uintptr_t* count) {
    return guarded([&] {
        CHECK_POINTER(block);
        CHECK_POINTER(parameters);
        CHECK_POINTER(count);
        *parameters = block->gradient_names.data();
        *count = block->gradient_names.size();
    });
}

mts_status_t mts_labels_free(mts_labels_t* labels) {
    return guarded([&] {
        if (labels) {
            labels->names = nullptr;
            labels->values = nullptr;
            labels->count = 0;
            labels->size = 0;
        }
    });
}

featomic_status_t featomic_b200_block_values(const mts_block_t* block, double** data, const uintptr_t** shape,
                                             uintptr_t* shape_count, int32_t* on_device) {
    return guarded([&] {
        CHECK_POINTER(block);
        CHECK_POINTER(data);
        CHECK_POINTER(shape);
        CHECK_POINTER(shape_count);
        auto* b = const_cast<mts_block_t*>(block);
        b->shape.assign(b->block->shape.begin(), b->block->shape.end());
        *data = b->block->data;
        *shape = b->shape.data();
        *shape_count = b->shape.size();
        if (on_device) *on_device = b->on_device ? 1 : 0;
    });
}

featomic_status_t featomic_b200_cg_coefficients(int32_t l1, int32_t l2, int32_t lambda, double* coefficients,
                                                uintptr_t count) {
    return guarded([&] {
        CHECK_POINTER(coefficients);
        const auto cg = fb200::real_cg_coefficients(l1, l2, lambda);
        if (count != cg.size())
            throw invalid_parameter("expected " + std::to_string(cg.size()) + " coefficients, got space for " +
                                    std::to_string(count));
        std::memcpy(coefficients, cg.data(), cg.size() * sizeof(double));
    });
}

featomic_status_t featomic_b200_cg_product(const featomic_b200_cg_task_t* tasks, uintptr_t n_tasks,
                                           int32_t precision, void* stream) {
    return guarded([&] {
        if (n_tasks == 0) return;
        CHECK_POINTER(tasks);
        fb200::cg_product(tasks, (size_t)n_tasks, precision, static_cast<cudaStream_t>(stream));
    });
}

featomic_status_t featomic_b200_cg_couple(const featomic_b200_cg_couple_task_t* tasks, uintptr_t n_tasks,
                                          int32_t precision, void* stream) {
    return guarded([&] {
        if (n_tasks == 0) return;
        CHECK_POINTER(tasks);
        fb200::cg_couple(tasks, (size_t)n_tasks, precision, static_cast<cudaStream_t>(stream));
    });
}

}  // extern "C"

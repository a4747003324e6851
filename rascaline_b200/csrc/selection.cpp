// Samples / properties / keys selections of a compute call
// (featomic/src/calculator.rs:20-158 LabelsSelection::select, :287-310 keys),
// applied to the output of the full calculation, on the host or, for device
// output, by a gather kernel on the device.
//
// featomic computes only the selected entries; their values do not depend on
// what else is computed, so selecting rows and columns of the full output
// gives the same numbers.  Semantics kept:
//   keys       same names as the calculator's keys: exactly these keys, in
//              this order (a key the systems do not produce gets an empty
//              block); fewer names: the default keys matching any row
//   Subset     per block, the default entries matching any row of the
//              selection on the selection's names, in default order
//   Predefined per block, the labels of the predefined TensorMap's block
//              with the same key, in that order.  A predefined sample the
//              full calculation does not have (a centre of the key's
//              center_type without neighbours of one of the key's neighbour
//              types) is a zero row, as featomic computes it, with zero
//              gradient rows for the atoms featomic lists
//              (atom_centered.rs:103-147); predefined properties must be
//              properties of the calculator
// Gradient rows follow their samples (positions rows keep their order within
// a sample, their "sample" column is renumbered); properties are selected on
// the last axis of every array.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cstdlib>
#include <cstring>
#include <map>

#include "host.hpp"

namespace fb200 {

namespace {

std::string join(const std::vector<std::string>& names) {
    std::string out;
    for (auto& n : names) out += (out.empty() ? "" : ", ") + n;
    return out;
}

// columns of `selection` inside `labels` (error when a name is unknown)
std::vector<size_t> columns_of(const Labels& labels, const Labels& selection, const char* kind) {
    std::vector<size_t> cols;
    for (auto& name : selection.names) {
        size_t c = 0;
        while (c < labels.names.size() && labels.names[c] != name) c++;
        if (c == labels.names.size())
            throw invalid_parameter("'" + name + "' in " + kind + " selection is not part of the " + kind +
                                    " of this calculator");
        cols.push_back(c);
    }
    return cols;
}

// indices of the entries of `labels` matching any row of `selection`
std::vector<int64_t> select_subset(const Labels& labels, const Labels& selection, const char* kind) {
    const std::vector<size_t> cols = columns_of(labels, selection, kind);
    const size_t w = labels.names.size(), sw = selection.names.size();
    std::map<std::vector<int32_t>, bool> wanted;
    for (size_t r = 0; r < selection.count(); r++)
        wanted[std::vector<int32_t>(selection.values.begin() + r * sw, selection.values.begin() + (r + 1) * sw)] = true;
    std::vector<int64_t> out;
    std::vector<int32_t> key(sw);
    for (size_t r = 0; r < labels.count(); r++) {
        for (size_t k = 0; k < sw; k++) key[k] = labels.values[r * w + cols[k]];
        if (wanted.count(key)) out.push_back((int64_t)r);
    }
    return out;
}

// indices of the predefined entries inside `labels` (same names required);
// an entry the full calculation does not have is -1 when `allow_absent`
std::vector<int64_t> select_predefined(const Labels& labels, const Labels& predefined, const char* kind,
                                       bool allow_absent) {
    if (predefined.names != labels.names)
        throw invalid_parameter(std::string("invalid predefined ") + kind + " names: expected [" + join(labels.names) +
                                "], but got [" + join(predefined.names) + "]");
    const size_t w = labels.names.size();
    std::map<std::vector<int32_t>, int64_t> index;
    for (size_t r = 0; r < labels.count(); r++)
        index[std::vector<int32_t>(labels.values.begin() + r * w, labels.values.begin() + (r + 1) * w)] = (int64_t)r;
    std::vector<int64_t> out;
    for (size_t r = 0; r < predefined.count(); r++) {
        auto it = index.find(std::vector<int32_t>(predefined.values.begin() + r * w,
                                                  predefined.values.begin() + (r + 1) * w));
        if (it == index.end() && !allow_absent)
            throw invalid_parameter(std::string("predefined ") + kind +
                                    " selection contains an entry outside of this calculator's " + kind);
        out.push_back(it == index.end() ? -1 : it->second);
    }
    return out;
}

// value of the key column `name` of key k, or INT32_MIN without that column
int32_t key_value(const Labels& keys, size_t k, const std::string& name) {
    const size_t w = keys.names.size();
    for (size_t c = 0; c < w; c++)
        if (keys.names[c] == name) return keys.values[k * w + c];
    return INT32_MIN;
}

// A predefined sample (system, atom) of key k that the full calculation did
// not produce: a centre of the key's center_type lacking neighbours of one
// of the key's neighbour types, whose values and gradients are all zero
// (its coefficients for that neighbour type vanish).  Returns its positions
// gradient samples: featomic's AtomCenteredSamples::gradients_for
// (labels/samples/atom_centered.rs:103-147) with self pairs, the atoms of
// the key's neighbour types within the cutoff plus the centre itself when
// one matched or its own type is one of them, by atom index.
std::vector<int32_t> absent_sample(const Selection& sel, const Labels& keys, size_t k, int32_t system, int32_t atom,
                                   bool positions) {
    const int32_t center_type = key_value(keys, k, "center_type");
    std::vector<int32_t> wanted;
    for (const char* name : {"neighbor_type", "neighbor_1_type", "neighbor_2_type"}) {
        const int32_t t = key_value(keys, k, name);
        if (t != INT32_MIN) wanted.push_back(t);
    }
    if (center_type == INT32_MIN || wanted.empty() || !sel.systems)
        throw invalid_parameter("predefined samples selection contains a sample this calculator does not produce");
    if (system < 0 || (size_t)system >= sel.systems->size() || atom < 0 ||
        atom >= (int32_t)(*sel.systems)[system].n_atoms)
        throw invalid_parameter("predefined samples selection contains (system=" + std::to_string(system) +
                                ", atom=" + std::to_string(atom) + "), which is not an atom of the systems");
    const std::vector<int32_t>& types = (*sel.systems)[system].types;
    if (types[atom] != center_type)
        throw invalid_parameter("predefined samples selection contains (system=" + std::to_string(system) +
                                ", atom=" + std::to_string(atom) + ") of atomic type " + std::to_string(types[atom]) +
                                " in a block with center_type=" + std::to_string(center_type) +
                                "; featomic-b200 computes the atoms of the block's center_type only");
    std::vector<int32_t> atoms;
    if (!positions) return atoms;
    auto matches = [&](int32_t t) { return std::find(wanted.begin(), wanted.end(), t) != wanted.end(); };
    bool with_centre = matches(types[atom]);
    for (int32_t j : sel.neighbors(system, atom)) {
        if (!matches(types[j])) continue;
        atoms.push_back(j);
        with_centre = true;
    }
    if (with_centre) atoms.push_back(atom);
    std::sort(atoms.begin(), atoms.end());
    atoms.erase(std::unique(atoms.begin(), atoms.end()), atoms.end());
    return atoms;
}

Labels rows_of(const Labels& labels, const std::vector<int64_t>& rows) {
    Labels out;
    out.names = labels.names;
    const size_t w = labels.names.size();
    for (int64_t r : rows) out.values.insert(out.values.end(), labels.values.begin() + r * w, labels.values.begin() + (r + 1) * w);
    return out;
}

const Block* predefined_block(const TensorMap& tm, const Labels& keys, size_t k, const char* kind) {
    if (tm.keys.names != keys.names)
        throw invalid_parameter(std::string("invalid key names in predefined ") + kind + ": expected [" +
                                join(keys.names) + "], but got [" + join(tm.keys.names) + "]");
    const size_t w = keys.names.size();
    for (size_t r = 0; r < tm.keys.count(); r++)
        if (std::equal(keys.values.begin() + k * w, keys.values.begin() + (k + 1) * w, tm.keys.values.begin() + r * w))
            return tm.blocks[r].get();
    std::string print;
    for (size_t c = 0; c < w; c++)
        print += (c ? ", " : "") + keys.names[c] + "=" + std::to_string(keys.values[k * w + c]);
    throw invalid_parameter("expected a block for (" + print + ") in predefined " + kind + " selection");
}

// one array of the output: rows of `src` (-1: a zero row), every middle
// axis, the block's selected properties
struct Gather {
    const double* src;  // null: all rows zero
    std::vector<int64_t> rows;
    int64_t inner, src_props;
    const std::vector<int64_t>* props;
    double* dst;
};

void gather_host(const Gather& g) {
    const std::vector<int64_t>& props = *g.props;
    size_t o = 0;
    for (int64_t r : g.rows)
        for (int64_t m = 0; m < g.inner; m++) {
            if (r < 0 || !g.src) {
                for (size_t p = 0; p < props.size(); p++) g.dst[o++] = 0.0;
                continue;
            }
            const double* s = g.src + ((size_t)r * g.inner + m) * g.src_props;
            for (int64_t p : props) g.dst[o++] = s[p];
        }
}

void check_cuda(cudaError_t status) {
    if (status != cudaSuccess) {
        cudaGetLastError();
        throw internal_error(std::string("CUDA error in a device selection: ") + cudaGetErrorString(status));
    }
}

void gather_device(const std::vector<Gather>& gathers) {
    // every index array in one upload
    std::vector<int64_t> index;
    std::vector<size_t> at;
    std::map<const std::vector<int64_t>*, size_t> props_at;
    for (auto& g : gathers) {
        at.push_back(index.size());
        for (int64_t r : g.rows) index.push_back(g.src ? r : -1);
        if (!props_at.count(g.props)) {
            props_at[g.props] = index.size();
            index.insert(index.end(), g.props->begin(), g.props->end());
        }
    }
    int64_t* d_index = nullptr;
    check_cuda(cudaMalloc(&d_index, sizeof(int64_t) * std::max<size_t>(1, index.size())));
    std::shared_ptr<void> keep(d_index, [](void* q) { cudaFree(q); });
    if (!index.empty())
        check_cuda(cudaMemcpy(d_index, index.data(), sizeof(int64_t) * index.size(), cudaMemcpyHostToDevice));
    for (size_t k = 0; k < gathers.size(); k++) {
        const Gather& g = gathers[k];
        if (g.rows.empty() || g.props->empty()) continue;
        launch_gather_rows(g.src, d_index + at[k], (int64_t)g.rows.size(), g.inner, g.src_props,
                           d_index + props_at[g.props], (int64_t)g.props->size(), g.dst);
        check_cuda(cudaGetLastError());
    }
    // the source TensorMap and the index arrays are released after return
    check_cuda(cudaDeviceSynchronize());
}

}  // namespace

std::unique_ptr<TensorMap> apply_selection(std::unique_ptr<TensorMap> full, const Selection& sel) {
    if (!sel.any()) return full;
    const TensorMap& tm = *full;

    // keys
    Labels keys = tm.keys;
    std::vector<int64_t> source;  // block of `tm` for every output key, -1 when absent
    if (sel.keys) {
        const Labels& ks = *sel.keys;
        if (ks.count() == 0) throw invalid_parameter("selected keys can not be empty");
        if (ks.names == tm.keys.names) {
            keys = ks;
        } else {
            keys = rows_of(tm.keys, select_subset(tm.keys, ks, "keys"));
        }
    }
    const size_t kw = keys.names.size();
    for (size_t k = 0; k < keys.count(); k++) {
        int64_t found = -1;
        for (size_t r = 0; r < tm.keys.count() && found < 0; r++)
            if (std::equal(keys.values.begin() + k * kw, keys.values.begin() + (k + 1) * kw,
                           tm.keys.values.begin() + r * kw))
                found = (int64_t)r;
        source.push_back(found);
    }
    if (tm.blocks.empty()) throw invalid_parameter("selections need at least one computed block");
    const Block& any = *tm.blocks[0];
    bool any_positions = false;
    for (auto& g : any.gradients) any_positions |= g.first == "positions";

    // per output block: selected sample rows (-1: a predefined sample the
    // full calculation does not have) and property columns
    struct Plan {
        const Block* src;
        std::vector<int64_t> rows, props;
        std::vector<Labels> components;
        Labels samples, properties;
        std::map<size_t, std::vector<int32_t>> absent_atoms;  // output row -> positions gradient atoms
    };
    std::vector<Plan> plans(keys.count());
    size_t total = 0;
    for (size_t k = 0; k < keys.count(); k++) {
        Plan& p = plans[k];
        p.src = source[k] >= 0 ? tm.blocks[source[k]].get() : nullptr;
        if (p.src) {
            p.components = p.src->components;
            p.samples = p.src->samples;
            p.properties = p.src->properties;
        } else {
            // a key the systems do not produce: no samples; components from
            // the key's o3_lambda when the calculator has them
            p.samples.names = any.samples.names;
            p.properties = any.properties;
            if (!any.components.empty()) {
                size_t lc = 0;
                while (lc < kw && keys.names[lc] != "o3_lambda") lc++;
                if (lc == kw) throw internal_error("selection: no o3_lambda key for the components");
                const int l = keys.values[k * kw + lc];
                if (l < 0 || l > sel.max_angular)
                    throw invalid_parameter("selected key with o3_lambda = " + std::to_string(l) +
                                            " is outside of this calculator's max_angular");
                Labels mu;
                mu.names = {"o3_mu"};
                for (int m = -l; m <= l; m++) mu.values.push_back(m);
                p.components = {mu};
            }
        }
        for (size_t r = 0; r < p.samples.count(); r++) p.rows.push_back((int64_t)r);
        for (size_t c = 0; c < p.properties.count(); c++) p.props.push_back((int64_t)c);
        if (sel.samples) {
            p.rows = select_subset(p.samples, *sel.samples, "samples");
            p.samples = rows_of(p.samples, p.rows);
        }
        if (sel.samples_predefined) {
            const Labels& wanted = predefined_block(*sel.samples_predefined, keys, k, "samples")->samples;
            p.rows = select_predefined(p.samples, wanted, "samples", true);
            p.samples = wanted;
            const size_t sw = wanted.names.size();
            for (size_t r = 0; r < p.rows.size(); r++) {
                if (p.rows[r] >= 0) continue;
                if (sw != 2 || wanted.names[0] != "system" || wanted.names[1] != "atom")
                    throw invalid_parameter("predefined samples selection contains a sample this calculator does not "
                                            "produce");
                p.absent_atoms[r] = absent_sample(sel, keys, k, wanted.values[r * sw], wanted.values[r * sw + 1],
                                                  any_positions);
            }
        }
        if (sel.properties) p.props = select_subset(p.properties, *sel.properties, "properties");
        if (sel.properties_predefined)
            p.props = select_predefined(
                p.properties, predefined_block(*sel.properties_predefined, keys, k, "properties")->properties,
                "properties", false);
        p.properties = rows_of(p.properties, p.props);
        size_t comp = 1;
        for (auto& c : p.components) comp *= c.count();
        total += p.rows.size() * comp * p.props.size();
        for (auto& named : any.gradients) {
            size_t inner = 1;
            const Block& g = *named.second;
            for (size_t a = 1; a + 1 < g.shape.size(); a++) inner *= g.shape[a];
            inner = inner / std::max<size_t>(1, [&] {
                size_t c = 1;
                for (auto& l : any.components) c *= l.count();
                return c;
            }()) * comp;
            size_t rows = 0;
            if (named.first == "positions") {
                if (p.src)
                    for (auto& sg : p.src->gradients)
                        if (sg.first == "positions") rows += sg.second->shape[0];  // upper bound
                for (auto& a : p.absent_atoms) rows += a.second.size();
            } else {
                rows = p.rows.size();
            }
            total += rows * inner * p.props.size();
        }
    }

    auto out = std::make_unique<TensorMap>();
    out->keys = keys;
    out->on_device = tm.on_device;
    out->device = tm.device;
    double* buffer = nullptr;
    const size_t bytes = std::max<size_t>(8, sizeof(double) * total);
    if (tm.on_device) {
        check_cuda(cudaMalloc(&buffer, bytes));
        out->storage = std::shared_ptr<void>(buffer, [](void* q) { cudaFree(q); });
    } else {
        buffer = static_cast<double*>(std::malloc(bytes));
        if (!buffer) throw std::bad_alloc();
        out->storage = std::shared_ptr<void>(buffer, std::free);
    }
    std::vector<Gather> gathers;
    size_t off = 0;
    for (size_t k = 0; k < keys.count(); k++) {
        Plan& p = plans[k];
        auto blk = std::make_unique<Block>();
        blk->samples = p.samples;
        blk->components = p.components;
        blk->properties = p.properties;
        blk->shape = {p.rows.size()};
        for (auto& c : p.components) blk->shape.push_back(c.count());
        blk->shape.push_back(p.props.size());
        blk->data = buffer + off;
        {
            size_t comp = 1;
            for (auto& c : p.components) comp *= c.count();
            gathers.push_back(Gather{p.src ? p.src->data : nullptr, p.rows, (int64_t)comp,
                                     p.src ? (int64_t)p.src->shape.back() : 0, &p.props, blk->data});
        }
        off += blk->size();
        // gradients present in the full output (all blocks carry the same set)
        for (auto& named : any.gradients) {
            const std::string& name = named.first;
            const Block* gsrc = nullptr;
            if (p.src)
                for (auto& g : p.src->gradients)
                    if (g.first == name) gsrc = g.second.get();
            auto gb = std::make_unique<Block>();
            gb->components = gsrc ? gsrc->components : named.second->components;
            if (!gsrc) {
                // the template block's components end with its own o3_mu:
                // swap in this key's
                gb->components.resize(gb->components.size() - any.components.size());
                gb->components.insert(gb->components.end(), p.components.begin(), p.components.end());
            }
            gb->properties = p.properties;
            gb->samples.names = named.second->samples.names;
            std::vector<int64_t> grows;
            if (name == "positions") {
                // rows of each kept sample, in their order, renumbered; zero
                // rows for the samples the full calculation does not have
                std::vector<std::vector<int64_t>> by_sample(gsrc ? p.src->samples.count() : 0);
                const size_t gw = named.second->samples.names.size();
                if (gsrc)
                    for (size_t r = 0; r < gsrc->samples.count(); r++)
                        by_sample[gsrc->samples.values[r * gw]].push_back((int64_t)r);
                for (size_t s = 0; s < p.rows.size(); s++) {
                    if (p.rows[s] < 0) {
                        const int32_t system = p.samples.values[2 * s];
                        for (int32_t a : p.absent_atoms[s]) {
                            grows.push_back(-1);
                            gb->samples.values.insert(gb->samples.values.end(), {(int32_t)s, system, a});
                        }
                        continue;
                    }
                    for (int64_t r : by_sample[p.rows[s]]) {
                        grows.push_back(r);
                        gb->samples.values.push_back((int32_t)s);
                        gb->samples.values.insert(gb->samples.values.end(), gsrc->samples.values.begin() + r * gw + 1,
                                                  gsrc->samples.values.begin() + (r + 1) * gw);
                    }
                }
            } else {
                // strain / cell: one row per sample
                for (size_t s = 0; s < p.rows.size(); s++) {
                    grows.push_back(gsrc ? p.rows[s] : -1);
                    gb->samples.values.push_back((int32_t)s);
                }
            }
            gb->shape = {grows.size()};
            for (auto& c : gb->components) gb->shape.push_back(c.count());
            gb->shape.push_back(p.props.size());
            gb->data = buffer + off;
            size_t inner = 1;
            for (size_t a = 1; a + 1 < gb->shape.size(); a++) inner *= gb->shape[a];
            gathers.push_back(Gather{gsrc ? gsrc->data : nullptr, grows, (int64_t)inner,
                                     gsrc ? (int64_t)gsrc->shape.back() : 0, &p.props, gb->data});
            off += gb->size();
            blk->gradients.emplace_back(name, std::move(gb));
        }
        out->blocks.push_back(std::move(blk));
    }
    if (off > std::max<size_t>(total, 1)) throw internal_error("selection: output buffer overflow");
    if (tm.on_device) {
        gather_device(gathers);
    } else {
        for (auto& g : gathers) gather_host(g);
    }
    return out;
}

}  // namespace fb200

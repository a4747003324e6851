// Samples / properties / keys selections of a compute call
// (featomic/src/calculator.rs:20-158 LabelsSelection::select, :287-310 keys),
// applied to the host TensorMap of the full calculation.
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
//              with the same key, in that order
// Gradient rows follow their samples (positions rows keep their order within
// a sample, their "sample" column is renumbered); properties are selected on
// the last axis of every array.
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

// indices of the predefined entries inside `labels` (same names required)
std::vector<int64_t> select_predefined(const Labels& labels, const Labels& predefined, const char* kind) {
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
        if (it == index.end())
            throw invalid_parameter(std::string("predefined ") + kind +
                                    " selection contains an entry that the systems do not produce; featomic-b200 only "
                                    "selects among the computed entries");
        out.push_back(it->second);
    }
    return out;
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

// copy of `src` restricted to `rows` of axis 0 and `props` of the last axis
void copy_rows(const Block& src, const std::vector<int64_t>& rows, const std::vector<int64_t>& props, double* dst) {
    const size_t n_props = src.shape.back();
    size_t inner = 1;  // product of the middle axes
    for (size_t a = 1; a + 1 < src.shape.size(); a++) inner *= src.shape[a];
    size_t o = 0;
    for (int64_t r : rows)
        for (size_t m = 0; m < inner; m++) {
            const double* s = src.data + ((size_t)r * inner + m) * n_props;
            for (int64_t p : props) dst[o++] = s[p];
        }
}

}  // namespace

std::unique_ptr<TensorMap> apply_selection(std::unique_ptr<TensorMap> full, const Selection& sel) {
    if (!sel.any()) return full;
    if (full->on_device) throw invalid_parameter("selections are only supported with host output");
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

    // per output block: selected sample rows and property columns
    struct Plan {
        const Block* src;
        std::vector<int64_t> rows, props;
        std::vector<Labels> components;
        Labels samples, properties;
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
        if (sel.samples) p.rows = select_subset(p.samples, *sel.samples, "samples");
        if (sel.samples_predefined)
            p.rows = select_predefined(p.samples, predefined_block(*sel.samples_predefined, keys, k, "samples")->samples,
                                       "samples");
        if (sel.properties) p.props = select_subset(p.properties, *sel.properties, "properties");
        if (sel.properties_predefined)
            p.props = select_predefined(
                p.properties, predefined_block(*sel.properties_predefined, keys, k, "properties")->properties,
                "properties");
        p.samples = rows_of(p.samples, p.rows);
        p.properties = rows_of(p.properties, p.props);
        size_t comp = 1;
        for (auto& c : p.components) comp *= c.count();
        total += p.rows.size() * comp * p.props.size();
        if (p.src)
            for (auto& g : p.src->gradients) {
                size_t inner = 1;
                for (size_t a = 1; a + 1 < g.second->shape.size(); a++) inner *= g.second->shape[a];
                total += g.second->shape[0] * inner * p.props.size();  // upper bound for positions rows
            }
    }

    auto out = std::make_unique<TensorMap>();
    out->keys = keys;
    out->on_device = false;
    out->device = tm.device;
    double* buffer = static_cast<double*>(std::malloc(std::max<size_t>(8, sizeof(double) * total)));
    if (!buffer) throw std::bad_alloc();
    out->storage = std::shared_ptr<void>(buffer, std::free);
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
        if (p.src) copy_rows(*p.src, p.rows, p.props, blk->data);
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
            if (gsrc && name == "positions") {
                // rows of each kept sample, in their order, renumbered
                std::vector<std::vector<int64_t>> by_sample(p.src->samples.count());
                const size_t gw = gsrc->samples.names.size();
                for (size_t r = 0; r < gsrc->samples.count(); r++)
                    by_sample[gsrc->samples.values[r * gw]].push_back((int64_t)r);
                for (size_t s = 0; s < p.rows.size(); s++)
                    for (int64_t r : by_sample[p.rows[s]]) {
                        grows.push_back(r);
                        gb->samples.values.push_back((int32_t)s);
                        gb->samples.values.insert(gb->samples.values.end(), gsrc->samples.values.begin() + r * gw + 1,
                                                  gsrc->samples.values.begin() + (r + 1) * gw);
                    }
            } else if (gsrc) {
                // strain / cell: one row per sample
                for (size_t s = 0; s < p.rows.size(); s++) {
                    grows.push_back(p.rows[s]);
                    gb->samples.values.push_back((int32_t)s);
                }
            }
            gb->shape = {grows.size()};
            for (auto& c : gb->components) gb->shape.push_back(c.count());
            gb->shape.push_back(p.props.size());
            gb->data = buffer + off;
            if (gsrc) copy_rows(*gsrc, grows, p.props, gb->data);
            off += gb->size();
            blk->gradients.emplace_back(name, std::move(gb));
        }
        out->blocks.push_back(std::move(blk));
    }
    if (off > std::max<size_t>(total, 1)) throw internal_error("selection: output buffer overflow");
    return out;
}

}  // namespace fb200

// Metadata of a compute call.  Restates featomic's labels builders on sorted
// arrays instead of BTreeSets:
//   keys       featomic/src/labels/keys.rs:61-159
//   samples    featomic/src/labels/samples/atom_centered.rs:31-101
//   gradients  featomic/src/labels/samples/atom_centered.rs:103-147
//   blocks     featomic/src/calculator.rs:414-495
//   power spectrum keys / samples: featomic/src/calculators/soap/power_spectrum.rs:423-481
//   spherical expansion keys / samples: spherical_expansion.rs:662-742
#include "plan.hpp"

#include <algorithm>
#include <map>
#include <tuple>

namespace fb200 {

Neighborhoods build_neighborhoods(const std::vector<HostSystem>& systems, int64_t n_pairs, const int32_t* first,
                                  const int32_t* second) {
    Neighborhoods nh;
    nh.atom_offset.push_back(0);
    std::vector<int32_t> types;
    for (size_t s = 0; s < systems.size(); s++) {
        for (int64_t i = 0; i < systems[s].n_atoms; i++) {
            types.push_back(systems[s].types[i]);
            nh.atom_system.push_back((int32_t)s);
            nh.atom_local.push_back((int32_t)i);
        }
        nh.atom_offset.push_back(nh.atom_offset.back() + systems[s].n_atoms);
    }
    nh.n_atoms = (int64_t)types.size();
    nh.species_types = types;
    std::sort(nh.species_types.begin(), nh.species_types.end());
    nh.species_types.erase(std::unique(nh.species_types.begin(), nh.species_types.end()), nh.species_types.end());
    nh.n_species = (int)nh.species_types.size();
    const int S = nh.n_species;
    nh.atom_species.resize(nh.n_atoms);
    for (int64_t a = 0; a < nh.n_atoms; a++)
        nh.atom_species[a] = (int32_t)(std::lower_bound(nh.species_types.begin(), nh.species_types.end(), types[a]) -
                                       nh.species_types.begin());

    // directions, counting sort on (centre, species of the other atom), stable in pair order
    std::vector<int64_t> count((size_t)nh.n_atoms * S + 1, 0);
    for (int64_t p = 0; p < n_pairs; p++) {
        count[(size_t)first[p] * S + nh.atom_species[second[p]]]++;
        count[(size_t)second[p] * S + nh.atom_species[first[p]]]++;
    }
    nh.seg_offset.assign((size_t)nh.n_atoms * S + 1, 0);
    for (size_t k = 0; k + 1 < nh.seg_offset.size(); k++) nh.seg_offset[k + 1] = nh.seg_offset[k] + count[k];
    std::vector<int64_t> fill(nh.seg_offset.begin(), nh.seg_offset.end() - 1);
    nh.dir_code.resize(2 * (size_t)n_pairs);
    for (int64_t p = 0; p < n_pairs; p++) {
        nh.dir_code[fill[(size_t)first[p] * S + nh.atom_species[second[p]]]++] = (int32_t)(p << 1);
        nh.dir_code[fill[(size_t)second[p] * S + nh.atom_species[first[p]]]++] = (int32_t)((p << 1) | 1);
    }

    // unique neighbours.  Inside a segment the other atoms are sorted (pairs
    // with the centre second come first, ordered by first; then the centre's
    // own pairs, ordered by second), so equal atoms are contiguous.
    nh.species_mask.assign((size_t)nh.n_atoms * S, 0);
    nh.entry_offset.assign(nh.n_atoms + 1, 0);
    std::vector<PsEntry> tmp;
    for (int64_t c = 0; c < nh.n_atoms; c++) {
        tmp.clear();
        nh.species_mask[(size_t)c * S + nh.atom_species[c]] = 1;
        for (int t = 0; t < S; t++) {
            int64_t d0 = nh.seg_offset[(size_t)c * S + t], d1 = nh.seg_offset[(size_t)c * S + t + 1];
            if (d1 > d0) nh.species_mask[(size_t)c * S + t] = 1;
            int64_t d = d0;
            while (d < d1) {
                int32_t code = nh.dir_code[d];
                int32_t p = code >> 1;
                int32_t other = (code & 1) ? first[p] : second[p];
                int64_t e = d + 1;
                while (e < d1) {
                    int32_t c2 = nh.dir_code[e];
                    int32_t p2 = c2 >> 1;
                    int32_t o2 = (c2 & 1) ? first[p2] : second[p2];
                    if (o2 != other) break;
                    e++;
                }
                if (other != (int32_t)c) tmp.push_back(PsEntry{other, t, (int32_t)d, (int32_t)e});
                d = e;
            }
        }
        tmp.push_back(PsEntry{(int32_t)c, nh.atom_species[c], -1, -1});
        std::sort(tmp.begin(), tmp.end(), [](const PsEntry& x, const PsEntry& y) { return x.atom < y.atom; });
        nh.entries.insert(nh.entries.end(), tmp.begin(), tmp.end());
        nh.entry_offset[c + 1] = (int64_t)nh.entries.size();
    }
    return nh;
}

std::vector<Labels> ps_components() { return {}; }

Labels ps_properties(const Hypers& h) {
    Labels p;
    p.names = {"l", "n_1", "n_2"};
    for (int l = 0; l <= h.max_angular; l++)
        for (int n1 = 0; n1 < h.nmax(); n1++)
            for (int n2 = 0; n2 < h.nmax(); n2++) p.values.insert(p.values.end(), {l, n1, n2});
    return p;
}

Labels se_properties(const Hypers& h) {
    Labels p;
    p.names = {"n"};
    for (int n = 0; n < h.nmax(); n++) p.values.push_back(n);
    return p;
}

namespace {

void assign_offsets(OutputPlan& plan, int64_t per_value_row, const GradientOptions& g,
                    const std::vector<int64_t>& per_block_width) {
    int64_t off = 0;
    for (size_t b = 0; b < plan.blocks.size(); b++) {
        auto& bp = plan.blocks[b];
        int64_t w = per_block_width.empty() ? per_value_row : per_block_width[b];
        bp.off_values = off;
        off += bp.n_samples * w;
        if (g.positions) {
            bp.off_positions = off;
            off += bp.n_grad_rows * 3 * w;
        }
        if (g.strain) {
            bp.off_strain = off;
            off += bp.n_samples * 9 * w;
        }
        if (g.cell) {
            bp.off_cell = off;
            off += bp.n_samples * 9 * w;
        }
    }
    plan.total_doubles = off;
}

}  // namespace

OutputPlan plan_power_spectrum(const Neighborhoods& nh, const Hypers& h, const GradientOptions& g) {
    OutputPlan plan;
    const int S = nh.n_species;
    // keys: (center, a, b) with a <= b among the species around every centre
    std::vector<uint8_t> present((size_t)S * S * S, 0);
    for (int64_t c = 0; c < nh.n_atoms; c++) {
        const uint8_t* mask = &nh.species_mask[(size_t)c * S];
        for (int a = 0; a < S; a++) {
            if (!mask[a]) continue;
            for (int b = a; b < S; b++)
                if (mask[b]) present[((size_t)nh.atom_species[c] * S + a) * S + b] = 1;
        }
    }
    std::vector<int32_t> key_index((size_t)S * S * S, -1);
    plan.keys.names = {"center_type", "neighbor_1_type", "neighbor_2_type"};
    for (int ct = 0; ct < S; ct++)
        for (int a = 0; a < S; a++)
            for (int b = a; b < S; b++) {
                if (!present[((size_t)ct * S + a) * S + b]) continue;
                key_index[((size_t)ct * S + a) * S + b] = (int32_t)plan.blocks.size();
                plan.keys.values.insert(plan.keys.values.end(), {nh.species_types[ct], nh.species_types[a], nh.species_types[b]});
                plan.blocks.emplace_back();
            }
    for (auto& bp : plan.blocks) {
        bp.samples.names = {"system", "atom"};
        bp.gradient_samples.names = {"sample", "system", "atom"};
    }

    // samples (AllOf{a, b}) and gradient samples (OneOf[a, b]), centre by centre
    plan.slot_offset.assign(nh.n_atoms + 1, 0);
    plan.row_offset.assign(nh.n_atoms + 1, 0);
    for (int64_t c = 0; c < nh.n_atoms; c++) {
        const uint8_t* mask = &nh.species_mask[(size_t)c * S];
        int64_t e0 = nh.entry_offset[c], e1 = nh.entry_offset[c + 1];
        int64_t first_slot = (int64_t)plan.slots.size();
        for (int a = 0; a < S; a++) {
            if (!mask[a]) continue;
            for (int b = a; b < S; b++) {
                if (!mask[b]) continue;
                int32_t k = key_index[((size_t)nh.atom_species[c] * S + a) * S + b];
                auto& bp = plan.blocks[k];
                int32_t sample = (int32_t)bp.n_samples++;
                bp.samples.values.insert(bp.samples.values.end(), {nh.atom_system[c], nh.atom_local[c]});
                plan.slots.push_back(PsKeySlot{k, sample, a, b});
            }
        }
        int64_t ns = (int64_t)plan.slots.size() - first_slot;
        plan.slot_offset[c + 1] = (int64_t)plan.slots.size();
        if (g.positions) {
            int64_t base = (int64_t)plan.rows.size();
            plan.rows.resize(base + (e1 - e0) * ns, -1);
            // rows of one sample are contiguous and sorted by neighbour atom
            for (int64_t s = 0; s < ns; s++) {
                const PsKeySlot& slot = plan.slots[first_slot + s];
                auto& bp = plan.blocks[slot.block];
                for (int64_t e = e0; e < e1; e++) {
                    const PsEntry& en = nh.entries[e];
                    if (en.atom != (int32_t)c && en.species != slot.a && en.species != slot.b) continue;
                    plan.rows[base + (e - e0) * ns + s] = bp.n_grad_rows++;
                    bp.gradient_samples.values.insert(bp.gradient_samples.values.end(),
                                                      {slot.sample, nh.atom_system[c], nh.atom_local[en.atom]});
                }
            }
        }
        plan.row_offset[c + 1] = (int64_t)plan.rows.size();
    }
    int64_t n_props = (int64_t)(h.max_angular + 1) * h.nmax() * h.nmax();
    assign_offsets(plan, n_props, g, {});
    return plan;
}

OutputPlan plan_spherical_expansion(const Neighborhoods& nh, const Hypers& h, const GradientOptions& g) {
    OutputPlan plan;
    const int S = nh.n_species;
    const int L = h.max_angular;
    std::vector<uint8_t> present((size_t)S * S, 0);
    for (int64_t c = 0; c < nh.n_atoms; c++)
        for (int t = 0; t < S; t++)
            if (nh.species_mask[(size_t)c * S + t]) present[(size_t)nh.atom_species[c] * S + t] = 1;
    // keys: (l, 1, center, neighbor) with l varying fastest
    std::vector<int32_t> pair_block((size_t)S * S, -1);
    plan.keys.names = {"o3_lambda", "o3_sigma", "center_type", "neighbor_type"};
    for (int ct = 0; ct < S; ct++)
        for (int nt = 0; nt < S; nt++) {
            if (!present[(size_t)ct * S + nt]) continue;
            pair_block[(size_t)ct * S + nt] = (int32_t)plan.blocks.size();
            for (int l = 0; l <= L; l++) {
                plan.keys.values.insert(plan.keys.values.end(), {l, 1, nh.species_types[ct], nh.species_types[nt]});
                plan.blocks.emplace_back();
                plan.blocks.back().l = l;
                plan.blocks.back().species = nt;
                plan.blocks.back().samples.names = {"system", "atom"};
                plan.blocks.back().gradient_samples.names = {"sample", "system", "atom"};
                plan.block_l.push_back(l);
                plan.block_species.push_back(nt);
            }
        }
    for (int64_t c = 0; c < nh.n_atoms; c++) {
        for (int nt = 0; nt < S; nt++) {
            if (!nh.species_mask[(size_t)c * S + nt]) continue;
            int32_t b0 = pair_block[(size_t)nh.atom_species[c] * S + nt];
            for (int l = 0; l <= L; l++) {
                auto& bp = plan.blocks[b0 + l];
                int32_t sample = (int32_t)bp.n_samples++;
                bp.samples.values.insert(bp.samples.values.end(), {nh.atom_system[c], nh.atom_local[c]});
                plan.row_centre.push_back((int32_t)c);
                plan.row_block.push_back(b0 + l);
                plan.row_sample.push_back(sample);
                if (!g.positions) continue;
                for (int64_t e = nh.entry_offset[c]; e < nh.entry_offset[c + 1]; e++) {
                    const PsEntry& en = nh.entries[e];
                    if (en.atom != (int32_t)c && en.species != nt) continue;
                    plan.grad_block.push_back(b0 + l);
                    plan.grad_row.push_back(bp.n_grad_rows++);
                    plan.grad_centre.push_back((int32_t)c);
                    plan.grad_atom.push_back(en.atom);
                    plan.grad_d0.push_back(en.d0);
                    plan.grad_d1.push_back(en.d1);
                    bp.gradient_samples.values.insert(bp.gradient_samples.values.end(),
                                                      {sample, nh.atom_system[c], nh.atom_local[en.atom]});
                }
            }
        }
    }
    std::vector<int64_t> widths;
    for (auto& bp : plan.blocks) widths.push_back((int64_t)(2 * bp.l + 1) * h.nmax());
    assign_offsets(plan, 0, g, widths);
    return plan;
}

}  // namespace fb200

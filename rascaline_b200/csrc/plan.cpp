// Metadata of a compute call.  Restates featomic's labels builders on sorted
// arrays instead of BTreeSets:
//   keys       featomic/src/labels/keys.rs:61-159
//   samples    featomic/src/labels/samples/atom_centered.rs:31-101
//   gradients  featomic/src/labels/samples/atom_centered.rs:103-147
//   blocks     featomic/src/calculator.rs:414-495
//   power spectrum keys / samples: featomic/src/calculators/soap/power_spectrum.rs:423-481
//   spherical expansion keys / samples: spherical_expansion.rs:662-742
//
// Every table is built in O(pairs + rows) with exact pre-sizing; the
// gradient sample labels are the only per-row work.
#include "plan.hpp"

#include <omp.h>

#include <algorithm>

namespace fb200 {

void build_neighborhoods(const std::vector<HostSystem>& systems, int64_t n_pairs, const int32_t* first,
                         const int32_t* second, Neighborhoods& nh) {
    // every vector is resized, not reallocated: a Neighborhoods kept by the
    // caller between calls reuses its storage (no page faults on the host)
    int64_t n_atoms = 0;
    for (auto& s : systems) n_atoms += s.n_atoms;
    nh.n_atoms = n_atoms;
    nh.atom_offset.resize(systems.size() + 1);
    nh.atom_system.resize(n_atoms);
    nh.atom_local.resize(n_atoms);
    nh.atom_species.resize(n_atoms);
    {
        int64_t a = 0;
        nh.atom_offset[0] = 0;
        for (size_t s = 0; s < systems.size(); s++) {
            for (int64_t i = 0; i < systems[s].n_atoms; i++, a++) {
                nh.atom_system[a] = (int32_t)s;
                nh.atom_local[a] = (int32_t)i;
            }
            nh.atom_offset[s + 1] = a;
        }
    }
    nh.species_types.clear();
    for (auto& s : systems) nh.species_types.insert(nh.species_types.end(), s.types.begin(), s.types.end());
    std::sort(nh.species_types.begin(), nh.species_types.end());
    nh.species_types.erase(std::unique(nh.species_types.begin(), nh.species_types.end()), nh.species_types.end());
    const int S = nh.n_species = (int)nh.species_types.size();
    if (S > 64) throw invalid_parameter("more than 64 atomic types are not supported");
    {
        int64_t a = 0;
        for (auto& s : systems)
            for (int32_t t : s.types)
                nh.atom_species[a++] = (int32_t)(std::lower_bound(nh.species_types.begin(), nh.species_types.end(), t) -
                                                 nh.species_types.begin());
    }
    const int32_t* sp = nh.atom_species.data();

    // directions: counting sort on (centre, species of the other atom),
    // stable in pair order.  Each thread counts a contiguous range of pairs;
    // a thread's slice of every bin starts after the slices of the threads
    // before it, so the parallel fill keeps pair order inside every bin.
    const int64_t n_bins = n_atoms * S;
    nh.seg_offset.assign((size_t)n_bins + 1, 0);
    nh.dir_code.resize(2 * (size_t)n_pairs);
    int64_t* seg = nh.seg_offset.data();
    int32_t* dir = nh.dir_code.data();
    const int n_threads = std::max(1, std::min(omp_get_max_threads(), (int)std::min<int64_t>(64, n_pairs / 2048 + 1)));
    nh.bin_scratch.assign((size_t)n_threads * n_bins, 0);
    int64_t* local = nh.bin_scratch.data();
#pragma omp parallel num_threads(n_threads)
    {
        const int t = omp_get_thread_num(), nt = omp_get_num_threads();
        const int64_t p0 = n_pairs * t / nt, p1 = n_pairs * (t + 1) / nt;
        int64_t* mine = local + (size_t)t * n_bins;
        for (int64_t p = p0; p < p1; p++) {
            mine[(size_t)first[p] * S + sp[second[p]]]++;
            mine[(size_t)second[p] * S + sp[first[p]]]++;
        }
#pragma omp barrier
        // bin totals and each thread's starting position, by bin ranges
        const int64_t b0 = n_bins * t / nt, b1 = n_bins * (t + 1) / nt;
        for (int64_t b = b0; b < b1; b++) {
            int64_t total = 0;
            for (int k = 0; k < nt; k++) {
                const int64_t c = local[(size_t)k * n_bins + b];
                local[(size_t)k * n_bins + b] = total;
                total += c;
            }
            seg[b + 1] = total;
        }
#pragma omp barrier
#pragma omp single
        for (int64_t b = 1; b <= n_bins; b++) seg[b] += seg[b - 1];
        for (int64_t p = p0; p < p1; p++) {
            const size_t bf = (size_t)first[p] * S + sp[second[p]], bs = (size_t)second[p] * S + sp[first[p]];
            dir[seg[bf] + mine[bf]++] = (int32_t)(p << 1);
            dir[seg[bs] + mine[bs]++] = (int32_t)((p << 1) | 1);
        }
    }
    // the other atom of every direction, in segment order: the merges below
    // then read one contiguous array per segment
    nh.other_atom.resize(2 * (size_t)n_pairs);
    int32_t* other = nh.other_atom.data();
#pragma omp parallel for schedule(static)
    for (int64_t k = 0; k < 2 * n_pairs; k++) {
        const int32_t code = dir[k];
        other[k] = (code & 1) ? first[code >> 1] : second[code >> 1];
    }

    // unique neighbours.  Inside a segment the other atoms are sorted (pairs
    // with the centre second come first, ordered by first; then the centre's
    // own pairs, ordered by second), so an S-way merge of the segments lists
    // every centre's neighbours by atom index.  Centres are independent: a
    // counting pass sizes every centre's list, a second pass fills it.
    nh.species_mask.assign((size_t)n_atoms * S, 0);
    nh.species_count.assign((size_t)n_atoms * S, 0);
    nh.entry_offset.assign(n_atoms + 1, 0);
    auto merge = [&](int64_t c, PsEntry* out, int32_t* cum_out, int32_t* count_out) -> int64_t {
        int64_t pos[64], end[64];
        int32_t cum[65];
        const int sc = sp[c];
        for (int t = 0; t < S; t++) {
            pos[t] = seg[(size_t)c * S + t];
            end[t] = seg[(size_t)c * S + t + 1];
        }
        for (int t = 0; t <= S; t++) cum[t] = 0;
        bool self_done = false;
        int64_t n = 0;
        auto emit = [&](const PsEntry& e) {
            if (out) {
                out[n] = e;
                for (int t = 0; t <= S; t++) cum_out[n * (S + 1) + t] = cum[t];
            }
            n++;
        };
        while (true) {
            int best = -1;
            int32_t best_atom = 0;
            for (int t = 0; t < S; t++) {
                if (pos[t] < end[t]) {
                    int32_t o = other[pos[t]];
                    if (best < 0 || o < best_atom) {
                        best = t;
                        best_atom = o;
                    }
                }
            }
            if (!self_done && (best < 0 || best_atom >= (int32_t)c)) {
                emit(PsEntry{(int32_t)c, sc, -1, -1});
                cum[S] = 1;
                self_done = true;
            }
            if (best < 0) break;
            int64_t d0 = pos[best], d = d0 + 1;
            while (d < end[best] && other[d] == best_atom) d++;
            pos[best] = d;
            if (best_atom == (int32_t)c) continue;  // periodic images of the centre itself
            emit(PsEntry{best_atom, best, (int32_t)d0, (int32_t)d});
            cum[best]++;
        }
        if (count_out)
            for (int t = 0; t < S; t++) count_out[t] = cum[t];
        return n;
    };
#pragma omp parallel for schedule(static)
    for (int64_t c = 0; c < n_atoms; c++) {
        nh.entry_offset[c + 1] = merge(c, nullptr, nullptr, &nh.species_count[(size_t)c * S]);
        for (int t = 0; t < S; t++)
            nh.species_mask[(size_t)c * S + t] = (seg[(size_t)c * S + t + 1] > seg[(size_t)c * S + t] || t == sp[c]) ? 1 : 0;
    }
    for (int64_t c = 0; c < n_atoms; c++) nh.entry_offset[c + 1] += nh.entry_offset[c];
    nh.entries.resize(nh.entry_offset[n_atoms]);
    nh.entry_cum.resize((size_t)nh.entry_offset[n_atoms] * (S + 1));
#pragma omp parallel for schedule(static)
    for (int64_t c = 0; c < n_atoms; c++)
        merge(c, nh.entries.data() + nh.entry_offset[c], nh.entry_cum.data() + nh.entry_offset[c] * (S + 1), nullptr);
}

Neighborhoods build_neighborhoods(const std::vector<HostSystem>& systems, int64_t n_pairs, const int32_t* first,
                                  const int32_t* second) {
    Neighborhoods nh;
    build_neighborhoods(systems, n_pairs, first, second, nh);
    return nh;
}

Labels ps_properties(const Hypers& h) {
    Labels p;
    p.names = {"l", "n_1", "n_2"};
    p.values.reserve((size_t)(h.max_angular + 1) * h.nmax() * h.nmax() * 3);
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

void assign_offsets(OutputPlan& plan, const GradientOptions& g, const std::vector<int64_t>& width) {
    int64_t off = 0;
    for (size_t b = 0; b < plan.blocks.size(); b++) {
        auto& bp = plan.blocks[b];
        int64_t w = width[b];
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

OutputPlan plan_power_spectrum(const Neighborhoods& nh, const Hypers& h, const GradientOptions& g, bool with_labels) {
    OutputPlan plan;
    const int S = nh.n_species;
    const int64_t N = nh.n_atoms;
    // keys: (center, a, b) with a <= b among the species around every centre
    std::vector<int32_t> key_index((size_t)S * S * S, -1);
    for (int64_t c = 0; c < N; c++) {
        const uint8_t* mask = &nh.species_mask[(size_t)c * S];
        for (int a = 0; a < S; a++) {
            if (!mask[a]) continue;
            for (int b = a; b < S; b++)
                if (mask[b]) key_index[((size_t)nh.atom_species[c] * S + a) * S + b] = 0;
        }
    }
    plan.keys.names = {"center_type", "neighbor_1_type", "neighbor_2_type"};
    int32_t nb = 0;
    for (size_t k = 0; k < key_index.size(); k++) {
        if (key_index[k] < 0) continue;
        key_index[k] = nb++;
        int ct = (int)(k / ((size_t)S * S)), a = (int)((k / S) % S), b = (int)(k % S);
        plan.keys.values.insert(plan.keys.values.end(), {nh.species_types[ct], nh.species_types[a], nh.species_types[b]});
    }
    plan.blocks.resize(nb);

    // slots, sample rows and the first gradient row of every slot
    plan.slot_offset.assign(N + 1, 0);
    for (int64_t c = 0; c < N; c++) {
        const uint8_t* mask = &nh.species_mask[(size_t)c * S];
        const int32_t* count = &nh.species_count[(size_t)c * S];
        for (int a = 0; a < S; a++) {
            if (!mask[a]) continue;
            for (int b = a; b < S; b++) {
                if (!mask[b]) continue;
                int32_t k = key_index[((size_t)nh.atom_species[c] * S + a) * S + b];
                auto& bp = plan.blocks[k];
                plan.slots.push_back(PsKeySlot{k, (int32_t)bp.n_samples++, a, b});
                plan.slot_row.push_back(bp.n_grad_rows);
                bp.n_grad_rows += count[a] + (a != b ? count[b] : 0) + 1;
            }
        }
        plan.slot_offset[c + 1] = (int64_t)plan.slots.size();
    }

    int64_t n_props = (int64_t)(h.max_angular + 1) * h.nmax() * h.nmax();
    assign_offsets(plan, g, std::vector<int64_t>(nb, n_props));
    if (with_labels) fill_power_spectrum_labels(nh, g, plan);
    return plan;
}

void fill_power_spectrum_labels(const Neighborhoods& nh, const GradientOptions& g, OutputPlan& plan) {
    const int64_t N = nh.n_atoms;
    const int S = nh.n_species;
    const int32_t nb = (int32_t)plan.blocks.size();
    // labels, written in place: every slot knows its sample row and its first
    // gradient row, so centres fill their rows independently
    std::vector<int32_t*> sample_w(nb), grad_w(nb);
#pragma omp parallel for schedule(static)
    for (int32_t k = 0; k < nb; k++) {
        auto& bp = plan.blocks[k];
        bp.samples.names = {"system", "atom"};
        bp.samples.values.resize((size_t)bp.n_samples * 2);
        sample_w[k] = bp.samples.values.data();
        bp.gradient_samples.names = {"sample", "system", "atom"};
        if (g.positions) {
            bp.gradient_samples.values.resize((size_t)bp.n_grad_rows * 3);
            grad_w[k] = bp.gradient_samples.values.data();
        }
    }
#pragma omp parallel
    {
        // per centre: the write position of every slot's next gradient row,
        // and the slots of each neighbour species
        std::vector<int32_t*> w;
        std::vector<int32_t> by_species, n_by_species(S);
#pragma omp for schedule(static)
        for (int64_t c = 0; c < N; c++) {
            const int32_t sys = nh.atom_system[c];
            const int64_t s0 = plan.slot_offset[c], ns = plan.slot_offset[c + 1] - s0;
            for (int64_t i = 0; i < ns; i++) {
                const PsKeySlot& slot = plan.slots[s0 + i];
                int32_t* sw = sample_w[slot.block] + 2 * (size_t)slot.sample;
                sw[0] = sys;
                sw[1] = nh.atom_local[c];
            }
            if (!g.positions) continue;
            w.resize(ns);
            by_species.resize((size_t)S * ns);
            std::fill(n_by_species.begin(), n_by_species.end(), 0);
            for (int64_t i = 0; i < ns; i++) {
                const PsKeySlot& slot = plan.slots[s0 + i];
                w[i] = grad_w[slot.block] + 3 * (size_t)plan.slot_row[s0 + i];
                by_species[(size_t)slot.a * ns + n_by_species[slot.a]++] = (int32_t)i;
                if (slot.b != slot.a) by_species[(size_t)slot.b * ns + n_by_species[slot.b]++] = (int32_t)i;
            }
            // entries in atom order: each row goes to the end of its slots' rows
            for (int64_t e = nh.entry_offset[c]; e < nh.entry_offset[c + 1]; e++) {
                const PsEntry& en = nh.entries[e];
                const int32_t local = nh.atom_local[en.atom];
                if (en.atom == (int32_t)c) {
                    for (int64_t i = 0; i < ns; i++) {
                        int32_t* gw = w[i];
                        gw[0] = plan.slots[s0 + i].sample;
                        gw[1] = sys;
                        gw[2] = local;
                        w[i] = gw + 3;
                    }
                    continue;
                }
                for (int j = 0; j < n_by_species[en.species]; j++) {
                    const int32_t i = by_species[(size_t)en.species * ns + j];
                    int32_t* gw = w[i];
                    gw[0] = plan.slots[s0 + i].sample;
                    gw[1] = sys;
                    gw[2] = local;
                    w[i] = gw + 3;
                }
            }
        }
    }
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
    assign_offsets(plan, g, widths);
    return plan;
}

// spherical_expansion_by_pair (spherical_expansion_pair.rs:547-700) with the
// samples of FullNeighborList (calculators/neighbor_list.rs:372-490): for
// each (first type, second type) the pairs of each system in pair order
// (both directions when the types are equal, else the matching one), then,
// for l = 0 only, that system's self pairs (i, i, 0 0 0).  Every direction
// lands in exactly one row of the blocks of its type pair.
OutputPlan plan_by_pair(const Neighborhoods& nh, const Hypers& h, const GradientOptions& g, int64_t n_pairs,
                        const int32_t* first, const int32_t* second, const int32_t* shift) {
    OutputPlan plan;
    const int L = h.max_angular;
    auto type_of = [&](int64_t atom) { return nh.species_types[nh.atom_species[atom]]; };
    std::vector<std::pair<int32_t, int32_t>> tps;
    for (int64_t p = 0; p < n_pairs; p++) {
        tps.push_back({type_of(first[p]), type_of(second[p])});
        tps.push_back({type_of(second[p]), type_of(first[p])});
    }
    for (int64_t a = 0; a < nh.n_atoms; a++) tps.push_back({type_of(a), type_of(a)});
    std::sort(tps.begin(), tps.end());
    tps.erase(std::unique(tps.begin(), tps.end()), tps.end());
    auto tp_index = [&](int32_t a, int32_t b) {
        return (int32_t)(std::lower_bound(tps.begin(), tps.end(), std::make_pair(a, b)) - tps.begin());
    };
    plan.keys.names = {"o3_lambda", "o3_sigma", "first_atom_type", "second_atom_type"};
    for (auto& t : tps)
        for (int l = 0; l <= L; l++) {
            plan.keys.values.insert(plan.keys.values.end(), {l, 1, t.first, t.second});
            plan.blocks.emplace_back();
            BlockPlan& b = plan.blocks.back();
            b.l = l;
            b.samples.names = {"system", "first_atom", "second_atom", "cell_shift_a", "cell_shift_b", "cell_shift_c"};
            b.gradient_samples.names = {"sample", "system", "atom"};
        }
    const size_t T = tps.size();
    std::vector<int64_t> n0(T, 0), n1(T, 0), ngrad(T, 0);
    plan.bp_block0.resize(2 * n_pairs);
    plan.bp_row0.resize(2 * n_pairs);
    plan.bp_row1.resize(2 * n_pairs);
    plan.bp_grow.resize(2 * n_pairs);
    auto add_direction = [&](int64_t d, int32_t system, int64_t a, int64_t b, int32_t s0, int32_t s1, int32_t s2) {
        const int32_t ti = tp_index(type_of(a), type_of(b));
        const int32_t la = nh.atom_local[a], lb = nh.atom_local[b];
        const int64_t r0 = n0[ti]++, r1 = n1[ti]++;
        plan.bp_block0[d] = ti * (L + 1);
        plan.bp_row0[d] = r0;
        plan.bp_row1[d] = r1;
        plan.bp_grow[d] = ngrad[ti];
        ngrad[ti] += la == lb ? 1 : 2;
        for (int l = 0; l <= L; l++) {
            BlockPlan& bp = plan.blocks[(size_t)ti * (L + 1) + l];
            const int32_t row = (int32_t)(l == 0 ? r0 : r1);
            bp.samples.values.insert(bp.samples.values.end(), {system, la, lb, s0, s1, s2});
            if (!g.positions) continue;
            bp.gradient_samples.values.insert(bp.gradient_samples.values.end(), {row, system, la});
            if (la != lb) bp.gradient_samples.values.insert(bp.gradient_samples.values.end(), {row, system, lb});
        }
    };
    int64_t p = 0;
    const int64_t n_systems = (int64_t)nh.atom_offset.size() - 1;
    for (int64_t s = 0; s < n_systems; s++) {
        for (; p < n_pairs && nh.atom_system[first[p]] == s; p++) {
            const int32_t* sh = shift + 3 * p;
            add_direction(2 * p, (int32_t)s, first[p], second[p], sh[0], sh[1], sh[2]);
            add_direction(2 * p + 1, (int32_t)s, second[p], first[p], -sh[0], -sh[1], -sh[2]);
        }
        for (int64_t a = nh.atom_offset[s]; a < nh.atom_offset[s + 1]; a++) {
            const int32_t ti = tp_index(type_of(a), type_of(a));
            BlockPlan& bp = plan.blocks[(size_t)ti * (L + 1)];
            plan.bp_self_block.push_back(ti * (L + 1));
            plan.bp_self_row.push_back(n0[ti]++);
            bp.samples.values.insert(bp.samples.values.end(), {(int32_t)s, nh.atom_local[a], nh.atom_local[a], 0, 0, 0});
        }
    }
    if (p != n_pairs) throw internal_error("spherical_expansion_by_pair: pairs are not grouped by system");
    for (size_t ti = 0; ti < T; ti++)
        for (int l = 0; l <= L; l++) {
            BlockPlan& bp = plan.blocks[ti * (L + 1) + l];
            bp.n_samples = l == 0 ? n0[ti] : n1[ti];
            bp.n_grad_rows = g.positions ? ngrad[ti] : 0;
        }
    std::vector<int64_t> widths;
    for (auto& bp : plan.blocks) widths.push_back((int64_t)(2 * bp.l + 1) * h.nmax());
    assign_offsets(plan, g, widths);
    return plan;
}

}  // namespace fb200

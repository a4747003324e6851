// Host-side metadata of one compute call: neighbour bookkeeping, the keys /
// samples / gradient samples of the output TensorMap, and the index tables
// the kernels consume.
#pragma once

#include <cstdint>
#include <vector>

#include "engine.hpp"
#include "host.hpp"

namespace fb200 {

// Neighbourhood bookkeeping shared by both calculators
struct Neighborhoods {
    int64_t n_atoms = 0;
    int n_species = 0;
    std::vector<int32_t> species_types;  // sorted unique atomic types
    std::vector<int32_t> atom_species;   // [n_atoms]
    std::vector<int32_t> atom_system;    // [n_atoms]
    std::vector<int32_t> atom_local;     // index inside its system
    std::vector<int64_t> atom_offset;    // [n_systems + 1]
    // directions (pair << 1 | reversed), grouped by (centre, neighbour species)
    // and ordered by pair inside a group
    std::vector<int64_t> seg_offset;     // [n_atoms * S + 1]
    std::vector<int32_t> dir_code;
    // unique neighbours of every centre plus the centre itself, by atom index
    std::vector<int64_t> entry_offset;   // [n_atoms + 1]
    std::vector<PsEntry> entries;
    // per entry: S prefix counts of earlier neighbours by species, then 1 if
    // the centre itself comes earlier in the list
    std::vector<int32_t> entry_cum;      // [entries][S + 1]
    // per centre: number of unique neighbours of each species
    std::vector<int32_t> species_count;  // [n_atoms * S]
    // species present around each centre (own species included)
    std::vector<uint8_t> species_mask;   // [n_atoms * S]
    // working storage of the build, kept with the rest for reuse
    std::vector<int32_t> other_atom;     // the other atom of every direction
    std::vector<int64_t> bin_scratch;    // per-thread counting-sort bins
};

Neighborhoods build_neighborhoods(const std::vector<HostSystem>& systems, int64_t n_pairs, const int32_t* first,
                                  const int32_t* second);
// the same into `nh`, reusing its storage
void build_neighborhoods(const std::vector<HostSystem>& systems, int64_t n_pairs, const int32_t* first,
                         const int32_t* second, Neighborhoods& nh);

// Output plan: labels of every block and where the block lives in the
// output buffer (offsets in doubles)
struct BlockPlan {
    Labels samples;
    Labels gradient_samples;  // positions
    int64_t n_samples = 0, n_grad_rows = 0;
    int64_t off_values = 0, off_positions = -1, off_strain = -1, off_cell = -1;
    int l = 0;        // spherical expansion blocks
    int species = 0;  // neighbour species (spherical expansion)
};

struct OutputPlan {
    Labels keys;
    std::vector<BlockPlan> blocks;
    int64_t total_doubles = 0;
    // power spectrum tables
    std::vector<int64_t> slot_offset;  // [n_atoms + 1]
    std::vector<PsKeySlot> slots;
    std::vector<int64_t> slot_row;     // first gradient row of every slot
    // spherical expansion tables
    std::vector<int32_t> row_centre, row_block, row_sample;
    std::vector<int32_t> grad_block, grad_centre, grad_atom, grad_d0, grad_d1;
    std::vector<int64_t> grad_row;
    std::vector<int32_t> block_l, block_species;
    // spherical expansion by pair, per direction d = 2 pair + reversed: the
    // block of l = 0 of its type pair (block of l = block0 + l), its row in
    // the l = 0 and l > 0 blocks and its first positions gradient row; and
    // the self pairs (l = 0 block, row)
    std::vector<int32_t> bp_block0;
    std::vector<int64_t> bp_row0, bp_row1, bp_grow;
    std::vector<int32_t> bp_self_block;
    std::vector<int64_t> bp_self_row;
};

// without labels, the kernel tables and offsets only: the sample and
// gradient-sample labels can then be written by fill_power_spectrum_labels
// while the kernels run
OutputPlan plan_power_spectrum(const Neighborhoods& nh, const Hypers& h, const GradientOptions& g,
                               bool with_labels = true);
void fill_power_spectrum_labels(const Neighborhoods& nh, const GradientOptions& g, OutputPlan& plan);
OutputPlan plan_spherical_expansion(const Neighborhoods& nh, const Hypers& h, const GradientOptions& g);
OutputPlan plan_by_pair(const Neighborhoods& nh, const Hypers& h, const GradientOptions& g, int64_t n_pairs,
                        const int32_t* first, const int32_t* second, const int32_t* shift);

// Labels of the properties of each calculator
Labels ps_properties(const Hypers& h);
Labels se_properties(const Hypers& h);

}  // namespace fb200

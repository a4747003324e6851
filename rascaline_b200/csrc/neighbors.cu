// Kernel (a): periodic cell-list neighbour search on the GPU.
//
// Produces featomic's half neighbour list (featomic/src/systems/neighbors.rs:
// CellList::new :101-163, add_atom :167-201, pairs :217-309,
// NeighborsList::new :349-403) for a batch of systems in one pass:
//
//   1. bin atoms: fractional coordinates (vector x inverse cell), floor, Python
//      divmod wrap (one thread per atom; atomics only on integer cell counts)
//   2. count the candidate pairs of every atom i over the (2 n_search + 1)^3
//      neighbouring cells (j >= i, the self-image half-space rules), keeping
//      those with |r_ij|^2 < rc^2 -- one warp per atom, lanes over candidates
//   3. exclusive scan of the counts (CUB)
//   4. the same warp compacts its kept pairs by ballot into a scratch list,
//      then places every pair at its rank in (second, shift) order
//
// The list is therefore ordered by (first, second, shift); featomic sorts by
// (first, second) with an unstable sort, so only ties between periodic images
// of the same two atoms can be ordered differently (tests compare those runs
// as multisets).  Distances and vectors use explicit round-to-nearest
// intrinsics so that no FMA is contracted and the bits match the CPU
// evaluation order: vector = (r_j - r_i) + (H^T s), d^2 = x x + y y + z z.
#include <cub/cub.cuh>

#include <mutex>

#include "engine.hpp"
#include "featomic_b200.h"

namespace fb200 {

namespace {

__device__ __forceinline__ void divmod_i(int a, int b, int* q, int* r) {
    int quotient = a / b;
    int remainder = a % b;
    if (remainder < 0) {
        remainder += b;
        quotient -= 1;
    }
    *q = quotient;
    *r = remainder;
}

__global__ void nl_assign_cells(const NlSystem* __restrict__ systems, const int32_t* __restrict__ atom_system,
                                const double* __restrict__ positions, int64_t n_atoms, int32_t* __restrict__ cell_of,
                                int32_t* __restrict__ atom_shift, int32_t* __restrict__ cell_count) {
    int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= n_atoms) return;
    const NlSystem& s = systems[atom_system[g]];
    double p0 = positions[3 * g], p1 = positions[3 * g + 1], p2 = positions[3 * g + 2];
    double f[3];
    if (s.infinite) {
        f[0] = p0;
        f[1] = p1;
        f[2] = p2;
    } else {
        // row vector times inverse matrix, matrix.rs:399-407
        for (int k = 0; k < 3; k++) {
            f[k] = __dadd_rn(__dadd_rn(__dmul_rn(p0, s.inv[0 * 3 + k]), __dmul_rn(p1, s.inv[1 * 3 + k])),
                             __dmul_rn(p2, s.inv[2 * 3 + k]));
        }
    }
    int idx[3], sh[3];
    for (int k = 0; k < 3; k++) {
        int ci = (int)floor(__dmul_rn(f[k], (double)s.n_cells[k]));
        if (s.infinite) {
            // `cell_index as usize` then usize::clamp(.., 0, n - 1): negative
            // values wrap to huge numbers and land in the last cell
            unsigned long long u = (unsigned long long)(long long)ci;
            unsigned long long hi = (unsigned long long)(s.n_cells[k] - 1);
            idx[k] = (int)(u > hi ? hi : u);
            sh[k] = 0;
        } else {
            divmod_i(ci, s.n_cells[k], &sh[k], &idx[k]);
        }
    }
    int32_t cell = (int32_t)(s.cell_offset + ((int64_t)idx[0] * s.n_cells[1] + idx[1]) * s.n_cells[2] + idx[2]);
    cell_of[g] = cell;
    atom_shift[3 * g] = sh[0];
    atom_shift[3 * g + 1] = sh[1];
    atom_shift[3 * g + 2] = sh[2];
    atomicAdd(&cell_count[cell], 1);
}

__global__ void nl_fill_cells(const int32_t* __restrict__ cell_of, int64_t n_atoms, const int32_t* __restrict__ cell_start,
                              int32_t* __restrict__ cell_fill, int32_t* __restrict__ cell_atoms) {
    int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= n_atoms) return;
    int32_t c = cell_of[g];
    int slot = atomicAdd(&cell_fill[c], 1);
    cell_atoms[cell_start[c] + slot] = (int32_t)g;
}

// Candidate pairs of atom g, enumerated by one warp: the lanes stride over
// the atoms of every neighbouring cell.  `visit(keep, j, shift, v, d2)` is
// called by every lane for every round (keep is false for lanes without a
// kept pair), so that the caller can use warp-wide ballots.
template <typename Visit>
__device__ __forceinline__ void nl_warp_enumerate(const NlSystem& s, int64_t g, const double* __restrict__ positions,
                                                  const int32_t* __restrict__ cell_of, const int32_t* __restrict__ atom_shift,
                                                  const int32_t* __restrict__ cell_start, const int32_t* __restrict__ cell_count,
                                                  const int32_t* __restrict__ cell_atoms, int lane, Visit visit) {
    const int local = (int)(cell_of[g] - s.cell_offset);
    const int cz = local % s.n_cells[2];
    const int cy = (local / s.n_cells[2]) % s.n_cells[1];
    const int cx = local / (s.n_cells[2] * s.n_cells[1]);
    const int si[3] = {atom_shift[3 * g], atom_shift[3 * g + 1], atom_shift[3 * g + 2]};
    const double pi[3] = {positions[3 * g], positions[3 * g + 1], positions[3 * g + 2]};
    for (int dx = -s.n_search[0]; dx <= s.n_search[0]; dx++)
    for (int dy = -s.n_search[1]; dy <= s.n_search[1]; dy++)
    for (int dz = -s.n_search[2]; dz <= s.n_search[2]; dz++) {
        int cs[3], ni[3];
        divmod_i(cx + dx, s.n_cells[0], &cs[0], &ni[0]);
        divmod_i(cy + dy, s.n_cells[1], &cs[1], &ni[1]);
        divmod_i(cz + dz, s.n_cells[2], &cs[2], &ni[2]);
        const int32_t nc = (int32_t)(s.cell_offset + ((int64_t)ni[0] * s.n_cells[1] + ni[1]) * s.n_cells[2] + ni[2]);
        const int32_t start = cell_start[nc], count = cell_count[nc];
        for (int32_t q0 = 0; q0 < count; q0 += 32) {
            const int32_t q = q0 + lane;
            bool keep = false;
            int32_t j = -1;
            int sh[3] = {0, 0, 0};
            double v[3] = {0.0, 0.0, 0.0};
            double d2 = 0.0;
            if (q < count) {
                j = cell_atoms[start + q];
                keep = g <= j;
                for (int k = 0; k < 3; k++) sh[k] = cs[k] + si[k] - atom_shift[3 * (int64_t)j + k];
                const bool zero = sh[0] == 0 && sh[1] == 0 && sh[2] == 0;
                if (keep && g == j) {
                    // self images: one of each +/- shift pair (neighbors.rs:253-286)
                    const int sum = sh[0] + sh[1] + sh[2];
                    if (zero || sum < 0 || (sum == 0 && (sh[2] < 0 || (sh[2] == 0 && sh[1] < 0)))) keep = false;
                }
                if (s.infinite && !zero) keep = false;
                if (keep) {
                    for (int k = 0; k < 3; k++) {
                        // CellShift::cartesian, neighbors.rs:52-57
                        const double c = __dadd_rn(__dadd_rn(__dmul_rn(s.H[0 * 3 + k], (double)sh[0]),
                                                             __dmul_rn(s.H[1 * 3 + k], (double)sh[1])),
                                                   __dmul_rn(s.H[2 * 3 + k], (double)sh[2]));
                        v[k] = __dadd_rn(__dsub_rn(positions[3 * (int64_t)j + k], pi[k]), c);
                    }
                    d2 = __dadd_rn(__dadd_rn(__dmul_rn(v[0], v[0]), __dmul_rn(v[1], v[1])), __dmul_rn(v[2], v[2]));
                    keep = d2 < s.cutoff2;
                }
            }
            visit(keep, j, sh, v, d2);
        }
    }
}

__global__ void nl_count(const NlSystem* __restrict__ systems, const int32_t* __restrict__ atom_system,
                         const double* __restrict__ positions, int64_t n_atoms, const int32_t* __restrict__ cell_of,
                         const int32_t* __restrict__ atom_shift, const int32_t* __restrict__ cell_start,
                         const int32_t* __restrict__ cell_count, const int32_t* __restrict__ cell_atoms,
                         int64_t* __restrict__ pair_count) {
    const int64_t g = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (g >= n_atoms) return;
    const NlSystem& s = systems[atom_system[g]];
    int64_t count = 0;
    nl_warp_enumerate(s, g, positions, cell_of, atom_shift, cell_start, cell_count, cell_atoms, lane,
                      [&](bool keep, int32_t, const int*, const double*, double) {
                          count += __popc(__ballot_sync(0xffffffffu, keep));
                      });
    if (lane == 0) pair_count[g] = count;
}

__device__ __forceinline__ bool pair_key_less(int32_t j1, const int32_t* s1, int32_t j2, const int32_t* s2) {
    if (j1 != j2) return j1 < j2;
    for (int k = 0; k < 3; k++)
        if (s1[k] != s2[k]) return s1[k] < s2[k];
    return false;
}

// kept pairs of atom g in enumeration order into `scratch`, then every lane
// places its pairs at their rank in (second, shift) order
__global__ void nl_write(const NlSystem* __restrict__ systems, const int32_t* __restrict__ atom_system,
                         const double* __restrict__ positions, int64_t n_atoms, const int32_t* __restrict__ cell_of,
                         const int32_t* __restrict__ atom_shift, const int32_t* __restrict__ cell_start,
                         const int32_t* __restrict__ cell_count, const int32_t* __restrict__ cell_atoms,
                         const int64_t* __restrict__ pair_start, DevicePairs scratch, DevicePairs pairs) {
    const int64_t g = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (g >= n_atoms) return;
    const NlSystem& s = systems[atom_system[g]];
    const int64_t base = pair_start[g];
    int64_t written = 0;
    nl_warp_enumerate(s, g, positions, cell_of, atom_shift, cell_start, cell_count, cell_atoms, lane,
                      [&](bool keep, int32_t j, const int* sh, const double* v, double d2) {
                          const unsigned mask = __ballot_sync(0xffffffffu, keep);
                          if (keep) {
                              const int64_t w = base + written + __popc(mask & ((1u << lane) - 1u));
                              scratch.second[w] = j;
                              scratch.distance[w] = __dsqrt_rn(d2);
                              for (int k = 0; k < 3; k++) {
                                  scratch.vector[3 * w + k] = v[k];
                                  scratch.shift[3 * w + k] = sh[k];
                              }
                          }
                          written += __popc(mask);
                      });
    __syncwarp();
    for (int64_t a = lane; a < written; a += 32) {
        const int32_t j = scratch.second[base + a];
        const int32_t* sh = &scratch.shift[3 * (base + a)];
        int64_t rank = 0;
        for (int64_t b = 0; b < written; b++)
            if (pair_key_less(scratch.second[base + b], &scratch.shift[3 * (base + b)], j, sh)) rank++;
        const int64_t w = base + rank;
        pairs.first[w] = (int32_t)g;
        pairs.second[w] = j;
        pairs.distance[w] = scratch.distance[base + a];
        for (int k = 0; k < 3; k++) {
            pairs.vector[3 * w + k] = scratch.vector[3 * (base + a) + k];
            pairs.shift[3 * w + k] = sh[k];
        }
    }
}

}  // namespace

// Host-side cell-list parameters, CellList::new (neighbors.rs:101-163) and
// UnitCell (cell.rs:34-66, :154-169).  Compiled with FMA contraction off.
NlSystem make_nl_system(const double* cell, double cutoff, int64_t atom_offset, int64_t n_atoms, int64_t cell_offset);

int64_t NeighborBuilder::build(const std::vector<NlSystem>& systems, const std::vector<int32_t>& atom_system,
                               const double* d_positions, int64_t n_atoms, DeviceArena& arena, cudaStream_t stream) {
    int64_t n_systems = (int64_t)systems.size();
    int64_t n_cells = 0;
    for (auto& s : systems) n_cells = std::max<int64_t>(n_cells, s.cell_offset + (int64_t)s.n_cells[0] * s.n_cells[1] * s.n_cells[2]);
    if (n_cells >= (int64_t)INT32_MAX || n_atoms >= (int64_t)INT32_MAX) throw internal_error("too many atoms or cells for the neighbour list");

    NlSystem* d_sys = arena.alloc<NlSystem>("nl.systems", n_systems);
    int32_t* d_atom_system = arena.alloc<int32_t>("nl.atom_system", n_atoms);
    int32_t* d_cell_of = arena.alloc<int32_t>("nl.cell_of", n_atoms);
    int32_t* d_atom_shift = arena.alloc<int32_t>("nl.atom_shift", 3 * n_atoms);
    int32_t* d_cell_count = arena.alloc<int32_t>("nl.cell_count", n_cells + 1);
    int32_t* d_cell_start = arena.alloc<int32_t>("nl.cell_start", n_cells + 1);
    int32_t* d_cell_fill = arena.alloc<int32_t>("nl.cell_fill", n_cells + 1);
    int32_t* d_cell_atoms = arena.alloc<int32_t>("nl.cell_atoms", n_atoms);
    int64_t* d_pair_count = arena.alloc<int64_t>("nl.pair_count", n_atoms + 1);
    int64_t* d_pair_start = arena.alloc<int64_t>("nl.pair_start", n_atoms + 1);

    CUDA_CHECK(cudaMemcpyAsync(d_sys, systems.data(), sizeof(NlSystem) * n_systems, cudaMemcpyHostToDevice, stream));
    CUDA_CHECK(cudaMemcpyAsync(d_atom_system, atom_system.data(), sizeof(int32_t) * n_atoms, cudaMemcpyHostToDevice, stream));
    CUDA_CHECK(cudaMemsetAsync(d_cell_count, 0, sizeof(int32_t) * (n_cells + 1), stream));
    CUDA_CHECK(cudaMemsetAsync(d_cell_fill, 0, sizeof(int32_t) * (n_cells + 1), stream));
    CUDA_CHECK(cudaMemsetAsync(d_pair_count, 0, sizeof(int64_t) * (n_atoms + 1), stream));

    int threads = 128;
    int blocks = (int)((n_atoms + threads - 1) / threads);
    // one warp per atom for the pair search
    int warp_blocks = (int)((n_atoms * 32 + threads - 1) / threads);
    if (n_atoms > 0) {
        nl_assign_cells<<<blocks, threads, 0, stream>>>(d_sys, d_atom_system, d_positions, n_atoms, d_cell_of, d_atom_shift, d_cell_count);
        CUDA_CHECK(cudaGetLastError());
    }
    arena.exclusive_scan(d_cell_count, d_cell_start, n_cells + 1, stream);
    if (n_atoms > 0) {
        nl_fill_cells<<<blocks, threads, 0, stream>>>(d_cell_of, n_atoms, d_cell_start, d_cell_fill, d_cell_atoms);
        CUDA_CHECK(cudaGetLastError());
        nl_count<<<warp_blocks, threads, 0, stream>>>(d_sys, d_atom_system, d_positions, n_atoms, d_cell_of,
                                                      d_atom_shift, d_cell_start, d_cell_count, d_cell_atoms, d_pair_count);
        CUDA_CHECK(cudaGetLastError());
    }
    arena.exclusive_scan(d_pair_count, d_pair_start, n_atoms + 1, stream);
    pair_start = d_pair_start;
    int64_t total = 0;
    CUDA_CHECK(cudaMemcpyAsync(&total, d_pair_start + n_atoms, sizeof(int64_t), cudaMemcpyDeviceToHost, stream));
    CUDA_CHECK(cudaStreamSynchronize(stream));
    if (total >= (int64_t)INT32_MAX) throw internal_error("too many pairs for the neighbour list");

    pairs.first = arena.alloc<int32_t>("pairs.first", total);
    pairs.second = arena.alloc<int32_t>("pairs.second", total);
    pairs.distance = arena.alloc<double>("pairs.distance", total);
    pairs.vector = arena.alloc<double>("pairs.vector", 3 * total);
    pairs.shift = arena.alloc<int32_t>("pairs.shift", 3 * total);
    pairs.count = total;
    DevicePairs scratch;
    scratch.second = arena.alloc<int32_t>("nl.scratch.second", total);
    scratch.distance = arena.alloc<double>("nl.scratch.distance", total);
    scratch.vector = arena.alloc<double>("nl.scratch.vector", 3 * total);
    scratch.shift = arena.alloc<int32_t>("nl.scratch.shift", 3 * total);
    scratch.count = total;
    if (n_atoms > 0 && total > 0) {
        nl_write<<<warp_blocks, threads, 0, stream>>>(d_sys, d_atom_system, d_positions, n_atoms, d_cell_of,
                                                      d_atom_shift, d_cell_start, d_cell_count, d_cell_atoms,
                                                      d_pair_start, scratch, pairs);
        CUDA_CHECK(cudaGetLastError());
    }
    return total;
}

std::vector<Pair> neighbor_list(const double* positions, int64_t n_atoms, const double* cell, double cutoff) {
    DeviceArena arena;
    NeighborBuilder nb;
    cudaStream_t stream = nullptr;
    std::vector<NlSystem> systems = {make_nl_system(cell, cutoff, 0, n_atoms, 0)};
    std::vector<int32_t> atom_system(n_atoms, 0);
    double* d_pos = arena.alloc<double>("positions", 3 * n_atoms);
    if (n_atoms) CUDA_CHECK(cudaMemcpy(d_pos, positions, sizeof(double) * 3 * n_atoms, cudaMemcpyHostToDevice));
    int64_t n = nb.build(systems, atom_system, d_pos, n_atoms, arena, stream);
    std::vector<int32_t> first(n), second(n), shift(3 * n);
    std::vector<double> dist(n), vec(3 * n);
    if (n) {
        CUDA_CHECK(cudaMemcpy(first.data(), nb.pairs.first, 4 * n, cudaMemcpyDeviceToHost));
        CUDA_CHECK(cudaMemcpy(second.data(), nb.pairs.second, 4 * n, cudaMemcpyDeviceToHost));
        CUDA_CHECK(cudaMemcpy(shift.data(), nb.pairs.shift, 12 * n, cudaMemcpyDeviceToHost));
        CUDA_CHECK(cudaMemcpy(dist.data(), nb.pairs.distance, 8 * n, cudaMemcpyDeviceToHost));
        CUDA_CHECK(cudaMemcpy(vec.data(), nb.pairs.vector, 24 * n, cudaMemcpyDeviceToHost));
    }
    std::vector<Pair> out(n);
    for (int64_t k = 0; k < n; k++) {
        out[k].first = (uint64_t)first[k];
        out[k].second = (uint64_t)second[k];
        out[k].distance = dist[k];
        for (int x = 0; x < 3; x++) {
            out[k].vector[x] = vec[3 * k + x];
            out[k].shift[x] = shift[3 * k + x];
        }
    }
    return out;
}

// ---------------------------------------------------------------------------
// The same neighbour list without any device allocation
// ---------------------------------------------------------------------------
//
// Every table of the cell list lives in one fixed array in device memory
// (defined below, about 3.7 MB per device), so the call never asks the CUDA
// runtime or any allocator for memory.  The caller owns the positions and the
// output pairs.  The atom and cell kernels are the ones above; the scans are a
// single-block kernel instead of CUB (which needs allocated temporary storage)
// and the pairs are sorted per atom in shared memory and written straight into
// the caller's featomic_pair_t array.

namespace {

constexpr int64_t NOALLOC_MAX_ATOMS = 65536;
// featomic caps the number of cells of one cell list at 1e5
// (CellList::new, neighbors.rs:128-139); make_nl_system does the same
constexpr int64_t NOALLOC_MAX_CELLS = 100000;
// pairs of one atom in the half list (j >= i), sorted in shared memory
constexpr int NOALLOC_MAX_PAIRS_PER_ATOM = 2048;

constexpr size_t align256(size_t x) { return (x + 255) / 256 * 256; }

// byte offsets of the tables inside the scratch array
constexpr size_t NOALLOC_SYSTEM = 0;
constexpr size_t NOALLOC_ATOM_SYSTEM = align256(NOALLOC_SYSTEM + sizeof(NlSystem));
constexpr size_t NOALLOC_CELL_OF = align256(NOALLOC_ATOM_SYSTEM + 4 * NOALLOC_MAX_ATOMS);
constexpr size_t NOALLOC_ATOM_SHIFT = align256(NOALLOC_CELL_OF + 4 * NOALLOC_MAX_ATOMS);
constexpr size_t NOALLOC_CELL_ATOMS = align256(NOALLOC_ATOM_SHIFT + 12 * NOALLOC_MAX_ATOMS);
constexpr size_t NOALLOC_CELL_COUNT = align256(NOALLOC_CELL_ATOMS + 4 * NOALLOC_MAX_ATOMS);
constexpr size_t NOALLOC_CELL_START = align256(NOALLOC_CELL_COUNT + 4 * (NOALLOC_MAX_CELLS + 1));
constexpr size_t NOALLOC_CELL_FILL = align256(NOALLOC_CELL_START + 4 * (NOALLOC_MAX_CELLS + 1));
constexpr size_t NOALLOC_PAIR_COUNT = align256(NOALLOC_CELL_FILL + 4 * (NOALLOC_MAX_CELLS + 1));
constexpr size_t NOALLOC_PAIR_START = align256(NOALLOC_PAIR_COUNT + 8 * (NOALLOC_MAX_ATOMS + 1));
constexpr size_t NOALLOC_OVERFLOW = align256(NOALLOC_PAIR_START + 8 * (NOALLOC_MAX_ATOMS + 1));
constexpr size_t NOALLOC_BYTES = align256(NOALLOC_OVERFLOW + 8);

}  // namespace

// One copy per device, shared by every call on that device
static __device__ __align__(256) unsigned char nl_noalloc_scratch[NOALLOC_BYTES];

namespace {

__global__ void nl_noalloc_store_system(NlSystem system, NlSystem* __restrict__ out) { *out = system; }

// Exclusive scan of `n` counts into out[0..n] (out[n] = total) by one block of
// 1024 threads, each over a contiguous chunk.  Counts above `limit` (when
// limit >= 0) set *over.
template <typename T>
__global__ void __launch_bounds__(1024) nl_noalloc_scan(const T* __restrict__ in, T* __restrict__ out, int64_t n,
                                                        int64_t limit, int32_t* __restrict__ over) {
    __shared__ T warp_total[32];
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const int64_t chunk = (n + blockDim.x - 1) / blockDim.x;
    const int64_t lo = (int64_t)t * chunk < n ? (int64_t)t * chunk : n;
    const int64_t hi = lo + chunk < n ? lo + chunk : n;
    T local = 0;
    for (int64_t i = lo; i < hi; i++) {
        const T c = in[i];
        if (limit >= 0 && (int64_t)c > limit) atomicOr(over, 1);
        local += c;
    }
    T incl = local;
    for (int off = 1; off < 32; off <<= 1) {
        const T y = __shfl_up_sync(0xffffffffu, incl, off);
        if (lane >= off) incl += y;
    }
    if (lane == 31) warp_total[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        T w = lane < (int)(blockDim.x >> 5) ? warp_total[lane] : T(0);
        for (int off = 1; off < 32; off <<= 1) {
            const T y = __shfl_up_sync(0xffffffffu, w, off);
            if (lane >= off) w += y;
        }
        warp_total[lane] = w;
    }
    __syncthreads();
    T prefix = incl - local + (warp > 0 ? warp_total[warp - 1] : T(0));
    for (int64_t i = lo; i < hi; i++) {
        out[i] = prefix;
        prefix += in[i];
    }
    if (t == (int)blockDim.x - 1) out[n] = prefix;
}

// One warp (one block) per atom.  First pass: the keys (second, shift) of the
// atom's kept pairs go to shared memory in enumeration order.  Second pass:
// the same enumeration again, every kept pair written at base + its rank among
// the keys, which is featomic's (first, second, shift) order.
__global__ void __launch_bounds__(32) nl_noalloc_write(
    const NlSystem* __restrict__ systems, const int32_t* __restrict__ atom_system, const double* __restrict__ positions,
    int64_t n_atoms, const int32_t* __restrict__ cell_of, const int32_t* __restrict__ atom_shift,
    const int32_t* __restrict__ cell_start, const int32_t* __restrict__ cell_count,
    const int32_t* __restrict__ cell_atoms, const int64_t* __restrict__ pair_start, featomic_pair_t* __restrict__ out,
    int64_t capacity) {
    __shared__ int32_t key_second[NOALLOC_MAX_PAIRS_PER_ATOM];
    __shared__ int32_t key_shift[3 * NOALLOC_MAX_PAIRS_PER_ATOM];
    const int64_t g = blockIdx.x;
    const int lane = threadIdx.x & 31;
    if (g >= n_atoms) return;
    const int64_t base = pair_start[g];
    const int64_t n = pair_start[g + 1] - base;
    // both are rejected on the host before this kernel is launched
    if (n > NOALLOC_MAX_PAIRS_PER_ATOM || base + n > capacity) return;
    const NlSystem& s = systems[atom_system[g]];
    int64_t written = 0;
    nl_warp_enumerate(s, g, positions, cell_of, atom_shift, cell_start, cell_count, cell_atoms, lane,
                      [&](bool keep, int32_t j, const int* sh, const double*, double) {
                          const unsigned mask = __ballot_sync(0xffffffffu, keep);
                          if (keep) {
                              const int64_t w = written + __popc(mask & ((1u << lane) - 1u));
                              if (w < n) {
                                  key_second[w] = j;
                                  for (int k = 0; k < 3; k++) key_shift[3 * w + k] = sh[k];
                              }
                          }
                          written += __popc(mask);
                      });
    __syncwarp();
    nl_warp_enumerate(s, g, positions, cell_of, atom_shift, cell_start, cell_count, cell_atoms, lane,
                      [&](bool keep, int32_t j, const int* sh, const double* v, double d2) {
                          if (!keep) return;
                          int64_t rank = 0;
                          for (int64_t b = 0; b < n; b++)
                              if (pair_key_less(key_second[b], &key_shift[3 * b], j, sh)) rank++;
                          if (rank >= n) return;
                          featomic_pair_t* p = out + base + rank;
                          p->first = (uintptr_t)g;
                          p->second = (uintptr_t)j;
                          p->distance = __dsqrt_rn(d2);
                          for (int k = 0; k < 3; k++) {
                              p->vector[k] = v[k];
                              p->cell_shift_indices[k] = sh[k];
                          }
                      });
}

std::mutex noalloc_setup_mutex;
constexpr int NOALLOC_MAX_DEVICES = 64;
unsigned char* noalloc_scratch_address[NOALLOC_MAX_DEVICES] = {};

// Set-up, once per device: the address of this device's copy of the scratch
// array, looked up with that device current.
unsigned char* noalloc_scratch_for_current_device() {
    int device = -1;
    CUDA_CHECK(cudaGetDevice(&device));
    if (device < 0 || device >= NOALLOC_MAX_DEVICES) throw internal_error("unsupported CUDA device index");
    std::lock_guard<std::mutex> lock(noalloc_setup_mutex);
    if (noalloc_scratch_address[device] == nullptr) {
        void* address = nullptr;
        cudaError_t status = cudaGetSymbolAddress(&address, nl_noalloc_scratch);
        if (status != cudaSuccess || address == nullptr) {
            throw internal_error(std::string("could not find the neighbour-list scratch array on device ") +
                                 std::to_string(device) + ": " + cudaGetErrorString(status));
        }
        noalloc_scratch_address[device] = static_cast<unsigned char*>(address);
    }
    return noalloc_scratch_address[device];
}

void check_device_buffer(const void* ptr, size_t alignment, const char* what) {
    cudaPointerAttributes attributes;
    CUDA_CHECK(cudaPointerGetAttributes(&attributes, ptr));
    int device = -1;
    CUDA_CHECK(cudaGetDevice(&device));
    const bool on_device = attributes.type == cudaMemoryTypeDevice || attributes.type == cudaMemoryTypeManaged;
    if (!on_device || (attributes.type == cudaMemoryTypeDevice && attributes.device != device)) {
        throw invalid_parameter(std::string(what) + " must be device memory of the current CUDA device");
    }
    if (reinterpret_cast<uintptr_t>(ptr) % alignment != 0) {
        throw invalid_parameter(std::string(what) + " must be aligned to " + std::to_string(alignment) + " bytes");
    }
}

}  // namespace

void neighbor_list_noalloc(const double* positions, int64_t n_atoms, const double* cell, double cutoff,
                           featomic_pair_t* pairs, int64_t capacity, uintptr_t* count, void* stream_ptr) {
    cudaStream_t stream = static_cast<cudaStream_t>(stream_ptr);
    if (n_atoms > NOALLOC_MAX_ATOMS) {
        throw invalid_parameter("featomic_b200_neighbor_list_noalloc handles at most " +
                                std::to_string(NOALLOC_MAX_ATOMS) + " atoms, got " + std::to_string(n_atoms));
    }
    const NlSystem system = make_nl_system(cell, cutoff, 0, n_atoms, 0);
    const int64_t n_cells = (int64_t)system.n_cells[0] * system.n_cells[1] * system.n_cells[2];
    if (n_cells < 1 || n_cells > NOALLOC_MAX_CELLS) {
        throw invalid_parameter("featomic_b200_neighbor_list_noalloc handles at most " +
                                std::to_string(NOALLOC_MAX_CELLS) + " cells, got " + std::to_string(n_cells));
    }
    unsigned char* scratch = noalloc_scratch_for_current_device();
    *count = 0;
    if (n_atoms == 0) return;
    check_device_buffer(positions, alignof(double), "positions");

    NlSystem* d_system = reinterpret_cast<NlSystem*>(scratch + NOALLOC_SYSTEM);
    int32_t* d_atom_system = reinterpret_cast<int32_t*>(scratch + NOALLOC_ATOM_SYSTEM);
    int32_t* d_cell_of = reinterpret_cast<int32_t*>(scratch + NOALLOC_CELL_OF);
    int32_t* d_atom_shift = reinterpret_cast<int32_t*>(scratch + NOALLOC_ATOM_SHIFT);
    int32_t* d_cell_atoms = reinterpret_cast<int32_t*>(scratch + NOALLOC_CELL_ATOMS);
    int32_t* d_cell_count = reinterpret_cast<int32_t*>(scratch + NOALLOC_CELL_COUNT);
    int32_t* d_cell_start = reinterpret_cast<int32_t*>(scratch + NOALLOC_CELL_START);
    int32_t* d_cell_fill = reinterpret_cast<int32_t*>(scratch + NOALLOC_CELL_FILL);
    int64_t* d_pair_count = reinterpret_cast<int64_t*>(scratch + NOALLOC_PAIR_COUNT);
    int64_t* d_pair_start = reinterpret_cast<int64_t*>(scratch + NOALLOC_PAIR_START);
    int32_t* d_overflow = reinterpret_cast<int32_t*>(scratch + NOALLOC_OVERFLOW);

    // must start at zero: the system index of every atom (one system), the two
    // per-cell atomic counters and the per-atom overflow flag
    CUDA_CHECK(cudaMemsetAsync(d_atom_system, 0, sizeof(int32_t) * n_atoms, stream));
    CUDA_CHECK(cudaMemsetAsync(d_cell_count, 0, sizeof(int32_t) * (n_cells + 1), stream));
    CUDA_CHECK(cudaMemsetAsync(d_cell_fill, 0, sizeof(int32_t) * (n_cells + 1), stream));
    CUDA_CHECK(cudaMemsetAsync(d_overflow, 0, sizeof(int32_t), stream));

    const int threads = 128;
    const int blocks = (int)((n_atoms + threads - 1) / threads);
    const int warp_blocks = (int)((n_atoms * 32 + threads - 1) / threads);
    nl_noalloc_store_system<<<1, 1, 0, stream>>>(system, d_system);
    CUDA_CHECK(cudaGetLastError());
    nl_assign_cells<<<blocks, threads, 0, stream>>>(d_system, d_atom_system, positions, n_atoms, d_cell_of,
                                                    d_atom_shift, d_cell_count);
    CUDA_CHECK(cudaGetLastError());
    nl_noalloc_scan<int32_t><<<1, 1024, 0, stream>>>(d_cell_count, d_cell_start, n_cells, -1, nullptr);
    CUDA_CHECK(cudaGetLastError());
    nl_fill_cells<<<blocks, threads, 0, stream>>>(d_cell_of, n_atoms, d_cell_start, d_cell_fill, d_cell_atoms);
    CUDA_CHECK(cudaGetLastError());
    nl_count<<<warp_blocks, threads, 0, stream>>>(d_system, d_atom_system, positions, n_atoms, d_cell_of, d_atom_shift,
                                                  d_cell_start, d_cell_count, d_cell_atoms, d_pair_count);
    CUDA_CHECK(cudaGetLastError());
    nl_noalloc_scan<int64_t><<<1, 1024, 0, stream>>>(d_pair_count, d_pair_start, n_atoms, NOALLOC_MAX_PAIRS_PER_ATOM,
                                                     d_overflow);
    CUDA_CHECK(cudaGetLastError());

    int64_t total = 0;
    int32_t overflow = 0;
    CUDA_CHECK(cudaMemcpyAsync(&total, d_pair_start + n_atoms, sizeof(int64_t), cudaMemcpyDeviceToHost, stream));
    CUDA_CHECK(cudaMemcpyAsync(&overflow, d_overflow, sizeof(int32_t), cudaMemcpyDeviceToHost, stream));
    CUDA_CHECK(cudaStreamSynchronize(stream));
    if (overflow != 0) {
        throw invalid_parameter("featomic_b200_neighbor_list_noalloc handles at most " +
                                std::to_string(NOALLOC_MAX_PAIRS_PER_ATOM) +
                                " pairs per atom in the half list; use a smaller cutoff or featomic_b200_neighbor_list");
    }
    *count = (uintptr_t)total;
    if (total > capacity) {
        throw Error(STATUS_BUFFER_SIZE_ERROR, "pair buffer is too small: got space for " + std::to_string(capacity) +
                                                  " pairs, need " + std::to_string(total));
    }
    if (total == 0) return;
    check_device_buffer(pairs, alignof(featomic_pair_t), "pairs");
    nl_noalloc_write<<<(unsigned)n_atoms, 32, 0, stream>>>(d_system, d_atom_system, positions, n_atoms, d_cell_of,
                                                          d_atom_shift, d_cell_start, d_cell_count, d_cell_atoms,
                                                          d_pair_start, pairs, capacity);
    CUDA_CHECK(cudaGetLastError());
}

}  // namespace fb200

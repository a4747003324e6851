// Compute pipeline of one calculator on the GPU:
//
//   positions (H2D, or already resident)
//     -> kernel (a) neighbour list            [neighbors.cu]
//     -> D2H of the pair indices, host metadata (keys, samples, gradient
//        samples, direction segments)         [plan.cpp]
//     -> kernel (b) pair features + per-centre accumulation  [expansion.cu]
//     -> kernel (c) power spectrum rows, or the spherical expansion blocks
//                                            [power_spectrum.cu, expansion.cu]
//     -> output TensorMap on the device, or D2H into pinned host memory
#include <cub/cub.cuh>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>

#include "dense.hpp"
#include "engine.hpp"
#include "plan.hpp"

namespace fb200 {

// ---------------------------------------------------------------------------
// DeviceArena
// ---------------------------------------------------------------------------
DeviceArena::~DeviceArena() { release(); }

void DeviceArena::release() {
    for (auto& kv : buffers_)
        if (kv.second.ptr) cudaFree(kv.second.ptr);
    buffers_.clear();
}

void* DeviceArena::alloc_bytes(const std::string& name, size_t bytes) {
    auto& b = buffers_[name];
    if (b.bytes >= bytes && b.ptr) return b.ptr;
    if (b.ptr) {
        // the previous buffer may still be read by queued work
        CUDA_CHECK(cudaDeviceSynchronize());
        CUDA_CHECK(cudaFree(b.ptr));
        b.ptr = nullptr;
    }
    size_t grow = std::max(bytes, b.bytes + b.bytes / 4);
    grow = (grow + 255) / 256 * 256;
    CUDA_CHECK(cudaMalloc(&b.ptr, grow));
    b.bytes = grow;
    return b.ptr;
}

size_t DeviceArena::bytes_reserved() const {
    size_t s = 0;
    for (auto& kv : buffers_) s += kv.second.bytes;
    return s;
}

void DeviceArena::exclusive_scan(const int32_t* in, int32_t* out, int64_t n, cudaStream_t stream) {
    size_t temp = 0;
    CUDA_CHECK(cub::DeviceScan::ExclusiveSum(nullptr, temp, in, out, (int)n, stream));
    void* t = alloc_bytes("scan.temp", temp);
    CUDA_CHECK(cub::DeviceScan::ExclusiveSum(t, temp, in, out, (int)n, stream));
}

void DeviceArena::exclusive_scan(const int64_t* in, int64_t* out, int64_t n, cudaStream_t stream) {
    size_t temp = 0;
    CUDA_CHECK(cub::DeviceScan::ExclusiveSum(nullptr, temp, in, out, (int)n, stream));
    void* t = alloc_bytes("scan.temp", temp);
    CUDA_CHECK(cub::DeviceScan::ExclusiveSum(t, temp, in, out, (int)n, stream));
}

// ---------------------------------------------------------------------------
// Cell-list parameters (neighbors.rs:101-163, cell.rs:34-66 and :154-169,
// matrix.rs:210-247).  This translation unit is compiled with
// -ffp-contract=off so that the host arithmetic keeps the reference order.
// ---------------------------------------------------------------------------
namespace {

double det3(const double* m) {
    return m[0] * (m[4] * m[8] - m[7] * m[5]) - m[1] * (m[3] * m[8] - m[5] * m[6]) + m[2] * (m[3] * m[7] - m[4] * m[6]);
}

void cross3(const double* a, const double* b, double* r) {
    r[0] = a[1] * b[2] - a[2] * b[1];
    r[1] = a[2] * b[0] - a[0] * b[2];
    r[2] = a[0] * b[1] - a[1] * b[0];
}

double dot3(const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

}  // namespace

NlSystem make_nl_system(const double* cell, double cutoff, int64_t atom_offset, int64_t n_atoms, int64_t cell_offset) {
    NlSystem s;
    std::memset(&s, 0, sizeof(s));
    s.atom_offset = atom_offset;
    s.cell_offset = cell_offset;
    s.n_atoms = (int32_t)n_atoms;
    s.cutoff2 = cutoff * cutoff;
    bool zero = true;
    for (int k = 0; k < 9; k++) {
        s.H[k] = cell[k];
        if (cell[k] != 0.0) zero = false;
    }
    s.infinite = zero ? 1 : 0;
    double dbf[3] = {1.0, 1.0, 1.0};
    if (!zero) {
        double det = det3(cell);
        if (!(std::fabs(det) > 1e-6)) throw invalid_parameter("the unit cell matrix is not invertible");
        double id = 1.0 / det;
        const double* m = cell;
        s.inv[0] = (m[4] * m[8] - m[7] * m[5]) * id;
        s.inv[1] = (m[2] * m[7] - m[1] * m[8]) * id;
        s.inv[2] = (m[1] * m[5] - m[2] * m[4]) * id;
        s.inv[3] = (m[5] * m[6] - m[3] * m[8]) * id;
        s.inv[4] = (m[0] * m[8] - m[2] * m[6]) * id;
        s.inv[5] = (m[3] * m[2] - m[0] * m[5]) * id;
        s.inv[6] = (m[3] * m[7] - m[6] * m[4]) * id;
        s.inv[7] = (m[6] * m[1] - m[0] * m[7]) * id;
        s.inv[8] = (m[0] * m[4] - m[3] * m[1]) * id;
        const double* a = &cell[0];
        const double* b = &cell[3];
        const double* c = &cell[6];
        double na[3], nb[3], nc[3];
        cross3(b, c, na);
        cross3(c, a, nb);
        cross3(a, b, nc);
        double la = std::sqrt(dot3(na, na)), lb = std::sqrt(dot3(nb, nb)), lc = std::sqrt(dot3(nc, nc));
        for (int k = 0; k < 3; k++) {
            na[k] = na[k] / la;
            nb[k] = nb[k] / lb;
            nc[k] = nc[k] / lc;
        }
        dbf[0] = std::fabs(dot3(na, a));
        dbf[1] = std::fabs(dot3(nb, b));
        dbf[2] = std::fabs(dot3(nc, c));
    }
    double nf[3];
    for (int k = 0; k < 3; k++) {
        double v = std::trunc(dbf[k] / cutoff);
        nf[k] = v < 1.0 ? 1.0 : v;
    }
    double total = nf[0] * nf[1] * nf[2];
    if (total > 1e5) {
        double rxy = nf[0] / nf[1];
        double ryz = nf[1] / nf[2];
        nf[2] = std::trunc(std::cbrt(1e5 / (rxy * ryz * ryz)));
        nf[1] = std::trunc(ryz * nf[2]);
        nf[0] = std::trunc(rxy * nf[1]);
    }
    for (int k = 0; k < 3; k++) {
        s.n_search[k] = (int32_t)std::ceil(cutoff * nf[k] / dbf[k]);
        s.n_cells[k] = (int32_t)nf[k];
        if (s.n_search[k] < 1) s.n_search[k] = 1;
        if (s.n_cells[k] == 1 && s.infinite) s.n_search[k] = 0;
    }
    return s;
}

// ---------------------------------------------------------------------------
// pinned host memory for outputs, recycled across calls
// ---------------------------------------------------------------------------
namespace {

struct PinnedPool {
    std::mutex mutex;
    std::vector<std::pair<void*, size_t>> free_list;
    size_t cached = 0;

    // returns the buffer and its real size (a recycled buffer can be larger)
    void* get(size_t bytes, size_t* actual) {
        {
            std::lock_guard<std::mutex> lock(mutex);
            size_t best = (size_t)-1;
            for (size_t k = 0; k < free_list.size(); k++)
                if (free_list[k].second >= bytes && (best == (size_t)-1 || free_list[k].second < free_list[best].second)) best = k;
            if (best != (size_t)-1) {
                void* p = free_list[best].first;
                *actual = free_list[best].second;
                cached -= free_list[best].second;
                free_list.erase(free_list.begin() + best);
                return p;
            }
        }
        void* p = nullptr;
        *actual = bytes;
        if (cudaHostAlloc(&p, bytes, cudaHostAllocDefault) != cudaSuccess) {
            cudaGetLastError();
            p = std::malloc(bytes);
            if (!p) throw internal_error("out of host memory");
            return p;  // plain memory, freed with free()
        }
        return p;
    }

    void put(void* p, size_t bytes, bool pinned) {
        if (!pinned) {
            std::free(p);
            return;
        }
        std::lock_guard<std::mutex> lock(mutex);
        free_list.emplace_back(p, bytes);
        cached += bytes;
        // keep at most 4 buffers
        while (free_list.size() > 4) {
            cudaFreeHost(free_list.front().first);
            cached -= free_list.front().second;
            free_list.erase(free_list.begin());
        }
    }
};

PinnedPool& pinned_pool() {
    static PinnedPool* pool = new PinnedPool();  // never destroyed: buffers may outlive static destruction
    return *pool;
}

bool is_pinned(void* p) {
    cudaPointerAttributes attr;
    if (cudaPointerGetAttributes(&attr, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return attr.type == cudaMemoryTypeHost;
}

template <typename T>
T* upload(DeviceArena& arena, const std::string& name, const std::vector<T>& host, cudaStream_t stream) {
    T* d = arena.alloc<T>(name, (int64_t)host.size());
    if (!host.empty()) CUDA_CHECK(cudaMemcpyAsync(d, host.data(), sizeof(T) * host.size(), cudaMemcpyHostToDevice, stream));
    return d;
}

// A non-blocking stream per device for the metadata work beside the
// spherical-expansion kernel (neighbourhood tables, uploads).  It has the
// highest priority: its small kernels take SMs as soon as blocks of the
// expansion retire instead of waiting for the whole grid.
cudaStream_t copy_stream() {
    static std::mutex mutex;
    static std::map<int, cudaStream_t> streams;
    int device = 0;
    CUDA_CHECK(cudaGetDevice(&device));
    std::lock_guard<std::mutex> lock(mutex);
    auto it = streams.find(device);
    if (it != streams.end()) return it->second;
    cudaStream_t s = nullptr;
    int least = 0, greatest = 0;
    CUDA_CHECK(cudaDeviceGetStreamPriorityRange(&least, &greatest));
    CUDA_CHECK(cudaStreamCreateWithPriority(&s, cudaStreamNonBlocking, greatest));
    streams[device] = s;
    return s;
}

// a stream per device for device-to-host copies that nothing on the device
// waits for
cudaStream_t readback_stream() {
    static std::mutex mutex;
    static std::map<int, cudaStream_t> streams;
    int device = 0;
    CUDA_CHECK(cudaGetDevice(&device));
    std::lock_guard<std::mutex> lock(mutex);
    auto it = streams.find(device);
    if (it != streams.end()) return it->second;
    cudaStream_t s = nullptr;
    CUDA_CHECK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    streams[device] = s;
    return s;
}

// makes `stream` wait for the uploads issued on the copy stream so far
void join_uploads(cudaStream_t stream) {
    cudaEvent_t done = nullptr;
    CUDA_CHECK(cudaEventCreateWithFlags(&done, cudaEventDisableTiming));
    CUDA_CHECK(cudaEventRecord(done, copy_stream()));
    CUDA_CHECK(cudaStreamWaitEvent(stream, done, 0));
    CUDA_CHECK(cudaEventDestroy(done));  // released once the recorded work has completed
}

double elapsed_ms(cudaEvent_t a, cudaEvent_t b) {
    float ms = 0.0f;
    if (cudaEventElapsedTime(&ms, a, b) != cudaSuccess) {
        cudaGetLastError();  // an event of a phase that did not run: not an error of the call
        return 0.0;
    }
    return (double)ms;
}

Labels xyz_labels(const char* name) {
    Labels l;
    l.names = {name};
    l.values = {0, 1, 2};
    return l;
}

}  // namespace

// ---------------------------------------------------------------------------
// Engine
// ---------------------------------------------------------------------------
Engine::Engine(const Hypers& h) : h_(h) {
    radial_ = build_radial_tables(h);
    ylm_ = build_ylm_tables(h.max_angular);
}

Engine::~Engine() {
    for (void* p : table_buffers_) cudaFree(p);
    if (staging_) cudaFreeHost(staging_);
    if (dense_marks_ready_)
        for (auto& e : dense_marks_) cudaEventDestroy(e);
}

void* Engine::staging(size_t bytes) {
    if (bytes > staging_bytes_) {
        if (staging_) CUDA_CHECK(cudaFreeHost(staging_));
        staging_ = nullptr;
        staging_bytes_ = 0;
        CUDA_CHECK(cudaHostAlloc(&staging_, bytes, cudaHostAllocDefault));
        staging_bytes_ = bytes;
    }
    return staging_;
}

cudaEvent_t* Engine::dense_marks() {
    if (!dense_marks_ready_) {
        for (auto& e : dense_marks_) CUDA_CHECK(cudaEventCreate(&e));
        dense_marks_ready_ = true;
    }
    return dense_marks_;
}

std::vector<double> Engine::dense_times() {
    std::vector<double> t(6, 0.0);
    if (!dense_marks_ready_) return t;
    // the last marks of the forward and backward passes
    if (cudaEventSynchronize(dense_marks_[3]) != cudaSuccess || cudaEventSynchronize(dense_marks_[7]) != cudaSuccess) {
        cudaGetLastError();  // a pass that never ran: no times
        return t;
    }
    for (int k = 0; k < 3; k++) t[k] = elapsed_ms(dense_marks_[k], dense_marks_[k + 1]);
    for (int k = 0; k < 3; k++) t[3 + k] = elapsed_ms(dense_marks_[4 + k], dense_marks_[5 + k]);
    return t;
}

void Engine::upload_tables() {
    int dev = 0;
    CUDA_CHECK(cudaGetDevice(&dev));
    if (tables_ready_ && dev == device_) return;
    if (tables_ready_) throw invalid_parameter("a calculator can only be used on the device it first ran on");
    device_ = dev;
    // keep the memory of freed device TensorMaps in the default pool
    cudaMemPool_t pool;
    CUDA_CHECK(cudaDeviceGetDefaultMemPool(&pool, dev));
    uint64_t threshold = UINT64_MAX;
    CUDA_CHECK(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &threshold));
    auto put = [&](const void* src, size_t bytes) -> void* {
        void* d = nullptr;
        CUDA_CHECK(cudaMalloc(&d, bytes > 0 ? bytes : 8));
        if (bytes) CUDA_CHECK(cudaMemcpy(d, src, bytes, cudaMemcpyHostToDevice));
        table_buffers_.push_back(d);
        return d;
    };
    auto putv = [&](const std::vector<double>& v) { return (const double*)put(v.data(), v.size() * sizeof(double)); };
    d_radial_.lmax = radial_.lmax;
    d_radial_.nmax = radial_.nmax;
    d_radial_.splined = radial_.splined ? 1 : 0;
    d_radial_.knot_offset = (const int32_t*)put(radial_.knot_offset.data(), radial_.knot_offset.size() * 4);
    d_radial_.knot_count = (const int32_t*)put(radial_.knot_count.data(), radial_.knot_count.size() * 4);
    d_radial_.positions = putv(radial_.positions);
    d_radial_.values = putv(radial_.values);
    d_radial_.derivs = putv(radial_.derivs);
    d_radial_.c = radial_.c;
    d_radial_.width2 = radial_.width2;
    d_radial_.bn = putv(radial_.bn);
    d_radial_.ortho = putv(radial_.ortho);
    d_ylm_.lmax = ylm_.lmax;
    d_ylm_.A = putv(ylm_.A);
    d_ylm_.B = putv(ylm_.B);
    d_ylm_.sq_plus = putv(ylm_.sq_plus);
    d_ylm_.sq_minus = putv(ylm_.sq_minus);
    d_ylm_.sq_2l1 = putv(ylm_.sq_2l1);
    d_ylm_.sq_half = putv(ylm_.sq_half);
    d_ylm_.sq_ll1 = putv(ylm_.sq_ll1);
    d_ylm_.inv_ll = putv(ylm_.inv_ll);
    d_self_ = (double*)putv(radial_.self_contribution);

    // the same tables for the dense kernels, in FP64 and rounded to FP32
    auto putf = [&](const std::vector<double>& v) {
        std::vector<float> f(v.begin(), v.end());
        return (const float*)put(f.data(), f.size() * sizeof(float));
    };
    dense_d_.ylm = d_ylm_;
    dense_d_.spline = {d_radial_.lmax, d_radial_.nmax, d_radial_.splined, d_radial_.knot_offset,
                       d_radial_.knot_count, d_radial_.positions, d_radial_.values, d_radial_.derivs};
    dense_d_.self_contribution = d_self_;
    dense_f_.ylm = {ylm_.lmax,          putf(ylm_.A),      putf(ylm_.B),       putf(ylm_.sq_plus), putf(ylm_.sq_minus),
                    putf(ylm_.sq_2l1), putf(ylm_.sq_half), putf(ylm_.sq_ll1), putf(ylm_.inv_ll)};
    dense_f_.spline = {d_radial_.lmax,        d_radial_.nmax,       d_radial_.splined,    d_radial_.knot_offset,
                       d_radial_.knot_count,  d_radial_.positions, putf(radial_.values), putf(radial_.derivs)};
    dense_f_.self_contribution = putf(radial_.self_contribution);
    tables_ready_ = true;
}

std::unique_ptr<TensorMap> Engine::compute(int kind, std::vector<HostSystem>& systems, const GradientOptions& g,
                                           bool device_output, const double* d_positions_in, cudaStream_t stream) {
    auto t_start = std::chrono::steady_clock::now();
    const bool ps = kind == OUTPUT_POWER_SPECTRUM, by_pair = kind == OUTPUT_BY_PAIR;
    upload_tables();
    cudaEvent_t ev[16];
    for (auto& e : ev) CUDA_CHECK(cudaEventCreate(&e));
    struct EventGuard {
        cudaEvent_t* e;
        ~EventGuard() {
            for (int k = 0; k < 16; k++) cudaEventDestroy(e[k]);
        }
    } guard{ev};
    CUDA_CHECK(cudaEventRecord(ev[0], stream));

    // ---- gather atoms -------------------------------------------------------
    int64_t n_atoms = 0;
    bool user_pairs = false, native_pairs = false;
    for (auto& s : systems) {
        n_atoms += s.n_atoms;
        if (s.has_pairs) user_pairs = true;
        else native_pairs = true;
    }
    if (user_pairs && native_pairs) throw internal_error("mixing systems with and without neighbour lists");
    if (n_atoms >= (int64_t)INT32_MAX / 2) throw invalid_parameter("too many atoms");
    std::vector<int32_t> atom_system;
    atom_system.reserve(n_atoms);
    for (size_t s = 0; s < systems.size(); s++)
        for (int64_t i = 0; i < systems[s].n_atoms; i++) atom_system.push_back((int32_t)s);

    const double* d_positions = d_positions_in;
    if (!d_positions && !user_pairs) {
        double* d = arena_.alloc<double>("positions", 3 * n_atoms);
        int64_t off = 0;
        for (auto& s : systems) {
            if (s.n_atoms)
                CUDA_CHECK(cudaMemcpyAsync(d + 3 * off, s.positions.data(), sizeof(double) * 3 * s.n_atoms,
                                           cudaMemcpyHostToDevice, stream));
            off += s.n_atoms;
        }
        d_positions = d;
    }

    // atomic types -> species indices, uploaded while the stream is idle (a
    // copy from pageable memory waits for the stream)
    std::vector<int32_t> species_types, atom_species_h(n_atoms);
    {
        for (auto& s : systems) species_types.insert(species_types.end(), s.types.begin(), s.types.end());
        std::sort(species_types.begin(), species_types.end());
        species_types.erase(std::unique(species_types.begin(), species_types.end()), species_types.end());
        int64_t a = 0;
        for (auto& s : systems)
            for (int32_t t : s.types)
                atom_species_h[a++] =
                    (int32_t)(std::lower_bound(species_types.begin(), species_types.end(), t) - species_types.begin());
    }
    const int S = (int)species_types.size();
    int32_t* d_species = (!by_pair && n_atoms > 0) ? upload(arena_, "meta.atom_species", atom_species_h, stream) : nullptr;

    // ---- kernel (a): neighbour list ------------------------------------------
    DevicePairs pairs;
    if (!user_pairs) {
        std::vector<NlSystem> nls;
        int64_t atom_off = 0, cell_off = 0;
        for (auto& s : systems) {
            NlSystem n = make_nl_system(s.cell, h_.cutoff, atom_off, s.n_atoms, cell_off);
            cell_off += (int64_t)n.n_cells[0] * n.n_cells[1] * n.n_cells[2];
            atom_off += s.n_atoms;
            nls.push_back(n);
        }
        nl_.build(nls, atom_system, d_positions, n_atoms, arena_, stream);
        pairs = nl_.pairs;
    } else {
        // neighbour list given by the caller's systems
        std::vector<int32_t> f, sd, sh;
        std::vector<double> dist, vec;
        int64_t off = 0;
        for (auto& s : systems) {
            for (auto& p : s.pairs) {
                if ((int64_t)p.first >= s.n_atoms || (int64_t)p.second >= s.n_atoms)
                    throw Error(STATUS_SYSTEM_ERROR, "pair index out of bounds in the system's neighbour list");
                f.push_back((int32_t)(p.first + off));
                sd.push_back((int32_t)(p.second + off));
                dist.push_back(p.distance);
                vec.insert(vec.end(), p.vector, p.vector + 3);
                sh.insert(sh.end(), p.shift, p.shift + 3);
            }
            off += s.n_atoms;
        }
        pairs.count = (int64_t)f.size();
        pairs.first = upload(arena_, "pairs.first", f, stream);
        pairs.second = upload(arena_, "pairs.second", sd, stream);
        pairs.distance = upload(arena_, "pairs.distance", dist, stream);
        pairs.vector = upload(arena_, "pairs.vector", vec, stream);
        pairs.shift = upload(arena_, "pairs.shift", sh, stream);
    }
    CUDA_CHECK(cudaEventRecord(ev[1], stream));

    // ---- pair indices to the host, then the per-pair features run on the GPU
    // while the host builds the metadata ----------------------------------------
    // the power spectrum builds its neighbourhood tables on the device: the
    // host needs no pair list
    const bool device_tables = ps && n_atoms > 0;
    std::vector<int32_t> h_first(device_tables ? 0 : pairs.count), h_second(device_tables ? 0 : pairs.count),
        h_shift(by_pair ? 3 * pairs.count : 0);
    if (pairs.count && !device_tables) {
        CUDA_CHECK(cudaMemcpyAsync(h_first.data(), pairs.first, sizeof(int32_t) * pairs.count, cudaMemcpyDeviceToHost, stream));
        CUDA_CHECK(cudaMemcpyAsync(h_second.data(), pairs.second, sizeof(int32_t) * pairs.count, cudaMemcpyDeviceToHost, stream));
        if (by_pair)
            CUDA_CHECK(cudaMemcpyAsync(h_shift.data(), pairs.shift, sizeof(int32_t) * 3 * pairs.count,
                                       cudaMemcpyDeviceToHost, stream));
    }
    CUDA_CHECK(cudaEventRecord(ev[6], stream));

    FeatureLayout layout = FeatureLayout::make(h_.max_angular, h_.nmax(), g.any());
    // the spherical expansion builds its pair terms itself (fused kernel) or
    // reads them from per-pair records
    const bool fused_se = !by_pair && n_atoms > 0 && se_fused_enabled() && se_fused_supported(layout, d_radial_);
    double* features = fused_se ? nullptr : arena_.alloc<double>("features", pairs.count * layout.stride);
    int32_t* status = arena_.alloc<int32_t>("status", 1);
    CUDA_CHECK(cudaMemsetAsync(status, 0, sizeof(int32_t), stream));
    CutoffParams cut{h_.cutoff, h_.smoothing_width, h_.smoothing, h_.scaling ? 1 : 0,
                     h_.scaling_scale, h_.scaling_rate, h_.scaling_exponent};
    if (!fused_se) launch_pair_features(pairs, d_radial_, d_ylm_, cut, layout, features, status, stream);
    CUDA_CHECK(cudaEventRecord(ev[2], stream));

    // ---- kernel (b): spherical expansion.  It needs the directions sorted by
    // (centre, neighbour species) in pair order, which the GPU sorts itself,
    // so it runs right after the pair features while the host builds the
    // neighbourhood tables and the output plan -------------------------------
    auto t_meta0 = std::chrono::steady_clock::now();
    SeArgs se{};
    const bool run_se = !by_pair && n_atoms > 0;
    DeviceNeighborhoods nb;
    int32_t* nb_host_count = nullptr;
    uint8_t* nb_host_mask = nullptr;
    int64_t nb_capacity = 0;
    int64_t* nb_host_offset = nullptr;
    PsEntry* nb_host_entries = nullptr;
    if (run_se) {
        const int K = layout.L2 * layout.nmax;
        se.layout = layout;
        se.n_centres = n_atoms;
        se.n_species = S;
        int32_t* d_dir = arena_.alloc<int32_t>("meta.dir_code", 2 * pairs.count);
        int64_t* d_seg = arena_.alloc<int64_t>("meta.seg_offset", n_atoms * S + 1);
        // the same order as the host's counting sort (stable radix sort of
        // (centre, species) keys over pair << 1 | reversed)
        launch_dense_directions(pairs, d_species, S, n_atoms, d_dir, d_seg, arena_, stream);
        if (device_tables) {
            // the power spectrum's neighbourhood tables, built on the copy
            // stream beside the expansion: the per-centre species counts come
            // back first (the output plan needs them), then the entries (the
            // labels need them); the contraction kernels wait for the copy
            // stream (join_uploads)
            cudaStream_t up = copy_stream();
            CUDA_CHECK(cudaEventRecord(ev[14], stream));
            CUDA_CHECK(cudaStreamWaitEvent(up, ev[14], 0));
            // pinned staging: [entry offsets][entries][species counts][species mask]
            nb_capacity = 2 * pairs.count + n_atoms;
            const size_t b_offset = sizeof(int64_t) * (n_atoms + 1), b_entries = sizeof(PsEntry) * nb_capacity;
            const size_t b_count = sizeof(int32_t) * n_atoms * S;
            char* host = (char*)staging(b_offset + b_entries + b_count + n_atoms * S);
            nb_host_offset = (int64_t*)host;
            nb_host_entries = (PsEntry*)(host + b_offset);
            nb_host_count = (int32_t*)(host + b_offset + b_entries);
            nb_host_mask = (uint8_t*)(host + b_offset + b_entries + b_count);
            // the species counts come back as soon as they are counted (ev[12]),
            // before the scan and the fill of the entries
            nb = launch_neighborhoods(pairs, d_species, d_dir, d_seg, S, n_atoms, arena_, up, nb_host_count,
                                      nb_host_mask, ev[12]);
            // the entries go back to the host (for the labels) on a stream of
            // their own, so that the contraction kernels, which join the copy
            // stream, do not wait for this copy
            cudaStream_t back = readback_stream();
            CUDA_CHECK(cudaEventRecord(ev[15], up));
            CUDA_CHECK(cudaStreamWaitEvent(back, ev[15], 0));
            CUDA_CHECK(cudaMemcpyAsync(nb_host_offset, nb.entry_offset, sizeof(int64_t) * (n_atoms + 1),
                                       cudaMemcpyDeviceToHost, back));
            CUDA_CHECK(cudaMemcpyAsync(nb_host_entries, nb.entries, sizeof(PsEntry) * nb_capacity,
                                       cudaMemcpyDeviceToHost, back));
            CUDA_CHECK(cudaEventRecord(ev[13], back));
        }
        se.centre_species = d_species;
        se.seg_offset = d_seg;
        se.dir_code = d_dir;
        se.features = features;
        se.self_contribution = d_self_;
        se.do_positions = g.positions;
        se.do_strain = g.strain;
        se.do_cell = g.cell;
        se.coef = arena_.alloc<double>("se.coef", n_atoms * S * K);
        se.pair_grad = g.positions ? arena_.alloc<double>("se.pair_grad", pairs.count * 3 * K) : nullptr;
        se.self_grad = g.positions ? arena_.alloc<double>("se.self_grad", n_atoms * S * 3 * K) : nullptr;
        se.strain = g.strain ? arena_.alloc<double>("se.strain", n_atoms * S * 9 * K) : nullptr;
        se.cellg = g.cell ? arena_.alloc<double>("se.cell", n_atoms * S * 9 * K) : nullptr;
        CUDA_CHECK(cudaEventRecord(ev[7], stream));
        if (fused_se) launch_se_fused(se, pairs, d_radial_, d_ylm_, cut, stream);
        else launch_se_accumulate(se, stream);
        CUDA_CHECK(cudaEventRecord(ev[3], stream));
    }

    if (!nh_) nh_ = std::make_unique<Neighborhoods>();
    Neighborhoods& nh = *nh_;
    if (device_tables) {
        // the atoms' bookkeeping here, the per-centre species tables from the
        // device; the entries follow before the labels are written
        CUDA_CHECK(cudaEventSynchronize(ev[12]));
        nh.n_atoms = n_atoms;
        nh.n_species = S;
        nh.species_types = species_types;
        nh.atom_species = atom_species_h;
        nh.atom_offset.resize(systems.size() + 1);
        nh.atom_system.resize(n_atoms);
        nh.atom_local.resize(n_atoms);
        int64_t a = 0;
        nh.atom_offset[0] = 0;
        for (size_t s = 0; s < systems.size(); s++) {
            for (int64_t i = 0; i < systems[s].n_atoms; i++, a++) {
                nh.atom_system[a] = (int32_t)s;
                nh.atom_local[a] = (int32_t)i;
            }
            nh.atom_offset[s + 1] = a;
        }
        nh.species_count.assign(nb_host_count, nb_host_count + n_atoms * S);
        nh.species_mask.assign(nb_host_mask, nb_host_mask + n_atoms * S);
    } else {
        CUDA_CHECK(cudaEventSynchronize(ev[6]));
        build_neighborhoods(systems, pairs.count, h_first.data(), h_second.data(), nh);
        if (nh.n_species != S) throw internal_error("species tables disagree");
    }

    OutputPlan plan = ps        ? plan_power_spectrum(nh, h_, g, /*with_labels=*/false)
                      : by_pair ? plan_by_pair(nh, h_, g, pairs.count, h_first.data(), h_second.data(), h_shift.data())
                                : plan_spherical_expansion(nh, h_, g);
    // the device's entries into the host tables, for the labels
    auto load_entries = [&]() {
        if (!device_tables) return;
        CUDA_CHECK(cudaEventSynchronize(ev[13]));
        nh.entry_offset.assign(nb_host_offset, nb_host_offset + n_atoms + 1);
        const int64_t n_entries = nh.entry_offset[n_atoms];
        if (n_entries > nb_capacity) throw internal_error("neighbour tables overflow");
        nh.entries.assign(nb_host_entries, nb_host_entries + n_entries);
    };
    auto t_meta1 = std::chrono::steady_clock::now();
    auto t_launch = t_meta1;  // host time when the contraction kernels are queued
    double meta_extra = 0.0;  // host metadata work done later, overlapped with kernels

    auto tm = std::make_unique<TensorMap>();
    tm->keys = plan.keys;
    tm->on_device = device_output;
    tm->device = device_;

    int64_t total = plan.total_doubles;
    double* d_out = nullptr;
    if (device_output) {
        // stream-ordered allocation from the device's default pool, which keeps
        // freed memory for reuse: no device-wide synchronisation per call
        void* p = nullptr;
        CUDA_CHECK(cudaMallocAsync(&p, std::max<size_t>(8, sizeof(double) * (size_t)total), stream));
        tm->storage = std::shared_ptr<void>(p, [](void* q) { cudaFreeAsync(q, nullptr); });
        d_out = (double*)p;
    } else {
        d_out = arena_.alloc<double>("output", total);
    }

    if (by_pair && !plan.blocks.empty()) {
        // ---- spherical expansion by pair: scatter of the pair records --------
        CUDA_CHECK(cudaEventRecord(ev[7], stream));
        CUDA_CHECK(cudaMemsetAsync(d_out, 0, sizeof(double) * (size_t)total, stream));
        std::vector<int64_t> offv, offp, offs, offc;
        for (auto& b : plan.blocks) {
            offv.push_back(b.off_values);
            offp.push_back(b.off_positions);
            offs.push_back(b.off_strain);
            offc.push_back(b.off_cell);
        }
        ByPairArgs bp{};
        bp.layout = layout;
        bp.n_dirs = 2 * pairs.count;
        bp.pairs = pairs;
        bp.features = features;
        bp.dir_block0 = upload(arena_, "bp.block0", plan.bp_block0, stream);
        bp.dir_row0 = upload(arena_, "bp.row0", plan.bp_row0, stream);
        bp.dir_row1 = upload(arena_, "bp.row1", plan.bp_row1, stream);
        bp.dir_grow = upload(arena_, "bp.grow", plan.bp_grow, stream);
        bp.off_values = upload(arena_, "bp.offv", offv, stream);
        bp.off_positions = upload(arena_, "bp.offp", offp, stream);
        bp.off_strain = upload(arena_, "bp.offs", offs, stream);
        bp.off_cell = upload(arena_, "bp.offc", offc, stream);
        bp.n_self = (int64_t)plan.bp_self_row.size();
        bp.self_block = upload(arena_, "bp.self_block", plan.bp_self_block, stream);
        bp.self_row = upload(arena_, "bp.self_row", plan.bp_self_row, stream);
        bp.self_contribution = d_self_;
        bp.out = d_out;
        CUDA_CHECK(cudaEventRecord(ev[3], stream));
        CUDA_CHECK(cudaEventRecord(ev[8], stream));
        CUDA_CHECK(cudaEventRecord(ev[9], stream));
        launch_by_pair(bp, g.positions, g.strain, g.cell, stream);
        CUDA_CHECK(cudaEventRecord(ev[4], stream));
        int32_t h_status = 0;
        CUDA_CHECK(cudaMemcpyAsync(&h_status, status, sizeof(int32_t), cudaMemcpyDeviceToHost, stream));
        CUDA_CHECK(cudaStreamSynchronize(stream));
        if (h_status != 0) {
            throw internal_error("Failed to compute radial integral with GTO basis. Try increasing decreasing the "
                                 "`cutoff`, or increasing the Gaussian's `width`.");
        }
    } else if (run_se && !plan.blocks.empty()) {
        // the metadata goes up on the copy stream while the expansion runs
        cudaStream_t up = copy_stream();
        std::vector<int64_t> offv, offp, offs, offc;
        for (auto& b : plan.blocks) {
            offv.push_back(b.off_values);
            offp.push_back(b.off_positions);
            offs.push_back(b.off_strain);
            offc.push_back(b.off_cell);
        }
        if (ps) {
            // ---- kernel (c): power spectrum ------------------------------------
            PsArgs pa{};
            pa.lmax = h_.max_angular;
            pa.nmax = h_.nmax();
            pa.n_species = S;
            pa.n_centres = nh.n_atoms;
            pa.n_props = (int64_t)(h_.max_angular + 1) * h_.nmax() * h_.nmax();
            pa.coef = se.coef;
            pa.pair_grad = se.pair_grad;
            pa.self_grad = se.self_grad;
            pa.strain = se.strain;
            pa.cellg = se.cellg;
            pa.dir_code = se.dir_code;
            pa.slot_offset = upload(arena_, "ps.slot_offset", plan.slot_offset, up);
            pa.slots = upload(arena_, "ps.slots", plan.slots, up);
            pa.entry_offset = nb.entry_offset;
            pa.entries = nb.entries;
            pa.entry_cum = nb.entry_cum;
            pa.slot_row = upload(arena_, "ps.slot_row", plan.slot_row, up);
            pa.off_values = upload(arena_, "ps.offv", offv, up);
            pa.off_positions = upload(arena_, "ps.offp", offp, up);
            pa.off_strain = upload(arena_, "ps.offs", offs, up);
            pa.off_cell = upload(arena_, "ps.offc", offc, up);
            pa.out = d_out;
            join_uploads(stream);
            PsEvents pe;
            pe.after_values = ev[8];
            pe.after_strain_cell = ev[11];
            pe.before_positions = ev[10];
            pe.after_positions = ev[9];
            t_launch = std::chrono::steady_clock::now();
            launch_power_spectrum(pa, g.positions, g.strain, g.cell, stream, pe);
            // the labels only describe the output: written while the kernels run
            auto t_labels = std::chrono::steady_clock::now();
            load_entries();
            fill_power_spectrum_labels(nh, g, plan);
            meta_extra += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_labels).count();
        } else {
            SeOutArgs so{};
            so.lmax = h_.max_angular;
            so.nmax = h_.nmax();
            so.n_species = S;
            so.coef = se.coef;
            so.pair_grad = se.pair_grad;
            so.self_grad = se.self_grad;
            so.strain = se.strain;
            so.cellg = se.cellg;
            so.dir_code = se.dir_code;
            so.n_rows = (int64_t)plan.row_centre.size();
            so.row_centre = upload(arena_, "so.row_centre", plan.row_centre, up);
            so.row_block = upload(arena_, "so.row_block", plan.row_block, up);
            so.row_sample = upload(arena_, "so.row_sample", plan.row_sample, up);
            so.n_grad_rows = (int64_t)plan.grad_block.size();
            so.grad_block = upload(arena_, "so.grad_block", plan.grad_block, up);
            so.grad_row = upload(arena_, "so.grad_row", plan.grad_row, up);
            so.grad_centre = upload(arena_, "so.grad_centre", plan.grad_centre, up);
            so.grad_atom = upload(arena_, "so.grad_atom", plan.grad_atom, up);
            so.grad_d0 = upload(arena_, "so.grad_d0", plan.grad_d0, stream);
            so.grad_d1 = upload(arena_, "so.grad_d1", plan.grad_d1, stream);
            so.block_l = upload(arena_, "so.block_l", plan.block_l, up);
            so.block_species = upload(arena_, "so.block_species", plan.block_species, up);
            so.off_values = upload(arena_, "so.offv", offv, up);
            so.off_positions = upload(arena_, "so.offp", offp, up);
            so.off_strain = upload(arena_, "so.offs", offs, up);
            so.off_cell = upload(arena_, "so.offc", offc, up);
            so.out = d_out;
            join_uploads(stream);
            CUDA_CHECK(cudaEventRecord(ev[8], stream));
            CUDA_CHECK(cudaEventRecord(ev[9], stream));
            t_launch = std::chrono::steady_clock::now();
            launch_se_output(so, g.positions, g.strain, g.cell, stream);
        }
        CUDA_CHECK(cudaEventRecord(ev[4], stream));
        int32_t h_status = 0;
        CUDA_CHECK(cudaMemcpyAsync(&h_status, status, sizeof(int32_t), cudaMemcpyDeviceToHost, stream));
        CUDA_CHECK(cudaStreamSynchronize(stream));
        if (h_status != 0) {
            throw internal_error("Failed to compute radial integral with GTO basis. Try increasing decreasing the "
                                 "`cutoff`, or increasing the Gaussian's `width`.");
        }
    } else {
        if (ps) {
            load_entries();
            fill_power_spectrum_labels(nh, g, plan);
        }
        for (int k : {7, 3, 8, 9, 4}) CUDA_CHECK(cudaEventRecord(ev[k], stream));
    }

    // ---- output TensorMap ------------------------------------------------------
    double* base = d_out;
    if (!device_output) {
        size_t bytes = std::max<size_t>(8, sizeof(double) * (size_t)total);
        size_t actual = 0;
        void* host = pinned_pool().get(bytes, &actual);
        bool pinned = is_pinned(host);
        tm->storage = std::shared_ptr<void>(host, [actual, pinned](void* q) { pinned_pool().put(q, actual, pinned); });
        if (total) CUDA_CHECK(cudaMemcpyAsync(host, d_out, sizeof(double) * total, cudaMemcpyDeviceToHost, stream));
        base = (double*)host;
    }
    CUDA_CHECK(cudaEventRecord(ev[5], stream));
    CUDA_CHECK(cudaStreamSynchronize(stream));

    std::vector<Labels> components_base;
    Labels properties = ps ? ps_properties(h_) : se_properties(h_);
    for (size_t b = 0; b < plan.blocks.size(); b++) {
        auto& bp = plan.blocks[b];
        auto blk = std::make_unique<Block>();
        blk->samples = std::move(bp.samples);
        blk->properties = properties;
        std::vector<Labels> comps;
        std::vector<size_t> comp_shape;
        if (!ps) {
            Labels mu;
            mu.names = {"o3_mu"};
            for (int m = -bp.l; m <= bp.l; m++) mu.values.push_back(m);
            comps.push_back(mu);
            comp_shape.push_back(2 * bp.l + 1);
        }
        blk->components = comps;
        blk->shape = {(size_t)bp.n_samples};
        blk->shape.insert(blk->shape.end(), comp_shape.begin(), comp_shape.end());
        blk->shape.push_back(properties.count());
        blk->data = base + bp.off_values;
        if (g.positions) {
            auto gb = std::make_unique<Block>();
            gb->samples = std::move(bp.gradient_samples);
            gb->components = {xyz_labels("xyz")};
            gb->components.insert(gb->components.end(), comps.begin(), comps.end());
            gb->properties = properties;
            gb->shape = {(size_t)bp.n_grad_rows, 3};
            gb->shape.insert(gb->shape.end(), comp_shape.begin(), comp_shape.end());
            gb->shape.push_back(properties.count());
            gb->data = base + bp.off_positions;
            blk->gradients.emplace_back("positions", std::move(gb));
        }
        // calculator.rs:448-490: cell components [xyz, abc, ...], strain [xyz_2, xyz_1, ...]
        for (int which = 0; which < 2; which++) {
            bool want = which == 0 ? g.cell : g.strain;
            if (!want) continue;
            auto gb = std::make_unique<Block>();
            gb->samples.names = {"sample"};
            for (int64_t s = 0; s < bp.n_samples; s++) gb->samples.values.push_back((int32_t)s);
            if (which == 0) gb->components = {xyz_labels("xyz"), xyz_labels("abc")};
            else gb->components = {xyz_labels("xyz_2"), xyz_labels("xyz_1")};
            gb->components.insert(gb->components.end(), comps.begin(), comps.end());
            gb->properties = properties;
            gb->shape = {(size_t)bp.n_samples, 3, 3};
            gb->shape.insert(gb->shape.end(), comp_shape.begin(), comp_shape.end());
            gb->shape.push_back(properties.count());
            gb->data = base + (which == 0 ? bp.off_cell : bp.off_strain);
            blk->gradients.emplace_back(which == 0 ? "cell" : "strain", std::move(gb));
        }
        tm->blocks.push_back(std::move(blk));
    }

    times_.neighbors = elapsed_ms(ev[0], ev[1]);
    times_.metadata_before_launch = std::chrono::duration<double, std::milli>(t_launch - t_meta0).count();
    times_.labels = meta_extra;
    times_.metadata = times_.metadata_before_launch + meta_extra;
    times_.features = elapsed_ms(ev[6], ev[2]);
    times_.expansion = elapsed_ms(ev[7], ev[3]);
    times_.contraction = elapsed_ms(ev[3], ev[4]);
    if (ps && run_se) {
        // values, strain and cell run beside the positions kernel
        times_.ps_values = elapsed_ms(ev[3], ev[8]);
        times_.ps_positions = elapsed_ms(ev[10], ev[9]);
        times_.ps_strain_cell = elapsed_ms(ev[8], ev[11]);
    } else {
        times_.ps_values = elapsed_ms(ev[3], ev[8]);
        times_.ps_positions = elapsed_ms(ev[8], ev[9]);
        times_.ps_strain_cell = elapsed_ms(ev[9], ev[4]);
    }
    times_.transfer = elapsed_ms(ev[4], ev[5]);
    times_.total = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_start).count();
    return tm;
}

// ---------------------------------------------------------------------------
// Dense power spectrum and its adjoint
// ---------------------------------------------------------------------------
DenseState::~DenseState() {
    for (void* p : allocations_) cudaFreeAsync(p, stream);
}

void* DenseState::alloc(size_t bytes) {
    void* p = nullptr;
    CUDA_CHECK(cudaMallocAsync(&p, std::max<size_t>(bytes, 8), stream));
    allocations_.push_back(p);
    return p;
}

template <typename T>
void Engine::dense_args(const DenseState& st, bool grad, DenseArgs<T>& a) {
    a = DenseArgs<T>{};
    a.lmax = h_.max_angular;
    a.nmax = h_.nmax();
    a.n_species = st.n_species;
    a.n_keys = st.n_keys;
    a.K = st.K;
    a.n_atoms = st.n_atoms;
    a.n_props = st.n_props;
    a.n_systems = st.n_systems;
    a.layout = FeatureLayout::make(h_.max_angular, h_.nmax(), grad);
    a.pairs = st.pairs;
    a.atom_species = st.atom_species;
    a.seg_offset = st.seg_offset;
    a.dir_code = st.dir_code;
    a.pair_start = st.pair_start;
    a.atom_offset = st.d_atom_offset;
    a.exact = d_radial_;
    if constexpr (sizeof(T) == 8) {
        a.tab = dense_d_;
    } else {
        a.tab = dense_f_;
        a.surrogate = active_surrogate_;
    }
    a.cut = CutoffParams{h_.cutoff, h_.smoothing_width, h_.smoothing, h_.scaling ? 1 : 0,
                         h_.scaling_scale, h_.scaling_rate, h_.scaling_exponent};
    a.coef = static_cast<T*>(st.coef);
}

std::unique_ptr<DenseState> Engine::forward_dense(int precision, std::vector<HostSystem>& systems,
                                                  const double* d_positions, const std::vector<int32_t>& species,
                                                  void* values, int64_t values_count, cudaStream_t stream,
                                                  bool expansion, bool backward_follows) {
    if (precision != 32 && precision != 64) throw invalid_parameter("precision must be 32 or 64");
    upload_tables();
    const std::shared_ptr<RadialSurrogate> hold = surrogate_.lock();
    active_surrogate_ = hold.get();
    struct Release {
        RadialSurrogate** p;
        ~Release() { *p = nullptr; }
    } release{&active_surrogate_};
    auto st = std::make_unique<DenseState>();
    st->engine = this;
    st->device = device_;
    st->precision = precision;
    st->stream = stream;
    st->n_systems = (int64_t)systems.size();

    std::vector<int32_t> types, atom_system;
    st->atom_offset.assign(1, 0);
    for (size_t s = 0; s < systems.size(); s++) {
        types.insert(types.end(), systems[s].types.begin(), systems[s].types.end());
        atom_system.insert(atom_system.end(), (size_t)systems[s].n_atoms, (int32_t)s);
        st->atom_offset.push_back(st->atom_offset.back() + systems[s].n_atoms);
    }
    const int64_t n_atoms = st->n_atoms = (int64_t)types.size();
    if (n_atoms >= (int64_t)INT32_MAX / 2) throw invalid_parameter("too many atoms");
    std::vector<int32_t> sp = species.empty() ? types : species;
    std::sort(sp.begin(), sp.end());
    sp.erase(std::unique(sp.begin(), sp.end()), sp.end());
    std::vector<int32_t> atom_species(n_atoms);
    for (int64_t i = 0; i < n_atoms; i++) {
        auto it = std::lower_bound(sp.begin(), sp.end(), types[i]);
        if (it == sp.end() || *it != types[i])
            throw invalid_parameter("atomic type " + std::to_string(types[i]) + " is not in the list of species");
        atom_species[i] = (int32_t)(it - sp.begin());
    }
    st->species_types = sp;
    const int S = st->n_species = (int)sp.size();
    st->n_keys = S * (S + 1) / 2;
    st->n_props = (int64_t)(h_.max_angular + 1) * h_.nmax() * h_.nmax();
    st->K = (h_.max_angular + 1) * (h_.max_angular + 1) * h_.nmax();
    const int64_t expected = expansion ? n_atoms * S * st->K : n_atoms * st->n_keys * st->n_props;
    if (values_count != expected) {
        throw invalid_parameter(std::string("the values buffer must hold ") +
                                (expansion ? "n_atoms x n_species x (max_angular + 1)^2 (max_radial + 1) = "
                                           : "n_atoms x n_keys x n_properties = ") +
                                std::to_string(expected) + " elements, got " + std::to_string(values_count));
    }
    if (n_atoms > 0 && !values) throw invalid_parameter("values must not be NULL");
    const size_t T_size = precision == 64 ? 8 : 4;

    st->d_atom_offset = (int64_t*)st->alloc(sizeof(int64_t) * st->atom_offset.size());
    CUDA_CHECK(cudaMemcpyAsync(st->d_atom_offset, st->atom_offset.data(), sizeof(int64_t) * st->atom_offset.size(),
                               cudaMemcpyHostToDevice, stream));
    if (n_atoms == 0) return st;
    st->atom_species = (int32_t*)st->alloc(sizeof(int32_t) * n_atoms);
    CUDA_CHECK(cudaMemcpyAsync(st->atom_species, atom_species.data(), sizeof(int32_t) * n_atoms,
                               cudaMemcpyHostToDevice, stream));

    // neighbour list (kernel a), then a private copy for the backward pass
    std::vector<NlSystem> nls;
    int64_t atom_off = 0, cell_off = 0;
    for (auto& s : systems) {
        NlSystem n = make_nl_system(s.cell, h_.cutoff, atom_off, s.n_atoms, cell_off);
        cell_off += (int64_t)n.n_cells[0] * n.n_cells[1] * n.n_cells[2];
        atom_off += s.n_atoms;
        nls.push_back(n);
    }
    const int64_t P = nl_.build(nls, atom_system, d_positions, n_atoms, arena_, stream);
    st->n_pairs = P;
    st->pairs.count = P;
    st->pairs.first = (int32_t*)st->alloc(sizeof(int32_t) * P);
    st->pairs.second = (int32_t*)st->alloc(sizeof(int32_t) * P);
    st->pairs.distance = (double*)st->alloc(sizeof(double) * P);
    st->pairs.vector = (double*)st->alloc(sizeof(double) * 3 * P);
    st->pairs.shift = (int32_t*)st->alloc(sizeof(int32_t) * 3 * P);
    st->pair_start = (int64_t*)st->alloc(sizeof(int64_t) * (n_atoms + 1));
    if (P > 0) {
        CUDA_CHECK(cudaMemcpyAsync(st->pairs.first, nl_.pairs.first, 4 * P, cudaMemcpyDeviceToDevice, stream));
        CUDA_CHECK(cudaMemcpyAsync(st->pairs.second, nl_.pairs.second, 4 * P, cudaMemcpyDeviceToDevice, stream));
        CUDA_CHECK(cudaMemcpyAsync(st->pairs.distance, nl_.pairs.distance, 8 * P, cudaMemcpyDeviceToDevice, stream));
        CUDA_CHECK(cudaMemcpyAsync(st->pairs.vector, nl_.pairs.vector, 24 * P, cudaMemcpyDeviceToDevice, stream));
        CUDA_CHECK(cudaMemcpyAsync(st->pairs.shift, nl_.pairs.shift, 12 * P, cudaMemcpyDeviceToDevice, stream));
    }
    CUDA_CHECK(cudaMemcpyAsync(st->pair_start, nl_.pair_start, sizeof(int64_t) * (n_atoms + 1),
                               cudaMemcpyDeviceToDevice, stream));

    // direction segments, coefficients, power spectrum
    st->dir_code = (int32_t*)st->alloc(sizeof(int32_t) * 2 * P);
    st->seg_offset = (int64_t*)st->alloc(sizeof(int64_t) * (n_atoms * S + 1));
    launch_dense_directions(st->pairs, st->atom_species, S, n_atoms, st->dir_code, st->seg_offset, arena_, stream);
    st->coef = st->alloc(T_size * (size_t)n_atoms * S * st->K);
    int32_t* status = arena_.alloc<int32_t>("dense.status", 1);
    CUDA_CHECK(cudaMemsetAsync(status, 0, sizeof(int32_t), stream));
    // with the learned surrogate, the FP32 backward recomputes the pair
    // features with their derivatives; when the caller announces a backward
    // pass, the forward computes them once and leaves them in the state
    const bool keep = backward_follows && precision == 32 && active_surrogate_ != nullptr && !expansion;
    const FeatureLayout layout = FeatureLayout::make(h_.max_angular, h_.nmax(), keep);
    const size_t feature_bytes = T_size * (size_t)std::max<int64_t>(P, 1) * layout.stride;
    void* features = keep ? st->alloc(feature_bytes) : arena_.alloc_bytes("dense.features", feature_bytes);
    if (keep) st->features_grad = features;
    cudaEvent_t* marks = dense_marks();
    if (precision == 64) {
        DenseArgs<double> a;
        dense_args(*st, false, a);
        a.marks = marks;
        a.features = (double*)features;
        a.values = expansion ? nullptr : (double*)values;
        a.status = status;
        launch_dense_forward<double>(a, P, stream);
    } else {
        DenseArgs<float> a;
        dense_args(*st, keep, a);
        a.gradient_features = keep;
        a.marks = marks;
        a.features = (float*)features;
        a.values = expansion ? nullptr : (float*)values;
        a.status = status;
        launch_dense_forward<float>(a, P, stream);
    }
    if (expansion) {
        CUDA_CHECK(cudaMemcpyAsync(values, st->coef, T_size * (size_t)n_atoms * S * st->K, cudaMemcpyDeviceToDevice,
                                   stream));
    }
    if (!radial_.splined) {
        int32_t h_status = 0;
        CUDA_CHECK(cudaMemcpyAsync(&h_status, status, sizeof(int32_t), cudaMemcpyDeviceToHost, stream));
        CUDA_CHECK(cudaStreamSynchronize(stream));
        if (h_status) throw internal_error("the analytic radial integral did not converge");
    }
    return st;
}

void Engine::jvp_dense(DenseState& st, const void* tangent_positions, const void* tangent_cell, void* tangent_coef,
                       void* tangent_values, cudaStream_t stream) {
    int dev = -1;
    CUDA_CHECK(cudaGetDevice(&dev));
    if (dev != st.device) throw invalid_parameter("the derivative must run on the device of the forward pass");
    const std::shared_ptr<RadialSurrogate> hold = surrogate_.lock();
    active_surrogate_ = hold.get();
    struct Release {
        RadialSurrogate** p;
        ~Release() { *p = nullptr; }
    } release{&active_surrogate_};
    if (st.n_atoms == 0) return;
    if (!tangent_positions) throw invalid_parameter("tangent_positions must not be NULL");
    const size_t T_size = st.precision == 64 ? 8 : 4;
    const int64_t P = st.n_pairs;
    const FeatureLayout layout = FeatureLayout::make(h_.max_angular, h_.nmax(), true);
    void* features = arena_.alloc_bytes("dense.features_grad", T_size * (size_t)std::max<int64_t>(P, 1) * layout.stride);
    void* pair_tangent = arena_.alloc_bytes("dense.pair_tangent", T_size * (size_t)std::max<int64_t>(P, 1) * st.K);
    void* tcoef = tangent_coef ? tangent_coef
                               : arena_.alloc_bytes("dense.tangent_coef", T_size * (size_t)st.n_atoms * st.n_species * st.K);
    int32_t* status = arena_.alloc<int32_t>("dense.status", 1);
    CUDA_CHECK(cudaMemsetAsync(status, 0, sizeof(int32_t), stream));
    if (st.precision == 64) {
        DenseArgs<double> a;
        dense_args(st, true, a);
        a.features = (double*)features;
        a.status = status;
        launch_dense_jvp<double>(a, P, (const double*)tangent_positions, (const double*)tangent_cell,
                                 (double*)pair_tangent, (double*)tcoef, (double*)tangent_values, stream);
    } else {
        DenseArgs<float> a;
        dense_args(st, true, a);
        a.features = (float*)features;
        a.status = status;
        launch_dense_jvp<float>(a, P, (const float*)tangent_positions, (const float*)tangent_cell, (float*)pair_tangent,
                                (float*)tcoef, (float*)tangent_values, stream);
    }
}

void Engine::backward_dense(DenseState& st, const void* grad_values, void* grad_positions, void* grad_strain,
                            void* grad_cell, cudaStream_t stream, bool by_species, bool coefficients) {
    int dev = -1;
    CUDA_CHECK(cudaGetDevice(&dev));
    if (dev != st.device) throw invalid_parameter("the backward pass must run on the device of the forward pass");
    const std::shared_ptr<RadialSurrogate> hold = surrogate_.lock();
    active_surrogate_ = hold.get();
    struct Release {
        RadialSurrogate** p;
        ~Release() { *p = nullptr; }
    } release{&active_surrogate_};
    if (st.n_atoms == 0) return;
    if (!grad_values || !grad_positions) throw invalid_parameter("grad_values and grad_positions must not be NULL");
    const size_t T_size = st.precision == 64 ? 8 : 4;
    const int64_t P = st.n_pairs;
    const FeatureLayout layout = FeatureLayout::make(h_.max_angular, h_.nmax(), true);
    // the forward's features with derivatives when it kept them (and the
    // surrogate that made them is still the active radial integral)
    const bool kept = st.features_grad != nullptr && active_surrogate_ != nullptr;
    void* features = kept ? st.features_grad
                          : arena_.alloc_bytes("dense.features_grad", T_size * (size_t)std::max<int64_t>(P, 1) * layout.stride);
    void* grad_coef = coefficients ? const_cast<void*>(grad_values)
                                   : arena_.alloc_bytes("dense.grad_coef", T_size * (size_t)st.n_atoms * st.n_species * st.K);
    void* pair_grad = arena_.alloc_bytes("dense.pair_grad", T_size * 3 * (size_t)std::max<int64_t>(P, 1));
    void* partial = arena_.alloc_bytes("dense.atom_partial", T_size * 18 * (size_t)st.n_atoms);
    int32_t* status = arena_.alloc<int32_t>("dense.status", 1);
    cudaEvent_t* marks = dense_marks();
    if (st.precision == 64) {
        DenseArgs<double> a;
        dense_args(st, true, a);
        a.marks = marks;
        a.features = (double*)features;
        a.grad_values = (const double*)grad_values;
        a.grad_species = by_species ? st.atom_species : nullptr;
        a.grad_coef = (double*)grad_coef;
        a.pair_grad = (double*)pair_grad;
        a.atom_partial = (double*)partial;
        a.grad_positions = (double*)grad_positions;
        a.grad_strain = (double*)grad_strain;
        a.grad_cell = (double*)grad_cell;
        a.status = status;
        launch_dense_backward<double>(a, P, stream, coefficients);
    } else {
        DenseArgs<float> a;
        dense_args(st, true, a);
        a.gradient_features = kept;
        a.marks = marks;
        a.features = (float*)features;
        a.grad_values = (const float*)grad_values;
        a.grad_species = by_species ? st.atom_species : nullptr;
        a.grad_coef = (float*)grad_coef;
        a.pair_grad = (float*)pair_grad;
        a.atom_partial = (float*)partial;
        a.grad_positions = (float*)grad_positions;
        a.grad_strain = (float*)grad_strain;
        a.grad_cell = (float*)grad_cell;
        a.status = status;
        launch_dense_backward<float>(a, P, stream, coefficients);
    }
}

}  // namespace fb200

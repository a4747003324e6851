// Kernel (c): SOAP power spectrum and its gradients on the GPU, FP64.
//
//   P[l, n1, n2] = sum_m c_a[l m n1] c_b[l m n2] * (sqrt 2 if a != b) / ((-1)^l sqrt(2l+1))
//
// featomic/src/calculators/soap/power_spectrum.rs:571-764.  One CTA per
// centre: the centre's key slots (block, sample row, neighbour species a, b)
// and its unique-neighbour entries are precomputed on the host, so every
// output row is written exactly once, contiguously, straight into the final
// TensorMap block layout ([sample][property], [gradient row][xyz][property],
// [sample][3][3][property]).
//
// positions gradient of row (centre i, atom j):
//   j == i : sum_m c_b dself_a + c_a dself_b
//   j != i : sum_m c_b dc_a(i<-j) [type(j) == a] + c_a dc_b(i<-j) [type(j) == b]
// with dc(i<-j) = sum over the pairs between i and j of g_pair (i first) or
// -(-1)^l g_pair (i second), in pair order.
#include "engine.hpp"

namespace fb200 {

namespace {

struct PropIndex {
    int l, n1, n2;
};

__device__ __forceinline__ PropIndex decode_prop(int64_t p, int nmax) {
    PropIndex r;
    int nn = nmax * nmax;
    r.l = (int)(p / nn);
    int rem = (int)(p - (int64_t)r.l * nn);
    r.n1 = rem / nmax;
    r.n2 = rem - r.n1 * nmax;
    return r;
}

__device__ __forceinline__ double ps_norm(int l) {
    double s = sqrt((double)(2 * l + 1));
    return (l % 2 == 0) ? s : -s;
}

__global__ void ps_values_kernel(PsArgs a) {
    const int64_t c = blockIdx.x;
    const int K = (a.lmax + 1) * (a.lmax + 1) * a.nmax;
    const int S = a.n_species;
    for (int64_t s = a.slot_offset[c]; s < a.slot_offset[c + 1]; s++) {
        const PsKeySlot slot = a.slots[s];
        const double* ca = a.coef + ((int64_t)c * S + slot.a) * K;
        const double* cb = a.coef + ((int64_t)c * S + slot.b) * K;
        double* out = a.out + a.off_values[slot.block] + (int64_t)slot.sample * a.n_props;
        const double scale = slot.a != slot.b ? 1.4142135623730951 : 1.0;
        for (int64_t p = threadIdx.x; p < a.n_props; p += blockDim.x) {
            PropIndex q = decode_prop(p, a.nmax);
            double sum = 0.0;
            const int base = q.l * q.l * a.nmax;
            for (int m = 0; m < 2 * q.l + 1; m++)
                sum += __ldg(ca + base + m * a.nmax + q.n1) * __ldg(cb + base + m * a.nmax + q.n2);
            if (slot.a != slot.b) sum *= scale;
            out[p] = sum / ps_norm(q.l);
        }
    }
}

__global__ void ps_positions_kernel(PsArgs a) {
    const int64_t c = blockIdx.x;
    const int K = (a.lmax + 1) * (a.lmax + 1) * a.nmax;
    const int S = a.n_species;
    const int64_t s0 = a.slot_offset[c], ns = a.slot_offset[c + 1] - s0;
    const int64_t e0 = a.entry_offset[c], ne = a.entry_offset[c + 1] - e0;
    const int64_t rbase = a.row_offset[c];
    for (int64_t e = 0; e < ne; e++) {
        const PsEntry entry = a.entries[e0 + e];
        const bool self = entry.atom == (int32_t)c;
        for (int64_t s = 0; s < ns; s++) {
            const int64_t row = a.rows[rbase + e * ns + s];
            if (row < 0) continue;
            const PsKeySlot slot = a.slots[s0 + s];
            const double* ca = a.coef + ((int64_t)c * S + slot.a) * K;
            const double* cb = a.coef + ((int64_t)c * S + slot.b) * K;
            const bool has1 = self || entry.species == slot.a;
            const bool has2 = self || entry.species == slot.b;
            double* out = a.out + a.off_positions[slot.block] + row * 3 * a.n_props;
            for (int64_t qi = threadIdx.x; qi < 3 * a.n_props; qi += blockDim.x) {
                const int x = (int)(qi / a.n_props);
                const int64_t p = qi - x * a.n_props;
                PropIndex q = decode_prop(p, a.nmax);
                const int base = q.l * q.l * a.nmax;
                const double sign_l = (q.l & 1) ? -1.0 : 1.0;
                double sum = 0.0;
                for (int pass = 0; pass < 2; pass++) {
                    if (pass == 0 && !has1) continue;
                    if (pass == 1 && !has2) continue;
                    // pass 0: value of b, gradient of a (column n1); pass 1: value of a, gradient of b (column n2)
                    const double* cv = pass == 0 ? cb : ca;
                    const int nv = pass == 0 ? q.n2 : q.n1;
                    const int ng = pass == 0 ? q.n1 : q.n2;
                    const int tg = pass == 0 ? slot.a : slot.b;
                    for (int m = 0; m < 2 * q.l + 1; m++) {
                        const int idx = base + m * a.nmax + ng;
                        double g;
                        if (self) {
                            g = __ldg(a.self_grad + (((int64_t)c * S + tg) * 3 + x) * K + idx);
                        } else {
                            g = 0.0;
                            for (int d = entry.d0; d < entry.d1; d++) {
                                const int32_t code = a.dir_code[d];
                                const int64_t pr = code >> 1;
                                const double factor = (code & 1) ? -sign_l : 1.0;
                                g += factor * __ldg(a.pair_grad + (pr * 3 + x) * K + idx);
                            }
                        }
                        sum += __ldg(cv + base + m * a.nmax + nv) * g;
                    }
                }
                if (slot.a != slot.b) sum *= 1.4142135623730951;
                out[qi] = sum / ps_norm(q.l);
            }
        }
    }
}

__global__ void ps_strain_cell_kernel(PsArgs a, int which) {
    const int64_t c = blockIdx.x;
    const int K = (a.lmax + 1) * (a.lmax + 1) * a.nmax;
    const int S = a.n_species;
    const double* src = which == 0 ? a.strain : a.cellg;
    const int64_t* offs = which == 0 ? a.off_strain : a.off_cell;
    for (int64_t s = a.slot_offset[c]; s < a.slot_offset[c + 1]; s++) {
        const PsKeySlot slot = a.slots[s];
        const double* ca = a.coef + ((int64_t)c * S + slot.a) * K;
        const double* cb = a.coef + ((int64_t)c * S + slot.b) * K;
        const double* ga = src + ((int64_t)c * S + slot.a) * 9 * K;
        const double* gb = src + ((int64_t)c * S + slot.b) * 9 * K;
        double* out = a.out + offs[slot.block] + (int64_t)slot.sample * 9 * a.n_props;
        for (int64_t qi = threadIdx.x; qi < 9 * a.n_props; qi += blockDim.x) {
            const int x = (int)(qi / a.n_props);
            const int64_t p = qi - x * a.n_props;
            PropIndex q = decode_prop(p, a.nmax);
            const int base = q.l * q.l * a.nmax;
            double sum = 0.0;
            for (int m = 0; m < 2 * q.l + 1; m++)
                sum += __ldg(cb + base + m * a.nmax + q.n2) * __ldg(ga + (int64_t)x * K + base + m * a.nmax + q.n1);
            for (int m = 0; m < 2 * q.l + 1; m++)
                sum += __ldg(ca + base + m * a.nmax + q.n1) * __ldg(gb + (int64_t)x * K + base + m * a.nmax + q.n2);
            if (slot.a != slot.b) sum *= 1.4142135623730951;
            out[qi] = sum / ps_norm(q.l);
        }
    }
}

}  // namespace

void launch_ps_values(const PsArgs& args, cudaStream_t stream) {
    if (args.n_centres == 0) return;
    ps_values_kernel<<<(unsigned)args.n_centres, 128, 0, stream>>>(args);
    CUDA_CHECK(cudaGetLastError());
}

void launch_ps_positions(const PsArgs& args, cudaStream_t stream) {
    if (args.n_centres == 0) return;
    ps_positions_kernel<<<(unsigned)args.n_centres, 256, 0, stream>>>(args);
    CUDA_CHECK(cudaGetLastError());
}

void launch_ps_strain_cell(const PsArgs& args, bool strain, bool cell, cudaStream_t stream) {
    if (args.n_centres == 0) return;
    if (strain) {
        ps_strain_cell_kernel<<<(unsigned)args.n_centres, 256, 0, stream>>>(args, 0);
        CUDA_CHECK(cudaGetLastError());
    }
    if (cell) {
        ps_strain_cell_kernel<<<(unsigned)args.n_centres, 256, 0, stream>>>(args, 1);
        CUDA_CHECK(cudaGetLastError());
    }
}

}  // namespace fb200

// Clebsch-Gordan coefficients and block tensor products (clebsch_gordan.cu).
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "../../include/featomic_b200.h"

namespace fb200 {

// Real CG coefficients of (l1, l2) -> lambda, dense [2 l1 + 1][2 l2 + 1][2 lambda + 1].
std::vector<double> real_cg_coefficients(int l1, int l2, int lambda);

// Launch every task on `stream` (precision 32 or 64).
void cg_product(const featomic_b200_cg_task_t* tasks, size_t n_tasks, int precision, cudaStream_t stream);

// Couple two spherical axes of each task's input to lambda, on `stream`.
void cg_couple(const featomic_b200_cg_couple_task_t* tasks, size_t n_tasks, int precision, cudaStream_t stream);

}  // namespace fb200

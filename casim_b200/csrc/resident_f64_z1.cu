// Resident-path kernels for double fields and 1 cleft layer(s): one translation
// unit per (precision, layers) so the specialisations compile in parallel.
#include "resident_kernel.cuh"

cudaError_t cb_res_f64_z1(const cbres::rs_args& a, int NI, int NP, int C, int threads, cudaStream_t st, int n, int* dry, int known) {
    return cbres::dispatch<double, 1>(a, NI, NP, C, threads, st, n, dry, known);
}

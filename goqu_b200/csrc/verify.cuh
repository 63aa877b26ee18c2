// Circuit equivalence on the device (transpile/verify/verify.go).
//
// goqu builds a circuit's unitary column by column: 2^n separate statevector
// runs, each starting from X gates that prepare |col> (verify.go:45-90).
// Here every column evolves at once: the unitary is one 2n-qubit vector with
// the row index in the low n bits and the column index in the high n bits,
// entry (col << n) | row = U[row][col], starting from the identity. The
// circuit's ops act on the low n qubits only, so one pass sequence over 4^n
// amplitudes applies the circuit to every column.
//
// The comparisons follow verify.go's rules: the global phase comes from the
// first entry of B (in index order; column 0 for unitaries) whose modulus
// exceeds tol, and every entry must then satisfy |a - phase * b| <= tol. The
// first index is an atomicMin over threads; the mismatch test sets a flag.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "tile_core.cuh"

namespace gq {

// Identity columns: entry (c << n) | c = 1 (the rest was cleared).
__global__ void k_unit_columns(cplx<double>* __restrict__ st, int n) {
    const uint64_t c = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (c < (1ull << n)) st[(c << n) | c] = {1.0, 0.0};
}

// *first = min(*first, smallest i < len with |v[i]| > tol).
__global__ void k_first_above(const cplx<double>* __restrict__ v, uint64_t len, double tol,
                              unsigned long long* __restrict__ first) {
    unsigned long long best = ~0ull;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < len; i += (uint64_t)gridDim.x * blockDim.x)
        if (hypot(v[i].x, v[i].y) > tol) {
            best = i;
            break;  // indices grow along the thread's stride
        }
    if (best != ~0ull) atomicMin(first, best);
}

// *bad = 1 when some |a[i] - phase * b[i]| > tol.
__global__ void k_phase_mismatch(const cplx<double>* __restrict__ a, const cplx<double>* __restrict__ b, uint64_t len,
                                 double pr, double pi, double tol, int* __restrict__ bad) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < len; i += (uint64_t)gridDim.x * blockDim.x) {
        const double dr = a[i].x - (pr * b[i].x - pi * b[i].y);
        const double di = a[i].y - (pr * b[i].y + pi * b[i].x);
        if (hypot(dr, di) > tol) {
            *bad = 1;
            return;
        }
    }
}

}  // namespace gq

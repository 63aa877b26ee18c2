// Batched MaxCut QAOA on the device: energies and adjoint gradients of many
// circuits of goqu's qaoa.Run form (algorithm/qaoa/qaoa.go:68-93, 164-196;
// MaxCutHamiltonian, maxcut.go:13-35), complex64 amplitudes with FP64
// reductions.
//
// The circuit is H on every qubit, then per layer k one RZZ(gamma_k) per edge
// (RZZ(2 * 0.5 * gamma_k), the cost layer of the edge's 0.5 Z_i Z_j term) and
// RX(2 beta_k) on every qubit; the energy is <psi| H |psi> with
// H = sum_e (-1/2 + 1/2 Z_i Z_j). In the computational basis both cost layer
// and Hamiltonian are functions of the cut count C(z), the number of edges
// whose two bits differ in z:
//   cost layer  D_k(z) = exp(-i gamma_k (|E| - 2 C(z)) / 2)
//   Hamiltonian H(z)   = -C(z)
// so a per-circuit table of C(z) (one byte per amplitude, built by the first
// pass) turns every cost layer into one lookup and one complex multiply, and
// lambda = H psi into a multiply. A mixer layer is the same RX on every qubit:
// butterflies in rounds of four qubits inside a tile of 4096 amplitudes held
// in shared memory (16 per thread, 256 threads).
//
// Gradients (adjoint method): with G = dU U^dagger,
//   beta_k:  G = -i sum_q X_q, so dE/dbeta_k = 2 sum_q Im <lambda| X_q |psi>;
//   gamma_k: G = -i A / 2 with A(z) = |E| - 2 C(z), so
//            dE/dgamma_k = sum_z A(z) Im(conj(lambda_z) psi_z).
// Both are invariant under the layer's own rotations (X_q commutes with
// RX_q; diagonal phases cancel in conj(lambda) psi), so each term is taken in
// whichever pass holds the qubit.
//
// Circuits of n <= 12 qubits run whole in one CTA: state, lambda and cut table
// in shared memory, forward, energy and reverse sweep without touching global
// memory. Larger circuits run one launch per pass over all circuits of the
// same (n, p): per layer a pass over tile qubits 0..11 and, for the qubits
// above 11, group passes whose tile is qubits 0..3 (coalescing), up to eight
// of the high qubits and filler qubits. Per-tile gradient and energy partials
// are summed in a fixed order, so results do not depend on scheduling.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/gqb200.h"

namespace gq {
void set_last_error(const std::string& msg);  // engine.cu
}

namespace {

constexpr int TB = 12;                 // tile bits
constexpr int TILE = 1 << TB;          // amplitudes per tile
constexpr int NT = TILE / 16;          // threads per tile (16 amplitudes each)
constexpr int MAX_LAYERS = 64;
constexpr int MAX_EDGES = 255;         // cut counts are bytes
constexpr int MAX_QUBITS = 26;
constexpr int kSmemForward = TILE * 8 + TILE;       // one tile of complex64 + its cut counts
constexpr int kSmemReverse = 2 * TILE * 8 + TILE;   // psi and lambda tiles + cut counts

// Pass flags.
constexpr int F_INIT = 1;        // the state is H^n |0>: synthesised, the cut table computed and stored
constexpr int F_D_BEFORE = 2;    // apply D_layer before the rotations (first group pass of layer 0)
constexpr int F_D_AFTER = 4;     // apply D_(layer+1) after the rotations (low pass, not the last layer)
constexpr int F_ENERGY = 8;      // after the rotations: energy partial and lambda = H psi (last pass)
// reverse
constexpr int F_UNDO_D = 16;     // start: gradient of gamma_(layer+1), then undo D_(layer+1)
constexpr int F_GRAD_G0 = 32;    // end: gradient of gamma_0 (the last reverse pass)

struct Pass {
    int32_t tq[TB];        // global qubit of each tile bit (tile bits 0..3 are qubits 0..3)
    int32_t outer_q[MAX_QUBITS];
    int32_t n_outer;
    uint32_t rot;          // tile bits rotated by this pass's RX
    int32_t layer;
    int32_t flags;
    int32_t slot;          // gradient slot of this pass within its layer (0: low pass)
};

// One (n, p) group of circuits; per-circuit arrays are strided by circuit.
struct Group {
    int n, p, nslots;                 // nslots: passes per layer (1 + group passes)
    float2* psi;                      // [circuit][2^n]           (n > 12)
    float2* lam;
    uint8_t* cut;                     // [circuit][2^n]
    const float2* phase;              // [circuit][layer][256]: D_k for each cut count
    const float2* rx;                 // [circuit][layer]: (cos beta_k, sin beta_k)
    const int2* edges;                // [circuit][max_edges]
    const int32_t* n_edges;           // [circuit]
    int max_edges;
    double* partial;                  // [circuit][1 + 2 p nslots][tiles]: energy, then (param, slot)
    int tiles;                        // tiles per circuit (1 for n <= 12)
};

union Cut16 {  // 16 cut counts, loaded and stored as one aligned 16-byte word
    uint4 v;
    uint8_t b[16];
};

__device__ __forceinline__ uint32_t sw(uint32_t l) { return l ^ ((l >> 4) & 15u); }  // bank-conflict-free slots

__device__ __forceinline__ float2 cmulf(float2 a, float2 b) {
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cmulcf(float2 a, float2 b) {  // conj(a) * b
    return make_float2(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x);
}

// RX(2 beta) on register bit S of 16 amplitudes: (a0, a1) <- (c a0 - i s a1, -i s a0 + c a1).
template <int S>
__device__ __forceinline__ void rx16(float2 (&a)[16], float c, float s) {
#pragma unroll
    for (int j = 0; j < 16; ++j) {
        if (j & (1 << S)) continue;
        const float2 x = a[j], y = a[j | (1 << S)];
        a[j] = make_float2(c * x.x + s * y.y, c * x.y - s * y.x);
        a[j | (1 << S)] = make_float2(c * y.x + s * x.y, c * y.y - s * x.x);
    }
}

// sum over the pairs of register bit S of 2 Im(conj(l0) p1 + conj(l1) p0): 2 Im <lambda| X_q |psi>.
template <int S>
__device__ __forceinline__ double xgrad16(const float2 (&p)[16], const float2 (&l)[16]) {
    float acc = 0.f;
#pragma unroll
    for (int j = 0; j < 16; ++j) {
        if (j & (1 << S)) continue;
        const float2 p0 = p[j], p1 = p[j | (1 << S)], l0 = l[j], l1 = l[j | (1 << S)];
        acc += (l0.x * p1.y - l0.y * p1.x) + (l1.x * p0.y - l1.y * p0.x);
    }
    return 2.0 * (double)acc;
}

__device__ __forceinline__ void rx_masked(float2 (&a)[16], uint32_t m, float c, float s) {
    if (m & 1) rx16<0>(a, c, s);
    if (m & 2) rx16<1>(a, c, s);
    if (m & 4) rx16<2>(a, c, s);
    if (m & 8) rx16<3>(a, c, s);
}
__device__ __forceinline__ double xgrad_masked(const float2 (&p)[16], const float2 (&l)[16], uint32_t m) {
    double g = 0.0;
    if (m & 1) g += xgrad16<0>(p, l);
    if (m & 2) g += xgrad16<1>(p, l);
    if (m & 4) g += xgrad16<2>(p, l);
    if (m & 8) g += xgrad16<3>(p, l);
    return g;
}

// Local tile index of register slot j in round r (register bits = tile bits
// 4r..4r+3) for thread t (its 8 bits fill the other tile bits in order).
__device__ __forceinline__ uint32_t local_index(int r, uint32_t t, uint32_t j) {
    const uint32_t lo_mask = (1u << (4 * r)) - 1u;
    const uint32_t thread_part = (t & lo_mask) | ((t & ~lo_mask) << 4);
    return thread_part | (j << (4 * r));
}

// Global index of local tile index l (tile bits -> qubits tq) plus the tile's base.
__device__ __forceinline__ uint64_t global_index(const Pass& ps, uint32_t l, uint64_t base) {
    uint64_t g = base;
#pragma unroll
    for (int b = 0; b < TB; ++b) g |= (uint64_t)((l >> b) & 1u) << ps.tq[b];
    return g;
}

__device__ __forceinline__ uint64_t tile_base(const Pass& ps, uint64_t tile) {
    uint64_t g = 0;
    for (int k = 0; k < ps.n_outer; ++k) g |= ((tile >> k) & 1ull) << ps.outer_q[k];
    return g;
}

// Cut count of basis state z: edges whose two bits differ.
__device__ __forceinline__ uint32_t cut_of(uint64_t z, const int2* e, int ne) {
    uint32_t c = 0;
    for (int k = 0; k < ne; ++k) c += (uint32_t)(((z >> e[k].x) ^ (z >> e[k].y)) & 1ull);
    return c;
}

// Block sum of v (FP64) in a fixed order; valid in thread 0.
__device__ __forceinline__ double block_sum(double v, double* red) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    __syncthreads();
    if (lane == 0) red[w] = v;
    __syncthreads();
    double s = 0.0;
    if (threadIdx.x == 0)
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) s += red[k];
    return s;
}

// ---- large circuits: one pass per launch ---------------------------------------

// Forward pass over one tile of one circuit (blockIdx.x: tile, blockIdx.y: circuit).
// Four CTAs per SM (64 registers): 2% faster on the 4096-circuit batch than
// three; the reverse pass stays at two (three spill and measured 7% slower).
__global__ void __launch_bounds__(NT, 4) k_qaoa_forward(const Group g, const Pass ps) {
    extern __shared__ float2 dyn_f[];  // tile (TILE amplitudes) | cut counts (TILE bytes)
    float2* sm = dyn_f;
    uint8_t* cs = (uint8_t*)(dyn_f + TILE);
    __shared__ double red[NT / 32];
    const uint32_t t = threadIdx.x;
    const uint64_t c = blockIdx.y, amps = 1ull << g.n;
    float2* psi = g.psi + c * amps;
    float2* lam = g.lam + c * amps;
    uint8_t* cut = g.cut + c * amps;
    const uint64_t base = tile_base(ps, blockIdx.x);
    const float2 rx = g.rx[c * g.p + ps.layer];
    float2 a[16];
    // round 0: tile bits 0..3 = qubits 0..3, 16 contiguous amplitudes
    const uint64_t g0 = global_index(ps, local_index(0, t, 0), base);
    Cut16 cv;
    cv.v = make_uint4(0u, 0u, 0u, 0u);
    if (ps.flags & F_INIT) {
        const float amp0 = (float)(1.0 / sqrt((double)amps));  // H^n |0>
        const int ne = g.n_edges[c];
        const int2* e = g.edges + c * g.max_edges;
#pragma unroll
        for (int j = 0; j < 16; ++j) {
            a[j] = make_float2(amp0, 0.f);
            cv.b[j] = (uint8_t)cut_of(g0 + j, e, ne);
        }
        *(uint4*)(cut + g0) = cv.v;
    } else {
        const float4* src = (const float4*)(psi + g0);
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const float4 v = src[j];
            a[2 * j] = make_float2(v.x, v.y);
            a[2 * j + 1] = make_float2(v.z, v.w);
        }
        if (ps.flags & (F_D_BEFORE | F_D_AFTER | F_ENERGY)) cv.v = *(const uint4*)(cut + g0);
    }
    if (ps.flags & F_D_BEFORE) {
        const float2* ph = g.phase + (c * g.p + ps.layer) * 256;
#pragma unroll
        for (int j = 0; j < 16; ++j) a[j] = cmulf(ph[cv.b[j]], a[j]);
    }
    rx_masked(a, ps.rot & 15u, rx.x, rx.y);
#pragma unroll
    for (int j = 0; j < 16; ++j) sm[sw(local_index(0, t, j))] = a[j];
    ((uint4*)cs)[t] = cv.v;  // local indices 16t..16t+15: one conflict-free 16-byte store
    __syncthreads();
    for (int r = 1; r < 3; ++r) {
#pragma unroll
        for (int j = 0; j < 16; ++j) a[j] = sm[sw(local_index(r, t, j))];
        rx_masked(a, (ps.rot >> (4 * r)) & 15u, rx.x, rx.y);
        if (r == 2) break;  // the last round writes global memory from registers
#pragma unroll
        for (int j = 0; j < 16; ++j) sm[sw(local_index(r, t, j))] = a[j];
        __syncthreads();
    }
    // round 2 layout: tile bits 8..11 in registers, lanes along tile bits 0..4
    double en = 0.0;
    if (ps.flags & F_D_AFTER) {
        const float2* ph = g.phase + (c * g.p + ps.layer + 1) * 256;
#pragma unroll
        for (int j = 0; j < 16; ++j) a[j] = cmulf(ph[cs[local_index(2, t, j)]], a[j]);
    }
#pragma unroll
    for (int j = 0; j < 16; ++j) {
        const uint32_t l = local_index(2, t, j);
        const uint64_t gi = global_index(ps, l, base);
        psi[gi] = a[j];
        if (ps.flags & F_ENERGY) {
            const float cc = (float)cs[l];
            en -= (double)cc * ((double)a[j].x * a[j].x + (double)a[j].y * a[j].y);
            lam[gi] = make_float2(-cc * a[j].x, -cc * a[j].y);
        }
    }
    if (ps.flags & F_ENERGY) {
        const double s = block_sum(en, red);
        if (t == 0) g.partial[c * (1 + 2ull * g.p * g.nslots) * g.tiles + blockIdx.x] = s;
    }
}

// Reverse pass over one tile of one circuit: psi and lambda together.
__global__ void __launch_bounds__(NT) k_qaoa_reverse(const Group g, const Pass ps) {
    extern __shared__ float2 dyn_r[];  // psi tile | lambda tile | cut counts
    float2* smp = dyn_r;
    float2* sml = dyn_r + TILE;
    uint8_t* cs = (uint8_t*)(dyn_r + 2 * TILE);
    __shared__ double red[NT / 32];
    const uint32_t t = threadIdx.x;
    const uint64_t c = blockIdx.y, amps = 1ull << g.n;
    float2* psi = g.psi + c * amps;
    float2* lam = g.lam + c * amps;
    const uint8_t* cut = g.cut + c * amps;
    const uint64_t base = tile_base(ps, blockIdx.x);
    const float2 rx = g.rx[c * g.p + ps.layer];
    const float sneg = -rx.y;  // RX^dagger = RX(-2 beta)
    const int ne = g.n_edges[c];
    float2 p[16], l[16];
    Cut16 cv;
    const uint64_t g0 = global_index(ps, local_index(0, t, 0), base);
    {
        const float4* sp = (const float4*)(psi + g0);
        const float4* sl = (const float4*)(lam + g0);
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const float4 v = sp[j], w = sl[j];
            p[2 * j] = make_float2(v.x, v.y);
            p[2 * j + 1] = make_float2(v.z, v.w);
            l[2 * j] = make_float2(w.x, w.y);
            l[2 * j + 1] = make_float2(w.z, w.w);
        }
        cv.v = *(const uint4*)(cut + g0);
    }
    double g_gamma = 0.0, g_beta = 0.0;
    if (ps.flags & F_UNDO_D) {  // gradient of gamma_(layer+1), then D_(layer+1)^dagger on both
        const float2* ph = g.phase + (c * g.p + ps.layer + 1) * 256;
        float acc = 0.f;
#pragma unroll
        for (int j = 0; j < 16; ++j) {
            const float2 w = cmulcf(l[j], p[j]);
            acc += (float)(ne - 2 * (int)cv.b[j]) * w.y;
            const float2 d = ph[cv.b[j]];
            const float2 dc = make_float2(d.x, -d.y);
            p[j] = cmulf(dc, p[j]);
            l[j] = cmulf(dc, l[j]);
        }
        g_gamma += (double)acc;
    }
    g_beta += xgrad_masked(p, l, ps.rot & 15u);
    rx_masked(p, ps.rot & 15u, rx.x, sneg);
    rx_masked(l, ps.rot & 15u, rx.x, sneg);
#pragma unroll
    for (int j = 0; j < 16; ++j) {
        const uint32_t li = sw(local_index(0, t, j));
        smp[li] = p[j];
        sml[li] = l[j];
    }
    ((uint4*)cs)[t] = cv.v;
    __syncthreads();
    for (int r = 1; r < 3; ++r) {
#pragma unroll
        for (int j = 0; j < 16; ++j) {
            const uint32_t li = sw(local_index(r, t, j));
            p[j] = smp[li];
            l[j] = sml[li];
        }
        const uint32_t m = (ps.rot >> (4 * r)) & 15u;
        g_beta += xgrad_masked(p, l, m);
        rx_masked(p, m, rx.x, sneg);
        rx_masked(l, m, rx.x, sneg);
        if (r == 2) break;
#pragma unroll
        for (int j = 0; j < 16; ++j) {
            const uint32_t li = sw(local_index(r, t, j));
            smp[li] = p[j];
            sml[li] = l[j];
        }
        __syncthreads();
    }
    if (ps.flags & F_GRAD_G0) {  // gradient of gamma_0, after the whole of mixer 0 is undone
        float acc = 0.f;
#pragma unroll
        for (int j = 0; j < 16; ++j) {
            const float2 w = cmulcf(l[j], p[j]);
            acc += (float)(ne - 2 * (int)cs[local_index(2, t, j)]) * w.y;
        }
        g_gamma += (double)acc;
    }
    const bool last = (ps.flags & F_GRAD_G0) != 0;
    if (!last) {  // the last reverse pass's states are not needed again
#pragma unroll
        for (int j = 0; j < 16; ++j) {
            const uint64_t gi = global_index(ps, local_index(2, t, j), base);
            psi[gi] = p[j];
            lam[gi] = l[j];
        }
    }
    const double sb = block_sum(g_beta, red);
    const double sg = block_sum(g_gamma, red);
    if (t == 0) {
        const uint64_t stride = (uint64_t)g.tiles;
        double* part = g.partial + c * (1 + 2ull * g.p * g.nslots) * stride;
        // (param, slot) rows: beta_k at 1 + (2k + 1) nslots + slot, gamma_k at 1 + 2k nslots + slot
        part[(1 + (2ull * ps.layer + 1) * g.nslots + ps.slot) * stride + blockIdx.x] = sb;
        if (ps.flags & F_UNDO_D)
            part[(1 + 2ull * (ps.layer + 1) * g.nslots + 0) * stride + blockIdx.x] = sg;
        if (ps.flags & F_GRAD_G0) part[(1 + 0) * stride + blockIdx.x] = sg;
    }
}

// ---- small circuits: the whole evaluation in one CTA ----------------------------

// Rounds of four qubits covering n <= 12 qubits: round r's register bits are
// qubits 4r..4r+3 taken mod n (a qubit appears once among rotated bits).
template <bool REV>
__device__ void small_mixer(float2* sp, float2* sl, int n, uint32_t t, float c, float s, double* gb) {
    const int rounds = (n + 3) / 4;
    // 2^(n-4) threads hold 16 amplitudes each; the block's other threads (a
    // warp is the smallest block) only pass the same barriers: every thread
    // executes both __syncthreads of every round, at the same instructions.
    const bool active = t < (1u << (n - 4));
    for (int r = 0; r < rounds; ++r) {
        // register bits: qubits q[0..3]; rotated: those < n not yet rotated
        int q[4];
        uint32_t m = 0;
        for (int k = 0; k < 4; ++k) {
            const int qq = 4 * r + k;
            q[k] = qq < n ? qq : (qq - n);  // wrap onto low qubits, not rotated again
            if (qq < n) m |= 1u << k;
        }
        // the thread's bits fill the other n - 4 qubit positions in order
        uint32_t others[TB];
        int no = 0;
        for (int b = 0; b < n; ++b)
            if (b != q[0] && b != q[1] && b != q[2] && b != q[3]) others[no++] = b;
        uint32_t basei = 0;
        for (int k = 0; k < no; ++k) basei |= ((t >> k) & 1u) << others[k];
        uint32_t idx[16];
#pragma unroll
        for (int j = 0; j < 16; ++j) {
            uint32_t v = basei;
#pragma unroll
            for (int k = 0; k < 4; ++k) v |= ((j >> k) & 1u) << q[k];
            idx[j] = v;
        }
        float2 a[16], b[16];
        if (active) {
#pragma unroll
            for (int j = 0; j < 16; ++j) a[j] = sp[idx[j]];
            if (REV) {
#pragma unroll
                for (int j = 0; j < 16; ++j) b[j] = sl[idx[j]];
                *gb += xgrad_masked(a, b, m);
                rx_masked(a, m, c, -s);
                rx_masked(b, m, c, -s);
            } else {
                rx_masked(a, m, c, s);
            }
        }
        __syncthreads();
        if (active) {
#pragma unroll
            for (int j = 0; j < 16; ++j) sp[idx[j]] = a[j];
            if (REV) {
#pragma unroll
                for (int j = 0; j < 16; ++j) sl[idx[j]] = b[j];
            }
        }
        __syncthreads();
    }
}

// One CTA per circuit of 4 <= n <= 12 qubits (max(32, 2^(n-4)) threads).
__global__ void __launch_bounds__(NT) k_qaoa_small(const Group g, double* __restrict__ energy_out,
                                                   double* __restrict__ grad_out) {
    extern __shared__ float2 dyn[];
    __shared__ double red[NT / 32];
    const int n = g.n, p = g.p;
    const uint32_t amps = 1u << n, t = threadIdx.x;
    float2* sp = dyn;
    float2* sl = dyn + amps;
    uint8_t* cs = (uint8_t*)(dyn + 2 * amps);
    const uint64_t c = blockIdx.x;
    const int ne = g.n_edges[c];
    const int2* e = g.edges + c * g.max_edges;
    const float amp0 = (float)(1.0 / sqrt((double)amps));
    for (uint32_t z = t; z < amps; z += blockDim.x) {
        sp[z] = make_float2(amp0, 0.f);
        cs[z] = (uint8_t)cut_of(z, e, ne);
    }
    __syncthreads();
    for (int k = 0; k < p; ++k) {
        const float2* ph = g.phase + (c * p + k) * 256;
        for (uint32_t z = t; z < amps; z += blockDim.x) sp[z] = cmulf(ph[cs[z]], sp[z]);
        __syncthreads();
        const float2 rx = g.rx[c * p + k];
        small_mixer<false>(sp, sl, n, t, rx.x, rx.y, nullptr);
    }
    double en = 0.0;
    for (uint32_t z = t; z < amps; z += blockDim.x) {
        const float2 a = sp[z];
        const float cc = (float)cs[z];
        en -= (double)cc * ((double)a.x * a.x + (double)a.y * a.y);
        sl[z] = make_float2(-cc * a.x, -cc * a.y);
    }
    const double e_sum = block_sum(en, red);
    if (t == 0) energy_out[c] = e_sum;
    __syncthreads();
    for (int k = p - 1; k >= 0; --k) {
        const float2 rx = g.rx[c * p + k];
        double gb = 0.0;
        small_mixer<true>(sp, sl, n, t, rx.x, rx.y, &gb);
        const double sb = block_sum(gb, red);
        if (t == 0) grad_out[c * 2 * p + 2 * k + 1] = sb;
        // gamma_k at the point just after D_k, then undo D_k
        const float2* ph = g.phase + (c * p + k) * 256;
        float acc = 0.f;
        for (uint32_t z = t; z < amps; z += blockDim.x) {
            const float2 w = cmulcf(sl[z], sp[z]);
            acc += (float)(ne - 2 * (int)cs[z]) * w.y;
            if (k > 0) {
                const float2 d = ph[cs[z]];
                const float2 dc = make_float2(d.x, -d.y);
                sp[z] = cmulf(dc, sp[z]);
                sl[z] = cmulf(dc, sl[z]);
            }
        }
        const double sg = block_sum((double)acc, red);
        if (t == 0) grad_out[c * 2 * p + 2 * k] = sg;
        __syncthreads();
    }
}

// Energies and gradients of the large circuits from the per-tile partials, in a
// fixed order: one block per circuit, thread i < 1 + 2p sums row group i.
__global__ void k_qaoa_reduce(const Group g, double* __restrict__ energy_out, double* __restrict__ grad_out) {
    const uint64_t c = blockIdx.x;
    const int rows = 1 + 2 * g.p;
    const uint64_t stride = (uint64_t)g.tiles;
    const double* part = g.partial + c * (1 + 2ull * g.p * g.nslots) * stride;
    for (int i = threadIdx.x; i < rows; i += blockDim.x) {
        double s = 0.0;
        if (i == 0) {
            for (uint64_t k = 0; k < stride; ++k) s += part[k];
            energy_out[c] = s;
        } else {
            const int prm = i - 1;  // gamma_k = 2k, beta_k = 2k + 1
            for (int sl = 0; sl < g.nslots; ++sl)
                for (uint64_t k = 0; k < stride; ++k) s += part[(1 + (uint64_t)prm * g.nslots + sl) * stride + k];
            grad_out[c * 2 * g.p + prm] = s;
        }
    }
}

int qfail(int code, const std::string& msg) {
    gq::set_last_error(msg);
    return code;
}

#define QCUDA(x)                                                                                     \
    do {                                                                                             \
        cudaError_t e_ = (x);                                                                        \
        if (e_ != cudaSuccess) return qfail(GQ_ECUDA, std::string(#x) + ": " + cudaGetErrorString(e_)); \
    } while (0)

struct DevMem {
    void* p = nullptr;
    size_t cap = 0;
    int ensure(size_t b) {
        if (b <= cap) return GQ_OK;
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
        if (cudaMalloc(&p, b) != cudaSuccess) {
            cudaGetLastError();
            return qfail(GQ_ENOMEM, "cudaMalloc of " + std::to_string(b) + " bytes failed");
        }
        cap = b;
        return GQ_OK;
    }
    ~DevMem() {
        if (p) cudaFree(p);
    }
};

// The passes of one (n, p) group with n > 12 (see the header comment).
std::vector<Pass> forward_passes(int n, int p, std::vector<Pass>* reverse) {
    const int high = n - TB, ngroups = (high + 7) / 8, nslots = 1 + ngroups;
    auto make = [&](const std::vector<int>& tq, uint32_t rot, int layer, int flags, int slot) {
        Pass ps{};
        for (int b = 0; b < TB; ++b) ps.tq[b] = tq[b];
        int no = 0;
        for (int q = 0; q < n; ++q)
            if (std::find(tq.begin(), tq.end(), q) == tq.end()) ps.outer_q[no++] = q;
        ps.n_outer = no;
        ps.rot = rot;
        ps.layer = layer;
        ps.flags = flags;
        ps.slot = slot;
        return ps;
    };
    std::vector<int> low(TB);
    for (int b = 0; b < TB; ++b) low[b] = b;
    // group j: tile bits 0..3 = qubits 0..3, 4..(4+len) = the group's qubits, the rest fillers from 4..
    std::vector<std::vector<int>> gtq(ngroups);
    std::vector<uint32_t> grot(ngroups);
    for (int j = 0; j < ngroups; ++j) {
        const int q0 = TB + 8 * j, len = std::min(8, n - q0);
        std::vector<int> tq = {0, 1, 2, 3};
        for (int k = 0; k < len; ++k) tq.push_back(q0 + k);
        for (int f = 4; (int)tq.size() < TB; ++f) tq.push_back(f);
        gtq[j] = tq;
        grot[j] = ((1u << len) - 1u) << 4;
    }
    std::vector<Pass> fwd;
    for (int k = 0; k < p; ++k) {
        for (int j = 0; j < ngroups; ++j) {
            int fl = 0;
            if (k == 0 && j == 0) fl |= F_INIT | F_D_BEFORE;
            fwd.push_back(make(gtq[j], grot[j], k, fl, 1 + j));
        }
        fwd.push_back(make(low, (1u << TB) - 1u, k, k + 1 < p ? F_D_AFTER : F_ENERGY, 0));
    }
    reverse->clear();
    for (int k = p - 1; k >= 0; --k) {
        reverse->push_back(make(low, (1u << TB) - 1u, k, k + 1 < p ? F_UNDO_D : 0, 0));
        for (int j = ngroups - 1; j >= 0; --j)
            reverse->push_back(make(gtq[j], grot[j], k, (k == 0 && j == 0) ? F_GRAD_G0 : 0, 1 + j));
    }
    (void)nslots;
    return fwd;
}


struct PinnedMem {
    void* p = nullptr;
    size_t cap = 0;
    int ensure(size_t b) {
        if (b <= cap) return GQ_OK;
        if (p) cudaFreeHost(p);
        p = nullptr;
        cap = 0;
        if (cudaMallocHost(&p, b) != cudaSuccess) {
            cudaGetLastError();
            return qfail(GQ_ENOMEM, "cudaMallocHost of " + std::to_string(b) + " bytes failed");
        }
        cap = b;
        return GQ_OK;
    }
};

// Buffers and streams reused by later calls on the same device (a call holds
// the workspace's lock, so concurrent calls run one after the other).
struct Workspace {
    std::mutex mu;
    int device = -1;
    cudaStream_t big = nullptr, small = nullptr;  // tile passes | one-CTA circuits
    cudaEvent_t small_done = nullptr;
    DevMem states, in, out;
    PinnedMem host_in, host_out;
    bool attrs = false;
};

Workspace& workspace(int dev) {
    static std::mutex mu;
    static std::map<int, Workspace*> all;  // kept until exit, like the library's other caches
    std::lock_guard<std::mutex> lk(mu);
    Workspace*& w = all[dev];
    if (!w) w = new Workspace();
    return *w;
}

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

}  // namespace

extern "C" int gq_qaoa_maxcut_batch(int precision, const gq_qaoa_item* items, size_t n_items, int want_gradients,
                                    double* energies_out, double* grads_out) {
    if (precision != GQ_C64) return qfail(GQ_EUNSUPPORTED, "qaoa batch: complex64 only (use gq_batch_run)");
    if (n_items && !items) return qfail(GQ_EINVAL, "null items");
    if (n_items && !energies_out) return qfail(GQ_EINVAL, "null energies");
    size_t total_params = 0;
    for (size_t i = 0; i < n_items; ++i) {
        const gq_qaoa_item& it = items[i];
        if (it.num_qubits < 4 || it.num_qubits > MAX_QUBITS)
            return qfail(GQ_EINVAL, "qaoa item " + std::to_string(i) + ": num_qubits out of range [4, 26]");
        if (it.p < 1 || it.p > MAX_LAYERS) return qfail(GQ_EINVAL, "qaoa item " + std::to_string(i) + ": p out of range");
        if (it.n_edges < 1 || it.n_edges > (size_t)MAX_EDGES || !it.edges || !it.gammas || !it.betas)
            return qfail(GQ_EINVAL, "qaoa item " + std::to_string(i) + ": bad edges or angles");
        for (size_t k = 0; k < it.n_edges; ++k) {
            const int a = it.edges[2 * k], b = it.edges[2 * k + 1];
            if (a < 0 || b < 0 || a >= it.num_qubits || b >= it.num_qubits || a == b)
                return qfail(GQ_EINVAL, "qaoa item " + std::to_string(i) + ": edge out of range");
        }
        total_params += 2 * (size_t)it.p;
    }
    if (want_gradients && total_params && !grads_out) return qfail(GQ_EINVAL, "null gradients");
    if (n_items == 0) return GQ_OK;
    int dev = 0;
    QCUDA(cudaGetDevice(&dev));
    Workspace& W = workspace(dev);
    std::lock_guard<std::mutex> lock(W.mu);
    if (!W.big) {
        QCUDA(cudaStreamCreateWithFlags(&W.big, cudaStreamNonBlocking));
        QCUDA(cudaStreamCreateWithFlags(&W.small, cudaStreamNonBlocking));
        QCUDA(cudaEventCreateWithFlags(&W.small_done, cudaEventDisableTiming));
    }
    if (!W.attrs) {
        QCUDA(cudaFuncSetAttribute(k_qaoa_small, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemReverse));
        QCUDA(cudaFuncSetAttribute(k_qaoa_forward, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemForward));
        QCUDA(cudaFuncSetAttribute(k_qaoa_reverse, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemReverse));
        W.attrs = true;
    }
    // groups of equal (n, p)
    std::map<std::pair<int, int>, std::vector<size_t>> groups;
    for (size_t i = 0; i < n_items; ++i) groups[{items[i].num_qubits, items[i].p}].push_back(i);
    std::vector<size_t> grad_off(n_items);
    for (size_t i = 0, o = 0; i < n_items; ++i) {
        grad_off[i] = o;
        o += 2 * (size_t)items[i].p;
    }
    // layout of every group's inputs (one upload), outputs (one download) and states
    struct GL {
        int n, p, nslots, tiles, max_e;
        const std::vector<size_t>* idx;
        size_t o_phase, o_rx, o_edge, o_ne;  // in the input block
        size_t o_e, o_g, o_part, part_rows;  // in the output block
        size_t o_state;                      // in the state block (n > 12)
    };
    std::vector<GL> gl;
    size_t in_bytes = 0, out_bytes = 0, state_bytes = 0;
    for (const auto& kv : groups) {
        GL g{};
        g.n = kv.first.first;
        g.p = kv.first.second;
        g.idx = &kv.second;
        const size_t nc = kv.second.size();
        const uint64_t amps = 1ull << g.n;
        const int ngroups = g.n > TB ? (g.n - TB + 7) / 8 : 0;
        g.nslots = 1 + ngroups;
        g.tiles = g.n > TB ? (int)(amps >> TB) : 1;
        g.max_e = 0;
        for (size_t i : kv.second) g.max_e = std::max(g.max_e, (int)items[i].n_edges);
        g.o_phase = in_bytes;
        in_bytes = align256(in_bytes + nc * g.p * 256 * 8);
        g.o_rx = in_bytes;
        in_bytes = align256(in_bytes + nc * g.p * 8);
        g.o_edge = in_bytes;
        in_bytes = align256(in_bytes + nc * g.max_e * 8);
        g.o_ne = in_bytes;
        in_bytes = align256(in_bytes + nc * 4);
        g.part_rows = 1 + 2ull * g.p * g.nslots;
        g.o_e = out_bytes;
        out_bytes = align256(out_bytes + nc * 8);
        g.o_g = out_bytes;
        out_bytes = align256(out_bytes + nc * 2 * g.p * 8);
        g.o_part = out_bytes;
        if (g.n > TB) out_bytes = align256(out_bytes + nc * g.part_rows * g.tiles * 8);
        g.o_state = state_bytes;
        if (g.n > TB) state_bytes = align256(state_bytes + nc * amps * (8 + 8 + 1));
        gl.push_back(g);
    }
    int rc = W.host_in.ensure(in_bytes);
    if (rc == GQ_OK) rc = W.in.ensure(in_bytes);
    if (rc == GQ_OK) rc = W.out.ensure(out_bytes);
    if (rc == GQ_OK && state_bytes) rc = W.states.ensure(state_bytes);
    if (rc != GQ_OK) return rc;
    // host tables: D_k for every cut count, the mixers' (cos, sin), edges
    char* hin = (char*)W.host_in.p;
    for (const GL& g : gl) {
        float2* phase = (float2*)(hin + g.o_phase);
        float2* rxv = (float2*)(hin + g.o_rx);
        int2* edges = (int2*)(hin + g.o_edge);
        int32_t* ne = (int32_t*)(hin + g.o_ne);
        for (size_t ci = 0; ci < g.idx->size(); ++ci) {
            const gq_qaoa_item& it = items[(*g.idx)[ci]];
            ne[ci] = (int32_t)it.n_edges;
            for (size_t k = 0; k < it.n_edges; ++k)
                edges[ci * g.max_e + k] = make_int2(it.edges[2 * k], it.edges[2 * k + 1]);
            for (int k = 0; k < g.p; ++k) {
                // D_k(C) = exp(-i gamma (|E| - 2 C) / 2): the product of the layer's RZZ(gamma)
                const double gm = it.gammas[k];
                for (int cc = 0; cc <= (int)it.n_edges; ++cc) {  // cut counts reach |E| at most
                    const double ang = -gm * ((double)it.n_edges - 2.0 * cc) / 2.0;
                    phase[(ci * g.p + k) * 256 + cc] = make_float2((float)std::cos(ang), (float)std::sin(ang));
                }
                rxv[ci * g.p + k] = make_float2((float)std::cos(it.betas[k]), (float)std::sin(it.betas[k]));
            }
        }
    }
    QCUDA(cudaMemcpyAsync(W.in.p, hin, in_bytes, cudaMemcpyHostToDevice, W.big));
    QCUDA(cudaEventRecord(W.small_done, W.big));
    QCUDA(cudaStreamWaitEvent(W.small, W.small_done, 0));  // the small stream needs the inputs too
    const char* din = (const char*)W.in.p;
    char* dout = (char*)W.out.p;
    bool any_small = false;
    for (const GL& g : gl) {
        const size_t nc = g.idx->size();
        const uint64_t amps = 1ull << g.n;
        Group gr{};
        gr.n = g.n;
        gr.p = g.p;
        gr.nslots = g.nslots;
        gr.phase = (const float2*)(din + g.o_phase);
        gr.rx = (const float2*)(din + g.o_rx);
        gr.edges = (const int2*)(din + g.o_edge);
        gr.n_edges = (const int32_t*)(din + g.o_ne);
        gr.max_edges = g.max_e;
        gr.tiles = g.tiles;
        double* d_e = (double*)(dout + g.o_e);
        double* d_g = (double*)(dout + g.o_g);
        if (g.n <= TB) {  // whole circuits in one CTA, beside the tile passes
            const unsigned threads = std::max(32u, 1u << (g.n - 4));
            k_qaoa_small<<<(unsigned)nc, threads, 2 * 8 * amps + amps, W.small>>>(gr, d_e, d_g);
            any_small = true;
        } else {
            gr.psi = (float2*)((char*)W.states.p + g.o_state);
            gr.lam = gr.psi + nc * amps;
            gr.cut = (uint8_t*)(gr.lam + nc * amps);
            gr.partial = (double*)(dout + g.o_part);
            QCUDA(cudaMemsetAsync(gr.partial, 0, nc * g.part_rows * g.tiles * 8, W.big));
            std::vector<Pass> rev;
            const std::vector<Pass> fwd = forward_passes(g.n, g.p, &rev);
            const dim3 grid((unsigned)g.tiles, (unsigned)nc);
            for (const Pass& ps : fwd) k_qaoa_forward<<<grid, NT, kSmemForward, W.big>>>(gr, ps);
            if (want_gradients)
                for (const Pass& ps : rev) k_qaoa_reverse<<<grid, NT, kSmemReverse, W.big>>>(gr, ps);
            k_qaoa_reduce<<<(unsigned)nc, 64, 0, W.big>>>(gr, d_e, d_g);
        }
        QCUDA(cudaGetLastError());
    }
    if (any_small) {
        QCUDA(cudaEventRecord(W.small_done, W.small));
        QCUDA(cudaStreamWaitEvent(W.big, W.small_done, 0));
    }
    rc = W.host_out.ensure(out_bytes);
    if (rc != GQ_OK) return rc;
    QCUDA(cudaMemcpyAsync(W.host_out.p, dout, out_bytes, cudaMemcpyDeviceToHost, W.big));
    QCUDA(cudaStreamSynchronize(W.big));
    const char* hout = (const char*)W.host_out.p;
    for (const GL& g : gl)
        for (size_t ci = 0; ci < g.idx->size(); ++ci) {
            const size_t i = (*g.idx)[ci];
            energies_out[i] = ((const double*)(hout + g.o_e))[ci];
            if (want_gradients)
                std::memcpy(grads_out + grad_off[i], (const double*)(hout + g.o_g) + ci * 2 * g.p, 2 * g.p * 8);
        }
    return GQ_OK;
}

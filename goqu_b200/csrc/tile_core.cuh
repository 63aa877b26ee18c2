// Tile-pass core shared by the sm_100a kernel and the host emulator.
//
// A pass streams the state through the SMs once. Each CTA owns a tile of 2^m
// amplitudes: the amplitudes whose index bits outside the pass's m tile qubits
// equal the CTA's base. The tile is staged in shared memory under an XOR
// swizzle; the pass then runs "phases": in each phase every thread holds 16
// amplitudes in registers, spanning 4 register qubits, and applies the gates
// of that phase to them (controls and diagonal factors may sit on any qubit,
// since every amplitude's global index is known). Phases exchange data through
// shared memory. Everything the device needs (tile qubits, swizzle columns,
// per-phase index tables, ops, matrices) comes from a program the host
// scheduler emits, so the code below is pure index arithmetic plus complex
// FMAs and is compiled both for sm_100a and for the host emulator.
#pragma once
#if !defined(__CUDACC_RTC__)
#include <math.h>
#include <stdint.h>
#endif

#if defined(__CUDACC__)
#define GQ_HD __host__ __device__ __forceinline__
#else
#define GQ_HD inline
#endif

namespace gq {

constexpr int RQ = 4;          // register qubits per thread
constexpr int NREG = 1 << RQ;  // amplitudes per thread
constexpr int MAX_TILE = 13;   // tile qubits (2^13 amplitudes per CTA)
constexpr int MAX_QUBITS = 48; // physical qubits of a state (DM: 2n)

template <class T>
struct alignas(2 * sizeof(T)) cplx {
    T x, y;
};

template <class T>
GQ_HD cplx<T> cmul(cplx<T> a, cplx<T> b) {
    return {a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x};
}
template <class T>
GQ_HD cplx<T> cfma(cplx<T> m, cplx<T> a, cplx<T> acc) {  // acc + m*a
    acc.x = acc.x + m.x * a.x;
    acc.x = acc.x - m.y * a.y;
    acc.y = acc.y + m.x * a.y;
    acc.y = acc.y + m.y * a.x;
    return acc;
}

enum KType : uint8_t {
    K_NONE = 0,
    K_U1 = 1,    // dense 2x2 on register bit t0
    K_U2 = 2,    // dense 4x4 on register bits t0 < t1 (t0 is local index bit 0)
    K_U3 = 3,    // dense 8x8 on t0 < t1 < t2
    K_U4 = 4,    // dense 16x16 on all four register bits
    K_X = 5,     // [[0,p0],[p1,0]] on t0 (pure swap when flags & 1)
    K_SWAP = 6,  // swap of register bits t0 < t1
    K_DIAG = 7,  // diagonal factor d[index]; index = pext(g, dmask) << nreg | ridx[j]
    K_PHASE = 8, // scalar factor when all controls are set
    K_RESET = 9, // deterministic reset of register bit t0 (sim/statevector/sim.go:168-186)
    K_GRAD = 10, // adjoint: Re <lambda| G |psi> into gradient slot `slot`; flags = the
                 // structure of G (K_U1..K_U4 dense on t0.., K_DIAG, K_PHASE, K_PAIRSUM)
    K_PAIRSUM = 11, // nreg = K qubit pairs: factor T[c] where c is the number of pairs
                    // whose two bits differ at the amplitude (a run of identical
                    // parity-symmetric 2-qubit diagonals, e.g. the RZZ(gamma) of a QAOA
                    // layer). Pool: K pair codes (re, im = code of each qubit: register
                    // bit 0..3, or 16 + global qubit), then T[0..K].
};

constexpr int MAX_GRAD_SLOTS = 64;  // gradient ops per pass

// One op as placed in a phase (40 bytes).
struct KOp {
    uint8_t type;
    uint8_t t0, t1, t2;  // target register bits, ascending
    uint8_t creg;        // control register bits (all must be 1)
    uint8_t nreg;        // K_DIAG: register-bit part of the table index
    uint8_t flags;
    uint8_t pad;
    uint32_t mat;        // offset into the complex pool
    uint32_t slot;       // K_GRAD: gradient slot of the pass
    uint64_t cmask;      // controls outside the registers (global mask)
    uint64_t dmask;      // K_DIAG: diagonal qubits outside the registers (global mask)
    uint64_t ridx;       // K_DIAG: 4-bit register part of the index for each slot j
};

// Thread bits of a phase: thread t's shared-memory base and global-index base
// are XOR / OR of per-bit columns, tabulated for the low 4 and high 5 bits of t.
constexpr int TLO = 16, THI = 32;

struct PhaseDesc {
    int32_t op_begin, op_end;
    uint32_t rslot[NREG];      // shared-memory slot offset of register slot j
    uint32_t tlo_slot[TLO];    // slot base of thread bits 0..3
    uint32_t thi_slot[THI];    // slot base of thread bits 4..8
    uint64_t tlo_glob[TLO];    // global index base of thread bits 0..3
    uint64_t thi_glob[THI];    // global index base of thread bits 4..8
};

struct PassDesc {
    int32_t m;        // tile qubits
    int32_t n_phases;
    int32_t phase0;   // first PhaseDesc of this pass
    int32_t n_outer;  // qubits outside the tile (CTA index bits)
    uint32_t acol[MAX_TILE];     // shared-memory slot of tile bit b (linear staging)
    int32_t tile_q[MAX_TILE];    // global qubit of tile bit b (ascending)
    int32_t outer_q[MAX_QUBITS]; // global qubit of CTA-index bit k
};

// Read-only load of a complex constant (all threads of a CTA read the same
// program data, so these are broadcasts through the L1 cache).
GQ_HD cplx<double> ldc(const cplx<double>* p, uint32_t i) {
#if defined(__CUDA_ARCH__)
    const double2 v = __ldg(reinterpret_cast<const double2*>(p + i));
    return {v.x, v.y};
#else
    return p[i];
#endif
}
GQ_HD cplx<float> ldc(const cplx<float>* p, uint32_t i) {
#if defined(__CUDA_ARCH__)
    const float2 v = __ldg(reinterpret_cast<const float2*>(p + i));
    return {v.x, v.y};
#else
    return p[i];
#endif
}

// Same load, but not merged or hoisted by the compiler: used where a matrix
// is too large to keep in registers across the unrolled amplitude groups.
GQ_HD cplx<double> ldc_v(const cplx<double>* p, uint32_t i) {
#if defined(__CUDA_ARCH__)
    double x, y;
    asm volatile("ld.global.nc.v2.f64 {%0, %1}, [%2];" : "=d"(x), "=d"(y) : "l"(p + i));
    return {x, y};
#else
    return p[i];
#endif
}
GQ_HD cplx<float> ldc_v(const cplx<float>* p, uint32_t i) {
#if defined(__CUDA_ARCH__)
    float x, y;
    asm volatile("ld.global.nc.v2.f32 {%0, %1}, [%2];" : "=f"(x), "=f"(y) : "l"(p + i));
    return {x, y};
#else
    return p[i];
#endif
}

// Asynchronous global -> shared copy of one amplitude (cp.async; persistent
// specialised kernels prefetch their next tile while the current one
// finishes). Host code copies directly.
#if defined(__CUDA_ARCH__)
__device__ __forceinline__ void cp_async_amp(cplx<double>* dst, const cplx<double>* src) {
    const uint32_t d = (uint32_t)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_amp(cplx<float>* dst, const cplx<float>* src) {
    const uint32_t d = (uint32_t)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
// Waits until every committed copy of this thread has landed.
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }
#endif

// Matrix held in kernel parameter space (the specialised pass kernels pass
// each pass's matrices by value): indexed with compile-time offsets, so the
// entries become constant-bank operands.
template <class T>
struct PMat {
    const cplx<T>* p;
};
template <class T>
GQ_HD cplx<T> ldc(PMat<T> m, uint32_t i) {
    return m.p[i];
}
template <class T>
GQ_HD cplx<T> ldc_v(PMat<T> m, uint32_t i) {
    return m.p[i];
}

GQ_HD uint64_t pext64(uint64_t v, uint64_t mask) {
    uint64_t r = 0;
    int k = 0;
    while (mask) {
#if defined(__CUDA_ARCH__)
        int b = __ffsll((long long)mask) - 1;
#else
        int b = __builtin_ctzll(mask);
#endif
        r |= ((v >> b) & 1ull) << k;
        ++k;
        mask &= mask - 1;
    }
    return r;
}

// ---- register-level gate bodies (S* are register bits, compile-time) -------

template <class T, int S, bool C, class MP>
GQ_HD void k_u1(cplx<T> (&a)[NREG], MP m, uint32_t creg) {
    const cplx<T> m0 = ldc(m, 0), m1 = ldc(m, 1), m2 = ldc(m, 2), m3 = ldc(m, 3);
#pragma unroll
    for (int j = 0; j < NREG; ++j) {
        if (j & (1 << S)) continue;
        if (C && (j & creg) != creg) continue;
        const cplx<T> a0 = a[j], a1 = a[j | (1 << S)];
        cplx<T> o0 = {T(0), T(0)}, o1 = {T(0), T(0)};
        o0 = cfma(m0, a0, o0);
        o0 = cfma(m1, a1, o0);
        o1 = cfma(m2, a0, o1);
        o1 = cfma(m3, a1, o1);
        a[j] = o0;
        a[j | (1 << S)] = o1;
    }
}

// The same for a real matrix (only the real parts of m are read): each
// output takes two real multiply-adds per component instead of four.
template <class T, int S, bool C, class MP>
GQ_HD void k_u1r(cplx<T> (&a)[NREG], MP m, uint32_t creg) {
    const T m0 = ldc(m, 0).x, m1 = ldc(m, 1).x, m2 = ldc(m, 2).x, m3 = ldc(m, 3).x;
#pragma unroll
    for (int j = 0; j < NREG; ++j) {
        if (j & (1 << S)) continue;
        if (C && (j & creg) != creg) continue;
        const cplx<T> a0 = a[j], a1 = a[j | (1 << S)];
        a[j] = {m0 * a0.x + m1 * a1.x, m0 * a0.y + m1 * a1.y};
        a[j | (1 << S)] = {m2 * a0.x + m3 * a1.x, m2 * a0.y + m3 * a1.y};
    }
}

template <class T, int S0, int S1, bool C, class MP>
GQ_HD void k_u2(cplx<T> (&a)[NREG], MP m, uint32_t creg) {
#pragma unroll
    for (int j = 0; j < NREG; ++j) {
        if (j & ((1 << S0) | (1 << S1))) continue;
        if (C && (j & creg) != creg) continue;
        const int idx[4] = {j, j | (1 << S0), j | (1 << S1), j | (1 << S0) | (1 << S1)};
        cplx<T> v[4];
#pragma unroll
        for (int c = 0; c < 4; ++c) v[c] = a[idx[c]];
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            cplx<T> o = {T(0), T(0)};
#pragma unroll
            for (int c = 0; c < 4; ++c) o = cfma(ldc_v(m, r * 4 + c), v[c], o);
            a[idx[r]] = o;
        }
    }
}

// A real 4x4 matrix (only the real parts of m are read).
template <class T, int S0, int S1, bool C, class MP>
GQ_HD void k_u2r(cplx<T> (&a)[NREG], MP m, uint32_t creg) {
#pragma unroll
    for (int j = 0; j < NREG; ++j) {
        if (j & ((1 << S0) | (1 << S1))) continue;
        if (C && (j & creg) != creg) continue;
        const int idx[4] = {j, j | (1 << S0), j | (1 << S1), j | (1 << S0) | (1 << S1)};
        cplx<T> v[4];
#pragma unroll
        for (int c = 0; c < 4; ++c) v[c] = a[idx[c]];
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            T ox = T(0), oy = T(0);
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                const T mr = ldc_v(m, r * 4 + c).x;
                ox += mr * v[c].x;
                oy += mr * v[c].y;
            }
            a[idx[r]] = {ox, oy};
        }
    }
}

template <class T, int S0, int S1, int S2, class MP>
GQ_HD void k_u3(cplx<T> (&a)[NREG], MP m, uint32_t creg) {
#pragma unroll
    for (int j = 0; j < NREG; ++j) {
        if (j & ((1 << S0) | (1 << S1) | (1 << S2))) continue;
        if ((j & creg) != creg) continue;
        int idx[8];
#pragma unroll
        for (int c = 0; c < 8; ++c)
            idx[c] = j | ((c & 1) ? (1 << S0) : 0) | ((c & 2) ? (1 << S1) : 0) | ((c & 4) ? (1 << S2) : 0);
        cplx<T> v[8];
#pragma unroll
        for (int c = 0; c < 8; ++c) v[c] = a[idx[c]];
#pragma unroll
        for (int r = 0; r < 8; ++r) {
            cplx<T> o = {T(0), T(0)};
#pragma unroll
            for (int c = 0; c < 8; ++c) o = cfma(ldc_v(m, r * 8 + c), v[c], o);
            a[idx[r]] = o;
        }
    }
}

// 16x16 on all register bits. Four output rows at a time, each summed in two
// interleaved partial sums (16 independent FMA chains); the outputs go to the
// thread's own shared-memory slots, so only the 16 inputs stay in registers,
// and are read back at the end (no other thread touches those slots in this
// phase).
template <class T, class MP>
GQ_HD void k_u4(cplx<T> (&a)[NREG], MP m, cplx<T>* sm, uint32_t sbase, const uint32_t* rslot) {
#pragma unroll 1
    for (int r0 = 0; r0 < NREG; r0 += 4) {
        cplx<T> o[4], e[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) o[q] = e[q] = cplx<T>{T(0), T(0)};
#pragma unroll
        for (int c = 0; c < NREG; c += 2) {
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                o[q] = cfma(ldc_v(m, (r0 + q) * NREG + c), a[c], o[q]);
                e[q] = cfma(ldc_v(m, (r0 + q) * NREG + c + 1), a[c + 1], e[q]);
            }
        }
#pragma unroll
        for (int q = 0; q < 4; ++q) sm[sbase ^ rslot[r0 + q]] = cplx<T>{o[q].x + e[q].x, o[q].y + e[q].y};
    }
#pragma unroll
    for (int r = 0; r < NREG; ++r) a[r] = sm[sbase ^ rslot[r]];
}

template <class T, int S, bool C, class MP>
GQ_HD void k_x(cplx<T> (&a)[NREG], MP m, uint32_t creg, bool pure) {
    if (pure) {
#pragma unroll
        for (int j = 0; j < NREG; ++j) {
            if (j & (1 << S)) continue;
            if (C && (j & creg) != creg) continue;
            const cplx<T> t = a[j];
            a[j] = a[j | (1 << S)];
            a[j | (1 << S)] = t;
        }
        return;
    }
    const cplx<T> p0 = ldc(m, 0), p1 = ldc(m, 1);
#pragma unroll
    for (int j = 0; j < NREG; ++j) {
        if (j & (1 << S)) continue;
        if (C && (j & creg) != creg) continue;
        const cplx<T> a0 = a[j], a1 = a[j | (1 << S)];
        a[j] = cmul(p0, a1);
        a[j | (1 << S)] = cmul(p1, a0);
    }
}

// Shear [[1, -t], [t, 1]] on register bit S (t real): the rotation part of a
// one-qubit unitary once its phases and cos(theta/2) are factored out (the
// specialised kernels keep those as pending per-slot factors).
template <class T, int S, bool C>
GQ_HD void k_shear(cplx<T> (&a)[NREG], T t, uint32_t creg) {
#pragma unroll
    for (int j = 0; j < NREG; ++j) {
        if (j & (1 << S)) continue;
        if (C && (j & creg) != creg) continue;
        const cplx<T> a0 = a[j], a1 = a[j | (1 << S)];
        a[j] = {a0.x - t * a1.x, a0.y - t * a1.y};
        a[j | (1 << S)] = {a1.x + t * a0.x, a1.y + t * a0.y};
    }
}

template <class T, int S0, int S1>
GQ_HD void k_swap(cplx<T> (&a)[NREG], uint32_t creg) {
#pragma unroll
    for (int j = 0; j < NREG; ++j) {
        if (!(j & (1 << S0)) || (j & (1 << S1))) continue;  // j has S0=1, S1=0
        if ((j & creg) != creg) continue;
        const int k = (j & ~(1 << S0)) | (1 << S1);
        const cplx<T> t = a[j];
        a[j] = a[k];
        a[k] = t;
    }
}

template <class T, int S>
GQ_HD void k_reset(cplx<T> (&a)[NREG]) {
#pragma unroll
    for (int j = 0; j < NREG; ++j) {
        if (j & (1 << S)) continue;
        const cplx<T> a0 = a[j], a1 = a[j | (1 << S)];
        const T s = a0.x * a0.x + a0.y * a0.y + a1.x * a1.x + a1.y * a1.y;
#if defined(__CUDA_ARCH__)
        const T norm = sqrt(s);
#else
        const T norm = (T)__builtin_sqrt((double)s);
#endif
        a[j] = norm > T(1e-15) ? cplx<T>{norm, T(0)} : cplx<T>{T(0), T(0)};
        a[j | (1 << S)] = {T(0), T(0)};
    }
}

// Diagonal with its table index's global part `hi` already extracted.
template <class T>
GQ_HD void k_diag_hi(cplx<T> (&a)[NREG], const cplx<T>* d, uint32_t hi, uint32_t nreg, uint32_t creg,
                     uint64_t ridx) {
    if (nreg == 0) {
        const cplx<T> f = ldc(d, hi);
        if (f.x == T(1) && f.y == T(0)) return;
#pragma unroll
        for (int j = 0; j < NREG; ++j)
            if ((j & creg) == creg) a[j] = cmul(f, a[j]);
        return;
    }
#pragma unroll
    for (int j = 0; j < NREG; ++j) {
        if ((j & creg) != creg) continue;
        const uint32_t idx = hi | (uint32_t)((ridx >> (4 * j)) & 15u);
        a[j] = cmul(ldc(d, idx), a[j]);
    }
}

template <class T>
GQ_HD void k_diag(cplx<T> (&a)[NREG], const KOp& op, const cplx<T>* d, uint64_t g0) {
    k_diag_hi<T>(a, d, (uint32_t)(pext64(g0, op.dmask) << op.nreg), op.nreg, op.creg, op.ridx);
}

template <class T>
GQ_HD void k_phase(cplx<T> (&a)[NREG], const cplx<T> s, uint32_t creg) {
#pragma unroll
    for (int j = 0; j < NREG; ++j)
        if ((j & creg) == creg) a[j] = cmul(s, a[j]);
}

// Per-slot counts of a K_PAIRSUM's odd pairs, one byte per register slot
// (slots 0..7 in lo, 8..15 in hi). slot_bits(r, h): byte j = bit r of slot j
// (h: of j + 8).
GQ_HD uint64_t slot_bits(int r, bool h) {
    return r == 0 ? 0x0100010001000100ull
                  : (r == 1 ? 0x0101000001010000ull : (r == 2 ? 0x0101010100000000ull : (h ? 0x0101010101010101ull : 0ull)));
}

GQ_HD uint32_t popc64(uint64_t v) {
#if defined(__CUDA_ARCH__)
    return (uint32_t)__popcll(v);
#else
    return (uint32_t)__builtin_popcountll(v);
#endif
}

// The op's data, classified on the host (all values small integers, exact in
// FP32), then its factor table T[0..K]:
//   d[0..1], d[2..3]: lo and hi counts of the pairs on two register bits, as
//     16-bit chunks (fixed per slot);
//   d[4 + 2r], d[5 + 2r]: pairs of register bit r with global qubits: their
//     qubit mask M_r (three 16-bit chunks) and number n_r. Slots with bit r
//     set differ from the pairs whose qubit bit of g0 is 0 (n_r - m_r of
//     them, m_r = popcount(g0 & M_r)), slots with bit r clear from the m_r
//     others;
//   d[12].x = G pairs of two global qubits, packed q0 | q1 << 6, two per
//     entry from d[13]: they add the same count to every slot.
// Returns the factor table.
template <class T>
GQ_HD const cplx<T>* pair_counts(const cplx<T>* d, uint64_t g0, uint64_t& lo, uint64_t& hi) {
    auto u = [](T v) { return (uint64_t)(uint32_t)v; };
    lo = u(d[0].x) | (u(d[0].y) << 16) | (u(d[1].x) << 32) | (u(d[1].y) << 48);
    hi = u(d[2].x) | (u(d[2].y) << 16) | (u(d[3].x) << 32) | (u(d[3].y) << 48);
    constexpr uint64_t ONES = 0x0101010101010101ull;
#pragma unroll
    for (int r = 0; r < RQ; ++r) {
        const cplx<T> c0 = d[4 + 2 * r], c1 = d[5 + 2 * r];
        const uint64_t n = u(c1.y);
        if (n == 0) continue;
        const uint64_t M = u(c0.x) | (u(c0.y) << 16) | (u(c1.x) << 32);
        const uint64_t m = popc64(g0 & M);
        const uint64_t sl = slot_bits(r, false), sh = slot_bits(r, true);
        lo += (n - m) * sl + m * (ONES - sl);
        hi += (n - m) * sh + m * (ONES - sh);
    }
    const uint32_t G = (uint32_t)d[12].x;
    uint64_t ng = 0;
    for (uint32_t k = 0; k < G; ++k) {
        const cplx<T> c = d[13 + (k >> 1)];
        const uint32_t pq = (uint32_t)((k & 1) ? c.y : c.x);
        ng += ((g0 >> (pq & 63u)) ^ (g0 >> (pq >> 6))) & 1ull;
    }
    lo += ng * ONES;
    hi += ng * ONES;
    return d + 13 + ((G + 1) >> 1);
}

// The factor table of a K_PAIRSUM's data (after its classified pairs).
template <class T>
GQ_HD const cplx<T>* pair_counts_table(const cplx<T>* d) {
    return d + 13 + (((uint32_t)d[12].x + 1) >> 1);
}

GQ_HD uint32_t slot_count(uint64_t lo, uint64_t hi, int j) {
    return (uint32_t)(((j < 8 ? lo : hi) >> (8 * (j & 7))) & 0xffull);
}

// The pair sum's factor T[c] per slot, given its counts.
template <class T>
GQ_HD void k_pairsum_lh(cplx<T> (&a)[NREG], const cplx<T>* table, uint64_t lo, uint64_t hi) {
#pragma unroll
    for (int j = 0; j < NREG; ++j) a[j] = cmul(ldc(table, slot_count(lo, hi, j)), a[j]);
}

template <class T>
GQ_HD void k_pairsum(cplx<T> (&a)[NREG], const cplx<T>* d, uint64_t g0) {
    uint64_t lo, hi;
    const cplx<T>* table = pair_counts<T>(d, g0, lo, hi);
    k_pairsum_lh<T>(a, table, lo, hi);
}

// Decodes one op and hands its body to `each`: each(body) calls body(a, sm)
// with a thread's 16 amplitudes and its shared-memory tile (U4's scratch).
// g0 is the global index of the thread's register slot 0 (its thread bits
// and the CTA's base).
template <class T, class Each>
GQ_HD void dispatch_op(const KOp& op, const cplx<T>* pool, uint64_t g0, uint32_t sbase, const uint32_t* rslot,
                       Each each) {
    if ((g0 & op.cmask) != op.cmask) return;
    const cplx<T>* m = pool + op.mat;
    const uint32_t creg = op.creg;
    switch (op.type) {
        case K_U1:
            if (creg == 0) {
                switch (op.t0) {
                    case 0: each([&](cplx<T>(&x)[NREG], cplx<T>*) { k_u1<T, 0, false>(x, m, 0); }); break;
                    case 1: each([&](cplx<T>(&x)[NREG], cplx<T>*) { k_u1<T, 1, false>(x, m, 0); }); break;
                    case 2: each([&](cplx<T>(&x)[NREG], cplx<T>*) { k_u1<T, 2, false>(x, m, 0); }); break;
                    default: each([&](cplx<T>(&x)[NREG], cplx<T>*) { k_u1<T, 3, false>(x, m, 0); }); break;
                }
            } else {
                switch (op.t0) {
                    case 0: each([&](cplx<T>(&x)[NREG], cplx<T>*) { k_u1<T, 0, true>(x, m, creg); }); break;
                    case 1: each([&](cplx<T>(&x)[NREG], cplx<T>*) { k_u1<T, 1, true>(x, m, creg); }); break;
                    case 2: each([&](cplx<T>(&x)[NREG], cplx<T>*) { k_u1<T, 2, true>(x, m, creg); }); break;
                    default: each([&](cplx<T>(&x)[NREG], cplx<T>*) { k_u1<T, 3, true>(x, m, creg); }); break;
                }
            }
            break;
        case K_U2:
            if (creg == 0) {
                switch (op.t0 * 4 + op.t1) {
                    case 1: each([&](cplx<T>(&x)[NREG], cplx<T>*) { k_u2<T, 0, 1, false>(x, m, 0); }); break;
                    case 2: each([&](cplx<T>(&x)[NREG], cplx<T>*) { k_u2<T, 0, 2, false>(x, m, 0); }); break;
                    case 3: each([&](cplx<T>(&x)[NREG], cplx<T>*) { k_u2<T, 0, 3, false>(x, m, 0); }); break;
                    case 6: each([&](cplx<T>(&x)[NREG], cplx<T>*) { k_u2<T, 1, 2, false>(x, m, 0); }); break;
                    case 7: each([&](cplx<T>(&x)[NREG], cplx<T>*) { k_u2<T, 1, 3, false>(x, m, 0); }); break;
                    default: each([&](cplx<T>(&x)[NREG], cplx<T>*) { k_u2<T, 2, 3, false>(x, m, 0); }); break;
                }
            } else {
                switch (op.t0 * 4 + op.t1) {
                    case 1: each([&](cplx<T>(&x)[NREG], cplx<T>*) { k_u2<T, 0, 1, true>(x, m, creg); }); break;
                    case 2: each([&](cplx<T>(&x)[NREG], cplx<T>*) { k_u2<T, 0, 2, true>(x, m, creg); }); break;
                    case 3: each([&](cplx<T>(&x)[NREG], cplx<T>*) { k_u2<T, 0, 3, true>(x, m, creg); }); break;
                    case 6: each([&](cplx<T>(&x)[NREG], cplx<T>*) { k_u2<T, 1, 2, true>(x, m, creg); }); break;
                    case 7: each([&](cplx<T>(&x)[NREG], cplx<T>*) { k_u2<T, 1, 3, true>(x, m, creg); }); break;
                    default: each([&](cplx<T>(&x)[NREG], cplx<T>*) { k_u2<T, 2, 3, true>(x, m, creg); }); break;
                }
            }
            break;
        case K_U3:
            switch (op.t0 * 16 + op.t1 * 4 + op.t2) {
                case 0 * 16 + 1 * 4 + 2: each([&](cplx<T>(&x)[NREG], cplx<T>*) { k_u3<T, 0, 1, 2>(x, m, creg); }); break;
                case 0 * 16 + 1 * 4 + 3: each([&](cplx<T>(&x)[NREG], cplx<T>*) { k_u3<T, 0, 1, 3>(x, m, creg); }); break;
                case 0 * 16 + 2 * 4 + 3: each([&](cplx<T>(&x)[NREG], cplx<T>*) { k_u3<T, 0, 2, 3>(x, m, creg); }); break;
                default: each([&](cplx<T>(&x)[NREG], cplx<T>*) { k_u3<T, 1, 2, 3>(x, m, creg); }); break;
            }
            break;
        case K_U4:
            each([&](cplx<T>(&x)[NREG], cplx<T>* xs) { k_u4<T>(x, m, xs, sbase, rslot); });
            break;
        case K_X: {
            const bool pure = op.flags & 1;
            if (creg == 0) {
                switch (op.t0) {
                    case 0: each([&](cplx<T>(&x)[NREG], cplx<T>*) { k_x<T, 0, false>(x, m, 0, pure); }); break;
                    case 1: each([&](cplx<T>(&x)[NREG], cplx<T>*) { k_x<T, 1, false>(x, m, 0, pure); }); break;
                    case 2: each([&](cplx<T>(&x)[NREG], cplx<T>*) { k_x<T, 2, false>(x, m, 0, pure); }); break;
                    default: each([&](cplx<T>(&x)[NREG], cplx<T>*) { k_x<T, 3, false>(x, m, 0, pure); }); break;
                }
            } else {
                switch (op.t0) {
                    case 0: each([&](cplx<T>(&x)[NREG], cplx<T>*) { k_x<T, 0, true>(x, m, creg, pure); }); break;
                    case 1: each([&](cplx<T>(&x)[NREG], cplx<T>*) { k_x<T, 1, true>(x, m, creg, pure); }); break;
                    case 2: each([&](cplx<T>(&x)[NREG], cplx<T>*) { k_x<T, 2, true>(x, m, creg, pure); }); break;
                    default: each([&](cplx<T>(&x)[NREG], cplx<T>*) { k_x<T, 3, true>(x, m, creg, pure); }); break;
                }
            }
            break;
        }
        case K_SWAP:
            switch (op.t0 * 4 + op.t1) {
                case 1: each([&](cplx<T>(&x)[NREG], cplx<T>*) { k_swap<T, 0, 1>(x, creg); }); break;
                case 2: each([&](cplx<T>(&x)[NREG], cplx<T>*) { k_swap<T, 0, 2>(x, creg); }); break;
                case 3: each([&](cplx<T>(&x)[NREG], cplx<T>*) { k_swap<T, 0, 3>(x, creg); }); break;
                case 6: each([&](cplx<T>(&x)[NREG], cplx<T>*) { k_swap<T, 1, 2>(x, creg); }); break;
                case 7: each([&](cplx<T>(&x)[NREG], cplx<T>*) { k_swap<T, 1, 3>(x, creg); }); break;
                default: each([&](cplx<T>(&x)[NREG], cplx<T>*) { k_swap<T, 2, 3>(x, creg); }); break;
            }
            break;
        case K_DIAG:
            each([&](cplx<T>(&x)[NREG], cplx<T>*) { k_diag<T>(x, op, m, g0); });
            break;
        case K_PHASE:
            each([&](cplx<T>(&x)[NREG], cplx<T>*) { k_phase<T>(x, ldc(m, 0), creg); });
            break;
        case K_PAIRSUM:
            each([&](cplx<T>(&x)[NREG], cplx<T>*) { k_pairsum<T>(x, m, g0); });
            break;
        case K_RESET:
            switch (op.t0) {
                case 0: each([&](cplx<T>(&x)[NREG], cplx<T>*) { k_reset<T, 0>(x); }); break;
                case 1: each([&](cplx<T>(&x)[NREG], cplx<T>*) { k_reset<T, 1>(x); }); break;
                case 2: each([&](cplx<T>(&x)[NREG], cplx<T>*) { k_reset<T, 2>(x); }); break;
                default: each([&](cplx<T>(&x)[NREG], cplx<T>*) { k_reset<T, 3>(x); }); break;
            }
            break;
        default:
            break;
    }
}

// Applies one op to the thread's 16 amplitudes.
template <class T>
GQ_HD void apply_op(cplx<T> (&a)[NREG], const KOp& op, const cplx<T>* pool, uint64_t g0, cplx<T>* sm,
                    uint32_t sbase, const uint32_t* rslot) {
    dispatch_op<T>(op, pool, g0, sbase, rslot, [&](auto body) { body(a, sm); });
}

// Global index base of a CTA: bit k of the CTA index goes to outer_q[k].
GQ_HD uint64_t cta_base(const PassDesc& p, uint64_t cta) {
    uint64_t g = 0;
    for (int k = 0; k < p.n_outer; ++k) g |= ((cta >> k) & 1ull) << p.outer_q[k];
    return g;
}

// Linear staging: element it*TPB + t of the tile. Returns its global index
// offset (without the CTA base) and its shared-memory slot.
GQ_HD void linear_slot(const PassDesc& p, uint32_t lin, uint64_t& goff, uint32_t& slot) {
    uint64_t g = 0;
    uint32_t s = 0;
    for (int b = 0; b < p.m; ++b)
        if ((lin >> b) & 1u) {
            g |= 1ull << p.tile_q[b];
            s ^= p.acol[b];
        }
    goff = g;
    slot = s;
}

// One thread's work in one phase: gather 16 amplitudes from the staged tile,
// apply the phase's ops, scatter them back. Threads of a phase touch disjoint
// slots, so phases only need a barrier between them.
template <class T>
GQ_HD void run_phase(cplx<T>* sm, const PhaseDesc& ph, const KOp* ops, const cplx<T>* pool, uint32_t t,
                     uint64_t base) {
    const uint32_t sbase = ph.tlo_slot[t & (TLO - 1)] ^ ph.thi_slot[(t >> 4) & (THI - 1)];
    const uint64_t g0 = base | ph.tlo_glob[t & (TLO - 1)] | ph.thi_glob[(t >> 4) & (THI - 1)];
    cplx<T> a[NREG];
#pragma unroll
    for (int j = 0; j < NREG; ++j) a[j] = sm[sbase ^ ph.rslot[j]];
    const int ob = ph.op_begin, oe = ph.op_end;
    for (int o = ob; o < oe; ++o) apply_op<T>(a, ops[o], pool, g0, sm, sbase, ph.rslot);
#pragma unroll
    for (int j = 0; j < NREG; ++j) sm[sbase ^ ph.rslot[j]] = a[j];
}

// ---- adjoint differentiation ----------------------------------------------


template <class T>
GQ_HD double cdot_re(cplx<T> b, cplx<T> v) {  // Re(conj(b) * v) in FP64
    return (double)b.x * (double)v.x + (double)b.y * (double)v.y;
}
// complex64: the product of two FP32 amplitudes is formed in FP32 (one fused
// multiply-add, the precision of the amplitudes) and the sums over
// amplitudes accumulate in FP64.
GQ_HD double cdot_re(cplx<float> b, cplx<float> v) { return (double)fmaf(b.x, v.x, b.y * v.y); }

// Gradient partials with the op's fields as arguments (the specialised dual
// kernels pass literals; grad_partial below passes the op record's).
template <class T>
GQ_HD double dot_re_creg(const cplx<T> (&b)[NREG], const cplx<T> (&v)[NREG], uint32_t creg) {
    double acc = 0.0;
#pragma unroll
    for (int j = 0; j < NREG; ++j)
        if ((j & creg) == creg) acc += cdot_re(b[j], v[j]);
    return acc;
}

template <class T>
GQ_HD double grad_phase_c(const cplx<T> (&a)[NREG], const cplx<T> (&b)[NREG], cplx<T> sc, uint32_t creg) {
    double acc = 0.0;
#pragma unroll
    for (int j = 0; j < NREG; ++j)
        if ((j & creg) == creg) acc += cdot_re(b[j], cmul(sc, a[j]));
    return acc;
}

template <class T>
GQ_HD double grad_diag_c(const cplx<T> (&a)[NREG], const cplx<T> (&b)[NREG], const cplx<T>* d, uint32_t hi,
                         uint32_t creg, uint64_t ridx) {
    double acc = 0.0;
#pragma unroll
    for (int j = 0; j < NREG; ++j) {
        if ((j & creg) != creg) continue;
        const uint32_t idx = hi | (uint32_t)((ridx >> (4 * j)) & 15u);
        acc += cdot_re(b[j], cmul(ldc(d, idx), a[j]));
    }
    return acc;
}

// G = [[0, p0], [p1, 0]] on register bit S (a Pauli-X generator such as
// RX's -i/2 X): sum over the pairs of Re(conj(b_0) p0 a_1 + conj(b_1) p1 a_0).
template <class T, int S>
GQ_HD double grad_x_c(const cplx<T> (&a)[NREG], const cplx<T> (&b)[NREG], cplx<T> p0, cplx<T> p1, uint32_t creg) {
    double acc = 0.0;
#pragma unroll
    for (int j = 0; j < NREG; ++j) {
        if ((j & (1 << S)) || (j & creg) != creg) continue;
        acc += cdot_re(b[j], cmul(p0, a[j | (1 << S)])) + cdot_re(b[j | (1 << S)], cmul(p1, a[j]));
    }
    return acc;
}

template <class T>
GQ_HD double grad_pairsum_lh(const cplx<T> (&a)[NREG], const cplx<T> (&b)[NREG], const cplx<T>* table, uint64_t lo,
                             uint64_t hi) {
    double acc = 0.0;
#pragma unroll
    for (int j = 0; j < NREG; ++j) acc += cdot_re(b[j], cmul(ldc(table, slot_count(lo, hi, j)), a[j]));
    return acc;
}

template <class T>
GQ_HD double grad_pairsum_c(const cplx<T> (&a)[NREG], const cplx<T> (&b)[NREG], const cplx<T>* d, uint64_t g0) {
    uint64_t lo, hi;
    const cplx<T>* table = pair_counts<T>(d, g0, lo, hi);
    return grad_pairsum_lh<T>(a, b, table, lo, hi);
}

// Re sum_j conj(lambda_j) (G psi)_j over the thread's amplitudes, G being the
// op's matrix restricted to the amplitudes whose controls are set (zero
// elsewhere). a = psi, b = lambda; neither is modified.
template <class T>
GQ_HD double grad_partial(const cplx<T> (&a)[NREG], const cplx<T> (&b)[NREG], const KOp& op, const cplx<T>* pool,
                          uint64_t g0) {
    if ((g0 & op.cmask) != op.cmask) return 0.0;
    const cplx<T>* m = pool + op.mat;
    const uint32_t creg = op.creg;
    switch (op.flags) {
        case K_PHASE:
            return grad_phase_c<T>(a, b, ldc(m, 0), creg);
        case K_DIAG:
            return grad_diag_c<T>(a, b, m, (uint32_t)(pext64(g0, op.dmask) << op.nreg), creg, op.ridx);
        case K_PAIRSUM:  // G = sum of the pairs' generators: T[c] per slot
            return grad_pairsum_c<T>(a, b, m, g0);
        case K_X: {
            const cplx<T> p0 = ldc(m, 0), p1 = ldc(m, 1);
            switch (op.t0) {
                case 0: return grad_x_c<T, 0>(a, b, p0, p1, creg);
                case 1: return grad_x_c<T, 1>(a, b, p0, p1, creg);
                case 2: return grad_x_c<T, 2>(a, b, p0, p1, creg);
                default: return grad_x_c<T, 3>(a, b, p0, p1, creg);
            }
        }
        default: {
            // dense G on the target register bits: apply it to a copy of psi
            // (the amplitudes whose controls are unset keep psi's values and
            // are excluded from the sum)
            return 0.0;
        }
    }
}

template <class T>
GQ_HD double grad_partial_dense(const cplx<T> (&a)[NREG], const cplx<T> (&b)[NREG], const KOp& op,
                                const cplx<T>* pool, uint64_t g0, cplx<T>* sm, uint32_t sbase, const uint32_t* rslot) {
    if ((g0 & op.cmask) != op.cmask) return 0.0;
    KOp d = op;
    d.type = op.flags;
    d.cmask = 0;
    cplx<T> v[NREG];
#pragma unroll
    for (int j = 0; j < NREG; ++j) v[j] = a[j];
    apply_op<T>(v, d, pool, g0, sm, sbase, rslot);
    double acc = 0.0;
    const uint32_t creg = op.creg;
#pragma unroll
    for (int j = 0; j < NREG; ++j)
        if ((j & creg) == creg) acc += cdot_re(b[j], v[j]);
    return acc;
}

template <class T>
GQ_HD void load_regs(cplx<T> (&a)[NREG], const cplx<T>* sm, uint32_t sbase, const uint32_t* rslot) {
#pragma unroll
    for (int j = 0; j < NREG; ++j) a[j] = sm[sbase ^ rslot[j]];
}
template <class T>
GQ_HD void store_regs(const cplx<T> (&a)[NREG], cplx<T>* sm, uint32_t sbase, const uint32_t* rslot) {
#pragma unroll
    for (int j = 0; j < NREG; ++j) sm[sbase ^ rslot[j]] = a[j];
}

// One thread's work in one phase of an adjoint (reverse) pass: the same ops
// are applied to psi (tile sm_a) and lambda (tile sm_b); gradient ops return
// their partial sums through `grad(slot, value)`.
template <class T, class Grad>
GQ_HD void run_phase_dual(cplx<T>* sm_a, cplx<T>* sm_b, const PhaseDesc& ph, const KOp* ops, const cplx<T>* pool,
                          uint32_t t, uint64_t base, Grad grad) {
    const uint32_t sbase = ph.tlo_slot[t & (TLO - 1)] ^ ph.thi_slot[(t >> 4) & (THI - 1)];
    const uint64_t g0 = base | ph.tlo_glob[t & (TLO - 1)] | ph.thi_glob[(t >> 4) & (THI - 1)];
    cplx<T> a[NREG], b[NREG];
    load_regs(a, sm_a, sbase, ph.rslot);
    load_regs(b, sm_b, sbase, ph.rslot);
    const int ob = ph.op_begin, oe = ph.op_end;
    // Pair sums: counts computed once for both states, and once for a
    // gradient pair sum and the unitary one after it (KOp.flags bit 1).
    uint64_t plo = 0, phi = 0;
    const cplx<T>* ptab = nullptr;
    bool pcount = false;
    for (int o = ob; o < oe; ++o) {
        const KOp& op = ops[o];
        if (op.type == K_GRAD) {
            double v;
            if (op.flags == K_PAIRSUM) {
                ptab = pair_counts<T>(pool + op.mat, g0, plo, phi);
                pcount = true;
                v = grad_pairsum_lh<T>(a, b, ptab, plo, phi);
            } else {
                pcount = false;
                v = (op.flags == K_PHASE || op.flags == K_DIAG || op.flags == K_X)
                        ? grad_partial<T>(a, b, op, pool, g0)
                        : grad_partial_dense<T>(a, b, op, pool, g0, sm_a, sbase, ph.rslot);
            }
            grad(op.slot, v);
            continue;
        }
        if (op.type == K_PAIRSUM) {
            // the unitary's own table: its data has the same pair layout as the gradient's
            const cplx<T>* tab = pair_counts_table<T>(pool + op.mat);
            if (!((op.flags & 2) && pcount)) pair_counts<T>(pool + op.mat, g0, plo, phi);
            pcount = true;
            k_pairsum_lh<T>(a, tab, plo, phi);
            k_pairsum_lh<T>(b, tab, plo, phi);
            continue;
        }
        pcount = false;
        // Each state decodes the op on its own: one decode for both holds
        // both states' operands live at once and measured slower (register
        // pressure). U4 spills through the thread's own slots of each tile.
        apply_op<T>(a, op, pool, g0, sm_a, sbase, ph.rslot);
        apply_op<T>(b, op, pool, g0, sm_b, sbase, ph.rslot);
    }
    store_regs(a, sm_a, sbase, ph.rslot);
    store_regs(b, sm_b, sbase, ph.rslot);
}

}  // namespace gq
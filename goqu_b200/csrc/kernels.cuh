// sm_100a kernels of the engine: the tile pass, probability / sampling
// kernels and FP64 reductions (expectations, density-matrix traces).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "tile_core.cuh"

namespace gq {

// ---------------------------------------------------------------------------
// Tile pass: one CTA per tile, 2^(m-4) threads, 2^m amplitudes of shared memory.
// The CTA stages its tile (16 coalesced loads per thread), runs the pass's
// phases with a barrier between them, and writes the tile back in place.
// Launch shapes. THREADS = 2^(m-4) bounds the tile size of a variant; MINB is
// the CTAs per SM the register allocation is sized for (65536 / (THREADS *
// MINB) registers per thread).
struct TileVariant {
    int threads, min_blocks;
};
constexpr TileVariant kVariantsC128[] = {{128, 3}, {128, 4}, {256, 2}, {64, 6}};
constexpr TileVariant kVariantsC64[] = {{256, 2}, {128, 4}, {512, 1}, {128, 3}};
constexpr int kNumVariants = 4;

// One CTA's share of a pass over the state `st` (CTA index `cta` of pass pd).
template <class T>
__device__ __forceinline__ void tile_pass_body(cplx<T>* __restrict__ st, const PassDesc& pd,
                                               const PhaseDesc* __restrict__ phases, const KOp* __restrict__ ops,
                                               const cplx<T>* __restrict__ pool, uint64_t cta, cplx<T>* sm) {
    const int m = pd.m;
    const int tbits = m - RQ;
    const uint32_t t = threadIdx.x;
    const uint64_t base = cta_base(pd, cta);

    // Linear staging index lin = it * 2^tbits + t: thread bits are tile bits
    // [0, tbits), `it` supplies tile bits [tbits, m).
    uint64_t gt = 0;
    uint32_t stt = 0;
    for (int b = 0; b < tbits; ++b)
        if ((t >> b) & 1u) {
            gt |= 1ull << pd.tile_q[b];
            stt ^= pd.acol[b];
        }
    uint64_t gq[RQ];
    uint32_t sq[RQ];
#pragma unroll
    for (int k = 0; k < RQ; ++k) {
        gq[k] = 1ull << pd.tile_q[tbits + k];
        sq[k] = pd.acol[tbits + k];
    }
    {
        cplx<T> v[NREG];
#pragma unroll
        for (int it = 0; it < NREG; ++it) {
            uint64_t g = base | gt;
#pragma unroll
            for (int k = 0; k < RQ; ++k)
                if ((it >> k) & 1) g |= gq[k];
            v[it] = st[g];
        }
#pragma unroll
        for (int it = 0; it < NREG; ++it) {
            uint32_t s = stt;
#pragma unroll
            for (int k = 0; k < RQ; ++k)
                if ((it >> k) & 1) s ^= sq[k];
            sm[s] = v[it];
        }
    }
    __syncthreads();
    const int nph = pd.n_phases;
    for (int p = 0; p < nph; ++p) {
        run_phase<T>(sm, phases[pd.phase0 + p], ops, pool, t, base);
        __syncthreads();
    }
#pragma unroll
    for (int k = 0; k < RQ; ++k) {
        gq[k] = 1ull << pd.tile_q[tbits + k];
        sq[k] = pd.acol[tbits + k];
    }
    {
        cplx<T> v[NREG];
#pragma unroll
        for (int it = 0; it < NREG; ++it) {
            uint32_t s = stt;
#pragma unroll
            for (int k = 0; k < RQ; ++k)
                if ((it >> k) & 1) s ^= sq[k];
            v[it] = sm[s];
        }
#pragma unroll
        for (int it = 0; it < NREG; ++it) {
            uint64_t g = base | gt;
#pragma unroll
            for (int k = 0; k < RQ; ++k)
                if ((it >> k) & 1) g |= gq[k];
            st[g] = v[it];
        }
    }
}

template <class T, int THREADS, int MINB>
__global__ void __launch_bounds__(THREADS, MINB)
    k_tile_pass(cplx<T>* __restrict__ st, const PassDesc* __restrict__ pdp, const PhaseDesc* __restrict__ phases,
                const KOp* __restrict__ ops, const cplx<T>* __restrict__ pool) {
    extern __shared__ __align__(16) unsigned char smraw[];
    tile_pass_body<T>(st, *pdp, phases, ops, pool, blockIdx.x, reinterpret_cast<cplx<T>*>(smraw));
}

// A batch of independent states. A batched launch runs one pass of many
// states: descriptor d (state, pass) takes 2^n_outer consecutive blocks.
// Descriptors with the same CTA count form a run, so block b finds its
// descriptor arithmetically after a scan over the launch's few runs.
struct BDesc {
    uint64_t state;  // first amplitude of the state
    uint64_t part0;  // reverse passes: its gradient partials start here (cta * nslots + slot)
    uint32_t pass;
    uint32_t nslots;
};
struct BRun {
    uint32_t block0;     // first block of the run in the launch
    uint32_t desc0;      // its first descriptor
    uint32_t log2_ctas;  // CTAs per descriptor
    uint32_t pad;
};

__device__ __forceinline__ BDesc batch_desc(const BRun* __restrict__ runs, int nruns, const BDesc* __restrict__ descs,
                                            uint32_t b, uint32_t& cta) {
    int r = 0;
    while (r + 1 < nruns && runs[r + 1].block0 <= b) ++r;
    const BRun R = runs[r];
    const uint32_t off = b - R.block0;
    cta = off & ((1u << R.log2_ctas) - 1u);
    return descs[R.desc0 + (off >> R.log2_ctas)];
}

template <class T, int THREADS, int MINB>
__global__ void __launch_bounds__(THREADS, MINB)
    k_tile_pass_batch(cplx<T>* __restrict__ states, const BRun* __restrict__ runs, int nruns,
                      const BDesc* __restrict__ descs, const PassDesc* __restrict__ passes,
                      const PhaseDesc* __restrict__ phases, const KOp* __restrict__ ops,
                      const cplx<T>* __restrict__ pool) {
    extern __shared__ __align__(16) unsigned char smraw[];
    uint32_t cta;
    const BDesc d = batch_desc(runs, nruns, descs, blockIdx.x, cta);
    tile_pass_body<T>(states + d.state, passes[d.pass], phases, ops, pool, cta, reinterpret_cast<cplx<T>*>(smraw));
}

// ---------------------------------------------------------------------------
// Adjoint reverse pass: the tile pass on two states (psi, lambda) at once,
// with gradient ops. Each warp writes its sum for every gradient slot once
// per pass into shared memory; the CTA's per-slot totals go to
// partial[cta * nslots + slot] (summed per slot by k_slot_sums).
template <class T>
__device__ __forceinline__ void adjoint_pass_body(cplx<T>* __restrict__ psi, cplx<T>* __restrict__ lam,
                                                  const PassDesc& pd, const PhaseDesc* __restrict__ phases,
                                                  const KOp* __restrict__ ops, const cplx<T>* __restrict__ pool,
                                                  uint64_t cta, double* __restrict__ partial_out, int nslots,
                                                  unsigned char* smraw) {
    const int m = pd.m;
    const int tbits = m - RQ;
    cplx<T>* sa = reinterpret_cast<cplx<T>*>(smraw);
    cplx<T>* sb = sa + (1u << m);
    double* gsm = reinterpret_cast<double*>(sb + (1u << m));  // [warps][MAX_GRAD_SLOTS]
    const uint32_t t = threadIdx.x;
    const uint64_t base = cta_base(pd, cta);
    uint64_t gt = 0;
    uint32_t stt = 0;
    for (int b = 0; b < tbits; ++b)
        if ((t >> b) & 1u) {
            gt |= 1ull << pd.tile_q[b];
            stt ^= pd.acol[b];
        }
    for (int it = 0; it < NREG; ++it) {
        uint64_t g = base | gt;
        uint32_t s = stt;
        for (int k = 0; k < RQ; ++k)
            if ((it >> k) & 1) {
                g |= 1ull << pd.tile_q[tbits + k];
                s ^= pd.acol[tbits + k];
            }
        sa[s] = psi[g];
        sb[s] = lam[g];
    }
    const int nwarps = (int)((blockDim.x + 31) >> 5);
    for (int i = (int)t; i < nwarps * MAX_GRAD_SLOTS; i += (int)blockDim.x) gsm[i] = 0.0;
    __syncthreads();
    const int warp = t >> 5, lane = t & 31;
    // Tiles below 2^9 amplitudes have fewer than 32 threads: reduce over the
    // lanes that exist (the mask of a shuffle must name only live lanes).
    const unsigned nlanes = blockDim.x < 32 ? blockDim.x : 32u;
    const unsigned lanes = nlanes == 32 ? 0xffffffffu : ((1u << nlanes) - 1u);
    // A slot is a parameter of the pass: consecutive gradient ops of one
    // parameter (every RZZ of a QAOA layer, say) add up in a register, and
    // the warp reduces once per run (all lanes call grad() in the same order).
    double acc = 0.0;
    int cur = -1;
    auto flush = [&]() {
        if (cur < 0) return;
        double v = acc;
        for (unsigned o = 16; o > 0; o >>= 1) {
            const double y = __shfl_xor_sync(lanes, v, o);
            if ((lane ^ o) < (int)nlanes) v += y;
        }
        if (lane == 0) gsm[warp * MAX_GRAD_SLOTS + cur] += v;
        acc = 0.0;
        cur = -1;
    };
    auto grad = [&](uint32_t slot, double v) {
        if ((int)slot != cur) {
            flush();
            cur = (int)slot;
        }
        acc += v;
    };
    for (int p = 0; p < pd.n_phases; ++p) {
        run_phase_dual<T>(sa, sb, phases[pd.phase0 + p], ops, pool, t, base, grad);
        flush();
        __syncthreads();
    }
    for (int it = 0; it < NREG; ++it) {
        uint64_t g = base | gt;
        uint32_t s = stt;
        for (int k = 0; k < RQ; ++k)
            if ((it >> k) & 1) {
                g |= 1ull << pd.tile_q[tbits + k];
                s ^= pd.acol[tbits + k];
            }
        psi[g] = sa[s];
        lam[g] = sb[s];
    }
    __syncthreads();
    for (int sl = (int)t; sl < nslots; sl += (int)blockDim.x) {  // tiles may have fewer threads than slots
        double tot = 0.0;
        for (int w = 0; w < nwarps; ++w) tot += gsm[w * MAX_GRAD_SLOTS + sl];
        partial_out[sl] = tot;
    }
}

template <class T, int THREADS, int MINB>
__global__ void __launch_bounds__(THREADS, MINB)
    k_adjoint_pass(cplx<T>* __restrict__ psi, cplx<T>* __restrict__ lam, const PassDesc* __restrict__ pdp,
                   const PhaseDesc* __restrict__ phases, const KOp* __restrict__ ops, const cplx<T>* __restrict__ pool,
                   double* __restrict__ partial, int nslots) {
    extern __shared__ __align__(16) unsigned char smraw[];
    adjoint_pass_body<T>(psi, lam, *pdp, phases, ops, pool, blockIdx.x, partial + (uint64_t)blockIdx.x * nslots,
                         nslots, smraw);
}

// Batched reverse passes: CTA c of descriptor d writes its gradient partials
// to partial[d.part0 + c * d.nslots .. + d.nslots].
template <class T, int THREADS, int MINB>
__global__ void __launch_bounds__(THREADS, MINB)
    k_adjoint_pass_batch(cplx<T>* __restrict__ psi, cplx<T>* __restrict__ lam, const BRun* __restrict__ runs,
                         int nruns, const BDesc* __restrict__ descs, const PassDesc* __restrict__ passes,
                         const PhaseDesc* __restrict__ phases, const KOp* __restrict__ ops,
                         const cplx<T>* __restrict__ pool, double* __restrict__ partial) {
    extern __shared__ __align__(16) unsigned char smraw[];
    uint32_t cta;
    const BDesc d = batch_desc(runs, nruns, descs, blockIdx.x, cta);
    adjoint_pass_body<T>(psi + d.state, lam + d.state, passes[d.pass], phases, ops, pool, cta,
                         partial + d.part0 + (uint64_t)cta * d.nslots, (int)d.nslots, smraw);
}

// Gradient reduction of many reverse passes at once: block s sums slot s
// over its pass's CTAs, partial[off[s] + c * stride[s]] for c < nctas[s],
// into sums[s]; then k_param_sums adds 2 x (the sums of each parameter's
// slots, in slot order) to grad[param]. Both orders are fixed
// (deterministic).
__global__ void k_slot_sums(const double* __restrict__ partial, const uint64_t* __restrict__ off,
                            const uint64_t* __restrict__ nctas, const uint32_t* __restrict__ stride,
                            double* __restrict__ sums) {
    const uint64_t s = blockIdx.x;
    double v = 0.0;
    for (uint64_t c = threadIdx.x; c < nctas[s]; c += blockDim.x) v += partial[off[s] + c * stride[s]];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    __shared__ double red[32];
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double tot = 0.0;
        for (unsigned w = 0; w < (blockDim.x >> 5); ++w) tot += red[w];
        sums[s] = tot;
    }
}

__global__ void k_param_sums(const double* __restrict__ sums, const int* __restrict__ slot_param, int nslots,
                             int nparams, double* __restrict__ grad) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= nparams) return;
    double acc = 0.0;
    bool any = false;
    for (int s = 0; s < nslots; ++s)
        if (slot_param[s] == p) {
            acc += sums[s];
            any = true;
        }
    if (any) grad[p] += 2.0 * acc;
}

template <class T>
__global__ void k_set_amp(cplx<T>* st, uint64_t idx, T re, T im) {
    st[idx] = {re, im};
}

// ---------------------------------------------------------------------------
// Probabilities. p = re*re + im*im with each product and the sum rounded
// separately (no FMA contraction), the arithmetic of goqu's probabilities()
// (sim/statevector/sim.go:274-280) compiled by Go on amd64.
__device__ __forceinline__ double prob_of(cplx<double> a) {
    return __dadd_rn(__dmul_rn(a.x, a.x), __dmul_rn(a.y, a.y));
}
__device__ __forceinline__ double prob_of(cplx<float> a) {
    const double x = a.x, y = a.y;
    return __dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y));
}

template <class T>
struct ProbState {
    const cplx<T>* st;
    __device__ __forceinline__ double operator()(uint64_t i) const { return prob_of(st[i]); }
};
struct ProbArray {
    const double* p;
    __device__ __forceinline__ double operator()(uint64_t i) const { return p[i]; }
};

template <class T>
__global__ void k_probs(const cplx<T>* __restrict__ st, uint64_t n, double* __restrict__ out) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        out[i] = prob_of(st[i]);
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Per-chunk probability sums (chunk = 2^chunk_log entries, one CTA each).
template <class P>
__global__ void k_chunk_sums(P prob, uint64_t n, int chunk_log, double* __restrict__ sums) {
    const uint64_t c0 = (uint64_t)blockIdx.x << chunk_log;
    const uint64_t len = (uint64_t)1 << chunk_log;
    double s = 0.0;
    for (uint64_t j = threadIdx.x; j < len; j += blockDim.x)
        if (c0 + j < n) s += prob(c0 + j);
    s = warp_sum(s);
    __shared__ double ws[32];
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        double v = threadIdx.x < (blockDim.x >> 5) ? ws[threadIdx.x] : 0.0;
        v = warp_sum(v);
        if (threadIdx.x == 0) sums[blockIdx.x] = v;
    }
}

// Inclusive prefix of the chunk sums (single CTA of 1024 threads).
__global__ void k_scan_chunks(const double* __restrict__ sums, uint64_t nchunks, double* __restrict__ incl) {
    __shared__ double part[1024];
    const uint64_t per = (nchunks + blockDim.x - 1) / blockDim.x;
    const uint64_t b = threadIdx.x * per, e = b + per < nchunks ? b + per : nchunks;
    double s = 0.0;
    for (uint64_t c = b; c < e; ++c) s += sums[c];
    part[threadIdx.x] = s;
    __syncthreads();
    if (threadIdx.x == 0) {  // 1024 sequential adds, negligible
        double acc = 0.0;
        for (unsigned i = 0; i < blockDim.x; ++i) {
            const double v = part[i];
            part[i] = acc;
            acc += v;
        }
    }
    __syncthreads();
    double acc = part[threadIdx.x];
    for (uint64_t c = b; c < e; ++c) {
        acc += sums[c];
        incl[c] = acc;
    }
}

// ---------------------------------------------------------------------------
// Exact inverse-CDF sampling.
//
// goqu's sampleIndex (sim/statevector/sim.go:288-298) scans cum += p_j in FP64
// and returns the first j with r < cum. The sum is reproduced exactly here
// without a 2^n-long dependency chain: while the running sum s stays in one
// binade [2^e, 2^(e+1)), every step rounds s + p_j to the grid u = 2^(e-52),
// so s advances by an integer number of grid steps, round-to-nearest(p_j / u)
// (an exact-half tie would depend on the parity of s: such chunks are handled
// sequentially). A chunk whose running sum stays inside one binade therefore
// advances s by u * (an exact int64 sum of per-element steps). Chunks that
// start at zero, straddle a binade boundary or contain a tie (a few dozen at
// most) are summed sequentially with the same FP64 additions as goqu.
//   k_chunk_sums / k_scan_chunks: approximate chunk-end sums (FP64 tree),
//       used only to predict each chunk's binade;
//   k_chunk_steps: per chunk, the exact int64 step count for the predicted
//       binade (or "not clean");
//   k_chunk_walk: one thread walks the chunks with the exact running sum,
//       taking clean chunks in O(1) and the others element by element;
//   k_sample_find: per shot, a binary search on the exact chunk ends and an
//       exact sequential scan inside the chunk.
__device__ __forceinline__ int exponent_of(double x) { return ilogb(x); }

template <class P>
__global__ void k_chunk_steps(P prob, uint64_t n, int chunk_log, const double* __restrict__ incl,
                              long long* __restrict__ steps, int* __restrict__ cexp, int* __restrict__ clean) {
    const uint64_t c = blockIdx.x;
    const double s0 = c ? incl[c - 1] : 0.0, s1 = incl[c];
    // Predicted binade of the whole chunk: that of the approximate sum before
    // it, with the chunk's end kept below the binade's top by a margin far
    // above the error of the approximate sums (~1e-12 relative).
    // (The walk checks the exact running sum's binade and end, so a wrong
    // prediction only sends the chunk to the element-by-element path; s0 on
    // a power of two, as after a basis state, is the common case that must
    // stay clean.)
    bool ok = s0 > 0x1p-1000;
    int e = 0;
    if (ok) {
        e = exponent_of(s0);
        const double hi = ldexp(1.0, e + 1);
        ok = s1 <= hi * (1.0 - 0x1p-30);
    }
    if (!ok) {
        if (threadIdx.x == 0) {
            steps[c] = 0;
            cexp[c] = e;
            clean[c] = 0;
        }
        return;
    }
    const uint64_t c0 = c << chunk_log;
    const uint64_t len = (uint64_t)1 << chunk_log;
    long long sum = 0;
    int tie = 0;
    for (uint64_t j = threadIdx.x; j < len; j += blockDim.x) {
        if (c0 + j >= n) break;
        const double q = ldexp(prob(c0 + j), 52 - e);  // exact: a power-of-two scaling
        const double f = floor(q);
        const double fr = q - f;                       // exact
        long long k = (long long)f;
        if (fr > 0.5) ++k;
        if (fr == 0.5) tie = 1;
        sum += k;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        sum += __shfl_xor_sync(0xffffffffu, sum, o);
        tie |= __shfl_xor_sync(0xffffffffu, tie, o);
    }
    __shared__ long long ws[32];
    __shared__ int wt[32];
    if ((threadIdx.x & 31) == 0) {
        ws[threadIdx.x >> 5] = sum;
        wt[threadIdx.x >> 5] = tie;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        long long t = 0;
        int ti = 0;
        for (unsigned w = 0; w < (blockDim.x >> 5); ++w) {
            t += ws[w];
            ti |= wt[w];
        }
        steps[c] = t;
        cexp[c] = e;
        clean[c] = !ti;
    }
}

// One warp walks the chunks with the exact running sum s, a window of
// 32 x kWalkK chunks at a time (kWalkK consecutive chunks per lane, loaded
// together). A chunk is taken in O(1) when it is clean in s's binade and
// s plus its exact step count stays below 2^(e+1): the ends of the window's
// leading run of such chunks are s plus the int64 window prefix times the
// ulp of the binade (exact). The first chunk after that run is summed in
// sub-chunks of 64 elements with the same rule, now against the exact s: a
// sub-chunk whose elements all round without a tie in s's binade and whose
// end stays below 2^(e+1) adds its int64 step count times the ulp; any other
// sub-chunk is summed element by element with goqu's own additions (every
// lane adds the 64 elements in order, so s stays warp-uniform). Then the
// next window starts after the chunk.
constexpr int kWalkK = 8;
constexpr int kSubChunk = 64;

template <class P>
__global__ void k_chunk_walk(P prob, uint64_t n, int chunk_log, const long long* __restrict__ steps,
                             const int* __restrict__ cexp, const int* __restrict__ clean, uint64_t nchunks,
                             double* __restrict__ ends, int* __restrict__ n_seq) {
    if (blockIdx.x != 0 || threadIdx.x >= 32) return;
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x;
    constexpr int W = 32 * kWalkK;
    double s = 0.0;
    int seq = 0;
    const uint64_t len = (uint64_t)1 << chunk_log;
    uint64_t c = 0;
    while (c < nchunks) {
        const bool pos = s > 0.0;
        const int se = pos ? exponent_of(s) : 0;
        const double lim = pos ? ldexp(1.0, se + 1) : 0.0;
        // ulp of s's binade; run * ulp equals ldexp(run, se - 52) exactly (a
        // power-of-two scaling; it is only used for clean chunks, whose
        // binade has se >= -1000)
        const double ulp = pos ? ldexp(1.0, se - 52) : 0.0;
        long long st[kWalkK];
        bool ok[kWalkK];
        long long lsum = 0;
#pragma unroll
        for (int k = 0; k < kWalkK; ++k) {
            const uint64_t idx = c + (uint64_t)lane * kWalkK + k;
            const bool in = idx < nchunks;
            st[k] = in ? steps[idx] : 0;
            ok[k] = in && pos && clean[idx] && cexp[idx] == se;
            lsum += st[k];
        }
        long long pre = lsum;  // inclusive prefix over the lanes
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const long long y = __shfl_up_sync(full, pre, o);
            if (lane >= o) pre += y;
        }
        // first chunk (window order) that cannot be taken in O(1)
        long long run = pre - lsum;
        int bad = W;
#pragma unroll
        for (int k = 0; k < kWalkK; ++k) {
            run += st[k];
            const bool good = ok[k] && s + (double)run * ulp < lim;
            if (!good && bad == W) bad = lane * kWalkK + k;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) bad = min(bad, __shfl_xor_sync(full, bad, o));
        // ends of the leading good run, and s after it
        run = pre - lsum;
        long long upto = 0;
#pragma unroll
        for (int k = 0; k < kWalkK; ++k) {
            run += st[k];
            const int p = lane * kWalkK + k;
            if (p < bad) ends[c + p] = s + (double)run * ulp;
            if (p == bad - 1) upto = run;
        }
        if (bad > 0) {
            upto = __shfl_sync(full, upto, (bad - 1) / kWalkK);
            s = s + (double)upto * ulp;
        }
        c += (uint64_t)bad;
        if (bad == W || c >= nchunks) continue;
        // chunk c: sub-chunk by sub-chunk
        ++seq;
        const uint64_t c0 = c << chunk_log;
        const uint64_t e1 = c0 + len < n ? c0 + len : n;
        for (uint64_t b = c0; b < e1; b += kSubChunk) {
            const double p0 = b + lane < e1 ? prob(b + lane) : 0.0;
            const double p1 = b + 32 + lane < e1 ? prob(b + 32 + lane) : 0.0;
            bool taken = false;
            if (s > 0x1p-1000) {  // s normal: binade e, ulp 2^(e-52)
                const int e = exponent_of(s);
                const double lim = ldexp(1.0, e + 1);
                double tot = p0 + p1;  // approximate sum (guards the scaling below against overflow)
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) tot += __shfl_xor_sync(full, tot, o);
                if (s + tot < lim * (1.0 - 0x1p-30)) {
                    long long ks = 0;
                    int tie = 0;
#pragma unroll
                    for (int h = 0; h < 2; ++h) {
                        const double q = ldexp(h ? p1 : p0, 52 - e);  // exact: a power-of-two scaling, q < 2^53
                        const double f = floor(q);
                        const double fr = q - f;  // exact
                        long long kk = (long long)f;
                        if (fr > 0.5) ++kk;
                        if (fr == 0.5) tie = 1;
                        ks += kk;
                    }
#pragma unroll
                    for (int o = 16; o > 0; o >>= 1) {
                        ks += __shfl_xor_sync(full, ks, o);
                        tie |= __shfl_xor_sync(full, tie, o);
                    }
                    if (!tie) {
                        const double sn = s + ldexp((double)ks, e - 52);  // exact: on the binade's grid, below lim
                        if (sn < lim) {
                            s = sn;
                            taken = true;
                        }
                    }
                }
            }
            if (!taken) {
                const int cnt = e1 - b < (uint64_t)kSubChunk ? (int)(e1 - b) : kSubChunk;
                for (int k = 0; k < cnt; ++k) s = __dadd_rn(s, __shfl_sync(full, k < 32 ? p0 : p1, k & 31));
            }
        }
        if (lane == 0) ends[c] = s;
        ++c;
    }
    if (lane == 0) *n_seq = seq;
}

template <class P>
__global__ void k_sample_find(P prob, uint64_t n, int chunk_log, const double* __restrict__ ends, uint64_t nchunks,
                              const double* __restrict__ uniforms, uint64_t shots, uint64_t* __restrict__ out) {
    const uint64_t shot = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (shot >= shots) return;
    const double r = uniforms[shot];
    uint64_t lo = 0, hi = nchunks;
    while (lo < hi) {
        const uint64_t mid = (lo + hi) >> 1;
        if (r < ends[mid])
            hi = mid;
        else
            lo = mid + 1;
    }
    uint64_t idx = n - 1;
    if (lo < nchunks) {
        double cum = lo ? ends[lo - 1] : 0.0;
        const uint64_t c0 = lo << chunk_log;
        const uint64_t e = (c0 + ((uint64_t)1 << chunk_log)) < n ? c0 + ((uint64_t)1 << chunk_log) : n;
        for (uint64_t j = c0; j < e; ++j) {
            cum = __dadd_rn(cum, prob(j));
            if (r < cum) {
                idx = j;
                break;
            }
        }
    }
    out[shot] = idx;
}

// ---------------------------------------------------------------------------
// FP64 reductions.
struct DTerm {
    double wre, wim;  // coeff * i^(number of Y)
    uint64_t z;
};
struct DGroup {
    uint64_t x;
    int32_t t0, t1;
};

__device__ __forceinline__ void block_reduce_store(double re, double im, double2* __restrict__ partial) {
    re = warp_sum(re);
    im = warp_sum(im);
    __shared__ double sre[32], sim[32];
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) {
        sre[w] = re;
        sim[w] = im;
    }
    __syncthreads();
    if (w == 0) {
        const int nw = blockDim.x >> 5;
        re = l < nw ? sre[l] : 0.0;
        im = l < nw ? sim[l] : 0.0;
        re = warp_sum(re);
        im = warp_sum(im);
        if (l == 0) partial[blockIdx.x] = make_double2(re, im);
    }
}

// Projective measurement of qubit q (measureQubit, sim/statevector/dynamic.go:
// 179-230): per block, the sums of |a_i|^2 over the amplitudes with bit q
// clear (x) and set (y).
template <class T>
__global__ void k_prob_bit(const cplx<T>* __restrict__ st, uint64_t n, int q, double2* __restrict__ partial) {
    double p0 = 0.0, p1 = 0.0;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const cplx<T> a = st[i];
        const double p = (double)a.x * (double)a.x + (double)a.y * (double)a.y;
        if ((i >> q) & 1ull)
            p1 += p;
        else
            p0 += p;
    }
    block_reduce_store(p0, p1, partial);
}

// Collapse onto `outcome` of qubit q: amplitudes with the other bit value are
// zeroed, the rest scaled by `scale` (1 / sqrt of the outcome's probability).
template <class T>
__global__ void k_collapse(cplx<T>* __restrict__ st, uint64_t n, int q, int outcome, double scale) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        cplx<T> a = st[i];
        if ((int)((i >> q) & 1ull) == outcome) {
            a.x = (T)((double)a.x * scale);
            a.y = (T)((double)a.y * scale);
        } else {
            a.x = T(0);
            a.y = T(0);
        }
        st[i] = a;
    }
}

// measureQubitDM (sim/densitymatrix/dynamic.go:198-255): per block, the sums
// of rho[i,i] over i with bit q clear (x) and set (y).
__global__ void k_dm_prob_bit(const cplx<double>* __restrict__ rho, uint64_t dim, int q, double2* __restrict__ partial) {
    double p0 = 0.0, p1 = 0.0;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < dim; i += (uint64_t)gridDim.x * blockDim.x) {
        const double d = rho[i * dim + i].x;
        if ((i >> q) & 1ull)
            p1 += d;
        else
            p0 += d;
    }
    block_reduce_store(p0, p1, partial);
}

// Projection onto `outcome` of qubit q: rho[r,c] kept (times `scale`) where
// both r and c have bit q equal to the outcome, zeroed elsewhere.
__global__ void k_dm_collapse(cplx<double>* __restrict__ rho, uint64_t dim, int q, int outcome, double scale) {
    const uint64_t n = dim * dim;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t r = i / dim, c = i % dim;
        cplx<double> a = rho[i];
        if ((int)((r >> q) & 1ull) == outcome && (int)((c >> q) & 1ull) == outcome) {
            a.x *= scale;
            a.y *= scale;
        } else {
            a.x = 0.0;
            a.y = 0.0;
        }
        rho[i] = a;
    }
}

// sum_t coeff_t <psi|P_t|psi>: for each amplitude i and each group of terms
// sharing an x mask, conj(psi[i^x]) psi[i] times sum_t w_t (-1)^popcount(i&z_t)
// (the formula of pauli.Expect, sim/pauli/expect_sv.go:21-47).
template <class T>
__global__ void k_expect(const cplx<T>* __restrict__ st, uint64_t n, const DGroup* __restrict__ groups, int ngroups,
                         const DTerm* __restrict__ terms, double2* __restrict__ partial) {
    double are = 0.0, aim = 0.0;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const cplx<T> ai = st[i];
        const double xr = (double)ai.x, xi = (double)ai.y;
        for (int g = 0; g < ngroups; ++g) {
            const DGroup gr = groups[g];
            const cplx<T> aj = st[i ^ gr.x];
            const double yr = (double)aj.x, yi = (double)aj.y;
            // conj(a_j) * a_i
            const double pr = yr * xr + yi * xi, pi = yr * xi - yi * xr;
            double fr = 0.0, fi = 0.0;
            for (int k = gr.t0; k < gr.t1; ++k) {
                const DTerm tm = terms[k];
                const double sg = (__popcll(i & tm.z) & 1) ? -1.0 : 1.0;
                fr += sg * tm.wre;
                fi += sg * tm.wim;
            }
            are += fr * pr - fi * pi;
            aim += fr * pi + fi * pr;
        }
    }
    block_reduce_store(are, aim, partial);
}

// Tr(rho P) for a row-major rho of dimension dim = 2^nq: sum_i rho[i, i^x]
// times the same term factors (pauli.ExpectDM, sim/pauli/expect_dm.go:9-21).
__global__ void k_dm_expect(const cplx<double>* __restrict__ rho, uint64_t dim, const DGroup* __restrict__ groups,
                            int ngroups, const DTerm* __restrict__ terms, double2* __restrict__ partial) {
    double are = 0.0, aim = 0.0;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < dim; i += (uint64_t)gridDim.x * blockDim.x) {
        for (int g = 0; g < ngroups; ++g) {
            const DGroup gr = groups[g];
            const cplx<double> v = rho[i * dim + (i ^ gr.x)];
            double fr = 0.0, fi = 0.0;
            for (int k = gr.t0; k < gr.t1; ++k) {
                const DTerm tm = terms[k];
                const double sg = (__popcll(i & tm.z) & 1) ? -1.0 : 1.0;
                fr += sg * tm.wre;
                fi += sg * tm.wim;
            }
            are += fr * v.x - fi * v.y;
            aim += fr * v.y + fi * v.x;
        }
    }
    block_reduce_store(are, aim, partial);
}

// sum_{i,j} rho_ij conj(rho_ji): the sum goqu's Purity takes
// (sim/densitymatrix/sim.go:265-276). 32x32 tiles through shared memory.
__global__ void k_dm_purity(const cplx<double>* __restrict__ rho, uint64_t dim, double2* __restrict__ partial) {
    __shared__ cplx<double> tile[32][33];
    const uint64_t ntile = dim >= 32 ? dim / 32 : 1;
    const uint64_t tdim = dim >= 32 ? 32 : dim;
    double are = 0.0, aim = 0.0;
    for (uint64_t tb = blockIdx.x; tb < ntile * ntile; tb += gridDim.x) {
        const uint64_t bi = tb / ntile, bj = tb % ntile;
        const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 32 x 8 threads
        __syncthreads();
        for (int yy = ty; yy < 32; yy += 8)
            if ((uint64_t)yy < tdim && (uint64_t)tx < tdim)
                tile[yy][tx] = rho[(bj * 32 + yy) * dim + bi * 32 + tx];  // block (j, i)
        __syncthreads();
        for (int yy = ty; yy < 32; yy += 8) {
            if ((uint64_t)yy >= tdim || (uint64_t)tx >= tdim) continue;
            const cplx<double> a = rho[(bi * 32 + yy) * dim + bj * 32 + tx];  // rho_ij
            const cplx<double> b = tile[tx][yy];                              // rho_ji
            are += a.x * b.x + a.y * b.y;  // a * conj(b)
            aim += a.y * b.x - a.x * b.y;
        }
    }
    block_reduce_store(are, aim, partial);
}

// sum_i conj(psi_i) sum_j rho_ij psi_j (Fidelity, sim/densitymatrix/sim.go:280-291).
__global__ void k_dm_fidelity(const cplx<double>* __restrict__ rho, uint64_t dim, const cplx<double>* __restrict__ psi,
                              double2* __restrict__ partial) {
    double are = 0.0, aim = 0.0;
    const uint64_t warps = (uint64_t)gridDim.x * (blockDim.x >> 5);
    const int lane = threadIdx.x & 31;
    for (uint64_t i = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5; i < dim; i += warps) {
        double rr = 0.0, ri = 0.0;
        for (uint64_t j = lane; j < dim; j += 32) {
            const cplx<double> a = rho[i * dim + j], p = psi[j];
            rr += a.x * p.x - a.y * p.y;
            ri += a.x * p.y + a.y * p.x;
        }
        const cplx<double> q = psi[i];
        // conj(q) * (rr + i ri), accumulated by every lane's partial row sum
        are += q.x * rr + q.y * ri;
        aim += q.x * ri - q.y * rr;
    }
    block_reduce_store(are, aim, partial);
}

__global__ void k_dm_diag_probs(const cplx<double>* __restrict__ rho, uint64_t dim, double* __restrict__ out) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < dim; i += (uint64_t)gridDim.x * blockDim.x) {
        const double v = rho[i * dim + i].x;
        out[i] = v < 0 ? 0.0 : v;
    }
}

// One qubit of ApplyReadoutError (sim/densitymatrix/measure.go:29-71):
// out[k] = in[k]*(1-P) + in[k^m]*P' with the reference's rounding.
__global__ void k_readout_qubit(const double* __restrict__ in, double* __restrict__ out, uint64_t dim, uint64_t mask,
                                double p01, double p10) {
    for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < dim; k += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t f = k ^ mask;
        // contribution of i = k (stays) and of i = f (flips into k)
        const double a = (k & mask) ? __dmul_rn(in[k], __dsub_rn(1.0, p10)) : __dmul_rn(in[k], __dsub_rn(1.0, p01));
        const double b = (f & mask) ? __dmul_rn(in[f], p10) : __dmul_rn(in[f], p01);
        out[k] = __dadd_rn(a, b);
    }
}

__global__ void k_final_reduce(const double2* __restrict__ partial, int n, double2* __restrict__ out) {
    double re = 0.0, im = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        re += partial[i].x;
        im += partial[i].y;
    }
    re = warp_sum(re);
    im = warp_sum(im);
    __shared__ double sre[32], sim[32];
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) {
        sre[w] = re;
        sim[w] = im;
    }
    __syncthreads();
    if (w == 0) {
        const int nw = blockDim.x >> 5;
        re = l < nw ? sre[l] : 0.0;
        im = l < nw ? sim[l] : 0.0;
        re = warp_sum(re);
        im = warp_sum(im);
        if (l == 0) *out = make_double2(re, im);
    }
}

// lambda = sum_t Re(c_t) P_t psi, with (P psi)_i = i^nY (-1)^popcount((i^x)&z)
// psi[i^x]; also accumulates Re <psi|lambda> = E into partial (per block).
template <class T>
__global__ void k_apply_terms(const cplx<T>* __restrict__ psi, cplx<T>* __restrict__ lam, uint64_t n,
                              const DGroup* __restrict__ groups, int ngroups, const DTerm* __restrict__ terms,
                              double2* __restrict__ partial) {
    double e = 0.0;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        double lr = 0.0, li = 0.0;
        for (int g = 0; g < ngroups; ++g) {
            const DGroup gr = groups[g];
            const uint64_t j = i ^ gr.x;
            const cplx<T> v = psi[j];
            double fr = 0.0, fi = 0.0;
            for (int k = gr.t0; k < gr.t1; ++k) {
                const DTerm tm = terms[k];
                const double sg = (__popcll(j & tm.z) & 1) ? -1.0 : 1.0;
                fr += sg * tm.wre;
                fi += sg * tm.wim;
            }
            lr += fr * (double)v.x - fi * (double)v.y;
            li += fr * (double)v.y + fi * (double)v.x;
        }
        lam[i] = {(T)lr, (T)li};
        const cplx<T> a = psi[i];
        e += (double)a.x * lr + (double)a.y * li;
    }
    block_reduce_store(e, 0.0, partial);
}

// ---------------------------------------------------------------------------
// Batched reductions for many small states.
struct BCircuit {
    uint64_t state;   // first amplitude of the circuit's state (and lambda)
    uint64_t n_amps;
    int32_t group0, ngroups;  // its Pauli groups in the concatenated arrays
};
struct BChunk {
    uint32_t circuit;
    uint32_t begin;  // first amplitude of this block's chunk
};

// lambda = sum_t Re(c_t) P_t psi per circuit, and per-block partials of
// Re <psi|lambda> (summed per circuit by k_segment_reduce).
template <class T>
__global__ void k_apply_terms_batch(const cplx<T>* __restrict__ psi_all, cplx<T>* __restrict__ lam_all,
                                    const BCircuit* __restrict__ circ, const BChunk* __restrict__ chunks,
                                    uint32_t chunk_len, const DGroup* __restrict__ groups,
                                    const DTerm* __restrict__ terms, double* __restrict__ partial) {
    const BChunk ch = chunks[blockIdx.x];
    const BCircuit c = circ[ch.circuit];
    const cplx<T>* psi = psi_all + c.state;
    cplx<T>* lam = lam_all + c.state;
    const uint64_t end = (uint64_t)ch.begin + chunk_len < c.n_amps ? (uint64_t)ch.begin + chunk_len : c.n_amps;
    // The circuit's groups and terms, read by every amplitude, are staged in
    // shared memory once per block when they fit (global loads of them
    // otherwise throttle the load pipe).
    constexpr int kSharedGroups = 64, kSharedTerms = 384;
    __shared__ DGroup sgr[kSharedGroups];
    __shared__ DTerm stm[kSharedTerms];
    const int t_lo = c.ngroups ? groups[c.group0].t0 : 0;
    const int t_hi = c.ngroups ? groups[c.group0 + c.ngroups - 1].t1 : 0;
    const bool staged = c.ngroups <= kSharedGroups && t_hi - t_lo <= kSharedTerms;
    if (staged) {
        for (int k = threadIdx.x; k < c.ngroups; k += blockDim.x) sgr[k] = groups[c.group0 + k];
        for (int k = threadIdx.x; k < t_hi - t_lo; k += blockDim.x) stm[k] = terms[t_lo + k];
    }
    __syncthreads();
    double e = 0.0;
    // The loop is instantiated once for the shared copies and once for the
    // global arrays, so that each reads its terms with its own load kind.
    auto run = [&](const DGroup* gp, const DTerm* tp) {
        for (uint64_t i = ch.begin + threadIdx.x; i < end; i += blockDim.x) {
            double lr = 0.0, li = 0.0;
            for (int g = 0; g < c.ngroups; ++g) {
                const DGroup gr = gp[g];
                const uint64_t j = i ^ gr.x;
                const cplx<T> v = psi[j];
                double fr = 0.0, fi = 0.0;
                for (int k = gr.t0 - t_lo; k < gr.t1 - t_lo; ++k) {
                    const DTerm tm = tp[k];
                    const double sg = (__popcll(j & tm.z) & 1) ? -1.0 : 1.0;
                    fr += sg * tm.wre;
                    fi += sg * tm.wim;
                }
                lr += fr * (double)v.x - fi * (double)v.y;
                li += fr * (double)v.y + fi * (double)v.x;
            }
            lam[i] = {(T)lr, (T)li};
            const cplx<T> a = psi[i];
            e += (double)a.x * lr + (double)a.y * li;
        }
    };
    if (staged)
        run(sgr, stm);
    else
        run(groups + c.group0, terms + t_lo);
    e = warp_sum(e);
    __shared__ double ws[32];
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = e;
    __syncthreads();
    if (threadIdx.x == 0) {
        double tot = 0.0;
        for (unsigned w = 0; w < (blockDim.x >> 5); ++w) tot += ws[w];
        partial[blockIdx.x] = tot;
    }
}

// out[s] = sum of partial[seg[s] .. seg[s+1]) (one block per segment).
__global__ void k_segment_reduce(const double* __restrict__ partial, const uint64_t* __restrict__ seg,
                                 double* __restrict__ out) {
    const uint64_t b = seg[blockIdx.x], e = seg[blockIdx.x + 1];
    double v = 0.0;
    for (uint64_t i = b + threadIdx.x; i < e; i += blockDim.x) v += partial[i];
    v = warp_sum(v);
    __shared__ double ws[32];
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double tot = 0.0;
        for (unsigned w = 0; w < (blockDim.x >> 5); ++w) tot += ws[w];
        out[blockIdx.x] = tot;
    }
}

// Gradient partials of one reverse wave: group g is one circuit's pass, its
// nctas CTAs holding nslots partials each from part0;
// grad[slot_grad[slot0 + s]] += 2 * sum over the group's CTAs.
struct BGradGroup {
    uint64_t part0;   // partials of one reverse pass of one state: part0 + cta * nslots + slot
    uint32_t nctas;
    uint32_t slot0;   // into slot_grad
    uint32_t nslots;
    uint32_t pad;
};
__global__ void k_grad_reduce_batch(const double* __restrict__ partial, const BGradGroup* __restrict__ grp,
                                    const uint32_t* __restrict__ slot_grad, double* __restrict__ grad) {
    const BGradGroup g = grp[blockIdx.x];
    __shared__ double ws[32];
    for (uint32_t s = 0; s < g.nslots; ++s) {
        double v = 0.0;
        for (uint32_t c = threadIdx.x; c < g.nctas; c += blockDim.x) v += partial[g.part0 + (uint64_t)c * g.nslots + s];
        v = warp_sum(v);
        if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = v;
        __syncthreads();
        if (threadIdx.x == 0) {
            double tot = 0.0;
            for (unsigned w = 0; w < (blockDim.x >> 5); ++w) tot += ws[w];
            grad[slot_grad[g.slot0 + s]] += 2.0 * tot;
        }
        __syncthreads();
    }
}

// |0...0> in every state of a batch (after a memset to zero).
template <class T>
__global__ void k_batch_basis(cplx<T>* __restrict__ states, const uint64_t* __restrict__ offs, uint64_t n) {
    const uint64_t c = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (c < n) states[offs[c]] = {T(1), T(0)};
}

}  // namespace gq

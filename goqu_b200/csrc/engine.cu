// C ABI of the engine (include/gqb200.h): handles, program upload, launches.
//
// A handle owns its device state, a program buffer, a scratch buffer and a
// CUDA stream; nothing is allocated per gate. Statevectors hold 2^max(n,4)
// amplitudes (qubits above n stay |0>), density matrices are vectorised as a
// 2n-qubit state (row index in the high n bits), so both run the same tile
// passes. There is no CPU fallback: without an sm_100 device every call fails.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <atomic>
#include <chrono>
#include <mutex>
#include <string>
#include <thread>
#include <future>
#include <vector>

#include "../../include/gqb200.h"
#include "counts.cuh"
#include "kernels.cuh"
#include "verify.cuh"
#include "jit.hpp"
#include "params.hpp"
#include "schedule.hpp"

using namespace gq;

namespace {

thread_local std::string g_err;

int fail(int code, const std::string& msg) {
    g_err = msg;
    return code;
}

#define GQ_CUDA(x)                                                                        \
    do {                                                                                  \
        cudaError_t e_ = (x);                                                             \
        if (e_ != cudaSuccess) return fail(GQ_ECUDA, std::string(#x) + ": " + cudaGetErrorString(e_)); \
    } while (0)

#define GQ_TRY(x)                  \
    do {                           \
        int rc_ = (x);             \
        if (rc_ != GQ_OK) return rc_; \
    } while (0)

int check_device(int* dev_out) {
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0) return fail(GQ_ENODEVICE, "no CUDA device visible");
    int dev = 0;
    GQ_CUDA(cudaGetDevice(&dev));
    cudaDeviceProp p;
    GQ_CUDA(cudaGetDeviceProperties(&p, dev));
    if (p.major != 10) return fail(GQ_ENODEVICE, std::string("device is not sm_100: ") + p.name);
    *dev_out = dev;
    return GQ_OK;
}

struct DevBuf {
    void* p = nullptr;
    size_t cap = 0;
    int ensure(size_t bytes) {
        if (bytes <= cap) return GQ_OK;
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
        if (cudaMalloc(&p, bytes) != cudaSuccess) {
            cudaGetLastError();
            return fail(GQ_ENOMEM, "cudaMalloc of " + std::to_string(bytes) + " bytes failed");
        }
        cap = bytes;
        return GQ_OK;
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
    }
};

struct PinnedBuf {
    void* p = nullptr;
    size_t cap = 0;
    int ensure(size_t bytes) {
        if (bytes <= cap) return GQ_OK;
        if (p) cudaFreeHost(p);
        p = nullptr;
        cap = 0;
        if (cudaMallocHost(&p, bytes) != cudaSuccess) {
            cudaGetLastError();
            return fail(GQ_ENOMEM, "cudaMallocHost failed");
        }
        cap = bytes;
        return GQ_OK;
    }
    void release() {
        if (p) cudaFreeHost(p);
        p = nullptr;
        cap = 0;
    }
};

size_t align16(size_t x) { return (x + 15) & ~size_t(15); }

// FMA-per-amplitude budget of a pass: the measured optimum of the 28-qubit
// layered benchmark (larger budgets trade passes for compute per pass).
constexpr int kDefaultBudget = 320;

// Tile-pass kernel instantiations (see kVariants* in kernels.cuh).
using TileKernelD = void (*)(cplx<double>*, const PassDesc*, const PhaseDesc*, const KOp*, const cplx<double>*);
using TileKernelF = void (*)(cplx<float>*, const PassDesc*, const PhaseDesc*, const KOp*, const cplx<float>*);
const TileKernelD kTileD[kNumVariants] = {
    k_tile_pass<double, kVariantsC128[0].threads, kVariantsC128[0].min_blocks>,
    k_tile_pass<double, kVariantsC128[1].threads, kVariantsC128[1].min_blocks>,
    k_tile_pass<double, kVariantsC128[2].threads, kVariantsC128[2].min_blocks>,
    k_tile_pass<double, kVariantsC128[3].threads, kVariantsC128[3].min_blocks>};
const TileKernelF kTileF[kNumVariants] = {
    k_tile_pass<float, kVariantsC64[0].threads, kVariantsC64[0].min_blocks>,
    k_tile_pass<float, kVariantsC64[1].threads, kVariantsC64[1].min_blocks>,
    k_tile_pass<float, kVariantsC64[2].threads, kVariantsC64[2].min_blocks>,
    k_tile_pass<float, kVariantsC64[3].threads, kVariantsC64[3].min_blocks>};

// Adjoint (two-state) pass: 128 threads (tiles of up to 2^11 amplitudes).
using AdjKernelD = void (*)(cplx<double>*, cplx<double>*, const PassDesc*, const PhaseDesc*, const KOp*,
                            const cplx<double>*, double*, int);
using AdjKernelF = void (*)(cplx<float>*, cplx<float>*, const PassDesc*, const PhaseDesc*, const KOp*,
                            const cplx<float>*, double*, int);
constexpr int kAdjThreads = 128;
// CTAs per SM of the batched reverse pass: complex64 keeps both states'
// 16 amplitudes in 64 registers and fits 4 (128 registers; measured faster
// than 3 with 168 on 4096 QAOA circuits, 394 against 439 ms).
template <class T>
constexpr int kAdjBatchMinB = sizeof(T) == 4 ? 4 : 2;
const AdjKernelD kAdjD = k_adjoint_pass<double, kAdjThreads, 2>;
const AdjKernelF kAdjF = k_adjoint_pass<float, kAdjThreads, 3>;
template <class T>
struct AdjTable;
template <>
struct AdjTable<double> {
    static AdjKernelD get() { return kAdjD; }
};
template <>
struct AdjTable<float> {
    static AdjKernelF get() { return kAdjF; }
};
size_t adj_smem(size_t amp, int m) { return 2 * (amp << m) + (kAdjThreads / 32) * MAX_GRAD_SLOTS * sizeof(double); }

template <class T>
struct TileTable;
template <>
struct TileTable<double> {
    static TileKernelD get(int v) { return kTileD[v]; }
    static int threads(int v) { return kVariantsC128[v].threads; }
};
template <>
struct TileTable<float> {
    static TileKernelF get(int v) { return kTileF[v]; }
    static int threads(int v) { return kVariantsC64[v].threads; }
};

int log2i(int x) {
    int r = 0;
    while ((1 << (r + 1)) <= x) ++r;
    return r;
}

template <class T>
int set_smem_attr() {
    static std::once_flag once;
    static cudaError_t err = cudaSuccess;
    std::call_once(once, [] {
        for (int v = 0; v < kNumVariants && err == cudaSuccess; ++v) {
            const int m = log2i(TileTable<T>::threads(v)) + RQ;
            err = cudaFuncSetAttribute(TileTable<T>::get(v), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)(sizeof(cplx<T>) << m));
        }
        if (err == cudaSuccess)
            err = cudaFuncSetAttribute(AdjTable<T>::get(), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)adj_smem(sizeof(cplx<T>), log2i(kAdjThreads) + RQ));
    });
    if (err != cudaSuccess) return fail(GQ_ECUDA, std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(err));
    return GQ_OK;
}

// State of one simulator: device amplitudes plus the buffers to drive them.
struct Engine {
    int device = 0;
    int prec = GQ_C128;
    int nphys = 0;              // physical qubits of the vector
    uint64_t n_amps = 0;
    cudaStream_t stream = nullptr;
    DevBuf state, prog, scratch, scratch2, aux;
    DevBuf lam, ckpt, adj_partial, adj_grad;  // adjoint differentiation
    DevBuf hist;                              // shot histograms (counts.cuh)
    int adj_nparams = 0;                      // parameters of the current gradient
    int adj_segments = 0;                     // forward checkpoints (0: automatic)
    // Two host staging buffers used in turn: a program is packed into one
    // while the upload from the other may still wait behind running passes.
    PinnedBuf staging[2], hostio;
    cudaEvent_t staged[2] = {nullptr, nullptr};
    int stage_slot = 0;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr, ev_pass0 = nullptr, ev_pass1 = nullptr;
    bool pass_timed = false;
    bool staged_pending[2] = {false, false};
    SchedOptions opt;
    bool timing = false;
    gq_stats stats{};

    int variant = 0;
    int jit_mode = 1;         // GQ_OPT_JIT
    int jit_min_qubits = 20;  // GQ_OPT_JIT_MIN_QUBITS
    int jit_min_blocks = 0;   // GQ_OPT_JIT_MIN_BLOCKS (0: the variant's)
    int jit_persistent = 0;   // GQ_OPT_JIT_PERSISTENT (an autotuner candidate)
    int jit_minb = 4;         // CTAs per SM of the last specialised launch shape
    bool skip_zero_tiles = true;  // GQ_OPT_ZERO_TILES
    int num_sms = 148;
    template <class T>
    size_t jit_smem(int m) const {
        return sizeof(cplx<T>) << m;  // one tile buffer (persistent CTAs refill it in place)
    }
    size_t amp_bytes() const { return prec == GQ_C64 ? 8 : 16; }
    int max_tile() const {
        return RQ + log2i(prec == GQ_C64 ? kVariantsC64[variant].threads : kVariantsC128[variant].threads);
    }

    int init(int nphys_, int prec_) {
        GQ_TRY(check_device(&device));
        prec = prec_;
        nphys = nphys_;
        n_amps = 1ull << nphys;
        GQ_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
        GQ_CUDA(cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, device));
        for (cudaEvent_t& ev : staged) GQ_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
        GQ_CUDA(cudaEventCreate(&ev0));
        GQ_CUDA(cudaEventCreate(&ev1));
        GQ_CUDA(cudaEventCreate(&ev_pass0));
        GQ_CUDA(cudaEventCreate(&ev_pass1));
        GQ_TRY(state.ensure(n_amps * amp_bytes()));
        opt.low_qubits = prec == GQ_C64 ? 4 : 3;
        opt.swizzle_width = prec == GQ_C64 ? 4 : 3;
        variant = prec == GQ_C64 ? 1 : 0;
        opt.tile_qubits = max_tile();
        opt.budget = kDefaultBudget;
        stats.state_bytes = (int64_t)(n_amps * amp_bytes());
        GQ_TRY(prec == GQ_C64 ? set_smem_attr<float>() : set_smem_attr<double>());
        return reset_basis(0);
    }

    void destroy() {
        if (stream) cudaStreamSynchronize(stream);
        state.release();
        prog.release();
        scratch.release();
        scratch2.release();
        aux.release();
        lam.release();
        ckpt.release();
        adj_partial.release();
        adj_grad.release();
        hist.release();
        for (PinnedBuf& b : staging) b.release();
        hostio.release();
        for (cudaEvent_t& ev : staged)
            if (ev) cudaEventDestroy(ev);
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        if (ev_pass0) cudaEventDestroy(ev_pass0);
        if (ev_pass1) cudaEventDestroy(ev_pass1);
        if (stream) cudaStreamDestroy(stream);
        stream = nullptr;
    }

    int reset_basis(uint64_t idx) {
        GQ_CUDA(cudaMemsetAsync(state.p, 0, n_amps * amp_bytes(), stream));
        if (prec == GQ_C64)
            k_set_amp<float><<<1, 1, 0, stream>>>((cplx<float>*)state.p, idx, 1.f, 0.f);
        else
            k_set_amp<double><<<1, 1, 0, stream>>>((cplx<double>*)state.p, idx, 1.0, 0.0);
        GQ_CUDA(cudaGetLastError());
        stats.kernel_launches += 1;
        return GQ_OK;
    }

    // The next staging buffer: wait for the upload that last used it.
    int stage(size_t bytes, void** host) {
        stage_slot ^= 1;
        if (staged_pending[stage_slot]) {
            GQ_CUDA(cudaEventSynchronize(staged[stage_slot]));
            staged_pending[stage_slot] = false;
        }
        GQ_TRY(staging[stage_slot].ensure(bytes));
        *host = staging[stage_slot].p;
        return GQ_OK;
    }
    int upload(DevBuf& dst, size_t bytes) {
        GQ_TRY(dst.ensure(bytes));
        stats.h2d_bytes += (int64_t)bytes;
        GQ_CUDA(cudaMemcpyAsync(dst.p, staging[stage_slot].p, bytes, cudaMemcpyHostToDevice, stream));
        GQ_CUDA(cudaEventRecord(staged[stage_slot], stream));
        staged_pending[stage_slot] = true;
        return GQ_OK;
    }

    template <class T>
    int run_program_t(const Program& pr) {
        if (pr.passes.empty()) return GQ_OK;
        const size_t o_pass = 0;
        const size_t o_phase = align16(o_pass + sizeof(PassDesc) * pr.passes.size());
        const size_t o_ops = align16(o_phase + sizeof(PhaseDesc) * pr.phases.size());
        const size_t o_pool = align16(o_ops + sizeof(KOp) * pr.ops.size());
        const size_t total = align16(o_pool + sizeof(cplx<T>) * std::max<size_t>(1, pr.pool.size()));
        void* hp = nullptr;
        GQ_TRY(stage(total, &hp));
        char* h = (char*)hp;
        std::memcpy(h + o_pass, pr.passes.data(), sizeof(PassDesc) * pr.passes.size());
        std::memcpy(h + o_phase, pr.phases.data(), sizeof(PhaseDesc) * pr.phases.size());
        if (!pr.ops.empty()) std::memcpy(h + o_ops, pr.ops.data(), sizeof(KOp) * pr.ops.size());
        cplx<T>* pool = (cplx<T>*)(h + o_pool);
        for (size_t i = 0; i < pr.pool.size(); ++i) pool[i] = {(T)pr.pool[i].re, (T)pr.pool[i].im};
        GQ_TRY(upload(prog, total));
        char* d = (char*)prog.p;
        // Specialised kernels for the passes whose compilation has finished
        // (or, with GQ_OPT_JIT = 2, once it has); the others run interpreted.
        const size_t np = pr.passes.size();
        std::vector<const void*> jfn(np, nullptr);
        std::vector<const CachedPlan*> plans(np, nullptr);
        if (jit_on()) {
            // One tile per CTA: 4 CTAs of 128 threads per SM (128 registers)
            // measured fastest for both precisions. Persistent: the launch
            // shape's CTAs per SM, as far as one tile buffer each allows.
            const TileVariant tv = prec == GQ_C64 ? kVariantsC64[variant] : kVariantsC128[variant];
            int minb = tv.threads == 128 ? std::max(tv.min_blocks, 4) : tv.min_blocks;
            if (jit_persistent) minb = std::max(1, std::min(minb, (int)((227u << 10) / (sizeof(cplx<T>) << max_tile()))));
            if (jit_min_blocks > 0) minb = jit_min_blocks;
            jit_minb = minb;
            for (size_t i = 0; i < np; ++i) {
                const PassDesc& pd = pr.passes[i];
                plans[i] = jit_cached_plan(pr, i, prec == GQ_C64, 1 << (pd.m - RQ), minb, jit_persistent != 0);
                if (plans[i]->ok) jfn[i] = jit_plan_kernel(plans[i], jit_smem<T>(pd.m));
            }
            if (jit_mode == 2) {
                jit_wait(600000.0);
                for (size_t i = 0; i < np; ++i)
                    if (plans[i]->ok && !jfn[i]) jfn[i] = jit_plan_kernel(plans[i], jit_smem<T>(pr.passes[i].m));
            }
        }
        // the span from the call's first pass to its last (a call may run
        // several programs: checkpoint segments, a split density-matrix stream)
        if (timing && !pass_timed) GQ_CUDA(cudaEventRecord(ev_pass0, stream));
        std::vector<cplx<T>> pblock;
        int64_t jitted = 0;
        for (size_t i = 0; i < np; ++i) {
            const PassDesc& pd = pr.passes[i];
            const unsigned threads = 1u << (pd.m - RQ);
            const size_t smem = sizeof(cplx<T>) << pd.m;
            const unsigned grid = 1u << pd.n_outer;
            if (jfn[i]) pblock.resize(plans[i]->plan.n_param);
            if (jfn[i] && jit_pack(pr, i, plans[i]->plan, prec == GQ_C64, pblock.data())) {
                uint32_t op_base, pool_base;
                jit_bases(pr, i, &op_base, &pool_base);
                cplx<T>* stp = (cplx<T>*)state.p;
                const cplx<T>* poolp = (const cplx<T>*)(d + o_pool) + pool_base;
                const PhaseDesc* php = (const PhaseDesc*)(d + o_phase) + pd.phase0;
                void* args[4] = {&stp, pblock.data(), &poolp, &php};
                const unsigned jgrid =
                    jit_persistent ? (unsigned)std::min<uint64_t>(grid, (uint64_t)num_sms * jit_minb) : grid;
                GQ_CUDA(cudaLaunchKernel(jfn[i], dim3(jgrid), dim3(threads), args, jit_smem<T>(pd.m), stream));
                ++jitted;
                continue;
            }
            TileTable<T>::get(variant)<<<grid, threads, smem, stream>>>(
                (cplx<T>*)state.p, (const PassDesc*)(d + o_pass) + i, (const PhaseDesc*)(d + o_phase),
                (const KOp*)(d + o_ops), (const cplx<T>*)(d + o_pool));
        }
        GQ_CUDA(cudaGetLastError());
        stats.jit_passes += jitted;
        if (timing) {
            GQ_CUDA(cudaEventRecord(ev_pass1, stream));
            pass_timed = true;
        }
        stats.passes += (int64_t)pr.passes.size();
        stats.kernel_launches += (int64_t)pr.passes.size();
        stats.phases += (int64_t)pr.phases.size();
        return GQ_OK;
    }

    // Reverse sweep of an adjoint gradient: two-state tile passes, then the
    // per-pass gradient reduction into adj_grad.
    template <class T>
    int run_adjoint_t(const Program& pr) {
        if (pr.passes.empty()) return GQ_OK;
        const size_t np = pr.passes.size();
        size_t nslot_total = 0;
        for (const auto& v : pr.pass_params) nslot_total += v.size();
        const size_t ns1 = std::max<size_t>(1, nslot_total);
        const size_t o_pass = 0;
        const size_t o_phase = align16(o_pass + sizeof(PassDesc) * np);
        const size_t o_ops = align16(o_phase + sizeof(PhaseDesc) * pr.phases.size());
        const size_t o_pool = align16(o_ops + sizeof(KOp) * pr.ops.size());
        const size_t o_slots = align16(o_pool + sizeof(cplx<T>) * std::max<size_t>(1, pr.pool.size()));
        const size_t o_soff = align16(o_slots + sizeof(int) * ns1);
        const size_t o_sn = align16(o_soff + sizeof(uint64_t) * ns1);
        const size_t o_sst = align16(o_sn + sizeof(uint64_t) * ns1);
        const size_t total = align16(o_sst + sizeof(uint32_t) * ns1);
        void* hp = nullptr;
        GQ_TRY(stage(total, &hp));
        char* h = (char*)hp;
        std::memcpy(h + o_pass, pr.passes.data(), sizeof(PassDesc) * np);
        std::memcpy(h + o_phase, pr.phases.data(), sizeof(PhaseDesc) * pr.phases.size());
        if (!pr.ops.empty()) std::memcpy(h + o_ops, pr.ops.data(), sizeof(KOp) * pr.ops.size());
        cplx<T>* pool = (cplx<T>*)(h + o_pool);
        for (size_t i = 0; i < pr.pool.size(); ++i) pool[i] = {(T)pr.pool[i].re, (T)pr.pool[i].im};
        // Gradient partials of consecutive passes share one buffer (up to
        // kPartialCap doubles) and are reduced by two launches per group of
        // passes (k_slot_sums, k_param_sums) instead of one per pass.
        constexpr uint64_t kPartialCap = 16ull << 20;
        int* slots = (int*)(h + o_slots);
        uint64_t* soff = (uint64_t*)(h + o_soff);
        uint64_t* sn = (uint64_t*)(h + o_sn);
        uint32_t* sst = (uint32_t*)(h + o_sst);
        std::vector<uint64_t> pass_off(np);
        std::vector<size_t> pass_slot0(np);
        std::vector<size_t> group_end;  // last pass of each group
        uint64_t used = 0, max_group = 1;
        size_t k = 0;
        for (size_t i = 0; i < np; ++i) {
            const uint64_t grid = 1ull << pr.passes[i].n_outer;
            const uint64_t ns = pr.pass_params[i].size();
            if (used && used + grid * ns > kPartialCap) {
                group_end.push_back(i - 1);
                used = 0;
            }
            pass_off[i] = used;
            pass_slot0[i] = k;
            for (uint64_t sl = 0; sl < ns; ++sl, ++k) {
                slots[k] = pr.pass_params[i][sl];
                soff[k] = used + sl;
                sn[k] = grid;
                sst[k] = (uint32_t)ns;
            }
            used += grid * ns;
            max_group = std::max(max_group, used);
        }
        group_end.push_back(np - 1);
        GQ_TRY(upload(prog, total));
        GQ_TRY(adj_partial.ensure((max_group + ns1) * sizeof(double)));
        double* partial = (double*)adj_partial.p;
        double* sums = partial + max_group;
        char* d = (char*)prog.p;
        // specialised dual kernels for the passes whose compilation has
        // finished (or, with GQ_OPT_JIT = 2, once it has)
        std::vector<const void*> jfn(np, nullptr);
        std::vector<const CachedPlan*> plans(np, nullptr);
        if (jit_on()) {
            const int minb = 2;  // both states' 16 amplitudes and a gradient copy in registers
            for (size_t i = 0; i < np; ++i) {
                const PassDesc& pd = pr.passes[i];
                plans[i] = jit_cached_plan(pr, i, prec == GQ_C64, 1 << (pd.m - RQ), minb, false, true);
                if (plans[i]->ok) jfn[i] = jit_plan_kernel(plans[i], adj_smem(sizeof(cplx<T>), pd.m));
            }
            if (jit_mode == 2) {
                jit_wait(600000.0);
                for (size_t i = 0; i < np; ++i)
                    if (plans[i]->ok && !jfn[i])
                        jfn[i] = jit_plan_kernel(plans[i], adj_smem(sizeof(cplx<T>), pr.passes[i].m));
            }
        }
        std::vector<cplx<T>> pblock;
        int64_t jitted = 0;
        size_t gi = 0, slot_lo = 0;
        for (size_t i = 0; i < np; ++i) {
            const PassDesc& pd = pr.passes[i];
            const int nslots = (int)pr.pass_params[i].size();
            const unsigned threads = 1u << (pd.m - RQ);
            const unsigned grid = 1u << pd.n_outer;
            const size_t smem = adj_smem(sizeof(cplx<T>), pd.m);
            double* part = partial + pass_off[i];
            if (jfn[i]) pblock.resize(plans[i]->plan.n_param);
            if (jfn[i] && jit_pack(pr, i, plans[i]->plan, prec == GQ_C64, pblock.data())) {
                uint32_t op_base, pool_base;
                jit_bases(pr, i, &op_base, &pool_base);
                cplx<T>* psi = (cplx<T>*)state.p;
                cplx<T>* lm = (cplx<T>*)lam.p;
                const cplx<T>* poolp = (const cplx<T>*)(d + o_pool) + pool_base;
                const PhaseDesc* php = (const PhaseDesc*)(d + o_phase) + pd.phase0;
                int ns = nslots;
                void* args[7] = {&psi, &lm, pblock.data(), &poolp, &php, &part, &ns};
                GQ_CUDA(cudaLaunchKernel(jfn[i], dim3(grid), dim3(threads), args, smem, stream));
                ++jitted;
            } else {
                AdjTable<T>::get()<<<grid, threads, smem, stream>>>(
                    (cplx<T>*)state.p, (cplx<T>*)lam.p, (const PassDesc*)(d + o_pass) + i,
                    (const PhaseDesc*)(d + o_phase), (const KOp*)(d + o_ops), (const cplx<T>*)(d + o_pool), part,
                    nslots);
            }
            ++stats.kernel_launches;
            if (i == group_end[gi]) {
                const size_t slot_hi = pass_slot0[i] + nslots;
                const int ns = (int)(slot_hi - slot_lo);
                if (ns > 0) {
                    k_slot_sums<<<ns, 256, 0, stream>>>(partial, (const uint64_t*)(d + o_soff) + slot_lo,
                                                         (const uint64_t*)(d + o_sn) + slot_lo,
                                                         (const uint32_t*)(d + o_sst) + slot_lo, sums);
                    k_param_sums<<<(adj_nparams + 255) / 256, 256, 0, stream>>>(
                        sums, (const int*)(d + o_slots) + slot_lo, ns, adj_nparams, (double*)adj_grad.p);
                    stats.kernel_launches += 2;
                }
                slot_lo = slot_hi;
                ++gi;
            }
        }
        GQ_CUDA(cudaGetLastError());
        stats.jit_passes += jitted;
        stats.passes += (int64_t)np;
        stats.phases += (int64_t)pr.phases.size();
        return GQ_OK;
    }

    // Scheduling options of the reverse sweep (two-state tiles of up to
    // 2^(log2 kAdjThreads + RQ) amplitudes).
    SchedOptions adjoint_options() const {
        SchedOptions o = opt;
        o.tile_qubits = std::min(o.tile_qubits, log2i(kAdjThreads) + RQ);
        return o;
    }
    int run_adjoint(const Program& pr) {
        return prec == GQ_C64 ? run_adjoint_t<float>(pr) : run_adjoint_t<double>(pr);
    }

    bool jit_on() const { return jit_mode != 0 && nphys >= jit_min_qubits && jit_available(); }

    // support: when given, the qubits that may be 1 in a nonzero amplitude of
    // the state before the gates (SchedOptions::support0); it receives the
    // support after them. Only callers that have just reset the state pass it.
    int run_gates(const std::vector<NGate>& gates, uint64_t* support = nullptr) {
        Program pr;
        schedule(gates, nphys, run_options(support), pr);
        return run_scheduled(pr, support);
    }
    // The scheduling options of run_gates.
    SchedOptions run_options(const uint64_t* support) const {
        SchedOptions o = opt;
        o.fuse_pairs = !jit_on();  // specialised kernels take diagonals as free pending factors
        if (support && skip_zero_tiles) o.support0 = *support;
        return o;
    }
    // Runs a program scheduled with run_options(support).
    int run_scheduled(const Program& pr, uint64_t* support) {
        if (support) *support = skip_zero_tiles ? pr.support_out : ~0ull;
        stats.gates_in += pr.gates;
        for (const PassDesc& pd : pr.passes) stats.tile_bytes += (int64_t)(2 * amp_bytes()) << (pd.m + pd.n_outer);
        return prec == GQ_C64 ? run_program_t<float>(pr) : run_program_t<double>(pr);
    }

    int set_jit_option(int key, int64_t value) {
        if (key == GQ_OPT_JIT) {
            if (value < 0 || value > 2) return fail(GQ_EINVAL, "jit mode out of range [0, 2]");
            jit_mode = (int)value;
        } else if (key == GQ_OPT_JIT_PERSISTENT) {
            jit_persistent = value != 0;
        } else if (key == GQ_OPT_JIT_MIN_BLOCKS) {
            if (value < 0 || value > 16) return fail(GQ_EINVAL, "jit min blocks out of range [0, 16]");
            jit_min_blocks = (int)value;
        } else {
            if (value < 0 || value > 64) return fail(GQ_EINVAL, "jit min qubits out of range [0, 64]");
            jit_min_qubits = (int)value;
        }
        return GQ_OK;
    }

    gq_stats get_stats() const {
        gq_stats s = stats;
        jit_counters(&s.jit_compile_ms, nullptr, nullptr);
        return s;
    }

    void clear_stats() {
        const int64_t sb = stats.state_bytes;
        stats = gq_stats{};
        stats.state_bytes = sb;
    }

    // Timing brackets of one apply/evolve call (GQ_OPT_TIMING): events on the
    // handle's stream around the whole call and around its tile passes.
    int time_begin() {
        pass_timed = false;
        if (timing) GQ_CUDA(cudaEventRecord(ev0, stream));
        return GQ_OK;
    }
    int time_end() {
        if (!timing) return GQ_OK;
        GQ_CUDA(cudaEventRecord(ev1, stream));
        GQ_CUDA(cudaEventSynchronize(ev1));
        float ms = 0.f;
        GQ_CUDA(cudaEventElapsedTime(&ms, ev0, ev1));
        stats.last_ms = ms;
        if (pass_timed) {
            GQ_CUDA(cudaEventElapsedTime(&ms, ev_pass0, ev_pass1));
            stats.pass_ms = ms;
        }
        return GQ_OK;
    }

    // ---- reductions -----------------------------------------------------
    int reduce_grid() const { return 148 * 4; }

    // The same without waiting: the sum lands in the second 16 bytes of
    // hostio once the stream has passed this point (read it after a sync).
    int finish_reduce_async(int nblocks) {
        k_final_reduce<<<1, 1024, 0, stream>>>((const double2*)scratch.p, nblocks, (double2*)scratch.p + nblocks);
        GQ_CUDA(cudaGetLastError());
        GQ_TRY(hostio.ensure(64));
        GQ_CUDA(cudaMemcpyAsync((char*)hostio.p + 16, (double2*)scratch.p + nblocks, sizeof(double2),
                                cudaMemcpyDeviceToHost, stream));
        stats.kernel_launches += 2;
        return GQ_OK;
    }

    int finish_reduce(int nblocks, double* re, double* im) {
        k_final_reduce<<<1, 1024, 0, stream>>>((const double2*)scratch.p, nblocks, (double2*)scratch.p + nblocks);
        GQ_CUDA(cudaGetLastError());
        GQ_TRY(hostio.ensure(64));
        GQ_CUDA(cudaMemcpyAsync(hostio.p, (double2*)scratch.p + nblocks, sizeof(double2), cudaMemcpyDeviceToHost,
                                stream));
        GQ_CUDA(cudaStreamSynchronize(stream));
        double2 v = *(double2*)hostio.p;
        if (re) *re = v.x;
        if (im) *im = v.y;
        stats.kernel_launches += 2;
        return GQ_OK;
    }

    // Groups Pauli terms by x mask; uploads them; returns the group count.
    int upload_terms(const gq_pauli_term* terms, size_t n_terms, uint64_t qmask, int* ngroups, size_t* o_terms) {
        std::vector<size_t> order(n_terms);
        for (size_t i = 0; i < n_terms; ++i) {
            if ((terms[i].x_mask | terms[i].z_mask) & ~qmask) return fail(GQ_EINVAL, "Pauli term on a qubit out of range");
            order[i] = i;
        }
        std::stable_sort(order.begin(), order.end(),
                         [&](size_t a, size_t b) { return terms[a].x_mask < terms[b].x_mask; });
        std::vector<DGroup> groups;
        std::vector<DTerm> dt;
        for (size_t k = 0; k < n_terms; ++k) {
            const gq_pauli_term& t = terms[order[k]];
            if (groups.empty() || groups.back().x != t.x_mask) groups.push_back({t.x_mask, (int32_t)k, (int32_t)k});
            groups.back().t1 = (int32_t)k + 1;
            const int ny = __builtin_popcountll(t.x_mask & t.z_mask) & 3;  // iPow (sim/pauli/pauli.go:205-217)
            double pr = 1, pi = 0;
            if (ny == 1) pr = 0, pi = 1;
            if (ny == 2) pr = -1, pi = 0;
            if (ny == 3) pr = 0, pi = -1;
            dt.push_back({t.coeff_re * pr - t.coeff_im * pi, t.coeff_re * pi + t.coeff_im * pr, t.z_mask});
        }
        const size_t og = 0, ot = align16(sizeof(DGroup) * std::max<size_t>(1, groups.size()));
        const size_t total = ot + sizeof(DTerm) * std::max<size_t>(1, dt.size());
        void* hp = nullptr;
        GQ_TRY(stage(total, &hp));
        if (!groups.empty()) std::memcpy((char*)hp + og, groups.data(), sizeof(DGroup) * groups.size());
        if (!dt.empty()) std::memcpy((char*)hp + ot, dt.data(), sizeof(DTerm) * dt.size());
        GQ_TRY(upload(scratch2, total));
        *ngroups = (int)groups.size();
        *o_terms = ot;
        return GQ_OK;
    }

    // ---- shot histograms ---------------------------------------------------
    struct CountsOut {
        uint64_t* outcomes;
        uint64_t* counts;
        size_t* n_distinct;
        int key_bits;  // significant bits of an outcome index
    };

    // The distinct values of the `shots` indices at d_idx (device) with their
    // counts, in increasing order, copied to the caller's host arrays.
    int counts_impl(uint64_t* d_idx, size_t shots, const CountsOut& co) {
        const uint64_t n = shots;
        const uint32_t ntiles = (uint32_t)((n + kHistTile - 1) / kHistTile);
        const uint64_t ncounts = 256ull * ntiles;
        const size_t o_alt = 0, o_cnt = align16(n * 8), o_flag = o_cnt + align16(ncounts * 4);
        const size_t o_start = o_flag + align16(n * 4), o_out = o_start + align16(n * 8);
        const size_t o_num = o_out + align16(n * 8), o_total = o_num + align16(n * 8);
        GQ_TRY(hist.ensure(o_total + 16));
        char* h = (char*)hist.p;
        uint64_t* src = d_idx;
        uint64_t* dst = (uint64_t*)(h + o_alt);
        uint32_t* cnt = (uint32_t*)(h + o_cnt);
        for (int shift = 0; shift < co.key_bits; shift += 8) {
            k_radix_counts<<<ntiles, kHistThreads, 0, stream>>>(src, n, shift, ntiles, cnt);
            k_scan_u32<<<1, 1024, 0, stream>>>(cnt, ncounts, nullptr);
            k_radix_scatter<<<ntiles, kHistThreads, 0, stream>>>(src, n, shift, ntiles, cnt, dst);
            std::swap(src, dst);
            stats.kernel_launches += 3;
        }
        uint32_t* flag = (uint32_t*)(h + o_flag);
        uint32_t* total = (uint32_t*)(h + o_total);
        const unsigned g = (unsigned)std::min<uint64_t>((n + 255) / 256, (uint64_t)reduce_grid());
        k_run_flags<<<g, 256, 0, stream>>>(src, n, flag);
        k_scan_u32<<<1, 1024, 0, stream>>>(flag, n, total);
        k_run_starts<<<g, 256, 0, stream>>>(src, n, flag, (uint64_t*)(h + o_out), (uint64_t*)(h + o_start));
        k_run_counts<<<g, 256, 0, stream>>>((const uint64_t*)(h + o_start), n, total, (uint64_t*)(h + o_num));
        GQ_CUDA(cudaGetLastError());
        stats.kernel_launches += 4;
        GQ_TRY(hostio.ensure(64));
        GQ_CUDA(cudaMemcpyAsync(hostio.p, total, 4, cudaMemcpyDeviceToHost, stream));
        GQ_CUDA(cudaStreamSynchronize(stream));
        const size_t nd = *(const uint32_t*)hostio.p;
        if (nd) {
            GQ_CUDA(cudaMemcpyAsync(co.outcomes, h + o_out, nd * 8, cudaMemcpyDeviceToHost, stream));
            GQ_CUDA(cudaMemcpyAsync(co.counts, h + o_num, nd * 8, cudaMemcpyDeviceToHost, stream));
            GQ_CUDA(cudaStreamSynchronize(stream));
        }
        *co.n_distinct = nd;
        stats.d2h_bytes += (int64_t)(4 + 16 * nd);
        return GQ_OK;
    }

    // ---- sampling --------------------------------------------------------
    // Exact inverse-CDF sampling (see k_chunk_steps in kernels.cuh). The
    // exact chunk-end sums are cached until the state changes. With `co`,
    // the indices stay on the device and become (outcome, count) pairs.
    template <class P>
    int sample_impl(P prob, uint64_t n, const double* uniforms, size_t shots, uint64_t* idx_out,
                    const CountsOut* co = nullptr) {
        if (shots == 0) {
            if (co) *co->n_distinct = 0;
            return GQ_OK;
        }
        const int chunk_log = n >= 2048 ? 11 : (int)std::max<uint64_t>(0, (uint64_t)std::log2((double)n));
        const uint64_t nchunks = (n + (1ull << chunk_log) - 1) >> chunk_log;
        // scratch: sums | incl | ends | steps | cexp | clean | n_seq
        const size_t o_sums = 0, o_incl = o_sums + align16(nchunks * 8), o_ends = o_incl + align16(nchunks * 8);
        const size_t o_steps = o_ends + align16(nchunks * 8), o_exp = o_steps + align16(nchunks * 8);
        const size_t o_clean = o_exp + align16(nchunks * 4), o_nseq = o_clean + align16(nchunks * 4);
        GQ_TRY(scratch.ensure(o_nseq + 16));
        char* sc = (char*)scratch.p;
        double* sums = (double*)(sc + o_sums);
        double* incl = (double*)(sc + o_incl);
        double* ends = (double*)(sc + o_ends);
        const size_t o_u = 0, o_out = align16(shots * 8);
        const size_t io = o_out + align16(shots * 8);
        void* hp = nullptr;
        GQ_TRY(stage(io, &hp));
        std::memcpy((char*)hp + o_u, uniforms, shots * 8);
        GQ_TRY(upload(scratch2, io));
        char* d = (char*)scratch2.p;
        k_chunk_sums<P><<<(unsigned)nchunks, 256, 0, stream>>>(prob, n, chunk_log, sums);
        k_scan_chunks<<<1, 1024, 0, stream>>>(sums, nchunks, incl);
        k_chunk_steps<P><<<(unsigned)nchunks, 256, 0, stream>>>(prob, n, chunk_log, incl, (long long*)(sc + o_steps),
                                                               (int*)(sc + o_exp), (int*)(sc + o_clean));
        k_chunk_walk<P><<<1, 32, 0, stream>>>(prob, n, chunk_log, (const long long*)(sc + o_steps),
                                             (const int*)(sc + o_exp), (const int*)(sc + o_clean), nchunks, ends,
                                             (int*)(sc + o_nseq));
        k_sample_find<P><<<(unsigned)((shots + 127) / 128), 128, 0, stream>>>(
            prob, n, chunk_log, ends, nchunks, (const double*)(d + o_u), shots, (uint64_t*)(d + o_out));
        GQ_CUDA(cudaGetLastError());
        stats.kernel_launches += 5;
        if (co) return counts_impl((uint64_t*)(d + o_out), shots, *co);
        stats.d2h_bytes += (int64_t)(shots * 8);
        GQ_CUDA(cudaMemcpyAsync(idx_out, d + o_out, shots * 8, cudaMemcpyDeviceToHost, stream));
        GQ_CUDA(cudaStreamSynchronize(stream));
        return GQ_OK;
    }
};

bool valid_prec(int p) { return p == GQ_C128 || p == GQ_C64; }

}  // namespace

namespace gq {
// The calling thread's last error, for entry points defined in other files.
void set_last_error(const std::string& msg) { g_err = msg; }
}  // namespace gq

// ============================================================================
struct gq_sv {
    Engine e;
    int nq = 0;
};

struct gq_dm {
    Engine e;
    int nq = 0;
    bool dense_channels = false;  // GQ_OPT_DM_DENSE_CHANNELS
};

extern "C" {

int gq_abi_version(void) { return GQ_ABI_VERSION; }

const char* gq_last_error(void) { return g_err.c_str(); }

int gq_device_count(int* count) {
    if (!count) return fail(GQ_EINVAL, "null count");
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) {
        cudaGetLastError();
        n = 0;
    }
    int ok = 0;
    for (int i = 0; i < n; ++i) {
        cudaDeviceProp p;
        if (cudaGetDeviceProperties(&p, i) == cudaSuccess && p.major == 10) ++ok;
    }
    *count = ok;
    return GQ_OK;
}

// ---- statevector ------------------------------------------------------------
int gq_sv_create(int num_qubits, int precision, gq_sv** out) {
    if (!out) return fail(GQ_EINVAL, "null output handle");
    *out = nullptr;
    if (num_qubits < 1 || num_qubits > 34)
        return fail(GQ_EINVAL, "statevector: numQubits " + std::to_string(num_qubits) + " out of range [1, 34]");
    if (!valid_prec(precision)) return fail(GQ_EINVAL, "unknown precision");
    gq_sv* h = new gq_sv();
    h->nq = num_qubits;
    int rc = h->e.init(std::max(num_qubits, RQ), precision);
    if (rc != GQ_OK) {
        h->e.destroy();
        delete h;
        return rc;
    }
    *out = h;
    return GQ_OK;
}

int gq_sv_destroy(gq_sv* sv) {
    if (!sv) return GQ_OK;
    sv->e.destroy();
    delete sv;
    return GQ_OK;
}

int gq_sv_num_qubits(const gq_sv* sv, int* out) {
    if (!sv || !out) return fail(GQ_EINVAL, "null argument");
    *out = sv->nq;
    return GQ_OK;
}

int gq_sv_reset(gq_sv* sv) {
    if (!sv) return fail(GQ_EINVAL, "null handle");
    return sv->e.reset_basis(0);
}

// support: see Engine::run_gates (null: the state is arbitrary).
static int sv_apply_impl(gq_sv* sv, const gq_op* ops, size_t n_ops, uint64_t* support = nullptr) {
    if (n_ops && !ops) return fail(GQ_EINVAL, "null ops");
    std::vector<NGate> gates;
    std::string err;
    for (size_t i = 0; i < n_ops; ++i) {
        if (ops[i].kind == GQ_OP_CHANNEL) return fail(GQ_EINVAL, "op " + std::to_string(i) + ": channel on a statevector");
        int rc = normalize_op(ops[i], sv->nq, gates, err);
        if (rc != GQ_OK) return fail(rc, "op " + std::to_string(i) + ": " + err);
        if (!gates.empty() && gates.back().src < 0) gates.back().src = (int)i;
    }
    return sv->e.run_gates(gates, support);
}

namespace {
int sv_apply_timed(gq_sv* sv, const gq_op* ops, size_t n_ops, bool reset) {
    if (!sv) return fail(GQ_EINVAL, "null handle");
    sv->e.clear_stats();
    GQ_TRY(sv->e.time_begin());
    uint64_t support = 0;  // |0...0>: no qubit is 1 in a nonzero amplitude
    if (reset) GQ_TRY(sv->e.reset_basis(0));
    GQ_TRY(sv_apply_impl(sv, ops, n_ops, reset ? &support : nullptr));
    return sv->e.time_end();
}
}  // namespace

int gq_sv_apply(gq_sv* sv, const gq_op* ops, size_t n_ops) { return sv_apply_timed(sv, ops, n_ops, false); }

int gq_sv_evolve(gq_sv* sv, const gq_op* ops, size_t n_ops) { return sv_apply_timed(sv, ops, n_ops, true); }

int gq_sv_get_state(gq_sv* sv, void* host_out, size_t bytes) {
    if (!sv || !host_out) return fail(GQ_EINVAL, "null argument");
    const size_t need = (1ull << sv->nq) * sv->e.amp_bytes();
    if (bytes < need) return fail(GQ_EINVAL, "output buffer too small");
    GQ_CUDA(cudaMemcpyAsync(host_out, sv->e.state.p, need, cudaMemcpyDeviceToHost, sv->e.stream));
    GQ_CUDA(cudaStreamSynchronize(sv->e.stream));
    return GQ_OK;
}

int gq_sv_set_state(gq_sv* sv, const void* host_in, size_t bytes) {
    if (!sv || !host_in) return fail(GQ_EINVAL, "null argument");
    const size_t need = (1ull << sv->nq) * sv->e.amp_bytes();
    if (bytes != need) return fail(GQ_EINVAL, "state size mismatch");
    if (sv->nq < RQ) GQ_CUDA(cudaMemsetAsync(sv->e.state.p, 0, sv->e.n_amps * sv->e.amp_bytes(), sv->e.stream));
    GQ_CUDA(cudaMemcpyAsync(sv->e.state.p, host_in, need, cudaMemcpyHostToDevice, sv->e.stream));
    GQ_CUDA(cudaStreamSynchronize(sv->e.stream));
    return GQ_OK;
}

int gq_sv_probabilities(gq_sv* sv, double* host_out, size_t n) {
    if (!sv || !host_out) return fail(GQ_EINVAL, "null argument");
    const uint64_t na = 1ull << sv->nq;
    if (n < na) return fail(GQ_EINVAL, "output buffer too small");
    Engine& e = sv->e;
    GQ_TRY(e.scratch.ensure(na * 8));
    if (e.prec == GQ_C64)
        k_probs<float><<<e.reduce_grid(), 256, 0, e.stream>>>((const cplx<float>*)e.state.p, na, (double*)e.scratch.p);
    else
        k_probs<double><<<e.reduce_grid(), 256, 0, e.stream>>>((const cplx<double>*)e.state.p, na, (double*)e.scratch.p);
    GQ_CUDA(cudaGetLastError());
    GQ_CUDA(cudaMemcpyAsync(host_out, e.scratch.p, na * 8, cudaMemcpyDeviceToHost, e.stream));
    GQ_CUDA(cudaStreamSynchronize(e.stream));
    return GQ_OK;
}

int gq_sv_sample(gq_sv* sv, const double* uniforms, size_t shots, uint64_t* idx_out) {
    if (!sv) return fail(GQ_EINVAL, "null handle");
    if (shots && (!uniforms || !idx_out)) return fail(GQ_EINVAL, "null argument");
    for (size_t i = 0; i < shots; ++i)
        if (!(uniforms[i] >= 0.0 && uniforms[i] < 1.0)) return fail(GQ_EINVAL, "uniform outside [0, 1)");
    const uint64_t na = 1ull << sv->nq;
    Engine& e = sv->e;
    if (e.prec == GQ_C64) return e.sample_impl(ProbState<float>{(const cplx<float>*)e.state.p}, na, uniforms, shots, idx_out);
    return e.sample_impl(ProbState<double>{(const cplx<double>*)e.state.p}, na, uniforms, shots, idx_out);
}

int gq_sv_run(gq_sv* sv, const gq_op* ops, size_t n_ops, const double* uniforms, size_t shots, uint64_t* idx_out) {
    GQ_TRY(gq_sv_evolve(sv, ops, n_ops));  // resets the counters of this call
    return gq_sv_sample(sv, uniforms, shots, idx_out);
}

int gq_sv_sample_counts(gq_sv* sv, const double* uniforms, size_t shots, uint64_t* outcomes_out, uint64_t* counts_out,
                        size_t* n_distinct) {
    if (!sv) return fail(GQ_EINVAL, "null handle");
    if (!n_distinct || (shots && (!uniforms || !outcomes_out || !counts_out))) return fail(GQ_EINVAL, "null argument");
    if (shots > 0xffffffffull) return fail(GQ_EINVAL, "more than 2^32 - 1 shots");
    for (size_t i = 0; i < shots; ++i)
        if (!(uniforms[i] >= 0.0 && uniforms[i] < 1.0)) return fail(GQ_EINVAL, "uniform outside [0, 1)");
    const uint64_t na = 1ull << sv->nq;
    Engine& e = sv->e;
    const Engine::CountsOut co{outcomes_out, counts_out, n_distinct, sv->nq};
    if (e.prec == GQ_C64)
        return e.sample_impl(ProbState<float>{(const cplx<float>*)e.state.p}, na, uniforms, shots, nullptr, &co);
    return e.sample_impl(ProbState<double>{(const cplx<double>*)e.state.p}, na, uniforms, shots, nullptr, &co);
}

int gq_sv_run_counts(gq_sv* sv, const gq_op* ops, size_t n_ops, const double* uniforms, size_t shots,
                     uint64_t* outcomes_out, uint64_t* counts_out, size_t* n_distinct) {
    GQ_TRY(gq_sv_evolve(sv, ops, n_ops));  // resets the counters of this call
    return gq_sv_sample_counts(sv, uniforms, shots, outcomes_out, counts_out, n_distinct);
}

int gq_sv_expect_pauli_sum(gq_sv* sv, const gq_pauli_term* terms, size_t n_terms, double* out_re, double* out_im) {
    if (!sv) return fail(GQ_EINVAL, "null handle");
    if (n_terms && !terms) return fail(GQ_EINVAL, "null terms");
    Engine& e = sv->e;
    int ng = 0;
    size_t ot = 0;
    GQ_TRY(e.upload_terms(terms, n_terms, (sv->nq >= 64) ? ~0ull : ((1ull << sv->nq) - 1), &ng, &ot));
    const int nb = e.reduce_grid();
    GQ_TRY(e.scratch.ensure((nb + 1) * sizeof(double2)));
    const char* d = (const char*)e.scratch2.p;
    const uint64_t na = 1ull << sv->nq;
    if (e.prec == GQ_C64)
        k_expect<float><<<nb, 256, 0, e.stream>>>((const cplx<float>*)e.state.p, na, (const DGroup*)d, ng,
                                                  (const DTerm*)(d + ot), (double2*)e.scratch.p);
    else
        k_expect<double><<<nb, 256, 0, e.stream>>>((const cplx<double>*)e.state.p, na, (const DGroup*)d, ng,
                                                   (const DTerm*)(d + ot), (double2*)e.scratch.p);
    GQ_CUDA(cudaGetLastError());
    return e.finish_reduce(nb, out_re, out_im);
}

int gq_sv_expect_z_mask(gq_sv* sv, uint64_t mask, double* out) {
    gq_pauli_term t{1.0, 0.0, 0, mask};
    return gq_sv_expect_pauli_sum(sv, &t, 1, out, nullptr);
}

int gq_sv_prob0(gq_sv* sv, int qubit, double* p0) {
    if (!sv || !p0) return fail(GQ_EINVAL, "null argument");
    if (qubit < 0 || qubit >= sv->nq) return fail(GQ_EINVAL, "qubit out of range");
    Engine& e = sv->e;
    const int nb = e.reduce_grid();
    GQ_TRY(e.scratch.ensure((nb + 1) * sizeof(double2)));
    const uint64_t na = 1ull << sv->nq;
    if (e.prec == GQ_C64)
        k_prob_bit<float><<<nb, 256, 0, e.stream>>>((const cplx<float>*)e.state.p, na, qubit, (double2*)e.scratch.p);
    else
        k_prob_bit<double><<<nb, 256, 0, e.stream>>>((const cplx<double>*)e.state.p, na, qubit, (double2*)e.scratch.p);
    GQ_CUDA(cudaGetLastError());
    return e.finish_reduce(nb, p0, nullptr);
}

int gq_sv_collapse(gq_sv* sv, int qubit, int outcome, double p0) {
    if (!sv) return fail(GQ_EINVAL, "null handle");
    if (qubit < 0 || qubit >= sv->nq) return fail(GQ_EINVAL, "qubit out of range");
    if (outcome != 0 && outcome != 1) return fail(GQ_EINVAL, "outcome must be 0 or 1");
    // dynamic.go:203-229: norm from prob0 (1 - prob0 for outcome 1); a
    // norm below 1e-15 means the outcome was certain and nothing changes
    const double norm = outcome == 0 ? std::sqrt(p0) : std::sqrt(1.0 - p0);
    if (!(norm >= 1e-15)) return GQ_OK;
    Engine& e = sv->e;
    const uint64_t na = 1ull << sv->nq;
    const int nb = e.reduce_grid();
    if (e.prec == GQ_C64)
        k_collapse<float><<<nb, 256, 0, e.stream>>>((cplx<float>*)e.state.p, na, qubit, outcome, 1.0 / norm);
    else
        k_collapse<double><<<nb, 256, 0, e.stream>>>((cplx<double>*)e.state.p, na, qubit, outcome, 1.0 / norm);
    GQ_CUDA(cudaGetLastError());
    e.stats.kernel_launches += 1;
    return GQ_OK;
}

int gq_sv_measure(gq_sv* sv, int qubit, double u, int* outcome) {
    if (!sv || !outcome) return fail(GQ_EINVAL, "null argument");
    double p0 = 0.0;
    GQ_TRY(gq_sv_prob0(sv, qubit, &p0));
    *outcome = u >= p0 ? 1 : 0;  // dynamic.go:197-200
    return gq_sv_collapse(sv, qubit, *outcome, p0);
}

int gq_sv_copy_state(gq_sv* dst, const gq_sv* src) {
    if (!dst || !src) return fail(GQ_EINVAL, "null handle");
    if (dst->nq != src->nq || dst->e.prec != src->e.prec)
        return fail(GQ_EINVAL, "handles differ in qubit count or precision");
    if (dst == src) return GQ_OK;
    // both streams are idle on return, so either state may be changed next
    GQ_CUDA(cudaStreamSynchronize(src->e.stream));
    GQ_CUDA(cudaMemcpyAsync(dst->e.state.p, src->e.state.p, src->e.n_amps * src->e.amp_bytes(),
                            cudaMemcpyDeviceToDevice, dst->e.stream));
    GQ_CUDA(cudaStreamSynchronize(dst->e.stream));
    return GQ_OK;
}

int gq_sv_stats(const gq_sv* sv, gq_stats* out) {
    if (!sv || !out) return fail(GQ_EINVAL, "null argument");
    *out = sv->e.get_stats();
    return GQ_OK;
}

int gq_sv_set_option(gq_sv* sv, int key, int64_t value) {
    if (!sv) return fail(GQ_EINVAL, "null handle");
    Engine& e = sv->e;
    switch (key) {
        case GQ_OPT_TILE_QUBITS:
            if (value < RQ || value > e.max_tile())
                return fail(GQ_EINVAL, "tile qubits out of range [4, " + std::to_string(e.max_tile()) + "]");
            e.opt.tile_qubits = (int)value;
            return GQ_OK;
        case GQ_OPT_PASS_BUDGET:
            if (value < 0) return fail(GQ_EINVAL, "negative budget");
            e.opt.budget = value == 0 ? kDefaultBudget : (int)value;
            return GQ_OK;
        case GQ_OPT_LOW_QUBITS:
            if (value < 0 || value > 6) return fail(GQ_EINVAL, "low qubits out of range [0, 6]");
            e.opt.low_qubits = (int)value;
            return GQ_OK;
        case GQ_OPT_TIMING:
            e.timing = value != 0;
            return GQ_OK;
        case GQ_OPT_KERNEL_VARIANT:
            if (value < 0 || value >= kNumVariants) return fail(GQ_EINVAL, "kernel variant out of range");
            e.variant = (int)value;
            e.opt.tile_qubits = e.max_tile();
            return GQ_OK;
        case GQ_OPT_ADJOINT_SEGMENTS:
            if (value < 0 || value > 4096) return fail(GQ_EINVAL, "adjoint segments out of range [0, 4096]");
            e.adj_segments = (int)value;
            return GQ_OK;
        case GQ_OPT_FUSE_DENSE:
            e.opt.fuse_dense = value != 0;
            return GQ_OK;
        case GQ_OPT_ZERO_TILES:
            e.skip_zero_tiles = value != 0;
            return GQ_OK;
        case GQ_OPT_JIT:
        case GQ_OPT_JIT_MIN_QUBITS:
        case GQ_OPT_JIT_MIN_BLOCKS:
        case GQ_OPT_JIT_PERSISTENT:
            return e.set_jit_option(key, value);
        default:
            return fail(GQ_EINVAL, "unknown option");
    }
}

int gq_sv_adjoint_gradient(gq_sv* sv, const gq_op* ops, size_t n_ops, const gq_pauli_term* terms, size_t n_terms,
                           size_t n_params, double* grad_out, double* energy_out) {
    if (!sv) return fail(GQ_EINVAL, "null handle");
    if ((n_ops && !ops) || (n_terms && !terms) || (n_params && !grad_out)) return fail(GQ_EINVAL, "null argument");
    Engine& e = sv->e;
    std::vector<NGate> fwd, rev;
    std::vector<int> fo, ro;
    {
        std::string err;
        int rc = adjoint_gates(sv->nq, ops, n_ops, n_params, fwd, rev, fo, ro, err);
        if (rc != GQ_OK) return fail(rc, err);
    }
    e.clear_stats();
    GQ_TRY(e.time_begin());
    const size_t sbytes = e.n_amps * e.amp_bytes();
    GQ_TRY(e.lam.ensure(sbytes));
    GQ_TRY(e.adj_grad.ensure(std::max<size_t>(1, n_params) * sizeof(double)));
    e.adj_nparams = (int)n_params;
    // Forward segments (checkpoints bound the drift of un-applying gates).
    // The automatic count only takes the device memory that is free: the
    // checkpoint buffer's current allocation is released before it grows.
    size_t mem_free = 0, mem_total = 0;
    GQ_CUDA(cudaMemGetInfo(&mem_free, &mem_total));
    const int segs = adjoint_segments(e.adj_segments, e.prec == GQ_C64, n_ops, sbytes, mem_free + e.ckpt.cap);
    std::vector<size_t> bound(segs + 1);
    for (int j = 0; j <= segs; ++j) bound[j] = n_ops * (size_t)j / (size_t)segs;
    if (segs > 1) GQ_TRY(e.ckpt.ensure(sbytes * (segs - 1)));
    auto seg_of = [&](int op_index) {
        int j = 0;
        while (j + 1 < segs && (size_t)op_index >= bound[j + 1]) ++j;
        return j;
    };
    // The reverse programs depend on the gates only: a worker thread
    // schedules them while this thread schedules and launches the forward
    // sweep (the future joins on every return path).
    std::vector<std::vector<NGate>> rparts(segs);
    for (size_t k = 0; k < rev.size(); ++k) rparts[seg_of(ro[k])].push_back(rev[k]);
    const SchedOptions ropt = e.adjoint_options();
    const int nphys = e.nphys;
    auto rprogs = std::async(std::launch::async, [&rparts, &ropt, nphys] {
        std::vector<Program> progs(rparts.size());
        for (size_t j = 0; j < rparts.size(); ++j) schedule(rparts[j], nphys, ropt, progs[j]);
        return progs;
    });
    GQ_TRY(e.reset_basis(0));
    uint64_t support = 0;
    for (int j = 0; j < segs; ++j) {
        std::vector<NGate> part;
        for (size_t k = 0; k < fwd.size(); ++k)
            if (seg_of(fo[k]) == j) part.push_back(fwd[k]);
        GQ_TRY(e.run_gates(part, &support));
        if (j + 1 < segs)
            GQ_CUDA(cudaMemcpyAsync((char*)e.ckpt.p + sbytes * j, e.state.p, sbytes, cudaMemcpyDeviceToDevice, e.stream));
    }
    // lambda = Re(H) psi and the energy
    std::vector<gq_pauli_term> rt(terms, terms + n_terms);
    for (auto& t : rt) t.coeff_im = 0.0;
    int ng = 0;
    size_t ot = 0;
    GQ_TRY(e.upload_terms(rt.data(), rt.size(), (1ull << sv->nq) - 1, &ng, &ot));
    const int nb = e.reduce_grid();
    GQ_TRY(e.scratch.ensure((nb + 1) * sizeof(double2)));
    {
        const char* d = (const char*)e.scratch2.p;
        const uint64_t na = 1ull << sv->nq;
        if (sv->nq < RQ) GQ_CUDA(cudaMemsetAsync(e.lam.p, 0, sbytes, e.stream));
        if (e.prec == GQ_C64)
            k_apply_terms<float><<<nb, 256, 0, e.stream>>>((const cplx<float>*)e.state.p, (cplx<float>*)e.lam.p, na,
                                                           (const DGroup*)d, ng, (const DTerm*)(d + ot),
                                                           (double2*)e.scratch.p);
        else
            k_apply_terms<double><<<nb, 256, 0, e.stream>>>((const cplx<double>*)e.state.p, (cplx<double>*)e.lam.p,
                                                            na, (const DGroup*)d, ng, (const DTerm*)(d + ot),
                                                            (double2*)e.scratch.p);
        GQ_CUDA(cudaGetLastError());
        GQ_TRY(e.finish_reduce_async(nb));  // read after the final synchronisation
        ++e.stats.kernel_launches;
    }
    // reverse sweep
    GQ_CUDA(cudaMemsetAsync(e.adj_grad.p, 0, std::max<size_t>(1, n_params) * sizeof(double), e.stream));
    const std::vector<Program> rp = rprogs.get();
    for (int j = segs - 1; j >= 0; --j) {
        if (j + 1 < segs)
            GQ_CUDA(cudaMemcpyAsync(e.state.p, (char*)e.ckpt.p + sbytes * j, sbytes, cudaMemcpyDeviceToDevice, e.stream));
        GQ_TRY(e.run_adjoint(rp[j]));
    }
    if (n_params) {
        GQ_CUDA(cudaMemcpyAsync(grad_out, e.adj_grad.p, n_params * sizeof(double), cudaMemcpyDeviceToHost, e.stream));
        e.stats.d2h_bytes += (int64_t)(n_params * sizeof(double));
    }
    GQ_CUDA(cudaStreamSynchronize(e.stream));
    if (energy_out) *energy_out = ((const double2*)((const char*)e.hostio.p + 16))->x;
    return e.time_end();
}

// ---- density matrix -----------------------------------------------------------

int gq_dm_create(int num_qubits, gq_dm** out) {
    if (!out) return fail(GQ_EINVAL, "null output handle");
    *out = nullptr;
    if (num_qubits < 1 || num_qubits > 15)
        return fail(GQ_EINVAL, "densitymatrix: numQubits " + std::to_string(num_qubits) + " out of range [1, 15]");
    gq_dm* h = new gq_dm();
    h->nq = num_qubits;
    int rc = h->e.init(std::max(2 * num_qubits, RQ), GQ_C128);
    if (rc != GQ_OK) {
        h->e.destroy();
        delete h;
        return rc;
    }
    *out = h;
    return GQ_OK;
}

int gq_dm_destroy(gq_dm* dm) {
    if (!dm) return GQ_OK;
    dm->e.destroy();
    delete dm;
    return GQ_OK;
}

int gq_dm_reset(gq_dm* dm) {
    if (!dm) return fail(GQ_EINVAL, "null handle");
    return dm->e.reset_basis(0);
}

// support: see Engine::run_gates (null: the state is arbitrary).
// Op streams at least this long are analysed and scheduled in two halves.
constexpr size_t kDmSplitOps = 256;

static int dm_apply_impl(gq_dm* dm, const gq_op* ops, size_t n_ops, uint64_t* support = nullptr) {
    if (n_ops && !ops) return fail(GQ_EINVAL, "null ops");
    const bool structured = !dm->dense_channels;
    // A long stream is split at a gate (a gate keeps the channel after it): a
    // worker thread analyses and schedules the second half while this thread
    // does the first and launches it. Nothing launches before both halves
    // passed the analysis, as for the whole stream.
    size_t mid = n_ops >= kDmSplitOps ? n_ops / 2 : n_ops;
    while (mid < n_ops && ops[mid].kind == GQ_OP_CHANNEL) ++mid;
    if (mid >= n_ops) {
        std::vector<NGate> gates;
        std::string err;
        int rc = dm_gates(dm->nq, ops, n_ops, gates, err, structured);
        if (rc != GQ_OK) return fail(rc, err);
        return dm->e.run_gates(gates, support);
    }
    const int nq = dm->nq, nphys = dm->e.nphys;
    const SchedOptions o2 = dm->e.run_options(nullptr);  // the second half's start state is arbitrary
    std::promise<int> analysed;
    std::future<int> analysed_rc = analysed.get_future();
    auto second = std::async(std::launch::async, [&analysed, &o2, ops, n_ops, mid, nq, nphys, structured] {
        std::vector<NGate> g;
        std::string err;
        const int rc = dm_gates(nq, ops + mid, n_ops - mid, g, err, structured);
        analysed.set_value(rc);
        Program pr;
        if (rc == GQ_OK) schedule(g, nphys, o2, pr);
        return pr;
    });
    std::vector<NGate> gates;
    std::string err;
    int rc = dm_gates(nq, ops, mid, gates, err, structured);
    if (rc != GQ_OK) return fail(rc, err);
    Program first;
    schedule(gates, nphys, dm->e.run_options(support), first);
    if (analysed_rc.get() != GQ_OK) {
        // the message names the op in the whole stream
        std::vector<NGate> all;
        rc = dm_gates(nq, ops, n_ops, all, err, structured);
        return fail(rc != GQ_OK ? rc : GQ_EINVAL, err);
    }
    GQ_TRY(dm->e.run_scheduled(first, support));
    const Program pr = second.get();
    return dm->e.run_scheduled(pr, support ? support : nullptr);
}

static int dm_apply_timed(gq_dm* dm, const gq_op* ops, size_t n_ops, bool reset) {
    if (!dm) return fail(GQ_EINVAL, "null handle");
    dm->e.clear_stats();
    GQ_TRY(dm->e.time_begin());
    uint64_t support = 0;  // |0...0><0...0| is entry 0 of the vectorised matrix
    if (reset) GQ_TRY(dm->e.reset_basis(0));
    GQ_TRY(dm_apply_impl(dm, ops, n_ops, reset ? &support : nullptr));
    return dm->e.time_end();
}

int gq_dm_apply(gq_dm* dm, const gq_op* ops, size_t n_ops) { return dm_apply_timed(dm, ops, n_ops, false); }

int gq_dm_evolve(gq_dm* dm, const gq_op* ops, size_t n_ops) { return dm_apply_timed(dm, ops, n_ops, true); }

int gq_dm_set_option(gq_dm* dm, int key, int64_t value) {
    if (!dm) return fail(GQ_EINVAL, "null handle");
    if (key == GQ_OPT_TIMING) {
        dm->e.timing = value != 0;
        return GQ_OK;
    }
    if (key == GQ_OPT_PASS_BUDGET) {
        if (value < 0) return fail(GQ_EINVAL, "negative budget");
        dm->e.opt.budget = value == 0 ? kDefaultBudget : (int)value;
        return GQ_OK;
    }
    if (key == GQ_OPT_TILE_QUBITS) {
        if (value < RQ || value > dm->e.max_tile()) return fail(GQ_EINVAL, "tile qubits out of range");
        dm->e.opt.tile_qubits = (int)value;
        return GQ_OK;
    }
    if (key == GQ_OPT_KERNEL_VARIANT) {
        if (value < 0 || value >= kNumVariants) return fail(GQ_EINVAL, "kernel variant out of range");
        dm->e.variant = (int)value;
        dm->e.opt.tile_qubits = dm->e.max_tile();
        return GQ_OK;
    }
    if (key == GQ_OPT_JIT || key == GQ_OPT_JIT_MIN_QUBITS || key == GQ_OPT_JIT_MIN_BLOCKS ||
        key == GQ_OPT_JIT_PERSISTENT)
        return dm->e.set_jit_option(key, value);
    if (key == GQ_OPT_DM_DENSE_CHANNELS) {
        dm->dense_channels = value != 0;
        return GQ_OK;
    }
    if (key == GQ_OPT_ZERO_TILES) {
        dm->e.skip_zero_tiles = value != 0;
        return GQ_OK;
    }
    return fail(GQ_EINVAL, "unknown option");
}

int gq_dm_get(gq_dm* dm, double* host_out, size_t bytes) {
    if (!dm || !host_out) return fail(GQ_EINVAL, "null argument");
    const size_t need = (1ull << (2 * dm->nq)) * 16;
    if (bytes < need) return fail(GQ_EINVAL, "output buffer too small");
    GQ_CUDA(cudaMemcpyAsync(host_out, dm->e.state.p, need, cudaMemcpyDeviceToHost, dm->e.stream));
    GQ_CUDA(cudaStreamSynchronize(dm->e.stream));
    return GQ_OK;
}

int gq_dm_set(gq_dm* dm, const double* host_in, size_t bytes) {
    if (!dm || !host_in) return fail(GQ_EINVAL, "null argument");
    const size_t need = (1ull << (2 * dm->nq)) * 16;
    if (bytes != need) return fail(GQ_EINVAL, "size mismatch");
    if (2 * dm->nq < RQ) GQ_CUDA(cudaMemsetAsync(dm->e.state.p, 0, dm->e.n_amps * 16, dm->e.stream));
    GQ_CUDA(cudaMemcpyAsync(dm->e.state.p, host_in, need, cudaMemcpyHostToDevice, dm->e.stream));
    GQ_CUDA(cudaStreamSynchronize(dm->e.stream));
    return GQ_OK;
}

int gq_dm_diagonal_probs(gq_dm* dm, double* host_out, size_t n) {
    if (!dm || !host_out) return fail(GQ_EINVAL, "null argument");
    const uint64_t dim = 1ull << dm->nq;
    if (n < dim) return fail(GQ_EINVAL, "output buffer too small");
    Engine& e = dm->e;
    GQ_TRY(e.scratch.ensure(dim * 8));
    k_dm_diag_probs<<<e.reduce_grid(), 256, 0, e.stream>>>((const cplx<double>*)e.state.p, dim, (double*)e.scratch.p);
    GQ_CUDA(cudaGetLastError());
    GQ_CUDA(cudaMemcpyAsync(host_out, e.scratch.p, dim * 8, cudaMemcpyDeviceToHost, e.stream));
    GQ_CUDA(cudaStreamSynchronize(e.stream));
    return GQ_OK;
}

int gq_dm_expect_pauli_sum(gq_dm* dm, const gq_pauli_term* terms, size_t n_terms, double* out_re, double* out_im) {
    if (!dm) return fail(GQ_EINVAL, "null handle");
    if (n_terms && !terms) return fail(GQ_EINVAL, "null terms");
    Engine& e = dm->e;
    int ng = 0;
    size_t ot = 0;
    GQ_TRY(e.upload_terms(terms, n_terms, (1ull << dm->nq) - 1, &ng, &ot));
    const int nb = e.reduce_grid();
    GQ_TRY(e.scratch.ensure((nb + 1) * sizeof(double2)));
    const char* d = (const char*)e.scratch2.p;
    k_dm_expect<<<nb, 256, 0, e.stream>>>((const cplx<double>*)e.state.p, 1ull << dm->nq, (const DGroup*)d, ng,
                                          (const DTerm*)(d + ot), (double2*)e.scratch.p);
    GQ_CUDA(cudaGetLastError());
    return e.finish_reduce(nb, out_re, out_im);
}

int gq_dm_trace(gq_dm* dm, double* out_re, double* out_im) {
    gq_pauli_term t{1.0, 0.0, 0, 0};
    return gq_dm_expect_pauli_sum(dm, &t, 1, out_re, out_im);
}

int gq_dm_purity(gq_dm* dm, double* out) {
    if (!dm || !out) return fail(GQ_EINVAL, "null argument");
    Engine& e = dm->e;
    const int nb = e.reduce_grid();
    GQ_TRY(e.scratch.ensure((nb + 1) * sizeof(double2)));
    k_dm_purity<<<nb, 256, 0, e.stream>>>((const cplx<double>*)e.state.p, 1ull << dm->nq, (double2*)e.scratch.p);
    GQ_CUDA(cudaGetLastError());
    double re = 0;
    GQ_TRY(e.finish_reduce(nb, &re, nullptr));
    *out = std::fabs(re);
    return GQ_OK;
}

int gq_dm_fidelity(gq_dm* dm, const double* psi, size_t n, double* out) {
    if (!dm || !psi || !out) return fail(GQ_EINVAL, "null argument");
    const uint64_t dim = 1ull << dm->nq;
    if (n != dim) return fail(GQ_EINVAL, "densitymatrix: pure state length mismatch");
    Engine& e = dm->e;
    void* hp = nullptr;
    GQ_TRY(e.stage(dim * 16, &hp));
    std::memcpy(hp, psi, dim * 16);
    GQ_TRY(e.upload(e.scratch2, dim * 16));
    const int nb = e.reduce_grid();
    GQ_TRY(e.scratch.ensure((nb + 1) * sizeof(double2)));
    k_dm_fidelity<<<nb, 256, 0, e.stream>>>((const cplx<double>*)e.state.p, dim, (const cplx<double>*)e.scratch2.p,
                                            (double2*)e.scratch.p);
    GQ_CUDA(cudaGetLastError());
    double re = 0;
    GQ_TRY(e.finish_reduce(nb, &re, nullptr));
    *out = std::fabs(re);
    return GQ_OK;
}

static int dm_sample_impl(gq_dm* dm, const double* p01, const double* p10, const double* uniforms, size_t shots,
                          uint64_t* idx_out, const Engine::CountsOut* co) {
    for (size_t i = 0; i < shots; ++i)
        if (!(uniforms[i] >= 0.0 && uniforms[i] < 1.0)) return fail(GQ_EINVAL, "uniform outside [0, 1)");
    Engine& e = dm->e;
    const uint64_t dim = 1ull << dm->nq;
    // probs live in `aux`; the sampler uses scratch / scratch2.
    GQ_TRY(e.aux.ensure(2 * dim * 8));
    double* a = (double*)e.aux.p;
    double* b = a + dim;
    k_dm_diag_probs<<<e.reduce_grid(), 256, 0, e.stream>>>((const cplx<double>*)e.state.p, dim, a);
    if (p01 && p10)
        for (int q = 0; q < dm->nq; ++q) {
            if (p01[q] < 0) continue;
            k_readout_qubit<<<e.reduce_grid(), 256, 0, e.stream>>>(a, b, dim, 1ull << q, p01[q], p10[q]);
            std::swap(a, b);
        }
    GQ_CUDA(cudaGetLastError());
    return e.sample_impl(ProbArray{a}, dim, uniforms, shots, idx_out, co);
}

int gq_dm_sample(gq_dm* dm, const double* p01, const double* p10, const double* uniforms, size_t shots,
                 uint64_t* idx_out) {
    if (!dm) return fail(GQ_EINVAL, "null handle");
    if (shots && (!uniforms || !idx_out)) return fail(GQ_EINVAL, "null argument");
    return dm_sample_impl(dm, p01, p10, uniforms, shots, idx_out, nullptr);
}

int gq_dm_sample_counts(gq_dm* dm, const double* p01, const double* p10, const double* uniforms, size_t shots,
                        uint64_t* outcomes_out, uint64_t* counts_out, size_t* n_distinct) {
    if (!dm) return fail(GQ_EINVAL, "null handle");
    if (!n_distinct || (shots && (!uniforms || !outcomes_out || !counts_out))) return fail(GQ_EINVAL, "null argument");
    if (shots > 0xffffffffull) return fail(GQ_EINVAL, "more than 2^32 - 1 shots");
    const Engine::CountsOut co{outcomes_out, counts_out, n_distinct, dm->nq};
    return dm_sample_impl(dm, p01, p10, uniforms, shots, nullptr, &co);
}

int gq_dm_prob0(gq_dm* dm, int qubit, double* p0) {
    if (!dm || !p0) return fail(GQ_EINVAL, "null argument");
    if (qubit < 0 || qubit >= dm->nq) return fail(GQ_EINVAL, "qubit out of range");
    Engine& e = dm->e;
    const int nb = e.reduce_grid();
    GQ_TRY(e.scratch.ensure((nb + 1) * sizeof(double2)));
    k_dm_prob_bit<<<nb, 256, 0, e.stream>>>((const cplx<double>*)e.state.p, 1ull << dm->nq, qubit,
                                            (double2*)e.scratch.p);
    GQ_CUDA(cudaGetLastError());
    return e.finish_reduce(nb, p0, nullptr);
}

int gq_dm_collapse(gq_dm* dm, int qubit, int outcome, double p0) {
    if (!dm) return fail(GQ_EINVAL, "null handle");
    if (qubit < 0 || qubit >= dm->nq) return fail(GQ_EINVAL, "qubit out of range");
    if (outcome != 0 && outcome != 1) return fail(GQ_EINVAL, "outcome must be 0 or 1");
    // dynamic.go:231-254: divide by the outcome's probability (1 - prob0 for
    // outcome 1); below 1e-15 the outcome was certain and nothing changes
    const double p = outcome == 0 ? p0 : 1.0 - p0;
    if (!(p >= 1e-15)) return GQ_OK;
    Engine& e = dm->e;
    k_dm_collapse<<<e.reduce_grid(), 256, 0, e.stream>>>((cplx<double>*)e.state.p, 1ull << dm->nq, qubit, outcome,
                                                         1.0 / p);
    GQ_CUDA(cudaGetLastError());
    e.stats.kernel_launches += 1;
    return GQ_OK;
}

int gq_dm_measure(gq_dm* dm, int qubit, double u, int* outcome) {
    if (!dm || !outcome) return fail(GQ_EINVAL, "null argument");
    double p0 = 0.0;
    GQ_TRY(gq_dm_prob0(dm, qubit, &p0));
    *outcome = u >= p0 ? 1 : 0;
    return gq_dm_collapse(dm, qubit, *outcome, p0);
}

int gq_dm_copy_state(gq_dm* dst, const gq_dm* src) {
    if (!dst || !src) return fail(GQ_EINVAL, "null handle");
    if (dst->nq != src->nq) return fail(GQ_EINVAL, "handles differ in qubit count");
    if (dst == src) return GQ_OK;
    GQ_CUDA(cudaStreamSynchronize(src->e.stream));
    GQ_CUDA(cudaMemcpyAsync(dst->e.state.p, src->e.state.p, src->e.n_amps * src->e.amp_bytes(),
                            cudaMemcpyDeviceToDevice, dst->e.stream));
    GQ_CUDA(cudaStreamSynchronize(dst->e.stream));
    return GQ_OK;
}

int gq_dm_stats(const gq_dm* dm, gq_stats* out) {
    if (!dm || !out) return fail(GQ_EINVAL, "null argument");
    *out = dm->e.get_stats();
    return GQ_OK;
}

}  // extern "C"

// ============================================================================
// Batches of independent circuits (sweep.RunSim-style parameter batches,
// sweep/run.go:27-171, and the QAOA / VQE evaluations of algorithm/*): every
// circuit's forward and reverse programs are concatenated into one device
// program. Wave w runs pass w of every circuit in one launch per tile size
// (a descriptor per state and pass, runs of descriptors with equal CTA
// counts), so no kernel waits on another; lambda,
// energies and gradients are reduced per circuit in fixed order. The launch
// sequence is captured in a CUDA graph and replayed while the circuits'
// structure (not their angles) stays the same.
namespace {

struct BLaunch {
    uint32_t run0, nrun;  // into the run array
    uint32_t count;       // blocks
    int m;
    bool adjoint;
    uint32_t grp0, ngrp;    // gradient groups reduced after an adjoint launch
};

struct BatchPlan {
    Program prog;                  // concatenated passes / phases / ops / pool
    std::vector<int> pass_nslots;  // gradient slots per pass
    std::vector<uint32_t> slot_grad;
    std::vector<uint32_t> pass_slot0;
    std::vector<BDesc> descs;
    std::vector<BRun> runs;
    std::vector<BLaunch> launches;  // forward waves, then reverse waves
    size_t n_forward_launches = 0;
    std::vector<BGradGroup> ggroups;
    std::vector<uint64_t> state_off;
    uint64_t total_amps = 0, total_partials = 0;
    std::vector<DGroup> groups;
    std::vector<DTerm> terms;
    std::vector<BCircuit> circ;
    std::vector<BChunk> chunks;
    std::vector<uint64_t> chunk_seg;
    size_t total_params = 0;
    uint64_t signature = 0;
};

// Structure signature (graph replay): a 64-bit multiply-xorshift hash over
// 8-byte words.
uint64_t fnv(uint64_t h, const void* p, size_t n) {
    const unsigned char* b = (const unsigned char*)p;
    size_t i = 0;
    for (; i + 8 <= n; i += 8) {
        uint64_t w;
        std::memcpy(&w, b + i, 8);
        h = (h ^ w) * 0x9E3779B97F4A7C15ull;
        h ^= h >> 29;
    }
    for (; i < n; ++i) h = (h ^ b[i]) * 1099511628211ull;
    return h;
}

template <class F>
void parallel_for(size_t n, size_t min_parallel, F fn);

// fnv over 1 MiB chunks hashed on the host's threads, combined in order.
uint64_t fnv_par(uint64_t h, const void* p, size_t n) {
    const size_t chunk = 1u << 20, nc = (n + chunk - 1) / chunk;
    if (nc <= 1) return fnv(h, p, n);
    std::vector<uint64_t> part(nc);
    parallel_for(nc, 4, [&](size_t i) {
        part[i] = fnv(1469598103934665603ull ^ i, (const char*)p + i * chunk, std::min(chunk, n - i * chunk));
    });
    return fnv(h, part.data(), nc * sizeof(uint64_t));
}

}  // namespace

struct gq_batch {
    Engine e;
    BatchPlan plan;  // of the segment being planned
    // per segment: captured launch sequence, its structure signature and the
    // buffer generation its pointers belong to
    std::vector<cudaGraphExec_t> graphs;
    std::vector<uint64_t> graph_sig, graph_gen;
    std::vector<int64_t> graph_launches;
    uint64_t buf_gen = 0;  // bumped when a device buffer is reallocated
    bool use_graph = true;
    DevBuf states, lams, partials, energies, grads, tables;
    // two host staging buffers: segment k packs into one while the upload of
    // segment k - 1 may still read the other
    PinnedBuf stage[2];
    cudaEvent_t staged[2] = {nullptr, nullptr};
    bool staged_pending[2] = {false, false};
    PinnedBuf results;  // energies and gradients of all segments (pinned: copies do not block)
    std::chrono::steady_clock::time_point call_t0;  // start of the current gq_batch_run
};

namespace {

// Batched tile pass per precision.
template <class T>
struct BatchTile;
template <>
struct BatchTile<double> {
    static constexpr auto kernel = k_tile_pass_batch<double, 128, 3>;
};
template <>
struct BatchTile<float> {
    // 3 CTAs of 256 threads per SM (80 registers, a few spilled): measured
    // 4.8% faster on 4096 QAOA circuits than 2 CTAs with 128 registers
    static constexpr auto kernel = k_tile_pass_batch<float, 256, 3>;
};

template <class T>
int set_batch_attrs() {
    static std::once_flag once;
    static cudaError_t err = cudaSuccess;
    std::call_once(once, [] {
        const int mt = log2i(TileTable<T>::threads(0)) + RQ;
        err = cudaFuncSetAttribute(BatchTile<T>::kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)(sizeof(cplx<T>) << mt));
        if (err == cudaSuccess)
            err = cudaFuncSetAttribute(k_adjoint_pass_batch<T, kAdjThreads, kAdjBatchMinB<T>>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)adj_smem(sizeof(cplx<T>), log2i(kAdjThreads) + RQ));
    });
    if (err != cudaSuccess) return fail(GQ_ECUDA, std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(err));
    return GQ_OK;
}

// Runs fn(i) for i < n on the host's threads (one thread for small n).
template <class F>
void parallel_for(size_t n, size_t min_parallel, F fn) {
    unsigned nt = std::thread::hardware_concurrency();
    nt = std::max(1u, std::min(nt == 0 ? 1u : nt, 32u));
    if (n < min_parallel) nt = 1;
    std::atomic<size_t> next{0};
    auto worker = [&]() {
        for (size_t i; (i = next.fetch_add(1)) < n;) fn(i);
    };
    std::vector<std::thread> pool;
    for (unsigned k = 1; k < nt; ++k) pool.emplace_back(worker);
    worker();
    for (std::thread& t : pool) t.join();
}

// Builds the concatenated program, launch descriptors and reduction tables.
int build_batch_plan(int prec, const gq_batch_item* items, size_t n, bool grads, const SchedOptions& base_opt,
                     BatchPlan& P) {
    P = BatchPlan();
    std::vector<std::vector<int>> fwd_passes(n), rev_passes(n);
    std::vector<uint64_t> grad_off(n);
    // Each circuit is analysed and scheduled on its own (worker threads);
    // the results are concatenated in order below.
    struct CircPlan {
        Program pf, pr;
        std::vector<DGroup> groups;  // term indices local to the circuit
        std::vector<DTerm> terms;
        int rc = GQ_OK;
        std::string err;
    };
    std::vector<CircPlan> cp(n);
    auto plan_one = [&](size_t c) {
        CircPlan& q = cp[c];
        const gq_batch_item& it = items[c];
        auto bad = [&](int rc, const std::string& why) {
            q.rc = rc;
            q.err = "batch item " + std::to_string(c) + ": " + why;
        };
        if (it.num_qubits < 1 || it.num_qubits > 30) return bad(GQ_EINVAL, "qubits out of range");
        if ((it.n_ops && !it.ops) || (it.n_terms && !it.terms)) return bad(GQ_EINVAL, "null ops or terms");
        const int nphys = std::max(it.num_qubits, RQ);
        std::vector<NGate> fwd, rev;
        std::vector<int> fo, ro;
        std::string err;
        int rc;
        if (grads) {
            rc = adjoint_gates(it.num_qubits, it.ops, it.n_ops, it.n_params, fwd, rev, fo, ro, err);
        } else {
            rc = GQ_OK;
            for (size_t k = 0; k < it.n_ops && rc == GQ_OK; ++k) rc = normalize_op(it.ops[k], it.num_qubits, fwd, err);
        }
        if (rc != GQ_OK) return bad(rc, err);
        // Pauli terms of this circuit: Re(c_t) only (lambda for the gradient
        // and Re <psi|H|psi>), grouped by x mask
        const uint64_t qmask = (1ull << it.num_qubits) - 1;
        std::vector<size_t> order(it.n_terms);
        for (size_t i = 0; i < it.n_terms; ++i) {
            if ((it.terms[i].x_mask | it.terms[i].z_mask) & ~qmask) return bad(GQ_EINVAL, "Pauli term out of range");
            order[i] = i;
        }
        SchedOptions o = base_opt;
        schedule(fwd, nphys, o, q.pf);
        if (grads) {
            o.tile_qubits = std::min(o.tile_qubits, log2i(kAdjThreads) + RQ);
            schedule(rev, nphys, o, q.pr);
        }
        std::stable_sort(order.begin(), order.end(),
                         [&](size_t a, size_t b) { return it.terms[a].x_mask < it.terms[b].x_mask; });
        for (size_t k = 0; k < it.n_terms; ++k) {
            const gq_pauli_term& t = it.terms[order[k]];
            if (q.groups.empty() || q.groups.back().x != t.x_mask)
                q.groups.push_back({t.x_mask, (int32_t)q.terms.size(), (int32_t)q.terms.size()});
            const int ny = __builtin_popcountll(t.x_mask & t.z_mask) & 3;
            double wr = t.coeff_re, wi = 0.0;
            if (ny == 1) wr = 0.0, wi = t.coeff_re;
            if (ny == 2) wr = -t.coeff_re;
            if (ny == 3) wr = 0.0, wi = -t.coeff_re;
            q.terms.push_back({wr, wi, t.z_mask});
            q.groups.back().t1 = (int32_t)q.terms.size();
        }
    };
    parallel_for(n, 64, plan_one);
    // Concatenation: every circuit's section of the arrays is sized first,
    // then filled in parallel (offsets of passes, phases, ops and pool fixed up).
    struct Sec {
        size_t pass, phase, op, pool, slot, group, term;
    };
    std::vector<Sec> sec(2 * n + 1);  // programs in order c0.pf, c0.pr, c1.pf, ...
    {
        Sec at{0, 0, 0, 0, 0, 0, 0};
        for (size_t c = 0; c < n; ++c) {
            const CircPlan& q = cp[c];
            if (q.rc != GQ_OK) return fail(q.rc, q.err);
            const gq_batch_item& it = items[c];
            grad_off[c] = P.total_params;
            P.total_params += it.n_params;
            P.state_off.push_back(P.total_amps);
            P.total_amps += 1ull << std::max(it.num_qubits, RQ);
            for (int k = 0; k < 2; ++k) {
                const Program& pg = k ? q.pr : q.pf;
                sec[2 * c + k] = at;
                at.pass += pg.passes.size();
                at.phase += pg.phases.size();
                at.op += pg.ops.size();
                at.pool += pg.pool.size();
                for (const auto& sp : pg.pass_params) at.slot += sp.size();
                if (k == 0) {
                    at.group += q.groups.size();
                    at.term += q.terms.size();
                }
            }
            const size_t pb = sec[2 * c].pass, rb = sec[2 * c + 1].pass;
            for (size_t i = 0; i < q.pf.passes.size(); ++i) fwd_passes[c].push_back((int)(pb + i));
            for (size_t i = 0; i < q.pr.passes.size(); ++i) rev_passes[c].push_back((int)(rb + i));
            BCircuit bc;
            bc.state = P.state_off[c];
            bc.n_amps = 1ull << it.num_qubits;
            bc.group0 = (int32_t)sec[2 * c].group;
            bc.ngroups = (int32_t)q.groups.size();
            P.circ.push_back(bc);
        }
        sec[2 * n] = at;
        P.prog.passes.resize(at.pass);
        P.prog.phases.resize(at.phase);
        P.prog.ops.resize(at.op);
        P.prog.pool.resize(at.pool);
        P.pass_slot0.resize(at.pass);
        P.pass_nslots.resize(at.pass);
        P.slot_grad.resize(at.slot);
        P.groups.resize(at.group);
        P.terms.resize(at.term);
    }
    parallel_for(2 * n, 64, [&](size_t k) {
        const size_t c = k / 2;
        CircPlan& q = cp[c];
        const Program& src = (k & 1) ? q.pr : q.pf;
        const Sec& o = sec[k];
        size_t slot = o.slot;
        for (size_t i = 0; i < src.passes.size(); ++i) {
            PassDesc pd = src.passes[i];
            pd.phase0 += (int32_t)o.phase;
            P.prog.passes[o.pass + i] = pd;
            P.pass_slot0[o.pass + i] = (uint32_t)slot;
            const size_t ns = i < src.pass_params.size() ? src.pass_params[i].size() : 0;
            P.pass_nslots[o.pass + i] = (int)ns;
            for (size_t j = 0; j < ns; ++j) P.slot_grad[slot++] = (uint32_t)(grad_off[c] + src.pass_params[i][j]);
        }
        for (size_t i = 0; i < src.phases.size(); ++i) {
            PhaseDesc ph = src.phases[i];
            ph.op_begin += (int32_t)o.op;
            ph.op_end += (int32_t)o.op;
            P.prog.phases[o.phase + i] = ph;
        }
        for (size_t i = 0; i < src.ops.size(); ++i) {
            KOp op = src.ops[i];
            op.mat += (uint32_t)o.pool;
            P.prog.ops[o.op + i] = op;
        }
        std::copy(src.pool.begin(), src.pool.end(), P.prog.pool.begin() + o.pool);
        if (!(k & 1)) {
            for (size_t i = 0; i < q.groups.size(); ++i) {
                DGroup g = q.groups[i];
                g.t0 += (int32_t)o.term;
                g.t1 += (int32_t)o.term;
                P.groups[o.group + i] = g;
            }
            std::copy(q.terms.begin(), q.terms.end(), P.terms.begin() + o.term);
        }
        { Program none; std::swap(none, (k & 1) ? q.pr : q.pf); }  // release the circuit's program here
    });
    cp.clear();
    // chunks of the lambda / energy kernel
    const uint32_t chunk_len = 4096;
    P.chunk_seg.push_back(0);
    for (size_t c = 0; c < n; ++c) {
        for (uint64_t b = 0; b < P.circ[c].n_amps; b += chunk_len) P.chunks.push_back({(uint32_t)c, (uint32_t)b});
        P.chunk_seg.push_back(P.chunks.size());
    }
    // waves: pass w of every circuit, one launch per tile size; inside a
    // launch, circuits with the same CTA count form one run
    auto add_waves = [&](const std::vector<std::vector<int>>& passes, bool adjoint) {
        size_t W = 0;
        for (auto& v : passes) W = std::max(W, v.size());
        std::vector<std::vector<size_t>> by_outer(64);
        for (size_t w = 0; w < W; ++w) {
            for (int m = RQ; m <= MAX_TILE; ++m) {
                for (auto& v : by_outer) v.clear();
                for (size_t c = 0; c < n; ++c) {
                    if (w >= passes[c].size()) continue;
                    const PassDesc& pd = P.prog.passes[passes[c][w]];
                    if (pd.m == m) by_outer[pd.n_outer].push_back(c);
                }
                BLaunch L{(uint32_t)P.runs.size(), 0, 0, m, adjoint, (uint32_t)P.ggroups.size(), 0};
                for (int k = 63; k >= 0; --k) {
                    if (by_outer[k].empty()) continue;
                    P.runs.push_back({L.count, (uint32_t)P.descs.size(), (uint32_t)k, 0u});
                    for (size_t c : by_outer[k]) {
                        const int gp = passes[c][w];
                        const uint32_t ns = (uint32_t)P.pass_nslots[gp];
                        P.descs.push_back({P.state_off[c], P.total_partials, (uint32_t)gp, ns});
                        if (adjoint && ns > 0)
                            P.ggroups.push_back({P.total_partials, 1u << k, P.pass_slot0[gp], ns, 0u});
                        P.total_partials += (uint64_t)ns << k;
                        L.count += 1u << k;
                    }
                }
                L.nrun = (uint32_t)P.runs.size() - L.run0;
                L.ngrp = (uint32_t)P.ggroups.size() - L.grp0;
                if (L.count) P.launches.push_back(L);
            }
        }
    };
    add_waves(fwd_passes, false);
    P.n_forward_launches = P.launches.size();
    if (grads) add_waves(rev_passes, true);
    // structure signature: everything but the matrix values
    uint64_t h = 1469598103934665603ull;
    h = fnv_par(h, P.prog.passes.data(), P.prog.passes.size() * sizeof(PassDesc));
    h = fnv_par(h, P.prog.phases.data(), P.prog.phases.size() * sizeof(PhaseDesc));
    h = fnv_par(h, P.prog.ops.data(), P.prog.ops.size() * sizeof(KOp));
    h = fnv_par(h, P.descs.data(), P.descs.size() * sizeof(BDesc));
    h = fnv(h, P.runs.data(), P.runs.size() * sizeof(BRun));
    h = fnv(h, P.groups.data(), P.groups.size() * sizeof(DGroup));
    const size_t ps = P.prog.pool.size(), nt = P.terms.size();
    h = fnv(h, &ps, sizeof(ps));
    h = fnv(h, &nt, sizeof(nt));
    h = fnv(h, &prec, sizeof(prec));
    const int g = grads;
    h = fnv(h, &g, sizeof(g));
    P.signature = h;
    return GQ_OK;
}

template <class T>
// One segment of a batch (b->plan, n circuits): packs its tables into staging
// buffer `slot`, uploads them and enqueues its launches (a captured graph,
// replayed while the segment's structure and buffers are unchanged), then
// the copies of its energies and gradients into res_e / res_g (pinned).
// Nothing here waits for the device, so the host can plan the next segment
// while this one runs.
int batch_segment_t(gq_batch* b, bool grads, size_t n, size_t seg, bool first, double* res_e, double* res_g) {
    Engine& e = b->e;
    BatchPlan& P = b->plan;
    const int slot = (int)(seg & 1);
    // ---- one upload: program, descriptors, runs, reduction tables
    struct Off {
        size_t pass, phase, ops, pool, descs, runs, ggroups, slotg, bcirc, chunks, seg, groups, terms, soff, total;
    } o{};
    size_t at = 0;
    auto put = [&](size_t bytes) {
        const size_t r = at;
        at = align16(at + std::max<size_t>(bytes, 1));
        return r;
    };
    o.pass = put(P.prog.passes.size() * sizeof(PassDesc));
    o.phase = put(P.prog.phases.size() * sizeof(PhaseDesc));
    o.ops = put(P.prog.ops.size() * sizeof(KOp));
    o.pool = put(P.prog.pool.size() * sizeof(cplx<T>));
    o.descs = put(P.descs.size() * sizeof(BDesc));
    o.runs = put(P.runs.size() * sizeof(BRun));
    o.ggroups = put(P.ggroups.size() * sizeof(BGradGroup));
    o.slotg = put(P.slot_grad.size() * sizeof(uint32_t));
    o.bcirc = put(P.circ.size() * sizeof(BCircuit));
    o.chunks = put(P.chunks.size() * sizeof(BChunk));
    o.seg = put(P.chunk_seg.size() * sizeof(uint64_t));
    o.groups = put(P.groups.size() * sizeof(DGroup));
    o.terms = put(P.terms.size() * sizeof(DTerm));
    o.soff = put(P.state_off.size() * sizeof(uint64_t));
    o.total = at;
    if (b->staged_pending[slot]) {
        GQ_CUDA(cudaEventSynchronize(b->staged[slot]));
        b->staged_pending[slot] = false;
    }
    GQ_TRY(b->stage[slot].ensure(o.total));
    char* h = (char*)b->stage[slot].p;
    auto cp = [&](size_t off, const void* src, size_t bytes) {
        const size_t chunk = 4u << 20;
        parallel_for((bytes + chunk - 1) / chunk, 4, [&](size_t i) {
            std::memcpy(h + off + i * chunk, (const char*)src + i * chunk, std::min(chunk, bytes - i * chunk));
        });
    };
    cp(o.pass, P.prog.passes.data(), P.prog.passes.size() * sizeof(PassDesc));
    cp(o.phase, P.prog.phases.data(), P.prog.phases.size() * sizeof(PhaseDesc));
    cp(o.ops, P.prog.ops.data(), P.prog.ops.size() * sizeof(KOp));
    {
        cplx<T>* pool = (cplx<T>*)(h + o.pool);
        const size_t np = P.prog.pool.size(), chunk = 1u << 18;
        parallel_for((np + chunk - 1) / chunk, 4, [&](size_t k) {
            for (size_t i = k * chunk; i < std::min(np, (k + 1) * chunk); ++i)
                pool[i] = {(T)P.prog.pool[i].re, (T)P.prog.pool[i].im};
        });
    }
    cp(o.descs, P.descs.data(), P.descs.size() * sizeof(BDesc));
    cp(o.runs, P.runs.data(), P.runs.size() * sizeof(BRun));
    cp(o.ggroups, P.ggroups.data(), P.ggroups.size() * sizeof(BGradGroup));
    cp(o.slotg, P.slot_grad.data(), P.slot_grad.size() * sizeof(uint32_t));
    cp(o.bcirc, P.circ.data(), P.circ.size() * sizeof(BCircuit));
    cp(o.chunks, P.chunks.data(), P.chunks.size() * sizeof(BChunk));
    cp(o.seg, P.chunk_seg.data(), P.chunk_seg.size() * sizeof(uint64_t));
    cp(o.groups, P.groups.data(), P.groups.size() * sizeof(DGroup));
    cp(o.terms, P.terms.data(), P.terms.size() * sizeof(DTerm));
    cp(o.soff, P.state_off.data(), P.state_off.size() * sizeof(uint64_t));
    const bool resized = o.total > b->tables.cap || P.total_amps * sizeof(cplx<T>) > b->states.cap ||
                         P.total_amps * sizeof(cplx<T>) > b->lams.cap ||
                         std::max<uint64_t>(P.total_partials, P.chunks.size()) * sizeof(double) > b->partials.cap ||
                         (n + 1) * sizeof(double) > b->energies.cap ||
                         std::max<size_t>(1, P.total_params) * sizeof(double) > b->grads.cap;
    if (resized) {
        // buffers grow: the previous segment's launches may still use them
        GQ_CUDA(cudaStreamSynchronize(e.stream));
        ++b->buf_gen;  // captured graphs hold the old pointers
    }
    GQ_TRY(b->states.ensure(P.total_amps * sizeof(cplx<T>)));
    GQ_TRY(b->lams.ensure(P.total_amps * sizeof(cplx<T>)));
    GQ_TRY(b->partials.ensure(std::max<uint64_t>(1, std::max<uint64_t>(P.total_partials, P.chunks.size())) * sizeof(double)));
    GQ_TRY(b->energies.ensure((n + 1) * sizeof(double)));
    GQ_TRY(b->grads.ensure(std::max<size_t>(1, P.total_params) * sizeof(double)));
    GQ_TRY(b->tables.ensure(o.total));
    GQ_CUDA(cudaMemcpyAsync(b->tables.p, b->stage[slot].p, o.total, cudaMemcpyHostToDevice, e.stream));
    GQ_CUDA(cudaEventRecord(b->staged[slot], e.stream));
    b->staged_pending[slot] = true;
    e.stats.h2d_bytes += (int64_t)o.total;
    char* d = (char*)b->tables.p;
    cplx<T>* states = (cplx<T>*)b->states.p;
    cplx<T>* lams = (cplx<T>*)b->lams.p;
    double* partial = (double*)b->partials.p;

    if (b->graphs.size() <= seg) {
        b->graphs.resize(seg + 1, nullptr);
        b->graph_sig.resize(seg + 1, 0);
        b->graph_gen.resize(seg + 1, 0);
        b->graph_launches.resize(seg + 1, 0);
    }
    const bool replay = b->use_graph && b->graphs[seg] && b->graph_sig[seg] == P.signature &&
                        b->graph_gen[seg] == b->buf_gen;
    int64_t launches = 0;
    auto record = [&]() -> int {
        GQ_CUDA(cudaMemsetAsync(states, 0, P.total_amps * sizeof(cplx<T>), e.stream));
        k_batch_basis<T><<<(unsigned)((n + 127) / 128), 128, 0, e.stream>>>(states, (const uint64_t*)(d + o.soff), n);
        ++launches;
        for (size_t li = 0; li < P.launches.size(); ++li) {
            const BLaunch& L = P.launches[li];
            const unsigned threads = 1u << (L.m - RQ);
            if (!L.adjoint) {
                BatchTile<T>::kernel<<<L.count, threads, sizeof(cplx<T>) << L.m, e.stream>>>(
                    states, (const BRun*)(d + o.runs) + L.run0, (int)L.nrun, (const BDesc*)(d + o.descs),
                    (const PassDesc*)(d + o.pass), (const PhaseDesc*)(d + o.phase), (const KOp*)(d + o.ops),
                    (const cplx<T>*)(d + o.pool));
                ++launches;
            } else {
                k_adjoint_pass_batch<T, kAdjThreads, kAdjBatchMinB<T>><<<L.count, threads, adj_smem(sizeof(cplx<T>), L.m),
                                                                         e.stream>>>(
                    states, lams, (const BRun*)(d + o.runs) + L.run0, (int)L.nrun, (const BDesc*)(d + o.descs),
                    (const PassDesc*)(d + o.pass), (const PhaseDesc*)(d + o.phase), (const KOp*)(d + o.ops),
                    (const cplx<T>*)(d + o.pool), partial);
                ++launches;
                if (L.ngrp) {
                    k_grad_reduce_batch<<<L.ngrp, 256, 0, e.stream>>>(partial,
                                                                      (const BGradGroup*)(d + o.ggroups) + L.grp0,
                                                                      (const uint32_t*)(d + o.slotg),
                                                                      (double*)b->grads.p);
                    ++launches;
                }
            }
            if (li + 1 == P.n_forward_launches) {
                // after the forward waves: lambda and the energies
                k_apply_terms_batch<T><<<(unsigned)P.chunks.size(), 256, 0, e.stream>>>(
                    states, lams, (const BCircuit*)(d + o.bcirc), (const BChunk*)(d + o.chunks), 4096,
                    (const DGroup*)(d + o.groups), (const DTerm*)(d + o.terms), partial);
                k_segment_reduce<<<(unsigned)n, 256, 0, e.stream>>>(partial, (const uint64_t*)(d + o.seg),
                                                                    (double*)b->energies.p);
                GQ_CUDA(cudaMemsetAsync(b->grads.p, 0, std::max<size_t>(1, P.total_params) * sizeof(double), e.stream));
                launches += 2;
            }
        }
        if (P.n_forward_launches == 0) {
            k_apply_terms_batch<T><<<(unsigned)P.chunks.size(), 256, 0, e.stream>>>(
                states, lams, (const BCircuit*)(d + o.bcirc), (const BChunk*)(d + o.chunks), 4096,
                (const DGroup*)(d + o.groups), (const DTerm*)(d + o.terms), partial);
            k_segment_reduce<<<(unsigned)n, 256, 0, e.stream>>>(partial, (const uint64_t*)(d + o.seg),
                                                                (double*)b->energies.p);
            GQ_CUDA(cudaMemsetAsync(b->grads.p, 0, std::max<size_t>(1, P.total_params) * sizeof(double), e.stream));
            launches += 2;
        }
        GQ_CUDA(cudaGetLastError());
        return GQ_OK;
    };
    // the batch's device work alone (pass_ms): from the first launch on
    auto mark0 = [&]() -> int {
        if (!first) return GQ_OK;
        e.stats.host_ms =
            std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - b->call_t0).count();
        if (e.timing) GQ_CUDA(cudaEventRecord(e.ev_pass0, e.stream));
        return GQ_OK;
    };
    if (replay) {
        GQ_TRY(mark0());
        GQ_CUDA(cudaGraphLaunch(b->graphs[seg], e.stream));
        launches = b->graph_launches[seg];  // the recorded sequence
    } else if (b->use_graph) {
        if (b->graphs[seg]) {
            cudaGraphExecDestroy(b->graphs[seg]);
            b->graphs[seg] = nullptr;
        }
        cudaGraph_t g = nullptr;
        GQ_CUDA(cudaStreamBeginCapture(e.stream, cudaStreamCaptureModeThreadLocal));
        int rc = record();
        cudaError_t ce = cudaStreamEndCapture(e.stream, &g);
        if (rc != GQ_OK) {
            if (g) cudaGraphDestroy(g);
            return rc;
        }
        if (ce != cudaSuccess) return fail(GQ_ECUDA, std::string("graph capture: ") + cudaGetErrorString(ce));
        ce = cudaGraphInstantiate(&b->graphs[seg], g, 0);
        cudaGraphDestroy(g);
        if (ce != cudaSuccess) {
            b->graphs[seg] = nullptr;
            return fail(GQ_ECUDA, std::string("graph instantiate: ") + cudaGetErrorString(ce));
        }
        b->graph_sig[seg] = P.signature;
        b->graph_gen[seg] = b->buf_gen;
        b->graph_launches[seg] = launches;
        GQ_TRY(mark0());
        GQ_CUDA(cudaGraphLaunch(b->graphs[seg], e.stream));
    } else {
        GQ_TRY(mark0());
        GQ_TRY(record());
    }
    e.stats.kernel_launches += launches;
    GQ_CUDA(cudaMemcpyAsync(res_e, b->energies.p, n * sizeof(double), cudaMemcpyDeviceToHost, e.stream));
    if (grads && P.total_params)
        GQ_CUDA(cudaMemcpyAsync(res_g, b->grads.p, P.total_params * sizeof(double), cudaMemcpyDeviceToHost, e.stream));
    e.stats.d2h_bytes += (int64_t)(n * sizeof(double) + (grads ? P.total_params * sizeof(double) : 0));
    return GQ_OK;
}

}  // namespace

extern "C" {

int gq_batch_create(int precision, gq_batch** out) {
    if (!out) return fail(GQ_EINVAL, "null output handle");
    *out = nullptr;
    if (!valid_prec(precision)) return fail(GQ_EINVAL, "unknown precision");
    gq_batch* b = new gq_batch();
    int rc = b->e.init(RQ, precision);
    if (rc == GQ_OK) rc = precision == GQ_C64 ? set_batch_attrs<float>() : set_batch_attrs<double>();
    if (rc != GQ_OK) {
        b->e.destroy();
        delete b;
        return rc;
    }
    b->e.opt.tile_qubits = precision == GQ_C64 ? 12 : 11;
    for (int k = 0; k < 2 && rc == GQ_OK; ++k)
        if (cudaEventCreateWithFlags(&b->staged[k], cudaEventDisableTiming) != cudaSuccess) {
            (void)cudaGetLastError();
            rc = fail(GQ_ECUDA, "cudaEventCreate failed");
        }
    if (rc != GQ_OK) {
        for (cudaEvent_t ev : b->staged)
            if (ev) cudaEventDestroy(ev);
        b->e.destroy();
        delete b;
        return rc;
    }
    *out = b;
    return GQ_OK;
}

int gq_batch_destroy(gq_batch* b) {
    if (!b) return GQ_OK;
    if (b->e.stream) cudaStreamSynchronize(b->e.stream);
    for (cudaGraphExec_t g : b->graphs)
        if (g) cudaGraphExecDestroy(g);
    for (cudaEvent_t ev : b->staged)
        if (ev) cudaEventDestroy(ev);
    b->stage[0].release();
    b->stage[1].release();
    b->results.release();
    b->states.release();
    b->lams.release();
    b->partials.release();
    b->energies.release();
    b->grads.release();
    b->tables.release();
    b->e.destroy();
    delete b;
    return GQ_OK;
}

int gq_batch_run(gq_batch* b, const gq_batch_item* items, size_t n_items, int want_gradients, double* energies_out,
                 double* grads_out) {
    if (!b) return fail(GQ_EINVAL, "null handle");
    if (n_items == 0) return GQ_OK;
    if (!items) return fail(GQ_EINVAL, "null items");
    Engine& e = b->e;
    e.clear_stats();
    b->call_t0 = std::chrono::steady_clock::now();
    GQ_TRY(e.time_begin());
    const bool grads = want_gradients != 0;
    // Segments of about equal work (state size x ops), planned one after
    // another on the host while the device runs the previous one.
    const size_t nseg = std::max<size_t>(1, std::min<size_t>(8, n_items / 512));
    std::vector<double> work(n_items);
    double wsum = 0.0;
    size_t total_params = 0;
    for (size_t c = 0; c < n_items; ++c) {
        const int nq = std::max(1, std::min(30, items[c].num_qubits));
        work[c] = std::ldexp((double)(items[c].n_ops + 1), std::max(nq, RQ));
        wsum += work[c];
        total_params += items[c].n_params;
    }
    std::vector<size_t> cut{0};
    {
        double acc = 0.0;
        for (size_t c = 0; c < n_items; ++c) {
            acc += work[c];
            if (cut.size() < nseg && acc >= wsum * (double)cut.size() / (double)nseg && c + 1 < n_items)
                cut.push_back(c + 1);
        }
        cut.push_back(n_items);
    }
    GQ_TRY(b->results.ensure((n_items + std::max<size_t>(1, total_params)) * sizeof(double)));
    double* res_e = (double*)b->results.p;
    double* res_g = res_e + n_items;
    size_t poff = 0;
    int64_t passes = 0, phases = 0, state_bytes = 0;
    for (size_t sg = 0; sg + 1 < cut.size(); ++sg) {
        const size_t c0 = cut[sg], cnt = cut[sg + 1] - c0;
        GQ_TRY(build_batch_plan(e.prec, items + c0, cnt, grads, e.opt, b->plan));
        const int rc = e.prec == GQ_C64 ? batch_segment_t<float>(b, grads, cnt, sg, sg == 0, res_e + c0, res_g + poff)
                                        : batch_segment_t<double>(b, grads, cnt, sg, sg == 0, res_e + c0, res_g + poff);
        if (rc != GQ_OK) {
            cudaStreamSynchronize(e.stream);
            return rc;
        }
        poff += b->plan.total_params;
        passes += (int64_t)b->plan.prog.passes.size();
        phases += (int64_t)b->plan.prog.phases.size();
        state_bytes = std::max<int64_t>(state_bytes, (int64_t)(b->plan.total_amps * e.amp_bytes()));
    }
    if (e.timing) {
        GQ_CUDA(cudaEventRecord(e.ev_pass1, e.stream));
        e.pass_timed = true;
    }
    GQ_CUDA(cudaStreamSynchronize(e.stream));
    if (energies_out) std::memcpy(energies_out, res_e, n_items * sizeof(double));
    if (grads && grads_out && total_params) std::memcpy(grads_out, res_g, total_params * sizeof(double));
    e.stats.passes = passes;
    e.stats.phases = phases;
    e.stats.state_bytes = state_bytes;
    return e.time_end();
}

int gq_batch_set_option(gq_batch* b, int key, int64_t value) {
    if (!b) return fail(GQ_EINVAL, "null handle");
    switch (key) {
        case GQ_OPT_TIMING: b->e.timing = value != 0; return GQ_OK;
        case GQ_OPT_PASS_BUDGET: b->e.opt.budget = value == 0 ? kDefaultBudget : (int)value; return GQ_OK;
        case GQ_OPT_USE_GRAPH: b->use_graph = value != 0; return GQ_OK;
        default: return fail(GQ_EINVAL, "unknown option");
    }
}

int gq_batch_stats(const gq_batch* b, gq_stats* out) {
    if (!b || !out) return fail(GQ_EINVAL, "null argument");
    *out = b->e.get_stats();
    return GQ_OK;
}

}  // extern "C"

// ---- sweeps ------------------------------------------------------------------
namespace {

// sweep.RunSim / RunDensitySim (sweep/run.go:27-171): a pool of workers
// takes the points in order; each worker owns one handle (its own device
// state and stream), so points overlap on the device while every point is a
// fresh Evolve followed by sampling with the histogram built on the device.
// Workers: at most the host's threads, 8, the point count, and as many
// states as the free device memory holds next to 1 GiB of headroom.
int sweep_impl(bool density, int nq, int prec, const double* p01, const double* p10, const gq_sweep_point* pts,
               size_t n_pts, size_t shots, uint64_t* outcomes_out, uint64_t* counts_out, size_t* n_distinct_out,
               int32_t* status_out) {
    if (n_pts && (!pts || !n_distinct_out || !status_out)) return fail(GQ_EINVAL, "null argument");
    if (shots && n_pts && (!outcomes_out || !counts_out)) return fail(GQ_EINVAL, "null argument");
    if (density ? (nq < 1 || nq > 15) : (nq < 1 || nq > 34)) return fail(GQ_EINVAL, "num_qubits out of range");
    if (!density && prec != GQ_C128 && prec != GQ_C64) return fail(GQ_EINVAL, "unknown precision");
    for (size_t i = 0; i < n_pts; ++i)
        if ((pts[i].n_ops && !pts[i].ops) || (shots && !pts[i].uniforms)) return fail(GQ_EINVAL, "null point data");
    if (n_pts == 0) return GQ_OK;
    int dev = 0;
    GQ_TRY(check_device(&dev));
    const uint64_t outcomes = 1ull << nq;
    const size_t stride = (size_t)std::max<uint64_t>(1, std::min<uint64_t>(shots, outcomes));
    const uint64_t state_bytes =
        density ? (1ull << (2 * nq)) * 16 : std::max<uint64_t>(16, outcomes) * (prec == GQ_C64 ? 8 : 16);
    size_t mem_free = 0, mem_total = 0;
    GQ_CUDA(cudaMemGetInfo(&mem_free, &mem_total));
    const uint64_t headroom = 1ull << 30;
    const uint64_t by_mem = mem_free > headroom ? (mem_free - headroom) / (2 * state_bytes) : 0;
    unsigned hw = std::thread::hardware_concurrency();
    const size_t nworkers = std::max<size_t>(
        1, std::min<size_t>({n_pts, (size_t)8, (size_t)std::max(1u, hw), (size_t)std::max<uint64_t>(1, by_mem)}));
    std::atomic<size_t> next{0};
    std::mutex err_mu;
    std::string first_err;
    size_t first_bad = n_pts;
    auto worker = [&]() {
        cudaSetDevice(dev);
        gq_sv* sv = nullptr;
        gq_dm* dm = nullptr;
        int rc_create = density ? gq_dm_create(nq, &dm) : gq_sv_create(nq, prec, &sv);
        for (size_t i; (i = next.fetch_add(1)) < n_pts;) {
            int rc = rc_create;
            if (rc == GQ_OK) {
                uint64_t* oc = shots ? outcomes_out + i * stride : nullptr;
                uint64_t* ct = shots ? counts_out + i * stride : nullptr;
                if (density) {
                    rc = gq_dm_evolve(dm, pts[i].ops, pts[i].n_ops);
                    if (rc == GQ_OK)
                        rc = gq_dm_sample_counts(dm, p01, p10, pts[i].uniforms, shots, oc, ct, &n_distinct_out[i]);
                } else {
                    rc = gq_sv_run_counts(sv, pts[i].ops, pts[i].n_ops, pts[i].uniforms, shots, oc, ct,
                                          &n_distinct_out[i]);
                }
            }
            status_out[i] = rc;
            if (rc != GQ_OK) {
                n_distinct_out[i] = 0;
                std::lock_guard<std::mutex> lk(err_mu);
                if (i < first_bad) {
                    first_bad = i;
                    first_err = "point " + std::to_string(i) + ": " + g_err;
                }
            }
        }
        if (sv) gq_sv_destroy(sv);
        if (dm) gq_dm_destroy(dm);
    };
    std::vector<std::thread> pool;
    for (size_t k = 1; k < nworkers; ++k) pool.emplace_back(worker);
    worker();
    for (std::thread& t : pool) t.join();
    if (first_bad < n_pts) g_err = first_err;  // the points' own statuses are in status_out
    return GQ_OK;
}

}  // namespace

extern "C" {

int gq_sweep_run(int num_qubits, int precision, const gq_sweep_point* points, size_t n_points, size_t shots,
                 uint64_t* outcomes_out, uint64_t* counts_out, size_t* n_distinct_out, int32_t* status_out) {
    return sweep_impl(false, num_qubits, precision, nullptr, nullptr, points, n_points, shots, outcomes_out,
                      counts_out, n_distinct_out, status_out);
}

int gq_sweep_run_density(int num_qubits, const double* p01, const double* p10, const gq_sweep_point* points,
                         size_t n_points, size_t shots, uint64_t* outcomes_out, uint64_t* counts_out,
                         size_t* n_distinct_out, int32_t* status_out) {
    return sweep_impl(true, num_qubits, GQ_C128, p01, p10, points, n_points, shots, outcomes_out, counts_out,
                      n_distinct_out, status_out);
}

}  // extern "C"

// ---- circuit equivalence (transpile/verify/verify.go) ------------------------
namespace {

// Applies `ops` (qubits < n) to the handle's state without resetting it.
int apply_on_low(gq_sv* sv, int n, const gq_op* ops, size_t n_ops) {
    if (n_ops && !ops) return fail(GQ_EINVAL, "null ops");
    std::vector<NGate> gates;
    std::string err;
    for (size_t i = 0; i < n_ops; ++i) {
        if (ops[i].kind == GQ_OP_CHANNEL) return fail(GQ_EINVAL, "op " + std::to_string(i) + ": channel in a circuit");
        int rc = normalize_op(ops[i], n, gates, err);
        if (rc != GQ_OK) return fail(rc, "op " + std::to_string(i) + ": " + err);
    }
    return sv->e.run_gates(gates);
}

// sv (2n qubits) <- every column of the unitary of `ops`: entry (col << n) | row.
int unitary_into(gq_sv* sv, int n, const gq_op* ops, size_t n_ops) {
    Engine& e = sv->e;
    GQ_CUDA(cudaMemsetAsync(e.state.p, 0, e.n_amps * e.amp_bytes(), e.stream));
    k_unit_columns<<<(unsigned)(((1ull << n) + 255) / 256), 256, 0, e.stream>>>((cplx<double>*)e.state.p, n);
    GQ_CUDA(cudaGetLastError());
    return apply_on_low(sv, n, ops, n_ops);
}

// First index i < len with |state[i]| > tol, or len when there is none.
int first_above(Engine& e, uint64_t len, double tol, uint64_t* out) {
    GQ_TRY(e.scratch.ensure(64));
    GQ_TRY(e.hostio.ensure(64));
    unsigned long long* d = (unsigned long long*)e.scratch.p;
    GQ_CUDA(cudaMemsetAsync(d, 0xff, 8, e.stream));
    const unsigned g = (unsigned)std::min<uint64_t>((len + 255) / 256, (uint64_t)e.reduce_grid());
    k_first_above<<<g, 256, 0, e.stream>>>((const cplx<double>*)e.state.p, len, tol, d);
    GQ_CUDA(cudaGetLastError());
    GQ_CUDA(cudaMemcpyAsync(e.hostio.p, d, 8, cudaMemcpyDeviceToHost, e.stream));
    GQ_CUDA(cudaStreamSynchronize(e.stream));
    const unsigned long long v = *(const unsigned long long*)e.hostio.p;
    *out = v == ~0ull ? len : (uint64_t)v;
    return GQ_OK;
}

int amplitude_at(Engine& e, uint64_t i, Z* out) {
    GQ_TRY(e.hostio.ensure(64));
    GQ_CUDA(cudaMemcpyAsync(e.hostio.p, (const char*)e.state.p + 16 * i, 16, cudaMemcpyDeviceToHost, e.stream));
    GQ_CUDA(cudaStreamSynchronize(e.stream));
    *out = *(const Z*)e.hostio.p;
    return GQ_OK;
}

// n / m by Smith's algorithm (R. L. Smith, Algorithm 116: Complex division,
// CACM 5(8), 1962), the division Go's complex128 arithmetic uses.
Z smith_div(Z n, Z m) {
    if (std::fabs(m.re) >= std::fabs(m.im)) {
        const double r = m.im / m.re, den = m.re + r * m.im;
        return Z{(n.re + n.im * r) / den, (n.im - n.re * r) / den};
    }
    const double r = m.re / m.im, den = m.im + r * m.re;
    return Z{(n.re * r + n.im) / den, (n.im * r - n.re) / den};
}

// Whether some |a[i] - phase * b[i]| > tol for i < len (a, b: the handles' states).
int phase_mismatch(Engine& ea, Engine& eb, uint64_t len, Z phase, double tol, bool* bad) {
    GQ_CUDA(cudaStreamSynchronize(eb.stream));
    GQ_TRY(ea.scratch.ensure(64));
    GQ_TRY(ea.hostio.ensure(64));
    int* d = (int*)ea.scratch.p;
    GQ_CUDA(cudaMemsetAsync(d, 0, 4, ea.stream));
    const unsigned g = (unsigned)std::min<uint64_t>((len + 255) / 256, (uint64_t)ea.reduce_grid());
    k_phase_mismatch<<<g, 256, 0, ea.stream>>>((const cplx<double>*)ea.state.p, (const cplx<double>*)eb.state.p,
                                                len, phase.re, phase.im, tol, d);
    GQ_CUDA(cudaGetLastError());
    GQ_CUDA(cudaMemcpyAsync(ea.hostio.p, d, 4, cudaMemcpyDeviceToHost, ea.stream));
    GQ_CUDA(cudaStreamSynchronize(ea.stream));
    *bad = *(const int*)ea.hostio.p != 0;
    return GQ_OK;
}

struct SvPair {
    gq_sv* a = nullptr;
    gq_sv* b = nullptr;
    ~SvPair() {
        gq_sv_destroy(a);
        gq_sv_destroy(b);
    }
};

int check_pair_args(int n, int max_n, const gq_op* a, size_t na, const gq_op* b, size_t nb, double tol, int* out) {
    if (!out) return fail(GQ_EINVAL, "null output");
    if ((na && !a) || (nb && !b)) return fail(GQ_EINVAL, "null ops");
    if (n < 1 || n > max_n)
        return fail(GQ_EINVAL, "verify: circuit too large for equivalence check: " + std::to_string(n) + " qubits");
    if (!(tol >= 0.0)) return fail(GQ_EINVAL, "verify: negative tolerance");
    return GQ_OK;
}

}  // namespace

extern "C" {

int gq_unitary(int num_qubits, const gq_op* ops, size_t n_ops, double* host_out, size_t bytes) {
    if (!host_out) return fail(GQ_EINVAL, "null output");
    if (num_qubits < 1 || num_qubits > 16) return fail(GQ_EINVAL, "num_qubits out of range [1, 16]");
    const uint64_t len = 1ull << (2 * num_qubits);
    if (bytes < len * 16) return fail(GQ_EINVAL, "output buffer too small");
    gq_sv* sv = nullptr;
    GQ_TRY(gq_sv_create(2 * num_qubits, GQ_C128, &sv));
    int rc = unitary_into(sv, num_qubits, ops, n_ops);
    if (rc == GQ_OK) {
        cudaError_t e = cudaMemcpyAsync(host_out, sv->e.state.p, len * 16, cudaMemcpyDeviceToHost, sv->e.stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(sv->e.stream);
        if (e != cudaSuccess) rc = fail(GQ_ECUDA, std::string("unitary copy: ") + cudaGetErrorString(e));
    }
    gq_sv_destroy(sv);
    return rc;
}

int gq_equivalent(int num_qubits, const gq_op* a, size_t na, const gq_op* b, size_t nb, double tol, int* equal_out) {
    GQ_TRY(check_pair_args(num_qubits, 15, a, na, b, nb, tol, equal_out));
    const int n = num_qubits;
    SvPair p;
    GQ_TRY(gq_sv_create(2 * n, GQ_C128, &p.a));
    GQ_TRY(gq_sv_create(2 * n, GQ_C128, &p.b));
    GQ_TRY(unitary_into(p.a, n, a, na));
    GQ_TRY(unitary_into(p.b, n, b, nb));
    // global phase from the first entry of B's column 0 above tol (unitariesClose)
    const uint64_t dim = 1ull << n;
    uint64_t ib = 0;
    GQ_TRY(first_above(p.b->e, dim, tol, &ib));
    if (ib == dim) {
        *equal_out = 1;
        return GQ_OK;
    }
    Z va, vb;
    GQ_CUDA(cudaStreamSynchronize(p.a->e.stream));
    GQ_TRY(amplitude_at(p.a->e, ib, &va));
    GQ_TRY(amplitude_at(p.b->e, ib, &vb));
    if (std::hypot(va.re, va.im) < tol) {
        *equal_out = 0;
        return GQ_OK;
    }
    bool bad = false;
    GQ_TRY(phase_mismatch(p.a->e, p.b->e, dim * dim, smith_div(va, vb), tol, &bad));
    *equal_out = bad ? 0 : 1;
    return GQ_OK;
}

int gq_equivalent_on_zero(int num_qubits, const gq_op* a, size_t na, const gq_op* b, size_t nb, double tol,
                          int* equal_out) {
    GQ_TRY(check_pair_args(num_qubits, 30, a, na, b, nb, tol, equal_out));
    const int n = num_qubits;
    SvPair p;
    GQ_TRY(gq_sv_create(n, GQ_C128, &p.a));
    GQ_TRY(gq_sv_create(n, GQ_C128, &p.b));
    GQ_TRY(gq_sv_reset(p.a));
    GQ_TRY(apply_on_low(p.a, n, a, na));
    GQ_TRY(gq_sv_reset(p.b));
    GQ_TRY(apply_on_low(p.b, n, b, nb));
    // stateVectorsClose: the first index where either state exceeds tol
    // decides; B's entry there gives the global phase, of modulus 1 +- tol
    const uint64_t len = 1ull << n;
    uint64_t ia = 0, ib = 0;
    GQ_TRY(first_above(p.a->e, len, tol, &ia));
    GQ_TRY(first_above(p.b->e, len, tol, &ib));
    if (ib == len || ia < ib) {
        *equal_out = (ib == len && ia == len) ? 1 : 0;
        return GQ_OK;
    }
    Z va, vb;
    GQ_TRY(amplitude_at(p.a->e, ib, &va));
    GQ_TRY(amplitude_at(p.b->e, ib, &vb));
    if (std::hypot(va.re, va.im) < tol) {
        *equal_out = 0;
        return GQ_OK;
    }
    const Z phase = smith_div(va, vb);
    if (std::fabs(std::hypot(phase.re, phase.im) - 1.0) > tol) {
        *equal_out = 0;
        return GQ_OK;
    }
    bool bad = false;
    GQ_TRY(phase_mismatch(p.a->e, p.b->e, len, phase, tol, &bad));
    *equal_out = bad ? 0 : 1;
    return GQ_OK;
}

}  // extern "C"

// ---- parameterized templates and the Adam loop ---------------------------------
extern "C" {

int gq_sv_adjoint_template(gq_sv* sv, const gq_op* ops, size_t n_ops, const gq_param_gate* pgates, size_t n_pgates,
                           const double* theta, size_t n_params, const gq_pauli_term* terms, size_t n_terms,
                           double* grad_out, double* energy_out) {
    if (!sv) return fail(GQ_EINVAL, "null handle");
    if ((n_ops && !ops) || (n_pgates && !pgates) || (n_params && !theta)) return fail(GQ_EINVAL, "null argument");
    BoundTemplate bt;
    std::string err;
    const int rc = bind_template(ops, n_ops, pgates, n_pgates, theta, n_params, bt, err);
    if (rc != GQ_OK) return fail(rc, err);
    return gq_sv_adjoint_gradient(sv, bt.ops.data(), bt.ops.size(), terms, n_terms, n_params, grad_out, energy_out);
}

int gq_sv_minimize_adam(gq_sv* sv, const gq_op* ops, size_t n_ops, const gq_param_gate* pgates, size_t n_pgates,
                        const gq_pauli_term* terms, size_t n_terms, size_t n_params, double* x,
                        const gq_adam_options* opts, gq_optim_result* result, double* history_out,
                        size_t history_cap) {
    if (!sv || !result) return fail(GQ_EINVAL, "null argument");
    if (n_params == 0) return fail(GQ_EINVAL, "adam: x0 must be non-empty");
    if (!x) return fail(GQ_EINVAL, "null x");
    const gq_adam_options o = opts ? *opts : gq_adam_options{};
    const double lr = o.lr > 0 ? o.lr : 0.001, b1 = o.beta1 > 0 ? o.beta1 : 0.9;
    const double b2 = o.beta2 > 0 ? o.beta2 : 0.999, eps = o.epsilon > 0 ? o.epsilon : 1e-8;
    const int max_iter = o.max_iter > 0 ? o.max_iter : 1000;
    const double fun_tol = o.fun_tol > 0 ? o.fun_tol : 1e-8, grad_tol = o.grad_tol > 0 ? o.grad_tol : 0.0;
    const size_t n = n_params;
    std::vector<double> m(n, 0.0), v(n, 0.0), g(n);
    size_t nh = 0;
    auto record = [&](double f) {
        if (history_out && nh < history_cap) history_out[nh] = f;
        ++nh;
    };
    // (energy, gradient) at x: goqu's f(x) and, for the next iteration, grad(x)
    double fx = 0.0;
    GQ_TRY(gq_sv_adjoint_template(sv, ops, n_ops, pgates, n_pgates, x, n, terms, n_terms, g.data(), &fx));
    record(fx);
    int f_evals = 1, g_evals = 0, iter = 0;
    bool converged = false;
    double prev = fx;
    for (iter = 0; iter < max_iter; ++iter) {
        ++g_evals;  // g holds grad(x) at the current x
        if (grad_tol > 0) {
            double s = 0.0;
            for (double gj : g) s += gj * gj;
            if (std::sqrt(s) < grad_tol) {
                converged = true;
                break;
            }
        }
        const double t = (double)(iter + 1);
        for (size_t j = 0; j < n; ++j) {
            m[j] = b1 * m[j] + (1 - b1) * g[j];
            v[j] = b2 * v[j] + (1 - b2) * g[j] * g[j];
            const double mh = m[j] / (1 - std::pow(b1, t));
            const double vh = v[j] / (1 - std::pow(b2, t));
            x[j] -= lr * mh / (std::sqrt(vh) + eps);
        }
        GQ_TRY(gq_sv_adjoint_template(sv, ops, n_ops, pgates, n_pgates, x, n, terms, n_terms, g.data(), &fx));
        ++f_evals;
        record(fx);
        if (std::fabs(fx - prev) < fun_tol) {
            converged = true;
            ++iter;
            break;
        }
        prev = fx;
    }
    result->fun = fx;
    result->iterations = iter;
    result->func_evals = f_evals;
    result->grad_evals = g_evals;
    result->converged = converged ? 1 : 0;
    return GQ_OK;
}

}  // extern "C"

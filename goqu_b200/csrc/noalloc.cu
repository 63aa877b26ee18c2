// Pauli-sum expectation that allocates nothing (gq_expect_pauli_sum_noalloc).
//
// Who needs it: callers that own their device memory and cannot let a
// library call cudaMalloc / cudaFree, for instance an application whose
// allocator has reserved the GPU's memory for its own pool (a cudaMalloc
// would fail or fragment it), or a latency-critical loop in which the device
// synchronisation that cudaFree may imply is not acceptable. They pass a
// device state they allocated themselves; this entry point works entirely in
// a fixed scratch array compiled into the library.
//
// The scratch is a file-scope __device__ array of kScratchBytes (256 KiB):
// every GPU that loads the library holds it until the process exits. It bounds
// the Pauli sum to GQ_NOALLOC_MAX_TERMS terms. Host code cannot use the
// symbol `g_scratch` as a device address, so the address is looked up with
// cudaGetSymbolAddress once per device, on the first call made with that
// device current, and again only when the device's context has changed (after
// a cudaDeviceReset, or under another driver-API context). All calls share the
// array and it keeps the last call's contents: two calls that overlap on the
// GPU (different streams or threads) race on it.
//
// The call is synchronous: it copies the term tables from host memory and
// waits for its result on `stream`, so it cannot be recorded into a CUDA graph
// (a stream that is capturing is refused with GQ_EINVAL). The state must be
// device (or managed) memory of the current device.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/gqb200.h"
#include "tile_core.cuh"

using gq::cplx;

namespace gq {
void set_last_error(const std::string& msg);  // engine.cu
}

namespace {

// Pauli terms grouped by x mask; w = coeff * i^(number of Y).
struct NTerm {
    double wre, wim;
    uint64_t z;
};
struct NGroup {
    uint64_t x;
    int32_t t0, t1;
};

__device__ __forceinline__ double nwarp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// sum_t w_t sum_i (-1)^popcount(i & z_t) conj(psi[i ^ x_t]) psi[i], per block
// (the formula of pauli.Expect, sim/pauli/expect_sv.go:21-47), into the
// scratch's partial sums.
template <class T>
__global__ void k_expect_noalloc(const cplx<T>* __restrict__ st, uint64_t n, const NGroup* __restrict__ groups,
                                 int ngroups, const NTerm* __restrict__ terms, double2* __restrict__ partial) {
    double are = 0.0, aim = 0.0;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const cplx<T> ai = st[i];
        const double xr = (double)ai.x, xi = (double)ai.y;
        for (int g = 0; g < ngroups; ++g) {
            const NGroup gr = groups[g];
            const cplx<T> aj = st[i ^ gr.x];
            const double yr = (double)aj.x, yi = (double)aj.y;
            const double pr = yr * xr + yi * xi, pi = yr * xi - yi * xr;
            double fr = 0.0, fi = 0.0;
            for (int k = gr.t0; k < gr.t1; ++k) {
                const NTerm tm = terms[k];
                const double sg = (__popcll(i & tm.z) & 1) ? -1.0 : 1.0;
                fr += sg * tm.wre;
                fi += sg * tm.wim;
            }
            are += fr * pr - fi * pi;
            aim += fr * pi + fi * pr;
        }
    }
    are = nwarp_sum(are);
    aim = nwarp_sum(aim);
    __shared__ double sre[32], sim[32];
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) {
        sre[w] = are;
        sim[w] = aim;
    }
    __syncthreads();
    if (w == 0) {
        const int nw = blockDim.x >> 5;
        are = l < nw ? sre[l] : 0.0;
        aim = l < nw ? sim[l] : 0.0;
        are = nwarp_sum(are);
        aim = nwarp_sum(aim);
        if (l == 0) partial[blockIdx.x] = make_double2(are, aim);
    }
}

// Sum of the per-block partials (one block; fixed order).
__global__ void k_reduce_noalloc(const double2* __restrict__ partial, int n, double2* __restrict__ out) {
    double re = 0.0, im = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        re += partial[i].x;
        im += partial[i].y;
    }
    re = nwarp_sum(re);
    im = nwarp_sum(im);
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
        re = nwarp_sum(re);
        im = nwarp_sum(im);
        if (l == 0) *out = make_double2(re, im);
    }
}

constexpr int kReduceBlocks = 148 * 4;
constexpr size_t kGroupsBytes = sizeof(NGroup) * GQ_NOALLOC_MAX_TERMS;
constexpr size_t kTermsBytes = sizeof(NTerm) * GQ_NOALLOC_MAX_TERMS;
constexpr size_t kPartialBytes = sizeof(double2) * (kReduceBlocks + 1);
constexpr size_t kScratchBytes = 256 * 1024;
static_assert(kGroupsBytes + kTermsBytes + kPartialBytes <= kScratchBytes, "scratch layout exceeds its size");

__device__ __align__(256) unsigned char g_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
struct ScratchAddr {
    unsigned long long ctx_id = 0;  // driver context the address belongs to (0: none yet)
    void* ptr = nullptr;
};
ScratchAddr g_scratch_addr[kMaxDevices];
std::mutex g_setup_mutex;

int fail(int code, const std::string& msg) {
    gq::set_last_error(msg);  // reported by gq_last_error()
    return code;
}

// Unique id (for the life of the process) of the calling thread's current
// driver context, 0 when none is current. The two driver functions come
// through the runtime's entry-point query, so the library needs no link
// against libcuda.
unsigned long long current_context_id() {
    using GetCurrent = CUresult (*)(CUcontext*);
    using GetId = CUresult (*)(CUcontext, unsigned long long*);
    static GetCurrent get_current = nullptr;
    static GetId get_id = nullptr;
    static bool looked_up = false;
    if (!looked_up) {
        cudaDriverEntryPointQueryResult q1, q2;
        void* f1 = nullptr;
        void* f2 = nullptr;
        if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &f1, 12000, cudaEnableDefault, &q1) == cudaSuccess &&
            cudaGetDriverEntryPointByVersion("cuCtxGetId", &f2, 12000, cudaEnableDefault, &q2) == cudaSuccess &&
            q1 == cudaDriverEntryPointSuccess && q2 == cudaDriverEntryPointSuccess) {
            get_current = (GetCurrent)f1;
            get_id = (GetId)f2;
        }
        cudaGetLastError();
        looked_up = true;
    }
    if (!get_current || !get_id) return 0;
    CUcontext ctx = nullptr;
    unsigned long long id = 0;
    if (get_current(&ctx) != CUDA_SUCCESS || !ctx) return 0;
    if (get_id(ctx, &id) != CUDA_SUCCESS) return 0;
    return id;
}

// Device address of g_scratch in the current device's context: looked up
// with cudaGetSymbolAddress on the first call on a device and again when that
// device's current context is not the one the cached address came from.
int scratch_address(int dev, void** out) {
    if (dev < 0 || dev >= kMaxDevices) return fail(GQ_EINVAL, "device ordinal beyond the supported range");
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    ScratchAddr& a = g_scratch_addr[dev];
    const unsigned long long ctx = current_context_id();
    if (!a.ptr || ctx == 0 || a.ctx_id != ctx) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_scratch);
        if (e != cudaSuccess) return fail(GQ_ECUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
        a.ptr = p;
        a.ctx_id = current_context_id();  // the lookup made the device's context current
    }
    *out = a.ptr;
    return GQ_OK;
}

}  // namespace

extern "C" {

int gq_expect_pauli_sum_noalloc(const void* device_state, int num_qubits, int precision, const gq_pauli_term* terms,
                                size_t n_terms, void* stream, double* out_re, double* out_im) {
    if (!device_state || (n_terms && !terms)) return fail(GQ_EINVAL, "null argument");
    if (num_qubits < 1 || num_qubits > 40) return fail(GQ_EINVAL, "num_qubits out of range [1, 40]");
    if (precision != GQ_C128 && precision != GQ_C64) return fail(GQ_EINVAL, "unknown precision");
    if (n_terms > GQ_NOALLOC_MAX_TERMS)
        return fail(GQ_EINVAL, "too many Pauli terms: " + std::to_string(n_terms) + " > GQ_NOALLOC_MAX_TERMS (" +
                                   std::to_string(GQ_NOALLOC_MAX_TERMS) + ")");
    const uint64_t qmask = (1ull << num_qubits) - 1;
    // Terms grouped by x mask, with coeff * i^(number of Y) folded in
    // (the same tables as the allocating entry point builds).
    std::vector<size_t> order(n_terms);
    for (size_t i = 0; i < n_terms; ++i) {
        if ((terms[i].x_mask | terms[i].z_mask) & ~qmask) return fail(GQ_EINVAL, "Pauli term on a qubit out of range");
        order[i] = i;
    }
    std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) { return terms[a].x_mask < terms[b].x_mask; });
    std::vector<NGroup> groups;
    std::vector<NTerm> dt;
    for (size_t k = 0; k < n_terms; ++k) {
        const gq_pauli_term& t = terms[order[k]];
        if (groups.empty() || groups.back().x != t.x_mask) groups.push_back({t.x_mask, (int32_t)k, (int32_t)k});
        groups.back().t1 = (int32_t)k + 1;
        const int ny = __builtin_popcountll(t.x_mask & t.z_mask) & 3;
        double pr = 1, pi = 0;
        if (ny == 1) pr = 0, pi = 1;
        if (ny == 2) pr = -1, pi = 0;
        if (ny == 3) pr = 0, pi = -1;
        dt.push_back({t.coeff_re * pr - t.coeff_im * pi, t.coeff_re * pi + t.coeff_im * pr, t.z_mask});
    }
    cudaStream_t s = (cudaStream_t)stream;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return fail(GQ_ECUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    // The call copies from host memory and waits for its result: it cannot
    // be recorded into a graph.
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    e = cudaStreamIsCapturing(s, &cap);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(GQ_EINVAL, std::string("stream capture query failed: ") + cudaGetErrorString(e));
    }
    if (cap != cudaStreamCaptureStatusNone)
        return fail(GQ_EINVAL, "gq_expect_pauli_sum_noalloc is synchronous and cannot be called on a capturing stream");
    // The state must be device memory the current device can address; a host
    // pointer or another device's allocation would fault the kernel.
    cudaPointerAttributes attr;
    e = cudaPointerGetAttributes(&attr, device_state);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(GQ_EINVAL, std::string("device_state is not a CUDA pointer: ") + cudaGetErrorString(e));
    }
    if (attr.type != cudaMemoryTypeDevice && attr.type != cudaMemoryTypeManaged)
        return fail(GQ_EINVAL, "device_state is not device memory");
    if (attr.type == cudaMemoryTypeDevice && attr.device != dev)
        return fail(GQ_EINVAL, "device_state belongs to device " + std::to_string(attr.device) +
                                   ", but device " + std::to_string(dev) + " is current");
    void* base = nullptr;
    int rc = scratch_address(dev, &base);
    if (rc != GQ_OK) return rc;
    char* sc = (char*)base;
    NGroup* d_groups = (NGroup*)sc;
    NTerm* d_terms = (NTerm*)(sc + kGroupsBytes);
    double2* d_partial = (double2*)(sc + kGroupsBytes + kTermsBytes);
    if (!groups.empty()) e = cudaMemcpyAsync(d_groups, groups.data(), sizeof(NGroup) * groups.size(), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess && !dt.empty())
        e = cudaMemcpyAsync(d_terms, dt.data(), sizeof(NTerm) * dt.size(), cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return fail(GQ_ECUDA, std::string("cudaMemcpyAsync: ") + cudaGetErrorString(e));
    const uint64_t n = 1ull << num_qubits;
    if (precision == GQ_C64)
        k_expect_noalloc<float><<<kReduceBlocks, 256, 0, s>>>((const cplx<float>*)device_state, n, d_groups,
                                                              (int)groups.size(), d_terms, d_partial);
    else
        k_expect_noalloc<double><<<kReduceBlocks, 256, 0, s>>>((const cplx<double>*)device_state, n, d_groups,
                                                               (int)groups.size(), d_terms, d_partial);
    k_reduce_noalloc<<<1, 1024, 0, s>>>(d_partial, kReduceBlocks, d_partial + kReduceBlocks);
    e = cudaGetLastError();
    if (e != cudaSuccess) return fail(GQ_ECUDA, std::string("kernel launch: ") + cudaGetErrorString(e));
    double2 v;
    e = cudaMemcpyAsync(&v, d_partial + kReduceBlocks, sizeof(double2), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return fail(GQ_ECUDA, std::string("result copy: ") + cudaGetErrorString(e));
    if (out_re) *out_re = v.x;
    if (out_im) *out_im = v.y;
    return GQ_OK;
}

}  // extern "C"

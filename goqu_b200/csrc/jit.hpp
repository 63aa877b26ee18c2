// Specialised tile-pass kernels compiled at run time (NVRTC, sm_100a).
//
// The interpreted pass kernel (k_tile_pass) reads every op of a pass from the
// program at run time and dispatches on its kind, target register bits and
// controls. For a pass whose structure is known, jit_plan() emits the same
// pass as straight-line CUDA C++: the same tile_core.cuh op bodies, but with
// target bits, controls, shared-memory slots and global index columns as
// compile-time constants, and the pass's matrices passed by value as a kernel
// parameter block (constant-bank operands of the FMAs). The kernel text holds
// no matrix values, so passes with the same structure and different angles
// share one compiled kernel.
//
// Compilation runs on background threads; until a pass's kernel is ready the
// engine launches the interpreted kernel for it (GQ_OPT_JIT = 1), or waits
// for it (GQ_OPT_JIT = 2).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "schedule.hpp"

namespace gq {

struct JitPlan {
    std::string source;  // kernel text (the cache key)
    // Matrix entries packed into the parameter block, in order: (pool offset, count).
    std::vector<std::pair<uint32_t, uint32_t>> copies;
    uint32_t n_param = 0;  // complex entries of the parameter block (>= 1)
};

// Kernel text for pass `pass` of `pr` at precision c64 / c128 with the given
// launch bounds. Returns false for passes the generator does not cover
// (gradient ops), which stay on the interpreted kernel.
bool jit_plan(const Program& pr, size_t pass, bool c64, int threads, int min_blocks, JitPlan& out);

// Process-wide cache of compiled kernels, keyed by kernel text.
enum JitState { JIT_MISSING = 0, JIT_PENDING = 1, JIT_READY = 2, JIT_FAILED = 3 };

bool jit_available();  // libnvrtc could be loaded
// Returns the state of the kernel for `source`; queues its compilation when
// it is missing. On JIT_READY, *fn is the launchable kernel (cudaKernel_t),
// allowed `smem_bytes` of dynamic shared memory on the current device.
JitState jit_lookup(const std::string& source, size_t smem_bytes, bool queue, const void** fn);
// Blocks until no queued compilation is pending (or `max_ms` have passed).
void jit_wait(double max_ms);
// Compiles `source` to a cubin on the calling thread (no device needed).
// Returns "" on success, else the compiler log.
std::string jit_compile_only(const std::string& source, std::vector<char>* cubin, std::string* log);
// Milliseconds spent compiling (all threads) and kernels compiled so far.
void jit_counters(double* compile_ms, int64_t* compiled, int64_t* failed);

}  // namespace gq

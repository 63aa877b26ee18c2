// Specialised tile-pass kernels compiled at run time (NVRTC, sm_100a).
//
// The interpreted pass kernel (k_tile_pass) reads every op of a pass from the
// program at run time and dispatches on its kind, target register bits and
// controls. For a pass whose structure is known, jit_plan() emits the same
// pass as straight-line CUDA C++: the tile_core.cuh op bodies with target
// bits, controls, shared-memory slots and global index columns as
// compile-time constants, and the pass's numbers passed by value as a kernel
// parameter block (constant-bank operands of the FMAs).
//
// Within a phase the generator also keeps a pending factor per register slot
// (a product of "atoms": diagonal entries, phases): diagonal ops and
// permutations without run-time conditions cost no arithmetic, and a general
// one-qubit unitary U = g diag(1, e^{i phi}) cos(theta/2) [[1, -t], [t, 1]]
// diag(1, e^{i lambda}) (t = tan(theta/2)) costs one complex multiply on half
// the slots (to equalise the pair's factors) plus a real shear. Factors are
// folded into the amplitudes before any op that needs them equal across its
// group and at the end of the phase. Products and ratios of atoms are
// evaluated on the host by jit_pack() when the pass is launched.
//
// The kernel text holds no numbers, so passes with the same structure and
// other angles share one compiled kernel. Compilation runs on background
// threads; until a pass's kernel is ready the engine launches the
// interpreted kernel for it (GQ_OPT_JIT = 1), or waits for it (GQ_OPT_JIT = 2).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "schedule.hpp"

namespace gq {

// A factor value: pool[ref] (kind 0), or for the one-qubit unitary at
// ops[ref]: e^{i lambda} (1), g cos(theta/2) (2), g cos(theta/2) e^{i phi} (3);
// kinds 4-6 are the same three for the product of chain ref / 4 under the
// predicate values ref % 4 (JitChain).
struct JitAtom {
    uint8_t kind;
    uint32_t ref;
};

// One parameter-block entry: `count` pool values from pool[ref] (kind 0), the
// shear t of the one-qubit unitary ops[ref] (kind 1, real part), the product
// of atoms `num` divided by the product of atoms `den` (kind 2), or the shear
// t of chain ref / 4 under predicate values ref % 4 (kind 3).
struct JitEntry {
    uint8_t kind;
    uint32_t ref, count;
    std::vector<uint32_t> num, den;
};

// A chain of one-qubit ops on one register bit inside a phase: uncontrolled
// one-qubit unitaries and X-type ops, each X either unconditional (pred -1)
// or controlled by CTA-uniform predicate `pred` (0 or 1, local to the chain).
// No other op of the phase touches the bit between them, so the chain acts as
// one unitary per combination of its (at most two) predicates. Ops are pass
// relative, in order of application.
struct JitChain {
    std::vector<uint32_t> ops;
    std::vector<int8_t> pred;
};

struct JitPlan {
    std::string source;       // device kernel text (the cache key)
    std::string host_source;  // the same pass as a host function (CPU tests), when asked for
    std::vector<JitAtom> atoms;
    std::vector<JitEntry> entries;
    std::vector<JitChain> chains;
    uint32_t n_param = 0;                             // complex entries of the parameter block (>= 1)
    std::vector<std::vector<uint32_t>> phase_shears;  // shear ops of each phase (range check)
    std::vector<std::vector<uint32_t>> phase_chains;  // chains of each phase (range check)
};

// Kernel text for pass `pass` of `pr` at precision c64 / c128 with the given
// launch bounds (and, with `host`, the host-function form in host_source).
// persistent: the kernel is launched with fewer CTAs than tiles; each CTA
// walks tiles blockIdx.x, + gridDim.x, ... with two tile buffers (2 x 2^m
// amplitudes of dynamic shared memory), copying the next tile in with
// cp.async while the current one runs. Otherwise one CTA per tile.
// Returns false for passes the generator does not cover (gradient ops, or a
// parameter block over the kernel-parameter limit): they stay interpreted.
bool jit_plan(const Program& pr, size_t pass, bool c64, int threads, int min_blocks, bool persistent, JitPlan& out,
              bool host = false);
// The reverse (adjoint) pass on psi and lambda at once (kernel gqj_dual):
// every op on both states, gradient ops adding Re <lambda|G|psi> into
// per-warp slots that each CTA sums into partial[cta * nslots + slot], as
// k_adjoint_pass does. Dense ops stay dense (no pending factors). With
// `host`, host_source holds the same pass as a host function (CPU tests).
bool jit_plan_dual(const Program& pr, size_t pass, bool c64, int threads, int min_blocks, JitPlan& out,
                   bool host = false);
// Op and pool indices in a plan and its kernel text are relative to the
// pass: to its first op and that op's first pool entry (jit_bases). The
// kernel is launched with `pool` advanced by pool_base and `phases` by the
// pass's phase0, so passes of the same structure anywhere in any program
// share a plan and a kernel.
void jit_bases(const Program& pr, size_t pass, uint32_t* op_base, uint32_t* pool_base);
// Fills the parameter block (n_param complex values of float or double) from
// pass `pass` of the program's current numbers. Returns false when the pass's
// shears could leave the floating-point range; the pass then runs interpreted.
bool jit_pack(const Program& pr, size_t pass, const JitPlan& plan, bool c64, void* block);
// Decomposition of a one-qubit unitary m (row major) into the shear form
// above. False when m is not unitary to 1e-12 or cos / sin(theta/2) is below
// 1e-150 (the generator then keeps the dense 2x2).
bool u1_decompose(const Z* m, double* t, Z* lam, Z* post0, Z* post1);

// Candidate chains (JitChain) of pass `pass`, per phase, with the outer-qubit
// control mask of each predicate, and whether every product of the chain
// decomposes into the shear form with the program's current numbers. A chain
// holds at least two one-qubit unitaries.
struct ChainCand {
    int phase;
    JitChain chain;
    uint64_t pmask[2];
    bool fusable;
};
std::vector<ChainCand> jit_chains(const Program& pr, size_t pass);

// A pass's plan as cached per process, keyed by the pass's structure (launch
// shape, tile and phase tables, op kinds, bits, controls, relative pool
// offsets, which one-qubit unitaries decompose): every pass of that
// structure reuses the text and, once compiled, the kernel, without
// generating the text again.
struct CachedPlan {
    bool ok = false;        // jit_plan covered the pass
    JitPlan plan;
    const void* fn = nullptr;  // compiled kernel, once ready
    bool failed = false;    // compilation or loading failed
};
// Compiles with NVRTC through an on-disk cache: a cubin stored under a hash of
// everything it depends on (options, NVRTC version, the tile header, the
// kernel text) is reused when its stored identity equals this one byte for
// byte; new binaries are written through a temporary file and a rename.
// Directory: $GQ_JIT_CACHE_DIR ("off" disables), else
// $XDG_CACHE_HOME/goqu_b200/jit, else ~/.cache/goqu_b200/jit.
std::string jit_cache_dir();
std::string jit_compile_cached(const std::string& source, std::vector<char>* cubin, std::string* log, bool* from_disk);
// The plan cache's key of pass `pass`: everything the generated kernel's text
// depends on (launch shape, tile and phase tables, op kinds, bits, controls
// and pass-relative pool offsets, which unitaries take the shear form, which
// chains fuse), not the numbers.
std::string jit_plan_key(const Program& pr, size_t pass, bool c64, int threads, int min_blocks, bool persistent,
                         bool dual);
const CachedPlan* jit_cached_plan(const Program& pr, size_t pass, bool c64, int threads, int min_blocks,
                                  bool persistent, bool dual = false);
// The compiled kernel of a cached plan (queues its compilation on first call);
// nullptr until it is ready.
const void* jit_plan_kernel(const CachedPlan* cp, size_t smem_bytes);

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

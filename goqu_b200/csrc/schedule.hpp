// Host-side gate analysis and pass scheduling for the tile-pass kernel.
//
// normalize(): each gq_op becomes an NGate by reading its matrix: control
//   qubits (identity on their |0> block) are split off, and what remains is
//   classified as a scalar phase, a diagonal, an X-type swap with phases, a
//   SWAP, or a dense unitary on 1-4 target qubits. goqu routes gates through
//   pointer-equality and interface tiers (sim/statevector/kernel2q.go:24-114);
//   reading the structure from the matrix covers those tiers and every other
//   gate with the same structure.
// schedule(): packs the gate list into passes (one launch each) and phases
//   (register sets of 4 qubits) and emits the device program.
#pragma once
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/gqb200.h"
#include "tile_core.cuh"

namespace gq {

struct Z {
    double re, im;
};

struct NGate {
    KType type = K_NONE;
    std::vector<int> targets;  // U: matrix order (first = MSB); DIAG: table order
    uint64_t ctrl = 0;         // control qubits (all must be 1)
    std::vector<Z> data;       // U: 4^t matrix; X: {p0,p1}; DIAG: 2^t table; PHASE: {s}
    bool pure = false;         // X: plain swap
    uint64_t nd_mask = 0;      // qubits acted on non-diagonally (must be in registers)
    uint64_t d_mask = 0;       // qubits acted on diagonally (controls, diagonal targets)
    bool barrier = false;      // reset: nonlinear, commutes with nothing
    KType grad_kind = K_NONE;  // K_GRAD: structure of G (dense K_U*, K_DIAG or K_PHASE)
    int param = -1;            // K_GRAD: circuit parameter the slot accumulates into
    int cost = 0;              // FMA per amplitude, for the pass budget
    int src = -1;              // index of the gq_op it came from
};

struct SchedOptions {
    int tile_qubits = 12;  // m
    int low_qubits = 3;    // lowest qubits always in a tile (coalesced runs)
    int budget = 96;       // FMA-per-amplitude budget of a pass
    int swizzle_width = 3; // log2 of the 16-byte (c128) / 8-byte (c64) slots of one bank sweep
    bool fuse_pairs = true;   // fold runs of identical parity-symmetric 2-qubit diagonals into one
                              // K_PAIRSUM (the interpreted kernels; the specialised kernels keep
                              // diagonals as pending factors at no cost and take K_PAIRSUM off)
    bool fuse_dense = false;  // fold runs of register-local gates of a phase into one dense block
                              // (measured slower on the layered benchmark: dense blocks reload
                              // their matrix per amplitude group)
    // Qubits that may be 1 in a nonzero amplitude of the state the program
    // starts from (every amplitude whose index has a bit outside the mask is
    // exactly zero); all ones when nothing is known. A pass maps an all-zero
    // tile to an all-zero tile, so a pass launches only the CTAs whose outer
    // bits lie inside the support reached so far: the others keep their
    // zeros in place. After a reset to |0...0> the support is empty, and each
    // pass adds the qubits its non-diagonal ops act on.
    uint64_t support0 = ~0ull;
};

struct Program {
    std::vector<PassDesc> passes;
    std::vector<PhaseDesc> phases;
    std::vector<KOp> ops;
    std::vector<Z> pool;
    int64_t gates = 0;
    int64_t conflict_phases = 0;  // phases whose lane groups could not be made conflict free
    std::vector<std::vector<int>> pass_params;  // K_GRAD: parameter of each slot, per pass
    uint64_t support_out = ~0ull;  // the support after the last pass (SchedOptions::support0)
};

// Appends the NGates of one op (0 when it is an identity or a barrier).
// Returns GQ_OK or an error code with `err` set.
int normalize_op(const gq_op& op, int nphys, std::vector<NGate>& out, std::string& err);
// Builds an NGate from a dense matrix on `qubits` (first = MSB) with extra
// controls; used for gates and for density-matrix superoperators.
int analyze_matrix(const std::vector<Z>& m, const std::vector<int>& qubits, uint64_t ctrl, int src,
                   std::vector<NGate>& out, std::string& err);
void schedule(const std::vector<NGate>& gates, int nphys, const SchedOptions& opt, Program& prog);
// Density matrix ops -> NGates on the 2n-qubit vectorised rho (row qubit q is
// vector bit q+n, column qubit q is bit q): U on rows and conj(U) on columns,
// channels as sum_k E_k (x) conj(E_k), a gate and the channel that follows it
// on the same qubits folded into one superoperator. With `structured`, a
// channel whose superoperator only mixes populations among themselves and
// scales coherences (depolarizing, amplitude and phase damping) is applied
// after its gate as permutations, a diagonal and the population map on a
// 2^-k share of the entries instead.
int dm_gates(int nq, const gq_op* ops, size_t n_ops, std::vector<NGate>& gates, std::string& err,
             bool structured = true);
// Adjoint differentiation: `forward` are the gates of `ops`; `reverse` is the
// reverse sweep: for each op from last to first, one K_GRAD gate per
// parameter it depends on (G = dU/dtheta * U^dagger, zero where its controls
// are unset), then the inverse of the op. Ops must be unitary. `seg_ends`
// receives, per forward gate, the op index it came from (for checkpoints).
int adjoint_gates(int nq, const gq_op* ops, size_t n_ops, size_t n_params, std::vector<NGate>& forward,
                  std::vector<NGate>& reverse, std::vector<int>& fwd_op, std::vector<int>& rev_op, std::string& err);
// Forward checkpoints of an adjoint gradient. requested > 0 (the caller's
// GQ_OPT_ADJOINT_SEGMENTS) is kept, capped at the op count. Automatic (0):
// complex64 circuits of more than 256 ops take one segment per 128 ops (at most
// 8), others none; the count is then cut so that the (segments - 1) stored
// states of state_bytes fit in avail_bytes less kAdjointHeadroom, down to 1.
constexpr size_t kAdjointHeadroom = size_t(256) << 20;
int adjoint_segments(int requested, bool c64, size_t n_ops, size_t state_bytes, size_t avail_bytes);

}  // namespace gq

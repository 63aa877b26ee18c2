/*
 * gqb200.h - C ABI of the B200 (sm_100a) statevector / density-matrix engine.
 *
 * The engine sits behind goqu's simulator API (github.com/splch/goqu):
 *   sim/sim.go:9-22                 sim.Simulator {Run, Evolve, StateVector, Close}
 *   sim/statevector/sim.go:27-382   statevector.New/Run/Evolve/Apply/StateVector/Expect*
 *   sim/densitymatrix/sim.go:32-313 densitymatrix.New/WithNoise/Run/Evolve/DensityMatrix/...
 *   algorithm/gradient/gradient.go  CostFunc / ParameterShift (plus a new adjoint method)
 *   sweep/run.go:27-171             RunSim (batches of bound circuits)
 * Every function is plain C: pointers, sizes and integer status codes. No
 * CUDA or C++ types cross the boundary. All functions return GQ_OK (0) on
 * success; on failure they return a GQ_E* code and gq_last_error() returns a
 * message for the calling thread.
 *
 * Conventions (identical to goqu):
 *  - amplitude index bit q is qubit q (qubit 0 is the least significant bit);
 *  - a k-qubit gate matrix is row-major, 2^k x 2^k, interleaved (re, im)
 *    doubles; its local index uses the FIRST listed qubit as the most
 *    significant bit (circuit/gate/fixed.go:169-171, 316-317);
 *  - a density matrix is row-major rho[r * 2^n + c].
 * A handle is not thread-safe; distinct handles may be used concurrently.
 */
#ifndef GQB200_H
#define GQB200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GQ_ABI_VERSION 5

/* ---- status codes ------------------------------------------------------ */
#define GQ_OK 0
#define GQ_EINVAL 1        /* bad argument (qubit out of range, size mismatch, ...) */
#define GQ_ENOMEM 2        /* device or host allocation failed                      */
#define GQ_ECUDA 3         /* a CUDA runtime call failed                            */
#define GQ_EUNSUPPORTED 4  /* op kind / size the engine does not handle             */
#define GQ_ENODEVICE 5     /* no usable sm_100 device                               */
#define GQ_EDEVICE 6       /* a kernel reported an error status (bounded wait, ...) */

/* ---- precision ----------------------------------------------------------- */
#define GQ_C128 0 /* complex128 state, FP64 arithmetic                        */
#define GQ_C64 1  /* complex64 state, FP32 gate arithmetic, FP64 reductions   */

/* ---- op kinds --------------------------------------------------------------
 * The kind mirrors the dispatch goqu's CPU simulator performs, so the Go shim
 * can forward what its own type switch found:
 *   sim/statevector/sim.go:92-157       (Apply: 1q / 2q / 3q / controlled)
 *   sim/statevector/kernel2q.go:24-114  (pointer-equality and interface tiers)
 *   sim/statevector/kernel3q.go:10-47
 *   sim/statevector/kernel_controlled.go:11-41
 * The GPU engine analyses the matrix itself (diagonal / permutation / control
 * structure), so the kind is a hint for it; the matrix is always required.   */
#define GQ_OP_MATRIX 0          /* generic 1-, 2- or 3-qubit matrix                */
#define GQ_OP_CNOT 1            /* gate.CNOT  (fixed.go:183)                       */
#define GQ_OP_CZ 2              /* gate.CZ    (fixed.go:199)                       */
#define GQ_OP_SWAP 3            /* gate.SWAP  (fixed.go:215)                       */
#define GQ_OP_CY 4              /* gate.CY    (fixed.go:229)                       */
#define GQ_OP_ISWAP 5           /* gate.ISWAP (fixed.go:245)                       */
#define GQ_OP_SYCAMORE 6        /* gate.Sycamore (fixed.go:387)                    */
#define GQ_OP_CCX 7             /* gate.CCX   (fixed.go:329)                       */
#define GQ_OP_CSWAP 8           /* gate.CSWAP (fixed.go:349)                       */
#define GQ_OP_CCZ 9             /* gate.CCZ   (fixed.go:364)                       */
#define GQ_OP_CTRL_DIAG_2Q 10   /* gate.ControlDiagonal2Q (CP, CRZ; gate.go:62-66) */
#define GQ_OP_DIAG_2Q 11        /* gate.Diagonal2Q (RZZ, ZZ; gate.go:55-59)         */
#define GQ_OP_CTRL_U_2Q 12      /* gate.ControlU2Q (CRX, CRY; gate.go:69-75)        */
#define GQ_OP_CONTROLLED 13     /* gate.ControlledGate with >= 4 qubits: controls
                                   first, `matrix` is the INNER gate's matrix      */
#define GQ_OP_RESET 14          /* deterministic reset (sim/statevector/sim.go:168) */
#define GQ_OP_CHANNEL 15        /* density matrix only: Kraus channel; `matrix`
                                   holds num_kraus matrices back to back           */
#define GQ_OP_BARRIER 16        /* no-op (barrier / delay / measure on the SV path) */

#define GQ_MAX_OP_QUBITS 16
#define GQ_MAX_OP_PARAMS 3

/* One operation of a circuit, in circuit order. */
typedef struct gq_op {
    int32_t kind;
    int32_t num_qubits;   /* qubits listed in `qubits`                           */
    int32_t num_controls; /* GQ_OP_CONTROLLED: how many leading qubits are controls */
    int32_t num_kraus;    /* GQ_OP_CHANNEL: number of Kraus matrices             */
    int32_t qubits[GQ_MAX_OP_QUBITS];
    const double* matrix; /* interleaved complex, row-major (see conventions)    */
    /* Adjoint differentiation (optional): the op's matrix depends on up to three
     * circuit parameters; dmatrix[k] = d(matrix)/d(param[param_index[k]]) with
     * the chain rule of the bound expression already applied. Unused slots
     * have param_index = -1 and dmatrix = NULL.                                 */
    int32_t param_index[GQ_MAX_OP_PARAMS];
    int32_t reserved;
    const double* dmatrix[GQ_MAX_OP_PARAMS];
} gq_op;

/* One Pauli string in symplectic form (sim/pauli/pauli.go:19-24, 146-169):
 * bit q of x_mask set for X or Y on qubit q, bit q of z_mask set for Z or Y. */
typedef struct gq_pauli_term {
    double coeff_re;
    double coeff_im;
    uint64_t x_mask;
    uint64_t z_mask;
} gq_pauli_term;

/* Work counters of the most recent apply / run on a handle. */
typedef struct gq_stats {
    int64_t gates_in;        /* ops received (unitary gates, after skipping no-ops) */
    int64_t passes;          /* full-state passes launched                       */
    int64_t kernel_launches; /* kernels of this library launched                  */
    int64_t phases;          /* register phases summed over all passes            */
    int64_t state_bytes;     /* bytes of one state (2^n * amplitude size)          */
    double last_ms;          /* device time of the last apply/evolve call, CUDA events
                                on the handle's stream (GQ_OPT_TIMING only)           */
    double pass_ms;          /* device time of its tile passes alone (first to last) */
    int64_t h2d_bytes;       /* host->device bytes the last call copied (program, inputs) */
    int64_t d2h_bytes;       /* device->host bytes the last call copied (results)   */
    int64_t jit_passes;      /* passes of the last call run by a specialised kernel */
    double jit_compile_ms;   /* process total: milliseconds spent compiling them    */
    double host_ms;          /* batches: host time of the last call before its first
                                launch (analysis, scheduling, table packing, upload) */
    int64_t tile_bytes;      /* bytes the last call's tile passes read and wrote: 2 x
                                amplitude size x amplitudes of the CTAs launched
                                (passes x 2 x state_bytes unless GQ_OPT_ZERO_TILES
                                skipped tiles)                                      */
} gq_stats;

/* ---- library ------------------------------------------------------------- */
int gq_abi_version(void);
/* Message of the last failed call on this thread ("" if none). */
const char* gq_last_error(void);
/* Number of visible sm_100 devices. */
int gq_device_count(int* count);

/* ---- statevector: replaces statevector.New/Sim (sim/statevector/sim.go) ---- */
typedef struct gq_sv gq_sv;

/* New(n): state |0...0>. num_qubits in [1, 34] (goqu caps at 28; the GPU
 * engine is bounded by device memory). Replaces sim/statevector/sim.go:27-35. */
int gq_sv_create(int num_qubits, int precision, gq_sv** out);
int gq_sv_destroy(gq_sv* sv);
int gq_sv_num_qubits(const gq_sv* sv, int* out);
/* Reset to |0...0> (sim/statevector/sim.go:71-76). */
int gq_sv_reset(gq_sv* sv);
/* Apply ops to the current state (sim/statevector/sim.go:92-157). */
int gq_sv_apply(gq_sv* sv, const gq_op* ops, size_t n_ops);
/* Evolve: reset then apply (sim/statevector/sim.go:83-86). */
int gq_sv_evolve(gq_sv* sv, const gq_op* ops, size_t n_ops);
/* Copy the state to host memory: 2^n interleaved complex values, double for
 * GQ_C128, float for GQ_C64 (StateVector, sim/statevector/sim.go:61-65).       */
int gq_sv_get_state(gq_sv* sv, void* host_out, size_t bytes);
int gq_sv_set_state(gq_sv* sv, const void* host_in, size_t bytes);
/* p_i = re^2 + im^2 in FP64 (sim/statevector/sim.go:274-280). */
int gq_sv_probabilities(gq_sv* sv, double* host_out, size_t n);
/* Inverse-CDF sampling: for each uniform r (caller-supplied, in [0,1)), the
 * first index i with r < sum_{j<=i} p_j summed sequentially in FP64, else
 * 2^n - 1 (sampleIndex, sim/statevector/sim.go:288-298). Bit-exact with that
 * sequential sum. */
int gq_sv_sample(gq_sv* sv, const double* uniforms, size_t shots, uint64_t* idx_out);
/* Run for static circuits: Evolve then sample (sim/statevector/sim.go:40-58). */
int gq_sv_run(gq_sv* sv, const gq_op* ops, size_t n_ops, const double* uniforms,
              size_t shots, uint64_t* idx_out);
/* Sampling with the histogram built on the device: the distinct sampled
 * outcomes in increasing index order with their counts, i.e. the entries of
 * the map[bitstring]int that Run returns (sim/statevector/sim.go:40-58; the
 * bitstring is formatBitstring of the outcome, :306-316). outcomes_out and
 * counts_out need room for min(shots, 2^n) entries; *n_distinct receives how
 * many were written. Same uniforms, same outcomes as gq_sv_sample. At most
 * 2^32 - 1 shots per call. */
int gq_sv_sample_counts(gq_sv* sv, const double* uniforms, size_t shots, uint64_t* outcomes_out,
                        uint64_t* counts_out, size_t* n_distinct);
/* Run with counts: Evolve, then gq_sv_sample_counts. */
int gq_sv_run_counts(gq_sv* sv, const gq_op* ops, size_t n_ops, const double* uniforms, size_t shots,
                     uint64_t* outcomes_out, uint64_t* counts_out, size_t* n_distinct);
/* sum_t coeff_t <psi|P_t|psi> as a complex number (pauli.ExpectSum,
 * sim/pauli/expect_sv.go:21-97); ExpectPauliSum is its real part.            */
int gq_sv_expect_pauli_sum(gq_sv* sv, const gq_pauli_term* terms, size_t n_terms,
                           double* out_re, double* out_im);
/* sum_i (-1)^popcount(i & mask) p_i, unrounded (ExpectationValue before its
 * 1e-14 rounding, sim/statevector/sim.go:368-382).                           */
int gq_sv_expect_z_mask(gq_sv* sv, uint64_t mask, double* out);
/* Adjoint-method gradient of E(theta) = Re <psi(theta)|H|psi(theta)> for the
 * circuit `ops` applied to |0...0> (new: goqu only has ParameterShift and
 * FiniteDifference, algorithm/gradient/gradient.go:49-86). grad_out has
 * n_params entries; op parameters use gq_op.param_index / dmatrix.
 * The reverse sweep runs on the handle's state in place and stops at the
 * first parameterised op: evolve again before reading the state.            */
int gq_sv_adjoint_gradient(gq_sv* sv, const gq_op* ops, size_t n_ops,
                           const gq_pauli_term* terms, size_t n_terms,
                           size_t n_params, double* grad_out, double* energy_out);
/* ---- parameterized templates: the optimisation loop ------------------------
 * A template is the op stream of a circuit whose symbolic gates
 * (circuit/param/gate.go:13-142) are rebound from parameter values by the
 * library: each gq_param_gate names an op of the stream (its matrix pointer
 * is ignored), the gate family (goqu's parameterized gates,
 * circuit/gate/parameterized.go:91-564) and, per angle k,
 *   angle_k = scale[k] * theta[param[k]] + shift[k]   (param[k] = -1: shift only).
 * The library computes the matrix and d(matrix)/d(parameter) (closed forms;
 * chain rule over the angles that share a parameter) for every call. */
#define GQ_PG_RX 1
#define GQ_PG_RY 2
#define GQ_PG_RZ 3
#define GQ_PG_PHASE 4        /* P(phi) */
#define GQ_PG_U1 5
#define GQ_PG_U2 6           /* (phi, lambda) */
#define GQ_PG_U3 7           /* (theta, phi, lambda) */
#define GQ_PG_ROT 8          /* (phi, theta, omega) */
#define GQ_PG_CP 9
#define GQ_PG_RXX 10
#define GQ_PG_RYY 11
#define GQ_PG_RZZ 12
#define GQ_PG_FSIM 13        /* (theta, phi) */
#define GQ_PG_PSWAP 14
#define GQ_PG_GLOBAL_PHASE 15

typedef struct gq_param_gate {
    int32_t op_index;   /* op of the template this entry binds               */
    int32_t gate;       /* GQ_PG_* family                                     */
    int32_t num_angles; /* the family's angle count (1, 2 or 3)               */
    int32_t param[3];
    double scale[3];
    double shift[3];
} gq_param_gate;

/* Adjoint gradient (as gq_sv_adjoint_gradient) of the template bound at theta. */
int gq_sv_adjoint_template(gq_sv* sv, const gq_op* ops, size_t n_ops, const gq_param_gate* pgates, size_t n_pgates,
                           const double* theta, size_t n_params, const gq_pauli_term* terms, size_t n_terms,
                           double* grad_out, double* energy_out);

/* Adam options (algorithm/optim/adam.go:9-49, optim.go:21-58); zero or
 * negative fields take goqu's defaults: lr 0.001, beta1 0.9, beta2 0.999,
 * epsilon 1e-8, max_iter 1000, fun_tol 1e-8; grad_tol 0 disables that test. */
typedef struct gq_adam_options {
    double lr, beta1, beta2, epsilon;
    int32_t max_iter;
    int32_t reserved;
    double fun_tol;
    double grad_tol;
} gq_adam_options;

/* optim.Result (algorithm/optim/optim.go:60-69). */
typedef struct gq_optim_result {
    double fun;
    int32_t iterations;
    int32_t func_evals;
    int32_t grad_evals;
    int32_t converged;
} gq_optim_result;

/* optim.Adam.Minimize (adam.go:51-140) of E(theta) = Re <psi(theta)|H|psi(theta)>
 * with adjoint gradients (vqe.Run with the Adam optimizer and an adjoint
 * GradientFunc, algorithm/vqe/vqe.go:50-89). The loop runs inside the library:
 * each iteration binds the template, and one forward + reverse sweep yields
 * both the energy goqu evaluates after an update and the gradient of the
 * next iteration, so there is one device evaluation per iteration and the
 * state stays on the device. x holds x0 and receives the result's X;
 * history_out (optional, history_cap entries) receives every energy
 * evaluated, in order (vqe.Result.History). Counts follow goqu's. */
int gq_sv_minimize_adam(gq_sv* sv, const gq_op* ops, size_t n_ops, const gq_param_gate* pgates, size_t n_pgates,
                        const gq_pauli_term* terms, size_t n_terms, size_t n_params, double* x,
                        const gq_adam_options* opts, gq_optim_result* result, double* history_out,
                        size_t history_cap);

/* ---- dynamic circuits: replaces measureQubit (sim/statevector/dynamic.go:179-230) ----
 * The per-shot control flow of RunDynamic (dynamic.go:14-177) stays on the
 * host; shots sharing a measurement history share one device state. */
/* P(qubit = 0): sum of |a_i|^2 over the amplitudes with the qubit's bit clear
 * (dynamic.go:183-194), FP64. */
int gq_sv_prob0(gq_sv* sv, int qubit, double* p0);
/* Collapse onto `outcome` given P(0) = p0: the other half is zeroed and the
 * kept half scaled by 1/sqrt(p0) (outcome 0) or 1/sqrt(1 - p0) (outcome 1);
 * nothing changes when that norm is below 1e-15 (dynamic.go:203-229). */
int gq_sv_collapse(gq_sv* sv, int qubit, int outcome, double p0);
/* measureQubit with the caller's uniform u: outcome 1 iff u >= P(0)
 * (dynamic.go:197-200), then the collapse. */
int gq_sv_measure(gq_sv* sv, int qubit, double u, int* outcome);
/* dst's state <- src's state (same qubit count and precision): the branch
 * of a measurement history that both outcomes continue from. */
int gq_sv_copy_state(gq_sv* dst, const gq_sv* src);
int gq_sv_stats(const gq_sv* sv, gq_stats* out);

/* Engine options (per handle). */
#define GQ_OPT_TILE_QUBITS 1    /* qubits staged per CTA tile (4..13, bounded by the variant) */
#define GQ_OPT_PASS_BUDGET 2    /* FMA-per-amplitude budget of one pass (0 = auto) */
#define GQ_OPT_LOW_QUBITS 3     /* lowest qubits always in a tile (coalescing)      */
#define GQ_OPT_TIMING 4         /* 1: record CUDA events around every apply        */
#define GQ_OPT_KERNEL_VARIANT 5 /* tile-pass launch shape (0..3); sets the tile size */
#define GQ_OPT_ADJOINT_SEGMENTS 6 /* adjoint: forward checkpoints (0 = automatic, 1 = none) */
#define GQ_OPT_USE_GRAPH 7      /* batches: capture launches in a CUDA graph (default 1) */
#define GQ_OPT_FUSE_DENSE 8     /* 1: fold register-local gate runs into dense blocks (default 0) */
/* Specialised pass kernels (NVRTC, compiled on background threads and cached
 * per process by pass structure): 0 off, 1 use when compiled and run the
 * interpreted kernel until then (default), 2 wait for the compilation. */
#define GQ_OPT_JIT 9
#define GQ_OPT_JIT_MIN_QUBITS 10 /* smallest state (physical qubits) that uses them (default 20) */
#define GQ_OPT_JIT_MIN_BLOCKS 11 /* their CTAs per SM (register bound); 0 = the launch shape's */
/* 1: persistent CTAs (SMs x CTAs per SM), one tile buffer each, refilled with
 * the next tile (cp.async) while the current tile's last phase computes and
 * stores; 0: one CTA per tile (default). */
#define GQ_OPT_JIT_PERSISTENT 12
/* Density matrices: channels that only mix populations and scale coherences
 * (depolarizing, amplitude and phase damping) run as permutations, a
 * diagonal and the population map (default 0); 1 folds every channel into a
 * dense superoperator with the gate before it. */
#define GQ_OPT_DM_DENSE_CHANNELS 13
/* Evolve and Run from the reset state (and the adjoint's forward sweep):
 * every amplitude whose index has a 1 on a qubit that no earlier pass acted
 * on with a non-diagonal op is exactly zero, and a pass maps an all-zero tile
 * to an all-zero tile, so each pass launches only the CTAs whose outer
 * qubits lie in that support; the skipped tiles keep the zeros of the reset
 * (default 1; results are identical either way; Apply never skips). */
#define GQ_OPT_ZERO_TILES 14
int gq_sv_set_option(gq_sv* sv, int key, int64_t value);

/* ---- density matrix: replaces densitymatrix.New/Sim ---------------------- */
typedef struct gq_dm gq_dm;

/* New(n): rho = |0><0|, num_qubits in [1, 15] (goqu: [1, 14],
 * sim/densitymatrix/sim.go:32-40). */
int gq_dm_create(int num_qubits, gq_dm** out);
int gq_dm_destroy(gq_dm* dm);
int gq_dm_reset(gq_dm* dm);
/* Apply gates (rho <- U rho U^dagger) and Kraus channels (GQ_OP_CHANNEL,
 * rho <- sum_k E_k rho E_k^dagger) in order (sim/densitymatrix/sim.go:87-191,
 * 220-255). GQ_OP_RESET is the trace-preserving reset of sim.go:195-217.     */
int gq_dm_apply(gq_dm* dm, const gq_op* ops, size_t n_ops);
int gq_dm_evolve(gq_dm* dm, const gq_op* ops, size_t n_ops);
/* Copy rho (dim*dim interleaved complex doubles) to host. */
int gq_dm_get(gq_dm* dm, double* host_out, size_t bytes);
int gq_dm_set(gq_dm* dm, const double* host_in, size_t bytes);
/* diag(rho), negatives clamped to 0 (diagonalProbs, measure.go:11-20). */
int gq_dm_diagonal_probs(gq_dm* dm, double* host_out, size_t n);
/* sum_t coeff_t Tr(rho P_t) (pauli.ExpectSumDM, sim/pauli/expect_dm.go:9-30). */
int gq_dm_expect_pauli_sum(gq_dm* dm, const gq_pauli_term* terms, size_t n_terms,
                           double* out_re, double* out_im);
int gq_dm_trace(gq_dm* dm, double* out_re, double* out_im);
/* |Tr(rho^2)| (Purity, sim/densitymatrix/sim.go:265-276). */
int gq_dm_purity(gq_dm* dm, double* out);
/* |<psi|rho|psi>| for a host pure state (Fidelity, sim.go:280-291). */
int gq_dm_fidelity(gq_dm* dm, const double* psi, size_t n, double* out);
/* Readout-error mixing of `probs` in place, qubit by qubit with (p01, p10)
 * pairs (ApplyReadoutError, measure.go:29-71); p01[q] < 0 skips qubit q.     */
int gq_dm_sample(gq_dm* dm, const double* p01, const double* p10, const double* uniforms,
                 size_t shots, uint64_t* idx_out);
/* The same sampling with the histogram built on the device (densitymatrix
 * Run's counts, sim/densitymatrix/sim.go:48-66): distinct outcomes in
 * increasing order and their counts, as gq_sv_sample_counts. */
int gq_dm_sample_counts(gq_dm* dm, const double* p01, const double* p10, const double* uniforms,
                        size_t shots, uint64_t* outcomes_out, uint64_t* counts_out, size_t* n_distinct);
/* Dynamic circuits: measureQubitDM (sim/densitymatrix/dynamic.go:198-255).
 * P(0) = sum of rho[i,i] over i with the qubit's bit clear; the collapse keeps
 * rho[r,c] with both bits equal to the outcome, divided by its probability
 * (1 - p0 for outcome 1), unless that probability is below 1e-15. */
int gq_dm_prob0(gq_dm* dm, int qubit, double* p0);
int gq_dm_collapse(gq_dm* dm, int qubit, int outcome, double p0);
int gq_dm_measure(gq_dm* dm, int qubit, double u, int* outcome);
int gq_dm_copy_state(gq_dm* dst, const gq_dm* src);
int gq_dm_stats(const gq_dm* dm, gq_stats* out);
int gq_dm_set_option(gq_dm* dm, int key, int64_t value);

/* ---- batches of independent circuits ------------------------------------
 * Replaces the per-point loop of sweep.RunSim (sweep/run.go:27-97) and the
 * cost / gradient evaluations of algorithm/qaoa (qaoa.go:100-126) and
 * algorithm/vqe: every item is a circuit applied to |0...0> with a Pauli sum;
 * gq_batch_run returns Re <psi|H|psi> per item and, with want_gradients, the
 * adjoint gradient of each item (n_params entries per item, concatenated in
 * item order). Items run as batched launches in up to 8 segments of about
 * equal work: the host's threads analyse and schedule a segment while the
 * device runs the one before, and each segment's launches are a captured CUDA
 * graph, replayed while its structure (not its angles) stays the same.
 * Stats: last_ms covers the whole call, pass_ms the span of the launches,
 * host_ms the host time before the first launch.                            */
typedef struct gq_batch gq_batch;
typedef struct gq_batch_item {
    int32_t num_qubits;
    int32_t reserved;
    const gq_op* ops;
    size_t n_ops;
    const gq_pauli_term* terms;
    size_t n_terms;
    size_t n_params;
} gq_batch_item;

int gq_batch_create(int precision, gq_batch** out);
int gq_batch_destroy(gq_batch* b);
int gq_batch_run(gq_batch* b, const gq_batch_item* items, size_t n_items, int want_gradients,
                 double* energies_out, double* grads_out);
int gq_batch_set_option(gq_batch* b, int key, int64_t value);
int gq_batch_stats(const gq_batch* b, gq_stats* out);

/* ---- MaxCut QAOA batches: the evaluations of algorithm/qaoa -----------------
 * Energies and gradients of many QAOA circuits of goqu's qaoa.Run form
 * (qaoa.go:68-93, 164-196) for MaxCut Hamiltonians (maxcut.go:13-35): H on
 * every qubit, then per layer k an RZZ(gamma_k) per edge and RX(2 beta_k) on
 * every qubit; energy <H> with H = sum_e (-1/2 + 1/2 Z_i Z_j). The same
 * circuits as gq_batch_run items built from those gates, evaluated by a
 * dedicated path: a per-circuit table of cut counts makes each cost layer a
 * lookup, circuits of up to 12 qubits run whole in one CTA's shared memory,
 * larger ones in batched tile passes. grads_out receives 2p values per item,
 * [gamma_0, beta_0, gamma_1, beta_1, ...] (the circuit's FreeParameters
 * order), items concatenated. complex64 only (GQ_EUNSUPPORTED otherwise);
 * 4 <= num_qubits <= 26, 1 <= n_edges <= 255, 1 <= p <= 64. */
typedef struct gq_qaoa_item {
    int32_t num_qubits;
    int32_t p;
    const int32_t* edges; /* n_edges pairs (i, j), 0 <= i != j < num_qubits */
    size_t n_edges;
    const double* gammas; /* p values */
    const double* betas;  /* p values */
} gq_qaoa_item;

int gq_qaoa_maxcut_batch(int precision, const gq_qaoa_item* items, size_t n_items, int want_gradients,
                         double* energies_out, double* grads_out);

/* ---- sweeps: replaces sweep.RunSim / RunDensitySim (sweep/run.go:27-171) ----
 * Every point is the same circuit bound to different values: `num_qubits`
 * qubits from |0...0> (rho = |0><0| for density matrices), the point's op
 * stream applied (density matrices: gates and their channels, GQ_OP_CHANNEL,
 * as for gq_dm_apply), then `shots` samples drawn with the point's uniforms
 * (Run, sim/statevector/sim.go:40-58 and sim/densitymatrix/sim.go:48-66) and
 * returned as (outcome, count) pairs in increasing outcome order. Point i's
 * pairs are written at offset i * S of outcomes_out / counts_out, with
 * S = max(1, min(shots, 2^num_qubits)); n_distinct_out[i] receives their
 * number and status_out[i] the point's status (goqu's PointResult.Err), so a
 * failing point does not stop the others; gq_last_error() then describes the
 * first failing point. Points run on a pool of workers, each with its own
 * device state and stream (at most 8, and as many as device memory holds).
 * The density variant applies readout error with p01 / p10 (num_qubits
 * entries each, a negative p01[q] skips qubit q; both may be NULL). */
typedef struct gq_sweep_point {
    const gq_op* ops;
    size_t n_ops;
    const double* uniforms; /* `shots` values in [0, 1) */
} gq_sweep_point;

int gq_sweep_run(int num_qubits, int precision, const gq_sweep_point* points, size_t n_points, size_t shots,
                 uint64_t* outcomes_out, uint64_t* counts_out, size_t* n_distinct_out, int32_t* status_out);
int gq_sweep_run_density(int num_qubits, const double* p01, const double* p10, const gq_sweep_point* points,
                         size_t n_points, size_t shots, uint64_t* outcomes_out, uint64_t* counts_out,
                         size_t* n_distinct_out, int32_t* status_out);

/* ---- circuit equivalence: replaces transpile/verify (verify.go:16-155) ------
 * gq_unitary: the unitary of a circuit on num_qubits (<= 16) qubits, every
 * column evolved at once (goqu builds it from 2^n runs that prepend X gates,
 * verify.go:45-90). host_out receives 4^n complex128 values, column by
 * column: entry col * 2^n + row = U[row][col] (goqu's unitary[col][row]).
 * gq_equivalent: verify.Equivalent, the unitaries equal up to a global phase
 * taken from the first entry of B's column 0 whose modulus exceeds tol, every
 * entry then within tol (unitariesClose); num_qubits <= 15 (goqu: 10).
 * gq_equivalent_on_zero: verify.EquivalentOnZero, the states from |0...0>
 * compared the same way, the phase's modulus within tol of 1
 * (stateVectorsClose); num_qubits <= 30 (goqu: 14). *equal_out is 1 or 0. */
int gq_unitary(int num_qubits, const gq_op* ops, size_t n_ops, double* host_out, size_t bytes);
int gq_equivalent(int num_qubits, const gq_op* a, size_t n_a, const gq_op* b, size_t n_b, double tol, int* equal_out);
int gq_equivalent_on_zero(int num_qubits, const gq_op* a, size_t n_a, const gq_op* b, size_t n_b, double tol,
                          int* equal_out);

/* ---- expectation without allocation ---------------------------------------
 * No counterpart in the reference: an extra entry point for callers that own
 * their device memory and must not have the library call cudaMalloc or
 * cudaFree (an application allocator that has reserved the GPU's memory, a
 * latency-critical loop that cannot take the synchronisation cudaFree may
 * imply). Computes sum_t coeff_t <psi|P_t|psi> of a state the caller
 * allocated (2^num_qubits interleaved complex128 or complex64 amplitudes at
 * device_state) on `stream` (a cudaStream_t, NULL for the default stream).
 * Its scratch is a 256 KiB array compiled into the library, so at most
 * GQ_NOALLOC_MAX_TERMS terms are accepted (larger sums return GQ_EINVAL).
 * The first call on a device looks up the array's device address (again after
 * the device's context changes). The call is synchronous: it copies the term
 * tables from host memory and waits for the result, so it cannot be captured
 * into a CUDA graph, and a capturing `stream` is refused with GQ_EINVAL, as is
 * a device_state that is not device (or managed) memory of the current
 * device. Calls share the array: calls that overlap on the GPU race and must
 * be serialised by the caller.                                               */
#define GQ_NOALLOC_MAX_TERMS 2048
int gq_expect_pauli_sum_noalloc(const void* device_state, int num_qubits, int precision,
                                const gq_pauli_term* terms, size_t n_terms, void* stream,
                                double* out_re, double* out_im);

#ifdef __cplusplus
}
#endif

#endif /* GQB200_H */

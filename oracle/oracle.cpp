// CPU oracle: an FP64 restatement of goqu's pure-Go simulator kernels.
//
// THIS IS TEST INFRASTRUCTURE. Only tests/, __graft_entry__.smoke() and
// bench.py's CPU-baseline leg may load it, and only as the checker or as the
// timed CPU baseline. The product path (goqu_b200, libgqb200.so) never calls it.
//
// Every routine follows the cited Go source of github.com/splch/goqu, loop for
// loop, so that the arithmetic (operation order, no fused multiply-add: built
// with -ffp-contract=off, like Go on amd64) is that of the reference:
//   sim/statevector/sim.go, kernel2q.go, kernel3q.go, kernel_controlled.go
//   sim/pauli/expect_sv.go, expect_dm.go
//   sim/densitymatrix/sim.go, kernel1q.go, kernel2q.go, measure.go
// The op stream is the same gq_op array the GPU engine consumes (gqb200.h), so
// both sides see identical matrices. "threads" plays GOMAXPROCS: 0 runs the
// serial kernels, >0 runs the goroutine-parallel variants (same per-element
// arithmetic; only the Pauli expectation's partial-sum grouping differs).
//
// Deliberate difference: gates on more than two qubits in the density-matrix
// path are applied as U rho U^dagger directly instead of through goqu's
// H/T/CNOT decompositions (sim/densitymatrix/sim.go:321-506); both are exact
// up to rounding (~1e-15).
#include <cmath>
#include <cstdint>
#include <cstring>
#include <functional>
#include <thread>
#include <vector>

#include "../include/gqb200.h"

namespace {

struct cd {
    double re, im;
};
// Go complex128 arithmetic (cmd/compile: (a+bi)(c+di) = (ac-bd) + (ad+bc)i).
inline cd mul(cd a, cd b) { return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
inline cd add(cd a, cd b) { return {a.re + b.re, a.im + b.im}; }
inline cd neg(cd a) { return {-a.re, -a.im}; }
inline cd conjc(cd a) { return {a.re, -a.im}; }
const cd kI = {0.0, 1.0};
const cd kMinusI = {0.0, -1.0};

inline cd* C(double* p) { return reinterpret_cast<cd*>(p); }
inline const cd* C(const double* p) { return reinterpret_cast<const cd*>(p); }

// optimalWorkers (sim/statevector/sim.go:327-341; same rule in sim/pauli).
int optimal_workers(int nq, int gomaxprocs) {
    if (nq <= 16) return 1;
    long long n_amps = 1LL << nq;
    long long by_work = n_amps / 8192;
    if (by_work < 1) by_work = 1;
    if (gomaxprocs < by_work) return gomaxprocs;
    return (int)by_work;
}

// Runs body(start, end) over [0, n) in `workers` contiguous chunks, the last
// chunk taking the remainder (the split used by every *Parallel kernel).
void parallel_chunks(long long n, int workers, const std::function<void(long long, long long)>& body) {
    if (workers <= 1 || n <= 1) {
        body(0, n);
        return;
    }
    if (workers > n) workers = (int)n;
    long long per = n / workers;
    std::vector<std::thread> ts;
    for (int w = 0; w < workers; ++w) {
        long long s = w * per, e = (w == workers - 1) ? n : s + per;
        ts.emplace_back(body, s, e);
    }
    for (auto& t : ts) t.join();
}

struct SV {
    int nq;
    cd* st;
    long long n;
    int threads;
    bool par() const { return threads > 0 && nq >= 17; }
    int workers() const { return optimal_workers(nq, threads); }
};

// applyGate1 / applyGate1Parallel (sim/statevector/sim.go:211-272).
void gate1(SV& s, int q, const cd* m) {
    long long half = 1LL << q, block = half << 1, nblocks = s.n / block;
    auto body = [&](long long b_s, long long b_e) {
        for (long long b = b_s; b < b_e; ++b) {
            long long b0 = b * block;
            for (long long off = 0; off < half; ++off) {
                long long i0 = b0 + off, i1 = i0 + half;
                cd a0 = s.st[i0], a1 = s.st[i1];
                s.st[i0] = add(mul(m[0], a0), mul(m[1], a1));
                s.st[i1] = add(mul(m[2], a0), mul(m[3], a1));
            }
        }
    };
    if (s.par()) {
        int w = s.workers();
        if (nblocks < w) w = (int)nblocks;
        parallel_chunks(nblocks, w, body);
    } else {
        body(0, nblocks);
    }
}

// 2q block-stride iteration (blockStride2, kernel2q.go:128-136) over the
// canonical offsets (both gate bits zero). The parallel twins split the outer
// hi-blocks across workers (runParallel2q, kernel2q.go:365-409).
template <class F>
void for2(SV& s, int q0, int q1, F f) {
    int lo = q0 < q1 ? q0 : q1, hi = q0 < q1 ? q1 : q0;
    long long lo_m = 1LL << lo, hi_m = 1LL << hi;
    long long mask0 = 1LL << q0, mask1 = 1LL << q1;
    long long n_outer = s.n / (hi_m << 1);
    auto body = [&](long long o_s, long long o_e) {
        for (long long o = o_s; o < o_e; ++o) {
            long long hi0 = o * (hi_m << 1);
            for (long long lo0 = hi0; lo0 < hi0 + hi_m; lo0 += lo_m << 1)
                for (long long off = lo0; off < lo0 + lo_m; ++off) f(off, mask0, mask1);
        }
    };
    if (s.par()) {
        int w = s.workers();
        if (n_outer < w) w = (int)n_outer;
        parallel_chunks(n_outer, w, body);
    } else {
        body(0, n_outer);
    }
}

template <class F>
void for3(SV& s, int q0, int q1, int q2, F f) {
    int a = q0, b = q1, c = q2;  // sortThree (kernel3q.go:50-62)
    if (a > b) std::swap(a, b);
    if (b > c) std::swap(b, c);
    if (a > b) std::swap(a, b);
    long long lo_m = 1LL << a, mid_m = 1LL << b, hi_m = 1LL << c;
    long long m0 = 1LL << q0, m1 = 1LL << q1, m2 = 1LL << q2;
    long long n_outer = s.n / (hi_m << 1);
    auto body = [&](long long o_s, long long o_e) {
        for (long long o = o_s; o < o_e; ++o) {
            long long hi0 = o * (hi_m << 1);
            for (long long mid0 = hi0; mid0 < hi0 + hi_m; mid0 += mid_m << 1)
                for (long long lo0 = mid0; lo0 < mid0 + mid_m; lo0 += lo_m << 1)
                    for (long long off = lo0; off < lo0 + lo_m; ++off) f(off, m0, m1, m2);
        }
    };
    if (s.par()) {
        int w = s.workers();
        if (n_outer < w) w = (int)n_outer;
        parallel_chunks(n_outer, w, body);
    } else {
        body(0, n_outer);
    }
}

// dispatchGate2 (kernel2q.go:24-114) with the serial bodies of :152-346.
void gate2(SV& s, int kind, int q0, int q1, const cd* m) {
    cd* st = s.st;
    switch (kind) {
        case GQ_OP_CNOT:
            for2(s, q0, q1, [&](long long o, long long m0, long long m1) {
                long long i10 = o | m0, i11 = o | m0 | m1;
                std::swap(st[i10], st[i11]);
            });
            return;
        case GQ_OP_CZ:
            for2(s, q0, q1, [&](long long o, long long m0, long long m1) {
                long long i11 = o | m0 | m1;
                st[i11] = neg(st[i11]);
            });
            return;
        case GQ_OP_SWAP:
            for2(s, q0, q1, [&](long long o, long long m0, long long m1) {
                std::swap(st[o | m1], st[o | m0]);
            });
            return;
        case GQ_OP_CY:
            for2(s, q0, q1, [&](long long o, long long m0, long long m1) {
                long long i10 = o | m0, i11 = o | m0 | m1;
                cd a2 = st[i10], a3 = st[i11];
                st[i10] = mul(kMinusI, a3);
                st[i11] = mul(kI, a2);
            });
            return;
        case GQ_OP_ISWAP:
            for2(s, q0, q1, [&](long long o, long long m0, long long m1) {
                long long i01 = o | m1, i10 = o | m0;
                cd a1 = st[i01], a2 = st[i10];
                st[i01] = mul(kI, a2);
                st[i10] = mul(kI, a1);
            });
            return;
        case GQ_OP_SYCAMORE: {
            cd d11 = m[15];
            for2(s, q0, q1, [&](long long o, long long m0, long long m1) {
                long long i01 = o | m1, i10 = o | m0, i11 = o | m0 | m1;
                cd a1 = st[i01], a2 = st[i10];
                st[i01] = mul(kMinusI, a2);
                st[i10] = mul(kMinusI, a1);
                st[i11] = mul(st[i11], d11);
            });
            return;
        }
        case GQ_OP_CTRL_DIAG_2Q: {
            cd d2 = m[10], d3 = m[15];
            for2(s, q0, q1, [&](long long o, long long m0, long long m1) {
                long long i10 = o | m0, i11 = o | m0 | m1;
                st[i10] = mul(st[i10], d2);
                st[i11] = mul(st[i11], d3);
            });
            return;
        }
        case GQ_OP_DIAG_2Q: {
            cd d0 = m[0], d1 = m[5], d2 = m[10], d3 = m[15];
            for2(s, q0, q1, [&](long long o, long long m0, long long m1) {
                st[o] = mul(st[o], d0);
                st[o | m1] = mul(st[o | m1], d1);
                st[o | m0] = mul(st[o | m0], d2);
                st[o | m0 | m1] = mul(st[o | m0 | m1], d3);
            });
            return;
        }
        case GQ_OP_CTRL_U_2Q: {
            cd u00 = m[10], u01 = m[11], u10 = m[14], u11 = m[15];
            for2(s, q0, q1, [&](long long o, long long m0, long long m1) {
                long long i10 = o | m0, i11 = o | m0 | m1;
                cd a2 = st[i10], a3 = st[i11];
                st[i10] = add(mul(u00, a2), mul(u01, a3));
                st[i11] = add(mul(u10, a2), mul(u11, a3));
            });
            return;
        }
        default:  // kernel2qGeneric (kernel2q.go:284-304)
            for2(s, q0, q1, [&](long long o, long long m0, long long m1) {
                long long i00 = o, i01 = o | m1, i10 = o | m0, i11 = o | m0 | m1;
                cd a0 = st[i00], a1 = st[i01], a2 = st[i10], a3 = st[i11];
                st[i00] = add(add(add(mul(m[0], a0), mul(m[1], a1)), mul(m[2], a2)), mul(m[3], a3));
                st[i01] = add(add(add(mul(m[4], a0), mul(m[5], a1)), mul(m[6], a2)), mul(m[7], a3));
                st[i10] = add(add(add(mul(m[8], a0), mul(m[9], a1)), mul(m[10], a2)), mul(m[11], a3));
                st[i11] = add(add(add(mul(m[12], a0), mul(m[13], a1)), mul(m[14], a2)), mul(m[15], a3));
            });
            return;
    }
}

// dispatchGate3 (kernel3q.go:10-47) with the bodies of :76-180.
void gate3(SV& s, int kind, int q0, int q1, int q2, const cd* m) {
    cd* st = s.st;
    switch (kind) {
        case GQ_OP_CCX:
            for3(s, q0, q1, q2, [&](long long o, long long m0, long long m1, long long m2) {
                std::swap(st[o | m0 | m1], st[o | m0 | m1 | m2]);
            });
            return;
        case GQ_OP_CSWAP:
            for3(s, q0, q1, q2, [&](long long o, long long m0, long long m1, long long m2) {
                std::swap(st[o | m0 | m2], st[o | m0 | m1]);
            });
            return;
        case GQ_OP_CCZ:
            for3(s, q0, q1, q2, [&](long long o, long long m0, long long m1, long long m2) {
                long long i = o | m0 | m1 | m2;
                st[i] = neg(st[i]);
            });
            return;
        default:
            for3(s, q0, q1, q2, [&](long long o, long long m0, long long m1, long long m2) {
                long long idx[8];
                cd a[8];
                for (int r = 0; r < 8; ++r) {
                    long long i = o;
                    if (r & 4) i |= m0;
                    if (r & 2) i |= m1;
                    if (r & 1) i |= m2;
                    idx[r] = i;
                }
                for (int j = 0; j < 8; ++j) a[j] = st[idx[j]];
                for (int r = 0; r < 8; ++r) {
                    cd sum = {0.0, 0.0};
                    for (int c = 0; c < 8; ++c) sum = add(sum, mul(m[r * 8 + c], a[c]));
                    st[idx[r]] = sum;
                }
            });
            return;
    }
}

// applyControlledGate1/2(+Parallel) and applyControlledGateN
// (kernel_controlled.go:59-292): a full scan with mask tests.
void controlled(SV& s, const gq_op& op) {
    int nc = op.num_controls, nt = op.num_qubits - nc;
    long long cmask = 0;
    for (int i = 0; i < nc; ++i) cmask |= 1LL << op.qubits[i];
    const cd* m = C(op.matrix);
    cd* st = s.st;
    if (nt == 1 || nt == 2) {
        long long t0 = 1LL << op.qubits[nc], t1 = nt == 2 ? 1LL << op.qubits[nc + 1] : 0;
        long long tmask = t0 | t1;
        auto body = [&](long long b, long long e) {
            for (long long i = b; i < e; ++i) {
                if ((i & cmask) != cmask) continue;
                if ((i & tmask) != 0) continue;
                if (nt == 1) {
                    long long i0 = i, i1 = i | t0;
                    cd a0 = st[i0], a1 = st[i1];
                    st[i0] = add(mul(m[0], a0), mul(m[1], a1));
                    st[i1] = add(mul(m[2], a0), mul(m[3], a1));
                } else {
                    long long idx[4] = {i, i | t1, i | t0, i | t0 | t1};
                    cd a[4];
                    for (int j = 0; j < 4; ++j) a[j] = st[idx[j]];
                    for (int r = 0; r < 4; ++r) {
                        cd sum = {0.0, 0.0};
                        for (int c = 0; c < 4; ++c) sum = add(sum, mul(m[r * 4 + c], a[c]));
                        st[idx[r]] = sum;
                    }
                }
            }
        };
        if (s.par()) {
            int w = s.workers();
            long long chunk = s.n / w;
            if (chunk < 1) w = 1;
            parallel_chunks(s.n, w, body);
        } else {
            body(0, s.n);
        }
        return;
    }
    // Generic: the full controlled matrix (controlled.go:84-110) on all qubits.
    int tot = op.num_qubits;
    long long dim = 1LL << tot, inner = 1LL << nt, start = dim - inner;
    std::vector<cd> full(dim * dim, cd{0.0, 0.0});
    for (long long i = 0; i < start; ++i) full[i * dim + i] = {1.0, 0.0};
    for (long long r = 0; r < inner; ++r)
        for (long long c = 0; c < inner; ++c) full[(start + r) * dim + (start + c)] = m[r * inner + c];
    long long all = 0;
    std::vector<long long> masks(tot);
    for (int i = 0; i < tot; ++i) {
        masks[i] = 1LL << op.qubits[i];
        all |= masks[i];
    }
    std::vector<long long> idx(dim);
    std::vector<cd> a(dim);
    for (long long base = 0; base < s.n; ++base) {
        if (base & all) continue;
        for (long long r = 0; r < dim; ++r) {
            long long i = base;
            for (int bit = 0; bit < tot; ++bit)
                if (r & (1LL << (tot - 1 - bit))) i |= masks[bit];
            idx[r] = i;
        }
        for (long long j = 0; j < dim; ++j) a[j] = st[idx[j]];
        for (long long r = 0; r < dim; ++r) {
            cd sum = {0.0, 0.0};
            for (long long c = 0; c < dim; ++c) sum = add(sum, mul(full[r * dim + c], a[c]));
            st[idx[r]] = sum;
        }
    }
}

// resetQubit (sim/statevector/sim.go:168-186).
void reset_qubit(SV& s, int q) {
    long long half = 1LL << q, block = half << 1;
    for (long long b0 = 0; b0 < s.n; b0 += block)
        for (long long off = 0; off < half; ++off) {
            long long i0 = b0 + off, i1 = i0 + half;
            cd a0 = s.st[i0], a1 = s.st[i1];
            double norm = std::sqrt(a0.re * a0.re + a0.im * a0.im + a1.re * a1.re + a1.im * a1.im);
            s.st[i0] = norm > 1e-15 ? cd{norm, 0.0} : cd{0.0, 0.0};
            s.st[i1] = {0.0, 0.0};
        }
}

int popcount_parity(uint64_t v) { return __builtin_popcountll(v) & 1; }

// iPow (sim/pauli/pauli.go:205-217).
cd ipow(int k) {
    switch (k % 4) {
        case 0: return {1.0, 0.0};
        case 1: return {0.0, 1.0};
        case 2: return {-1.0, 0.0};
        default: return {0.0, -1.0};
    }
}

// ---- density matrix ---------------------------------------------------------
struct DM {
    int nq;
    long long dim;
    cd* rho;
    int threads;
    bool par() const { return threads > 0 && nq >= 9; }  // parallelThreshold (sim.go:21)
    int workers() const {
        // densitymatrix optimalWorkers (kernel1q.go:165-179).
        long long by_work = (dim * dim) / 8192;
        if (by_work < 1) by_work = 1;
        return threads < by_work ? threads : (int)by_work;
    }
};

// gate1Rows / gate1Cols (kernel1q.go:21-68). Rows parallelise over row
// blocks, columns over rows.
void dm_gate1(DM& s, int q, const cd* m) {
    long long dim = s.dim, half = 1LL << q, block = half << 1;
    cd* rho = s.rho;
    auto rows = [&](long long b_s, long long b_e) {
        for (long long b = b_s; b < b_e; ++b) {
            long long b0 = b * block;
            for (long long off = 0; off < half; ++off) {
                long long base0 = (b0 + off) * dim, base1 = (b0 + off + half) * dim;
                for (long long c = 0; c < dim; ++c) {
                    cd a0 = rho[base0 + c], a1 = rho[base1 + c];
                    rho[base0 + c] = add(mul(m[0], a0), mul(m[1], a1));
                    rho[base1 + c] = add(mul(m[2], a0), mul(m[3], a1));
                }
            }
        }
    };
    cd u00 = conjc(m[0]), u01 = conjc(m[1]), u10 = conjc(m[2]), u11 = conjc(m[3]);
    auto cols = [&](long long r_s, long long r_e) {
        for (long long r = r_s; r < r_e; ++r) {
            long long base = r * dim;
            for (long long b0 = 0; b0 < dim; b0 += block)
                for (long long off = 0; off < half; ++off) {
                    long long c0 = b0 + off, c1 = c0 + half;
                    cd a0 = rho[base + c0], a1 = rho[base + c1];
                    rho[base + c0] = add(mul(u00, a0), mul(u01, a1));
                    rho[base + c1] = add(mul(u10, a0), mul(u11, a1));
                }
        }
    };
    long long nblocks = dim / block;
    if (s.par()) {
        int w = s.workers();
        parallel_chunks(nblocks, w > nblocks ? (int)nblocks : w, rows);
        parallel_chunks(dim, w, cols);
    } else {
        rows(0, nblocks);
        cols(0, dim);
    }
}

// gate2Rows / gate2Cols (kernel2q.go:19-96).
void dm_gate2(DM& s, int q0, int q1, const cd* m) {
    long long dim = s.dim;
    long long mask0 = 1LL << q0, mask1 = 1LL << q1;
    int lo = q0 < q1 ? q0 : q1, hi = q0 < q1 ? q1 : q0;
    long long lo_m = 1LL << lo, hi_m = 1LL << hi;
    cd* rho = s.rho;
    long long n_outer = dim / (hi_m << 1);
    auto rows = [&](long long o_s, long long o_e) {
        for (long long o = o_s; o < o_e; ++o) {
            long long hi0 = o * (hi_m << 1);
            for (long long lo0 = hi0; lo0 < hi0 + hi_m; lo0 += lo_m << 1)
                for (long long off = lo0; off < lo0 + lo_m; ++off) {
                    long long b00 = off * dim, b01 = (off | mask1) * dim, b10 = (off | mask0) * dim,
                              b11 = (off | mask0 | mask1) * dim;
                    for (long long c = 0; c < dim; ++c) {
                        cd a0 = rho[b00 + c], a1 = rho[b01 + c], a2 = rho[b10 + c], a3 = rho[b11 + c];
                        rho[b00 + c] = add(add(add(mul(m[0], a0), mul(m[1], a1)), mul(m[2], a2)), mul(m[3], a3));
                        rho[b01 + c] = add(add(add(mul(m[4], a0), mul(m[5], a1)), mul(m[6], a2)), mul(m[7], a3));
                        rho[b10 + c] = add(add(add(mul(m[8], a0), mul(m[9], a1)), mul(m[10], a2)), mul(m[11], a3));
                        rho[b11 + c] = add(add(add(mul(m[12], a0), mul(m[13], a1)), mul(m[14], a2)), mul(m[15], a3));
                    }
                }
        }
    };
    cd uc[16];
    for (int i = 0; i < 16; ++i) uc[i] = conjc(m[i]);
    auto cols = [&](long long r_s, long long r_e) {
        for (long long r = r_s; r < r_e; ++r) {
            long long base = r * dim;
            for (long long hi0 = 0; hi0 < dim; hi0 += hi_m << 1)
                for (long long lo0 = hi0; lo0 < hi0 + hi_m; lo0 += lo_m << 1)
                    for (long long off = lo0; off < lo0 + lo_m; ++off) {
                        long long c00 = off, c01 = off | mask1, c10 = off | mask0, c11 = off | mask0 | mask1;
                        cd a0 = rho[base + c00], a1 = rho[base + c01], a2 = rho[base + c10], a3 = rho[base + c11];
                        rho[base + c00] = add(add(add(mul(uc[0], a0), mul(uc[1], a1)), mul(uc[2], a2)), mul(uc[3], a3));
                        rho[base + c01] = add(add(add(mul(uc[4], a0), mul(uc[5], a1)), mul(uc[6], a2)), mul(uc[7], a3));
                        rho[base + c10] = add(add(add(mul(uc[8], a0), mul(uc[9], a1)), mul(uc[10], a2)), mul(uc[11], a3));
                        rho[base + c11] = add(add(add(mul(uc[12], a0), mul(uc[13], a1)), mul(uc[14], a2)), mul(uc[15], a3));
                    }
        }
    };
    if (s.par()) {
        int w = s.workers();
        parallel_chunks(n_outer, w > n_outer ? (int)n_outer : w, rows);
        parallel_chunks(dim, w, cols);
    } else {
        rows(0, n_outer);
        cols(0, dim);
    }
}

// U rho U^dagger for k > 2 qubits: left multiply on the row index, right
// multiply by U^dagger on the column index (the same two-pass scheme).
void dm_gateN(DM& s, const int* qubits, int k, const cd* m) {
    long long dim = s.dim, kd = 1LL << k;
    std::vector<long long> masks(k);
    long long all = 0;
    for (int i = 0; i < k; ++i) {
        masks[i] = 1LL << qubits[i];
        all |= masks[i];
    }
    std::vector<long long> idx(kd);
    std::vector<cd> a(kd);
    cd* rho = s.rho;
    auto local = [&](long long base) {
        for (long long r = 0; r < kd; ++r) {
            long long i = base;
            for (int b = 0; b < k; ++b)
                if (r & (1LL << (k - 1 - b))) i |= masks[b];
            idx[r] = i;
        }
    };
    for (long long base = 0; base < dim; ++base) {  // rows
        if (base & all) continue;
        local(base);
        for (long long c = 0; c < dim; ++c) {
            for (long long j = 0; j < kd; ++j) a[j] = rho[idx[j] * dim + c];
            for (long long r = 0; r < kd; ++r) {
                cd sum = {0.0, 0.0};
                for (long long j = 0; j < kd; ++j) sum = add(sum, mul(m[r * kd + j], a[j]));
                rho[idx[r] * dim + c] = sum;
            }
        }
    }
    for (long long base = 0; base < dim; ++base) {  // columns
        if (base & all) continue;
        local(base);
        for (long long r0 = 0; r0 < dim; ++r0) {
            for (long long j = 0; j < kd; ++j) a[j] = rho[r0 * dim + idx[j]];
            for (long long r = 0; r < kd; ++r) {
                cd sum = {0.0, 0.0};
                for (long long j = 0; j < kd; ++j) sum = add(sum, mul(conjc(m[r * kd + j]), a[j]));
                rho[r0 * dim + idx[r]] = sum;
            }
        }
    }
}

void dm_gate(DM& s, const int* qubits, int k, const cd* m) {
    if (k == 1)
        dm_gate1(s, qubits[0], m);
    else if (k == 2)
        dm_gate2(s, qubits[0], qubits[1], m);
    else
        dm_gateN(s, qubits, k, m);
}

// Full matrix of a GQ_OP_CONTROLLED op (controlled.go:84-110).
std::vector<cd> controlled_full(const gq_op& op) {
    int tot = op.num_qubits, nt = op.num_qubits - op.num_controls;
    long long dim = 1LL << tot, inner = 1LL << nt, start = dim - inner;
    std::vector<cd> full(dim * dim, cd{0.0, 0.0});
    for (long long i = 0; i < start; ++i) full[i * dim + i] = {1.0, 0.0};
    const cd* m = C(op.matrix);
    for (long long r = 0; r < inner; ++r)
        for (long long c = 0; c < inner; ++c) full[(start + r) * dim + (start + c)] = m[r * inner + c];
    return full;
}

// resetQubit (sim/densitymatrix/sim.go:195-217).
void dm_reset(DM& s, int q) {
    long long dim = s.dim, mask = 1LL << q;
    cd* rho = s.rho;
    for (long long r = 0; r < dim; ++r) {
        if ((r >> q) & 1) continue;
        for (long long c = 0; c < dim; ++c) {
            if ((c >> q) & 1) continue;
            rho[r * dim + c] = add(rho[r * dim + c], rho[(r | mask) * dim + (c | mask)]);
        }
    }
    for (long long r = 0; r < dim; ++r)
        for (long long c = 0; c < dim; ++c)
            if (((r >> q) & 1) || ((c >> q) & 1)) rho[r * dim + c] = {0.0, 0.0};
}

// applyChannel (sim/densitymatrix/sim.go:220-255).
void dm_channel(DM& s, const gq_op& op) {
    int k = op.num_qubits;
    long long kd = 1LL << k;
    const cd* kraus = C(op.matrix);
    if (op.num_kraus == 1) {
        dm_gate(s, op.qubits, k, kraus);
        return;
    }
    long long n = s.dim * s.dim;
    // goqu runs the restore, accumulate and final copy loops serially; in the
    // threaded mode they are split across workers. Each element's additions
    // are the same in the same order, so the result is bit-identical.
    const int w = s.par() ? s.workers() : 1;
    std::vector<cd> temp(n), saved(n);
    parallel_chunks(n, w, [&](long long a, long long b) {
        std::memcpy(saved.data() + a, s.rho + a, (b - a) * sizeof(cd));
        for (long long i = a; i < b; ++i) temp[i] = cd{0.0, 0.0};
    });
    for (int e = 0; e < op.num_kraus; ++e) {
        parallel_chunks(n, w, [&](long long a, long long b) {
            std::memcpy(s.rho + a, saved.data() + a, (b - a) * sizeof(cd));
        });
        dm_gate(s, op.qubits, k, kraus + e * kd * kd);
        parallel_chunks(n, w, [&](long long a, long long b) {
            for (long long i = a; i < b; ++i) temp[i] = add(temp[i], s.rho[i]);
        });
    }
    parallel_chunks(n, w, [&](long long a, long long b) {
        std::memcpy(s.rho + a, temp.data() + a, (b - a) * sizeof(cd));
    });
}

}  // namespace

extern "C" {

// Apply (sim/statevector/sim.go:92-157) over an op stream; returns GQ_OK or
// GQ_EUNSUPPORTED for a >= 4-qubit op that is not GQ_OP_CONTROLLED.
int or_sv_apply(int nq, double* state, const gq_op* ops, size_t n_ops, int threads) {
    SV s{nq, C(state), 1LL << nq, threads};
    for (size_t i = 0; i < n_ops; ++i) {
        const gq_op& op = ops[i];
        if (op.kind == GQ_OP_BARRIER) continue;
        if (op.kind == GQ_OP_RESET) {
            reset_qubit(s, op.qubits[0]);
            continue;
        }
        if (op.kind == GQ_OP_CONTROLLED && op.num_qubits >= 4) {
            controlled(s, op);
            continue;
        }
        const cd* m = C(op.matrix);
        switch (op.num_qubits) {
            case 1: gate1(s, op.qubits[0], m); break;
            case 2: gate2(s, op.kind, op.qubits[0], op.qubits[1], m); break;
            case 3: gate3(s, op.kind, op.qubits[0], op.qubits[1], op.qubits[2], m); break;
            default: return GQ_EUNSUPPORTED;
        }
    }
    return GQ_OK;
}

// probabilities (sim/statevector/sim.go:274-280).
void or_sv_probabilities(int nq, const double* state, double* probs) {
    long long n = 1LL << nq;
    const cd* st = C(state);
    for (long long i = 0; i < n; ++i) probs[i] = st[i].re * st[i].re + st[i].im * st[i].im;
}

// measureQubit (sim/statevector/dynamic.go:179-230) with a caller-supplied
// uniform in place of the shot's PCG draw: P(0) summed over the blocks in
// index order, outcome 1 iff u >= P(0), then zero the other half and scale
// the kept half by 1/norm unless norm < 1e-15. Returns the outcome.
int or_sv_measure(int nq, double* state, int qubit, double u) {
    const long long half = 1LL << qubit, block = half << 1, n = 1LL << nq;
    cd* st = C(state);
    double p0 = 0.0;
    for (long long b0 = 0; b0 < n; b0 += block)
        for (long long off = 0; off < half; ++off) {
            const cd a = st[b0 + off];
            p0 += a.re * a.re + a.im * a.im;
        }
    const int outcome = u >= p0 ? 1 : 0;
    const double norm = outcome == 0 ? std::sqrt(p0) : std::sqrt(1 - p0);
    if (norm < 1e-15) return outcome;
    const double inv = 1.0 / norm;
    for (long long b0 = 0; b0 < n; b0 += block)
        for (long long off = 0; off < half; ++off) {
            cd& a0 = st[b0 + off];
            cd& a1 = st[b0 + off + half];
            if (outcome == 0) {
                a0 = {a0.re * inv, a0.im * inv};
                a1 = {0.0, 0.0};
            } else {
                a0 = {0.0, 0.0};
                a1 = {a1.re * inv, a1.im * inv};
            }
        }
    return outcome;
}

// measureQubitDM (sim/densitymatrix/dynamic.go:198-255) with a caller-supplied
// uniform: P(0) = sum of Re rho[i,i] over i with the bit clear (index order),
// outcome 1 iff u >= P(0); entries with both row and column bit equal to the
// outcome are divided by its probability, the others zeroed, unless that
// probability is below 1e-15. Returns the outcome.
int or_dm_measure(int nq, double* rho_, int qubit, double u) {
    const long long dim = 1LL << nq, mask = 1LL << qubit;
    cd* rho = C(rho_);
    double p0 = 0.0;
    for (long long i = 0; i < dim; ++i)
        if (!(i & mask)) p0 += rho[i * dim + i].re;
    const int outcome = u >= p0 ? 1 : 0;
    const double p = outcome == 0 ? p0 : 1 - p0;
    if (p < 1e-15) return outcome;
    const double inv = 1.0 / p;
    for (long long r = 0; r < dim; ++r) {
        const int rb = (int)((r >> qubit) & 1);
        for (long long c = 0; c < dim; ++c) {
            const int cb = (int)((c >> qubit) & 1);
            cd& a = rho[r * dim + c];
            if (rb == outcome && cb == outcome)
                a = {a.re * inv, a.im * inv};
            else
                a = {0.0, 0.0};
        }
    }
    return outcome;
}

// sampleIndex (sim/statevector/sim.go:288-298) for caller-supplied uniforms.
void or_sample(const double* probs, uint64_t len, const double* uniforms, size_t shots, uint64_t* out) {
    for (size_t k = 0; k < shots; ++k) {
        double r = uniforms[k], cum = 0.0;
        uint64_t hit = len - 1;
        for (uint64_t i = 0; i < len; ++i) {
            cum += probs[i];
            if (r < cum) {
                hit = i;
                break;
            }
        }
        out[k] = hit;
    }
}

// Sequential FP64 running sum sum_{j<=i} p_j at the requested indices (the
// `cum` of sampleIndex), for checking boundary cases.
void or_cumsum_at(const double* probs, uint64_t len, const uint64_t* at, size_t n_at, double* out) {
    double cum = 0.0;
    size_t k = 0;
    for (uint64_t i = 0; i < len && k < n_at; ++i) {
        cum += probs[i];
        while (k < n_at && at[k] == i) out[k++] = cum;
    }
}

// The full sequential running sum cum_i = (((p_0 + p_1) + p_2) + ... + p_i),
// so that sampleIndex(r) = first i with r < cum_i (a sorted search).
void or_cumsum(const double* probs, uint64_t len, double* out) {
    double cum = 0.0;
    for (uint64_t i = 0; i < len; ++i) {
        cum += probs[i];
        out[i] = cum;
    }
}

// pauli.Expect / ExpectSum (sim/pauli/expect_sv.go:21-97).
void or_sv_expect_pauli_sum(int nq, const double* state, const gq_pauli_term* terms, size_t n_terms,
                            int threads, double* out_re, double* out_im) {
    const cd* st = C(state);
    long long n = 1LL << nq;
    cd total = {0.0, 0.0};
    for (size_t t = 0; t < n_terms; ++t) {
        uint64_t xm = terms[t].x_mask, zm = terms[t].z_mask;
        cd yphase = ipow(__builtin_popcountll(xm & zm));
        cd coeff = {terms[t].coeff_re, terms[t].coeff_im};
        auto range = [&](long long b, long long e) {
            cd s = {0.0, 0.0};
            for (long long i = b; i < e; ++i) {
                long long j = i ^ (long long)xm;
                cd sg = {popcount_parity(i & zm) ? -1.0 : 1.0, 0.0};
                s = add(s, mul(mul(mul(conjc(st[j]), sg), yphase), st[i]));
            }
            return s;
        };
        cd sum;
        if (threads > 0 && nq >= 17) {  // expectParallel (expect_sv.go:49-88)
            int w = optimal_workers(nq, threads);
            if (w > n) w = (int)n;
            std::vector<cd> partial(w);
            long long chunk = n / w;
            std::vector<std::thread> ts;
            for (int k = 0; k < w; ++k) {
                long long s0 = k * chunk, e0 = (k == w - 1) ? n : s0 + chunk;
                ts.emplace_back([&, k, s0, e0] { partial[k] = range(s0, e0); });
            }
            for (auto& th : ts) th.join();
            sum = {0.0, 0.0};
            for (auto& p : partial) sum = add(sum, p);
        } else {
            sum = range(0, n);
        }
        total = add(total, mul(coeff, sum));
    }
    *out_re = total.re;
    *out_im = total.im;
}

// ExpectationValue (sim/statevector/sim.go:368-382); rounded != 0 applies its
// math.Round(ev*1e14)/1e14.
double or_sv_expect_z(int nq, const double* state, uint64_t mask, int rounded) {
    const cd* st = C(state);
    long long n = 1LL << nq;
    double ev = 0.0;
    for (long long i = 0; i < n; ++i) {
        double p = st[i].re * st[i].re + st[i].im * st[i].im;
        if (popcount_parity(i & mask) == 0)
            ev += p;
        else
            ev -= p;
    }
    return rounded ? std::round(ev * 1e14) / 1e14 : ev;
}

// densitymatrix Apply (sim/densitymatrix/sim.go:87-191) for an op stream in
// which the caller has already inserted the noise channels after each gate.
int or_dm_apply(int nq, double* rho, const gq_op* ops, size_t n_ops, int threads) {
    DM s{nq, 1LL << nq, C(rho), threads};
    for (size_t i = 0; i < n_ops; ++i) {
        const gq_op& op = ops[i];
        if (op.kind == GQ_OP_BARRIER) continue;
        if (op.kind == GQ_OP_RESET) {
            dm_reset(s, op.qubits[0]);
            continue;
        }
        if (op.kind == GQ_OP_CHANNEL) {
            dm_channel(s, op);
            continue;
        }
        if (op.kind == GQ_OP_CONTROLLED) {
            std::vector<cd> full = controlled_full(op);
            dm_gate(s, op.qubits, op.num_qubits, full.data());
            continue;
        }
        dm_gate(s, op.qubits, op.num_qubits, C(op.matrix));
    }
    return GQ_OK;
}

// pauli.ExpectSumDM (sim/pauli/expect_dm.go:9-30).
void or_dm_expect_pauli_sum(int nq, const double* rho_, const gq_pauli_term* terms, size_t n_terms,
                            double* out_re, double* out_im) {
    const cd* rho = C(rho_);
    long long dim = 1LL << nq;
    cd total = {0.0, 0.0};
    for (size_t t = 0; t < n_terms; ++t) {
        uint64_t xm = terms[t].x_mask, zm = terms[t].z_mask;
        cd yphase = ipow(__builtin_popcountll(xm & zm));
        cd sum = {0.0, 0.0};
        for (long long i = 0; i < dim; ++i) {
            long long j = i ^ (long long)xm;
            cd sg = {popcount_parity(i & zm) ? -1.0 : 1.0, 0.0};
            sum = add(sum, mul(mul(rho[i * dim + j], sg), yphase));
        }
        total = add(total, mul(cd{terms[t].coeff_re, terms[t].coeff_im}, sum));
    }
    *out_re = total.re;
    *out_im = total.im;
}

// Purity (sim/densitymatrix/sim.go:265-276).
double or_dm_purity(int nq, const double* rho_) {
    const cd* rho = C(rho_);
    long long dim = 1LL << nq;
    cd tr = {0.0, 0.0};
    for (long long i = 0; i < dim; ++i)
        for (long long j = 0; j < dim; ++j) tr = add(tr, mul(rho[i * dim + j], conjc(rho[j * dim + i])));
    return std::fabs(tr.re);
}

// Fidelity (sim/densitymatrix/sim.go:280-291).
double or_dm_fidelity(int nq, const double* rho_, const double* psi_) {
    const cd* rho = C(rho_);
    const cd* psi = C(psi_);
    long long dim = 1LL << nq;
    cd f = {0.0, 0.0};
    for (long long i = 0; i < dim; ++i)
        for (long long j = 0; j < dim; ++j) f = add(f, mul(mul(conjc(psi[i]), rho[i * dim + j]), psi[j]));
    return std::fabs(f.re);
}

// diagonalProbs (sim/densitymatrix/measure.go:11-20).
void or_dm_diagonal_probs(int nq, const double* rho_, double* probs) {
    const cd* rho = C(rho_);
    long long dim = 1LL << nq;
    for (long long i = 0; i < dim; ++i) {
        probs[i] = rho[i * dim + i].re;
        if (probs[i] < 0) probs[i] = 0;
    }
}

// ApplyReadoutError (sim/densitymatrix/measure.go:29-71); p01[q] < 0 means no
// readout error registered for qubit q. probs is updated in place.
void or_dm_readout(int nq, double* probs, const double* p01, const double* p10) {
    long long dim = 1LL << nq;
    std::vector<double> result(dim, 0.0);
    for (long long i = 0; i < dim; ++i) {
        double p = probs[i];
        if (p == 0) continue;
        result[i] += p;
    }
    for (int q = 0; q < nq; ++q) {
        if (p01[q] < 0) continue;
        std::vector<double> nr(dim, 0.0);
        long long mask = 1LL << q;
        for (long long i = 0; i < dim; ++i) {
            if (result[i] == 0) continue;
            long long f = i ^ mask;
            if ((i & mask) == 0) {
                nr[i] += result[i] * (1 - p01[q]);
                nr[f] += result[i] * p01[q];
            } else {
                nr[i] += result[i] * (1 - p10[q]);
                nr[f] += result[i] * p10[q];
            }
        }
        result.swap(nr);
    }
    std::memcpy(probs, result.data(), dim * sizeof(double));
}

}  // extern "C"

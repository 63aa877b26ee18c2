// Gate analysis and pass / phase scheduling (see schedule.hpp).
#include "schedule.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <string>
#include <random>

namespace gq {

namespace {

inline bool is_one(Z z) { return z.re == 1.0 && z.im == 0.0; }
inline bool is_zero(Z z) { return z.re == 0.0 && z.im == 0.0; }
inline bool eq(Z a, Z b) { return a.re == b.re && a.im == b.im; }

int popc(uint64_t v) { return __builtin_popcountll(v); }

// Is local position p (bit k-1-p of the local index) a control of m?
bool is_control(const std::vector<Z>& m, int k, int p) {
    const int dim = 1 << k, bit = 1 << (k - 1 - p);
    for (int r = 0; r < dim; ++r)
        for (int c = 0; c < dim; ++c) {
            if ((r & bit) && (c & bit)) continue;
            const Z v = m[r * dim + c];
            if (r == c ? !is_one(v) : !is_zero(v)) return false;
        }
    return true;
}

// Restricts m to the block where local position p is 1.
std::vector<Z> restrict_to_one(const std::vector<Z>& m, int k, int p) {
    const int dim = 1 << k, bit = 1 << (k - 1 - p), nd = dim >> 1;
    std::vector<Z> out(nd * nd);
    auto squeeze = [&](int x) {  // drop bit `bit` from x
        const int lo = x & (bit - 1), hi = (x >> 1) & ~(bit - 1);
        return hi | lo;
    };
    for (int r = 0; r < dim; ++r) {
        if (!(r & bit)) continue;
        for (int c = 0; c < dim; ++c) {
            if (!(c & bit)) continue;
            out[squeeze(r) * nd + squeeze(c)] = m[r * dim + c];
        }
    }
    return out;
}

int cost_of(KType t) {
    switch (t) {
        case K_GRAD: return 16;
        case K_U1: return 8;
        case K_U2: return 16;
        case K_U3: return 32;
        case K_U4: return 64;
        case K_DIAG: return 3;
        case K_RESET: return 4;
        case K_PAIRSUM: return 6;
        default: return 1;
    }
}

// Bit 63 is no qubit: it marks ops that commute with every unitary but not
// with a reset (a phase on the whole state), so only a deferred reset, which
// blocks all bits, holds them back.
constexpr uint64_t kGlobalBit = 1ull << 63;

void finish(NGate& g) {
    g.nd_mask = 0;
    g.d_mask = g.ctrl | kGlobalBit;
    const KType kind = g.type == K_GRAD ? g.grad_kind : g.type;
    if (kind == K_DIAG) {
        for (int q : g.targets) g.d_mask |= 1ull << q;
    } else if (kind != K_PHASE) {
        for (int q : g.targets) g.nd_mask |= 1ull << q;
    }
    g.cost = cost_of(kind) + (g.type == K_GRAD ? cost_of(K_GRAD) : 0);
}

}  // namespace

int analyze_matrix(const std::vector<Z>& m0, const std::vector<int>& qubits0, uint64_t ctrl, int src,
                   std::vector<NGate>& out, std::string& err) {
    std::vector<Z> m = m0;
    std::vector<int> qubits = qubits0;
    // Split off controls until none is left.
    for (bool found = true; found && !qubits.empty();) {
        found = false;
        const int k = (int)qubits.size();
        for (int p = 0; p < k; ++p) {
            if (is_control(m, k, p)) {
                ctrl |= 1ull << qubits[p];
                m = restrict_to_one(m, k, p);
                qubits.erase(qubits.begin() + p);
                found = true;
                break;
            }
        }
    }
    const int t = (int)qubits.size();
    const int dim = 1 << t;
    NGate g;
    g.ctrl = ctrl;
    g.src = src;
    g.targets = qubits;
    if (t == 0) {
        if (is_one(m[0])) return GQ_OK;  // identity
        g.type = K_PHASE;
        g.data = {m[0]};
        finish(g);
        out.push_back(g);
        return GQ_OK;
    }
    bool diag = true;
    for (int r = 0; r < dim && diag; ++r)
        for (int c = 0; c < dim; ++c)
            if (r != c && !is_zero(m[r * dim + c])) {
                diag = false;
                break;
            }
    if (diag) {
        bool all_eq = true, all_one = true;
        for (int i = 0; i < dim; ++i) {
            all_eq = all_eq && eq(m[i * dim + i], m[0]);
            all_one = all_one && is_one(m[i * dim + i]);
        }
        if (all_one) return GQ_OK;
        if (all_eq) {  // a phase times identity on the targets
            g.type = K_PHASE;
            g.targets.clear();
            g.data = {m[0]};
        } else {
            g.type = K_DIAG;
            g.data.resize(dim);
            for (int i = 0; i < dim; ++i) g.data[i] = m[i * dim + i];
        }
        finish(g);
        out.push_back(g);
        return GQ_OK;
    }
    if (t == 1 && is_zero(m[0]) && is_zero(m[3])) {
        g.type = K_X;
        g.data = {m[1], m[2]};
        g.pure = is_one(m[1]) && is_one(m[2]);
        finish(g);
        out.push_back(g);
        return GQ_OK;
    }
    if (t == 2) {
        bool swap = true;
        for (int r = 0; r < 4 && swap; ++r)
            for (int c = 0; c < 4; ++c) {
                const int want = (r == 1) ? 2 : (r == 2) ? 1 : r;
                const Z v = m[r * 4 + c];
                if (c == want ? !is_one(v) : !is_zero(v)) {
                    swap = false;
                    break;
                }
            }
        if (swap) {
            g.type = K_SWAP;
            finish(g);
            out.push_back(g);
            return GQ_OK;
        }
    }
    if (t > RQ) {
        err = "gate acts densely on " + std::to_string(t) + " qubits after control extraction (max 4)";
        return GQ_EUNSUPPORTED;
    }
    g.type = (KType)(K_U1 + (t - 1));
    g.data = m;
    finish(g);
    out.push_back(g);
    return GQ_OK;
}

int normalize_op(const gq_op& op, int nphys, std::vector<NGate>& out, std::string& err) {
    if (op.kind == GQ_OP_BARRIER) return GQ_OK;
    if (op.num_qubits < 1 || op.num_qubits > GQ_MAX_OP_QUBITS) {
        err = "op has " + std::to_string(op.num_qubits) + " qubits";
        return GQ_EINVAL;
    }
    uint64_t seen = 0;
    for (int i = 0; i < op.num_qubits; ++i) {
        const int q = op.qubits[i];
        if (q < 0 || q >= nphys) {
            err = "qubit " + std::to_string(q) + " out of range";
            return GQ_EINVAL;
        }
        if (seen & (1ull << q)) {
            err = "duplicate qubit " + std::to_string(q);
            return GQ_EINVAL;
        }
        seen |= 1ull << q;
    }
    if (op.kind == GQ_OP_RESET) {
        NGate g;
        g.type = K_RESET;
        g.targets = {op.qubits[0]};
        finish(g);
        g.barrier = true;
        out.push_back(g);
        return GQ_OK;
    }
    if (op.kind == GQ_OP_CHANNEL) {
        err = "Kraus channels apply to density matrices only";
        return GQ_EINVAL;
    }
    if (!op.matrix) {
        err = "op has no matrix";
        return GQ_EINVAL;
    }
    int nc = 0;
    uint64_t ctrl = 0;
    if (op.kind == GQ_OP_CONTROLLED) {
        nc = op.num_controls;
        if (nc < 0 || nc >= op.num_qubits) {
            err = "bad control count";
            return GQ_EINVAL;
        }
        for (int i = 0; i < nc; ++i) ctrl |= 1ull << op.qubits[i];
    }
    const int k = op.num_qubits - nc;
    if (k > 10) {
        err = "inner gate on " + std::to_string(k) + " qubits";
        return GQ_EUNSUPPORTED;
    }
    const int dim = 1 << k;
    std::vector<Z> m(dim * dim);
    std::memcpy(m.data(), op.matrix, sizeof(Z) * dim * dim);
    std::vector<int> qs(op.qubits + nc, op.qubits + op.num_qubits);
    return analyze_matrix(m, qs, ctrl, -1, out, err);
}

namespace {

struct PhasePlan {
    uint64_t rmask = 0;
    std::vector<int> gates;
};

// Greedy partition of `list` (a valid order) into groups whose non-diagonal
// qubits fit in `limit` qubits of `allowed`. A gate that does not fit is
// deferred, and every later gate that does not commute with a deferred gate
// (shares a qubit non-diagonally) is deferred behind it, so each group is a
// valid reordering of the sequence.
template <class Fits>
void greedy_groups(const std::vector<NGate>& gates, std::vector<int> list, Fits fits,
                   std::vector<std::vector<int>>& groups, std::vector<uint64_t>& masks, uint64_t seed_mask) {
    while (!list.empty()) {
        uint64_t used = seed_mask, bnd = 0, bd = 0;
        std::vector<int> take, rest;
        int budget_used = 0;
        for (size_t i = 0; i < list.size(); ++i) {
            const NGate& g = gates[list[i]];
            const bool free = !(g.nd_mask & (bnd | bd)) && !(g.d_mask & bnd) && (!g.barrier || (bnd | bd) == 0);
            if (free && fits(used | g.nd_mask, budget_used + g.cost, take.empty())) {
                used |= g.nd_mask;
                budget_used += g.cost;
                take.push_back(list[i]);
                continue;
            }
            rest.push_back(list[i]);
            bnd |= g.barrier ? ~0ull : g.nd_mask;
            bd |= g.d_mask;
        }
        groups.push_back(take);
        masks.push_back(used);
        list.swap(rest);
    }
}

// ---- dense fusion inside a phase ---------------------------------------------
// Every thread holds all 2^4 amplitudes of the phase's register qubits, so a
// run of gates whose qubits (controls included) all lie in the register set
// acts on them as one dense 2^k x 2^k matrix, k = qubits the run touches. The
// run is replaced by that product when it costs fewer FMA per amplitude than
// the separate ops plus their per-op overhead.
constexpr int kOpOverhead = 6;

Z zmul(Z a, Z b) { return Z{a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }

// Applies gate g to v, a state over the qubits qs (local bit p <-> qs[p]).
void apply_small(const NGate& g, const std::vector<int>& qs, std::vector<Z>& v) {
    auto pos = [&](int q) {
        for (size_t p = 0; p < qs.size(); ++p)
            if (qs[p] == q) return (int)p;
        return -1;
    };
    uint32_t cm = 0;
    for (size_t p = 0; p < qs.size(); ++p)
        if (g.ctrl & (1ull << qs[p])) cm |= 1u << p;
    const int t = (int)g.targets.size();
    std::vector<int> tb(t);
    uint32_t tm = 0;
    for (int i = 0; i < t; ++i) {
        tb[i] = pos(g.targets[i]);
        tm |= 1u << tb[i];
    }
    const uint32_t dim = 1u << qs.size();
    auto sub = [&](uint32_t x, uint32_t r) {  // x with the target bits set from r (first target = MSB)
        for (int i = 0; i < t; ++i)
            if ((r >> (t - 1 - i)) & 1) x |= 1u << tb[i];
        return x;
    };
    switch (g.type) {
        case K_PHASE:
            for (uint32_t x = 0; x < dim; ++x)
                if ((x & cm) == cm) v[x] = zmul(g.data[0], v[x]);
            return;
        case K_DIAG:
            for (uint32_t x = 0; x < dim; ++x) {
                if ((x & cm) != cm) continue;
                uint32_t idx = 0;
                for (int i = 0; i < t; ++i) idx |= ((x >> tb[i]) & 1u) << (t - 1 - i);
                v[x] = zmul(g.data[idx], v[x]);
            }
            return;
        case K_X:
            for (uint32_t x = 0; x < dim; ++x) {
                if ((x & cm) != cm || (x & tm)) continue;
                const uint32_t y = x | tm;
                const Z a0 = v[x], a1 = v[y];
                v[x] = zmul(g.data[0], a1);
                v[y] = zmul(g.data[1], a0);
            }
            return;
        case K_SWAP:
            for (uint32_t x = 0; x < dim; ++x) {
                if ((x & cm) != cm) continue;
                const uint32_t b0 = (x >> tb[0]) & 1u, b1 = (x >> tb[1]) & 1u;
                if (b0 == 1 && b1 == 0) std::swap(v[x], v[(x & ~(1u << tb[0])) | (1u << tb[1])]);
            }
            return;
        default: {  // K_U1..K_U4
            const uint32_t td = 1u << t;
            std::vector<Z> in(td), out(td);
            for (uint32_t x = 0; x < dim; ++x) {
                if ((x & cm) != cm || (x & tm)) continue;
                for (uint32_t r = 0; r < td; ++r) in[r] = v[sub(x, r)];
                for (uint32_t r = 0; r < td; ++r) {
                    Z acc{0, 0};
                    for (uint32_t c = 0; c < td; ++c) {
                        const Z p = zmul(g.data[r * td + c], in[c]);
                        acc.re += p.re;
                        acc.im += p.im;
                    }
                    out[r] = acc;
                }
                for (uint32_t r = 0; r < td; ++r) v[sub(x, r)] = out[r];
            }
            return;
        }
    }
}

bool foldable(const NGate& g, uint64_t R) {
    if (g.type == K_GRAD || g.type == K_RESET || g.type == K_NONE) return false;
    uint64_t q = g.ctrl;
    for (int x : g.targets) q |= 1ull << x;
    return (q & ~R) == 0;
}

// The phase's gates, with runs of register-local gates folded into dense
// blocks where that is cheaper. rq[k] is the qubit of register bit k.
std::vector<NGate> fuse_phase(const std::vector<NGate>& gates, const std::vector<int>& group, uint64_t R,
                              const int* rq, bool enable) {
    std::vector<NGate> out;
    std::vector<int> run;
    auto flush = [&]() {
        if (run.empty()) return;
        uint64_t touched = 0;
        int sparse = 0;
        for (int gi : run) {
            const NGate& g = gates[gi];
            touched |= g.ctrl;
            for (int x : g.targets) touched |= 1ull << x;
            sparse += g.cost + kOpOverhead;
        }
        std::vector<int> qs;  // ascending register bit
        for (int k = 0; k < RQ; ++k)
            if (touched & (1ull << rq[k])) qs.push_back(rq[k]);
        const int k = (int)qs.size();
        const int dense = k ? cost_of((KType)(K_U1 + k - 1)) + kOpOverhead : 1 << 30;
        if (!enable || run.size() < 2 || dense >= sparse) {
            for (int gi : run) out.push_back(gates[gi]);
            run.clear();
            return;
        }
        const uint32_t dim = 1u << k;
        std::vector<Z> B(dim * dim, Z{0, 0});  // column c = image of basis state c
        for (uint32_t c = 0; c < dim; ++c) {
            std::vector<Z> v(dim, Z{0, 0});
            v[c] = Z{1, 0};
            for (int gi : run) apply_small(gates[gi], qs, v);
            for (uint32_t r = 0; r < dim; ++r) B[r * dim + c] = v[r];
        }
        NGate d;
        d.type = (KType)(K_U1 + k - 1);
        for (int p = k - 1; p >= 0; --p) d.targets.push_back(qs[p]);  // MSB first: local bit p <-> qs[p]
        d.data = B;
        d.src = gates[run.front()].src;
        finish(d);
        out.push_back(d);
        run.clear();
    };
    for (int gi : group) {
        if (foldable(gates[gi], R)) {
            run.push_back(gi);
        } else {
            flush();
            out.push_back(gates[gi]);
        }
    }
    flush();
    return out;
}

// Runs of commuting diagonal ops (phases, diagonals, and their gradient ops)
// in a phase's op list: identical parity-symmetric 2-qubit diagonals
// (d00 = d11, d01 = d10, no controls: RZZ(g), ZZ(g) of one layer) fold into
// one K_PAIRSUM with T[c] = d00^(K-c) d01^c; gradient ops of one parameter
// with such a G fold into one K_GRAD(K_PAIRSUM) with T[c] = (K-c) g00 + c g01.
// Inside such a run every op commutes with every other, and a gradient op
// measures the same Re <lambda|G|psi> anywhere in it when the run's
// diagonals are unitary (<D lambda|G|D psi> = <lambda|G|psi>), so gradient
// ops are moved ahead of the run's unitaries only when all of them are.
bool pair_sym(const NGate& g) {
    const KType k = g.type == K_GRAD ? g.grad_kind : g.type;
    return k == K_DIAG && g.ctrl == 0 && g.targets.size() == 2 && g.data.size() == 4 && eq(g.data[0], g.data[3]) &&
           eq(g.data[1], g.data[2]);
}

bool diag_class(const NGate& g) {
    const KType k = g.type == K_GRAD ? g.grad_kind : g.type;
    return (k == K_DIAG || k == K_PHASE) && !g.barrier;
}

bool unit_modulus(const NGate& g) {
    for (const Z& z : g.data)
        if (std::fabs(z.re * z.re + z.im * z.im - 1.0) > 1e-12) return false;
    return true;
}

// The classified pair data of a K_PAIRSUM (layout in tile_core.cuh,
// pair_counts): counts of the pairs on two register bits per slot, a qubit
// mask per register bit for its pairs with global qubits, the packed pairs of
// two global qubits. Every value is an integer below 2^16, exact in FP32.
void pair_data(const std::vector<int>& targets, uint64_t R, const int* rq, std::vector<Z>& data) {
    auto regbit = [&](int q) {
        for (int k = 0; k < RQ; ++k)
            if (rq[k] == q && (R >> q & 1ull)) return k;
        return -1;
    };
    uint64_t lo = 0, hi = 0, M[RQ] = {0, 0, 0, 0};
    int nr[RQ] = {0, 0, 0, 0};
    std::vector<int> gg;
    for (size_t p = 0; p + 1 < targets.size(); p += 2) {
        const int a = targets[p], b = targets[p + 1], ka = regbit(a), kb = regbit(b);
        if (ka >= 0 && kb >= 0) {
            for (int j = 0; j < NREG; ++j)
                if (((j >> ka) ^ (j >> kb)) & 1) (j < 8 ? lo : hi) += 1ull << (8 * (j & 7));
        } else if (ka >= 0 || kb >= 0) {
            const int r = ka >= 0 ? ka : kb, q = ka >= 0 ? b : a;
            M[r] |= 1ull << q;
            ++nr[r];
        } else {
            gg.push_back(a | (b << 6));
        }
    }
    auto c16 = [](uint64_t v, int i) { return (double)((v >> (16 * i)) & 0xffffull); };
    data.push_back(Z{c16(lo, 0), c16(lo, 1)});
    data.push_back(Z{c16(lo, 2), c16(lo, 3)});
    data.push_back(Z{c16(hi, 0), c16(hi, 1)});
    data.push_back(Z{c16(hi, 2), c16(hi, 3)});
    for (int r = 0; r < RQ; ++r) {
        data.push_back(Z{c16(M[r], 0), c16(M[r], 1)});
        data.push_back(Z{c16(M[r], 2), (double)nr[r]});
    }
    data.push_back(Z{(double)gg.size(), 0.0});
    for (size_t k = 0; k < gg.size(); k += 2)
        data.push_back(Z{(double)gg[k], k + 1 < gg.size() ? (double)gg[k + 1] : 0.0});
}

std::vector<NGate> fuse_pairsums(const std::vector<NGate>& in, uint64_t R, const int* rq) {
    std::vector<NGate> out;
    size_t i = 0;
    while (i < in.size()) {
        if (!diag_class(in[i])) {
            out.push_back(in[i++]);
            continue;
        }
        size_t j = i;
        bool has_grad = false, unitary = true;
        while (j < in.size() && diag_class(in[j])) {
            if (in[j].type == K_GRAD)
                has_grad = true;
            else if (!unit_modulus(in[j]))
                unitary = false;
            ++j;
        }
        if (has_grad && !unitary) {  // keep the run as it is
            for (size_t k = i; k < j; ++k) out.push_back(in[k]);
            i = j;
            continue;
        }
        // groups of fusable ops, in first-appearance order
        std::vector<std::vector<size_t>> groups;
        std::vector<size_t> singles;
        for (size_t k = i; k < j; ++k) {
            const NGate& g = in[k];
            if (!pair_sym(g)) {
                singles.push_back(k);
                continue;
            }
            bool placed = false;
            for (auto& grp : groups) {
                const NGate& h = in[grp[0]];
                if (h.type == g.type && h.param == g.param && eq(h.data[0], g.data[0]) && eq(h.data[1], g.data[1]) &&
                    grp.size() < 200) {
                    // a pair at most once per op (its qubit masks hold each pair once)
                    bool dup = false;
                    for (size_t q : grp)
                        dup = dup || (std::min(in[q].targets[0], in[q].targets[1]) == std::min(g.targets[0], g.targets[1]) &&
                                      std::max(in[q].targets[0], in[q].targets[1]) == std::max(g.targets[0], g.targets[1]));
                    if (dup) continue;
                    grp.push_back(k);
                    placed = true;
                    break;
                }
            }
            if (!placed) groups.push_back({k});
        }
        std::vector<NGate> grads, units;
        for (size_t k : singles) (in[k].type == K_GRAD ? grads : units).push_back(in[k]);
        for (const auto& grp : groups) {
            const NGate& h = in[grp[0]];
            if (grp.size() < 2) {
                (h.type == K_GRAD ? grads : units).push_back(h);
                continue;
            }
            const int K = (int)grp.size();
            NGate f;
            f.type = h.type == K_GRAD ? K_GRAD : K_PAIRSUM;
            f.grad_kind = h.type == K_GRAD ? K_PAIRSUM : K_NONE;
            f.param = h.param;
            f.src = h.src;
            for (size_t k : grp) {
                f.targets.push_back(in[k].targets[0]);
                f.targets.push_back(in[k].targets[1]);
            }
            pair_data(f.targets, R, rq, f.data);
            const Z e = h.data[0], o = h.data[1];
            if (h.type == K_GRAD) {
                for (int c = 0; c <= K; ++c)
                    f.data.push_back(Z{(K - c) * e.re + c * o.re, (K - c) * e.im + c * o.im});
            } else {
                std::vector<Z> pe(K + 1), po(K + 1);
                pe[0] = po[0] = Z{1, 0};
                for (int c = 1; c <= K; ++c) {
                    pe[c] = Z{pe[c - 1].re * e.re - pe[c - 1].im * e.im, pe[c - 1].re * e.im + pe[c - 1].im * e.re};
                    po[c] = Z{po[c - 1].re * o.re - po[c - 1].im * o.im, po[c - 1].re * o.im + po[c - 1].im * o.re};
                }
                for (int c = 0; c <= K; ++c) {
                    const Z a = pe[K - c], b = po[c];
                    f.data.push_back(Z{a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re});
                }
            }
            (h.type == K_GRAD ? grads : units).push_back(f);
        }
        // A unitary pair sum right after the gradient pair sum of the same
        // pairs reuses the pair counts (flag `pure` here, KOp.flags bit 1).
        if (!grads.empty() && !units.empty() && grads.back().type == K_GRAD &&
            grads.back().grad_kind == K_PAIRSUM && units.front().type == K_PAIRSUM &&
            units.front().targets == grads.back().targets)
            units.front().pure = true;
        out.insert(out.end(), grads.begin(), grads.end());
        out.insert(out.end(), units.begin(), units.end());
        i = j;
    }
    return out;
}

int rank_gf2(std::vector<uint32_t> v) {
    int r = 0;
    for (int bit = 31; bit >= 0; --bit) {
        int piv = -1;
        for (size_t i = r; i < v.size(); ++i)
            if ((v[i] >> bit) & 1u) {
                piv = (int)i;
                break;
            }
        if (piv < 0) continue;
        std::swap(v[r], v[piv]);
        for (size_t i = 0; i < v.size(); ++i)
            if ((int)i != r && ((v[i] >> bit) & 1u)) v[i] ^= v[r];
        ++r;
    }
    return r;
}

}  // namespace

void schedule(const std::vector<NGate>& gates, int nphys, const SchedOptions& opt, Program& prog) {
    const int m = std::min(opt.tile_qubits, nphys);
    const int low = std::min(opt.low_qubits, m);
    const int W = opt.swizzle_width;
    const uint64_t all = (nphys >= 64) ? ~0ull : ((1ull << nphys) - 1);
    const uint64_t low_mask = (1ull << low) - 1;
    prog.gates += (int64_t)gates.size();

    std::vector<int> remaining(gates.size());
    for (size_t i = 0; i < gates.size(); ++i) remaining[i] = (int)i;

    std::mt19937_64 rng(12345);
    // Support of the state before the current pass (SchedOptions::support0).
    uint64_t support = opt.support0 | ~all;
    while (!remaining.empty()) {
        // ---- pass: the tile holds the targets of every absorbed gate.
        std::vector<std::vector<int>> pgroups;
        std::vector<uint64_t> pmasks;
        // A pass launches at most 2^(support qubits outside the low ones) CTAs
        // (SchedOptions::support0): while that is below a full pass's
        // 2^(nphys - m), its arithmetic costs proportionally less, and its
        // budget grows by the same factor (up to 64x).
        int budget = opt.budget;
        {
            const int full_outer = nphys - m, sup_outer = popc(support & all & ~low_mask);
            if (sup_outer < full_outer)
                budget = (int)std::min<int64_t>((int64_t)opt.budget << std::min(6, full_outer - sup_outer), 1 << 28);
        }
        {
            std::vector<int> take, rest;
            uint64_t T = low_mask, bnd = 0, bd = 0;
            int used = 0, ngrad = 0;
            for (size_t i = 0; i < remaining.size(); ++i) {
                const NGate& g = gates[remaining[i]];
                const bool free =
                    !(g.nd_mask & (bnd | bd)) && !(g.d_mask & bnd) && (!g.barrier || (bnd | bd) == 0);
                const uint64_t nt = T | g.nd_mask;
                const bool grad_ok = g.type != K_GRAD || ngrad < MAX_GRAD_SLOTS;
                if (free && grad_ok && popc(nt) <= m && (used + g.cost <= budget || take.empty())) {
                    T = nt;
                    used += g.cost;
                    ngrad += g.type == K_GRAD;
                    take.push_back(remaining[i]);
                    continue;
                }
                rest.push_back(remaining[i]);
                bnd |= g.barrier ? ~0ull : g.nd_mask;
                bd |= g.d_mask;
                if ((bnd & all) == all) {  // only unconditioned global phases could still pass
                    rest.insert(rest.end(), remaining.begin() + i + 1, remaining.end());
                    break;
                }
            }
            pgroups.push_back(take);
            pmasks.push_back(T);
            remaining.swap(rest);
        }
        uint64_t T = pmasks[0];
        for (int q = 0; q < nphys && popc(T) < m; ++q) T |= 1ull << q;  // fill with low qubits
        const std::vector<int>& absorbed = pgroups[0];

        // ---- phases: register sets of RQ qubits inside the tile.
        std::vector<std::vector<int>> groups;
        std::vector<uint64_t> rmasks;
        greedy_groups(
            gates, absorbed, [&](uint64_t u, int, bool) { return popc(u) <= RQ; }, groups, rmasks, 0);
        if (groups.empty()) {  // a pass with no gate cannot happen; keep one empty phase
            groups.push_back({});
            rmasks.push_back(0);
        }

        PassDesc pd;
        std::memset(&pd, 0, sizeof(pd));
        pd.m = m;
        pd.phase0 = (int32_t)prog.phases.size();
        pd.n_phases = (int32_t)groups.size();
        int tile_q[MAX_TILE], tb_of[64];
        int nt = 0;
        for (int q = 0; q < nphys; ++q) {
            if (T & (1ull << q)) {
                tb_of[q] = nt;
                tile_q[nt++] = q;
            } else if (support & (1ull << q)) {
                pd.outer_q[pd.n_outer++] = q;
            }
        }
        for (int b = 0; b < m; ++b) pd.tile_q[b] = tile_q[b];

        // Register sets filled to RQ qubits (highest free tile qubits first).
        std::vector<uint64_t> rfull(groups.size());
        for (size_t p = 0; p < groups.size(); ++p) {
            uint64_t R = rmasks[p];
            for (int b = m - 1; b >= 0 && popc(R) < RQ; --b) R |= 1ull << tile_q[b];
            rfull[p] = R;
        }

        // Swizzle: slot = i ^ S*(i >> W) on the low W bits; choose S so that the
        // W lowest thread bits of every phase hit distinct bank groups.
        uint32_t S[MAX_TILE] = {0};
        const int tbits = m - RQ;
        if (W > 0 && m > W && tbits >= W) {
            int best_ok = -1;
            uint32_t best[MAX_TILE] = {0};
            for (int attempt = 0; attempt < 512; ++attempt) {
                uint32_t cand[MAX_TILE] = {0};
                if (attempt > 0)
                    for (int b = W; b < m; ++b) cand[b] = (uint32_t)(rng() & ((1u << W) - 1));
                int ok = 0;
                for (size_t p = 0; p < groups.size(); ++p) {
                    std::vector<uint32_t> cols;
                    for (int b = 0; b < m && (int)cols.size() < W; ++b) {
                        if (rfull[p] & (1ull << tile_q[b])) continue;
                        cols.push_back(((b < W) ? (1u << b) : 0u) ^ cand[b]);
                    }
                    if (rank_gf2(cols) == W) ++ok;
                }
                if (ok > best_ok) {
                    best_ok = ok;
                    std::memcpy(best, cand, sizeof(best));
                }
                if (ok == (int)groups.size()) break;
            }
            std::memcpy(S, best, sizeof(S));
            prog.conflict_phases += (int64_t)groups.size() - best_ok;
        }
        for (int b = 0; b < m; ++b) pd.acol[b] = (1u << b) ^ S[b];

        std::vector<int> slot_params;
        for (size_t p = 0; p < groups.size(); ++p) {
            PhaseDesc ph;
            std::memset(&ph, 0, sizeof(ph));
            const uint64_t R = rfull[p];
            int rq[RQ], rtb[RQ], nr = 0;
            for (int b = 0; b < m; ++b)
                if (R & (1ull << tile_q[b])) {
                    rq[nr] = tile_q[b];
                    rtb[nr] = b;
                    ++nr;
                }
            uint32_t tslot[MAX_TILE];
            uint64_t tglob[MAX_TILE];
            int nb = 0;
            for (int b = 0; b < m; ++b)
                if (!(R & (1ull << tile_q[b]))) {
                    tslot[nb] = pd.acol[b];
                    tglob[nb] = 1ull << tile_q[b];
                    ++nb;
                }
            for (int v = 0; v < TLO; ++v) {
                uint32_t sv = 0;
                uint64_t gv = 0;
                for (int b = 0; b < 4 && b < nb; ++b)
                    if ((v >> b) & 1) {
                        sv ^= tslot[b];
                        gv |= tglob[b];
                    }
                ph.tlo_slot[v] = sv;
                ph.tlo_glob[v] = gv;
            }
            for (int v = 0; v < THI; ++v) {
                uint32_t sv = 0;
                uint64_t gv = 0;
                for (int b = 0; b < 5 && b + 4 < nb; ++b)
                    if ((v >> b) & 1) {
                        sv ^= tslot[b + 4];
                        gv |= tglob[b + 4];
                    }
                ph.thi_slot[v] = sv;
                ph.thi_glob[v] = gv;
            }
            for (int j = 0; j < NREG; ++j) {
                uint32_t s = 0;
                for (int k = 0; k < RQ; ++k)
                    if ((j >> k) & 1) s ^= pd.acol[rtb[k]];
                ph.rslot[j] = s;
            }
            auto kbit = [&](int q) {
                for (int k = 0; k < RQ; ++k)
                    if (rq[k] == q) return k;
                return -1;
            };
            ph.op_begin = (int32_t)prog.ops.size();
            std::vector<NGate> fused = fuse_phase(gates, groups[p], R, rq, opt.fuse_dense);
            if (opt.fuse_pairs) fused = fuse_pairsums(fused, R, rq);
            for (const NGate& g : fused) {
                KOp op;
                std::memset(&op, 0, sizeof(op));
                op.type = g.type;
                const KType kind = g.type == K_GRAD ? g.grad_kind : g.type;
                if (g.type == K_GRAD) {  // one slot per parameter of the pass
                    const auto at = std::find(slot_params.begin(), slot_params.end(), g.param);
                    op.slot = (uint32_t)(at - slot_params.begin());
                    if (at == slot_params.end()) slot_params.push_back(g.param);
                }
                for (int k = 0; k < RQ; ++k)
                    if (g.ctrl & (1ull << rq[k])) op.creg |= (uint8_t)(1u << k);
                op.cmask = g.ctrl & ~R;
                op.mat = (uint32_t)prog.pool.size();
                const int t = (int)g.targets.size();
                if (kind >= K_U1 && kind <= K_U4) {
                    // order[p] = target index whose register bit is the p-th smallest
                    std::vector<int> order(t);
                    for (int i = 0; i < t; ++i) order[i] = i;
                    std::sort(order.begin(), order.end(),
                              [&](int a, int b) { return kbit(g.targets[a]) < kbit(g.targets[b]); });
                    uint8_t tk[4] = {0, 0, 0, 0};
                    for (int i = 0; i < t; ++i) tk[i] = (uint8_t)kbit(g.targets[order[i]]);
                    op.t0 = tk[0];
                    op.t1 = tk[1];
                    op.t2 = tk[2];
                    const int dim = 1 << t;
                    auto mapidx = [&](int x) {
                        int o = 0;
                        for (int pp = 0; pp < t; ++pp)
                            if ((x >> pp) & 1) o |= 1 << (t - 1 - order[pp]);
                        return o;
                    };
                    for (int r = 0; r < dim; ++r)
                        for (int c = 0; c < dim; ++c) prog.pool.push_back(g.data[mapidx(r) * dim + mapidx(c)]);
                } else if (kind == K_X || kind == K_RESET) {
                    op.t0 = (uint8_t)kbit(g.targets[0]);
                    op.flags = g.pure ? 1 : 0;
                    prog.pool.insert(prog.pool.end(), g.data.begin(), g.data.end());
                } else if (kind == K_PAIRSUM) {
                    op.nreg = (uint8_t)(g.targets.size() / 2);  // pairs; the table has nreg + 1 entries
                    op.flags = g.pure ? 2 : 0;  // counts of the preceding gradient pair sum
                    prog.pool.insert(prog.pool.end(), g.data.begin(), g.data.end());
                } else if (kind == K_SWAP) {
                    int a = kbit(g.targets[0]), b = kbit(g.targets[1]);
                    op.t0 = (uint8_t)std::min(a, b);
                    op.t1 = (uint8_t)std::max(a, b);
                } else if (kind == K_PHASE) {
                    prog.pool.push_back(g.data[0]);
                } else if (kind == K_DIAG) {
                    // Index layout: register targets (ascending register bit)
                    // in the low bits, the others (ascending qubit) above.
                    std::vector<int> reg_t, oth_t;  // target positions
                    for (int i = 0; i < t; ++i) (kbit(g.targets[i]) >= 0 ? reg_t : oth_t).push_back(i);
                    std::sort(reg_t.begin(), reg_t.end(),
                              [&](int a, int b) { return kbit(g.targets[a]) < kbit(g.targets[b]); });
                    std::sort(oth_t.begin(), oth_t.end(), [&](int a, int b) { return g.targets[a] < g.targets[b]; });
                    op.nreg = (uint8_t)reg_t.size();
                    for (int i : oth_t) op.dmask |= 1ull << g.targets[i];
                    const int dim = 1 << t;
                    for (int v = 0; v < dim; ++v) {
                        int orig = 0;
                        for (size_t pp = 0; pp < reg_t.size(); ++pp)
                            if ((v >> pp) & 1) orig |= 1 << (t - 1 - reg_t[pp]);
                        for (size_t pp = 0; pp < oth_t.size(); ++pp)
                            if ((v >> (reg_t.size() + pp)) & 1) orig |= 1 << (t - 1 - oth_t[pp]);
                        prog.pool.push_back(g.data[orig]);
                    }
                    for (int j = 0; j < NREG; ++j) {
                        uint64_t ri = 0;
                        for (size_t pp = 0; pp < reg_t.size(); ++pp)
                            if ((j >> kbit(g.targets[reg_t[pp]])) & 1) ri |= 1ull << pp;
                        op.ridx |= ri << (4 * j);
                    }
                }
                if (g.type == K_GRAD) op.flags = (uint8_t)kind;
                prog.ops.push_back(op);
            }
            ph.op_end = (int32_t)prog.ops.size();
            prog.phases.push_back(ph);
        }
        (void)tb_of;
        prog.passes.push_back(pd);
        prog.pass_params.push_back(slot_params);
        for (int gi : absorbed) support |= gates[gi].barrier ? ~0ull : gates[gi].nd_mask;
    }
    prog.support_out = (support & all) == all ? ~0ull : (support & all);
}

// ---- density matrix ----------------------------------------------------
namespace {


// Superoperator sum_k E_k (x) conj(E_k) of a Kraus set on k qubits, as a
// matrix on the 2k vectorised qubits (row qubits first, then column qubits).
std::vector<Z> superop(const Z* kraus, int nk, int k) {
    const int d = 1 << k, D = d * d;
    std::vector<Z> s(D * D, Z{0, 0});
    for (int e = 0; e < nk; ++e) {
        const Z* E = kraus + e * d * d;
        for (int r = 0; r < d; ++r)
            for (int c = 0; c < d; ++c)
                for (int r2 = 0; r2 < d; ++r2)
                    for (int c2 = 0; c2 < d; ++c2) {
                        const Z a = E[r * d + r2], b = E[c * d + c2];  // E[r,r'] * conj(E[c,c'])
                        Z& o = s[(r * d + c) * D + (r2 * d + c2)];
                        o.re += a.re * b.re + a.im * b.im;
                        o.im += a.im * b.re - a.re * b.im;
                    }
    }
    return s;
}

std::vector<Z> matmul(const std::vector<Z>& a, const std::vector<Z>& b, int D) {
    std::vector<Z> c(D * D, Z{0, 0});
    for (int i = 0; i < D; ++i)
        for (int k = 0; k < D; ++k) {
            const Z x = a[i * D + k];
            if (x.re == 0 && x.im == 0) continue;
            for (int j = 0; j < D; ++j) {
                const Z y = b[k * D + j];
                c[i * D + j].re += x.re * y.re - x.im * y.im;
                c[i * D + j].im += x.re * y.im + x.im * y.re;
            }
        }
    return c;
}

// U (x) conj(U) on (row qubits, column qubits), local index row bits high.
std::vector<Z> unitary_superop(const std::vector<Z>& u, int k) {
    return superop(u.data(), 1, k);
}

// A channel superoperator S (4^k x 4^k, index (a << k) | b for the row
// pattern a and column pattern b) is in population / coherence form when it
// maps the populations rho[a,a] only among themselves, by
// T[a][a'] = S[(a,a),(a',a')], and scales each coherence rho[a,b], a != b, by
// D[(a,b)] = S[(a,b),(a,b)]. Depolarizing (1q: T = (1-2p/3) I + (2p/3) X on the
// populations, coherences x (1-4p/3); 2q: T = (1-16p/15) I + (4p/15) J,
// coherences x (1-16p/15)), amplitude damping and phase damping have it, with
// the other entries exactly zero in the FP64 sum over Kraus operators.
bool population_coherence(const std::vector<Z>& S, int k, std::vector<Z>& T, std::vector<Z>& D) {
    const int d = 1 << k, dd = d * d;
    for (int R = 0; R < dd; ++R)
        for (int C = 0; C < dd; ++C) {
            if (R == C || (S[R * dd + C].re == 0.0 && S[R * dd + C].im == 0.0)) continue;
            const int a = R >> k, b = R & (d - 1), a2 = C >> k, b2 = C & (d - 1);
            if (!(a == b && a2 == b2)) return false;
        }
    T.assign(d * d, Z{0, 0});
    D.assign(dd, Z{1, 0});
    for (int a = 0; a < d; ++a)
        for (int a2 = 0; a2 < d; ++a2) T[a * d + a2] = S[((a << k) | a) * dd + ((a2 << k) | a2)];
    for (int R = 0; R < dd; ++R)
        if ((R >> k) != (R & (d - 1))) D[R] = S[R * dd + R];
    return true;
}

// Emits a population / coherence channel on row qubits rq and column qubits
// cq as cheap ops instead of a dense superoperator. With
// V = prod_i X(c_i) CNOT(r_i -> c_i), which maps |a, b> to |a, b ^ a ^ 1..1>
// and is its own inverse, S = V S'' V where S'' scales (a, b'') by
// D[(a, b'' ^ a ^ 1..1)] for b'' != 1..1 (a diagonal) and applies T to the
// row qubits where every column qubit is 1 (T controlled by the c_i). The
// CNOTs and X are permutations, the diagonal a pending factor; only T does
// arithmetic, on a 2^-k share of the entries.
int emit_population_coherence(const std::vector<Z>& T, const std::vector<Z>& D, const std::vector<int>& rq,
                              const std::vector<int>& cq, int src, std::vector<NGate>& out, std::string& err) {
    const int k = (int)rq.size(), d = 1 << k, dd = d * d;
    const std::vector<Z> cnot = {Z{1, 0}, Z{0, 0}, Z{0, 0}, Z{0, 0}, Z{0, 0}, Z{1, 0}, Z{0, 0}, Z{0, 0},
                                 Z{0, 0}, Z{0, 0}, Z{0, 0}, Z{1, 0}, Z{0, 0}, Z{0, 0}, Z{1, 0}, Z{0, 0}};
    const std::vector<Z> x = {Z{0, 0}, Z{1, 0}, Z{1, 0}, Z{0, 0}};
    auto emit_v = [&]() {
        for (int i = 0; i < k; ++i) {
            int rc = analyze_matrix(cnot, {rq[i], cq[i]}, 0, src, out, err);
            if (rc == GQ_OK) rc = analyze_matrix(x, {cq[i]}, 0, src, out, err);
            if (rc != GQ_OK) return rc;
        }
        return (int)GQ_OK;
    };
    int rc = emit_v();
    if (rc != GQ_OK) return rc;
    std::vector<Z> diag(dd * dd, Z{0, 0});
    for (int a = 0; a < d; ++a)
        for (int b2 = 0; b2 < d; ++b2) {
            const int R = (a << k) | b2;
            diag[R * dd + R] = b2 == d - 1 ? Z{1, 0} : D[(a << k) | (b2 ^ a ^ (d - 1))];
        }
    std::vector<int> all(rq);
    all.insert(all.end(), cq.begin(), cq.end());
    rc = analyze_matrix(diag, all, 0, src, out, err);
    uint64_t cmask = 0;
    for (int c : cq) cmask |= 1ull << c;
    if (rc == GQ_OK) rc = analyze_matrix(T, rq, cmask, src, out, err);
    if (rc == GQ_OK) rc = emit_v();
    return rc;
}

std::vector<Z> full_controlled(const gq_op& op) {
    const int tot = op.num_qubits, nt = op.num_qubits - op.num_controls;
    const int dim = 1 << tot, inner = 1 << nt, start = dim - inner;
    std::vector<Z> f(dim * dim, Z{0, 0});
    for (int i = 0; i < start; ++i) f[i * dim + i] = Z{1, 0};
    const Z* m = (const Z*)op.matrix;
    for (int r = 0; r < inner; ++r)
        for (int c = 0; c < inner; ++c) f[(start + r) * dim + start + c] = m[r * inner + c];
    return f;
}

}  // namespace

int dm_gates(int nq, const gq_op* ops, size_t n_ops, std::vector<NGate>& gates, std::string& err, bool structured) {
    auto vec_qubits = [&](const gq_op& op) {
        std::vector<int> q;
        for (int i = 0; i < op.num_qubits; ++i) q.push_back(op.qubits[i] + nq);  // row qubits
        for (int i = 0; i < op.num_qubits; ++i) q.push_back(op.qubits[i]);       // column qubits
        return q;
    };
    // A noise model applies the same few Kraus sets after many gates: each
    // distinct set's superoperator and population / coherence form is
    // computed once per call (keyed by its arity and Kraus entries).
    struct ChanForm {
        std::vector<Z> sop, pop_t, coh_d;
        bool pc = false;
    };
    std::map<std::string, ChanForm> chan_forms;
    auto chan_form = [&](const gq_op& c) -> const ChanForm& {
        const int kk = c.num_qubits, dd = 1 << kk;
        std::string key((const char*)&kk, sizeof(kk));
        key.append((const char*)c.matrix, sizeof(Z) * (size_t)c.num_kraus * dd * dd);
        auto it = chan_forms.find(key);
        if (it != chan_forms.end()) return it->second;
        ChanForm f;
        f.sop = superop((const Z*)c.matrix, c.num_kraus, kk);
        f.pc = kk <= 2 && population_coherence(f.sop, kk, f.pop_t, f.coh_d);
        return chan_forms.emplace(std::move(key), std::move(f)).first->second;
    };
    for (size_t i = 0; i < n_ops; ++i) {
        const gq_op& op = ops[i];
        if (op.kind == GQ_OP_BARRIER) continue;
        if (op.num_qubits < 1 || op.num_qubits > 8) { err = "op " + std::to_string(i) + ": bad qubit count"; return GQ_EINVAL; }
        for (int j = 0; j < op.num_qubits; ++j)
            if (op.qubits[j] < 0 || op.qubits[j] >= nq) { err = "op " + std::to_string(i) + ": qubit out of range"; return GQ_EINVAL; }
        const int k = op.num_qubits;
        const int d = 1 << k;
        if (op.kind == GQ_OP_RESET) {
            // sim/densitymatrix/sim.go:195-217: rho[r,c] += rho[r|m, c|m] on the
            // (0,0) block, everything with the bit set cleared.
            std::vector<Z> s(16, Z{0, 0});
            s[0 * 4 + 0] = Z{1, 0};
            s[0 * 4 + 3] = Z{1, 0};
            int rc = analyze_matrix(s, {op.qubits[0] + nq, op.qubits[0]}, 0, (int)i, gates, err);
            if (rc != GQ_OK) return rc;
            continue;
        }
        if (!op.matrix) { err = "op " + std::to_string(i) + ": no matrix"; return GQ_EINVAL; }
        std::vector<int> rq, cq;  // row and column vector qubits of the op
        for (int j = 0; j < k; ++j) {
            rq.push_back(op.qubits[j] + nq);
            cq.push_back(op.qubits[j]);
        }
        std::vector<Z> sop;
        if (op.kind == GQ_OP_CHANNEL) {
            if (op.num_kraus < 1) { err = "channel without Kraus operators"; return GQ_EINVAL; }
            const ChanForm& cf = chan_form(op);
            if (structured && cf.pc) {
                int rc = emit_population_coherence(cf.pop_t, cf.coh_d, rq, cq, (int)i, gates, err);
                if (rc != GQ_OK) { err = "op " + std::to_string(i) + ": " + err; return rc; }
                continue;
            }
            sop = cf.sop;
        } else {
            std::vector<Z> u;
            if (op.kind == GQ_OP_CONTROLLED)
                u = full_controlled(op);
            else
                u.assign((const Z*)op.matrix, (const Z*)op.matrix + d * d);
            const bool fold = k <= 2 && i + 1 < n_ops && ops[i + 1].kind == GQ_OP_CHANNEL &&
                              ops[i + 1].num_qubits == k && std::equal(ops[i + 1].qubits, ops[i + 1].qubits + k, op.qubits) &&
                              ops[i + 1].matrix && ops[i + 1].num_kraus >= 1;
            const ChanForm* cf = fold ? &chan_form(ops[i + 1]) : nullptr;
            if (fold && !(structured && cf->pc)) {
                // The channel that follows on the same qubits folds into one
                // superoperator S * (U (x) conj(U)).
                sop = matmul(cf->sop, unitary_superop(u, k), d * d);
                ++i;
            } else {
                // U on the row qubits, conj(U) on the column qubits, then the
                // following channel's cheap population / coherence form.
                std::vector<Z> uc(u);
                for (auto& z : uc) z.im = -z.im;
                int rc = analyze_matrix(u, rq, 0, (int)i, gates, err);
                if (rc == GQ_OK) rc = analyze_matrix(uc, cq, 0, (int)i, gates, err);
                if (rc == GQ_OK && fold) {
                    rc = emit_population_coherence(cf->pop_t, cf->coh_d, rq, cq, (int)(i + 1), gates, err);
                    ++i;
                }
                if (rc != GQ_OK) { err = "op " + std::to_string(i) + ": " + err; return rc; }
                continue;
            }
        }
        int rc = analyze_matrix(sop, vec_qubits(op), 0, (int)i, gates, err);
        if (rc != GQ_OK) { err = "op " + std::to_string(i) + ": " + err; return rc; }
    }
    return GQ_OK;
}


// ---- adjoint differentiation ---------------------------------------------
namespace {

std::vector<Z> dagger(const std::vector<Z>& m, int dim) {
    std::vector<Z> o(dim * dim);
    for (int r = 0; r < dim; ++r)
        for (int c = 0; c < dim; ++c) o[r * dim + c] = Z{m[c * dim + r].re, -m[c * dim + r].im};
    return o;
}

std::vector<Z> mul(const std::vector<Z>& a, const std::vector<Z>& b, int dim) {
    std::vector<Z> c(dim * dim, Z{0, 0});
    for (int i = 0; i < dim; ++i)
        for (int k = 0; k < dim; ++k) {
            const Z x = a[i * dim + k];
            for (int j = 0; j < dim; ++j) {
                const Z y = b[k * dim + j];
                c[i * dim + j].re += x.re * y.re - x.im * y.im;
                c[i * dim + j].im += x.re * y.im + x.im * y.re;
            }
        }
    return c;
}

bool zero_control(const std::vector<Z>& m, int k, int p) {
    const int dim = 1 << k, bit = 1 << (k - 1 - p);
    for (int r = 0; r < dim; ++r)
        for (int c = 0; c < dim; ++c) {
            if ((r & bit) && (c & bit)) continue;
            const Z v = m[r * dim + c];
            if (v.re != 0.0 || v.im != 0.0) return false;
        }
    return true;
}

// G as a K_GRAD gate: qubits on whose |0> rows and columns G vanishes become
// controls; the rest is a phase, a diagonal or a dense matrix on <= 4 qubits.
int grad_gate(std::vector<Z> m, std::vector<int> qubits, uint64_t ctrl, int param, std::vector<NGate>& out,
              std::string& err) {
    for (bool found = true; found && !qubits.empty();) {
        found = false;
        const int k = (int)qubits.size();
        for (int p = 0; p < k; ++p)
            if (zero_control(m, k, p)) {
                ctrl |= 1ull << qubits[p];
                m = restrict_to_one(m, k, p);
                qubits.erase(qubits.begin() + p);
                found = true;
                break;
            }
    }
    const int t = (int)qubits.size(), dim = 1 << t;
    NGate g;
    g.type = K_GRAD;
    g.param = param;
    g.ctrl = ctrl;
    g.targets = qubits;
    bool diag = true;
    for (int r = 0; r < dim && diag; ++r)
        for (int c = 0; c < dim; ++c)
            if (r != c && (m[r * dim + c].re != 0.0 || m[r * dim + c].im != 0.0)) {
                diag = false;
                break;
            }
    const bool xtype = t == 1 && m[0].re == 0.0 && m[0].im == 0.0 && m[3].re == 0.0 && m[3].im == 0.0;
    if (t == 0) {
        g.grad_kind = K_PHASE;
        g.data = {m[0]};
    } else if (xtype) {  // Pauli-X generators (RX, and X-type parts): G a_0 = p0 a_1, G a_1 = p1 a_0
        g.grad_kind = K_X;
        g.data = {m[1], m[2]};
    } else if (diag) {
        g.grad_kind = K_DIAG;
        g.data.resize(dim);
        for (int i = 0; i < dim; ++i) g.data[i] = m[i * dim + i];
    } else if (t <= RQ) {
        g.grad_kind = (KType)(K_U1 + (t - 1));
        g.data = m;
    } else {
        err = "derivative acts densely on more than 4 qubits";
        return GQ_EUNSUPPORTED;
    }
    finish(g);
    out.push_back(g);
    return GQ_OK;
}

}  // namespace

int adjoint_gates(int nq, const gq_op* ops, size_t n_ops, size_t n_params, std::vector<NGate>& forward,
                  std::vector<NGate>& reverse, std::vector<int>& fwd_op, std::vector<int>& rev_op, std::string& err) {
    for (size_t i = 0; i < n_ops; ++i) {
        const size_t before = forward.size();
        const gq_op& op = ops[i];
        if (op.kind == GQ_OP_RESET || op.kind == GQ_OP_CHANNEL) {
            err = "op " + std::to_string(i) + ": adjoint differentiation needs a unitary circuit";
            return GQ_EUNSUPPORTED;
        }
        int rc = normalize_op(op, nq, forward, err);
        if (rc != GQ_OK) {
            err = "op " + std::to_string(i) + ": " + err;
            return rc;
        }
        for (size_t k = before; k < forward.size(); ++k) fwd_op.push_back((int)i);
    }
    for (size_t ii = n_ops; ii-- > 0;) {
        const gq_op& op = ops[ii];
        if (op.kind == GQ_OP_BARRIER) continue;
        const int nc = op.kind == GQ_OP_CONTROLLED ? op.num_controls : 0;
        const int k = op.num_qubits - nc, dim = 1 << k;
        uint64_t ctrl = 0;
        for (int c = 0; c < nc; ++c) ctrl |= 1ull << op.qubits[c];
        std::vector<int> qs(op.qubits + nc, op.qubits + op.num_qubits);
        std::vector<Z> u((const Z*)op.matrix, (const Z*)op.matrix + dim * dim);
        const std::vector<Z> ud = dagger(u, dim);
        const size_t before = reverse.size();
        for (int p = 0; p < GQ_MAX_OP_PARAMS; ++p) {
            const int pi = op.param_index[p];
            if (pi < 0) continue;
            if ((size_t)pi >= n_params || !op.dmatrix[p]) {
                err = "op " + std::to_string(ii) + ": parameter index out of range or missing derivative";
                return GQ_EINVAL;
            }
            std::vector<Z> du((const Z*)op.dmatrix[p], (const Z*)op.dmatrix[p] + dim * dim);
            // G = dU U^dagger. For rotations it does not depend on the angle
            // (-i/2 times a Pauli string), but the product's zero entries
            // carry rounding noise of a few ulps that depends on it. Entries
            // below 1e-12 of the largest are zero, so G's structure (controls,
            // diagonal, X-type), and with it the specialised kernels' cache
            // key, stays the same when the angles change.
            std::vector<Z> g = mul(du, ud, dim);
            double gmax = 0.0;
            for (const Z& v : g) gmax = std::max(gmax, std::hypot(v.re, v.im));
            for (Z& v : g)
                if (std::hypot(v.re, v.im) <= 1e-12 * gmax) v = Z{0.0, 0.0};
            int rc = grad_gate(g, qs, ctrl, pi, reverse, err);
            if (rc != GQ_OK) {
                err = "op " + std::to_string(ii) + ": " + err;
                return rc;
            }
        }
        int rc = analyze_matrix(ud, qs, ctrl, (int)ii, reverse, err);
        if (rc != GQ_OK) {
            err = "op " + std::to_string(ii) + ": " + err;
            return rc;
        }
        for (size_t kk = before; kk < reverse.size(); ++kk) rev_op.push_back((int)ii);
    }
    // Ops ahead of the first parameterised op (an initial H layer, say) need no
    // un-applying: no gradient is taken below them.
    size_t keep = 0;
    for (size_t k = 0; k < reverse.size(); ++k)
        if (reverse[k].type == K_GRAD) keep = k + 1;
    reverse.resize(keep);
    rev_op.resize(keep);
    return GQ_OK;
}

int adjoint_segments(int requested, bool c64, size_t n_ops, size_t state_bytes, size_t avail_bytes) {
    const int most = (int)std::max<size_t>(1, n_ops);
    if (requested > 0) return std::min(requested, most);
    // Un-applying gates in FP32 drifts: complex64 circuits of more than 256
    // ops restart the reverse sweep from a stored forward state every 128 ops,
    // up to 8 segments. complex128 circuits need none.
    int segs = (c64 && n_ops > 256) ? (int)std::min<size_t>(8, n_ops / 128) : 1;
    segs = std::max(1, std::min(segs, most));
    // The (segs - 1) checkpoint copies must fit in the memory left for them,
    // keeping kAdjointHeadroom for the program and reduction buffers; with too
    // little room take fewer segments, down to none.
    if (segs > 1 && state_bytes > 0) {
        const size_t usable = avail_bytes > kAdjointHeadroom ? avail_bytes - kAdjointHeadroom : 0;
        const size_t fit = usable / state_bytes;
        segs = (int)std::min<size_t>((size_t)segs, fit + 1);
    }
    return std::max(1, segs);
}

}  // namespace gq

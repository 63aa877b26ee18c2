// Specialised tile-pass kernels: code generation, parameter packing and
// NVRTC compilation (see jit.hpp). Needs no device; the emulator library
// links it for the CPU tests.
#include "jit.hpp"

#include <dlfcn.h>
#include <sys/stat.h>
#include <unistd.h>
#include <nvrtc.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <map>
#include <thread>

namespace gq {

namespace {

// tile_core.cuh as text: the op bodies the generated kernels call.
const char* kTileCore =
#include "tile_core_src.inc"
    ;

std::string hex64(uint64_t v) {
    char b[32];
    std::snprintf(b, sizeof b, "0x%llxull", (unsigned long long)v);
    return b;
}
std::string hex32(uint32_t v) {
    char b[24];
    std::snprintf(b, sizeof b, "0x%xu", v);
    return b;
}
std::string num(long long v) { return std::to_string(v); }

int ctz64(uint64_t v) { return __builtin_ctzll(v); }

// Emits `dst |= ((src >> k) & mask) << q[k]` for every run of bits k of `src`
// (k = 0..n-1) going to consecutive positions q[k].
void emit_deposit(std::string& s, const char* ind, const char* dst, const char* src, const int* q, int n) {
    int k = 0;
    while (k < n) {
        int len = 1;
        while (k + len < n && q[k + len] == q[k] + len) ++len;
        const uint64_t mask = len >= 64 ? ~0ull : ((1ull << len) - 1);
        s += ind;
        s += dst;
        s += " |= ((uint64_t)(";
        s += src;
        s += " >> " + num(k) + ") & " + hex64(mask) + ") << " + num(q[k]) + ";\n";
        k += len;
    }
}

Z zmul(Z a, Z b) { return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
Z zadd(Z a, Z b) { return {a.re + b.re, a.im + b.im}; }
Z zdiv(Z a, Z b) {
    const double d = b.re * b.re + b.im * b.im;
    return {(a.re * b.re + a.im * b.im) / d, (a.im * b.re - a.re * b.im) / d};
}
double zabs(Z a) { return std::hypot(a.re, a.im); }

using Pend = std::vector<uint32_t>;  // sorted atom ids

// Code generation state of one pass.
struct Gen {
    const Program& pr;
    JitPlan& out;
    uint32_t cap;
    uint32_t np = 0;
    bool overflow = false;
    std::map<std::pair<uint8_t, uint32_t>, uint32_t> atom_ids;
    std::map<std::string, uint32_t> entry_ids;  // dedupe key -> parameter offset

    Gen(const Program& p, JitPlan& o, uint32_t c) : pr(p), out(o), cap(c) {}

    uint32_t atom(uint8_t kind, uint32_t ref) {
        auto it = atom_ids.find({kind, ref});
        if (it != atom_ids.end()) return it->second;
        const uint32_t id = (uint32_t)out.atoms.size();
        out.atoms.push_back({kind, ref});
        atom_ids[{kind, ref}] = id;
        return id;
    }
    uint32_t add_entry(const std::string& key, JitEntry e) {
        auto it = entry_ids.find(key);
        if (it != entry_ids.end()) return it->second;
        const uint32_t n = e.kind == 0 ? e.count : 1;
        if (np + n > cap) {
            overflow = true;
            return 0;
        }
        const uint32_t off = np;
        np += n;
        out.entries.push_back(std::move(e));
        entry_ids[key] = off;
        return off;
    }
    uint32_t copy(uint32_t ref, uint32_t count) {
        return add_entry("C" + num(ref) + ":" + num(count), JitEntry{0, ref, count, {}, {}});
    }
    uint32_t shear_t(uint32_t op) { return add_entry("T" + num(op), JitEntry{1, op, 1, {}, {}}); }
    // Offset of the 2^nl shear values of chain `fid` (one per predicate combination).
    uint32_t chain_t(uint32_t fid, int nl) {
        const std::string key = "F" + num(fid);
        auto it = entry_ids.find(key);
        if (it != entry_ids.end()) return it->second;
        const uint32_t n = 1u << nl;
        if (np + n > cap) {
            overflow = true;
            return 0;
        }
        const uint32_t off = np;
        for (uint32_t e = 0; e < n; ++e) out.entries.push_back(JitEntry{3, fid * 4 + e, 1, {}, {}});
        np += n;
        entry_ids[key] = off;
        return off;
    }
    // prod(n0) / prod(d0) with common atoms cancelled, and its dedupe key.
    static std::string reduce(const Pend& n0, const Pend& d0, Pend& n, Pend& d) {
        n.clear();
        d.clear();
        std::set_difference(n0.begin(), n0.end(), d0.begin(), d0.end(), std::back_inserter(n));
        std::set_difference(d0.begin(), d0.end(), n0.begin(), n0.end(), std::back_inserter(d));
        std::string key;
        for (uint32_t a : n) key += num(a) + ",";
        key += "/";
        for (uint32_t a : d) key += num(a) + ",";
        return key;
    }
    // Offset of prod(num) / prod(den) after cancelling common atoms; -1 if 1.
    long ratio(const Pend& n0, const Pend& d0) {
        Pend n, d;
        const std::string key = reduce(n0, d0, n, d);
        if (n.empty() && d.empty()) return -1;
        return add_entry("P" + key, JitEntry{2, 0, 1, n, d});
    }
    // Offset of a block of consecutive ratios prod(nums[e]) / prod(dens[e]).
    uint32_t ratio_table(const std::vector<Pend>& nums, const std::vector<Pend>& dens) {
        std::vector<Pend> ns(nums.size()), ds(nums.size());
        std::string key = "Q";
        for (size_t e = 0; e < nums.size(); ++e) key += reduce(nums[e], dens[e], ns[e], ds[e]) + ";";
        auto it = entry_ids.find(key);
        if (it != entry_ids.end()) return it->second;
        if (np + nums.size() > cap) {
            overflow = true;
            return 0;
        }
        const uint32_t off = np;
        for (size_t e = 0; e < nums.size(); ++e) out.entries.push_back(JitEntry{2, 0, 1, ns[e], ds[e]});
        np += (uint32_t)nums.size();
        entry_ids[key] = off;
        return off;
    }
};

void pend_add(Pend& p, uint32_t a) { p.insert(std::upper_bound(p.begin(), p.end(), a), a); }

// A register slot's pending factor as a function of the phase's uniform
// predicates: entry c holds the atoms that apply when predicate k holds for
// exactly the bits k set in c.
using PendT = std::vector<Pend>;

}  // namespace

namespace {
template <class V>
void put_key(std::string& k, const V& v) {
    k.append(reinterpret_cast<const char*>(&v), sizeof(V));
}
}  // namespace

// Whether the `count` pool entries from `at` are all real (the generator then
// emits the real-matrix op bodies, which read only the real parts).
static bool pool_real(const Program& pr, uint32_t at, uint32_t count) {
    for (uint32_t k = 0; k < count; ++k)
        if (pr.pool[at + k].im != 0.0) return false;
    return true;
}

std::string jit_plan_key(const Program& pr, size_t pi, bool c64, int threads, int min_blocks, bool persistent,
                         bool dual) {
    const PassDesc& pd = pr.passes[pi];
    uint32_t op_base, pool_base;
    jit_bases(pr, pi, &op_base, &pool_base);
    std::string key;
    key.reserve(4096);
    put_key(key, (int)c64);
    put_key(key, threads);
    put_key(key, min_blocks);
    put_key(key, (int)persistent);
    put_key(key, (int)dual);
    put_key(key, pd.m);
    put_key(key, pd.n_outer);
    put_key(key, pd.n_phases);
    key.append((const char*)pd.tile_q, sizeof(int32_t) * pd.m);
    key.append((const char*)pd.acol, sizeof(uint32_t) * pd.m);
    key.append((const char*)pd.outer_q, sizeof(int32_t) * pd.n_outer);
    for (int p = 0; p < pd.n_phases; ++p) {
        const PhaseDesc& ph = pr.phases[pd.phase0 + p];
        key.append((const char*)ph.rslot, sizeof(ph.rslot));
        key.append((const char*)ph.tlo_slot, sizeof(ph.tlo_slot));
        key.append((const char*)ph.thi_slot, sizeof(ph.thi_slot));
        key.append((const char*)ph.tlo_glob, sizeof(ph.tlo_glob));
        key.append((const char*)ph.thi_glob, sizeof(ph.thi_glob));
        put_key(key, ph.op_end - ph.op_begin);
        for (int o = ph.op_begin; o < ph.op_end; ++o) {
            const KOp& op = pr.ops[o];
            const uint8_t b[8] = {op.type, op.t0, op.t1, op.t2, op.creg, op.nreg, op.flags, (uint8_t)op.slot};
            key.append((const char*)b, 8);
            put_key(key, op.mat - pool_base);
            put_key(key, op.cmask);
            put_key(key, op.dmask);
            put_key(key, op.ridx);
            bool dense = op.type == K_U1 && op.cmask;
            if (op.type == K_U1 && !op.cmask) {
                double t;
                Z l, a, c;
                const bool dec = u1_decompose(&pr.pool[op.mat], &t, &l, &a, &c);
                put_key(key, (int)dec);
                dense = !dec;
            }
            // dense one- and two-qubit matrices with real entries take the real op bodies
            if (!dual && dense) put_key(key, (int)pool_real(pr, op.mat, 4));
            if (!dual && op.type == K_U2) put_key(key, (int)pool_real(pr, op.mat, 16));
        }
    }
    if (!dual)  // which one-qubit chains the forward kernel fuses
        for (const ChainCand& cc : jit_chains(pr, pi)) put_key(key, (int)cc.fusable);
    return key;
}

bool u1_decompose(const Z* m, double* t, Z* lam, Z* post0, Z* post1) {
    // unitary: columns orthonormal
    const double n0 = m[0].re * m[0].re + m[0].im * m[0].im + m[2].re * m[2].re + m[2].im * m[2].im;
    const double n1 = m[1].re * m[1].re + m[1].im * m[1].im + m[3].re * m[3].re + m[3].im * m[3].im;
    const Z ip = {m[0].re * m[1].re + m[0].im * m[1].im + m[2].re * m[3].re + m[2].im * m[3].im,
                  m[0].re * m[1].im - m[0].im * m[1].re + m[2].re * m[3].im - m[2].im * m[3].re};
    if (std::fabs(n0 - 1) > 1e-12 || std::fabs(n1 - 1) > 1e-12 || zabs(ip) > 1e-12) return false;
    const double c = zabs(m[0]), s = zabs(m[2]);
    if (c < 1e-150 || s < 1e-150) return false;
    const Z g = {m[0].re / c, m[0].im / c};
    const Z eph = zdiv({m[2].re / s, m[2].im / s}, g);      // e^{i phi}
    const Z elam = zdiv({-m[1].re / s, -m[1].im / s}, g);   // e^{i lambda}
    *t = s / c;
    *lam = elam;
    *post0 = {g.re * c, g.im * c};
    *post1 = zmul(*post0, eph);
    return true;
}

void jit_bases(const Program& pr, size_t pi, uint32_t* op_base, uint32_t* pool_base) {
    const PassDesc& pd = pr.passes[pi];
    const uint32_t ob = pd.n_phases > 0 ? (uint32_t)pr.phases[pd.phase0].op_begin : 0;
    *op_base = ob;
    *pool_base = ob < pr.ops.size() ? pr.ops[ob].mat : 0;
}

namespace {

// Register bits an op reads or mixes in any way (targets, controls, the
// register part of a diagonal's table index).
uint32_t op_reg_bits(const KOp& op) {
    uint32_t b = op.creg;
    const uint8_t kind = op.type == K_GRAD ? op.flags : op.type;
    switch (kind) {
        case K_U1: case K_X: b |= 1u << op.t0; break;
        case K_U2: case K_SWAP: b |= (1u << op.t0) | (1u << op.t1); break;
        case K_U3: b |= (1u << op.t0) | (1u << op.t1) | (1u << op.t2); break;
        case K_U4: case K_PAIRSUM: b = 15u; break;
        case K_RESET: b = 15u; break;  // nonlinear: commutes with no unitary on any register bit
        case K_DIAG:
            for (int k = 0; k < RQ; ++k)
                for (int j = 0; j < NREG; ++j)
                    if (((op.ridx >> (4 * j)) & 15u) != ((op.ridx >> (4 * (j ^ (1 << k)))) & 15u)) b |= 1u << k;
            break;
        default: break;
    }
    return b;
}

// The product of a chain's ops (row major) when its predicates take the
// values of the bits of e.
void chain_matrix(const Program& pr, uint32_t op_base, const JitChain& ch, int e, Z* out) {
    Z m[4] = {{1, 0}, {0, 0}, {0, 0}, {1, 0}};
    for (size_t i = 0; i < ch.ops.size(); ++i) {
        const KOp& op = pr.ops[op_base + ch.ops[i]];
        Z f[4];
        if (op.type == K_U1) {
            for (int k = 0; k < 4; ++k) f[k] = pr.pool[op.mat + k];
        } else {
            if (ch.pred[i] >= 0 && !((e >> ch.pred[i]) & 1)) continue;
            const bool pure = op.flags & 1;
            f[0] = f[3] = Z{0, 0};
            f[1] = pure ? Z{1, 0} : pr.pool[op.mat];
            f[2] = pure ? Z{1, 0} : pr.pool[op.mat + 1];
        }
        const Z r[4] = {zadd(zmul(f[0], m[0]), zmul(f[1], m[2])), zadd(zmul(f[0], m[1]), zmul(f[1], m[3])),
                        zadd(zmul(f[2], m[0]), zmul(f[3], m[2])), zadd(zmul(f[2], m[1]), zmul(f[3], m[3]))};
        for (int k = 0; k < 4; ++k) m[k] = r[k];
    }
    for (int k = 0; k < 4; ++k) out[k] = m[k];
}

}  // namespace

std::vector<ChainCand> jit_chains(const Program& pr, size_t pi) {
    const PassDesc& pd = pr.passes[pi];
    uint32_t op_base, pool_base;
    jit_bases(pr, pi, &op_base, &pool_base);
    uint64_t outer = 0;
    for (int k = 0; k < pd.n_outer; ++k) outer |= 1ull << pd.outer_q[k];
    std::vector<ChainCand> res;
    for (int p = 0; p < pd.n_phases; ++p) {
        const PhaseDesc& ph = pr.phases[pd.phase0 + p];
        for (int r = 0; r < RQ; ++r) {
            auto element = [&](const KOp& op) {
                if (op.t0 != r || op.creg) return false;
                if (op.type == K_U1) return op.cmask == 0;
                return op.type == K_X && (op.cmask & ~outer) == 0;
            };
            std::vector<int> run;
            auto finish = [&]() {
                int first = -1, last = -1, nu = 0;
                for (size_t i = 0; i < run.size(); ++i)
                    if (pr.ops[run[i]].type == K_U1) {
                        if (first < 0) first = (int)i;
                        last = (int)i;
                        ++nu;
                    }
                if (nu >= 2) {
                    ChainCand cc;
                    cc.phase = p;
                    cc.pmask[0] = cc.pmask[1] = 0;
                    int np = 0;
                    bool ok = true;
                    for (int i = first; i <= last; ++i) {
                        const KOp& op = pr.ops[run[i]];
                        int8_t pv = -1;
                        if (op.cmask) {
                            int k = 0;
                            while (k < np && cc.pmask[k] != op.cmask) ++k;
                            if (k == np) {
                                if (np == 2) {
                                    ok = false;
                                    break;
                                }
                                cc.pmask[np++] = op.cmask;
                            }
                            pv = (int8_t)k;
                        }
                        cc.chain.ops.push_back((uint32_t)run[i] - op_base);
                        cc.chain.pred.push_back(pv);
                    }
                    if (ok) {
                        cc.fusable = true;
                        for (int e = 0; e < (1 << np) && cc.fusable; ++e) {
                            Z mm[4], l, a0, a1;
                            double t;
                            chain_matrix(pr, op_base, cc.chain, e, mm);
                            cc.fusable = u1_decompose(mm, &t, &l, &a0, &a1);
                        }
                        res.push_back(cc);
                    }
                }
                run.clear();
            };
            for (int o = ph.op_begin; o < ph.op_end; ++o) {
                const KOp& op = pr.ops[o];
                if (!(op_reg_bits(op) & (1u << r))) continue;
                if (element(op)) {
                    run.push_back(o);
                } else {
                    finish();
                }
            }
            finish();
        }
    }
    return res;
}

namespace {

enum PlanResult { PLAN_OK = 0, PLAN_UNCOVERED = 1, PLAN_OVERFLOW = 2 };

// jit_plan with at most `kmax` uniform predicates per phase.
PlanResult plan_forward(const Program& pr, size_t pi, bool c64, int threads, int min_blocks, bool persistent,
                        JitPlan& out, bool host, int kmax) {
    const PassDesc& pd = pr.passes[pi];
    uint32_t op_base, pool_base;
    jit_bases(pr, pi, &op_base, &pool_base);
    const int m = pd.m, tbits = m - RQ;
    if (tbits < 0 || (1 << tbits) != threads) return PLAN_UNCOVERED;
    out.atoms.clear();
    out.entries.clear();
    out.phase_shears.clear();
    out.chains.clear();
    out.phase_chains.clear();
    Gen gen(pr, out, c64 ? 3900u : 1950u);  // 32 KB of kernel parameters
    uint64_t outer_mask = 0;
    for (int k = 0; k < pd.n_outer; ++k) outer_mask |= 1ull << pd.outer_q[k];
    const std::vector<ChainCand> cands = jit_chains(pr, pi);

    // ---- prologue: CTA base, staging columns (thread bits = tile bits [0, tbits))
    auto make_pro = [&](const char* ctav) {
        std::string r;
        r += "    uint64_t base = 0;\n";
        emit_deposit(r, "    ", "base", ctav, pd.outer_q, pd.n_outer);
        r += "    uint64_t gt = base;\n    uint32_t stt = 0;\n";
        emit_deposit(r, "    ", "gt", "t", pd.tile_q, tbits);
        for (int k = 0; k < tbits; ++k)
            r += "    stt ^= (0u - ((t >> " + num(k) + ") & 1u)) & " + hex32(pd.acol[k]) + ";\n";
        r += "    (void)gt;\n    (void)stt;\n";
        return r;
    };
    const std::string pro = make_pro("cta");
    uint64_t G[NREG];
    uint32_t S[NREG];
    for (int it = 0; it < NREG; ++it) {
        G[it] = 0;
        S[it] = 0;
        for (int k = 0; k < RQ; ++k)
            if ((it >> k) & 1) {
                G[it] |= 1ull << pd.tile_q[tbits + k];
                S[it] ^= pd.acol[tbits + k];
            }
    }
    std::string seg_in = "    {\n        cplx<T> v[16];\n";
    for (int it = 0; it < NREG; ++it) seg_in += "        v[" + num(it) + "] = st[gt | " + hex64(G[it]) + "];\n";
    for (int it = 0; it < NREG; ++it) seg_in += "        sm[stt ^ " + hex32(S[it]) + "] = v[" + num(it) + "];\n";
    seg_in += "    }\n";
    std::string seg_out = "    {\n        cplx<T> v[16];\n";
    for (int it = 0; it < NREG; ++it) seg_out += "        v[" + num(it) + "] = sm[stt ^ " + hex32(S[it]) + "];\n";
    for (int it = 0; it < NREG; ++it) seg_out += "        st[gt | " + hex64(G[it]) + "] = v[" + num(it) + "];\n";
    seg_out += "    }\n";

    std::vector<std::string> seg_ph;
    // The first phase may load its amplitudes straight from global memory and
    // the last store them straight back (no staging through shared memory, two
    // barriers fewer) when the phase's lanes run along the lowest qubits
    // (128-byte runs, as the staging copies) and each register bit is one
    // tile qubit. direct_in / direct_out record whether they do.
    bool direct_in = false, direct_out = false;
    const int lane_run = c64 ? 4 : 3;  // lowest qubits a 128-byte run spans
    for (int p = 0; p < pd.n_phases; ++p) {
        const PhaseDesc& ph = pr.phases[pd.phase0 + p];
        out.phase_shears.emplace_back();
        uint32_t tslot[MAX_TILE];
        int tq[MAX_TILE];
        for (int k = 0; k < tbits; ++k) {
            const uint32_t sv = k < 4 ? ph.tlo_slot[1u << k] : ph.thi_slot[1u << (k - 4)];
            const uint64_t g = k < 4 ? ph.tlo_glob[1u << k] : ph.thi_glob[1u << (k - 4)];
            if (g == 0 || (g & (g - 1))) return PLAN_UNCOVERED;
            tslot[k] = sv;
            tq[k] = ctz64(g);
        }
        for (int v = 0; v < TLO && v < (1 << tbits); ++v) {  // the tables are XOR / OR of those columns
            uint32_t sv = 0;
            uint64_t g = 0;
            for (int k = 0; k < 4 && k < tbits; ++k)
                if ((v >> k) & 1) {
                    sv ^= tslot[k];
                    g |= 1ull << tq[k];
                }
            if (sv != ph.tlo_slot[v] || g != ph.tlo_glob[v]) return PLAN_UNCOVERED;
        }
        // Uniform predicates: controls of X-type and phase ops that lie in the
        // CTA's outer bits hold for a whole CTA. Such an op costs no arithmetic:
        // the X swaps registers under a CTA-uniform branch, and both become
        // predicate-dependent pending factors, read from a table indexed by
        // the predicates' values when they are applied.
        std::vector<uint64_t> upred;
        for (int oa = ph.op_begin; oa < ph.op_end && (int)upred.size() < kmax; ++oa) {
            const KOp& op = pr.ops[oa];
            if (op.type != K_X || !op.cmask || (op.cmask & ~outer_mask)) continue;
            if (std::find(upred.begin(), upred.end(), op.cmask) == upred.end()) upred.push_back(op.cmask);
        }
        const int K = (int)upred.size(), NC = 1 << K;
        auto upred_of = [&](uint64_t cmask) {
            for (int k = 0; k < K; ++k)
                if (upred[k] == cmask) return k;
            return -1;
        };
        // Chains fused into one unitary per predicate combination, applied
        // at the chain's last op; its other ops are skipped.
        out.phase_chains.emplace_back();
        struct Fused {
            uint32_t fid;
            int nl, ubit[2];
        };
        std::map<int, Fused> fused_at;
        std::vector<char> skip(ph.op_end - ph.op_begin, 0);
        for (const ChainCand& cc : cands) {
            if (cc.phase != p || !cc.fusable) continue;
            Fused f;
            f.nl = 0;
            bool ok = true;
            for (int k = 0; k < 2 && cc.pmask[k]; ++k) {
                f.ubit[k] = upred_of(cc.pmask[k]);
                ok = ok && f.ubit[k] >= 0;
                ++f.nl;
            }
            if (!ok) continue;
            f.fid = (uint32_t)out.chains.size();
            out.chains.push_back(cc.chain);
            out.phase_chains.back().push_back(f.fid);
            for (size_t i = 0; i + 1 < cc.chain.ops.size(); ++i) skip[op_base + cc.chain.ops[i] - ph.op_begin] = 1;
            fused_at[(int)(op_base + cc.chain.ops.back())] = f;
        }

        std::string b = "    {\n        uint32_t sb = 0;\n        uint64_t g0 = base;\n";
        for (int k = 0; k < tbits; ++k)
            b += "        sb ^= (0u - ((t >> " + num(k) + ") & 1u)) & " + hex32(tslot[k]) + ";\n";
        emit_deposit(b, "        ", "g0", "t", tq, tbits);
        b += "        (void)g0;\n";
        if (K > 0) {
            b += "        const uint32_t pc = 0u";
            for (int k = 0; k < K; ++k)
                b += " | (((base & " + hex64(upred[k]) + ") == " + hex64(upred[k]) + ") ? " + hex32(1u << k) + " : 0u)";
            b += ";\n";
        }
        // global offset of each register slot: register bit k is the tile
        // qubit whose staging column is rslot[1 << k]
        uint64_t greg[NREG];
        bool direct = tbits >= lane_run;
        for (int k = 0; k < lane_run && direct; ++k) direct = tq[k] == k;
        for (int k = 0; k < RQ && direct; ++k) {
            int hit = -1;
            for (int bb = 0; bb < m; ++bb)
                if (pd.acol[bb] == ph.rslot[1 << k]) hit = bb;
            if (hit < 0) direct = false;
            else greg[1 << k] = 1ull << pd.tile_q[hit];
        }
        if (direct) {
            greg[0] = 0;
            for (int j = 1; j < NREG; ++j) greg[j] = greg[j & (j - 1)] | greg[j & -j];
        }
        // (persistent CTAs find their tile in shared memory, prefetched)
        const bool load_global = direct && p == 0 && !persistent;
        const bool store_global = direct && p == pd.n_phases - 1;
        if (p == 0) direct_in = load_global;
        if (p == pd.n_phases - 1) direct_out = store_global;
        b += "        cplx<T> a[16];\n";
        for (int j = 0; j < NREG; ++j)
            b += load_global ? "        a[" + num(j) + "] = st[g0 | " + hex64(greg[j]) + "];\n"
                             : "        a[" + num(j) + "] = sm[sb ^ " + hex32(ph.rslot[j]) + "];\n";
        // the last phase's registers are loaded: a persistent CTA may refill
        // the tile buffer with its next tile from here on
        if (store_global && persistent) {
            // every thread's registers of this tile are loaded: each thread
            // refills its own sixteen slots with the next tile's amplitudes
            b += "        __syncthreads();\n        if (nxt < ntiles) {\n            uint64_t nb = 0;\n";
            emit_deposit(b, "            ", "nb", "nxt", pd.outer_q, pd.n_outer);
            b += "            const uint64_t gq = nb | (g0 ^ base);\n";
            for (int j = 0; j < NREG; ++j)
                b += "            cp_async_amp(sm + (sb ^ " + hex32(ph.rslot[j]) + "), st + (gq | " + hex64(greg[j]) + "));\n";
            b += "        }\n        cp_async_commit();\n";
        }

        PendT pend[NREG];
        for (int j = 0; j < NREG; ++j) pend[j].assign(NC, Pend());
        auto add_all = [&](int j, uint32_t atom) {
            for (Pend& e : pend[j]) pend_add(e, atom);
        };
        // Multiplies a[j] by num[c] / den[c] for the current predicate values c.
        auto scale_by = [&](int j, const PendT& nm, const PendT& dn) {
            uint32_t dep = 0;  // predicates the ratio depends on
            Pend n0, d0, n1, d1;
            std::vector<std::string> keys(NC);
            for (int c = 0; c < NC; ++c) keys[c] = Gen::reduce(nm[c], dn[c], n0, d0);
            for (int c = 0; c < NC; ++c)
                for (int k = 0; k < K; ++k)
                    if (keys[c] != keys[c ^ (1 << k)]) dep |= 1u << k;
            if (dep == 0) {
                const long off = gen.ratio(nm[0], dn[0]);
                if (off >= 0) b += "        a[" + num(j) + "] = cmul(p.m[" + num(off) + "], a[" + num(j) + "]);\n";
                return;
            }
            std::vector<int> bits;
            for (int k = 0; k < K; ++k)
                if ((dep >> k) & 1) bits.push_back(k);
            PendT tn, td;
            for (int e = 0; e < (1 << (int)bits.size()); ++e) {
                int c = 0;
                for (size_t i = 0; i < bits.size(); ++i)
                    if ((e >> i) & 1) c |= 1 << bits[i];
                tn.push_back(nm[c]);
                td.push_back(dn[c]);
            }
            const uint32_t off = gen.ratio_table(tn, td);
            std::string idx;
            for (size_t i = 0; i < bits.size(); ++i) {
                if (i) idx += " | ";
                idx += "(((pc >> " + num(bits[i]) + ") & 1u) << " + num((long long)i) + ")";
            }
            b += "        a[" + num(j) + "] = cmul(p.m[" + num(off) + " + (" + idx + ")], a[" + num(j) + "]);\n";
        };
        // Groups of an op on target bits `tm` under register controls `creg`.
        auto groups = [&](uint32_t tm, uint32_t creg) {
            std::vector<std::vector<int>> gs;
            for (int j = 0; j < NREG; ++j) {
                if ((j & tm) || (j & creg) != creg) continue;
                std::vector<int> g;
                for (int sub = 0; sub < NREG; ++sub)
                    if ((sub & ~tm) == 0) g.push_back(j | sub);
                gs.push_back(g);
            }
            return gs;
        };
        auto normalize = [&](const std::vector<int>& g) {
            for (size_t i = 1; i < g.size(); ++i)
                if (pend[g[i]] != pend[g[0]]) {
                    scale_by(g[i], pend[g[i]], pend[g[0]]);
                    pend[g[i]] = pend[g[0]];
                }
        };
        // Other phases with run-time controls accumulate per register-control
        // pattern M into a per-thread factor rq<M> (one complex multiply per
        // thread and op), applied to the slots of M before an op that mixes
        // them with other slots, and at the end of the phase.
        uint32_t racc = 0, rdecl = 0;  // bit M: rq<M> pending / declared
        auto flush = [&](uint32_t mixed) {
            for (uint32_t M = 0; M < NREG; ++M) {
                if (!((racc >> M) & 1u) || ((M & mixed) == 0 && mixed != 0xffffffffu)) continue;
                for (int j = 0; j < NREG; ++j)
                    if ((j & (int)M) == (int)M)
                        b += "        a[" + num(j) + "] = cmul(rq" + num(M) + ", a[" + num(j) + "]);\n";
                racc &= ~(1u << M);
            }
        };
        auto resolve = [&](int j) {
            bool any = false;
            for (const Pend& e : pend[j]) any = any || !e.empty();
            if (!any) return;
            scale_by(j, pend[j], PendT(NC));
            pend[j].assign(NC, Pend());
        };

        for (int oa = ph.op_begin; oa < ph.op_end; ++oa) {
            const KOp& op = pr.ops[oa];
            if (op.type == K_GRAD || op.type == K_NONE || op.type > K_RESET) return PLAN_UNCOVERED;
            if (skip[oa - ph.op_begin]) continue;
            // indices relative to the pass (its first op and first pool entry),
            // so the kernel text and plan do not depend on the pass's position
            const uint32_t o = (uint32_t)oa - op_base, rm = op.mat - pool_base;
            const std::string creg = num(op.creg) + "u";
            const std::string C = op.creg ? "true" : "false";
            std::string cond;
            if (op.cmask) cond = "if ((g0 & " + hex64(op.cmask) + ") == " + hex64(op.cmask) + ") ";
            const int uk = op.cmask ? upred_of(op.cmask) : -1;
            const std::string S0 = num(op.t0), S1 = num(op.t1), S2 = num(op.t2);
            auto pm = [&](uint32_t off) { return "PMat<T>{p.m + " + num(off) + "}"; };
            switch (op.type) {  // register bits the op mixes
                case K_U1: case K_X: flush(1u << op.t0); break;
                case K_U2: case K_SWAP: flush((1u << op.t0) | (1u << op.t1)); break;
                case K_U3: flush((1u << op.t0) | (1u << op.t1) | (1u << op.t2)); break;
                case K_U4: case K_RESET: flush(0xffffffffu); break;
                default: break;
            }
            switch (op.type) {
                case K_U1: {
                    const uint32_t tm = 1u << op.t0;
                    double tv;
                    Z lam, p0, p1;
                    const auto fu = fused_at.find(oa);
                    if (fu != fused_at.end()) {
                        // the chain's product under this CTA's predicate values:
                        // atoms and shear read at index e (the chain's predicates)
                        const Fused& f = fu->second;
                        auto local = [&](int c) {
                            int e = 0;
                            for (int k = 0; k < f.nl; ++k) e |= ((c >> f.ubit[k]) & 1) << k;
                            return (uint32_t)e;
                        };
                        const auto gs = groups(tm, 0u);
                        for (const auto& g : gs) {
                            for (int c = 0; c < NC; ++c) pend_add(pend[g[1]][c], gen.atom(4, f.fid * 4 + local(c)));
                            normalize(g);
                        }
                        std::string idx = "0u";
                        for (int k = 0; k < f.nl; ++k)
                            idx += " | (((pc >> " + num(f.ubit[k]) + ") & 1u) << " + num(k) + ")";
                        b += "        k_shear<T, " + S0 + ", false>(a, p.m[" + num(gen.chain_t(f.fid, f.nl)) + " + (" +
                             idx + ")].x, 0u);\n";
                        for (const auto& g : gs) {
                            pend[g[1]] = pend[g[0]];
                            for (int c = 0; c < NC; ++c) {
                                pend_add(pend[g[1]][c], gen.atom(6, f.fid * 4 + local(c)));
                                pend_add(pend[g[0]][c], gen.atom(5, f.fid * 4 + local(c)));
                            }
                        }
                    } else if (!op.cmask && u1_decompose(&pr.pool[op.mat], &tv, &lam, &p0, &p1)) {
                        const uint32_t a_l = gen.atom(1, (uint32_t)o), a_0 = gen.atom(2, (uint32_t)o),
                                       a_1 = gen.atom(3, (uint32_t)o);
                        const auto gs = groups(tm, op.creg);
                        for (const auto& g : gs) {
                            add_all(g[1], a_l);
                            normalize(g);
                        }
                        b += "        k_shear<T, " + S0 + ", " + C + ">(a, p.m[" + num(gen.shear_t((uint32_t)o)) +
                             "].x, " + creg + ");\n";
                        for (const auto& g : gs) {
                            pend[g[1]] = pend[g[0]];
                            add_all(g[1], a_1);
                            add_all(g[0], a_0);
                        }
                        out.phase_shears.back().push_back((uint32_t)o);
                    } else {
                        for (const auto& g : groups(tm, op.creg)) normalize(g);
                        const char* fn = pool_real(pr, op.mat, 4) ? "k_u1r<T, " : "k_u1<T, ";
                        b += "        " + cond + fn + S0 + ", " + C + ">(a, " + pm(gen.copy(rm, 4)) + ", " + creg +
                             ");\n";
                    }
                    break;
                }
                case K_U2: {
                    for (const auto& g : groups((1u << op.t0) | (1u << op.t1), op.creg)) normalize(g);
                    const char* fn = pool_real(pr, op.mat, 16) ? "k_u2r<T, " : "k_u2<T, ";
                    b += "        " + cond + fn + S0 + ", " + S1 + ", " + C + ">(a, " + pm(gen.copy(rm, 16)) + ", " +
                         creg + ");\n";
                    break;
                }
                case K_U3:
                    for (const auto& g : groups((1u << op.t0) | (1u << op.t1) | (1u << op.t2), op.creg)) normalize(g);
                    b += "        " + cond + "k_u3<T, " + S0 + ", " + S1 + ", " + S2 + ">(a, " +
                         pm(gen.copy(rm, 64)) + ", " + creg + ");\n";
                    break;
                case K_U4:
                    for (const auto& g : groups(15u, 0u)) normalize(g);
                    b += "        " + cond + "k_u4<T>(a, " + pm(gen.copy(rm, 256)) + ", sm, sb, phases[" + num(p) +
                         "].rslot);\n";
                    break;
                case K_X: {
                    const uint32_t tm = 1u << op.t0;
                    const bool pure = op.flags & 1;
                    if (op.cmask && uk < 0) {
                        for (const auto& g : groups(tm, op.creg)) normalize(g);
                        b += "        " + cond + "k_x<T, " + S0 + ", " + C + ">(a, " +
                             (pure ? std::string("pool") : pm(gen.copy(rm, 2))) + ", " + creg + ", " +
                             (pure ? "true" : "false") + ");\n";
                    } else {
                        // a permutation (for a uniform predicate, under a CTA-uniform
                        // branch); the phases p0, p1 become pending factors
                        b += "        " + std::string(uk >= 0 ? "if ((pc >> " + num(uk) + ") & 1u) " : "") + "k_x<T, " +
                             S0 + ", " + C + ">(a, pool, " + creg + ", true);\n";
                        for (const auto& g : groups(tm, op.creg))
                            for (int c = 0; c < NC; ++c) {
                                if (uk >= 0 && !((c >> uk) & 1)) continue;
                                std::swap(pend[g[0]][c], pend[g[1]][c]);
                                if (!pure) {
                                    pend_add(pend[g[0]][c], gen.atom(0, rm));
                                    pend_add(pend[g[1]][c], gen.atom(0, rm + 1));
                                }
                            }
                    }
                    break;
                }
                case K_SWAP: {
                    std::vector<std::pair<int, int>> prs;
                    for (int j = 0; j < NREG; ++j) {
                        if (!(j & (1 << op.t0)) || (j & (1 << op.t1))) continue;
                        if ((j & op.creg) != op.creg) continue;
                        prs.push_back({j, (j & ~(1 << op.t0)) | (1 << op.t1)});
                    }
                    if (op.cmask)
                        for (const auto& q : prs) normalize({q.first, q.second});
                    else
                        for (const auto& q : prs) std::swap(pend[q.first], pend[q.second]);
                    b += "        " + cond + "k_swap<T, " + S0 + ", " + S1 + ">(a, " + creg + ");\n";
                    break;
                }
                case K_PHASE:
                    if (op.cmask && uk < 0) {
                        const uint32_t M = op.creg;
                        const std::string rv = "rq" + num(M), v = "p.m[" + num(gen.copy(rm, 1)) + "]";
                        if ((racc >> M) & 1u) {
                            b += "        " + cond + rv + " = cmul(" + v + ", " + rv + ");\n";
                        } else {
                            b += "        " + std::string((rdecl >> M) & 1u ? "" : "cplx<T> ") + rv +
                                 " = cplx<T>{T(1), T(0)};\n        " + cond + rv + " = " + v + ";\n";
                            racc |= 1u << M;
                            rdecl |= 1u << M;
                        }
                    } else {
                        const uint32_t a_s = gen.atom(0, rm);
                        for (int j = 0; j < NREG; ++j)
                            if ((j & op.creg) == op.creg)
                                for (int c = 0; c < NC; ++c)
                                    if (uk < 0 || ((c >> uk) & 1)) pend_add(pend[j][c], a_s);
                    }
                    break;
                case K_DIAG:
                    if (op.cmask || op.dmask) {
                        std::string h = "{ uint32_t hi = 0; ";
                        int k = 0;
                        for (uint64_t dm = op.dmask; dm; dm &= dm - 1, ++k)
                            h += "hi |= (uint32_t)((g0 >> " + num(ctz64(dm)) + ") & 1ull) << " + num(k) + "; ";
                        h += "k_diag_hi<T>(a, pool + " + num(rm) + "u, hi << " + num(op.nreg) + ", " +
                             num(op.nreg) + "u, " + creg + ", " + hex64(op.ridx) + "); }";
                        b += "        " + cond + h + "\n";
                    } else {
                        for (int j = 0; j < NREG; ++j)
                            if ((j & op.creg) == op.creg) add_all(j, gen.atom(0, rm + (uint32_t)((op.ridx >> (4 * j)) & 15u)));
                    }
                    break;
                case K_RESET:
                    for (int j = 0; j < NREG; ++j) resolve(j);
                    b += "        " + cond + "k_reset<T, " + S0 + ">(a);\n";
                    break;
                default:
                    return PLAN_UNCOVERED;
            }
            if (gen.overflow) return PLAN_OVERFLOW;
        }
        flush(0xffffffffu);
        for (int j = 0; j < NREG; ++j) resolve(j);
        if (gen.overflow) return PLAN_OVERFLOW;
        for (int j = 0; j < NREG; ++j)
            b += store_global ? "        st[g0 | " + hex64(greg[j]) + "] = a[" + num(j) + "];\n"
                              : "        sm[sb ^ " + hex32(ph.rslot[j]) + "] = a[" + num(j) + "];\n";
        b += "    }\n";
        seg_ph.push_back(b);
    }

    out.n_param = gen.np > 0 ? gen.np : 1;
    const std::string T = c64 ? "float" : "double";
    const std::string jp = "namespace gq {\nstruct JP {\n    cplx<" + T + "> m[" + num(out.n_param) + "];\n};\n}\n";
    std::string& s = out.source;
    s.clear();
    s += "// goqu_b200 specialised tile pass\n";
    s += "typedef unsigned char uint8_t;\ntypedef int int32_t;\ntypedef unsigned int uint32_t;\n";
    s += "typedef long long int64_t;\ntypedef unsigned long long uint64_t;\n";
    s += "#include \"tile_core.cuh\"\n" + jp;
    s += "extern \"C\" __global__ void __launch_bounds__(" + num(threads) + ", " + num(min_blocks) + ")\n";
    s += "gqj_pass(gq::cplx<" + T + ">* __restrict__ st, const __grid_constant__ gq::JP p, const gq::cplx<" + T +
         ">* __restrict__ pool, const gq::PhaseDesc* __restrict__ phases) {\n";
    s += "    using namespace gq;\n    using T = " + T + ";\n";
    s += "    extern __shared__ __align__(16) unsigned char smraw[];\n";
    s += "    (void)pool;\n    (void)phases;\n";
    s += "    const uint32_t t = threadIdx.x;\n";
    if (!persistent) {
        s += "    cplx<T>* sm = reinterpret_cast<cplx<T>*>(smraw);\n";
        s += "    const uint64_t cta = blockIdx.x;\n";
        s += pro;
        if (!direct_in) s += seg_in + "    __syncthreads();\n";
        for (size_t k = 0; k < seg_ph.size(); ++k) {
            s += seg_ph[k];
            if (k + 1 < seg_ph.size() || !direct_out) s += "    __syncthreads();\n";
        }
        if (!direct_out) s += seg_out;
        s += "}\n";
    } else {
        // Persistent CTAs (grid = SMs x CTAs per SM), one tile buffer each: the
        // next tile's amplitudes are copied in asynchronously (cp.async) once
        // the current tile's last phase has loaded its registers (each thread
        // into the slots it read), so the copy overlaps that phase's
        // arithmetic and its direct stores; the CTA waits for the copy before
        // the next tile's first phase. Without direct stores the last phase
        // writes the buffer back first and the copy starts after the staged
        // write-out.
        auto issue = [&]() {
            std::string r = "    if (nxt < ntiles) {\n" + make_pro("nxt");
            for (int it = 0; it < NREG; ++it)
                r += "    cp_async_amp(sm + (stt ^ " + hex32(S[it]) + "), st + (gt | " + hex64(G[it]) + "));\n";
            r += "    }\n    cp_async_commit();\n";
            return r;
        };
        s += "    cplx<T>* const sm = reinterpret_cast<cplx<T>*>(smraw);\n";
        s += "    const uint64_t ntiles = 1ull << " + num(pd.n_outer) + ";\n";
        s += "    uint64_t cta = blockIdx.x;\n    if (cta >= ntiles) return;\n";
        s += "    {\n" + pro + seg_in + "    }\n    __syncthreads();\n";
        s += "    for (;;) {\n";
        s += "    const uint64_t nxt = cta + gridDim.x;\n";
        s += "    {\n" + pro;
        for (size_t k = 0; k < seg_ph.size(); ++k) {
            s += seg_ph[k];  // the last one, with direct stores, issues the copy itself
            if (k + 1 < seg_ph.size()) s += "    __syncthreads();\n";
        }
        if (!direct_out) s += "    __syncthreads();\n" + seg_out + "    __syncthreads();\n    {\n" + issue() + "    }\n";
        s += "    }\n    cp_async_wait_all();\n    __syncthreads();\n";
        s += "    cta = nxt;\n    if (cta >= ntiles) break;\n    }\n}\n";
    }

    if (host) {
        // the same segments, threads of a CTA run one after another between barriers
        std::string& h = out.host_source;
        h.clear();
        h += "#include \"tile_core.cuh\"\n";
        h += "extern \"C\" void gqj_host_" + num((long long)pi) + "(gq::cplx<" + T + ">* st, const gq::cplx<" + T +
             ">* pm, const gq::cplx<" + T + ">* pool, const gq::PhaseDesc* phases, gq::cplx<" + T + ">* sm) {\n";
        h += "    using namespace gq;\n    using T = " + T + ";\n    (void)pool;\n    (void)phases;\n";
        h += "    const struct {\n        const cplx<T>* m;\n    } p{pm};\n";
        h += "    for (uint64_t cta = 0; cta < (1ull << " + num(pd.n_outer) + "); ++cta) {\n";
        auto loop = [&](const std::string& seg) {
            h += "    for (uint32_t t = 0; t < " + num(threads) + "u; ++t) {\n" + pro + seg + "    }\n";
        };
        if (!direct_in) loop(seg_in);
        for (const std::string& ph : seg_ph) loop(ph);
        if (!direct_out) loop(seg_out);
        h += "    }\n}\n";
    }
    return PLAN_OK;
}

}  // namespace

bool jit_plan(const Program& pr, size_t pi, bool c64, int threads, int min_blocks, bool persistent, JitPlan& out,
              bool host) {
    // predicate tables grow the parameter block: fewer predicates per phase
    // when it does not fit
    for (int kmax : {4, 2, 0}) {
        const PlanResult r = plan_forward(pr, pi, c64, threads, min_blocks, persistent, out, host, kmax);
        if (r != PLAN_OVERFLOW) return r == PLAN_OK;
    }
    return false;
}

bool jit_plan_dual(const Program& pr, size_t pi, bool c64, int threads, int min_blocks, JitPlan& out, bool host) {
    const PassDesc& pd = pr.passes[pi];
    uint32_t op_base, pool_base;
    jit_bases(pr, pi, &op_base, &pool_base);
    const int m = pd.m, tbits = m - RQ;
    if (tbits < 0 || (1 << tbits) != threads) return false;
    out.atoms.clear();
    out.entries.clear();
    out.phase_shears.clear();
    Gen gen(pr, out, c64 ? 3900u : 1950u);

    std::string pro = "    uint64_t base = 0;\n";
    emit_deposit(pro, "    ", "base", "cta", pd.outer_q, pd.n_outer);
    pro += "    uint64_t gt = base;\n    uint32_t stt = 0;\n";
    emit_deposit(pro, "    ", "gt", "t", pd.tile_q, tbits);
    for (int k = 0; k < tbits; ++k)
        pro += "    stt ^= (0u - ((t >> " + num(k) + ") & 1u)) & " + hex32(pd.acol[k]) + ";\n";
    pro += "    (void)gt;\n    (void)stt;\n";
    uint64_t G[NREG];
    uint32_t S[NREG];
    for (int it = 0; it < NREG; ++it) {
        G[it] = 0;
        S[it] = 0;
        for (int k = 0; k < RQ; ++k)
            if ((it >> k) & 1) {
                G[it] |= 1ull << pd.tile_q[tbits + k];
                S[it] ^= pd.acol[tbits + k];
            }
    }
    std::string seg_in = "    {\n        cplx<T> v[16], w[16];\n";
    for (int it = 0; it < NREG; ++it)
        seg_in += "        v[" + num(it) + "] = psi[gt | " + hex64(G[it]) + "];\n        w[" + num(it) + "] = lam[gt | " +
                  hex64(G[it]) + "];\n";
    for (int it = 0; it < NREG; ++it)
        seg_in += "        sa[stt ^ " + hex32(S[it]) + "] = v[" + num(it) + "];\n        sbuf[stt ^ " + hex32(S[it]) +
                  "] = w[" + num(it) + "];\n";
    seg_in += "    }\n";
    std::string seg_out = "    {\n";
    for (int it = 0; it < NREG; ++it)
        seg_out += "        psi[gt | " + hex64(G[it]) + "] = sa[stt ^ " + hex32(S[it]) + "];\n        lam[gt | " +
                   hex64(G[it]) + "] = sbuf[stt ^ " + hex32(S[it]) + "];\n";
    seg_out += "    }\n";
    const std::string SL = num(MAX_GRAD_SLOTS);
    // per-warp slot sums: the device reduces a warp's lanes with shuffles;
    // the host form (threads in turn) adds each thread's value
    auto flush = [&](int slot, bool hst) -> std::string {
        if (hst) return "        gsm[(t >> 5) * " + SL + " + " + num(slot) + "] += gacc; gacc = 0.0;\n";
        return "        { double fv = gacc; for (unsigned o = 16; o > 0; o >>= 1) { const double y = "
               "__shfl_xor_sync(lanes, fv, o); if ((lane ^ o) < (int)nlanes) fv += y; } if (lane == 0) gsm[warp * " +
               SL + " + " + num(slot) + "] += fv; gacc = 0.0; }\n";
    };
    std::vector<std::string> ph_dev, ph_host;
    for (int p = 0; p < pd.n_phases; ++p) {
        const PhaseDesc& ph = pr.phases[pd.phase0 + p];
        uint32_t tslot[MAX_TILE];
        int tq[MAX_TILE];
        for (int k = 0; k < tbits; ++k) {
            const uint32_t sv = k < 4 ? ph.tlo_slot[1u << k] : ph.thi_slot[1u << (k - 4)];
            const uint64_t g = k < 4 ? ph.tlo_glob[1u << k] : ph.thi_glob[1u << (k - 4)];
            if (g == 0 || (g & (g - 1))) return false;
            tslot[k] = sv;
            tq[k] = ctz64(g);
        }
        for (int v = 0; v < TLO && v < (1 << tbits); ++v) {
            uint32_t sv = 0;
            uint64_t g = 0;
            for (int k = 0; k < 4 && k < tbits; ++k)
                if ((v >> k) & 1) {
                    sv ^= tslot[k];
                    g |= 1ull << tq[k];
                }
            if (sv != ph.tlo_slot[v] || g != ph.tlo_glob[v]) return false;
        }
        std::string head = "    {\n        uint32_t sb = 0;\n        uint64_t g0 = base;\n";
        for (int k = 0; k < tbits; ++k)
            head += "        sb ^= (0u - ((t >> " + num(k) + ") & 1u)) & " + hex32(tslot[k]) + ";\n";
        emit_deposit(head, "        ", "g0", "t", tq, tbits);
        head += "        (void)g0;\n        cplx<T> a[16], bb[16];\n        double gacc = 0.0;\n        (void)gacc;\n";
        for (int j = 0; j < NREG; ++j)
            head += "        a[" + num(j) + "] = sa[sb ^ " + hex32(ph.rslot[j]) + "];\n        bb[" + num(j) +
                    "] = sbuf[sb ^ " + hex32(ph.rslot[j]) + "];\n";
        std::string bd, bh;  // op bodies, device / host flush
        int cur = -1;
        for (int oa = ph.op_begin; oa < ph.op_end; ++oa) {
            const KOp& op = pr.ops[oa];
            const uint32_t rm = op.mat - pool_base;
            const bool grad = op.type == K_GRAD;
            const uint8_t kind = grad ? op.flags : op.type;
            if (kind == K_NONE || kind == K_RESET || kind == K_GRAD || kind > K_PAIRSUM) return false;
            const std::string creg = num(op.creg) + "u";
            const std::string C = op.creg ? "true" : "false";
            const std::string S0 = num(op.t0), S1 = num(op.t1), S2 = num(op.t2);
            std::string cond;
            if (op.cmask) cond = "if ((g0 & " + hex64(op.cmask) + ") == " + hex64(op.cmask) + ") ";
            auto pm = [&](uint32_t off) { return "PMat<T>{p.m + " + num(off) + "}"; };
            const bool pure_x = kind == K_X && !grad && (op.flags & 1);
            // the op's body on register array x (xs: its shared-memory tile, U4's scratch)
            auto body = [&](const std::string& x, const std::string& xs) -> std::string {
                switch (kind) {
                    case K_U1:
                        return "k_u1<T, " + S0 + ", " + C + ">(" + x + ", " + pm(gen.copy(rm, 4)) + ", " + creg + ");";
                    case K_U2:
                        return "k_u2<T, " + S0 + ", " + S1 + ", " + C + ">(" + x + ", " + pm(gen.copy(rm, 16)) + ", " +
                               creg + ");";
                    case K_U3:
                        return "k_u3<T, " + S0 + ", " + S1 + ", " + S2 + ">(" + x + ", " + pm(gen.copy(rm, 64)) +
                               ", " + creg + ");";
                    case K_U4:
                        return "k_u4<T>(" + x + ", " + pm(gen.copy(rm, 256)) + ", " + xs + ", sb, phases[" + num(p) +
                               "].rslot);";
                    case K_X:
                        return "k_x<T, " + S0 + ", " + C + ">(" + x + ", " +
                               (pure_x ? std::string("pool") : pm(gen.copy(rm, 2))) + ", " + creg + ", " +
                               (pure_x ? "true" : "false") + ");";
                    case K_SWAP: return "k_swap<T, " + S0 + ", " + S1 + ">(" + x + ", " + creg + ");";
                    case K_PHASE: return "k_phase<T>(" + x + ", p.m[" + num(gen.copy(rm, 1)) + "], " + creg + ");";
                    case K_PAIRSUM:
                        return "k_pairsum<T>(" + x + ", pool + " + num(rm) + "u, g0);";
                    case K_DIAG: {
                        std::string h = "{ uint32_t hi = 0; ";
                        int k = 0;
                        for (uint64_t dm = op.dmask; dm; dm &= dm - 1, ++k)
                            h += "hi |= (uint32_t)((g0 >> " + num(ctz64(dm)) + ") & 1ull) << " + num(k) + "; ";
                        h += "k_diag_hi<T>(" + x + ", pool + " + num(rm) + "u, hi << " + num(op.nreg) + ", " +
                             num(op.nreg) + "u, " + creg + ", " + hex64(op.ridx) + "); }";
                        return h;
                    }
                    default: return "";
                }
            };
            if (!grad) {
                const std::string line = "        " + cond + body("a", "sa") + "\n        " + cond + body("bb", "sbuf") + "\n";
                bd += line;
                bh += line;
                continue;
            }
            if ((int)op.slot != cur) {  // slot runs: reduce once per run
                if (cur >= 0) {
                    bd += flush(cur, false);
                    bh += flush(cur, true);
                }
                cur = (int)op.slot;
            }
            std::string e;
            if (kind == K_PHASE) {
                e = "gv = grad_phase_c<T>(a, bb, p.m[" + num(gen.copy(rm, 1)) + "], " + creg + ");";
            } else if (kind == K_DIAG) {
                std::string h = "uint32_t hi = 0; ";
                int k = 0;
                for (uint64_t dm = op.dmask; dm; dm &= dm - 1, ++k)
                    h += "hi |= (uint32_t)((g0 >> " + num(ctz64(dm)) + ") & 1ull) << " + num(k) + "; ";
                e = h + "gv = grad_diag_c<T>(a, bb, pool + " + num(rm) + "u, hi << " + num(op.nreg) + ", " + creg +
                    ", " + hex64(op.ridx) + ");";
            } else if (kind == K_PAIRSUM) {
                e = "gv = grad_pairsum_c<T>(a, bb, pool + " + num(rm) + "u, g0);";
            } else if (kind == K_X) {
                const uint32_t px = gen.copy(rm, 2);
                e = "gv = grad_x_c<T, " + S0 + ">(a, bb, p.m[" + num(px) + "], p.m[" + num(px + 1) + "], " + creg + ");";
            } else {  // dense G, applied to a copy of psi
                e = "cplx<T> v[16]; for (int j = 0; j < 16; ++j) v[j] = a[j]; " + body("v", "sa") +
                    " gv = dot_re_creg<T>(bb, v, " + creg + ");";
            }
            const std::string line = "        { double gv = 0.0; " + cond + "{ " + e + " } gacc += gv; }\n";
            bd += line;
            bh += line;
        }
        if (cur >= 0) {
            bd += flush(cur, false);
            bh += flush(cur, true);
        }
        std::string tail;
        for (int j = 0; j < NREG; ++j)
            tail += "        sa[sb ^ " + hex32(ph.rslot[j]) + "] = a[" + num(j) + "];\n        sbuf[sb ^ " +
                    hex32(ph.rslot[j]) + "] = bb[" + num(j) + "];\n";
        tail += "    }\n";
        ph_dev.push_back(head + bd + tail);
        ph_host.push_back(head + bh + tail);
        if (gen.overflow) return false;
    }

    out.n_param = gen.np > 0 ? gen.np : 1;
    const std::string T = c64 ? "float" : "double";
    const std::string tile = num(1ll << m);
    std::string& s = out.source;
    s.clear();
    s += "// goqu_b200 specialised reverse (adjoint) pass\n";
    s += "typedef unsigned char uint8_t;\ntypedef int int32_t;\ntypedef unsigned int uint32_t;\n";
    s += "typedef long long int64_t;\ntypedef unsigned long long uint64_t;\n";
    s += "#include \"tile_core.cuh\"\n";
    s += "namespace gq {\nstruct JP {\n    cplx<" + T + "> m[" + num(out.n_param) + "];\n};\n}\n";
    s += "extern \"C\" __global__ void __launch_bounds__(" + num(threads) + ", " + num(min_blocks) + ")\n";
    s += "gqj_dual(gq::cplx<" + T + ">* __restrict__ psi, gq::cplx<" + T + ">* __restrict__ lam, const "
         "__grid_constant__ gq::JP p, const gq::cplx<" + T + ">* __restrict__ pool, const gq::PhaseDesc* __restrict__ "
         "phases, double* __restrict__ partial, int nslots) {\n";
    s += "    using namespace gq;\n    using T = " + T + ";\n";
    s += "    extern __shared__ __align__(16) unsigned char smraw[];\n";
    s += "    cplx<T>* const sa = reinterpret_cast<cplx<T>*>(smraw);\n";
    s += "    cplx<T>* const sbuf = sa + " + tile + ";\n";
    s += "    double* const gsm = reinterpret_cast<double*>(sbuf + " + tile + ");\n";
    s += "    (void)pool;\n    (void)phases;\n";
    s += "    const uint32_t t = threadIdx.x;\n    const uint64_t cta = blockIdx.x;\n";
    s += "    const int nwarps = (int)((blockDim.x + 31) >> 5);\n";
    s += "    const int warp = (int)(t >> 5), lane = (int)(t & 31);\n";
    s += "    const unsigned nlanes = blockDim.x < 32 ? blockDim.x : 32u;\n";
    s += "    const unsigned lanes = nlanes == 32 ? 0xffffffffu : ((1u << nlanes) - 1u);\n";
    s += pro + seg_in;
    s += "    for (int i = (int)t; i < nwarps * " + SL + "; i += (int)blockDim.x) gsm[i] = 0.0;\n";
    s += "    __syncthreads();\n";
    for (const std::string& ph : ph_dev) s += ph + "    __syncthreads();\n";
    s += seg_out;
    s += "    for (int sl = (int)t; sl < nslots; sl += (int)blockDim.x) {\n        double tot = 0.0;\n"
         "        for (int w = 0; w < nwarps; ++w) tot += gsm[w * " + SL + " + sl];\n"
         "        partial[cta * (uint64_t)nslots + sl] = tot;\n    }\n}\n";
    if (host) {
        std::string& h = out.host_source;
        h.clear();
        h += "#include \"tile_core.cuh\"\n";
        h += "extern \"C\" void gqj_hostdual_" + num((long long)pi) + "(gq::cplx<" + T + ">* psi, gq::cplx<" + T +
             ">* lam, const gq::cplx<" + T + ">* pm, const gq::cplx<" + T + ">* pool, const gq::PhaseDesc* phases, "
             "double* partial, int nslots, gq::cplx<" + T + ">* sa, double* gsm) {\n";
        h += "    using namespace gq;\n    using T = " + T + ";\n    (void)pool;\n    (void)phases;\n";
        h += "    const struct {\n        const cplx<T>* m;\n    } p{pm};\n";
        h += "    cplx<T>* const sbuf = sa + " + tile + ";\n";
        h += "    const int nwarps = " + num((threads + 31) >> 5) + ";\n";
        h += "    for (uint64_t cta = 0; cta < (1ull << " + num(pd.n_outer) + "); ++cta) {\n";
        auto loop = [&](const std::string& seg) {
            h += "    for (uint32_t t = 0; t < " + num(threads) + "u; ++t) {\n" + pro + seg + "    }\n";
        };
        loop(seg_in);
        h += "    for (int i = 0; i < nwarps * " + SL + "; ++i) gsm[i] = 0.0;\n";
        for (const std::string& ph : ph_host) loop(ph);
        loop(seg_out);
        h += "    for (int sl = 0; sl < nslots; ++sl) {\n        double tot = 0.0;\n"
             "        for (int w = 0; w < nwarps; ++w) tot += gsm[w * " + SL + " + sl];\n"
             "        partial[cta * (uint64_t)nslots + sl] = tot;\n    }\n";
        h += "    }\n}\n";
    }
    return true;
}

bool jit_pack(const Program& pr, size_t pi, const JitPlan& plan, bool c64, void* block) {
    uint32_t op_base, pool_base;
    jit_bases(pr, pi, &op_base, &pool_base);
    const size_t nops = pr.ops.size() - op_base;
    // atom values
    std::vector<Z> av(plan.atoms.size());
    std::vector<double> tv(nops, 0.0);
    std::vector<char> have(nops, 0);
    auto dec = [&](uint32_t o, Z* lam, Z* p0, Z* p1) {
        double t;
        if (o >= nops || !u1_decompose(&pr.pool[pr.ops[op_base + o].mat], &t, lam, p0, p1)) return false;
        tv[o] = t;
        have[o] = 1;
        return true;
    };
    // chain products under each predicate combination
    struct ChainDec {
        double t;
        Z lam, p0, p1;
        bool have = false;
    };
    std::vector<ChainDec> cd(plan.chains.size() * 4);
    auto cdec = [&](uint32_t ref) -> const ChainDec* {
        if (ref / 4 >= plan.chains.size()) return nullptr;
        ChainDec& d = cd[ref];
        if (!d.have) {
            Z mm[4];
            chain_matrix(pr, op_base, plan.chains[ref / 4], (int)(ref % 4), mm);
            if (!u1_decompose(mm, &d.t, &d.lam, &d.p0, &d.p1)) return nullptr;
            d.have = true;
        }
        return &d;
    };
    for (size_t i = 0; i < plan.atoms.size(); ++i) {
        const JitAtom& a = plan.atoms[i];
        if (a.kind == 0) {
            av[i] = pr.pool[pool_base + a.ref];
            continue;
        }
        if (a.kind >= 4) {
            const ChainDec* d = cdec(a.ref);
            if (!d) return false;
            av[i] = a.kind == 4 ? d->lam : (a.kind == 5 ? d->p0 : d->p1);
            continue;
        }
        Z lam, p0, p1;
        if (!dec(a.ref, &lam, &p0, &p1)) return false;  // no longer decomposable: run interpreted
        av[i] = a.kind == 1 ? lam : (a.kind == 2 ? p0 : p1);
    }
    // range check: within a phase the amplitudes grow by at most prod(1 + |t|)
    const double limit = c64 ? 60.0 : 600.0;  // log2 bound
    for (size_t p = 0; p < plan.phase_shears.size(); ++p) {
        double lg = 0;
        for (uint32_t o : plan.phase_shears[p]) {
            if (o >= nops) return false;
            if (!have[o]) {
                Z l, a, b;
                if (!dec(o, &l, &a, &b)) return false;
            }
            lg += std::log2(1.0 + std::fabs(tv[o]));
        }
        if (p < plan.phase_chains.size())
            for (uint32_t f : plan.phase_chains[p]) {
                double tmax = 0;
                int npred = 0;
                for (int8_t k : plan.chains[f].pred) npred = std::max(npred, k + 1);
                for (int e = 0; e < (1 << npred); ++e) {
                    const ChainDec* d = cdec(f * 4 + (uint32_t)e);
                    if (!d) return false;
                    tmax = std::max(tmax, std::fabs(d->t));
                }
                lg += std::log2(1.0 + tmax);
            }
        if (lg > limit) return false;
    }
    std::vector<Z> vals;
    vals.reserve(plan.n_param);
    for (const JitEntry& e : plan.entries) {
        if (e.kind == 0) {
            for (uint32_t k = 0; k < e.count; ++k) vals.push_back(pr.pool[pool_base + e.ref + k]);
        } else if (e.kind == 1) {
            if (!have[e.ref]) {
                Z l, a, b;
                if (!dec(e.ref, &l, &a, &b)) return false;
            }
            vals.push_back({tv[e.ref], 0.0});
        } else if (e.kind == 3) {
            const ChainDec* d = cdec(e.ref);
            if (!d) return false;
            vals.push_back({d->t, 0.0});
        } else {
            Z nv = {1, 0}, dv = {1, 0};
            for (uint32_t a : e.num) nv = zmul(nv, av[a]);
            for (uint32_t a : e.den) dv = zmul(dv, av[a]);
            if (zabs(dv) < 1e-280) return false;
            vals.push_back(e.den.empty() ? nv : zdiv(nv, dv));
        }
    }
    vals.resize(plan.n_param, Z{0, 0});
    if (c64) {
        float* f = (float*)block;
        for (size_t i = 0; i < vals.size(); ++i) {
            f[2 * i] = (float)vals[i].re;
            f[2 * i + 1] = (float)vals[i].im;
        }
    } else {
        std::memcpy(block, vals.data(), sizeof(Z) * vals.size());
    }
    return true;
}

// ---- NVRTC -----------------------------------------------------------------

namespace {

struct Nvrtc {
    bool ok = false;
    nvrtcResult (*create)(nvrtcProgram*, const char*, const char*, int, const char* const*, const char* const*);
    nvrtcResult (*compile)(nvrtcProgram, int, const char* const*);
    nvrtcResult (*log_size)(nvrtcProgram, size_t*);
    nvrtcResult (*log)(nvrtcProgram, char*);
    nvrtcResult (*cubin_size)(nvrtcProgram, size_t*);
    nvrtcResult (*cubin)(nvrtcProgram, char*);
    nvrtcResult (*destroy)(nvrtcProgram*);
    nvrtcResult (*version)(int*, int*) = nullptr;
    Nvrtc() {
        const char* names[] = {"libnvrtc.so.12", "libnvrtc.so", "/usr/local/cuda/lib64/libnvrtc.so.12"};
        void* h = nullptr;
        for (const char* n : names)
            if ((h = dlopen(n, RTLD_NOW | RTLD_LOCAL))) break;
        if (!h) return;
        create = (decltype(create))dlsym(h, "nvrtcCreateProgram");
        compile = (decltype(compile))dlsym(h, "nvrtcCompileProgram");
        log_size = (decltype(log_size))dlsym(h, "nvrtcGetProgramLogSize");
        log = (decltype(log))dlsym(h, "nvrtcGetProgramLog");
        cubin_size = (decltype(cubin_size))dlsym(h, "nvrtcGetCUBINSize");
        cubin = (decltype(cubin))dlsym(h, "nvrtcGetCUBIN");
        destroy = (decltype(destroy))dlsym(h, "nvrtcDestroyProgram");
        version = (decltype(version))dlsym(h, "nvrtcVersion");
        ok = create && compile && log_size && log && cubin_size && cubin && destroy;
    }
};

Nvrtc& nvrtc() {
    static Nvrtc n;
    return n;
}

}  // namespace

bool jit_available() { return nvrtc().ok; }

namespace {
const char* const kJitOpts[] = {"--gpu-architecture=sm_100a", "-std=c++17", "--ptxas-options=-v"};
constexpr int kJitNumOpts = 3;
}  // namespace

std::string jit_compile_only(const std::string& source, std::vector<char>* cubin, std::string* log) {
    Nvrtc& N = nvrtc();
    if (!N.ok) return "libnvrtc not found";
    nvrtcProgram prog;
    const char* hdr_src[] = {kTileCore};
    const char* hdr_name[] = {"tile_core.cuh"};
    if (N.create(&prog, source.c_str(), "gqj_pass.cu", 1, hdr_src, hdr_name) != NVRTC_SUCCESS)
        return "nvrtcCreateProgram failed";
    const nvrtcResult rc = N.compile(prog, kJitNumOpts, kJitOpts);
    size_t ls = 0;
    N.log_size(prog, &ls);
    std::string lg(ls, '\0');
    if (ls) N.log(prog, &lg[0]);
    if (log) *log = lg;
    if (rc != NVRTC_SUCCESS) {
        N.destroy(&prog);
        return "compile failed: " + lg;
    }
    size_t cs = 0;
    N.cubin_size(prog, &cs);
    if (cubin) {
        cubin->resize(cs);
        N.cubin(prog, cubin->data());
    }
    N.destroy(&prog);
    return "";
}

// ---- on-disk cache of compiled kernels -------------------------------------

namespace {

// Everything the binary depends on: cache format, compiler options, NVRTC
// version, the embedded tile header and the kernel text.
std::string jit_identity(const std::string& source) {
    std::string id = "goqu_b200 jit cubin v1\n";
    for (int i = 0; i < kJitNumOpts; ++i) id += std::string(kJitOpts[i]) + "\n";
    int maj = 0, mnr = 0;
    if (nvrtc().version) nvrtc().version(&maj, &mnr);
    id += "nvrtc " + std::to_string(maj) + "." + std::to_string(mnr) + "\n";
    id += kTileCore;
    id += "\n";
    id += source;
    return id;
}

uint64_t fnv1a(const std::string& s) {
    uint64_t h = 1469598103934665603ull;
    for (unsigned char c : s) h = (h ^ c) * 1099511628211ull;
    return h;
}

}  // namespace

std::string jit_cache_dir() {
    const char* env = std::getenv("GQ_JIT_CACHE_DIR");
    if (env) return std::string(env) == "off" ? std::string() : std::string(env);
    const char* xdg = std::getenv("XDG_CACHE_HOME");
    if (xdg && *xdg) return std::string(xdg) + "/goqu_b200/jit";
    const char* home = std::getenv("HOME");
    return home && *home ? std::string(home) + "/.cache/goqu_b200/jit" : std::string();
}

std::string jit_compile_cached(const std::string& source, std::vector<char>* cubin, std::string* log, bool* from_disk) {
    *from_disk = false;
    const std::string dir = jit_cache_dir();
    if (dir.empty()) return jit_compile_only(source, cubin, log);
    const std::string id = jit_identity(source);
    char name[32];
    std::snprintf(name, sizeof(name), "%016llx.cubin", (unsigned long long)fnv1a(id));
    const std::string path = dir + "/" + name;
    // a hit needs the stored identity to equal this one byte for byte
    if (FILE* f = std::fopen(path.c_str(), "rb")) {
        uint64_t idn = 0, cn = 0;
        std::string stored;
        std::vector<char> bin;
        bool ok = std::fread(&idn, 8, 1, f) == 1 && idn == id.size();
        if (ok) {
            stored.resize(idn);
            ok = std::fread(&stored[0], 1, idn, f) == idn && stored == id && std::fread(&cn, 8, 1, f) == 1 &&
                 cn > 0 && cn < (1ull << 30);
        }
        if (ok) {
            bin.resize(cn);
            ok = std::fread(bin.data(), 1, cn, f) == cn;
        }
        std::fclose(f);
        if (ok) {
            if (cubin) cubin->swap(bin);
            if (log) log->clear();
            *from_disk = true;
            return "";
        }
    }
    std::vector<char> bin;
    const std::string err = jit_compile_only(source, &bin, log);
    if (!err.empty()) return err;
    // write to a private temporary file, then rename over the final name
    std::string cmd_dir = dir;
    for (size_t i = 1; i <= cmd_dir.size(); ++i)
        if (i == cmd_dir.size() || cmd_dir[i] == '/') mkdir(cmd_dir.substr(0, i).c_str(), 0700);
    const std::string tmp = path + "." + std::to_string((long long)getpid()) + "." +
                            std::to_string((unsigned long long)std::hash<std::thread::id>()(std::this_thread::get_id())) +
                            ".tmp";
    if (FILE* f = std::fopen(tmp.c_str(), "wb")) {
        const uint64_t idn = id.size(), cn = bin.size();
        const bool ok = std::fwrite(&idn, 8, 1, f) == 1 && std::fwrite(id.data(), 1, idn, f) == idn &&
                        std::fwrite(&cn, 8, 1, f) == 1 && std::fwrite(bin.data(), 1, cn, f) == cn;
        const bool closed = std::fclose(f) == 0;
        if (ok && closed) std::rename(tmp.c_str(), path.c_str());
        else std::remove(tmp.c_str());
    }
    if (cubin) cubin->swap(bin);
    return "";
}

}  // namespace gq

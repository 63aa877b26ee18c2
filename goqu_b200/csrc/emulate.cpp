// Host emulation of the tile-pass programs, for CPU tests of the scheduler.
//
// Runs the exact device code path of tile_core.cuh (the same run_phase /
// apply_op functions and the same program tables) with CTAs, phases and
// threads executed one after another, so that scheduling, swizzle and index
// tables can be checked against the oracle without a GPU. It is built into
// libgqb200_emu.so, which only the tests load.
#include <dlfcn.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include <set>

#include "jit.hpp"
#include "schedule.hpp"
#include "params.hpp"
#include "tile_core.cuh"

namespace {

thread_local std::string g_err;
// Support of the start state the next scheduling hooks assume
// (SchedOptions::support0; gqx_set_support0), and the CTAs their programs
// launch (gqx_last_ctas).
thread_local uint64_t g_support0 = ~0ull;
thread_local int64_t g_ctas = 0;
// Persistent kernel texts in gqx_jit_check (gqx_set_persistent).
thread_local bool g_persistent = false;

int64_t count_ctas(const gq::Program& prog) {
    int64_t c = 0;
    for (const gq::PassDesc& pd : prog.passes) c += 1ll << pd.n_outer;
    return c;
}

template <class T>
void run_pass(std::vector<gq::cplx<T>>& st, const gq::Program& prog, const std::vector<gq::cplx<T>>& pool, size_t pi) {
    const gq::PassDesc& pd = prog.passes[pi];
    const int m = pd.m;
    const uint32_t tpb = 1u << (m - gq::RQ);
    const uint64_t n_cta = 1ull << pd.n_outer;
    std::vector<gq::cplx<T>> sm(1u << m);
    for (uint64_t cta = 0; cta < n_cta; ++cta) {
        const uint64_t base = gq::cta_base(pd, cta);
        for (uint32_t lin = 0; lin < (1u << m); ++lin) {
            uint64_t goff;
            uint32_t slot;
            gq::linear_slot(pd, lin, goff, slot);
            sm[slot] = st[base | goff];
        }
        for (int p = 0; p < pd.n_phases; ++p) {
            const gq::PhaseDesc& ph = prog.phases[pd.phase0 + p];
            for (uint32_t t = 0; t < tpb; ++t) gq::run_phase<T>(sm.data(), ph, prog.ops.data(), pool.data(), t, base);
        }
        for (uint32_t lin = 0; lin < (1u << m); ++lin) {
            uint64_t goff;
            uint32_t slot;
            gq::linear_slot(pd, lin, goff, slot);
            st[base | goff] = sm[slot];
        }
    }
}

template <class T>
std::vector<gq::cplx<T>> pool_of(const gq::Program& prog) {
    std::vector<gq::cplx<T>> pool(prog.pool.size());
    for (size_t i = 0; i < pool.size(); ++i) pool[i] = {(T)prog.pool[i].re, (T)prog.pool[i].im};
    return pool;
}

template <class T>
void run_program(std::vector<gq::cplx<T>>& st, const gq::Program& prog) {
    const std::vector<gq::cplx<T>> pool = pool_of<T>(prog);
    for (size_t i = 0; i < prog.passes.size(); ++i) run_pass<T>(st, prog, pool, i);
}

// Runs a program through the specialised kernels' host form: every pass's
// generated code is compiled with the host compiler into one library and
// called with its packed parameter block; passes without a plan or whose
// block does not pack run through the emulated interpreter.
template <class T>
int run_program_jit(std::vector<gq::cplx<T>>& st, const gq::Program& prog, bool c64, const char* csrc,
                    const char* work, int64_t* jitted) {
    std::vector<gq::JitPlan> plans(prog.passes.size());
    std::vector<char> ok(prog.passes.size(), 0);
    std::string src;
    for (size_t i = 0; i < prog.passes.size(); ++i) {
        const int threads = 1 << (prog.passes[i].m - gq::RQ);
        if (!gq::jit_plan(prog, i, c64, threads, 1, false, plans[i], true)) continue;
        ok[i] = 1;
        src += plans[i].host_source;
    }
    const std::string dir = work;
    const std::string cpp = dir + "/gqj_host.cpp", so = dir + "/gqj_host.so";
    {
        FILE* f = std::fopen(cpp.c_str(), "w");
        if (!f) {
            g_err = "cannot write " + cpp;
            return GQ_EINVAL;
        }
        std::fwrite(src.data(), 1, src.size(), f);
        std::fclose(f);
    }
    const std::string cmd = "g++ -O1 -std=c++17 -shared -fPIC -w -I'" + std::string(csrc) + "' '" + cpp + "' -o '" +
                            so + "' 2>'" + dir + "/gqj_host.log'";
    if (std::system(cmd.c_str()) != 0) {
        g_err = "host compile of the generated passes failed (" + dir + "/gqj_host.log)";
        return GQ_EINVAL;
    }
    void* h = dlopen(so.c_str(), RTLD_NOW | RTLD_LOCAL);
    if (!h) {
        g_err = dlerror();
        return GQ_EINVAL;
    }
    typedef void (*PassFn)(gq::cplx<T>*, const gq::cplx<T>*, const gq::cplx<T>*, const gq::PhaseDesc*, gq::cplx<T>*);
    const std::vector<gq::cplx<T>> pool = pool_of<T>(prog);
    *jitted = 0;
    for (size_t i = 0; i < prog.passes.size(); ++i) {
        std::vector<gq::cplx<T>> block;
        PassFn fn = nullptr;
        if (ok[i]) {
            block.resize(plans[i].n_param);
            if (gq::jit_pack(prog, i, plans[i], c64, block.data()))
                fn = (PassFn)dlsym(h, ("gqj_host_" + std::to_string(i)).c_str());
        }
        if (!fn) {
            run_pass<T>(st, prog, pool, i);
            continue;
        }
        uint32_t op_base, pool_base;
        gq::jit_bases(prog, i, &op_base, &pool_base);
        std::vector<gq::cplx<T>> sm(1u << prog.passes[i].m);
        fn(st.data(), block.data(), pool.data() + pool_base, prog.phases.data() + prog.passes[i].phase0, sm.data());
        ++*jitted;
    }
    dlclose(h);
    return GQ_OK;
}

}  // namespace

extern "C" {

const char* gqx_last_error(void) { return g_err.c_str(); }

void gqx_set_support0(uint64_t support0) { g_support0 = support0; }
void gqx_set_persistent(int on) { g_persistent = on != 0; }
int64_t gqx_last_ctas(void) { return g_ctas; }

// Applies ops to a host state (2^nq interleaved doubles) through the
// scheduler and the tile-pass code, emulated on the CPU. precision GQ_C64
// runs the float instantiation. Returns GQ_OK or an error code.
static int emulate_sv_impl(int nq, int precision, double* state, const gq_op* ops, size_t n_ops, int tile_qubits,
                           int budget, int fuse, int64_t* passes_out, int64_t* phases_out);

int gqx_emulate_sv(int nq, int precision, double* state, const gq_op* ops, size_t n_ops, int tile_qubits,
                   int budget, int64_t* passes_out, int64_t* phases_out) {
    return emulate_sv_impl(nq, precision, state, ops, n_ops, tile_qubits, budget, 0, passes_out, phases_out);
}

// The same with dense fusion of register-local gate runs switched on.
int gqx_emulate_sv_fused(int nq, int precision, double* state, const gq_op* ops, size_t n_ops, int tile_qubits,
                         int budget, int64_t* passes_out, int64_t* phases_out) {
    return emulate_sv_impl(nq, precision, state, ops, n_ops, tile_qubits, budget, 1, passes_out, phases_out);
}

static int emulate_sv_impl(int nq, int precision, double* state, const gq_op* ops, size_t n_ops, int tile_qubits,
                           int budget, int fuse, int64_t* passes_out, int64_t* phases_out) {
    const int nphys = nq < gq::RQ ? gq::RQ : nq;
    std::vector<gq::NGate> gates;
    for (size_t i = 0; i < n_ops; ++i) {
        int rc = gq::normalize_op(ops[i], nq, gates, g_err);
        if (rc != GQ_OK) return rc;
    }
    gq::SchedOptions opt;
    if (tile_qubits > 0) opt.tile_qubits = tile_qubits;
    if (budget > 0) opt.budget = budget;
    opt.swizzle_width = precision == GQ_C64 ? 4 : 3;
    opt.low_qubits = precision == GQ_C64 ? 4 : 3;
    opt.fuse_dense = fuse != 0;
    opt.support0 = g_support0;
    gq::Program prog;
    gq::schedule(gates, nphys, opt, prog);
    g_ctas = count_ctas(prog);
    const uint64_t n = 1ull << nphys;
    if (precision == GQ_C64) {
        std::vector<gq::cplx<float>> st(n, {0.f, 0.f});
        for (uint64_t i = 0; i < (1ull << nq); ++i) st[i] = {(float)state[2 * i], (float)state[2 * i + 1]};
        run_program<float>(st, prog);
        for (uint64_t i = 0; i < (1ull << nq); ++i) {
            state[2 * i] = st[i].x;
            state[2 * i + 1] = st[i].y;
        }
    } else {
        std::vector<gq::cplx<double>> st(n, {0.0, 0.0});
        std::memcpy(st.data(), state, sizeof(double) * 2 * (1ull << nq));
        run_program<double>(st, prog);
        std::memcpy(state, st.data(), sizeof(double) * 2 * (1ull << nq));
    }
    if (passes_out) *passes_out = (int64_t)prog.passes.size();
    if (phases_out) *phases_out = (int64_t)prog.phases.size();
    return GQ_OK;
}

// Schedule only: out = {passes, phases, ops, sum over ops of their FMA-per-
// amplitude cost, K_PAIRSUM ops}, for comparing scheduler settings without
// running anything.
int gqx_schedule_stats(int nq, int precision, const gq_op* ops, size_t n_ops, int tile_qubits, int budget, int fuse,
                       int64_t* out) {
    const int nphys = nq < gq::RQ ? gq::RQ : nq;
    std::vector<gq::NGate> gates;
    for (size_t i = 0; i < n_ops; ++i) {
        int rc = gq::normalize_op(ops[i], nq, gates, g_err);
        if (rc != GQ_OK) return rc;
    }
    gq::SchedOptions opt;
    if (tile_qubits > 0) opt.tile_qubits = tile_qubits;
    if (budget > 0) opt.budget = budget;
    opt.swizzle_width = precision == GQ_C64 ? 4 : 3;
    opt.low_qubits = precision == GQ_C64 ? 4 : 3;
    opt.fuse_dense = fuse != 0;
    gq::Program prog;
    gq::schedule(gates, nphys, opt, prog);
    int64_t cost = 0, pairsums = 0;
    for (const gq::KOp& op : prog.ops) {
        static const int c[] = {0, 8, 16, 32, 64, 1, 1, 3, 1, 4, 16, 6};
        cost += c[op.type] + 6;
        pairsums += op.type == gq::K_PAIRSUM;
    }
    out[0] = (int64_t)prog.passes.size();
    out[1] = (int64_t)prog.phases.size();
    out[2] = (int64_t)prog.ops.size();
    out[3] = cost;
    out[4] = pairsums;
    return GQ_OK;
}

// Per pass of the statevector schedule: out[5*i ..] = {phases, ops, FMA-per-
// amplitude cost, tile qubit mask, CTA-index bits}; returns the pass count
// (at most `max_passes` rows are written) or a negative error code.
int64_t gqx_schedule_passes(int nq, int precision, const gq_op* ops, size_t n_ops, int tile_qubits, int budget,
                            int64_t* out, int64_t max_passes) {
    const int nphys = nq < gq::RQ ? gq::RQ : nq;
    std::vector<gq::NGate> gates;
    for (size_t i = 0; i < n_ops; ++i) {
        int rc = gq::normalize_op(ops[i], nq, gates, g_err);
        if (rc != GQ_OK) return -rc;
    }
    gq::SchedOptions opt;
    if (tile_qubits > 0) opt.tile_qubits = tile_qubits;
    if (budget > 0) opt.budget = budget;
    opt.swizzle_width = precision == GQ_C64 ? 4 : 3;
    opt.low_qubits = precision == GQ_C64 ? 4 : 3;
    opt.support0 = g_support0;
    gq::Program prog;
    gq::schedule(gates, nphys, opt, prog);
    g_ctas = count_ctas(prog);
    for (size_t p = 0; p < prog.passes.size() && (int64_t)p < max_passes; ++p) {
        const gq::PassDesc& pd = prog.passes[p];
        int64_t n = 0, cost = 0, tmask = 0;
        for (int b = 0; b < pd.m; ++b) tmask |= 1ll << pd.tile_q[b];
        for (int f = pd.phase0; f < pd.phase0 + pd.n_phases; ++f)
            for (int k = prog.phases[f].op_begin; k < prog.phases[f].op_end; ++k) {
                static const int c[] = {0, 8, 16, 32, 64, 1, 1, 3, 1, 4, 16, 6};
                const gq::KOp& op = prog.ops[k];
                cost += c[op.type];
                ++n;
            }
        int64_t* o = out + 5 * p;
        o[0] = pd.n_phases;
        o[1] = n;
        o[2] = cost;
        o[3] = tmask;
        o[4] = pd.n_outer;
    }
    return (int64_t)prog.passes.size();
}

// Density matrix: rho (dim*dim interleaved doubles, row-major) evolved by the
// density-matrix op stream through dm_gates, the scheduler and the tile code.
int gqx_emulate_dm(int nq, double* rho, const gq_op* ops, size_t n_ops, int tile_qubits, int budget) {
    const int nvec = 2 * nq;
    const int nphys = nvec < gq::RQ ? gq::RQ : nvec;
    std::vector<gq::NGate> gates;
    int rc = gq::dm_gates(nq, ops, n_ops, gates, g_err);
    if (rc != GQ_OK) return rc;
    gq::SchedOptions opt;
    opt.tile_qubits = tile_qubits > 0 ? tile_qubits : 11;
    if (budget > 0) opt.budget = budget;
    gq::Program prog;
    gq::schedule(gates, nphys, opt, prog);
    std::vector<gq::cplx<double>> st(1ull << nphys, {0.0, 0.0});
    std::memcpy(st.data(), rho, sizeof(double) * 2 * (1ull << nvec));
    run_program<double>(st, prog);
    std::memcpy(rho, st.data(), sizeof(double) * 2 * (1ull << nvec));
    return GQ_OK;
}

// Adjoint gradient on the host through the same reverse program and dual
// tile code as the device: psi forward, lambda = sum_t Re(c_t) P_t psi, then
// the reverse passes accumulating 2 Re <lambda| G |psi> per parameter.
static int emulate_adjoint_impl(int nq, const gq_op* ops, size_t n_ops, const gq_pauli_term* terms, size_t n_terms,
                                size_t n_params, int tile_qubits, int budget, double* grad_out, double* energy_out,
                                const char* csrc, const char* work, int64_t* jitted);

int gqx_emulate_adjoint(int nq, const gq_op* ops, size_t n_ops, const gq_pauli_term* terms, size_t n_terms,
                        size_t n_params, int tile_qubits, int budget, double* grad_out, double* energy_out) {
    return emulate_adjoint_impl(nq, ops, n_ops, terms, n_terms, n_params, tile_qubits, budget, grad_out, energy_out,
                                nullptr, nullptr, nullptr);
}

// The same gradient with the reverse passes run through the host form of the
// specialised dual kernels (jit_plan_dual): the generated code is compiled
// with the host compiler in `work` (tile_core.cuh from `csrc`).
// *jitted = reverse passes that ran generated code.
int gqx_jit_emulate_adjoint(int nq, const gq_op* ops, size_t n_ops, const gq_pauli_term* terms, size_t n_terms,
                            size_t n_params, int tile_qubits, int budget, double* grad_out, double* energy_out,
                            const char* csrc, const char* work, int64_t* jitted) {
    return emulate_adjoint_impl(nq, ops, n_ops, terms, n_terms, n_params, tile_qubits, budget, grad_out, energy_out,
                                csrc, work, jitted);
}

static int emulate_adjoint_impl(int nq, const gq_op* ops, size_t n_ops, const gq_pauli_term* terms, size_t n_terms,
                                size_t n_params, int tile_qubits, int budget, double* grad_out, double* energy_out,
                                const char* csrc, const char* work, int64_t* jitted) {
    const int nphys = nq < gq::RQ ? gq::RQ : nq;
    std::vector<gq::NGate> fwd, rev;
    std::vector<int> fo, ro;
    int rc = gq::adjoint_gates(nq, ops, n_ops, n_params, fwd, rev, fo, ro, g_err);
    if (rc != GQ_OK) return rc;
    gq::SchedOptions opt;
    if (tile_qubits > 0) opt.tile_qubits = tile_qubits;
    if (budget > 0) opt.budget = budget;
    gq::Program pf, pr;
    gq::schedule(fwd, nphys, opt, pf);
    gq::schedule(rev, nphys, opt, pr);
    const uint64_t n = 1ull << nphys;
    std::vector<gq::cplx<double>> psi(n, {0.0, 0.0}), lam(n, {0.0, 0.0});
    psi[0] = {1.0, 0.0};
    run_program<double>(psi, pf);
    double energy = 0.0;
    for (size_t t = 0; t < n_terms; ++t) {
        const uint64_t x = terms[t].x_mask, z = terms[t].z_mask;
        const int ny = __builtin_popcountll(x & z) & 3;
        const double c = terms[t].coeff_re;
        double wr = c, wi = 0;
        if (ny == 1) wr = 0, wi = c;
        if (ny == 2) wr = -c, wi = 0;
        if (ny == 3) wr = 0, wi = -c;
        for (uint64_t i = 0; i < (1ull << nq); ++i) {
            const uint64_t j = i ^ x;
            const double sg = (__builtin_popcountll(j & z) & 1) ? -1.0 : 1.0;
            const gq::cplx<double> v = psi[j];
            lam[i].x += sg * (wr * v.x - wi * v.y);
            lam[i].y += sg * (wr * v.y + wi * v.x);
        }
    }
    for (uint64_t i = 0; i < n; ++i) energy += psi[i].x * lam[i].x + psi[i].y * lam[i].y;
    std::vector<double> grad(n_params, 0.0);
    std::vector<gq::cplx<double>> pool(pr.pool.size());
    for (size_t i = 0; i < pool.size(); ++i) pool[i] = {pr.pool[i].re, pr.pool[i].im};
    // generated dual passes (host form), when asked for
    typedef void (*DualFn)(gq::cplx<double>*, gq::cplx<double>*, const gq::cplx<double>*, const gq::cplx<double>*,
                           const gq::PhaseDesc*, double*, int, gq::cplx<double>*, double*);
    std::vector<gq::JitPlan> plans(csrc ? pr.passes.size() : 0);
    std::vector<char> planned(plans.size(), 0);
    void* lib = nullptr;
    if (csrc) {
        std::string src;
        for (size_t i = 0; i < pr.passes.size(); ++i) {
            const int threads = 1 << (pr.passes[i].m - gq::RQ);
            if (!gq::jit_plan_dual(pr, i, false, threads, 1, plans[i], true)) continue;
            planned[i] = 1;
            src += plans[i].host_source;
        }
        const std::string dir = work;
        const std::string cpp = dir + "/gqj_hostdual.cpp", so = dir + "/gqj_hostdual.so";
        FILE* f = std::fopen(cpp.c_str(), "w");
        if (!f) {
            g_err = "cannot write " + cpp;
            return GQ_EINVAL;
        }
        std::fwrite(src.data(), 1, src.size(), f);
        std::fclose(f);
        const std::string cmd = "g++ -O1 -std=c++17 -shared -fPIC -w -I'" + std::string(csrc) + "' '" + cpp +
                                "' -o '" + so + "' 2>'" + dir + "/gqj_hostdual.log'";
        if (std::system(cmd.c_str()) != 0) {
            g_err = "host compile of the generated dual passes failed (" + dir + "/gqj_hostdual.log)";
            return GQ_EINVAL;
        }
        lib = dlopen(so.c_str(), RTLD_NOW | RTLD_LOCAL);
        if (!lib) {
            g_err = dlerror();
            return GQ_EINVAL;
        }
        *jitted = 0;
    }
    for (size_t pi = 0; pi < pr.passes.size(); ++pi) {
        const gq::PassDesc& pd = pr.passes[pi];
        DualFn fn = nullptr;
        std::vector<gq::cplx<double>> block;
        if (lib && planned[pi]) {
            block.resize(plans[pi].n_param);
            if (gq::jit_pack(pr, pi, plans[pi], false, block.data()))
                fn = (DualFn)dlsym(lib, ("gqj_hostdual_" + std::to_string(pi)).c_str());
        }
        if (fn) {
            const int nslots = (int)pr.pass_params[pi].size();
            const uint64_t nc = 1ull << pd.n_outer;
            std::vector<double> part(nc * (size_t)std::max(1, nslots)), gsm(4 * gq::MAX_GRAD_SLOTS);
            std::vector<gq::cplx<double>> smem(2u << pd.m);
            uint32_t op_base, pool_base;
            gq::jit_bases(pr, pi, &op_base, &pool_base);
            fn(psi.data(), lam.data(), block.data(), pool.data() + pool_base, pr.phases.data() + pd.phase0,
               part.data(), nslots, smem.data(), gsm.data());
            for (int sl = 0; sl < nslots; ++sl) {
                double tot = 0.0;
                for (uint64_t c = 0; c < nc; ++c) tot += part[c * nslots + sl];
                grad[pr.pass_params[pi][sl]] += 2.0 * tot;
            }
            ++*jitted;
            continue;
        }
        const int m = pd.m;
        const uint32_t tpb = 1u << (m - gq::RQ);
        std::vector<gq::cplx<double>> sa(1u << m), sb(1u << m);
        std::vector<double> slots(gq::MAX_GRAD_SLOTS, 0.0);
        for (uint64_t cta = 0; cta < (1ull << pd.n_outer); ++cta) {
            const uint64_t base = gq::cta_base(pd, cta);
            for (uint32_t lin = 0; lin < (1u << m); ++lin) {
                uint64_t goff;
                uint32_t slot;
                gq::linear_slot(pd, lin, goff, slot);
                sa[slot] = psi[base | goff];
                sb[slot] = lam[base | goff];
            }
            for (int p = 0; p < pd.n_phases; ++p)
                for (uint32_t t = 0; t < tpb; ++t)
                    gq::run_phase_dual<double>(sa.data(), sb.data(), pr.phases[pd.phase0 + p], pr.ops.data(), pool.data(),
                                               t, base, [&](uint32_t s, double v) { slots[s] += v; });
            for (uint32_t lin = 0; lin < (1u << m); ++lin) {
                uint64_t goff;
                uint32_t slot;
                gq::linear_slot(pd, lin, goff, slot);
                psi[base | goff] = sa[slot];
                lam[base | goff] = sb[slot];
            }
        }
        for (size_t sl = 0; sl < pr.pass_params[pi].size(); ++sl) grad[pr.pass_params[pi][sl]] += 2.0 * slots[sl];
    }
    if (lib) dlclose(lib);
    for (size_t i = 0; i < n_params; ++i) grad_out[i] = grad[i];
    if (energy_out) *energy_out = energy;
    return GQ_OK;
}

// Specialised pass kernels without a device: schedules `ops` (a statevector
// program, or with dm != 0 the density-matrix program of an n-qubit rho) the
// way the engine does, generates the kernel text of every pass and compiles
// up to `max_compile` distinct texts with NVRTC for sm_100a.
// out: [passes, passes with a kernel text, distinct texts, compiled, compiled
// with register spills]. GQ_EUNSUPPORTED when libnvrtc cannot be loaded.
int gqx_jit_check(int nq, int precision, const gq_op* ops, size_t n_ops, int tile_qubits, int budget, int dm,
                  int max_compile, int64_t* out) {
    if (!gq::jit_available()) {
        g_err = "libnvrtc not found";
        return GQ_EUNSUPPORTED;
    }
    std::vector<gq::NGate> gates;
    int nphys;
    if (dm) {
        nphys = 2 * nq < gq::RQ ? gq::RQ : 2 * nq;
        const int rc = gq::dm_gates(nq, ops, n_ops, gates, g_err);
        if (rc != GQ_OK) return rc;
    } else {
        nphys = nq < gq::RQ ? gq::RQ : nq;
        for (size_t i = 0; i < n_ops; ++i) {
            const int rc = gq::normalize_op(ops[i], nphys, gates, g_err);
            if (rc != GQ_OK) return rc;
        }
    }
    gq::SchedOptions opt;
    opt.tile_qubits = tile_qubits > 0 ? tile_qubits : 11;  // the engine's default launch shapes: 128 threads
    opt.budget = budget > 0 ? budget : 320;
    opt.swizzle_width = precision == GQ_C64 ? 4 : 3;
    opt.low_qubits = precision == GQ_C64 ? 4 : 3;
    gq::Program prog;
    gq::schedule(gates, nphys, opt, prog);
    std::set<std::string> texts;
    int64_t planned = 0, compiled = 0, spills = 0;
    for (size_t i = 0; i < prog.passes.size(); ++i) {
        gq::JitPlan pl;
        const int threads = 1 << (prog.passes[i].m - gq::RQ);
        // the engine's default shape (persistent: the 12-qubit-tile shape's 2 CTAs per SM)
        if (!gq::jit_plan(prog, i, precision == GQ_C64, threads, g_persistent ? 2 : 4, g_persistent, pl)) continue;
        ++planned;
        if (!texts.insert(pl.source).second || compiled >= max_compile) continue;
        std::string log;
        const std::string err = gq::jit_compile_only(pl.source, nullptr, &log);
        if (!err.empty()) {
            g_err = err.substr(0, 4000);
            return GQ_ECUDA;
        }
        ++compiled;
        if (log.find(" 0 bytes spill stores") == std::string::npos) ++spills;
    }
    out[0] = (int64_t)prog.passes.size();
    out[1] = planned;
    out[2] = (int64_t)texts.size();
    out[3] = compiled;
    out[4] = spills;
    return GQ_OK;
}

// The specialised kernels' code run on the CPU (see run_program_jit): a
// statevector program (dm = 0, `state` 2^nq amplitudes) or the density-matrix
// program of an nq-qubit rho (dm = 1, `state` 4^nq amplitudes), scheduled
// as the engine does. csrc: directory of tile_core.cuh; work: a writable
// directory for the generated library. out = {passes, passes run specialised}.
int gqx_jit_emulate(int nq, int precision, double* state, const gq_op* ops, size_t n_ops, int tile_qubits,
                    int budget, int dm, const char* csrc, const char* work, int64_t* out) {
    std::vector<gq::NGate> gates;
    const int nvec = dm ? 2 * nq : nq;
    const int nphys = nvec < gq::RQ ? gq::RQ : nvec;
    if (dm) {
        const int rc = gq::dm_gates(nq, ops, n_ops, gates, g_err);
        if (rc != GQ_OK) return rc;
    } else {
        for (size_t i = 0; i < n_ops; ++i) {
            const int rc = gq::normalize_op(ops[i], nphys, gates, g_err);
            if (rc != GQ_OK) return rc;
        }
    }
    gq::SchedOptions opt;
    opt.tile_qubits = tile_qubits > 0 ? tile_qubits : 11;
    opt.budget = budget > 0 ? budget : 320;
    opt.swizzle_width = precision == GQ_C64 ? 4 : 3;
    opt.low_qubits = precision == GQ_C64 ? 4 : 3;
    opt.support0 = g_support0;
    gq::Program prog;
    gq::schedule(gates, nphys, opt, prog);
    g_ctas = count_ctas(prog);
    const uint64_t n = 1ull << nphys, nv = 1ull << nvec;
    int64_t jitted = 0;
    int rc;
    if (precision == GQ_C64) {
        std::vector<gq::cplx<float>> st(n, {0.f, 0.f});
        for (uint64_t i = 0; i < nv; ++i) st[i] = {(float)state[2 * i], (float)state[2 * i + 1]};
        rc = run_program_jit<float>(st, prog, true, csrc, work, &jitted);
        for (uint64_t i = 0; i < nv; ++i) {
            state[2 * i] = st[i].x;
            state[2 * i + 1] = st[i].y;
        }
    } else {
        std::vector<gq::cplx<double>> st(n, {0.0, 0.0});
        std::memcpy(st.data(), state, sizeof(double) * 2 * nv);
        rc = run_program_jit<double>(st, prog, false, csrc, work, &jitted);
        std::memcpy(state, st.data(), sizeof(double) * 2 * nv);
    }
    out[0] = (int64_t)prog.passes.size();
    out[1] = jitted;
    return rc;
}

// What the specialised statevector kernels of `ops` use, scheduled as the
// engine does: out = [passes, passes with a kernel text, fused one-qubit
// chains, chain candidates, phases with CTA-uniform predicates, phases with
// run-time phase accumulators].
int gqx_jit_plan_stats(int nq, int precision, const gq_op* ops, size_t n_ops, int tile_qubits, int budget,
                       int64_t* out) {
    std::vector<gq::NGate> gates;
    const int nphys = nq < gq::RQ ? gq::RQ : nq;
    for (size_t i = 0; i < n_ops; ++i) {
        const int rc = gq::normalize_op(ops[i], nphys, gates, g_err);
        if (rc != GQ_OK) return rc;
    }
    gq::SchedOptions opt;
    opt.tile_qubits = tile_qubits > 0 ? tile_qubits : 11;
    opt.budget = budget > 0 ? budget : 320;
    opt.swizzle_width = precision == GQ_C64 ? 4 : 3;
    opt.low_qubits = precision == GQ_C64 ? 4 : 3;
    gq::Program prog;
    gq::schedule(gates, nphys, opt, prog);
    int64_t planned = 0, chains = 0, cands = 0, pred_phases = 0, acc_phases = 0;
    for (size_t i = 0; i < prog.passes.size(); ++i) {
        gq::JitPlan pl;
        cands += (int64_t)gq::jit_chains(prog, i).size();
        if (!gq::jit_plan(prog, i, precision == GQ_C64, 1 << (prog.passes[i].m - gq::RQ), 4, false, pl)) continue;
        ++planned;
        chains += (int64_t)pl.chains.size();
        for (size_t at = 0; (at = pl.source.find("const uint32_t pc =", at)) != std::string::npos; ++at) ++pred_phases;
        for (size_t at = 0; (at = pl.source.find("cplx<T> rq", at)) != std::string::npos; ++at) ++acc_phases;
    }
    out[0] = (int64_t)prog.passes.size();
    out[1] = planned;
    out[2] = chains;
    out[3] = cands;
    out[4] = pred_phases;
    out[5] = acc_phases;
    return GQ_OK;
}

// The reverse sweep of an adjoint gradient as specialised dual kernels: the
// reverse program of `ops` scheduled as the engine does (11-qubit tiles),
// each pass's dual kernel text compiled with NVRTC at the engine's launch
// bounds. out: [passes, passes with a kernel text, compiled].
int gqx_jit_check_dual(int nq, int precision, const gq_op* ops, size_t n_ops, size_t n_params, int max_compile,
                       int64_t* out) {
    if (!gq::jit_available()) {
        g_err = "libnvrtc not found";
        return GQ_EUNSUPPORTED;
    }
    const int nphys = nq < gq::RQ ? gq::RQ : nq;
    std::vector<gq::NGate> fwd, rev;
    std::vector<int> fo, ro;
    int rc = gq::adjoint_gates(nq, ops, n_ops, n_params, fwd, rev, fo, ro, g_err);
    if (rc != GQ_OK) return rc;
    gq::SchedOptions opt;
    opt.tile_qubits = 11;
    opt.budget = 320;
    opt.swizzle_width = precision == GQ_C64 ? 4 : 3;
    opt.low_qubits = precision == GQ_C64 ? 4 : 3;
    gq::Program pr;
    gq::schedule(rev, nphys, opt, pr);
    std::set<std::string> texts;
    int64_t planned = 0, compiled = 0;
    for (size_t i = 0; i < pr.passes.size(); ++i) {
        gq::JitPlan pl;
        const int threads = 1 << (pr.passes[i].m - gq::RQ);
        if (!gq::jit_plan_dual(pr, i, precision == GQ_C64, threads, 2, pl)) continue;
        ++planned;
        if (!texts.insert(pl.source).second || compiled >= max_compile) continue;
        std::string log;
        const std::string err = gq::jit_compile_only(pl.source, nullptr, &log);
        if (!err.empty()) {
            g_err = err.substr(0, 4000);
            return GQ_ECUDA;
        }
        ++compiled;
    }
    out[0] = (int64_t)pr.passes.size();
    out[1] = planned;
    out[2] = compiled;
    return GQ_OK;
}

// The adjoint's checkpoint policy (gq::adjoint_segments) with the device's
// free memory given by the caller: the same host function the engine calls
// after cudaMemGetInfo.
int gqx_adjoint_segments(int requested, int c64, uint64_t n_ops, uint64_t state_bytes, uint64_t avail_bytes) {
    return gq::adjoint_segments(requested, c64 != 0, (size_t)n_ops, (size_t)state_bytes, (size_t)avail_bytes);
}

// A parameterized gate family's matrix (k < 0) or its derivative with
// respect to angle k, as the engine binds it; out holds 2 * dim^2 doubles.
int gqx_param_gate(int family, const double* angles, int n_angles, int k, double* out) {
    std::vector<gq::Z> m;
    const bool ok = k < 0 ? gq::param_gate_matrix(family, angles, n_angles, m)
                          : gq::param_gate_dmatrix(family, angles, n_angles, k, m);
    if (!ok) return GQ_EINVAL;
    std::memcpy(out, m.data(), m.size() * sizeof(gq::Z));
    return (int)m.size();
}

// FNV-1a digest of the plan-cache keys of every reverse (adjoint) pass the
// engine would run for `ops`: equal digests mean the specialised kernels
// compiled for one binding serve the other.
int gqx_adjoint_plan_digest(int nq, int precision, const gq_op* ops, size_t n_ops, size_t n_params, uint64_t* digest,
                            int64_t* passes) {
    const int nphys = nq < gq::RQ ? gq::RQ : nq;
    std::vector<gq::NGate> fwd, rev;
    std::vector<int> fo, ro;
    int rc = gq::adjoint_gates(nq, ops, n_ops, n_params, fwd, rev, fo, ro, g_err);
    if (rc != GQ_OK) return rc;
    gq::SchedOptions opt;
    opt.tile_qubits = 11;
    opt.budget = 320;
    opt.swizzle_width = precision == GQ_C64 ? 4 : 3;
    opt.low_qubits = precision == GQ_C64 ? 4 : 3;
    gq::Program pr;
    gq::schedule(rev, nphys, opt, pr);
    uint64_t h = 1469598103934665603ull;
    for (size_t i = 0; i < pr.passes.size(); ++i) {
        const std::string k = gq::jit_plan_key(pr, i, precision == GQ_C64, 1 << (pr.passes[i].m - gq::RQ), 2, false, true);
        for (unsigned char ch : k) h = (h ^ ch) * 1099511628211ull;
    }
    *digest = h;
    *passes = (int64_t)pr.passes.size();
    return GQ_OK;
}

// jit_compile_cached on a kernel text (cache directory from the environment):
// *from_disk tells whether the cubin came from the cache; returns its size.
int64_t gqx_jit_compile_cached(const char* source, int* from_disk) {
    std::vector<char> bin;
    std::string log;
    bool disk = false;
    const std::string err = gq::jit_compile_cached(source, &bin, &log, &disk);
    if (!err.empty()) {
        g_err = err.substr(0, 4000);
        return -1;
    }
    *from_disk = disk ? 1 : 0;
    return (int64_t)bin.size();
}

}  // extern "C"

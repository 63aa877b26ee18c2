// Specialised tile-pass kernels: code generation and NVRTC compilation (see
// jit.hpp). Needs no device; the emulator library links it for the CPU tests.
#include "jit.hpp"

#include <dlfcn.h>
#include <nvrtc.h>

#include <cstdio>
#include <cstring>

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

int ctz64(uint64_t v) { return __builtin_ctzll(v); }

// Emits `dst |= (uint64_t)((src >> from) & mask) << to` for every run of bit k
// of `src` (k = 0..n-1) going to qubit q[k], merging runs of consecutive
// positions into one shift.
void emit_deposit(std::string& s, const char* dst, const char* src, const int* q, int n) {
    int k = 0;
    while (k < n) {
        int len = 1;
        while (k + len < n && q[k + len] == q[k] + len) ++len;
        const uint64_t mask = len >= 64 ? ~0ull : ((1ull << len) - 1);
        s += "    ";
        s += dst;
        s += " |= ((uint64_t)(";
        s += src;
        s += " >> " + std::to_string(k) + ") & " + hex64(mask) + ") << " + std::to_string(q[k]) + ";\n";
        k += len;
    }
}

int mat_len(const KOp& op) {
    switch (op.type) {
        case K_U1: return 4;
        case K_U2: return 16;
        case K_U3: return 64;
        case K_U4: return 256;
        case K_X: return (op.flags & 1) ? 0 : 2;
        case K_PHASE: return 1;
        default: return 0;
    }
}

}  // namespace

bool jit_plan(const Program& pr, size_t pi, bool c64, int threads, int min_blocks, JitPlan& out) {
    const PassDesc& pd = pr.passes[pi];
    const int m = pd.m, tbits = m - RQ;
    if (tbits < 0 || (1 << tbits) != threads) return false;
    out.copies.clear();
    const uint32_t cap = c64 ? 3900u : 1950u;  // parameter block entries (32 KB of kernel parameters)
    uint32_t np = 0;

    std::string b;  // kernel body
    b.reserve(1 << 16);
    b += "    const uint32_t t = threadIdx.x;\n    const uint64_t cta = blockIdx.x;\n    uint64_t base = 0;\n";
    emit_deposit(b, "base", "cta", pd.outer_q, pd.n_outer);
    // staging: thread bits are tile bits [0, tbits), the 16 register slots
    // of the linear staging are tile bits [tbits, m)
    b += "    uint64_t gt = base;\n    uint32_t stt = 0;\n";
    emit_deposit(b, "gt", "t", pd.tile_q, tbits);
    for (int k = 0; k < tbits; ++k)
        b += "    stt ^= (0u - ((t >> " + std::to_string(k) + ") & 1u)) & " + hex32(pd.acol[k]) + ";\n";
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
    b += "    {\n        cplx<T> v[16];\n";
    for (int it = 0; it < NREG; ++it) b += "        v[" + std::to_string(it) + "] = st[gt | " + hex64(G[it]) + "];\n";
    for (int it = 0; it < NREG; ++it)
        b += "        sm[stt ^ " + hex32(S[it]) + "] = v[" + std::to_string(it) + "];\n";
    b += "    }\n    __syncthreads();\n";

    for (int p = 0; p < pd.n_phases; ++p) {
        const int phi = pd.phase0 + p;
        const PhaseDesc& ph = pr.phases[phi];
        // thread-bit columns of the phase's tables
        uint32_t tslot[MAX_TILE];
        int tq[MAX_TILE];
        for (int k = 0; k < tbits; ++k) {
            const uint32_t s = k < 4 ? ph.tlo_slot[1u << k] : ph.thi_slot[1u << (k - 4)];
            const uint64_t g = k < 4 ? ph.tlo_glob[1u << k] : ph.thi_glob[1u << (k - 4)];
            if (g == 0 || (g & (g - 1))) return false;
            tslot[k] = s;
            tq[k] = ctz64(g);
        }
        // the tables must be the XOR / OR of those columns
        for (int v = 0; v < TLO && v < (1 << tbits); ++v) {
            uint32_t s = 0;
            uint64_t g = 0;
            for (int k = 0; k < 4 && k < tbits; ++k)
                if ((v >> k) & 1) {
                    s ^= tslot[k];
                    g |= 1ull << tq[k];
                }
            if (s != ph.tlo_slot[v] || g != ph.tlo_glob[v]) return false;
        }
        b += "    {\n        uint32_t sb = 0;\n        uint64_t g0 = base;\n";
        for (int k = 0; k < tbits; ++k)
            b += "        sb ^= (0u - ((t >> " + std::to_string(k) + ") & 1u)) & " + hex32(tslot[k]) + ";\n";
        {
            std::string d;
            emit_deposit(d, "g0", "t", tq, tbits);
            b += d;
        }
        b += "        cplx<T> a[16];\n";
        for (int j = 0; j < NREG; ++j)
            b += "        a[" + std::to_string(j) + "] = sm[sb ^ " + hex32(ph.rslot[j]) + "];\n";
        for (int o = ph.op_begin; o < ph.op_end; ++o) {
            const KOp& op = pr.ops[o];
            if (op.type == K_GRAD || op.type == K_NONE || op.type > K_RESET) return false;
            const int ml = mat_len(op);
            std::string M;
            if (ml > 0 && np + (uint32_t)ml <= cap) {
                M = "PMat<T>{p.m + " + std::to_string(np) + "}";
                out.copies.push_back({op.mat, (uint32_t)ml});
                np += (uint32_t)ml;
            } else {
                M = "(pool + " + std::to_string(op.mat) + "u)";
            }
            const std::string creg = std::to_string(op.creg) + "u";
            const std::string C = op.creg ? "true" : "false";
            std::string cond;
            if (op.cmask) cond = "if ((g0 & " + hex64(op.cmask) + ") == " + hex64(op.cmask) + ") ";
            const std::string S0 = std::to_string(op.t0), S1 = std::to_string(op.t1), S2 = std::to_string(op.t2);
            std::string call;
            switch (op.type) {
                case K_U1: call = "k_u1<T, " + S0 + ", " + C + ">(a, " + M + ", " + creg + ");"; break;
                case K_U2: call = "k_u2<T, " + S0 + ", " + S1 + ", " + C + ">(a, " + M + ", " + creg + ");"; break;
                case K_U3: call = "k_u3<T, " + S0 + ", " + S1 + ", " + S2 + ">(a, " + M + ", " + creg + ");"; break;
                case K_U4:
                    call = "k_u4<T>(a, " + M + ", sm, sb, phases[" + std::to_string(phi) + "].rslot);";
                    break;
                case K_X:
                    call = "k_x<T, " + S0 + ", " + C + ">(a, " + ((op.flags & 1) ? std::string("pool") : M) + ", " +
                           creg + ", " + ((op.flags & 1) ? "true" : "false") + ");";
                    break;
                case K_SWAP: call = "k_swap<T, " + S0 + ", " + S1 + ">(a, " + creg + ");"; break;
                case K_PHASE: call = "k_phase<T>(a, ldc(" + M + ", 0), " + creg + ");"; break;
                case K_RESET: call = "k_reset<T, " + S0 + ">(a);"; break;
                case K_DIAG: {
                    std::string h = "{ uint32_t hi = 0; ";
                    int k = 0;
                    for (uint64_t dm = op.dmask; dm; dm &= dm - 1, ++k)
                        h += "hi |= (uint32_t)((g0 >> " + std::to_string(ctz64(dm)) + ") & 1ull) << " +
                             std::to_string(k) + "; ";
                    h += "k_diag_hi<T>(a, pool + " + std::to_string(op.mat) + "u, hi << " + std::to_string(op.nreg) +
                         ", " + std::to_string(op.nreg) + "u, " + creg + ", " + hex64(op.ridx) + "); }";
                    call = h;
                    break;
                }
                default: return false;
            }
            b += "        " + cond + call + "\n";
        }
        for (int j = 0; j < NREG; ++j)
            b += "        sm[sb ^ " + hex32(ph.rslot[j]) + "] = a[" + std::to_string(j) + "];\n";
        b += "    }\n    __syncthreads();\n";
    }
    b += "    {\n        cplx<T> v[16];\n";
    for (int it = 0; it < NREG; ++it)
        b += "        v[" + std::to_string(it) + "] = sm[stt ^ " + hex32(S[it]) + "];\n";
    for (int it = 0; it < NREG; ++it) b += "        st[gt | " + hex64(G[it]) + "] = v[" + std::to_string(it) + "];\n";
    b += "    }\n";

    out.n_param = np > 0 ? np : 1;
    const char* T = c64 ? "float" : "double";
    std::string& s = out.source;
    s.clear();
    s.reserve(b.size() + 1024);
    s += "// goqu_b200 specialised tile pass\n";
    s += "typedef unsigned char uint8_t;\ntypedef int int32_t;\ntypedef unsigned int uint32_t;\n";
    s += "typedef long long int64_t;\ntypedef unsigned long long uint64_t;\n";
    s += "#include \"tile_core.cuh\"\n";
    s += "namespace gq {\nstruct JP {\n    cplx<" + std::string(T) + "> m[" + std::to_string(out.n_param) + "];\n};\n}\n";
    s += "extern \"C\" __global__ void __launch_bounds__(" + std::to_string(threads) + ", " +
         std::to_string(min_blocks) + ")\n";
    s += "gqj_pass(gq::cplx<" + std::string(T) + ">* __restrict__ st, const __grid_constant__ gq::JP p, const gq::cplx<" +
         std::string(T) + ">* __restrict__ pool, const gq::PhaseDesc* __restrict__ phases) {\n";
    s += "    using namespace gq;\n    using T = " + std::string(T) + ";\n";
    s += "    extern __shared__ __align__(16) unsigned char smraw[];\n";
    s += "    cplx<T>* sm = reinterpret_cast<cplx<T>*>(smraw);\n";
    s += "    (void)pool;\n    (void)phases;\n";
    s += b;
    s += "}\n";
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
        ok = create && compile && log_size && log && cubin_size && cubin && destroy;
    }
};

Nvrtc& nvrtc() {
    static Nvrtc n;
    return n;
}

}  // namespace

bool jit_available() { return nvrtc().ok; }

std::string jit_compile_only(const std::string& source, std::vector<char>* cubin, std::string* log) {
    Nvrtc& N = nvrtc();
    if (!N.ok) return "libnvrtc not found";
    nvrtcProgram prog;
    const char* hdr_src[] = {kTileCore};
    const char* hdr_name[] = {"tile_core.cuh"};
    if (N.create(&prog, source.c_str(), "gqj_pass.cu", 1, hdr_src, hdr_name) != NVRTC_SUCCESS)
        return "nvrtcCreateProgram failed";
    const char* opts[] = {"--gpu-architecture=sm_100a", "-std=c++17", "--ptxas-options=-v"};
    const nvrtcResult rc = N.compile(prog, 3, opts);
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

}  // namespace gq

// Specialised tile-pass kernels: the process-wide cache, compilation on
// worker threads and loading (see jit.hpp).
#include "jit.hpp"

#include <chrono>
#include <cstdlib>
#include <condition_variable>
#include <deque>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>

namespace gq {

namespace {

struct Entry {
    JitState state = JIT_PENDING;
    std::vector<char> cubin;
    cudaLibrary_t lib = nullptr;
    cudaKernel_t kernel = nullptr;
    uint64_t smem_devices = 0;  // devices the shared-memory attribute was raised on
    std::string log;
};

struct Cache {
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::unordered_map<std::string, std::unique_ptr<Entry>> map;
    std::deque<const std::string*> queue;
    int busy = 0;
    bool stopping = false;
    std::vector<std::thread> workers;
    double compile_ms = 0;
    int64_t compiled = 0, failed = 0, from_cache = 0;

    void start() {
        if (!workers.empty()) return;
        unsigned n = std::thread::hardware_concurrency();
        n = n == 0 ? 2 : (n > 16 ? 16 : n);
        for (unsigned i = 0; i < n; ++i) {
            workers.emplace_back([this] { run(); });
            workers.back().detach();
        }
        std::atexit(drain_at_exit);
    }
    // At process exit: drop queued work and let compilations in flight end
    // before the compiler library is unloaded under them.
    static void drain_at_exit();
    void run() {
        for (;;) {
            const std::string* key;
            {
                std::unique_lock<std::mutex> lk(mu);
                cv_work.wait(lk, [&] { return !queue.empty() || stopping; });
                if (stopping) return;
                key = queue.front();
                queue.pop_front();
                ++busy;
            }
            std::vector<char> bin;
            std::string log;
            const auto t0 = std::chrono::steady_clock::now();
            bool from_disk = false;
            const std::string err = jit_compile_cached(*key, &bin, &log, &from_disk);
            const double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
            {
                std::lock_guard<std::mutex> lk(mu);
                Entry& e = *map[*key];
                compile_ms += ms;
                if (err.empty()) {
                    e.cubin.swap(bin);
                    e.state = JIT_PENDING;  // compiled (or read from disk); loaded by the next lookup
                    ++compiled;
                    if (from_disk) ++from_cache;
                } else {
                    e.state = JIT_FAILED;
                    ++failed;
                }
                e.log = err.empty() ? log : err;
                --busy;
            }
            cv_done.notify_all();
        }
    }
};

Cache& cache() {
    static Cache* c = new Cache();  // never destroyed: worker threads are detached
    return *c;
}

void Cache::drain_at_exit() {
    Cache& c = cache();
    std::unique_lock<std::mutex> lk(c.mu);
    c.stopping = true;
    for (const std::string* k : c.queue) c.map[*k]->state = JIT_FAILED;
    c.queue.clear();
    c.cv_work.notify_all();
    c.cv_done.wait_for(lk, std::chrono::seconds(60), [&] { return c.busy == 0; });
}

}  // namespace

JitState jit_lookup(const std::string& source, size_t smem_bytes, bool queue, const void** fn) {
    Cache& c = cache();
    std::lock_guard<std::mutex> lk(c.mu);
    auto it = c.map.find(source);
    if (it == c.map.end()) {
        if (!queue || !jit_available()) return JIT_MISSING;
        c.start();
        auto ins = c.map.emplace(source, std::unique_ptr<Entry>(new Entry()));
        c.queue.push_back(&ins.first->first);
        c.cv_work.notify_one();
        return JIT_PENDING;
    }
    Entry& e = *it->second;
    if (e.state == JIT_PENDING && !e.cubin.empty()) {
        // libraries and kernels are context independent: one load serves every device
        cudaError_t err = cudaLibraryLoadData(&e.lib, e.cubin.data(), nullptr, nullptr, 0, nullptr, nullptr, 0);
        const char* name = source.find("\ngqj_dual(") != std::string::npos ? "gqj_dual" : "gqj_pass";
        if (err == cudaSuccess) err = cudaLibraryGetKernel(&e.kernel, e.lib, name);
        if (err != cudaSuccess) {
            e.state = JIT_FAILED;
            e.log = cudaGetErrorString(err);
            (void)cudaGetLastError();
            return JIT_FAILED;
        }
        std::vector<char>().swap(e.cubin);
        e.state = JIT_READY;
    }
    if (e.state != JIT_READY) return e.state;
    if (smem_bytes > 48 * 1024) {
        int dev = 0;
        if (cudaGetDevice(&dev) != cudaSuccess || dev >= 64) return JIT_FAILED;
        if (!((e.smem_devices >> dev) & 1)) {
            if (cudaKernelSetAttributeForDevice(e.kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_bytes,
                                                dev) != cudaSuccess) {
                (void)cudaGetLastError();
                return JIT_FAILED;
            }
            e.smem_devices |= 1ull << dev;
        }
    }
    if (fn) *fn = (const void*)e.kernel;
    return JIT_READY;
}

namespace {

struct PlanCache {
    std::mutex mu;
    std::unordered_map<std::string, std::unique_ptr<CachedPlan>> map;
};

PlanCache& plan_cache() {
    static PlanCache* c = new PlanCache();
    return *c;
}


}  // namespace

const CachedPlan* jit_cached_plan(const Program& pr, size_t pi, bool c64, int threads, int min_blocks,
                                  bool persistent, bool dual) {
    const std::string key = jit_plan_key(pr, pi, c64, threads, min_blocks, persistent, dual);
    PlanCache& pc = plan_cache();
    std::lock_guard<std::mutex> lk(pc.mu);
    auto it = pc.map.find(key);
    if (it != pc.map.end()) return it->second.get();
    if (pc.map.size() >= 8192) pc.map.clear();  // bound the cache; plans are regenerated on demand
    std::unique_ptr<CachedPlan> cp(new CachedPlan());
    cp->ok = dual ? jit_plan_dual(pr, pi, c64, threads, min_blocks, cp->plan)
                  : jit_plan(pr, pi, c64, threads, min_blocks, persistent, cp->plan);
    const CachedPlan* r = cp.get();
    pc.map.emplace(std::move(key), std::move(cp));
    return r;
}

const void* jit_plan_kernel(const CachedPlan* ccp, size_t smem_bytes) {
    CachedPlan* cp = const_cast<CachedPlan*>(ccp);
    {
        std::lock_guard<std::mutex> lk(plan_cache().mu);
        if (cp->fn || cp->failed || !cp->ok) return cp->fn;
    }
    const void* fn = nullptr;
    const JitState st = jit_lookup(cp->plan.source, smem_bytes, true, &fn);
    std::lock_guard<std::mutex> lk(plan_cache().mu);
    if (st == JIT_READY) cp->fn = fn;
    if (st == JIT_FAILED) cp->failed = true;
    return cp->fn;
}

void jit_wait(double max_ms) {
    Cache& c = cache();
    std::unique_lock<std::mutex> lk(c.mu);
    c.cv_done.wait_for(lk, std::chrono::duration<double, std::milli>(max_ms),
                       [&] { return c.queue.empty() && c.busy == 0; });
}

void jit_counters(double* compile_ms, int64_t* compiled, int64_t* failed) {
    Cache& c = cache();
    std::lock_guard<std::mutex> lk(c.mu);
    if (compile_ms) *compile_ms = c.compile_ms;
    if (compiled) *compiled = c.compiled;
    if (failed) *failed = c.failed;
}

}  // namespace gq

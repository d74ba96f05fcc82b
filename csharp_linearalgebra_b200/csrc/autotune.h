// The autotuner: for the products that have more than one launch shape with
// identical results (the DMMA GEMM's small and big tiles, bit-identical by
// construction; the modular GEMM's 128- and 256-column tiles, exact integer
// arithmetic either way), the first launch of a size class runs both, timed
// with CUDA events on the context's stream, and records the faster for that
// class on that device. Later launches of the class take the recorded shape.
// A size class is (product kind, log2 of the launch's tiles at the big shape,
// log2 of its depth). Off by default (tns_set_autotune): the fixed rule is
// "big tiles when they fill the GPU".
#pragma once

#include "tns_internal.h"

#include <map>
#include <mutex>
#include <tuple>

namespace tns {

enum class TuneKind : int { kDmmaReal = 0, kDmmaComplex = 1, kSplitReal = 2, kSplitComplex = 3 };

struct TuneTable {
    std::mutex mu;
    std::map<std::tuple<int, int, int, int>, int> choice;  // (device, kind, tiles class, depth class) -> variant
};
inline TuneTable& tune_table() {
    static TuneTable t;
    return t;
}
inline int log2_class(long long v) {
    int b = 0;
    while (v > 1) {
        v >>= 1;
        ++b;
    }
    return b;
}
// The recorded variant (0 small, 1 big) for a size class, or -1.
inline int tuned_variant(int device, TuneKind kind, long long tiles, long long depth) {
    TuneTable& t = tune_table();
    std::lock_guard<std::mutex> g(t.mu);
    auto it = t.choice.find({device, (int)kind, log2_class(tiles), log2_class(depth)});
    return it == t.choice.end() ? -1 : it->second;
}
inline void record_variant(int device, TuneKind kind, long long tiles, long long depth, int variant) {
    TuneTable& t = tune_table();
    std::lock_guard<std::mutex> g(t.mu);
    t.choice[{device, (int)kind, log2_class(tiles), log2_class(depth)}] = variant;
}
inline void clear_tuning() {
    TuneTable& t = tune_table();
    std::lock_guard<std::mutex> g(t.mu);
    t.choice.clear();
}
// Device time of f()'s launches on the context's stream (waits for them).
template <class F>
float time_launches(Context& ctx, F&& f) {
    cudaEvent_t a = ctx.take_event(), b = ctx.take_event();
    TNS_CUDA(cudaEventRecord(a, ctx.stream));
    f();
    TNS_CUDA(cudaEventRecord(b, ctx.stream));
    TNS_CUDA(cudaEventSynchronize(b));
    float ms = 0.f;
    TNS_CUDA(cudaEventElapsedTime(&ms, a, b));
    ctx.event_pool.push_back(a);
    ctx.event_pool.push_back(b);
    return ms;
}

}  // namespace tns

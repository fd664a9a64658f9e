// Region timers (fsd_profile.h) and their C ABI.
#include <cuda_runtime.h>

#include <vector>

#include "fsd_profile.h"

namespace fsd {

struct Profiler {
    bool on = false;
    std::vector<cudaEvent_t> pool;
    size_t next = 0;
    std::vector<int> open[R_COUNT];                 // stack of start-event slots per region
    std::vector<std::pair<int, int>> pairs[R_COUNT];  // recorded (start, end) slots
    double ms[R_COUNT] = {};
    long long count[R_COUNT] = {};
    long long dropped = 0;  // regions not timed because no event could be had
};

static Profiler* prof(fsd_handle* h) { return (Profiler*)h->profiler; }

static void resolve(fsd_handle* h) {
    Profiler* p = prof(h);
    cudaStreamSynchronize(h->stream);
    for (int r = 0; r < R_COUNT; ++r) {
        for (auto& pr : p->pairs[r]) {
            float t = 0.f;
            if (cudaEventElapsedTime(&t, p->pool[pr.first], p->pool[pr.second]) == cudaSuccess) p->ms[r] += t;
            p->count[r] += 1;
        }
        p->pairs[r].clear();
    }
    p->next = 0;
}

// Next free event.  A full pool is resolved (one stream synchronisation) when
// no region is open; with regions open it grows instead, so no region is lost.
static int take(fsd_handle* h) {
    Profiler* p = prof(h);
    bool busy = false;
    for (int r = 0; r < R_COUNT; ++r) busy |= !p->open[r].empty();
    if (p->next >= p->pool.size() && !busy) resolve(h);
    if (p->next >= p->pool.size()) {
        cudaEvent_t e;
        if (cudaEventCreate(&e) != cudaSuccess) return -1;
        p->pool.push_back(e);
    }
    return (int)p->next++;
}

void profile_begin(fsd_handle* h, int region) {
    Profiler* p = prof(h);
    if (!p || !p->on) return;
    const int e = take(h);
    if (e < 0) {
        ++p->dropped;
        return;
    }
    cudaEventRecord(p->pool[e], h->stream);
    p->open[region].push_back(e);
}

void profile_end(fsd_handle* h, int region) {
    Profiler* p = prof(h);
    if (!p || !p->on || p->open[region].empty()) return;
    const int s = p->open[region].back();
    p->open[region].pop_back();
    const int e = take(h);
    if (e < 0) {
        ++p->dropped;
        return;
    }
    cudaEventRecord(p->pool[e], h->stream);
    p->pairs[region].push_back({s, e});
}

void profile_destroy(fsd_handle* h) {
    Profiler* p = prof(h);
    if (!p) return;
    for (auto e : p->pool) cudaEventDestroy(e);
    delete p;
    h->profiler = nullptr;
}

}  // namespace fsd

using namespace fsd;

extern "C" {

int fsd_profile_enable(fsd_handle* h, int on) {
    if (!h) return FSD_ERR_BAD_PARAMS;
    if (!h->profiler) {
        Profiler* p = new Profiler();
        p->pool.resize(16384);
        for (auto& e : p->pool)
            if (cudaEventCreate(&e) != cudaSuccess) return FSD_ERR_CUDA;
        h->profiler = p;
    }
    Profiler* p = prof(h);
    resolve(h);
    p->on = on != 0;
    return FSD_OK;
}

int fsd_profile_read(fsd_handle* h, double* ms, long long* counts, int n, int reset) {
    if (!h || !h->profiler || !ms || !counts || n < R_COUNT) return FSD_ERR_BAD_PARAMS;
    Profiler* p = prof(h);
    resolve(h);
    for (int r = 0; r < R_COUNT; ++r) {
        ms[r] = p->ms[r];
        counts[r] = p->count[r];
        if (reset) {
            p->ms[r] = 0.0;
            p->count[r] = 0;
        }
    }
    if (n > R_COUNT) {
        ms[R_COUNT] = 0.0;
        counts[R_COUNT] = p->dropped;
        if (reset) p->dropped = 0;
    }
    return FSD_OK;
}

}  // extern "C"

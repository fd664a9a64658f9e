// Batched stepping of independent suspensions (replicas): each handle steps
// on its own stream, driven by one of a pool of host threads, so the kernels
// of small replicas overlap on the GPU.  Every replica's step keeps its own
// host-side control flow (GMRES convergence polling, Lanczos), which is why
// the concurrency lives in host threads rather than in one device launch.
#include <algorithm>
#include <atomic>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

#include "fsd.h"
#include "fsd_internal.h"

extern "C" int fsd_step_batch(fsd_handle* const* hs, const fsd_step_args* args, int n, int nthreads,
                              int* status) {
    if (!hs || !args || n < 0) return FSD_ERR_BAD_PARAMS;
    for (int i = 0; i < n; ++i)
        if (!hs[i]) return FSD_ERR_BAD_PARAMS;
    const int nt = std::max(1, std::min(nthreads > 0 ? nthreads : n, n));
    std::atomic<int> next{0};
    std::vector<int> st(n, FSD_OK);
    auto work = [&]() {
        for (;;) {
            const int i = next.fetch_add(1);
            if (i >= n) return;
            if (cudaSetDevice(hs[i]->device) != cudaSuccess) {
                st[i] = FSD_ERR_CUDA;
                continue;
            }
            st[i] = fsd_step(hs[i], &args[i]);
        }
    };
    if (nt == 1) {
        work();
    } else {
        std::vector<std::thread> pool;
        pool.reserve(nt);
        for (int t = 0; t < nt; ++t) pool.emplace_back(work);
        for (auto& t : pool) t.join();
    }
    int first = FSD_OK;
    for (int i = 0; i < n; ++i) {
        if (status) status[i] = st[i];
        if (first == FSD_OK && st[i] != FSD_OK && st[i] != FSD_ERR_LANCZOS_MAXIT) first = st[i];
    }
    return first;
}

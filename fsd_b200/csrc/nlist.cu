// Neighbour list: every pair within r_list = ewald_cut + buffer, both
// directions, no self.  Replaces HOOMD's NeighborListGPUBinned as configured by
// PSEv3 (integrate.py:80-85: cell list, r_buff 0.4, rebuilt every step).
//
// Particles are binned into cells no narrower than r_list (measured between
// opposite faces of the sheared box), each cell's members are sorted by index,
// and each particle scans its 27 neighbouring cells in a fixed order, so row
// contents and order are deterministic.  Boxes with fewer than three cells
// along an axis fall back to an all-pairs scan.
#include <mutex>

#include "fsd.h"
#include "fsd_device.cuh"
#include "fsd_kernels.cuh"
#include "fsd_profile.h"

namespace fsd {

// ---------------------------------------------------------------- scan utility
// Exclusive scan of n unsigned values, out may alias in.  out[n] receives the
// total.  Uses block-level scans plus one pass over the block sums.
namespace {
constexpr int kScanThreads = 1024;
constexpr int kScanItems = 4;
constexpr int kScanTile = kScanThreads * kScanItems;

__device__ __forceinline__ unsigned block_exclusive_scan(unsigned v, unsigned* sh, unsigned* total) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    unsigned x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        unsigned y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) sh[wid] = x;
    __syncthreads();
    if (wid == 0) {
        unsigned s = (lane < (int)(blockDim.x >> 5)) ? sh[lane] : 0u;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            unsigned y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += y;
        }
        sh[lane] = s;
    }
    __syncthreads();
    const unsigned warp_off = wid ? sh[wid - 1] : 0u;
    if (total) *total = sh[(blockDim.x >> 5) - 1];
    return warp_off + x - v;
}

__global__ void scan_tiles(const unsigned* in, unsigned* out, unsigned* sums, int n) {
    __shared__ unsigned sh[32];
    const int base = blockIdx.x * kScanTile + threadIdx.x * kScanItems;
    unsigned v[kScanItems], s = 0;
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
        v[i] = (base + i < n) ? in[base + i] : 0u;
        s += v[i];
    }
    unsigned total;
    unsigned off = block_exclusive_scan(s, sh, &total);
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
        if (base + i < n) out[base + i] = off;
        off += v[i];
    }
    if (threadIdx.x == 0) sums[blockIdx.x] = total;
}

__global__ void scan_sums(unsigned* sums, int nb, unsigned* out_total) {
    __shared__ unsigned sh[32];
    unsigned carry = 0;
    for (int base = 0; base < nb; base += blockDim.x) {
        const int i = base + threadIdx.x;
        const unsigned v = (i < nb) ? sums[i] : 0u;
        unsigned total;
        const unsigned ex = block_exclusive_scan(v, sh, &total);
        if (i < nb) sums[i] = ex + carry;
        carry += total;
        __syncthreads();
    }
    if (threadIdx.x == 0) *out_total = carry;
}

__global__ void scan_add(unsigned* out, const unsigned* sums, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] += sums[i / kScanTile];
}
}  // namespace

size_t scan_scratch_elems(int n) { return (size_t)(n + kScanTile - 1) / kScanTile + 1; }

void exclusive_scan(const unsigned* in, unsigned* out, int n, unsigned* scratch, cudaStream_t st) {
    const int nb = (n + kScanTile - 1) / kScanTile;
    count_launch();
    scan_tiles<<<nb, kScanThreads, 0, st>>>(in, out, scratch, n);
    count_launch();
    scan_sums<<<1, kScanThreads, 0, st>>>(scratch, nb, out + n);
    count_launch();
    scan_add<<<(n + 255) / 256, 256, 0, st>>>(out, scratch, n);
}

// ----------------------------------------------------------- counting sort bins
__global__ void k_bin_fill(const unsigned* key, int n, const unsigned* start, unsigned* fill, unsigned* items) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const unsigned c = key[i];
    const unsigned slot = atomicAdd(&fill[c], 1u);
    items[start[c] + slot] = i;
}

// Sort each bin's members by particle index (bins hold few members).
__global__ void k_bin_sort(const unsigned* start, int nbins, unsigned* items) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nbins) return;
    const unsigned b = start[c], e = start[c + 1];
    for (unsigned i = b + 1; i < e; ++i) {
        const unsigned key = items[i];
        unsigned j = i;
        while (j > b && items[j - 1] > key) {
            items[j] = items[j - 1];
            --j;
        }
        items[j] = key;
    }
}

__global__ void k_bin_count(const unsigned* key, int n, unsigned* count) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) atomicAdd(&count[key[i]], 1u);
}

void counting_sort(const unsigned* key, int n, int nbins, unsigned* count, unsigned* start, unsigned* fill,
                   unsigned* items, unsigned* scan_scratch, cudaStream_t st) {
    cudaMemsetAsync(count, 0, sizeof(unsigned) * nbins, st);
    cudaMemsetAsync(fill, 0, sizeof(unsigned) * nbins, st);
    count_launch();
    k_bin_count<<<(n + 255) / 256, 256, 0, st>>>(key, n, count);
    exclusive_scan(count, start, nbins, scan_scratch, st);
    count_launch();
    k_bin_fill<<<(n + 255) / 256, 256, 0, st>>>(key, n, start, fill, items);
    count_launch();
    k_bin_sort<<<(nbins + 255) / 256, 256, 0, st>>>(start, nbins, items);
}

// ------------------------------------------------------------------ cell list
__global__ void k_cell_key(const float4* pos, int n, Box b, int3 nc, unsigned* key) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 p = pos[i];
    const float3 f = make_fraction(make_float3(p.x, p.y, p.z), b);
    int cx = (int)floorf(f.x * nc.x), cy = (int)floorf(f.y * nc.y), cz = (int)floorf(f.z * nc.z);
    cx = ((cx % nc.x) + nc.x) % nc.x;
    cy = ((cy % nc.y) + nc.y) % nc.y;
    cz = ((cz % nc.z) + nc.z) % nc.z;
    key[i] = (unsigned)((cx * nc.y + cy) * nc.z + cz);
}

__global__ void k_nlist_cells(const float4* __restrict__ pos, int n, Box b, int3 nc, const unsigned* __restrict__ key,
                              const unsigned* __restrict__ cstart, const unsigned* __restrict__ cparts, float rlist2,
                              unsigned* nneigh, unsigned* nlist, int stride, int* max_count) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 pi = pos[i];
    const unsigned c = key[i];
    const int cz = c % nc.z, cy = (c / nc.z) % nc.y, cx = c / (nc.z * nc.y);
    unsigned cnt = 0;
    unsigned* row = nlist + (size_t)i * stride;
    for (int dx = -1; dx <= 1; ++dx) {
        const int x = (cx + dx + nc.x) % nc.x;
        for (int dy = -1; dy <= 1; ++dy) {
            const int y = (cy + dy + nc.y) % nc.y;
            for (int dz = -1; dz <= 1; ++dz) {
                const int z = (cz + dz + nc.z) % nc.z;
                const unsigned cc = (unsigned)((x * nc.y + y) * nc.z + z);
                for (unsigned k = cstart[cc]; k < cstart[cc + 1]; ++k) {
                    const unsigned j = cparts[k];
                    if (j == (unsigned)i) continue;
                    const float4 pj = pos[j];
                    const float3 r = min_image_rn(make_float3(pi.x - pj.x, pi.y - pj.y, pi.z - pj.z), b);
                    if (dist2_rn(r) < rlist2) {
                        if (cnt < (unsigned)stride) row[cnt] = j;
                        ++cnt;
                    }
                }
            }
        }
    }
    nneigh[i] = cnt < (unsigned)stride ? cnt : (unsigned)stride;
    atomicMax(max_count, (int)cnt);
}

__global__ void k_nlist_allpairs(const float4* __restrict__ pos, int n, Box b, float rlist2, unsigned* nneigh,
                                 unsigned* nlist, int stride, int* max_count) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 pi = pos[i];
    unsigned cnt = 0;
    unsigned* row = nlist + (size_t)i * stride;
    for (int j = 0; j < n; ++j) {
        if (j == i) continue;
        const float4 pj = pos[j];
        const float3 r = min_image_rn(make_float3(pi.x - pj.x, pi.y - pj.y, pi.z - pj.z), b);
        if (dist2_rn(r) < rlist2) {
            if (cnt < (unsigned)stride) row[cnt] = j;
            ++cnt;
        }
    }
    nneigh[i] = cnt < (unsigned)stride ? cnt : (unsigned)stride;
    atomicMax(max_count, (int)cnt);
}

// Cells per axis so that a cell is at least r_list wide between faces.
int3 cell_dims(const Box& b, float rlist) {
    const float wx = b.Lx / sqrtf(1.0f + b.xy * b.xy);
    int3 nc;
    nc.x = (int)floorf(wx / rlist);
    nc.y = (int)floorf(b.Ly / rlist);
    nc.z = (int)floorf(b.Lz / rlist);
    return nc;
}

// Builds the list; returns the largest neighbour count in *max_count_host.
int build_neighbor_list(fsd_handle* h, const float4* pos, int* max_count_host) {
    Workspace& w = h->w;
    const int n = h->p.N;
    const float rlist = h->ewald_cut + h->p.nlist_buffer;
    const float rlist2 = rlist * rlist;
    const int3 nc = cell_dims(h->box, rlist);
    cudaStream_t st = h->stream;
    ProfRegion pr(h, R_NLIST);
    FSD_CHECK_CUDA(cudaMemsetAsync(w.nl_overflow, 0, sizeof(int), st));
    if (nc.x >= 3 && nc.y >= 3 && nc.z >= 3 && (size_t)nc.x * nc.y * nc.z <= w.ncell_cap) {
        const int ncells = nc.x * nc.y * nc.z;
        count_launch();
        k_cell_key<<<(n + 255) / 256, 256, 0, st>>>(pos, n, h->box, nc, w.part_cell);
        counting_sort(w.part_cell, n, ncells, w.cell_count, w.cell_start, w.cell_fill, w.cell_parts, w.scan_scratch, st);
        count_launch();
        k_nlist_cells<<<(n + 127) / 128, 128, 0, st>>>(pos, n, h->box, nc, w.part_cell, w.cell_start, w.cell_parts,
                                                       rlist2, w.nneigh, w.nlist, w.nl_stride, w.nl_overflow);
        FSD_CHECK_CUDA(cudaMemcpyAsync(w.order, w.cell_parts, sizeof(unsigned) * n, cudaMemcpyDeviceToDevice, st));
    } else {
        count_launch();
        k_nlist_allpairs<<<(n + 127) / 128, 128, 0, st>>>(pos, n, h->box, rlist2, w.nneigh, w.nlist, w.nl_stride,
                                                          w.nl_overflow);
    }
    FSD_CHECK_CUDA(cudaGetLastError());
    FSD_CHECK_CUDA(cudaMemcpyAsync(w.host_flag, w.nl_overflow, sizeof(int), cudaMemcpyDeviceToHost, st));
    FSD_CHECK_CUDA(cudaStreamSynchronize(st));
    *max_count_host = *w.host_flag;
    return FSD_OK;
}

__global__ void k_iota(unsigned* v, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) v[i] = (unsigned)i;
}

int init_particle_order(fsd_handle* h) {
    count_launch();
    k_iota<<<(h->p.N + 255) / 256, 256, 0, h->stream>>>(h->w.order, h->p.N);
    FSD_CHECK_CUDA(cudaGetLastError());
    return FSD_OK;
}

// Entries of each particle's neighbour list closer than sqrt(r2), in list
// order (so pair sums over them add in the same order as over the full list).
__global__ void k_sublist(const float4* __restrict__ pos, int n, Box b, const unsigned* __restrict__ nneigh,
                          const unsigned* __restrict__ nlist, int stride, float r2, unsigned* __restrict__ sub_n,
                          unsigned* __restrict__ sub) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 pi = pos[i];
    const unsigned* row = nlist + (size_t)i * stride;
    unsigned* out = sub + (size_t)i * stride;
    const unsigned nn = nneigh[i];
    unsigned k = 0;
    for (unsigned q = 0; q < nn; ++q) {
        const unsigned j = row[q];
        const float4 pj = pos[j];
        const float3 r = min_image(make_float3(pj.x - pi.x, pj.y - pi.y, pj.z - pi.z), b);
        if (r.x * r.x + r.y * r.y + r.z * r.z < r2) out[k++] = j;
    }
    sub_n[i] = k;
}

// The lubrication kernels' list: pairs within rlub plus the list buffer, so
// the sub-list stays complete for as long as the full list does.
int build_lub_list(fsd_handle* h, const float4* pos) {
    Workspace& w = h->w;
    const float r = h->p.rlub + h->p.nlist_buffer;
    count_launch();
    k_sublist<<<(h->p.N + 127) / 128, 128, 0, h->stream>>>(pos, h->p.N, h->box, w.nneigh, w.nlist, w.nl_stride,
                                                           r * r, w.lub_n, w.lub_list);
    FSD_CHECK_CUDA(cudaGetLastError());
    return FSD_OK;
}

// ------------------------------------------- allocation-free neighbour list
// Scratch of fsd_neighbor_list_noalloc: the cell key and cell members of every
// particle and the counting-sort arrays of every cell, in one file-scope
// device array (about 1.25 MiB, held on each device that loads the library
// until the process exits).  All calls on a device share it.
namespace {
constexpr int kNoAllocMaxN = FSD_NOALLOC_MAX_N;
constexpr int kNoAllocMaxCells = FSD_NOALLOC_MAX_CELLS;
constexpr size_t kNoAllocScan = (size_t)(kNoAllocMaxCells + kScanTile - 1) / kScanTile + 1;
constexpr size_t kOffKey = 0;
constexpr size_t kOffParts = kOffKey + kNoAllocMaxN;
constexpr size_t kOffCount = kOffParts + kNoAllocMaxN;
constexpr size_t kOffStart = kOffCount + kNoAllocMaxCells;
constexpr size_t kOffFill = kOffStart + kNoAllocMaxCells + 1;
constexpr size_t kOffScan = kOffFill + kNoAllocMaxCells;
constexpr size_t kNoAllocElems = kOffScan + kNoAllocScan;

static __device__ __align__(256) unsigned g_nlist_scratch[kNoAllocElems];

// Device address of g_nlist_scratch on the current device, looked up once per
// device.  In host code the array's name is only a host-side stand-in, so the
// kernels are always given this address instead.
constexpr int kMaxDevices = 64;
std::mutex g_scratch_mu;
unsigned* g_scratch_addr[kMaxDevices] = {};

int noalloc_scratch(unsigned** out) {
    int dev = -1;
    FSD_CHECK_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) return FSD_ERR_BAD_PARAMS;
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    if (!g_scratch_addr[dev]) {
        void* p = nullptr;
        FSD_CHECK_CUDA(cudaGetSymbolAddress(&p, g_nlist_scratch));
        g_scratch_addr[dev] = (unsigned*)p;
    }
    *out = g_scratch_addr[dev];
    return FSD_OK;
}
}  // namespace

int neighbor_list_noalloc(const float4* pos, int n, Box b, float rlist, unsigned* nneigh, unsigned* nlist,
                          int stride, int* max_count, cudaStream_t st) {
    unsigned* scratch = nullptr;
    const int e = noalloc_scratch(&scratch);
    if (e != FSD_OK) return e;
    const float rlist2 = rlist * rlist;
    // Cells per axis, clamped to the scratch's cell capacity before the
    // conversion to int (a large box over a small r_list would overflow it).
    const float wx = b.Lx / sqrtf(1.0f + b.xy * b.xy);
    auto axis_cells = [](float len, float r) {
        return (int)fminf(floorf(len / r), (float)kNoAllocMaxCells);
    };
    int3 nc = make_int3(axis_cells(wx, rlist), axis_cells(b.Ly, rlist), axis_cells(b.Lz, rlist));
    // Wider cells than r_list stay correct, so a box with more cells than the
    // scratch holds uses fewer, wider cells along its longest cell axis.
    while ((size_t)nc.x * nc.y * nc.z > (size_t)kNoAllocMaxCells) {
        if (nc.x >= nc.y && nc.x >= nc.z) --nc.x;
        else if (nc.y >= nc.z) --nc.y;
        else --nc.z;
    }
    FSD_CHECK_CUDA(cudaMemsetAsync(max_count, 0, sizeof(int), st));
    if (nc.x >= 3 && nc.y >= 3 && nc.z >= 3) {
        const int ncells = nc.x * nc.y * nc.z;
        unsigned* key = scratch + kOffKey;
        unsigned* parts = scratch + kOffParts;
        unsigned* start = scratch + kOffStart;
        count_launch();
        k_cell_key<<<(n + 255) / 256, 256, 0, st>>>(pos, n, b, nc, key);
        // counting_sort clears the per-cell counters it accumulates into.
        counting_sort(key, n, ncells, scratch + kOffCount, start, scratch + kOffFill, parts, scratch + kOffScan, st);
        count_launch();
        k_nlist_cells<<<(n + 127) / 128, 128, 0, st>>>(pos, n, b, nc, key, start, parts, rlist2, nneigh, nlist,
                                                       stride, max_count);
    } else {
        count_launch();
        k_nlist_allpairs<<<(n + 127) / 128, 128, 0, st>>>(pos, n, b, rlist2, nneigh, nlist, stride, max_count);
    }
    FSD_CHECK_CUDA(cudaGetLastError());
    return FSD_OK;
}

}  // namespace fsd

extern "C" int fsd_neighbor_list_noalloc(const float* d_pos, int N, float Lx, float Ly, float Lz, float xy,
                                         float rlist, unsigned int* d_nneigh, unsigned int* d_nlist, int stride,
                                         int* d_max_count, void* cuda_stream) {
    if (!d_pos || !d_nneigh || !d_nlist || !d_max_count) return FSD_ERR_BAD_PARAMS;
    if (N < 1 || N > FSD_NOALLOC_MAX_N || stride < 1) return FSD_ERR_BAD_PARAMS;
    if (!(rlist > 0.f) || !(Lx > 0.f) || !(Ly > 0.f) || !(Lz > 0.f) || !std::isfinite(rlist) ||
        !std::isfinite(Lx) || !std::isfinite(Ly) || !std::isfinite(Lz) || !std::isfinite(xy))
        return FSD_ERR_BAD_PARAMS;
    return fsd::neighbor_list_noalloc((const float4*)d_pos, N, fsd::Box{Lx, Ly, Lz, xy}, rlist, d_nneigh, d_nlist,
                                      stride, d_max_count, (cudaStream_t)cuda_stream);
}

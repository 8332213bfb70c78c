// edm_static.cu — cell list of caller-provided positions without any device
// allocation.
//
// Who needs this: callers that must not allocate device memory on the fly —
// code running inside a pre-sized memory pool or arena (a host framework
// that owns every allocation on the device), a process that has handed the
// whole device memory to another allocator, or a latency-critical loop where
// a cudaMalloc (which can synchronise the device) is not acceptable.  They
// pass their own positions and output buffers; the scratch this routine
// needs (per-cell counters, fill cursors, scan block sums) lives in one
// file-scope __device__ array that every GPU loading the library holds
// until the process exits.
//
// The array's host-side name is only a stand-in: host code gets the device
// address once per device with cudaGetSymbolAddress (the first call on a
// device does that set-up, so make the first call before any stream
// capture), and passes it to the kernels.  All calls share the one array:
// calls that overlap on the GPU (different streams, or different threads
// without ordering) race on it.  Each call clears what must start at zero.
#include <algorithm>
#include <cstdint>
#include <mutex>
#include <string>

#include <cuda_runtime.h>

#include "../../include/edm_b200.h"
#include "edm_error.h"

namespace {

constexpr int kThreads = 256;
constexpr int kScanThreads = 512;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;
constexpr int64_t kMaxBlocks = (EDM_STATIC_MAX_CELLS + kScanTile - 1) / kScanTile;

// [0, MAX)          per-cell counts
// [MAX, 2*MAX)      per-cell fill cursors
// [2*MAX, +blocks)  scan block sums
__device__ __align__(256) int32_t g_edm_static_scratch[2 * EDM_STATIC_MAX_CELLS + kMaxBlocks + 64];

std::mutex g_mu;
int32_t* g_scratch_ptr[64] = {nullptr};
int fail(int code, const std::string& m) { return edm::report_error(code, m); }

__device__ __forceinline__ int clampi(int v, int n) {
  v = v >= n ? n - 1 : v;
  return v < 0 ? 0 : v;
}

__device__ __forceinline__ int cell_of(const double* pos, int64_t i, double csx, double csy, int nx, int ny) {
  const int cx = clampi((int)__ddiv_rn(pos[2 * i], csx), nx);
  const int cy = clampi((int)__ddiv_rn(pos[2 * i + 1], csy), ny);
  return cx * ny + cy;
}

__global__ void k_zero(int32_t* a, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) a[i] = 0;
}

__global__ void k_count(const double* pos, int64_t n, double csx, double csy, int nx, int ny, int32_t* cnt) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) atomicAdd(&cnt[cell_of(pos, i, csx, csy, nx, ny)], 1);
}

__device__ __forceinline__ int block_scan(int v, int& total) {
  __shared__ int ws[32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  int x = v;
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) ws[wid] = x;
  __syncthreads();
  if (wid == 0) {
    const int nw = blockDim.x >> 5;
    int w = lane < nw ? ws[lane] : 0;
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += y;
    }
    if (lane < nw) ws[lane] = w;
  }
  __syncthreads();
  const int base = wid > 0 ? ws[wid - 1] : 0;
  total = ws[(blockDim.x >> 5) - 1];
  __syncthreads();
  return base + x - v;
}

__global__ void k_reduce(const int32_t* cnt, int64_t n, int32_t* bsum) {
  const int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanItems;
  int v = 0;
  for (int i = 0; i < kScanItems; ++i)
    if (base + i < n) v += cnt[base + i];
  int total;
  block_scan(v, total);
  if (threadIdx.x == 0) bsum[blockIdx.x] = total;
}

__global__ void k_bsum(int32_t* bsum, int nb, int32_t* big_count) {
  if (threadIdx.x == 0) *big_count = 0;
  int carry = 0;
  for (int off = 0; off < nb; off += blockDim.x) {
    const int i = off + threadIdx.x;
    const int v = i < nb ? bsum[i] : 0;
    int total;
    const int ex = block_scan(v, total);
    if (i < nb) bsum[i] = carry + ex;
    carry += total;
  }
}

__global__ void k_down(const int32_t* cnt, int64_t n, const int32_t* bsum, int32_t* start, int32_t* cursor) {
  const int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanItems;
  int vals[kScanItems];
  int v = 0;
  for (int i = 0; i < kScanItems; ++i) {
    vals[i] = base + i < n ? cnt[base + i] : 0;
    v += vals[i];
  }
  int total;
  int run = block_scan(v, total) + bsum[blockIdx.x];
  for (int i = 0; i < kScanItems; ++i) {
    if (base + i < n) {
      start[base + i] = run;
      cursor[base + i] = run;
    }
    run += vals[i];
  }
  if (base < n && base + kScanItems >= n) start[n] = run;
}

__global__ void k_fill(const double* pos, int64_t n, double csx, double csy, int nx, int ny, int32_t* cursor,
                       int32_t* members) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) members[atomicAdd(&cursor[cell_of(pos, i, csx, csy, nx, ny)], 1)] = (int32_t)i;
}

// Members of each cell in ascending particle index (deterministic output).
// The fill above leaves each cell's members in atomic order; every class of
// cell is then put in order with bounded work:
//  - up to kSmallCell members: one thread, insertion sort (<= 496 moves);
//  - up to kMidCell: one block, each member's rank counted in shared memory
//    (O(m^2 / kBigThreads) per thread);
//  - larger: one block scans particle indices 0..n-1 in order and writes the
//    cell's members as it meets them (O(n) per such cell; at most
//    n / kMidCell of them, and n <= EDM_STATIC_MAX_PARTICLES).
constexpr int kSmallCell = 32;
constexpr int kMidCell = 8192;
constexpr int kBigThreads = 512;

__global__ void k_sort_small(const int32_t* start, int64_t n_cells, int32_t* members, int32_t* big_list,
                             int32_t* big_count) {
  const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n_cells) return;
  const int a = start[c], b = start[c + 1];
  if (b - a > kSmallCell) {
    big_list[atomicAdd(big_count, 1)] = (int32_t)c;
    return;
  }
  for (int i = a + 1; i < b; ++i) {
    const int32_t v = members[i];
    int j = i - 1;
    while (j >= a && members[j] > v) {
      members[j + 1] = members[j];
      --j;
    }
    members[j + 1] = v;
  }
}

__global__ void __launch_bounds__(kBigThreads) k_sort_large(const double* pos, int64_t n, double csx, double csy,
                                                            int nx, int ny, const int32_t* start, int32_t* members,
                                                            const int32_t* big_list, const int32_t* big_count) {
  __shared__ int32_t buf[kMidCell];
  __shared__ int32_t warp_tot[kBigThreads / 32];
  const int nbig = *big_count;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int k = blockIdx.x; k < nbig; k += gridDim.x) {
    const int c = big_list[k];
    const int a = start[c], m = start[c + 1] - a;
    if (m <= kMidCell) {
      for (int i = threadIdx.x; i < m; i += kBigThreads) buf[i] = members[a + i];
      __syncthreads();
      for (int i = threadIdx.x; i < m; i += kBigThreads) {
        const int32_t v = buf[i];
        int rank = 0;
        for (int q = 0; q < m; ++q) rank += buf[q] < v ? 1 : 0;  // indices are distinct
        members[a + rank] = v;
      }
      __syncthreads();
    } else {
      int run = 0;
      for (int64_t base = 0; base < n; base += kBigThreads) {
        const int64_t i = base + threadIdx.x;
        const bool hit = i < n && cell_of(pos, i, csx, csy, nx, ny) == c;
        const unsigned bits = __ballot_sync(0xffffffffu, hit);
        if (lane == 0) warp_tot[wid] = __popc(bits);
        __syncthreads();
        int before = 0, total = 0;
        for (int w = 0; w < kBigThreads / 32; ++w) {
          const int t = warp_tot[w];
          before += w < wid ? t : 0;
          total += t;
        }
        if (hit) members[a + run + before + __popc(bits & ((1u << lane) - 1u))] = (int32_t)i;
        run += total;
        __syncthreads();
      }
    }
  }
}

int scratch_for_current_device(int32_t** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fail(EDM_ECUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
  if (dev < 0 || dev >= 64) return fail(EDM_EINVAL, "device index out of range");
  std::lock_guard<std::mutex> lock(g_mu);
  if (!g_scratch_ptr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_edm_static_scratch);
    if (e != cudaSuccess) return fail(EDM_ECUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    g_scratch_ptr[dev] = (int32_t*)p;
  }
  *out = g_scratch_ptr[dev];
  return EDM_OK;
}

}  // namespace

extern "C" int edm_cell_list_static(const double* positions_dev, int64_t n, double Lx, double Ly, int32_t nx,
                                    int32_t ny, int32_t* cell_start_dev, int32_t* members_dev, void* stream) {
  if (n < 0 || nx < 1 || ny < 1 || !(Lx > 0.0) || !(Ly > 0.0))
    return fail(EDM_EINVAL, "edm_cell_list_static: bad size or box");
  if (n > EDM_STATIC_MAX_PARTICLES)
    return fail(EDM_EINVAL, "edm_cell_list_static: n exceeds EDM_STATIC_MAX_PARTICLES (" +
                                std::to_string((long long)EDM_STATIC_MAX_PARTICLES) + ")");
  const int64_t n_cells = (int64_t)nx * (int64_t)ny;
  if (n_cells > EDM_STATIC_MAX_CELLS)
    return fail(EDM_EINVAL, "edm_cell_list_static: nx*ny exceeds EDM_STATIC_MAX_CELLS (" +
                                std::to_string((long long)EDM_STATIC_MAX_CELLS) + ")");
  if (!cell_start_dev || (n > 0 && (!positions_dev || !members_dev)))
    return fail(EDM_EINVAL, "edm_cell_list_static: null buffer");
  int32_t* scratch = nullptr;
  int rc = scratch_for_current_device(&scratch);
  if (rc != EDM_OK) return rc;
  // [0, MAX): per-cell counts, then (once the scan has read them) the list of
  // cells with more than kSmallCell members; [MAX, 2 MAX): fill cursors;
  // then the scan block sums and the list's length
  int32_t* cnt = scratch;
  int32_t* big_list = scratch;
  int32_t* cursor = scratch + EDM_STATIC_MAX_CELLS;
  int32_t* bsum = scratch + 2 * EDM_STATIC_MAX_CELLS;
  int32_t* big_count = bsum + kMaxBlocks;
  cudaStream_t s = (cudaStream_t)stream;
  const double csx = Lx / nx, csy = Ly / ny;  // cell side = box side / cells
  const int nb = (int)((n_cells + kScanTile - 1) / kScanTile);
  cudaGetLastError();  // a launch error left by earlier, unrelated work is not this call's
  auto check = [&](const char* kernel) -> int {
    const cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) return EDM_OK;
    return fail(EDM_ECUDA, std::string("edm_cell_list_static: launch of ") + kernel + ": " + cudaGetErrorString(e));
  };
  k_zero<<<(unsigned)std::min<int64_t>((n_cells + kThreads - 1) / kThreads, 4096), kThreads, 0, s>>>(cnt, n_cells);
  if ((rc = check("k_zero")) != EDM_OK) return rc;
  if (n > 0) {
    k_count<<<(unsigned)((n + kThreads - 1) / kThreads), kThreads, 0, s>>>(positions_dev, n, csx, csy, nx, ny, cnt);
    if ((rc = check("k_count")) != EDM_OK) return rc;
  }
  k_reduce<<<nb, kScanThreads, 0, s>>>(cnt, n_cells, bsum);
  if ((rc = check("k_reduce")) != EDM_OK) return rc;
  k_bsum<<<1, 1024, 0, s>>>(bsum, nb, big_count);
  if ((rc = check("k_bsum")) != EDM_OK) return rc;
  k_down<<<nb, kScanThreads, 0, s>>>(cnt, n_cells, bsum, cell_start_dev, cursor);
  if ((rc = check("k_down")) != EDM_OK) return rc;
  if (n > 0) {
    k_fill<<<(unsigned)((n + kThreads - 1) / kThreads), kThreads, 0, s>>>(positions_dev, n, csx, csy, nx, ny, cursor,
                                                                        members_dev);
    if ((rc = check("k_fill")) != EDM_OK) return rc;
    k_sort_small<<<(unsigned)((n_cells + kThreads - 1) / kThreads), kThreads, 0, s>>>(cell_start_dev, n_cells,
                                                                                    members_dev, big_list, big_count);
    if ((rc = check("k_sort_small")) != EDM_OK) return rc;
    k_sort_large<<<296, kBigThreads, 0, s>>>(positions_dev, n, csx, csy, nx, ny, cell_start_dev, members_dev, big_list,
                                             big_count);
    if ((rc = check("k_sort_large")) != EDM_OK) return rc;
  }
  return EDM_OK;
}

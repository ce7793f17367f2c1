// agimp_refine_levels_noalloc: the free-surface refinement rule of refine.cu
// for callers that cannot allocate device memory.
//
// Who needs it: a host that gives the whole device memory budget to its own
// arena or pool allocator at start-up (a game or visual-effects engine, or a
// framework that reserves all of HBM) cannot let a library call cudaMalloc:
// the call fails once the pool has the memory, or bypasses the host's
// accounting; a real-time loop may also not accept the device-wide
// synchronisation that cudaMalloc/cudaFree can imply.  Such a caller owns its
// particle positions and the output levels, but not a simulator handle (whose
// agimp_create allocates), so this entry point takes no handle.
//
// Its scratch (the depth of every finest cell plus the particles' bounding
// box) lives in the file-scope array below, which every GPU that loads the
// library holds until the process exits.  All calls share it: they must not
// overlap on the GPU (calls on different streams, or from different host
// threads without ordering, race on it).  Each call resets what it reads.
#include <climits>
#include <mutex>

#include "../../include/agimp.h"
#include "common.cuh"

namespace agimp {
namespace {

// 16 MiB of cell depths: finest^dim <= 16,777,216 (3D up to 256^3, 2D up to 4096^2)
constexpr long long NOALLOC_MAX_CELLS = 16ll << 20;
constexpr int NOALLOC_HEADER = 256;  // bounding box: int lo[3], hi[3]
// longest line of a distance-transform pass: the finest size (2D at most
// 4096, 3D at most 256 under the cell limit)
constexpr int NOALLOC_MAX_LINE = 4096;
static __device__ __align__(256) uint8_t g_noalloc_scratch[NOALLOC_HEADER + NOALLOC_MAX_CELLS];

constexpr int NOALLOC_MAX_DEVICES = 64;
uint8_t* g_scratch_ptr[NOALLOC_MAX_DEVICES] = {};
std::mutex g_scratch_mu;

struct NA {
  const float* x;  // [n][dim] (the C ABI's particle layout)
  long long n;
  int dim, L, sz, band;
  int32_t* g;
  int* bb;         // scratch header
  uint8_t* depth;  // scratch cells, finest^dim
};

#define GS_LOOP(i, n) \
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < (n); i += (long long)gridDim.x * blockDim.x)

__global__ void k_na_bb_init(NA a) {
  if (threadIdx.x < 3) {
    a.bb[threadIdx.x] = INT_MAX;
    a.bb[3 + threadIdx.x] = -1;
  }
}

template <int D>
__device__ __forceinline__ bool na_cell(const NA& a, long long p, int* cell) {
  bool ok = true;
#pragma unroll
  for (int d = 0; d < D; ++d) {
    const float x = a.x[p * D + d];
    if (!(x >= 0.f && x < 1.f)) ok = false;
    cell[d] = ok ? (int)floorf(x * (float)a.sz) : 0;
  }
  return ok;
}

template <int D>
__device__ __forceinline__ long long na_vol(const NA& a, int* lo, int* n) {
  long long v = 1;
#pragma unroll
  for (int d = 0; d < D; ++d) {
    lo[d] = a.bb[d];
    n[d] = a.bb[3 + d] - lo[d] + 1;
    if (n[d] <= 0) return 0;
    v *= n[d];
  }
  return v;
}

template <int D>
__device__ __forceinline__ long long na_idx(const NA& a, const int* cell) {
  long long o = 0;
#pragma unroll
  for (int d = 0; d < D; ++d) o = o * a.sz + cell[d];
  return o;
}

// bounding box of the particles' finest cells: a fixed grid of CTAs, each
// reducing its share of the particles across its warps in shared memory, then
// one atomic per CTA and bound
template <int D>
__global__ void __launch_bounds__(256) k_na_bb(NA a) {
  __shared__ int s_lo[8][D], s_hi[8][D];
  int lo[D], hi[D];
#pragma unroll
  for (int d = 0; d < D; ++d) {
    lo[d] = INT_MAX;
    hi[d] = -1;
  }
  GS_LOOP(p, a.n) {
    int cell[D];
    if (na_cell<D>(a, p, cell))
#pragma unroll
      for (int d = 0; d < D; ++d) {
        lo[d] = min(lo[d], cell[d]);
        hi[d] = max(hi[d], cell[d]);
      }
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int d = 0; d < D; ++d) {
#pragma unroll
    for (int o = 16; o; o >>= 1) {
      lo[d] = min(lo[d], __shfl_xor_sync(0xffffffffu, lo[d], o));
      hi[d] = max(hi[d], __shfl_xor_sync(0xffffffffu, hi[d], o));
    }
    if (lane == 0) {
      s_lo[warp][d] = lo[d];
      s_hi[warp][d] = hi[d];
    }
  }
  __syncthreads();
  if (threadIdx.x < D) {
    const int d = threadIdx.x;
    int mn = INT_MAX, mx = -1;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
      mn = min(mn, s_lo[w][d]);
      mx = max(mx, s_hi[w][d]);
    }
    if (mx >= 0) {
      atomicMin(&a.bb[d], mn);
      atomicMax(&a.bb[3 + d], mx);
    }
  }
}

template <int D>
__global__ void k_na_clear(NA a) {
  int lo[D], n[D];
  const long long vol = na_vol<D>(a, lo, n);
  GS_LOOP(i, vol) {
    long long t = i;
    int cell[D];
#pragma unroll
    for (int d = D - 1; d >= 0; --d) {
      cell[d] = lo[d] + (int)(t % n[d]);
      t /= n[d];
    }
    a.depth[na_idx<D>(a, cell)] = 0;
  }
}

template <int D>
__global__ void k_na_mark(NA a) {
  const long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  int cell[D];
  if (p < a.n && na_cell<D>(a, p, cell)) a.depth[na_idx<D>(a, cell)] = 1;
}

// One pass of the separable distance transform of refine.cu along `axis`,
// in place: a CTA takes one line of the bounding box at a time and reads it
// into shared memory before writing it back, so the pass needs no second
// buffer (lines are at most NOALLOC_MAX_LINE cells long).  With f_0 = 0 on
// empty and K on occupied cells (the first pass reads occupancy 0 / 1),
//   f_a(c) = min over x' on the line of c of max(f_{a-1}(c|x'), |x - x'|),
// positions outside the box counting as empty, so after the last axis every
// cell holds min(K, its Chebyshev distance to the nearest empty cell).
template <int D>
__global__ void __launch_bounds__(256) k_na_dt_line(NA a, int axis, int K, int first) {
  __shared__ uint8_t line[NOALLOC_MAX_LINE];
  int lo[D], n[D];
  const long long vol = na_vol<D>(a, lo, n);
  if (vol == 0) return;
  const int nx = n[axis];
  const long long nlines = vol / nx;
  long long stride = 1;
  for (int d = D - 1; d > axis; --d) stride *= a.sz;
  for (long long li = blockIdx.x; li < nlines; li += gridDim.x) {
    // the line's first cell: li runs over the other axes' box coordinates
    int cell[D];
    long long t = li;
#pragma unroll
    for (int d = D - 1; d >= 0; --d) {
      if (d == axis) {
        cell[d] = lo[d];
        continue;
      }
      cell[d] = lo[d] + (int)(t % n[d]);
      t /= n[d];
    }
    uint8_t* base = a.depth + na_idx<D>(a, cell);
    for (int x = threadIdx.x; x < nx; x += blockDim.x) {
      const int v = base[x * stride];
      line[x] = (uint8_t)(first ? (v ? K : 0) : v);
    }
    __syncthreads();
    for (int x = threadIdx.x; x < nx; x += blockDim.x) {
      auto val = [&](int q) -> int { return (q < 0 || q >= nx) ? 0 : line[q]; };
      int best = val(x);
      for (int o = 1; o < best; ++o) best = min(best, max(min(val(x - o), val(x + o)), o));
      base[x * stride] = (uint8_t)best;
    }
    __syncthreads();
  }
}

template <int D>
__global__ void k_na_assign(NA a) {
  const long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  int cell[D];
  if (p >= a.n || !na_cell<D>(a, p, cell)) return;
  const int dd = a.depth[na_idx<D>(a, cell)];
  int lv = 0;
  for (int k = 0; k < a.L - 1; ++k) {
    if (dd <= a.band * ((1 << (k + 1)) - 1)) {
      lv = a.L - 1 - k;
      break;
    }
  }
  a.g[p] = lv;
}

template <int D>
void na_launch(const NA& a, int sms, cudaStream_t s) {
  const int Gp = (int)((a.n + 255) / 256);
  const int G = sms * 8;
  // the largest depth the rule compares is band (2^(L-1) - 1); the entry
  // point keeps it below 250, so K fits the uint8 cells
  const int K = a.band * ((1 << (a.L - 1)) - 1) + 1;
  k_na_bb_init<<<1, 32, 0, s>>>(a);
  k_na_bb<D><<<sms * 2, 256, 0, s>>>(a);  // 256 threads: 8 warps (s_lo / s_hi)
  k_na_clear<D><<<G, 256, 0, s>>>(a);
  k_na_mark<D><<<Gp, 256, 0, s>>>(a);
  for (int k = 0; k < D; ++k) k_na_dt_line<D><<<G, 256, 0, s>>>(a, D - 1 - k, K, k == 0);
  k_na_assign<D><<<Gp, 256, 0, s>>>(a);
}

}  // namespace
}  // namespace agimp

extern "C" agimp_status agimp_refine_levels_noalloc(const float* x, int64_t n, int32_t dim, int32_t level,
                                                    int32_t coarsest_size, int32_t band, int32_t* g, void* stream) {
  using namespace agimp;
  if ((dim != 2 && dim != 3) || level < 1 || level > MAXL || coarsest_size < 4 ||
      (coarsest_size & (coarsest_size - 1)) || band < 1 || band > 32 || n < 0 || (n > 0 && (!x || !g)))
    return AGIMP_INVALID_ARG;
  // depths are kept in bytes: the deepest threshold must stay below 250
  if ((long long)band * ((1ll << (level - 1)) - 1) >= 250) return AGIMP_INVALID_ARG;
  const long long sz = (long long)coarsest_size << (level - 1);
  long long cells = 1;
  for (int d = 0; d < dim; ++d) {
    cells *= sz;
    if (cells > NOALLOC_MAX_CELLS) return AGIMP_CAPACITY;  // finest^dim beyond the static scratch
  }
  if (n == 0) return AGIMP_OK;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= NOALLOC_MAX_DEVICES) return AGIMP_CUDA_ERROR;
  uint8_t* base = nullptr;
  {
    // First call on a device: look up the scratch array's device address with
    // that device current.  The host-side symbol is only a stand-in and must
    // never be passed to a kernel.
    std::lock_guard<std::mutex> lk(g_scratch_mu);
    if (!g_scratch_ptr[dev]) {
      void* p = nullptr;
      if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return AGIMP_CUDA_ERROR;
      g_scratch_ptr[dev] = (uint8_t*)p;
    }
    base = g_scratch_ptr[dev];
  }
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  NA a;
  a.x = x;
  a.n = n;
  a.dim = dim;
  a.L = level;
  a.sz = (int)sz;
  a.band = band;
  a.g = g;
  a.bb = (int*)base;
  a.depth = base + NOALLOC_HEADER;
  cudaStream_t s = (cudaStream_t)stream;
  if (dim == 2)
    na_launch<2>(a, sms, s);
  else
    na_launch<3>(a, sms, s);
  return cudaGetLastError() == cudaSuccess ? AGIMP_OK : AGIMP_CUDA_ERROR;
}

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

template <int D>
__global__ void k_na_bb(NA a) {
  const long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  int cell[D];
  const bool ok = p < a.n && na_cell<D>(a, p, cell);
#pragma unroll
  for (int d = 0; d < D; ++d) {
    int lo = ok ? cell[d] : INT_MAX, hi = ok ? cell[d] : -1;
#pragma unroll
    for (int o = 16; o; o >>= 1) {
      lo = min(lo, __shfl_xor_sync(0xffffffffu, lo, o));
      hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, o));
    }
    if ((threadIdx.x & 31) == 0 && hi >= 0) {
      atomicMin(&a.bb[d], lo);
      atomicMax(&a.bb[3 + d], hi);
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

template <int D>
__global__ void k_na_erode(NA a, int k) {
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
    uint8_t* me = &a.depth[na_idx<D>(a, cell)];
    if (*me != k) continue;
    bool all = true;
#pragma unroll
    for (int q = 0; q < ((D == 2) ? 9 : 27); ++q) {
      int c[D];
      int tt = q;
      bool in = true;
#pragma unroll
      for (int d = D - 1; d >= 0; --d) {
        c[d] = cell[d] + tt % 3 - 1;
        tt /= 3;
        in = in && c[d] >= lo[d] && c[d] < lo[d] + n[d];
      }
      if (!in || a.depth[na_idx<D>(a, c)] < k) all = false;
    }
    if (all) *me = (uint8_t)(k + 1);
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
  int kmax = a.band * ((1 << (a.L - 1)) - 1) + 1;
  if (kmax > 250) kmax = 250;
  k_na_bb_init<<<1, 32, 0, s>>>(a);
  k_na_bb<D><<<Gp, 256, 0, s>>>(a);
  k_na_clear<D><<<G, 256, 0, s>>>(a);
  k_na_mark<D><<<Gp, 256, 0, s>>>(a);
  for (int k = 1; k < kmax; ++k) k_na_erode<D><<<G, 256, 0, s>>>(a, k);
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

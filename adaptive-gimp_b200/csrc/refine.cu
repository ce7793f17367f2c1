// Free-surface refinement rule (extension; the reference fixes g_p once at
// initialisation, init.py:17-29 and run_3d.py:151-156).
//
// depth(c) = Chebyshev distance in finest cells from occupied finest cell c to
// the nearest empty one (cells outside the domain are empty), found by
// iterated 3^d erosion over the bounding box of the particles.  A particle's
// prescribed level is L-1 when depth <= band, L-2 when depth <= 3*band, L-3
// when depth <= 7*band, ..., and 0 deeper inside.
#include <climits>

#include "common.cuh"

namespace agimp {

enum { CTR_BB = 16 };  // ctr[16..18] = bbox lo, ctr[19..21] = bbox hi (finest cells)

#define GS_LOOP(i, n) \
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < (n); i += (long long)gridDim.x * blockDim.x)

__global__ void k_bb_init(Ctx c) {
  if (threadIdx.x < 3) {
    c.ctr[CTR_BB + threadIdx.x] = INT_MAX;
    c.ctr[CTR_BB + 3 + threadIdx.x] = -1;
  }
}

template <int D>
__device__ __forceinline__ bool particle_cell(const Ctx& c, int p, int* cell) {
  bool ok = true;
#pragma unroll
  for (int d = 0; d < D; ++d) {
    const float x = c.P.x[(long long)d * c.N + p];
    if (!(x >= 0.f && x < 1.f)) ok = false;
    cell[d] = ok ? (int)floorf(x * (float)c.sz) : 0;
  }
  return ok;
}

template <int D>
__global__ void k_bb(Ctx c) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  int cell[D];
  const bool ok = p < c.N && particle_cell<D>(c, p, cell);
#pragma unroll
  for (int d = 0; d < D; ++d) {
    int lo = ok ? cell[d] : INT_MAX, hi = ok ? cell[d] : -1;
#pragma unroll
    for (int o = 16; o; o >>= 1) {
      lo = min(lo, __shfl_xor_sync(0xffffffffu, lo, o));
      hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, o));
    }
    if ((threadIdx.x & 31) == 0 && hi >= 0) {
      atomicMin(&c.ctr[CTR_BB + d], lo);
      atomicMax(&c.ctr[CTR_BB + 3 + d], hi);
    }
  }
}

template <int D>
__device__ __forceinline__ long long bb_volume(const Ctx& c, int* lo, int* n) {
  long long v = 1;
#pragma unroll
  for (int d = 0; d < D; ++d) {
    lo[d] = c.ctr[CTR_BB + d];
    n[d] = c.ctr[CTR_BB + 3 + d] - lo[d] + 1;
    if (n[d] <= 0) return 0;
    v *= n[d];
  }
  return v;
}

template <int D>
__device__ __forceinline__ long long occ_index(const Ctx& c, const int* cell) {
  long long o = 0;
#pragma unroll
  for (int d = 0; d < D; ++d) o = o * c.sz + cell[d];
  return o;
}

template <int D>
__global__ void k_occ_clear(Ctx c) {
  int lo[D], n[D];
  const long long vol = bb_volume<D>(c, lo, n);
  GS_LOOP(i, vol) {
    long long t = i;
    int cell[D];
#pragma unroll
    for (int d = D - 1; d >= 0; --d) {
      cell[d] = lo[d] + (int)(t % n[d]);
      t /= n[d];
    }
    c.occ[occ_index<D>(c, cell)] = 0;
  }
}

template <int D>
__global__ void k_occ_mark(Ctx c) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  int cell[D];
  if (p < c.N && particle_cell<D>(c, p, cell)) c.occ[occ_index<D>(c, cell)] = 1;
}

template <int D>
__global__ void k_erode(Ctx c, int k) {
  int lo[D], n[D];
  const long long vol = bb_volume<D>(c, lo, n);
  GS_LOOP(i, vol) {
    long long t = i;
    int cell[D];
#pragma unroll
    for (int d = D - 1; d >= 0; --d) {
      cell[d] = lo[d] + (int)(t % n[d]);
      t /= n[d];
    }
    uint8_t* me = &c.occ[occ_index<D>(c, cell)];
    if (*me != k) continue;
    bool all = true;
#pragma unroll
    for (int a = 0; a < ((D == 2) ? 9 : 27); ++a) {
      int q[D];
      int tt = a;
      bool in = true;
#pragma unroll
      for (int d = D - 1; d >= 0; --d) {
        q[d] = cell[d] + tt % 3 - 1;
        tt /= 3;
        in = in && q[d] >= lo[d] && q[d] < lo[d] + n[d];
      }
      // cells outside the particles' bounding box are empty
      if (!in || c.occ[occ_index<D>(c, q)] < k) all = false;
    }
    if (all) *me = (uint8_t)(k + 1);
  }
}

template <int D>
__global__ void k_assign(Ctx c, int band) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  int cell[D];
  if (p >= c.N || !particle_cell<D>(c, p, cell)) return;
  const int dd = c.occ[occ_index<D>(c, cell)];
  int lv = 0;
  for (int k = 0; k < c.L - 1; ++k) {
    if (dd <= band * ((1 << (k + 1)) - 1)) {
      lv = c.L - 1 - k;
      break;
    }
  }
  c.P.g[p] = lv;
}

template <int D>
static void run_refine(const Ctx& c, int band, cudaStream_t s) {
  if (c.N == 0) return;
  const int Gp = (c.N + 255) / 256;
  const int G = c.sms * 8;
  int kmax = band * ((1 << (c.L - 1)) - 1) + 1;
  if (kmax > 250) kmax = 250;
  k_bb_init<<<1, 32, 0, s>>>(c);
  k_bb<D><<<Gp, 256, 0, s>>>(c);
  k_occ_clear<D><<<G, 256, 0, s>>>(c);
  k_occ_mark<D><<<Gp, 256, 0, s>>>(c);
  for (int k = 1; k < kmax; ++k) k_erode<D><<<G, 256, 0, s>>>(c, k);
  k_assign<D><<<Gp, 256, 0, s>>>(c, band);
}

void launch_refine(const Ctx& c, int band, cudaStream_t s) {
  if (c.dim == 2)
    run_refine<2>(c, band, s);
  else
    run_refine<3>(c, band, s);
}

}  // namespace agimp

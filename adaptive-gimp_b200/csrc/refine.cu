// Free-surface refinement rule (extension; the reference fixes g_p once at
// initialisation, init.py:17-29 and run_3d.py:151-156).
//
// depth(c) = Chebyshev distance in finest cells from occupied finest cell c to
// the nearest empty one (cells outside the particles' bounding box are
// empty), capped at K = 1 + band (2^(L-1) - 1): the value that iterated 3^d
// erosion over the bounding box reaches.  It is computed as a separable
// distance transform, one pass per axis: with f_0 = 0 on empty and K on
// occupied cells,
//   f_a(c) = min over x' on the line of c along axis a of max(f_{a-1}(c|x'), |x - x'|)
// (positions outside the box count as empty), so f_d = min(K, depth) exactly
// (min and max of integers).  A particle's prescribed level is L-1 when
// depth <= band, L-2 when depth <= 3*band, L-3 when depth <= 7*band, ..., and
// 0 deeper inside.
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

// bounding box of the particles' finest cells: every CTA reduces its share of
// the particles, then one atomic per CTA and bound (a few hundred CTAs: the
// six addresses see few atomics)
template <int D>
__global__ void k_bb(Ctx c) {
  __shared__ int s_lo[8][D], s_hi[8][D];
  int lo[D], hi[D];
#pragma unroll
  for (int d = 0; d < D; ++d) {
    lo[d] = INT_MAX;
    hi[d] = -1;
  }
  GS_LOOP(p, c.N) {
    int cell[D];
    if (particle_cell<D>(c, (int)p, cell))
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
    int a = INT_MAX, b = -1;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
      a = min(a, s_lo[w][d]);
      b = max(b, s_hi[w][d]);
    }
    if (b >= 0) {
      atomicMin(&c.ctr[CTR_BB + d], a);
      atomicMax(&c.ctr[CTR_BB + 3 + d], b);
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

// cell i of the bounding box (row-major, first axis slowest); box volumes stay
// below 2^31 (finest <= 1024 in 3D, 8192 in 2D), so 32-bit division
template <int D>
__device__ __forceinline__ void box_cell(const int* lo, const int* n, long long i, int* cell) {
  unsigned t = (unsigned)i;
#pragma unroll
  for (int d = D - 1; d >= 0; --d) {
    cell[d] = lo[d] + (int)(t % (unsigned)n[d]);
    t /= (unsigned)n[d];
  }
}

template <int D>
__global__ void k_occ_clear(Ctx c) {
  int lo[D], n[D];
  const long long vol = bb_volume<D>(c, lo, n);
  GS_LOOP(i, vol) {
    int cell[D];
    box_cell<D>(lo, n, i, cell);
    c.occ[occ_index<D>(c, cell)] = 0;
  }
}

template <int D>
__global__ void k_occ_mark(Ctx c) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  int cell[D];
  if (p < c.N && particle_cell<D>(c, p, cell)) c.occ[occ_index<D>(c, cell)] = 1;
}

// one pass of the distance transform along `axis`, from `in` to `out`
// (first pass: `in` holds occupancy 0 / 1, read as 0 / K)
template <int D>
__global__ void k_dt_axis(Ctx c, const uint8_t* __restrict__ in, uint8_t* __restrict__ out, int axis, int K,
                          int first) {
  int lo[D], n[D];
  const long long vol = bb_volume<D>(c, lo, n);
  long long stride = 1;
  for (int d = D - 1; d > axis; --d) stride *= c.sz;
  GS_LOOP(i, vol) {
    int cell[D];
    box_cell<D>(lo, n, i, cell);
    const long long idx = occ_index<D>(c, cell);
    const int x = cell[axis] - lo[axis], nx = n[axis];
    auto val = [&](int q) -> int {  // f at position q of the line (outside the box: empty)
      if (q < 0 || q >= nx) return 0;
      const int v = in[idx + (long long)(q - x) * stride];
      return first ? (v ? K : 0) : v;
    };
    int best = val(x);
    for (int o = 1; o < best; ++o) best = min(best, max(min(val(x - o), val(x + o)), o));
    out[idx] = (uint8_t)best;
  }
}

template <int D>
__global__ void k_assign(Ctx c, const uint8_t* depth, int band) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  int cell[D];
  if (p >= c.N || !particle_cell<D>(c, p, cell)) return;
  const int dd = depth[occ_index<D>(c, cell)];
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
  // agimp_refine_levels keeps band (2^(L-1) - 1) below 250: K fits the uint8 cells
  const int kmax = band * ((1 << (c.L - 1)) - 1) + 1;
  k_bb_init<<<1, 32, 0, s>>>(c);
  k_bb<D><<<c.sms * 2, 256, 0, s>>>(c);  // 256 threads: 8 warps (s_lo / s_hi)
  k_occ_clear<D><<<G, 256, 0, s>>>(c);
  k_occ_mark<D><<<Gp, 256, 0, s>>>(c);
  // passes alternate between the two buffers, the innermost axis first
  uint8_t* buf[2] = {c.occ, c.occ2};
  for (int k = 0; k < D; ++k)
    k_dt_axis<D><<<G, 256, 0, s>>>(c, buf[k & 1], buf[(k + 1) & 1], D - 1 - k, kmax, k == 0);
  k_assign<D><<<Gp, 256, 0, s>>>(c, buf[D & 1], band);
}

void launch_refine(const Ctx& c, int band, cudaStream_t s) {
  if (c.dim == 2)
    run_refine<2>(c, band, s);
  else
    run_refine<3>(c, band, s);
}

}  // namespace agimp

// Scene initialisers on the device: the particle fields and static level maps
// that the reference fills with Taichi kernels (init.py:3-98,
// run_3d.py:14-32), generated on the GPU from a small description so that a
// large scene needs neither host arrays nor an upload.
//
// * agimp_lattice_count / agimp_lattice_fill: points of a jittered
//   sub-lattice inside boxes and spheres (the scenes of the benchmark
//   configurations).  Count, scan of the per-tile counts, then an ordered
//   compaction: shape after shape, row-major lattice order inside a shape.
// * agimp_random_fill: particles uniform in boxes with the level bands of
//   init.py:3-32 (two boxes, g_p from the position inside the box) and
//   run_3d.py:14-32.
// * agimp_set_level_map_rule: init.py's initialize_mask1..5 tabulated over the
//   finest cells on the device; agimp_set_coarse_level_map: a map constant on
//   each coarsest cell, expanded on the device.
//
// Random numbers: Philox4x32-10 (J. Salmon, M. Moraes, R. Dror, D. Shaw,
// "Parallel random numbers: as easy as 1, 2, 3", SC 2011), a counter-based
// generator: the numbers of particle / lattice point k are a pure function of
// (seed, k), so the result does not depend on the launch shape.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "sim.h"

namespace agimp {

agimp_status install_level_map(agimp_sim* s, int8_t* dev_table, int halo, int n);

namespace {

struct U4 {
  uint32_t x, y, z, w;
};

// Philox4x32 with 10 rounds: each round multiplies words 0 and 2 by the
// round constants, swaps the halves and mixes in the key, which is bumped by
// the Weyl constants between rounds.
__host__ __device__ __forceinline__ U4 philox(U4 c, uint32_t k0, uint32_t k1) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    const uint64_t p0 = (uint64_t)0xD2511F53u * c.x;
    const uint64_t p1 = (uint64_t)0xCD9E8D57u * c.z;
    c = U4{(uint32_t)(p1 >> 32) ^ c.y ^ k0, (uint32_t)p1, (uint32_t)(p0 >> 32) ^ c.w ^ k1, (uint32_t)p0};
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  return c;
}

// 53-bit uniform double in [0, 1) from two words (a high, b low)
__device__ __forceinline__ double u53(uint32_t a, uint32_t b) {
  return (double)(((uint64_t)a << 32 | b) >> 11) * 0x1p-53;
}

// 24-bit uniform float in [0, 1)
__device__ __forceinline__ float u24(uint32_t a) { return (float)(a >> 8) * 0x1p-24f; }

// ---------------------------------------------------------------------------
// Jittered lattice
struct LatticeShape {
  int kind, level;
  double lo[3], hi[3], centre[3], r2;  // inside test
  double start[3];                     // first lattice index per axis (an integer)
  long long n[3];                      // lattice points per axis
  long long tile0;                     // first tile of this shape
  long long points;
  float vel[3], mass;
};

constexpr int TILE = 1024;  // lattice points per tile (one CTA)
constexpr int MAXSH = 64;

struct LatticeArgs {
  int dim, jitter, nsh;
  uint32_t k0, k1;
  double h;
  LatticeShape sh[MAXSH];
};

// lattice point k of shape j: position (double) and whether it is inside
template <int D>
__device__ __forceinline__ bool lattice_point(const LatticeArgs& A, int j, long long k, double* x) {
  const LatticeShape& S = A.sh[j];
  long long idx[D];
  long long t = k;
#pragma unroll
  for (int d = D - 1; d >= 0; --d) {
    idx[d] = t % S.n[d];
    t /= S.n[d];
  }
  double u[3] = {0.0, 0.0, 0.0};
  if (A.jitter) {
    const U4 a = philox(U4{(uint32_t)k, (uint32_t)((unsigned long long)k >> 32), (uint32_t)j, 0u}, A.k0, A.k1);
    u[0] = u53(a.x, a.y);
    u[1] = u53(a.z, a.w);
    if (D == 3) {
      const U4 b = philox(U4{(uint32_t)k, (uint32_t)((unsigned long long)k >> 32), (uint32_t)j, 1u}, A.k0, A.k1);
      u[2] = u53(b.x, b.y);
    }
  }
  const double hh = __dmul_rn(0.5, A.h);
  bool in = true;
  double s2 = 0.0;
#pragma unroll
  for (int d = 0; d < D; ++d) {
    // centre (start + i) h + h / 2, then the offset -h/2 + h u (u in [0, 1))
    const double c = __dadd_rn(__dmul_rn(S.start[d] + (double)idx[d], A.h), hh);
    x[d] = A.jitter ? __dadd_rn(c, __dadd_rn(-hh, __dmul_rn(A.h, u[d]))) : c;
    if (S.kind == AGIMP_SHAPE_BOX) {
      in = in && x[d] >= S.lo[d] && x[d] < S.hi[d];
    } else {
      const double e = __dsub_rn(x[d], S.centre[d]);
      s2 = d == 0 ? __dmul_rn(e, e) : __dadd_rn(s2, __dmul_rn(e, e));
    }
  }
  if (S.kind == AGIMP_SHAPE_SPHERE) in = s2 < S.r2;
  return in;
}

__device__ __forceinline__ int tile_shape(const LatticeArgs& A, long long tile) {
  int j = 0;
  while (j + 1 < A.nsh && A.sh[j + 1].tile0 <= tile) ++j;
  return j;
}

template <int D>
__global__ void __launch_bounds__(TILE) k_lattice_count(LatticeArgs A, long long ntiles, int* counts) {
  __shared__ int wc[TILE / 32];
  for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int j = tile_shape(A, tile);
    const long long k = (tile - A.sh[j].tile0) * TILE + threadIdx.x;
    double x[3];
    const bool in = k < A.sh[j].points && lattice_point<D>(A, j, k, x);
    const unsigned b = __ballot_sync(0xffffffffu, in);
    if ((threadIdx.x & 31) == 0) wc[threadIdx.x >> 5] = __popc(b);
    __syncthreads();
    if (threadIdx.x < 32) {
      int v = wc[threadIdx.x];
#pragma unroll
      for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
      if (threadIdx.x == 0) counts[tile] = v;
    }
    __syncthreads();
  }
}

// exclusive scan of n counts into offs (one CTA); offs[n] = total
__global__ void __launch_bounds__(1024) k_scan_counts(const int* counts, long long n, long long* offs) {
  __shared__ long long part[1024];
  const long long per = (n + blockDim.x - 1) / blockDim.x;
  const long long a = min(n, per * threadIdx.x), b = min(n, a + per);
  long long s = 0;
  for (long long i = a; i < b; ++i) s += counts[i];
  part[threadIdx.x] = s;
  __syncthreads();
  for (int o = 1; o < (int)blockDim.x; o <<= 1) {  // inclusive Hillis-Steele scan
    const long long v = threadIdx.x >= (unsigned)o ? part[threadIdx.x - o] : 0;
    __syncthreads();
    part[threadIdx.x] += v;
    __syncthreads();
  }
  long long run = part[threadIdx.x] - s;
  for (long long i = a; i < b; ++i) {
    offs[i] = run;
    run += counts[i];
  }
  if (threadIdx.x == blockDim.x - 1) offs[n] = part[threadIdx.x];
}

template <int D>
__global__ void __launch_bounds__(TILE) k_lattice_fill(LatticeArgs A, long long ntiles, const long long* offs,
                                                       Particles P, long long N) {
  __shared__ int wc[TILE / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int j = tile_shape(A, tile);
    const LatticeShape& S = A.sh[j];
    const long long k = (tile - S.tile0) * TILE + threadIdx.x;
    double x[3];
    const bool in = k < S.points && lattice_point<D>(A, j, k, x);
    const unsigned b = __ballot_sync(0xffffffffu, in);
    if (lane == 0) wc[warp] = __popc(b);
    __syncthreads();
    int before = 0;
    for (int w = 0; w < warp; ++w) before += wc[w];
    __syncthreads();
    if (in) {
      const long long p = offs[tile] + before + __popc(b & ((1u << lane) - 1u));
      if (p < N) {
#pragma unroll
        for (int d = 0; d < D; ++d) {
          P.x[d * N + p] = __double2float_rn(x[d]);
          P.v[d * N + p] = S.vel[d];
        }
#pragma unroll
        for (int e = 0; e < D * D; ++e) {
          P.F[e * N + p] = (e % (D + 1) == 0) ? 1.f : 0.f;
          P.C[e * N + p] = 0.f;
        }
        P.m[p] = S.mass;
        P.Jp[p] = 1.f;
        P.g[p] = S.level;
        P.id[p] = (int)p;
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Uniform particles in boxes with level bands (init.py:3-32, run_3d.py:14-32)
struct RandomBox {
  long long first, count;
  float lo[3], size[3], vel[3], mass;
  int nb, level;
  float blo[4], bhi[4];
  int blev[4];
};

constexpr int MAXBOX = 16;

struct RandomArgs {
  int nbox;
  uint32_t k0, k1;
  RandomBox b[MAXBOX];
};

template <int D>
__global__ void k_random_fill(RandomArgs A, Particles P, long long N) {
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < N; p += (long long)gridDim.x * blockDim.x) {
    int j = 0;
    while (j + 1 < A.nbox && A.b[j + 1].first <= p) ++j;
    const RandomBox& B = A.b[j];
    const U4 r = philox(U4{(uint32_t)p, (uint32_t)((unsigned long long)p >> 32), 0u, 0u}, A.k0, A.k1);
    const float u[3] = {u24(r.x), u24(r.y), u24(r.z)};
    // x = u * size + lo in f32 (explicitly rounded: no contraction)
#pragma unroll
    for (int d = 0; d < D; ++d) {
      P.x[d * N + p] = __fadd_rn(__fmul_rn(u[d], B.size[d]), B.lo[d]);
      P.v[d * N + p] = B.vel[d];
    }
    int g = B.level;
    for (int k = B.nb - 1; k >= 0; --k) {  // the first matching band wins
      bool in = true;
#pragma unroll
      for (int d = 0; d < D; ++d) in = in && B.blo[k] <= u[d] && u[d] <= B.bhi[k];
      if (in) g = B.blev[k];
    }
#pragma unroll
    for (int e = 0; e < D * D; ++e) {
      P.F[e * N + p] = (e % (D + 1) == 0) ? 1.f : 0.f;
      P.C[e * N + p] = 0.f;
    }
    P.m[p] = B.mass;
    P.Jp[p] = 1.f;
    P.g[p] = g;
    P.id[p] = (int)p;
  }
}

// ---------------------------------------------------------------------------
// Level maps.  Entry: level in bits 0-3, bit 6 = no activation; table over
// finest cells [-H, sz + H)^dim, first axis slowest.
__device__ __forceinline__ bool inner8(const int* I, int D, int sz) {
  bool r = true;
  for (int d = 0; d < D; ++d) r = r && I[d] >= 8 && I[d] < sz - 8;
  return r;
}

__device__ __forceinline__ bool in_range(const int* I, int D, int sz) {
  bool r = true;
  for (int d = 0; d < D; ++d) r = r && I[d] >= 0 && I[d] < sz;
  return r;
}

// initialize_mask1..5 (init.py:34-98) at finest cell I
__device__ __forceinline__ int8_t mask_rule(int rule, const int* I, int D, int sz, int L) {
  const double half = (double)sz / 2.0, quarter = (double)sz / 4.0;  // `sz / 2` is true division
  const bool inner = inner8(I, D, sz);
  switch (rule) {
    case 1:  // every cell at the finest level
      return (int8_t)(L - 1);
    case 2:  // level 0 in the left half (8-cell margin), level 3 elsewhere
      return (int8_t)((I[0] < half && inner) ? 0 : 3);
    case 3:  // levels 0 / 1 / 2 in vertical bands
      return (int8_t)((I[0] < quarter && inner) ? 0 : (I[0] < half && inner) ? 1 : 2);
    case 4: {  // levels 1 / 2 in the left half, 3 elsewhere in range, else 3 without activation
      if (I[0] < half && inner) return (int8_t)(I[1] < half ? 1 : 2);
      return (int8_t)(in_range(I, D, sz) ? 3 : (3 | 64));
    }
    default: {  // 5: levels 0 / 1 / 2 in the left half, 3 elsewhere in range
      if (I[0] < half && inner) return (int8_t)(I[1] < quarter ? 0 : I[1] < half ? 1 : 2);
      return (int8_t)(in_range(I, D, sz) ? 3 : (3 | 64));
    }
  }
}

__global__ void k_map_rule(int rule, int D, int sz, int L, int H, int n, long long total, int8_t* table) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    int I[3];
    long long t = e;
    for (int d = D - 1; d >= 0; --d) {
      I[d] = (int)(t % n) - H;
      t /= n;
    }
    table[e] = mask_rule(rule, I, D, sz, L);
  }
}

__global__ void k_map_coarse(const int8_t* coarse, int D, int sz, int nc, int L, int H, int n, long long total,
                             int8_t* table) {
  const int s = L - 1;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    int I[3];
    long long t = e;
    for (int d = D - 1; d >= 0; --d) {
      I[d] = (int)(t % n) - H;
      t /= n;
    }
    int8_t v;
    if (in_range(I, D, sz)) {
      long long c = 0;
      for (int d = 0; d < D; ++d) c = c * nc + (I[d] >> s);
      v = coarse[c];
    } else {
      v = (int8_t)((L - 1) | 64);
    }
    table[e] = v;
  }
}

int grid_for(long long n, int threads) { return (int)std::max<long long>(1, std::min<long long>((n + threads - 1) / threads, 148LL * 32)); }

// host side of the lattice: per-shape index ranges and tiles
agimp_status lattice_setup(int dim, int finest, int per_axis, int jitter, uint64_t seed, const agimp_shape* shapes,
                           int nsh, LatticeArgs& A, long long& ntiles, std::string& err) {
  if ((dim != 2 && dim != 3) || finest < 1 || per_axis < 1 || nsh < 0 || nsh > MAXSH || (nsh && !shapes)) {
    err = "lattice: dim 2 or 3, finest >= 1, per_axis >= 1, 0 <= n_shapes <= 64";
    return AGIMP_INVALID_ARG;
  }
  std::memset(&A, 0, sizeof(A));
  A.dim = dim;
  A.jitter = jitter != 0;
  A.nsh = nsh;
  A.k0 = (uint32_t)seed;
  A.k1 = (uint32_t)(seed >> 32);
  A.h = 1.0 / (double)((long long)finest * per_axis);
  ntiles = 0;
  for (int j = 0; j < nsh; ++j) {
    const agimp_shape& q = shapes[j];
    LatticeShape& S = A.sh[j];
    if (q.kind != AGIMP_SHAPE_BOX && q.kind != AGIMP_SHAPE_SPHERE) {
      err = "lattice: unknown shape kind";
      return AGIMP_INVALID_ARG;
    }
    S.kind = q.kind;
    S.level = q.level;
    S.r2 = q.radius * q.radius;
    long long pts = 1;
    for (int d = 0; d < dim; ++d) {
      S.lo[d] = q.lo[d];
      S.hi[d] = q.hi[d];
      S.centre[d] = q.centre[d];
      S.vel[d] = q.velocity[d];
      // the region's bounding box: the box itself, or centre -+ radius
      const double a = q.kind == AGIMP_SHAPE_BOX ? q.lo[d] : q.centre[d] - q.radius;
      const double b = q.kind == AGIMP_SHAPE_BOX ? q.hi[d] : q.centre[d] + q.radius;
      const double i0 = std::floor(a / A.h), i1 = std::ceil(b / A.h);
      if (!(std::isfinite(i0) && std::isfinite(i1)) || std::fabs(i0) > 1e15 || std::fabs(i1) > 1e15) {
        err = "lattice: shape bounds out of range";
        return AGIMP_INVALID_ARG;
      }
      S.start[d] = i0;
      S.n[d] = std::max(0LL, (long long)(i1 - i0));
      pts *= S.n[d];
    }
    S.mass = q.mass;
    S.points = pts;
    S.tile0 = ntiles;
    ntiles += (pts + TILE - 1) / TILE;
  }
  return AGIMP_OK;
}

// counts and offsets of the tiles (device scratch owned by the caller)
cudaError_t lattice_offsets(const LatticeArgs& A, long long ntiles, int** counts, long long** offs, long long* total,
                            cudaStream_t st) {
  *counts = nullptr;
  *offs = nullptr;
  cudaError_t e = cudaMalloc(counts, sizeof(int) * std::max(1LL, ntiles));
  if (e == cudaSuccess) e = cudaMalloc(offs, sizeof(long long) * (ntiles + 1));
  if (e != cudaSuccess) return e;
  if (ntiles) {
    if (A.dim == 2)
      k_lattice_count<2><<<grid_for(ntiles, 1), TILE, 0, st>>>(A, ntiles, *counts);
    else
      k_lattice_count<3><<<grid_for(ntiles, 1), TILE, 0, st>>>(A, ntiles, *counts);
    k_scan_counts<<<1, 1024, 0, st>>>(*counts, ntiles, *offs);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(total, *offs + ntiles, sizeof(long long), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  } else {
    *total = 0;
  }
  return e;
}

}  // namespace
}  // namespace agimp

using namespace agimp;

extern "C" {

agimp_status agimp_lattice_count(int32_t dim, int32_t finest, int32_t per_axis, int32_t jitter, uint64_t seed,
                                 const agimp_shape* shapes, int32_t n_shapes, int64_t* count, int32_t device) {
  if (!count) return AGIMP_INVALID_ARG;
  LatticeArgs A;
  long long ntiles = 0;
  std::string err;
  agimp_status st = lattice_setup(dim, finest, per_axis, jitter, seed, shapes, n_shapes, A, ntiles, err);
  if (st != AGIMP_OK) return st;
  if (cudaSetDevice(device) != cudaSuccess) return AGIMP_CUDA_ERROR;
  int* counts = nullptr;
  long long* offs = nullptr;
  long long total = 0;
  cudaError_t e = lattice_offsets(A, ntiles, &counts, &offs, &total, 0);
  if (counts) cudaFree(counts);
  if (offs) cudaFree(offs);
  if (e != cudaSuccess) return AGIMP_CUDA_ERROR;
  *count = total;
  return AGIMP_OK;
}

agimp_status agimp_lattice_fill(agimp_sim* s, int32_t per_axis, int32_t jitter, uint64_t seed,
                                const agimp_shape* shapes, int32_t n_shapes, void* stream) {
  if (!s) return AGIMP_INVALID_ARG;
  LatticeArgs A;
  long long ntiles = 0;
  agimp_status st = lattice_setup(s->c.dim, s->c.sz, per_axis, jitter, seed, shapes, n_shapes, A, ntiles, s->err);
  if (st != AGIMP_OK) return st;
  if (cudaSetDevice(s->device) != cudaSuccess) return AGIMP_CUDA_ERROR;
  cudaStream_t use = stream ? (cudaStream_t)stream : s->internal;
  wait_readback(s, s->par, use);  // the fill overwrites the state being read
  int* counts = nullptr;
  long long* offs = nullptr;
  long long total = 0;
  cudaError_t e = lattice_offsets(A, ntiles, &counts, &offs, &total, use);
  if (e == cudaSuccess && total != s->c.N) {
    cudaFree(counts);
    cudaFree(offs);
    s->err = "lattice fill: the shapes hold " + std::to_string(total) + " points, the simulator " +
             std::to_string(s->c.N) + " particles";
    return AGIMP_INVALID_ARG;
  }
  if (e == cudaSuccess && ntiles) {
    const Particles& P = s->buf[s->par];
    if (A.dim == 2)
      k_lattice_fill<2><<<grid_for(ntiles, 1), TILE, 0, use>>>(A, ntiles, offs, P, s->c.N);
    else
      k_lattice_fill<3><<<grid_for(ntiles, 1), TILE, 0, use>>>(A, ntiles, offs, P, s->c.N);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaEventRecord(s->ev_state, use);  // later asynchronous readbacks follow the fill
    if (e == cudaSuccess) e = cudaStreamSynchronize(use);  // before the scratch is freed
    s->state_marked = true;
  }
  if (counts) cudaFree(counts);
  if (offs) cudaFree(offs);
  if (e != cudaSuccess) {
    s->err = std::string("lattice fill: ") + cudaGetErrorString(e);
    return AGIMP_CUDA_ERROR;
  }
  return AGIMP_OK;
}

agimp_status agimp_random_fill(agimp_sim* s, uint64_t seed, const agimp_random_box* boxes, int32_t n_boxes,
                               void* stream) {
  if (!s) return AGIMP_INVALID_ARG;
  if (n_boxes < 1 || n_boxes > MAXBOX || !boxes) {
    s->err = "random fill: 1 <= n_boxes <= 16";
    return AGIMP_INVALID_ARG;
  }
  RandomArgs A;
  std::memset(&A, 0, sizeof(A));
  A.nbox = n_boxes;
  A.k0 = (uint32_t)seed;
  A.k1 = (uint32_t)(seed >> 32);
  long long first = 0;
  for (int j = 0; j < n_boxes; ++j) {
    const agimp_random_box& q = boxes[j];
    RandomBox& B = A.b[j];
    if (q.count < 0 || q.n_bands < 0 || q.n_bands > 4) {
      s->err = "random fill: count >= 0 and 0 <= n_bands <= 4";
      return AGIMP_INVALID_ARG;
    }
    B.first = first;
    B.count = q.count;
    first += q.count;
    for (int d = 0; d < 3; ++d) {
      B.lo[d] = q.lo[d];
      B.size[d] = q.size[d];
      B.vel[d] = q.velocity[d];
    }
    B.mass = q.mass;
    B.nb = q.n_bands;
    B.level = q.level;
    for (int k = 0; k < 4; ++k) {
      B.blo[k] = q.band_lo[k];
      B.bhi[k] = q.band_hi[k];
      B.blev[k] = q.band_level[k];
    }
  }
  if (first != s->c.N) {
    s->err = "random fill: the box counts sum to " + std::to_string(first) + ", the simulator has " +
             std::to_string(s->c.N) + " particles";
    return AGIMP_INVALID_ARG;
  }
  if (cudaSetDevice(s->device) != cudaSuccess) return AGIMP_CUDA_ERROR;
  cudaStream_t use = stream ? (cudaStream_t)stream : s->internal;
  wait_readback(s, s->par, use);
  const Particles& P = s->buf[s->par];
  if (s->c.N) {
    if (s->c.dim == 2)
      k_random_fill<2><<<grid_for(s->c.N, 256), 256, 0, use>>>(A, P, s->c.N);
    else
      k_random_fill<3><<<grid_for(s->c.N, 256), 256, 0, use>>>(A, P, s->c.N);
  }
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaEventRecord(s->ev_state, use);  // later asynchronous readbacks follow the fill
  s->state_marked = true;
  if (e == cudaSuccess && !stream) e = cudaStreamSynchronize(use);
  if (e != cudaSuccess) {
    s->err = std::string("random fill: ") + cudaGetErrorString(e);
    return AGIMP_CUDA_ERROR;
  }
  return AGIMP_OK;
}

agimp_status agimp_set_level_map_rule(agimp_sim* s, int32_t rule, void* stream) {
  if (!s) return AGIMP_INVALID_ARG;
  const int L = s->c.L, D = s->c.dim, sz = s->c.sz;
  static const int need[6] = {0, 1, 4, 3, 4, 4};  // levels each rule uses
  if (rule < 1 || rule > 5 || L < need[rule]) {
    s->err = "level map rule: 1..5 (rules 2, 4, 5 need 4 levels, rule 3 needs 3)";
    return AGIMP_INVALID_ARG;
  }
  if (cudaSetDevice(s->device) != cudaSuccess) return AGIMP_CUDA_ERROR;
  const int H = std::max(2, 1 << (L - 1)), n = sz + 2 * H;
  long long total = 1;
  for (int d = 0; d < D; ++d) total *= n;
  int8_t* table = nullptr;
  cudaError_t e = cudaMalloc(&table, (size_t)total);
  cudaStream_t use = stream ? (cudaStream_t)stream : s->internal;
  if (e == cudaSuccess) {
    k_map_rule<<<grid_for(total, 256), 256, 0, use>>>(rule, D, sz, L, H, n, total, table);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(use);
  if (e != cudaSuccess) {
    if (table) cudaFree(table);
    s->err = std::string("level map rule: ") + cudaGetErrorString(e);
    return AGIMP_CUDA_ERROR;
  }
  return install_level_map(s, table, H, n);
}

agimp_status agimp_set_coarse_level_map(agimp_sim* s, const int8_t* coarse_levels, int32_t memory, void* stream) {
  if (!s || !coarse_levels || (memory != AGIMP_MEM_HOST && memory != AGIMP_MEM_DEVICE)) return AGIMP_INVALID_ARG;
  const int L = s->c.L, D = s->c.dim, sz = s->c.sz, nc = s->c.coarsest;
  long long nco = 1;
  for (int d = 0; d < D; ++d) nco *= nc;
  std::vector<int8_t> host((size_t)nco);
  if (cudaSetDevice(s->device) != cudaSuccess) return AGIMP_CUDA_ERROR;
  cudaStream_t use = stream ? (cudaStream_t)stream : s->internal;
  if (memory == AGIMP_MEM_HOST) {
    std::memcpy(host.data(), coarse_levels, (size_t)nco);
  } else if (cudaMemcpyAsync(host.data(), coarse_levels, (size_t)nco, cudaMemcpyDeviceToHost, use) != cudaSuccess ||
             cudaStreamSynchronize(use) != cudaSuccess) {
    return AGIMP_CUDA_ERROR;
  }
  for (long long i = 0; i < nco; ++i)
    if (host[i] < 0 || host[i] >= L) {
      s->err = "coarse level map: entry out of [0, level) at " + std::to_string(i);
      return AGIMP_INVALID_ARG;
    }
  const int H = std::max(2, 1 << (L - 1)), n = sz + 2 * H;
  long long total = 1;
  for (int d = 0; d < D; ++d) total *= n;
  int8_t* table = nullptr;
  int8_t* dco = nullptr;
  cudaError_t e = cudaMalloc(&table, (size_t)total);
  if (e == cudaSuccess) e = cudaMalloc(&dco, (size_t)nco);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dco, host.data(), (size_t)nco, cudaMemcpyHostToDevice, use);
  if (e == cudaSuccess) {
    k_map_coarse<<<grid_for(total, 256), 256, 0, use>>>(dco, D, sz, nc, L, H, n, total, table);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(use);
  if (dco) cudaFree(dco);
  if (e != cudaSuccess) {
    if (table) cudaFree(table);
    s->err = std::string("coarse level map: ") + cudaGetErrorString(e);
    return AGIMP_CUDA_ERROR;
  }
  return install_level_map(s, table, H, n);
}

}  // extern "C"

// Shared definitions of the B200 adaptive GIMP substep.
//
// Data layout in HBM (one simulator):
//  * Every level l stores cells and nodes over indices [-4, size_l + 8) per
//    axis, blocked in 4^d tiles: element (i,j[,k]) lives at
//      block(i>>2 +1, j>>2 +1 [, k>>2 +1]) * 4^d + local(i&3, j&3 [, k&3]),
//    blocks in row-major order (first axis slowest).  A 4^d tile is the
//    reference's leaf block (adaptive_gimp.py:28-42) and is contiguous
//    (64 B of masks / 1 KB of node records in 3D).
//  * node record: float4 {p_x | v_x, p_y | v_y, p_z | v_z, m}: momentum until
//    grid_op, velocity after, exactly like ad_grid_v / ad_grid_m.
//  * cell mask: u32 per cell (utils.py:5-9 flags, plus CULLING kept internally
//    until the next substep; readback masks it out).
//  * node mask: u32 on the finest lattice, same blocked layout as the finest
//    level (adaptive_gimp.py:23-26: one mask shared by all levels through
//    _map, adaptive_gimp.py:126-128).
//  * per level: bmap (block -> index in the active list, -1 if inactive) and
//    the active block list itself.  Active blocks are the 4^d blocks within
//    one block of any particle's position at that level; every nonzero cell,
//    node value or node flag of a substep lies inside them.
//  * particles: SoA, one f32 array per component ([c * N + p]).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace agimp {

constexpr int MAXL = 8;
constexpr int CHUNK = 256;      // default P2G work item (particles of one bin) = P2G CTA size
constexpr int MAX_CHUNK = 512;  // largest work item the tuning may choose
constexpr int MIN_CHUNK = 64;   // smallest work item (sizes the work-item buffer)
constexpr int HALO = 4;

enum : uint32_t { ACT = 1u, GHO = 2u, TJ = 4u, CUL = 8u };
enum : uint32_t { ERR_OOB = 1u, ERR_ESCAPED = 2u, ERR_MAP_OOB = 4u, ERR_NOBIN = 8u, ERR_MLP = 16u };

// device counters
enum {
  CTR_LEVEL = 0,   // [0, MAXL): active blocks per level
  CTR_TOUCH = 8,   // touched finest blocks
  CTR_BINCUR = 9,  // particles placed by the bin allocator
  CTR_CHUNKS = 10, // P2G/G2P work items
  CTR_ERR = 11,    // error bits
  CTR_UNBIN = 12,  // particles without a level (fl_p = -1) in the last substep
  CTR_SUR = 13,    // particles handed to the surrogate MLP in the last substep
  CTR_REC = 14,    // recorded (features, projected state) pairs since the recorder was armed
  CTR_SURFB = 15,  // surrogate predictions rejected (exact return map used instead)
  // [16, 22): particle bounding box used by the refinement rule
  CTR_PROJ = 22,   // particles whose trial state needs the return map this substep
  CTR_FULL = 23,   // non-empty bins this substep (listed in full_bins)
  CTR_COUNT = 24
};

struct LevelDev {
  int size;          // cells per axis at this level
  int nb;            // stored blocks per axis (size/4 + 3)
  long long nblocks; // nb^dim
  uint32_t* cell;
  float4* node;
  int32_t* bmap;
  int32_t* blist;
  // node mask of this level's nodes, in the level's own blocked layout
  // (node_mask[_map(l, I)], adaptive_gimp.py:126-128): the finest level's is
  // the node mask itself; coarser levels get a copy after ghost / T-junction
  // marking, so the level transfers read whole blocks of it
  uint32_t* nm;
  // levels below the finest: per block, 1 + the largest radius around which
  // k_dilate has activated this substep's blocks (0: none; cleared through
  // the touch list), so touched blocks with a common ancestor walk its
  // neighbourhood once
  uint32_t* dflag;
};

struct Particles {
  float* x;    // [dim][N]
  float* v;    // [dim][N]
  float* F;    // [dim*dim][N]
  float* C;    // [dim*dim][N]
  float* m;    // [N]
  float* Jp;   // [N]
  int32_t* g;  // [N] prescribed level
  int32_t* fl; // [N] level used by the last substep
  int32_t* id; // [N] the particle's index in the caller's arrays
};

struct Ctx {
  int dim, L, coarsest, sz;
  int N;
  int sms;  // multiprocessors of the device (grid-stride launch width)
  int is_static, gap, bmode, plast, ncol, map_h, map_n;
  int inv_norm;  // 1: normalise nodes that are not activated (extension)
  int chunk;     // particles per P2G work item: 64, 128 or 256 (launch tuning)
  float radius, mu, la, theta_c, theta_s, xi, dt;
  float grav[3];
  double col[4][6];  // collider boxes, compared in double like the oracle
  LevelDev lev[MAXL];
  uint32_t* nmask;
  int32_t* ctr;
  uint32_t* touch_flag;
  int32_t* touch_list;
  uint32_t* touch_occ;  // static mode, [finest blocks][1 (2D) or 5 (3D)]: base cells of the block's particles
  int32_t* bin_count;   // [bins]: particles per bin
  int32_t* cell_count;  // [bins][4^d]: particles per (bin, base cell inside the bin's block)
  int32_t* cell_off;    // [bins][4^d]: their offsets inside the bin (particles of a bin are cell-sorted)
  int32_t* bin_start;
  int32_t* full_bins;   // [bins]: the non-empty bins of this substep
  int4* chunks;  // {level, block (stored linear id), start, count}
  int32_t* bin_of;      // per particle: bin * 4^d + base cell
  int32_t* rank_of;
  int32_t* perm;
  int32_t* proj;  // [N] slots of the particles listed for the return map (CTR_PROJ of them)
  // Particle state, SoA.  P holds the state the substep starts from, in the
  // bin order of the previous substep; G2P writes the new state into Q in this
  // substep's bin order (the host swaps P and Q between substeps).
  Particles P, Q;
  const int8_t* map;
  uint8_t* occ;   // refinement scratch over the finest cells
  uint8_t* occ2;  // its second buffer (the distance transform's passes alternate)
  // surrogate return map and training-pair recorder (extension)
  int sur;                   // 1: G2P hands particles that need a projection to the MLP
  int rec_stride;            // recorder: particles whose new slot is a multiple of this
  long long rec_cap;         // recorder capacity (pairs)
  float sur_tol;             // accepted residual of a prediction
  float sur_xmax[8];         // trained range of each feature
  float* sur_X;              // [N][7]
  float* sur_Y;              // [N][4]
  float* sur_meta;           // [N][SUR_META]
  float* rec_X;              // [rec_cap][7]
  float* rec_T;              // [rec_cap][4]
  const void* mlp_packed;    // bf16 operand tiles of the MLP
  const float* mlp_P;        // f32 parameters of the MLP
  // Slot counter of the surrogate buffers: this scene's ctr[CTR_SUR] when the
  // simulator steps alone, or one counter shared by every scene of a batch
  // whose scenes share one set of buffers (then `scene` tells k_sur_finish
  // whose particle a slot holds).
  int32_t* sur_ctr;
  int scene;                 // index of the scene in the batch being stepped
};

// Surrogate features of a trial elastic state with singular values sig and
// plastic volume ratio jp (snow, Stomakhin et al. 2013): 7 inputs
//   (sig_i - 1) / 0.05 (i < 3; 0 for the missing one in 2D), log(jp) / 0.5,
//   xi (1 - jp) / 5 (the log of the hardening scale), theta_c / 0.025 - 1,
//   theta_s / 0.0075 - 1,
// and 4 outputs, the return map's change of those quantities:
//   (projected sig_i - sig_i) / 0.02, (log(new jp) - log(jp)) / 0.02.
// Outputs as changes are exactly 0 along elastic directions, so the network's
// bf16 resolution only limits the plastic part of the map.
constexpr float SUR_SIG = 0.05f, SUR_LJ = 0.5f, SUR_H = 5.f;
constexpr float SUR_DSIG = 0.02f, SUR_DLJ = 0.02f;
constexpr int SUR_META = 24;  // slot, U[9], V[9], sig[3], jp, scene

template <int D>
__host__ __device__ __forceinline__ void snow_features(const float* sig, float jp, float xi, float tc, float ts,
                                                       float* x) {
#pragma unroll
  for (int d = 0; d < 3; ++d) x[d] = d < D ? (sig[d] - 1.f) / SUR_SIG : 0.f;
  x[3] = logf(jp) / SUR_LJ;
  x[4] = xi * (1.f - jp) / SUR_H;
  x[5] = tc / 0.025f - 1.f;
  x[6] = ts / 0.0075f - 1.f;
}

// ---------------------------------------------------------------------------
// index helpers
template <int D>
__host__ __device__ __forceinline__ bool in_store(const LevelDev& V, const int* I) {
#pragma unroll
  for (int d = 0; d < D; ++d)
    if ((unsigned)(I[d] + HALO) >= (unsigned)(4 * V.nb)) return false;
  return true;
}

// Element and block indices fit in 32 bits (agimp_create rejects lattices of
// more than 2^31 elements per level), so the index arithmetic is 32-bit.
template <int D>
__host__ __device__ __forceinline__ long long elem_of(const LevelDev& V, const int* I) {
  unsigned b = 0, loc = 0;
#pragma unroll
  for (int d = 0; d < D; ++d) {
    const unsigned a = (unsigned)(I[d] + HALO);
    b = b * (unsigned)V.nb + (a >> 2);
    loc = (loc << 2) | (a & 3u);
  }
  return (long long)((b << (2 * D)) | loc);
}

// The 2^D elements I0 + {0,1}^D of one level (corner a adds bit D-1-d of a
// on axis d, the order of the corner loops): each axis's share of the
// element index (block part and local part) is formed once for I0[d] and
// I0[d] + 1, so a corner costs D-1 additions instead of a full elem_of.
template <int D>
struct Corners {
  unsigned t[D][2];
  bool v[D][2];
  __host__ __device__ __forceinline__ Corners(const LevelDev& V, const int* I0) {
    const unsigned nb = (unsigned)V.nb;
    unsigned m = 1;  // nb^(D-1-d)
#pragma unroll
    for (int d = D - 1; d >= 0; --d) {
#pragma unroll
      for (int k = 0; k < 2; ++k) {
        const unsigned a = (unsigned)(I0[d] + k + HALO);
        v[d][k] = a < 4u * nb;
        t[d][k] = (((a >> 2) * m) << (2 * D)) | ((a & 3u) << (2 * (D - 1 - d)));
      }
      m *= nb;
    }
  }
  // element index of corner a (equal to elem_of of I0 + corner offsets)
  __host__ __device__ __forceinline__ unsigned idx(int a) const {
    unsigned r = 0;
#pragma unroll
    for (int d = 0; d < D; ++d) r += t[d][(a >> (D - 1 - d)) & 1];
    return r;
  }
  // corner a lies in the store (in_store)
  __host__ __device__ __forceinline__ bool ok(int a) const {
    bool r = true;
#pragma unroll
    for (int d = 0; d < D; ++d) r = r && v[d][(a >> (D - 1 - d)) & 1];
    return r;
  }
};

template <int D>
__device__ __forceinline__ long long block_of(const LevelDev& V, const int* I) {
  unsigned b = 0;
#pragma unroll
  for (int d = 0; d < D; ++d) b = b * (unsigned)V.nb + ((unsigned)(I[d] + HALO) >> 2);
  return (long long)b;
}

// element coordinates of local index `loc` in stored block `blk`
template <int D>
__device__ __forceinline__ void elem_coords(const LevelDev& V, long long blk, int loc, int* I) {
  unsigned b = (unsigned)blk;
  const unsigned nb = (unsigned)V.nb;
#pragma unroll
  for (int d = D - 1; d >= 0; --d) {
    const unsigned q = b / nb;
    const int bd = (int)(b - q * nb);
    b = q;
    I[d] = (bd << 2) + ((loc >> (2 * (D - 1 - d))) & 3) - HALO;
  }
}

// node_mask[_map(l, I)] (adaptive_gimp.py:126-131); positions outside the
// finest lattice [0, sz] read 0.
template <int D>
__device__ __forceinline__ uint32_t nm_get(const Ctx& c, int l, const int* I) {
  const int s = c.L - 1 - l;
  int P[D];
#pragma unroll
  for (int d = 0; d < D; ++d) {
    P[d] = I[d] * (1 << s);
    if (P[d] < 0 || P[d] > c.sz) return 0u;
  }
  return c.nmask[elem_of<D>(c.lev[c.L - 1], P)];
}

template <int D>
__device__ __forceinline__ void nm_or(const Ctx& c, int l, const int* I, uint32_t bits) {
  const int s = c.L - 1 - l;
  int P[D];
#pragma unroll
  for (int d = 0; d < D; ++d) {
    P[d] = I[d] * (1 << s);
    if (P[d] < 0 || P[d] > c.sz) return;  // unobservable: never read by a predicate
  }
  uint32_t* w = &c.nmask[elem_of<D>(c.lev[c.L - 1], P)];
  if ((*w & bits) != bits) atomicOr(w, bits);
}

__device__ __forceinline__ bool is_valid(uint32_t nm) { return nm > 0u; }
__device__ __forceinline__ bool is_activated(uint32_t nm) { return (nm & (ACT | TJ)) == ACT; }
__device__ __forceinline__ bool is_tj(uint32_t nm) { return (nm & TJ) == TJ; }
__device__ __forceinline__ bool is_ghost(uint32_t nm) { return (nm & (ACT | GHO | TJ)) == GHO; }

__device__ __forceinline__ void set_err(const Ctx& c, uint32_t bits) {
  if ((((volatile uint32_t*)c.ctr)[CTR_ERR] & bits) != bits) atomicOr((unsigned*)&c.ctr[CTR_ERR], bits);
}

// Decode flat element e over the active lists of levels [l0, l1) -> level,
// block, local index.  Returns false past the end.
template <int D>
__device__ __forceinline__ bool decode_elem(const Ctx& c, int l0, int l1, long long e, int& l, long long& blk,
                                            int& loc) {
  const int per = 1 << (2 * D);
  long long bi = e >> (2 * D);
  loc = (int)(e & (per - 1));
  for (int q = l0; q < l1; ++q) {
    int n = c.ctr[CTR_LEVEL + q];
    if (bi < n) {
      l = q;
      blk = c.lev[q].blist[bi];
      return true;
    }
    bi -= n;
  }
  return false;
}

// Warp-aggregated slot reservation for the lanes that call it together (one
// atomic per warp instead of one per lane: counters shared by a whole grid
// serialise at L2)
__device__ __forceinline__ int reserve_slot(int32_t* counter) {
  const unsigned mask = __activemask();
  const int lane = threadIdx.x & 31;
  const int leader = __ffs(mask) - 1;
  int base = 0;
  if (lane == leader) base = atomicAdd(counter, __popc(mask));
  base = __shfl_sync(mask, base, leader);
  return base + __popc(mask & ((1u << lane) - 1u));
}

// First entry of each level's active blocks in the level-by-level block
// numbering (s[q] = active blocks of the levels below q, s[L] = all of them),
// read from the counters once per CTA: the per-element loops then decode an
// element from shared memory instead of re-reading the counters.  Every
// thread of the CTA calls it (it ends with a barrier).
struct BlockRanges {
  int s[MAXL + 1];
};

__device__ __forceinline__ void load_block_ranges(const Ctx& c, BlockRanges& r) {
  if (threadIdx.x == 0) {
    int t = 0;
    for (int q = 0; q < c.L; ++q) {
      r.s[q] = t;
      t += c.ctr[CTR_LEVEL + q];
    }
    r.s[c.L] = t;
  }
  __syncthreads();
}

// element e of the active blocks of levels [l0, l1): its level, stored
// block and local index (decode_elem through the CTA's BlockRanges)
template <int D>
__device__ __forceinline__ void decode_elem_r(const Ctx& c, const BlockRanges& r, int l0, int l1, long long e, int& l,
                                              long long& blk, int& loc) {
  const int bi = (int)(e >> (2 * D)) + r.s[l0];
  loc = (int)(e & ((1 << (2 * D)) - 1));
  int q = l0;
  while (q + 1 < l1 && bi >= r.s[q + 1]) ++q;
  l = q;
  blk = c.lev[q].blist[bi - r.s[q]];
}

__device__ __forceinline__ long long total_elems_r(const BlockRanges& r, int l0, int l1, int D) {
  return (long long)(r.s[l1] - r.s[l0]) << (2 * D);
}

__device__ __forceinline__ long long total_elems(const Ctx& c, int l0, int l1, int D) {
  long long t = 0;
  for (int q = l0; q < l1; ++q) t += c.ctr[CTR_LEVEL + q];
  return t << (2 * D);
}

// ---------------------------------------------------------------------------
// small dense linear algebra (row-major)
template <int D>
__host__ __device__ __forceinline__ float det(const float* F) {
  if (D == 2) return F[0] * F[3] - F[1] * F[2];
  return F[0] * (F[4] * F[8] - F[5] * F[7]) - F[1] * (F[3] * F[8] - F[5] * F[6]) +
         F[2] * (F[3] * F[7] - F[4] * F[6]);
}

// 2x2: polar rotation in closed form.  R maximises tr(R^T F) over rotations,
// which is U V^T of the rotation-variant SVD used by the reference's
// get_stress (utils.py:11-16).
__host__ __device__ __forceinline__ void polar2(const float* F, float& c, float& s) {
  float a = F[0] + F[3], b = F[2] - F[1];
  float n2 = a * a + b * b;
  if (n2 > 0.f) {
    float inv = 1.0f / sqrtf(n2);
    c = a * inv;
    s = b * inv;
  } else {
    c = 1.f;
    s = 0.f;
  }
}

// 2x2 SVD with det U = det V = +1: R from polar2, then the symmetric factor
// S = R^T F is diagonalised by one exact Jacobi rotation.
__host__ __device__ __forceinline__ void svd2(const float* F, float* U, float* sig, float* V) {
  float c, s;
  polar2(F, c, s);
  // S = R^T F
  float s00 = c * F[0] + s * F[2], s01 = c * F[1] + s * F[3];
  float s11 = -s * F[1] + c * F[3];
  float cv = 1.f, sv = 0.f;
  if (s01 != 0.f) {
    float tau = (s11 - s00) / (2.f * s01);
    float t = copysignf(1.f, tau) / (fabsf(tau) + sqrtf(1.f + tau * tau));
    cv = 1.f / sqrtf(1.f + t * t);
    sv = t * cv;
  }
  // eigenvalues: Q^T S Q with Q = [[cv, sv], [-sv, cv]]
  float e0 = cv * cv * s00 - 2.f * cv * sv * s01 + sv * sv * s11;
  float e1 = sv * sv * s00 + 2.f * cv * sv * s01 + cv * cv * s11;
  float V00 = cv, V01 = sv, V10 = -sv, V11 = cv;
  if (fabsf(e1) > fabsf(e0)) {  // sort descending, keep det V = +1
    float t = e0; e0 = e1; e1 = t;
    float a0 = V00, a1 = V10;
    V00 = V01; V10 = V11;
    V01 = -a0; V11 = -a1;
  }
  sig[0] = e0; sig[1] = e1;
  V[0] = V00; V[1] = V01; V[2] = V10; V[3] = V11;
  // U = R V
  U[0] = c * V00 - s * V10; U[1] = c * V01 - s * V11;
  U[2] = s * V00 + c * V10; U[3] = s * V01 + c * V11;
}

// 3x3 SVD, A = U diag(sig) V^T with det U = det V = +1 (rotation-variant).
// Method: cyclic Jacobi eigenanalysis of A^T A with exact rotations (Golub &
// Van Loan, Matrix Computations, 4th ed., Alg. 8.5.3), columns of B = A V
// sorted by norm, then a Givens QR of B gives U and sig (the approach of
// McAdams et al. 2011, "Computing the SVD of 3x3 matrices with minimal
// branching and elementary floating point operations", with exact instead of
// approximate Givens angles).
__host__ __device__ __forceinline__ void jacobi_rot(float* S, float* V, int p, int q) {
  // symmetric S (row-major 3x3), zero S[p][q]
  float apq = S[p * 3 + q];
  if (apq == 0.f) return;
  float app = S[p * 3 + p], aqq = S[q * 3 + q];
  float tau = (aqq - app) / (2.f * apq);
  float t = copysignf(1.f, tau) / (fabsf(tau) + sqrtf(1.f + tau * tau));
  float c = 1.f / sqrtf(1.f + t * t), s = t * c;
  // S <- J^T S J, J = rotation in (p,q) with J[p][p]=c, J[p][q]=s, J[q][p]=-s, J[q][q]=c
#pragma unroll
  for (int k = 0; k < 3; ++k) {  // columns
    float skp = S[k * 3 + p], skq = S[k * 3 + q];
    S[k * 3 + p] = c * skp - s * skq;
    S[k * 3 + q] = s * skp + c * skq;
  }
#pragma unroll
  for (int k = 0; k < 3; ++k) {  // rows
    float spk = S[p * 3 + k], sqk = S[q * 3 + k];
    S[p * 3 + k] = c * spk - s * sqk;
    S[q * 3 + k] = s * spk + c * sqk;
  }
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    float vkp = V[k * 3 + p], vkq = V[k * 3 + q];
    V[k * 3 + p] = c * vkp - s * vkq;
    V[k * 3 + q] = s * vkp + c * vkq;
  }
}

__host__ __device__ __forceinline__ void givens_qr(float* B, float* U, int i, int j) {
  // zero B[i][j] (i > j) using rows j and i; U <- U G^T
  float a = B[j * 3 + j], b = B[i * 3 + j];
  float r2 = a * a + b * b;
  float c = 1.f, s = 0.f;
  if (r2 > 0.f) {
    float inv = 1.0f / sqrtf(r2);
    c = a * inv;
    s = b * inv;
  }
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    float bj = B[j * 3 + k], bi = B[i * 3 + k];
    B[j * 3 + k] = c * bj + s * bi;
    B[i * 3 + k] = -s * bj + c * bi;
  }
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    float uj = U[k * 3 + j], ui = U[k * 3 + i];
    U[k * 3 + j] = c * uj + s * ui;
    U[k * 3 + i] = -s * uj + c * ui;
  }
}

__host__ __device__ __forceinline__ void svd3(const float* A, float* U, float* sig, float* V) {
  float S[9];
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      float a = 0.f;
#pragma unroll
      for (int k = 0; k < 3; ++k) a += A[k * 3 + i] * A[k * 3 + j];
      S[i * 3 + j] = a;
    }
#pragma unroll
  for (int i = 0; i < 9; ++i) V[i] = (i % 4 == 0) ? 1.f : 0.f;
#pragma unroll 1
  for (int sweep = 0; sweep < 5; ++sweep) {
    float off = fabsf(S[1]) + fabsf(S[2]) + fabsf(S[5]);
    float dg = fabsf(S[0]) + fabsf(S[4]) + fabsf(S[8]);
    if (off <= 1e-9f * dg) break;
    jacobi_rot(S, V, 0, 1);
    jacobi_rot(S, V, 0, 2);
    jacobi_rot(S, V, 1, 2);
  }
  // B = A V
  float B[9];
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      float a = 0.f;
#pragma unroll
      for (int k = 0; k < 3; ++k) a += A[i * 3 + k] * V[k * 3 + j];
      B[i * 3 + j] = a;
    }
  // sort columns by norm, descending; each swap negates one column to keep det V = +1
  auto cn = [&](int j) { return B[j] * B[j] + B[3 + j] * B[3 + j] + B[6 + j] * B[6 + j]; };
  auto swapc = [&](int a, int b) {
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      float t = B[k * 3 + a]; B[k * 3 + a] = B[k * 3 + b]; B[k * 3 + b] = -t;
      t = V[k * 3 + a]; V[k * 3 + a] = V[k * 3 + b]; V[k * 3 + b] = -t;
    }
  };
  float n0 = cn(0), n1 = cn(1), n2 = cn(2);
  if (n0 < n1) { swapc(0, 1); float t = n0; n0 = n1; n1 = t; }
  if (n0 < n2) { swapc(0, 2); float t = n0; n0 = n2; n2 = t; }
  if (n1 < n2) { swapc(1, 2); }
  // QR by Givens: B = U R
#pragma unroll
  for (int i = 0; i < 9; ++i) U[i] = (i % 4 == 0) ? 1.f : 0.f;
  givens_qr(B, U, 1, 0);
  givens_qr(B, U, 2, 0);
  givens_qr(B, U, 2, 1);
  sig[0] = B[0];
  sig[1] = B[4];
  sig[2] = B[8];
  // det U = +1 by construction; make sig[0], sig[1] non-negative by flipping
  // column pairs of U and V together (keeps both determinants).
  if (sig[0] < 0.f) {
    sig[0] = -sig[0]; sig[2] = -sig[2];
#pragma unroll
    for (int k = 0; k < 3; ++k) { U[k * 3 + 0] = -U[k * 3 + 0]; U[k * 3 + 2] = -U[k * 3 + 2]; }
  }
  if (sig[1] < 0.f) {
    sig[1] = -sig[1]; sig[2] = -sig[2];
#pragma unroll
    for (int k = 0; k < 3; ++k) { U[k * 3 + 1] = -U[k * 3 + 1]; U[k * 3 + 2] = -U[k * 3 + 2]; }
  }
}

// Polar rotation of a 3x3 F with det F > 0 by the scaled Newton iteration
// X <- (g X + X^{-T} / g) / 2 (Higham, "Computing the polar decomposition
// with applications", SIAM J. Sci. Stat. Comput. 7, 1986), with the
// Frobenius-norm scaling g = (|X^{-1}| / |X|)^(1/2) in the first iterations.
// For det F > 0 the limit is U V^T of the SVD.  Returns false (R undefined)
// when det X <= 0 is met or the iteration has not settled after 12 steps.
__host__ __device__ __forceinline__ bool polar_newton3(const float* F, float* R) {
  float X[9];
#pragma unroll
  for (int i = 0; i < 9; ++i) X[i] = F[i];
#pragma unroll 1
  for (int it = 0; it < 12; ++it) {
    float Y[9];
    Y[0] = X[4] * X[8] - X[5] * X[7];
    Y[1] = X[5] * X[6] - X[3] * X[8];
    Y[2] = X[3] * X[7] - X[4] * X[6];
    Y[3] = X[2] * X[7] - X[1] * X[8];
    Y[4] = X[0] * X[8] - X[2] * X[6];
    Y[5] = X[1] * X[6] - X[0] * X[7];
    Y[6] = X[1] * X[5] - X[2] * X[4];
    Y[7] = X[2] * X[3] - X[0] * X[5];
    Y[8] = X[0] * X[4] - X[1] * X[3];
    const float dt = X[0] * Y[0] + X[1] * Y[1] + X[2] * Y[2];
    if (!(dt > 1e-20f)) return false;
    const float id = 1.0f / dt;  // Y = cofactor(X) / det X = X^{-T}
#pragma unroll
    for (int i = 0; i < 9; ++i) Y[i] *= id;
    float g = 1.f, gi = 1.f;
    if (it < 3) {
      float nx = 0.f, ny = 0.f;
#pragma unroll
      for (int i = 0; i < 9; ++i) {
        nx += X[i] * X[i];
        ny += Y[i] * Y[i];
      }
      g = sqrtf(sqrtf(ny / nx));
      gi = 1.0f / g;
    }
    float diff = 0.f;
#pragma unroll
    for (int i = 0; i < 9; ++i) {
      const float xn = 0.5f * (g * X[i] + gi * Y[i]);
      diff = fmaxf(diff, fabsf(xn - X[i]));
      X[i] = xn;
    }
    if (diff <= 1e-6f) {
#pragma unroll
      for (int i = 0; i < 9; ++i) R[i] = X[i];
      return true;
    }
  }
  return false;
}

// R = U V^T of the rotation-variant SVD
template <int D>
__host__ __device__ __forceinline__ void polar_rot(const float* F, float* R) {
  if (D == 2) {
    float c, s;
    polar2(F, c, s);
    R[0] = c; R[1] = -s; R[2] = s; R[3] = c;
  } else {
    if (polar_newton3(F, R)) return;
    float U[9], sg[3], V[9];
    svd3(F, U, sg, V);
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) R[i * 3 + j] = U[i * 3] * V[j * 3] + U[i * 3 + 1] * V[j * 3 + 1] + U[i * 3 + 2] * V[j * 3 + 2];
  }
}

// Fixed-corotated Kirchhoff stress (utils.py:11-16) as a symmetric matrix:
//   tau = 2 mu (F - R) F^T + la J (J - 1) I,  R = U V^T,
// passed as tmu = 2 mu and diag = la J (J - 1).  tau is symmetric, and its
// entries are written in the order xx, xy, yy (2D) / xx, xy, yy, xz, yz, zz (3D).
//
// 3D near rotations (det F > 0, |F F^T - I|_F < 0.1, which holds in the snow
// range, singular values within a few percent of 1): with the left polar
// decomposition F = P R, R F^T = P = (F F^T)^(1/2), so
//   (F - R) F^T = F F^T - (F F^T)^(1/2) = (I + E) - (I + E)^(1/2),  E = F F^T - I,
// a power series in E: E/2 + E^2/8 - E^3/16 + 5 E^4/128 - 7 E^5/256 + ...
// (the binomial series of the matrix square root, Higham, "Functions of
// Matrices", SIAM 2008, ch. 6), summed by Horner's rule to the E^5 term: the
// first omitted term, 21 E^6 / 1024, is below 2.1e-8 for |E| < 0.1.  Every
// product is a polynomial in E (symmetric, commuting), so each needs only its
// 6 upper entries.  Elsewhere (inverted or strongly stretched F) R comes from
// polar_rot.  In 2D the closed-form polar rotation is cheap and used always.
template <int D>
__host__ __device__ __forceinline__ void kirchhoff_sym(const float* F, float tmu, float diag, float* tau) {
  if (D == 2) {
    float R[4];
    polar_rot<2>(F, R);
    float t[4];
#pragma unroll
    for (int r = 0; r < 2; ++r)
#pragma unroll
      for (int b = 0; b < 2; ++b) {
        float acc = 0.f;
#pragma unroll
        for (int k = 0; k < 2; ++k) acc += (tmu * (F[r * 2 + k] - R[r * 2 + k])) * F[b * 2 + k];
        t[r * 2 + b] = acc;
      }
    tau[0] = t[0] + diag;
    tau[1] = 0.5f * (t[1] + t[2]);
    tau[2] = t[3] + diag;
    return;
  }
  // E = F F^T - I, upper entries (xx, xy, yy, xz, yz, zz)
  float e[6];
  e[0] = fmaf(F[0], F[0], fmaf(F[1], F[1], F[2] * F[2])) - 1.f;
  e[1] = fmaf(F[0], F[3], fmaf(F[1], F[4], F[2] * F[5]));
  e[2] = fmaf(F[3], F[3], fmaf(F[4], F[4], F[5] * F[5])) - 1.f;
  e[3] = fmaf(F[0], F[6], fmaf(F[1], F[7], F[2] * F[8]));
  e[4] = fmaf(F[3], F[6], fmaf(F[4], F[7], F[5] * F[8]));
  e[5] = fmaf(F[6], F[6], fmaf(F[7], F[7], F[8] * F[8])) - 1.f;
  const float fro2 = e[0] * e[0] + e[2] * e[2] + e[5] * e[5] + 2.f * (e[1] * e[1] + e[3] * e[3] + e[4] * e[4]);
  if (fro2 < 0.01f && det<3>(F) > 0.f) {
    // T <- c I + E T, starting from T = c4 I + c5 E
    float t[6];
    const float c5 = -7.f / 256.f, c4 = 5.f / 128.f, c3 = -1.f / 16.f, c2 = 1.f / 8.f, c1 = 0.5f;
#pragma unroll
    for (int i = 0; i < 6; ++i) t[i] = c5 * e[i];
    t[0] += c4;
    t[2] += c4;
    t[5] += c4;
    auto sym_mul = [](const float* a, const float* b, float* o) {
      // o = a b for symmetric commuting a, b (upper entries)
      o[0] = fmaf(a[0], b[0], fmaf(a[1], b[1], a[3] * b[3]));
      o[1] = fmaf(a[0], b[1], fmaf(a[1], b[2], a[3] * b[4]));
      o[2] = fmaf(a[1], b[1], fmaf(a[2], b[2], a[4] * b[4]));
      o[3] = fmaf(a[0], b[3], fmaf(a[1], b[4], a[3] * b[5]));
      o[4] = fmaf(a[1], b[3], fmaf(a[2], b[4], a[4] * b[5]));
      o[5] = fmaf(a[3], b[3], fmaf(a[4], b[4], a[5] * b[5]));
    };
    const float cs[3] = {c3, c2, c1};
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      float o[6];
      sym_mul(e, t, o);
#pragma unroll
      for (int i = 0; i < 6; ++i) t[i] = o[i];
      t[0] += cs[k];
      t[2] += cs[k];
      t[5] += cs[k];
    }
    float x[6];
    sym_mul(e, t, x);
#pragma unroll
    for (int i = 0; i < 6; ++i) tau[i] = tmu * x[i];
  } else {
    float R[9];
    polar_rot<3>(F, R);
    float t[9];
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
      for (int b = 0; b < 3; ++b) {
        float acc = 0.f;
#pragma unroll
        for (int k = 0; k < 3; ++k) acc += (tmu * (F[r * 3 + k] - R[r * 3 + k])) * F[b * 3 + k];
        t[r * 3 + b] = acc;
      }
    tau[0] = t[0];
    tau[1] = 0.5f * (t[1] + t[3]);
    tau[2] = t[4];
    tau[3] = 0.5f * (t[2] + t[6]);
    tau[4] = 0.5f * (t[5] + t[7]);
    tau[5] = t[8];
  }
  tau[0] += diag;
  tau[2] += diag;
  tau[5] += diag;
}

// True when every singular value of F provably lies in [lo, hi] and det F > 0
// (Gershgorin discs of F^T F inside [lo^2, hi^2]): a clamp of the singular
// values to [lo, hi] then leaves F unchanged.
template <int D>
__host__ __device__ __forceinline__ bool singular_values_within(const float* F, float lo, float hi) {
  if (!(det<D>(F) > 0.f)) return false;
  float S[D * D];
#pragma unroll
  for (int i = 0; i < D; ++i)
#pragma unroll
    for (int j = 0; j < D; ++j) {
      float a = 0.f;
#pragma unroll
      for (int k = 0; k < D; ++k) a += F[k * D + i] * F[k * D + j];
      S[i * D + j] = a;
    }
  const float lo2 = lo * lo, hi2 = hi * hi;
#pragma unroll
  for (int i = 0; i < D; ++i) {
    float r = 0.f;
#pragma unroll
    for (int j = 0; j < D; ++j)
      if (j != i) r += fabsf(S[i * D + j]);
    if (S[i * D + i] - r < lo2 || S[i * D + i] + r > hi2) return false;
  }
  return true;
}

// singular_values_within for a matrix given by its Gram matrix S = F^T F
// (upper entries, row by row: 2D s00 s01 s11, 3D s00 s01 s02 s11 s12 s22) and
// its determinant: the same Gershgorin test.
template <int D>
__host__ __device__ __forceinline__ bool gram_within(const float* S, float detF, float lo, float hi) {
  if (!(detF > 0.f)) return false;
  const float lo2 = lo * lo, hi2 = hi * hi;
  if (D == 2) {
    const float r = fabsf(S[1]);
    return S[0] - r >= lo2 && S[0] + r <= hi2 && S[2] - r >= lo2 && S[2] + r <= hi2;
  }
  const float r0 = fabsf(S[1]) + fabsf(S[2]), r1 = fabsf(S[1]) + fabsf(S[4]), r2 = fabsf(S[2]) + fabsf(S[4]);
  return S[0] - r0 >= lo2 && S[0] + r0 <= hi2 && S[3] - r1 >= lo2 && S[3] + r1 <= hi2 && S[5] - r2 >= lo2 &&
         S[5] + r2 <= hi2;
}

// GIMP weights factorised per axis.  get_weight_stencil (adaptive_gimp.py:
// 218-228) sums get_linear_weight (utils.py:18-42) over the 2^d cells dI and
// 2^d corners cell_ that meet at node n = dI + cell_; the summand is a product
// over axes, so the sum is the product of per-axis sums:
//   w[n] = prod_d W_d[n_d] / (2^d (2r)^d),
//   dw[n]_a = G_a[n_a] prod_{d!=a} W_d[n_d] / (2^(d-1) (2r)^d).
__host__ __device__ __forceinline__ void axis_weights(float t, float r, float* W, float* G) {
  // dI = 0: interval around t + 1; dI = 1: around t
  const float bmin0 = fminf(fmaxf(t + 1.f - r, 0.f), 1.f), bmax0 = fminf(fmaxf(t + 1.f + r, 0.f), 1.f);
  const float bmin1 = fminf(fmaxf(t - r, 0.f), 1.f), bmax1 = fminf(fmaxf(t + r, 0.f), 1.f);
  // corner cell_ = 0: mx = 1 - bmin, mn = 1 - bmax; cell_ = 1: mx = bmax, mn = bmin
  const float a0 = 1.f - bmin0, b0 = 1.f - bmax0;
  const float a1 = 1.f - bmin1, b1 = 1.f - bmax1;
  const float w00 = a0 * a0 - b0 * b0, g00 = b0 - a0;                 // dI 0, cell 0 -> node 0
  const float w01 = bmax0 * bmax0 - bmin0 * bmin0, g01 = bmax0 - bmin0; // dI 0, cell 1 -> node 1
  const float w10 = a1 * a1 - b1 * b1, g10 = b1 - a1;                 // dI 1, cell 0 -> node 1
  const float w11 = bmax1 * bmax1 - bmin1 * bmin1, g11 = bmax1 - bmin1; // dI 1, cell 1 -> node 2
  W[0] = w00;
  W[1] = w01 + w10;
  W[2] = w11;
  G[0] = g00;
  G[1] = g01 + g10;
  G[2] = g11;
}

// axis_weights for the reference's radius r = 0.5 (adaptive_gimp.py:48) and
// t in [-0.5, 0.5] (every in-domain particle): none of the clamps binds, and
// the per-axis sums reduce to W = ((1/2 - t)^2, 3/2 - 2 t^2, (1/2 + t)^2),
// G = (t - 1/2, -2 t, t + 1/2).
__host__ __device__ __forceinline__ void axis_weights_half(float t, float* W, float* G) {
  const float a = 0.5f - t, b = 0.5f + t;
  W[0] = a * a;
  W[1] = fmaf(-2.f * t, t, 1.5f);
  W[2] = b * b;
  G[0] = -a;
  G[1] = -2.f * t;
  G[2] = b;
}

// ---------------------------------------------------------------------------
// Batches.  One launch per kernel serves every scene of a batch (a single
// simulator is a batch of one).  For each kind of launch the CTAs are cut into
// consecutive ranges, one per scene; a CTA finds its scene by binary search
// over the range starts and copies the scene's context into shared memory.
enum { MAP_G = 0,  // grid-stride kernels over particles, active blocks or work items
       MAP_O = 1,  // bin allocation (1024-thread CTAs)
       MAP_T = 2,  // staged level transfers (one 4^d block per CTA at a time: 4x MAP_G's CTAs)
       MAP_P = 3,  // P2G: whole waves of the CTAs that fit an SM at once
       NMAP = 4 };

struct Batch {
  const Ctx* ctx;  // [n] scene contexts in device memory
  const int* ofs;  // [NMAP][n + 1] first CTA of each scene, per launch kind
  int n;
};

// What the host needs to launch a batch's substep.
struct BatchLaunch {
  Batch b;
  int dim;
  int sms;           // multiprocessors of the device
  int maxL;          // most levels of any scene (per-level launches run to it)
  int nct[NMAP];     // CTAs of each launch kind
  int chunk;         // P2G work-item size of every scene
  int any_dynamic;   // some scene activates cells from g_p (runs k_mark_hier)
  int any_plastic;   // some scene has snow plasticity (runs k_project)
  const Ctx* single; // host context of a single simulator, else null
  // surrogate return map of the substep (sur != 0): the MLP runs over the
  // *sur_n slots of sur_X / sur_Y, then k_sur_finish applies them
  int sur;
  const void* mlp_packed;
  const float* mlp_P;
  const float* sur_X;
  float* sur_Y;
  const float* sur_meta;
  const int32_t* sur_n;
  long long sur_cap;
  int32_t* sur_err;
  // second stream of the substep (null: everything on the caller's stream):
  // k_ghost_tj runs on it beside the binning kernels and P2G, which read no
  // node mask and only the exact-ACTIVATED cell tests that k_ghost_tj leaves
  // unchanged; the restriction waits for it
  cudaStream_t side;
  cudaEvent_t fork, join;
  // programmatic dependent launches between consecutive substep kernels on
  // one stream (launch_k); off for phase timing
  bool pdl;
};

// The calling CTA's scene: its context (copied to *sc), its rank among the
// scene's CTAs and their number.  Every thread of the CTA must call it.
template <int KIND>
__device__ __forceinline__ const Ctx& scene_slice(const Batch& B, Ctx* sc, int& bid, int& nblk) {
  const int* o = B.ofs + KIND * (B.n + 1);
  const int cta = (int)blockIdx.x;
  int lo = 0, hi = B.n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (__ldg(&o[mid]) <= cta)
      lo = mid;
    else
      hi = mid - 1;
  }
  bid = cta - __ldg(&o[lo]);
  nblk = __ldg(&o[lo + 1]) - __ldg(&o[lo]);
  const unsigned* src = (const unsigned*)(B.ctx + lo);
  unsigned* dst = (unsigned*)sc;
  for (int i = threadIdx.x; i < (int)(sizeof(Ctx) / 4); i += blockDim.x) dst[i] = __ldg(&src[i]);
  __syncthreads();
  // The next kernel on the stream (a programmatic dependent, launch_k with
  // pdl) may be scheduled once every CTA of this one has started: its CTAs
  // fill the SM slots this kernel's last wave leaves free and run their own
  // prologue, then wait below for this kernel to complete.
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  // Launched as a programmatic dependent of the previous kernel on the stream
  // (launch_k with pdl), the CTA may have started before that kernel finished:
  // everything above reads only host-written launch data; wait here until the
  // previous kernel has completed and its writes are visible.  Without the
  // launch attribute this returns at once.
  asm volatile("griddepcontrol.wait;" ::: "memory");
  return *sc;
}

// Kernel prologue: binds `c` (this CTA's scene), `bid_` and `nblk_`.
#define SCENE_CTA(B, KIND)  \
  __shared__ Ctx s_ctx_;    \
  int bid_, nblk_;          \
  const Ctx& c = scene_slice<KIND>(B, &s_ctx_, bid_, nblk_)

// grid-stride loop over [0, n) across the CTAs of this CTA's scene
#define SCENE_LOOP(i, n) \
  for (long long i = bid_ * (long long)blockDim.x + threadIdx.x; i < (n); i += (long long)nblk_ * blockDim.x)

// the same over the scene's particle slots, with a trip count uniform across
// the CTA (for warp-collective bodies): p = p0 + threadIdx.x may be >= c.N
#define SCENE_PARTICLES(p0) \
  for (int p0 = bid_ * (int)blockDim.x; p0 < c.N; p0 += nblk_ * (int)blockDim.x)

// Launch kernel k on stream s; with pdl as a programmatic dependent launch:
// the launch may begin while the previous kernel on s is still finishing, so
// launch latency and each CTA's prologue (scene lookup and context copy in
// scene_slice) overlap that kernel's tail.  Every kernel launched this way
// starts with SCENE_CTA, which waits for the previous kernel before touching
// its results.
template <typename... P, typename... A>
inline cudaError_t launch_k(bool pdl, void (*k)(P...), int grid, int block, size_t smem, cudaStream_t s, A... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)grid);
  cfg.blockDim = dim3((unsigned)block);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = pdl ? 1 : 0;
  return cudaLaunchKernelEx(&cfg, k, args...);
}

// ---------------------------------------------------------------------------
// host-side launchers (defined in topology.cu / transfer.cu)
// ev (optional): PHASES+1 events recorded at the phase boundaries
constexpr int PHASES = 8;  // blocks, topology, binning, p2g, restrict, gridop, prolong, g2p
void launch_substep(const BatchLaunch& bl, cudaStream_t s, cudaEvent_t* ev = nullptr);
void launch_refine(const Ctx& c, int band, cudaStream_t s);
void prepare_transfer_kernels();  // kernel attributes (shared-memory opt-in); once per device
int p2g_resident(int dim, int chunk);  // k_p2g CTAs an SM holds at once
// surrogate MLP forward over a device-side sample count (mlp.cu)
void launch_mlp_forward_dev(const void* packed, const float* P, const float* X, float* Y, const int32_t* n_dev,
                            long long cap, int32_t* err, int sms, cudaStream_t s);
int kernels_per_substep(const BatchLaunch& bl);

}  // namespace agimp

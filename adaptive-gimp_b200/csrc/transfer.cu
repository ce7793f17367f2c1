// Particle/grid transfer kernels of the adaptive GIMP substep.
//
// Reference steps (adaptive_gimp.py, g1n0st/adaptive-gimp):
//   230-250 p2g               -> k_p2g      (all levels in one launch)
//   289-301 grid_restriction  -> k_restrict (one launch per level, fine->coarse)
//   277-287 grid_op           -> level 0 in the last k_restrict, level l in
//                                k_prolong(l); k_gridop (all levels) only
//                                when every scene has one level
//   303-321 grid_prolongation -> k_prolong  (one launch per level, coarse->fine)
//   252-275 g2p               -> k_g2p      (all levels in one launch)
//
// P2G: one CTA per work item = up to CH particles of one bin (one 4^d block of
// one level).  A bin's particles touch only the (4+2)^d nodes from the block
// origin, so P2G accumulates into that tile in shared memory and flushes it
// with one float4 atomic per touched node.  G2P: one thread per particle slot
// in bin order; neighbouring threads gather the same nodes through L1.
//
// Every kernel serves a batch of scenes (a single simulator is a batch of
// one): each CTA works for the scene its launch range assigns it to.
//
// Restriction and prolongation are written as gathers (each destination node
// sums its sources) instead of the reference's scatters, so they need no
// atomics; the set of terms and their weights are the reference's.
#include "common.cuh"
#include "umma.cuh"

namespace agimp {

// first stored cell of block `blk` (block indices are 32-bit: 32-bit division)
template <int D>
__device__ __forceinline__ void chunk_origin(const LevelDev& V, long long blk, int* O) {
  unsigned b = (unsigned)blk;
  const unsigned nb = (unsigned)V.nb;
#pragma unroll
  for (int d = D - 1; d >= 0; --d) {
    O[d] = (int)(b % nb) * 4 - HALO;
    b /= nb;
  }
}

// ---------------------------------------------------------------------------
// Packed f32x2 arithmetic (sm_100 fma/mul/add .f32x2): each half is rounded
// exactly like the scalar fmaf / multiply / add, at one instruction per pair.
__device__ __forceinline__ unsigned long long pk2(float2 a) {
  unsigned long long r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a.x), "f"(a.y));
  return r;
}
__device__ __forceinline__ float2 upk2(unsigned long long r) {
  float2 a;
  asm("mov.b64 {%0, %1}, %2;" : "=f"(a.x), "=f"(a.y) : "l"(r));
  return a;
}
__device__ __forceinline__ float2 ffma2(float2 a, float2 b, float2 c) {
  unsigned long long d;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(pk2(a)), "l"(pk2(b)), "l"(pk2(c)));
  return upk2(d);
}
__device__ __forceinline__ float2 fmul2(float2 a, float2 b) {
  unsigned long long d;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(pk2(a)), "l"(pk2(b)));
  return upk2(d);
}
__device__ __forceinline__ float2 fadd2(float2 a, float2 b) {
  unsigned long long d;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(pk2(a)), "l"(pk2(b)));
  return upk2(d);
}
__device__ __forceinline__ float2 dup2(float a) { return make_float2(a, a); }

// ---------------------------------------------------------------------------
// P2G (adaptive_gimp.py:230-250).  Per work item (up to CH particles of one
// 4^d block of one level, in base-cell order: bins store their particles
// sorted by cell, the last axis fastest):
//  1. one thread per particle computes the scaled Kirchhoff stress S
//     (utils.py:11-16, adaptive_gimp.py:240; symmetric, kirchhoff_sym), its
//     per-axis GIMP weights and gradients, m, a = m (v - C (tc+1)) and
//     B = m C, and its base cell inside the block, forms each node row's
//     share A of the momentum term (below) and stores the record in shared
//     memory at its thread index;
//  2. each warp cuts its own 32 particles into ranges: in 3D SLOTS = 3
//     contiguous ranges of equal length (11/11/10), which keeps every slot
//     busy for the same number of steps; in 2D runs of one base cell (about 4
//     particles), 10 at a time.  A lane owns one row of three
//     stencil nodes (the last axis runs along the row; 3^(d-1) rows per cell)
//     of one range and walks its particles, reading its row's float4 and the
//     record's shared part (3D 18 floats, 2D 16, of 52 / 28).  It sums the
//     three nodes' w m and w (a + B n) + S grad w in registers; when the base
//     cell moves one or two cells along the row, the nodes left behind go to
//     the (4+2)^d node tile in shared memory and the others move down the
//     row; any other change, and the end, sends all three;
//  3. a CTA takes a contiguous range of work items, so consecutive items of
//     one block (a dense block holds many) keep summing into the same tile;
//     when the next item is another block, the tile is flushed after one
//     barrier with one float4 atomic per touched node and cleared.  Two tiles
//     alternate between blocks, so the next block's records and sums need no
//     further barrier.
template <int D, int CH>
struct P2GLayout {
  static constexpr int ROWS = (D == 2) ? 3 : 9;   // node rows per stencil
  static constexpr int SLOTS = 32 / ROWS;         // particle ranges served by one warp at once
  static constexpr int TN = (D == 2) ? 36 : 216;  // nodes of the (4+2)^d tile
  // per-particle record (floats): one float4 per node row (a lane reads only
  // its own row and the part every row shares):
  //  3D  4 r: A_x A_y A_z cw of row r = 3 n0 + n1 (r < 9) | 36 Bk_x Bk_y Bk_z m |
  //     40 SL_x SL_y SL_z cell | 44 W2[0..2] G2[0] | 48 G2[1] G2[2] - -
  //  2D  4 r: A_x A_y cw cell of row r = n0 (r < 3) | 12 Bk_x Bk_y SL_x SL_y |
  //     16 W1[0..2] m | 20 G1[0..2] - | 24 - - - -
  // Strides are odd multiples of four floats: the float4 stores of eight
  // consecutive threads (one shared-memory wavefront) fall in distinct banks.
  static constexpr int STRIDE = (D == 3) ? 52 : 28;
  static constexpr int TMAX = 16;  // 2D: longest run of one base cell walked by one slot
  static constexpr size_t bytes() {
    return sizeof(float) * ((size_t)CH * STRIDE + 2 * 4 * TN) + sizeof(int) * (CH / 32) * 33;
  }
};

// Node k of a lane's row of base cell cc sits at tile index row_tile + k.
template <int D>
__device__ __forceinline__ int p2g_row_tile(int cc, int n0, int n1) {
  if (D == 2) return (((cc >> 2) & 3) + n0) * 6 + (cc & 3);
  return ((((cc >> 4) & 3) + n0) * 6 + ((cc >> 2) & 3) + n1) * 6 + (cc & 3);
}

// One node's sums into the node tile ([4][TN]: p_x, p_y, p_z, m).
template <int D>
__device__ __forceinline__ void p2g_node_flush(float* tile, int TN, int ti, float2 axy, float az, float am) {
  atomicAdd(&tile[ti], axy.x);
  atomicAdd(&tile[TN + ti], axy.y);
  if (D == 3) atomicAdd(&tile[2 * TN + ti], az);
  atomicAdd(&tile[3 * TN + ti], am);
}

// A lane's three node sums of one base cell into the node tile.
template <int D>
__device__ __forceinline__ void p2g_row_flush(float* tile, int TN, int cc, int n0, int n1, const float2* axy,
                                              const float* az, const float* am) {
  const int ti = p2g_row_tile<D>(cc, n0, n1);
#pragma unroll
  for (int k = 0; k < 3; ++k) p2g_node_flush<D>(tile, TN, ti + k, axy[k], az[k], am[k]);
}

template <int D, int CH>
__global__ void __launch_bounds__(CH, 1024 / CH) k_p2g(Batch B) {
  SCENE_CTA(B, MAP_P);
  using Y = P2GLayout<D, CH>;
  extern __shared__ float4 dsm4[];
  float* pd = (float*)dsm4;             // [CH][STRIDE]
  float* tiles = pd + CH * Y::STRIDE;   // [2][4][TN]: p_x, p_y, p_z, m
  int* starts = (int*)(tiles + 2 * 4 * Y::TN);  // 2D: [warps][33] run starts
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nch = c.ctr[CTR_CHUNKS];
  const float pw = (D == 2) ? 0.25f : 0.125f;                                        // 0.5**dim
  const float rd = (D == 2) ? c.radius * c.radius : c.radius * c.radius * c.radius;  // radius**dim
  const float r2 = 2.f * c.radius;
  const float kw = (D == 2) ? 1.f / (4.f * r2 * r2) : 1.f / (8.f * r2 * r2 * r2);
  const bool half = c.radius == 0.5f;
  // the tiles start at zero; each flush leaves its tile at zero again
  for (int i = threadIdx.x; i < 2 * 4 * Y::TN; i += blockDim.x) tiles[i] = 0.f;
  __syncthreads();
  int tb = 0;
  const int per = (nch + nblk_ - 1) / nblk_;
  const int c0 = bid_ * per, c1 = min(nch, c0 + per);
  // this lane's slot and node row
  const int q = lane / Y::ROWS, row = lane % Y::ROWS;
  const int n0 = (D == 2) ? row : row / 3, n1 = (D == 2) ? 0 : row % 3;
  for (int ch = c0; ch < c1; ++ch) {
    const int4 wd = c.chunks[ch];
    const int l = wd.x;
    if (l < 0) continue;  // particles without a level: no transfer (uniform over the CTA)
    // the tile is flushed when the next work item of this CTA is another block
    bool last = ch + 1 == c1;
    if (!last) {
      const int4 nx = c.chunks[ch + 1];
      last = nx.x != wd.x || nx.y != wd.y;
    }
    const LevelDev& V = c.lev[l];
    int O[D];
    chunk_origin<D>(V, wd.y, O);
    float* tile = tiles + tb * 4 * Y::TN;
    // -- 1. per-particle records -----------------------------------------------
    const int i = threadIdx.x;
    int cell = -1;
    if (i < wd.w) {
      const int p = __ldg(&c.perm[wd.z + i]);
      const long long N = c.N;
      const float inv = (float)(c.coarsest << l);
      const float dx = 1.f / inv;
      float xp[D], vp[D], F[D * D], Cm[D * D];
#pragma unroll
      for (int d = 0; d < D; ++d) {
        xp[d] = __ldg(&c.P.x[d * N + p]);
        vp[d] = __ldg(&c.P.v[d * N + p]);
      }
#pragma unroll
      for (int k = 0; k < D * D; ++k) {
        F[k] = __ldg(&c.P.F[k * N + p]);
        Cm[k] = __ldg(&c.P.C[k * N + p]);
      }
      const float mp = __ldg(&c.P.m[p]);
      const float jp = c.plast == 1 ? __ldg(&c.P.Jp[p]) : 1.f;
      float tc[D];
      cell = 0;
#pragma unroll
      for (int d = 0; d < D; ++d) {
        const float xs = xp[d] * inv;
        const int base = (int)(xs + 0.5f) - 1;
        tc[d] = xs - (float)(base + 1);
        cell = (cell << 2) | ((base - O[d]) & 3);
      }
      float mu = c.mu, la = c.la;
      if (c.plast == 1) {
        const float h = expf(c.xi * (1.f - jp));
        mu *= h;
        la *= h;
      }
      const float J = det<D>(F);
      float tau[(D == 2) ? 3 : 6];
      kirchhoff_sym<D>(F, 2.f * mu, la * J * (J - 1.f), tau);
      const float sc = (-c.dt * pw) / (rd * dx);
      float a[D];
#pragma unroll
      for (int r = 0; r < D; ++r) {
        float cd = 0.f;
#pragma unroll
        for (int b = 0; b < D; ++b) cd += Cm[r * D + b] * (tc[b] + 1.f);
        a[r] = mp * (vp[r] - cd);
      }
      // axis factors, scaled so that a node's weight is the product of its
      // W's and the gradient's factors need no constant: axis 0 carries kw,
      // every G carries kg / kw = 2
      float W[D][3], G[D][3];
#pragma unroll
      for (int d = 0; d < D; ++d) {
        if (half)
          axis_weights_half(tc[d], W[d], G[d]);
        else
          axis_weights(tc[d], c.radius, W[d], G[d]);
        const float sw = d == 0 ? kw : 1.f;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          W[d][k] *= sw;
          G[d][k] *= 2.f * sw;
        }
      }
      float4* P4 = (float4*)(pd + i * Y::STRIDE);
      const float cf = __int_as_float(cell);
      if (D == 3) {
        // row r = 3 n0 + n1: A = cw (a + B[:,0] n0 + B[:,1] n1) + S[:,0] cg0 + S[:,1] cg1
        // with cw = W0[n0] W1[n1], cg0 = G0[n0] W1[n1], cg1 = W0[n0] G1[n1]
        const float Bx0 = mp * Cm[0], By0 = mp * Cm[D], Bz0 = mp * Cm[(2 * D) % (D * D)];
        const float Bx1 = mp * Cm[1], By1 = mp * Cm[D + 1], Bz1 = mp * Cm[(2 * D + 1) % (D * D)];
        const float Sxx = sc * tau[0], Sxy = sc * tau[1], Syy = sc * tau[2];
        const float Sxz = sc * tau[3 % (D == 3 ? 6 : 3)], Syz = sc * tau[4 % (D == 3 ? 6 : 3)];
        const float Szz = sc * tau[5 % (D == 3 ? 6 : 3)];
#pragma unroll
        for (int r0 = 0; r0 < 3; ++r0) {
#pragma unroll
          for (int r1 = 0; r1 < 3; ++r1) {
            const float cw = W[0][r0] * W[1][r1], cg0 = G[0][r0] * W[1][r1], cg1 = W[0][r0] * G[1][r1];
            const float fn0 = (float)r0, fn1 = (float)r1;
            const float ux = fmaf(Bx1, fn1, fmaf(Bx0, fn0, a[0]));
            const float uy = fmaf(By1, fn1, fmaf(By0, fn0, a[1]));
            const float uz = fmaf(Bz1, fn1, fmaf(Bz0, fn0, a[D - 1]));
            P4[3 * r0 + r1] = make_float4(fmaf(cw, ux, fmaf(Sxx, cg0, Sxy * cg1)),
                                          fmaf(cw, uy, fmaf(Sxy, cg0, Syy * cg1)),
                                          fmaf(cw, uz, fmaf(Sxz, cg0, Syz * cg1)), cw);
          }
        }
        P4[9] = make_float4(mp * Cm[2 % (D * D)], mp * Cm[(D + 2) % (D * D)], mp * Cm[D * D - 1], mp);
        P4[10] = make_float4(Sxz, Syz, Szz, cf);
        P4[11] = make_float4(W[D - 1][0], W[D - 1][1], W[D - 1][2], G[D - 1][0]);
        *(float2*)(P4 + 12) = make_float2(G[D - 1][1], G[D - 1][2]);
      } else {
        // row r = n0: A = cw (a + B[:,0] n0) + S[:,0] cg0 with cw = W0[n0], cg0 = G0[n0]
        const float Bx0 = mp * Cm[0], By0 = mp * Cm[D];
        const float Sxx = sc * tau[0], Sxy = sc * tau[1], Syy = sc * tau[2];
#pragma unroll
        for (int r0 = 0; r0 < 3; ++r0) {
          const float cw = W[0][r0], cg0 = G[0][r0], fn0 = (float)r0;
          const float ux = fmaf(Bx0, fn0, a[0]), uy = fmaf(By0, fn0, a[1]);
          P4[r0] = make_float4(fmaf(cw, ux, Sxx * cg0), fmaf(cw, uy, Sxy * cg0), cw, cf);
        }
        P4[3] = make_float4(mp * Cm[1], mp * Cm[D + 1 < D * D ? D + 1 : 0], Sxy, Syy);
        P4[4] = make_float4(W[D - 1][0], W[D - 1][1], W[D - 1][2], mp);
        P4[5] = make_float4(G[D - 1][0], G[D - 1][1], G[D - 1][2], 0.f);
      }
    }
    __syncwarp();
    // -- 2. this warp's particles in SLOTS ranges, lane <-> node row -------------
    const int wbase = warp * 32;
    const int nvalid = max(0, min(32, wd.w - wbase));
    auto walk = [&](const int j0, const int j1) {
      float2 axy[3];
      float az[3], am[3];
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        axy[k] = make_float2(0.f, 0.f);
        az[k] = am[k] = 0.f;
      }
      int cur = -1;
#pragma unroll 2
      for (int j = j0; j < j1; ++j) {
        const float* R = pd + (wbase + j) * Y::STRIDE;
        const float4 rw = *(const float4*)(R + 4 * row);  // this row's A (and cw, 2D: and the cell)
        const float4 sl = D == 3 ? *(const float4*)(R + 40) : make_float4(0.f, 0.f, 0.f, 0.f);  // SL, cell
        const int cc = __float_as_int(D == 3 ? sl.w : rw.w);
        if (cc != cur) {
          // Cells ascend with the row axis fastest: the next cell one or two
          // steps further along the same line shares the row's last nodes,
          // so only the nodes it leaves behind go to the tile and the others
          // move down the row.
          const int dz = cc - cur;
          if (cur >= 0 && (cc >> 2) == (cur >> 2) && dz > 0 && dz < 3) {
            const int ti = p2g_row_tile<D>(cur, n0, n1);
            p2g_node_flush<D>(tile, Y::TN, ti, axy[0], az[0], am[0]);
            if (dz == 2) p2g_node_flush<D>(tile, Y::TN, ti + 1, axy[1], az[1], am[1]);
            const float2 zz = make_float2(0.f, 0.f);
            axy[0] = dz == 1 ? axy[1] : axy[2];
            az[0] = dz == 1 ? az[1] : az[2];
            am[0] = dz == 1 ? am[1] : am[2];
            axy[1] = dz == 1 ? axy[2] : zz;
            az[1] = dz == 1 ? az[2] : 0.f;
            am[1] = dz == 1 ? am[2] : 0.f;
            axy[2] = zz;
            az[2] = am[2] = 0.f;
          } else {
            if (cur >= 0) p2g_row_flush<D>(tile, Y::TN, cur, n0, n1, axy, az, am);
#pragma unroll
            for (int k = 0; k < 3; ++k) {
              axy[k] = make_float2(0.f, 0.f);
              az[k] = am[k] = 0.f;
            }
          }
          cur = cc;
        }
        // Node k of the row has weight cw wL[k] and gradient
        // (cg_0 wL[k], .., cg_{d-2} wL[k], cw gL[k]); its momentum term is
        //   w (a + B n) + S grad w = wL[k] (A + k Bk) + gL[k] s_L
        // with A = cw (a + B n_row) + sum_{b<d-1} S[:, b] cg_b (the record's
        // row part), Bk = cw B[:, d-1] and s_L = cw S[:, d-1]; the mass term
        // is wL[k] cw m.
        float wL[3], gL[3], cw, mp;
        float2 Axy, bkxy, slxy;
        if (D == 3) {
          const float4 bm = *(const float4*)(R + 36);           // Bk_x Bk_y Bk_z m
          const float4 wl = *(const float4*)(R + 44);           // W2[0..2] G2[0]
          const float2 gh = *(const float2*)(R + 48);           // G2[1] G2[2]
          wL[0] = wl.x, wL[1] = wl.y, wL[2] = wl.z;
          gL[0] = wl.w, gL[1] = gh.x, gL[2] = gh.y;
          cw = rw.w;
          mp = bm.w;
          Axy = make_float2(rw.x, rw.y);
          bkxy = fmul2(dup2(cw), make_float2(bm.x, bm.y));
          slxy = fmul2(dup2(cw), make_float2(sl.x, sl.y));
          const float Az = rw.z, bkz = cw * bm.z, slz = cw * sl.z;
          az[0] = fmaf(gL[0], slz, fmaf(wL[0], Az, az[0]));
          az[1] = fmaf(gL[1], slz, fmaf(wL[1], Az + bkz, az[1]));
          az[2] = fmaf(gL[2], slz, fmaf(wL[2], fmaf(2.f, bkz, Az), az[2]));
        } else {
          const float4 bs = *(const float4*)(R + 12);  // Bk_x Bk_y SL_x SL_y
          const float4 wl = *(const float4*)(R + 16);  // W1[0..2] m
          const float4 gl = *(const float4*)(R + 20);  // G1[0..2]
          wL[0] = wl.x, wL[1] = wl.y, wL[2] = wl.z;
          gL[0] = gl.x, gL[1] = gl.y, gL[2] = gl.z;
          cw = rw.z;
          mp = wl.w;
          Axy = make_float2(rw.x, rw.y);
          bkxy = fmul2(dup2(cw), make_float2(bs.x, bs.y));
          slxy = fmul2(dup2(cw), make_float2(bs.z, bs.w));
        }
        const float2 A1xy = fadd2(Axy, bkxy), A2xy = ffma2(dup2(2.f), bkxy, Axy);
        axy[0] = ffma2(dup2(gL[0]), slxy, ffma2(dup2(wL[0]), Axy, axy[0]));
        axy[1] = ffma2(dup2(gL[1]), slxy, ffma2(dup2(wL[1]), A1xy, axy[1]));
        axy[2] = ffma2(dup2(gL[2]), slxy, ffma2(dup2(wL[2]), A2xy, axy[2]));
        const float cm = cw * mp;
#pragma unroll
        for (int k = 0; k < 3; ++k) am[k] = fmaf(wL[k], cm, am[k]);
      }
      if (cur >= 0) p2g_row_flush<D>(tile, Y::TN, cur, n0, n1, axy, az, am);
    };
    if (D == 3) {
      // 3D: SLOTS equal ranges of consecutive particles in one pass (11, 11,
      // 10)
      if (q < Y::SLOTS) walk((q * nvalid) / Y::SLOTS, ((q + 1) * nvalid) / Y::SLOTS);
    } else {
      // 2D: runs of one base cell (found with ballots, at most TMAX long; a
      // cell holds about 4 particles), SLOTS runs at a time, one tile update
      // per run (equal ranges of 3-4 particles would mostly straddle two
      // cells: twice the tile updates)
      const bool valid = lane < nvalid;
      const int prev = __shfl_up_sync(0xffffffffu, cell, 1);
      const unsigned runs = __ballot_sync(0xffffffffu, valid && (lane == 0 || cell != prev));
      const int rs = valid ? 31 - __clz(runs & ((2u << lane) - 1u)) : 0;  // start of this lane's run
      const bool tstart = valid && (lane - rs) % Y::TMAX == 0;
      const unsigned tmask = __ballot_sync(0xffffffffu, tstart);
      const int ntask = __popc(tmask);
      int* ws = starts + warp * 33;  // task k starts at ws[k]; ws[ntask] = nvalid
      if (tstart) ws[__popc(tmask & ((1u << lane) - 1u))] = lane;
      if (lane == 0) ws[ntask] = nvalid;
      __syncwarp();
      for (int t0 = 0; t0 < ntask; t0 += Y::SLOTS) {
        const int t = t0 + q;
        if (q < Y::SLOTS && t < ntask) walk(ws[t], ws[t + 1]);
      }
    }
    // the next work item's step 1 overwrites this warp's records and task
    // starts, which lanes of this warp may still be reading above
    __syncwarp();
    if (!last) continue;  // the same block follows: keep summing into this tile
    __syncthreads();
    // -- 3. flush and clear ---------------------------------------------------
    for (int t = threadIdx.x; t < Y::TN; t += blockDim.x) {
      const float4 val = make_float4(tile[t], tile[Y::TN + t], D == 3 ? tile[2 * Y::TN + t] : 0.f, tile[3 * Y::TN + t]);
      if (val.x == 0.f && val.y == 0.f && val.z == 0.f && val.w == 0.f) continue;
      int I[D];
      int tt = t;
#pragma unroll
      for (int d = D - 1; d >= 0; --d) {
        I[d] = O[d] + tt % 6;
        tt /= 6;
      }
      tile[t] = tile[Y::TN + t] = tile[3 * Y::TN + t] = 0.f;
      if (D == 3) tile[2 * Y::TN + t] = 0.f;
      if (!in_store<D>(V, I)) {
        set_err(c, ERR_OOB);
        continue;
      }
      atomicAdd(&V.node[elem_of<D>(V, I)], val);
    }
    tb ^= 1;
  }
}

// grid_op (adaptive_gimp.py:277-287) of node I of level l, stored at idx: an
// activated node's momentum becomes its velocity (gravity, walls, colliders);
// with inv_norm the other nodes with mass are divided by it.  I lies in
// [0, size]^d.
// Node mask of node I of level l stored at idx: 3D scenes read the level's
// own copy (k_level_masks), which the staged transfers copy by whole blocks;
// 2D scenes, whose transfers gather node by node, read the node mask itself.
template <int D>
__device__ __forceinline__ uint32_t level_mask(const Ctx& c, int l, const int* I, long long idx) {
  if (D == 3) return c.lev[l].nm[idx];
  return nm_get<D>(c, l, I);
}

template <int D>
__device__ __forceinline__ void gridop_node(const Ctx& c, int l, const int* I, long long idx) {
  const LevelDev& V = c.lev[l];
  const float4 nd = V.node[idx];
  if (!(nd.w > 0.f)) return;
  if (!is_activated(level_mask<D>(c, l, I, idx))) {
    if (c.inv_norm) V.node[idx] = make_float4(nd.x / nd.w, nd.y / nd.w, D == 3 ? nd.z / nd.w : nd.z, nd.w);
    return;
  }
  float vv[3] = {nd.x, nd.y, nd.z};
  const int s = c.L - 1 - l;
  bool band = false;
#pragma unroll
  for (int d = 0; d < D; ++d) {
    vv[d] = vv[d] / nd.w;
    vv[d] = vv[d] + c.grav[d] * c.dt;
    const int P = I[d] * (1 << s);
    if (P < c.gap || P > c.sz - c.gap) {
      band = true;
      if (c.bmode == 0) vv[d] = 0.f;
    }
  }
  if (c.bmode == 1 && band)
#pragma unroll
    for (int d = 0; d < D; ++d) vv[d] = 0.f;
  if (c.ncol) {
    const double ldx = 1.0 / (double)(c.coarsest << l);
    for (int k = 0; k < c.ncol; ++k) {
      bool in = true;
#pragma unroll
      for (int d = 0; d < D; ++d) {
        const double pos = (double)I[d] * ldx;
        in = in && pos >= c.col[k][d] && pos <= c.col[k][3 + d];
      }
      if (in)
#pragma unroll
        for (int d = 0; d < D; ++d) vv[d] = 0.f;
    }
  }
  V.node[idx] = make_float4(vv[0], vv[1], vv[2], nd.w);
}

// ---------------------------------------------------------------------------
// Level transfers staged through shared memory by the TMA engine.  A CTA takes
// one destination block at a time; one thread issues bulk copies
// (cp.async.bulk, global -> shared, completion counted in bytes on an
// mbarrier) of the source level's node blocks and node-mask blocks the
// destination block reads, every thread waits on the mbarrier (bounded), and
// the gather then reads shared memory only.  Blocks are contiguous in HBM
// (PER nodes of 16 B, PER masks of 4 B), so every copy is one aligned run.
template <int D>
struct Stage {
  static constexpr int PER = 1 << (2 * D);
  static constexpr uint32_t NODE_BYTES = PER * 16, MASK_BYTES = PER * 4;
  // the lanes of the first warp (a 2D CTA has 16 threads)
  static constexpr unsigned WARP0 = PER >= 32 ? 0xffffffffu : ((1u << PER) - 1u);
};

__device__ __forceinline__ void mbar_expect_tx(uint64_t* m, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(umma::smem_u32(m)), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ void bulk_to_shared(void* dst, const void* src, uint32_t bytes, uint64_t* m) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   umma::smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(umma::smem_u32(m))
               : "memory");
}

// Wait for the staged copies of this phase.  When the bounded wait gives up,
// the CTA records ERR_MLP (a bounded device wait gave up), waits once more
// (bounded) for its copies in flight and returns false.
__device__ __forceinline__ bool stage_wait(const Ctx& c, uint64_t* m, uint32_t phase) {
  if (umma::mbar_wait(m, phase)) return true;
  if (threadIdx.x == 0) set_err(c, ERR_MLP);
  umma::mbar_wait(m, phase);
  return false;
}

__device__ __forceinline__ void stage_init(uint64_t* m) {
  if (threadIdx.x == 0) {
    umma::mbar_init(m, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
}

// stored block coordinates of linear block index b (first axis slowest)
template <int D>
__device__ __forceinline__ void block_coords(unsigned b, unsigned nb, int* Bc) {
#pragma unroll
  for (int d = D - 1; d >= 0; --d) {
    Bc[d] = (int)(b % nb);
    b /= nb;
  }
}

// grid_restriction(l) (adaptive_gimp.py:289-301) as a gather over the coarse
// nodes K of level l-1: the restricted sum onto K of the fine nodes 2K - dI
// that are (activated and even), T-junctions or ghosts, weight 0.5^|dI|_1.
// The fine nodes of a coarse block lie in the 3^d fine blocks 2B-2 .. 2B (B:
// the coarse block's stored coordinates).  The last restriction (into level
// 0) also applies grid_op to level 0, whose momentum no later pass reads; in a
// scene of one level it only does that.
template <int D>
__global__ void __launch_bounds__(Stage<D>::PER) k_restrict(Batch B, int l) {
  SCENE_CTA(B, MAP_T);
  using S = Stage<D>;
  constexpr int NB = (D == 2) ? 9 : 27;
  __shared__ __align__(128) float4 fn[NB][S::PER];
  __shared__ __align__(128) uint32_t fm[NB][S::PER];
  __shared__ int fok[NB];
  __shared__ __align__(8) uint64_t mbar;
  const bool restrict_l = l < c.L;
  if (!restrict_l && l != 1) return;
  const LevelDev& Vc = c.lev[l - 1];
  const LevelDev& Vf = c.lev[restrict_l ? l : l - 1];
  const int nblk = c.ctr[CTR_LEVEL + l - 1];
  const int lsz = Vf.size, l0sz = Vc.size;
  const int loc = threadIdx.x;
  stage_init(&mbar);
  uint32_t phase = 0;
  for (int bi = bid_; bi < nblk; bi += nblk_) {
    const unsigned blk = (unsigned)Vc.blist[bi];
    int Bc[D];
    block_coords<D>(blk, (unsigned)Vc.nb, Bc);
    if (restrict_l) {
      if (threadIdx.x < 32) {
        // lane t of the first warp stages fine block t (NB <= 32)
        const int t = threadIdx.x;
        uint32_t bytes = 0;
        if (t < NB) {
          bool ok = true;
          unsigned fb = 0;
          int tt = t, fc[D];
#pragma unroll
          for (int d = D - 1; d >= 0; --d) {
            fc[d] = 2 * Bc[d] - 2 + tt % 3;
            tt /= 3;
            ok = ok && fc[d] >= 0 && fc[d] < Vf.nb;
          }
#pragma unroll
          for (int d = 0; d < D; ++d) fb = fb * (unsigned)Vf.nb + (unsigned)fc[d];
          fok[t] = ok ? (int)fb : -1;
          if (ok) bytes = S::NODE_BYTES + S::MASK_BYTES;
        }
        bytes = __reduce_add_sync(S::WARP0, bytes);
        // earlier generic reads of the tile finished at the barrier that
        // ended the previous block; order them before the async writes
        umma::fence_proxy_async();
        if (t == 0) mbar_expect_tx(&mbar, bytes);
        __syncwarp(S::WARP0);
        if (t < NB && fok[t] >= 0) {
          bulk_to_shared(fn[t], Vf.node + ((long long)fok[t] << (2 * D)), S::NODE_BYTES, &mbar);
          bulk_to_shared(fm[t], Vf.nm + ((long long)fok[t] << (2 * D)), S::MASK_BYTES, &mbar);
        }
      }
      __syncthreads();  // fok
      const bool ok = stage_wait(c, &mbar, phase);
      phase ^= 1;
      if (!ok) return;
    }
    int K[D];
#pragma unroll
    for (int d = D - 1, t = loc; d >= 0; --d, t >>= 2) K[d] = ((Bc[d] - 1) << 2) + (t & 3);
    bool inr = true;
#pragma unroll
    for (int d = 0; d < D; ++d) inr = inr && K[d] >= 0 && K[d] <= l0sz;
    const long long cidx = ((long long)blk << (2 * D)) | loc;
    if (inr && restrict_l && is_valid(Vc.nm[cidx])) {
      float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
      bool any = false;
#pragma unroll
      for (int a = 0; a < ((D == 2) ? 9 : 27); ++a) {
        int t = a, nrm = 0, tile = 0, li = 0;
        bool okI = true;
#pragma unroll
        for (int d = D - 1; d >= 0; --d) {
          const int dI = t % 3 - 1;
          t /= 3;
          const int I = 2 * K[d] - dI;
          nrm += dI != 0;
          okI = okI && I >= 0 && I <= lsz;
        }
        if (!okI) continue;
        // tile and local index of fine node 2K - dI
        t = a;
        int mul = 1, lmul = 1;
#pragma unroll
        for (int d = D - 1; d >= 0; --d) {
          const int dI = t % 3 - 1;
          t /= 3;
          const int q = 2 * K[d] - dI + HALO;
          tile += ((q >> 2) - (2 * Bc[d] - 2)) * mul;
          li += (q & 3) * lmul;
          mul *= 3;
          lmul *= 4;
        }
        if (fok[tile] < 0) continue;
        const uint32_t nm = fm[tile][li];
        if (!((is_activated(nm) && nrm == 0) || is_tj(nm) || is_ghost(nm))) continue;
        const float w = (nrm == 0) ? 1.f : (nrm == 1) ? 0.5f : (nrm == 2) ? 0.25f : 0.125f;
        const float4 f = fn[tile][li];
        acc.x += f.x * w;
        acc.y += f.y * w;
        acc.z += f.z * w;
        acc.w += f.w * w;
        any = true;
      }
      if (any) {
        float4 o = Vc.node[cidx];
        o.x += acc.x;
        o.y += acc.y;
        o.z += acc.z;
        o.w += acc.w;
        Vc.node[cidx] = o;
      }
    }
    if (inr && l == 1) gridop_node<D>(c, 0, K, cidx);
    __syncthreads();  // the tile is free for the next block's copies
  }
}

// ---------------------------------------------------------------------------
// The same two transfers as direct gathers through L1 (one thread per
// destination node): used for 2D scenes, whose 16-node blocks are too small
// for a staging round trip per block to pay.
template <int D>
__global__ void k_restrict_gather(Batch B, int l) {
  SCENE_CTA(B, MAP_G);
  const bool restrict_l = l < c.L;
  if (!restrict_l && l != 1) return;
  const LevelDev& Vc = c.lev[l - 1];
  const LevelDev& Vf = c.lev[restrict_l ? l : l - 1];
  const long long tot = (long long)c.ctr[CTR_LEVEL + l - 1] << (2 * D);
  const int lsz = Vf.size, l0sz = Vc.size;
  SCENE_LOOP(e, tot) {
    const long long blk = Vc.blist[e >> (2 * D)];
    const int loc = (int)(e & ((1 << (2 * D)) - 1));
    int K[D];
    elem_coords<D>(Vc, blk, loc, K);
    bool inr = true;
#pragma unroll
    for (int d = 0; d < D; ++d) inr = inr && K[d] >= 0 && K[d] <= l0sz;
    if (!inr) continue;
    const long long cidx = (blk << (2 * D)) | loc;
    if (restrict_l && is_valid(level_mask<D>(c, l - 1, K, cidx))) {
      float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
      bool any = false;
#pragma unroll
      for (int a = 0; a < ((D == 2) ? 9 : 27); ++a) {
        int I[D], nrm = 0, t = a;
        bool ok = true;
#pragma unroll
        for (int d = D - 1; d >= 0; --d) {
          const int dI = t % 3 - 1;
          t /= 3;
          I[d] = 2 * K[d] - dI;
          nrm += dI != 0;
          ok = ok && I[d] >= 0 && I[d] <= lsz;
        }
        if (!ok) continue;
        const long long fidx = elem_of<D>(Vf, I);
        const uint32_t nm = level_mask<D>(c, l, I, fidx);
        if (!((is_activated(nm) && nrm == 0) || is_tj(nm) || is_ghost(nm))) continue;
        const float w = (nrm == 0) ? 1.f : (nrm == 1) ? 0.5f : (nrm == 2) ? 0.25f : 0.125f;
        const float4 f = Vf.node[fidx];
        acc.x += f.x * w;
        acc.y += f.y * w;
        acc.z += f.z * w;
        acc.w += f.w * w;
        any = true;
      }
      if (any) {
        float4 o = Vc.node[cidx];
        o.x += acc.x;
        o.y += acc.y;
        o.z += acc.z;
        o.w += acc.w;
        Vc.node[cidx] = o;
      }
    }
    if (l == 1) gridop_node<D>(c, 0, K, cidx);
  }
}

template <int D>
__global__ void k_prolong_gather(Batch B, int l) {
  SCENE_CTA(B, MAP_G);
  if (l >= c.L) return;
  const LevelDev& Vc = c.lev[l - 1];
  const LevelDev& Vf = c.lev[l];
  const long long tot = (long long)c.ctr[CTR_LEVEL + l] << (2 * D);
  const int lsz = Vf.size;
  SCENE_LOOP(e, tot) {
    const long long blk = Vf.blist[e >> (2 * D)];
    const int loc = (int)(e & ((1 << (2 * D)) - 1));
    int J[D];
    elem_coords<D>(Vf, blk, loc, J);
    bool inr = true, even = true;
#pragma unroll
    for (int d = 0; d < D; ++d) {
      inr = inr && J[d] >= 0 && J[d] <= lsz;
      even = even && (J[d] & 1) == 0;
    }
    if (!inr) continue;
    const long long fidx = (blk << (2 * D)) | loc;
    gridop_node<D>(c, l, J, fidx);
    const uint32_t nm = level_mask<D>(c, l, J, fidx);
    const bool tg = is_tj(nm) || is_ghost(nm);
    if (!tg && !even) continue;
    float acc[3] = {0.f, 0.f, 0.f};
    if (tg) {
      int nodd = 0;
#pragma unroll
      for (int d = 0; d < D; ++d) nodd += J[d] & 1;
      const float w = (nodd == 0) ? 1.f : (nodd == 1) ? 0.5f : (nodd == 2) ? 0.25f : 0.125f;
#pragma unroll
      for (int a = 0; a < (1 << D); ++a) {
        int K[D];
        bool use = true;
#pragma unroll
        for (int d = 0; d < D; ++d) {
          const int bit = (a >> d) & 1;
          if (J[d] & 1)
            K[d] = (J[d] - 1) / 2 + bit;
          else {
            K[d] = J[d] / 2;
            use = use && bit == 0;
          }
        }
        if (!use) continue;
        const long long cidx = elem_of<D>(Vc, K);
        if (!is_valid(level_mask<D>(c, l - 1, K, cidx))) continue;
        const float4 cv = Vc.node[cidx];
        acc[0] += cv.x * w;
        acc[1] += cv.y * w;
        acc[2] += cv.z * w;
      }
    } else if (is_activated(nm)) {
      int K[D];
#pragma unroll
      for (int d = 0; d < D; ++d) K[d] = J[d] / 2;
      const long long cidx = elem_of<D>(Vc, K);
      if (is_valid(level_mask<D>(c, l - 1, K, cidx))) {
        const float4 cv = Vc.node[cidx];
        acc[0] = cv.x;
        acc[1] = cv.y;
        acc[2] = cv.z;
      }
    }
    float4 o = Vf.node[fidx];
    o.x = acc[0];
    o.y = acc[1];
    o.z = acc[2];
    Vf.node[fidx] = o;
  }
}

// 3D scenes stage their transfers through shared memory, 2D scenes gather
template <int D>
constexpr bool staged_transfers() {
  return D == 3;
}

// ---------------------------------------------------------------------------
// grid_op for every level at once.  Only substeps whose scenes all have one
// level launch it; otherwise the last restriction applies grid_op to level 0
// and each prolongation to its own level (see there).
template <int D>
__global__ void k_gridop(Batch B) {
  SCENE_CTA(B, MAP_G);
  __shared__ BlockRanges br;
  load_block_ranges(c, br);
  const long long tot = total_elems_r(br, 0, c.L, D);
  SCENE_LOOP(e, tot) {
    int l, loc;
    long long blk;
    decode_elem_r<D>(c, br, 0, c.L, e, l, blk, loc);
    const LevelDev& V = c.lev[l];
    int I[D];
    elem_coords<D>(V, blk, loc, I);
    bool inr = true;
#pragma unroll
    for (int d = 0; d < D; ++d) inr = inr && I[d] >= 0 && I[d] <= V.size;
    if (inr) gridop_node<D>(c, l, I, (blk << (2 * D)) | loc);
  }
}

// ---------------------------------------------------------------------------
// grid_prolongation(l) (adaptive_gimp.py:303-321) as a gather over the fine
// nodes J of level l: T-junction and ghost nodes take the weighted sum of
// their valid coarse neighbours, other all-even nodes take the coincident
// coarse velocity if they are activated and it is valid, else 0; the rest keep
// their value.  The coarse nodes of a fine block B lie in the 2^d coarse
// blocks (2B + 1) / 4 .. (2B + 1) / 4 + 1 per axis, staged like the
// restriction's.  Level l's grid_op runs first on each node: its momentum is
// no longer read (the restrictions are done) and its coarser neighbour is
// final.
template <int D>
__global__ void __launch_bounds__(Stage<D>::PER) k_prolong(Batch B, int l) {
  SCENE_CTA(B, MAP_T);
  using S = Stage<D>;
  constexpr int NB = 1 << D;
  __shared__ __align__(128) float4 cn[NB][S::PER];
  __shared__ __align__(128) uint32_t cm[NB][S::PER];
  __shared__ int cok[NB];
  __shared__ __align__(8) uint64_t mbar;
  if (l >= c.L) return;
  const LevelDev& Vc = c.lev[l - 1];
  const LevelDev& Vf = c.lev[l];
  const int nblk = c.ctr[CTR_LEVEL + l];
  const int lsz = Vf.size;
  const int loc = threadIdx.x;
  stage_init(&mbar);
  uint32_t phase = 0;
  for (int bi = bid_; bi < nblk; bi += nblk_) {
    const unsigned blk = (unsigned)Vf.blist[bi];
    int Bf[D], C0[D];
    block_coords<D>(blk, (unsigned)Vf.nb, Bf);
#pragma unroll
    for (int d = 0; d < D; ++d) C0[d] = (2 * Bf[d] + 1) >> 2;
    if (threadIdx.x < 32) {
      // lane t of the first warp stages coarse block t
      const int t = threadIdx.x;
      uint32_t bytes = 0;
      if (t < NB) {
        bool ok = true;
        unsigned cb = 0;
#pragma unroll
        for (int d = 0; d < D; ++d) {
          const int q = C0[d] + ((t >> (D - 1 - d)) & 1);
          ok = ok && q < Vc.nb;
          cb = cb * (unsigned)Vc.nb + (unsigned)q;
        }
        cok[t] = ok ? (int)cb : -1;
        if (ok) bytes = S::NODE_BYTES + S::MASK_BYTES;
      }
      bytes = __reduce_add_sync(S::WARP0, bytes);
      umma::fence_proxy_async();
      if (t == 0) mbar_expect_tx(&mbar, bytes);
      __syncwarp(S::WARP0);
      if (t < NB && cok[t] >= 0) {
        bulk_to_shared(cn[t], Vc.node + ((long long)cok[t] << (2 * D)), S::NODE_BYTES, &mbar);
        bulk_to_shared(cm[t], Vc.nm + ((long long)cok[t] << (2 * D)), S::MASK_BYTES, &mbar);
      }
    }
    __syncthreads();  // cok
    const bool okw = stage_wait(c, &mbar, phase);
    phase ^= 1;
    if (!okw) return;
    int J[D];
#pragma unroll
    for (int d = D - 1, t = loc; d >= 0; --d, t >>= 2) J[d] = ((Bf[d] - 1) << 2) + (t & 3);
    bool inr = true, even = true;
#pragma unroll
    for (int d = 0; d < D; ++d) {
      inr = inr && J[d] >= 0 && J[d] <= lsz;
      even = even && (J[d] & 1) == 0;
    }
    const long long fidx = ((long long)blk << (2 * D)) | loc;
    if (inr) {
      gridop_node<D>(c, l, J, fidx);
      const uint32_t nm = Vf.nm[fidx];
      const bool tg = is_tj(nm) || is_ghost(nm);
      if (tg || even) {
        // coarse node K: staged tile and local index
        auto coarse = [&](const int* K, float4& v) -> bool {
          int tile = 0, li = 0;
#pragma unroll
          for (int d = 0; d < D; ++d) {
            const int q = K[d] + HALO;
            tile = tile * 2 + ((q >> 2) - C0[d]);
            li = li * 4 + (q & 3);
          }
          if (cok[tile] < 0 || !is_valid(cm[tile][li])) return false;
          v = cn[tile][li];
          return true;
        };
        float acc[3] = {0.f, 0.f, 0.f};
        if (tg) {
          int nodd = 0;
#pragma unroll
          for (int d = 0; d < D; ++d) nodd += J[d] & 1;
          const float w = (nodd == 0) ? 1.f : (nodd == 1) ? 0.5f : (nodd == 2) ? 0.25f : 0.125f;
#pragma unroll
          for (int a = 0; a < (1 << D); ++a) {
            int K[D];
            bool use = true;
#pragma unroll
            for (int d = 0; d < D; ++d) {
              const int bit = (a >> d) & 1;
              if (J[d] & 1)
                K[d] = (J[d] - 1) / 2 + bit;
              else {
                K[d] = J[d] / 2;
                use = use && bit == 0;
              }
            }
            float4 cv;
            if (!use || !coarse(K, cv)) continue;
            acc[0] += cv.x * w;
            acc[1] += cv.y * w;
            acc[2] += cv.z * w;
          }
        } else if (is_activated(nm)) {
          int K[D];
#pragma unroll
          for (int d = 0; d < D; ++d) K[d] = J[d] / 2;
          float4 cv;
          if (coarse(K, cv)) {
            acc[0] = cv.x;
            acc[1] = cv.y;
            acc[2] = cv.z;
          }
        }
        float4 o = Vf.node[fidx];
        o.x = acc[0];
        o.y = acc[1];
        o.z = acc[2];
        Vf.node[fidx] = o;
      }
    }
    __syncthreads();  // the tile is free for the next block's copies
  }
}

// ---------------------------------------------------------------------------
// g2p (adaptive_gimp.py:252-275), plus the snow return map (extension).
template <int D>
__device__ __forceinline__ void svd_d(const float* F, float* U, float* sg, float* V) {
  if (D == 2)
    svd2(F, U, sg, V);
  else
    svd3(F, U, sg, V);
}

// Exact snow return map (Stomakhin et al. 2013) on an SVD: clamp the singular
// values to [1-theta_c, 1+theta_s], update Jp, rebuild F.  Written with
// explicitly rounded operations (no contraction choices left to the compiler)
// so that every inlined copy, in G2P and in the surrogate's finishing kernel,
// gives the same bits for the same SVD.
template <int D>
__device__ __forceinline__ void snow_clamp_rebuild(const Ctx& c, const float* U, const float* sg, const float* V,
                                                   float* F, float& jp) {
  const float lo = 1.f - c.theta_c, hi = 1.f + c.theta_s;
  float Jo = 1.f, Jn = 1.f, sc[D];
#pragma unroll
  for (int d = 0; d < D; ++d) {
    const float cl = fminf(fmaxf(sg[d], lo), hi);
    Jo = __fmul_rn(Jo, sg[d]);
    Jn = __fmul_rn(Jn, cl);
    sc[d] = cl;
  }
  jp = __fdiv_rn(__fmul_rn(jp, Jo), Jn);
#pragma unroll
  for (int i = 0; i < D; ++i)
#pragma unroll
    for (int j = 0; j < D; ++j) {
      float a = 0.f;
#pragma unroll
      for (int k = 0; k < D; ++k) a = __fmaf_rn(__fmul_rn(U[i * D + k], sc[k]), V[j * D + k], a);
      F[i * D + j] = a;
    }
}


// The surrogate's domain: a non-inverted trial state with positive singular
// values and plastic ratio.
template <int D>
__device__ __forceinline__ bool sur_domain(const float* F, const float* sg, float jp) {
  bool ok = jp > 0.f && det<D>(F) > 0.f;
#pragma unroll
  for (int d = 0; d < D; ++d) ok = ok && sg[d] > 0.f;
  return ok;
}

// Recorder: the surrogate's training pair (features, exact projected state)
// of a trial state with singular values sg and plastic ratio jp.
template <int D>
__device__ __forceinline__ void record_pair(const Ctx& c, const float* sg, float jp) {
  float x[7], y[4];
  snow_features<D>(sg, jp, c.xi, c.theta_c, c.theta_s, x);
  float Jo = 1.f, Jn = 1.f;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    if (d < D) {
      const float cl = fminf(fmaxf(sg[d], 1.f - c.theta_c), 1.f + c.theta_s);
      Jo *= sg[d];
      Jn *= cl;
      y[d] = (cl - sg[d]) / SUR_DSIG;
    } else {
      y[d] = 0.f;
    }
  }
  y[3] = logf(Jo / Jn) / SUR_DLJ;
  const int slot = reserve_slot(&c.ctr[CTR_REC]);
  if ((long long)slot >= c.rec_cap) return;
#pragma unroll
  for (int k = 0; k < 7; ++k) c.rec_X[(long long)slot * 7 + k] = x[k];
#pragma unroll
  for (int k = 0; k < 4; ++k) c.rec_T[(long long)slot * 4 + k] = y[k];
}

// Surrogate hand-off of a trial state with SVD (U, sg, V): its features go to
// the MLP's input buffer and U, V, sig, jp to the metadata buffer, and
// k_sur_finish writes F and Jp.  Returns false when the features leave the
// trained range (the caller then applies the exact return map).
template <int D>
__device__ __forceinline__ bool sur_handoff(const Ctx& c, const float* U, const float* sg, const float* V, float jp,
                                            int j) {
  float x[7];
  snow_features<D>(sg, jp, c.xi, c.theta_c, c.theta_s, x);
  bool ok = true;
#pragma unroll
  for (int k = 0; k < 7; ++k) ok = ok && fabsf(x[k]) <= c.sur_xmax[k];
  if (!ok) return false;
  const int slot = reserve_slot(c.sur_ctr);
  float* meta = c.sur_meta + (long long)slot * SUR_META;
  meta[0] = __int_as_float(j);
  meta[23] = __int_as_float(c.scene);
#pragma unroll
  for (int k = 0; k < D * D; ++k) {
    meta[1 + k] = U[k];
    meta[10 + k] = V[k];
  }
#pragma unroll
  for (int d = 0; d < D; ++d) meta[19 + d] = sg[d];
  meta[22] = jp;
#pragma unroll
  for (int k = 0; k < 7; ++k) c.sur_X[(long long)slot * 7 + k] = x[k];
  return true;
}

// Snow return map of G2P's trial state F (in place): states whose singular
// values are provably inside the clamp interval are unchanged; the others get
// an SVD, are recorded when the recorder samples this particle, and are
// projected exactly or handed to the surrogate.
template <int D>
__device__ __forceinline__ void snow_return_map(const Ctx& c, float* F, float& jp, int j) {
  if (singular_values_within<D>(F, 1.f - c.theta_c, 1.f + c.theta_s)) return;
  float U[D * D], sg[D], V[D * D];
  svd_d<D>(F, U, sg, V);
  const bool dom = (c.rec_X || c.sur) && sur_domain<D>(F, sg, jp);
  if (c.rec_X && dom && j % c.rec_stride == 0) record_pair<D>(c, sg, jp);
  if (c.sur && dom && sur_handoff<D>(c, U, sg, V, jp, j)) return;
  snow_clamp_rebuild<D>(c, U, sg, V, F, jp);
}

// Apply the MLP's predictions: decode the projected singular values sig' and
// the change of log Jp, reject them when sig' leaves the clamp interval (the
// yield surface) or the change breaks the plastic-volume balance
// log Jp' - log Jp = sum log sig - sum log sig' by more than sur_tol (then the
// exact return map is used), and write F and Jp.
template <int D>
__global__ void k_sur_finish(Batch B, const float* __restrict__ meta_all, const float* __restrict__ Y,
                             const int32_t* __restrict__ n_dev) {
  const int n = *n_dev;
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
    const float* meta = meta_all + (long long)s * SUR_META;
    const int j = __float_as_int(meta[0]);
    const Ctx& c = B.ctx[__float_as_int(meta[23])];  // the slot's scene
    float U[D * D], V[D * D], sg[D];
#pragma unroll
    for (int k = 0; k < D * D; ++k) {
      U[k] = meta[1 + k];
      V[k] = meta[10 + k];
    }
#pragma unroll
    for (int d = 0; d < D; ++d) sg[d] = meta[19 + d];
    float jp = meta[22];
    const float* y = Y + (long long)s * 4;
    const float ts = c.theta_s, tcr = c.theta_c;
    float sp[D], r = 0.f, lsum = 0.f;
#pragma unroll
    for (int d = 0; d < D; ++d) {
      sp[d] = sg[d] + SUR_DSIG * y[d];
      r = fmaxf(r, fmaxf(sp[d] - (1.f + ts), (1.f - tcr) - sp[d]));
      lsum += logf(sg[d]) - logf(fmaxf(sp[d], 1e-6f));
    }
    const float dljp = SUR_DLJ * y[3];
    r = fmaxf(r, fabsf(dljp - lsum));
    float F[D * D];
    if (!(r <= c.sur_tol)) {
      snow_clamp_rebuild<D>(c, U, sg, V, F, jp);
      atomicAdd(&c.ctr[CTR_SURFB], 1);
    } else {
      jp = jp * expf(dljp);
#pragma unroll
      for (int a = 0; a < D; ++a)
#pragma unroll
        for (int b = 0; b < D; ++b) {
          float acc = 0.f;
#pragma unroll
          for (int k = 0; k < D; ++k) acc += U[a * D + k] * sp[k] * V[b * D + k];
          F[a * D + b] = acc;
        }
    }
    const long long N = c.N;
    float* QF = c.Q.F;
    float* QJ = c.Q.Jp;
#pragma unroll
    for (int k = 0; k < D * D; ++k) __stwb(&QF[k * N + j], F[k]);
    __stwb(&QJ[j], jp);
  }
}

// G2P writes the updated particles into Q in this substep's bin order, so the
// next substep reads every particle array with contiguous loads.  m, g and id
// travel with the particle; fl records the level used; particles without a
// level (the extra bin, level -1) are copied unchanged.
template <int D>
__device__ __forceinline__ void copy_particle(const Ctx& c, int p, int j) {
  const long long N = c.N;
#pragma unroll
  for (int d = 0; d < D; ++d) {
    __stwb(&c.Q.x[d * N + j], __ldg(&c.P.x[d * N + p]));
    __stwb(&c.Q.v[d * N + j], __ldg(&c.P.v[d * N + p]));
  }
#pragma unroll
  for (int k = 0; k < D * D; ++k) {
    __stwb(&c.Q.F[k * N + j], __ldg(&c.P.F[k * N + p]));
    __stwb(&c.Q.C[k * N + j], __ldg(&c.P.C[k * N + p]));
  }
  __stwb(&c.Q.m[j], __ldg(&c.P.m[p]));
  __stwb(&c.Q.Jp[j], __ldg(&c.P.Jp[p]));
  __stwb(&c.Q.g[j], __ldg(&c.P.g[p]));
  __stwb(&c.Q.id[j], __ldg(&c.P.id[p]));
  __stwb(&c.Q.fl[j], -1);
}

// One particle, slot j of this substep's bin order; the 3^d nodes come
// through L1 (particles of a bin share a (4+2)^d node tile).
template <int D>
__device__ __forceinline__ void g2p_one(const Ctx& c, int j) {
  const float pw = (D == 2) ? 0.25f : 0.125f;
  const float rd = (D == 2) ? c.radius * c.radius : c.radius * c.radius * c.radius;
  const long long N = c.N;
  const int p = __ldg(&c.perm[j]);
  const int l = __ldg(&c.P.fl[p]);
  // the fields read after the gather start moving into L1 now (no registers held)
#pragma unroll
  for (int k = 0; k < D * D; ++k) asm volatile("prefetch.global.L1 [%0];" ::"l"(&c.P.F[k * N + p]));
  asm volatile("prefetch.global.L1 [%0];" ::"l"(&c.P.m[p]));
  asm volatile("prefetch.global.L1 [%0];" ::"l"(&c.P.g[p]));
  asm volatile("prefetch.global.L1 [%0];" ::"l"(&c.P.id[p]));
  if (c.plast == 1) asm volatile("prefetch.global.L1 [%0];" ::"l"(&c.P.Jp[p]));
  if (l < 0) {
    copy_particle<D>(c, p, j);
    return;
  }
  float xp[D];
#pragma unroll
  for (int d = 0; d < D; ++d) xp[d] = __ldg(&c.P.x[d * N + p]);
  const LevelDev& V = c.lev[l];
  const float inv = (float)(c.coarsest << l);
  const float dx = 1.f / inv;
  int base[D];
  float tc[D];
#pragma unroll
  for (int d = 0; d < D; ++d) {
    const float xs = xp[d] * inv;
    base[d] = (int)(xs + 0.5f) - 1;
    tc[d] = xs - (float)(base[d] + 1);
  }
  // Gather by rows along the last axis: the weights are products of per-axis
  // terms, so a row's nodes are first summed with the last axis's weight (S)
  // and gradient (T), and the other axes' factors are applied once per row.
  // Only the last axis's factors are kept; the others are formed when their
  // row starts (closed form for radius 1/2), which keeps G2P inside 64
  // registers with a slab of nodes in flight.
  const bool half = c.radius == 0.5f;
  float W2[3], G2[3];
  if (half)
    axis_weights_half(tc[D - 1], W2, G2);
  else
    axis_weights(tc[D - 1], c.radius, W2, G2);
  auto axis_factor = [&](float t, int k, float& w, float& g) {
    if (half) {
      const float a = 0.5f - t, b = 0.5f + t;
      w = k == 0 ? a * a : (k == 1 ? fmaf(-2.f * t, t, 1.5f) : b * b);
      g = k == 0 ? -a : (k == 1 ? -2.f * t : b);
    } else {
      float Wk[3], Gk[3];
      axis_weights(t, c.radius, Wk, Gk);
      w = k == 0 ? Wk[0] : (k == 1 ? Wk[1] : Wk[2]);
      g = k == 0 ? Gk[0] : (k == 1 ? Gk[1] : Gk[2]);
    }
  };
  const float r2 = 2.f * c.radius;
  const float kw = (D == 2) ? 1.f / (4.f * r2 * r2) : 1.f / (8.f * r2 * r2 * r2);
  const float kg = (D == 2) ? 1.f / (2.f * r2 * r2) : 1.f / (4.f * r2 * r2 * r2);
  float nv[D], G[D * D];
#pragma unroll
  for (int i = 0; i < D; ++i) nv[i] = 0.f;
#pragma unroll
  for (int i = 0; i < D * D; ++i) G[i] = 0.f;
#pragma unroll(D == 3 ? 1 : 3)
  for (int n0 = 0; n0 < 3; ++n0) {
    float w0, g0;
    axis_factor(tc[0], n0, w0, g0);
    // one row (3 nodes) in flight at a time: measured faster than a slab of
    // 9 gathers, which does not fit the 64-register budget
#pragma unroll 1
    for (int n1 = 0; n1 < ((D == 2) ? 1 : 3); ++n1) {
      float S[D], T[D];
#pragma unroll
      for (int i = 0; i < D; ++i) S[i] = T[i] = 0.f;
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        int I[D];
        I[0] = base[0] + n0;
        if (D == 3) I[1] = base[1] + n1;
        I[D - 1] = base[D - 1] + k;
        // base lies in [-1, size-1] for an in-domain particle: always in store
        const float4 nd = __ldg(&V.node[elem_of<D>(V, I)]);
        const float gv[3] = {nd.x, nd.y, nd.z};
#pragma unroll
        for (int i = 0; i < D; ++i) {
          S[i] += gv[i] * W2[k];
          T[i] += gv[i] * G2[k];
        }
      }
      // row factors: weight, and the gradient components of the other axes
      float cw, cg[D];
      if (D == 2) {
        cw = w0 * kw;
        cg[0] = g0 * kg;
        cg[1] = w0 * kg;
      } else {
        float w1, g1;
        axis_factor(tc[1], n1, w1, g1);
        const float wxy = w0 * w1;
        cw = wxy * kw;
        cg[0] = g0 * w1 * kg;
        cg[1] = w0 * g1 * kg;
        cg[D - 1] = wxy * kg;
      }
#pragma unroll
      for (int i = 0; i < D; ++i) {
        nv[i] += cw * S[i];
#pragma unroll
        for (int q = 0; q < D - 1; ++q) G[i * D + q] += cg[q] * S[i];
        G[i * D + D - 1] += cg[D - 1] * T[i];
      }
    }
  }
#pragma unroll
  for (int d = 0; d < D; ++d) {
    __stwb(&c.Q.v[d * N + j], nv[d]);
    __stwb(&c.Q.x[d * N + j], xp[d] + c.dt * nv[d]);
  }
#pragma unroll
  for (int i = 0; i < D * D; ++i) __stwb(&c.Q.C[i * N + j], G[i]);
  // the rest of the particle is read only now (fewer live registers during
  // the gather); m, g, id and Jp travel unchanged
  __stwb(&c.Q.m[j], __ldg(&c.P.m[p]));
  __stwb(&c.Q.g[j], __ldg(&c.P.g[p]));
  __stwb(&c.Q.id[j], __ldg(&c.P.id[p]));
  __stwb(&c.Q.Jp[j], c.plast == 1 ? __ldg(&c.P.Jp[p]) : 1.f);
  __stwb(&c.Q.fl[j], l);
  float F[D * D];
#pragma unroll
  for (int k = 0; k < D * D; ++k) F[k] = __ldg(&c.P.F[k * N + p]);
  const float s = (c.dt * pw) / (rd * dx);
  // F' = (I + s G) F row by row, each row stored at once; the Gram matrix
  // F'^T F' is summed from the rows for the return-map test below
  float Sg[(D == 2) ? 3 : 6];
#pragma unroll
  for (int k = 0; k < ((D == 2) ? 3 : 6); ++k) Sg[k] = 0.f;
#pragma unroll
  for (int i = 0; i < D; ++i) {
    float row[D];
#pragma unroll
    for (int q = 0; q < D; ++q) {
      float a = 0.f;
#pragma unroll
      for (int k = 0; k < D; ++k) a += ((i == k ? 1.f : 0.f) + s * G[i * D + k]) * F[k * D + q];
      row[q] = a;
      __stwb(&c.Q.F[(i * D + q) * N + j], a);
    }
    int u = 0;
#pragma unroll
    for (int a = 0; a < D; ++a)
#pragma unroll
      for (int b = a; b < D; ++b) Sg[u++] += row[a] * row[b];
  }
  // trial states that may leave the elastic interval get the return map in
  // k_project (it needs an SVD, whose registers would halve G2P's occupancy);
  // det F' = det(I + s G) det F
  if (c.plast == 1) {
    float A[D * D];
#pragma unroll
    for (int i = 0; i < D; ++i)
#pragma unroll
      for (int k = 0; k < D; ++k) A[i * D + k] = (i == k ? 1.f : 0.f) + s * G[i * D + k];
    if (!gram_within<D>(Sg, det<D>(A) * det<D>(F), 1.f - c.theta_c, 1.f + c.theta_s))
      c.proj[reserve_slot(&c.ctr[CTR_PROJ])] = j;
  }
}

// 2D G2P: one thread per particle slot, grid-stride (a 2D block holds about
// one work item, too little to pay for staging its nodes).
template <int D>
__global__ void __launch_bounds__(256, 4) k_g2p_gather(Batch B) {
  SCENE_CTA(B, MAP_G);
  SCENE_LOOP(j, c.N) g2p_one<D>(c, (int)j);
}

// The new state of particle p (slot j of this substep's bin order) whose
// base cell lies in the block with first node O, from the block's staged
// node velocities: txy[t] = (v_x, v_y), tz[t] = v_z of tile node t (the
// (4+2)^d nodes O..O+5, last axis fastest).
template <int D>
__device__ __forceinline__ void g2p_staged(const Ctx& c, int l, int p, int j, const float* xp, const int* O,
                                           const float2* txy, const float* tz) {
  const float pw = (D == 2) ? 0.25f : 0.125f;
  const float rd = (D == 2) ? c.radius * c.radius : c.radius * c.radius * c.radius;
  const long long N = c.N;
  const float inv = (float)(c.coarsest << l);
  const float dx = 1.f / inv;
  float tc[D];
  int t0 = 0;
  bool inside = true;
#pragma unroll
  for (int d = 0; d < D; ++d) {
    const float xs = xp[d] * inv;
    const int base = (int)(xs + 0.5f) - 1;
    tc[d] = xs - (float)(base + 1);
    // the binning put the base cell in this block; a cell outside it would
    // read another tile's nodes, so it is clamped and reported
    int r = base - O[d];
    inside = inside && r >= 0 && r <= 3;
    r = min(max(r, 0), 3);
    t0 = t0 * 6 + r;
  }
  if (!inside) set_err(c, ERR_OOB);
  const bool half = c.radius == 0.5f;
  float W2[3], G2[3];
  if (half)
    axis_weights_half(tc[D - 1], W2, G2);
  else
    axis_weights(tc[D - 1], c.radius, W2, G2);
  auto axis_factor = [&](float t, int k, float& w, float& g) {
    if (half) {
      const float a = 0.5f - t, b = 0.5f + t;
      w = k == 0 ? a * a : (k == 1 ? fmaf(-2.f * t, t, 1.5f) : b * b);
      g = k == 0 ? -a : (k == 1 ? -2.f * t : b);
    } else {
      float Wk[3], Gk[3];
      axis_weights(t, c.radius, Wk, Gk);
      w = k == 0 ? Wk[0] : (k == 1 ? Wk[1] : Wk[2]);
      g = k == 0 ? Gk[0] : (k == 1 ? Gk[1] : Gk[2]);
    }
  };
  const float r2 = 2.f * c.radius;
  const float kw = (D == 2) ? 1.f / (4.f * r2 * r2) : 1.f / (8.f * r2 * r2 * r2);
  const float kg = (D == 2) ? 1.f / (2.f * r2 * r2) : 1.f / (4.f * r2 * r2 * r2);
  float nv[D], G[D * D];
#pragma unroll
  for (int i = 0; i < D; ++i) nv[i] = 0.f;
#pragma unroll
  for (int i = 0; i < D * D; ++i) G[i] = 0.f;
  // Rows along the last axis: a row's nodes are summed with the last axis's
  // weight (S) and gradient (T) first; the other axes' factors are applied
  // once per row.
#pragma unroll
  for (int n0 = 0; n0 < 3; ++n0) {
    float w0, g0;
    axis_factor(tc[0], n0, w0, g0);
#pragma unroll
    for (int n1 = 0; n1 < ((D == 2) ? 1 : 3); ++n1) {
      const int tr = t0 + n0 * ((D == 2) ? 6 : 36) + ((D == 2) ? 0 : n1 * 6);
      float2 Sxy = make_float2(0.f, 0.f), Txy = make_float2(0.f, 0.f);
      float Sz = 0.f, Tz = 0.f;
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        const float2 v = txy[tr + k];
        Sxy = ffma2(v, dup2(W2[k]), Sxy);
        Txy = ffma2(v, dup2(G2[k]), Txy);
        if (D == 3) {
          const float vz = tz[tr + k];
          Sz = fmaf(vz, W2[k], Sz);
          Tz = fmaf(vz, G2[k], Tz);
        }
      }
      const float S[3] = {Sxy.x, Sxy.y, Sz}, T[3] = {Txy.x, Txy.y, Tz};
      // row factors: weight, and the gradient components of the other axes
      float cw, cg[D];
      if (D == 2) {
        cw = w0 * kw;
        cg[0] = g0 * kg;
        cg[1] = w0 * kg;
      } else {
        float w1, g1;
        axis_factor(tc[1], n1, w1, g1);
        const float wxy = w0 * w1;
        cw = wxy * kw;
        cg[0] = g0 * w1 * kg;
        cg[1] = w0 * g1 * kg;
        cg[D - 1] = wxy * kg;
      }
#pragma unroll
      for (int i = 0; i < D; ++i) {
        nv[i] = fmaf(cw, S[i], nv[i]);
#pragma unroll
        for (int q = 0; q < D - 1; ++q) G[i * D + q] = fmaf(cg[q], S[i], G[i * D + q]);
        G[i * D + D - 1] = fmaf(cg[D - 1], T[i], G[i * D + D - 1]);
      }
    }
  }
#pragma unroll
  for (int d = 0; d < D; ++d) {
    __stwb(&c.Q.v[d * N + j], nv[d]);
    __stwb(&c.Q.x[d * N + j], xp[d] + c.dt * nv[d]);
  }
#pragma unroll
  for (int i = 0; i < D * D; ++i) __stwb(&c.Q.C[i * N + j], G[i]);
  // m, g, id and Jp travel unchanged
  __stwb(&c.Q.m[j], __ldg(&c.P.m[p]));
  __stwb(&c.Q.g[j], __ldg(&c.P.g[p]));
  __stwb(&c.Q.id[j], __ldg(&c.P.id[p]));
  __stwb(&c.Q.Jp[j], c.plast == 1 ? __ldg(&c.P.Jp[p]) : 1.f);
  __stwb(&c.Q.fl[j], l);
  float F[D * D];
#pragma unroll
  for (int k = 0; k < D * D; ++k) F[k] = __ldg(&c.P.F[k * N + p]);
  const float s = (c.dt * pw) / (rd * dx);
  // F' = (I + s G) F row by row, each row stored at once; the Gram matrix
  // F'^T F' is summed from the rows for the return-map test below
  float Sg[(D == 2) ? 3 : 6];
#pragma unroll
  for (int k = 0; k < ((D == 2) ? 3 : 6); ++k) Sg[k] = 0.f;
#pragma unroll
  for (int i = 0; i < D; ++i) {
    float row[D];
#pragma unroll
    for (int q = 0; q < D; ++q) {
      float a = 0.f;
#pragma unroll
      for (int k = 0; k < D; ++k) a += ((i == k ? 1.f : 0.f) + s * G[i * D + k]) * F[k * D + q];
      row[q] = a;
      __stwb(&c.Q.F[(i * D + q) * N + j], a);
    }
    int u = 0;
#pragma unroll
    for (int a = 0; a < D; ++a)
#pragma unroll
      for (int b = a; b < D; ++b) Sg[u++] += row[a] * row[b];
  }
  // trial states that may leave the elastic interval get the return map in
  // k_project (it needs an SVD, whose registers would halve G2P's occupancy);
  // det F' = det(I + s G) det F
  if (c.plast == 1) {
    float A[D * D];
#pragma unroll
    for (int i = 0; i < D; ++i)
#pragma unroll
      for (int k = 0; k < D; ++k) A[i * D + k] = (i == k ? 1.f : 0.f) + s * G[i * D + k];
    if (!gram_within<D>(Sg, det<D>(A) * det<D>(F), 1.f - c.theta_c, 1.f + c.theta_s))
      c.proj[reserve_slot(&c.ctr[CTR_PROJ])] = j;
  }
}

// 3D G2P (adaptive_gimp.py:289-321) over the P2G work items: a CTA takes a
// contiguous range of them (up to CH particles of one 4^3 block each); when
// the block changes it stages the block's 6^3 node velocities in shared
// memory (two tiles alternate, so one barrier per block suffices: a thread
// that passed the previous barrier has finished reading the tile from two
// blocks ago), and each thread then computes one particle from the tile.
// Particles without a level (the extra bin) are copied unchanged.
template <int D, int CH>
__global__ void __launch_bounds__(CH, 1024 / CH) k_g2p(Batch B) {
  SCENE_CTA(B, MAP_G);
  constexpr int TN = (D == 2) ? 36 : 216;
  __shared__ float2 txy[2][TN];
  __shared__ float tz[2][(D == 3) ? TN : 1];
  const int nch = c.ctr[CTR_CHUNKS];
  const int per = (nch + nblk_ - 1) / nblk_;
  const int c0 = bid_ * per, c1 = min(nch, c0 + per);
  const long long N = c.N;
  int tb = 1, tl = -1, tk = -1;
  for (int ch = c0; ch < c1; ++ch) {
    const int4 wd = c.chunks[ch];
    const int i = threadIdx.x, j = wd.z + i;
    const bool mine = i < wd.w;
    if (wd.x < 0) {  // uniform over the CTA
      if (mine) copy_particle<D>(c, __ldg(&c.perm[j]), j);
      continue;
    }
    const int l = wd.x;
    const LevelDev& V = c.lev[l];
    int O[D];
    chunk_origin<D>(V, wd.y, O);
    // the particle's position and the fields read after the gather start
    // moving before the tile load, so both latencies overlap
    int p = 0;
    float xp[D];
    if (mine) {
      p = __ldg(&c.perm[j]);
#pragma unroll
      for (int d = 0; d < D; ++d) xp[d] = __ldg(&c.P.x[d * N + p]);
#pragma unroll
      for (int k = 0; k < D * D; ++k) asm volatile("prefetch.global.L1 [%0];" ::"l"(&c.P.F[k * N + p]));
      asm volatile("prefetch.global.L1 [%0];" ::"l"(&c.P.m[p]));
      asm volatile("prefetch.global.L1 [%0];" ::"l"(&c.P.g[p]));
      asm volatile("prefetch.global.L1 [%0];" ::"l"(&c.P.id[p]));
      if (c.plast == 1) asm volatile("prefetch.global.L1 [%0];" ::"l"(&c.P.Jp[p]));
    }
    if (l != tl || wd.y != tk) {  // uniform over the CTA
      tb ^= 1;
      tl = l;
      tk = wd.y;
      for (int t = threadIdx.x; t < TN; t += CH) {
        int I[D], r = t;
#pragma unroll
        for (int d = D - 1; d >= 0; --d) {
          I[d] = O[d] + r % 6;
          r /= 6;
        }
        float4 nd = make_float4(0.f, 0.f, 0.f, 0.f);
        if (in_store<D>(V, I)) nd = __ldg(&V.node[elem_of<D>(V, I)]);
        txy[tb][t] = make_float2(nd.x, nd.y);
        if (D == 3) tz[tb][t] = nd.z;
      }
      __syncthreads();
    }
    if (mine) g2p_staged<D>(c, l, p, j, xp, O, txy[tb], tz[tb]);
  }
}

// Snow return map (extension) of the particles G2P listed: the trial state
// written to Q is projected in place (or handed to the surrogate).
template <int D>
__global__ void __launch_bounds__(256) k_project(Batch B) {
  SCENE_CTA(B, MAP_G);
  if (c.plast != 1) return;
  const int n = c.ctr[CTR_PROJ];
  const long long N = c.N;
  SCENE_LOOP(s, n) {
    const int j = c.proj[s];
    float F[D * D];
#pragma unroll
    for (int k = 0; k < D * D; ++k) F[k] = c.Q.F[k * N + j];
    float jp = c.Q.Jp[j];
    snow_return_map<D>(c, F, jp, j);
#pragma unroll
    for (int k = 0; k < D * D; ++k) __stwb(&c.Q.F[k * N + j], F[k]);
    __stwb(&c.Q.Jp[j], jp);
  }
}

// ---------------------------------------------------------------------------
template <int D, int CH>
static void set_p2g_smem() {
  cudaFuncSetAttribute(k_p2g<D, CH>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)P2GLayout<D, CH>::bytes());
}

// CTAs of k_p2g<dim, chunk> that one SM holds at once (shared memory bound)
int p2g_resident(int dim, int chunk) {
  int n = 0;
  auto occ = [&](auto k, int ch, size_t smem) { cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k, ch, smem); };
  if (dim == 2) {
    switch (chunk) {
      case 64: occ(k_p2g<2, 64>, 64, P2GLayout<2, 64>::bytes()); break;
      case 128: occ(k_p2g<2, 128>, 128, P2GLayout<2, 128>::bytes()); break;
      case 512: occ(k_p2g<2, 512>, 512, P2GLayout<2, 512>::bytes()); break;
      default: occ(k_p2g<2, 256>, 256, P2GLayout<2, 256>::bytes()); break;
    }
  } else {
    switch (chunk) {
      case 64: occ(k_p2g<3, 64>, 64, P2GLayout<3, 64>::bytes()); break;
      case 128: occ(k_p2g<3, 128>, 128, P2GLayout<3, 128>::bytes()); break;
      case 512: occ(k_p2g<3, 512>, 512, P2GLayout<3, 512>::bytes()); break;
      default: occ(k_p2g<3, 256>, 256, P2GLayout<3, 256>::bytes()); break;
    }
  }
  return n > 0 ? n : 1;
}

void prepare_transfer_kernels() {
  set_p2g_smem<2, 64>();
  set_p2g_smem<2, 128>();
  set_p2g_smem<2, 256>();
  set_p2g_smem<3, 64>();
  set_p2g_smem<3, 128>();
  set_p2g_smem<3, 256>();
  set_p2g_smem<2, 512>();
  set_p2g_smem<3, 512>();
}

template <int D>
static void launch_p2g(const BatchLaunch& bl, cudaStream_t s, bool pdl) {
  const int G = bl.nct[MAP_P];
  switch (bl.chunk) {
    case 64: launch_k(pdl, k_p2g<D, 64>, G, 64, P2GLayout<D, 64>::bytes(), s, bl.b); break;
    case 128: launch_k(pdl, k_p2g<D, 128>, G, 128, P2GLayout<D, 128>::bytes(), s, bl.b); break;
    case 512: launch_k(pdl, k_p2g<D, 512>, G, 512, P2GLayout<D, 512>::bytes(), s, bl.b); break;
    default: launch_k(pdl, k_p2g<D, 256>, G, 256, P2GLayout<D, 256>::bytes(), s, bl.b); break;
  }
}

template <int D>
static void launch_g2p(const BatchLaunch& bl, cudaStream_t s, bool pdl) {
  const int G = bl.nct[MAP_G];
  if constexpr (D == 2) {
    launch_k(pdl, k_g2p_gather<D>, G, 256, 0, s, bl.b);
  } else {
    switch (bl.chunk) {
      case 64: launch_k(pdl, k_g2p<D, 64>, G, 64, 0, s, bl.b); break;
      case 128: launch_k(pdl, k_g2p<D, 128>, G, 128, 0, s, bl.b); break;
      case 512: launch_k(pdl, k_g2p<D, 512>, G, 512, 0, s, bl.b); break;
      default: launch_k(pdl, k_g2p<D, 256>, G, 256, 0, s, bl.b); break;
    }
  }
}

template <int D>
void launch_transfer(const BatchLaunch& bl, cudaStream_t s, cudaEvent_t* ev) {
  const int G = bl.nct[MAP_G];
  const bool pdl = bl.pdl && !ev;
  launch_p2g<D>(bl, s, pdl);
  if (bl.side) cudaStreamWaitEvent(s, bl.join, 0);  // k_ghost_tj's node mask
  if (ev) cudaEventRecord(ev[4], s);
  // the first launch after the join is a plain one
  bool first = true;
  for (int l = bl.maxL - 1; l >= 1; --l, first = false) {
    if (staged_transfers<D>())
      launch_k(pdl && !(first && bl.side), k_restrict<D>, bl.nct[MAP_T], Stage<D>::PER, 0, s, bl.b, l);
    else
      launch_k(pdl && !(first && bl.side), k_restrict_gather<D>, G, 256, 0, s, bl.b, l);
  }
  if (ev) cudaEventRecord(ev[5], s);
  // with more than one level grid_op runs inside the restriction into level 0
  // and the prolongations
  if (bl.maxL == 1) launch_k(pdl && !bl.side, k_gridop<D>, G, 256, 0, s, bl.b);
  if (ev) cudaEventRecord(ev[6], s);
  for (int l = 1; l < bl.maxL; ++l) {
    if (staged_transfers<D>())
      launch_k(pdl, k_prolong<D>, bl.nct[MAP_T], Stage<D>::PER, 0, s, bl.b, l);
    else
      launch_k(pdl, k_prolong_gather<D>, G, 256, 0, s, bl.b, l);
  }
  if (ev) cudaEventRecord(ev[7], s);
  launch_g2p<D>(bl, s, pdl);
  if (bl.any_plastic) launch_k(pdl, k_project<D>, G, 256, 0, s, bl.b);
  if (bl.sur) {
    launch_mlp_forward_dev(bl.mlp_packed, bl.mlp_P, bl.sur_X, bl.sur_Y, bl.sur_n, bl.sur_cap, bl.sur_err, bl.sms, s);
    k_sur_finish<D><<<G, 256, 0, s>>>(bl.b, bl.sur_meta, bl.sur_Y, bl.sur_n);
  }
  if (ev) cudaEventRecord(ev[8], s);
}

template void launch_transfer<2>(const BatchLaunch&, cudaStream_t, cudaEvent_t*);
template void launch_transfer<3>(const BatchLaunch&, cudaStream_t, cudaEvent_t*);

}  // namespace agimp

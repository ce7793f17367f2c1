// Topology and binning kernels of the adaptive GIMP substep.
//
// Reference steps (adaptive_gimp.py, g1n0st/adaptive-gimp):
//   324-326 deactivate_all            -> k_clear (only the blocks the previous
//                                         substep touched)
//   72-96   activate_cell_*           -> k_touch_activate
//   98-124  _mark_hier_ / _split_hier_-> k_mark_hier + k_resolve
//   142-153 _activate_mask            -> k_resolve (same pass)
//   155-187 ghost / T-junction        -> k_ghost_tj (all levels in one pass)
//   189-216 level_mapping             -> k_bin + k_offsets + k_scatter
//
// The reference runs its sparse sweeps level by level.  Here each pass covers
// every level at once: the reads each pass depends on are not written in the
// same pass (CULLING bits in k_resolve, == ACTIVATED tests in k_ghost_tj), so
// the result does not depend on the order.  The one order-dependent bit in the
// reference (GHOST on a node that also gets T_JUNCTION, adaptive_gimp.py:174
// against 182-183) never changes a node's class.
#include "common.cuh"

namespace agimp {

template <int D>
__device__ __forceinline__ void cell_or(const Ctx& c, int l, const int* I, uint32_t bits) {
  const LevelDev& V = c.lev[l];
  if (!in_store<D>(V, I)) {
    set_err(c, ERR_OOB);
    return;
  }
  uint32_t* w = &V.cell[elem_of<D>(V, I)];
  if ((*w & bits) != bits) atomicOr(w, bits);
}

template <int D>
__device__ __forceinline__ uint32_t cell_get(const Ctx& c, int l, const int* I) {
  const LevelDev& V = c.lev[l];
  if (!in_store<D>(V, I)) return 0u;
  return V.cell[elem_of<D>(V, I)];
}

// ---------------------------------------------------------------------------
// Clear everything the previous substep wrote (its active blocks), reset the
// per-substep counters.
template <int D>
__global__ void k_clear(Batch B) {
  SCENE_CTA(B, MAP_G);
  if (bid_ == 0 && threadIdx.x == 0) {
    c.ctr[CTR_TOUCH] = 0;
    c.ctr[CTR_BINCUR] = 0;
    c.ctr[CTR_CHUNKS] = 0;
    c.ctr[CTR_UNBIN] = 0;
    c.ctr[CTR_SUR] = 0;
    c.ctr[CTR_SURFB] = 0;
    if (c.sur) *c.sur_ctr = 0;  // a batch's shared slot counter (every scene clears it)
    c.ctr[CTR_PROJ] = 0;
    c.ctr[CTR_FULL] = 0;
  }
  __shared__ BlockRanges br;
  load_block_ranges(c, br);
  const long long tot = total_elems_r(br, 0, c.L, D);
  SCENE_LOOP(e, tot) {
    int l, loc;
    long long blk;
    decode_elem_r<D>(c, br, 0, c.L, e, l, blk, loc);
    const LevelDev& V = c.lev[l];
    const long long idx = (blk << (2 * D)) | loc;
    V.cell[idx] = 0u;
    V.node[idx] = make_float4(0.f, 0.f, 0.f, 0.f);
    if (D == 3 && l < c.L - 1) V.nm[idx] = 0u;
    if (loc == 0) V.bmap[blk] = -1;
    int I[D];
    elem_coords<D>(V, blk, loc, I);
    const int s = c.L - 1 - l;
    int P[D];
    bool ok = true;
#pragma unroll
    for (int d = 0; d < D; ++d) {
      P[d] = I[d] * (1 << s);
      ok = ok && P[d] >= 0 && P[d] <= c.sz;
    }
    if (ok) c.nmask[elem_of<D>(c.lev[c.L - 1], P)] = 0u;
  }
}

// ---------------------------------------------------------------------------
// Per particle: record the finest block holding it (for the active-block
// lists) and activate cells, dynamically from g_p (adaptive_gimp.py:87-96) or
// through the level map (adaptive_gimp.py:72-85).
// the tabulated level map at finest cell I: bits 0-3 the level, bit 6 "no
// activation"; outside the table: an error and level L-1 without activation
template <int D>
__device__ __forceinline__ int map_entry(const Ctx& c, const int* I) {
  long long o = 0;
#pragma unroll
  for (int d = 0; d < D; ++d) {
    int a = I[d] + c.map_h;
    if (a < 0 || a >= c.map_n) {
      set_err(c, ERR_MAP_OOB);
      return (c.L - 1) | 64;
    }
    o = o * c.map_n + a;
  }
  return c.map[o];
}

template <int D>
__device__ __forceinline__ int grid_init(const Ctx& c, const int* I) {
  // grid_initializer(sim, I) with the tabulated map: activate_cell(l, I)
  // (adaptive_gimp.py:68-70) unless bit 6 is set; returns l.
  const int e = map_entry<D>(c, I);
  const int l = e & 15;
  if (!(e & 64)) {
    int A[D];
    const int s = c.L - 1 - l;
#pragma unroll
    for (int d = 0; d < D; ++d) A[d] = I[d] >> s;
    cell_or<D>(c, l, A, ACT);
  }
  return l;
}

// one particle slot p (may be >= N)
template <int D>
__device__ __forceinline__ void touch_one(const Ctx& c, int p) {
  const bool valid = p < c.N;
  float xp[D];
  bool esc = !valid;
#pragma unroll
  for (int d = 0; d < D; ++d) {
    xp[d] = valid ? c.P.x[(long long)d * c.N + p] : 0.f;
    if (!(xp[d] >= 0.f && xp[d] < 1.f)) esc = true;
  }
  if (valid && esc) set_err(c, ERR_ESCAPED);
  if (esc) return;
  // the finest cell holding the particle and its block (the touched block)
  const LevelDev& Vf = c.lev[c.L - 1];
  int pc[D];
  unsigned b = 0;
#pragma unroll
  for (int d = 0; d < D; ++d) {
    pc[d] = (int)(xp[d] * (float)c.sz);
    b = b * (unsigned)Vf.nb + (unsigned)((pc[d] >> 2) + 1);
  }
  const int key = (int)b;
  // reach of this particle's activations, recorded with its finest block: 1
  // in dynamic mode, L - (level of its level-map cell) in static mode
  unsigned reach = 1;
  if (!c.is_static) {
    const int gl = c.P.g[p];
    const bool ok = gl >= 0 && gl < c.L;
    int base[D];
    long long bk = ok ? gl : -1;
    if (ok) {
      const float inv = (float)(c.coarsest << gl);
#pragma unroll
      for (int d = 0; d < D; ++d) {
        base[d] = (int)(xp[d] * inv + 0.5f) - 1;
        bk = bk * (c.sz + 4) + (base[d] + 2);
      }
    }
    // particles with the same (level, base cell) activate the same 2^d
    // cells: the lanes of such a group share the activations
    const int lane = threadIdx.x & 31;
    const unsigned g = __match_any_sync(__activemask(), bk);
    const int r = __popc(g & ((1u << lane) - 1u)), n = __popc(g);
    if (ok)
      for (int a = r; a < (1 << D); a += n) {
        int I[D];
#pragma unroll
        for (int d = 0; d < D; ++d) I[d] = base[d] + ((a >> (D - 1 - d)) & 1);
        cell_or<D>(c, gl, I, ACT);
      }
  } else {
    // The lookups depend on the finest base cell fb, then on (level, base):
    // lanes of a warp that share them would repeat identical lookups and
    // activations, so the first lane of each group does them for the group.
    // The 4^d cells around fb (adaptive_gimp.py:77-78) are looked up by
    // k_dilate, once per cell, from the base cells recorded here.
    const unsigned act = __activemask();
    const int lane = threadIdx.x & 31;
    int fb[D];
    long long fk = 0;
#pragma unroll
    for (int d = 0; d < D; ++d) {
      fb[d] = (int)(xp[d] * (float)c.sz + 0.5f) - 1;
      fk = fk * (c.sz + 4) + (fb[d] + 2);
    }
    const unsigned g1 = __match_any_sync(act, fk);
    const int lead1 = __ffs(g1) - 1;
    int level = 0;
    // fb's own activation is one of its window's (k_dilate): only the level here
    if (lane == lead1) level = map_entry<D>(c, fb) & 15;
    {
      // fb lies in [T0 - 1, T0 + 3] on every axis (T0: the touched block's
      // first cell); bit (j_1, .., j_{d-1}) of word j_0 with j = fb - T0 + 1
      int j[D];
#pragma unroll
      for (int d = 0; d < D; ++d) j[d] = fb[d] - (pc[d] & ~3) + 1;
      const unsigned wi = (D == 2) ? (unsigned)key : (unsigned)key * 5u + (unsigned)j[0];
      const unsigned bit = (D == 2) ? 1u << (5 * j[0] + j[1]) : 1u << (5 * j[1] + j[D - 1]);
      const unsigned g3 = __match_any_sync(act, wi);
      const unsigned bits = __reduce_or_sync(g3, bit);
      uint32_t* w = &c.touch_occ[wi];
      if (lane == __ffs(g3) - 1 && (*w & bits) != bits) atomicOr(w, bits);
    }
    level = __shfl_sync(g1, level, lead1);
    reach = (unsigned)(c.L - level);
    const float inv = (float)(c.coarsest << level);
    int base[D];
    long long bk = level;
#pragma unroll
    for (int d = 0; d < D; ++d) {
      base[d] = (int)(xp[d] * inv + 0.5f) - 1;
      bk = bk * (c.sz + 4) + (base[d] + 2);
    }
    // at the finest level base = fb: its 2^d corners are cells of fb's window,
    // so a warp whose particles all map to the finest level skips this part
    if (!__all_sync(act, level == c.L - 1)) {
      const unsigned g2 = __match_any_sync(act, bk);
      const int r2 = __popc(g2 & ((1u << lane) - 1u)), n2 = __popc(g2);
#pragma unroll 1
      for (int a = level < c.L - 1 ? r2 : (1 << D); a < (1 << D); a += n2) {
        int I[D];
#pragma unroll
        for (int d = 0; d < D; ++d) I[d] = (base[d] + ((a >> (D - 1 - d)) & 1)) * (1 << (c.L - 1 - level));
        grid_init<D>(c, I);
      }
    }
  }
  // record the finest block for the active-block lists (first toucher appends)
  const unsigned grp = __match_any_sync(__activemask(), key);
  const unsigned rmax = __reduce_max_sync(grp, reach);
  if ((int)(threadIdx.x & 31) == __ffs(grp) - 1 && c.touch_flag[key] < rmax &&
      atomicMax(&c.touch_flag[key], rmax) == 0u) {
    const int i = reserve_slot(&c.ctr[CTR_TOUCH]);
    c.touch_list[i] = key;
  }
}

template <int D>
__global__ void k_touch_activate(Batch B) {
  SCENE_CTA(B, MAP_G);
  // the active-block counts were read by k_clear; k_dilate rebuilds them
  if (bid_ == 0 && threadIdx.x < MAXL) c.ctr[CTR_LEVEL + threadIdx.x] = 0;
  SCENE_PARTICLES(p0) touch_one<D>(c, p0 + (int)threadIdx.x);
}

// ---------------------------------------------------------------------------
// Active-block lists: level l gets the blocks within R_l blocks of each
// touched finest block (shifted to that level).  Dynamic activation, culling,
// ghost/T marking and the transfers stay within 2 cells of a particle at every
// level, so R_l = 1.  A static level-map lookup (adaptive_gimp.py:82-85) lands
// up to two cells of the level the map gives at the particle (lv) away, i.e.
// rho = max(2, 2^(L - lv)) finest cells, and activates a cell of any level
// there; with the ghost / T / corner reach on top (6 cells), level l needs
// ceil((ceil(rho / 2^(L-1-l)) + 6) / 4) blocks.  The touched block records
// L - lv of its coarsest-mapped particle (`reach`; 1 in dynamic mode).
__device__ __forceinline__ int dilate_radius(const Ctx& c, int l, unsigned reach) {
  if (!c.is_static) return 1;
  const int rho = max(2, 1 << (int)reach);  // reach = L - lv
  const int div = 1 << (c.L - 1 - l);
  return ((rho + div - 1) / div + 9) / 4;
}

// Static mode: grid_initializer on the 4^d cells f_base + [-1, 2]^d of every
// particle (adaptive_gimp.py:77-78), once per distinct cell.  k_touch_activate
// recorded the particles' base cells per touched block (fb - T0 + 1 in
// [0, 4]^d); a cell X = T0 + r (r in [-2, 5]^d) is looked up when a recorded
// base cell lies in [X - 2, X + 1] on every axis.
// Blocks next to each other may both look up a cell of their common border;
// the second lookup finds the cell already set.
__device__ __forceinline__ unsigned axis_window(int r) {
  const int lo = max(0, r - 1), hi = min(4, r + 2);
  return lo > hi ? 0u : ((2u << hi) - (1u << lo));
}

// bits j of a 5-bit axis mask m, spread to bit 5 j (one 5-bit row per j)
__device__ __forceinline__ unsigned spread_rows(unsigned m) {
  unsigned o = 0;
#pragma unroll
  for (int j = 0; j < 5; ++j)
    if (m >> j & 1u) o |= 1u << (5 * j);
  return o;
}

template <int D>
__device__ __forceinline__ void static_window(const Ctx& c, int key, const int* fb, int lane) {
  constexpr int W = (D == 2) ? 1 : 5;
  uint32_t occ[W];
#pragma unroll
  for (int w = 0; w < W; ++w) occ[w] = c.touch_occ[(long long)key * W + w];
  for (int r = lane; r < (1 << (3 * D)); r += 32) {
    int X[D];
    unsigned m[D];
#pragma unroll
    for (int d = 0; d < D; ++d) {
      const int rel = ((r >> (3 * (D - 1 - d))) & 7) - 2;
      X[d] = fb[d] * 4 + rel;
      m[d] = axis_window(rel);
    }
    // recorded base cells inside the window of X
    const unsigned plane = m[D - 1] * spread_rows(m[D - 2]);
    bool hit;
    if (D == 2) {
      hit = (occ[0] & plane) != 0u;
    } else {
      hit = false;
#pragma unroll
      for (int j = 0; j < 5; ++j) hit = hit || ((m[0] >> j & 1u) && (occ[j] & plane));
    }
    if (hit) grid_init<D>(c, X);
  }
}

template <int D>
__global__ void k_dilate(Batch B) {
  SCENE_CTA(B, MAP_G);
  // one warp per touched finest block; its lanes walk the block's
  // (2R_l + 1)^d neighbourhood at every level
  const int lane = threadIdx.x & 31;
  const int wid = bid_ * (blockDim.x >> 5) + (threadIdx.x >> 5), nw = nblk_ * (blockDim.x >> 5);
  const LevelDev& Vf = c.lev[c.L - 1];
  const int ntouch = c.ctr[CTR_TOUCH];
  for (int t = wid; t < ntouch; t += nw) {
    const int key = c.touch_list[t];
    const unsigned reach = c.touch_flag[key];
    int fb[D];
    unsigned k = (unsigned)key;
#pragma unroll
    for (int d = D - 1; d >= 0; --d) {
      fb[d] = (int)(k % (unsigned)Vf.nb) - 1;
      k /= (unsigned)Vf.nb;
    }
    for (int l = 0; l < c.L; ++l) {
      const int R = dilate_radius(c, l, reach);
      const int w = 2 * R + 1;
      const int items = (D == 2) ? w * w : w * w * w;
      const LevelDev& V = c.lev[l];
      const int s = c.L - 1 - l;
      if (l < c.L - 1) {
        // the touched blocks under one block of this level share its
        // neighbourhood: only the first with at least this radius walks it
        unsigned ba = 0;
#pragma unroll
        for (int d = 0; d < D; ++d) ba = ba * (unsigned)V.nb + (unsigned)((fb[d] >> s) + 1);
        int done = 0;
        if (lane == 0) done = atomicMax(&V.dflag[ba], (unsigned)R + 1u) >= (unsigned)R + 1u;
        if (__shfl_sync(0xffffffffu, done, 0)) continue;
      }
      for (int r = lane; r < items; r += 32) {
        int tt = r;
        unsigned b = 0;
        bool ok = true;
        int cb[D];
#pragma unroll
        for (int d = D - 1; d >= 0; --d) {
          cb[d] = (fb[d] >> s) + (tt % w - R) + 1;
          tt /= w;
          ok = ok && cb[d] >= 0 && cb[d] < V.nb;
        }
        if (!ok) continue;  // beyond the stored lattice: nothing can be written there
#pragma unroll
        for (int d = 0; d < D; ++d) b = b * (unsigned)V.nb + (unsigned)cb[d];
        int* bm = &V.bmap[b];
        if (*bm == -1 && atomicCAS(bm, -1, -2) == -1) {
          const int i = reserve_slot(&c.ctr[CTR_LEVEL + l]);
          V.blist[i] = (int)b;
          *bm = i;
        }
      }
    }
    if (c.is_static) static_window<D>(c, key, fb, lane);
  }
}

// ---------------------------------------------------------------------------
// _mark_hier_ for every level l >= 1 (adaptive_gimp.py:98-109): an ACTIVATED
// cell whose finest ACTIVATED ancestor sits at level l0 marks CULLING on its
// ancestors at levels l0..l-1.  Only ACTIVATED bits are read and only CULLING
// bits written, so all levels run in one pass.
template <int D>
__global__ void k_mark_hier(Batch B) {
  SCENE_CTA(B, MAP_G);
  if (c.is_static) return;  // static mode has no culling (adaptive_gimp.py:335-337)
  __shared__ BlockRanges br;
  load_block_ranges(c, br);
  const long long tot = total_elems_r(br, 1, c.L, D);
  SCENE_LOOP(e, tot) {
    int l, loc;
    long long blk;
    decode_elem_r<D>(c, br, 1, c.L, e, l, blk, loc);
    const LevelDev& V = c.lev[l];
    const uint32_t v = V.cell[(blk << (2 * D)) | loc];
    if (!(v & ACT)) continue;
    int I[D];
    elem_coords<D>(V, blk, loc, I);
    int l0 = -1;
    for (int q = 0; q < l; ++q) {
      int A[D];
#pragma unroll
      for (int d = 0; d < D; ++d) A[d] = I[d] >> (l - q);
      if (cell_get<D>(c, q, A) & ACT) l0 = q;
    }
    if (l0 < 0) continue;
    for (int q = l0; q < l; ++q) {
      int A[D];
#pragma unroll
      for (int d = 0; d < D; ++d) A[d] = I[d] >> (l - q);
      cell_or<D>(c, q, A, CUL);
    }
  }
}

// ---------------------------------------------------------------------------
// _split_hier_ for all levels (adaptive_gimp.py:111-118) resolved in one pass:
// a cell with CULLING is emptied; a cell whose parent has CULLING becomes
// ACTIVATED.  CULLING bits are not written here, so the pass is order-free.
// Cells that end exactly ACTIVATED then mark their corner nodes
// (_activate_mask, adaptive_gimp.py:142-149).  The CULLING bit itself stays
// set until the next substep clears the block; readback masks it out.
template <int D>
__global__ void k_resolve(Batch B) {
  SCENE_CTA(B, MAP_G);
  // k_dilate has read the touched blocks' reach: clear the flags for the next
  // substep (they are read again only by k_touch_activate)
  SCENE_LOOP(t, c.ctr[CTR_TOUCH]) {
    const int key = c.touch_list[t];
    c.touch_flag[key] = 0u;
    if (c.is_static)
      for (int w = 0; w < ((D == 2) ? 1 : 5); ++w) c.touch_occ[(long long)key * ((D == 2) ? 1 : 5) + w] = 0u;
    // k_dilate's per-ancestor marks of this touched block
    const LevelDev& Vf = c.lev[c.L - 1];
    int fb[D];
    unsigned k = (unsigned)key;
#pragma unroll
    for (int d = D - 1; d >= 0; --d) {
      fb[d] = (int)(k % (unsigned)Vf.nb) - 1;
      k /= (unsigned)Vf.nb;
    }
    for (int l = 0; l < c.L - 1; ++l) {
      const LevelDev& V = c.lev[l];
      const int s = c.L - 1 - l;
      unsigned ba = 0;
#pragma unroll
      for (int d = 0; d < D; ++d) ba = ba * (unsigned)V.nb + (unsigned)((fb[d] >> s) + 1);
      if (V.dflag[ba]) V.dflag[ba] = 0u;
    }
  }
  __shared__ BlockRanges br;
  load_block_ranges(c, br);
  const long long tot = total_elems_r(br, 0, c.L, D);
  SCENE_LOOP(e, tot) {
    int l, loc;
    long long blk;
    decode_elem_r<D>(c, br, 0, c.L, e, l, blk, loc);
    const LevelDev& V = c.lev[l];
    const long long idx = (blk << (2 * D)) | loc;
    const uint32_t v = V.cell[idx];
    int I[D];
    bool have_I = false;
    uint32_t nv = v;
    if (!c.is_static) {
      bool pc = false;
      if (l > 0) {
        elem_coords<D>(V, blk, loc, I);
        have_I = true;
        int A[D];
#pragma unroll
        for (int d = 0; d < D; ++d) A[d] = I[d] >> 1;
        pc = (cell_get<D>(c, l - 1, A) & CUL) != 0u;
      }
      if (v & CUL)
        nv = v & ~ACT;
      else if ((v & ACT) || pc)
        nv = v | ACT;
      if (nv != v) V.cell[idx] = nv;
    }
    if (nv != ACT) continue;
    if (!have_I) elem_coords<D>(V, blk, loc, I);
#pragma unroll
    for (int a = 0; a < (1 << D); ++a) {
      int J[D];
#pragma unroll
      for (int d = 0; d < D; ++d) J[d] = I[d] + ((a >> (D - 1 - d)) & 1);
      nm_or<D>(c, l, J, ACT);
    }
  }
}

// ---------------------------------------------------------------------------
// _mark_ghost_and_T_junction for every level (adaptive_gimp.py:155-187).
template <int D>
__global__ void k_ghost_tj(Batch B) {
  SCENE_CTA(B, MAP_G);
  __shared__ BlockRanges br;
  load_block_ranges(c, br);
  const long long tot = total_elems_r(br, 0, c.L, D);
  SCENE_LOOP(e, tot) {
    int l, loc;
    long long blk;
    decode_elem_r<D>(c, br, 0, c.L, e, l, blk, loc);
    const LevelDev& V = c.lev[l];
    if (V.cell[(blk << (2 * D)) | loc] != ACT) continue;
    int I[D];
    elem_coords<D>(V, blk, loc, I);
    const int lsz = V.size;
#pragma unroll 1
    for (int f = 0; f < 2 * D; ++f) {
      const int ax = f >> 1, side = f & 1;
      int I1[D];
#pragma unroll
      for (int d = 0; d < D; ++d) I1[d] = I[d];
      I1[ax] += side ? -1 : 1;
      bool inr = true;
#pragma unroll
      for (int d = 0; d < D; ++d) inr = inr && I1[d] >= 0 && I1[d] < lsz;
      if (!inr) continue;
      if (V.cell[elem_of<D>(V, I1)] == ACT) continue;
      int lp = -1;  // _heriarchical_check
      for (int q = 0; q <= l; ++q) {
        int A[D];
#pragma unroll
        for (int d = 0; d < D; ++d) A[d] = I1[d] >> (l - q);
        if (cell_get<D>(c, q, A) == ACT) lp = q;
      }
      if (lp < 0) continue;
      const int md = (1 << (l - lp)) - 1;
#pragma unroll
      for (int a = 0; a < (1 << D); ++a) {
        int J[D];
        bool off = false;
        bool face = true;
#pragma unroll
        for (int d = 0; d < D; ++d) {
          const int bit = (a >> (D - 1 - d)) & 1;
          if (d == ax && bit != side) face = false;
          J[d] = I1[d] + bit;
          off = off || (J[d] & md) != 0;
        }
        if (face && off) nm_or<D>(c, l, J, TJ);
      }
      for (int l0 = lp + 1; l0 <= l; ++l0) {
        int Ip[D];
#pragma unroll
        for (int d = 0; d < D; ++d) Ip[d] = I1[d] >> (l - l0);
        cell_or<D>(c, l0, Ip, GHO);
#pragma unroll
        for (int a = 0; a < (1 << D); ++a) {
          int J[D];
#pragma unroll
          for (int d = 0; d < D; ++d) J[d] = Ip[d] + ((a >> (D - 1 - d)) & 1);
          if (nm_get<D>(c, l0, J) == 0u) nm_or<D>(c, l0, J, GHO);
        }
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Per-level node masks for the levels below the finest (3D scenes, whose
// level transfers copy them by whole blocks): node I of level l gets
// node_mask[_map(l, I)] (adaptive_gimp.py:126-128), 0 outside [0, size].
// Runs after ghost / T-junction marking, the last writer of the node mask.
template <int D>
__global__ void k_level_masks(Batch B) {
  SCENE_CTA(B, MAP_G);
  __shared__ BlockRanges br;
  load_block_ranges(c, br);
  const long long tot = total_elems_r(br, 0, c.L - 1, D);
  SCENE_LOOP(e, tot) {
    int l, loc;
    long long blk;
    decode_elem_r<D>(c, br, 0, c.L - 1, e, l, blk, loc);
    const LevelDev& V = c.lev[l];
    int I[D];
    elem_coords<D>(V, blk, loc, I);
    bool inr = true;
#pragma unroll
    for (int d = 0; d < D; ++d) inr = inr && I[d] >= 0 && I[d] <= V.size;
    V.nm[(blk << (2 * D)) | loc] = inr ? nm_get<D>(c, l, I) : 0u;
  }
}

// ---------------------------------------------------------------------------
// level_mapping (adaptive_gimp.py:189-216): fl_p = finest level with an
// ACTIVATED cell among the 2^d cells around the particle; bin = (fl_p, block
// of base).  Particles without a level go to one extra bin after all block
// bins, so that every particle gets a slot in the new order.  The rank inside
// the bin comes from a warp-aggregated atomic.
// lb: lb[l] = bins of the levels below l (block bins are numbered level by
// level); lb[L] = all block bins, the index of the extra bin
template <int D>
__device__ __forceinline__ void bin_one(const Ctx& c, int p, const int* lb) {
  const int lane = threadIdx.x & 31;
  int bin = -1;
  if (p < c.N) {
    float xp[D];
    bool esc = false;
#pragma unroll
    for (int d = 0; d < D; ++d) {
      xp[d] = c.P.x[(long long)d * c.N + p];
      if (!(xp[d] >= 0.f && xp[d] < 1.f)) esc = true;
    }
    int fl = -1;
    if (!esc) {
      // the finest level with an ACTIVATED cell: search from the finest down
      for (int l = c.L - 1; l >= 0 && fl < 0; --l) {
        const float inv = (float)(c.coarsest << l);
        int base[D];
#pragma unroll
        for (int d = 0; d < D; ++d) base[d] = (int)(xp[d] * inv + 0.5f) - 1;
        const LevelDev& V = c.lev[l];
        const Corners<D> K(V, base);
#pragma unroll
        for (int a = 0; a < (1 << D); ++a)
          if (K.ok(a) && V.cell[K.idx(a)] == ACT) fl = l;
      }
      if (fl >= 0) {
        const float inv = (float)(c.coarsest << fl);
        const LevelDev& V = c.lev[fl];
        long long b = 0;
        bool ok = true;
        int cell = 0;
#pragma unroll
        for (int d = 0; d < D; ++d) {
          const int base = ((int)(xp[d] * inv + 0.5f)) - 1;
          const int cb = (base >> 2) + 1;
          ok = ok && cb >= 0 && cb < V.nb;
          b = b * V.nb + cb;
          cell = (cell << 2) | (base & 3);  // base cell inside the block
        }
        const int bi = ok ? V.bmap[b] : -1;
        if (bi < 0) {
          set_err(c, ERR_NOBIN);
          fl = -1;
        } else {
          bin = ((lb[fl] + bi) << (2 * D)) | cell;
        }
      }
    }
    if (fl < 0) bin = lb[c.L] << (2 * D);  // the extra bin
    c.P.fl[p] = fl;
  }
  // bin sizes and the rank inside the (bin, cell): warp-aggregated atomics
  {
    const int b = bin >= 0 ? bin >> (2 * D) : -1;
    const unsigned gb = __match_any_sync(0xffffffffu, b);
    if (b >= 0 && lane == __ffs(gb) - 1) atomicAdd(&c.bin_count[b], __popc(gb));
  }
  const unsigned grp = __match_any_sync(0xffffffffu, bin);
  const int leader = __ffs(grp) - 1;
  const int rank = __popc(grp & ((1u << lane) - 1u));
  int base = 0;
  if (bin >= 0 && lane == leader) base = atomicAdd(&c.cell_count[bin], __popc(grp));
  base = __shfl_sync(0xffffffffu, base, leader);
  if (bin >= 0) {
    c.bin_of[p] = bin;
    c.rank_of[p] = base + rank;
  }
}

template <int D>
__global__ void k_bin(Batch B) {
  SCENE_CTA(B, MAP_G);
  __shared__ int lb[MAXL + 1];
  if (threadIdx.x == 0) {
    int t = 0;
    for (int q = 0; q < c.L; ++q) {
      lb[q] = t;
      t += c.ctr[CTR_LEVEL + q];
    }
    lb[c.L] = t;
  }
  __syncthreads();
  SCENE_PARTICLES(p0) bin_one<D>(c, p0 + (int)threadIdx.x, lb);
}

// ---------------------------------------------------------------------------
// Bin storage: each CTA scans 1024 bins, reserves their particles and work
// items with one atomic each, and writes the work-item descriptors.  Bins of
// different CTAs land in any order; a bin's particles stay contiguous.
__device__ __forceinline__ int2 block_incl_scan2(int a, int b, int2* warp_sums) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int ya = __shfl_up_sync(0xffffffffu, a, o);
    const int yb = __shfl_up_sync(0xffffffffu, b, o);
    if (lane >= o) {
      a += ya;
      b += yb;
    }
  }
  if (lane == 31) warp_sums[w] = make_int2(a, b);
  __syncthreads();
  if (w == 0) {
    const int nw = blockDim.x >> 5;
    int2 s = lane < nw ? warp_sums[lane] : make_int2(0, 0);
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int ya = __shfl_up_sync(0xffffffffu, s.x, o);
      const int yb = __shfl_up_sync(0xffffffffu, s.y, o);
      if (lane >= o) {
        s.x += ya;
        s.y += yb;
      }
    }
    if (lane < nw) warp_sums[lane] = s;
  }
  __syncthreads();
  if (w > 0) {
    const int2 pre = warp_sums[w - 1];
    a += pre.x;
    b += pre.y;
  }
  return make_int2(a, b);
}

template <int D>
__global__ void __launch_bounds__(1024) k_offsets(Batch B) {
  SCENE_CTA(B, MAP_O);
  __shared__ int2 warp_sums[32];
  __shared__ int2 s_base;
  const int CH = c.chunk;
  long long nblk = 0;
  for (int q = 0; q < c.L; ++q) nblk += c.ctr[CTR_LEVEL + q];
  const long long nb = nblk + 1;  // block bins + the extra bin of particles without a level
  for (long long t0 = (long long)bid_ * blockDim.x; t0 < nb; t0 += (long long)nblk_ * blockDim.x) {
    const long long b = t0 + threadIdx.x;
    int cnt = 0;
    if (b < nb) {
      cnt = c.bin_count[b];
      if (cnt) c.bin_count[b] = 0;
    }
    const int nch = (cnt + CH - 1) / CH;
    const int2 inc = block_incl_scan2(cnt, nch, warp_sums);
    if (threadIdx.x == blockDim.x - 1) {
      s_base.x = inc.x ? atomicAdd(&c.ctr[CTR_BINCUR], inc.x) : 0;
      s_base.y = inc.y ? atomicAdd(&c.ctr[CTR_CHUNKS], inc.y) : 0;
    }
    __syncthreads();
    if (cnt > 0) {
      const int start = s_base.x + inc.x - cnt;
      c.bin_start[b] = start;
      c.full_bins[reserve_slot(&c.ctr[CTR_FULL])] = (int)b;
      const int ch0 = s_base.y + inc.y - nch;
      int l = -1, blk = 0;  // level -1 marks the extra bin
      if (b < nblk) {
        l = 0;
        long long r = b;
        while (l < c.L - 1 && r >= c.ctr[CTR_LEVEL + l]) {
          r -= c.ctr[CTR_LEVEL + l];
          ++l;
        }
        blk = c.lev[l].blist[r];
      } else {
        c.ctr[CTR_UNBIN] = cnt;
      }
      for (int j = 0; j < nch; ++j) c.chunks[ch0 + j] = make_int4(l, blk, start + j * CH, min(CH, cnt - j * CH));
    }
    __syncthreads();
  }
}

// Offsets of the cells inside each bin (the bin's particles are stored in
// cell order); one warp per bin, cell counts cleared for the next substep.
template <int D>
__global__ void k_cell_offsets(Batch B) {
  SCENE_CTA(B, MAP_G);
  constexpr int NC = 1 << (2 * D), PER = (NC + 31) / 32;
  const int lane = threadIdx.x & 31;
  const int wid = bid_ * (blockDim.x >> 5) + (threadIdx.x >> 5), nw = nblk_ * (blockDim.x >> 5);
  const int nfull = c.ctr[CTR_FULL];
  for (int t = wid; t < nfull; t += nw) {
    const int b = c.full_bins[t];
    int* cc = c.cell_count + ((long long)b << (2 * D));
    int n[PER], tot = 0;
#pragma unroll
    for (int k = 0; k < PER; ++k) {
      const int cell = lane * PER + k;
      n[k] = cell < NC ? cc[cell] : 0;
      tot += n[k];
    }
    int inc = tot;  // inclusive scan of the lanes' totals
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, inc, o);
      if (lane >= o) inc += y;
    }
    int run = inc - tot;
    int* co = c.cell_off + ((long long)b << (2 * D));
#pragma unroll
    for (int k = 0; k < PER; ++k) {
      const int cell = lane * PER + k;
      if (cell < NC) {
        co[cell] = run;
        run += n[k];
        if (n[k]) cc[cell] = 0;
      }
    }
  }
}

template <int D>
__global__ void k_scatter(Batch B) {
  SCENE_CTA(B, MAP_G);
  SCENE_LOOP(p, c.N) {
    const int key = c.bin_of[p];
    c.perm[c.bin_start[key >> (2 * D)] + c.cell_off[key] + c.rank_of[p]] = (int)p;
  }
}

// ---------------------------------------------------------------------------
// launch sequence (transfer kernels are in transfer.cu)
template <int D>
void launch_transfer(const BatchLaunch& bl, cudaStream_t s, cudaEvent_t* ev);

template <int D>
static void run_topology(const BatchLaunch& bl, cudaStream_t s, cudaEvent_t* ev) {
  const Batch& B = bl.b;
  const int G = bl.nct[MAP_G], Go = bl.nct[MAP_O];
  if (ev) cudaEventRecord(ev[0], s);
  const bool pdl = bl.pdl && !ev;
  // the first kernel follows whatever preceded the substep: a plain launch
  launch_k(false, k_clear<D>, G, 256, 0, s, B);
  launch_k(pdl, k_touch_activate<D>, G, 256, 0, s, B);
  launch_k(pdl, k_dilate<D>, G, 256, 0, s, B);
  if (ev) cudaEventRecord(ev[1], s);
  if (bl.any_dynamic) launch_k(pdl, k_mark_hier<D>, G, 256, 0, s, B);
  launch_k(pdl, k_resolve<D>, G, 256, 0, s, B);
  if (bl.side) {
    cudaEventRecord(bl.fork, s);
    cudaStreamWaitEvent(bl.side, bl.fork, 0);
    k_ghost_tj<D><<<G, 256, 0, bl.side>>>(B);
    if (D == 3 && bl.maxL > 1) launch_k(true, k_level_masks<D>, G, 256, 0, bl.side, B);
    cudaEventRecord(bl.join, bl.side);
  } else {
    launch_k(pdl, k_ghost_tj<D>, G, 256, 0, s, B);
    if (D == 3 && bl.maxL > 1) launch_k(pdl, k_level_masks<D>, G, 256, 0, s, B);
  }
  if (ev) cudaEventRecord(ev[2], s);
  // after an event record or wait the next launch is a plain one
  launch_k(pdl && !bl.side, k_bin<D>, G, 256, 0, s, B);
  launch_k(pdl, k_offsets<D>, Go, 1024, 0, s, B);
  launch_k(pdl, k_cell_offsets<D>, G, 256, 0, s, B);
  launch_k(pdl, k_scatter<D>, G, 256, 0, s, B);
  if (ev) cudaEventRecord(ev[3], s);
}

void launch_substep(const BatchLaunch& bl, cudaStream_t s, cudaEvent_t* ev) {
  if (bl.dim == 2) {
    run_topology<2>(bl, s, ev);
    launch_transfer<2>(bl, s, ev);
  } else {
    run_topology<3>(bl, s, ev);
    launch_transfer<3>(bl, s, ev);
  }
}

int kernels_per_substep(const BatchLaunch& bl) {
  const int topo = 10 - (bl.any_dynamic ? 0 : 1) + (bl.dim == 3 && bl.maxL > 1 ? 1 : 0);
  return topo + 2 + (bl.maxL == 1 ? 1 : 0) + (bl.any_plastic ? 1 : 0) + 2 * (bl.maxL - 1);
}

}  // namespace agimp

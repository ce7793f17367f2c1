// CPU restatement of the reference's adaptive GIMP substep.
//
// TEST INFRASTRUCTURE ONLY.  This file is the parity oracle: only tests/,
// __graft_entry__.smoke() and bench.py's cpu_baseline / reference legs may
// load it, and only as the checker or the timed CPU baseline, never as the
// product path.
//
// What it restates (file:line are in the reference project g1n0st/adaptive-gimp):
//   utils.py:5-9        mask flags
//   utils.py:11-16      get_stress (fixed-corotated Kirchhoff stress)
//   utils.py:18-42      get_linear_weight (GIMP per-cell weight / gradient)
//   adaptive_gimp.py:68-96   activate_cell, activate_cell_static/_dynamic
//   adaptive_gimp.py:98-124  _mark_hier_, _split_hier_, culling_hierarchy_duplicate
//   adaptive_gimp.py:126-140 _map and node predicates
//   adaptive_gimp.py:142-187 _activate_mask, ghost / T-junction marking
//   adaptive_gimp.py:189-216 get_finest_level_near_particle, level_mapping
//   adaptive_gimp.py:218-228 get_weight_stencil
//   adaptive_gimp.py:230-275 p2g, g2p
//   adaptive_gimp.py:277-321 grid_op, grid_restriction, grid_prolongation
//   adaptive_gimp.py:323-352 substep ordering
//
// Parity status: pinned against golden vectors produced by running the
// reference's own adaptive_gimp.py / utils.py source under a Taichi-semantics
// shim (tests/golden/make_golden.py).  The Taichi runtime itself (its sparse
// storage, fast-math code generation and ti.svd) is not available here, so
// those parts are restated, not pinned.
//
// Storage is dense with per-4^d-block activity flags, emulating Taichi's
// pointer/bitmasked SNodes: reads of never-written elements return zero and
// struct-for loops visit only active blocks.  Loops run serially in a fixed
// order when nthreads == 0 (deterministic), or under OpenMP with atomics when
// nthreads > 0 (the timed CPU baseline).
//
// Extensions that have no counterpart in the reference (parameters default to
// the reference's behaviour): a sticky-wall boundary mode, box colliders,
// snow plasticity (Stomakhin et al. 2013) and the free-surface refinement rule
// that recomputes the prescribed particle levels.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <type_traits>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

enum : int32_t { UNACTIVATED = 0, ACTIVATED = 1, GHOST = 2, T_JUNCTION = 4, CULLING = 8 };
enum : uint32_t { ERR_OOB = 1u, ERR_ESCAPED = 2u, ERR_MAP_OOB = 4u, ERR_BAD_ARG = 8u };

constexpr int HALO = 4;  // level arrays cover indices [-HALO, size + 2*HALO)

// ---- atomics (serial mode executes them in program order) --------------------
inline void at_or(int32_t* a, int32_t b) {
#pragma omp atomic update
  *a |= b;
}
template <typename R> inline void at_add(R* a, R b) {
#pragma omp atomic update
  *a += b;
}
inline void at_flag(uint8_t* a) {
#pragma omp atomic write
  *a = 1;
}
inline void at_err(uint32_t* e, uint32_t b) {
#pragma omp atomic update
  *e |= b;
}

// ---- small dense matrices -------------------------------------------------
// Polar rotation / SVD in double precision by one-sided (Hestenes) Jacobi.
// Returns U, sig, V with A = U diag(sig) V^T, det(U) = det(V) = +1, sig sorted
// by magnitude descending, the last entry carrying the sign when det(A) < 0.
// This is the oracle's own method; ti.svd (the reference's, utils.py:13) is a
// third-party routine that only needs to agree on U V^T and sig up to rounding.
template <int D> void svd_d(const double* A, double* U, double* sig, double* V) {
  double B[D][D], W[D][D];
  for (int i = 0; i < D; ++i)
    for (int j = 0; j < D; ++j) { B[i][j] = A[i * D + j]; W[i][j] = (i == j); }
  for (int sweep = 0; sweep < 60; ++sweep) {
    double off = 0.0;
    for (int p = 0; p < D - 1; ++p)
      for (int q = p + 1; q < D; ++q) {
        double a = 0, b = 0, g = 0;
        for (int i = 0; i < D; ++i) { a += B[i][p] * B[i][p]; b += B[i][q] * B[i][q]; g += B[i][p] * B[i][q]; }
        if (std::fabs(g) <= 1e-300 || std::fabs(g) <= 1e-17 * std::sqrt(a * b)) continue;
        off = std::max(off, std::fabs(g) / std::sqrt(a * b));
        double zeta = (b - a) / (2.0 * g);
        double t = (zeta >= 0 ? 1.0 : -1.0) / (std::fabs(zeta) + std::sqrt(1.0 + zeta * zeta));
        double c = 1.0 / std::sqrt(1.0 + t * t), s = c * t;
        for (int i = 0; i < D; ++i) {
          double bp = B[i][p], bq = B[i][q];
          B[i][p] = c * bp - s * bq; B[i][q] = s * bp + c * bq;
          double wp = W[i][p], wq = W[i][q];
          W[i][p] = c * wp - s * wq; W[i][q] = s * wp + c * wq;
        }
      }
    if (off < 1e-16) break;
  }
  double s[D]; int ord[D];
  for (int j = 0; j < D; ++j) {
    double n = 0; for (int i = 0; i < D; ++i) n += B[i][j] * B[i][j];
    s[j] = std::sqrt(n); ord[j] = j;
  }
  std::sort(ord, ord + D, [&](int a, int b) { return s[a] > s[b]; });
  double Uc[D][D], Vc[D][D], sg[D];
  for (int k = 0; k < D; ++k) {
    int j = ord[k]; sg[k] = s[j];
    for (int i = 0; i < D; ++i) { Vc[i][k] = W[i][j]; Uc[i][k] = (s[j] > 1e-300) ? B[i][j] / s[j] : 0.0; }
  }
  // complete U where singular values vanish
  if (D == 2) {
    if (sg[0] <= 1e-300) { Uc[0][0] = 1; Uc[1][0] = 0; }
    if (sg[1] <= 1e-300 * std::max(1.0, sg[0]) || sg[1] == 0) { Uc[0][1] = -Uc[1][0]; Uc[1][1] = Uc[0][0]; }
  } else {
    if (sg[0] <= 1e-300) { for (int i = 0; i < D; ++i) Uc[i][0] = (i == 0); }
    if (sg[1] <= 1e-300) {
      // any unit vector orthogonal to U0
      double a[3] = {Uc[0][0], Uc[1][0], Uc[2][0]}, e[3] = {0, 0, 0};
      int m = (std::fabs(a[0]) < 0.6) ? 0 : 1; e[m] = 1;
      double d = a[0] * e[0] + a[1] * e[1] + a[2] * e[2];
      double u1[3] = {e[0] - d * a[0], e[1] - d * a[1], e[2] - d * a[2]};
      double n = std::sqrt(u1[0] * u1[0] + u1[1] * u1[1] + u1[2] * u1[2]);
      for (int i = 0; i < 3; ++i) Uc[i][1] = u1[i] / n;
    }
    if (sg[2] <= 1e-300) {
      Uc[0][2] = Uc[1][0] * Uc[2][1] - Uc[2][0] * Uc[1][1];
      Uc[1][2] = Uc[2][0] * Uc[0][1] - Uc[0][0] * Uc[2][1];
      Uc[2][2] = Uc[0][0] * Uc[1][1] - Uc[1][0] * Uc[0][1];
    }
  }
  auto det = [](double M[D][D]) {
    if (D == 2) return M[0][0] * M[1][1] - M[0][1] * M[1][0];
    return M[0][0] * (M[1][1] * M[2][2] - M[1][2] * M[2][1]) - M[0][1] * (M[1][0] * M[2][2] - M[1][2] * M[2][0]) +
           M[0][2] * (M[1][0] * M[2][1] - M[1][1] * M[2][0]);
  };
  if (det(Vc) < 0) for (int i = 0; i < D; ++i) { Vc[i][D - 1] = -Vc[i][D - 1]; Uc[i][D - 1] = -Uc[i][D - 1]; }
  if (det(Uc) < 0) { for (int i = 0; i < D; ++i) Uc[i][D - 1] = -Uc[i][D - 1]; sg[D - 1] = -sg[D - 1]; }
  for (int i = 0; i < D; ++i) {
    sig[i] = sg[i];
    for (int j = 0; j < D; ++j) { U[i * D + j] = Uc[i][j]; V[i * D + j] = Vc[i][j]; }
  }
}

template <int D, typename R> R det(const R* F) {
  if (D == 2) return F[0] * F[3] - F[1] * F[2];
  return F[0] * (F[4] * F[8] - F[5] * F[7]) - F[1] * (F[3] * F[8] - F[5] * F[6]) + F[2] * (F[3] * F[7] - F[4] * F[6]);
}

// utils.py:11-16: stress = 2*mu*(F - U V^T) @ F^T + I * la * J * (J - 1)
template <int D, typename R> void get_stress(const R* F, R mu, R la, R* out) {
  double Fd[D * D], U[D * D], S[D], V[D * D];
  for (int i = 0; i < D * D; ++i) Fd[i] = (double)F[i];
  svd_d<D>(Fd, U, S, V);
  R Rm[D * D];
  for (int i = 0; i < D; ++i)
    for (int j = 0; j < D; ++j) {
      double a = 0; for (int k = 0; k < D; ++k) a += U[i * D + k] * V[j * D + k];
      Rm[i * D + j] = (R)a;
    }
  R J = det<D, R>(F);
  R tmu = (R)2 * mu;
  R X[D * D];
  for (int i = 0; i < D * D; ++i) X[i] = tmu * (F[i] - Rm[i]);
  R diag = la * J * (J - (R)1);
  for (int i = 0; i < D; ++i)
    for (int j = 0; j < D; ++j) {
      R a = 0; for (int k = 0; k < D; ++k) a += X[i * D + k] * F[j * D + k];
      out[i * D + j] = a + (i == j ? diag : (R)0);
    }
}

// utils.py:18-42 get_linear_weight and adaptive_gimp.py:218-228 get_weight_stencil.
// W[k][0] = weight, W[k][1..D] = gradient, k = sum_d n_d 3^d over node offsets n.
template <int D, typename R> void weight_stencil(const R* tc, R radius, R W[][D + 1]) {
  constexpr int NN = (D == 2) ? 9 : 27;
  for (int k = 0; k < NN; ++k) for (int c = 0; c <= D; ++c) W[k][c] = 0;
  const R r2 = radius * (R)2.0;
  const R wden = (D == 2) ? (R)4.0 * r2 * r2 : (R)8.0 * r2 * r2 * r2;
  const R gden = (D == 2) ? (R)2.0 * r2 * r2 : (R)4.0 * r2 * r2 * r2;
  for (int a = 0; a < (1 << D); ++a) {      // dI in ndrange(2,..), last axis fastest
    int dI[D]; for (int d = 0; d < D; ++d) dI[d] = (a >> (D - 1 - d)) & 1;
    for (int b = 0; b < (1 << D); ++b) {    // cell_
      int cl[D]; for (int d = 0; d < D; ++d) cl[d] = (b >> (D - 1 - d)) & 1;
      R w[D], gw[D];
      for (int d = 0; d < D; ++d) {
        R t = tc[d] + (R)(1 - dI[d]);
        R bmin = std::min(std::max(t - radius, (R)0.0), (R)1.0);
        R bmax = std::min(std::max(t + radius, (R)0.0), (R)1.0);
        R mx, mn;
        if (cl[d]) { mx = bmax; mn = bmin; } else { mx = (R)1.0 - bmin; mn = (R)1.0 - bmax; }
        w[d] = mx * mx - mn * mn;
        gw[d] = cl[d] ? (mx - mn) : (mn - mx);
      }
      int k = 0, cv = 1;
      for (int d = 0; d < D; ++d) { k += (dI[d] + cl[d]) * cv; cv *= 3; }
      if (D == 2) {
        W[k][0] += w[0] * w[1] / wden;
        W[k][1] += gw[0] * w[1] / gden;
        W[k][2] += w[0] * gw[1] / gden;
      } else {
        W[k][0] += w[0] * w[1] * w[2] / wden;
        W[k][1] += gw[0] * w[1] * w[2] / gden;
        W[k][2] += w[0] * gw[1] * w[2] / gden;
        W[k][3] += w[0] * w[1] * gw[2] / gden;
      }
    }
  }
}

}  // namespace

extern "C" {
// Parameters of the restated simulator.  Defaults reproducing the reference
// (adaptive_gimp.py:18, 48-53): radius 0.5, gravity (0,-100,0), E 5e3, nu 0.2,
// boundary_gap 4, boundary_mode 0 (per-axis normal clamp), no plasticity.
typedef struct {
  int32_t dim, level, coarsest_size;
  int32_t boundary_gap;
  int32_t boundary_mode;  // 0: per-axis clamp (reference), 1: sticky walls
  int32_t plasticity;     // 0: none (reference), 1: snow
  double radius;
  double gravity[3];
  double E, nu;
  double theta_c, theta_s, hardening;
  int32_t n_colliders;
  double colliders[4][6];  // sticky boxes: lo[3], hi[3] in domain units
  int32_t invalid_nodes;   // 0: reference (raw momentum kept), 1: normalised
} orc_params;
}

namespace {

struct SimBase {
  virtual ~SimBase() {}
  uint32_t err = 0;
};

template <int D, typename R> struct Sim : SimBase {
  static constexpr int NC = 1 << D;          // 2^d
  static constexpr int NS = (D == 2) ? 9 : 27;  // 3^d
  struct Lev {
    int size, n, nb;
    std::vector<int32_t> cell;
    std::vector<R> m, v;
    std::vector<uint8_t> blk;
  };
  int L, coarsest, sz, gap, bmode, plast, inv_norm;
  double coarsest_dx;
  R radius, grav[3], mu, la, theta_c, theta_s, xi;
  int ncol; double col[4][6];
  int64_t N;
  std::vector<R> x, v, F, C, m, Jp;
  std::vector<int32_t> g, fl;
  std::vector<Lev> lev;
  int nm_n, nm_nb;
  std::vector<int32_t> nmask;
  std::vector<uint8_t> nm_blk;
  bool is_static = false;
  int map_h = 0, map_n = 0;
  std::vector<int8_t> map;
  std::vector<std::vector<int32_t>> pid;  // per level, particles sorted by (block, index)
  std::vector<std::vector<int64_t>> pid_blk;
  bool par = false;

  Sim(const orc_params* p, int64_t n) {
    L = p->level; coarsest = p->coarsest_size; sz = coarsest << (L - 1);
    gap = p->boundary_gap; bmode = p->boundary_mode; plast = p->plasticity;
    inv_norm = p->invalid_nodes;
    coarsest_dx = 1.0 / coarsest;
    radius = (R)p->radius;
    for (int d = 0; d < 3; ++d) grav[d] = (R)p->gravity[d];
    double mu_d = p->E / (2 * (1 + p->nu)), la_d = p->E * p->nu / ((1 + p->nu) * (1 - 2 * p->nu));
    mu = (R)mu_d; la = (R)la_d;
    theta_c = (R)p->theta_c; theta_s = (R)p->theta_s; xi = (R)p->hardening;
    ncol = p->n_colliders; std::memcpy(col, p->colliders, sizeof(col));
    N = n;
    x.assign(N * D, 0); v.assign(N * D, 0); F.assign(N * D * D, 0); C.assign(N * D * D, 0);
    m.assign(N, 0); Jp.assign(N, 1); g.assign(N, 0); fl.assign(N, -1);
    lev.resize(L);
    for (int l = 0; l < L; ++l) {
      Lev& A = lev[l];
      A.size = coarsest << l; A.n = A.size + 3 * HALO; A.nb = A.n / 4;
      int64_t cnt = 1, bc = 1;
      for (int d = 0; d < D; ++d) { cnt *= A.n; bc *= A.nb; }
      A.cell.assign(cnt, 0); A.m.assign(cnt, 0); A.v.assign(cnt * D, 0); A.blk.assign(bc, 0);
    }
    nm_n = sz + 4; nm_nb = nm_n / 4;
    int64_t cnt = 1, bc = 1;
    for (int d = 0; d < D; ++d) { cnt *= nm_n; bc *= nm_nb; }
    nmask.assign(cnt, 0); nm_blk.assign(bc, 0);
    pid.resize(L); pid_blk.resize(L);
  }

  // ---- indexing ----------------------------------------------------------
  bool lidx(const Lev& A, const int* I, int64_t& out, int64_t& ob) const {
    int64_t o = 0, b = 0;
    for (int d = 0; d < D; ++d) {
      int a = I[d] + HALO;
      if (a < 0 || a >= A.n) return false;
      o = o * A.n + a; b = b * A.nb + (a >> 2);
    }
    out = o; ob = b; return true;
  }
  void unlin(const Lev& A, int64_t o, int* I) const {
    for (int d = D - 1; d >= 0; --d) { I[d] = (int)(o % A.n) - HALO; o /= A.n; }
  }
  int32_t cell_get(int l, const int* I) const {
    int64_t o, b; if (!lidx(lev[l], I, o, b)) return 0; return lev[l].cell[o];
  }
  void cell_or(int l, const int* I, int32_t bits) {
    int64_t o, b; Lev& A = lev[l];
    if (!lidx(A, I, o, b)) { at_err(&err, ERR_OOB); return; }
    at_or(&A.cell[o], bits); at_flag(&A.blk[b]);
  }
  // node mask on the finest lattice; writes outside [0, sz] are unobservable
  // (every predicate read happens at in-range nodes) and are dropped.
  bool nm_idx(const int* P, int64_t& o, int64_t& b) const {
    int64_t oo = 0, bb = 0;
    for (int d = 0; d < D; ++d) {
      if (P[d] < 0 || P[d] > sz) return false;
      oo = oo * nm_n + P[d]; bb = bb * nm_nb + (P[d] >> 2);
    }
    o = oo; b = bb; return true;
  }
  int32_t nm_get_map(int l, const int* I) const {  // node_mask[_map(l, I)]
    int P[D]; int s = L - 1 - l;
    for (int d = 0; d < D; ++d) P[d] = I[d] * (1 << s);
    int64_t o, b; if (!nm_idx(P, o, b)) return 0; return nmask[o];
  }
  void nm_or_map(int l, const int* I, int32_t bits) {
    int P[D]; int s = L - 1 - l;
    for (int d = 0; d < D; ++d) P[d] = I[d] * (1 << s);
    int64_t o, b; if (!nm_idx(P, o, b)) return;
    at_or(&nmask[o], bits); at_flag(&nm_blk[b]);
  }
  // adaptive_gimp.py:130-140
  bool is_valid(int l, const int* I) const { return nm_get_map(l, I) > 0; }
  bool is_activated(int l, const int* I) const { return (nm_get_map(l, I) & (ACTIVATED | T_JUNCTION)) == ACTIVATED; }
  bool is_T(int l, const int* I) const { return (nm_get_map(l, I) & T_JUNCTION) == T_JUNCTION; }
  bool is_ghost(int l, const int* I) const {
    return (nm_get_map(l, I) & (ACTIVATED | GHOST | T_JUNCTION)) == GHOST;
  }

  // iterate active blocks of level l in linear order, all elements inside
  template <typename Fn> void for_active(int l, Fn fn) {
    Lev& A = lev[l];
    int64_t nblk = (int64_t)A.blk.size();
    std::vector<int64_t> act;
    for (int64_t b = 0; b < nblk; ++b) if (A.blk[b]) act.push_back(b);
    auto body = [&](int64_t bi) {
      int64_t b = act[bi];
      int B[D]; int64_t t = b;
      for (int d = D - 1; d >= 0; --d) { B[d] = (int)(t % A.nb); t /= A.nb; }
      for (int e = 0; e < (1 << (2 * D)); ++e) {
        int I[D];
        for (int d = 0; d < D; ++d) I[d] = B[d] * 4 + ((e >> (2 * (D - 1 - d))) & 3) - HALO;
        fn(I);
      }
    };
    if (par) {
#pragma omp parallel for schedule(dynamic, 4)
      for (int64_t bi = 0; bi < (int64_t)act.size(); ++bi) body(bi);
    } else {
      for (int64_t bi = 0; bi < (int64_t)act.size(); ++bi) body(bi);
    }
  }
  template <typename Fn> void for_particles(Fn fn) {
    if (par) {
#pragma omp parallel for schedule(static)
      for (int64_t p = 0; p < N; ++p) fn(p);
    } else {
      for (int64_t p = 0; p < N; ++p) fn(p);
    }
  }

  bool escaped(int64_t p) const {
    for (int d = 0; d < D; ++d) {
      R a = x[p * D + d];
      if (!(a >= (R)0 && a < (R)1)) return true;
    }
    return false;
  }
  R level_dx(int l) const { return (R)(coarsest_dx / (double)(1 << l)); }
  void base_at(int64_t p, R dx, int* base) const {
    for (int d = 0; d < D; ++d) base[d] = (int)(x[p * D + d] / dx + (R)0.5) - 1;
  }

  // ---- adaptive_gimp.py:324-326 --------------------------------------------
  void clear_all() {
    for (int l = 0; l < L; ++l) {
      Lev& A = lev[l];
      int64_t per = 1; for (int d = 0; d < D; ++d) per *= 4;
      for (int64_t b = 0; b < (int64_t)A.blk.size(); ++b) {
        if (!A.blk[b]) continue;
        A.blk[b] = 0;
        int B[D]; int64_t t = b;
        for (int d = D - 1; d >= 0; --d) { B[d] = (int)(t % A.nb); t /= A.nb; }
        for (int e = 0; e < per; ++e) {
          int64_t o = 0;
          for (int d = 0; d < D; ++d) o = o * A.n + (B[d] * 4 + ((e >> (2 * (D - 1 - d))) & 3));
          A.cell[o] = 0; A.m[o] = 0; for (int c = 0; c < D; ++c) A.v[o * D + c] = 0;
        }
      }
    }
    for (int64_t b = 0; b < (int64_t)nm_blk.size(); ++b) {
      if (!nm_blk[b]) continue;
      nm_blk[b] = 0;
      int B[D]; int64_t t = b;
      for (int d = D - 1; d >= 0; --d) { B[d] = (int)(t % nm_nb); t /= nm_nb; }
      for (int e = 0; e < (1 << (2 * D)); ++e) {
        int64_t o = 0;
        for (int d = 0; d < D; ++d) o = o * nm_n + (B[d] * 4 + ((e >> (2 * (D - 1 - d))) & 3));
        nmask[o] = 0;
      }
    }
  }

  // ---- adaptive_gimp.py:68-85: static activation through the level map ------
  // The reference's grid_initializer(sim, I) calls sim.activate_cell(l, I) and
  // returns l.  Here it is a table over finest cells: low nibble = l, bit 6 set
  // = return l without activating.
  int map_lookup(const int* I, bool& ok) const {
    int64_t o = 0;
    for (int d = 0; d < D; ++d) {
      int a = I[d] + map_h;
      if (a < 0 || a >= map_n) { ok = false; return L - 1; }
      o = o * map_n + a;
    }
    ok = true; return map[o];
  }
  int grid_initializer(const int* I) {
    bool ok; int e = map_lookup(I, ok);
    if (!ok) { at_err(&err, ERR_MAP_OOB); return L - 1; }
    int l = e & 15;
    if (!(e & 64)) {  // activate_cell (adaptive_gimp.py:68-70)
      int c[D]; int s = L - 1 - l;
      for (int d = 0; d < D; ++d) c[d] = I[d] >> s;
      cell_or(l, c, ACTIVATED);
    }
    return l;
  }
  void activate_cell_static() {
    for_particles([&](int64_t p) {
      if (escaped(p)) { at_err(&err, ERR_ESCAPED); return; }
      R f_dx = (R)(coarsest_dx / (double)(1 << (L - 1)));
      int fb[D]; base_at(p, f_dx, fb);
      for (int a = 0; a < (1 << (2 * D)); ++a) {  // dI in ndrange((-1,3),..)
        int I[D];
        for (int d = 0; d < D; ++d) I[d] = fb[d] + ((a >> (2 * (D - 1 - d))) & 3) - 1;
        grid_initializer(I);
      }
      int level = grid_initializer(fb);
      R dx = (R)(coarsest_dx / (double)(1 << level));
      int base[D]; base_at(p, dx, base);
      for (int a = 0; a < NC; ++a) {
        int I[D];
        for (int d = 0; d < D; ++d) I[d] = (base[d] + ((a >> (D - 1 - d)) & 1)) * (1 << (L - 1 - level));
        grid_initializer(I);
      }
    });
  }
  // adaptive_gimp.py:87-96
  void activate_cell_dynamic() {
    for_particles([&](int64_t p) {
      if (escaped(p)) { at_err(&err, ERR_ESCAPED); return; }
      int gl = g[p];
      if (gl < 0 || gl >= L) return;
      R dx = level_dx(gl);
      int base[D]; base_at(p, dx, base);
      for (int a = 0; a < NC; ++a) {
        int I[D];
        for (int d = 0; d < D; ++d) I[d] = base[d] + ((a >> (D - 1 - d)) & 1);
        cell_or(gl, I, ACTIVATED);
      }
    });
  }
  // adaptive_gimp.py:98-109
  void mark_hier(int l) {
    for_active(l, [&](const int* I) {
      if (!(cell_get(l, I) & ACTIVATED)) return;
      int l0 = -1;
      for (int q = 0; q < l; ++q) {
        int A[D]; for (int d = 0; d < D; ++d) A[d] = I[d] >> (l - q);
        if (cell_get(q, A) & ACTIVATED) l0 = std::max(l0, q);
      }
      if (l0 != -1)
        for (int q = l0; q < l; ++q) {
          int A[D]; for (int d = 0; d < D; ++d) A[d] = I[d] >> (l - q);
          cell_or(q, A, CULLING);
        }
    });
  }
  // adaptive_gimp.py:111-118
  void split_hier(int l) {
    for_active(l, [&](const int* I) {
      if (!(cell_get(l, I) & CULLING)) return;
      for (int a = 0; a < NC; ++a) {
        int Ch[D];
        for (int d = 0; d < D; ++d) Ch[d] = I[d] * 2 + ((a >> (D - 1 - d)) & 1);
        cell_or(l + 1, Ch, ACTIVATED);
      }
      int64_t o, b; lidx(lev[l], I, o, b); lev[l].cell[o] = 0;
    });
  }
  // adaptive_gimp.py:142-153
  void activate_mask(int l) {
    for_active(l, [&](const int* I) {
      if (cell_get(l, I) != ACTIVATED) return;
      for (int a = 0; a < NC; ++a) {
        int J[D];
        for (int d = 0; d < D; ++d) J[d] = I[d] + ((a >> (D - 1 - d)) & 1);
        nm_or_map(l, J, ACTIVATED);
      }
    });
  }
  // adaptive_gimp.py:155-158
  int hier_check(int l, const int* I) const {
    int best = -1;
    for (int q = 0; q <= l; ++q) {
      int A[D]; for (int d = 0; d < D; ++d) A[d] = I[d] >> (l - q);
      if (cell_get(q, A) == ACTIVATED) best = std::max(best, q);
    }
    return best;
  }
  // adaptive_gimp.py:160-183
  void mark_ghost_T(int l) {
    const int lsz = lev[l].size;
    for_active(l, [&](const int* I) {
      if (cell_get(l, I) != ACTIVATED) return;
      for (int f = 0; f < 2 * D; ++f) {
        int ax = f / 2, side = f % 2;
        int I1[D]; for (int d = 0; d < D; ++d) I1[d] = I[d];
        I1[ax] += side ? -1 : 1;
        bool inr = true; for (int d = 0; d < D; ++d) inr = inr && (I1[d] >= 0 && I1[d] < lsz);
        if (!inr) continue;
        if (cell_get(l, I1) == ACTIVATED) continue;
        int lp = hier_check(l, I1);
        if (lp <= -1) continue;
        for (int a = 0; a < NC; ++a) {
          int c[D]; for (int d = 0; d < D; ++d) c[d] = (a >> (D - 1 - d)) & 1;
          if (c[ax] != side) continue;
          int J[D]; bool anyoff = false; int md = 1 << (l - lp);
          for (int d = 0; d < D; ++d) { J[d] = I1[d] + c[d]; if (J[d] % md != 0) anyoff = true; }
          if (anyoff) nm_or_map(l, J, T_JUNCTION);
        }
        for (int l0 = lp + 1; l0 <= l; ++l0) {
          int Ip[D]; for (int d = 0; d < D; ++d) Ip[d] = I1[d] >> (l - l0);
          cell_or(l0, Ip, GHOST);
          for (int a = 0; a < NC; ++a) {
            int J[D]; for (int d = 0; d < D; ++d) J[d] = Ip[d] + ((a >> (D - 1 - d)) & 1);
            if (nm_get_map(l0, J) == UNACTIVATED) nm_or_map(l0, J, GHOST);
          }
        }
      }
    });
  }
  // adaptive_gimp.py:189-216 (the per-block particle lists are built here in
  // (block, particle index) order; Taichi's atomic append order is unspecified)
  void level_mapping() {
    std::vector<int64_t> key(N, -1);
    for_particles([&](int64_t p) {
      if (escaped(p)) { fl[p] = -1; return; }
      int f = -1;
      for (int l = 0; l < L; ++l) {
        R dx = level_dx(l);
        int base[D]; base_at(p, dx, base);
        for (int a = 0; a < NC; ++a) {
          int I[D]; for (int d = 0; d < D; ++d) I[d] = base[d] + ((a >> (D - 1 - d)) & 1);
          if (cell_get(l, I) == ACTIVATED) f = std::max(f, l);
        }
      }
      fl[p] = f;
      if (f >= 0) {
        int base[D]; base_at(p, level_dx(f), base);
        int64_t b = 0; const Lev& A = lev[f];
        bool ok = true;
        for (int d = 0; d < D; ++d) {
          int bb = (base[d] >> 2) + 1;  // block index with one block of halo
          if (bb < 0 || bb >= A.nb) ok = false;
          b = b * A.nb + bb;
        }
        if (!ok) { at_err(&err, ERR_OOB); fl[p] = -1; return; }
        key[p] = b;
      }
    });
    for (int l = 0; l < L; ++l) { pid[l].clear(); pid_blk[l].clear(); }
    std::vector<int64_t> order;
    order.reserve(N);
    for (int64_t p = 0; p < N; ++p) if (fl[p] >= 0) order.push_back(p);
    std::stable_sort(order.begin(), order.end(), [&](int64_t a, int64_t b) {
      if (fl[a] != fl[b]) return fl[a] < fl[b];
      return key[a] < key[b];
    });
    for (int64_t p : order) { pid[fl[p]].push_back((int32_t)p); pid_blk[fl[p]].push_back(key[p]); }
  }

  template <typename Fn> void for_pid(int l, Fn fn) {
    const std::vector<int32_t>& P = pid[l];
    if (par) {
#pragma omp parallel for schedule(dynamic, 256)
      for (int64_t i = 0; i < (int64_t)P.size(); ++i) fn((int64_t)P[i]);
    } else {
      for (int64_t i = 0; i < (int64_t)P.size(); ++i) fn((int64_t)P[i]);
    }
  }

  void node_add(int l, const int* I, R dm, const R* dv) {
    int64_t o, b; Lev& A = lev[l];
    if (!lidx(A, I, o, b)) { at_err(&err, ERR_OOB); return; }
    at_add(&A.m[o], dm);
    for (int c = 0; c < D; ++c) at_add(&A.v[o * D + c], dv[c]);
    at_flag(&A.blk[b]);
  }
  void node_addv(int l, const int* I, const R* dv) {
    int64_t o, b; Lev& A = lev[l];
    if (!lidx(A, I, o, b)) { at_err(&err, ERR_OOB); return; }
    for (int c = 0; c < D; ++c) at_add(&A.v[o * D + c], dv[c]);
    at_flag(&A.blk[b]);
  }
  bool node_get(int l, const int* I, R& mm, R* vv) const {
    int64_t o, b; const Lev& A = lev[l];
    if (!lidx(A, I, o, b)) { mm = 0; for (int c = 0; c < D; ++c) vv[c] = 0; return false; }
    mm = A.m[o]; for (int c = 0; c < D; ++c) vv[c] = A.v[o * D + c];
    return true;
  }

  // adaptive_gimp.py:230-250
  void p2g(int l, R dt) {
    R dx = level_dx(l);
    const R pw = (D == 2) ? (R)0.25 : (R)0.125;              // 0.5**dim
    const R rd = (D == 2) ? radius * radius : radius * radius * radius;  // radius**dim
    for_pid(l, [&](int64_t p) {
      int base[D]; base_at(p, dx, base);
      R tc[D];
      for (int d = 0; d < D; ++d) tc[d] = x[p * D + d] / dx - (R)(base[d] + 1);
      R mu_p = mu, la_p = la;
      if (plast == 1) {  // snow hardening (extension)
        R h = (R)std::exp((double)(xi * ((R)1 - Jp[p])));
        mu_p = mu * h; la_p = la * h;
      }
      R S[D * D];
      get_stress<D, R>(&F[p * D * D], mu_p, la_p, S);
      R sc = (-dt * pw) / (rd * dx);
      for (int i = 0; i < D * D; ++i) S[i] = sc * S[i];
      R W[NS][D + 1];
      weight_stencil<D, R>(tc, radius, W);
      const R* vp = &v[p * D];
      const R* Cp = &C[p * D * D];
      for (int k = 0; k < NS; ++k) {  // ndrange(3,..), last axis fastest
        int dI[D]; int t = k;
        for (int d = D - 1; d >= 0; --d) { dI[d] = t % 3; t /= 3; }
        int kk = 0, cv = 1;
        for (int d = 0; d < D; ++d) { kk += dI[d] * cv; cv *= 3; }
        R w = W[kk][0];
        R dpos[D];
        for (int d = 0; d < D; ++d) dpos[d] = (R)dI[d] - (tc[d] + (R)1);
        R wm = w * m[p];
        R dv[D];
        for (int i = 0; i < D; ++i) {
          R cd = 0; for (int j = 0; j < D; ++j) cd += Cp[i * D + j] * dpos[j];
          R sg = 0; for (int j = 0; j < D; ++j) sg += S[i * D + j] * W[kk][1 + j];
          dv[i] = wm * (vp[i] + cd) + sg;
        }
        int I[D]; for (int d = 0; d < D; ++d) I[d] = base[d] + dI[d];
        node_add(l, I, wm, dv);
      }
    });
  }

  // snow plasticity return map (extension; Stomakhin et al. 2013)
  void snow_project(int64_t p) {
    R* Fp = &F[p * D * D];
    double Fd[D * D], U[D * D], sg[D], V[D * D];
    for (int i = 0; i < D * D; ++i) Fd[i] = (double)Fp[i];
    svd_d<D>(Fd, U, sg, V);
    R J_old = 1, J_new = 1, sc[D];
    for (int d = 0; d < D; ++d) {
      R s = (R)sg[d];
      R c = std::min(std::max(s, (R)1 - theta_c), (R)1 + theta_s);
      J_old *= s; J_new *= c; sc[d] = c;
    }
    Jp[p] = Jp[p] * J_old / J_new;
    for (int i = 0; i < D; ++i)
      for (int j = 0; j < D; ++j) {
        R a = 0; for (int k = 0; k < D; ++k) a += (R)U[i * D + k] * sc[k] * (R)V[j * D + k];
        Fp[i * D + j] = a;
      }
  }

  // adaptive_gimp.py:252-275
  void g2p(int l, R dt) {
    R dx = level_dx(l);
    const R pw = (D == 2) ? (R)0.25 : (R)0.125;
    const R rd = (D == 2) ? radius * radius : radius * radius * radius;
    for_pid(l, [&](int64_t p) {
      int base[D]; base_at(p, dx, base);
      R tc[D];
      for (int d = 0; d < D; ++d) tc[d] = x[p * D + d] / dx - (R)(base[d] + 1);
      R nv[D] = {}, G[D * D] = {};
      R W[NS][D + 1];
      weight_stencil<D, R>(tc, radius, W);
      for (int k = 0; k < NS; ++k) {
        int dI[D]; int t = k;
        for (int d = D - 1; d >= 0; --d) { dI[d] = t % 3; t /= 3; }
        int kk = 0, cv = 1;
        for (int d = 0; d < D; ++d) { kk += dI[d] * cv; cv *= 3; }
        int I[D]; for (int d = 0; d < D; ++d) I[d] = base[d] + dI[d];
        R mm, gv[D];
        if (!node_get(l, I, mm, gv)) at_err(&err, ERR_OOB);
        R w = W[kk][0];
        for (int i = 0; i < D; ++i) nv[i] += gv[i] * w;
        for (int i = 0; i < D; ++i)
          for (int j = 0; j < D; ++j) G[i * D + j] += gv[i] * W[kk][1 + j];
      }
      for (int i = 0; i < D; ++i) v[p * D + i] = nv[i];
      for (int i = 0; i < D * D; ++i) C[p * D * D + i] = G[i];
      for (int i = 0; i < D; ++i) x[p * D + i] += dt * v[p * D + i];
      R s = (dt * pw) / (rd * dx);
      R A[D * D];
      for (int i = 0; i < D; ++i)
        for (int j = 0; j < D; ++j) A[i * D + j] = (i == j ? (R)1 : (R)0) + s * G[i * D + j];
      R Fo[D * D];
      for (int i = 0; i < D * D; ++i) Fo[i] = F[p * D * D + i];
      for (int i = 0; i < D; ++i)
        for (int j = 0; j < D; ++j) {
          R a = 0; for (int k = 0; k < D; ++k) a += A[i * D + k] * Fo[k * D + j];
          F[p * D * D + i * D + j] = a;
        }
      if (plast == 1) snow_project(p);
    });
  }

  // adaptive_gimp.py:277-287 (+ sticky walls and box colliders as extensions)
  void grid_op(int l, R dt) {
    const int lsz = lev[l].size;
    const int s = L - 1 - l;
    const double ldx = coarsest_dx / (double)(1 << l);
    for_active(l, [&](const int* I) {
      for (int d = 0; d < D; ++d) if (I[d] < 0 || I[d] > lsz) return;
      int64_t o, b; Lev& A = lev[l];
      if (!lidx(A, I, o, b)) return;
      if (!(A.m[o] > 0)) return;
      if (!is_activated(l, I)) {
        // extension (invalid_nodes = 1): normalise the momentum the
        // reference leaves raw on nodes it does not update
        if (inv_norm) for (int c = 0; c < D; ++c) A.v[o * D + c] /= A.m[o];
        return;
      }
      R* vv = &A.v[o * D];
      for (int c = 0; c < D; ++c) vv[c] /= A.m[o];
      for (int c = 0; c < D; ++c) vv[c] += grav[c] * dt;
      bool inband = false;
      for (int c = 0; c < D; ++c) {
        int P = I[c] * (1 << s);
        if (P < gap || P > sz - gap) { if (bmode == 0) vv[c] = 0; inband = true; }
      }
      if (bmode == 1 && inband) for (int c = 0; c < D; ++c) vv[c] = 0;
      for (int k = 0; k < ncol; ++k) {
        bool in = true;
        for (int c = 0; c < D; ++c) {
          double pos = (double)I[c] * ldx;
          in = in && (pos >= col[k][c] && pos <= col[k][3 + c]);
        }
        if (in) for (int c = 0; c < D; ++c) vv[c] = 0;
      }
    });
  }
  // adaptive_gimp.py:289-301
  void grid_restriction(int l) {
    const int lsz = lev[l].size;
    for_active(l, [&](const int* I) {
      for (int d = 0; d < D; ++d) if (I[d] < 0 || I[d] > lsz) return;
      bool even = true; for (int d = 0; d < D; ++d) even = even && (I[d] % 2 == 0);
      if (!((is_activated(l, I) && even) || is_T(l, I) || is_ghost(l, I))) return;
      R mm, vv[D];
      node_get(l, I, mm, vv);
      for (int a = 0; a < NS; ++a) {  // ndrange((-1,2),..)
        int dI[D]; int t = a;
        for (int d = D - 1; d >= 0; --d) { dI[d] = t % 3 - 1; t /= 3; }
        int J[D]; bool ok = true; int nrm = 0;
        for (int d = 0; d < D; ++d) {
          J[d] = I[d] + dI[d];
          if (J[d] < 0 || J[d] > lsz || (J[d] % 2) != 0) ok = false;
          nrm += std::abs(dI[d]);
        }
        if (!ok) continue;
        int K[D]; for (int d = 0; d < D; ++d) K[d] = J[d] / 2;
        if (!is_valid(l - 1, K)) continue;
        R w = (R)std::pow(0.5, (double)nrm);
        R dv[D]; for (int c = 0; c < D; ++c) dv[c] = vv[c] * w;
        node_add(l - 1, K, mm * w, dv);
      }
    });
  }
  // adaptive_gimp.py:303-321
  void grid_prolongation(int l) {
    const int l0 = l - 1;
    const int l0sz = lev[l0].size, lsz = l0sz * 2;
    for_active(l, [&](const int* I) {
      for (int d = 0; d < D; ++d) if (I[d] < 0 || I[d] > lsz) return;
      bool even = true; for (int d = 0; d < D; ++d) even = even && (I[d] % 2 == 0);
      if (is_T(l, I) || is_ghost(l, I) || even) {
        int64_t o, b; Lev& A = lev[l];
        if (lidx(A, I, o, b)) for (int c = 0; c < D; ++c) A.v[o * D + c] = 0;
      }
    });
    for_active(l0, [&](const int* I) {
      for (int d = 0; d < D; ++d) if (I[d] < 0 || I[d] > l0sz) return;
      if (!is_valid(l0, I)) return;
      R mm, vv[D];
      node_get(l0, I, mm, vv);
      for (int a = 0; a < NS; ++a) {
        int dI[D]; int t = a;
        for (int d = D - 1; d >= 0; --d) { dI[d] = t % 3 - 1; t /= 3; }
        int J[D]; bool ok = true; int nrm = 0; bool zero = true;
        for (int d = 0; d < D; ++d) {
          J[d] = I[d] * 2 + dI[d];
          if (J[d] < 0 || J[d] > lsz) ok = false;
          nrm += std::abs(dI[d]); if (dI[d] != 0) zero = false;
        }
        if (!ok) continue;
        if (!(is_T(l, J) || is_ghost(l, J) || (is_activated(l, J) && zero))) continue;
        R w = (R)std::pow(0.5, (double)nrm);
        R dv[D]; for (int c = 0; c < D; ++c) dv[c] = vv[c] * w;
        node_addv(l, J, dv);
      }
    });
  }

  // adaptive_gimp.py:323-352
  void substep(R dt) {
    clear_all();
    if (is_static) {
      activate_cell_static();
    } else {
      activate_cell_dynamic();
      for (int l = L - 1; l >= 0; --l) if (l != 0) mark_hier(l);
      for (int l = 0; l < L; ++l) if (l != L - 1) split_hier(l);
    }
    for (int l = 0; l < L; ++l) activate_mask(l);
    for (int l = L - 1; l >= 0; --l) mark_ghost_T(l);
    level_mapping();
    for (int l = 0; l < L; ++l) p2g(l, dt);
    for (int l = L - 1; l >= 0; --l) if (l != 0) grid_restriction(l);
    for (int l = 0; l < L; ++l) grid_op(l, dt);
    for (int l = 0; l < L; ++l) if (l != 0) grid_prolongation(l);
    for (int l = 0; l < L; ++l) g2p(l, dt);
  }

  // Free-surface refinement rule (extension): a particle's prescribed level
  // is the finest level when its finest cell lies within `band` finest cells
  // (Chebyshev distance) of an empty finest cell, the next coarser level
  // within band*3, then band*7, ..., and level 0 deeper inside.
  void refine_levels(int band) {
    const int n = sz;
    int64_t cnt = 1; for (int d = 0; d < D; ++d) cnt *= n;
    std::vector<uint8_t> depth(cnt, 0);
    auto cidx = [&](const int* c) { int64_t o = 0; for (int d = 0; d < D; ++d) o = o * n + c[d]; return o; };
    for (int64_t p = 0; p < N; ++p) {
      if (escaped(p)) continue;
      int c[D]; for (int d = 0; d < D; ++d) c[d] = (int)std::floor(x[p * D + d] * (R)n);
      depth[cidx(c)] = 1;
    }
    int kmax = band * ((1 << (L - 1)) - 1) + 1;
    if (kmax > 250) kmax = 250;
    std::vector<uint8_t> nxt;
    for (int k = 1; k < kmax; ++k) {
      nxt = depth;
      bool changed = false;
      for (int64_t o = 0; o < cnt; ++o) {
        if (depth[o] != k) continue;
        int c[D]; int64_t t = o;
        for (int d = D - 1; d >= 0; --d) { c[d] = (int)(t % n); t /= n; }
        bool all = true;
        for (int a = 0; a < NS && all; ++a) {
          int q[D]; int tt = a;
          for (int d = D - 1; d >= 0; --d) { q[d] = c[d] + tt % 3 - 1; tt /= 3; }
          bool in = true; for (int d = 0; d < D; ++d) in = in && (q[d] >= 0 && q[d] < n);
          if (!in || depth[cidx(q)] < k) all = false;
        }
        if (all) { nxt[o] = (uint8_t)(k + 1); changed = true; }
      }
      depth.swap(nxt);
      if (!changed) break;
    }
    for (int64_t p = 0; p < N; ++p) {
      if (escaped(p)) continue;
      int c[D]; for (int d = 0; d < D; ++d) c[d] = (int)std::floor(x[p * D + d] * (R)n);
      int dd = depth[cidx(c)];
      int lv = 0;
      for (int k = 0; k < L - 1; ++k) {
        int T = band * ((1 << (k + 1)) - 1);
        if (dd <= T) { lv = L - 1 - k; break; }
      }
      g[p] = lv;
    }
  }
};

template <typename Fn> auto dispatch(SimBase* h, int dim, int f64, Fn fn) {
  if (dim == 2) {
    if (f64) return fn(static_cast<Sim<2, double>*>(h));
    return fn(static_cast<Sim<2, float>*>(h));
  }
  if (f64) return fn(static_cast<Sim<3, double>*>(h));
  return fn(static_cast<Sim<3, float>*>(h));
}

struct Handle {
  int dim, f64;
  SimBase* s;
};

}  // namespace

extern "C" {

void* orc_create(const orc_params* p, int32_t use_f64, int64_t n) {
  if (!p || (p->dim != 2 && p->dim != 3) || p->level < 1 || p->level > 8 || p->coarsest_size < 4 ||
      (p->coarsest_size & (p->coarsest_size - 1)) || n < 0)
    return nullptr;
  Handle* h = new Handle{p->dim, use_f64 ? 1 : 0, nullptr};
  if (p->dim == 2) h->s = use_f64 ? (SimBase*)new Sim<2, double>(p, n) : (SimBase*)new Sim<2, float>(p, n);
  else h->s = use_f64 ? (SimBase*)new Sim<3, double>(p, n) : (SimBase*)new Sim<3, float>(p, n);
  return h;
}

void orc_destroy(void* hh) {
  Handle* h = (Handle*)hh;
  if (!h) return;
  delete h->s;
  delete h;
}

int32_t orc_set_particles(void* hh, const double* x, const double* v, const double* F, const double* C,
                          const double* m, const int32_t* g, const double* Jp) {
  Handle* h = (Handle*)hh;
  return dispatch(h->s, h->dim, h->f64, [&](auto* s) {
    constexpr int D = std::remove_pointer_t<decltype(s)>::NC == 4 ? 2 : 3;
    using R = std::remove_reference_t<decltype(s->x[0])>;
    for (int64_t i = 0; i < s->N * D; ++i) { s->x[i] = (R)x[i]; s->v[i] = (R)v[i]; }
    for (int64_t i = 0; i < s->N * D * D; ++i) { s->F[i] = (R)F[i]; s->C[i] = (R)C[i]; }
    for (int64_t i = 0; i < s->N; ++i) { s->m[i] = (R)m[i]; s->g[i] = g[i]; s->Jp[i] = Jp ? (R)Jp[i] : (R)1; }
    return 0;
  });
}

int32_t orc_set_g(void* hh, const int32_t* g) {
  Handle* h = (Handle*)hh;
  return dispatch(h->s, h->dim, h->f64, [&](auto* s) {
    for (int64_t i = 0; i < s->N; ++i) s->g[i] = g[i];
    return 0;
  });
}

int32_t orc_set_level_map(void* hh, const int8_t* table, int32_t halo) {
  Handle* h = (Handle*)hh;
  return dispatch(h->s, h->dim, h->f64, [&](auto* s) {
    constexpr int D = std::remove_pointer_t<decltype(s)>::NC == 4 ? 2 : 3;
    s->map_h = halo; s->map_n = s->sz + 2 * halo;
    int64_t cnt = 1; for (int d = 0; d < D; ++d) cnt *= s->map_n;
    s->map.assign(table, table + cnt);
    s->is_static = true;
    return 0;
  });
}

int32_t orc_substep(void* hh, double dt, int32_t nsteps, int32_t nthreads) {
  Handle* h = (Handle*)hh;
  return dispatch(h->s, h->dim, h->f64, [&](auto* s) {
    using R = std::remove_reference_t<decltype(s->x[0])>;
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
    s->par = nthreads > 0;
    for (int i = 0; i < nsteps; ++i) s->substep((R)dt);
    s->par = false;
    return 0;
  });
}

int32_t orc_refine_levels(void* hh, int32_t band) {
  Handle* h = (Handle*)hh;
  return dispatch(h->s, h->dim, h->f64, [&](auto* s) { s->refine_levels(band); return 0; });
}

int32_t orc_get_particles(void* hh, double* x, double* v, double* F, double* C, double* m, int32_t* g, int32_t* fl,
                          double* Jp) {
  Handle* h = (Handle*)hh;
  return dispatch(h->s, h->dim, h->f64, [&](auto* s) {
    constexpr int D = std::remove_pointer_t<decltype(s)>::NC == 4 ? 2 : 3;
    for (int64_t i = 0; i < s->N * D; ++i) { if (x) x[i] = s->x[i]; if (v) v[i] = s->v[i]; }
    for (int64_t i = 0; i < s->N * D * D; ++i) { if (F) F[i] = s->F[i]; if (C) C[i] = s->C[i]; }
    for (int64_t i = 0; i < s->N; ++i) {
      if (m) m[i] = s->m[i]; if (g) g[i] = s->g[i]; if (fl) fl[i] = s->fl[i]; if (Jp) Jp[i] = s->Jp[i];
    }
    return 0;
  });
}

// Dense readback of level l over node/cell indices [lo, lo + n) per axis
// (row-major, first axis slowest).  Indices outside the stored range read 0.
int32_t orc_get_grid(void* hh, int32_t l, int32_t lo, int32_t n, double* m, double* v, int32_t* cell) {
  Handle* h = (Handle*)hh;
  return dispatch(h->s, h->dim, h->f64, [&](auto* s) {
    constexpr int D = std::remove_pointer_t<decltype(s)>::NC == 4 ? 2 : 3;
    if (l < 0 || l >= s->L) return 1;
    int64_t cnt = 1; for (int d = 0; d < D; ++d) cnt *= n;
    for (int64_t o = 0; o < cnt; ++o) {
      int I[D]; int64_t t = o;
      for (int d = D - 1; d >= 0; --d) { I[d] = (int)(t % n) + lo; t /= n; }
      int64_t li, lb;
      bool ok = s->lidx(s->lev[l], I, li, lb);
      if (m) m[o] = ok ? (double)s->lev[l].m[li] : 0.0;
      if (v) for (int c = 0; c < D; ++c) v[o * D + c] = ok ? (double)s->lev[l].v[li * D + c] : 0.0;
      if (cell) cell[o] = ok ? s->lev[l].cell[li] : 0;
    }
    return 0;
  });
}

// Node mask over the finest lattice [0, sz] per axis.
int32_t orc_get_node_mask(void* hh, int32_t* out) {
  Handle* h = (Handle*)hh;
  return dispatch(h->s, h->dim, h->f64, [&](auto* s) {
    constexpr int D = std::remove_pointer_t<decltype(s)>::NC == 4 ? 2 : 3;
    int n = s->sz + 1;
    int64_t cnt = 1; for (int d = 0; d < D; ++d) cnt *= n;
    for (int64_t o = 0; o < cnt; ++o) {
      int P[D]; int64_t t = o;
      for (int d = D - 1; d >= 0; --d) { P[d] = (int)(t % n); t /= n; }
      int64_t li, lb;
      out[o] = s->nm_idx(P, li, lb) ? s->nmask[li] : 0;
    }
    return 0;
  });
}

uint32_t orc_errors(void* hh) {
  Handle* h = (Handle*)hh;
  return h->s->err;
}

void orc_clear_errors(void* hh) { ((Handle*)hh)->s->err = 0; }

// ---- unit-level entry points ------------------------------------------------
void orc_weight_stencil(int32_t dim, int32_t use_f64, double radius, const double* tc, double* out) {
  if (dim == 2) {
    if (use_f64) { double W[9][3]; weight_stencil<2, double>(tc, radius, W); std::memcpy(out, W, sizeof(W)); }
    else {
      float t[2] = {(float)tc[0], (float)tc[1]}; float W[9][3];
      weight_stencil<2, float>(t, (float)radius, W);
      for (int i = 0; i < 9; ++i) for (int j = 0; j < 3; ++j) out[i * 3 + j] = W[i][j];
    }
  } else {
    if (use_f64) { double W[27][4]; weight_stencil<3, double>(tc, radius, W); std::memcpy(out, W, sizeof(W)); }
    else {
      float t[3] = {(float)tc[0], (float)tc[1], (float)tc[2]}; float W[27][4];
      weight_stencil<3, float>(t, (float)radius, W);
      for (int i = 0; i < 27; ++i) for (int j = 0; j < 4; ++j) out[i * 4 + j] = W[i][j];
    }
  }
}

void orc_stress(int32_t dim, int32_t use_f64, const double* F, double mu, double la, double* out) {
  if (dim == 2) {
    if (use_f64) get_stress<2, double>(F, mu, la, out);
    else {
      float f[4], o[4]; for (int i = 0; i < 4; ++i) f[i] = (float)F[i];
      get_stress<2, float>(f, (float)mu, (float)la, o);
      for (int i = 0; i < 4; ++i) out[i] = o[i];
    }
  } else {
    if (use_f64) get_stress<3, double>(F, mu, la, out);
    else {
      float f[9], o[9]; for (int i = 0; i < 9; ++i) f[i] = (float)F[i];
      get_stress<3, float>(f, (float)mu, (float)la, o);
      for (int i = 0; i < 9; ++i) out[i] = o[i];
    }
  }
}

void orc_svd(int32_t dim, const double* A, double* U, double* S, double* V) {
  if (dim == 2) svd_d<2>(A, U, S, V);
  else svd_d<3>(A, U, S, V);
}

}  // extern "C"

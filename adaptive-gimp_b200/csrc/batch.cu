// Batches of scenes: one launch per kernel for all scenes of a batch, under a
// CUDA graph per step phase, with launch sizes chosen by a measuring
// autotuner.  A single simulator steps through this same path as a batch of
// one.
//
// Launch layout.  Each launch kind (grid-stride kernels, the bin allocator)
// gives every scene a consecutive range of CTAs:
//   grid-stride kernels (over particles, active blocks or work items):
//     sms * ctas_per_sm CTAs shared in proportion to the scenes' particle
//     counts (at least one each);
//   bin allocator: a quarter of the scene's grid-stride CTAs (at least one).
// The kernels find their scene by binary search over the range starts.
#include <cstdlib>
#include <algorithm>
#include <cmath>
#include <cstring>

#include "sim.h"

namespace agimp {

#define BCK(call)                                                            \
  do {                                                                       \
    cudaError_t e_ = (call);                                                 \
    if (e_ != cudaSuccess) {                                                 \
      b->err = std::string(#call) + ": " + cudaGetErrorString(e_);           \
      return AGIMP_CUDA_ERROR;                                               \
    }                                                                        \
  } while (0)

Ctx& sim_ctx(agimp_sim* s) {
  s->c.P = s->buf[s->par];
  s->c.Q = s->buf[1 - s->par];
  return s->c;
}

agimp_status batch_init(agimp_batch* b) {
  const int n = (int)b->sims.size();
  {
    const char* e = std::getenv("AGIMP_PDL");
    b->pdl = !(e && e[0] == '0');
  }
  b->device = b->sims[0]->device;
  b->dim = b->sims[0]->c.dim;
  b->sms = b->sims[0]->c.sms;
  for (int k = 0; k < 2; ++k) {
    BCK(cudaMalloc(&b->dctx[k], sizeof(Ctx) * n));
    b->hctx[k].resize(n);
    std::memset(b->hctx[k].data(), 0, sizeof(Ctx) * n);
    b->hvalid[k].assign(n, 0);
  }
  BCK(cudaMalloc(&b->dofs, sizeof(int) * NMAP * (n + 1)));
  b->hofs.assign(NMAP * (n + 1), 0);
  BCK(cudaStreamCreateWithFlags(&b->side, cudaStreamNonBlocking));
  BCK(cudaEventCreateWithFlags(&b->ev_fork, cudaEventDisableTiming));
  BCK(cudaEventCreateWithFlags(&b->ev_join, cudaEventDisableTiming));
  if (!b->single) {
    BCK(cudaStreamCreateWithFlags(&b->internal, cudaStreamNonBlocking));
    BCK(cudaEventCreateWithFlags(&b->ev_in, cudaEventDisableTiming));
    BCK(cudaEventCreateWithFlags(&b->ev_out, cudaEventDisableTiming));
    BCK(cudaEventCreateWithFlags(&b->ev_done, cudaEventDisableTiming));
    BCK(cudaEventCreateWithFlags(&b->ev_read, cudaEventDisableTiming));
    BCK(cudaStreamCreateWithFlags(&b->gather, cudaStreamNonBlocking));
    for (int k = 0; k < 2; ++k) {
      BCK(cudaEventCreateWithFlags(&b->ev_xs[k], cudaEventDisableTiming));
      BCK(cudaEventCreateWithFlags(&b->ev_hsrc[k], cudaEventDisableTiming));
      BCK(cudaEventCreateWithFlags(&b->ev_gath[k], cudaEventDisableTiming));
    }
  }
  return AGIMP_OK;
}

void batch_drop_graphs(agimp_batch* b) {
  for (int k = 0; k < 2; ++k)
    if (b->gexec[k]) {
      cudaGraphExecDestroy(b->gexec[k]);
      b->gexec[k] = nullptr;
    }
}

// The batch's shared surrogate: slot buffers over all scenes' particles
// (allocated on first use), the MLP's parameters and the acceptance rule.
// packed == nullptr switches it off.
agimp_status batch_set_surrogate(agimp_batch* b, const void* packed, const float* P, const float* xmax, float tol) {
  BCK(cudaSetDevice(b->device));
  BCK(cudaDeviceSynchronize());
  batch_drop_graphs(b);
  for (int k = 0; k < 2; ++k) std::fill(b->hvalid[k].begin(), b->hvalid[k].end(), 0);
  if (!packed) {
    b->sur = 0;
    return AGIMP_OK;
  }
  long long tot = 0;
  for (agimp_sim* s : b->sims) tot += s->c.N;
  if (tot > b->scap) {
    if (b->sX) cudaFree(b->sX);
    if (b->sY) cudaFree(b->sY);
    if (b->smeta) cudaFree(b->smeta);
    b->sX = b->sY = b->smeta = nullptr;
    b->scap = 0;
    BCK(cudaMalloc(&b->sX, sizeof(float) * (tot * 7 + 8)));
    BCK(cudaMalloc(&b->sY, sizeof(float) * (tot * 4 + 8)));
    BCK(cudaMalloc(&b->smeta, sizeof(float) * (tot * SUR_META + 8)));
    b->scap = tot;
  }
  if (!b->sctr) {
    BCK(cudaMalloc(&b->sctr, 2 * sizeof(int32_t)));
    BCK(cudaMemset(b->sctr, 0, 2 * sizeof(int32_t)));
  }
  b->mlp_packed = packed;
  b->mlp_P = P;
  for (int k = 0; k < 8; ++k) b->sur_xmax[k] = k < 7 ? xmax[k] : 0.f;
  b->sur_tol = tol;
  b->sur = 1;
  return AGIMP_OK;
}

void batch_free(agimp_batch* b) {
  batch_drop_graphs(b);
  if (b->sX) cudaFree(b->sX);
  if (b->sY) cudaFree(b->sY);
  if (b->smeta) cudaFree(b->smeta);
  if (b->sctr) cudaFree(b->sctr);
  b->sX = b->sY = b->smeta = nullptr;
  b->sctr = nullptr;
  for (int k = 0; k < 2; ++k)
    if (b->dctx[k]) cudaFree(b->dctx[k]);
  if (b->dofs) cudaFree(b->dofs);
  if (b->internal) cudaStreamDestroy(b->internal);
  if (b->side) cudaStreamDestroy(b->side);
  if (b->ev_fork) cudaEventDestroy(b->ev_fork);
  if (b->ev_join) cudaEventDestroy(b->ev_join);
  if (b->ev_in) cudaEventDestroy(b->ev_in);
  if (b->ev_out) cudaEventDestroy(b->ev_out);
  if (b->ev_done) cudaEventDestroy(b->ev_done);
  if (b->ev_read) cudaEventDestroy(b->ev_read);
  if (b->xstage) cudaFree(b->xstage);
  if (b->dsrc) cudaFree(b->dsrc);
  if (b->hsrc) cudaFreeHost(b->hsrc);
  if (b->ustage) cudaFree(b->ustage);
  if (b->utab) cudaFree(b->utab);
  if (b->utab_h) cudaFreeHost(b->utab_h);
  b->ustage = nullptr;
  b->utab = b->utab_h = nullptr;
  b->ustage_floats = 0;
  if (b->gather) cudaStreamDestroy(b->gather);
  for (int k = 0; k < 2; ++k)
    for (cudaEvent_t* e : {&b->ev_xs[k], &b->ev_hsrc[k], &b->ev_gath[k]}) {
      if (*e) cudaEventDestroy(*e);
      *e = nullptr;
    }
  b->ev_done = b->ev_read = nullptr;
  b->xstage = nullptr;
  b->dsrc = nullptr;
  b->hsrc = nullptr;
  b->gather = nullptr;
  b->xstage_floats = 0;
  b->xs_busy[0] = b->xs_busy[1] = b->hsrc_busy[0] = b->hsrc_busy[1] = false;
  b->dctx[0] = b->dctx[1] = nullptr;
  b->dofs = nullptr;
  b->internal = nullptr;
  b->ev_in = b->ev_out = nullptr;
}

// CTA ranges of every launch kind (host copy in b->hofs, uploaded on `use`).
static agimp_status build_maps(agimp_batch* b, cudaStream_t use) {
  const int n = (int)b->sims.size();
  long long sumN = 0;
  for (agimp_sim* s : b->sims) sumN += s->c.N;
  const long long G = (long long)b->sms * b->tune.ctas_per_sm;
  // P2G: whole waves of resident CTAs (a partly filled last wave leaves SMs
  // idle at the end of the kernel), at least as many CTAs as the other kinds
  const int res = p2g_resident(b->dim, b->tune.chunk);
  const long long wave = (long long)b->sms * res;
  const long long GP = std::max<long long>(1, (G + wave - 1) / wave) * wave;
  int* Gm = b->hofs.data() + MAP_G * (n + 1);
  int* O = b->hofs.data() + MAP_O * (n + 1);
  int* T = b->hofs.data() + MAP_T * (n + 1);
  int* Pm = b->hofs.data() + MAP_P * (n + 1);
  Gm[0] = O[0] = T[0] = Pm[0] = 0;
  auto share = [&](long long tot, long long N) {
    return n == 1 ? (int)std::max<long long>(1, tot)
                  : (int)std::max<long long>(1, sumN ? (long long)std::llround((double)tot * N / sumN) : 1);
  };
  for (int i = 0; i < n; ++i) {
    const long long N = b->sims[i]->c.N;
    const int cg = share(G, N);
    Gm[i + 1] = Gm[i] + cg;
    O[i + 1] = O[i] + std::max(1, cg / 4);
    T[i + 1] = T[i] + 4 * cg;
    Pm[i + 1] = Pm[i] + share(GP, N);
  }
  b->nct[MAP_G] = Gm[n];
  b->nct[MAP_O] = O[n];
  b->nct[MAP_T] = T[n];
  b->nct[MAP_P] = Pm[n];
  BCK(cudaMemcpyAsync(b->dofs, b->hofs.data(), sizeof(int) * b->hofs.size(), cudaMemcpyHostToDevice, use));
  b->maps_valid = true;
  return AGIMP_OK;
}

// Bring the device contexts of phase `ph` up to date with the scenes' state.
static agimp_status sync_contexts(agimp_batch* b, int ph, float dt, cudaStream_t use) {
  const int n = (int)b->sims.size();
  int lo = n, hi = -1;
  for (int i = 0; i < n; ++i) {
    Ctx& c = sim_ctx(b->sims[i]);
    c.dt = dt;
    c.chunk = b->tune.chunk;
    // what this batch uploads: the scene's context with its index here and,
    // in a batch of several, the batch's surrogate setting in place of the
    // scene's own
    Ctx t = c;
    t.scene = i;
    if (!b->single) {
      t.sur = b->sur && c.plast == 1;
      if (b->sur) {
        t.mlp_packed = b->mlp_packed;
        t.mlp_P = b->mlp_P;
        t.sur_X = b->sX;
        t.sur_Y = b->sY;
        t.sur_meta = b->smeta;
        t.sur_ctr = b->sctr;
        t.sur_tol = b->sur_tol;
        for (int k = 0; k < 8; ++k) t.sur_xmax[k] = b->sur_xmax[k];
      }
    }
    Ctx& h = b->hctx[ph][i];
    if (!b->hvalid[ph][i] || std::memcmp(&h, &t, sizeof(Ctx)) != 0) {
      std::memcpy(&h, &t, sizeof(Ctx));
      b->hvalid[ph][i] = 1;
      lo = std::min(lo, i);
      hi = std::max(hi, i);
    }
  }
  if (hi >= lo)
    BCK(cudaMemcpyAsync(b->dctx[ph] + lo, b->hctx[ph].data() + lo, sizeof(Ctx) * (hi - lo + 1),
                        cudaMemcpyHostToDevice, use));
  return AGIMP_OK;
}

static BatchLaunch make_launch(agimp_batch* b, int ph) {
  BatchLaunch bl;
  const int n = (int)b->sims.size();
  bl.b.ctx = b->dctx[ph];
  bl.b.ofs = b->dofs;
  bl.b.n = n;
  bl.dim = b->dim;
  bl.maxL = 1;
  bl.any_dynamic = 0;
  bl.any_plastic = 0;
  for (agimp_sim* s : b->sims) {
    bl.maxL = std::max(bl.maxL, s->c.L);
    if (!s->c.is_static) bl.any_dynamic = 1;
    if (s->c.plast == 1) bl.any_plastic = 1;
  }
  for (int k = 0; k < NMAP; ++k) bl.nct[k] = b->nct[k];
  bl.chunk = b->tune.chunk;
  bl.single = b->single ? &b->hctx[ph][0] : nullptr;
  bl.side = b->side;
  bl.fork = b->ev_fork;
  bl.join = b->ev_join;
  bl.pdl = b->pdl;
  bl.sms = b->sms;
  bl.sur = 0;
  if (b->single) {
    const Ctx& c = b->hctx[ph][0];
    if (c.sur && c.plast == 1 && c.N) {
      bl.sur = 1;
      bl.mlp_packed = c.mlp_packed;
      bl.mlp_P = c.mlp_P;
      bl.sur_X = c.sur_X;
      bl.sur_Y = c.sur_Y;
      bl.sur_meta = c.sur_meta;
      bl.sur_n = c.sur_ctr;
      bl.sur_cap = c.N;
      bl.sur_err = c.ctr + CTR_ERR;
    }
  } else if (b->sur && bl.any_plastic && b->scap) {
    bl.sur = 1;
    bl.mlp_packed = b->mlp_packed;
    bl.mlp_P = b->mlp_P;
    bl.sur_X = b->sX;
    bl.sur_Y = b->sY;
    bl.sur_meta = b->smeta;
    bl.sur_n = b->sctr;
    bl.sur_cap = b->scap;
    bl.sur_err = b->sctr + 1;
  }
  return bl;
}

static agimp_batch::Key launch_key(const BatchLaunch& bl, cudaStream_t use) {
  agimp_batch::Key k;
  std::memset(&k, 0, sizeof(k));
  k.maxL = bl.maxL;
  k.any_dynamic = bl.any_dynamic;
  k.any_plastic = bl.any_plastic;
  k.chunk = bl.chunk;
  k.sur = bl.sur;
  for (int i = 0; i < NMAP; ++i) k.nct[i] = bl.nct[i];
  k.stream = use;
  return k;
}

agimp_status batch_step(agimp_batch* b, float dt, int n, cudaStream_t use, cudaEvent_t* ev) {
  BCK(cudaSetDevice(b->device));
  if (!b->maps_valid) {
    const agimp_status st = build_maps(b, use);
    if (st != AGIMP_OK) return st;
  }
  for (int i = 0; i < n; ++i) {
    // the substep writes each scene's other buffer: wait for readbacks of it
    for (agimp_sim* s : b->sims) wait_readback(s, 1 - s->par, use);
    if (b->read_pending && b->steps > b->read_step) {  // the batch copy read those buffers
      BCK(cudaStreamWaitEvent(use, b->ev_read, 0));
      b->read_pending = false;
    }
    const int ph = b->single ? b->sims[0]->par : (int)(b->steps & 1);
    agimp_status st = sync_contexts(b, ph, dt, use);
    if (st != AGIMP_OK) return st;
    BatchLaunch bl = make_launch(b, ph);
    if (ev) bl.side = nullptr;  // phase timing: one stream
    if (ev || !b->graphs) {
      launch_substep(bl, use, ev);
      BCK(cudaGetLastError());
    } else {
      const agimp_batch::Key key = launch_key(bl, use);
      if (!b->gexec[ph] || std::memcmp(&key, &b->gkey[ph], sizeof(key)) != 0) {
        if (b->gexec[ph]) {
          cudaGraphExecDestroy(b->gexec[ph]);
          b->gexec[ph] = nullptr;
        }
        cudaGraph_t graph = nullptr;
        BCK(cudaStreamBeginCapture(use, cudaStreamCaptureModeThreadLocal));
        launch_substep(bl, use, nullptr);
        BCK(cudaStreamEndCapture(use, &graph));
        const cudaError_t e = cudaGraphInstantiate(&b->gexec[ph], graph, 0);
        cudaGraphDestroy(graph);
        BCK(e);
        std::memcpy(&b->gkey[ph], &key, sizeof(key));
      }
      BCK(cudaGraphLaunch(b->gexec[ph], use));
    }
    for (agimp_sim* s : b->sims) {
      s->par ^= 1;  // the new state is in the other buffer
      s->substeps += 1;
      s->bins_valid = true;
    }
    b->steps += 1;
  }
  // state-ready marks for asynchronous readbacks (a batch of one always
  // records it; larger batches only for scenes that read asynchronously)
  for (agimp_sim* s : b->sims)
    if (n > 0) {
      const bool mark = b->single || s->async_used;
      if (mark) BCK(cudaEventRecord(s->ev_state, use));
      s->state_marked = mark;
    }
  if (b->ev_done && n > 0) BCK(cudaEventRecord(b->ev_done, use));
  return AGIMP_OK;
}

namespace {
struct GatherSrc {
  const float* x;
  const int32_t* id;
  long long N, off;
};

// every scene's positions, in its caller's particle order, at its offset
template <int D>
__global__ void k_gather_x(const int* ofs, int n, const GatherSrc* src, float* out) {
  const int cta = (int)blockIdx.x;
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (ofs[mid] <= cta)
      lo = mid;
    else
      hi = mid - 1;
  }
  const GatherSrc g = src[lo];
  const int bid = cta - ofs[lo], nblk = ofs[lo + 1] - ofs[lo];
  for (long long s = bid * (long long)blockDim.x + threadIdx.x; s < g.N; s += (long long)nblk * blockDim.x) {
    const long long o = (g.off + g.id[s]) * D;
#pragma unroll
    for (int d = 0; d < D; ++d) out[o + d] = g.x[d * g.N + s];
  }
}
}  // namespace

agimp_status batch_positions_async(agimp_batch* b, float* x, cudaStream_t use) {
  BCK(cudaSetDevice(b->device));
  if (b->single || !x) {
    b->err = "batch positions: a batch of several scenes and an output are required";
    return AGIMP_INVALID_ARG;
  }
  if (!b->maps_valid) {
    const agimp_status st = build_maps(b, use);
    if (st != AGIMP_OK) return st;
  }
  const int n = (int)b->sims.size();
  long long tot = 0;
  for (agimp_sim* s : b->sims) tot += s->c.N;
  if (!b->xstage) {
    const long long per = std::max<long long>(tot * b->dim, 1);
    BCK(cudaMalloc(&b->xstage, 2 * per * sizeof(float)));
    BCK(cudaMalloc(&b->dsrc, 2 * sizeof(GatherSrc) * n));
    BCK(cudaMallocHost(&b->hsrc, 2 * sizeof(GatherSrc) * n));
    b->xstage_floats = per;
  }
  // Two slots.  The source table goes to the device from pinned memory (an
  // upload from pageable memory would wait for the stream); the gather runs
  // on the batch's gather stream behind the last substep and the slot's
  // previous host copy, so it frees the scenes' state without waiting for
  // the previous readback's copy; the host copy runs on the caller's stream.
  const int slot = b->xs_next;
  b->xs_next ^= 1;
  GatherSrc* hs = (GatherSrc*)b->hsrc + (size_t)slot * n;
  GatherSrc* ds = (GatherSrc*)b->dsrc + (size_t)slot * n;
  float* xs = b->xstage + (size_t)slot * b->xstage_floats;
  if (b->hsrc_busy[slot]) BCK(cudaEventSynchronize(b->ev_hsrc[slot]));  // its last upload has run
  long long off = 0;
  for (int i = 0; i < n; ++i) {
    agimp_sim* s = b->sims[i];
    hs[i] = GatherSrc{s->buf[s->par].x, s->buf[s->par].id, (long long)s->c.N, off};
    off += s->c.N;
  }
  cudaStream_t gs = b->gather;
  BCK(cudaStreamWaitEvent(gs, b->ev_done, 0));  // the batch's last substep is written
  if (b->xs_busy[slot]) BCK(cudaStreamWaitEvent(gs, b->ev_xs[slot], 0));  // the slot's last copy is done
  BCK(cudaMemcpyAsync(ds, hs, sizeof(GatherSrc) * n, cudaMemcpyHostToDevice, gs));
  BCK(cudaEventRecord(b->ev_hsrc[slot], gs));
  b->hsrc_busy[slot] = true;
  const int G = b->nct[MAP_G];
  if (b->dim == 2)
    k_gather_x<2><<<G, 256, 0, gs>>>(b->dofs + MAP_G * (n + 1), n, ds, xs);
  else
    k_gather_x<3><<<G, 256, 0, gs>>>(b->dofs + MAP_G * (n + 1), n, ds, xs);
  BCK(cudaGetLastError());
  // the scenes' state has been read: the substep that overwrites it may run
  BCK(cudaEventRecord(b->ev_read, gs));
  b->read_pending = true;
  b->read_step = b->steps;
  BCK(cudaEventRecord(b->ev_gath[slot], gs));
  BCK(cudaStreamWaitEvent(use, b->ev_gath[slot], 0));
  BCK(cudaMemcpyAsync(x, xs, tot * b->dim * sizeof(float), cudaMemcpyDeviceToHost, use));
  BCK(cudaEventRecord(b->ev_xs[slot], use));
  b->xs_busy[slot] = true;
  return AGIMP_OK;
}

namespace {
struct ScatterDst {
  void* dst;           // the scene's field: comps x N, slot-major per component
  const int32_t* id;   // storage slot -> caller index
  long long N, off;    // particles; first index in the concatenated arrays
};

// every scene's field from the concatenated caller arrays (particle-major,
// comps values each, scenes in batch order) into its storage
template <typename T>
__global__ void k_scatter_in(const int* ofs, int n, const ScatterDst* tab, const T* src, int comps) {
  const int cta = (int)blockIdx.x;
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (ofs[mid] <= cta)
      lo = mid;
    else
      hi = mid - 1;
  }
  const ScatterDst t = tab[lo];
  T* dst = (T*)t.dst;
  const int bid = cta - ofs[lo], nblk = ofs[lo + 1] - ofs[lo];
  for (long long s = bid * (long long)blockDim.x + threadIdx.x; s < t.N; s += (long long)nblk * blockDim.x) {
    const long long o = (t.off + t.id[s]) * comps;
    for (int c = 0; c < comps; ++c) dst[c * t.N + s] = src[o + c];
  }
}
}  // namespace

agimp_status batch_set_particles(agimp_batch* b, const float* x, const float* v, const float* F, const float* C,
                                 const float* m, const int32_t* g, const float* Jp, int memory, cudaStream_t use) {
  BCK(cudaSetDevice(b->device));
  if (b->single || (memory != AGIMP_MEM_DEVICE && memory != AGIMP_MEM_HOST)) {
    b->err = "batch upload: a batch of several scenes and a memory kind are required";
    return AGIMP_INVALID_ARG;
  }
  if (!b->maps_valid) {
    const agimp_status st = build_maps(b, use);
    if (st != AGIMP_OK) return st;
  }
  const int n = (int)b->sims.size(), D = b->dim;
  long long tot = 0;
  for (agimp_sim* s : b->sims) tot += s->c.N;
  // the state being overwritten may still be read by asynchronous readbacks
  for (agimp_sim* s : b->sims) {
    wait_readback(s, s->par, use);
    s->bins_valid = false;
  }
  if (b->read_pending) BCK(cudaStreamWaitEvent(use, b->ev_read, 0));
  const void* fields[7] = {x, v, F, C, m, Jp, g};
  const int comps[7] = {D, D, D * D, D * D, 1, 1, 1};
  const size_t need = (size_t)std::max<long long>(tot, 1) * D * D;
  if (memory == AGIMP_MEM_HOST && need > b->ustage_floats) {
    if (b->ustage) BCK(cudaFree(b->ustage));
    b->ustage = nullptr;
    b->ustage_floats = 0;
    BCK(cudaMalloc(&b->ustage, need * sizeof(float)));
    b->ustage_floats = need;
  }
  if (!b->utab) {
    BCK(cudaMalloc(&b->utab, 7 * sizeof(ScatterDst) * n));
    BCK(cudaMallocHost(&b->utab_h, 7 * sizeof(ScatterDst) * n));
  }
  ScatterDst* th = (ScatterDst*)b->utab_h;
  long long off = 0;
  for (int i = 0; i < n; ++i) {
    agimp_sim* s = b->sims[i];
    const Particles& P = s->buf[s->par];
    void* dst[7] = {P.x, P.v, P.F, P.C, P.m, P.Jp, P.g};
    for (int f = 0; f < 7; ++f) th[f * n + i] = ScatterDst{dst[f], P.id, (long long)s->c.N, off};
    off += s->c.N;
  }
  BCK(cudaMemcpyAsync(b->utab, th, 7 * sizeof(ScatterDst) * n, cudaMemcpyHostToDevice, use));
  const int G = b->nct[MAP_G];
  for (int f = 0; f < 7; ++f) {
    if (!fields[f] || tot == 0) continue;
    const void* src = fields[f];
    if (memory == AGIMP_MEM_HOST) {
      // one field at a time through the staging buffer (stream order keeps
      // the next field's copy behind this field's scatter)
      BCK(cudaMemcpyAsync(b->ustage, src, tot * comps[f] * sizeof(float), cudaMemcpyHostToDevice, use));
      src = b->ustage;
    }
    const ScatterDst* td = (const ScatterDst*)b->utab + (size_t)f * n;
    if (f == 6)
      k_scatter_in<int32_t><<<G, 256, 0, use>>>(b->dofs + MAP_G * (n + 1), n, td, (const int32_t*)src, 1);
    else
      k_scatter_in<float><<<G, 256, 0, use>>>(b->dofs + MAP_G * (n + 1), n, td, (const float*)src, comps[f]);
    BCK(cudaGetLastError());
  }
  for (agimp_sim* s : b->sims) {
    BCK(cudaEventRecord(s->ev_state, use));  // later asynchronous readbacks follow the upload
    s->state_marked = true;
  }
  // the pinned table (and host arrays) may be reused on return
  BCK(cudaStreamSynchronize(use));
  return AGIMP_OK;
}

void wait_readback(agimp_sim* s, int buf, cudaStream_t use) {
  if (s->read_pending[buf]) {
    cudaStreamWaitEvent(use, s->ev_read[buf], 0);
    s->read_pending[buf] = false;
  }
}

int batch_kernels(agimp_batch* b) {
  const BatchLaunch bl = make_launch(b, 0);
  const Ctx& c = b->sims[0]->c;
  return kernels_per_substep(bl) + ((b->single && c.sur && c.plast == 1 && c.N) ? 2 : 0);
}

agimp_status batch_set_tuning(agimp_batch* b, const agimp_tuning* t) {
  if (!t || (t->chunk != 64 && t->chunk != 128 && t->chunk != 256 && t->chunk != 512) || t->ctas_per_sm < 1 ||
      t->ctas_per_sm > 32) {
    b->err = "tuning: chunk must be 64, 128, 256 or 512 and ctas_per_sm in [1, 32]";
    return AGIMP_INVALID_ARG;
  }
  b->tune.chunk = t->chunk;
  b->tune.ctas_per_sm = t->ctas_per_sm;
  b->tune.ms_per_substep = t->ms_per_substep;
  b->maps_valid = false;
  batch_drop_graphs(b);
  return AGIMP_OK;
}

// ---------------------------------------------------------------------------
// Autotuner.  Every candidate (P2G work-item size x grid-stride CTAs per SM)
// runs `trials` timed substeps after two warm-up substeps (which capture its
// graphs) from the same saved particle state; the fastest is kept.  The saved
// state is put back after each candidate, so tuning leaves the simulation
// where it was.  The grid itself needs no restoring: every substep clears the
// blocks the previous substep activated, whichever they were.
namespace {

struct Saved {
  agimp_sim* s;
  int par;
  long long substeps;
  int32_t err, rec;
  char* data;  // particle arrays of buf[par]
};

size_t state_bytes(const agimp_sim* s) {
  const size_t N = s->c.N, D = s->c.dim;
  return (2 * D + 2 * D * D + 5) * N * 4;
}

template <class F>
void for_each_array(agimp_sim* s, const Particles& P, F f) {
  const size_t N = s->c.N, D = s->c.dim;
  f(P.x, D * N * 4);
  f(P.v, D * N * 4);
  f(P.F, D * D * N * 4);
  f(P.C, D * D * N * 4);
  f(P.m, N * 4);
  f(P.Jp, N * 4);
  f(P.g, N * 4);
  f(P.fl, N * 4);
  f(P.id, N * 4);
}

}  // namespace

agimp_status batch_autotune(agimp_batch* b, float dt, int trials, agimp_tuning* best, cudaStream_t use) {
  BCK(cudaSetDevice(b->device));
  if (trials < 1 || trials > 1000) {
    b->err = "trials must be in [1, 1000]";
    return AGIMP_INVALID_ARG;
  }
  size_t total = 0;
  for (agimp_sim* s : b->sims) total += state_bytes(s);
  char* scratch = nullptr;
  BCK(cudaMalloc(&scratch, std::max<size_t>(total, 16)));
  std::vector<Saved> saved;
  size_t off = 0;
  for (agimp_sim* s : b->sims) {
    Saved v{s, s->par, s->substeps, 0, 0, scratch + off};
    int32_t h[2];
    cudaMemcpyAsync(&h[0], s->c.ctr + CTR_ERR, 4, cudaMemcpyDeviceToHost, use);
    cudaMemcpyAsync(&h[1], s->c.ctr + CTR_REC, 4, cudaMemcpyDeviceToHost, use);
    cudaStreamSynchronize(use);
    v.err = h[0];
    v.rec = h[1];
    size_t o = 0;
    for_each_array(s, s->buf[s->par], [&](const void* p, size_t nb) {
      cudaMemcpyAsync(v.data + o, p, nb, cudaMemcpyDeviceToDevice, use);
      o += nb;
    });
    off += state_bytes(s);
    saved.push_back(v);
  }
  auto restore = [&]() {
    for (Saved& v : saved) {
      agimp_sim* s = v.s;
      s->par = v.par;
      s->substeps = v.substeps;
      s->bins_valid = false;  // the restored state was not binned by the last substep
      size_t o = 0;
      for_each_array(s, s->buf[v.par], [&](void* p, size_t nb) {
        cudaMemcpyAsync(p, v.data + o, nb, cudaMemcpyDeviceToDevice, use);
        o += nb;
      });
      cudaMemcpyAsync(s->c.ctr + CTR_ERR, &v.err, 4, cudaMemcpyHostToDevice, use);
      cudaMemcpyAsync(s->c.ctr + CTR_REC, &v.rec, 4, cudaMemcpyHostToDevice, use);
      cudaEventRecord(s->ev_state, use);  // the restored state is the last write
      s->state_marked = true;
    }
    return cudaStreamSynchronize(use);
  };
  const agimp_tuning old = b->tune;
  agimp_tuning top{0, 0, INFINITY};
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  agimp_status st = AGIMP_OK;
  const int chunks[4] = {64, 128, 256, 512};
  const int cps[4] = {2, 4, 8, 16};
  for (int ci = 0; ci < 4 && st == AGIMP_OK; ++ci)
    for (int gi = 0; gi < 4 && st == AGIMP_OK; ++gi) {
      agimp_tuning t{chunks[ci], cps[gi], 0.f};
      st = batch_set_tuning(b, &t);
      if (st == AGIMP_OK) st = batch_step(b, dt, 2, use, nullptr);
      if (st != AGIMP_OK) break;
      cudaEventRecord(e0, use);
      st = batch_step(b, dt, trials, use, nullptr);
      cudaEventRecord(e1, use);
      const cudaError_t e = cudaEventSynchronize(e1);
      float ms = 0.f;
      if (e == cudaSuccess) cudaEventElapsedTime(&ms, e0, e1);
      const cudaError_t r = restore();
      if (st == AGIMP_OK && (e != cudaSuccess || r != cudaSuccess)) {
        b->err = std::string("autotune: ") + cudaGetErrorString(e != cudaSuccess ? e : r);
        st = AGIMP_CUDA_ERROR;
      }
      t.ms_per_substep = ms / trials;
      if (st == AGIMP_OK && t.ms_per_substep < top.ms_per_substep) top = t;
    }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(scratch);
  if (st != AGIMP_OK) {
    batch_set_tuning(b, &old);
    return st;
  }
  st = batch_set_tuning(b, &top);
  if (best) *best = top;
  return st;
}

}  // namespace agimp

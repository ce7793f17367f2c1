// C ABI of libagimp.so (declared in include/agimp.h).
//
// Host side of the reference's AdaptiveGIMP class (adaptive_gimp.py:4-352):
// storage allocation (__init__), particle and level-map upload (the
// particle_initializer / grid_initializer hooks), substep() and field
// readback.  Every kernel launch is stream-ordered; the substep is captured as
// a CUDA graph once per (dt, stream) and replayed.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "sim.h"

using namespace agimp;

namespace agimp {
void mlp_buffers(const agimp_mlp* m, const void** packed, const float** P);
}

namespace {

// the simulator's kernel context with P = current state, Q = the other buffer
Ctx& cur(agimp_sim* s) { return sim_ctx(s); }

// captured substeps depend on the launch structure and the surrogate settings
void drop_graphs(agimp_sim* s) {
  if (s->self) batch_drop_graphs(s->self);
}

// status of a batch call on the simulator's own batch, with its message
agimp_status from_batch(agimp_sim* s, agimp_status st) {
  if (st != AGIMP_OK) s->err = s->self->err;
  return st;
}

agimp_status fail(agimp_sim* s, agimp_status st, const std::string& msg) {
  if (s) s->err = msg;
  return st;
}

agimp_status cuda_fail(agimp_sim* s, cudaError_t e, const char* what) {
  return fail(s, AGIMP_CUDA_ERROR, std::string(what) + ": " + cudaGetErrorString(e));
}

#define CK(call)                                        \
  do {                                                  \
    cudaError_t e_ = (call);                            \
    if (e_ != cudaSuccess) return cuda_fail(s, e_, #call); \
  } while (0)

template <typename T>
cudaError_t dalloc(agimp_sim* s, T** ptr, size_t count) {
  void* p = nullptr;
  cudaError_t e = cudaMalloc(&p, count * sizeof(T) + 16);
  if (e != cudaSuccess) return e;
  s->allocs.push_back(p);
  *ptr = (T*)p;
  return cudaSuccess;
}

// RAII: run library work on the caller's stream, or on an internal stream
// ordered after / before the legacy default stream when the caller passes NULL
// (a graph cannot be captured on the legacy stream).
struct StreamUse {
  agimp_sim* s;
  cudaStream_t user, use;
  StreamUse(agimp_sim* s_, void* stream) : s(s_), user((cudaStream_t)stream) {
    use = user ? user : s->internal;
    if (!user) {
      cudaEventRecord(s->ev_in, 0);
      cudaStreamWaitEvent(s->internal, s->ev_in, 0);
    }
  }
  ~StreamUse() {
    if (!user) {
      cudaEventRecord(s->ev_out, s->internal);
      cudaStreamWaitEvent(0, s->ev_out, 0);
    }
  }
};

// Caller arrays are in the caller's particle order; storage slot i holds
// particle id[i].
__global__ void k_aos_to_soa(const float* __restrict__ aos, const int32_t* __restrict__ id, float* __restrict__ soa,
                             long long n, int comps) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n * comps;
       i += (long long)gridDim.x * blockDim.x) {
    const long long slot = i / comps;
    const int c = (int)(i % comps);
    soa[c * n + slot] = aos[(long long)id[slot] * comps + c];
  }
}

__global__ void k_soa_to_aos(const float* __restrict__ soa, const int32_t* __restrict__ id, float* __restrict__ aos,
                             long long n, int comps) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n * comps;
       i += (long long)gridDim.x * blockDim.x) {
    const long long slot = i / comps;
    const int c = (int)(i % comps);
    aos[(long long)id[slot] * comps + c] = soa[c * n + slot];
  }
}

__global__ void k_i32_in(const int32_t* __restrict__ src, const int32_t* __restrict__ id, int32_t* __restrict__ dst,
                         long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    dst[i] = src[id[i]];
}

__global__ void k_i32_out(const int32_t* __restrict__ src, const int32_t* __restrict__ id, int32_t* __restrict__ dst,
                          long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    dst[id[i]] = src[i];
}

// Bin key of every particle in the last substep (adaptive_gimp.py:208-216:
// particle p goes to pid[fl_p] at block base // 4 of level fl_p): the level in
// bits 60-63 and per axis the block coordinate plus one (floor(base / 4) + 1,
// the stored block index) in a 20-bit field, first axis highest; ~0 for
// particles without a level.  Slot j of the current state came from slot
// perm[j] of the binned state, whose bin_of holds the bin.
template <int D>
__global__ void k_get_bins(Ctx c, const int32_t* __restrict__ id, unsigned long long* __restrict__ out) {
  long long nbins = 0;
  for (int q = 0; q < c.L; ++q) nbins += c.ctr[CTR_LEVEL + q];
  for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < c.N; j += (long long)gridDim.x * blockDim.x) {
    const long long b = (long long)(c.bin_of[c.perm[j]] >> (2 * D));
    unsigned long long key = ~0ull;
    if (b < nbins) {
      int l = 0;
      long long r = b;
      while (l < c.L - 1 && r >= c.ctr[CTR_LEVEL + l]) {
        r -= c.ctr[CTR_LEVEL + l];
        ++l;
      }
      unsigned blk = (unsigned)c.lev[l].blist[r];
      const unsigned nb = (unsigned)c.lev[l].nb;
      key = (unsigned long long)l << 60;
#pragma unroll
      for (int d = D - 1; d >= 0; --d) {
        key |= (unsigned long long)(blk % nb) << (20 * (D - 1 - d));
        blk /= nb;
      }
    }
    out[id[j]] = key;
  }
}

__global__ void k_iota(int32_t* __restrict__ id, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    id[i] = (int32_t)i;
}

template <int D>
__global__ void k_get_grid(Ctx c, int l, int lo, int n, long long off, long long cnt, float* m, float* v,
                           int32_t* cell) {
  const LevelDev& V = c.lev[l];
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < cnt; i += (long long)gridDim.x * blockDim.x) {
    long long o = off + i;
    int I[D];
#pragma unroll
    for (int d = D - 1; d >= 0; --d) {
      I[d] = (int)(o % n) + lo;
      o /= n;
    }
    float4 nd = make_float4(0.f, 0.f, 0.f, 0.f);
    uint32_t cm = 0;
    if (in_store<D>(V, I)) {
      const long long e = elem_of<D>(V, I);
      nd = V.node[e];
      cm = V.cell[e] & ~CUL;
    }
    if (m) m[i] = nd.w;
    if (v) {
      v[i * D] = nd.x;
      v[i * D + 1] = nd.y;
      if (D == 3) v[i * D + 2] = nd.z;
    }
    if (cell) cell[i] = (int32_t)cm;
  }
}

template <int D>
__global__ void k_get_nmask(Ctx c, long long off, long long cnt, int32_t* out) {
  const int n = c.sz + 1;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < cnt; i += (long long)gridDim.x * blockDim.x) {
    long long o = off + i;
    int P[D];
#pragma unroll
    for (int d = D - 1; d >= 0; --d) {
      P[d] = (int)(o % n);
      o /= n;
    }
    out[i] = (int32_t)c.nmask[elem_of<D>(c.lev[c.L - 1], P)];
  }
}

int gs_blocks(long long n) {
  long long b = (n + 255) / 256;
  if (b > 65535) b = 65535;
  return (int)(b < 1 ? 1 : b);
}

}  // namespace

namespace agimp {
// Makes the device table (ownership passes to the simulator) its level map
// and switches the substep to static activation.
agimp_status install_level_map(agimp_sim* s, int8_t* dev_table, int halo, int n) {
  CK(cudaDeviceSynchronize());  // substeps in flight may read the old map
  if (s->map_dev) cudaFree(s->map_dev);
  s->map_dev = dev_table;
  if (!s->c.touch_occ) {
    // base-cell records of the touched blocks (static mode only)
    const size_t words = (size_t)s->c.lev[s->c.L - 1].nblocks * (s->c.dim == 2 ? 1 : 5);
    CK(cudaMalloc(&s->c.touch_occ, words * sizeof(uint32_t)));
    CK(cudaMemset(s->c.touch_occ, 0, words * sizeof(uint32_t)));
  }
  s->c.map = s->map_dev;
  s->c.map_h = halo;
  s->c.map_n = n;
  s->c.is_static = 1;
  drop_graphs(s);
  return AGIMP_OK;
}
}  // namespace agimp

extern "C" {

int agimp_abi_version(void) { return AGIMP_ABI_VERSION; }

const char* agimp_status_string(agimp_status st) {
  switch (st) {
    case AGIMP_OK: return "ok";
    case AGIMP_INVALID_ARG: return "invalid argument";
    case AGIMP_CAPACITY: return "capacity exceeded";
    case AGIMP_NAN: return "non-finite value";
    case AGIMP_DEVICE_TIMEOUT: return "device wait timed out";
    case AGIMP_CUDA_ERROR: return "CUDA error";
    case AGIMP_NOT_READY: return "not ready";
    case AGIMP_OUT_OF_MEMORY: return "out of device memory";
  }
  return "unknown status";
}

void agimp_default_params(agimp_params* p, int32_t dim, int32_t level, int32_t coarsest_size, int64_t n) {
  std::memset(p, 0, sizeof(*p));
  p->dim = dim;
  p->level = level;
  p->coarsest_size = coarsest_size;
  p->boundary_gap = 4;
  p->boundary_mode = 0;
  p->plasticity = 0;
  p->invalid_nodes = 0;
  p->n_particles = n;
  p->radius = 0.5;
  p->gravity[1] = -100.0;
  p->E = 5e3;
  p->nu = 0.2;
  p->theta_c = 2.5e-2;
  p->theta_s = 7.5e-3;
  p->hardening = 10.0;
}

const char* agimp_last_error(const agimp_sim* s) { return s ? s->err.c_str() : "null handle"; }

agimp_status agimp_create(const agimp_params* p, int32_t device, agimp_sim** out) {
  if (!p || !out) return AGIMP_INVALID_ARG;
  *out = nullptr;
  if ((p->dim != 2 && p->dim != 3) || p->level < 1 || p->level > MAXL || p->coarsest_size < 4 ||
      (p->coarsest_size & (p->coarsest_size - 1)) || p->n_particles < 0 || p->n_particles > (int64_t)1 << 30 ||
      p->n_colliders < 0 || p->n_colliders > 4 || !(p->radius > 0.0 && p->radius <= 0.5) ||
      (p->coarsest_size << (p->level - 1)) > (1 << 13) || p->plasticity < 0 || p->plasticity > 1 ||
      p->invalid_nodes < 0 || p->invalid_nodes > 1)
    return AGIMP_INVALID_ARG;
  agimp_sim* s = new agimp_sim();
  s->p = *p;
  s->device = device;
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) {
    delete s;
    return AGIMP_CUDA_ERROR;
  }
  Ctx& c = s->c;
  std::memset(&c, 0, sizeof(c));
  const int D = p->dim;
  c.dim = D;
  c.L = p->level;
  c.coarsest = p->coarsest_size;
  c.sz = p->coarsest_size << (p->level - 1);
  c.N = (int)p->n_particles;
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  c.sms = sms;
  prepare_transfer_kernels();
  c.gap = p->boundary_gap;
  c.bmode = p->boundary_mode;
  c.plast = p->plasticity;
  c.inv_norm = p->invalid_nodes;
  c.radius = (float)p->radius;
  const double mu = p->E / (2.0 * (1.0 + p->nu)), la = p->E * p->nu / ((1.0 + p->nu) * (1.0 - 2.0 * p->nu));
  c.mu = (float)mu;
  c.la = (float)la;
  c.theta_c = (float)p->theta_c;
  c.theta_s = (float)p->theta_s;
  c.xi = (float)p->hardening;
  for (int d = 0; d < 3; ++d) c.grav[d] = (float)p->gravity[d];
  c.ncol = p->n_colliders;
  for (int k = 0; k < 4; ++k)
    for (int j = 0; j < 6; ++j) c.col[k][j] = p->colliders[k][j];
  const int per = 1 << (2 * D);
  long long tot_blocks = 0;
#define AL(ptr, n)                                   \
  do {                                               \
    if (dalloc(s, &(ptr), (size_t)(n)) != cudaSuccess) { \
      agimp_destroy(s);                              \
      return AGIMP_OUT_OF_MEMORY;                    \
    }                                                \
  } while (0)
  for (int l = 0; l < c.L; ++l) {
    LevelDev& V = c.lev[l];
    V.size = c.coarsest << l;
    V.nb = V.size / 4 + 3;
    V.nblocks = 1;
    for (int d = 0; d < D; ++d) V.nblocks *= V.nb;
    if (V.nblocks * per > 0x7fffffffLL) {  // element indices are 32-bit in the kernels
      s->err = "lattice too large: a level holds more than 2^31 stored elements";
      agimp_destroy(s);
      return AGIMP_CAPACITY;
    }
    tot_blocks += V.nblocks;
    AL(V.cell, V.nblocks * per);
    AL(V.node, V.nblocks * per);
    AL(V.bmap, V.nblocks);
    AL(V.blist, V.nblocks);
    cudaMemset(V.cell, 0, V.nblocks * per * sizeof(uint32_t));
    cudaMemset(V.node, 0, V.nblocks * per * sizeof(float4));
    cudaMemset(V.bmap, 0xff, V.nblocks * sizeof(int32_t));
  }
  const LevelDev& Vf = c.lev[c.L - 1];
  AL(c.nmask, Vf.nblocks * per);
  {
    long long cells = 1;
    for (int d = 0; d < D; ++d) cells *= c.sz;
    AL(c.occ, cells);
    AL(c.occ2, cells);
  }
  cudaMemset(c.nmask, 0, Vf.nblocks * per * sizeof(uint32_t));
  for (int l = 0; l < c.L; ++l) {
    LevelDev& V = c.lev[l];
    if (l == c.L - 1) {
      V.nm = c.nmask;
    } else if (D == 3) {  // 2D transfers read the node mask itself
      AL(V.nm, V.nblocks * per);
      cudaMemset(V.nm, 0, V.nblocks * per * sizeof(uint32_t));
    }
    if (l < c.L - 1) {
      AL(V.dflag, V.nblocks);
      cudaMemset(V.dflag, 0, V.nblocks * sizeof(uint32_t));
    }
  }
  AL(c.ctr, CTR_COUNT);
  cudaMemset(c.ctr, 0, CTR_COUNT * sizeof(int32_t));
  c.sur_ctr = c.ctr + CTR_SUR;  // stepping alone, the surrogate slots count here
  AL(c.touch_flag, Vf.nblocks);
  AL(c.touch_list, Vf.nblocks);
  cudaMemset(c.touch_flag, 0, Vf.nblocks * sizeof(uint32_t));
  AL(c.bin_count, tot_blocks + 1);  // + the bin of particles without a level
  cudaMemset(c.bin_count, 0, (tot_blocks + 1) * sizeof(int32_t));
  AL(c.cell_count, (tot_blocks + 1) * per);
  AL(c.cell_off, (tot_blocks + 1) * per);
  AL(c.bin_start, tot_blocks + 1);
  AL(c.full_bins, tot_blocks + 1);
  cudaMemset(c.cell_count, 0, (tot_blocks + 1) * per * sizeof(int32_t));
  const long long N = c.N;
  AL(c.chunks, N / MIN_CHUNK + tot_blocks + 2);  // enough for any work-item size
  c.chunk = CHUNK;
  AL(c.bin_of, N + 1);
  AL(c.rank_of, N + 1);
  AL(c.perm, N + 1);
  AL(c.proj, N + 1);
  for (int k = 0; k < 2; ++k) {
    Particles& P = s->buf[k];
    AL(P.x, D * N + 1);
    AL(P.v, D * N + 1);
    AL(P.F, D * D * N + 1);
    AL(P.C, D * D * N + 1);
    AL(P.m, N + 1);
    AL(P.Jp, N + 1);
    AL(P.g, N + 1);
    AL(P.fl, N + 1);
    AL(P.id, N + 1);
    cudaMemset(P.x, 0, (D * N + 1) * sizeof(float));
    cudaMemset(P.v, 0, (D * N + 1) * sizeof(float));
    cudaMemset(P.F, 0, (D * D * N + 1) * sizeof(float));
    cudaMemset(P.C, 0, (D * D * N + 1) * sizeof(float));
    cudaMemset(P.m, 0, (N + 1) * sizeof(float));
    cudaMemset(P.g, 0, (N + 1) * sizeof(int32_t));
    cudaMemset(P.fl, 0xff, (N + 1) * sizeof(int32_t));
  }
  s->staging_floats = std::max<size_t>((size_t)1 << 20, (size_t)(D * D * N));
  AL(s->staging, s->staging_floats);
  {
    // Jp starts at 1
    std::vector<float> ones(N + 1, 1.0f);
    cudaMemcpy(s->buf[0].Jp, ones.data(), (N + 1) * sizeof(float), cudaMemcpyHostToDevice);
  }
#undef AL
  if (cudaStreamCreateWithFlags(&s->internal, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&s->ev_in, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&s->ev_out, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&s->ev_state, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&s->ev_read[0], cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&s->ev_read[1], cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&s->ev_stage[0], cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&s->ev_stage[1], cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&s->ev_gath[0], cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&s->ev_gath[1], cudaEventDisableTiming) != cudaSuccess ||
      cudaStreamCreateWithFlags(&s->gather, cudaStreamNonBlocking) != cudaSuccess) {
    agimp_destroy(s);
    return AGIMP_CUDA_ERROR;
  }
  // storage slot i starts with caller particle i (on the simulator's own
  // stream; the synchronisation below orders it before any use)
  if (N) k_iota<<<gs_blocks(N), 256, 0, s->internal>>>(s->buf[0].id, N);
  s->self = new agimp_batch();
  s->self->sims.push_back(s);
  s->self->single = true;
  if (batch_init(s->self) != AGIMP_OK) {
    agimp_destroy(s);
    return AGIMP_CUDA_ERROR;
  }
  e = cudaDeviceSynchronize();
  if (e != cudaSuccess) {
    agimp_destroy(s);
    return AGIMP_CUDA_ERROR;
  }
  *out = s;
  return AGIMP_OK;
}

agimp_status agimp_destroy(agimp_sim* s) {
  if (!s) return AGIMP_INVALID_ARG;
  cudaSetDevice(s->device);
  cudaDeviceSynchronize();
  if (s->self) {
    batch_free(s->self);
    delete s->self;
    s->self = nullptr;
  }
  for (void* p : s->allocs) cudaFree(p);
  if (s->rimg) cudaFree(s->rimg);
  if (s->astage) cudaFree(s->astage);
  for (cudaEvent_t e : {s->ev_state, s->ev_read[0], s->ev_read[1], s->ev_stage[0], s->ev_stage[1], s->ev_gath[0],
                        s->ev_gath[1]})
    if (e) cudaEventDestroy(e);
  if (s->gather) cudaStreamDestroy(s->gather);
  if (s->rwin) cudaFree(s->rwin);
  if (s->rkey) cudaFree(s->rkey);
  if (s->rdir) cudaFree(s->rdir);
  if (s->rslot) cudaFree(s->rslot);
  if (s->map_dev) cudaFree(s->map_dev);
  if (s->c.touch_occ) cudaFree(s->c.touch_occ);
  if (s->internal) cudaStreamDestroy(s->internal);
  if (s->ev_in) cudaEventDestroy(s->ev_in);
  if (s->ev_out) cudaEventDestroy(s->ev_out);
  delete s;
  return AGIMP_OK;
}

static agimp_status upload_soa(agimp_sim* s, const float* src, float* dst, int comps, int memory, cudaStream_t st) {
  const long long N = s->c.N;
  if (N == 0) return AGIMP_OK;
  const float* aos = src;
  if (memory == AGIMP_MEM_HOST) {
    CK(cudaMemcpyAsync(s->staging, src, N * comps * sizeof(float), cudaMemcpyHostToDevice, st));
    aos = s->staging;
  }
  k_aos_to_soa<<<gs_blocks(N * comps), 256, 0, st>>>(aos, s->buf[s->par].id, dst, N, comps);
  CK(cudaGetLastError());
  return AGIMP_OK;
}

static agimp_status download_soa(agimp_sim* s, const float* src, float* dst, int comps, int memory, cudaStream_t st) {
  const long long N = s->c.N;
  if (N == 0) return AGIMP_OK;
  float* aos = (memory == AGIMP_MEM_HOST) ? s->staging : dst;
  k_soa_to_aos<<<gs_blocks(N * comps), 256, 0, st>>>(src, s->buf[s->par].id, aos, N, comps);
  CK(cudaGetLastError());
  if (memory == AGIMP_MEM_HOST) {
    CK(cudaMemcpyAsync(dst, s->staging, N * comps * sizeof(float), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
  }
  return AGIMP_OK;
}

static agimp_status copy_i32(agimp_sim* s, const int32_t* src, int32_t* dst, int to_dev, int memory, cudaStream_t st) {
  const long long N = s->c.N;
  if (N == 0) return AGIMP_OK;
  const int32_t* id = s->buf[s->par].id;
  int32_t* tmp = (int32_t*)s->staging;
  if (to_dev) {
    const int32_t* from = src;
    if (memory == AGIMP_MEM_HOST) {
      CK(cudaMemcpyAsync(tmp, src, N * sizeof(int32_t), cudaMemcpyHostToDevice, st));
      from = tmp;
    }
    k_i32_in<<<gs_blocks(N), 256, 0, st>>>(from, id, dst, N);
    CK(cudaGetLastError());
  } else {
    int32_t* to = memory == AGIMP_MEM_HOST ? tmp : dst;
    k_i32_out<<<gs_blocks(N), 256, 0, st>>>(src, id, to, N);
    CK(cudaGetLastError());
    if (memory == AGIMP_MEM_HOST) {
      CK(cudaMemcpyAsync(dst, tmp, N * sizeof(int32_t), cudaMemcpyDeviceToHost, st));
      CK(cudaStreamSynchronize(st));
    }
  }
  return AGIMP_OK;
}

agimp_status agimp_set_particles(agimp_sim* s, const float* x, const float* v, const float* F, const float* C,
                                 const float* m, const int32_t* g, const float* Jp, int32_t memory, void* stream) {
  if (!s || (memory != AGIMP_MEM_DEVICE && memory != AGIMP_MEM_HOST)) return fail(s, AGIMP_INVALID_ARG, "bad args");
  CK(cudaSetDevice(s->device));
  StreamUse su(s, stream);
  wait_readback(s, s->par, su.use);  // the upload overwrites the state being read
  s->bins_valid = false;
  const int D = s->c.dim;
  const Particles& P = s->buf[s->par];
  agimp_status r;
  if (x && (r = upload_soa(s, x, P.x, D, memory, su.use))) return r;
  if (v && (r = upload_soa(s, v, P.v, D, memory, su.use))) return r;
  if (F && (r = upload_soa(s, F, P.F, D * D, memory, su.use))) return r;
  if (C && (r = upload_soa(s, C, P.C, D * D, memory, su.use))) return r;
  if (m && (r = upload_soa(s, m, P.m, 1, memory, su.use))) return r;
  if (Jp && (r = upload_soa(s, Jp, P.Jp, 1, memory, su.use))) return r;
  if (g && (r = copy_i32(s, g, P.g, 1, memory, su.use))) return r;
  CK(cudaEventRecord(s->ev_state, su.use));  // later asynchronous readbacks follow the upload
  s->state_marked = true;
  if (memory == AGIMP_MEM_HOST) CK(cudaStreamSynchronize(su.use));  // host buffers may be reused on return
  return AGIMP_OK;
}

agimp_status agimp_get_particles(agimp_sim* s, float* x, float* v, float* F, float* C, float* m, int32_t* g,
                                 int32_t* fl, float* Jp, int32_t memory, void* stream) {
  if (!s || (memory != AGIMP_MEM_DEVICE && memory != AGIMP_MEM_HOST)) return fail(s, AGIMP_INVALID_ARG, "bad args");
  CK(cudaSetDevice(s->device));
  StreamUse su(s, stream);
  const int D = s->c.dim;
  const Particles& P = s->buf[s->par];
  agimp_status r;
  if (x && (r = download_soa(s, P.x, x, D, memory, su.use))) return r;
  if (v && (r = download_soa(s, P.v, v, D, memory, su.use))) return r;
  if (F && (r = download_soa(s, P.F, F, D * D, memory, su.use))) return r;
  if (C && (r = download_soa(s, P.C, C, D * D, memory, su.use))) return r;
  if (m && (r = download_soa(s, P.m, m, 1, memory, su.use))) return r;
  if (Jp && (r = download_soa(s, P.Jp, Jp, 1, memory, su.use))) return r;
  if (g && (r = copy_i32(s, P.g, g, 0, memory, su.use))) return r;
  if (fl && (r = copy_i32(s, P.fl, fl, 0, memory, su.use))) return r;
  return AGIMP_OK;
}

agimp_status agimp_get_bins(agimp_sim* s, uint64_t* keys, int32_t memory, void* stream) {
  if (!s || !keys || (memory != AGIMP_MEM_DEVICE && memory != AGIMP_MEM_HOST))
    return fail(s, AGIMP_INVALID_ARG, "bad args");
  if (!s->bins_valid) return fail(s, AGIMP_NOT_READY, "no substep has binned the current state");
  CK(cudaSetDevice(s->device));
  StreamUse su(s, stream);
  const long long N = s->c.N;
  if (N == 0) return AGIMP_OK;
  Ctx& c = cur(s);
  unsigned long long* dst = (unsigned long long*)keys;
  unsigned long long* tmp = nullptr;
  if (memory == AGIMP_MEM_HOST) {
    CK(cudaMallocAsync((void**)&tmp, N * sizeof(unsigned long long), su.use));
    dst = tmp;
  }
  if (c.dim == 2)
    k_get_bins<2><<<gs_blocks(N), 256, 0, su.use>>>(c, c.P.id, dst);
  else
    k_get_bins<3><<<gs_blocks(N), 256, 0, su.use>>>(c, c.P.id, dst);
  CK(cudaGetLastError());
  if (memory == AGIMP_MEM_HOST) {
    CK(cudaMemcpyAsync(keys, tmp, N * sizeof(unsigned long long), cudaMemcpyDeviceToHost, su.use));
    CK(cudaFreeAsync(tmp, su.use));
    CK(cudaStreamSynchronize(su.use));
  }
  return AGIMP_OK;
}

agimp_status agimp_get_particles_async(agimp_sim* s, float* x, float* v, float* F, float* C, float* m, int32_t* g,
                                       int32_t* fl, float* Jp, void* stream) {
  if (!s) return AGIMP_INVALID_ARG;
  CK(cudaSetDevice(s->device));
  StreamUse su(s, stream);
  const long long N = s->c.N;
  const int D = s->c.dim;
  const int k = s->par;
  const Particles& P = s->buf[k];
  if (!s->async_used) {
    // from now on every substep marks when the state is ready; if nothing
    // marked the last write yet (a scene stepped only in a batch of several),
    // the work issued so far on the caller's stream is the state
    s->async_used = true;
    if (!s->state_marked) CK(cudaEventRecord(s->ev_state, su.use));
    s->state_marked = true;
  }
  // Two staging slots: the fields are first gathered into caller order in
  // this call's slot (a short kernel on the gather stream, behind the state
  // and the slot's previous host copy), which frees the particle state for
  // the substep that overwrites it; the host copies out of the slot run on
  // the caller's stream and overlap the following substeps.  A slot is
  // reused two calls later, after its copies.
  cudaStream_t gs = s->gather;
  CK(cudaStreamWaitEvent(gs, s->ev_state, 0));  // the state is written
  const int slot = s->stage_next;
  s->stage_next ^= 1;
  if (s->stage_busy[slot]) CK(cudaStreamWaitEvent(gs, s->ev_stage[slot], 0));
  const int comps = (x ? D : 0) + (v ? D : 0) + (F ? D * D : 0) + (C ? D * D : 0) + (m ? 1 : 0) + (Jp ? 1 : 0) +
                    (g ? 1 : 0) + (fl ? 1 : 0);
  const size_t need = (size_t)N * comps + 16;
  if (need > s->astage_floats) {
    CK(cudaDeviceSynchronize());  // both slots idle before they move
    if (s->astage) cudaFree(s->astage);
    s->astage = nullptr;
    s->astage_floats = 0;
    CK(cudaMalloc(&s->astage, 2 * need * sizeof(float)));
    s->astage_floats = need;
  }
  float* const st0 = s->astage + (size_t)slot * s->astage_floats;
  struct Copy {
    void* dst;
    const float* src;
    size_t bytes;
  };
  Copy copies[8];
  int ncopy = 0;
  float* st = st0;
  auto field = [&](const float* src, float* dst, int comps) -> cudaError_t {
    if (!dst || !N) return cudaSuccess;
    k_soa_to_aos<<<gs_blocks(N * comps), 256, 0, gs>>>(src, P.id, st, N, comps);
    copies[ncopy++] = {dst, st, N * comps * sizeof(float)};
    st += N * comps;
    return cudaGetLastError();
  };
  auto ifield = [&](const int32_t* src, int32_t* dst) -> cudaError_t {
    if (!dst || !N) return cudaSuccess;
    k_i32_out<<<gs_blocks(N), 256, 0, gs>>>(src, P.id, (int32_t*)st, N);
    copies[ncopy++] = {dst, st, N * sizeof(int32_t)};
    st += N;
    return cudaGetLastError();
  };
  CK(field(P.x, x, D));
  CK(field(P.v, v, D));
  CK(field(P.F, F, D * D));
  CK(field(P.C, C, D * D));
  CK(field(P.m, m, 1));
  CK(field(P.Jp, Jp, 1));
  CK(ifield(P.g, g));
  CK(ifield(P.fl, fl));
  // the state has been read: a substep may overwrite it from here on
  CK(cudaEventRecord(s->ev_read[k], gs));
  s->read_pending[k] = true;
  s->last_read = k;
  CK(cudaEventRecord(s->ev_gath[slot], gs));
  CK(cudaStreamWaitEvent(su.use, s->ev_gath[slot], 0));
  for (int i = 0; i < ncopy; ++i)
    CK(cudaMemcpyAsync(copies[i].dst, copies[i].src, copies[i].bytes, cudaMemcpyDeviceToHost, su.use));
  CK(cudaEventRecord(s->ev_stage[slot], su.use));
  s->stage_busy[slot] = true;
  return AGIMP_OK;
}

agimp_status agimp_set_level_map(agimp_sim* s, const int8_t* table, int32_t halo, int32_t memory, void* stream) {
  if (!s || !table) return fail(s, AGIMP_INVALID_ARG, "null table");
  const int need = std::max(2, 1 << (s->c.L - 1));
  if (halo < need) return fail(s, AGIMP_INVALID_ARG, "level map halo must be >= max(2, 2^(level-1))");
  CK(cudaSetDevice(s->device));
  const int n = s->c.sz + 2 * halo;
  size_t bytes = 1;
  for (int d = 0; d < s->c.dim; ++d) bytes *= (size_t)n;
  std::vector<int8_t> host(bytes);
  if (memory == AGIMP_MEM_HOST)
    std::memcpy(host.data(), table, bytes);
  else
    CK(cudaMemcpy(host.data(), table, bytes, cudaMemcpyDeviceToHost));
  for (size_t i = 0; i < bytes; ++i) {
    const int e = host[i];
    if (e < 0 || (e & 15) >= s->c.L || (e & ~(15 | 64)))
      return fail(s, AGIMP_INVALID_ARG, "level map entry out of range at " + std::to_string(i));
  }
  int8_t* table_dev = nullptr;
  CK(cudaMalloc(&table_dev, bytes));
  const cudaError_t e = cudaMemcpy(table_dev, host.data(), bytes, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    cudaFree(table_dev);
    return cuda_fail(s, e, "level map upload");
  }
  (void)stream;
  return install_level_map(s, table_dev, halo, n);
}

agimp_status agimp_get_level_map(agimp_sim* s, int8_t* table, int32_t* halo, int32_t memory, void* stream) {
  if (!s || (memory != AGIMP_MEM_DEVICE && memory != AGIMP_MEM_HOST)) return fail(s, AGIMP_INVALID_ARG, "bad args");
  if (!s->c.is_static || !s->map_dev) return fail(s, AGIMP_INVALID_ARG, "no level map selected");
  if (halo) *halo = s->c.map_h;
  if (!table) return AGIMP_OK;
  CK(cudaSetDevice(s->device));
  StreamUse su(s, stream);
  size_t bytes = 1;
  for (int d = 0; d < s->c.dim; ++d) bytes *= (size_t)s->c.map_n;
  CK(cudaMemcpyAsync(table, s->map_dev, bytes, memory == AGIMP_MEM_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice,
                     su.use));
  if (memory == AGIMP_MEM_HOST) CK(cudaStreamSynchronize(su.use));
  return AGIMP_OK;
}

agimp_status agimp_clear_level_map(agimp_sim* s) {
  if (!s) return AGIMP_INVALID_ARG;
  s->c.is_static = 0;
  drop_graphs(s);
  return AGIMP_OK;
}

agimp_status agimp_set_graphs(agimp_sim* s, int32_t enable) {
  if (!s) return AGIMP_INVALID_ARG;
  s->self->graphs = enable != 0;
  if (!s->self->graphs) drop_graphs(s);
  return AGIMP_OK;
}

agimp_status agimp_substep(agimp_sim* s, float dt, int32_t n_steps, void* stream) {
  if (!s || n_steps < 0 || !std::isfinite(dt)) return fail(s, AGIMP_INVALID_ARG, "bad substep args");
  CK(cudaSetDevice(s->device));
  StreamUse su(s, stream);
  return from_batch(s, batch_step(s->self, dt, n_steps, su.use, nullptr));
}

agimp_status agimp_refine_levels(agimp_sim* s, int32_t band, void* stream) {
  if (!s || band < 1 || band > 32) return fail(s, AGIMP_INVALID_ARG, "band must be in [1, 32]");
  // depths are kept in bytes: the deepest threshold, band (2^(L-1) - 1), must stay below 250
  if ((long long)band * ((1ll << (s->c.L - 1)) - 1) >= 250)
    return fail(s, AGIMP_INVALID_ARG, "band * (2^(levels-1) - 1) must be below 250");
  CK(cudaSetDevice(s->device));
  StreamUse su(s, stream);
  wait_readback(s, s->par, su.use);  // g_p of the state being read is rewritten
  launch_refine(cur(s), band, su.use);
  CK(cudaGetLastError());
  CK(cudaEventRecord(s->ev_state, su.use));  // later asynchronous readbacks follow it
  s->state_marked = true;
  return AGIMP_OK;
}

agimp_status agimp_get_grid(agimp_sim* s, int32_t level, int32_t lo, int32_t n, float* m, float* v, int32_t* cell,
                            int32_t memory, void* stream) {
  if (!s || level < 0 || level >= s->c.L || n <= 0) return fail(s, AGIMP_INVALID_ARG, "bad grid readback args");
  CK(cudaSetDevice(s->device));
  StreamUse su(s, stream);
  const int D = s->c.dim;
  long long total = 1;
  for (int d = 0; d < D; ++d) total *= n;
  if (memory == AGIMP_MEM_DEVICE) {
    if (D == 2)
      k_get_grid<2><<<gs_blocks(total), 256, 0, su.use>>>(s->c, level, lo, n, 0, total, m, v, cell);
    else
      k_get_grid<3><<<gs_blocks(total), 256, 0, su.use>>>(s->c, level, lo, n, 0, total, m, v, cell);
    CK(cudaGetLastError());
    return AGIMP_OK;
  }
  // host: slabs through the staging buffer (m | v | cell)
  const long long slab = (long long)(s->staging_floats / (2 + D));
  for (long long off = 0; off < total; off += slab) {
    const long long cnt = std::min(slab, total - off);
    float* sm = s->staging;
    float* sv = s->staging + cnt;
    int32_t* sc = (int32_t*)(s->staging + cnt * (1 + D));
    if (D == 2)
      k_get_grid<2><<<gs_blocks(cnt), 256, 0, su.use>>>(s->c, level, lo, n, off, cnt, m ? sm : nullptr,
                                                        v ? sv : nullptr, cell ? sc : nullptr);
    else
      k_get_grid<3><<<gs_blocks(cnt), 256, 0, su.use>>>(s->c, level, lo, n, off, cnt, m ? sm : nullptr,
                                                        v ? sv : nullptr, cell ? sc : nullptr);
    CK(cudaGetLastError());
    if (m) CK(cudaMemcpyAsync(m + off, sm, cnt * sizeof(float), cudaMemcpyDeviceToHost, su.use));
    if (v) CK(cudaMemcpyAsync(v + off * D, sv, cnt * D * sizeof(float), cudaMemcpyDeviceToHost, su.use));
    if (cell) CK(cudaMemcpyAsync(cell + off, sc, cnt * sizeof(int32_t), cudaMemcpyDeviceToHost, su.use));
    CK(cudaStreamSynchronize(su.use));
  }
  return AGIMP_OK;
}

agimp_status agimp_get_node_mask(agimp_sim* s, int32_t* out, int32_t memory, void* stream) {
  if (!s || !out) return fail(s, AGIMP_INVALID_ARG, "bad node mask readback args");
  CK(cudaSetDevice(s->device));
  StreamUse su(s, stream);
  const int D = s->c.dim;
  long long total = 1;
  for (int d = 0; d < D; ++d) total *= (s->c.sz + 1);
  const long long slab = memory == AGIMP_MEM_HOST ? (long long)s->staging_floats : total;
  for (long long off = 0; off < total; off += slab) {
    const long long cnt = std::min(slab, total - off);
    int32_t* dst = memory == AGIMP_MEM_HOST ? (int32_t*)s->staging : out + off;
    if (D == 2)
      k_get_nmask<2><<<gs_blocks(cnt), 256, 0, su.use>>>(s->c, off, cnt, dst);
    else
      k_get_nmask<3><<<gs_blocks(cnt), 256, 0, su.use>>>(s->c, off, cnt, dst);
    CK(cudaGetLastError());
    if (memory == AGIMP_MEM_HOST) {
      CK(cudaMemcpyAsync(out + off, dst, cnt * sizeof(int32_t), cudaMemcpyDeviceToHost, su.use));
      CK(cudaStreamSynchronize(su.use));
    }
  }
  return AGIMP_OK;
}

agimp_status agimp_errors(agimp_sim* s, uint32_t* bits, int32_t clear) {
  if (!s || !bits) return AGIMP_INVALID_ARG;
  CK(cudaSetDevice(s->device));
  CK(cudaDeviceSynchronize());
  int32_t v = 0;
  CK(cudaMemcpy(&v, s->c.ctr + CTR_ERR, sizeof(int32_t), cudaMemcpyDeviceToHost));
  *bits = (uint32_t)v;
  if (clear) CK(cudaMemset(s->c.ctr + CTR_ERR, 0, sizeof(int32_t)));
  return AGIMP_OK;
}

agimp_status agimp_get_stats(agimp_sim* s, agimp_stats* out) {
  if (!s || !out) return AGIMP_INVALID_ARG;
  CK(cudaSetDevice(s->device));
  CK(cudaDeviceSynchronize());
  int32_t h[CTR_COUNT];
  CK(cudaMemcpy(h, s->c.ctr, sizeof(h), cudaMemcpyDeviceToHost));
  std::memset(out, 0, sizeof(*out));
  for (int l = 0; l < MAXL; ++l) out->active_blocks[l] = l < s->c.L ? h[CTR_LEVEL + l] : 0;
  out->n_binned = h[CTR_BINCUR] - h[CTR_UNBIN];
  out->n_surrogate = h[CTR_SUR];
  out->n_fallback = h[CTR_SURFB];
  out->n_chunks = h[CTR_CHUNKS];
  out->substeps = s->substeps;
  return AGIMP_OK;
}

int32_t agimp_kernels_per_substep(const agimp_sim* s) {
  if (!s) return 0;
  return batch_kernels(s->self);
}

agimp_status agimp_set_surrogate(agimp_sim* s, const agimp_mlp* m, const float* xmax, float tol) {
  if (!s) return AGIMP_INVALID_ARG;
  CK(cudaSetDevice(s->device));
  CK(cudaDeviceSynchronize());
  drop_graphs(s);
  if (!m) {
    s->c.sur = 0;
    return AGIMP_OK;
  }
  if (s->c.plast != 1) return fail(s, AGIMP_INVALID_ARG, "the surrogate replaces the snow return map: plasticity must be snow");
  if (!xmax || !(tol > 0.f)) return fail(s, AGIMP_INVALID_ARG, "surrogate needs xmax[7] and tol > 0");
  const long long N = s->c.N;
  if (!s->c.sur_X) {
    CK(dalloc(s, &s->c.sur_X, (size_t)N * 7 + 8));
    CK(dalloc(s, &s->c.sur_Y, (size_t)N * 4 + 8));
    CK(dalloc(s, &s->c.sur_meta, (size_t)N * SUR_META + 8));
  }
  mlp_buffers(m, &s->c.mlp_packed, &s->c.mlp_P);
  for (int k = 0; k < 8; ++k) s->c.sur_xmax[k] = k < 7 ? xmax[k] : 0.f;
  s->c.sur_tol = tol;
  s->c.sur_ctr = s->c.ctr + CTR_SUR;
  s->c.sur = 1;
  return AGIMP_OK;
}

agimp_status agimp_set_recorder(agimp_sim* s, float* X, float* T, int64_t capacity, int32_t stride) {
  if (!s || (X && (!T || capacity <= 0 || stride < 1))) return fail(s, AGIMP_INVALID_ARG, "bad recorder args");
  CK(cudaSetDevice(s->device));
  CK(cudaDeviceSynchronize());
  drop_graphs(s);
  s->c.rec_X = X;
  s->c.rec_T = T;
  s->c.rec_cap = X ? capacity : 0;
  s->c.rec_stride = X ? stride : 1;
  CK(cudaMemset(s->c.ctr + CTR_REC, 0, sizeof(int32_t)));
  return AGIMP_OK;
}

agimp_status agimp_recorded(agimp_sim* s, int64_t* count, int32_t reset) {
  if (!s || !count) return AGIMP_INVALID_ARG;
  CK(cudaSetDevice(s->device));
  CK(cudaDeviceSynchronize());
  int32_t v = 0;
  CK(cudaMemcpy(&v, s->c.ctr + CTR_REC, sizeof(v), cudaMemcpyDeviceToHost));
  *count = v;
  if (reset) CK(cudaMemset(s->c.ctr + CTR_REC, 0, sizeof(int32_t)));
  return AGIMP_OK;
}

agimp_status agimp_profile_substep(agimp_sim* s, float dt, float* ms, int32_t n, void* stream) {
  if (!s || !ms || n < PHASES || !std::isfinite(dt)) return fail(s, AGIMP_INVALID_ARG, "bad profile args");
  CK(cudaSetDevice(s->device));
  StreamUse su(s, stream);
  cudaEvent_t ev[PHASES + 1];
  for (int i = 0; i <= PHASES; ++i) CK(cudaEventCreate(&ev[i]));
  const agimp_status st = batch_step(s->self, dt, 1, su.use, ev);
  cudaError_t e = st == AGIMP_OK ? cudaEventSynchronize(ev[PHASES]) : cudaSuccess;
  for (int i = 0; i < PHASES && e == cudaSuccess && st == AGIMP_OK; ++i)
    e = cudaEventElapsedTime(&ms[i], ev[i], ev[i + 1]);
  for (int i = 0; i <= PHASES; ++i) cudaEventDestroy(ev[i]);
  if (st != AGIMP_OK) return from_batch(s, st);
  if (e != cudaSuccess) return cuda_fail(s, e, "profile substep");
  return AGIMP_OK;
}

// ---------------------------------------------------------------------------
// headless drawing (gui.py)
agimp_status agimp_render_mask(agimp_sim* s, int32_t res, int32_t show_ghost, int32_t show_node, float* img,
                               int32_t memory, void* stream) {
  if (!s) return AGIMP_INVALID_ARG;
  CK(cudaSetDevice(s->device));
  StreamUse su(s, stream);
  return render_mask(s, res, show_ghost, show_node, img, memory, su.use);
}

agimp_status agimp_render_particles(agimp_sim* s, int32_t res, float radius, const float* colors,
                                    int32_t colors_memory, float* img, int32_t memory, void* stream) {
  if (!s) return AGIMP_INVALID_ARG;
  CK(cudaSetDevice(s->device));
  StreamUse su(s, stream);
  return render_particles(s, res, radius, colors, colors_memory, img, memory, su.use);
}

agimp_status agimp_render_scene3d(agimp_sim* s, int32_t res, const agimp_view3d* view, float* img, int32_t memory,
                                  void* stream) {
  if (!s) return AGIMP_INVALID_ARG;
  CK(cudaSetDevice(s->device));
  StreamUse su(s, stream);
  return render_scene3d(s, res, view, img, memory, su.use);
}

agimp_status agimp_cell_lines(agimp_sim* s, float* vertices, int64_t capacity, int64_t* count, int32_t memory,
                              void* stream) {
  if (!s) return AGIMP_INVALID_ARG;
  CK(cudaSetDevice(s->device));
  StreamUse su(s, stream);
  long long n = 0;
  const agimp_status st = cell_lines(s, vertices, capacity, &n, memory, su.use);
  if (count) *count = n;
  return st;
}

// ---------------------------------------------------------------------------
// launch tuning of one simulator
agimp_status agimp_set_tuning(agimp_sim* s, const agimp_tuning* t) {
  if (!s) return AGIMP_INVALID_ARG;
  return from_batch(s, batch_set_tuning(s->self, t));
}

agimp_status agimp_get_tuning(const agimp_sim* s, agimp_tuning* t) {
  if (!s || !t) return AGIMP_INVALID_ARG;
  *t = s->self->tune;
  return AGIMP_OK;
}

agimp_status agimp_autotune(agimp_sim* s, float dt, int32_t trials, agimp_tuning* best, void* stream) {
  if (!s || !std::isfinite(dt)) return fail(s, AGIMP_INVALID_ARG, "bad autotune args");
  CK(cudaSetDevice(s->device));
  StreamUse su(s, stream);
  return from_batch(s, batch_autotune(s->self, dt, trials, best, su.use));
}

// ---------------------------------------------------------------------------
// batches of simulators
static agimp_status bfail(agimp_batch* b, agimp_status st, const char* msg) {
  if (b) b->err = msg;
  return st;
}

// library work of a batch on the caller's stream, or on the batch's internal
// stream ordered after / before the legacy default stream
struct BatchStream {
  agimp_batch* b;
  cudaStream_t user, use;
  BatchStream(agimp_batch* b_, void* stream) : b(b_), user((cudaStream_t)stream) {
    use = user ? user : b->internal;
    if (!user) {
      cudaEventRecord(b->ev_in, 0);
      cudaStreamWaitEvent(b->internal, b->ev_in, 0);
    }
  }
  ~BatchStream() {
    if (!user) {
      cudaEventRecord(b->ev_out, b->internal);
      cudaStreamWaitEvent(0, b->ev_out, 0);
    }
  }
};

agimp_status agimp_batch_create(agimp_sim* const* sims, int32_t n, agimp_batch** out) {
  if (!sims || !out || n < 1 || n > (1 << 16)) return AGIMP_INVALID_ARG;
  *out = nullptr;
  for (int i = 0; i < n; ++i) {
    if (!sims[i]) return AGIMP_INVALID_ARG;
    if (sims[i]->device != sims[0]->device || sims[i]->c.dim != sims[0]->c.dim) return AGIMP_INVALID_ARG;
    for (int j = 0; j < i; ++j)
      if (sims[j] == sims[i]) return AGIMP_INVALID_ARG;
  }
  if (cudaSetDevice(sims[0]->device) != cudaSuccess) return AGIMP_CUDA_ERROR;
  agimp_batch* b = new agimp_batch();
  b->sims.assign(sims, sims + n);
  b->single = false;
  if (batch_init(b) != AGIMP_OK) {
    batch_free(b);
    delete b;
    return AGIMP_CUDA_ERROR;
  }
  *out = b;
  return AGIMP_OK;
}

agimp_status agimp_batch_destroy(agimp_batch* b) {
  if (!b) return AGIMP_INVALID_ARG;
  cudaSetDevice(b->device);
  cudaDeviceSynchronize();
  batch_free(b);
  delete b;
  return AGIMP_OK;
}

const char* agimp_batch_last_error(const agimp_batch* b) { return b ? b->err.c_str() : "null handle"; }

agimp_status agimp_batch_substep(agimp_batch* b, float dt, int32_t n_steps, void* stream) {
  if (!b || n_steps < 0 || !std::isfinite(dt)) return bfail(b, AGIMP_INVALID_ARG, "bad substep args");
  if (cudaSetDevice(b->device) != cudaSuccess) return bfail(b, AGIMP_CUDA_ERROR, "cudaSetDevice failed");
  BatchStream bs(b, stream);
  return batch_step(b, dt, n_steps, bs.use, nullptr);
}

agimp_status agimp_batch_set_graphs(agimp_batch* b, int32_t enable) {
  if (!b) return AGIMP_INVALID_ARG;
  b->graphs = enable != 0;
  if (!b->graphs) batch_drop_graphs(b);
  return AGIMP_OK;
}

agimp_status agimp_batch_set_tuning(agimp_batch* b, const agimp_tuning* t) {
  if (!b) return AGIMP_INVALID_ARG;
  return batch_set_tuning(b, t);
}

agimp_status agimp_batch_get_tuning(const agimp_batch* b, agimp_tuning* t) {
  if (!b || !t) return AGIMP_INVALID_ARG;
  *t = b->tune;
  return AGIMP_OK;
}

agimp_status agimp_batch_autotune(agimp_batch* b, float dt, int32_t trials, agimp_tuning* best, void* stream) {
  if (!b || !std::isfinite(dt)) return bfail(b, AGIMP_INVALID_ARG, "bad autotune args");
  if (cudaSetDevice(b->device) != cudaSuccess) return bfail(b, AGIMP_CUDA_ERROR, "cudaSetDevice failed");
  BatchStream bs(b, stream);
  return batch_autotune(b, dt, trials, best, bs.use);
}

agimp_status agimp_batch_profile_substep(agimp_batch* b, float dt, float* ms, int32_t n, void* stream) {
  if (!b || !ms || n < PHASES || !std::isfinite(dt)) return bfail(b, AGIMP_INVALID_ARG, "bad profile args");
  if (cudaSetDevice(b->device) != cudaSuccess) return bfail(b, AGIMP_CUDA_ERROR, "cudaSetDevice failed");
  BatchStream bs(b, stream);
  cudaEvent_t ev[PHASES + 1];
  for (int i = 0; i <= PHASES; ++i)
    if (cudaEventCreate(&ev[i]) != cudaSuccess) return bfail(b, AGIMP_CUDA_ERROR, "cudaEventCreate failed");
  const agimp_status st = batch_step(b, dt, 1, bs.use, ev);
  cudaError_t e = st == AGIMP_OK ? cudaEventSynchronize(ev[PHASES]) : cudaSuccess;
  for (int i = 0; i < PHASES && e == cudaSuccess && st == AGIMP_OK; ++i)
    e = cudaEventElapsedTime(&ms[i], ev[i], ev[i + 1]);
  for (int i = 0; i <= PHASES; ++i) cudaEventDestroy(ev[i]);
  if (st != AGIMP_OK) return st;
  if (e != cudaSuccess) return bfail(b, AGIMP_CUDA_ERROR, cudaGetErrorString(e));
  return AGIMP_OK;
}

agimp_status agimp_batch_positions_async(agimp_batch* b, float* x, void* stream) {
  if (!b) return AGIMP_INVALID_ARG;
  BatchStream bs(b, stream);
  return batch_positions_async(b, x, bs.use);
}

agimp_status agimp_batch_set_particles(agimp_batch* b, const float* x, const float* v, const float* F, const float* C,
                                       const float* m, const int32_t* g, const float* Jp, int32_t memory, void* stream) {
  if (!b) return AGIMP_INVALID_ARG;
  BatchStream bs(b, stream);
  return batch_set_particles(b, x, v, F, C, m, g, Jp, memory, bs.use);
}

agimp_status agimp_batch_set_surrogate(agimp_batch* b, const agimp_mlp* m, const float* xmax, float tol) {
  if (!b) return AGIMP_INVALID_ARG;
  if (!m) return batch_set_surrogate(b, nullptr, nullptr, nullptr, 0.f);
  if (!xmax || !(tol > 0.f)) return bfail(b, AGIMP_INVALID_ARG, "surrogate needs xmax[7] and tol > 0");
  bool any = false;
  for (agimp_sim* s : b->sims) any = any || s->c.plast == 1;
  if (!any) return bfail(b, AGIMP_INVALID_ARG, "the surrogate replaces the snow return map: no scene has snow plasticity");
  const void* packed = nullptr;
  const float* P = nullptr;
  mlp_buffers(m, &packed, &P);
  return batch_set_surrogate(b, packed, P, xmax, tol);
}

agimp_status agimp_batch_surrogate_stats(agimp_batch* b, int64_t* handed, int64_t* rejected, uint32_t* errors) {
  if (!b) return AGIMP_INVALID_ARG;
  if (cudaSetDevice(b->device) != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess) return AGIMP_CUDA_ERROR;
  int32_t h[2] = {0, 0};
  if (b->single) {
    agimp_sim* s = b->sims[0];
    if (cudaMemcpy(h, s->c.ctr + CTR_SUR, sizeof(int32_t), cudaMemcpyDeviceToHost) != cudaSuccess)
      return AGIMP_CUDA_ERROR;
  } else if (b->sctr &&
             cudaMemcpy(h, b->sctr, 2 * sizeof(int32_t), cudaMemcpyDeviceToHost) != cudaSuccess) {
    return AGIMP_CUDA_ERROR;
  }
  long long rej = 0;
  for (agimp_sim* s : b->sims) {
    int32_t v = 0;
    if (cudaMemcpy(&v, s->c.ctr + CTR_SURFB, sizeof(int32_t), cudaMemcpyDeviceToHost) != cudaSuccess)
      return AGIMP_CUDA_ERROR;
    rej += v;
  }
  if (handed) *handed = h[0];
  if (rejected) *rejected = rej;
  if (errors) *errors = h[1] ? AGIMP_ERR_WAIT : 0u;
  return AGIMP_OK;
}

int32_t agimp_batch_kernels_per_substep(const agimp_batch* b) {
  return b ? batch_kernels(const_cast<agimp_batch*>(b)) : 0;
}

}  // extern "C"

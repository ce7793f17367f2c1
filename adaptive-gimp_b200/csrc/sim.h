// Host-side state of a simulator (agimp_sim) and of a batch of simulators
// stepped by shared launches (agimp_batch).  Internal to libagimp.so.
#pragma once
#include <string>
#include <vector>

#include "../../include/agimp.h"
#include "common.cuh"

struct agimp_batch;

struct agimp_sim {
  agimp::Ctx c;
  agimp::Particles buf[2];  // particle state ping-pongs between the two buffers
  int par = 0;              // buf[par] holds the current state
  agimp_params p;
  int device = 0;
  std::string err;
  std::vector<void*> allocs;
  cudaStream_t internal = nullptr;
  cudaEvent_t ev_in = nullptr, ev_out = nullptr;
  float* staging = nullptr;
  size_t staging_floats = 0;
  int8_t* map_dev = nullptr;
  long long substeps = 0;
  bool bins_valid = false;  // perm / bin_of hold the binning of the current state's last substep
  agimp_batch* self = nullptr;  // the simulator as a batch of one (its substep path)
  // asynchronous readback: the state is ready after ev_state; a copy of
  // buffer k is in flight until ev_read[k]
  bool async_used = false;
  bool state_marked = false;  // ev_state was recorded after the last write of the state
  cudaEvent_t ev_state = nullptr;
  cudaEvent_t ev_read[2] = {nullptr, nullptr};
  bool read_pending[2] = {false, false};
  int last_read = -1;           // buffer of the last asynchronous readback (its staging is busy until ev_read)
  float* astage = nullptr;      // staging of asynchronous readbacks: two slots of astage_floats
  size_t astage_floats = 0;
  int stage_next = 0;           // slot of the next asynchronous readback
  bool stage_busy[2] = {false, false};
  cudaEvent_t ev_stage[2] = {nullptr, nullptr};  // the host copy out of slot k has been issued up to here
  // the gathers of asynchronous readbacks run on their own stream, so a
  // gather (and with it the release of the state) waits only for the state
  // and for its slot's previous host copy, not for the last readback's copy
  cudaStream_t gather = nullptr;
  cudaEvent_t ev_gath[2] = {nullptr, nullptr};  // slot k's gather is done
  float* rimg = nullptr;        // headless drawing: image scratch for host outputs
  size_t rimg_floats = 0;
  int* rwin = nullptr;          // headless drawing: particle covering each pixel
  size_t rwin_n = 0;
  unsigned long long* rkey = nullptr;  // 3D drawing: nearest sphere hit per pixel (depth, particle)
  float* rdir = nullptr;               // 3D drawing: ray direction per pixel
  int* rslot = nullptr;                // 3D drawing: storage slot of each caller particle index
  size_t rkey_n = 0, rslot_n = 0;
};

// Several simulators (scenes) stepped together: one launch per kernel serves
// all of them.  The kernels read each scene's context from device memory, one
// array per step phase (a scene's particle buffers alternate between steps);
// the host keeps a copy of what the device holds and uploads only entries
// that changed.
struct agimp_batch {
  struct Key {  // launch structure a captured substep holds
    int maxL, any_dynamic, any_plastic, chunk, sur;
    int nct[agimp::NMAP];
    cudaStream_t stream;
  };
  std::vector<agimp_sim*> sims;
  bool single = false;  // a simulator's own batch of one
  int device = 0, dim = 2, sms = 148;
  agimp_tuning tune{agimp::CHUNK, 8, 0.f};
  bool graphs = true;
  // programmatic dependent launches inside a substep (AGIMP_PDL=0 in the
  // environment switches them off, for comparison)
  bool pdl = true;
  agimp::Ctx* dctx[2] = {nullptr, nullptr};
  std::vector<agimp::Ctx> hctx[2];
  std::vector<char> hvalid[2];
  int* dofs = nullptr;  // [NMAP][n + 1]
  std::vector<int> hofs;
  int nct[agimp::NMAP] = {0, 0, 0, 0};
  bool maps_valid = false;
  cudaGraphExec_t gexec[2] = {nullptr, nullptr};
  Key gkey[2];
  long long steps = 0;
  cudaStream_t internal = nullptr;  // used when the caller passes no stream (own batches only)
  cudaStream_t side = nullptr;      // second stream inside a substep
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  cudaEvent_t ev_in = nullptr, ev_out = nullptr;
  std::string err;
  // batch readback of positions (own batches only): the last step's work is
  // done at ev_done; a copy started after `read_step` steps ends at ev_read
  cudaEvent_t ev_done = nullptr, ev_read = nullptr;
  bool read_pending = false;
  long long read_step = 0;
  // two slots: gathered positions (xstage, tot*dim floats each), the
  // per-scene gather sources in pinned host memory (hsrc) and on the device
  // (dsrc); the gathers run on their own stream (see agimp_sim::gather)
  float* xstage = nullptr;
  void* dsrc = nullptr;
  void* hsrc = nullptr;
  long long xstage_floats = 0;
  int xs_next = 0;
  bool xs_busy[2] = {false, false}, hsrc_busy[2] = {false, false};
  cudaEvent_t ev_xs[2] = {nullptr, nullptr};    // slot k's host copy is done
  cudaEvent_t ev_hsrc[2] = {nullptr, nullptr};  // slot k's source table is on the device
  cudaEvent_t ev_gath[2] = {nullptr, nullptr};  // slot k's gather is done
  cudaStream_t gather = nullptr;
  // batch upload (agimp_batch_set_particles): one field of all scenes in the
  // staging at a time, the per-scene destinations of all fields in utab
  float* ustage = nullptr;
  size_t ustage_floats = 0;
  void* utab = nullptr;
  void* utab_h = nullptr;
  // surrogate return map shared by the scenes of a batch of several
  // (agimp_batch_set_surrogate): one set of slot buffers over all scenes'
  // particles and one slot counter, so one MLP launch serves the batch
  int sur = 0;
  const void* mlp_packed = nullptr;
  const float* mlp_P = nullptr;
  float sur_xmax[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  float sur_tol = 0.f;
  float* sX = nullptr;        // [cap][7]
  float* sY = nullptr;        // [cap][4]
  float* smeta = nullptr;     // [cap][SUR_META]
  int32_t* sctr = nullptr;    // [0] slots this substep, [1] error bits of the MLP
  long long scap = 0;
};

namespace agimp {
// The simulator's context with P = its current state, Q = the other buffer.
Ctx& sim_ctx(agimp_sim* s);
// Allocate a batch's device arrays for its simulators (b->sims, b->single set).
agimp_status batch_init(agimp_batch* b);
void batch_free(agimp_batch* b);
void batch_drop_graphs(agimp_batch* b);
// n substeps of every scene on `use`; with ev, one substep with phase events
// and no graph.
agimp_status batch_step(agimp_batch* b, float dt, int n, cudaStream_t use, cudaEvent_t* ev);
int batch_kernels(agimp_batch* b);
agimp_status batch_positions_async(agimp_batch* b, float* x, cudaStream_t use);
agimp_status batch_set_particles(agimp_batch* b, const float* x, const float* v, const float* F, const float* C,
                                 const float* m, const int32_t* g, const float* Jp, int memory, cudaStream_t use);
// make `use` wait for asynchronous readbacks of the buffer the next work writes
void wait_readback(agimp_sim* s, int buf, cudaStream_t use);
agimp_status batch_autotune(agimp_batch* b, float dt, int trials, agimp_tuning* best, cudaStream_t use);
agimp_status batch_set_tuning(agimp_batch* b, const agimp_tuning* t);
agimp_status batch_set_surrogate(agimp_batch* b, const void* packed, const float* P, const float* xmax, float tol);
// headless drawing (render.cu)
agimp_status render_mask(agimp_sim* s, int res, int show_ghost, int show_node, float* img, int memory, cudaStream_t st);
agimp_status render_scene3d(agimp_sim* s, int res, const agimp_view3d* v, float* img, int memory, cudaStream_t st);
agimp_status cell_lines(agimp_sim* s, float* vert, long long cap, long long* count, int memory, cudaStream_t st);
agimp_status render_particles(agimp_sim* s, int res, float radius, const float* colors, int colors_memory, float* img,
                              int memory, cudaStream_t st);
}  // namespace agimp

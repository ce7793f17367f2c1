// Headless drawing of a 2D simulator: the reference GUI's mask view
// (gui.py:12-43, GUI.visualize_mask) and its particle circles (gui.py:69,
// canvas.circles), rendered by CUDA kernels into an RGB f32 image
// img[res][res][3] indexed [i][j] like the reference's bg_img[i, j] (i along x,
// j along y).  There is no window: the image stays in device memory or is
// copied to the caller.
//
// Order of the reference's parallel writes.  visualize_mask's second loop
// paints a 3x3 square around every finest node that is activated, a T
// junction or a ghost node; when the node spacing in pixels (res / finest) is
// below 3 the squares overlap and the Taichi result depends on thread order.
// Here every pixel takes the colour of the last covering node in row-major
// (i, j) order, the result of a serial run.  Particles are drawn in the
// caller's particle order (later particles on top); a pixel is covered when
// its centre lies within radius * res pixels of the particle.
#include <algorithm>
#include <cstring>

#include "sim.h"

namespace agimp {
namespace {

struct RGB {
  float r, g, b;
};

// gui.py:20-29 colours
__device__ __constant__ RGB kActFill = {0.28f, 0.68f, 0.99f};
__device__ __constant__ RGB kActEdge = {0.18f, 0.58f, 0.88f};
__device__ __constant__ RGB kGhoFill = {0.f, 0.f, 1.0f};
__device__ __constant__ RGB kGhoEdge = {0.f, 0.f, 0.77f};
// gui.py:32-43 node markers
__device__ __constant__ RGB kNodeAct = {1.0f, 0.f, 0.f};
__device__ __constant__ RGB kNodeTJ = {0.f, 1.0f, 0.f};
__device__ __constant__ RGB kNodeGho = {0.f, 0.f, 0.35f};

__device__ __forceinline__ void put(float* img, long long pix, RGB c) {
  img[pix * 3 + 0] = c.r;
  img[pix * 3 + 1] = c.g;
  img[pix * 3 + 2] = c.b;
}

// cell_mask[l][I] as the reference reads it (CULLING is internal)
__device__ __forceinline__ uint32_t cell_at(const Ctx& c, int l, int i, int j) {
  const LevelDev& V = c.lev[l];
  const int I[2] = {i, j};
  if (!in_store<2>(V, I)) return 0u;
  return V.cell[elem_of<2>(V, I)] & ~CUL;
}

// gui.py:17-29: per pixel, the levels from coarse to fine overwrite each other
__global__ void k_render_cells(Ctx c, int res, int show_ghost, int show_node, float* img) {
  const long long tot = (long long)res * res;
  const int fscale = res / c.sz;
  for (long long pix = blockIdx.x * (long long)blockDim.x + threadIdx.x; pix < tot;
       pix += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(pix / res), j = (int)(pix % res);
    RGB col = {0.f, 0.f, 0.f};
    for (int l = 0; l < c.L; ++l) {
      const int scale = res / (c.coarsest << l);
      const uint32_t cm = cell_at(c, l, i / scale, j / scale);
      const bool edge = i % scale == 0 || i % scale == scale - 1 || j % scale == 0 || j % scale == scale - 1;
      if (cm == ACT)
        col = edge ? kActEdge : kActFill;
      else if (cm == GHO && show_ghost)
        col = edge ? kGhoEdge : kGhoFill;
    }
    // gui.py:31-43: the last node (row-major) whose 3x3 marker covers the pixel
    if (show_node) {
      bool done = false;
      for (int di = 1; di >= -1 && !done; --di) {
        const int i0 = i + di;
        if (i0 < 0 || i0 >= res || i0 % fscale) continue;
        for (int dj = 1; dj >= -1 && !done; --dj) {
          const int j0 = j + dj;
          if (j0 < 0 || j0 >= res || j0 % fscale) continue;
          const int P[2] = {i0 / fscale, j0 / fscale};
          uint32_t nm = 0u;
          if (P[0] <= c.sz && P[1] <= c.sz) nm = c.nmask[elem_of<2>(c.lev[c.L - 1], P)];
          if (is_activated(nm)) {
            col = kNodeAct;
            done = true;
          } else if (is_tj(nm)) {
            col = kNodeTJ;
            done = true;
          } else if (is_ghost(nm)) {
            col = kNodeGho;
            done = true;
          }
        }
      }
    }
    put(img, pix, col);
  }
}

// particles: the highest caller index covering each pixel wins
__global__ void k_splat(Ctx c, int res, float rpix, int* winner) {
  const long long N = c.N;
  for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < N; s += (long long)gridDim.x * blockDim.x) {
    const float px = __fmul_rn(c.P.x[s], (float)res), py = __fmul_rn(c.P.x[N + s], (float)res);
    const int id = c.P.id[s];
    const int i0 = max(0, (int)floorf(px - rpix - 0.5f)), i1 = min(res - 1, (int)ceilf(px + rpix - 0.5f));
    const int j0 = max(0, (int)floorf(py - rpix - 0.5f)), j1 = min(res - 1, (int)ceilf(py + rpix - 0.5f));
    for (int i = i0; i <= i1; ++i)
      for (int j = j0; j <= j1; ++j) {
        // explicitly rounded f32 operations (no contraction): the same bits
        // as an f32 evaluation of (i+0.5-px)^2 + (j+0.5-py)^2 <= rpix^2
        const float dxp = __fsub_rn((float)i + 0.5f, px), dyp = __fsub_rn((float)j + 0.5f, py);
        if (__fadd_rn(__fmul_rn(dxp, dxp), __fmul_rn(dyp, dyp)) <= __fmul_rn(rpix, rpix))
          atomicMax(&winner[(long long)i * res + j], id + 1);
      }
  }
}

__global__ void k_splat_color(int res, const int* winner, const float* colors, float* img) {
  const long long tot = (long long)res * res;
  for (long long pix = blockIdx.x * (long long)blockDim.x + threadIdx.x; pix < tot;
       pix += (long long)gridDim.x * blockDim.x) {
    const int w = winner[pix];
    if (w > 0) {
      const long long q = (long long)(w - 1) * 3;
      img[pix * 3 + 0] = colors[q + 0];
      img[pix * 3 + 1] = colors[q + 1];
      img[pix * 3 + 2] = colors[q + 2];
    }
  }
}

int blocks_for(long long n) { return (int)std::min<long long>((n + 255) / 256, 148 * 16); }

}  // namespace

// image scratch of a simulator (allocated on first use, grown when needed)
static cudaError_t render_buffers(agimp_sim* s, int res, bool winner) {
  const size_t pix = (size_t)res * res;
  if (pix * 3 > s->rimg_floats) {
    if (s->rimg) cudaFree(s->rimg);
    s->rimg = nullptr;
    s->rimg_floats = 0;
    cudaError_t e = cudaMalloc(&s->rimg, pix * 3 * sizeof(float));
    if (e != cudaSuccess) return e;
    s->rimg_floats = pix * 3;
  }
  if (winner && pix > s->rwin_n) {
    if (s->rwin) cudaFree(s->rwin);
    s->rwin = nullptr;
    s->rwin_n = 0;
    cudaError_t e = cudaMalloc(&s->rwin, pix * sizeof(int));
    if (e != cudaSuccess) return e;
    s->rwin_n = pix;
  }
  return cudaSuccess;
}

agimp_status render_mask(agimp_sim* s, int res, int show_ghost, int show_node, float* img, int memory,
                         cudaStream_t st) {
  const Ctx& c = sim_ctx(s);
  if (c.dim != 2 || res < c.sz || res > 16384 || !img) {
    s->err = "render: 2D only, finest <= res <= 16384, img required";
    return AGIMP_INVALID_ARG;
  }
  cudaError_t e = cudaSuccess;
  float* out = img;
  if (memory == AGIMP_MEM_HOST) {
    e = render_buffers(s, res, false);
    out = s->rimg;
  }
  const long long tot = (long long)res * res;
  if (e == cudaSuccess) {
    k_render_cells<<<blocks_for(tot), 256, 0, st>>>(c, res, show_ghost, show_node, out);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess && memory == AGIMP_MEM_HOST) {
    e = cudaMemcpyAsync(img, out, tot * 3 * sizeof(float), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  }
  if (e != cudaSuccess) {
    s->err = std::string("render mask: ") + cudaGetErrorString(e);
    return AGIMP_CUDA_ERROR;
  }
  return AGIMP_OK;
}

agimp_status render_particles(agimp_sim* s, int res, float radius, const float* colors, int colors_memory, float* img,
                              int memory, cudaStream_t st) {
  const Ctx& c = sim_ctx(s);
  if (c.dim != 2 || res < 1 || res > 16384 || !img || !colors || !(radius >= 0.f && radius < 0.25f)) {
    s->err = "render: 2D only, 1 <= res <= 16384, 0 <= radius < 0.25, img and colors required";
    return AGIMP_INVALID_ARG;
  }
  const long long tot = (long long)res * res;
  cudaError_t e = render_buffers(s, res, true);
  float* work = img;
  const float* cols = colors;
  if (e == cudaSuccess && memory == AGIMP_MEM_HOST) {
    work = s->rimg;
    e = cudaMemcpyAsync(work, img, tot * 3 * sizeof(float), cudaMemcpyHostToDevice, st);
  }
  if (e == cudaSuccess && colors_memory == AGIMP_MEM_HOST && c.N) {
    // colours go into the staging buffer (at least N x 4 floats)
    e = cudaMemcpyAsync(s->staging, colors, (size_t)c.N * 3 * sizeof(float), cudaMemcpyHostToDevice, st);
    cols = s->staging;
  }
  if (e == cudaSuccess) e = cudaMemsetAsync(s->rwin, 0, tot * sizeof(int), st);
  if (e == cudaSuccess && c.N) {
    k_splat<<<blocks_for(c.N), 256, 0, st>>>(c, res, radius * (float)res, s->rwin);  // host f32 product
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) {
    k_splat_color<<<blocks_for(tot), 256, 0, st>>>(res, s->rwin, cols, work);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess && memory == AGIMP_MEM_HOST) {
    e = cudaMemcpyAsync(img, work, tot * 3 * sizeof(float), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  }
  if (e != cudaSuccess) {
    s->err = std::string("render particles: ") + cudaGetErrorString(e);
    return AGIMP_CUDA_ERROR;
  }
  return AGIMP_OK;
}

}  // namespace agimp

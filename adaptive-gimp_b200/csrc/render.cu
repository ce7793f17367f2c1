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

// ---------------------------------------------------------------------------
// 3D: GUI3D.show (gui_3d.py:50-64) without a window.  scene.particles draws
// x_p as spheres of one radius and colour, scene.mesh the unit floor quad,
// lit by point lights.  Here every pixel casts a ray from the camera; the
// nearest sphere (exact ray-sphere intersection) or the floor is shaded with
// Lambert terms of the point lights plus the ambient term (no shadows, no
// specular: the reference's GGUI shaders are not reproduced).  All
// arithmetic is explicitly rounded f32 (no contraction), so a serial f32
// evaluation in the same order gives the same image.  img[row][col][3],
// row 0 at the top of the picture.
__device__ __forceinline__ float dot3(const float* a, const float* b) {
  return __fadd_rn(__fadd_rn(__fmul_rn(a[0], b[0]), __fmul_rn(a[1], b[1])), __fmul_rn(a[2], b[2]));
}

// unit ray direction through the centre of pixel (row, col)
__global__ void k_rays(agimp_view3d v, int res, float* dir) {
  const long long tot = (long long)res * res;
  for (long long pix = blockIdx.x * (long long)blockDim.x + threadIdx.x; pix < tot;
       pix += (long long)gridDim.x * blockDim.x) {
    const int row = (int)(pix / res), col = (int)(pix % res);
    const float fr = (float)res;
    const float sx = __fmul_rn(__fsub_rn(__fdiv_rn(__fmul_rn(2.f, (float)col + 0.5f), fr), 1.f), v.tan_half_fov);
    const float sy = __fmul_rn(__fsub_rn(1.f, __fdiv_rn(__fmul_rn(2.f, (float)row + 0.5f), fr)), v.tan_half_fov);
    float d[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) d[k] = __fadd_rn(__fadd_rn(v.forward[k], __fmul_rn(sx, v.right[k])), __fmul_rn(sy, v.up[k]));
    const float inv = __fdiv_rn(1.f, __fsqrt_rn(dot3(d, d)));
#pragma unroll
    for (int k = 0; k < 3; ++k) dir[pix * 3 + k] = __fmul_rn(d[k], inv);
  }
}

// screen-coordinate range (x / z along one camera axis) of a sphere with
// camera-space centre (a, z) on that axis and radius R (z > R): the slopes of
// the two tangent lines from the eye
__device__ __forceinline__ void tangent_range(float a, float z, float R, float& lo, float& hi) {
  const float den = z * z - R * R;
  const float q = R * sqrtf(fmaxf(a * a + z * z - R * R, 0.f));
  lo = (a * z - q) / den;
  hi = (a * z + q) / den;
}

// every pixel the sphere of particle slot i may cover (its bound widened by
// one pixel) records (depth, caller index) of the nearest front hit
__global__ void k_splat3d(Ctx c, agimp_view3d v, int res, const float* dir, unsigned long long* key) {
  const long long N = c.N;
  const float R = v.radius;
  const float fr = (float)res;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
    float oc[3], w[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      w[k] = __fsub_rn(c.P.x[k * N + i], v.eye[k]);  // centre relative to the eye
      oc[k] = -w[k];
    }
    const float cz = dot3(w, v.forward);
    if (!(cz > R)) continue;  // spheres reaching the eye plane are not drawn
    const float cx = dot3(w, v.right), cy = dot3(w, v.up);
    float x0, x1, y0, y1;
    tangent_range(cx, cz, R, x0, x1);
    tangent_range(cy, cz, R, y0, y1);
    const float half = 0.5f * fr / v.tan_half_fov;
    const int c0 = max(0, (int)floorf(x0 * half + 0.5f * fr - 0.5f) - 1);
    const int c1 = min(res - 1, (int)ceilf(x1 * half + 0.5f * fr - 0.5f) + 1);
    const int r0 = max(0, (int)floorf(0.5f * fr - y1 * half - 0.5f) - 1);
    const int r1 = min(res - 1, (int)ceilf(0.5f * fr - y0 * half - 0.5f) + 1);
    if (c0 > c1 || r0 > r1) continue;
    const float cc = __fsub_rn(dot3(oc, oc), __fmul_rn(R, R));
    const unsigned long long id = (unsigned)c.P.id[i];
    for (int row = r0; row <= r1; ++row)
      for (int col = c0; col <= c1; ++col) {
        const long long pix = (long long)row * res + col;
        const float d[3] = {dir[pix * 3], dir[pix * 3 + 1], dir[pix * 3 + 2]};
        const float b = dot3(oc, d);
        const float disc = __fsub_rn(__fmul_rn(b, b), cc);
        if (!(disc >= 0.f)) continue;
        const float t = __fsub_rn(-b, __fsqrt_rn(disc));
        if (!(t > 0.f)) continue;
        atomicMin(&key[pix], ((unsigned long long)__float_as_uint(t) << 32) | id);
      }
  }
}

__global__ void k_slot_of(Ctx c, int* slot) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < c.N; i += (long long)gridDim.x * blockDim.x)
    slot[c.P.id[i]] = (int)i;
}

__device__ __forceinline__ void shade(const agimp_view3d& v, const float* base, const float* p, const float* n,
                                      float* out) {
#pragma unroll
  for (int k = 0; k < 3; ++k) out[k] = __fmul_rn(base[k], v.ambient[k]);
  for (int l = 0; l < v.n_lights; ++l) {
    float L[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) L[k] = __fsub_rn(v.light_pos[l][k], p[k]);
    const float inv = __fdiv_rn(1.f, __fsqrt_rn(dot3(L, L)));
#pragma unroll
    for (int k = 0; k < 3; ++k) L[k] = __fmul_rn(L[k], inv);
    const float ndl = fmaxf(dot3(n, L), 0.f);
#pragma unroll
    for (int k = 0; k < 3; ++k) out[k] = __fadd_rn(out[k], __fmul_rn(__fmul_rn(base[k], v.light_color[l][k]), ndl));
  }
}

__global__ void k_shade3d(Ctx c, agimp_view3d v, int res, const float* dir, const unsigned long long* key,
                          const int* slot, float* img) {
  const long long tot = (long long)res * res;
  const long long N = c.N;
  for (long long pix = blockIdx.x * (long long)blockDim.x + threadIdx.x; pix < tot;
       pix += (long long)gridDim.x * blockDim.x) {
    const float d[3] = {dir[pix * 3], dir[pix * 3 + 1], dir[pix * 3 + 2]};
    const unsigned long long k = key[pix];
    float ts = INFINITY;
    if (k != ~0ull) ts = __uint_as_float((unsigned)(k >> 32));
    float tf = INFINITY;
    float hf[3];
    if (v.floor && d[1] != 0.f) {
      const float t = __fdiv_rn(-v.eye[1], d[1]);
      if (t > 0.f) {
#pragma unroll
        for (int q = 0; q < 3; ++q) hf[q] = __fadd_rn(v.eye[q], __fmul_rn(t, d[q]));
        if (hf[0] >= 0.f && hf[0] <= 1.f && hf[2] >= 0.f && hf[2] <= 1.f) tf = t;
      }
    }
    float out[3] = {v.background[0], v.background[1], v.background[2]};
    if (tf < ts) {
      hf[1] = 0.f;
      const float n[3] = {0.f, v.eye[1] >= 0.f ? 1.f : -1.f, 0.f};  // two-sided: faces the camera
      shade(v, v.floor_color, hf, n, out);
    } else if (ts < INFINITY) {
      const long long i = slot[(unsigned)(k & 0xffffffffu)];
      float p[3], n[3];
#pragma unroll
      for (int q = 0; q < 3; ++q) {
        p[q] = __fadd_rn(v.eye[q], __fmul_rn(ts, d[q]));
        n[q] = __fdiv_rn(__fsub_rn(p[q], c.P.x[q * N + i]), v.radius);
      }
      shade(v, v.color, p, n, out);
    }
#pragma unroll
    for (int q = 0; q < 3; ++q) img[pix * 3 + q] = out[q];
  }
}

// _draw_lines (gui_3d.py:35-47): 24 vertices (the 12 edges, in the
// reference's stencil order) for every cell that is exactly ACTIVATED
__global__ void k_cell_lines(Ctx c, float* vert, long long cap, unsigned long long* count) {
  const long long tot = total_elems(c, 0, c.L, 3);
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < tot; e += (long long)gridDim.x * blockDim.x) {
    int l, loc;
    long long blk;
    decode_elem<3>(c, 0, c.L, e, l, blk, loc);
    const LevelDev& V = c.lev[l];
    if ((V.cell[(blk << 6) | loc] & ~CUL) != ACT) continue;
    int I[3];
    elem_coords<3>(V, blk, loc, I);
    const float dx = (1.f / (float)c.coarsest) / (float)(1 << l);
    const unsigned long long at = atomicAdd(count, 24ull);
    if ((long long)at + 24 > cap) continue;
    const int st[24] = {0, 1, 2, 3, 4, 5, 6, 7, 0, 2, 1, 3, 4, 6, 5, 7, 0, 4, 1, 5, 2, 6, 3, 7};
    for (int q = 0; q < 24; ++q) {
      const int k = st[q];  // corner dI with k = dI_0 + 2 dI_1 + 4 dI_2
#pragma unroll
      for (int a = 0; a < 3; ++a) vert[(at + q) * 3 + a] = (float)(I[a] + ((k >> a) & 1)) * dx;
    }
  }
}

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

namespace agimp {

agimp_status render_scene3d(agimp_sim* s, int res, const agimp_view3d* v, float* img, int memory, cudaStream_t st) {
  const Ctx& c = sim_ctx(s);
  if (c.dim != 3 || res < 1 || res > 16384 || !img || !v || !(v->radius > 0.f) || v->n_lights < 0 ||
      v->n_lights > 4 || !(v->tan_half_fov > 0.f)) {
    s->err = "render 3D: 3D only, 1 <= res <= 16384, radius > 0, tan_half_fov > 0, 0..4 lights, img required";
    return AGIMP_INVALID_ARG;
  }
  const size_t pix = (size_t)res * res;
  cudaError_t e = cudaSuccess;
  if (pix > s->rkey_n) {
    if (s->rkey) cudaFree(s->rkey);
    if (s->rdir) cudaFree(s->rdir);
    s->rkey = nullptr;
    s->rdir = nullptr;
    s->rkey_n = 0;
    e = cudaMalloc(&s->rkey, pix * sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMalloc(&s->rdir, pix * 3 * sizeof(float));
    if (e == cudaSuccess) s->rkey_n = pix;
  }
  if (e == cudaSuccess && (size_t)c.N + 1 > s->rslot_n) {
    if (s->rslot) cudaFree(s->rslot);
    s->rslot = nullptr;
    s->rslot_n = 0;
    e = cudaMalloc(&s->rslot, ((size_t)c.N + 1) * sizeof(int));
    if (e == cudaSuccess) s->rslot_n = (size_t)c.N + 1;
  }
  float* out = img;
  if (e == cudaSuccess && memory == AGIMP_MEM_HOST) {
    e = render_buffers(s, res, false);
    out = s->rimg;
  }
  if (e == cudaSuccess) e = cudaMemsetAsync(s->rkey, 0xff, pix * sizeof(unsigned long long), st);
  if (e == cudaSuccess) {
    k_rays<<<blocks_for((long long)pix), 256, 0, st>>>(*v, res, s->rdir);
    if (c.N) {
      k_slot_of<<<blocks_for(c.N), 256, 0, st>>>(c, s->rslot);
      k_splat3d<<<blocks_for(c.N), 256, 0, st>>>(c, *v, res, s->rdir, s->rkey);
    }
    k_shade3d<<<blocks_for((long long)pix), 256, 0, st>>>(c, *v, res, s->rdir, s->rkey, s->rslot, out);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess && memory == AGIMP_MEM_HOST) {
    e = cudaMemcpyAsync(img, out, pix * 3 * sizeof(float), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  }
  if (e != cudaSuccess) {
    s->err = std::string("render 3D: ") + cudaGetErrorString(e);
    return AGIMP_CUDA_ERROR;
  }
  return AGIMP_OK;
}

agimp_status cell_lines(agimp_sim* s, float* vert, long long cap, long long* count, int memory, cudaStream_t st) {
  const Ctx& c = sim_ctx(s);
  if (c.dim != 3 || !count || cap < 0 || (cap > 0 && !vert)) {
    s->err = "cell lines: 3D only; count required; vertices required when capacity > 0";
    return AGIMP_INVALID_ARG;
  }
  unsigned long long* dcount = nullptr;
  float* dv = nullptr;
  cudaError_t e = cudaMalloc(&dcount, sizeof(unsigned long long));
  if (e == cudaSuccess) e = cudaMemsetAsync(dcount, 0, sizeof(unsigned long long), st);
  float* target = vert;
  if (e == cudaSuccess && memory == AGIMP_MEM_HOST && cap > 0) {
    e = cudaMalloc(&dv, (size_t)cap * 3 * sizeof(float));
    target = dv;
  }
  if (e == cudaSuccess) {
    // the block lists and their counts are on the device: a grid-stride pass
    // over all of them
    k_cell_lines<<<148 * 8, 256, 0, st>>>(c, target, cap, dcount);
    e = cudaGetLastError();
  }
  unsigned long long n = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&n, dcount, sizeof(n), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e == cudaSuccess && memory == AGIMP_MEM_HOST && cap > 0)
    e = cudaMemcpy(vert, dv, (size_t)std::min<unsigned long long>(n, (unsigned long long)cap) * 3 * sizeof(float),
                   cudaMemcpyDeviceToHost);
  if (dcount) cudaFree(dcount);
  if (dv) cudaFree(dv);
  if (e != cudaSuccess) {
    s->err = std::string("cell lines: ") + cudaGetErrorString(e);
    return AGIMP_CUDA_ERROR;
  }
  *count = (long long)n;
  return AGIMP_OK;
}

}  // namespace agimp

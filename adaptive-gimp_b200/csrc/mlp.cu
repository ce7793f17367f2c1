// Surrogate return-map MLP (extension; the reference has no plasticity):
// 7 inputs -> 64 -> 64 -> 4 outputs, SiLU after the hidden layers, bf16
// weights and activations with f32 accumulation on the sm_100a tensor cores
// (tcgen05.mma, accumulators in tensor memory).
//
// Parameters are kept in f32 (the trainer's master copy) and packed into bf16
// tensor-core operand tiles after every change.  A CTA of 128 threads handles
// 128 samples per tile: thread t owns row t, which is TMEM lane t, so each
// warp reads its 32 rows back with tcgen05.ld.
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/agimp.h"
#include "common.cuh"
#include "umma.cuh"

namespace agimp {
namespace mlp {

constexpr int IN = 7, H = 64, OUT = 4;
constexpr int K1 = 16;  // input width padded to one MMA K step
constexpr int N3 = 16;  // output width padded to the smallest MMA N
constexpr int OW1 = 0, OB1 = OW1 + IN * H, OW2 = OB1 + H, OB2 = OW2 + H * H, OW3 = OB2 + H, OB3 = OW3 + H * OUT;
constexpr int NPARAM = OB3 + OUT;  // 4932
// packed bf16 operand tiles: B1 [64][16], B2 [64][64], B3 [16][64] (row = output unit, K-major)
constexpr int PB1 = 0, PB2 = PB1 + H * K1, PB3 = PB2 + H * H, NPACK = PB3 + N3 * H;  // 6144
constexpr int TILE = 128;

__device__ __forceinline__ float silu(float z) { return z / (1.f + __expf(-z)); }

__global__ void k_pack(const float* __restrict__ P, __nv_bfloat16* __restrict__ packed) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < NPACK; i += gridDim.x * blockDim.x) {
    float v;
    int dst;
    if (i < PB2) {
      const int n = i / K1, k = i % K1;
      v = k < IN ? P[OW1 + k * H + n] : 0.f;
      dst = PB1 + umma::tile_off(n, k, K1);
    } else if (i < PB3) {
      const int j = i - PB2, n = j / H, k = j % H;
      v = P[OW2 + k * H + n];
      dst = PB2 + umma::tile_off(n, k, H);
    } else {
      const int j = i - PB3, n = j / H, k = j % H;
      v = n < OUT ? P[OW3 + k * OUT + n] : 0.f;
      dst = PB3 + umma::tile_off(n, k, H);
    }
    packed[dst] = __float2bfloat16_rn(v);
  }
}

// shared-memory layout of the forward kernel (bytes)
struct FwdSmem {
  static constexpr int B1 = 0;
  static constexpr int B2 = B1 + 2 * H * K1;
  static constexpr int B3 = B2 + 2 * H * H;
  static constexpr int A1 = B3 + 2 * N3 * H;
  static constexpr int A2 = A1 + 2 * TILE * K1;
  static constexpr int A3 = A2 + 2 * TILE * H;
  static constexpr int BIAS = A3 + 2 * TILE * H;     // b1[64] b2[64] b3[16]
  static constexpr int MBAR = BIAS + 4 * (H + H + N3);
  static constexpr int TSLOT = MBAR + 8;
  static constexpr int BYTES = TSLOT + 16;
};

// Y[n][4] = MLP(X[n][7]) for n < N.
__global__ void __launch_bounds__(TILE) k_forward(const float* __restrict__ X, float* __restrict__ Y, long long N,
                                                  const __nv_bfloat16* __restrict__ packed,
                                                  const float* __restrict__ P, int32_t* __restrict__ err) {
  extern __shared__ __align__(128) unsigned char sm[];
  __nv_bfloat16* sB = (__nv_bfloat16*)(sm + FwdSmem::B1);
  __nv_bfloat16* sA1 = (__nv_bfloat16*)(sm + FwdSmem::A1);
  __nv_bfloat16* sA2 = (__nv_bfloat16*)(sm + FwdSmem::A2);
  __nv_bfloat16* sA3 = (__nv_bfloat16*)(sm + FwdSmem::A3);
  float* sb = (float*)(sm + FwdSmem::BIAS);
  uint64_t* mbar = (uint64_t*)(sm + FwdSmem::MBAR);
  uint32_t* tslot = (uint32_t*)(sm + FwdSmem::TSLOT);
  const int tid = threadIdx.x, warp = tid >> 5;
  for (int i = tid; i < NPACK; i += TILE) sB[i] = packed[i];
  for (int i = tid; i < H; i += TILE) {
    sb[i] = P[OB1 + i];
    sb[H + i] = P[OB2 + i];
  }
  if (tid < N3) sb[2 * H + tid] = tid < OUT ? P[OB3 + tid] : 0.f;
  if (tid == 0) {
    umma::mbar_init(mbar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) umma::tmem_alloc(tslot, 128);
  umma::fence_proxy_async();
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  const uint32_t tmem = *tslot;
  const uint32_t lane_base = (uint32_t)(warp * 32) << 16;
  const uint32_t aB1 = umma::smem_u32(sm + FwdSmem::B1), aB2 = umma::smem_u32(sm + FwdSmem::B2),
                 aB3 = umma::smem_u32(sm + FwdSmem::B3);
  const uint32_t aA1 = umma::smem_u32(sA1), aA2 = umma::smem_u32(sA2), aA3 = umma::smem_u32(sA3);
  uint32_t phase = 0;
  bool ok = true;
  const long long ntiles = (N + TILE - 1) / TILE;
  for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const long long row = tile * TILE + tid;
#pragma unroll
    for (int k = 0; k < K1; ++k) {
      const float v = (k < IN && row < N) ? X[row * IN + k] : 0.f;
      sA1[umma::tile_off(tid, k, K1)] = __float2bfloat16_rn(v);
    }
    umma::fence_proxy_async();
    umma::fence_before_sync();
    __syncthreads();
    umma::fence_after_sync();
    // layer 1: [128 x 16] x [16 x 64] -> TMEM columns [0, 64)
    if (tid == 0) {
      umma::mma_bf16(tmem, umma::smem_desc(aA1, 128, 2 * 128), umma::smem_desc(aB1, 128, 2 * 128),
                     umma::idesc_bf16_f32(TILE, H), 0);
      umma::mma_commit(mbar);
    }
    ok = umma::mbar_wait(mbar, phase) && ok;
    phase ^= 1;
    umma::fence_after_sync();
#pragma unroll
    for (int c = 0; c < H / 16; ++c) {
      float acc[16];
      umma::tmem_ld16(tmem + lane_base + c * 16, acc);
#pragma unroll
      for (int j = 0; j < 16; ++j)
        sA2[umma::tile_off(tid, c * 16 + j, H)] = __float2bfloat16_rn(silu(acc[j] + sb[c * 16 + j]));
    }
    umma::fence_proxy_async();
    umma::fence_before_sync();
    __syncthreads();
    umma::fence_after_sync();
    // layer 2: [128 x 64] x [64 x 64] -> TMEM columns [64, 128)
    if (tid == 0) {
#pragma unroll
      for (int kk = 0; kk < H / 16; ++kk)
        umma::mma_bf16(tmem + 64, umma::smem_desc(aA2 + kk * 256, 128, 8 * 128),
                       umma::smem_desc(aB2 + kk * 256, 128, 8 * 128), umma::idesc_bf16_f32(TILE, H), kk > 0);
      umma::mma_commit(mbar);
    }
    ok = umma::mbar_wait(mbar, phase) && ok;
    phase ^= 1;
    umma::fence_after_sync();
#pragma unroll
    for (int c = 0; c < H / 16; ++c) {
      float acc[16];
      umma::tmem_ld16(tmem + lane_base + 64 + c * 16, acc);
#pragma unroll
      for (int j = 0; j < 16; ++j)
        sA3[umma::tile_off(tid, c * 16 + j, H)] = __float2bfloat16_rn(silu(acc[j] + sb[H + c * 16 + j]));
    }
    umma::fence_proxy_async();
    umma::fence_before_sync();
    __syncthreads();
    umma::fence_after_sync();
    // layer 3: [128 x 64] x [64 x 16] -> TMEM columns [0, 16)
    if (tid == 0) {
#pragma unroll
      for (int kk = 0; kk < H / 16; ++kk)
        umma::mma_bf16(tmem, umma::smem_desc(aA3 + kk * 256, 128, 8 * 128),
                       umma::smem_desc(aB3 + kk * 256, 128, 8 * 128), umma::idesc_bf16_f32(TILE, N3), kk > 0);
      umma::mma_commit(mbar);
    }
    ok = umma::mbar_wait(mbar, phase) && ok;
    phase ^= 1;
    umma::fence_after_sync();
    {
      float acc[16];
      umma::tmem_ld16(tmem + lane_base, acc);
      if (row < N) {
#pragma unroll
        for (int j = 0; j < OUT; ++j) Y[row * OUT + j] = acc[j] + sb[2 * H + j];
      }
    }
    umma::fence_before_sync();
    __syncthreads();
    umma::fence_after_sync();
  }
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  if (warp == 0) umma::tmem_dealloc(tmem, 128);
  if (!ok && tid == 0) atomicOr((unsigned*)err, 1u);
}

}  // namespace mlp
}  // namespace agimp

using namespace agimp;

struct agimp_mlp {
  int device = 0;
  float* P = nullptr;               // f32 parameters
  __nv_bfloat16* packed = nullptr;  // bf16 operand tiles
  int32_t* err = nullptr;
  int sms = 148;
  std::string msg;
};

extern "C" {

agimp_status agimp_mlp_create(int32_t device, agimp_mlp** out) {
  if (!out) return AGIMP_INVALID_ARG;
  *out = nullptr;
  if (cudaSetDevice(device) != cudaSuccess) return AGIMP_CUDA_ERROR;
  agimp_mlp* m = new agimp_mlp();
  m->device = device;
  cudaDeviceGetAttribute(&m->sms, cudaDevAttrMultiProcessorCount, device);
  if (cudaMalloc(&m->P, mlp::NPARAM * sizeof(float)) != cudaSuccess ||
      cudaMalloc(&m->packed, mlp::NPACK * sizeof(__nv_bfloat16)) != cudaSuccess ||
      cudaMalloc(&m->err, sizeof(int32_t)) != cudaSuccess) {
    cudaFree(m->P);
    cudaFree(m->packed);
    cudaFree(m->err);
    delete m;
    return AGIMP_OUT_OF_MEMORY;
  }
  cudaMemset(m->P, 0, mlp::NPARAM * sizeof(float));
  cudaMemset(m->packed, 0, mlp::NPACK * sizeof(__nv_bfloat16));
  cudaMemset(m->err, 0, sizeof(int32_t));
  cudaFuncSetAttribute(mlp::k_forward, cudaFuncAttributeMaxDynamicSharedMemorySize, mlp::FwdSmem::BYTES);
  if (cudaDeviceSynchronize() != cudaSuccess) {
    delete m;
    return AGIMP_CUDA_ERROR;
  }
  *out = m;
  return AGIMP_OK;
}

agimp_status agimp_mlp_destroy(agimp_mlp* m) {
  if (!m) return AGIMP_INVALID_ARG;
  cudaSetDevice(m->device);
  cudaDeviceSynchronize();
  cudaFree(m->P);
  cudaFree(m->packed);
  cudaFree(m->err);
  delete m;
  return AGIMP_OK;
}

int32_t agimp_mlp_num_params(void) { return mlp::NPARAM; }

agimp_status agimp_mlp_set_params(agimp_mlp* m, const float* params, int32_t memory, void* stream) {
  if (!m || !params) return AGIMP_INVALID_ARG;
  if (cudaSetDevice(m->device) != cudaSuccess) return AGIMP_CUDA_ERROR;
  cudaStream_t s = (cudaStream_t)stream;
  const cudaMemcpyKind k = memory == AGIMP_MEM_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
  if (cudaMemcpyAsync(m->P, params, mlp::NPARAM * sizeof(float), k, s) != cudaSuccess) return AGIMP_CUDA_ERROR;
  mlp::k_pack<<<(mlp::NPACK + 255) / 256, 256, 0, s>>>(m->P, m->packed);
  if (memory == AGIMP_MEM_HOST && cudaStreamSynchronize(s) != cudaSuccess) return AGIMP_CUDA_ERROR;
  return cudaGetLastError() == cudaSuccess ? AGIMP_OK : AGIMP_CUDA_ERROR;
}

agimp_status agimp_mlp_get_params(agimp_mlp* m, float* params, int32_t memory, void* stream) {
  if (!m || !params) return AGIMP_INVALID_ARG;
  if (cudaSetDevice(m->device) != cudaSuccess) return AGIMP_CUDA_ERROR;
  cudaStream_t s = (cudaStream_t)stream;
  const cudaMemcpyKind k = memory == AGIMP_MEM_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
  if (cudaMemcpyAsync(params, m->P, mlp::NPARAM * sizeof(float), k, s) != cudaSuccess) return AGIMP_CUDA_ERROR;
  if (memory == AGIMP_MEM_HOST && cudaStreamSynchronize(s) != cudaSuccess) return AGIMP_CUDA_ERROR;
  return AGIMP_OK;
}

agimp_status agimp_mlp_forward(agimp_mlp* m, const float* X, float* Y, int64_t n, void* stream) {
  if (!m || n < 0 || (n > 0 && (!X || !Y))) return AGIMP_INVALID_ARG;
  if (n == 0) return AGIMP_OK;
  if (cudaSetDevice(m->device) != cudaSuccess) return AGIMP_CUDA_ERROR;
  const long long ntiles = (n + mlp::TILE - 1) / mlp::TILE;
  const int grid = (int)std::min<long long>(ntiles, (long long)m->sms * 4);
  mlp::k_forward<<<grid, mlp::TILE, mlp::FwdSmem::BYTES, (cudaStream_t)stream>>>(X, Y, n, m->packed, m->P, m->err);
  return cudaGetLastError() == cudaSuccess ? AGIMP_OK : AGIMP_CUDA_ERROR;
}

agimp_status agimp_mlp_errors(agimp_mlp* m, uint32_t* bits, int32_t clear) {
  if (!m || !bits) return AGIMP_INVALID_ARG;
  if (cudaSetDevice(m->device) != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess) return AGIMP_CUDA_ERROR;
  int32_t v = 0;
  if (cudaMemcpy(&v, m->err, sizeof(v), cudaMemcpyDeviceToHost) != cudaSuccess) return AGIMP_CUDA_ERROR;
  *bits = (uint32_t)v;
  if (clear) cudaMemset(m->err, 0, sizeof(int32_t));
  return AGIMP_OK;
}

}  // extern "C"

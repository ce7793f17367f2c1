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
// packed bf16 operand tiles (K-major): forward B1 [64][16], B2 [64][64], B3 [16][64]
// (row = output unit), backward B3T [64][16] (row = hidden unit of layer 2,
// K = outputs) and B2T [64][64] (row = hidden unit of layer 1, K = layer-2 units)
constexpr int PB1 = 0, PB2 = PB1 + H * K1, PB3 = PB2 + H * H, NPACK_FWD = PB3 + N3 * H;  // 6144
constexpr int PB3T = NPACK_FWD, PB2T = PB3T + H * K1, NPACK = PB2T + H * H;           // 11264
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
    } else if (i < PB3T) {
      const int j = i - PB3, n = j / H, k = j % H;
      v = n < OUT ? P[OW3 + k * OUT + n] : 0.f;
      dst = PB3 + umma::tile_off(n, k, H);
    } else if (i < PB2T) {
      const int j = i - PB3T, n = j / K1, k = j % K1;  // (n, k) = W3[n][k]
      v = k < OUT ? P[OW3 + n * OUT + k] : 0.f;
      dst = PB3T + umma::tile_off(n, k, K1);
    } else {
      const int j = i - PB2T, n = j / H, k = j % H;  // (n, k) = W2[n][k]
      v = P[OW2 + n * H + k];
      dst = PB2T + umma::tile_off(n, k, H);
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
                                                  const float* __restrict__ P, int32_t* __restrict__ err,
                                                  const int32_t* __restrict__ n_dev, uint32_t err_bit) {
  if (n_dev) N = min((long long)*n_dev, N);  // device-side sample count, capped by the buffer size
  extern __shared__ __align__(128) unsigned char sm[];
  __nv_bfloat16* sB = (__nv_bfloat16*)(sm + FwdSmem::B1);
  __nv_bfloat16* sA1 = (__nv_bfloat16*)(sm + FwdSmem::A1);
  __nv_bfloat16* sA2 = (__nv_bfloat16*)(sm + FwdSmem::A2);
  __nv_bfloat16* sA3 = (__nv_bfloat16*)(sm + FwdSmem::A3);
  float* sb = (float*)(sm + FwdSmem::BIAS);
  uint64_t* mbar = (uint64_t*)(sm + FwdSmem::MBAR);
  uint32_t* tslot = (uint32_t*)(sm + FwdSmem::TSLOT);
  const int tid = threadIdx.x, warp = tid >> 5;
  for (int i = tid; i < NPACK_FWD; i += TILE) sB[i] = packed[i];
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
  if (!ok && tid == 0) atomicOr((unsigned*)err, err_bit);
}


// ---------------------------------------------------------------------------
// Training: loss and gradient of the mean squared error over n samples.
// Per tile of 128 samples (thread t = sample t = TMEM lane t):
//   forward  Z1 = X W1, A1 = silu(Z1 + b1), Z2 = A1 W2, A2 = silu(Z2 + b2),
//            Y = A2 W3 + b3                                  (3 MMAs)
//   backward dY = 2 (Y - T) / n, dA2 = dY W3^T, dZ2 = dA2 silu'(.),
//            dA1 = dZ2 W2^T, dZ1 = dA1 silu'(.)              (2 MMAs)
//   weights  G3 += [A2^T; 1] dY, G2 += [A1^T; 1] dZ2, G1 += [X^T; 1] dZ1
// The weight-gradient MMAs take the transposed activations as A (M = 128 rows:
// the real features, then one row of ones that yields the bias gradient, then
// zeros) and accumulate in TMEM over all tiles of the CTA; the CTA then adds
// them to the global gradient with atomics.
struct TrainSmem {
  static constexpr int B1 = 0;                       // [64][16]
  static constexpr int B2 = B1 + 2 * H * K1;         // [64][64]
  static constexpr int B3 = B2 + 2 * H * H;          // [16][64]
  static constexpr int B3T = B3 + 2 * N3 * H;        // [64][16]
  static constexpr int B2T = B3T + 2 * H * K1;       // [64][64]
  static constexpr int X = B2T + 2 * H * H;          // [128][16]
  static constexpr int A1 = X + 2 * TILE * K1;       // [128][64]
  static constexpr int A2 = A1 + 2 * TILE * H;       // [128][64]
  static constexpr int DY = A2 + 2 * TILE * H;       // [128][16]
  static constexpr int DZ2 = DY + 2 * TILE * K1;     // [128][64]
  static constexpr int XT = DZ2 + 2 * TILE * H;      // [128][128]
  static constexpr int A1T = XT + 2 * TILE * TILE;   // [128][128]
  static constexpr int A2T = A1T + 2 * TILE * TILE;  // [128][128]
  static constexpr int DZ1T = A2T + 2 * TILE * TILE; // [64][128]
  static constexpr int DZ2T = DZ1T + 2 * H * TILE;   // [64][128]
  static constexpr int DYT = DZ2T + 2 * H * TILE;    // [16][128]
  static constexpr int BIAS = DYT + 2 * N3 * TILE;   // b1[64] b2[64] b3[16]
  static constexpr int LOSS = BIAS + 4 * (H + H + N3);
  static constexpr int MBAR = LOSS + 8;
  static constexpr int TSLOT = MBAR + 8;
  static constexpr int BYTES = TSLOT + 16;
};
// TMEM columns
constexpr int TZ1 = 0, TZ2 = 64, TY = 128, TDA2 = 192, TDA1 = 256, TG1 = 320, TG2 = 384, TG3 = 448;

__device__ __forceinline__ float dsilu(float z) {
  const float s = 1.f / (1.f + __expf(-z));
  return s * (1.f + z * (1.f - s));
}

__global__ void __launch_bounds__(TILE) k_train(const float* __restrict__ Xg, const float* __restrict__ Tg, long long N,
                                                const __nv_bfloat16* __restrict__ packed, const float* __restrict__ P,
                                                float* __restrict__ grad, float* __restrict__ loss,
                                                int32_t* __restrict__ err) {
  extern __shared__ __align__(128) unsigned char sm[];
  using S = TrainSmem;
  __nv_bfloat16* sX = (__nv_bfloat16*)(sm + S::X);
  __nv_bfloat16* sA1 = (__nv_bfloat16*)(sm + S::A1);
  __nv_bfloat16* sA2 = (__nv_bfloat16*)(sm + S::A2);
  __nv_bfloat16* sDY = (__nv_bfloat16*)(sm + S::DY);
  __nv_bfloat16* sDZ2 = (__nv_bfloat16*)(sm + S::DZ2);
  __nv_bfloat16* sXT = (__nv_bfloat16*)(sm + S::XT);
  __nv_bfloat16* sA1T = (__nv_bfloat16*)(sm + S::A1T);
  __nv_bfloat16* sA2T = (__nv_bfloat16*)(sm + S::A2T);
  __nv_bfloat16* sDZ1T = (__nv_bfloat16*)(sm + S::DZ1T);
  __nv_bfloat16* sDZ2T = (__nv_bfloat16*)(sm + S::DZ2T);
  __nv_bfloat16* sDYT = (__nv_bfloat16*)(sm + S::DYT);
  float* sb = (float*)(sm + S::BIAS);
  float* sloss = (float*)(sm + S::LOSS);
  uint64_t* mbar = (uint64_t*)(sm + S::MBAR);
  uint32_t* tslot = (uint32_t*)(sm + S::TSLOT);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  __nv_bfloat16* sB = (__nv_bfloat16*)(sm + S::B1);
  for (int i = tid; i < NPACK; i += TILE) sB[i] = packed[i];
  for (int i = tid; i < H; i += TILE) {
    sb[i] = P[OB1 + i];
    sb[H + i] = P[OB2 + i];
  }
  if (tid < N3) sb[2 * H + tid] = tid < OUT ? P[OB3 + tid] : 0.f;
  // constant parts of the operand tiles: zero padding and the rows of ones
  const __nv_bfloat16 zero = __float2bfloat16_rn(0.f), one = __float2bfloat16_rn(1.f);
  for (int i = tid; i < TILE * TILE; i += TILE) {
    const int r = i / TILE, k = i % TILE;
    if (r >= IN) sXT[umma::tile_off(r, k, TILE)] = r == IN ? one : zero;
    if (r >= H) {
      sA1T[umma::tile_off(r, k, TILE)] = r == H ? one : zero;
      sA2T[umma::tile_off(r, k, TILE)] = r == H ? one : zero;
    }
    if (r >= OUT && r < N3) sDYT[umma::tile_off(r, k, TILE)] = zero;
  }
  for (int i = tid; i < TILE * K1; i += TILE) {
    const int r = i / K1, k = i % K1;
    if (k >= IN) sX[umma::tile_off(r, k, K1)] = zero;
    if (k >= OUT) sDY[umma::tile_off(r, k, K1)] = zero;
  }
  if (tid == 0) {
    *sloss = 0.f;
    umma::mbar_init(mbar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) umma::tmem_alloc(tslot, 512);
  umma::fence_proxy_async();
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  const uint32_t tmem = *tslot;
  const uint32_t lb = (uint32_t)(warp * 32) << 16;
  auto addr = [&](int off) { return umma::smem_u32(sm + off); };
  const uint32_t id_64 = umma::idesc_bf16_f32(TILE, H), id_16 = umma::idesc_bf16_f32(TILE, N3);
  uint32_t phase = 0;
  bool ok = true;
  float my_loss = 0.f;
  const float inv_n = 1.f / (float)N;
  const long long ntiles = (N + TILE - 1) / TILE;
  bool first = true;
  auto sync_for_mma = [&]() {
    umma::fence_proxy_async();
    umma::fence_before_sync();
    __syncthreads();
    umma::fence_after_sync();
  };
  auto wait_mma = [&]() {
    ok = umma::mbar_wait(mbar, phase) && ok;
    phase ^= 1;
    umma::fence_after_sync();
  };
  for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const long long row = tile * TILE + tid;
    const bool live = row < N;
    float t[OUT];
#pragma unroll
    for (int k = 0; k < IN; ++k) {
      const __nv_bfloat16 v = __float2bfloat16_rn(live ? Xg[row * IN + k] : 0.f);
      sX[umma::tile_off(tid, k, K1)] = v;
      sXT[umma::tile_off(k, tid, TILE)] = v;
    }
#pragma unroll
    for (int j = 0; j < OUT; ++j) t[j] = live ? Tg[row * OUT + j] : 0.f;
    sync_for_mma();
    if (tid == 0) {
      umma::mma_bf16(tmem + TZ1, umma::smem_desc(addr(S::X), 128, 2 * 128), umma::smem_desc(addr(S::B1), 128, 2 * 128),
                     id_64, 0);
      umma::mma_commit(mbar);
    }
    wait_mma();
#pragma unroll
    for (int c = 0; c < H / 16; ++c) {
      float acc[16];
      umma::tmem_ld16(tmem + lb + TZ1 + c * 16, acc);
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        const __nv_bfloat16 a = __float2bfloat16_rn(silu(acc[j] + sb[c * 16 + j]));
        sA1[umma::tile_off(tid, c * 16 + j, H)] = a;
        sA1T[umma::tile_off(c * 16 + j, tid, TILE)] = a;
      }
    }
    sync_for_mma();
    if (tid == 0) {
#pragma unroll
      for (int kk = 0; kk < H / 16; ++kk)
        umma::mma_bf16(tmem + TZ2, umma::smem_desc(addr(S::A1) + kk * 256, 128, 8 * 128),
                       umma::smem_desc(addr(S::B2) + kk * 256, 128, 8 * 128), id_64, kk > 0);
      umma::mma_commit(mbar);
    }
    wait_mma();
#pragma unroll
    for (int c = 0; c < H / 16; ++c) {
      float acc[16];
      umma::tmem_ld16(tmem + lb + TZ2 + c * 16, acc);
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        const __nv_bfloat16 a = __float2bfloat16_rn(silu(acc[j] + sb[H + c * 16 + j]));
        sA2[umma::tile_off(tid, c * 16 + j, H)] = a;
        sA2T[umma::tile_off(c * 16 + j, tid, TILE)] = a;
      }
    }
    sync_for_mma();
    if (tid == 0) {
#pragma unroll
      for (int kk = 0; kk < H / 16; ++kk)
        umma::mma_bf16(tmem + TY, umma::smem_desc(addr(S::A2) + kk * 256, 128, 8 * 128),
                       umma::smem_desc(addr(S::B3) + kk * 256, 128, 8 * 128), id_16, kk > 0);
      umma::mma_commit(mbar);
    }
    wait_mma();
    {
      float acc[16];
      umma::tmem_ld16(tmem + lb + TY, acc);
#pragma unroll
      for (int j = 0; j < OUT; ++j) {
        const float e = live ? acc[j] + sb[2 * H + j] - t[j] : 0.f;
        my_loss += e * e;
        const __nv_bfloat16 d = __float2bfloat16_rn(2.f * e * inv_n);
        sDY[umma::tile_off(tid, j, K1)] = d;
        sDYT[umma::tile_off(j, tid, TILE)] = d;
      }
    }
    sync_for_mma();
    // dA2 = dY W3^T ; G3 += [A2^T; 1] dY
    if (tid == 0) {
      umma::mma_bf16(tmem + TDA2, umma::smem_desc(addr(S::DY), 128, 2 * 128),
                     umma::smem_desc(addr(S::B3T), 128, 2 * 128), id_64, 0);
#pragma unroll
      for (int kk = 0; kk < TILE / 16; ++kk)
        umma::mma_bf16(tmem + TG3, umma::smem_desc(addr(S::A2T) + kk * 256, 128, 16 * 128),
                       umma::smem_desc(addr(S::DYT) + kk * 256, 128, 16 * 128), id_16, (!first || kk > 0) ? 1u : 0u);
      umma::mma_commit(mbar);
    }
    wait_mma();
#pragma unroll
    for (int c = 0; c < H / 16; ++c) {
      float da[16], z[16];
      umma::tmem_ld16(tmem + lb + TDA2 + c * 16, da);
      umma::tmem_ld16(tmem + lb + TZ2 + c * 16, z);
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        const __nv_bfloat16 d = __float2bfloat16_rn(da[j] * dsilu(z[j] + sb[H + c * 16 + j]));
        sDZ2[umma::tile_off(tid, c * 16 + j, H)] = d;
        sDZ2T[umma::tile_off(c * 16 + j, tid, TILE)] = d;
      }
    }
    sync_for_mma();
    // dA1 = dZ2 W2^T ; G2 += [A1^T; 1] dZ2
    if (tid == 0) {
#pragma unroll
      for (int kk = 0; kk < H / 16; ++kk)
        umma::mma_bf16(tmem + TDA1, umma::smem_desc(addr(S::DZ2) + kk * 256, 128, 8 * 128),
                       umma::smem_desc(addr(S::B2T) + kk * 256, 128, 8 * 128), id_64, kk > 0);
#pragma unroll
      for (int kk = 0; kk < TILE / 16; ++kk)
        umma::mma_bf16(tmem + TG2, umma::smem_desc(addr(S::A1T) + kk * 256, 128, 16 * 128),
                       umma::smem_desc(addr(S::DZ2T) + kk * 256, 128, 16 * 128), id_64, (!first || kk > 0) ? 1u : 0u);
      umma::mma_commit(mbar);
    }
    wait_mma();
#pragma unroll
    for (int c = 0; c < H / 16; ++c) {
      float da[16], z[16];
      umma::tmem_ld16(tmem + lb + TDA1 + c * 16, da);
      umma::tmem_ld16(tmem + lb + TZ1 + c * 16, z);
#pragma unroll
      for (int j = 0; j < 16; ++j)
        sDZ1T[umma::tile_off(c * 16 + j, tid, TILE)] = __float2bfloat16_rn(da[j] * dsilu(z[j] + sb[c * 16 + j]));
    }
    sync_for_mma();
    // G1 += [X^T; 1] dZ1
    if (tid == 0) {
#pragma unroll
      for (int kk = 0; kk < TILE / 16; ++kk)
        umma::mma_bf16(tmem + TG1, umma::smem_desc(addr(S::XT) + kk * 256, 128, 16 * 128),
                       umma::smem_desc(addr(S::DZ1T) + kk * 256, 128, 16 * 128), id_64, (!first || kk > 0) ? 1u : 0u);
      umma::mma_commit(mbar);
    }
    wait_mma();
    first = false;
    umma::fence_before_sync();
    __syncthreads();
    umma::fence_after_sync();
  }
  // loss
#pragma unroll
  for (int o = 16; o; o >>= 1) my_loss += __shfl_xor_sync(0xffffffffu, my_loss, o);
  if (lane == 0) atomicAdd(sloss, my_loss);
  // weight gradients: thread tid holds row tid of G1 / G2 / G3
  if (!first) {
#pragma unroll
    for (int c = 0; c < H / 16; ++c) {
      float g[16];
      umma::tmem_ld16(tmem + lb + TG1 + c * 16, g);
      if (tid < IN)
        for (int j = 0; j < 16; ++j) atomicAdd(&grad[OW1 + tid * H + c * 16 + j], g[j]);
      else if (tid == IN)
        for (int j = 0; j < 16; ++j) atomicAdd(&grad[OB1 + c * 16 + j], g[j]);
      umma::tmem_ld16(tmem + lb + TG2 + c * 16, g);
      if (tid < H)
        for (int j = 0; j < 16; ++j) atomicAdd(&grad[OW2 + tid * H + c * 16 + j], g[j]);
      else if (tid == H)
        for (int j = 0; j < 16; ++j) atomicAdd(&grad[OB2 + c * 16 + j], g[j]);
    }
    float g[16];
    umma::tmem_ld16(tmem + lb + TG3, g);
    if (tid < H)
      for (int j = 0; j < OUT; ++j) atomicAdd(&grad[OW3 + tid * OUT + j], g[j]);
    else if (tid == H)
      for (int j = 0; j < OUT; ++j) atomicAdd(&grad[OB3 + j], g[j]);
  }
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  if (tid == 0) atomicAdd(loss, *sloss * inv_n);
  if (warp == 0) umma::tmem_dealloc(tmem, 512);
  if (!ok && tid == 0) atomicOr((unsigned*)err, 1u);
}

// Adam (Kingma & Ba 2015) on the f32 parameters; step >= 1
__global__ void k_adam(float* __restrict__ P, const float* __restrict__ g, float* __restrict__ m1,
                       float* __restrict__ m2, float lr, float b1, float b2, float eps, int step) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= NPARAM) return;
  const float gi = g[i];
  const float a = b1 * m1[i] + (1.f - b1) * gi, b = b2 * m2[i] + (1.f - b2) * gi * gi;
  m1[i] = a;
  m2[i] = b;
  const float ah = a / (1.f - powf(b1, (float)step)), bh = b / (1.f - powf(b2, (float)step));
  P[i] -= lr * ah / (sqrtf(bh) + eps);
}

}  // namespace mlp

void launch_mlp_forward_dev(const void* packed, const float* P, const float* X, float* Y, const int32_t* n_dev,
                            long long cap, int32_t* err, int sms, cudaStream_t s) {
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(mlp::k_forward, cudaFuncAttributeMaxDynamicSharedMemorySize, mlp::FwdSmem::BYTES);
    attr = true;
  }
  const long long ntiles = (cap + mlp::TILE - 1) / mlp::TILE;
  const int grid = (int)std::min<long long>(ntiles, (long long)sms * 4);
  mlp::k_forward<<<grid, mlp::TILE, mlp::FwdSmem::BYTES, s>>>(X, Y, cap, (const __nv_bfloat16*)packed, P, err, n_dev,
                                                             ERR_MLP);
}

// Self-test of the bounded completion wait of the tensor-core kernels
// (umma::mbar_wait): one CTA waits on an mbarrier of one expected arrival.
// With arrive = 1 a thread arrives first and the wait succeeds; with
// arrive = 0 nothing ever arrives, the wait gives up after max_polls polls,
// the kernel records ERR_MLP in *err and returns normally, so the context
// stays usable.  This is how a lost tensor-core completion surfaces.
__global__ void k_wait_selftest(uint32_t* err, uint32_t max_polls, int arrive) {
  __shared__ uint64_t mbar;
  if (threadIdx.x == 0) {
    umma::mbar_init(&mbar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  if (arrive && threadIdx.x == 0)
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(umma::smem_u32(&mbar)) : "memory");
  const bool ok = umma::mbar_wait(&mbar, 0, max_polls);
  if (!ok && threadIdx.x == 0) atomicOr(err, ERR_MLP);
}

}  // namespace agimp

using namespace agimp;

struct agimp_mlp {
  int device = 0;
  float* P = nullptr;               // f32 parameters
  __nv_bfloat16* packed = nullptr;  // bf16 operand tiles
  float* grad = nullptr;            // gradient, Adam moments, loss
  float* m1 = nullptr;
  float* m2 = nullptr;
  float* loss = nullptr;
  int step = 0;
  int32_t* err = nullptr;
  int sms = 148;
  std::string msg;
};

namespace agimp {
void mlp_buffers(const agimp_mlp* m, const void** packed, const float** P) {
  *packed = m->packed;
  *P = m->P;
}
}  // namespace agimp

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
      cudaMalloc(&m->grad, mlp::NPARAM * sizeof(float)) != cudaSuccess ||
      cudaMalloc(&m->m1, mlp::NPARAM * sizeof(float)) != cudaSuccess ||
      cudaMalloc(&m->m2, mlp::NPARAM * sizeof(float)) != cudaSuccess ||
      cudaMalloc(&m->loss, sizeof(float)) != cudaSuccess || cudaMalloc(&m->err, sizeof(int32_t)) != cudaSuccess) {
    cudaFree(m->P);
    cudaFree(m->packed);
    cudaFree(m->grad);
    cudaFree(m->m1);
    cudaFree(m->m2);
    cudaFree(m->loss);
    cudaFree(m->err);
    delete m;
    return AGIMP_OUT_OF_MEMORY;
  }
  cudaMemset(m->m1, 0, mlp::NPARAM * sizeof(float));
  cudaMemset(m->m2, 0, mlp::NPARAM * sizeof(float));
  cudaMemset(m->P, 0, mlp::NPARAM * sizeof(float));
  cudaMemset(m->packed, 0, mlp::NPACK * sizeof(__nv_bfloat16));
  cudaMemset(m->err, 0, sizeof(int32_t));
  cudaFuncSetAttribute(mlp::k_forward, cudaFuncAttributeMaxDynamicSharedMemorySize, mlp::FwdSmem::BYTES);
  cudaFuncSetAttribute(mlp::k_train, cudaFuncAttributeMaxDynamicSharedMemorySize, mlp::TrainSmem::BYTES);
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
  cudaFree(m->grad);
  cudaFree(m->m1);
  cudaFree(m->m2);
  cudaFree(m->loss);
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
  mlp::k_forward<<<grid, mlp::TILE, mlp::FwdSmem::BYTES, (cudaStream_t)stream>>>(X, Y, n, m->packed, m->P, m->err,
                                                                                 nullptr, 1u);
  return cudaGetLastError() == cudaSuccess ? AGIMP_OK : AGIMP_CUDA_ERROR;
}

static agimp_status mlp_grad(agimp_mlp* m, const float* X, const float* T, int64_t n, cudaStream_t s) {
  cudaMemsetAsync(m->grad, 0, mlp::NPARAM * sizeof(float), s);
  cudaMemsetAsync(m->loss, 0, sizeof(float), s);
  if (n == 0) return AGIMP_OK;
  const long long ntiles = (n + mlp::TILE - 1) / mlp::TILE;
  const int grid = (int)std::min<long long>(ntiles, (long long)m->sms);
  mlp::k_train<<<grid, mlp::TILE, mlp::TrainSmem::BYTES, s>>>(X, T, n, m->packed, m->P, m->grad, m->loss, m->err);
  return cudaGetLastError() == cudaSuccess ? AGIMP_OK : AGIMP_CUDA_ERROR;
}

agimp_status agimp_mlp_grad(agimp_mlp* m, const float* X, const float* T, int64_t n, float* grad, float* loss,
                            void* stream) {
  if (!m || n < 0 || (n > 0 && (!X || !T))) return AGIMP_INVALID_ARG;
  if (cudaSetDevice(m->device) != cudaSuccess) return AGIMP_CUDA_ERROR;
  cudaStream_t s = (cudaStream_t)stream;
  agimp_status r = mlp_grad(m, X, T, n, s);
  if (r) return r;
  if (grad && cudaMemcpyAsync(grad, m->grad, mlp::NPARAM * sizeof(float), cudaMemcpyDeviceToDevice, s) != cudaSuccess)
    return AGIMP_CUDA_ERROR;
  if (loss && cudaMemcpyAsync(loss, m->loss, sizeof(float), cudaMemcpyDeviceToDevice, s) != cudaSuccess)
    return AGIMP_CUDA_ERROR;
  return AGIMP_OK;
}

agimp_status agimp_mlp_train_step(agimp_mlp* m, const float* X, const float* T, int64_t n, float lr, float* loss,
                                  void* stream) {
  if (!m || n <= 0 || !X || !T || !(lr > 0.f)) return AGIMP_INVALID_ARG;
  if (cudaSetDevice(m->device) != cudaSuccess) return AGIMP_CUDA_ERROR;
  cudaStream_t s = (cudaStream_t)stream;
  agimp_status r = mlp_grad(m, X, T, n, s);
  if (r) return r;
  m->step += 1;
  mlp::k_adam<<<(mlp::NPARAM + 255) / 256, 256, 0, s>>>(m->P, m->grad, m->m1, m->m2, lr, 0.9f, 0.999f, 1e-8f,
                                                         m->step);
  mlp::k_pack<<<(mlp::NPACK + 255) / 256, 256, 0, s>>>(m->P, m->packed);
  if (loss && cudaMemcpyAsync(loss, m->loss, sizeof(float), cudaMemcpyDeviceToDevice, s) != cudaSuccess)
    return AGIMP_CUDA_ERROR;
  return cudaGetLastError() == cudaSuccess ? AGIMP_OK : AGIMP_CUDA_ERROR;
}

agimp_status agimp_mlp_reset_optimizer(agimp_mlp* m) {
  if (!m) return AGIMP_INVALID_ARG;
  if (cudaSetDevice(m->device) != cudaSuccess) return AGIMP_CUDA_ERROR;
  cudaMemset(m->m1, 0, mlp::NPARAM * sizeof(float));
  cudaMemset(m->m2, 0, mlp::NPARAM * sizeof(float));
  m->step = 0;
  return AGIMP_OK;
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

agimp_status agimp_wait_selftest(int32_t device, int32_t arrive, uint32_t max_polls, uint32_t* bits) {
  if (!bits || max_polls == 0) return AGIMP_INVALID_ARG;
  if (cudaSetDevice(device) != cudaSuccess) return AGIMP_CUDA_ERROR;
  uint32_t* d = nullptr;
  if (cudaMalloc(&d, sizeof(uint32_t)) != cudaSuccess) return AGIMP_OUT_OF_MEMORY;
  uint32_t v = 0;
  bool good = cudaMemset(d, 0, sizeof(uint32_t)) == cudaSuccess;
  if (good) {
    k_wait_selftest<<<1, 128>>>(d, max_polls, arrive);
    good = cudaGetLastError() == cudaSuccess && cudaDeviceSynchronize() == cudaSuccess &&
           cudaMemcpy(&v, d, sizeof(v), cudaMemcpyDeviceToHost) == cudaSuccess;
  }
  cudaFree(d);
  if (!good) return AGIMP_CUDA_ERROR;
  *bits = v ? AGIMP_ERR_WAIT : 0u;
  return v ? AGIMP_DEVICE_TIMEOUT : AGIMP_OK;
}

}  // extern "C"

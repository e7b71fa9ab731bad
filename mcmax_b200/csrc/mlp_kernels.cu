/*
 * mlp_kernels.cu -- the opacity-surrogate network on sm_100a tensor cores.
 *
 * Network: 6 normalised inputs (log10 a, log10 lambda, n, log10 k,
 * porosity, fmax) -> 4 hidden layers of 256 SiLU units -> 64 outputs
 * (standardised log10 kappa_abs, log10 kappa_sca and Legendre moments of
 * F11, F12, F33 and F34; the targets are described at moments_kernel in
 * part_kernels.cu).  No counterpart in the reference: it
 * replaces calls of ComputePart's DHS inner loop (ComputePart.f:318-447)
 * inside its training box.
 *
 * Kernels (one tile = 128 samples):
 *   mlp_fwd_kernel     forward pass, two tiles in flight per CTA with warps
 *                      split into epilogue, MMA-issue and weight-copy roles.
 *                      Layer 0 (6 -> 256) on CUDA cores; layers 1-3
 *                      (256 -> 256) and the output layer (256 -> 64) as
 *                      tcgen05 BF16 MMAs with FP32 accumulators in tensor
 *                      memory; bias + SiLU epilogue from tensor memory back
 *                      into the shared A operand.  Optionally keeps
 *                      pre-activations (FP32) and activations (BF16) for
 *                      the backward pass.
 *   (the backward kernels use one warpgroup of 128 threads per CTA)
 *   mlp_dx_kernel      dZ_{l-1} = (dZ_l W_l) * SiLU'(Z_{l-1}), tcgen05 with
 *                      the transposed weights.
 *   mlp_dw_kernel      dW_l += dZ_l^T H_{l-1} over the batch, tcgen05 with
 *                      both operands transposed while staging; the 256-row
 *                      result is two M = 128 accumulators (512 TMEM columns).
 *   mlp_out_back_kernel, mlp_in_back_kernel, mlp_colsum_kernel
 *                      the thin layers and bias sums on CUDA cores.
 *   mlp_adam_kernel, mlp_pack_kernel
 *                      Adam on FP32 master weights; BF16 K-major copies of
 *                      W and W^T for the tensor cores.
 *   mlp_gemm_check_kernel
 *                      one 128 x N x 256 product, for the descriptor test.
 * Every mbarrier wait is bounded; a timeout sets *err and the CTA frees its
 * tensor memory and returns.
 */
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "tc_sm100.cuh"

namespace mlp {

constexpr int IN = 6, H = 256, OUT = 64, TILE = 128, NT = 128;
constexpr uint32_t A_BYTES = TILE * H * 2;   /* 64 KB activation tile */
constexpr uint32_t B_BYTES = H * H * 2;      /* 128 KB weight tile */

struct Params {
  const float *W0, *b0;          /* 256 x 6, 256 */
  const float *b123;             /* 3 x 256 */
  const float *b4;               /* OUT */
  const __nv_bfloat16 *Wc;       /* 3 x 4 chunks of 64 inputs, (out rows, in cols) */
  const __nv_bfloat16 *Wtc;      /* 3 x K-major (in rows, out cols) */
  const __nv_bfloat16 *W4c;      /* 4 chunks of 64 inputs, OUT rows */
};

__device__ __forceinline__ float dsilu(float z) {
  const float s = 1.0f / (1.0f + __expf(-z));
  return s * (1.0f + z * (1.0f - s));
}

__device__ __forceinline__ uint32_t pack2(float a, float b) {
  __nv_bfloat162 v = __floats2bfloat162_rn(a, b);
  return *reinterpret_cast<uint32_t *>(&v);
}

/* copy `bytes` (multiple of 16*NT) from global to shared, 16 B per access,
 * eight loads in flight per thread */
__device__ __forceinline__ void copy16(unsigned char *dst, const unsigned char *src, uint32_t bytes) {
  const uint4 *s = reinterpret_cast<const uint4 *>(src);
  uint4 *d = reinterpret_cast<uint4 *>(dst);
#pragma unroll 8
  for (uint32_t i = threadIdx.x; i < bytes / 16; i += NT) d[i] = s[i];
}

/* a row of 256 values (8 at a time) into the K-major A tile */
__device__ __forceinline__ void store_row8(unsigned char *A, int r, int k0, const float *v) {
  uint4 q;
  q.x = pack2(v[0], v[1]);
  q.y = pack2(v[2], v[3]);
  q.z = pack2(v[4], v[5]);
  q.w = pack2(v[6], v[7]);
  *reinterpret_cast<uint4 *>(A + tc_kmaj_off(r, k0, H)) = q;
}

struct Tc {
  uint32_t tmem;
  uint32_t phase;
};

/* issue one GEMM from the CTA's A and B tiles and wait for it; returns 0
 * when the wait timed out (uniform over the CTA) */
__device__ __forceinline__ int run_gemm(Tc &tc, uint64_t *mbar, uint32_t a0, uint32_t b0, int N, int K) {
  tc_fence_async_smem();
  __syncthreads();
  tc_fence_after();
  if (threadIdx.x == 0) {
    tc_gemm_issue(tc.tmem, a0, b0, TILE, N, K, 0);
    tc_commit(mbar);
  }
  const int ok = tc_mbar_wait(mbar, tc.phase);
  tc.phase ^= 1u;
  tc_fence_after();
  return __syncthreads_and(ok);
}

/* ------------------------------------------------------------------ forward */
/* SiLU z * sigmoid(z) with one special-function operation: u = 2^(-|z| log2 e)
 * by ex2.approx, then r = 1 / (1 + u) for 1 + u in (1, 2] by Newton-Raphson
 * from the linear minimax estimate 24/17 - 8/17 (1 + u), whose relative error
 * is at most 1/17; two steps bring it below 2e-5, far under the BF16 rounding
 * of the result.  sigmoid(z) = r for z >= 0 and u r for z < 0. */
__device__ __forceinline__ float silu_fast(float z) {
  float u;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(u) : "f"(-1.4426950408889634f * fabsf(z)));
  const float d = 1.0f + u;
  float r = fmaf(-0.47058823529411764f, d, 1.4117647058823529f);
  r = fmaf(r, fmaf(-d, r, 1.0f), r);
  r = fmaf(r, fmaf(-d, r, 1.0f), r);
  return z * (z >= 0.0f ? r : u * r);
}

/* Forward pass with two 128-row tiles (slots X = 0, Y = 1) in flight per CTA
 * and warps split by role:
 *   warps 0-15  epilogue: the input layer on CUDA cores, the bias + SiLU of
 *               each hidden layer from tensor memory into the slot's shared A
 *               operand, the output layer's bias into y.  The four warps of a
 *               TMEM lane quarter split the columns in four.
 *   warp 16     issues the MMAs (one lane);
 *   warp 17     streams the weights by bulk copy (one lane) through a ring of
 *               three 32 KB slots.
 * Weights are stored in chunks of 64 input columns (mlp_pack_kernel).  Each
 * chunk serves the same layer of both tiles: a layer's MMAs alternate X chunk
 * c, Y chunk c, so the weights cross L2 once per 256 rows.  While the tensor
 * cores run a layer of one tile, the epilogue warps work on the other.  When
 * there are no more tiles than CTAs, each CTA takes one tile (slot X only).
 * Barriers: full / empty per weight slot (copy landed / MMAs done reading it);
 * ready per tile slot (all 512 epilogue threads have written the A operand
 * and read the accumulator); done per tile slot (MMA commit: the accumulator
 * holds the layer).  Tensor memory: X accumulates in columns 0-255, Y in
 * 256-511.  Every wait is bounded and gives up once another role has; the
 * MMA and copy warps then wait (bounded) for their operations in flight
 * before the CTA frees tensor memory. */
constexpr int FW_EPI = 512, FW_NT = FW_EPI + 64, FW_SLOTS = 3, FW_KC = 64;
constexpr uint32_t FW_CHUNK = H * FW_KC * 2;    /* 32 KB: 256 output rows x 64 inputs */
constexpr uint32_t FW_CHUNK4 = OUT * FW_KC * 2; /* 8 KB: the output layer's chunk */
constexpr uint32_t FW_OFF_W = 2 * A_BYTES;      /* A_X | A_Y | weight slots | barriers */
constexpr uint32_t FW_OFF_BAR = FW_OFF_W + FW_SLOTS * FW_CHUNK;
constexpr uint32_t FW_NBAR = 2 * FW_SLOTS + 5;  /* full, empty, ready x2, done x2, drain */

/* the input layer of one tile into its A operand: this thread's row, its
 * quarter of the 256 units; KEEP also writes zs and hs */
template <bool KEEP>
__device__ __forceinline__ void fw_input_layer(const Params &P, const float *__restrict__ x, int n, int tile,
                                               int row, int c0, unsigned char *A, float *__restrict__ zs,
                                               __nv_bfloat16 *__restrict__ hs) {
  static_assert(IN == 6, "the vector loads below read six inputs per row");
  const int g = tile * TILE + row;
  const bool live = g < n;
  float xi[IN];
  {
    float2 a = make_float2(0.0f, 0.0f), b = a, c = a;
    if (live) {
      const float2 *xp = reinterpret_cast<const float2 *>(x + (size_t)g * IN); /* 8-byte aligned rows */
      a = __ldg(xp);
      b = __ldg(xp + 1);
      c = __ldg(xp + 2);
    }
    xi[0] = a.x, xi[1] = a.y, xi[2] = b.x, xi[3] = b.y, xi[4] = c.x, xi[5] = c.y;
  }
  for (int j0 = c0; j0 < c0 + H / 4; j0 += 8) {
    /* the 8 units' weights (48 floats) and biases, 16-byte aligned */
    float w[8 * IN], bj[8];
    const float4 *wp = reinterpret_cast<const float4 *>(P.W0 + j0 * IN);
#pragma unroll
    for (int k = 0; k < 2 * IN; ++k) {
      const float4 q = __ldg(wp + k);
      w[4 * k] = q.x, w[4 * k + 1] = q.y, w[4 * k + 2] = q.z, w[4 * k + 3] = q.w;
    }
    const float4 *bp = reinterpret_cast<const float4 *>(P.b0 + j0);
#pragma unroll
    for (int k = 0; k < 2; ++k) {
      const float4 q = __ldg(bp + k);
      bj[4 * k] = q.x, bj[4 * k + 1] = q.y, bj[4 * k + 2] = q.z, bj[4 * k + 3] = q.w;
    }
    float v[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      float z = bj[u];
#pragma unroll
      for (int i = 0; i < IN; ++i) z = fmaf(w[u * IN + i], xi[i], z);
      if (KEEP && live) zs[((size_t)g * 4 + 0) * H + j0 + u] = z;
      v[u] = silu_fast(z);
    }
    store_row8(A, row, j0, v);
    if (KEEP && live)
      *reinterpret_cast<uint4 *>(hs + ((size_t)g * 4 + 0) * H + j0) =
          *reinterpret_cast<const uint4 *>(A + tc_kmaj_off(row, j0, H));
  }
}

/* bias + SiLU of hidden layer l + 1 (the result of tensor-core product l,
 * l = 0..2) from the accumulator into the A operand */
template <bool KEEP>
__device__ __forceinline__ void fw_hidden(const Params &P, uint32_t acc, int l, int g, bool live, int row, int c0,
                                          unsigned char *A, float *__restrict__ zs, __nv_bfloat16 *__restrict__ hs) {
  for (int cc = c0; cc < c0 + H / 4; cc += 32) {
    float v[32];
    tc_ld32(acc + (uint32_t)cc, v);
    const float4 *bias = reinterpret_cast<const float4 *>(P.b123 + l * H + cc); /* 16-byte aligned */
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const float4 q = __ldg(bias + k);
      v[4 * k] += q.x, v[4 * k + 1] += q.y, v[4 * k + 2] += q.z, v[4 * k + 3] += q.w;
    }
#pragma unroll
    for (int u = 0; u < 32; ++u) {
      const float z = v[u];
      if (KEEP && live) zs[((size_t)g * 4 + l + 1) * H + cc + u] = z;
      v[u] = silu_fast(z);
    }
#pragma unroll
    for (int k = 0; k < 32; k += 8) {
      store_row8(A, row, cc + k, v + k);
      if (KEEP && live)
        *reinterpret_cast<uint4 *>(hs + ((size_t)g * 4 + l + 1) * H + cc + k) =
            *reinterpret_cast<const uint4 *>(A + tc_kmaj_off(row, cc + k, H));
    }
  }
}

/* KEEP: also write the pre-activations zs and activations hs (training) */
template <bool KEEP>
__global__ void __launch_bounds__(FW_NT, 1)
    mlp_fwd_kernel(Params P, const float *__restrict__ x, int n, float *__restrict__ y, float *__restrict__ zs,
                   __nv_bfloat16 *__restrict__ hs, int *err) {
  extern __shared__ __align__(1024) unsigned char smem[];
  uint64_t *bar = reinterpret_cast<uint64_t *>(smem + FW_OFF_BAR);
  uint64_t *full = bar, *empty = bar + FW_SLOTS, *ready = bar + 2 * FW_SLOTS, *done = ready + 2, *drain = done + 2;
  uint32_t *slot = reinterpret_cast<uint32_t *>(bar + FW_NBAR);
  volatile int *abort_flag = reinterpret_cast<volatile int *>(slot + 1);
  const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
  if (t == 0) {
    for (int i = 0; i < FW_SLOTS; ++i) {
      tc_mbar_init(full + i, 1);
      tc_mbar_init(empty + i, 1);
    }
    for (int s = 0; s < 2; ++s) {
      tc_mbar_init(ready + s, FW_EPI);
      tc_mbar_init(done + s, 1);
    }
    tc_mbar_init(drain, 1);
    *abort_flag = 0;
  }
  if (warp == 0) tc_alloc(slot, 512);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *slot;
  /* tiles per step: two (X, Y) while there are more tiles than CTAs, else
   * one (X); step p holds tiles per * p + s */
  const int ntiles = (n + TILE - 1) / TILE, per = ntiles <= (int)gridDim.x ? 1 : 2;
  const int nsteps = (ntiles + per - 1) / per, stride = (int)gridDim.x;
  int ok = 1;
  if (warp < FW_EPI / 32) {
    /* epilogue warps: thread = TMEM lane (row) x quarter of the columns */
    const int row = t & (TILE - 1), c0 = (t >> 7) * (H / 4);
    const uint32_t lanes = (uint32_t)((warp & 3) * 32) << 16;
    uint32_t dphase = 0u; /* bit s: parity of slot s's next done phase */
    int p = blockIdx.x;
    if (p < nsteps) {
      for (int s = 0; s < per; ++s) {
        fw_input_layer<KEEP>(P, x, n, per * p + s, row, c0, smem + s * A_BYTES, zs, hs);
        tc_fence_async_smem();
        tc_mbar_arrive(ready + s);
      }
    }
    for (; p < nsteps && ok; p += stride) {
      for (int L = 0; L < 4 && ok; ++L) {
        for (int s = 0; s < per; ++s) {
          ok = __all_sync(0xffffffffu, tc_mbar_wait_or_abort(done + s, (dphase >> s) & 1u, abort_flag));
          dphase ^= 1u << s;
          if (!ok) break;
          tc_fence_after();
          const uint32_t acc = tmem + lanes + 256u * (uint32_t)s;
          unsigned char *A = smem + s * A_BYTES;
          const int g = (per * p + s) * TILE + row;
          const bool live = g < n;
          if (L < 3) {
            fw_hidden<KEEP>(P, acc, L, g, live, row, c0, A, zs, hs);
          } else {
            /* output layer: 64 columns, 16 per column quarter */
            const int c = (t >> 7) * 16;
            float v[16];
            tc_ld16(acc + (uint32_t)c, v);
            if (live) {
              const float4 *bias = reinterpret_cast<const float4 *>(P.b4 + c);
              float4 *yo = reinterpret_cast<float4 *>(y + (size_t)g * OUT + c);
#pragma unroll
              for (int k = 0; k < 4; ++k) {
                const float4 q = __ldg(bias + k);
                yo[k] = make_float4(v[4 * k] + q.x, v[4 * k + 1] + q.y, v[4 * k + 2] + q.z, v[4 * k + 3] + q.w);
              }
            }
            if (p + stride >= nsteps) continue; /* no further product on this slot */
            /* the slot's A operand is free: the next step's input layer */
            fw_input_layer<KEEP>(P, x, n, per * (p + stride) + s, row, c0, A, zs, hs);
          }
          tc_fence_async_smem();
          tc_fence_before();
          tc_mbar_arrive(ready + s);
        }
      }
    }
  } else if (warp == FW_EPI / 32) {
    /* MMA warp: per step, layers L = 0..3 (three hidden products and the
     * output), per layer four weight chunks, each for X then Y */
    uint32_t rphase = 0u; /* bit s: parity of slot s's next ready phase */
    int q = 0;
    for (int p = blockIdx.x; p < nsteps && ok; p += stride) {
      for (int L = 0; L < 4 && ok; ++L) {
        const uint32_t idesc = tc_idesc_bf16(TILE, L < 3 ? H : OUT);
        for (int c = 0; c < 4 && ok; ++c, ++q) {
          const int ws = q % FW_SLOTS;
          ok = __all_sync(0xffffffffu,
                          tc_mbar_wait_or_abort(full + ws, (uint32_t)(q / FW_SLOTS) & 1u, abort_flag));
          if (!ok) break;
          const uint32_t b = tc_smem_addr(smem + FW_OFF_W + ws * FW_CHUNK);
          for (int s = 0; s < per; ++s) {
            if (c == 0) {
              ok = __all_sync(0xffffffffu, tc_mbar_wait_or_abort(ready + s, (rphase >> s) & 1u, abort_flag));
              rphase ^= 1u << s;
              if (!ok) break;
            }
            tc_fence_after();
            if (lane == 0) {
              const uint32_t a = tc_smem_addr(smem + s * A_BYTES);
#pragma unroll
              for (int j = 0; j < FW_KC / 16; ++j) {
                const uint64_t ad = tc_desc(a + 256u * (uint32_t)(4 * c + j), 128u, (uint32_t)H * 16u);
                const uint64_t bd = tc_desc(b + 256u * (uint32_t)j, 128u, (uint32_t)FW_KC * 16u);
                tc_mma(tmem + 256u * (uint32_t)s, ad, bd, idesc, (c > 0 || j > 0) ? 1u : 0u);
              }
              if (c == 3) tc_commit(done + s);
            }
            __syncwarp();
          }
          if (!ok) break;
          if (lane == 0) tc_commit(empty + ws);
          __syncwarp();
        }
      }
    }
    /* every MMA issued here completes before tensor memory is freed */
    if (lane == 0) tc_commit(drain);
    __syncwarp();
    (void)tc_mbar_wait(drain, 0u);
  } else {
    /* weight stream: 16 chunks per step, chunk q = (layer (q / 4) % 4,
     * columns 64 (q % 4) ..), slot q % 3 */
    const int mine = (int)blockIdx.x < nsteps ? (nsteps - 1 - (int)blockIdx.x) / stride + 1 : 0;
    int issued = 0; /* chunk q goes to slot q % 3 as its (q / 3)-th fill */
    for (int q = 0; q < 16 * mine && ok; ++q) {
      const int ws = q % FW_SLOTS, u = q / FW_SLOTS;
      if (u > 0) {
        ok = __all_sync(0xffffffffu, tc_mbar_wait_or_abort(empty + ws, (uint32_t)(u - 1) & 1u, abort_flag));
        if (!ok) break;
      }
      const int L = (q >> 2) & 3, c = q & 3;
      const unsigned char *src = L < 3 ? reinterpret_cast<const unsigned char *>(P.Wc) + (size_t)(L * 4 + c) * FW_CHUNK
                                       : reinterpret_cast<const unsigned char *>(P.W4c) + (size_t)c * FW_CHUNK4;
      if (lane == 0) tc_bulk_load(smem + FW_OFF_W + ws * FW_CHUNK, src, L < 3 ? FW_CHUNK : FW_CHUNK4, full + ws);
      __syncwarp();
      issued = q + 1;
    }
    /* every copy issued here lands before the CTA leaves: the last fill of
     * each slot */
    for (int ws = 0; ws < FW_SLOTS && ws < issued; ++ws) {
      const int last = ws + FW_SLOTS * ((issued - 1 - ws) / FW_SLOTS);
      (void)tc_mbar_wait(full + ws, (uint32_t)(last / FW_SLOTS) & 1u);
    }
  }
  if (!ok) {
    *abort_flag = 1;
    if (lane == 0) atomicExch(err, 1);
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0) tc_dealloc(tmem, 512);
}

/* ---------------------------------------------------------------- backward */
/* dZprev = (dZ W) * SiLU'(Zprev): A = dZ tile (from global), B = W^T */
__global__ void __launch_bounds__(NT, 1)
    mlp_dx_kernel(const __nv_bfloat16 *__restrict__ Wtc_l, const __nv_bfloat16 *__restrict__ dz, int n,
                  const float *__restrict__ zs, int lprev, __nv_bfloat16 *__restrict__ dzprev, int *err) {
  extern __shared__ __align__(1024) unsigned char smem[];
  unsigned char *A = smem;
  unsigned char *B = smem + A_BYTES;
  uint64_t *mbar = reinterpret_cast<uint64_t *>(B + B_BYTES);
  uint32_t *slot = reinterpret_cast<uint32_t *>(mbar + 1);
  const int t = threadIdx.x, warp = t >> 5;
  if (t == 0) tc_mbar_init(mbar, 1);
  if (warp == 0) tc_alloc(slot, 256);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  Tc tc{*slot, 0u};
  const uint32_t lane_base = tc.tmem + ((uint32_t)(warp * 32) << 16);
  const uint32_t a0 = tc_smem_addr(A), b0 = tc_smem_addr(B);
  copy16(B, reinterpret_cast<const unsigned char *>(Wtc_l), B_BYTES);
  const int ntiles = (n + TILE - 1) / TILE;
  int ok = 1;
  for (int tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
    const int g = tile * TILE + t;
    const bool live = g < n;
    __syncthreads();
#pragma unroll 8
    for (int k0 = 0; k0 < H; k0 += 8) {
      uint4 q = make_uint4(0, 0, 0, 0);
      if (live) q = *reinterpret_cast<const uint4 *>(dz + (size_t)g * H + k0);
      *reinterpret_cast<uint4 *>(A + tc_kmaj_off(t, k0, H)) = q;
    }
    ok = run_gemm(tc, mbar, a0, b0, H, H);
    if (!ok) break;
    for (int c = 0; c < H; c += 16) {
      float v[16];
      tc_ld16(lane_base + (uint32_t)c, v);
      if (live) {
        uint32_t w[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
          const float z0 = zs[((size_t)g * 4 + lprev) * H + c + 2 * u];
          const float z1 = zs[((size_t)g * 4 + lprev) * H + c + 2 * u + 1];
          w[u] = pack2(v[2 * u] * dsilu(z0), v[2 * u + 1] * dsilu(z1));
        }
        uint4 *d = reinterpret_cast<uint4 *>(dzprev + (size_t)g * H + c);
        d[0] = make_uint4(w[0], w[1], w[2], w[3]);
        d[1] = make_uint4(w[4], w[5], w[6], w[7]);
      }
    }
    tc_fence_before();
  }
  if (!ok && t == 0) atomicExch(err, 1);
  if (!ok) (void)tc_mbar_wait(mbar, tc.phase ^ 1u);
  __syncthreads();
  tc_fence_after();
  if (warp == 0) tc_dealloc(tc.tmem, 256);
}

/* dW += dZ^T Hprev over the batch: M = 256 output rows (two 128-row halves),
 * N = 256 inputs, K = samples in chunks of 128 */
__global__ void __launch_bounds__(NT, 1)
    mlp_dw_kernel(const __nv_bfloat16 *__restrict__ dz, const __nv_bfloat16 *__restrict__ hs, int lprev, int n,
                  float *__restrict__ dW, int *err) {
  extern __shared__ __align__(1024) unsigned char smem[];
  constexpr int KC = 128;
  unsigned char *A0 = smem;                 /* dZ^T rows 0..127: 128 x 128 */
  unsigned char *A1 = smem + 128 * KC * 2;  /* rows 128..255 */
  unsigned char *B = smem + 2 * 128 * KC * 2; /* Hprev^T: 256 x 128 */
  uint64_t *mbar = reinterpret_cast<uint64_t *>(B + 256 * KC * 2);
  uint32_t *slot = reinterpret_cast<uint32_t *>(mbar + 1);
  const int t = threadIdx.x, warp = t >> 5;
  if (t == 0) tc_mbar_init(mbar, 1);
  if (warp == 0) tc_alloc(slot, 512);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  Tc tc{*slot, 0u};
  const uint32_t a0 = tc_smem_addr(A0), a1 = tc_smem_addr(A1), b0 = tc_smem_addr(B);
  const int nchunks = (n + KC - 1) / KC;
  int ok = 1, first = 1;
  for (int ch = blockIdx.x; ch < nchunks && ok; ch += gridDim.x) {
    __syncthreads();
    /* transposed staging: element (row = feature, k = sample) */
    for (int s0 = 0; s0 < KC; s0 += 8) {
      float d0[8], d1[8], h0[8], h1[8];
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const int g = ch * KC + s0 + i;
        const bool live = g < n;
        d0[i] = live ? __bfloat162float(dz[(size_t)g * H + t]) : 0.0f;
        d1[i] = live ? __bfloat162float(dz[(size_t)g * H + 128 + t]) : 0.0f;
        h0[i] = live ? __bfloat162float(hs[((size_t)g * 4 + lprev) * H + t]) : 0.0f;
        h1[i] = live ? __bfloat162float(hs[((size_t)g * 4 + lprev) * H + 128 + t]) : 0.0f;
      }
      *reinterpret_cast<uint4 *>(A0 + tc_kmaj_off(t, s0, KC)) =
          make_uint4(pack2(d0[0], d0[1]), pack2(d0[2], d0[3]), pack2(d0[4], d0[5]), pack2(d0[6], d0[7]));
      *reinterpret_cast<uint4 *>(A1 + tc_kmaj_off(t, s0, KC)) =
          make_uint4(pack2(d1[0], d1[1]), pack2(d1[2], d1[3]), pack2(d1[4], d1[5]), pack2(d1[6], d1[7]));
      *reinterpret_cast<uint4 *>(B + tc_kmaj_off(t, s0, KC)) =
          make_uint4(pack2(h0[0], h0[1]), pack2(h0[2], h0[3]), pack2(h0[4], h0[5]), pack2(h0[6], h0[7]));
      *reinterpret_cast<uint4 *>(B + tc_kmaj_off(128 + t, s0, KC)) =
          make_uint4(pack2(h1[0], h1[1]), pack2(h1[2], h1[3]), pack2(h1[4], h1[5]), pack2(h1[6], h1[7]));
    }
    tc_fence_async_smem();
    __syncthreads();
    tc_fence_after();
    if (t == 0) {
      tc_gemm_issue(tc.tmem, a0, b0, TILE, H, KC, !first);
      tc_gemm_issue(tc.tmem + 256u, a1, b0, TILE, H, KC, !first);
      tc_commit(mbar);
    }
    const int w = tc_mbar_wait(mbar, tc.phase);
    tc.phase ^= 1u;
    tc_fence_after();
    ok = __syncthreads_and(w);
    first = 0;
  }
  if (ok && !first) {
    const uint32_t lane_base = tc.tmem + ((uint32_t)(warp * 32) << 16);
    for (int half = 0; half < 2; ++half)
      for (int c = 0; c < H; c += 16) {
        float v[16];
        tc_ld16(lane_base + (uint32_t)(half * 256 + c), v);
        float *row = dW + (size_t)(half * 128 + t) * H + c;
#pragma unroll
        for (int u = 0; u < 16; ++u) atomicAdd(row + u, v[u]);
      }
  }
  if (!ok && t == 0) atomicExch(err, 1);
  if (!ok) (void)tc_mbar_wait(mbar, tc.phase ^ 1u);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0) tc_dealloc(tc.tmem, 512);
}

/* loss = sum_o w_o (y - t)^2 / n; dY = 2 w_o (y - t) / n */
__global__ void mlp_loss_kernel(const float *__restrict__ y, const float *__restrict__ tgt,
                                const float *__restrict__ w, int n, float *__restrict__ dy, double *loss) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  float l = 0.0f;
  if (i < (long long)n * OUT) {
    const int o = (int)(i % OUT);
    const float d = y[i] - tgt[i];
    dy[i] = 2.0f * w[o] * d / (float)n;
    l = w[o] * d * d;
  }
  for (int s = 16; s > 0; s >>= 1) l += __shfl_down_sync(0xffffffffu, l, s);
  if ((threadIdx.x & 31) == 0 && l != 0.0f) atomicAdd(loss, (double)l / (double)n);
}

/* output layer backward on CUDA cores: dW4 += dY^T H3, db4 += sum dY,
 * dZ3 = (dY W4) * SiLU'(Z3); one block of 256 threads per 128 samples */
__global__ void __launch_bounds__(256)
    mlp_out_back_kernel(const float *__restrict__ W4, const float *__restrict__ dy, const float *__restrict__ zs,
                        const __nv_bfloat16 *__restrict__ hs, int n, float *__restrict__ dW4,
                        float *__restrict__ db4, __nv_bfloat16 *__restrict__ dz3) {
  __shared__ float sdy[TILE * OUT];
  const int k = threadIdx.x; /* hidden unit */
  float w4[OUT], acc[OUT];
#pragma unroll
  for (int o = 0; o < OUT; ++o) {
    w4[o] = W4[o * H + k];
    acc[o] = 0.0f;
  }
  for (int tile = blockIdx.x; tile * TILE < n; tile += gridDim.x) {
    __syncthreads();
    for (int i = k; i < TILE * OUT; i += 256) {
      const int g = tile * TILE + i / OUT;
      sdy[i] = g < n ? dy[(size_t)g * OUT + (i % OUT)] : 0.0f;
    }
    __syncthreads();
    for (int s = 0; s < TILE; ++s) {
      const int g = tile * TILE + s;
      if (g >= n) break;
      const float h = __bfloat162float(hs[((size_t)g * 4 + 3) * H + k]);
      float dh = 0.0f;
#pragma unroll
      for (int o = 0; o < OUT; ++o) {
        const float d = sdy[s * OUT + o];
        dh = fmaf(d, w4[o], dh);
        acc[o] = fmaf(d, h, acc[o]);
      }
      dz3[(size_t)g * H + k] = __float2bfloat16_rn(dh * dsilu(zs[((size_t)g * 4 + 3) * H + k]));
    }
  }
#pragma unroll
  for (int o = 0; o < OUT; ++o) atomicAdd(&dW4[o * H + k], acc[o]);
  if (k < OUT) {
    float s = 0.0f;
    for (int g = blockIdx.x * TILE; g < n; g += gridDim.x * TILE)
      for (int u = 0; u < TILE && g + u < n; ++u) s += dy[(size_t)(g + u) * OUT + k];
    atomicAdd(&db4[k], s);
  }
}

/* input layer backward: dW0 += dZ0^T X, db0 += sum dZ0 (one thread per unit) */
__global__ void __launch_bounds__(256)
    mlp_in_back_kernel(const __nv_bfloat16 *__restrict__ dz0, const float *__restrict__ x, int n,
                       float *__restrict__ dW0, float *__restrict__ db0) {
  const int j = threadIdx.x;
  float acc[IN + 1];
#pragma unroll
  for (int i = 0; i <= IN; ++i) acc[i] = 0.0f;
  for (int g = blockIdx.x; g < n; g += gridDim.x) {
    const float d = __bfloat162float(dz0[(size_t)g * H + j]);
#pragma unroll
    for (int i = 0; i < IN; ++i) acc[i] = fmaf(d, x[(size_t)g * IN + i], acc[i]);
    acc[IN] += d;
  }
#pragma unroll
  for (int i = 0; i < IN; ++i) atomicAdd(&dW0[j * IN + i], acc[i]);
  atomicAdd(&db0[j], acc[IN]);
}

/* db += column sums of dZ (n x 256, bf16) */
__global__ void __launch_bounds__(256)
    mlp_colsum_kernel(const __nv_bfloat16 *__restrict__ dz, int n, float *__restrict__ db) {
  const int j = threadIdx.x;
  float s = 0.0f;
  for (int g = blockIdx.x; g < n; g += gridDim.x) s += __bfloat162float(dz[(size_t)g * H + j]);
  atomicAdd(&db[j], s);
}

/* Adam step on the flat parameter vector */
__global__ void mlp_adam_kernel(float *__restrict__ p, const float *__restrict__ gr, float *__restrict__ m,
                                float *__restrict__ v, int np, float lr, float b1, float b2, float eps, float c1,
                                float c2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= np) return;
  const float g = gr[i];
  const float mi = b1 * m[i] + (1.0f - b1) * g;
  const float vi = b2 * v[i] + (1.0f - b2) * g * g;
  m[i] = mi;
  v[i] = vi;
  p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

/* BF16 K-major copies of the tensor-core weights from the FP32 masters:
 * Wc[l] (out rows, in cols) and W4c (OUT x 256) for the forward pass, in
 * chunks of 64 input columns, each chunk a K-major tile of its own (chunk
 * (l, c) at (4 l + c) x 32 KB); Wtc[l] (in rows, out cols), one 256-column
 * K-major tile per layer, for the backward pass */
__global__ void mlp_pack_kernel(const float *__restrict__ W123, const float *__restrict__ W4,
                                __nv_bfloat16 *__restrict__ Wc, __nv_bfloat16 *__restrict__ Wtc,
                                __nv_bfloat16 *__restrict__ W4c) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < 3 * H * H) {
    const int l = i / (H * H), r = (i / H) % H, c = i % H; /* W[l][r = out][c = in] */
    const __nv_bfloat16 v = __float2bfloat16_rn(W123[i]);
    unsigned char *wc = reinterpret_cast<unsigned char *>(Wc) + (size_t)(l * 4 + c / FW_KC) * FW_CHUNK;
    unsigned char *wt = reinterpret_cast<unsigned char *>(Wtc + (size_t)l * H * H);
    *reinterpret_cast<__nv_bfloat16 *>(wc + tc_kmaj_off(r, c % FW_KC, FW_KC)) = v;
    *reinterpret_cast<__nv_bfloat16 *>(wt + tc_kmaj_off(c, r, H)) = v;
  } else if (i < 3 * H * H + OUT * H) {
    const int j = i - 3 * H * H, r = j / H, c = j % H;
    unsigned char *w4 = reinterpret_cast<unsigned char *>(W4c) + (size_t)(c / FW_KC) * FW_CHUNK4;
    *reinterpret_cast<__nv_bfloat16 *>(w4 + tc_kmaj_off(r, c % FW_KC, FW_KC)) = __float2bfloat16_rn(W4[j]);
  }
}

/* one 128 x N x 256 product D = A B^T from row-major BF16 inputs */
__global__ void __launch_bounds__(NT, 1)
    mlp_gemm_check_kernel(const __nv_bfloat16 *__restrict__ Ain, const __nv_bfloat16 *__restrict__ Bin, int N,
                          float *__restrict__ D, int *err) {
  extern __shared__ __align__(1024) unsigned char smem[];
  unsigned char *A = smem;
  unsigned char *B = smem + A_BYTES;
  uint64_t *mbar = reinterpret_cast<uint64_t *>(B + B_BYTES);
  uint32_t *slot = reinterpret_cast<uint32_t *>(mbar + 1);
  const int t = threadIdx.x, warp = t >> 5;
  if (t == 0) tc_mbar_init(mbar, 1);
  if (warp == 0) tc_alloc(slot, 256);
  for (int k0 = 0; k0 < H; k0 += 8)
    *reinterpret_cast<uint4 *>(A + tc_kmaj_off(t, k0, H)) =
        *reinterpret_cast<const uint4 *>(Ain + (size_t)t * H + k0);
  for (int r = t; r < N; r += NT)
    for (int k0 = 0; k0 < H; k0 += 8)
      *reinterpret_cast<uint4 *>(B + tc_kmaj_off(r, k0, H)) =
          *reinterpret_cast<const uint4 *>(Bin + (size_t)r * H + k0);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  Tc tc{*slot, 0u};
  const int ok = run_gemm(tc, mbar, tc_smem_addr(A), tc_smem_addr(B), N, H);
  if (ok) {
    const uint32_t lane_base = tc.tmem + ((uint32_t)(warp * 32) << 16);
    for (int c = 0; c < N; c += 16) {
      float v[16];
      tc_ld16(lane_base + (uint32_t)c, v);
#pragma unroll
      for (int u = 0; u < 16; ++u) D[(size_t)t * N + c + u] = v[u];
    }
  } else {
    if (t == 0) atomicExch(err, 1);
    (void)tc_mbar_wait(mbar, tc.phase ^ 1u);
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0) tc_dealloc(tc.tmem, 256);
}

}  // namespace mlp

/* ======================================================================
 * Host side: parameters, optimizer state and batch buffers of the network
 * on a context, and the extern "C" entry points (include/mcmax_gpu.h).
 * ==================================================================== */
#include <algorithm>
#include <chrono>
#include <cstring>
#include <random>
#include <vector>

#include "mcg_internal.h"
#include "surrogate_phase.h"

namespace {

using namespace mlp;

constexpr int64_t OFF_W0 = 0, OFF_B0 = OFF_W0 + H * IN, OFF_W123 = OFF_B0 + H, OFF_B123 = OFF_W123 + 3 * H * H,
                  OFF_W4 = OFF_B123 + 3 * H, OFF_B4 = OFF_W4 + OUT * H, NPARAMS = OFF_B4 + OUT;
static_assert(NPARAMS == MCG_MLP_NPARAMS, "parameter count");

constexpr size_t SMEM_FWD = FW_OFF_BAR + FW_NBAR * 8 + 8;
constexpr size_t SMEM_DX = A_BYTES + B_BYTES + 16;
constexpr size_t SMEM_DW = 4 * 128 * 128 * 2 + 16;
constexpr size_t SMEM_CHECK = A_BYTES + B_BYTES + 16;

inline int nblk(long long n, int b) { return (int)((n + b - 1) / b); }

}  // namespace

struct MlpState {
  float *P = nullptr, *G = nullptr, *M = nullptr, *V = nullptr;
  __nv_bfloat16 *Wc = nullptr, *Wtc = nullptr, *W4c = nullptr;
  int *err = nullptr;
  double *loss = nullptr;
  float *wout = nullptr;
  int64_t cap = 0; /* batch rows the buffers hold */
  float *xb = nullptr, *tb = nullptr, *yb = nullptr, *dy = nullptr, *zs = nullptr;
  __nv_bfloat16 *hs = nullptr, *dza = nullptr, *dzb = nullptr;
  bool have_params = false;
  int64_t step = 0;
  std::vector<void *> own;
};

namespace {

template <typename T>
cudaError_t dalloc(MlpState &s, T **p, size_t n) {
  cudaError_t e = cudaMalloc((void **)p, std::max<size_t>(n, 1) * sizeof(T));
  if (e == cudaSuccess) s.own.push_back(*p);
  return e;
}

mcg_status mlp_init(mcg_ctx *ctx) {
  if (ctx->mlp) return MCG_OK;
  MlpState *s = new MlpState();
  ctx->mlp = s;
  cudaError_t e = cudaSuccess;
  if (e == cudaSuccess) e = dalloc(*s, &s->P, NPARAMS);
  if (e == cudaSuccess) e = dalloc(*s, &s->G, NPARAMS);
  if (e == cudaSuccess) e = dalloc(*s, &s->M, NPARAMS);
  if (e == cudaSuccess) e = dalloc(*s, &s->V, NPARAMS);
  if (e == cudaSuccess) e = dalloc(*s, &s->Wc, 3 * H * H);
  if (e == cudaSuccess) e = dalloc(*s, &s->Wtc, 3 * H * H);
  if (e == cudaSuccess) e = dalloc(*s, &s->W4c, OUT * H);
  if (e == cudaSuccess) e = dalloc(*s, &s->err, 1);
  if (e == cudaSuccess) e = dalloc(*s, &s->loss, 1);
  if (e == cudaSuccess) e = dalloc(*s, &s->wout, OUT);
  if (e != cudaSuccess) return mcg_fail(ctx, MCG_ERR_NOMEM, "mlp: cudaMalloc failed: %s", cudaGetErrorString(e));
  MCG_CUDA(ctx, cudaFuncSetAttribute(mlp_fwd_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)SMEM_FWD));
  MCG_CUDA(ctx, cudaFuncSetAttribute(mlp_fwd_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)SMEM_FWD));
  MCG_CUDA(ctx, cudaFuncSetAttribute(mlp_dx_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM_DX));
  MCG_CUDA(ctx, cudaFuncSetAttribute(mlp_dw_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM_DW));
  MCG_CUDA(ctx, cudaFuncSetAttribute(mlp_gemm_check_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)SMEM_CHECK));
  return MCG_OK;
}

mcg_status mlp_reserve(mcg_ctx *ctx, int64_t rows) {
  MlpState &s = *ctx->mlp;
  if (rows <= s.cap) return MCG_OK;
  void *old[] = {s.xb, s.tb, s.yb, s.dy, s.zs, s.hs, s.dza, s.dzb};
  for (void *p : old)
    if (p) {
      cudaFree(p);
      s.own.erase(std::remove(s.own.begin(), s.own.end(), p), s.own.end());
    }
  cudaError_t e = cudaSuccess;
  if (e == cudaSuccess) e = dalloc(s, &s.xb, (size_t)rows * IN);
  if (e == cudaSuccess) e = dalloc(s, &s.tb, (size_t)rows * OUT);
  if (e == cudaSuccess) e = dalloc(s, &s.yb, (size_t)rows * OUT);
  if (e == cudaSuccess) e = dalloc(s, &s.dy, (size_t)rows * OUT);
  if (e == cudaSuccess) e = dalloc(s, &s.zs, (size_t)rows * 4 * H);
  if (e == cudaSuccess) e = dalloc(s, &s.hs, (size_t)rows * 4 * H);
  if (e == cudaSuccess) e = dalloc(s, &s.dza, (size_t)rows * H);
  if (e == cudaSuccess) e = dalloc(s, &s.dzb, (size_t)rows * H);
  if (e != cudaSuccess) {
    s.cap = 0;
    s.xb = s.tb = s.yb = s.dy = s.zs = nullptr;
    s.hs = s.dza = s.dzb = nullptr;
    return mcg_fail(ctx, MCG_ERR_NOMEM, "mlp: batch buffers of %lld rows: %s", (long long)rows,
                    cudaGetErrorString(e));
  }
  s.cap = rows;
  return MCG_OK;
}

Params mlp_params(const MlpState &s) {
  Params p;
  p.W0 = s.P + OFF_W0;
  p.b0 = s.P + OFF_B0;
  p.b123 = s.P + OFF_B123;
  p.b4 = s.P + OFF_B4;
  p.Wc = s.Wc;
  p.Wtc = s.Wtc;
  p.W4c = s.W4c;
  return p;
}

void mlp_pack(mcg_ctx *ctx) {
  MlpState &s = *ctx->mlp;
  const int n = 3 * H * H + OUT * H;
  mlp_pack_kernel<<<nblk(n, 256), 256, 0, ctx->stream>>>(s.P + OFF_W123, s.P + OFF_W4, s.Wc, s.Wtc, s.W4c);
}

int grid_tiles(mcg_ctx *ctx, int64_t n) {
  const int tiles = (int)((n + TILE - 1) / TILE);
  return std::max(1, std::min(tiles, ctx->sm_count > 0 ? ctx->sm_count : 148));
}

/* the forward kernel: one tile per CTA while the tiles fit on the SMs, else
 * pairs of tiles (the kernel takes two per step when tiles > CTAs) */
int grid_fwd(mcg_ctx *ctx, int64_t n) {
  const int sms = ctx->sm_count > 0 ? ctx->sm_count : 148;
  const int tiles = (int)((n + TILE - 1) / TILE);
  if (tiles <= sms) return std::max(1, tiles);
  return std::min((tiles + 1) / 2, sms);
}

/* forward of rows already in s.xb; zs/hs kept when `keep` */
void mlp_fwd_launch(mcg_ctx *ctx, int64_t n, bool keep) {
  MlpState &s = *ctx->mlp;
  if (keep)
    mlp_fwd_kernel<true><<<grid_fwd(ctx, n), FW_NT, SMEM_FWD, ctx->stream>>>(mlp_params(s), s.xb, (int)n, s.yb,
                                                                             s.zs, s.hs, s.err);
  else
    mlp_fwd_kernel<false><<<grid_fwd(ctx, n), FW_NT, SMEM_FWD, ctx->stream>>>(mlp_params(s), s.xb, (int)n, s.yb,
                                                                              nullptr, nullptr, s.err);
}

/* loss and gradient of the batch in s.xb / s.tb into s.G (zeroed here) */
void mlp_backward_launch(mcg_ctx *ctx, int64_t n) {
  MlpState &s = *ctx->mlp;
  cudaStream_t st = ctx->stream;
  const int sms = ctx->sm_count > 0 ? ctx->sm_count : 148;
  cudaMemsetAsync(s.G, 0, NPARAMS * sizeof(float), st);
  cudaMemsetAsync(s.loss, 0, sizeof(double), st);
  mlp_fwd_launch(ctx, n, true);
  mlp_loss_kernel<<<nblk(n * OUT, 256), 256, 0, st>>>(s.yb, s.tb, s.wout, (int)n, s.dy, s.loss);
  const int tiles = (int)((n + TILE - 1) / TILE);
  mlp_out_back_kernel<<<std::min(tiles, 4 * sms), 256, 0, st>>>(s.P + OFF_W4, s.dy, s.zs, s.hs, (int)n,
                                                                 s.G + OFF_W4, s.G + OFF_B4, s.dza);
  __nv_bfloat16 *dz = s.dza, *dzn = s.dzb;
  for (int l = 2; l >= 0; --l) {
    /* dz holds dZ of tensor-core layer l (input H_l, output Z_{l+1}) */
    mlp_dw_kernel<<<std::min(tiles, sms), NT, SMEM_DW, st>>>(dz, s.hs, l, (int)n, s.G + OFF_W123 + (size_t)l * H * H,
                                                            s.err);
    mlp_colsum_kernel<<<std::min((int)n, 2 * sms), 256, 0, st>>>(dz, (int)n, s.G + OFF_B123 + (size_t)l * H);
    mlp_dx_kernel<<<grid_tiles(ctx, n), NT, SMEM_DX, st>>>(s.Wtc + (size_t)l * H * H, dz, (int)n, s.zs, l, dzn,
                                                           s.err);
    std::swap(dz, dzn);
  }
  mlp_in_back_kernel<<<std::min((int)n, 2 * sms), 256, 0, st>>>(dz, s.xb, (int)n, s.G + OFF_W0, s.G + OFF_B0);
}

mcg_status mlp_check_err(mcg_ctx *ctx, const char *what) {
  int herr = 0;
  MCG_CUDA(ctx, cudaMemcpyAsync(&herr, ctx->mlp->err, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  MCG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  if (herr) return mcg_fail(ctx, MCG_ERR_RUN, "%s: a tensor-core wait timed out", what);
  return MCG_OK;
}

mcg_status mlp_ready(mcg_ctx *ctx, const char *what) {
  if (!ctx->mlp || !ctx->mlp->have_params)
    return mcg_fail(ctx, MCG_ERR_STATE, "%s: mcg_mlp_set_params has not been called", what);
  return MCG_OK;
}

__global__ void gather_rows_kernel(const float *__restrict__ X, const float *__restrict__ T,
                                   const int *__restrict__ idx, int n, float *__restrict__ xb,
                                   float *__restrict__ tb) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n * OUT) return;
  const int r = i / OUT, c = i % OUT;
  const int g = idx[r];
  tb[i] = T[(size_t)g * OUT + c];
  if (c < IN) xb[(size_t)r * IN + c] = X[(size_t)g * IN + c];
}

}  // namespace

void mcg_free_mlp(mcg_ctx *ctx) {
  if (!ctx->mlp) return;
  for (void *p : ctx->mlp->own) cudaFree(p);
  delete ctx->mlp;
  ctx->mlp = nullptr;
}

extern "C" {

mcg_status mcg_mlp_set_params(mcg_ctx *ctx, const float *params, int64_t nparams) {
  if (!ctx) return MCG_ERR_ARG;
  cudaSetDevice(ctx->device);
  if (!params || nparams != NPARAMS)
    return mcg_fail(ctx, MCG_ERR_ARG, "mlp_set_params: %lld parameters expected", (long long)NPARAMS);
  mcg_status st = mlp_init(ctx);
  if (st != MCG_OK) return st;
  MlpState &s = *ctx->mlp;
  MCG_CUDA(ctx, cudaMemcpyAsync(s.P, params, NPARAMS * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
  MCG_CUDA(ctx, cudaMemsetAsync(s.M, 0, NPARAMS * sizeof(float), ctx->stream));
  MCG_CUDA(ctx, cudaMemsetAsync(s.V, 0, NPARAMS * sizeof(float), ctx->stream));
  MCG_CUDA(ctx, cudaMemsetAsync(s.err, 0, sizeof(int), ctx->stream));
  mlp_pack(ctx);
  MCG_CUDA(ctx, cudaGetLastError());
  MCG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  s.have_params = true;
  s.step = 0;
  return MCG_OK;
}

mcg_status mcg_mlp_get_params(mcg_ctx *ctx, float *params, int64_t nparams) {
  if (!ctx) return MCG_ERR_ARG;
  cudaSetDevice(ctx->device);
  mcg_status st = mlp_ready(ctx, "mlp_get_params");
  if (st != MCG_OK) return st;
  if (!params || nparams != NPARAMS)
    return mcg_fail(ctx, MCG_ERR_ARG, "mlp_get_params: %lld parameters expected", (long long)NPARAMS);
  MCG_CUDA(ctx, cudaMemcpyAsync(params, ctx->mlp->P, NPARAMS * sizeof(float), cudaMemcpyDeviceToHost,
                                ctx->stream));
  MCG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return MCG_OK;
}

mcg_status mcg_mlp_forward(mcg_ctx *ctx, int64_t n, const float *x, float *y) {
  if (!ctx) return MCG_ERR_ARG;
  cudaSetDevice(ctx->device);
  mcg_status st = mlp_ready(ctx, "mlp_forward");
  if (st != MCG_OK) return st;
  if (n < 1 || n > (int64_t)1 << 30 || !x || !y) return mcg_fail(ctx, MCG_ERR_ARG, "mlp_forward: bad arguments");
  MlpState &s = *ctx->mlp;
  const int64_t chunk = std::min<int64_t>(n, (int64_t)1 << 20);
  if ((st = mlp_reserve(ctx, chunk)) != MCG_OK) return st;
  for (int64_t i0 = 0; i0 < n; i0 += chunk) {
    const int64_t m = std::min(chunk, n - i0);
    MCG_CUDA(ctx, cudaMemcpyAsync(s.xb, x + i0 * IN, m * IN * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
    mlp_fwd_launch(ctx, m, false);
    MCG_CUDA(ctx, cudaGetLastError());
    MCG_CUDA(ctx, cudaMemcpyAsync(y + i0 * OUT, s.yb, m * OUT * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
  }
  return mlp_check_err(ctx, "mlp_forward");
}

mcg_status mcg_mlp_gradient(mcg_ctx *ctx, int64_t n, const float *x, const float *t, const float *w,
                            float *grad, double *loss) {
  if (!ctx) return MCG_ERR_ARG;
  cudaSetDevice(ctx->device);
  mcg_status st = mlp_ready(ctx, "mlp_gradient");
  if (st != MCG_OK) return st;
  if (n < 1 || n > (int64_t)1 << 20 || !x || !t || !w || !grad)
    return mcg_fail(ctx, MCG_ERR_ARG, "mlp_gradient: 1 <= n <= 2^20 and non-null arrays required");
  MlpState &s = *ctx->mlp;
  if ((st = mlp_reserve(ctx, n)) != MCG_OK) return st;
  MCG_CUDA(ctx, cudaMemcpyAsync(s.xb, x, n * IN * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
  MCG_CUDA(ctx, cudaMemcpyAsync(s.tb, t, n * OUT * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
  MCG_CUDA(ctx, cudaMemcpyAsync(s.wout, w, OUT * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
  mlp_backward_launch(ctx, n);
  MCG_CUDA(ctx, cudaGetLastError());
  MCG_CUDA(ctx, cudaMemcpyAsync(grad, s.G, NPARAMS * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
  double l = 0.0;
  MCG_CUDA(ctx, cudaMemcpyAsync(&l, s.loss, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  st = mlp_check_err(ctx, "mlp_gradient");
  if (loss) *loss = l;
  return st;
}

mcg_status mcg_mlp_train(mcg_ctx *ctx, int64_t n, const float *x, const float *t, const float *w,
                         const mcg_mlp_train_opts *o, mcg_mlp_train_report *rep) {
  if (!ctx) return MCG_ERR_ARG;
  cudaSetDevice(ctx->device);
  mcg_status st = mlp_ready(ctx, "mlp_train");
  if (st != MCG_OK) return st;
  if (n < 1 || n > (int64_t)1 << 28 || !x || !t || !w || !o)
    return mcg_fail(ctx, MCG_ERR_ARG, "mlp_train: bad arguments");
  if (o->epochs < 1 || o->batch < TILE || o->batch > (1 << 20) || !(o->lr > 0.0f))
    return mcg_fail(ctx, MCG_ERR_ARG, "mlp_train: epochs >= 1, 128 <= batch <= 2^20, lr > 0 required");
  MlpState &s = *ctx->mlp;
  const int64_t B = std::min<int64_t>(o->batch, n);
  if ((st = mlp_reserve(ctx, B)) != MCG_OK) return st;
  float *X = nullptr, *T = nullptr;
  int *idx = nullptr;
  cudaError_t e = cudaMalloc(&X, (size_t)n * IN * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc(&T, (size_t)n * OUT * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc(&idx, (size_t)n * sizeof(int));
  auto release = [&]() {
    cudaFree(X);
    cudaFree(T);
    cudaFree(idx);
  };
  if (e != cudaSuccess) {
    release();
    return mcg_fail(ctx, MCG_ERR_NOMEM, "mlp_train: dataset of %lld rows: %s", (long long)n, cudaGetErrorString(e));
  }
  cudaStream_t cs = ctx->stream;
  cudaMemcpyAsync(X, x, (size_t)n * IN * sizeof(float), cudaMemcpyHostToDevice, cs);
  cudaMemcpyAsync(T, t, (size_t)n * OUT * sizeof(float), cudaMemcpyHostToDevice, cs);
  cudaMemcpyAsync(s.wout, w, OUT * sizeof(float), cudaMemcpyHostToDevice, cs);
  std::vector<int> perm((size_t)n);
  for (int64_t i = 0; i < n; ++i) perm[(size_t)i] = (int)i;
  std::mt19937_64 rng(o->seed);
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  const int64_t steps_per_epoch = n / B;
  const int64_t total = std::max<int64_t>(1, steps_per_epoch * o->epochs);
  cudaEventRecord(ctx->ev0, cs);
  double last = 0.0;
  int64_t k = 0;
  for (int ep = 0; ep < o->epochs; ++ep) {
    std::shuffle(perm.begin(), perm.end(), rng);
    cudaMemcpyAsync(idx, perm.data(), (size_t)n * sizeof(int), cudaMemcpyHostToDevice, cs);
    double ep_loss = 0.0;
    for (int64_t b = 0; b < std::max<int64_t>(1, steps_per_epoch); ++b, ++k) {
      gather_rows_kernel<<<nblk(B * OUT, 256), 256, 0, cs>>>(X, T, idx + b * B, (int)B, s.xb, s.tb);
      mlp_backward_launch(ctx, B);
      /* cosine decay of the learning rate to lr_min */
      const double fr = (double)k / (double)total;
      const float lr = (float)(o->lr_min + 0.5 * (o->lr - o->lr_min) * (1.0 + cos(3.14159265358979 * fr)));
      ++s.step;
      const float c1 = 1.0f - powf(b1, (float)s.step), c2 = 1.0f - powf(b2, (float)s.step);
      mlp_adam_kernel<<<nblk(NPARAMS, 256), 256, 0, cs>>>(s.P, s.G, s.M, s.V, (int)NPARAMS, lr, b1, b2, eps, c1,
                                                           c2);
      mlp_pack(ctx);
      if (b == steps_per_epoch - 1 || steps_per_epoch <= 1) {
        double l = 0.0;
        cudaMemcpyAsync(&l, s.loss, sizeof(double), cudaMemcpyDeviceToHost, cs);
        cudaStreamSynchronize(cs);
        ep_loss = l;
      }
    }
    last = ep_loss;
    if (rep && ep < MCG_MLP_MAX_EPOCH_LOG) rep->epoch_loss[ep] = ep_loss;
  }
  cudaEventRecord(ctx->ev1, cs);
  e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaEventSynchronize(ctx->ev1);
  float ms = 0.0f;
  cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
  release();
  if (e != cudaSuccess) return mcg_fail(ctx, MCG_ERR_CUDA, "mlp_train: %s", cudaGetErrorString(e));
  if (rep) {
    rep->final_loss = last;
    rep->steps = k;
    rep->device_ms = ms;
  }
  return mlp_check_err(ctx, "mlp_train");
}

mcg_status mcg_mlp_gemm_check(mcg_ctx *ctx, int N, const uint16_t *A, const uint16_t *B, float *D) {
  if (!ctx) return MCG_ERR_ARG;
  cudaSetDevice(ctx->device);
  if (!A || !B || !D || N < 16 || N > 256 || N % 16 != 0)
    return mcg_fail(ctx, MCG_ERR_ARG, "mlp_gemm_check: 16 <= N <= 256, N % 16 == 0");
  mcg_status st = mlp_init(ctx);
  if (st != MCG_OK) return st;
  MlpState &s = *ctx->mlp;
  if ((st = mlp_reserve(ctx, TILE * 4)) != MCG_OK) return st;
  /* A (128 x 256) and B (N x 256) staged through the activation buffers */
  __nv_bfloat16 *dA = s.dza, *dB = s.dzb;
  float *dD = s.zs;
  MCG_CUDA(ctx, cudaMemsetAsync(s.err, 0, sizeof(int), ctx->stream));
  MCG_CUDA(ctx, cudaMemcpyAsync(dA, A, TILE * H * 2, cudaMemcpyHostToDevice, ctx->stream));
  MCG_CUDA(ctx, cudaMemcpyAsync(dB, B, (size_t)N * H * 2, cudaMemcpyHostToDevice, ctx->stream));
  mlp_gemm_check_kernel<<<1, NT, SMEM_CHECK, ctx->stream>>>(dA, dB, N, dD, s.err);
  MCG_CUDA(ctx, cudaGetLastError());
  MCG_CUDA(ctx, cudaMemcpyAsync(D, dD, (size_t)TILE * N * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
  return mlp_check_err(ctx, "mlp_gemm_check");
}

}  // extern "C"

/* ======================================================================
 * ComputePart through the surrogate (mcg_compute_part_surrogate).
 * ==================================================================== */
namespace {

constexpr int SURR_NMOM = 12; /* Legendre moments per Mueller element */
constexpr int NA = 180;       /* scattering-angle bins (ComputePart.f:41) */
static_assert(SURR_NMOM == SURR_PH_L && NA == SURR_PH_NA, "surrogate_phase.h works on the same moments and bins");

/* training box of the network inputs: log10 a [micron], log10 lambda
 * [micron], n, log10 k, porosity, fmax */
const double kBoxLo[6] = {-2.0, -1.0, 1.5, -3.5, 0.0, 0.0};
const double kBoxHi[6] = {3.0, 3.4771212547196626, 3.5, 0.3010299956639812, 0.6, 0.8};

struct SurrogatePart {
  int nlam = 0, ns = 0;
  double rho = 0.0, por = 0.0;
  std::vector<double> mw;  /* mass weight per size */
  int64_t row0 = 0;        /* first network row: (k, l) -> row0 + k * nlam + l */
};

/* sizes and mass weights of ComputePart.f:276-292 for one material */
bool part_sizes(const mcg_part_in &in, std::vector<double> &r, std::vector<double> &mw) {
  const int ns = in.ns;
  r.assign(ns, 0.0);
  mw.assign(ns, 0.0);
  const double minlog = log10(in.amin), maxlog = log10(in.amax), pw = -in.apow;
  if (ns == 1) {
    r[0] = pow(10.0, (minlog + maxlog) / 2.0);
    mw[0] = 1.0;
    return true;
  }
  double t = 0.0;
  for (int k = 0; k < ns; ++k) {
    r[k] = pow(10.0, minlog + (maxlog - minlog) * (double)k / (double)(ns - 1));
    mw[k] = pow(r[k], pw + 1.0) * r[k] * r[k] * r[k];
    t += mw[k];
  }
  if (!(t > 0.0)) return false;
  for (int k = 0; k < ns; ++k) mw[k] /= t;
  return true;
}

}  // namespace

extern "C" mcg_status mcg_compute_part_surrogate(mcg_ctx *ctx, int nparts, const mcg_part_in *in, mcg_part_out *out,
                                                 double rho_train, int nf_train, int *used) {
  if (!ctx) return MCG_ERR_ARG;
  cudaSetDevice(ctx->device);
  mcg_status st = mlp_ready(ctx, "compute_part_surrogate");
  if (st != MCG_OK) return st;
  if (nparts < 1 || !in || !out || !(rho_train > 0.0))
    return mcg_fail(ctx, MCG_ERR_ARG, "compute_part_surrogate: nparts >= 1, rho_train > 0, non-null in/out");
  std::vector<SurrogatePart> sp(nparts);
  std::vector<int> fallback;
  std::vector<float> X;
  int64_t rows = 0;
  for (int p = 0; p < nparts; ++p) {
    const mcg_part_in &q = in[p];
    if (!out[p].kabs || !out[p].ksca || !out[p].kext || !out[p].F)
      return mcg_fail(ctx, MCG_ERR_ARG, "compute_part_surrogate: null output array (part %d)", p);
    bool ok = q.nm == 1 && q.lam && q.e1 && q.e2 && q.rho && q.nlam >= 2 && q.ns >= 1 && q.nf == nf_train &&
              q.normalize_abun <= 0.0 && q.amin > 0.0 && q.amax > 0.0 && q.rho[0] > 0.0;
    const double por = (ok && q.blend) ? q.porosity : 0.0;
    std::vector<double> r, mw;
    if (ok) ok = part_sizes(q, r, mw);
    if (ok) {
      for (int k = 0; k < q.ns && ok; ++k)
        for (int l = 0; l < q.nlam && ok; ++l) {
          const double v[6] = {log10(r[k]), log10(q.lam[l]), q.e1[l], q.e2[l] > 0.0 ? log10(q.e2[l]) : -99.0, por,
                               q.fmax};
          for (int i = 0; i < 6; ++i) ok = ok && v[i] >= kBoxLo[i] && v[i] <= kBoxHi[i];
        }
    }
    if (!ok) {
      fallback.push_back(p);
      if (used) used[p] = 0;
      continue;
    }
    SurrogatePart &s = sp[p];
    s.nlam = q.nlam;
    s.ns = q.ns;
    s.rho = q.rho[0];
    s.por = por;
    s.mw = mw;
    s.row0 = rows;
    for (int k = 0; k < q.ns; ++k)
      for (int l = 0; l < q.nlam; ++l) {
        const double v[6] = {log10(r[k]), log10(q.lam[l]), q.e1[l], log10(q.e2[l]), por, q.fmax};
        for (int i = 0; i < 6; ++i) X.push_back((float)(2.0 * (v[i] - kBoxLo[i]) / (kBoxHi[i] - kBoxLo[i]) - 1.0));
      }
    rows += (int64_t)q.ns * q.nlam;
    if (used) used[p] = 1;
  }
  if (rows > 0) {
    std::vector<float> Y((size_t)rows * OUT);
    if ((st = mcg_mlp_forward(ctx, rows, X.data(), Y.data())) != MCG_OK) return st;
    static const SurrLegendre legendre; /* Legendre table of the 180 angle bins */
    for (int p = 0; p < nparts; ++p) {
      if (used && !used[p]) continue;
      if (!used && std::find(fallback.begin(), fallback.end(), p) != fallback.end()) continue;
      const SurrogatePart &s = sp[p];
      const double scale = rho_train / s.rho; /* kappa ~ 1 / material density */
      for (int l = 0; l < s.nlam; ++l) {
        double ka = 0.0, ks = 0.0, wsum = 0.0, chi[SURR_NMOM + 1] = {0}, beta[SURR_NMOM + 1] = {0},
               gam[SURR_NMOM + 1] = {0}, del[SURR_NMOM + 1] = {0};
        for (int k = 0; k < s.ns; ++k) {
          const float *y = Y.data() + (size_t)(s.row0 + (int64_t)k * s.nlam + l) * OUT;
          const double kak = pow(10.0, (double)y[0]) * scale, ksk = pow(10.0, (double)y[1]) * scale;
          ka += s.mw[k] * kak;
          ks += s.mw[k] * ksk;
          const double w = s.mw[k] * ksk;
          wsum += w;
          chi[0] += w;
          for (int m = 1; m <= SURR_NMOM; ++m) chi[m] += w * (double)y[1 + m];
          for (int m = 0; m <= SURR_NMOM; ++m) {
            beta[m] += w * (double)y[14 + m];
            gam[m] += w * (double)y[27 + m];
            del[m] += w * (double)y[40 + m];
          }
        }
        for (int m = 0; m <= SURR_NMOM; ++m) {
          chi[m] /= wsum;
          beta[m] /= wsum;
          gam[m] /= wsum;
          del[m] /= wsum;
        }
        out[p].kabs[l] = ka;
        out[p].ksca[l] = ks;
        out[p].kext[l] = ka + ks;
        /* phase matrix on the 180 bins from the moments, delta-M form */
        surr_phase_matrix(legendre, chi, beta, gam, del, 1, out[p].F + (size_t)l * 6 * NA);
      }
      out[p].rho_av = (1.0 - s.por) * s.rho;
      out[p].mscale = 1.0;
      out[p].rscale = 1.0;
      out[p].n_dhs = out[p].n_mie = out[p].n_dhs_fail = 0;
    }
  }
  if (!fallback.empty()) {
    std::vector<mcg_part_in> fin;
    std::vector<mcg_part_out> fout;
    for (int p : fallback) {
      fin.push_back(in[p]);
      fout.push_back(out[p]);
    }
    st = mcg_part_batch_impl(ctx, (int)fin.size(), fin.data(), fout.data());
    if (st != MCG_OK) return st;
    for (size_t i = 0; i < fallback.size(); ++i) out[fallback[i]] = fout[i];
  }
  return MCG_OK;
}

extern "C" mcg_status mcg_surrogate_targets(mcg_ctx *ctx, int64_t n, const double *in6, double rho, int nf,
                                            float *out) {
  if (!ctx) return MCG_ERR_ARG;
  cudaSetDevice(ctx->device);
  return mcg_surrogate_targets_impl(ctx, n, in6, rho, nf, out);
}

/* Device timing of the network: forward passes over n device-resident rows
 * and training steps (forward + backward + Adam) on batches of `batch` rows,
 * CUDA events on the context's stream.  The parameters are saved and
 * restored around the training steps. */
extern "C" mcg_status mcg_mlp_time(mcg_ctx *ctx, int64_t n, int iters, int batch, float *fwd_ms, float *step_ms) {
  if (!ctx) return MCG_ERR_ARG;
  cudaSetDevice(ctx->device);
  mcg_status st = mlp_ready(ctx, "mlp_time");
  if (st != MCG_OK) return st;
  if (n < TILE || n > ((int64_t)1 << 24) || iters < 1 || iters > 1000 || batch < TILE || batch > (1 << 20) || !fwd_ms ||
      !step_ms)
    return mcg_fail(ctx, MCG_ERR_ARG, "mlp_time: 128 <= n <= 2^24, 1 <= iters <= 1000, 128 <= batch <= 2^20");
  MlpState &s = *ctx->mlp;
  const int64_t rows = std::max<int64_t>(n, batch);
  if ((st = mlp_reserve(ctx, rows)) != MCG_OK) return st;
  cudaStream_t cs = ctx->stream;
  std::vector<float> P((size_t)NPARAMS);
  MCG_CUDA(ctx, cudaMemcpyAsync(P.data(), s.P, NPARAMS * sizeof(float), cudaMemcpyDeviceToHost, cs));
  /* inputs in [-1, 1] and zero targets, generated on the host once */
  {
    std::vector<float> x((size_t)rows * IN), w(OUT, 1.0f);
    std::mt19937 rng(7);
    std::uniform_real_distribution<float> u(-1.0f, 1.0f);
    for (auto &v : x) v = u(rng);
    MCG_CUDA(ctx, cudaMemcpyAsync(s.xb, x.data(), x.size() * sizeof(float), cudaMemcpyHostToDevice, cs));
    MCG_CUDA(ctx, cudaMemsetAsync(s.tb, 0, (size_t)rows * OUT * sizeof(float), cs));
    MCG_CUDA(ctx, cudaMemcpyAsync(s.wout, w.data(), OUT * sizeof(float), cudaMemcpyHostToDevice, cs));
    MCG_CUDA(ctx, cudaStreamSynchronize(cs));
  }
  for (int w = 0; w < 2; ++w) mlp_fwd_launch(ctx, n, false);
  cudaEventRecord(ctx->ev0, cs);
  for (int i = 0; i < iters; ++i) mlp_fwd_launch(ctx, n, false);
  cudaEventRecord(ctx->ev1, cs);
  MCG_CUDA(ctx, cudaEventSynchronize(ctx->ev1));
  float ms = 0.0f;
  cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
  *fwd_ms = ms / (float)iters;
  const float b1 = 0.9f, b2 = 0.999f;
  auto step = [&]() {
    mlp_backward_launch(ctx, batch);
    ++s.step;
    const float c1 = 1.0f - powf(b1, (float)s.step), c2 = 1.0f - powf(b2, (float)s.step);
    mlp_adam_kernel<<<nblk(NPARAMS, 256), 256, 0, cs>>>(s.P, s.G, s.M, s.V, (int)NPARAMS, 1e-6f, b1, b2, 1e-8f, c1, c2);
    mlp_pack(ctx);
  };
  for (int w = 0; w < 2; ++w) step();
  cudaEventRecord(ctx->ev0, cs);
  for (int i = 0; i < iters; ++i) step();
  cudaEventRecord(ctx->ev1, cs);
  MCG_CUDA(ctx, cudaEventSynchronize(ctx->ev1));
  cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
  *step_ms = ms / (float)iters;
  /* restore the parameters and a fresh optimizer state */
  st = mcg_mlp_set_params(ctx, P.data(), NPARAMS);
  if (st != MCG_OK) return st;
  return mlp_check_err(ctx, "mlp_time");
}

/*
 * tc_sm100.cuh -- the fifth-generation tensor-core (tcgen05) pieces used by
 * the opacity-surrogate network kernels: shared-memory matrix descriptors,
 * the instruction descriptor of a BF16 x BF16 -> FP32 MMA, tensor-memory
 * allocation, MMA issue and completion through an mbarrier, and loads of the
 * accumulator from tensor memory.  sm_100a only.
 *
 * Operand layout: K-major, no swizzle.  A tile of R rows and K columns of
 * bf16 is stored as 8-row x 16-byte "core matrices": element (r, k) sits at
 *   (r / 8) * SBO + (k / 8) * 128 + (r % 8) * 16 + (k % 8) * 2   bytes,
 * SBO = K * 16 (the 8-row groups follow one another after all K columns).
 * One MMA consumes K = 16 (two core matrices along K, 128 bytes apart: the
 * leading byte offset), so the descriptor of k-step s starts s * 256 bytes
 * after the tile.
 *
 * Every wait on an mbarrier is bounded: after TC_WAIT_LIMIT polls it gives
 * up and reports failure to the caller, which records an error status and
 * returns (nothing here traps).
 */
#ifndef MCMAX_TC_SM100_CUH
#define MCMAX_TC_SM100_CUH

#include <cuda_bf16.h>
#include <stdint.h>

#define TC_WAIT_LIMIT (1u << 20)

__device__ __forceinline__ uint32_t tc_smem_addr(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

/* byte offset of element (r, k) in a K-major no-swizzle tile with K columns */
__host__ __device__ __forceinline__ uint32_t tc_kmaj_off(int r, int k, int K) {
  return (uint32_t)((r >> 3) * (K * 16) + (k >> 3) * 128 + (r & 7) * 16 + (k & 7) * 2);
}

/* shared-memory matrix descriptor (sm_100 form: version 1 in bits 46-47,
 * no swizzle, base offset 0) */
__device__ __forceinline__ uint64_t tc_desc(uint32_t saddr, uint32_t lbo_bytes, uint32_t sbo_bytes) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo_bytes >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo_bytes >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1u << 46;
  return d;
}

/* instruction descriptor, kind::f16: D = F32 (bits 4-5 = 1), A = B = BF16
 * (bits 7-9 = 1, bits 10-12 = 1), both K-major, N >> 3 at bit 17, M >> 4 at
 * bit 24 */
__host__ __device__ constexpr uint32_t tc_idesc_bf16(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

/* tensor-memory allocation by one whole warp; the base address is written to
 * *slot (shared memory) */
__device__ __forceinline__ void tc_alloc(uint32_t *slot, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(tc_smem_addr(slot)),
               "r"(ncols));
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
}
__device__ __forceinline__ void tc_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols));
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
/* make generic-proxy shared-memory writes visible to the tensor cores */
__device__ __forceinline__ void tc_fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

/* D[tmem] (+)= A * B^T, one elected thread */
__device__ __forceinline__ void tc_mma(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                       uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}
/* arrive on the mbarrier when all MMAs issued so far by this thread are done */
__device__ __forceinline__ void tc_commit(uint64_t *mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   tc_smem_addr(mbar))
               : "memory");
}

__device__ __forceinline__ void tc_mbar_init(uint64_t *mbar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(tc_smem_addr(mbar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
/* bounded wait for the phase with the given parity; returns 1 on success */
__device__ __forceinline__ int tc_mbar_wait(uint64_t *mbar, uint32_t parity) {
  const uint32_t a = tc_smem_addr(mbar);
  for (uint32_t it = 0; it < TC_WAIT_LIMIT; ++it) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(a), "r"(parity)
        : "memory");
    if (ok) return 1;
  }
  return 0;
}

/* Asynchronous bulk copy global -> shared (the copy engine of the SM, no
 * multicast) that completes `bytes` of transaction count on the mbarrier.
 * The issuing thread first announces the total with tc_expect_tx.  Both
 * addresses 16-byte aligned, sizes multiples of 16. */
__device__ __forceinline__ void tc_expect_tx(uint64_t *mbar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(tc_smem_addr(mbar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void tc_bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *mbar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   tc_smem_addr(dst)),
               "l"(src), "r"(bytes), "r"(tc_smem_addr(mbar))
               : "memory");
}
/* one thread: announce and issue a copy of `bytes` in pieces of 32 KB */
__device__ __forceinline__ void tc_bulk_load(void *dst, const void *src, uint32_t bytes, uint64_t *mbar) {
  tc_expect_tx(mbar, bytes);
  for (uint32_t o = 0; o < bytes; o += 32768u) {
    const uint32_t n = bytes - o < 32768u ? bytes - o : 32768u;
    tc_bulk_g2s((unsigned char *)dst + o, (const unsigned char *)src + o, n, mbar);
  }
}

/* 16 consecutive FP32 accumulator columns of this thread's TMEM lane: warp w
 * of the warpgroup reads lanes 32w..32w+31, lane = row of the 128-row tile.
 * The load and its wait are one statement (as in tc_ld32). */
__device__ __forceinline__ void tc_ld16(uint32_t taddr, float *v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n\t"
      "tcgen05.wait::ld.sync.aligned;"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr)
      : "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

/* 32 consecutive FP32 accumulator columns of this thread's TMEM lane; the
 * load and its wait are one statement, so no use of the registers can be
 * scheduled before the data has arrived */
__device__ __forceinline__ void tc_ld32(uint32_t taddr, float *v) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n\t"
      "tcgen05.wait::ld.sync.aligned;"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr)
      : "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

/* plain arrival (release, CTA scope) on an mbarrier */
__device__ __forceinline__ void tc_mbar_arrive(uint64_t *mbar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(tc_smem_addr(mbar)) : "memory");
}

/* bounded wait that also gives up when *abort_flag is set (checked every 64
 * polls); returns 1 when the phase completed */
__device__ __forceinline__ int tc_mbar_wait_or_abort(uint64_t *mbar, uint32_t parity, volatile int *abort_flag) {
  const uint32_t a = tc_smem_addr(mbar);
  for (uint32_t it = 0; it < TC_WAIT_LIMIT; ++it) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(a), "r"(parity)
        : "memory");
    if (ok) return 1;
    if ((it & 63u) == 63u && *abort_flag) return 0;
  }
  return 0;
}

/* issue the K/16 MMAs of D = A (M x K) * B (N x K)^T from K-major tiles at
 * shared addresses a0 (M rows) and b0 (N rows) */
__device__ __forceinline__ void tc_gemm_issue(uint32_t tmem_d, uint32_t a0, uint32_t b0, int M, int N, int K,
                                              int accumulate_first) {
  const uint32_t idesc = tc_idesc_bf16(M, N);
  const uint32_t sbo = (uint32_t)K * 16u;
  for (int s = 0; s < K / 16; ++s) {
    const uint64_t ad = tc_desc(a0 + 256u * (uint32_t)s, 128u, sbo);
    const uint64_t bd = tc_desc(b0 + 256u * (uint32_t)s, 128u, sbo);
    tc_mma(tmem_d, ad, bd, idesc, (s > 0 || accumulate_first) ? 1u : 0u);
  }
}

#endif /* MCMAX_TC_SM100_CUH */

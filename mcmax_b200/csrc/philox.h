/*
 * philox.h -- Philox4x32-10 counter-based generator (Salmon, Moraes, Dror &
 * Shaw, "Parallel random numbers: as easy as 1, 2, 3", SC 2011), usable from
 * host C/C++ and CUDA device code.
 *
 * Every photon packet owns an independent stream: key = run seed, counter =
 * (block index, 0, packet id low, packet id high).  One block yields four
 * 32-bit words = two uniform doubles with 53 random bits each.  The stream of
 * a packet therefore does not depend on which thread, warp or launch
 * processes it, which is what lets the GPU kernels and the CPU oracle replay
 * identical random numbers.
 */
#ifndef MCMAX_PHILOX_H
#define MCMAX_PHILOX_H

#include <stdint.h>

#if defined(__CUDACC__)
#define PX_FN static __host__ __device__ __forceinline__
#else
#define PX_FN static inline
#endif

#define PX_M0 0xD2511F53u
#define PX_M1 0xCD9E8D57u
#define PX_W0 0x9E3779B9u
#define PX_W1 0xBB67AE85u

PX_FN void px_mulhilo(uint32_t a, uint32_t b, uint32_t *hi, uint32_t *lo) {
  uint64_t p = (uint64_t)a * (uint64_t)b;
  *hi = (uint32_t)(p >> 32);
  *lo = (uint32_t)p;
}

/* ten rounds of Philox4x32 on counter c[4] with key k[2]; result in out[4] */
PX_FN void px_philox4x32_10(const uint32_t c[4], const uint32_t k[2], uint32_t out[4]) {
  uint32_t x0 = c[0], x1 = c[1], x2 = c[2], x3 = c[3];
  uint32_t k0 = k[0], k1 = k[1];
  for (int r = 0; r < 10; ++r) {
    uint32_t hi0, lo0, hi1, lo1;
    px_mulhilo(PX_M0, x0, &hi0, &lo0);
    px_mulhilo(PX_M1, x2, &hi1, &lo1);
    uint32_t y0 = hi1 ^ x1 ^ k0;
    uint32_t y1 = lo1;
    uint32_t y2 = hi0 ^ x3 ^ k1;
    uint32_t y3 = lo0;
    x0 = y0; x1 = y1; x2 = y2; x3 = y3;
    k0 += PX_W0;
    k1 += PX_W1;
  }
  out[0] = x0; out[1] = x1; out[2] = x2; out[3] = x3;
}

/* two 32-bit words -> double uniform on the open interval (0,1) */
PX_FN double px_u01(uint32_t a, uint32_t b) {
  uint64_t v = ((uint64_t)a << 21) ^ (uint64_t)(b >> 11); /* 53 bits */
  return ((double)v + 0.5) * 0x1p-53;
}

/* per-packet stream state: 24 bytes, kept in registers by the kernels */
typedef struct {
  uint32_t key[2];
  uint32_t pid_lo, pid_hi;
  uint32_t block;   /* next Philox block index */
  uint32_t have;    /* 1 when `spare` holds an unused draw */
  double spare;
} px_stream;

PX_FN void px_init(px_stream *s, uint64_t seed, uint64_t packet_id) {
  s->key[0] = (uint32_t)seed;
  s->key[1] = (uint32_t)(seed >> 32);
  s->pid_lo = (uint32_t)packet_id;
  s->pid_hi = (uint32_t)(packet_id >> 32);
  s->block = 0;
  s->have = 0;
  s->spare = 0.0;
}

#if defined(__CUDA_ARCH__)
/* One Philox block for a device caller.  Kept out of line: the packet loops
 * draw random numbers at dozens of places, and one shared copy of the ten
 * rounds keeps those loops small in the instruction cache. */
static __device__ __noinline__ uint4 px_block_dev(uint32_t block, uint32_t pid_lo, uint32_t pid_hi, uint32_t k0,
                                                  uint32_t k1) {
  const uint32_t c[4] = {block, 0u, pid_lo, pid_hi};
  const uint32_t k[2] = {k0, k1};
  uint32_t o[4];
  px_philox4x32_10(c, k, o);
  return make_uint4(o[0], o[1], o[2], o[3]);
}
#endif

/* next uniform double in (0,1) of the packet's stream */
PX_FN double px_next(px_stream *s) {
  if (s->have) {
    s->have = 0;
    return s->spare;
  }
  uint32_t o[4];
#if defined(__CUDA_ARCH__)
  {
    const uint4 w = px_block_dev(s->block, s->pid_lo, s->pid_hi, s->key[0], s->key[1]);
    o[0] = w.x;
    o[1] = w.y;
    o[2] = w.z;
    o[3] = w.w;
  }
#else
  {
    const uint32_t c[4] = {s->block, 0u, s->pid_lo, s->pid_hi};
    px_philox4x32_10(c, s->key, o);
  }
#endif
  s->block += 1u;
  s->spare = px_u01(o[2], o[3]);
  s->have = 1;
  return px_u01(o[0], o[1]);
}

#endif /* MCMAX_PHILOX_H */

/*
 * hp_rng.h -- counter-based random numbers shared by the CUDA kernels and the
 * CPU checker, so that both draw bit-identical streams.
 *
 * Generator: Philox4x32-10 (J. K. Salmon, M. A. Moraes, R. O. Dror,
 * D. E. Shaw, "Parallel random numbers: as easy as 1, 2, 3", SC'11), with the
 * round multipliers and Weyl key increments published there.
 *
 * Stream layout.  Each particle owns one stream per step and per purpose:
 *     key     = (seed_lo, seed_hi)                  case seed
 *     counter = (slot, cell, step, species << 16 | block)
 * where slot is the particle's position inside its cell after the sort,
 * cell the cell index, step the time-step counter and block the index of the
 * 4-word Philox block inside the stream.  This replaces the reference's one
 * curand XORWOW state per (species, node) (src/cuda_Init.cu:80-86), whose
 * draw order depends on the per-cell loop; a per-particle key makes the
 * draws independent of how particles are mapped to threads.
 *
 * The null-collision test, the one draw every particle makes in a step,
 * comes from a separate block shared by four consecutive slots of a cell:
 *     counter = (slot / 4, cell, step, species << 16 | 0x8000 | sub)
 * slot 4g + t takes word t, and sub is the electron sub-cycle (0 for ions).
 * So one Philox evaluation tests four particles; a particle that collides
 * then draws everything else from its own stream above, starting at word 0
 * of block 0.  Particle streams use block numbers below 0x8000.
 *
 * Uniforms are (x >> 8 + 1) * 2^-24, in (0, 1] like curand_uniform.
 */
#ifndef HP_RNG_H
#define HP_RNG_H

#include <stdint.h>

#if defined(__CUDACC__)
#define HP_HD __host__ __device__ __forceinline__
#else
#define HP_HD static inline
#endif

#define HP_PHILOX_M0 0xD2511F53u
#define HP_PHILOX_M1 0xCD9E8D57u
#define HP_PHILOX_W0 0x9E3779B9u
#define HP_PHILOX_W1 0xBB67AE85u

typedef struct hp_u4 { uint32_t x, y, z, w; } hp_u4;

HP_HD void hp_mulhilo(uint32_t a, uint32_t b, uint32_t *hi, uint32_t *lo) {
    uint64_t p = (uint64_t)a * (uint64_t)b;
    *hi = (uint32_t)(p >> 32);
    *lo = (uint32_t)p;
}

HP_HD hp_u4 hp_philox4x32_10(hp_u4 c, uint32_t k0, uint32_t k1) {
#if defined(__CUDACC__)
#pragma unroll
#endif
    for (int r = 0; r < 10; r++) {
        uint32_t hi0, lo0, hi1, lo1;
        hp_mulhilo(HP_PHILOX_M0, c.x, &hi0, &lo0);
        hp_mulhilo(HP_PHILOX_M1, c.z, &hi1, &lo1);
        hp_u4 n;
        n.x = hi1 ^ c.y ^ k0;
        n.y = lo1;
        n.z = hi0 ^ c.w ^ k1;
        n.w = lo0;
        c = n;
        k0 += HP_PHILOX_W0;
        k1 += HP_PHILOX_W1;
    }
    return c;
}

HP_HD float hp_u01(uint32_t x) { return (float)((x >> 8) + 1u) * (1.0f / 16777216.0f); }

/* One particle's stream for one step and purpose. */
typedef struct hp_stream {
    hp_u4 ctr;
    uint32_t k0, k1;
    hp_u4 buf;
    int used; /* words of buf already consumed (4 = empty) */
} hp_stream;

HP_HD void hp_stream_init(hp_stream *s, uint64_t seed, uint32_t slot, uint32_t cell, uint32_t step,
                          uint32_t species) {
    s->k0 = (uint32_t)seed;
    s->k1 = (uint32_t)(seed >> 32);
    s->ctr.x = slot;
    s->ctr.y = cell;
    s->ctr.z = step;
    s->ctr.w = species << 16;
    s->used = 4;
    s->buf.x = s->buf.y = s->buf.z = s->buf.w = 0u;
}

HP_HD float hp_stream_next(hp_stream *s) {
    if (s->used == 4) {
        s->buf = hp_philox4x32_10(s->ctr, s->k0, s->k1);
        s->ctr.w += 1u;
        s->used = 0;
    }
    uint32_t v = (s->used == 0) ? s->buf.x : (s->used == 1) ? s->buf.y : (s->used == 2) ? s->buf.z : s->buf.w;
    s->used++;
    return hp_u01(v);
}

#define HP_TEST_BLOCK 0x8000u

/* The null-collision test block of slots 4*group .. 4*group+3. */
HP_HD hp_u4 hp_test_block(uint64_t seed, uint32_t group, uint32_t cell, uint32_t step, uint32_t species,
                          uint32_t sub) {
    hp_u4 ctr;
    ctr.x = group;
    ctr.y = cell;
    ctr.z = step;
    ctr.w = (species << 16) | HP_TEST_BLOCK | sub;
    return hp_philox4x32_10(ctr, (uint32_t)seed, (uint32_t)(seed >> 32));
}

HP_HD uint32_t hp_word(hp_u4 b, uint32_t t) { return t == 0 ? b.x : t == 1 ? b.y : t == 2 ? b.z : b.w; }

/* The null-collision test draw of one slot. */
HP_HD float hp_test_draw(uint64_t seed, uint32_t slot, uint32_t cell, uint32_t step, uint32_t species,
                         uint32_t sub) {
    return hp_u01(hp_word(hp_test_block(seed, slot >> 2, cell, step, species, sub), slot & 3u));
}

#endif /* HP_RNG_H */

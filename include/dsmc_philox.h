/*
 * dsmc_philox.h - counter-based random numbers for the DSMC engine.
 *
 * Philox4x32-10 (Salmon, Moraes, Dror and Shaw, "Parallel random numbers:
 * as easy as 1, 2, 3", SC'11), written from the published round function:
 * two 32x32->64 multiplies per round with the multipliers 0xD2511F53 and
 * 0xCD9E8D57, and a Weyl key schedule with increments 0x9E3779B9 and
 * 0xBB67AE85, ten rounds.
 *
 * The reference solver draws every random number from one global
 * multiply-with-carry stream (rng/BRNG.cxx:15-34), so the draw a particle gets
 * depends on every draw made before it.  Here every consumer owns a keyed
 * stream instead:
 *
 *     key     = (seed low word, seed high word)          one key per case
 *     counter = (draw / 4, entity, step, kind)           one stream per entity
 *
 * and the d-th draw of a stream is word (d % 4) of Philox(counter(d / 4), key).
 * A stream is therefore random-access: the GPU computes draw d directly, the
 * CPU oracle walks it sequentially, and both see the same numbers.
 *
 * Draws are mapped to doubles exactly as the reference maps its 32-bit words
 * (rng/BRNG.cxx:33): u = z * 2.328306435996595e-10, one IEEE multiply, so
 * u lies in [0, 1) and 0 is reachable.
 *
 * This header is plain C99 and compiles for the host and, under nvcc, for the
 * device.
 */
#ifndef DSMC_PHILOX_H
#define DSMC_PHILOX_H

#include <stdint.h>

#if defined(__CUDACC__)
#define DSMC_HD __host__ __device__ __forceinline__
#else
#define DSMC_HD static inline
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* Stream kinds: the fourth counter word. */
enum {
    DSMC_RNG_INIT = 1,    /* cold-start fill of the domain, entity 0          */
    DSMC_RNG_INJECT = 2,  /* inflow strip, entity = strip 0..3 (L, R, B, T)   */
    DSMC_RNG_MOVE = 3,    /* wall scattering, entity = particle slot          */
    DSMC_RNG_COLLIDE = 4, /* NTC selection, entity = cell k*NY + l            */
    DSMC_RNG_USER = 5,    /* host-side brng() of the drop-in surface           */
    DSMC_RNG_WARM = 6     /* warm start from a predicted field, entity = cell  */
};

#define DSMC_PHILOX_M0 0xD2511F53u
#define DSMC_PHILOX_M1 0xCD9E8D57u
#define DSMC_PHILOX_W0 0x9E3779B9u
#define DSMC_PHILOX_W1 0xBB67AE85u

/* The reference's 32-bit-word-to-double scale (rng/BRNG.cxx:33). */
#define DSMC_U32_TO_UNIT 2.328306435996595e-10

typedef struct dsmc_u32x4 {
    uint32_t v[4];
} dsmc_u32x4;

DSMC_HD void dsmc_mulhilo32(uint32_t a, uint32_t b, uint32_t *hi, uint32_t *lo)
{
    uint64_t p = (uint64_t)a * (uint64_t)b;
    *hi = (uint32_t)(p >> 32);
    *lo = (uint32_t)p;
}

DSMC_HD dsmc_u32x4 dsmc_philox4x32_10(dsmc_u32x4 c, uint32_t k0, uint32_t k1)
{
    for (int r = 0; r < 10; ++r) {
        if (r > 0) {
            k0 += DSMC_PHILOX_W0;
            k1 += DSMC_PHILOX_W1;
        }
        uint32_t hi0, lo0, hi1, lo1;
        dsmc_mulhilo32(DSMC_PHILOX_M0, c.v[0], &hi0, &lo0);
        dsmc_mulhilo32(DSMC_PHILOX_M1, c.v[2], &hi1, &lo1);
        dsmc_u32x4 n;
        n.v[0] = hi1 ^ c.v[1] ^ k0;
        n.v[1] = lo1;
        n.v[2] = hi0 ^ c.v[3] ^ k1;
        n.v[3] = lo0;
        c = n;
    }
    return c;
}

DSMC_HD double dsmc_u32_to_unit(uint32_t z)
{
    return (double)z * DSMC_U32_TO_UNIT;
}

/* A sequential cursor over one keyed stream. */
typedef struct dsmc_stream {
    uint32_t key0, key1;
    uint32_t entity, step, kind;
    uint32_t next;     /* counter word 0 of the next block to fetch */
    uint32_t used;     /* words of buf already handed out (0..4)    */
    uint32_t buf[4];
} dsmc_stream;

DSMC_HD void dsmc_stream_init(dsmc_stream *s, uint64_t seed, uint32_t kind,
                              uint32_t step, uint32_t entity)
{
    s->key0 = (uint32_t)seed;
    s->key1 = (uint32_t)(seed >> 32);
    s->entity = entity;
    s->step = step;
    s->kind = kind;
    s->next = 0;
    s->used = 4; /* forces a fetch of block 0 on the first draw */
    s->buf[0] = s->buf[1] = s->buf[2] = s->buf[3] = 0;
}

/* Position the cursor so the next draw is draw number d of the stream. */
DSMC_HD void dsmc_stream_seek(dsmc_stream *s, uint64_t d)
{
    dsmc_u32x4 c;
    c.v[0] = (uint32_t)(d >> 2);
    c.v[1] = s->entity;
    c.v[2] = s->step;
    c.v[3] = s->kind;
    dsmc_u32x4 o = dsmc_philox4x32_10(c, s->key0, s->key1);
    s->buf[0] = o.v[0];
    s->buf[1] = o.v[1];
    s->buf[2] = o.v[2];
    s->buf[3] = o.v[3];
    s->next = (uint32_t)(d >> 2) + 1u;
    s->used = (uint32_t)(d & 3u);
}

DSMC_HD uint32_t dsmc_stream_u32(dsmc_stream *s)
{
    if (s->used == 4) {
        dsmc_u32x4 c;
        c.v[0] = s->next;
        c.v[1] = s->entity;
        c.v[2] = s->step;
        c.v[3] = s->kind;
        dsmc_u32x4 o = dsmc_philox4x32_10(c, s->key0, s->key1);
        s->buf[0] = o.v[0];
        s->buf[1] = o.v[1];
        s->buf[2] = o.v[2];
        s->buf[3] = o.v[3];
        s->next += 1u;
        s->used = 0;
    }
    return s->buf[s->used++];
}

/* brng(): the next uniform double in [0, 1) of the stream. */
DSMC_HD double dsmc_stream_uniform(dsmc_stream *s)
{
    return dsmc_u32_to_unit(dsmc_stream_u32(s));
}

#ifdef __cplusplus
}
#endif

#endif /* DSMC_PHILOX_H */

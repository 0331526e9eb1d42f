/* SFMT-19937 restatement of lib/m_spring.f90:187-379 (spring_sfmt_init,
 * spring_sfmt_stream, spring_sfmt_source, spring_sfmt_kernel,
 * spring_sfmt_core).  Test infrastructure only.
 *
 * The reference stores the state as 64-bit halves of 128-bit words; this
 * restatement works on the equivalent little-endian 32-bit lanes.  The
 * recursion constants are the ones of the reference (POS1=122, SL1=18,
 * SL2=1 byte, SR1=11, SR2=1 byte, masks 8667995624701935 / 9007156306837503
 * for the low/high 64-bit halves, parity (1,0,0,331998852)). */
#include "orc_internal.h"

#define SFMT_N 156
#define SFMT_N32 624
#define SFMT_POS1 122

static const uint32_t MSK[4] = {0xdfffffefU, 0xddfecb7fU, 0xbffaffffU, 0xbffffff6U};
static const uint32_t PARITY[4] = {0x00000001U, 0x00000000U, 0x00000000U, 0x13c9e684U};

typedef struct { uint32_t u[4]; } w128;

static void lshift128(w128 *out, const w128 *in, int bytes) {
    uint64_t th = ((uint64_t)in->u[3] << 32) | in->u[2];
    uint64_t tl = ((uint64_t)in->u[1] << 32) | in->u[0];
    int s = bytes * 8;
    uint64_t oh = (th << s) | (tl >> (64 - s));
    uint64_t ol = tl << s;
    out->u[1] = (uint32_t)(ol >> 32); out->u[0] = (uint32_t)ol;
    out->u[3] = (uint32_t)(oh >> 32); out->u[2] = (uint32_t)oh;
}

static void rshift128(w128 *out, const w128 *in, int bytes) {
    uint64_t th = ((uint64_t)in->u[3] << 32) | in->u[2];
    uint64_t tl = ((uint64_t)in->u[1] << 32) | in->u[0];
    int s = bytes * 8;
    uint64_t oh = th >> s;
    uint64_t ol = (tl >> s) | (th << (64 - s));
    out->u[1] = (uint32_t)(ol >> 32); out->u[0] = (uint32_t)ol;
    out->u[3] = (uint32_t)(oh >> 32); out->u[2] = (uint32_t)oh;
}

/* spring_sfmt_core: r = a ^ (a <<8) ^ ((b >>11) & msk) ^ (c >>8) ^ (d << 18) */
static void recursion(w128 *r, const w128 *a, const w128 *b, const w128 *c, const w128 *d) {
    w128 x, y;
    lshift128(&x, a, 1);
    rshift128(&y, c, 1);
    for (int k = 0; k < 4; ++k)
        r->u[k] = a->u[k] ^ x.u[k] ^ ((b->u[k] >> 11) & MSK[k]) ^ y.u[k] ^ (d->u[k] << 18);
}

static void gen_all(orc_sfmt *s) {
    w128 *st = (w128 *)s->st;
    w128 *r1 = &st[SFMT_N - 2], *r2 = &st[SFMT_N - 1];
    int i;
    for (i = 0; i < SFMT_N - SFMT_POS1; ++i) {
        recursion(&st[i], &st[i], &st[i + SFMT_POS1], r1, r2);
        r1 = r2; r2 = &st[i];
    }
    for (; i < SFMT_N; ++i) {
        recursion(&st[i], &st[i], &st[i + SFMT_POS1 - SFMT_N], r1, r2);
        r1 = r2; r2 = &st[i];
    }
}

/* spring_sfmt_init (m_spring.f90:187-243).  The reference's `inner` flag has
 * an initialiser and hence keeps its value across calls; a run calls the
 * initialiser once, which this restatement models by starting from 0. */
void orc_sfmt_init(orc_sfmt *s, int32_t seed) {
    s->st[0] = (uint32_t)seed;
    for (int i = 1; i < SFMT_N32; ++i)
        s->st[i] = 1812433253U * (s->st[i - 1] ^ (s->st[i - 1] >> 30)) + (uint32_t)i;
    s->idx = SFMT_N32;
    uint32_t inner = 0;
    for (int i = 0; i < 4; ++i) inner ^= s->st[i] & PARITY[i];
    for (int i = 16; i > 0; i >>= 1) inner ^= inner >> i;
    inner &= 1;
    if (inner != 1) {
        for (int i = 0; i < 4; ++i) {
            uint32_t work = 1;
            for (int j = 0; j < 32; ++j) {
                if (work & PARITY[i]) { s->st[i] ^= work; return; }
                work <<= 1;
            }
        }
    }
}

uint32_t orc_sfmt_u32(orc_sfmt *s) {
    if (s->idx >= SFMT_N32) { gen_all(s); s->idx = 0; }
    return s->st[s->idx++];
}

/* spring_sfmt_stream: (u32 + 0.5) / 2^32, in (0,1) */
double orc_sfmt_stream(orc_sfmt *s) {
    return ((double)orc_sfmt_u32(s) + 0.5) * (1.0 / 4294967296.0);
}

/* src/dqmc_util.f90:72: abs((irank*1981+2008)*951049) in 32-bit integers
 * (two's-complement wrap, as the Fortran default integer does). */
int32_t orc_test_seed(int32_t irank) {
    uint32_t v = ((uint32_t)irank * 1981U + 2008U) * 951049U;
    int32_t s = (int32_t)v;
    if (s < 0) s = (int32_t)(0U - (uint32_t)s);
    return s;
}

/*
 * rng_shim.c - TEST INFRASTRUCTURE ONLY.
 *
 * Replaces the reference's mtwist.c when the reference sources are linked into the
 * harness, so that every Random::operator() draw the reference code makes comes from a
 * counter-based stream the harness chooses: draw d of (seed, stream, path) is word d&3
 * of Philox4x32-10 (Salmon et al., SC'11) on counter {d>>2, path, stream, 0x52454e5a},
 * key {seed, 0x4b5a4f52} - the same stream the CUDA kernels and the C oracle use.
 *
 * The reference inlines mt_lrand() from mtwist.h: it pops statevec[--stateptr] and
 * applies the MT19937 output tempering (published constants of Matsumoto & Nishimura,
 * 1998).  mts_refresh() below therefore stores the inverse-tempered Philox words, in
 * pop order, so the tempered output equals the Philox word exactly.
 */
#include <stdint.h>
#include <string.h>

#define MT_STATE_SIZE 624
typedef struct {
    uint32_t statevec[MT_STATE_SIZE];
    int stateptr;
    int initialized;
} mt_state;

mt_state mt_default_state;

static uint32_t g_seed = 2013u, g_stream = 0u, g_path = 0u, g_draw = 0u;

static uint32_t draw_u32(uint32_t seed, uint32_t stream, uint32_t path, uint32_t d) {
    uint32_t c0 = d >> 2, c1 = path, c2 = stream, c3 = 0x52454e5au;
    uint32_t k0 = seed, k1 = 0x4b5a4f52u;
    for (int r = 0; r < 10; ++r) {
        uint64_t p0 = (uint64_t)0xD2511F53u * c0;
        uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
        uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ k0;
        uint32_t n2 = (uint32_t)(p0 >> 32) ^ c3 ^ k1;
        c0 = n0; c1 = (uint32_t)p1; c2 = n2; c3 = (uint32_t)p0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    uint32_t w[4] = {c0, c1, c2, c3};
    return w[d & 3];
}

/* Inverse of y ^= y >> 11; y ^= (y << 7) & B; y ^= (y << 15) & C; y ^= y >> 18. */
static uint32_t undo_right(uint32_t y, int sh) {
    uint32_t x = y;
    for (int i = 0; i < 32; i += sh) x = y ^ (x >> sh);
    return x;
}
static uint32_t undo_left(uint32_t y, int sh, uint32_t mask) {
    uint32_t x = y;
    for (int i = 0; i < 32; i += sh) x = y ^ ((x << sh) & mask);
    return x;
}
static uint32_t untemper(uint32_t y) {
    y = undo_right(y, 18);
    y = undo_left(y, 15, 0xefc60000u);
    y = undo_left(y, 7, 0x9d2c5680u);
    y = undo_right(y, 11);
    return y;
}

void mts_refresh(mt_state *state) {
    /* mt_lrand pops statevec[623] first */
    for (int i = MT_STATE_SIZE - 1; i >= 0; --i)
        state->statevec[i] = untemper(draw_u32(g_seed, g_stream, g_path, g_draw++));
    state->stateptr = MT_STATE_SIZE;
    state->initialized = 1;
}

void mts_seed32(mt_state *state, uint32_t seed) {
    g_seed = seed; g_stream = 0u; g_path = 0u; g_draw = 0u;
    state->stateptr = 0;
    state->initialized = 1;
}
void mt_seed32(uint32_t seed) { mts_seed32(&mt_default_state, seed); }
void mts_seed32new(mt_state *state, uint32_t seed) { mts_seed32(state, seed); }
void mt_seed32new(uint32_t seed) { mts_seed32(&mt_default_state, seed); }
uint32_t mt_seed(void) { mt_seed32(2013u); return 2013u; }

/* Harness control: the next draw is draw 0 of (seed, stream, path). */
void rref_rng_stream(uint32_t seed, uint32_t stream, uint32_t path) {
    g_seed = seed; g_stream = stream; g_path = path; g_draw = 0u;
    mt_default_state.stateptr = 0;
    mt_default_state.initialized = 1;
}

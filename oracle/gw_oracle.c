/*
 * gw_oracle.c -- TEST INFRASTRUCTURE ONLY (see gw_oracle.h).
 *
 * Plain-C restatement of GraphWalker's walk hot path.  Only tests/,
 * __graft_entry__.smoke() and bench.py's cpu_baseline leg use it, as the
 * checker; the product (graphwalker_b200/) never links or loads it.
 */
#include "gw_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* ------------------------------------------------------------------------ */
/* Philox4x32-10, from the round function and constants published in        */
/* Salmon et al., SC'11 ("Parallel random numbers: as easy as 1, 2, 3").     */
/* ------------------------------------------------------------------------ */
#define PHILOX_M0 0xD2511F53u
#define PHILOX_M1 0xCD9E8D57u
#define PHILOX_W0 0x9E3779B9u
#define PHILOX_W1 0xBB67AE85u

static inline void mulhilo32(uint32_t a, uint32_t b, uint32_t *hi, uint32_t *lo) {
    uint64_t p = (uint64_t)a * (uint64_t)b;
    *hi = (uint32_t)(p >> 32);
    *lo = (uint32_t)p;
}

void gwo_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
    uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
    uint32_t k0 = key[0], k1 = key[1];
    for (int r = 0; r < 10; ++r) {
        uint32_t hi0, lo0, hi1, lo1;
        mulhilo32(PHILOX_M0, c0, &hi0, &lo0);
        mulhilo32(PHILOX_M1, c2, &hi1, &lo1);
        uint32_t n0 = hi1 ^ c1 ^ k0;
        uint32_t n2 = hi0 ^ c3 ^ k1;
        c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
        k0 += PHILOX_W0;
        k1 += PHILOX_W1;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

/* Per-hop draws: words 0 and 1 of Philox(key=seed, ctr=(id, hop, 0, 0)),
 * each shifted right by one so they span rand_r's [0, RAND_MAX].  The
 * engine's native-RNG layout (rng = 1) takes both draws of hop h from one
 * block per two hops: words 0, 1 (h even) or 2, 3 (h odd) of
 * Philox(ctr = (id, h / 2, 0, "NATV")). */
#define GWO_NATIVE_TAG 0x4E415456u
static inline void hop_draws(uint64_t seed, uint32_t rng, uint32_t id, uint32_t hop, uint32_t d[2]) {
    uint32_t ctr[4] = {id, hop, 0u, 0u};
    uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    uint32_t out[4];
    int w = 0;
    if (rng == 1) {
        ctr[1] = hop >> 1;
        ctr[3] = GWO_NATIVE_TAG;
        w = (hop & 1u) ? 2 : 0;
    }
    gwo_philox4x32_10(ctr, key, out);
    d[0] = out[w] >> 1;
    d[1] = out[w + 1] >> 1;
}

/* ------------------------------------------------------------------------ */
/* The continuation test of every live walk class:                          */
/*   if (outd > 0 && (float)rand_r(&seed)/RAND_MAX > 0.15)                  */
/* randomwalkwithjump.hpp:45, randomwalkwithstop.hpp:34,                    */
/* randomwalkwithprob.hpp:34, randomwalkwithrestartwithjoint.hpp:42.        */
/* ------------------------------------------------------------------------ */
#define GWO_RAND_MAX 2147483647 /* src/api/datatype.hpp:8 (an int) */

int gwo_continue_test(uint32_t r, double p) {
    volatile float q = (float)(int)r / GWO_RAND_MAX; /* float / int -> float */
    return (double)q > p;
}

uint64_t gwo_threshold_mismatches(double p) {
    uint32_t thr = gwo_continue_threshold(p);
    uint64_t bad = 0;
    for (uint32_t r = 0; r < 0x80000000u; ++r) {
        float q = (float)(int)r / GWO_RAND_MAX;
        bad += ((double)q > p) != (r >= thr);
    }
    return bad;
}

uint32_t gwo_continue_threshold(double p) {
    uint32_t lo = 0, hi = 0x80000000u; /* answer in [lo, hi] */
    if (!gwo_continue_test(0x7fffffffu, p)) return 0x80000000u;
    while (lo < hi) {
        uint32_t mid = lo + (hi - lo) / 2;
        if (gwo_continue_test(mid, p)) hi = mid; else lo = mid + 1;
    }
    return lo;
}

/* ------------------------------------------------------------------------ */
/* Walk word codec, src/walks/walk.hpp:69-91                                */
/* ------------------------------------------------------------------------ */
uint64_t gwo_encode(uint32_t source, uint32_t current, uint32_t hop) {
    return (((uint64_t)source & 0xffffffu) << 40) | (((uint64_t)current & 0x3ffffffu) << 14) |
           ((uint64_t)hop & 0x3fffu);
}
uint32_t gwo_get_source(uint64_t w) { return (uint32_t)(w >> 40) & 0xffffffu; }
uint32_t gwo_get_current(uint64_t w) { return (uint32_t)(w >> 14) & 0x3ffffffu; }
uint32_t gwo_get_hop(uint64_t w) { return (uint32_t)(w & 0x3fffu); }

/* ------------------------------------------------------------------------ */
/* One hop of one walk.  Restates the loop body shared by the four classes  */
/* (randomwalkwithjump.hpp:40-53 and siblings): the draw for the test is    */
/* only consumed when outd > 0 (short-circuit), the neighbour is            */
/* csr[beg_pos[v] - beg_pos[0] + r % outd], and the else-branch is the       */
/* class's own.  Returns 0 if the walk ended inside this hop (stop rules),  */
/* 1 if it moved (v updated, hop not yet incremented).                      */
/* ------------------------------------------------------------------------ */
static inline int hop_advance(const uint64_t *rowptr, const uint32_t *colidx, const gwo_params *p,
                              uint32_t thr, uint32_t id, uint32_t src, uint32_t hop, uint32_t *v) {
    uint32_t d[2];
    hop_draws(p->seed, p->rng, id, hop, d);
    uint64_t beg = rowptr[*v];
    uint64_t outd = rowptr[*v + 1] - beg;
    int di = 0;
    int pass = 0;
    if (outd > 0) pass = d[di++] >= thr;
    if (pass) {
        uint64_t r = d[di++];
        *v = colidx[beg + r % outd];
        return 1;
    }
    switch (p->rule) {
    case GWO_RULE_JUMP: *v = d[di++] % p->njump; return 1;           /* jump.hpp:50 */
    case GWO_RULE_STOP: return 0;                                    /* stop.hpp:37 */
    case GWO_RULE_PROB: return 0;                                    /* prob.hpp:41 */
    case GWO_RULE_RESTART: *v = src; return 1;                       /* joint.hpp:47-49 */
    case GWO_RULE_PPR:
        if (outd == 0) { *v = src; return 1; }
        return 0;
    }
    return 0;
}

static inline int rule_capped(uint32_t rule) {
    return rule == GWO_RULE_JUMP || rule == GWO_RULE_STOP || rule == GWO_RULE_PPR;
}

uint32_t gwo_run_walks(const uint64_t *rowptr, const uint32_t *colidx, uint32_t nv,
                       const uint32_t *cur, const uint32_t *id, const uint32_t *src,
                       const uint32_t *hop0, uint64_t nwalks, const gwo_params *p,
                       uint32_t *counts, uint32_t *paths, uint32_t stride, uint32_t *plen,
                       uint64_t *closure, uint32_t *final_cur, uint32_t *final_hop) {
    uint32_t status = 0;
    uint32_t thr = gwo_continue_threshold(p->jump_prob);
    /* Walks are independent (every draw is keyed on the walk's id and hop),
     * so they run on all host threads; the shared sinks are updated
     * atomically, which leaves every count equal to the sequential loop's. */
#pragma omp parallel for schedule(dynamic, 4096) reduction(| : status)
    for (uint64_t i = 0; i < nwalks; ++i) {
        uint32_t v = cur[i], h = hop0[i], s = src[i], wid = id[i];
        uint32_t k = 0;
        for (;;) {
            if (rule_capped(p->rule) && h >= p->L) break;
            if (p->rule == GWO_RULE_PROB && h >= p->max_hops) { status |= GWO_ST_HOP_OVF; break; }
            if (v >= nv) { status |= GWO_ST_BOUNDS; break; }
            /* updateInfo(sourId, dstId, threadid, hop) precedes the draws */
            if (counts) {
#pragma omp atomic
                counts[v] += 1;
            }
            if (paths) {
                if (k < stride) paths[i * (uint64_t)stride + k] = v;
                else status |= GWO_ST_PATH_OVF;
            }
            if (closure && (int64_t)h >= (int64_t)p->L - 1 && v == s) { /* graphlet.cpp:46-52 */
#pragma omp atomic
                *closure += 1;
            }
            k++;
            if (!hop_advance(rowptr, colidx, p, thr, wid, s, h, &v)) break;
            h++;
            if (p->rule == GWO_RULE_RESTART && p->L > 0 && h % p->L == p->L - 1) break; /* joint.hpp:52 */
        }
        if (plen) plen[i] = k;
        if (final_cur) final_cur[i] = v;
        if (final_hop) final_hop[i] = h;
    }
    return status;
}

uint32_t gwo_getblock(const uint32_t *blocks, uint32_t nblocks, uint32_t v) {
    for (uint32_t p = 0; p < nblocks; ++p)
        if (v < blocks[p + 1]) return p;
    return nblocks;
}

uint32_t gwo_block_step(const uint64_t *rowptr, const uint32_t *colidx, uint32_t nv,
                        const uint32_t *blocks, uint32_t nblocks, uint32_t b,
                        uint32_t *cur, const uint32_t *id, const uint32_t *src, uint32_t *hop,
                        uint64_t n, const gwo_params *p, uint32_t *counts, uint32_t *dest) {
    uint32_t status = 0;
    uint32_t thr = gwo_continue_threshold(p->jump_prob);
    uint32_t lo = blocks[b], hi = blocks[b + 1];
    for (uint64_t i = 0; i < n; ++i) {
        uint32_t v = cur[i], h = hop[i], s = src[i], wid = id[i];
        int ended = 0;
        /* while (dstId >= blocks[exec_block] && dstId < blocks[exec_block+1] && hop < L) */
        while (v >= lo && v < hi) {
            if (rule_capped(p->rule) && h >= p->L) break;
            if (p->rule == GWO_RULE_PROB && h >= p->max_hops) { status |= GWO_ST_HOP_OVF; ended = 1; break; }
            if (v >= nv) { status |= GWO_ST_BOUNDS; ended = 1; break; }
            if (counts) counts[v] += 1;
            if (!hop_advance(rowptr, colidx, p, thr, wid, s, h, &v)) { ended = 1; break; }
            h++;
            if (p->rule == GWO_RULE_RESTART && p->L > 0 && h % p->L == p->L - 1) { ended = 1; break; }
        }
        uint32_t d = 0xffffffffu;
        if (!ended) {
            int alive;
            if (rule_capped(p->rule)) alive = h < p->L;                    /* jump.hpp:55 */
            else if (p->rule == GWO_RULE_RESTART) alive = p->L == 0 || h % p->L != p->L - 1;
            else alive = 1;                                                /* prob.hpp:45 */
            if (alive) {
                uint32_t q = gwo_getblock(blocks, nblocks, v);
                if (q < nblocks) d = q;                                    /* jump.hpp:57 */
            }
        }
        cur[i] = v;
        hop[i] = h;
        dest[i] = d;
    }
    return status;
}

/* ------------------------------------------------------------------------ */
/* compute_block, src/preprocess/conversions.hpp:300-364, over the whole    */
/* row pointer at once (the reference reads it in VERT_SIZE chunks; the     */
/* result is the same except where it reads beg_pos[-1] of a later chunk).  */
/* ------------------------------------------------------------------------ */
uint32_t gwo_compute_blocks(const uint64_t *rowptr, uint32_t nv, uint64_t blocksize_kb,
                            uint32_t *blocks, uint32_t cap) {
    uint64_t mneb = blocksize_kb * 1024u / 4u;
    uint64_t ttv = (uint64_t)nv + 1; /* entries in the beg_pos file */
    uint64_t bgstvb = 0;
    uint32_t n = 0;
#define PUSH(x) do { if (n >= cap) return 0; blocks[n++] = (uint32_t)(x); } while (0)
    PUSH(0);
    for (uint64_t v = 0; v < ttv; ++v) {
        if (rowptr[v] - bgstvb > mneb) {
            if (rowptr[v] - rowptr[v - 1] > mneb) {
                PUSH(v - 1);
                PUSH(v);
                bgstvb = rowptr[v];
            } else {
                PUSH(v - 1);
                bgstvb = rowptr[v - 1];
            }
        }
    }
    PUSH(ttv - 1);
#undef PUSH
    return n;
}

/* ------------------------------------------------------------------------ */
/* Seeded R-MAT stream.                                                     */
/* ------------------------------------------------------------------------ */
static inline uint64_t splitmix64(uint64_t x) { /* Steele, Lea, Flood (OOPSLA'14) */
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

uint32_t gwo_rmat_permute(uint32_t v, uint32_t scale, uint64_t seed) {
    uint32_t mask = scale >= 32 ? 0xffffffffu : ((1u << scale) - 1u);
    uint32_t sh = (scale + 1) / 2;
    uint32_t x = v & mask;
    for (uint32_t r = 0; r < 4; ++r) {
        uint64_t k = splitmix64(seed ^ (0x5045524Dull + r)); /* "PERM" + round */
        x = (x ^ (uint32_t)k) & mask;
        x = (x * ((uint32_t)(k >> 32) | 1u)) & mask;
        if (sh > 0 && sh < 32) x ^= x >> sh;
    }
    return x;
}

void gwo_rmat_edge(uint64_t e, uint32_t scale, uint64_t seed,
                   uint32_t ta, uint32_t tab, uint32_t tabc,
                   uint32_t *src, uint32_t *dst) {
    uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32) ^ 0x524D4154u}; /* "RMAT" */
    uint32_t s = 0, d = 0;
    for (uint32_t l = 0; l < scale; l += 4) {
        uint32_t ctr[4] = {(uint32_t)e, (uint32_t)(e >> 32), l >> 2, 0u};
        uint32_t out[4];
        gwo_philox4x32_10(ctr, key, out);
        for (uint32_t j = 0; j < 4 && l + j < scale; ++j) {
            uint32_t u = out[j];
            uint32_t bit = 1u << (scale - 1 - (l + j));
            if (u < ta) {
            } else if (u < tab) {
                d |= bit;
            } else if (u < tabc) {
                s |= bit;
            } else {
                s |= bit;
                d |= bit;
            }
        }
    }
    *src = gwo_rmat_permute(s, scale, seed);
    *dst = gwo_rmat_permute(d, scale, seed);
}

/* LSD radix sort of 64-bit keys, 16 bits per pass.  Each thread counts and
 * scatters one contiguous chunk; the per-(digit, thread) offsets keep every
 * pass stable, so the result is the sequential sort's. */
static void radix_sort_u64(uint64_t *a, uint64_t *tmp, uint64_t n) {
    int nt = 1;
#ifdef _OPENMP
    nt = omp_get_max_threads();
#endif
    size_t *cnt = (size_t *)malloc((size_t)65536 * nt * sizeof(size_t));
    for (int pass = 0; pass < 4; ++pass) {
        int shift = pass * 16;
#pragma omp parallel num_threads(nt)
        {
            int t = 0;
#ifdef _OPENMP
            t = omp_get_thread_num();
#endif
            uint64_t lo = n * (uint64_t)t / nt, hi = n * (uint64_t)(t + 1) / nt;
            size_t *c = cnt + (size_t)65536 * t;
            memset(c, 0, 65536 * sizeof(size_t));
            for (uint64_t i = lo; i < hi; ++i) c[(a[i] >> shift) & 0xffff]++;
#pragma omp barrier
#pragma omp single
            {
                size_t sum = 0;
                for (int b = 0; b < 65536; ++b)
                    for (int u = 0; u < nt; ++u) {
                        size_t x = cnt[(size_t)65536 * u + b];
                        cnt[(size_t)65536 * u + b] = sum;
                        sum += x;
                    }
            }
            for (uint64_t i = lo; i < hi; ++i) tmp[c[(a[i] >> shift) & 0xffff]++] = a[i];
        }
        uint64_t *sw = a; a = tmp; tmp = sw;
    }
    /* four passes: the sorted keys are back in the caller's array */
    free(cnt);
}

uint64_t gwo_rmat_csr(uint32_t scale, uint64_t nedges_raw, uint64_t seed,
                      uint32_t ta, uint32_t tab, uint32_t tabc,
                      uint64_t *rowptr, uint32_t *colidx) {
    uint64_t nv = 1ull << scale;
    uint64_t *keys = (uint64_t *)malloc((nedges_raw ? nedges_raw : 1) * sizeof(uint64_t));
    uint64_t *tmp = (uint64_t *)malloc((nedges_raw ? nedges_raw : 1) * sizeof(uint64_t));
    /* edges are generated independently (Philox keyed on the edge index);
     * self-loops (dropped, conversions.hpp:237) become all-ones keys that
     * sort behind every real edge */
#pragma omp parallel for schedule(static)
    for (uint64_t e = 0; e < nedges_raw; ++e) {
        uint32_t s, d;
        gwo_rmat_edge(e, scale, seed, ta, tab, tabc, &s, &d);
        keys[e] = s == d ? ~0ull : ((uint64_t)s << 32) | d;
    }
    radix_sort_u64(keys, tmp, nedges_raw);
    uint64_t m = nedges_raw;
    while (m > 0 && keys[m - 1] == ~0ull) --m;
    memset(rowptr, 0, (nv + 1) * sizeof(uint64_t));
    for (uint64_t i = 0; i < m; ++i) rowptr[(keys[i] >> 32) + 1]++;
#pragma omp parallel for schedule(static)
    for (uint64_t i = 0; i < m; ++i) colidx[i] = (uint32_t)keys[i];
    for (uint64_t v = 0; v < nv; ++v) rowptr[v + 1] += rowptr[v];
    free(keys);
    free(tmp);
    return m;
}

/* ------------------------------------------------------------------------ */
/* FP64 expected visits (truncated power series).                           */
/* The per-hop continuation probability is the exact fraction of 31-bit     */
/* draws that pass the test; the neighbour choice is taken as uniform       */
/* (the r % outd bias is below outd / 2^31).                                */
/* ------------------------------------------------------------------------ */
void gwo_expected_visits(const uint64_t *rowptr, const uint32_t *colidx, uint32_t nv,
                         uint32_t src, uint32_t rule, uint32_t L, double alpha,
                         double *out) {
    uint32_t thr = gwo_continue_threshold(alpha);
    double q = (double)(0x80000000u - thr) / 2147483648.0; /* P(continue | outd > 0) */
    double *x = (double *)calloc(nv, sizeof(double));
    double *y = (double *)calloc(nv, sizeof(double));
    memset(out, 0, nv * sizeof(double));
    x[src] = 1.0;
    uint32_t nvisit_hops;
    if (rule == GWO_RULE_RESTART) nvisit_hops = L > 0 ? L - 1 : 0;
    else if (rule == GWO_RULE_PROB) nvisit_hops = 100000;
    else nvisit_hops = L;
    if (rule == GWO_RULE_RESTART && L == 1) nvisit_hops = 1;
    for (uint32_t h = 0; h < nvisit_hops; ++h) {
        double mass = 0.0;
        for (uint32_t v = 0; v < nv; ++v) { out[v] += x[v]; mass += x[v]; }
        if (mass < 1e-16) break;
        memset(y, 0, nv * sizeof(double));
        double to_src = 0.0, to_uniform = 0.0;
        for (uint32_t v = 0; v < nv; ++v) {
            double xv = x[v];
            if (xv == 0.0) continue;
            uint64_t beg = rowptr[v], deg = rowptr[v + 1] - beg;
            double fail;
            if (deg > 0) {
                double share = xv * q / (double)deg;
                for (uint64_t e = 0; e < deg; ++e) y[colidx[beg + e]] += share;
                fail = xv * (1.0 - q);
            } else {
                fail = xv;
            }
            if (rule == GWO_RULE_RESTART) to_src += fail;
            else if (rule == GWO_RULE_PPR && deg == 0) to_src += fail;
            else if (rule == GWO_RULE_JUMP) to_uniform += fail;
        }
        y[src] += to_src;
        if (to_uniform != 0.0) for (uint32_t v = 0; v < nv; ++v) y[v] += to_uniform / nv;
        double *t = x; x = y; y = t;
    }
    free(x);
    free(y);
}

/* ------------------------------------------------------------------------ */
/* SimRank meeting reduction: the triple loop of SimRank::computeResult     */
/* (apps/simrank.cpp:71-84), with the per-level pair counts kept as well.   */
/* ------------------------------------------------------------------------ */
float gwo_simrank(const uint32_t *a, const uint32_t *b, uint32_t R, uint32_t L, uint64_t *meet) {
    float simrank = 0;
    const uint64_t rr = (uint64_t)R * (uint64_t)R; /* wid_t is 64-bit (datatype.hpp:18) */
    memset(meet, 0, (size_t)L * sizeof(uint64_t));
    for (uint64_t i = 0; i < R; ++i)
        for (uint64_t j = 0; j < R; ++j)
            for (uint32_t l = 0; l < L; ++l) {
                const uint32_t x = a[i * L + l];
                if (x == b[j * L + l] && x != 0xffffffffu) {
                    simrank += (1.0 / rr) * pow(0.8, l);
                    meet[l]++;
                    break;
                }
            }
    return simrank;
}

/* ------------------------------------------------------------------------ */
/* Text edge list -> CSR: convert_to_csr (conversions.hpp:181-291).          */
/* ------------------------------------------------------------------------ */
static int is_delim(char c) { return c == '\t' || c == ',' || c == ' '; }   /* strtok(s, "\t, ") */

/* (vid_t)atoi(token): glibc atoi is (int)strtol(s, NULL, 10); leading
 * isspace() characters, an optional sign, decimal digits; strtol saturates at
 * LONG_MAX / LONG_MIN and the int conversion keeps the low 32 bits.  The
 * token never holds a delimiter, so [b, e) is the whole token. */
static uint32_t ref_atoi(const char *b, const char *e) {
    while (b < e && (*b == '\n' || *b == '\v' || *b == '\f' || *b == '\r')) ++b;
    int neg = 0;
    if (b < e && (*b == '+' || *b == '-')) { neg = *b == '-'; ++b; }
    uint64_t v = 0;
    int over = 0;
    for (; b < e && *b >= '0' && *b <= '9'; ++b) {
        if (!over) {
            if (v > (UINT64_MAX - 9) / 10) over = 1;
            else v = v * 10 + (uint64_t)(*b - '0');
        }
    }
    int64_t r;
    if (!neg) r = (over || v > (uint64_t)INT64_MAX) ? INT64_MAX : (int64_t)v;
    else r = (over || v > (uint64_t)INT64_MAX + 1) ? INT64_MIN : (int64_t)(0 - v);
    return (uint32_t)(uint64_t)r;
}

uint64_t gwo_convert_text(const char *text, uint64_t len, uint64_t *rowptr, uint32_t *colidx,
                          uint32_t *nv_out, uint64_t *ne_out) {
    uint64_t cap = 1024, ne = 0, lineno = 0;
    uint32_t *src = (uint32_t *)malloc(cap * 4), *dst = (uint32_t *)malloc(cap * 4);
    uint32_t max_vert = 0;
    uint64_t pos = 0, bad = 0;
    while (pos < len) {
        /* one fgets line: through '\n' or the end of the text */
        uint64_t end = pos;
        while (end < len && text[end] != '\n') ++end;
        if (end < len) ++end;
        ++lineno;
        if (end - pos > 1023) { bad = lineno; break; }
        const char *s = text + pos, *lim = text + end;
        pos = end;
        for (const char *z = s; z < lim; ++z) if (*z == '\0') { lim = z; break; }   /* C string end */
        if (s < lim && (s[0] == '#' || s[0] == '%')) continue;
        const char *t1 = s;
        while (t1 < lim && is_delim(*t1)) ++t1;
        const char *e1 = t1;
        while (e1 < lim && !is_delim(*e1)) ++e1;
        const char *t2 = e1;
        while (t2 < lim && is_delim(*t2)) ++t2;
        const char *e2 = t2;
        while (e2 < lim && !is_delim(*e2)) ++e2;
        if (t1 == e1 || t2 == e2) { bad = lineno; break; }
        const uint32_t from = ref_atoi(t1, e1), to = ref_atoi(t2, e2);
        if (from == to) continue;                       /* conversions.hpp:239 */
        if (from > max_vert) max_vert = from;
        if (to > max_vert) max_vert = to;
        if (ne == cap) {
            cap *= 2;
            src = (uint32_t *)realloc(src, cap * 4);
            dst = (uint32_t *)realloc(dst, cap * 4);
        }
        src[ne] = from;
        dst[ne] = to;
        ++ne;
    }
    if (!bad) {
        const uint64_t nv = (uint64_t)max_vert + 1;
        if (nv_out) *nv_out = (uint32_t)nv;
        if (ne_out) *ne_out = ne;
        if (rowptr && colidx) {   /* stable counting sort by source */
            memset(rowptr, 0, (nv + 1) * sizeof(uint64_t));
            for (uint64_t i = 0; i < ne; ++i) rowptr[src[i] + 1]++;
            for (uint64_t v = 0; v < nv; ++v) rowptr[v + 1] += rowptr[v];
            uint64_t *fill = (uint64_t *)malloc(nv * sizeof(uint64_t));
            memcpy(fill, rowptr, nv * sizeof(uint64_t));
            for (uint64_t i = 0; i < ne; ++i) colidx[fill[src[i]]++] = dst[i];
            free(fill);
        }
    }
    free(src);
    free(dst);
    return bad;
}

/*
 * gw_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of GraphWalker's random-walk hot path.  Its results
 * are those of a sequential loop; the loops over independent items (walks,
 * generated edges) run on the host's threads with OpenMP so that the
 * configs' full sizes can be checked in seconds.  It is used by tests/,
 * __graft_entry__.smoke() and bench.py's cpu_baseline leg as the checker.  Nothing in graphwalker_b200/ links, loads or calls
 * this code; the product path is the CUDA library only.
 *
 * Parity pin: the restatement is checked against golden vectors produced by
 * the reference's own engine and walk classes (compiled from source with a
 * test-only RNG shim, see oracle/ref_shim/) in tests/test_oracle_golden.py.
 *
 * Every function cites the reference file:line whose behaviour it restates
 * (paths relative to the GraphWalker project root).
 */
#ifndef GW_ORACLE_H
#define GW_ORACLE_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Walk update rules (one per live RandomWalk subclass, plus the PPR rule of
 * the single-source PPR workload, which is not a reference class). */
enum {
    GWO_RULE_JUMP = 0,    /* src/walks/randomwalkwithjump.hpp:30-62        */
    GWO_RULE_STOP = 1,    /* src/walks/randomwalkwithstop.hpp:20-52        */
    GWO_RULE_PROB = 2,    /* src/walks/randomwalkwithprob.hpp:20-57        */
    GWO_RULE_RESTART = 3, /* src/walks/randomwalkwithrestartwithjoint.hpp:29-61 */
    GWO_RULE_PPR = 4      /* stop w.p. alpha, dangling -> back to source   */
};

/* Status bits (mirrors the device status word). */
enum {
    GWO_ST_BOUNDS = 1,    /* a walk reached a vertex id >= nvertices       */
    GWO_ST_PATH_OVF = 2,  /* a walk made more visits than path_stride      */
    GWO_ST_HOP_OVF = 4    /* an uncapped walk exceeded max_hops            */
};

/* Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as
 * easy as 1, 2, 3", SC'11).  out = Philox(key, ctr). */
void gwo_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);

/* Smallest r in [0, 2^31) for which the reference's continuation test
 * `(float)r/RAND_MAX > p` holds (randomwalkwithjump.hpp:45 and siblings;
 * RAND_MAX from src/api/datatype.hpp:8).  Evaluates the float expression
 * itself by bisection; returns 2^31 if no r passes. */
uint32_t gwo_continue_threshold(double p);

/* Evaluates the reference's continuation test literally for one r: the
 * quotient is computed in float and compared with the double p, exactly as
 * the reference's `(float)rand_r(&seed)/RAND_MAX > 0.15` does. */
int gwo_continue_test(uint32_t r, double p);

/* Number of r in [0, 2^31) where `r >= gwo_continue_threshold(p)` disagrees
 * with the float test (exhaustive; 0 expected). */
uint64_t gwo_threshold_mismatches(double p);

/* The reference's 64-bit walk word (src/walks/walk.hpp:69-91). */
uint64_t gwo_encode(uint32_t source, uint32_t current, uint32_t hop);
uint32_t gwo_get_source(uint64_t w);
uint32_t gwo_get_current(uint64_t w);
uint32_t gwo_get_hop(uint64_t w);

typedef struct {
    uint32_t rule;         /* GWO_RULE_*                                      */
    uint32_t L;            /* walk length cap / restart segment length        */
    double   jump_prob;    /* else-branch probability (the double literal 0.15 in the ref) */
    uint32_t njump;        /* N of `rand_r % N` in the jump rule               */
    uint64_t seed;         /* Philox key                                      */
    uint32_t max_hops;     /* hop guard for the uncapped rule                 */
    uint32_t rng;          /* 0: draws of hop h = words 0, 1 of Philox(id, h, 0, 0)
                              (the reference's per-hop draw, shimmed); 1: the
                              engine's native-RNG layout, words 0-1 (even h) or
                              2-3 (odd h) of Philox(id, h / 2, 0, "NATV")      */
} gwo_params;

/*
 * Runs every walk to its end over a whole-graph CSR, exactly as the
 * reference's block engine would with every block resident (the engine's
 * block boundaries never change a trajectory once the per-hop draws are
 * keyed on (seed, walk id, hop)).
 *
 * walk i starts at vertex cur[i] with hop hop0[i]; id[i] keys its Philox
 * stream; src[i] is its source (restart target / sink key).
 *
 * Outputs (each may be NULL):
 *   counts[nv]          += 1 per visit of a vertex            (rwdomination sink)
 *   paths[i*stride + k]  = k-th visited vertex of walk i       (simrank sink)
 *   plen[i]              = number of visits of walk i
 *   closure             += walks with a visit at hop >= L-1 equal to src (graphlet)
 *   final_cur/final_hop  = state when the walk ended
 * Returns a bitmask of GWO_ST_*.
 */
uint32_t gwo_run_walks(const uint64_t *rowptr, const uint32_t *colidx, uint32_t nv,
                       const uint32_t *cur, const uint32_t *id, const uint32_t *src,
                       const uint32_t *hop0, uint64_t nwalks, const gwo_params *p,
                       uint32_t *counts, uint32_t *paths, uint32_t stride, uint32_t *plen,
                       uint64_t *closure, uint32_t *final_cur, uint32_t *final_hop);

/*
 * One block-engine superstep for the walks of one block, restating
 * updateByWalk's in-block loop: a walk advances while its vertex lies in
 * [blocks[b], blocks[b+1]) and it is alive; on leaving it is handed to
 * getblock(v) (src/walks/randomwalk.hpp:74-82).
 * dest[i] = destination block, or 0xffffffff when the walk ended.
 * cur/hop are updated in place.  counts may be NULL.
 */
uint32_t gwo_block_step(const uint64_t *rowptr, const uint32_t *colidx, uint32_t nv,
                        const uint32_t *blocks, uint32_t nblocks, uint32_t b,
                        uint32_t *cur, const uint32_t *id, const uint32_t *src, uint32_t *hop,
                        uint64_t n, const gwo_params *p, uint32_t *counts, uint32_t *dest);

/* Block boundaries from a CSR row pointer, restating compute_block
 * (src/preprocess/conversions.hpp:300-364) including its split rule for a
 * vertex whose degree alone exceeds the budget.  rowptr has nv+1 entries.
 * Writes up to cap entries into blocks; returns the number of boundary
 * entries (nblocks + 1), or 0 if cap is too small. */
uint32_t gwo_compute_blocks(const uint64_t *rowptr, uint32_t nv, uint64_t blocksize_kb,
                            uint32_t *blocks, uint32_t cap);

/* Linear block lookup, restating RandomWalk::getblock
 * (src/walks/randomwalk.hpp:74-82): returns nblocks when v >= blocks[nblocks]. */
uint32_t gwo_getblock(const uint32_t *blocks, uint32_t nblocks, uint32_t v);

/* --- seeded R-MAT graph (synthetic stand-in for the reference datasets) --- */

/* Keyed bijection of [0, 2^scale) used to permute vertex ids. */
uint32_t gwo_rmat_permute(uint32_t v, uint32_t scale, uint64_t seed);

/* Edge e of the R-MAT stream before self-loop removal, after permutation. */
void gwo_rmat_edge(uint64_t e, uint32_t scale, uint64_t seed,
                   uint32_t ta, uint32_t tab, uint32_t tabc,
                   uint32_t *src, uint32_t *dst);

/* Builds the CSR of R-MAT(scale, nedges_raw): edges generated by
 * gwo_rmat_edge, self-loops removed, duplicates kept, rows sorted by
 * (src, dst).  rowptr must hold 2^scale+1 entries, colidx nedges_raw.
 * Returns the number of edges kept. */
uint64_t gwo_rmat_csr(uint32_t scale, uint64_t nedges_raw, uint64_t seed,
                      uint32_t ta, uint32_t tab, uint32_t tabc,
                      uint64_t *rowptr, uint32_t *colidx);

/* --- FP64 truncated power series for the PPR-type rules --- */

/* Expected visits per vertex of ONE walk started at src, for rules STOP and
 * PPR (capped at L hops) and RESTART (L-1 visits per segment), computed by
 * propagating the exact per-hop distribution.  out[nv]. */
void gwo_expected_visits(const uint64_t *rowptr, const uint32_t *colidx, uint32_t nv,
                         uint32_t src, uint32_t rule, uint32_t L, double alpha,
                         double *out);

/* --- text edge list -> CSR (src/preprocess/conversions.hpp:181-291) --- */

/* The reference's convert_to_csr on text[0, len): lines as fgets reads them,
 * '#'/'%' comment lines skipped, the first two strtok tokens (delimiters tab,
 * comma, space) converted by atoi into vid_t (the low 32 bits of strtol),
 * self-loops dropped, duplicates kept.  Lines are grouped by source with a
 * stable sort (the reference expects them grouped already, in which case
 * the sort changes nothing).  nv = largest vertex id seen + 1 (1 when there
 * are no edges).  With rowptr/colidx NULL only *nv and *ne are computed;
 * otherwise rowptr[nv + 1] and colidx[ne] are filled.  Returns 0, or the
 * 1-based number of the first line the reference rejects (fewer than two
 * tokens) or that is longer than 1023 bytes (fgets would split it). */
uint64_t gwo_convert_text(const char *text, uint64_t len, uint64_t *rowptr, uint32_t *colidx,
                          uint32_t *nv, uint64_t *ne);

/* --- SimRank meeting reduction (apps/simrank.cpp:71-84, computeResult) --- */

/* a and b hold R walks of L visits each (walk i = a[i*L .. i*L+L-1],
 * 0xFFFFFFFF = no visit).  For every pair (i, j) the first l < L with
 * a[i*L+l] == b[j*L+l] != 0xFFFFFFFF is counted in meet[l] (meet[L] zeroed
 * first).  Returns the app's estimate accumulated as the app does: a float
 * sum over i, then j, of (1.0 / (R*R)) * pow(0.8, l), R*R in 64-bit. */
float gwo_simrank(const uint32_t *a, const uint32_t *b, uint32_t R, uint32_t L, uint64_t *meet);

#ifdef __cplusplus
}
#endif
#endif

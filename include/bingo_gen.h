/*
 * bingo_gen.h - seeded synthetic workloads for the walk engine (host code).
 *
 * The reference reads edge lists from ../dataset/<NAME> (include/graph.cuh:22-27)
 * and makes its update batches from copies of existing pairs
 * (include/graph.cuh:58-92); those datasets are not available, so the engine's
 * tests and benchmarks use these generators instead. All output is a pure
 * function of the arguments (counter-based Philox4x32-10 per item), so it does
 * not depend on the thread count.
 */
#ifndef BINGO_GEN_H
#define BINGO_GEN_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* weight distributions */
#define BINGO_W_UNIFORM 0    /* integer uniform in [lo, hi] */
#define BINGO_W_LOGUNIFORM 1 /* floor(lo * (hi/lo)^U), U uniform in [0,1), clamped to [lo, hi-1] */
#define BINGO_W_ZIPF 2       /* P(w = x) ~ x^-s on [lo, hi] (Hoermann-Derflinger rejection-inversion) */

/* R-MAT (Chakrabarti, Zhan, Faloutsos, SDM 2004): ef * 2^scale draws with
 * quadrant probabilities a, b, c (d = 1-a-b-c); self-loops and duplicate
 * (src, dst) pairs are dropped. Edges come out sorted by (src, dst).
 * src and dst must hold edge_factor << scale entries (NULL: count only).
 * Returns the edge count m. */
uint64_t bingo_gen_rmat(uint32_t scale, uint32_t edge_factor, double a, double b, double c, uint64_t seed,
                        uint32_t* src, uint32_t* dst);

/* w[i] for i in [0, m), drawn from stream (seed, i). */
void bingo_gen_weights(uint64_t m, int dist, double lo, double hi, double s, uint64_t seed, uint32_t* w);

/* Stateful update-batch generator mirroring the reference's insertGraph /
 * deleteGraph roles: it tracks every live (u, v, slot) and each vertex's
 * slot counter exactly as the engine assigns slots (append order). */
typedef struct bingo_updgen bingo_updgen;

bingo_updgen* bingo_updgen_create(uint32_t n, const uint32_t* src, const uint32_t* dst, uint64_t m, uint64_t seed);
void bingo_updgen_destroy(bingo_updgen* g);
/* k inserts of pairs absent from the live graph (no self-loops, distinct
 * within the batch), u and v uniform in [0, n), weights from dist. The
 * generator records the slots the engine will assign. Returns k. */
uint64_t bingo_updgen_inserts(bingo_updgen* g, uint64_t k, int dist, double lo, double hi, double s, uint32_t* src,
                              uint32_t* dst, uint32_t* w);
/* k deletes drawn uniformly without replacement from the live edges, as
 * (u, slot). Returns the number produced (<= live edges). */
uint64_t bingo_updgen_deletes(bingo_updgen* g, uint64_t k, uint32_t* u, uint32_t* slot);
uint64_t bingo_updgen_live(const bingo_updgen* g);

/* ---- The reference's own inputs ------------------------------------------
 * Edge-list files as the reference's loadGraph() reads them
 * (include/graph.cuh:22-27): whitespace-separated "u v" pairs of
 * non-negative decimal ids, one edge per pair, kept in file order (self-loops
 * and duplicates too, as the reference keeps them). Unlike the reference's
 * scanf loop, lines starting with '#' or '%' (SNAP / Matrix Market headers)
 * are skipped. Ids stay as in the file (the engine is 0-based; the reference
 * adds 1 and keeps vertex 0 as scratch), and n = largest id + 1.
 *
 * Two calls: bingo_edge_list_read(path, NULL, NULL, 0, &m, &n) counts;
 * a second call with arrays of at least m entries fills them. Returns 0, or
 * -1 (cannot open / read), -2 (malformed token at byte offset *m), -3
 * (arrays too small), -4 (an id above 2^32 - 2). */
int bingo_edge_list_read(const char* path, uint32_t* src, uint32_t* dst, uint64_t cap, uint64_t* m, uint32_t* n);

/* Load weights of the reference driver (include/graph.cuh:43-51,
 * include/api.h:29-30): w = trunc(bias(d(v))) + 1 with d(v) the out-degree
 * of the edge's destination over the edge list, bias(d) = d
 * (BINGO_DRIVER_DEGREE) or (float)pow(d, 0.3) (BINGO_DRIVER_DEGREE_POW03);
 * BINGO_DRIVER_AUTO picks the second when n > 1e7, as the reference does.
 * Returns 0, or -1 for an unknown kind or an id >= n. */
#define BINGO_DRIVER_AUTO 0
#define BINGO_DRIVER_DEGREE 1
#define BINGO_DRIVER_DEGREE_POW03 2
int bingo_driver_weights(int kind, const uint32_t* src, const uint32_t* dst, uint64_t m, uint32_t n, uint32_t* w);

#ifdef __cplusplus
}
#endif

#endif /* BINGO_GEN_H */

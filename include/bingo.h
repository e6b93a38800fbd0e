/*
 * bingo.h - C ABI of the B200 radix bias-factorization walk engine.
 *
 * The reference has no library boundary: its operator surface is a set of
 * C++ host functions and CUDA kernels called from its graph driver
 * (include/graph.cuh). Each entry point below names the reference interface
 * it replaces. Every function returns a bingo_status (0 = BINGO_OK); no C++
 * exception crosses this boundary. Vertex ids are 0-based in [0, n).
 *
 * Pointers: every array argument may be host memory (pageable or pinned) or
 * device memory on the handle's device; the library detects which. Calls are
 * ordered on the handle's CUDA stream. With cfg.synchronous != 0 (the
 * default) each call returns only after its device work is complete and
 * reports device-detected errors directly; otherwise such errors surface at
 * the next bingo_sync(), and walk rows bound for host memory are complete
 * only after it: they are copied out on a second stream while the next
 * calls' device work runs.
 *
 * Threading: one handle may be used by one host thread at a time.
 */
#ifndef BINGO_H
#define BINGO_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct bingo_handle bingo_handle;

typedef enum bingo_status {
  BINGO_OK = 0,
  BINGO_ERR_INVALID_ARGUMENT = 1, /* null pointer, bad enum, bad config */
  BINGO_ERR_OUT_OF_RANGE = 2,     /* a vertex id >= n */
  BINGO_ERR_ZERO_WEIGHT = 3,      /* an inserted or loaded weight of 0 */
  BINGO_ERR_INVALID_SLOT = 4,     /* delete of an absent or already deleted slot (skipped) */
  BINGO_ERR_CAPACITY = 5,         /* the graph arena (HBM budget) cannot hold the batch */
  BINGO_ERR_CUDA = 6,             /* a CUDA runtime call failed; see bingo_last_error */
  BINGO_ERR_NOT_LOADED = 7,       /* operation needs a loaded graph */
  BINGO_ERR_TIMEOUT = 8,          /* a bounded device wait expired */
  BINGO_ERR_NO_DEVICE = 9,        /* no usable CUDA device */
  BINGO_ERR_UNSUPPORTED = 10,     /* e.g. node2vec without the adjacency index */
  BINGO_ERR_BUSY = 11,            /* the handle is serving; only bingo_serve_* calls are allowed */
  BINGO_ERR_CORRUPT = 12          /* the graph store breaks an invariant (bingo_check; a restored snapshot) */
} bingo_status;

typedef enum bingo_app {
  BINGO_DEEPWALK = 0, /* include/operation.cuh:252 deepwalkKernel */
  BINGO_NODE2VEC = 1, /* include/operation.cuh:281 node2vecKernel */
  BINGO_PPR = 2,      /* include/operation.cuh:336 pprKernel */
  BINGO_SAMPLING = 3  /* include/operation.cuh:407 samplingKernel (one hop) */
} bingo_app;

/* bingo_walk_job.flags */
#define BINGO_WALK_PPR_TAIL 1u /* PPR keeps walking past the last slot and overwrites it,
                                  as include/operation.cuh:353-360 does */

/* bingo_walk() mode */
#define BINGO_WALK_BATCHED 0u /* all jobs in one persistent launch over a device work queue */
#define BINGO_WALK_PLAIN 1u   /* one launch per job, the reference's per-job form */

/* Weight modes. U32: integer weights >= 1 (the reference's wtype::Int).
 * F32: float weights in (0, 65536) (the reference's wtype::Float, whose
 * integer part is limited to MAXLOG = 16 bits, include/api.h:11), kept as
 * 16.16 fixed point q = round_half_even(w * 2^16): every kernel then runs
 * unchanged and draws exactly in proportion to q, so each probability is
 * within 2^-17 / w relative of the float weight's. In F32 mode every uint32
 * weight the API takes or returns (bingo_run, serving updates, dumps) is such
 * a fixed-point value; bingo_weights_to_fixed16 converts. */
#define BINGO_WEIGHTS_U32 0
#define BINGO_WEIGHTS_F32 1

typedef struct bingo_config {
  int32_t device;         /* CUDA device ordinal */
  uint32_t node2vec;      /* maintain the adjacency index node2vec needs (like NODE2VEC, include/api.h:25) */
  uint32_t synchronous;   /* 1: every call waits for its device work (default) */
  uint32_t weight_mode;   /* BINGO_WEIGHTS_U32 (default) or BINGO_WEIGHTS_F32 */
  double arena_factor;    /* graph arena = factor x bytes needed at load (default 2.0) */
  uint64_t arena_bytes;   /* minimum graph arena bytes; 0 = from arena_factor only */
} bingo_config;

typedef struct bingo_walk_job {
  int32_t app;            /* bingo_app */
  uint32_t length;        /* positions per walk, start included (reference LEN=80) */
  const uint32_t* starts; /* start vertices; NULL = the range [first, first + n_starts) */
  uint64_t n_starts;
  uint32_t first;
  uint32_t job_id;        /* Philox counter word 3 */
  uint64_t seed;          /* Philox key */
  uint32_t flags;         /* BINGO_WALK_* */
  uint32_t reserved0;
  double p, q;            /* node2vec return / in-out parameters (reference P=0.5, Q=2) */
  double stop_prob;       /* PPR termination probability (reference TP=0.0125) */
  int32_t* out;           /* [n_starts][length] vertex ids, -1 after a dead end or stop;
                             sampling: [n_starts]. Device outputs of walk apps must be
                             32-byte aligned (rows are written a sector at a time). */
} bingo_walk_job;

typedef struct bingo_stats {
  uint32_t n;             /* vertices */
  uint32_t weight_mode;   /* the handle's BINGO_WEIGHTS_* */
  uint64_t slots;         /* edge slots including tombstones */
  uint64_t live_edges;
  uint64_t arena_bytes;   /* bytes reserved for the graph arenas */
  uint64_t arena_used;    /* bytes handed out (live + abandoned by growth) */
  uint64_t scratch_bytes; /* staging and sort scratch currently held */
  uint64_t walk_steps;    /* walk steps produced since bingo_create (moves to a neighbour) */
  uint64_t kernel_launches; /* engine kernels launched since bingo_create (library sort/scan/select
                               kernels not included) */
  uint64_t walk_trials;   /* node2vec proposals drawn since bingo_create (one alias draw each) */
  uint64_t walk_probes;   /* node2vec adjacency-index lookups since bingo_create */
} bingo_stats;

/* Defaults for bingo_config (device 0, node2vec on, synchronous, factor 2). */
void bingo_config_init(bingo_config* cfg);

/* Replaces the global device state of include/graph.cuh:9-14 and MemPool::init
 * (include/gpuMem.cuh:15-24). */
int bingo_create(const bingo_config* cfg, bingo_handle** out);
int bingo_destroy(bingo_handle* h);

/* Message of the last failing call on this handle (or of bingo_create when h is NULL). */
const char* bingo_last_error(const bingo_handle* h);

/* Replaces build(Edges*, int amount, NodeData**, NodeData**, int* d, int** sizeManager, int n)
 * (include/operation.cuh:33). Edges of one source keep their input order as
 * slots 0..deg-1 (the stable bucket of include/operation.cuh:82-90). */
int bingo_load_edges(bingo_handle* h, const uint32_t* src, const uint32_t* dst, const uint32_t* w, uint64_t m,
                     uint32_t n);

/* Replaces insert(Edges*, int amount, NodeData**, NodeData**, int* d, int* sizeManager)
 * (include/operation.cuh:144). Edges append to their source in batch order
 * (the stable_sort of include/operation.cuh:147). out_slots (may be NULL)
 * receives each edge's slot id, the id the reference caller tracks as d[u]++
 * (include/graph.cuh:66) and later passes to delete. Weight 0 is rejected.
 * The call waits on the host until the batch is validated and its arena
 * space reserved (the apply kernel already runs meanwhile; a batch that did
 * not fit is applied again after the arenas grow), so even on an
 * asynchronous handle a rejected batch is reported by this call, with
 * nothing applied. */
int bingo_insert_batch(bingo_handle* h, const uint32_t* src, const uint32_t* dst, const uint32_t* w, uint64_t k,
                       uint32_t* out_slots);

/* Replaces deleteE(Deleted*, int amount, NodeData**) (include/operation.cuh:215)
 * with (u, slot) pairs (include/type.h:32-35). Deletes of one vertex apply in
 * batch order; a slot that is absent or already deleted is skipped and the
 * call returns BINGO_ERR_INVALID_SLOT after applying the rest. */
int bingo_delete_batch(bingo_handle* h, const uint32_t* u, const uint32_t* slot, uint64_t k);

/* Float-weight forms of bingo_load_edges / bingo_insert_batch for handles
 * created with weight_mode = BINGO_WEIGHTS_F32 (the reference's
 * wtype::Float load and insert, include/Bingo.cuh:65-69, :176-177, :189-190).
 * The reference keeps the fractional parts as one remainder group drawn by
 * rejection over all slots (include/Bingo.cuh:254-264); here the weight is
 * quantised to 16.16 fixed point and lands in the bit groups like any other.
 * A weight that is not in (0, 65536), or that rounds to 0 (w < 2^-17),
 * rejects the whole batch (BINGO_ERR_ZERO_WEIGHT for w <= 0, NaN or w
 * rounding to 0; BINGO_ERR_OUT_OF_RANGE for w >= 65536). */
int bingo_load_edges_f32(bingo_handle* h, const uint32_t* src, const uint32_t* dst, const float* w, uint64_t m,
                         uint32_t n);
int bingo_insert_batch_f32(bingo_handle* h, const uint32_t* src, const uint32_t* dst, const float* w, uint64_t k,
                           uint32_t* out_slots);
/* Host conversion to the F32 mode's fixed point (same rounding as the
 * device); invalid weights become 0. Returns the number of invalid weights. */
uint64_t bingo_weights_to_fixed16(const float* w, uint64_t k, uint32_t* out);

/* Delete by (u, v) pair; no reference counterpart (the reference deletes by
 * slot only, include/operation.cuh:215). The r-th occurrence of a pair in the
 * batch deletes the r-th lowest live slot of u whose neighbour is v; the
 * translated (u, slot) batch then applies exactly as bingo_delete_batch.
 * Pairs with no such slot are skipped and the call returns
 * BINGO_ERR_INVALID_SLOT after applying the rest. */
int bingo_delete_pairs(bingo_handle* h, const uint32_t* u, const uint32_t* v, uint64_t k);

/* Replaces the walk kernels deepwalkKernel / node2vecKernel / pprKernel /
 * samplingKernel<<<BLKSZ, THDSZ>>>(gId, pId, n, NodeData*, int* rwD, PIECESIZE, seed)
 * (include/operation.cuh:252, :281, :336, :407) and the randomWalk driver
 * (include/graph.cuh:93). Output rows match rwD ([walk][length]). mode is
 * BINGO_WALK_BATCHED or BINGO_WALK_PLAIN; both give identical results. */
int bingo_walk(bingo_handle* h, const bingo_walk_job* jobs, uint32_t n_jobs, uint32_t mode);

/* Allocation-free walks. No counterpart in the reference: this entry point
 * exists for callers that cannot call cudaMalloc while they run - a serving
 * loop whose HBM is already budgeted to the graph and its query outputs, or
 * an application that owns the device memory pool and forbids allocations
 * outside it. It runs the same walks as
 * bingo_walk(jobs, n_jobs, BINGO_WALK_BATCHED), with identical results, but
 * takes its scratch (job table, walk offsets and work counter, 6.4 KB) from a
 * fixed array compiled into the library instead of allocating it, and calls
 * neither cudaMalloc nor cudaFree nor any allocating library routine. The job
 * table reaches that array as a kernel parameter, so nothing is read from the
 * caller's host memory after the call returns.
 *
 * Limits: at most 64 jobs per call (more returns BINGO_ERR_INVALID_ARGUMENT);
 * every start array must be device memory or NULL and every output device
 * memory (32-byte aligned for walk apps), since host buffers would need
 * staging memory. The scratch array is shared by every call on a device and
 * keeps the last call's contents (the work counter is zeroed by each call);
 * calls whose work overlaps on the GPU (two streams, or two handles on one
 * device, at once) race on it, so issue them in order on one stream. The
 * first call on each device looks up the array's device address
 * (cudaGetSymbolAddress, with that device current); make that first call
 * before any stream capture. */
int bingo_walk_noalloc(bingo_handle* h, const bingo_walk_job* jobs, uint32_t n_jobs);

/* ---- Batched programs -------------------------------------------------
 * A program is an ordered list of walk-job sets and update batches executed
 * with no host synchronisation between them (the reference runs the same
 * sequence as separate synchronous calls, include/apps.cu:24-31). Each op
 * sees the graph as left by the ops before it. All arrays must be device
 * memory (starts may be NULL). With BINGO_RUN_GRAPH the program is captured
 * once into a CUDA graph and replayed while its shape (op kinds, batch sizes,
 * walk counts per job, array addresses) stays the same; walk-job contents
 * (apps, lengths, seeds, p/q, stop probabilities) may change between
 * replays. Update capacity is checked on the device: a batch that does not
 * fit the graph arenas is not applied and the call returns
 * BINGO_ERR_CAPACITY (the arenas are grown before the next call). */
typedef enum bingo_op_kind {
  BINGO_OP_WALK = 0,
  BINGO_OP_INSERT = 1,
  BINGO_OP_DELETE = 2,
  BINGO_OP_DELETE_PAIRS = 3 /* delete by (u, v) as bingo_delete_pairs */
} bingo_op_kind;

typedef struct bingo_op {
  int32_t kind;               /* bingo_op_kind */
  uint32_t n_jobs;            /* WALK: jobs in this set, run as one persistent launch */
  const bingo_walk_job* jobs; /* WALK */
  const uint32_t* a;          /* INSERT: src   DELETE: vertex   DELETE_PAIRS: u */
  const uint32_t* b;          /* INSERT: dst   DELETE: slot     DELETE_PAIRS: v */
  const uint32_t* c;          /* INSERT: weight */
  uint64_t k;                 /* INSERT / DELETE / DELETE_PAIRS: batch size */
  uint32_t* out_slots;        /* INSERT: slot ids (device, may be NULL) */
} bingo_op;

#define BINGO_RUN_GRAPH 1u

int bingo_run(bingo_handle* h, const bingo_op* ops, uint32_t n_ops, uint32_t flags);

/* ---- Serving -----------------------------------------------------------
 * Continuous batching of walk queries with interleaved update batches (the
 * reference has no serving mode). Walk queries are admitted into a running
 * device-resident walk loop as job slots and output memory free up, and
 * their walks run mixed with those of every other admitted query. An update
 * batch commits after every walk query submitted before it has finished,
 * and before any query submitted after it starts, so a query sees the graph
 * after exactly the updates submitted before it (its `version`), and its
 * rows equal those of the same query run alone on that graph.
 *
 * Query inputs are copied at submit; `out` (host or device) must stay valid
 * until the ticket is done. Admission: a query must fit the output budget
 * (rows + starts), at most max_jobs queries are in flight. While serving,
 * other calls on the handle return BINGO_ERR_BUSY. */
typedef struct bingo_serve_config {
  uint64_t output_budget_bytes; /* device memory for in-flight query rows and starts (default 1 GiB) */
  uint32_t max_jobs;            /* queries in flight, <= 4096 (default 4096) */
  uint32_t max_update_batch;    /* update batches apply in chunks of at most this many edges (default 2^20) */
  uint32_t idle_timeout_us;     /* the walk loop exits after this long without work (default 2000) */
  uint32_t reserved0;
} bingo_serve_config;

typedef struct bingo_serve_status {
  int32_t done;        /* 1 when the request has finished */
  int32_t status;      /* bingo_status of the request */
  int32_t kind;        /* 0 walk, 1 insert, 2 delete */
  int32_t reserved0;
  uint64_t version;    /* updates applied before this request (walks) / including it (updates) */
  uint64_t latency_ns; /* submit to result ready */
  uint64_t ready_ns;   /* when the result became ready, CLOCK_MONOTONIC nanoseconds */
} bingo_serve_status;

int bingo_serve_start(bingo_handle* h, const bingo_serve_config* cfg);
int bingo_serve_submit_walk(bingo_handle* h, const bingo_walk_job* job, uint64_t* ticket);
/* kind: BINGO_OP_INSERT (a = src, b = dst, c = weights, out_slots optional),
 * BINGO_OP_DELETE (a = vertex, b = slot) or BINGO_OP_DELETE_PAIRS (a = u,
 * b = v, as bingo_delete_pairs). The batch is copied at submission. It
 * applies after every walk submitted before it has finished on the device
 * and before any walk submitted after it starts; its ticket is done once the
 * batch has applied, with the batch's own status (a delete batch with absent
 * or repeated slots applies the rest and reports BINGO_ERR_INVALID_SLOT).
 * out_slots (host memory) holds the slot ids once the ticket is done. */
int bingo_serve_submit_update(bingo_handle* h, int32_t kind, const uint32_t* a, const uint32_t* b,
                              const uint32_t* c, uint64_t k, uint32_t* out_slots, uint64_t* ticket);
int bingo_serve_poll(bingo_handle* h, uint64_t ticket, bingo_serve_status* out);
/* Waits at most timeout_us; returns BINGO_ERR_TIMEOUT if the ticket is not done. */
int bingo_serve_wait(bingo_handle* h, uint64_t ticket, uint64_t timeout_us, bingo_serve_status* out);
/* ---- Snapshots ------------------------------------------------------------
 * No reference counterpart (the reference rebuilds its graph from the edge
 * list on every start). bingo_save writes the whole graph store (every slot,
 * tombstone, group list, back-pointer, alias table and adjacency entry) to a
 * file; bingo_restore replaces the handle's graph with a file's, so a
 * restored handle walks and updates exactly like the one that saved it. The
 * file is checksummed and tied to this build's record layout and to
 * config.node2vec; a restore that fails leaves the handle with no graph. */
int bingo_save(bingo_handle* h, const char* path);
/* The restored store is checked as by bingo_check before the handle takes
 * it; a file whose content breaks an invariant (with a valid checksum)
 * returns BINGO_ERR_CORRUPT and leaves the handle with no graph. */
int bingo_restore(bingo_handle* h, const char* path);

/* ---- Store check ----------------------------------------------------------
 * No reference counterpart (the reference has no consistency checker). One
 * device pass over the whole store verifies every structural invariant the
 * walk and update kernels rely on, reading each record only after the
 * offsets that lead to it were checked against the used part of its arena
 * (so a corrupt store yields a report, never an out-of-bounds access):
 *   EXTENT  a vertex's edge slots, back-pointer pool, group lists, alias
 *           table or adjacency index reach past the used part of its arena,
 *           or a count exceeds its capacity;
 *   COUNT   the live-slot count or a group's member count differs from the
 *           live slots carrying that weight bit;
 *   MEMBER  a group member names (through the back-pointer index it holds)
 *           a slot that is not live, lacks the group's bit or holds another
 *           neighbour, or its back-pointer disagrees;
 *   ALIAS   the alias table is not the exact table over the group masses
 *           cnt_k * 2^k (slot count, totals, own / alias groups, and for
 *           every group the scaled mass its slots carry);
 *   HASH    a live neighbour is missing from the adjacency index, or the
 *           index's key, multiplicity or weight totals disagree;
 *   RANGE   a live slot holds a neighbour id >= n.
 * Returns BINGO_OK with a clean report, BINGO_ERR_CORRUPT with the report
 * filled when any vertex fails. */
enum {
  BINGO_CHECK_EXTENT = 1,
  BINGO_CHECK_COUNT = 2,
  BINGO_CHECK_MEMBER = 4,
  BINGO_CHECK_ALIAS = 8,
  BINGO_CHECK_HASH = 16,
  BINGO_CHECK_RANGE = 32
};
typedef struct bingo_check_report {
  uint64_t vertices;       /* vertices checked (= n) */
  uint64_t live_edges;     /* live (non-tombstone) edge slots */
  uint64_t weight_sum;     /* sum of the live weights, modulo 2^64 */
  uint64_t members;        /* group members over all vertices (= sum of popcount(w) over live slots) */
  uint64_t alias_slots;    /* alias slots over all vertices (= nonzero groups) */
  uint64_t bad_vertices;   /* vertices failing at least one check */
  uint32_t kinds;          /* BINGO_CHECK_* bits seen */
  uint32_t first_bad;      /* lowest failing vertex id, or 0xffffffff */
} bingo_check_report;
int bingo_check(bingo_handle* h, bingo_check_report* out);

/* ---- Tuning -------------------------------------------------------------
 * Launch and batching parameters. None of them changes any result (walks,
 * slot ids, graph state); bingo_autotune picks them by measurement. */
typedef struct bingo_tuning {
  uint32_t walk_chunk;          /* walks a warp claims per refill, 1..1024; 0 (default) = each walk
                                   kernel's measured default: 8 for DeepWalk, 32 otherwise */
  uint32_t walk_blocks_per_sm;  /* resident walk blocks per SM, capped by occupancy; 0 (default) =
                                   each walk kernel's measured default: 4 for DeepWalk and PPR, the
                                   occupancy limit otherwise */
  uint32_t walk_split;          /* 1: one persistent launch per app; 0: one mixed launch (default) */
  uint32_t walk_order;          /* 1: jobs with the longest expected walks first (default); 0: job order */
  uint32_t update_chunk;        /* edges per update sub-batch of bingo_insert_batch / bingo_delete_batch,
                                   0 = the whole batch (default) */
  uint32_t apply_blocks_per_sm; /* blocks per SM of the insert / delete apply kernels, 1..32 (default 8) */
  uint32_t reserved[2];
} bingo_tuning;

int bingo_get_tuning(bingo_handle* h, bingo_tuning* out);
int bingo_set_tuning(bingo_handle* h, const bingo_tuning* t);

/* Sample workload for bingo_autotune. The walk jobs follow bingo_walk
 * (BINGO_WALK_BATCHED; their outputs are overwritten). The optional update
 * batch (inserts, then deletes by slot valid against the current graph) is
 * timed on the handle's graph and undone from a device copy taken first, so
 * the graph is unchanged when the call returns; without room for the copy
 * the update knobs are left as they are. */
typedef struct bingo_tune_request {
  const bingo_walk_job* jobs;
  uint32_t n_jobs;
  uint32_t repeats;  /* timed runs per candidate (0 = 3); the median counts */
  const uint32_t *ins_src, *ins_dst, *ins_w;
  uint64_t n_ins;
  const uint32_t *del_u, *del_slot;
  uint64_t n_del;
} bingo_tune_request;

typedef struct bingo_tune_report {
  bingo_tuning best;         /* also made current */
  double walk_ms_start;      /* median wall time of the job set with the starting knobs */
  double walk_ms_best;
  double update_ms_start;    /* median wall time of the update batch (-1: not tuned) */
  double update_ms_best;
  uint32_t candidates;       /* configurations timed */
  uint32_t reserved0;
} bingo_tune_report;

/* Coordinate search: walk_chunk, walk_split, walk_order, walk_blocks_per_sm,
 * then update_chunk and apply_blocks_per_sm; a candidate replaces the
 * current choice when its median is at least 1 % lower. */
int bingo_autotune(bingo_handle* h, const bingo_tune_request* req, bingo_tune_report* out);

/* Scheduler counters since bingo_serve_start (times in ns of scheduler-thread wall time). */
typedef struct bingo_serve_metrics {
  uint64_t submitted, completed;
  uint64_t walk_kernel_launches; /* serving-loop launches (relaunched after idle exits and updates) */
  uint64_t scheduler_passes;
  uint64_t admit_ns, complete_ns, update_ns, drain_wait_ns;
  uint64_t max_inflight;         /* most walk queries in flight at once */
  uint64_t queue_ns;             /* sum over walk queries of submit -> admission */
  uint64_t device_ns;            /* sum over walk queries of admission -> last walk finished (host-observed) */
  uint64_t copy_ns;              /* sum over walk queries of last walk finished -> result in caller memory */
  uint64_t drain_inflight_ns;    /* part of drain_wait_ns until earlier queries retired */
} bingo_serve_metrics;
int bingo_serve_get_metrics(bingo_handle* h, bingo_serve_metrics* out);

/* Finishes every submitted request, stops the walk loop, returns the handle to normal use. */
int bingo_serve_stop(bingo_handle* h);

/* Waits for all queued work; returns the first device-detected error since
 * the previous bingo_sync (or BINGO_OK). */
int bingo_sync(bingo_handle* h);

/* The CUDA stream calls are ordered on (cudaStream_t as void*); NULL restores
 * the handle's own stream. */
int bingo_set_stream(bingo_handle* h, void* stream);

int bingo_get_stats(bingo_handle* h, bingo_stats* out);

/* Graph-state dump for parity checks (the reference has none; its state is
 * the NodeData records of include/Bingo.cuh:6-58). sizes[0] = slots,
 * sizes[1] = group members, sizes[2] = alias slots. All outputs are host
 * arrays: ecnt/live/am [n]; ev/ew [slots] by vertex; gcnt [n*32];
 * mslot/mv/mbp [members] by (vertex, bit): member slot, neighbour, and the
 * slot's back-pointer (equals the member's position); athr/aT/aown/aalias
 * [alias slots] by vertex: threshold, total mass, own bit, alias bit. */
int bingo_dump_sizes(bingo_handle* h, uint64_t sizes[3]);
int bingo_dump_state(bingo_handle* h, uint32_t* ecnt, uint32_t* live, uint32_t* ev, uint32_t* ew, uint32_t* gcnt,
                     uint32_t* mslot, uint32_t* mv, uint32_t* mbp, uint32_t* am, uint64_t* athr, uint64_t* aT,
                     uint8_t* aown, uint8_t* aalias);

/* Philox4x32-10 as the device computes it (one block per counter), for
 * checking the walk random stream: out[4*i..4*i+3] = philox(ctr_i, key). */
int bingo_philox(bingo_handle* h, const uint32_t* ctr4, uint64_t count, uint64_t key, uint32_t* out4);

/* Diagnostic with no counterpart in the reference: measures this GPU's
 * random 32-byte-sector read rate from a table of table_bytes (allocated and
 * freed by the call). out[0] = sectors/s with 8 independent reads in flight
 * per thread, out[1] = sectors/s of dependent read chains (one per thread,
 * the shape of a walk step), out[2] = mean dependent-read latency in ns. */
int bingo_probe_gather(bingo_handle* h, uint64_t table_bytes, double out[3]);

#ifdef __cplusplus
}
#endif

#endif /* BINGO_H */

/*
 * gsofa.h -- C ABI of the B200-native gSoFa symbolic LU factorization.
 *
 * The reference exposes one host entry point,
 *     void symbfact_min_id(int args, char **argv, int myrank,
 *                          ull_t &fill_count, double &time)
 * (without_space_optimization/symbfact.cuh:991 and
 *  with_space_optimization/symbfact.cuh:1553), called from
 * without_space_optimization/main.cu:31.  It reads the colbeg/colend/csr text
 * files named in argv, runs the multi-source fill traversal on the GPU, and
 * reports the total fill count and the time; every error calls exit().
 *
 * This header replaces it with:
 *   - gsofa_symbfact_min_id(): the same argv contract, returning a status;
 *   - a structured API (context, device-resident matrix, parameters, result)
 *     that also returns the L+U pattern, per-line counts and the supernode
 *     partition, for one matrix or a batch of matrices in one launch.
 *
 * Conventions:
 *   - every function returns a gsofa_status and never exits the process;
 *   - input arrays are caller-owned host memory and are copied;
 *   - result arrays are library-owned host memory, valid until
 *     gsofa_result_free();
 *   - a context is used by one host thread at a time.
 *
 * Matrix convention: n lines; line v owns adj[beg[v] .. end[v]) (the
 * reference's colbeg/colend/csr triple).  Ranges may sit anywhere inside adj,
 * in any order; lists may be unsorted and may contain the diagonal or
 * duplicates.  The pattern computed is that of the LU factors of the matrix
 * whose row v holds the entries of line v:
 *   U by rows:    u_idx[u_ptr[s] .. u_ptr[s+1])  = sorted { j > s : (s,j) in L+U }
 *   L by columns: l_idx[l_ptr[j] .. l_ptr[j+1])  = sorted { i > j : (i,j) in L+U }
 * (entries are original nonzeros plus fill; the diagonal is implicit).
 */
#ifndef GSOFA_H
#define GSOFA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GSOFA_ABI_VERSION 1

typedef enum gsofa_status {
    GSOFA_OK = 0,
    GSOFA_ERR_INVALID_INPUT = 1, /* bad sizes, ranges or ids; bad argv     */
    GSOFA_ERR_OOM = 2,           /* device or host allocation failed       */
    GSOFA_ERR_QUEUE_OVERFLOW = 3,/* a frontier queue or the pattern pool
                                    ran out of room (retried internally)    */
    GSOFA_ERR_TIMEOUT = 4,       /* a bounded device-side wait gave up     */
    GSOFA_ERR_CUDA = 5,          /* a CUDA runtime call failed             */
    GSOFA_ERR_IO = 6,            /* an input file could not be read        */
    GSOFA_ERR_UNSUPPORTED = 7,   /* no usable GPU or too large for it      */
    GSOFA_ERR_BUSY = 8           /* no room for the request now: poll and
                                    fetch results, then submit again        */
} gsofa_status;

typedef struct gsofa_ctx gsofa_ctx;       /* device, stream, scratch pools */
typedef struct gsofa_matrix gsofa_matrix; /* device-resident G and G^T     */

/* Tuning and output parameters; zero means "choose automatically". */
typedef struct gsofa_params {
    int32_t src_chunk;          /* consecutive sources per work item; 0: 32 to
                                   512, about eight pieces per resident CTA  */
    int32_t block_size;         /* threads per CTA: 128, 256, 512, 768 (the
                                   two passes side by side only) or 1024      */
    int32_t threads_per_source; /* lanes expanding one frontier vertex:
                                   1 (default: one thread per vertex, a warp
                                   for rows longer than 32), 4, 8, 16 or 32   */
    int32_t ctas_per_sm;        /* resident CTAs per SM                       */
    int64_t queue_capacity;     /* frontier entries per CTA (>= n, else n)    */
    int64_t pool_capacity;      /* pattern entries kept on the device         */
    int32_t max_supernode_size; /* 0 or negative: unbounded                   */
    int32_t want_pattern;       /* 1: the pattern in CSR form (u/l index
                                   arrays in line order); 2: the ranges form,
                                   through gsofa_symbfact_ranges only          */
    int32_t reuse;              /* -1 (default) or 1: a source reuses the
                                   finished traversal of s-1 whenever s-1 is
                                   reachable from s; the two passes of a
                                   source run side by side in one CTA and
                                   exchange the flags that decide it (when
                                   two bitmaps fit, else as with 2);
                                   2: reuse only when s-1 is in adj(s);
                                   0: every source starts from scratch        */
    int32_t flags;              /* GSOFA_FLAG_* bits                          */
    int32_t part_count;         /* >1: process only the sources s with        */
    int32_t part_index;         /*     s % part_count == part_index (the
                                   reference's interleaved virtual-GPU
                                   partition, symbfact.cuh:1093); per-line
                                   outputs of other lines are zero            */
    int32_t line_lo;            /* either nonzero: process only the source   */
    int32_t line_hi;            /*   lines [line_lo, line_hi) of one matrix
                                   (a contiguous partition, see
                                   gsofa_partition_lines; [n, n) is empty);
                                   reuse and the pattern stay available;
                                   per-line outputs of other lines are zero;
                                   no supernode partition is formed from part
                                   of the lines (n_supernodes = 0; see
                                   gsofa_supernodes_from_lines)               */
} gsofa_params;

#define GSOFA_FLAG_NO_DOWNLOAD 0x1 /* keep per-line arrays on the device only */
#define GSOFA_FLAG_DEVICE_TIMING 0x2 /* record the traversal kernel time       */
#define GSOFA_FLAG_GRAPH 0x4       /* capture the launch in a CUDA graph and
                                      replay it while the same job (matrices,
                                      parameters, buffers) repeats            */
#define GSOFA_FLAG_GLOBAL_STATE 0x8 /* keep every traversal's visited bitmap
                                      in global memory (L2): many small
                                      traversals per SM, any n              */
#define GSOFA_FLAG_WIDE_REGS 0x40  /* the two passes side by side in 512-thread
                                      CTAs with up to 128 registers a thread
                                      (one CTA per SM): fastest on
                                      latency-bound matrices (small frontiers),
                                      slower on dense-fill ones               */
#define GSOFA_FLAG_DIRECT_HOST 0x20 /* gsofa_symbfact_ranges into host memory:
                                      the kernel writes the lists there
                                      itself (no device pool; slower than the
                                      default staging through device memory) */
#define GSOFA_FLAG_SHARED_STATE 0x10 /* keep them in shared memory (at most
                                      two per SM; GSOFA_ERR_UNSUPPORTED when
                                      they do not fit).  Neither flag: shared
                                      memory while two bitmaps fit, else
                                      global memory                         */

typedef struct gsofa_result {
    int32_t n;
    int32_t n_supernodes;
    uint64_t fill_count;     /* new nonzeros (original entries excluded);
                                with part_count > 1: of the processed lines */
    uint64_t nnz_lu;         /* |struct(A) u fill u diag|                  */
    uint64_t nnz_u;          /* strictly upper entries                      */
    uint64_t nnz_l;          /* strictly lower entries                      */
    uint64_t edges_inspected;/* adjacency entries the traversal read        */
    uint64_t sources;        /* traversals run (both passes)                */
    uint64_t x_total;        /* pass-G vertices expanded: sum |X(s)| when
                                every source starts from scratch          */
    uint64_t e_insp;         /* pass-G input-degree sum over the sources and
                                the vertices expanded, sum deg(s) + sum over
                                X(s) of deg(v) (input degrees, diagonal and
                                duplicates included)                      */
    uint64_t levels;         /* frontier levels summed over the traversals  */
    uint64_t reused_sources; /* traversals that started from s-1's state    */
    uint64_t cycles[7];      /* SM cycles summed over traversals: seeding,
                                level loop, range fold, count and link
                                flag, list output (once per chain of
                                sources), bitmap clearing, waiting for the
                                other pass                                  */
    uint64_t ctas;           /* CTAs of the persistent launch               */
    double kernel_ms;        /* factorization kernel time on the device     */
    /* per-line arrays (host, library-owned; NULL with NO_DOWNLOAD) */
    int32_t *u_row_count;    /* [n] |U row s|                               */
    int32_t *l_col_count;    /* [n] |L column j|                            */
    int32_t *l_row_count;    /* [n] |L row s| (with want_pattern only)      */
    int32_t *sn_start;       /* [n_supernodes] first line of each supernode */
    uint8_t *line_flags;     /* [n] bit 0: s+1 in U row s; bit 1: s+1 in
                                L column s (the supernode link flags)       */
    /* pattern (host, library-owned; NULL unless want_pattern) */
    int64_t *u_ptr;          /* [n+1] */
    int32_t *u_idx;          /* [nnz_u] */
    int64_t *l_ptr;          /* [n+1] */
    int32_t *l_idx;          /* [nnz_l] */
    void *internal;
    /* ranges form (gsofa_symbfact_ranges): begins into the caller's pool
     * (host, library-owned; NULL with NO_DOWNLOAD, see
     * gsofa_result_fetch_ranges) */
    int64_t *u_beg;          /* [n] U row s = pool[u_beg[s] .. + u_row_count[s])  */
    int64_t *l_beg;          /* [n] L col j = pool[l_beg[j] .. + l_col_count[j])  */
    int64_t pool_used;       /* pool entries the job wrote; after
                                GSOFA_ERR_QUEUE_OVERFLOW: the entries it needs */
} gsofa_result;

/* ---- reference-compatible entry ------------------------------------------
 * Replaces symbfact_min_id (without_space_optimization/symbfact.cuh:991;
 * with_space_optimization/symbfact.cuh:1553).  argv as the reference's CLI:
 *   argv[1] colbeg file, argv[2] colend file, argv[3] csr file,
 *   argv[4] N_GPU (source partitions, run back to back),
 *   optional argv[5] device memory pool in GB (the context's budget: it bounds
 *   the concurrent traversals, each holding an n-entry frontier queue, as the
 *   reference's pool bounds its sources per pass; GSOFA_ERR_OOM when not even
 *   one fits; 0: 90% of the free memory), argv[6] max_supernode_size,
 *   argv[7] GPUs per node.
 * The device is myrank % GPUs-per-node.  *fill_count receives the TOTAL over
 * all partitions; *time_ms the factorization time.  Returns a status. */
gsofa_status gsofa_symbfact_min_id(int argc, char **argv, int myrank,
                                   uint64_t *fill_count, double *time_ms);

/* ---- structured API ------------------------------------------------------ */
const char *gsofa_status_str(gsofa_status s);
int gsofa_abi_version(void);
void gsofa_default_params(gsofa_params *p);

/* Context on `device`; mem_budget_bytes bounds the device memory it may hold
 * (0: 90% of the free memory at creation). */
gsofa_status gsofa_create(gsofa_ctx **ctx, int device, size_t mem_budget_bytes);
void gsofa_destroy(gsofa_ctx *ctx);

/* Makes ctx issue its work on `cuda_stream` (a cudaStream_t of ctx's device;
 * NULL restores the context's own stream).  Calls still return only after
 * their work has finished. */
gsofa_status gsofa_set_stream(gsofa_ctx *ctx, void *cuda_stream);

/* Reads the reference's text files (csr: "nnz n" then nnz ids; colbeg and
 * colend: n ids each; without_space_optimization/symbfact.cuh:1022-1071) into
 * malloc'd arrays the caller frees with gsofa_free().  Each file may instead
 * be in the binary form gsofa_write_binary() produces (detected by its magic),
 * which loads without text parsing. */
gsofa_status gsofa_read_text(const char *beg_file, const char *end_file,
                             const char *csr_file, int32_t *n, int64_t *nnz,
                             int32_t **beg, int32_t **end, int32_t **adj);

/* Writes the three input files in binary form: the magic "GSOFAB01", then
 * little-endian int64 counts (csr: nnz, n; colbeg and colend: n) and the
 * int32 ids.  No counterpart in the reference, which reads text only. */
gsofa_status gsofa_write_binary(const char *beg_file, const char *end_file,
                                const char *csr_file, int32_t n, int64_t nnz,
                                const int32_t *beg, const int32_t *end,
                                const int32_t *adj);
void gsofa_free(void *p);

/* Copies the caller's host arrays to the device, validates them (every range
 * inside [0, nnz), every id inside [0, n)) and builds the compact graph and its
 * transpose.  The matrix belongs to ctx. */
gsofa_status gsofa_upload(gsofa_ctx *ctx, int32_t n, int64_t nnz,
                          const int32_t *beg, const int32_t *end,
                          const int32_t *adj, gsofa_matrix **out);
void gsofa_matrix_free(gsofa_matrix *m);
int32_t gsofa_matrix_n(const gsofa_matrix *m);

/* Symbolic factorization of one matrix (params may be NULL). */
gsofa_status gsofa_symbfact(gsofa_ctx *ctx, const gsofa_matrix *m,
                            const gsofa_params *params, gsofa_result *out);

/* `count` matrices in one persistent launch; out[i] belongs to mats[i]. */
gsofa_status gsofa_symbfact_batch(gsofa_ctx *ctx, int count,
                                  const gsofa_matrix *const *mats,
                                  const gsofa_params *params,
                                  gsofa_result *out);

void gsofa_result_free(gsofa_result *r);

/* The pattern in the reference's own begin/end layout (colbeg/colend into
 * one id array, without_space_optimization/symbfact.cuh:1022-1071), written
 * straight into caller memory: U row s is pool[u_beg[s] .. u_beg[s] +
 * u_row_count[s]) and L column j is pool[l_beg[j] .. l_beg[j] +
 * l_col_count[j]), each list sorted; lists sit in the order the traversals
 * finished them, with no gaps (pool_used = nnz_u + nnz_l of all `count`
 * matrices).  No compaction pass runs.
 *
 * `pool` is either device memory on ctx's device or page-locked host memory
 * (cudaHostAlloc, cudaHostRegister).  A host pool is staged through a device
 * pool of the same size when half the context's budget holds it, and copied
 * at full PCIe speed; otherwise (or with GSOFA_FLAG_DIRECT_HOST) the kernel
 * writes the lists into host memory while the traversals run, so the pattern
 * needs no device memory and may be larger than the device.  pool_capacity
 * counts int32 entries.  When
 * it is too small the call returns GSOFA_ERR_QUEUE_OVERFLOW with
 * out[i].pool_used set to the entries the job needs.  The other result
 * fields are as for gsofa_symbfact.  Results of a device pool can feed
 * gsofa_result_supernodal while the pool stays allocated. */
gsofa_status gsofa_symbfact_ranges(gsofa_ctx *ctx, int count,
                                   const gsofa_matrix *const *mats,
                                   const gsofa_params *params, int32_t *pool,
                                   int64_t pool_capacity, gsofa_result *out);

/* Copies the begins of a ranges-form result made with GSOFA_FLAG_NO_DOWNLOAD
 * into caller buffers of n entries each (either may be NULL); valid until the
 * next factorization on ctx. */
gsofa_status gsofa_result_fetch_ranges(gsofa_ctx *ctx, const gsofa_result *r,
                                       int64_t *u_beg, int64_t *l_beg);

/* Copies the arrays of a result made with GSOFA_FLAG_NO_DOWNLOAD into
 * caller-owned host buffers (page-locked buffers give full PCIe speed).  Any
 * pointer may be NULL; sizes follow the result: n for the per-line counts,
 * n_supernodes, n+1 for the offsets, nnz_u / nnz_l for the indices.  Valid
 * until the next factorization on ctx (GSOFA_ERR_INVALID_INPUT after it). */
gsofa_status gsofa_result_fetch(gsofa_ctx *ctx, const gsofa_result *r,
                                int32_t *u_row_count, int32_t *l_col_count,
                                int32_t *l_row_count, int32_t *sn_start,
                                int64_t *u_ptr, int32_t *u_idx,
                                int64_t *l_ptr, int32_t *l_idx);

/* SuperLU-style supernodal structure of a factorization with the pattern,
 * built on the device from the result and downloaded without the full
 * pattern.  Supernode k holds columns / rows xsup[k] .. xsup[k+1]-1:
 *   lsub[xlsub[k] .. xlsub[k+1]) -- its rows: the diagonal block xsup[k] ..
 *       xsup[k+1]-1, then the rows below the block of its last column, which
 *       hold those of every column of the supernode (L columns of a supernode
 *       nest, so this is the union: a relaxed supernode where they differ);
 *   usub[xusub[k] .. xusub[k+1]) -- the columns right of the block, the same
 *       for every row of the supernode;
 *   supno[j] -- the supernode of column j.
 * The consumer-side format of SuperLU_DIST's symbolic stage; no counterpart in
 * the reference, which returns no pattern.  Host arrays are library-owned until
 * gsofa_supernodal_free().  Needs the result of the last factorization on ctx,
 * made with the pattern (GSOFA_FLAG_NO_DOWNLOAD spares its download). */
typedef struct gsofa_supernodal {
    int32_t n, nsuper;
    int64_t nlsub, nusub;
    int32_t *xsup;    /* [nsuper + 1] */
    int32_t *supno;   /* [n] */
    int64_t *xlsub;   /* [nsuper + 1] */
    int32_t *lsub;    /* [nlsub] */
    int64_t *xusub;   /* [nsuper + 1] */
    int32_t *usub;    /* [nusub] */
} gsofa_supernodal;

gsofa_status gsofa_result_supernodal(gsofa_ctx *ctx, const gsofa_result *r,
                                     gsofa_supernodal *out);
void gsofa_supernodal_free(gsofa_supernodal *s);

/* The same structure into caller-owned (e.g. page-locked) buffers, in two
 * calls: the sizes first (nsuper + 1 entries for xsup, xlsub and xusub, n for
 * supno, nlsub for lsub, nusub for usub), then the fetch.  Any fetch pointer
 * may be NULL.  The fetch needs the sizes call for the same result just before
 * it on ctx. */
gsofa_status gsofa_result_supernodal_sizes(gsofa_ctx *ctx, const gsofa_result *r,
                                           int32_t *nsuper, int64_t *nlsub,
                                           int64_t *nusub);
gsofa_status gsofa_result_supernodal_fetch(gsofa_ctx *ctx, const gsofa_result *r,
                                           int32_t *xsup, int32_t *supno,
                                           int64_t *xlsub, int32_t *lsub,
                                           int64_t *xusub, int32_t *usub);

/* Supernode partition from per-line U row counts and link flags (as in
 * gsofa_result), computed on the host: used to finish a factorization whose
 * lines were computed in partitions (on several GPUs) and summed.  Writes the
 * starts to sn_start (capacity n) and returns their number (-1: bad input). */
int32_t gsofa_supernodes_from_lines(int32_t n, const int32_t *u_row_count,
                                    const uint8_t *line_flags,
                                    int32_t max_supernode_size, int32_t *sn_start);

/* Contiguous partition of the source lines into `parts` ranges of equal
 * predicted work, for factorizing one matrix on several GPUs with
 * gsofa_params.line_lo / line_hi (replaces the reference's interleaved
 * partition, with_space_optimization/symbfact.cuh:1084-1099, which leaves no
 * consecutive sources on one GPU and so no traversal reuse).  Work of line s:
 * a fixed cost per traversal plus a cost per list entry, the list lengths
 * predicted from the column counts of the Cholesky factor of A + A^T
 * (elimination tree and skeleton counts, near-linear time); each cut moves to
 * a nearby line that does not hold its predecessor.  Host-only.  cuts
 * receives parts + 1 entries (cuts[0] = 0, cuts[parts] = n); work, when
 * non-NULL, the predicted work of each part (SM cycles). */
gsofa_status gsofa_partition_lines(int32_t n, int64_t nnz, const int32_t *beg,
                                   const int32_t *end, const int32_t *adj,
                                   int32_t parts, int32_t *cuts, double *work);

/* Predicted list length of every line, the work model of
 * gsofa_partition_lines: counts[s] = |column s of the Cholesky factor of
 * A + A^T| minus the diagonal, an upper bound on both |U row s| and
 * |L column s| (equal to them when the pattern is symmetric).  Host-only. */
gsofa_status gsofa_predict_line_counts(int32_t n, int64_t nnz, const int32_t *beg,
                                       const int32_t *end, const int32_t *adj,
                                       int64_t *counts);

/* Fill-reducing ordering on the GPU, the step before the factorization (the
 * reference takes its colbeg/colend/csr input already ordered): reverse
 * Cuthill-McKee on the symmetric structure A + A^T of the host triple.  The
 * order is exactly the sequential algorithm's with every tie broken by
 * (degree, vertex id): each component (taken in that key order) starts at
 * George and Liu's pseudo-peripheral vertex, each vertex's unordered
 * neighbours follow it in key order, and the whole sequence is reversed.
 * perm (n entries) receives perm[new] = old.  Uses the context's device and
 * stream; scratch (about 40 bytes per entry and 60 per line) counts against
 * its budget.  GSOFA_ERR_UNSUPPORTED past 2^30 entries. */
gsofa_status gsofa_order_rcm(gsofa_ctx *ctx, int32_t n, int64_t nnz, const int32_t *colbeg,
                             const int32_t *colend, const int32_t *csr, int32_t *perm);

/* The symmetric permutation P A P^T of a host triple: new line k is old line
 * perm[k] with every id v renamed to the new position of v, each line sorted,
 * packed in order (out_colbeg[k] .. out_colend[k] in out_csr, which holds
 * the sum of the input lines' lengths).  Host-only. */
gsofa_status gsofa_permute_lines(int32_t n, int64_t nnz, const int32_t *colbeg, const int32_t *colend,
                                 const int32_t *csr, const int32_t *perm, int32_t *out_colbeg,
                                 int32_t *out_colend, int32_t *out_csr);

/* Device scratch bytes a factorization of an n-line, nnz-entry matrix needs
 * with these parameters, excluding the pattern pool (admission control). */
size_t gsofa_predict_scratch_bytes(const gsofa_ctx *ctx, int32_t n, int64_t nnz,
                                   const gsofa_params *params);

/* ---- serving: continuous batching over a persistent kernel ----------------
 * A server keeps one persistent kernel running on its device.  Every
 * submitted request (a matrix) is uploaded into device memory the server
 * reserved at creation, cut into work pieces and published to the running
 * kernel, whose CTAs take pieces of all live requests as they free up; a
 * request that arrives while others are being factorized starts on the next
 * free CTA.  Admission is by predicted device bytes (matrix, per-line state):
 * a request that does not fit now returns GSOFA_ERR_BUSY.  Results are counts
 * and supernodes (no pattern).  One host thread drives a server. */
typedef struct gsofa_server gsofa_server;

typedef struct gsofa_server_config {
    int32_t device;
    int32_t max_n;              /* largest request; 0: see flags            */
    int64_t mem_budget_bytes;   /* device bytes the server may hold; 0: 90%
                                   of the free memory                       */
    int32_t max_supernode_size; /* as in gsofa_params                       */
    int32_t src_chunk;          /* sources per work piece; 0: 32 to 512 from
                                   each request's n                         */
    int32_t max_requests;       /* requests in flight; 0: 4096             */
    int32_t idle_exit_us;       /* safety bound on how long an idle CTA
                                   waits for work (the host stops the kernel
                                   itself when nothing is in flight);
                                   0: 30 s                                  */
    int32_t max_n_out;          /* set by gsofa_server_create: the limit    */
    int32_t flags;              /* GSOFA_FLAG_SHARED_STATE: bitmaps in shared
                                   memory (two traversals per SM, n up to
                                   ~800K); default (or _GLOBAL_STATE): in
                                   global memory, six traversals per SM, max_n
                                   defaults to 1,048,576                    */
} gsofa_server_config;

gsofa_status gsofa_server_create(gsofa_server **srv, gsofa_server_config *cfg);
void gsofa_server_destroy(gsofa_server *srv);
/* Device bytes a request holds while it is in flight. */
size_t gsofa_server_request_bytes(const gsofa_server *srv, int32_t n, int64_t nnz);
/* Uploads and publishes one request (host arrays, copied); *id identifies it. */
gsofa_status gsofa_server_submit(gsofa_server *srv, int32_t n, int64_t nnz,
                                 const int32_t *beg, const int32_t *end,
                                 const int32_t *adj, int64_t *id);
/* Ids of requests finished since the last poll (up to `capacity`). */
gsofa_status gsofa_server_poll(gsofa_server *srv, int64_t *ids, int32_t capacity,
                               int32_t *count);
/* Waits until every published request has finished and the kernel has
 * exited, so other work (another library's kernels, gsofa_symbfact) gets the
 * whole device; the next submit restarts the kernel. */
gsofa_status gsofa_server_drain(gsofa_server *srv);
/* The result of a finished request (counts, line flags, supernodes, totals);
 * releases the request's device memory.  Free with gsofa_result_free. */
gsofa_status gsofa_server_result(gsofa_server *srv, int64_t id, gsofa_result *out);

/* ---- factorization without device allocation ------------------------------
 * No counterpart in the reference.  For callers that cannot call cudaMalloc:
 * code embedded in an application whose own allocator owns all device memory
 * (a solver plugin under a host framework's memory pool or budget), and code
 * on latency-critical paths where cudaMalloc's implicit device-wide
 * synchronisation is not acceptable.  The caller passes device pointers for
 * the input (the colbeg/colend/csr triple, already on `device`) and for the
 * outputs; every intermediate array lives in one file-scope static device
 * array of GSOFA_NOALLOC_SCRATCH_BYTES that each GPU loading this library
 * holds until the process exits.  Nothing here calls cudaMalloc, cudaFree or
 * an allocating library routine.
 *
 * Limits: n <= GSOFA_NOALLOC_MAX_N and the line ranges' total length
 * <= GSOFA_NOALLOC_MAX_NNZ; larger inputs return GSOFA_ERR_UNSUPPORTED before
 * any work is issued.  The array also holds one n-entry frontier queue per SM,
 * so the limits hold on GPUs with up to 200 SMs (the B200 has 148); on a
 * larger GPU an input near both limits returns GSOFA_ERR_UNSUPPORTED too.  Counts only (no pattern): per-line U row counts,
 * L column counts, the supernode starts and a host summary
 * summary[0] = fill count, [1] = nnz(L+U), [2] = number of supernodes.
 *
 * Every call looks up the static array's device address with `device`
 * current (the first call on a device also reads its properties); make the
 * first call on a device before any stream capture.  The caller's current
 * device is restored before the call returns.  All calls on a device share the one array and it keeps the last
 * call's contents (everything that must start at zero is cleared by the
 * call), so calls that overlap on the GPU race: issue them one at a time.
 * The call returns after its work on `cuda_stream` (NULL: the legacy default
 * stream) has finished. */
#define GSOFA_NOALLOC_MAX_N 16384
#define GSOFA_NOALLOC_MAX_NNZ 262144
#define GSOFA_NOALLOC_SCRATCH_BYTES (16u << 20)
gsofa_status gsofa_symbfact_counts_noalloc(int device, void *cuda_stream, int32_t n,
                                           int64_t nnz, const int32_t *d_beg,
                                           const int32_t *d_end, const int32_t *d_adj,
                                           int32_t max_supernode_size,
                                           int32_t *d_u_row_count,
                                           int32_t *d_l_col_count,
                                           int32_t *d_sn_start, uint64_t *summary);

#ifdef __cplusplus
}
#endif
#endif /* GSOFA_H */

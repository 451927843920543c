/*
 * gsofa_oracle.h -- CPU restatement of gSoFa's symbolic LU factorization.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the shipped library links, loads or
 * calls this code; only the test-suite, the smoke check and the CPU-baseline
 * leg of the benchmark use it, always as the checker, never as the thing being
 * measured or shipped.
 *
 * Input convention (the reference's driver format): a graph of n vertices
 * ("lines"); line v owns the entries adj[beg[v] .. end[v]).  Ranges may sit
 * anywhere inside adj and in any order; lists may be unsorted and may hold the
 * diagonal or duplicates.  This is the colbeg/colend/csr triple read by
 * without_space_optimization/symbfact.cuh:1022-1071.
 *
 * Two restatements are provided:
 *
 *  1. gsofa_oracle_maxid_fills(): the reference's own algorithm -- per-source
 *     "max-id" label propagation with a fill marker, seeded as in
 *     with_space_optimization/symbfact.cuh:639-721 and relaxed as in
 *     with_space_optimization/symbfact.cuh:989-1067.  It returns fill counts
 *     per line (the reference outputs only the total).
 *
 *  2. gsofa_oracle_counts()/gsofa_oracle_pattern(): the same fill set,
 *     computed as two reachability passes.  Pass G, source s, collects
 *     hi_G(s) = { j > s : j in adj(v), v in {s} u X_G(s) } where X_G(s) is the
 *     set of vertices < s reachable from s through vertices < s.  This is the
 *     upper part of line s (original entries plus fill).  Pass G^T does the
 *     same on the transposed graph; by the fill-path theorem,
 *     (s, j) with j < s is in the factor iff s is in hi_{G^T}(j), so pass G^T
 *     yields the lower part column by column.  The GPU library computes
 *     exactly these arrays, and they are compared bit for bit.
 *
 * Parity pin: on the bundled n = 11,948 matrix both restatements give
 * 980,136 fills, the total logged by the reference
 * (with_space_optimization/space_optimization_log_1_264_GPU_warp_centric.dat:2).
 */
#ifndef GSOFA_ORACLE_H
#define GSOFA_ORACLE_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

/* Threads the OpenMP functions use when given nthreads <= 0 (the OpenMP
 * default: OMP_NUM_THREADS, else the host's logical cores). */
int gsofa_oracle_threads(void);

/* Per-line outputs of one reachability pass over G (pass 0) or G^T (pass 1).
 * All arrays have n entries and are caller-allocated; any may be NULL.
 *   cnt[s]   = |hi(s)|               (entries > s in line s of that pass)
 *   orig[s]  = distinct original entries > s in line s of that pass
 *   next[s]  = 1 if s+1 is in hi(s)  (used by the supernode scan)
 * work[0] += |X(s)|, work[1] += E_insp(s) = deg(s) + sum_{v in X(s)} deg(v),
 * summed over the processed sources (only meaningful for pass 0).
 * sources/n_sources: restrict to these sources (NULL = all n sources).
 * Returns 0 on success, nonzero on invalid input or allocation failure. */
int gsofa_oracle_counts(int32_t n, const int32_t *beg, const int32_t *end,
                        const int32_t *adj, int64_t adj_len, int pass,
                        int nthreads, const int32_t *sources, int32_t n_sources,
                        int32_t *cnt, int32_t *orig, uint8_t *next,
                        uint64_t *work);

/* Writes the sorted hi(s) lists of one pass at idx[ptr[s] .. ptr[s+1]).
 * ptr has n+1 entries and must be the exclusive prefix sum of cnt. */
int gsofa_oracle_pattern(int32_t n, const int32_t *beg, const int32_t *end,
                         const int32_t *adj, int64_t adj_len, int pass,
                         int nthreads, const int64_t *ptr, int32_t *idx);

/* The sorted hi(s) lists of one pass for the listed sources only (distinct
 * ids; a repeated source fails with 3): list i goes to idx[ptr[i] ..
 * ptr[i+1]), where ptr (n_sources + 1 entries) is the exclusive prefix sum
 * of those sources' cnt values.  Lets a check cover sampled lines of a
 * matrix whose whole pattern is too large to hold. */
int gsofa_oracle_lists(int32_t n, const int32_t *beg, const int32_t *end,
                       const int32_t *adj, int64_t adj_len, int pass,
                       int nthreads, const int32_t *sources, int32_t n_sources,
                       const int64_t *ptr, int32_t *idx);

/* Supernode partition from the per-line upper counts and link flags.
 * Lines s-1 and s are in one supernode iff
 *   (i)   s-1 is in line s  (lnext[s-1] == 1: s is in hi_{G^T}(s-1)),
 *   (ii)  s   is in line s-1 (unext[s-1] == 1: s is in hi_G(s-1)),
 *   (iii) ucnt[s] == ucnt[s-1] - 1, and
 *   (iv)  the current supernode holds fewer than max_size lines
 *         (max_size <= 0: unbounded).
 * Writes the first line of each supernode to sn_start (capacity n) and
 * returns the number of supernodes. */
int32_t gsofa_oracle_supernodes(int32_t n, const int32_t *ucnt,
                                const uint8_t *unext, const uint8_t *lnext,
                                int32_t max_size, int32_t *sn_start);

/* Faithful restatement of the reference's max-id traversal.  For every line s,
 * fills_lo[s] / fills_hi[s] receive the number of fills (s, j) with j < s /
 * j > s.  Either may be NULL.  Returns the total fill count, or -1 on error. */
int64_t gsofa_oracle_maxid_fills(int32_t n, const int32_t *beg,
                                 const int32_t *end, const int32_t *adj,
                                 int64_t adj_len, int nthreads,
                                 int64_t *fills_lo, int64_t *fills_hi);

/* The same for the listed sources only (NULL: all n, highest first): the
 * reference's algorithm on a sample of its lines.  fills_lo / fills_hi are
 * indexed by line and written only at the listed lines. */
int64_t gsofa_oracle_maxid_counts(int32_t n, const int32_t *beg,
                                  const int32_t *end, const int32_t *adj,
                                  int64_t adj_len, int nthreads,
                                  const int32_t *sources, int32_t n_sources,
                                  int64_t *fills_lo, int64_t *fills_hi);

/* The fill pattern (both halves, sorted) of the single line s, from the max-id
 * traversal; out must hold n entries.  Returns the number written or -1. */
int32_t gsofa_oracle_maxid_line(int32_t n, const int32_t *beg,
                                const int32_t *end, const int32_t *adj,
                                int64_t adj_len, int32_t s, int32_t *out);

/* Reverse Cuthill-McKee ordering of the symmetric structure A + A^T (the
 * step before the path; the reference takes its input already ordered, so
 * this restates the published algorithms: Cuthill-McKee breadth-first levels,
 * George-Liu pseudo-peripheral start, ties broken by (degree, vertex id); the
 * rules are spelled out in gsofa_oracle.c).  perm[new] = old.  No reference
 * output exists for it: the GPU ordering is compared with this one bit for
 * bit, and its quality (bandwidth) with scipy's reverse_cuthill_mckee. */
int gsofa_oracle_rcm(int32_t n, const int32_t *beg, const int32_t *end, const int32_t *adj,
                     int64_t adj_len, int32_t *perm);

#ifdef __cplusplus
}
#endif
#endif

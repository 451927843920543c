/*
 * gsofa_oracle.c -- CPU restatement of gSoFa's symbolic factorization.
 *
 * TEST INFRASTRUCTURE ONLY (the checker, never the product).  See
 * gsofa_oracle.h for the conventions and for which reference lines each
 * function restates.
 *
 * Build: oracle/Makefile (gcc -O2 -fopenmp -shared).
 */
#include "gsofa_oracle.h"

#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* ------------------------------------------------------------------------ */
/* Input validation: every range inside [0, adj_len), every id inside [0, n). */
static int validate(int32_t n, const int32_t *beg, const int32_t *end,
                    const int32_t *adj, int64_t adj_len)
{
    if (n < 0 || adj_len < 0) return 1;
    if (n > 0 && (!beg || !end)) return 1;
    if (adj_len > 0 && !adj) return 1;
    for (int32_t v = 0; v < n; v++) {
        if (beg[v] < 0 || end[v] < beg[v] || (int64_t)end[v] > adj_len) return 1;
    }
    for (int64_t k = 0; k < adj_len; k++) {
        if (adj[k] < 0 || adj[k] >= n) return 1;
    }
    return 0;
}

/* Transposed graph in plain CSR form: tptr[n+1], tadj[adj_len].  Only entries
 * that some line's range covers are transposed. */
static int transpose(int32_t n, const int32_t *beg, const int32_t *end,
                     const int32_t *adj, int32_t **tbeg, int32_t **tend,
                     int32_t **tadj)
{
    int64_t total = 0;
    for (int32_t v = 0; v < n; v++) total += end[v] - beg[v];
    int32_t *cnt = (int32_t *)calloc((size_t)n + 1, sizeof(int32_t));
    int32_t *b = (int32_t *)malloc(((size_t)n + 1) * sizeof(int32_t));
    int32_t *e = (int32_t *)malloc(((size_t)n + 1) * sizeof(int32_t));
    int32_t *t = (int32_t *)malloc(((size_t)total + 1) * sizeof(int32_t));
    if (!cnt || !b || !e || !t) { free(cnt); free(b); free(e); free(t); return 1; }
    for (int32_t v = 0; v < n; v++)
        for (int32_t k = beg[v]; k < end[v]; k++) cnt[adj[k]]++;
    int32_t run = 0;
    for (int32_t v = 0; v < n; v++) { b[v] = run; e[v] = run; run += cnt[v]; }
    /* Lines are visited in increasing order, so each transposed list is
     * sorted by construction. */
    for (int32_t v = 0; v < n; v++)
        for (int32_t k = beg[v]; k < end[v]; k++) t[e[adj[k]]++] = v;
    free(cnt);
    *tbeg = b; *tend = e; *tadj = t;
    return 0;
}

static int cmp_i32(const void *a, const void *b)
{
    int32_t x = *(const int32_t *)a, y = *(const int32_t *)b;
    return (x > y) - (x < y);
}

/* One reachability traversal from source s restricted to vertices < s.
 * stamp[] holds s+1 for every vertex reached from s (a per-thread array that
 * never needs clearing because tags are unique per source).  On return
 * hi[0..*nhi) lists hi(s) (unsorted), *norig the distinct original entries
 * > s, *nx = |X(s)| and *einsp = deg(s) + sum_{v in X(s)} deg(v). */
static void reach_one(int32_t s, const int32_t *beg, const int32_t *end,
                      const int32_t *adj, int32_t *stamp, int32_t *queue,
                      int32_t *hi, int32_t *nhi, int32_t *norig,
                      uint64_t *nx, uint64_t *einsp)
{
    const int32_t tag = s + 1;
    int32_t qh = 0, qt = 0, h = 0, orig = 0;
    uint64_t e = (uint64_t)(end[s] - beg[s]);
    stamp[s] = tag;
    for (int32_t k = beg[s]; k < end[s]; k++) {
        int32_t m = adj[k];
        if (stamp[m] == tag) continue;
        stamp[m] = tag;
        if (m < s) queue[qt++] = m;
        else { hi[h++] = m; orig++; }
    }
    while (qh < qt) {
        int32_t v = queue[qh++];
        e += (uint64_t)(end[v] - beg[v]);
        for (int32_t k = beg[v]; k < end[v]; k++) {
            int32_t m = adj[k];
            if (stamp[m] == tag) continue;
            stamp[m] = tag;
            if (m < s) queue[qt++] = m;
            else hi[h++] = m;
        }
    }
    *nhi = h; *norig = orig; *nx = (uint64_t)qt; *einsp = e;
}

static int set_threads(int nthreads)
{
#ifdef _OPENMP
    if (nthreads <= 0) nthreads = omp_get_max_threads();
    return nthreads;
#else
    (void)nthreads;
    return 1;
#endif
}

int gsofa_oracle_threads(void) { return set_threads(0); }

int gsofa_oracle_counts(int32_t n, const int32_t *beg, const int32_t *end,
                        const int32_t *adj, int64_t adj_len, int pass,
                        int nthreads, const int32_t *sources, int32_t n_sources,
                        int32_t *cnt, int32_t *orig, uint8_t *next,
                        uint64_t *work)
{
    if (validate(n, beg, end, adj, adj_len)) return 1;
    if (pass != 0 && pass != 1) return 1;
    if (n == 0) return 0;
    const int32_t *B = beg, *E = end, *A = adj;
    int32_t *tb = NULL, *te = NULL, *ta = NULL;
    if (pass == 1) {
        if (transpose(n, beg, end, adj, &tb, &te, &ta)) return 2;
        B = tb; E = te; A = ta;
    }
    const int32_t ns = sources ? n_sources : n;
    for (int32_t i = 0; sources && i < ns; i++)
        if (sources[i] < 0 || sources[i] >= n) { free(tb); free(te); free(ta); return 1; }
    uint64_t wx = 0, we = 0;
    int failed = 0;
    nthreads = set_threads(nthreads);
#pragma omp parallel num_threads(nthreads) reduction(+ : wx, we) reduction(| : failed)
    {
        int32_t *stamp = (int32_t *)calloc((size_t)n, sizeof(int32_t));
        int32_t *queue = (int32_t *)malloc((size_t)n * sizeof(int32_t));
        int32_t *hi = (int32_t *)malloc((size_t)n * sizeof(int32_t));
        if (!stamp || !queue || !hi) failed = 1;
        else {
            /* One source per scheduling step, in the given order (by default
             * the highest, heaviest lines first): the threads take the
             * heavy lines one each instead of one thread taking a block of
             * them (longest-first list scheduling). */
#pragma omp for schedule(dynamic, 1)
            for (int32_t i = 0; i < ns; i++) {
                int32_t s = sources ? sources[i] : (n - 1 - i); /* heavy lines first */
                int32_t h, o; uint64_t x, e;
                reach_one(s, B, E, A, stamp, queue, hi, &h, &o, &x, &e);
                if (cnt) cnt[s] = h;
                if (orig) orig[s] = o;
                if (next) next[s] = (uint8_t)(s + 1 < n && stamp[s + 1] == s + 1);
                wx += x; we += e;
            }
        }
        free(stamp); free(queue); free(hi);
    }
    free(tb); free(te); free(ta);
    if (failed) return 2;
    if (work) { work[0] += wx; work[1] += we; }
    return 0;
}

int gsofa_oracle_pattern(int32_t n, const int32_t *beg, const int32_t *end,
                         const int32_t *adj, int64_t adj_len, int pass,
                         int nthreads, const int64_t *ptr, int32_t *idx)
{
    if (validate(n, beg, end, adj, adj_len)) return 1;
    if (pass != 0 && pass != 1) return 1;
    if (n == 0) return 0;
    if (!ptr || !idx) return 1;
    const int32_t *B = beg, *E = end, *A = adj;
    int32_t *tb = NULL, *te = NULL, *ta = NULL;
    if (pass == 1) {
        if (transpose(n, beg, end, adj, &tb, &te, &ta)) return 2;
        B = tb; E = te; A = ta;
    }
    int failed = 0;
    nthreads = set_threads(nthreads);
#pragma omp parallel num_threads(nthreads) reduction(| : failed)
    {
        int32_t *stamp = (int32_t *)calloc((size_t)n, sizeof(int32_t));
        int32_t *queue = (int32_t *)malloc((size_t)n * sizeof(int32_t));
        int32_t *hi = (int32_t *)malloc((size_t)n * sizeof(int32_t));
        if (!stamp || !queue || !hi) failed = 1;
        else {
#pragma omp for schedule(dynamic, 1)
            for (int32_t i = 0; i < n; i++) {
                int32_t s = n - 1 - i;
                int32_t h, o; uint64_t x, e;
                reach_one(s, B, E, A, stamp, queue, hi, &h, &o, &x, &e);
                if (ptr[s + 1] - ptr[s] != h) { failed = 1; continue; }
                qsort(hi, (size_t)h, sizeof(int32_t), cmp_i32);
                memcpy(idx + ptr[s], hi, (size_t)h * sizeof(int32_t));
            }
        }
        free(stamp); free(queue); free(hi);
    }
    free(tb); free(te); free(ta);
    return failed ? 3 : 0;
}

int gsofa_oracle_lists(int32_t n, const int32_t *beg, const int32_t *end,
                       const int32_t *adj, int64_t adj_len, int pass,
                       int nthreads, const int32_t *sources, int32_t n_sources,
                       const int64_t *ptr, int32_t *idx)
{
    if (validate(n, beg, end, adj, adj_len)) return 1;
    if (pass != 0 && pass != 1) return 1;
    if (n_sources < 0 || (n_sources > 0 && (!sources || !ptr || !idx))) return 1;
    for (int32_t i = 0; i < n_sources; i++)
        if (sources[i] < 0 || sources[i] >= n) return 1;
    if (n == 0 || n_sources == 0) return 0;
    const int32_t *B = beg, *E = end, *A = adj;
    int32_t *tb = NULL, *te = NULL, *ta = NULL;
    if (pass == 1) {
        if (transpose(n, beg, end, adj, &tb, &te, &ta)) return 2;
        B = tb; E = te; A = ta;
    }
    int failed = 0;
    nthreads = set_threads(nthreads);
#pragma omp parallel num_threads(nthreads) reduction(| : failed)
    {
        int32_t *stamp = (int32_t *)calloc((size_t)n, sizeof(int32_t));
        int32_t *queue = (int32_t *)malloc((size_t)n * sizeof(int32_t));
        int32_t *hi = (int32_t *)malloc((size_t)n * sizeof(int32_t));
        if (!stamp || !queue || !hi) failed = 1;
        else {
#pragma omp for schedule(dynamic, 1)
            for (int32_t i = 0; i < n_sources; i++) {
                int32_t s = sources[i];
                int32_t h, o; uint64_t x, e;
                reach_one(s, B, E, A, stamp, queue, hi, &h, &o, &x, &e);
                if (ptr[i + 1] - ptr[i] != h) { failed = 1; continue; }
                qsort(hi, (size_t)h, sizeof(int32_t), cmp_i32);
                memcpy(idx + ptr[i], hi, (size_t)h * sizeof(int32_t));
            }
        }
        free(stamp); free(queue); free(hi);
    }
    free(tb); free(te); free(ta);
    return failed ? 3 : 0;
}

int32_t gsofa_oracle_supernodes(int32_t n, const int32_t *ucnt,
                                const uint8_t *unext, const uint8_t *lnext,
                                int32_t max_size, int32_t *sn_start)
{
    if (n <= 0) return 0;
    int32_t k = 0, run = 0;
    for (int32_t s = 0; s < n; s++) {
        int linked = s > 0 && lnext[s - 1] && unext[s - 1] &&
                     ucnt[s] == ucnt[s - 1] - 1;
        if (linked && (max_size <= 0 || run < max_size)) {
            run++;
        } else {
            sn_start[k++] = s;
            run = 1;
        }
    }
    return k;
}

/* ------------------------------------------------------------------------ */
/* Faithful max-id restatement.
 *
 * Per source s (one slot of the reference's source chunk):
 *   cost[v]  : smallest known "maximum intermediate id" of a path s -> v;
 *              valid only where cstamp[v] == s+1 (the reference instead keeps
 *              per-chunk offsets, symbfact.cuh max_id_offset).
 *   mark[v]  : the fill marker fill_in_d[slot][v]; == s+1 once (s, v) is
 *              recorded as original structure or fill.
 * Seeding (with_space_optimization/symbfact.cuh:657-717): cost[s] = 0; for
 * every neighbour nb: mark[nb] = s+1; if nb < s: cost[nb] = 0 and enqueue nb.
 * Relaxation of a queue item f (symbfact.cuh:926, 989-1067):
 *   c = max(f, cost[f]);
 *   for m in adj(f):
 *     if m > s: record fill (s, m) unless marked; do not relax;
 *     else if cost[m] > c: cost[m] = c; enqueue m if m < s;
 *                          record fill (s, m) if m > c and unmarked.
 * The reference processes the queue level by level on the GPU with atomicMin;
 * a FIFO reaches the same fixpoint.
 */
static int64_t maxid_one(int32_t s, const int32_t *beg, const int32_t *end,
                         const int32_t *adj, uint32_t *cost, int32_t *cstamp,
                         int32_t *mark, int32_t *queue, int64_t qcap,
                         int64_t *lo, int64_t *hi, int32_t *out)
{
    const int32_t tag = s + 1;
    int64_t qh = 0, qt = 0, flo = 0, fhi = 0;
    int32_t nout = 0;
    cost[s] = 0; cstamp[s] = tag;
    for (int32_t k = beg[s]; k < end[s]; k++) {
        int32_t nb = adj[k];
        mark[nb] = tag;
        if (nb < s) {
            cost[nb] = 0; cstamp[nb] = tag;
            if (qt >= qcap) return -1;
            queue[qt++] = nb;
        }
    }
    while (qh < qt) {
        int32_t f = queue[qh++];
        uint32_t cf = cost[f];
        uint32_t c = (uint32_t)f > cf ? (uint32_t)f : cf;
        for (int32_t k = beg[f]; k < end[f]; k++) {
            int32_t m = adj[k];
            if (m > s) {
                if (mark[m] != tag) {
                    mark[m] = tag; fhi++;
                    if (out) out[nout++] = m;
                }
                continue;
            }
            uint32_t cm = (cstamp[m] == tag) ? cost[m] : UINT32_MAX;
            if (cm > c) {
                cost[m] = c; cstamp[m] = tag;
                if (m < s) {
                    if (qt >= qcap) {
                        /* compact the consumed prefix of the FIFO */
                        memmove(queue, queue + qh, (size_t)(qt - qh) * sizeof(int32_t));
                        qt -= qh; qh = 0;
                        if (qt >= qcap) return -1;
                    }
                    queue[qt++] = m;
                }
                if ((uint32_t)m > c && mark[m] != tag) {
                    mark[m] = tag; flo++;
                    if (out) out[nout++] = m;
                }
            }
        }
    }
    *lo = flo; *hi = fhi;
    return (int64_t)nout;
}

int64_t gsofa_oracle_maxid_counts(int32_t n, const int32_t *beg,
                                  const int32_t *end, const int32_t *adj,
                                  int64_t adj_len, int nthreads,
                                  const int32_t *sources, int32_t n_sources,
                                  int64_t *fills_lo, int64_t *fills_hi)
{
    if (validate(n, beg, end, adj, adj_len)) return -1;
    if (n == 0) return 0;
    const int32_t ns = sources ? n_sources : n;
    for (int32_t i = 0; sources && i < ns; i++)
        if (sources[i] < 0 || sources[i] >= n) return -1;
    int64_t total = 0;
    int failed = 0;
    /* A vertex re-enters the FIFO on every improvement of its label, so the
     * queue is sized generously and compacted when full. */
    const int64_t qcap = 4 * (int64_t)n + 1024;
    nthreads = set_threads(nthreads);
#pragma omp parallel num_threads(nthreads) reduction(+ : total) reduction(| : failed)
    {
        uint32_t *cost = (uint32_t *)malloc((size_t)n * sizeof(uint32_t));
        int32_t *cstamp = (int32_t *)calloc((size_t)n, sizeof(int32_t));
        int32_t *mark = (int32_t *)calloc((size_t)n, sizeof(int32_t));
        int32_t *queue = (int32_t *)malloc((size_t)qcap * sizeof(int32_t));
        if (!cost || !cstamp || !mark || !queue) failed = 1;
        else {
            /* one source per scheduling step, heaviest (given) order first */
#pragma omp for schedule(dynamic, 1)
            for (int32_t i = 0; i < ns; i++) {
                int32_t s = sources ? sources[i] : (n - 1 - i);
                int64_t lo = 0, hi = 0;
                if (maxid_one(s, beg, end, adj, cost, cstamp, mark, queue, qcap,
                              &lo, &hi, NULL) < 0) { failed = 1; continue; }
                if (fills_lo) fills_lo[s] = lo;
                if (fills_hi) fills_hi[s] = hi;
                total += lo + hi;
            }
        }
        free(cost); free(cstamp); free(mark); free(queue);
    }
    return failed ? -1 : total;
}

int64_t gsofa_oracle_maxid_fills(int32_t n, const int32_t *beg,
                                 const int32_t *end, const int32_t *adj,
                                 int64_t adj_len, int nthreads,
                                 int64_t *fills_lo, int64_t *fills_hi)
{
    return gsofa_oracle_maxid_counts(n, beg, end, adj, adj_len, nthreads, NULL, 0,
                                     fills_lo, fills_hi);
}

int32_t gsofa_oracle_maxid_line(int32_t n, const int32_t *beg,
                                const int32_t *end, const int32_t *adj,
                                int64_t adj_len, int32_t s, int32_t *out)
{
    if (validate(n, beg, end, adj, adj_len) || s < 0 || s >= n || !out) return -1;
    const int64_t qcap = 4 * (int64_t)n + 1024;
    uint32_t *cost = (uint32_t *)malloc((size_t)n * sizeof(uint32_t));
    int32_t *cstamp = (int32_t *)calloc((size_t)n, sizeof(int32_t));
    int32_t *mark = (int32_t *)calloc((size_t)n, sizeof(int32_t));
    int32_t *queue = (int32_t *)malloc((size_t)qcap * sizeof(int32_t));
    int64_t lo, hi, r = -1;
    if (cost && cstamp && mark && queue) {
        r = maxid_one(s, beg, end, adj, cost, cstamp, mark, queue, qcap, &lo,
                      &hi, out);
        if (r > 0) qsort(out, (size_t)r, sizeof(int32_t), cmp_i32);
    }
    free(cost); free(cstamp); free(mark); free(queue);
    return (int32_t)r;
}

/* ------------------------------------------------------------------------ */
/* Reverse Cuthill-McKee ordering (the step before the path: the reference
 * takes its input already ordered).  Restates the published algorithms --
 * Cuthill and McKee (1969), breadth-first levels with each vertex's unvisited
 * neighbours appended by increasing degree; George and Liu (1979), the
 * pseudo-peripheral start vertex; the order reversed at the end -- with every
 * tie broken by vertex id, so the result is one well-defined permutation:
 *
 *   S = A + A^T without the diagonal and duplicates; deg(v) = |S(v)|; the
 *   key of v is (deg(v), v).
 *   While vertices remain: start = the unordered vertex of least key.
 *     George-Liu: r = start; repeat { BFS from r; c = the vertex of least key
 *     in the last level; if ecc(c) > ecc(r) then r = c else stop }.
 *     Cuthill-McKee from r: a FIFO queue; each dequeued vertex appends its
 *     unordered neighbours in key order.
 *   perm[k] = the (n-1-k)-th vertex of the whole Cuthill-McKee sequence.
 *
 * perm[new] = old.  Returns 0, or nonzero on invalid input or allocation
 * failure. */
static int32_t *g_rcm_deg;   /* key order for qsort (single-threaded) */
static int cmp_key(const void *a, const void *b)
{
    const int32_t x = *(const int32_t *)a, y = *(const int32_t *)b;
    if (g_rcm_deg[x] != g_rcm_deg[y]) return g_rcm_deg[x] < g_rcm_deg[y] ? -1 : 1;
    return (x > y) - (x < y);
}

/* BFS from r over the unordered vertices (ord < 0), levels into lev[];
 * returns the eccentricity and the vertex of least key in the last level. */
static int32_t rcm_bfs(int32_t r, const int64_t *sp, const int32_t *sa, const int32_t *deg,
                       const int32_t *ord, int32_t *lev, int32_t *queue, int32_t *last_min)
{
    int64_t head = 0, tail = 0;
    queue[tail++] = r;
    lev[r] = 0;
    int32_t ecc = 0;
    while (head < tail) {
        const int32_t v = queue[head++];
        for (int64_t k = sp[v]; k < sp[v + 1]; k++) {
            const int32_t u = sa[k];
            if (ord[u] >= 0 || lev[u] >= 0) continue;
            lev[u] = lev[v] + 1;
            if (lev[u] > ecc) ecc = lev[u];
            queue[tail++] = u;
        }
    }
    int32_t best = -1;
    for (int64_t i = 0; i < tail; i++) {
        const int32_t v = queue[i];
        if (lev[v] == ecc && (best < 0 || deg[v] < deg[best] || (deg[v] == deg[best] && v < best))) best = v;
    }
    for (int64_t i = 0; i < tail; i++) lev[queue[i]] = -1;
    *last_min = best;
    return ecc;
}

int gsofa_oracle_rcm(int32_t n, const int32_t *beg, const int32_t *end, const int32_t *adj,
                     int64_t adj_len, int32_t *perm)
{
    if (validate(n, beg, end, adj, adj_len) || (n > 0 && !perm)) return 1;
    if (n == 0) return 0;
    /* S: both directions of every off-diagonal entry, each row sorted and
     * without duplicates */
    int64_t *cnt = (int64_t *)calloc((size_t)n + 1, sizeof(int64_t));
    if (!cnt) return 2;
    for (int32_t v = 0; v < n; v++)
        for (int32_t k = beg[v]; k < end[v]; k++)
            if (adj[k] != v) { cnt[v + 1]++; cnt[adj[k] + 1]++; }
    for (int32_t v = 0; v < n; v++) cnt[v + 1] += cnt[v];
    int32_t *sa = (int32_t *)malloc(((size_t)cnt[n] + 1) * sizeof(int32_t));
    int64_t *at = (int64_t *)malloc(((size_t)n + 1) * sizeof(int64_t));
    int64_t *sp = (int64_t *)malloc(((size_t)n + 1) * sizeof(int64_t));
    int32_t *deg = (int32_t *)malloc((size_t)n * sizeof(int32_t));
    int32_t *ord = (int32_t *)malloc((size_t)n * sizeof(int32_t));
    int32_t *lev = (int32_t *)malloc((size_t)n * sizeof(int32_t));
    int32_t *queue = (int32_t *)malloc((size_t)n * sizeof(int32_t));
    int32_t *bykey = (int32_t *)malloc((size_t)n * sizeof(int32_t));
    int32_t *cm = (int32_t *)malloc((size_t)n * sizeof(int32_t));
    int32_t *buf = (int32_t *)malloc((size_t)n * sizeof(int32_t));
    int rc = 0;
    if (!sa || !at || !sp || !deg || !ord || !lev || !queue || !bykey || !cm || !buf) { rc = 2; goto done; }
    for (int32_t v = 0; v < n; v++) at[v] = cnt[v];
    for (int32_t v = 0; v < n; v++)
        for (int32_t k = beg[v]; k < end[v]; k++)
            if (adj[k] != v) { sa[at[v]++] = adj[k]; sa[at[adj[k]]++] = v; }
    sp[0] = 0;
    for (int32_t v = 0; v < n; v++) {
        const int64_t b = cnt[v], e = cnt[v + 1];
        qsort(sa + b, (size_t)(e - b), sizeof(int32_t), cmp_i32);
        int64_t w = sp[v];
        for (int64_t k = b; k < e; k++)
            if (k == b || sa[k] != sa[k - 1]) sa[w++] = sa[k];
        sp[v + 1] = w;
        deg[v] = (int32_t)(w - sp[v]);
    }
    /* compacted rows: sa[sp[v] .. sp[v+1]) (sp[v] <= cnt[v], writes trail reads) */
    for (int32_t v = 0; v < n; v++) { ord[v] = -1; lev[v] = -1; bykey[v] = v; }
    g_rcm_deg = deg;
    qsort(bykey, (size_t)n, sizeof(int32_t), cmp_key);
    {
        int32_t pos = 0, cursor = 0;
        while (pos < n) {
            while (ord[bykey[cursor]] >= 0) cursor++;
            int32_t r = bykey[cursor], c = -1;
            int32_t ecc = rcm_bfs(r, sp, sa, deg, ord, lev, queue, &c);
            for (;;) {
                int32_t c2 = -1;
                const int32_t ecc_c = rcm_bfs(c, sp, sa, deg, ord, lev, queue, &c2);
                if (ecc_c <= ecc) break;
                r = c;
                ecc = ecc_c;
                c = c2;
            }
            /* Cuthill-McKee from r */
            int32_t head = pos;
            cm[pos] = r;
            ord[r] = pos++;
            while (head < pos) {
                const int32_t v = cm[head++];
                int32_t m = 0;
                for (int64_t k = sp[v]; k < sp[v + 1]; k++)
                    if (ord[sa[k]] < 0) { buf[m++] = sa[k]; ord[sa[k]] = n; }   /* taken */
                qsort(buf, (size_t)m, sizeof(int32_t), cmp_key);
                for (int32_t i = 0; i < m; i++) { cm[pos] = buf[i]; ord[buf[i]] = pos++; }
            }
        }
    }
    for (int32_t k = 0; k < n; k++) perm[k] = cm[n - 1 - k];
done:
    free(cnt); free(sa); free(at); free(sp); free(deg); free(ord); free(lev); free(queue);
    free(bykey); free(cm); free(buf);
    return rc;
}

// gsofa_device.cuh -- device code of the B200 symbolic factorization.
//
// Layout of one factorization job in HBM (all matrices of a batch share it):
//   per matrix  : n, line_base, G = (ptr[n+1], adj[]) and G^T = (ptr, adj),
//                 compact int32 CSR without diagonal entries;
//   per line l  : cnt[2][L] int32   -- |hi(s)| of pass 0 (U row) / 1 (L column)
//                 nxt[2][L] uint8   -- s+1 in hi(s)
//                 poff[2][L] int64  -- where the sorted hi(s) list sits in pool
//                 gptr[2][L+1] int64-- CSR offsets after compaction
//                 lrow[L] int32     -- |L row s| (histogram of the L columns)
//                 snind[L] uint8    -- line starts a supernode
//   pool / out  : int32 pattern entries (the traversals write pool, one range
//                 per chain of sources; compaction writes out in line order);
//   stamp       : pattern mode, per traversal: n uint16, the chain index at
//                 which each vertex was first set;
//   per CTA     : frontier queue of qcap int32 (every vertex enters at most
//                 once per source, so qcap >= n never overflows).
// The per-source visited set is an n-bit bitmap in shared memory.
#pragma once

#include <cooperative_groups.h>
#include <stdint.h>

namespace gsofa {
namespace dev {

namespace cg = cooperative_groups;

// Rows of at most SLOT_NB ids are also kept whole in a 32-byte slot per
// vertex -- {degree, row offset, up to six ids} -- so expanding a frontier
// vertex is one L2 round trip instead of two (row bounds, then ids); longer
// rows take their ids from adj at the slot's offset.  Matrices whose mean
// off-diagonal degree is above SLOT_NB have no slots (slot == nullptr): most
// of their rows would pay the 32-byte slot load and still read adj.
constexpr int SLOT_NB = 6;

struct PassGraph {
    const int32_t *ptr;  // [n+1]
    const int32_t *adj;  // [ptr[n]]
    const int4 *slot;    // [2n]: vertex v at slot[2v], slot[2v+1] (or null)
};

struct MatDesc {
    int32_t n;
    int32_t pad;
    int64_t line_base;   // first line of this matrix in the job's line space
    PassGraph g[2];      // 0: G, 1: G^T
    const int32_t *rawdeg; // [n] input degree of every line (work counters)
};

// The sources of one matrix, s = offset + stride * j for j in [0, nj), cut
// into pieces of consecutive j.  Piece k of a range covers pass k & 1 (one
// pass per piece unless paired) and piece k >> 1 (k, paired) counted from the
// top: the highest sources, which carry the largest traversals, are handed
// out first.  The top nj - tail sources go in pieces of `chunk`, the bottom
// `tail` ones in pieces of `small`, handed out last, so a launch ends on
// short pieces instead of waiting for a long one.
struct Range {
    int32_t mat;
    int32_t chunk;
    int32_t nj;
    int32_t stride;
    int32_t offset;
    int32_t small;       // piece length of the bottom `tail` sources
    int32_t tail;
    int32_t pad;
    int64_t piece_base;  // first global piece index of this range
    int64_t npieces;     // pieces of both passes
};

// Sources [j0, j1) of piece c of a range, counted from its top.
__host__ __device__ inline void piece_bounds(const Range &rg, int64_t c, int64_t &j0, int64_t &j1)
{
    const int64_t top = (int64_t)rg.nj - rg.tail;
    const int64_t nb = (top + rg.chunk - 1) / rg.chunk;
    if (c < nb) {
        j1 = (int64_t)rg.nj - c * rg.chunk;
        j0 = j1 - rg.chunk > (int64_t)rg.tail ? j1 - rg.chunk : (int64_t)rg.tail;
    } else {
        j1 = (int64_t)rg.tail - (c - nb) * rg.small;
        j0 = j1 - rg.small > 0 ? j1 - rg.small : 0;
    }
}

// Pieces of one pass of a range.
__host__ __device__ inline int64_t pieces_per_pass(const Range &rg)
{
    const int64_t top = (int64_t)rg.nj - rg.tail;
    return (top + rg.chunk - 1) / rg.chunk + ((int64_t)rg.tail + rg.small - 1) / rg.small;
}

// Error bits reported through JobArgs::status.
enum : uint32_t {
    ERR_POOL_OVERFLOW = 1u,
    ERR_QUEUE_OVERFLOW = 2u,
    ERR_COUNT_MISMATCH = 4u,   // a list's running count and its bitmap disagree
};

struct JobArgs {
    const MatDesc *mats;
    int32_t nmats;
    int32_t nranges;
    const Range *ranges;
    int64_t npieces;
    unsigned long long *piece_counter; // dynamic fetch of work pieces
    int32_t *queue;            // gridDim.x * qcap
    int64_t qcap;
    int32_t bitmap_words;      // shared-memory bitmap size (>= max n / 32, multiple of 128)
    int32_t state_words;       // bitmap + its two summary levels
    int32_t ring_size;         // shared-memory frontier ring entries (power of two)
    int32_t lanes;             // lanes per frontier vertex: 1 (thread per vertex,
                               // warp for long rows) or 4..32
    int32_t reuse;
    int32_t want_pattern;
    int32_t max_sn;
    int64_t L;                 // total lines
    int32_t *cnt;              // [2][L]
    uint8_t *nxt;              // [2][L]
    int64_t *poff;             // [2][L]
    int32_t *pool;
    int64_t pool_cap;
    unsigned long long *pool_tail;
    int64_t *gptr;             // [2][L+1]
    int32_t *out;              // pool_cap entries
    int32_t *lrow;             // [L]
    uint8_t *snind;            // [L]
    int32_t *sn_list;          // [L]
    int64_t *mat_info;         // [nmats][3] at each matrix's first line: pass-0 and
                               // pass-1 CSR offsets, supernodes before it
    int64_t ntiles;
    int64_t tile_lo, tile_hi;  // the post-traversal phases cover tiles [tile_lo, tile_hi)
                               // (all of them, unless only a line range was processed)
    int64_t *tile_sum;         // [2][ntiles] then exclusive prefix (in place)
    int64_t *tile_last;        // [ntiles] last supernode-run start, then prefix max
    int64_t *tile_sn;          // [ntiles] then exclusive prefix
    unsigned long long *counters; // [0] edges inspected, [1] sources, [2] sn total,
                                  // [3] pass-G expansions, [4] pass-G input degrees,
                                  // [5] levels, [6] sources that reused state,
                                  // [7..13] cycles: seeding, levels, fold, count,
                                  // list output, clearing, pair wait;
                                  // [14] ns until the traversals ended,
                                  // [15] CTAs' traversal ns, summed
    uint32_t *status;
    uint16_t *stamp;           // pattern mode: per traversal, stamp_stride entries:
    int64_t stamp_stride;      // the chain index at which each vertex was first set
    uint32_t *gbm;             // global-state kernels: per traversal, state_words
                               // words (bitmap and its summaries) in global memory
    unsigned int *blk_done;    // ranges form, streamed: entries written into each
    int32_t blk_shift;         // pool block of 2^blk_shift entries (or null)
};

constexpr int TILE = 2048;     // lines per tile in the post-traversal phases
constexpr int HEAVY_ROW = 32;  // rows longer than this are expanded by a whole warp

__device__ __forceinline__ int64_t warp_incl_scan(int64_t x)
{
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int64_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    return x;
}

// Exclusive scan over the block; *total receives the block sum.  Uses
// s_warp[32]; contains two __syncthreads and a trailing one.
template <int BLOCK>
__device__ __forceinline__ int64_t block_excl_scan(int64_t v, int64_t *total,
                                                   int64_t *s_warp)
{
    constexpr int NW = BLOCK / 32;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int64_t x = warp_incl_scan(v);
    if (lane == 31) s_warp[wid] = x;
    __syncthreads();
    if (wid == 0) {
        int64_t w = lane < NW ? s_warp[lane] : 0;
        w = warp_incl_scan(w);
        if (lane < NW) s_warp[lane] = w;
    }
    __syncthreads();
    int64_t pre = wid ? s_warp[wid - 1] : 0;
    *total = s_warp[NW - 1];
    __syncthreads();
    return pre + x - v;
}

template <int BLOCK>
__device__ __forceinline__ int64_t block_sum(int64_t v, int64_t *s_warp)
{
    int64_t t;
    block_excl_scan<BLOCK>(v, &t, s_warp);
    return t;
}

// Exclusive max-scan over the block (identity -1); *total receives the
// block maximum.
template <int BLOCK>
__device__ __forceinline__ int64_t block_excl_max(int64_t v, int64_t *total,
                                                  int64_t *s_warp)
{
    constexpr int NW = BLOCK / 32;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int64_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int64_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x = max(x, y);
    }
    int64_t ex = __shfl_up_sync(0xffffffffu, x, 1);
    if (lane == 0) ex = -1;
    if (lane == 31) s_warp[wid] = x;
    __syncthreads();
    if (wid == 0) {
        int64_t w = lane < NW ? s_warp[lane] : -1;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int64_t y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w = max(w, y);
        }
        if (lane < NW) s_warp[lane] = w;
    }
    __syncthreads();
    int64_t pre = wid ? s_warp[wid - 1] : -1;
    *total = s_warp[NW - 1];
    __syncthreads();
    return max(pre, ex);
}

// Global load; CG = true reads through L2 only (no L1), for data that the
// host may rewrite while a persistent kernel runs.
template <bool CG>
__device__ __forceinline__ int32_t ld(const int32_t *p)
{
    if (CG) return __ldcg(p);
    return *p;
}

template <bool CG>
__device__ __forceinline__ int4 ld4(const int4 *p)
{
    if (CG) return __ldcg(p);
    return *p;
}

// Words of a bitmap's first summary level (the bitmap is followed directly by
// its summary, so their distance is the bitmap size).
__device__ __forceinline__ int bm_summary_words(const uint32_t *bm, const uint32_t *summ)
{
    return (int)(summ - bm) >> 5;
}

// Bit test-and-set in the shared-memory bitmap; true when this call set it.
// summ holds one bit per bitmap word, set when that word first becomes
// nonzero, so output scans can skip empty stretches 32 words at a time.
// summ is followed by a second level (one bit per summary word, i.e. per
// 32K vertices) at summ + summary_words; SUMM2_OFF gives that offset.
// GBM: the bitmap lives in global memory (L2), where a read before the
// atomic would cost as much as the atomic itself, so the atomic goes first.
template <bool GBM>
__device__ __forceinline__ bool test_and_set(uint32_t *bm, uint32_t *summ, int32_t m)
{
    const uint32_t bit = 1u << (m & 31);
    const int wi = m >> 5;
    uint32_t *w = bm + wi;
    if (!GBM && (*reinterpret_cast<volatile uint32_t *>(w) & bit)) return false;
    const uint32_t old = atomicOr(w, bit);
    if (old == 0u) {
        const int si = wi >> 5;
        const uint32_t olds = atomicOr(summ + si, 1u << (wi & 31));
        if (olds == 0u) atomicOr(summ + (bm_summary_words(bm, summ)) + (si >> 5), 1u << (si & 31));
    }
    return !(old & bit);
}

// Reads a word of a traversal's state: from shared memory, or (GBM) from
// global memory through L2 only -- its words change by atomics in L2 and are
// cleared by plain stores, so an L1 copy could be stale.
template <bool GBM>
__device__ __forceinline__ uint32_t bm_word(const uint32_t *p)
{
    if (GBM) return __ldcg(p);
    return *p;
}

// Frontier queue of one source: absolute positions 0, 1, 2, ... in BFS order.
// A position p written while the writer's level started at w0 lives in the
// shared-memory ring (ring_size entries, a power of two) when
// p - w0 < ring_size and in the CTA's global spill array otherwise; readers
// apply the same rule with the same w0.  Ring entries of one level and of the
// level it feeds always lie within ring_size consecutive positions, so live
// ring slots never collide.
struct Frontier {
    int32_t *ring;    // shared memory
    int32_t *spill;   // global memory, qcap entries (this CTA's slice)
    int64_t qcap;
    uint32_t *status;
    int ring_size;
};

__device__ __forceinline__ void fr_put(const Frontier &f, int p, int w0, int32_t m)
{
    if (p - w0 < f.ring_size) f.ring[p & (f.ring_size - 1)] = m;
    else if ((int64_t)p < f.qcap) f.spill[p] = m;
    else atomicOr(f.status, ERR_QUEUE_OVERFLOW);  // cannot happen: p < n <= qcap
}

__device__ __forceinline__ int32_t fr_get(const Frontier &f, int p, int w0)
{
    return (p - w0 < f.ring_size) ? f.ring[p & (f.ring_size - 1)] : f.spill[p];
}

// Appends m to the next level; one shared atomic per coalesced group of lanes
// (warp-aggregated enqueue).  base: first position of the next level;
// w0: first position of the current level.
__device__ __forceinline__ void push(const Frontier &f, int *tail, int base, int w0, int32_t m)
{
    cg::coalesced_group g = cg::coalesced_threads();
    int b = 0;
    if (g.thread_rank() == 0) b = atomicAdd(tail, (int)g.size());
    b = g.shfl(b, 0);
    fr_put(f, base + b + (int)g.thread_rank(), w0, m);
}

// Seeding window: the rows of up to SEED_WIN consecutive sources (SEED_ADJ
// ids at most), loaded together -- consecutive rows are one stretch of the
// adjacency array -- so a source's seeding reads shared memory instead of
// waiting on two dependent L2 round trips.
constexpr int SEED_WIN = 32;
constexpr int SEED_ADJ = 512;

struct SharedState {
    long long piece;
    int flag;
    int tailc[3];     // level entry counts by phase (barrier-synchronised levels)
    int fetch[3];     // dynamic fetch counters by phase
    int chain_lo;     // lowest vertex set in the bitmap since the last clear
    int chain_hi;     // highest vertex set since the last clear
    int seg[2];       // piece boundaries after chain alignment
    int stail;        // entries of the next level, counted while warp 0 runs levels alone
    int solo_start, solo_wstart, solo_count;   // where such a run ended
    int64_t warp[32]; // per-warp entry counts of a chain's last list (list output)
    int64_t last_off; // pool offset of a chain's last list (-1: pool short)
    int last_cnt;     // its entries
    // tallies kept by the half's first thread only: levels, then cycles of
    // seeding, level loop, range fold, count and link flag, list output (per
    // chain), bitmap clearing, wait for the other pass; sources; reused
    // sources
    unsigned long long prof[8];
    unsigned long long nsrc, nreuse;
    int hcount;        // set bits above the current source (|hi(s)| once done)
    // the current chain -- consecutive sources sharing one bitmap -- whose
    // lists are written when it ends (pattern mode)
    uint16_t *stamp;   // this traversal's stamp row, or null (counts only)
    int chain_s0;      // its first source
    int chain_len;     // its sources so far (the current one included)
    int64_t chain_total;  // entries of its lists
    // the seeding window: sources [win_lo, win_hi) of the current piece
    int win_lo, win_hi;
    int32_t win_ptr[SEED_WIN + 1];   // their row bounds in adj
    int32_t win_raw[SEED_WIN];       // their input degrees (work counters)
    int32_t win_adj[SEED_ADJ];       // adj[win_ptr[0] .. win_ptr[win_hi - win_lo])
};

// Records that v was first set while the chain's source `idx` ran (sources
// of a chain are consecutive, so idx = s - chain_s0).  Only vertices above
// the chain's first source can appear in its lists.
__device__ __forceinline__ void stamp_set(const SharedState &sh, int32_t v, int idx, int32_t chain_s0)
{
    uint16_t *st = sh.stamp;
    if (st != nullptr && v > chain_s0) st[v] = (uint16_t)idx;
}

// Clears the bitmap words covering vertices [lo, hi]; gtid/GT: the calling
// thread's index and the size of the thread group that shares the bitmap.
template <int GT>
__device__ __forceinline__ void clear_range(uint32_t *bm, uint32_t *summ, int lo, int hi, int gtid)
{
    if (hi < lo) return;
    for (int w = (lo >> 5) + gtid; w <= (hi >> 5); w += GT) bm[w] = 0u;
    for (int w = (lo >> 10) + gtid; w <= (hi >> 10); w += GT) summ[w] = 0u;
    uint32_t *summ2 = summ + bm_summary_words(bm, summ);
    for (int w = (lo >> 15) + gtid; w <= (hi >> 15); w += GT) summ2[w] = 0u;
}

// Visits the nonzero chunks c in [c0, c1) (chunk = 32 bitmap words = one
// summary word) in increasing order, using the second summary level to skip
// empty stretches; fn(c) runs warp-uniformly.
template <bool GBM, class F>
__device__ __forceinline__ void for_nonzero_chunks(const uint32_t *summ2, int c0, int c1, F fn)
{
    int c = c0;
    while (c < c1) {
        const int wb = c & ~31;
        uint32_t m = bm_word<GBM>(summ2 + (wb >> 5)) & (~0u << (c & 31));
        if (c1 - wb < 32) m &= (1u << (c1 - wb)) - 1u;
        while (m) {
            const int b = __ffs(m) - 1;
            m &= m - 1u;
            fn(wb + b);
        }
        c = wb + 32;
    }
}

// Barrier of the GT threads that work on one traversal: the whole CTA
// (bar == 0) or one half of it (named barrier `bar`).
template <int GT>
__device__ __forceinline__ void gsync(int bar)
{
    if (bar == 0) __syncthreads();
    else if (bar == 1) asm volatile("bar.sync 1, %0;" ::"n"(GT) : "memory");
    else asm volatile("bar.sync 2, %0;" ::"n"(GT) : "memory");
}

// True when x-1 is in adj(x); evaluated by one whole warp.
__device__ __forceinline__ bool warp_has_prev(const PassGraph &g, int32_t x)
{
    const int lane = threadIdx.x & 31;
    bool hit = false;
    for (int32_t k = g.ptr[x] + lane; k < g.ptr[x + 1]; k += 32)
        hit |= (g.adj[k] == x - 1);
    return __any_sync(0xffffffffu, hit);
}

// The chain start at or below x: the lowest y with y+1 .. x each holding its
// predecessor, searched at most `limit - 1` steps down; x itself when the
// chain reaches further (then the cut is not aligned).  Warp 0 only.
__device__ __forceinline__ int32_t chain_start(const PassGraph &g, int32_t x, int32_t limit)
{
    int32_t y = x;
    for (int step = 0; step < limit - 1; step++) {
        if (y == 0 || !warp_has_prev(g, y)) return y;
        y--;
    }
    return (y == 0 || !warp_has_prev(g, y)) ? y : x;
}

// Visits neighbour m of a frontier vertex: marks it, and queues it for the
// next level when it lies below the source, else counts it in nh (new
// vertices above the source).
#define GSOFA_VISIT(m)                                                          \
    do {                                                                        \
        const int32_t _m = (m);                                                 \
        if (test_and_set<GBM>(bm, summ, _m)) {                                        \
            t_lo = min(t_lo, _m);                                               \
            t_hi = max(t_hi, _m);                                               \
            stamp_set(sh, _m, cidx, s - cidx);                                            \
            if (_m < s) push(f, tailp, end, start, _m);                         \
            else nh++;                                                          \
        }                                                                       \
    } while (0)

// One source s of one pass: seeds from adj(s), expands the frontier level by
// level through vertices < s, then records |hi(s)| and the s+1 link flag (the
// list itself is written when the chain of sources ends, output_chain).
// When the caller reuses state, the bitmap still holds the finished traversal
// of s-1, which is valid whenever s-1 is in X(s): then X(s-1) u {s-1} is inside
// X(s) and hi(s-1) minus {s} is inside hi(s).
// END_SYNC: finish with a barrier of the traversal's threads (not needed when
// the caller's next step is a barrier of the whole CTA).
//
// The level counters (tailc, fetch) are zero on entry: the previous source
// left them so.  s_end: the end of the piece (the seeding window stays within
// it); stride: the distance between the piece's sources; cidx: the index of
// s in its chain (every thread tracks it; a chain's sources are consecutive,
// so it starts at s - cidx).
template <int GT, bool CG, bool END_SYNC, bool GBM>
__device__ void process_source(const JobArgs &a, const PassGraph g, int32_t n,
                               int64_t line, int pass, int32_t s, int32_t s_end, int32_t stride,
                               int cidx, uint32_t *bm, uint32_t *summ,
                               const Frontier &f, SharedState &sh,
                               unsigned long long &edges, const int32_t *rawdeg,
                               unsigned long long &xcnt, unsigned long long &einsp,
                               unsigned long long *prof, const int gtid, const int bar)
{
    const int tid = gtid;
    const int lane = tid & 31;
    const int lanes = a.lanes;
    const int lane_in_group = tid & (lanes - 1);
    int t_lo = INT32_MAX, t_hi = -1;

    long long c0 = 0;
    if (tid == 0) c0 = clock64();
    // a new seeding window when s is past the current one (consecutive
    // sources only): row bounds, then the rows themselves, all threads
    int wlo = sh.win_lo, whi = sh.win_hi;   // stable: set behind earlier barriers
    if (stride == 1 && (s < wlo || s >= whi)) {
        const int hi0 = min(s_end, s + SEED_WIN);
        for (int i = tid; i <= hi0 - s; i += GT) {
            sh.win_ptr[i] = ld<CG>(g.ptr + s + i);
            if (i < hi0 - s) sh.win_raw[i] = ld<CG>(rawdeg + s + i);
        }
        gsync<GT>(bar);
        int k = hi0 - s;   // rows that fit
        while (k > 0 && sh.win_ptr[k] - sh.win_ptr[0] > SEED_ADJ) k--;
        const int32_t a0 = sh.win_ptr[0], na = sh.win_ptr[k] - a0;
        for (int i = tid; i < na; i += GT) sh.win_adj[i] = ld<CG>(g.adj + a0 + i);
        gsync<GT>(bar);
        wlo = s;
        whi = s + k;
        if (tid == 0) { sh.win_lo = wlo; sh.win_hi = whi; }   // read by later sources
    }
    const bool in_win = stride == 1 && s >= wlo && s < whi;
    if (tid == 0) {
        sh.chain_len = cidx + 1;
        if (test_and_set<GBM>(bm, summ, s)) { t_lo = s; t_hi = s; stamp_set(sh, s, cidx, s - cidx); }
        else atomicAdd(&sh.hcount, -1);   // s was in hi(s-1): counted, but not above s
    }
    // No barrier here: seeding pushes onto the zeroed level-0 counter, the
    // stamps take the thread's own cidx, and s itself (which no neighbour of
    // s is) is set before the level loop's first barrier.

    // seeding: every neighbour of s is structure of line s; level-0 items
    {
        int32_t b0, e0;
        if (in_win) {
            b0 = sh.win_ptr[s - wlo];
            e0 = sh.win_ptr[s - wlo + 1];
        } else {
            b0 = ld<CG>(g.ptr + s);
            e0 = ld<CG>(g.ptr + s + 1);
        }
        if (tid == 0) {
            edges += (unsigned long long)(e0 - b0);
            if (pass == 0) einsp += (unsigned long long)(in_win ? sh.win_raw[s - wlo] : ld<CG>(rawdeg + s));
        }
        int *tailp = &sh.tailc[0];
        const int end = 0, start = 0;
        int nh = 0;
        if (in_win) {
            const int32_t *wa = sh.win_adj - sh.win_ptr[0];
            for (int32_t k = b0 + tid; k < e0; k += GT) GSOFA_VISIT(wa[k]);
        } else {
            for (int32_t k = b0 + tid; k < e0; k += GT) GSOFA_VISIT(ld<CG>(g.adj + k));
        }
        nh = (int)__reduce_add_sync(0xffffffffu, (unsigned)nh);
        if (lane == 0 && nh) atomicAdd(&sh.hcount, nh);
    }
    long long cs = 0;
    if (tid == 0) { cs = clock64(); prof[1] += (unsigned long long)(cs - c0); }

    // One warp's step of a level (one thread per vertex): items base ..
    // base + 31 of the level [start, end), whose entries were written while
    // the level starting at wstart ran; new vertices below s go to the next
    // level through tailp.  Each lane loads its row bounds and then up to
    // eight adjacency ids at once (independent loads in flight hide the L2
    // latency).  The id loop runs to the warp's longest light row so every
    // step is warp-uniform and new vertices below s are enqueued with one
    // ballot and one shared atomic.  Rows longer than HEAVY_ROW are expanded
    // by the whole warp.
    auto warp_step = [&](const int base, const int start, const int end, const int wstart, int *const tailp) {
        const int it = base + lane;
        int32_t b = 0, d = 0;
        int4 sl0 = make_int4(0, 0, -1, -1), sl1 = make_int4(-1, -1, -1, -1);
        if (it < end) {
            const int32_t v = fr_get(f, it, wstart);
            if (g.slot != nullptr) {   // degree, offset and short rows in one 32-byte load
                sl0 = ld4<CG>(g.slot + 2 * (int64_t)v);
                sl1 = ld4<CG>(g.slot + 2 * (int64_t)v + 1);
                d = sl0.x;
                b = sl0.y;
            } else {
                b = ld<CG>(g.ptr + v);
                d = ld<CG>(g.ptr + v + 1) - b;
            }
            edges += (unsigned long long)d;
            if (pass == 0) { xcnt++; einsp += (unsigned long long)ld<CG>(rawdeg + v); }
        }
        // the row's ids are in the slot (first step of the id loop)
        const bool in_slot = g.slot != nullptr && d <= SLOT_NB;
        unsigned heavy = __ballot_sync(0xffffffffu, d > HEAVY_ROW);
        while (heavy) {
            const int src = __ffs(heavy) - 1;
            heavy &= heavy - 1u;
            const int32_t hb = __shfl_sync(0xffffffffu, b, src);
            const int32_t hd = __shfl_sync(0xffffffffu, d, src);
            for (int32_t k0 = 0; k0 < hd; k0 += 32) {
                const bool on = k0 + lane < hd;
                const int32_t m = on ? ld<CG>(g.adj + hb + k0 + lane) : 0;
                const bool fresh = on && test_and_set<GBM>(bm, summ, m);
                if (fresh) { t_lo = min(t_lo, m); t_hi = max(t_hi, m); stamp_set(sh, m, cidx, s - cidx); }
                const bool low = fresh && m < s;
                const unsigned bal = __ballot_sync(0xffffffffu, low);
                const unsigned bhi = __ballot_sync(0xffffffffu, fresh) & ~bal;
                if (lane == 0 && bhi) atomicAdd(&sh.hcount, __popc(bhi));
                if (bal) {
                    int pb = 0;
                    if (lane == 0) pb = atomicAdd(tailp, __popc(bal));
                    pb = __shfl_sync(0xffffffffu, pb, 0);
                    if (low) fr_put(f, end + pb + __popc(bal & ((1u << lane) - 1u)), start, m);
                }
            }
        }
        const int dl = d > HEAVY_ROW ? 0 : d;
        const int dmax = __reduce_max_sync(0xffffffffu, dl);
        for (int k0 = 0; k0 < dmax; k0 += 8) {
            int32_t buf[8];
            if (in_slot) {   // d <= 6 < 8: only this first step has ids
                const int32_t sv[SLOT_NB] = {sl0.z, sl0.w, sl1.x, sl1.y, sl1.z, sl1.w};
#pragma unroll
                for (int u = 0; u < 8; u++) buf[u] = (u < SLOT_NB && k0 + u < dl) ? sv[u < SLOT_NB ? u : 0] : -1;
            } else {
#pragma unroll
                for (int u = 0; u < 8; u++) buf[u] = (k0 + u < dl) ? ld<CG>(g.adj + b + k0 + u) : -1;
            }
            // independent bit tests and sets first, then one enqueue
            // (warp scan + one shared atomic) for all new low vertices
            unsigned fresh = 0u;
#pragma unroll
            for (int u = 0; u < 8; u++)
                if (buf[u] >= 0 && test_and_set<GBM>(bm, summ, buf[u])) fresh |= 1u << u;
            // new vertices below s in the low 16 bits, above s in
            // the high ones (a warp step finds at most 256)
            int nlh = 0;
#pragma unroll
            for (int u = 0; u < 8; u++)
                if ((fresh >> u) & 1u) {
                    t_lo = min(t_lo, buf[u]);
                    t_hi = max(t_hi, buf[u]);
                    nlh += buf[u] < s ? 1 : 0x10000;
                }
            if (fresh && sh.stamp != nullptr) {
#pragma unroll
                for (int u = 0; u < 8; u++)
                    if ((fresh >> u) & 1u) stamp_set(sh, buf[u], cidx, s - cidx);
            }
            int incl = nlh;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += y;
            }
            const int wsum = __shfl_sync(0xffffffffu, incl, 31);
            const int wtot = wsum & 0xffff;
            if (lane == 0 && (wsum >> 16)) atomicAdd(&sh.hcount, wsum >> 16);
            if (wtot) {
                int pb = 0;
                if (lane == 0) pb = atomicAdd(tailp, wtot);
                pb = __shfl_sync(0xffffffffu, pb, 0) + ((incl - nlh) & 0xffff);
#pragma unroll
                for (int u = 0; u < 8; u++)
                    if (((fresh >> u) & 1u) && buf[u] < s) fr_put(f, end + pb++, start, buf[u]);
            }
        }
    };

    // level-synchronous expansion through vertices < s, one barrier a level.
    // A level of at most 32 vertices (one per lane) is run by warp 0 alone
    // (solo), and so are the small levels after it, with warp barriers only,
    // while the traversal's other warps wait at the next barrier.  The
    // barrier-synchronised levels count their entries in tailc[] by phase c:
    // the current level's count in tailc[c % 3], the next level's in
    // tailc[(c + 1) % 3] (zero when the level starts), fetch counter
    // fetch[c % 3] (zero too).  Solo levels count in sh.stail only, touched by
    // lane 0 alone, and hand over through sh.solo_* after the next barrier:
    // the phase and its counters are then as they were when the run began.
    int start = 0, wstart = 0, c = 0;
    bool relay = false;   // warp 0 ran levels alone: take up its position
    for (;;) {
        gsync<GT>(bar);
        int end;
        if (relay) {
            start = sh.solo_start;
            wstart = sh.solo_wstart;
            end = start + sh.solo_count;
            relay = false;
        } else {
            end = start + sh.tailc[c % 3];
        }
        if (end == start) break;
        const bool solo = lanes == 1 && end - start <= 32;
        if (solo && tid >= 32) {
            relay = true;
            continue;
        }
        if (tid == 0) prof[0]++;   // levels
        if (!solo && tid == 0) { sh.tailc[(c + 2) % 3] = 0; sh.fetch[(c + 1) % 3] = 0; }
        int *const tailp = solo ? &sh.stail : &sh.tailc[(c + 1) % 3];
        int *const fetchp = &sh.fetch[c % 3];
        if (lanes == 1) {
            // a warp takes 32 queue items with one shared atomic; solo, warp
            // 0 takes the whole level, then the next while it is small
            for (;;) {
                int base = start;
                if (solo) {
                    if (lane == 0) sh.stail = 0;
                } else {
                    if (lane == 0) base = atomicAdd(fetchp, 32);
                    base = __shfl_sync(0xffffffffu, base, 0) + start;
                    if (base >= end) break;
                }
                warp_step(base, start, end, wstart, tailp);
                if (solo) {
                    __syncwarp();   // the level's queue entries, for every lane
                    int nn = 0;
                    if (lane == 0) nn = sh.stail;
                    nn = __shfl_sync(0xffffffffu, nn, 0);
                    wstart = start;
                    start = end;
                    end += nn;
                    if (nn == 0 || nn > 32) {
                        if (lane == 0) {
                            sh.solo_start = start;
                            sh.solo_wstart = wstart;
                            sh.solo_count = nn;
                        }
                        break;
                    }
                    if (lane == 0) prof[0]++;
                }
            }
            if (solo) {
                relay = true;
                continue;
            }
        } else {
            // groups of `lanes` threads per vertex
            const unsigned gmask = (lanes == 32)
                                       ? 0xffffffffu
                                       : (((1u << lanes) - 1u) << (lane & ~(lanes - 1)));
            int nh = 0;
            for (;;) {
                int it = 0;
                if (lane_in_group == 0) it = atomicAdd(fetchp, 1);
                it = __shfl_sync(gmask, it, 0, lanes) + start;
                if (it >= end) break;
                const int32_t v = fr_get(f, it, wstart);
                const int32_t b = ld<CG>(g.ptr + v), e = ld<CG>(g.ptr + v + 1);
                if (lane_in_group == 0) {
                    edges += (unsigned long long)(e - b);
                    if (pass == 0) { xcnt++; einsp += (unsigned long long)ld<CG>(rawdeg + v); }
                }
                for (int32_t k = b + lane_in_group; k < e; k += lanes) GSOFA_VISIT(ld<CG>(g.adj + k));
            }
            nh = (int)__reduce_add_sync(0xffffffffu, (unsigned)nh);
            if (lane == 0 && nh) atomicAdd(&sh.hcount, nh);
        }
        wstart = start;
        start = end;
        c++;
    }
    long long ce = 0;
    if (tid == 0) { ce = clock64(); prof[2] += (unsigned long long)(ce - cs); }

    // fold the touched range into the chain range (warp reduce + shared
    // atomics; it is read only when the bitmap is cleared, after later
    // barriers)
    {
        const int wl = __reduce_min_sync(0xffffffffu, t_lo);
        const int wh = __reduce_max_sync(0xffffffffu, t_hi);
        if (lane == 0) {
            if (wl != INT32_MAX) atomicMin(&sh.chain_lo, wl);
            if (wh >= 0) atomicMax(&sh.chain_hi, wh);
        }
    }
    long long c1 = 0;
    if (tid == 0) { c1 = clock64(); prof[3] += (unsigned long long)(c1 - ce); }

    // |hi(s)| = the bits above s: the traversal's running count, complete
    // since the level loop's last barrier.  The lists themselves are written
    // when the chain ends (output_chain); here only the count and the link
    // flag.
    if (tid == 0) {
        // the next source starts from zeroed level counters (every thread
        // read this one's last, empty level before leaving the loop; the
        // counters of that level are zero already)
        sh.tailc[0] = sh.tailc[1] = sh.tailc[2] = 0;
        sh.fetch[0] = sh.fetch[1] = sh.fetch[2] = 0;
        const int total = sh.hcount;
        const int64_t slot = (int64_t)pass * a.L + line;
        a.cnt[slot] = (int32_t)total;
        const int nx = (s + 1 < n) && ((bm_word<GBM>(bm + ((s + 1) >> 5)) >> ((s + 1) & 31)) & 1u);
        a.nxt[slot] = (uint8_t)nx;
        sh.flag = nx;
        sh.chain_total += total;
    }
    if (END_SYNC) gsync<GT>(bar);
    if (tid == 0) prof[4] += (unsigned long long)(clock64() - c1);
}
#undef GSOFA_VISIT

// Lane's bitmap word of chunk cc, without the bits below word w0 and below
// first_mask in word w0.
template <bool GBM>
__device__ __forceinline__ uint32_t last_word(const uint32_t *bm, const uint32_t *summ, int cc, int lane, int w0,
                                              uint32_t first_mask)
{
    const int w = (cc << 5) + lane;
    uint32_t x = ((bm_word<GBM>(summ + cc) >> lane) & 1u) ? bm_word<GBM>(bm + w) : 0u;
    if (w < w0) x = 0u;
    if (w == w0) x &= first_mask;
    return x;
}

// Writes the lists of the chain that just ended -- sources chain_s0 ..
// chain_s0 + chain_len - 1, which shared one bitmap -- while the bitmap still
// holds the last source's traversal.  Bits are only ever added along a chain,
// so the bits above source i of the chain that were set by the time it
// finished are its list: hi(s_i) = { v > s_i : v set, stamp(v) <= i }.  One
// pool range holds all of the chain's lists.
//
// The last source's list is every set bit above it: all warps write it at
// once from the bitmap (each a share of its chunks, offsets from a count
// pass), into the pool and into `scratch` (this traversal's frontier spill
// array, free once the traversal is done).  Every earlier list i is then the
// chain's own later sources that it reached, followed by the last list's
// entries of stamp <= i: a warp streams the last list from scratch (several
// coalesced loads and their stamps in flight at once) and keeps its entries
// by ballot -- no per-list walk of the bitmap.  Lists of pass G^T (columns
// of L) also count their entries into the L row histogram (fire-and-forget
// reductions that overlap other traversals).
template <int GT, bool GBM>
__device__ void output_chain(const JobArgs &a, int64_t line_base, int pass, const uint32_t *bm,
                             const uint32_t *summ, SharedState &sh, int32_t *scratch, int gtid, int bar)
{
    const int64_t line0 = line_base + sh.chain_s0;
    int32_t *const lrow = pass ? a.lrow + line_base : nullptr;
    constexpr int NWARP = GT / 32;
    const int lane = gtid & 31, wid = gtid >> 5;
    const unsigned below = (1u << lane) - 1u;
    const int s0 = sh.chain_s0, len = sh.chain_len;
    const int64_t row0 = (int64_t)pass * a.L + line0;   // cnt / poff entry of s0

    // The last source's list: set bits in words from w0 on (first_mask on
    // w0), chunks [c_lo, c_hi) shared out among the warps.  Every warp counts
    // its share (shared memory only) while warp 0 also takes the chain's pool
    // range and writes every list's offset; one barrier then covers both.
    const int s_last = s0 + len - 1;
    const int chain_hi = sh.chain_hi;
    const uint32_t *summ2 = summ + bm_summary_words(bm, summ);
    const int w0 = (s_last + 1) >> 5;
    const uint32_t first_mask = ~0u << ((s_last + 1) & 31);
    const int c_lo = w0 >> 5;
    const int c_hi = chain_hi > s_last ? (chain_hi >> 10) + 1 : c_lo;
    const int share = (max(c_hi - c_lo, 0) + NWARP - 1) / NWARP;
    const int my_lo = c_lo + wid * share, my_hi = min(c_hi, my_lo + share);
    if (wid == 0) {
        // one exact range per chain (one global atomic per chain of sources,
        // so the pool holds the lists with no gaps); past the capacity the
        // chain's lists are not written, the tail still advances, and its
        // final value is the capacity the job needs
        long long base = -1;
        if (lane == 0) {
            const int64_t total = sh.chain_total;
            base = 0;
            if (total > 0) {
                const unsigned long long o = atomicAdd(a.pool_tail, (unsigned long long)total);
                base = ((int64_t)o + total <= a.pool_cap) ? (long long)o : -1;
            }
            if (base < 0) atomicOr(a.status, ERR_POOL_OVERFLOW);
        }
        base = __shfl_sync(0xffffffffu, base, 0);
        long long carry = 0;
        for (int i0 = 0; i0 < len; i0 += 32) {
            const int i = i0 + lane;
            const long long c = i < len ? (long long)a.cnt[row0 + i] : 0;
            long long incl = c;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const long long y = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += y;
            }
            const long long off = base >= 0 ? base + carry + incl - c : -1;
            if (i < len) a.poff[row0 + i] = off;
            if (i == len - 1) {
                sh.last_off = off;
                sh.last_cnt = (int)c;
            }
            carry += __shfl_sync(0xffffffffu, incl, 31);
        }
    }
    int mine = 0;
    if (my_lo < my_hi)
        for_nonzero_chunks<GBM>(summ2, my_lo, my_hi, [&](int cc) {
            mine += __popc(last_word<GBM>(bm, summ, cc, lane, w0, first_mask));
        });
    mine = (int)__reduce_add_sync(0xffffffffu, (unsigned)mine);
    if (lane == 0) sh.warp[wid] = mine;
    gsync<GT>(bar);
    const int64_t off_last = sh.last_off;
    const int cnt_last = sh.last_cnt;
    const bool write = off_last >= 0;   // else the pool is short: nothing is written
    if (write) {
        int pos = 0, all = 0;
        for (int k = 0; k < NWARP; k++) {
            const int c = (int)sh.warp[k];
            pos += k < wid ? c : 0;
            all += c;
        }
        if (gtid == 0 && all != cnt_last) atomicOr(a.status, ERR_COUNT_MISMATCH);
        int32_t *const out = a.pool + off_last;
        if (my_lo < my_hi)
            for_nonzero_chunks<GBM>(summ2, my_lo, my_hi, [&](int cc) {
                uint32_t x = last_word<GBM>(bm, summ, cc, lane, w0, first_mask);
                const int pc = __popc(x);
                int incl = pc;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const int y = __shfl_up_sync(0xffffffffu, incl, o);
                    if (lane >= o) incl += y;
                }
                const int excl = incl - pc;
                const int wbase = cc << 5;
                // at most two entries a word: a word per lane; denser chunks
                // a word at a time across the warp (lane = bit), one
                // coalesced run per store.  Nothing lands past the list's
                // own cnt_last entries.
                if (__reduce_max_sync(0xffffffffu, (unsigned)pc) <= 2u) {
                    int at = pos + excl;
                    while (x) {
                        const int bit = __ffs(x) - 1;
                        x &= x - 1u;
                        const int32_t v = ((wbase + lane) << 5) + bit;
                        if (at < cnt_last) {
                            out[at] = v;
                            scratch[at] = v;
                            if (lrow) atomicAdd(lrow + v, 1);
                        }
                        at++;
                    }
                } else {
                    unsigned nzw = __ballot_sync(0xffffffffu, x != 0u);
                    while (nzw) {
                        const int j = __ffs(nzw) - 1;
                        nzw &= nzw - 1u;
                        const uint32_t xj = __shfl_sync(0xffffffffu, x, j);
                        const int pj = __shfl_sync(0xffffffffu, excl, j);
                        const int at = pos + pj + __popc(xj & below);
                        if (((xj >> lane) & 1u) && at < cnt_last) {
                            const int32_t v = ((wbase + j) << 5) + lane;
                            out[at] = v;
                            scratch[at] = v;
                            if (lrow) atomicAdd(lrow + v, 1);
                        }
                    }
                }
                pos += __shfl_sync(0xffffffffu, incl, 31);
            });
    }
    gsync<GT>(bar);

    // every earlier list i: its later chain sources (s_i, s_last] that were
    // reached by then, then the last list's entries of stamp <= i (all above
    // s_last, so the list stays sorted)
    const uint16_t *stamp = sh.stamp;
    for (int i = wid; write && i < len - 1; i += NWARP) {
        const int s = s0 + i;
        const int64_t off = a.poff[row0 + i];
        const int cnt = a.cnt[row0 + i];
        if (cnt == 0) continue;
        int32_t *const out = a.pool + off;
        int pos = 0;
        for (int k0 = s + 1; k0 <= s_last; k0 += 32) {
            const int v = k0 + lane;
            const bool in = v <= s_last && ((bm_word<GBM>(bm + (v >> 5)) >> (v & 31)) & 1u) && (int)stamp[v] <= i;
            const unsigned bal = __ballot_sync(0xffffffffu, in);
            const int at = pos + __popc(bal & below);
            if (in && at < cnt) {
                out[at] = v;
                if (lrow) atomicAdd(lrow + v, 1);
            }
            pos += __popc(bal);
        }
        // UNR loads of the last list and their stamps in flight at once (two
        // where 64 registers a thread must do)
        constexpr int UNR = GT > 384 ? 2 : 4;
        for (int k0 = 0; k0 < cnt_last; k0 += 32 * UNR) {
            int32_t e[UNR];
            int t[UNR];
#pragma unroll
            for (int u = 0; u < UNR; u++) {
                const int k = k0 + 32 * u + lane;
                e[u] = k < cnt_last ? __ldcg(scratch + k) : -1;
            }
#pragma unroll
            for (int u = 0; u < UNR; u++)   // only vertices of the last list (s_last, chain_hi] are read
                t[u] = (e[u] > s_last && e[u] <= chain_hi) ? (int)stamp[e[u]] : INT32_MAX;
#pragma unroll
            for (int u = 0; u < UNR; u++) {
                const bool in = t[u] <= i;
                const unsigned bal = __ballot_sync(0xffffffffu, in);
                const int at = pos + __popc(bal & below);
                if (in && at < cnt) {
                    out[at] = e[u];
                    if (lrow) atomicAdd(lrow + e[u], 1);
                }
                pos += __popc(bal);
            }
        }
        if (lane == 0 && pos != cnt) atomicOr(a.status, ERR_COUNT_MISMATCH);
    }
    gsync<GT>(bar);
    // Streaming: count the chain's entries into the pool blocks they fill.
    // Every list of the chain is written (the barrier above); one fence makes
    // those writes visible device-wide before the counts that let the host
    // copy a full block out while the traversals go on.
    if (a.blk_done != nullptr && gtid == 0 && sh.chain_total > 0) {
        const int64_t base = a.poff[row0];
        if (base >= 0) {
            __threadfence();
            const int64_t end = base + sh.chain_total;
            const int64_t bsz = (int64_t)1 << a.blk_shift;
            for (int64_t b = base >> a.blk_shift; b <= (end - 1) >> a.blk_shift; b++) {
                const int64_t lo = max(base, b * bsz), hi = min(end, (b + 1) * bsz);
                atomicAdd(a.blk_done + b, (unsigned int)(hi - lo));
            }
        }
    }
}

// Per-thread tallies of one CTA's traversals (summed over the CTA at the
// end); the per-source ones live in SharedState, kept by one thread.
struct Tally {
    unsigned long long edges = 0, xcnt = 0, einsp = 0;
};

// The sources s_lo, s_lo + stride, ... < s_hi of one work piece, in order,
// each starting from the previous source's state whenever that is valid.
template <int BLOCK, bool PAIRED, bool CG, bool GBM, bool LISTS = true>
__device__ void run_piece(const JobArgs &a, const MatDesc &md, const PassGraph &g, int pass,
                          int32_t s_lo, int32_t s_hi, int32_t stride, uint32_t *bm, uint32_t *summ,
                          const Frontier &fr, SharedState &sh, int (*pair_flag)[2], int half,
                          int gtid, int bar, Tally &acc)
{
    constexpr int GT = PAIRED ? BLOCK / 2 : BLOCK;
    const int tid = threadIdx.x;
    int prev = -2;
    int idx = 0;
    // the current chain, tracked by every thread alike (decisions never read
    // state another thread may be changing): index of the last source in it
    // (-1: none yet)
    int cidx = -1;
    for (int32_t s = s_lo; s < s_hi; s += stride, idx++) {
        int reuse = 0;
        // chain indices are 16-bit stamps: a chain ends after 65535 sources
        if (a.reuse && prev == s - 1 && !(a.want_pattern && cidx + 1 >= 65535)) {
            if (PAIRED) {
                reuse = pair_flag[(idx - 1) & 1][1 - half];
            } else {
                if (tid < 32) {
                    const bool h = warp_has_prev(g, s);
                    if (tid == 0) sh.flag = h ? 1 : 0;
                }
                __syncthreads();
                reuse = sh.flag;
            }
        }
        if (!reuse) {
            if (LISTS && a.want_pattern && cidx >= 0) {
                const long long co = clock64();
                output_chain<GT, GBM>(a, md.line_base, pass, bm, summ, sh, fr.spill, gtid, bar);
                if (gtid == 0) sh.prof[5] += (unsigned long long)(clock64() - co);
            }
            const long long cc = clock64();
            const int clo = sh.chain_lo, chi = sh.chain_hi;
            clear_range<GT>(bm, summ, clo, chi, gtid);
            // the new chain's counters, in place before the barrier that
            // precedes its first seeding (which adds to hcount)
            if (gtid == 0) { sh.hcount = 0; sh.chain_s0 = s; sh.chain_len = 0; sh.chain_total = 0; }
            gsync<GT>(bar);
            if (gtid == 0) {
                sh.chain_lo = INT32_MAX; sh.chain_hi = -1;
                sh.prof[6] += (unsigned long long)(clock64() - cc);
            }
            cidx = 0;
        } else {
            cidx++;
            if (gtid == 0) sh.nreuse++;
        }
        // paired: the pass-flag exchange below is a barrier of the whole CTA
        process_source<GT, CG, !PAIRED, GBM>(a, g, md.n, md.line_base + s, pass, s, s_hi, stride, cidx,
                                             bm, summ, fr, sh, acc.edges, md.rawdeg, acc.xcnt, acc.einsp,
                                             sh.prof, gtid, bar);
        if (PAIRED) {
            if (gtid == 0) pair_flag[idx & 1][half] = sh.flag;
            const long long cw = clock64();
            __syncthreads();
            if (gtid == 0) sh.prof[7] += (unsigned long long)(clock64() - cw);
        }
        prev = s;
        if (gtid == 0) sh.nsrc++;
    }
    // the piece's last chain
    if (LISTS && a.want_pattern && cidx >= 0) {
        const long long co = clock64();
        output_chain<GT, GBM>(a, md.line_base, pass, bm, summ, sh, fr.spill, gtid, bar);
        if (gtid == 0) {
            sh.prof[5] += (unsigned long long)(clock64() - co);
            sh.chain_len = 0;
        }
    }
}

// ---------------------------------------------------------------------------
// The persistent cooperative factorization kernel.
//
// PAIRED = false: every CTA runs one traversal at a time; a work piece is one
// pass of a run of sources, and s reuses s-1's state when s-1 is in adj(s).
// PAIRED = true: the CTA's two halves run pass G and pass G^T of the same
// source side by side, each with its own bitmap and frontier ring, and
// exchange their s+1 flags after every source.  By the fill-path theorem,
// s-1 is in X_G(s) exactly when s is in hi_{G^T}(s-1) (and likewise with G
// and G^T swapped), so each half reuses s-1's state whenever it is valid.
//
// GBM = true: every traversal's visited bitmap and summaries live in global
// memory (a.gbm, resident in L2 for the sizes that matter) instead of shared
// memory, which then holds only the frontier rings.  A traversal's state no
// longer bounds how many traversals an SM runs (shared memory holds two
// bitmaps of at most ~850K lines each), so small CTAs run many traversals per
// SM side by side, and n is bounded only by device memory.
//
// MINB: resident CTAs per SM the registers are budgeted for (the default
// fills the SM with 1024 threads; 1 gives a 512-thread CTA up to 128
// registers a thread, for launches that hold one CTA per SM anyway).
// LISTS: the list output is compiled in; counts-only jobs run an
// instantiation without it, whose registers go to the traversal alone.
template <int BLOCK, bool PAIRED, bool GBM, int MINB = (BLOCK >= 1024 ? 1 : 1024 / BLOCK), bool LISTS = true>
__global__ void __launch_bounds__(BLOCK, MINB) factor_kernel(JobArgs a)
{
    constexpr int GT = PAIRED ? BLOCK / 2 : BLOCK;
    constexpr int NS = PAIRED ? 2 : 1;
    extern __shared__ __align__(16) uint32_t smem_dyn[];
    __shared__ SharedState shs[NS];
    __shared__ int pair_flag[2][2];   // [source parity][pass]: s+1 in hi(s)
    __shared__ long long s_piece;
    cg::grid_group grid = cg::this_grid();
    const int tid = threadIdx.x;
    const int half = PAIRED ? tid / GT : 0;
    const int gtid = PAIRED ? tid % GT : tid;
    const int bar = PAIRED ? 1 + half : 0;
    SharedState &sh = shs[half];
    uint32_t *const state = GBM ? a.gbm + ((int64_t)blockIdx.x * NS) * a.state_words : smem_dyn;
    uint32_t *bm = state + (size_t)half * a.state_words;
    uint32_t *summ = bm + a.bitmap_words;
    int32_t *ring = (int32_t *)(GBM ? smem_dyn : smem_dyn + (size_t)NS * a.state_words) + (size_t)half * a.ring_size;

    // ---- phase 1: traversals ------------------------------------------------
    unsigned long long t_start = 0;
    if (tid == 0) asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t_start));
    for (int w = tid; w < NS * a.state_words; w += BLOCK) state[w] = 0u;
    if (gtid == 0) {
        sh.chain_lo = INT32_MAX; sh.chain_hi = -1; sh.hcount = 0;
        sh.stamp = a.want_pattern ? a.stamp + ((int64_t)blockIdx.x * NS + half) * a.stamp_stride : nullptr;
        sh.chain_s0 = 0; sh.chain_len = 0; sh.chain_total = 0;
        for (int q = 0; q < 8; q++) sh.prof[q] = 0;
        sh.nsrc = sh.nreuse = 0;
        sh.tailc[0] = sh.tailc[1] = sh.tailc[2] = 0;
        sh.fetch[0] = sh.fetch[1] = sh.fetch[2] = 0;
        sh.win_lo = sh.win_hi = 0;
    }
    const Frontier fr{ring, a.queue + ((int64_t)blockIdx.x * NS + half) * a.qcap, a.qcap, a.status,
                      a.ring_size};
    Tally acc;
    __syncthreads();
    for (;;) {
        if (tid == 0) s_piece = (long long)atomicAdd(a.piece_counter, 1ull);
        __syncthreads();
        const int64_t pc = s_piece;
        if (pc >= a.npieces) break;
        int r = 0;
        {
            int hi = a.nranges - 1;
            while (r < hi) {
                const int mid = (r + hi + 1) >> 1;
                if (a.ranges[mid].piece_base <= pc) r = mid; else hi = mid - 1;
            }
        }
        const Range rg = a.ranges[r];
        const int64_t k = pc - rg.piece_base;
        const int pass = PAIRED ? half : (int)(k & 1);
        const int64_t c = PAIRED ? k : (k >> 1);
        int64_t j0, j1;
        piece_bounds(rg, c, j0, j1);
        const MatDesc md = a.mats[rg.mat];
        const PassGraph g = md.g[pass];
        int32_t s_lo = rg.offset + (int32_t)j0 * rg.stride;
        int32_t s_hi = rg.offset + (int32_t)j1 * rg.stride;   // exclusive (stride 1)
        if (!PAIRED && a.reuse && rg.stride == 1) {
            // cut pieces where adjacency chains start, so a piece's first
            // source rarely has a predecessor it could have reused
            if (tid < 32) {
                const int32_t lim = min(rg.chunk, 64);
                const int32_t lo = (j0 == 0) ? s_lo : chain_start(g, s_lo, lim);
                const int32_t hi = (j1 == rg.nj) ? s_hi : chain_start(g, s_hi, lim);
                if (tid == 0) { sh.seg[0] = lo; sh.seg[1] = hi; }
            }
            __syncthreads();
            s_lo = sh.seg[0];
            s_hi = sh.seg[1];
        }
        run_piece<BLOCK, PAIRED, false, GBM, LISTS>(a, md, g, pass, s_lo, s_hi, rg.stride, bm, summ, fr, sh, pair_flag,
                                        half, gtid, bar, acc);
        // the next piece starts from an empty bitmap
        {
            const int clo = sh.chain_lo, chi = sh.chain_hi;
            clear_range<GT>(bm, summ, clo, chi, gtid);
            __syncthreads();
            // the next piece may be another matrix: no seeding window yet
            if (gtid == 0) { sh.chain_lo = INT32_MAX; sh.chain_hi = -1; sh.hcount = 0; sh.win_lo = sh.win_hi = 0; }
            __syncthreads();
        }
    }
    {
        if (tid == 0) {   // this CTA's busy time, summed over CTAs (load balance)
            unsigned long long t_done;
            asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t_done));
            atomicAdd(&a.counters[15], t_done - t_start);
        }
        int64_t *wsum = shs[0].warp;
        const int64_t e = block_sum<BLOCK>((int64_t)acc.edges, wsum);
        const int64_t x = block_sum<BLOCK>((int64_t)acc.xcnt, wsum);
        const int64_t ei = block_sum<BLOCK>((int64_t)acc.einsp, wsum);
        if (tid == 0) {
            unsigned long long ns = 0, nr = 0, pv[8] = {0, 0, 0, 0, 0, 0, 0, 0};
            for (int h = 0; h < NS; h++) {
                ns += shs[h].nsrc;
                nr += shs[h].nreuse;
                for (int q = 0; q < 8; q++) pv[q] += shs[h].prof[q];
            }
            atomicAdd(&a.counters[0], (unsigned long long)e);
            atomicAdd(&a.counters[1], (unsigned long long)ns);
            atomicAdd(&a.counters[3], (unsigned long long)x);
            atomicAdd(&a.counters[4], (unsigned long long)ei);
            atomicAdd(&a.counters[5], (unsigned long long)pv[0]);
            atomicAdd(&a.counters[6], (unsigned long long)nr);
            for (int q = 1; q < 8; q++) atomicAdd(&a.counters[6 + q], (unsigned long long)pv[q]);
        }
    }
    grid.sync();
    if (blockIdx.x == 0 && tid == 0) {   // nanoseconds from launch to the end of the traversals
        unsigned long long t_now;
        asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t_now));
        a.counters[14] = t_now - t_start;
    }

    const int64_t L = a.L;
    const int64_t ntiles = a.ntiles;

    // line -> matrix lookup (matrices are stored in line order)
    auto mat_of = [&](int64_t l) -> int {
        int lo = 0, hi = a.nmats - 1;
        while (lo < hi) {
            int mid = (lo + hi + 1) >> 1;
            if (a.mats[mid].line_base <= l) lo = mid; else hi = mid - 1;
        }
        return lo;
    };
    // supernode run boundary before line l: lines l-1 and l join when each
    // is in the other's line and line l's upper count is one less
    auto sn_flag = [&](int64_t l) -> bool {
        const MatDesc &md = a.mats[mat_of(l)];
        const int64_t s = l - md.line_base;
        if (s == 0) return true;
        const bool linked = a.nxt[L + l - 1] && a.nxt[l - 1] && (a.cnt[l] == a.cnt[l - 1] - 1);
        return !linked;
    };

    // ---- phase 2: tile partial sums ------------------------------------------
    for (int64_t t = a.tile_lo + blockIdx.x; t < a.tile_hi; t += gridDim.x) {
        int64_t s0 = 0, s1 = 0, last = -1;
        for (int64_t l = t * TILE + tid; l < min(L, (t + 1) * TILE); l += BLOCK) {
            s0 += a.cnt[l];
            s1 += a.cnt[L + l];
            if (sn_flag(l)) last = max(last, l);
        }
        int64_t t0 = block_sum<BLOCK>(s0, shs[0].warp);
        int64_t t1 = block_sum<BLOCK>(s1, shs[0].warp);
        int64_t tl;
        block_excl_max<BLOCK>(last, &tl, shs[0].warp);
        if (tid == 0) {
            a.tile_sum[t] = t0;
            a.tile_sum[ntiles + t] = t1;
            a.tile_last[t] = tl;
        }
    }
    grid.sync();

    // ---- phase 3: block 0 scans the tile partials -----------------------------
    if (blockIdx.x == 0) {
        int64_t c0 = 0, c1 = 0, cm = -1;
        for (int64_t base = a.tile_lo; base < a.tile_hi; base += BLOCK) {
            const int64_t t = base + tid;
            const int64_t v0 = t < a.tile_hi ? a.tile_sum[t] : 0;
            const int64_t v1 = t < a.tile_hi ? a.tile_sum[ntiles + t] : 0;
            const int64_t vm = t < a.tile_hi ? a.tile_last[t] : -1;
            int64_t tot0, tot1, totm;
            const int64_t e0 = block_excl_scan<BLOCK>(v0, &tot0, shs[0].warp);
            const int64_t e1 = block_excl_scan<BLOCK>(v1, &tot1, shs[0].warp);
            const int64_t em = block_excl_max<BLOCK>(vm, &totm, shs[0].warp);
            if (t < a.tile_hi) {
                a.tile_sum[t] = c0 + e0;
                a.tile_sum[ntiles + t] = c1 + e1;
                a.tile_last[t] = max(cm, em);
            }
            c0 += tot0; c1 += tot1; cm = max(cm, totm);
        }
        if (tid == 0) {
            a.gptr[L] = c0;                  // pass 0 total
            a.gptr[(L + 1) + L] = c1;        // pass 1 total
        }
    }
    grid.sync();

    // ---- phase 4: CSR offsets and supernode starts per tile -------------------
    for (int64_t t = a.tile_lo + blockIdx.x; t < a.tile_hi; t += gridDim.x) {
        int64_t c0 = a.tile_sum[t], c1 = a.tile_sum[ntiles + t], carry = a.tile_last[t];
        int64_t nsn = 0;
        for (int64_t base = t * TILE; base < min(L, (t + 1) * TILE); base += BLOCK) {
            const int64_t l = base + tid;
            const bool in = l < min(L, (t + 1) * TILE);
            int64_t v0 = in ? a.cnt[l] : 0;
            int64_t v1 = in ? a.cnt[L + l] : 0;
            bool f = in && sn_flag(l);
            int64_t tot0, tot1;
            int64_t e0 = block_excl_scan<BLOCK>(v0, &tot0, shs[0].warp);
            int64_t e1 = block_excl_scan<BLOCK>(v1, &tot1, shs[0].warp);
            int64_t sub_last;
            int64_t rs = block_excl_max<BLOCK>(f ? l : -1, &sub_last, shs[0].warp);
            rs = max(max(rs, f ? l : (int64_t)-1), carry);
            bool start = false;
            if (in) {
                a.gptr[l] = c0 + e0;
                a.gptr[(L + 1) + l] = c1 + e1;
                start = f || (a.max_sn > 0 && ((l - rs) % a.max_sn) == 0);
                a.snind[l] = start ? 1 : 0;
            }
            const int64_t ns = block_sum<BLOCK>(start ? 1 : 0, shs[0].warp);
            carry = max(carry, sub_last);   // run start carried to the next sub-tile
            c0 += tot0; c1 += tot1; nsn += ns;
        }
        if (tid == 0) a.tile_sn[t] = nsn;
    }
    grid.sync();

    // ---- phase 5: block 0 scans the supernode tile counts ---------------------
    if (blockIdx.x == 0) {
        int64_t c = 0;
        for (int64_t base = a.tile_lo; base < a.tile_hi; base += BLOCK) {
            const int64_t t = base + tid;
            int64_t v = t < a.tile_hi ? a.tile_sn[t] : 0;
            int64_t tot;
            int64_t e = block_excl_scan<BLOCK>(v, &tot, shs[0].warp);
            if (t < a.tile_hi) a.tile_sn[t] = c + e;
            c += tot;
        }
        if (tid == 0) a.counters[2] = (unsigned long long)c;
    }
    grid.sync();

    // ---- phase 6: supernode list, pattern compaction ---------------------------
    for (int64_t t = a.tile_lo + blockIdx.x; t < a.tile_hi; t += gridDim.x) {
        int64_t c = a.tile_sn[t];
        for (int64_t base = t * TILE; base < min(L, (t + 1) * TILE); base += BLOCK) {
            const int64_t l = base + tid;
            const bool in = l < min(L, (t + 1) * TILE);
            int64_t v = (in && a.snind[l]) ? 1 : 0;
            int64_t tot;
            int64_t e = block_excl_scan<BLOCK>(v, &tot, shs[0].warp);
            if (v) a.sn_list[c + e] = (int32_t)l;
            if (in && a.mat_info) {
                const int mi = mat_of(l);
                if (a.mats[mi].line_base == l) {
                    a.mat_info[3 * mi + 0] = a.gptr[l];
                    a.mat_info[3 * mi + 1] = a.gptr[(L + 1) + l];
                    a.mat_info[3 * mi + 2] = c + e;
                }
            }
            c += tot;
        }
    }
    // CSR form only (want_pattern == 1); the ranges form (2) leaves the
    // lists where the chains wrote them, at poff
    if (a.want_pattern == 1 && (*a.status & ERR_POOL_OVERFLOW) == 0) {
        const int warps = (gridDim.x * BLOCK) >> 5;
        const int gw = (blockIdx.x * BLOCK + tid) >> 5;
        const int lane = tid & 31;
        const int64_t tot0 = a.gptr[L];
        for (int64_t pl = gw; pl < 2 * L; pl += warps) {
            const int pass = pl >= L;
            const int64_t l = pass ? pl - L : pl;
            const int32_t c = a.cnt[pl];
            if (c == 0) continue;
            const int64_t src = a.poff[pl];
            const int64_t dst = (pass ? tot0 : 0) + a.gptr[pass * (L + 1) + l];
            // four loads in flight per lane before their stores
            const int32_t *from = a.pool + src;
            int32_t *to = a.out + dst;
            for (int32_t k0 = 0; k0 < c; k0 += 128) {
                int32_t v[4];
#pragma unroll
                for (int u = 0; u < 4; u++) {
                    const int32_t k = k0 + 32 * u + lane;
                    v[u] = k < c ? __ldcs(from + k) : 0;
                }
#pragma unroll
                for (int u = 0; u < 4; u++) {
                    const int32_t k = k0 + 32 * u + lane;
                    if (k < c) __stcs(to + k, v[u]);
                }
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Upload kernels: validation, diagonal removal, distinct-entry counts, G^T.

struct UploadArgs {
    int32_t n;
    int64_t nnz;
    const int32_t *beg, *end, *adj;  // staged input
    int32_t *deg;                    // [n]   distinct off-diagonal entries per line
    int32_t *indeg;                  // [n+1] entries per transposed line
    int32_t *orig_up;                // [n]   distinct entries > v in line v
    int32_t *orig_lo;                // [n]   distinct lines u > j holding j
    int32_t *rawdeg;                 // [n]   end[v] - beg[v]
    unsigned long long *counts;      // [0] distinct upper, [1] distinct lower
    uint32_t *status;                // bit 0: invalid input
};

// True when adj[k] is the first occurrence of its value in line [b, k].
__device__ __forceinline__ bool first_in_line(const int32_t *adj, int32_t b, int32_t k,
                                              bool sorted)
{
    const int32_t m = adj[k];
    if (sorted) return (k == b) || (adj[k - 1] != m);
    for (int32_t j = b; j < k; j++)
        if (adj[j] == m) return false;
    return true;
}

// One warp per line.  Checks the range and the ids, counts kept entries and
// transposed entries, and the distinct off-diagonal entries above/below.
__global__ void upload_count_kernel(UploadArgs u)
{
    const int lane = threadIdx.x & 31;
    const int64_t gw = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    unsigned long long up = 0, lo = 0;
    for (int64_t v = gw; v < u.n; v += nw) {
        const int32_t b = u.beg[v], e = u.end[v];
        if (b < 0 || e < b || (int64_t)e > u.nnz) {
            if (lane == 0) {
                atomicOr(u.status, 1u);
                u.deg[v] = 0; u.orig_up[v] = 0; u.rawdeg[v] = 0;
            }
            continue;
        }
        if (lane == 0) u.rawdeg[v] = e - b;
        // sorted lists allow a linear duplicate test
        bool sorted = true;
        for (int32_t k = b + lane; k + 1 < e; k += 32)
            if (u.adj[k] > u.adj[k + 1]) sorted = false;
        sorted = __all_sync(0xffffffffu, sorted);
        int kept = 0, kup = 0;
        for (int32_t k = b + lane; k < e; k += 32) {
            const int32_t m = u.adj[k];
            if (m < 0 || m >= u.n) { atomicOr(u.status, 1u); continue; }
            if (m == (int32_t)v) continue;
            if (!first_in_line(u.adj, b, k, sorted)) continue;
            kept++;
            atomicAdd(&u.indeg[m], 1);
            if (m > v) { up++; kup++; }
            else { lo++; atomicAdd(&u.orig_lo[m], 1); }
        }
        for (int o = 16; o; o >>= 1) {
            kept += __shfl_xor_sync(0xffffffffu, kept, o);
            kup += __shfl_xor_sync(0xffffffffu, kup, o);
        }
        if (lane == 0) { u.deg[v] = kept; u.orig_up[v] = kup; }
    }
    for (int o = 16; o; o >>= 1) {
        up += __shfl_xor_sync(0xffffffffu, up, o);
        lo += __shfl_xor_sync(0xffffffffu, lo, o);
    }
    if (lane == 0) {
        if (up) atomicAdd(&u.counts[0], up);
        if (lo) atomicAdd(&u.counts[1], lo);
    }
}

// One warp per line: copies the kept entries (order preserved) into G and
// scatters them into G^T through per-line cursors.
__global__ void upload_fill_kernel(UploadArgs u, const int32_t *gptr, int32_t *gadj,
                                   int32_t *tcursor, int32_t *tadj)
{
    const int lane = threadIdx.x & 31;
    const int64_t gw = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t v = gw; v < u.n; v += nw) {
        const int32_t b = u.beg[v], e = u.end[v];
        if (b < 0 || e < b || (int64_t)e > u.nnz) continue;
        bool sorted = true;
        for (int32_t k = b + lane; k + 1 < e; k += 32)
            if (u.adj[k] > u.adj[k + 1]) sorted = false;
        sorted = __all_sync(0xffffffffu, sorted);
        int32_t out = gptr[v];
        for (int32_t k0 = b; k0 < e; k0 += 32) {
            const int32_t k = k0 + lane;
            int32_t m = -1;
            bool keep = false;
            if (k < e) {
                m = u.adj[k];
                keep = (m >= 0 && m < u.n && m != (int32_t)v) &&
                       first_in_line(u.adj, b, k, sorted);
            }
            const unsigned bal = __ballot_sync(0xffffffffu, keep);
            if (keep) {
                gadj[out + __popc(bal & ((1u << lane) - 1u))] = m;
                const int32_t p = atomicAdd(&tcursor[m], 1);
                tadj[p] = (int32_t)v;
            }
            out += __popc(bal);
        }
    }
}

// Fills the 32-byte slot of every vertex of one pass graph: {degree, row
// offset, the first SLOT_NB ids (-1 past the degree)}.
__global__ void slot_fill_kernel(int32_t n, const int32_t *ptr, const int32_t *adj, int4 *slot)
{
    for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
        const int32_t b = ptr[v], d = ptr[v + 1] - b;
        int32_t x[SLOT_NB];
#pragma unroll
        for (int u = 0; u < SLOT_NB; u++) x[u] = u < d ? adj[b + u] : -1;
        slot[2 * v] = make_int4(d, b, x[0], x[1]);
        slot[2 * v + 1] = make_int4(x[2], x[3], x[4], x[5]);
    }
}

// Exclusive scan of int32 counts into int32 offsets: three kernels.
template <int BLOCK>
__global__ void scan_tiles_kernel(const int32_t *in, int64_t n, int64_t *tile_sums)
{
    __shared__ int64_t warp[32];
    const int64_t t = blockIdx.x;
    const int64_t i = t * BLOCK + threadIdx.x;
    int64_t v = i < n ? in[i] : 0;
    int64_t s = block_sum<BLOCK>(v, warp);
    if (threadIdx.x == 0) tile_sums[t] = s;
}

template <int BLOCK>
__global__ void scan_partials_kernel(int64_t *tile_sums, int64_t ntiles, int64_t *total)
{
    __shared__ int64_t warp[32];
    int64_t c = 0;
    for (int64_t base = 0; base < ntiles; base += BLOCK) {
        const int64_t t = base + threadIdx.x;
        int64_t v = t < ntiles ? tile_sums[t] : 0;
        int64_t tot;
        int64_t e = block_excl_scan<BLOCK>(v, &tot, warp);
        if (t < ntiles) tile_sums[t] = c + e;
        c += tot;
    }
    if (threadIdx.x == 0) *total = c;
}

template <int BLOCK>
__global__ void scan_apply_kernel(const int32_t *in, int64_t n, const int64_t *tile_sums,
                                  int32_t *out, const int64_t *total)
{
    __shared__ int64_t warp[32];
    const int64_t t = blockIdx.x;
    const int64_t i = t * BLOCK + threadIdx.x;
    int64_t v = i < n ? in[i] : 0;
    int64_t tot;
    int64_t e = block_excl_scan<BLOCK>(v, &tot, warp);
    if (i < n) out[i] = (int32_t)(tile_sums[t] + e);
    if (i == 0) out[n] = (int32_t)*total;
}

}  // namespace dev
}  // namespace gsofa

// gsofa_api.cu -- host side of the B200 symbolic factorization (C ABI).
//
// Replaces the reference's host orchestration symbfact_min_id
// (without_space_optimization/symbfact.cuh:991-1391,
//  with_space_optimization/symbfact.cuh:1553-2583): file reading, device
// selection, scratch sizing, the launch and the result report.  Unlike the
// reference, nothing here exits the process; every failure is a status code.
#include "../../include/gsofa.h"
#include "gsofa_device.cuh"
#include "gsofa_server.cuh"
#include "gsofa_supernodal.cuh"
#include "gsofa_partition.hpp"
#include "gsofa_order.cuh"

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <functional>
#include <thread>
#include <map>
#include <unordered_map>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <new>
#include <stdexcept>
#include <string>
#include <vector>

using namespace gsofa::dev;

namespace {

// ---------------------------------------------------------------------------
// Small helpers

struct CudaFail {
    cudaError_t e;
};

#define GS_CUDA(x)                                                     \
    do {                                                               \
        cudaError_t _e = (x);                                          \
        if (_e != cudaSuccess) throw CudaFail{_e};                     \
    } while (0)

thread_local char g_last_error[256];

gsofa_status fail_cuda(cudaError_t e)
{
    std::snprintf(g_last_error, sizeof(g_last_error), "%s", cudaGetErrorString(e));
    cudaGetLastError();
    return (e == cudaErrorMemoryAllocation) ? GSOFA_ERR_OOM : GSOFA_ERR_CUDA;
}

// cudaFuncSetAttribute(MaxDynamicSharedMemorySize) belongs to the kernel and
// is shared by every caller in the process: each launch sets it and launches
// under this lock, so another host thread cannot resize it in between.
std::mutex &kernel_attr_mutex()
{
    static std::mutex m;
    return m;
}

// Grow-only device buffer owned by a context.
struct DevBuf {
    void *p = nullptr;
    size_t bytes = 0;
};

}  // namespace

// A captured factorization job and what it was captured from.
struct GraphCache {
    cudaGraphExec_t exec = nullptr;
    std::vector<char> key;
    std::vector<MatDesc> md;     // host sources of the captured copies
    std::vector<Range> ranges;
    JobArgs args{};
    cudaStream_t stream = nullptr;
};

struct gsofa_ctx {
    int device = 0;
    int sm_count = 0;
    size_t smem_optin = 0;
    size_t budget = 0;
    size_t held = 0;          // bytes of grow-only scratch currently held
    cudaStream_t stream = nullptr;      // stream all work is issued on
    cudaStream_t own_stream = nullptr;  // the context's own stream
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    // job scratch
    DevBuf queue, cnt, nxt, poff, gptr, lrow, snind, snlist, tiles, misc, pool, out, mats, ranges, stamp;
    DevBuf gstate;            // visited bitmaps of the global-state kernels
    DevBuf blk;               // streaming: written entries per pool block
    DevBuf order;             // gsofa_order_rcm: symmetric structure, levels, sort space
    unsigned int *h_blk = nullptr;   // page-locked mirror of blk
    size_t h_blk_cap = 0;
    cudaStream_t s_poll = nullptr, s_copy = nullptr;   // streaming: counter reads, block copies
    DevBuf sn_head, sn_data;  // gsofa_result_supernodal: sizes and offsets; index lists
    std::vector<int64_t> sn_xl, sn_xu;   // supernodal offsets of the result sizes were taken for
    const void *sn_for = nullptr;        // ... that result (its internal record)
    uint64_t sn_job = 0;                 // ... and its job
    // upload staging
    DevBuf st_beg, st_end, st_adj, st_tmp;
    std::vector<gsofa_matrix *> matrices;
    uint64_t job_id = 0;      // incremented by every factorization
    DevBuf matinfo;
    GraphCache graph;         // last captured job (GSOFA_FLAG_GRAPH)
    // launch shapes already sized: (block, bitmap words) -> (ring, CTAs/SM)
    struct Shape { int block; int32_t words; bool paired; bool gbm; bool wide; bool lists; int ring; int occ; };
    std::vector<Shape> shapes;

    void *grow(DevBuf &b, size_t bytes)
    {
        bytes = std::max<size_t>(bytes, 256);
        if (b.bytes >= bytes) return b.p;
        if (b.p) {
            GS_CUDA(cudaFree(b.p));
            held -= b.bytes;
            b.p = nullptr;
            b.bytes = 0;
        }
        if (held + bytes > budget) throw CudaFail{cudaErrorMemoryAllocation};
        GS_CUDA(cudaMalloc(&b.p, bytes));
        b.bytes = bytes;
        held += bytes;
        return b.p;
    }
    void release(DevBuf &b)
    {
        if (b.p) {
            cudaFree(b.p);
            held -= b.bytes;
        }
        b.p = nullptr;
        b.bytes = 0;
    }

    // Device slabs of freed matrices, kept for later uploads so that a caller
    // who uploads, factorizes and frees matrix after matrix pays no
    // cudaMalloc / cudaFree (each of which synchronises the device) once the
    // cache is warm.  At most kSlabs slabs and budget / 8 bytes are kept.
    static constexpr size_t kSlabs = 8;
    std::vector<DevBuf> slabs;
    size_t slab_bytes = 0;
    void *slab_take(size_t bytes, size_t *got)
    {
        int best = -1;
        for (size_t i = 0; i < slabs.size(); i++)
            if (slabs[i].bytes >= bytes && slabs[i].bytes <= 2 * bytes &&
                (best < 0 || slabs[i].bytes < slabs[(size_t)best].bytes))
                best = (int)i;
        if (best >= 0) {
            DevBuf b = slabs[(size_t)best];
            slabs.erase(slabs.begin() + best);
            slab_bytes -= b.bytes;
            *got = b.bytes;
            return b.p;
        }
        void *p = nullptr;
        GS_CUDA(cudaMalloc(&p, bytes));
        *got = bytes;
        return p;
    }
    void slab_give(void *p, size_t bytes)
    {
        if (!p) return;
        if (slabs.size() < kSlabs && slab_bytes + bytes <= budget / 8) {
            slabs.push_back(DevBuf{p, bytes});
            slab_bytes += bytes;
        } else {
            cudaFree(p);
        }
    }
};

struct gsofa_matrix {
    gsofa_ctx *ctx = nullptr;
    int32_t n = 0;
    int64_t nnz_in = 0;
    int64_t nnz_g = 0;            // distinct off-diagonal entries kept
    int32_t *d_gptr = nullptr, *d_gadj = nullptr;
    int32_t *d_tptr = nullptr, *d_tadj = nullptr;
    int32_t *d_orig_up = nullptr, *d_orig_lo = nullptr, *d_rawdeg = nullptr;
    int4 *d_gslot = nullptr, *d_tslot = nullptr;   // 32-byte row slots of G and G^T
    void *slab = nullptr;          // one device allocation holding all of the above
    size_t slab_bytes = 0;
    uint64_t orig_up = 0, orig_lo = 0;
    int64_t last_pattern_total = -1;  // pool size the last run needed
};

namespace {

// Where a result's arrays sit in the context's device buffers (for
// gsofa_result_fetch); valid while ctx->job_id == job_id.
struct ResultInternal {
    uint64_t job_id;
    int64_t L, line_base, n;
    int64_t u0, l0;         // first index of the U rows / L columns in `out`
    int64_t sn0;            // first supernode of this matrix in the device list
    int pattern;            // the job's pattern form: 0 none, 1 CSR in `out`,
                            // 2 ranges in the caller's pool (begins in poff)
    const int32_t *pool;    // ranges form: the pool's device address
};

// The caller's pattern pool of the ranges form (gsofa_symbfact_ranges):
// a device address (device memory, or the device alias of page-locked host
// memory) and its capacity in entries.
struct ExtPool {
    int32_t *dev = nullptr;
    int64_t cap = 0;
    // streaming to host: per-block written-entry counters the kernel keeps,
    // and the host loop that copies full blocks out while the kernel runs
    unsigned int *blk_done = nullptr;
    int32_t blk_shift = 0;
    int64_t nblk = 0;
    std::function<void()> while_running;
};

int pick_block(int32_t max_n)
{
    if (max_n <= 8192) return 256;
    return 512;
}

template <int BLOCK, bool PAIRED, bool GBM, int MINB = (BLOCK >= 1024 ? 1 : 1024 / BLOCK), bool LISTS = true>
void *factor_fn()
{
    return (void *)factor_kernel<BLOCK, PAIRED, GBM, MINB, LISTS>;
}

// The factorization kernel for a launch shape: threads per CTA, the two
// passes side by side (paired), the visited bitmaps in global memory (gbm),
// registers budgeted for one CTA per SM (wide: the 512-thread paired form).
// lists: the job writes the pattern.  Counts-only jobs of the shapes that
// large matrices take run an instantiation without the list output (fewer
// registers: no spills where the list output's code would cause them).
void *factor_kernel_for(int block, bool paired, bool gbm = false, bool wide = false, bool lists = true)
{
    if (!lists && paired) {
        if (gbm && block == 256) return factor_fn<256, true, true, 4, false>();
        if (wide && block == 512) return factor_fn<512, true, false, 1, false>();
        if (!gbm && !wide && block == 768) return factor_fn<768, true, false, 1, false>();
        if (!gbm && !wide && block == 1024) return factor_fn<1024, true, false, 1, false>();
    }
    if (gbm) {
        switch (block) {
        case 128: return paired ? factor_fn<128, true, true>() : factor_fn<128, false, true>();
        case 256: return paired ? factor_fn<256, true, true>() : factor_fn<256, false, true>();
        case 512: return paired ? factor_fn<512, true, true>() : factor_fn<512, false, true>();
        default: return nullptr;
        }
    }
    if (wide) return (block == 512 && paired) ? factor_fn<512, true, false, 1>() : nullptr;
    switch (block) {
    case 128: return paired ? nullptr : factor_fn<128, false, false>();
    case 256: return paired ? factor_fn<256, true, false>() : factor_fn<256, false, false>();
    case 512: return paired ? factor_fn<512, true, false>() : factor_fn<512, false, false>();
    case 768: return paired ? factor_fn<768, true, false>() : factor_fn<768, false, false>();
    case 1024: return paired ? factor_fn<1024, true, false>() : factor_fn<1024, false, false>();
    default: return nullptr;
    }
}

void resolve_params(const gsofa_params *in, gsofa_params *p)
{
    gsofa_default_params(p);
    if (in) *p = *in;
}

// Copies a device array [off, off+count) of T into a fresh malloc'd host array.
template <class T>
T *download(cudaStream_t st, const T *d, int64_t off, int64_t count)
{
    T *h = (T *)std::malloc((size_t)std::max<int64_t>(count, 1) * sizeof(T));
    if (!h) throw std::bad_alloc();
    if (count > 0)
        GS_CUDA(cudaMemcpyAsync(h, d + off, (size_t)count * sizeof(T), cudaMemcpyDeviceToHost, st));
    return h;
}

void free_result_arrays(gsofa_result *r)
{
    std::free(r->u_row_count);
    std::free(r->l_col_count);
    std::free(r->l_row_count);
    std::free(r->sn_start);
    std::free(r->line_flags);
    r->line_flags = nullptr;
    std::free(r->u_ptr);
    std::free(r->u_idx);
    std::free(r->l_ptr);
    std::free(r->l_idx);
    std::free(r->u_beg);
    std::free(r->l_beg);
    r->u_beg = r->l_beg = nullptr;
    r->u_row_count = r->l_col_count = r->l_row_count = r->sn_start = nullptr;
    r->u_ptr = r->l_ptr = nullptr;
    r->u_idx = r->l_idx = nullptr;
}

// The factorization of `count` matrices in one cooperative launch.
double now_ms()
{
    using namespace std::chrono;
    return duration<double, std::milli>(steady_clock::now().time_since_epoch()).count();
}

gsofa_status run_job(gsofa_ctx *ctx, int count, const gsofa_matrix *const *mats,
                     const gsofa_params *pin, gsofa_result *out, const ExtPool *ext = nullptr)
{
    static const bool host_timing = std::getenv("GSOFA_HOST_TIMING") != nullptr;
    const double t_enter = now_ms();
    gsofa_params p;
    resolve_params(pin, &p);
    if (count <= 0 || !mats || !out) return GSOFA_ERR_INVALID_INPUT;
    for (int i = 0; i < count; i++) {
        if (!mats[i] || mats[i]->ctx != ctx) return GSOFA_ERR_INVALID_INPUT;
        std::memset(&out[i], 0, sizeof(gsofa_result));
        out[i].n = mats[i]->n;
    }
    const int part_count = p.part_count > 1 ? p.part_count : 1;
    const int part_index = p.part_count > 1 ? p.part_index : 0;
    if (part_index < 0 || part_index >= part_count) return GSOFA_ERR_INVALID_INPUT;
    // a contiguous range of source lines [line_lo, line_hi) of one matrix
    const bool line_range = p.line_lo != 0 || p.line_hi != 0;
    if (line_range && (count != 1 || part_count > 1 || p.line_lo < 0 || p.line_hi < p.line_lo))
        return GSOFA_ERR_INVALID_INPUT;
    const int32_t range_lo = line_range ? std::min(p.line_lo, mats[0]->n) : 0;
    const int32_t range_hi = line_range ? std::min(p.line_hi, mats[0]->n) : 0;
    const bool subset = part_count > 1 || line_range;   // some lines are not processed
    // pattern form: 1 CSR (lists compacted into line order), 2 ranges (lists
    // left where their chains wrote them, in the caller's pool)
    if (p.want_pattern == 2 && !ext) return GSOFA_ERR_INVALID_INPUT;
    if (ext && (p.want_pattern != 2 || part_count != 1)) return GSOFA_ERR_INVALID_INPUT;
    const int pattern_form = (p.want_pattern != 0 && part_count == 1) ? (ext ? 2 : 1) : 0;
    const bool want_pattern = pattern_form != 0;
    const bool restrict_tiles = line_range && pattern_form != 1;
    // reuse: -1 (auto) or 1 = paired passes with exact reuse when two bitmaps
    // fit in shared memory, else adjacency chains; 2 = adjacency chains;
    // 0 = every source from scratch.  Interleaved partitions have no
    // consecutive sources, so they run without reuse; line ranges keep it.
    const int reuse = (p.reuse != 0 && part_count == 1) ? 1 : 0;
    // distinct original entries of the processed lines (their fill count
    // subtracts them)
    auto processed_orig = [&](int i) -> uint64_t {
        const int64_t n = mats[i]->n;
        std::vector<int32_t> ou((size_t)n), ol((size_t)n);
        GS_CUDA(cudaMemcpy(ou.data(), mats[i]->d_orig_up, n * 4, cudaMemcpyDeviceToHost));
        GS_CUDA(cudaMemcpy(ol.data(), mats[i]->d_orig_lo, n * 4, cudaMemcpyDeviceToHost));
        uint64_t o = 0;
        if (line_range) {
            for (int64_t q = range_lo; q < range_hi; q++) o += (uint64_t)ou[q] + (uint64_t)ol[q];
        } else {
            for (int64_t q = part_index; q < n; q += part_count) o += (uint64_t)ou[q] + (uint64_t)ol[q];
        }
        return o;
    };

    // line space and per-matrix descriptors
    std::vector<MatDesc> md(count);
    int64_t L = 0;
    int32_t max_n = 1;
    for (int i = 0; i < count; i++) {
        md[i].n = mats[i]->n;
        md[i].pad = 0;
        md[i].line_base = L;
        md[i].g[0] = PassGraph{mats[i]->d_gptr, mats[i]->d_gadj, mats[i]->d_gslot};
        md[i].g[1] = PassGraph{mats[i]->d_tptr, mats[i]->d_tadj, mats[i]->d_tslot};
        md[i].rawdeg = mats[i]->d_rawdeg;
        L += mats[i]->n;
        max_n = std::max(max_n, mats[i]->n);
    }
    if (L == 0) return GSOFA_OK;

    // parameters
    // bitmap words rounded to 128 so its summary (one bit per word) is a
    // whole number of 16-byte groups
    const int32_t words_needed = ((max_n + 31) / 32 + 127) / 128 * 128;
    const int32_t state_needed = words_needed + words_needed / 32 + ((words_needed / 32 + 31) / 32 + 3) / 4 * 4;
    // Where the visited bitmaps live: shared memory holds two of them (the
    // paired kernel) up to ~850K lines and one up to ~1.7M; global memory
    // holds any number of any size.  GSOFA_FLAG_GLOBAL_STATE /
    // GSOFA_FLAG_SHARED_STATE choose; else shared memory while the pair fits.
    const size_t pair_smem = (size_t)2 * state_needed * 4 + 2 * 1024 * 4 + sizeof(SharedState) * 2 + 1024;
    if ((p.flags & GSOFA_FLAG_GLOBAL_STATE) && (p.flags & GSOFA_FLAG_SHARED_STATE)) return GSOFA_ERR_INVALID_INPUT;
    const size_t single_smem = (size_t)state_needed * 4 + 1024 * 4 + sizeof(SharedState) + 1024;
    const bool want_pair = reuse && p.reuse != 2;
    const bool gbm = (p.flags & GSOFA_FLAG_GLOBAL_STATE) ||
                     (!(p.flags & GSOFA_FLAG_SHARED_STATE) &&
                      ((want_pair && pair_smem > ctx->smem_optin) || single_smem > ctx->smem_optin));
    const bool paired = want_pair && (gbm || pair_smem <= ctx->smem_optin);
    // Shared-state pairs past 8K lines hold one CTA per SM (1024 threads at
    // 64 registers fill its register file): 768 threads with up to 80
    // registers a thread run without register spills, measured faster than
    // 1024 threads on the 80^3 stencil with and without the pattern.  Counts
    // of matrices with long rows (no row slots: mean degree above SLOT_NB)
    // take 1024 threads: their large frontiers keep every warp busy (9%
    // faster on the 659K-line power-law matrix).  512 threads with up to 128
    // registers -- GSOFA_FLAG_WIDE_REGS -- are faster still on latency-bound
    // matrices, counts only, but slower where large frontiers keep many warps
    // busy.
    const bool wide = (p.flags & GSOFA_FLAG_WIDE_REGS) != 0;
    bool long_rows = false;
    for (int i = 0; i < count; i++) long_rows |= mats[i]->n > 0 && mats[i]->d_gslot == nullptr;
    int block = p.block_size;
    if (wide) block = 512;
    if (!block) {
        if (gbm) block = paired ? 256 : 128;
        else if (paired && max_n > 8192) block = (!want_pattern && long_rows) ? 1024 : 768;
        else block = pick_block(max_n) * (paired ? 2 : 1);
    }
    if (wide && (!paired || gbm)) return GSOFA_ERR_INVALID_INPUT;
    void *kfn = factor_kernel_for(block, paired, gbm, wide, want_pattern != 0);
    if (!kfn) return GSOFA_ERR_INVALID_INPUT;
    const int NS = paired ? 2 : 1;
    int lanes = p.threads_per_source ? p.threads_per_source : 1;
    if (lanes != 1 && lanes != 4 && lanes != 8 && lanes != 16 && lanes != 32)
        return GSOFA_ERR_INVALID_INPUT;

    const int32_t bitmap_words = words_needed;
    const int32_t state_words = state_needed;
    const size_t static_smem = sizeof(SharedState) * NS + 1024;
    // shared memory per traversal: its bitmap and summaries (unless in global
    // memory) and its frontier ring
    const size_t smem_state = gbm ? 0 : (size_t)state_words * 4;
    if ((size_t)NS * (smem_state + 1024 * 4) + static_smem > ctx->smem_optin) return GSOFA_ERR_UNSUPPORTED;
    // frontier ring: the largest of 8K/4K/2K/1K entries that keeps the most
    // CTAs (each with its own bitmap) resident on an SM; sized once per shape
    int ring = 0, occ = 0;
    size_t smem = 0;
    bool cached = false;
    for (const auto &sh : ctx->shapes)
        if (sh.block == block && sh.words == bitmap_words && sh.paired == paired && sh.gbm == gbm && sh.wide == wide &&
            sh.lists == (want_pattern != 0)) {
            ring = sh.ring; occ = sh.occ; cached = true;
        }
    if (cached) {
        smem = (size_t)NS * (smem_state + (size_t)ring * 4);
    } else {
        std::lock_guard<std::mutex> lk(kernel_attr_mutex());
        for (int cand = 8192; cand >= 1024; cand >>= 1) {
            const size_t sm = (size_t)NS * (smem_state + (size_t)cand * 4);
            if (sm + static_smem > ctx->smem_optin) continue;
            GS_CUDA(cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
            int o = 0;
            GS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, kfn, block, sm));
            if (o > occ) { occ = o; ring = cand; smem = sm; }
        }
        if (occ <= 0) return GSOFA_ERR_UNSUPPORTED;
        ctx->shapes.push_back({block, bitmap_words, paired, gbm, wide, want_pattern != 0, ring, occ});
    }
    int per_sm = p.ctas_per_sm > 0 ? std::min(p.ctas_per_sm, occ) : occ;
    int grid = per_sm * ctx->sm_count;
    {
        // Concurrent traversals within the memory budget (the reference
        // shrinks its sources per pass until the state fits its pool,
        // with_space_optimization/symbfact.cuh:1465-1507): every traversal
        // holds a frontier queue of n entries and, with the pattern, a row of
        // n chain stamps; the per-line arrays and a minimal pool come first.
        const int64_t q = std::max<int64_t>(p.queue_capacity, max_n);
        const int64_t per_cta = (int64_t)NS * (q * 4 + (want_pattern ? (int64_t)words_needed * 32 * 2 : 0) +
                                               (gbm ? (int64_t)state_words * 4 : 0));
        // cnt, nxt, poff, gptr, lrow, snind, sn_list
        const int64_t per_line = 2 * 4 + 2 + 2 * 8 + 2 * 8 + 4 + 1 + 4;
        const int64_t fixed = L * per_line + ((L + TILE - 1) / TILE) * 32 + 64 * 1024 +
                              (want_pattern ? (int64_t)2 * 4 * (1 << 20) : 0);
        const int64_t others = (int64_t)ctx->held - (int64_t)ctx->queue.bytes - (int64_t)ctx->stamp.bytes -
                               (int64_t)ctx->gstate.bytes;
        const int64_t room = (int64_t)ctx->budget - others - fixed;
        if (room < per_cta) return GSOFA_ERR_OOM;
        grid = (int)std::min<int64_t>(grid, room / per_cta);
    }
    // sources per work piece: a piece's first source cannot reuse state, so
    // pieces are long (up to 512 sources) while there are still about eight
    // per concurrent traversal -- the last pieces handed out are the light,
    // low-numbered sources, so the launch's tail stays short
    int chunk = p.src_chunk;
    if (chunk <= 0) {
        // a line range keeps the pieces the whole matrix would have (smaller
        // ones start more traversals afresh, and a fresh start costs most in
        // the separator lines a range of the last lines holds) while every
        // CTA still gets about four pieces; shorter ranges take the length
        // that gives every CTA four, or eight, pieces
        const int64_t mult = paired ? 1 : 2;
        const int64_t lines = line_range ? (int64_t)(range_hi - range_lo) : L;
        const int64_t per = std::max(mult * lines / ((int64_t)8 * grid),
                                     std::min(mult * L / ((int64_t)8 * grid), mult * lines / ((int64_t)4 * grid)));
        chunk = reuse ? (int)std::min<int64_t>(512, std::max<int64_t>(32, per)) : 1;
    }

    // work ranges: biggest matrices first
    std::vector<int> order(count);
    for (int i = 0; i < count; i++) order[i] = i;
    std::stable_sort(order.begin(), order.end(),
                     [&](int x, int y) { return mats[x]->n > mats[y]->n; });
    std::vector<Range> ranges;
    int64_t npieces = 0;
    for (int i : order) {
        const int32_t n = mats[i]->n;
        if (n <= part_index) continue;
        Range r{};
        r.mat = i;
        r.chunk = chunk;
        r.stride = part_count;
        r.offset = part_index;
        r.nj = (n - part_index + part_count - 1) / part_count;
        if (line_range) {
            r.offset = range_lo;
            r.nj = range_hi - range_lo;
            if (r.nj <= 0) continue;
        }
        r.piece_base = npieces;
        // the bottom eighth in quarter-length pieces (the last handed out)
        r.tail = (reuse && chunk >= 64) ? r.nj / 8 : 0;
        r.small = r.tail ? std::max(32, chunk / 4) : chunk;
        r.npieces = (paired ? 1 : 2) * pieces_per_pass(r);
        npieces += r.npieces;
        ranges.push_back(r);
    }

    const int64_t qcap = std::max<int64_t>(p.queue_capacity, max_n);
    const int64_t ntiles = (L + TILE - 1) / TILE;

    // pool sizing: the last run's exact need (every chain takes an exact
    // range, so the pool holds the lists with no gaps), else a share of the
    // budget; the ranges form writes into the caller's pool
    auto pool_need = [&](int64_t entries) { return std::max<int64_t>(entries, 1); };
    int64_t pool_cap = 0;
    if (pattern_form == 2) {
        pool_cap = ext->cap;
    } else if (want_pattern) {
        if (p.pool_capacity > 0) {
            pool_cap = p.pool_capacity;
        } else {
            int64_t known = 0;
            bool all_known = true;
            for (int i = 0; i < count; i++) {
                if (mats[i]->last_pattern_total < 0) all_known = false;
                else known += mats[i]->last_pattern_total;
            }
            if (all_known) {
                pool_cap = pool_need(known);
            } else {
                size_t freeb = ctx->budget > ctx->held ? ctx->budget - ctx->held : 0;
                pool_cap = std::max<int64_t>((int64_t)(freeb / 4 / (2 * sizeof(int32_t))), 1 << 20);
                pool_cap = std::min<int64_t>(pool_cap, (int64_t)1 << 31);
            }
        }
    }

    ctx->job_id++;
    for (int attempt = 0; attempt < 2; attempt++) {
        // scratch
        int32_t *d_queue = (int32_t *)ctx->grow(ctx->queue, (size_t)grid * NS * qcap * sizeof(int32_t));
        int32_t *d_cnt = (int32_t *)ctx->grow(ctx->cnt, (size_t)2 * L * sizeof(int32_t));
        uint8_t *d_nxt = (uint8_t *)ctx->grow(ctx->nxt, (size_t)2 * L);
        int64_t *d_poff = (int64_t *)ctx->grow(ctx->poff, (size_t)2 * L * sizeof(int64_t));
        int64_t *d_gptr = (int64_t *)ctx->grow(ctx->gptr, (size_t)2 * (L + 1) * sizeof(int64_t));
        int32_t *d_lrow = (int32_t *)ctx->grow(ctx->lrow, (size_t)L * sizeof(int32_t));
        uint8_t *d_snind = (uint8_t *)ctx->grow(ctx->snind, (size_t)L);
        int32_t *d_sn = (int32_t *)ctx->grow(ctx->snlist, (size_t)L * sizeof(int32_t));
        int64_t *d_tiles = (int64_t *)ctx->grow(ctx->tiles, (size_t)4 * ntiles * sizeof(int64_t));
        // misc: piece counter, pool tail, counters[4], status
        char *d_misc = (char *)ctx->grow(ctx->misc, 256);
        unsigned long long *d_piece = (unsigned long long *)d_misc;
        unsigned long long *d_tail = (unsigned long long *)(d_misc + 8);
        unsigned long long *d_counters = (unsigned long long *)(d_misc + 16);   // 16 counters
        uint32_t *d_status = (uint32_t *)(d_misc + 192);
        int32_t *d_pool = nullptr, *d_out = nullptr;
        uint16_t *d_stamp = nullptr;
        // a 16-bit chain index per vertex for every traversal: its lists are
        // read off the bitmap when the chain ends
        const int64_t stamp_stride = (int64_t)bitmap_words * 32;
        if (pattern_form == 1) {
            d_pool = (int32_t *)ctx->grow(ctx->pool, (size_t)pool_cap * sizeof(int32_t));
            d_out = (int32_t *)ctx->grow(ctx->out, (size_t)pool_cap * sizeof(int32_t));
        } else if (pattern_form == 2) {
            d_pool = ext->dev;
        }
        if (want_pattern)
            d_stamp = (uint16_t *)ctx->grow(ctx->stamp, (size_t)grid * NS * stamp_stride * sizeof(uint16_t));
        uint32_t *d_gstate = gbm ? (uint32_t *)ctx->grow(ctx->gstate, (size_t)grid * NS * state_words * 4) : nullptr;
        MatDesc *d_mats = (MatDesc *)ctx->grow(ctx->mats, md.size() * sizeof(MatDesc));
        int64_t *d_minfo = (int64_t *)ctx->grow(ctx->matinfo, (size_t)3 * count * sizeof(int64_t));
        Range *d_ranges = (Range *)ctx->grow(ctx->ranges, std::max<size_t>(ranges.size(), 1) * sizeof(Range));

        cudaStream_t st = ctx->stream;
        JobArgs a{};
        a.mats = d_mats;
        a.nmats = count;
        a.nranges = (int32_t)ranges.size();
        a.ranges = d_ranges;
        a.npieces = npieces;
        a.piece_counter = d_piece;
        a.queue = d_queue;
        a.qcap = qcap;
        a.bitmap_words = bitmap_words;
        a.state_words = state_words;
        a.ring_size = ring;
        a.lanes = lanes;
        a.reuse = reuse;
        a.want_pattern = pattern_form;
        a.max_sn = p.max_supernode_size;
        a.L = L;
        a.cnt = d_cnt;
        a.nxt = d_nxt;
        a.poff = d_poff;
        a.pool = d_pool;
        a.pool_cap = pool_cap;
        a.pool_tail = d_tail;
        a.gptr = d_gptr;
        a.out = d_out;
        a.lrow = d_lrow;
        a.snind = d_snind;
        a.sn_list = d_sn;
        a.mat_info = d_minfo;
        a.ntiles = ntiles;
        // a line range without the CSR form needs its own lines only: the
        // scans cover its tiles (the totals are its lists' lengths, and no
        // supernode partition is formed from part of the lines)
        a.tile_lo = restrict_tiles ? (int64_t)range_lo / TILE : 0;
        a.tile_hi = restrict_tiles ? ((int64_t)range_hi + TILE - 1) / TILE : ntiles;
        a.tile_sum = d_tiles;
        a.tile_last = d_tiles + 2 * ntiles;
        a.tile_sn = d_tiles + 3 * ntiles;
        a.counters = d_counters;
        a.status = d_status;
        a.stamp = d_stamp;
        a.stamp_stride = stamp_stride;
        a.gbm = d_gstate;
        a.blk_done = ext ? ext->blk_done : nullptr;
        a.blk_shift = ext ? ext->blk_shift : 0;

        // The job: descriptor copies, clears and the cooperative launch.  With
        // GSOFA_FLAG_GRAPH it is captured once into a CUDA graph and replayed
        // while the same job (matrices, parameters, buffers) comes back.
        const MatDesc *md_src = md.data();
        const Range *rg_src = ranges.data();
        // The shared-memory attribute is set under the lock right before each
        // launch (and graph launch); inside a capture it was set beforehand.
        auto issue = [&](void *const *kargs, bool capturing) {
            GS_CUDA(cudaMemcpyAsync(d_mats, md_src, md.size() * sizeof(MatDesc), cudaMemcpyHostToDevice, st));
            if (!ranges.empty())
                GS_CUDA(cudaMemcpyAsync(d_ranges, rg_src, ranges.size() * sizeof(Range),
                                        cudaMemcpyHostToDevice, st));
            GS_CUDA(cudaMemsetAsync(d_misc, 0, 256, st));
            GS_CUDA(cudaMemsetAsync(d_lrow, 0, (size_t)L * sizeof(int32_t), st));
            if (a.blk_done) GS_CUDA(cudaMemsetAsync(a.blk_done, 0, (size_t)ext->nblk * 4, st));
            if (subset) {
                GS_CUDA(cudaMemsetAsync(d_cnt, 0, (size_t)2 * L * sizeof(int32_t), st));
                GS_CUDA(cudaMemsetAsync(d_nxt, 0, (size_t)2 * L, st));
            }
            std::unique_lock<std::mutex> lk(kernel_attr_mutex(), std::defer_lock);
            if (!capturing) {
                lk.lock();
                GS_CUDA(cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            }
            GS_CUDA(cudaLaunchCooperativeKernel(kfn, dim3(grid), dim3(block), (void **)kargs, smem, st));
        };
        void *args[] = {&a};
        bool graphed = false;
        if (p.flags & GSOFA_FLAG_GRAPH) {
            std::vector<char> key(sizeof(JobArgs) + md.size() * sizeof(MatDesc) +
                                  ranges.size() * sizeof(Range) + 4 * sizeof(int64_t));
            char *kp = key.data();
            std::memcpy(kp, &a, sizeof(JobArgs)); kp += sizeof(JobArgs);
            std::memcpy(kp, md.data(), md.size() * sizeof(MatDesc)); kp += md.size() * sizeof(MatDesc);
            if (!ranges.empty()) std::memcpy(kp, ranges.data(), ranges.size() * sizeof(Range));
            kp += ranges.size() * sizeof(Range);
            const int64_t extra[4] = {(int64_t)(intptr_t)kfn, grid, block, (int64_t)smem};
            std::memcpy(kp, extra, sizeof(extra));
            GraphCache &gc = ctx->graph;
            if (!(gc.exec && gc.key == key && gc.stream == st)) {
                if (gc.exec) { cudaGraphExecDestroy(gc.exec); gc.exec = nullptr; }
                gc.key = key;
                gc.md = md;
                gc.ranges = ranges;
                gc.stream = st;
                md_src = gc.md.data();
                rg_src = gc.ranges.data();
                gc.args = a;
                void *gargs[] = {&gc.args};
                cudaGraph_t graph = nullptr;
                {
                    std::lock_guard<std::mutex> lk(kernel_attr_mutex());
                    GS_CUDA(cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
                }
                bool ok = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
                if (ok) {
                    try {
                        issue(gargs, true);
                    } catch (CudaFail &) {
                        ok = false;
                    }
                    ok = (cudaStreamEndCapture(st, &graph) == cudaSuccess) && ok;
                }
                if (ok) ok = cudaGraphInstantiate(&gc.exec, graph, 0) == cudaSuccess;
                if (graph) cudaGraphDestroy(graph);
                if (!ok) {
                    cudaGetLastError();
                    gc.exec = nullptr;
                    gc.key.clear();
                }
            }
            graphed = gc.exec != nullptr;
        }
        const double t_launch = now_ms();
        GS_CUDA(cudaEventRecord(ctx->ev0, st));
        if (graphed) {
            std::lock_guard<std::mutex> lk(kernel_attr_mutex());
            GS_CUDA(cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            GS_CUDA(cudaGraphLaunch(ctx->graph.exec, st));
        } else {
            issue(args, false);
        }
        GS_CUDA(cudaEventRecord(ctx->ev1, st));
        if (ext && ext->while_running) ext->while_running();

        unsigned long long h_misc[25];
        GS_CUDA(cudaMemcpyAsync(h_misc, d_misc, sizeof(h_misc), cudaMemcpyDeviceToHost, st));
        int64_t tot[2];
        GS_CUDA(cudaMemcpyAsync(&tot[0], d_gptr + L, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
        GS_CUDA(cudaMemcpyAsync(&tot[1], d_gptr + (L + 1) + L, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
        GS_CUDA(cudaStreamSynchronize(st));
        const double t_done = now_ms();
        float ms = 0.f;
        GS_CUDA(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
        const uint32_t status = (uint32_t)(h_misc[24] & 0xffffffffu);
        const unsigned long long edges = h_misc[2], nsrc = h_misc[3], nsn = h_misc[4];
        const unsigned long long xtot = h_misc[5], einsp = h_misc[6];
        const unsigned long long levels = h_misc[7], reused = h_misc[8];

        if (status & ERR_QUEUE_OVERFLOW) return GSOFA_ERR_QUEUE_OVERFLOW;
        // a list's count and its pattern disagree: an internal fault, never
        // a property of the input
        if (status & ERR_COUNT_MISMATCH) return GSOFA_ERR_CUDA;
        if (want_pattern && (status & ERR_POOL_OVERFLOW)) {
            if (attempt == 0 && pattern_form == 1) {
                pool_cap = pool_need(tot[0] + tot[1]);
                continue;   // rerun with the pool the counts ask for
            }
            // the caller's pool is too small: report what the job needs
            for (int i = 0; i < count; i++) out[i].pool_used = (int64_t)h_misc[1];
            return GSOFA_ERR_QUEUE_OVERFLOW;
        }

        // per-matrix results: offsets at every matrix's first line come from
        // mat_info (empty matrices take their successor's values)
        std::vector<int64_t> mi((size_t)3 * count);
        GS_CUDA(cudaMemcpyAsync(mi.data(), d_minfo, mi.size() * sizeof(int64_t), cudaMemcpyDeviceToHost, st));
        GS_CUDA(cudaStreamSynchronize(st));
        std::vector<int64_t> s0(count + 1), s1(count + 1), ss(count + 1);
        s0[count] = tot[0];
        s1[count] = tot[1];
        ss[count] = (int64_t)nsn;
        for (int i = count - 1; i >= 0; i--) {
            if (restrict_tiles) {   // one matrix; its own lines only, no supernodes
                s0[i] = s1[i] = 0;
                ss[i] = ss[i + 1] = 0;
            } else if (md[i].n > 0) {
                s0[i] = mi[3 * i];
                s1[i] = mi[3 * i + 1];
                ss[i] = line_range ? 0 : mi[3 * i + 2];
                if (line_range) ss[i + 1] = 0;
            } else {
                s0[i] = s0[i + 1];
                s1[i] = s1[i + 1];
                ss[i] = ss[i + 1];
            }
        }
        const bool download_lines = !(p.flags & GSOFA_FLAG_NO_DOWNLOAD);
        std::vector<uint8_t *> lflags;
        for (int i = 0; i < count; i++) {
            const int64_t lb = md[i].line_base, n = md[i].n;
            gsofa_result &r = out[i];
            r.nnz_u = (uint64_t)(s0[i + 1] - s0[i]);
            r.nnz_l = (uint64_t)(s1[i + 1] - s1[i]);
            r.nnz_lu = r.nnz_u + r.nnz_l + (uint64_t)n;
            r.n_supernodes = (int32_t)(ss[i + 1] - ss[i]);
            r.kernel_ms = ms;
            r.edges_inspected = edges;
            r.sources = nsrc;
            r.x_total = xtot;
            r.e_insp = einsp;
            r.levels = levels;
            r.reused_sources = reused;
            for (int q = 0; q < 7; q++) r.cycles[q] = h_misc[9 + q];
            r.ctas = (uint64_t)grid;
            r.pool_used = want_pattern ? (int64_t)h_misc[1] : 0;
            if (!subset) {
                r.fill_count = r.nnz_u - mats[i]->orig_up + r.nnz_l - mats[i]->orig_lo;
                const_cast<gsofa_matrix *>(mats[i])->last_pattern_total = (int64_t)(r.nnz_u + r.nnz_l);
            }
            if (download_lines) {
                r.u_row_count = download(st, d_cnt, lb, n);
                r.l_col_count = download(st, d_cnt, L + lb, n);
                if (want_pattern) r.l_row_count = download(st, d_lrow, lb, n);
                r.sn_start = download(st, d_sn, ss[i], r.n_supernodes);
                // link flags: bit 0 from pass G, bit 1 from pass G^T (merged below)
                r.line_flags = download(st, d_nxt, lb, n);
                lflags.push_back(download(st, d_nxt, L + lb, n));
                if (pattern_form == 1) {
                    r.u_ptr = download(st, d_gptr, lb, n + 1);
                    r.l_ptr = download(st, d_gptr, (L + 1) + lb, n + 1);
                    r.u_idx = download(st, d_out, s0[i], (int64_t)r.nnz_u);
                    r.l_idx = download(st, d_out, tot[0] + s1[i], (int64_t)r.nnz_l);
                } else if (pattern_form == 2) {
                    r.u_beg = download(st, d_poff, lb, n);
                    r.l_beg = download(st, d_poff, L + lb, n);
                }
            }
            // where the result sits on the device, for gsofa_result_fetch and
            // gsofa_result_supernodal (valid until the next job on ctx)
            ResultInternal *ri = new ResultInternal();
            ri->job_id = ctx->job_id;
            ri->L = L;
            ri->line_base = lb;
            ri->n = n;
            ri->u0 = s0[i];
            ri->l0 = tot[0] + s1[i];
            ri->sn0 = ss[i];
            ri->pattern = pattern_form;
            ri->pool = pattern_form == 2 ? d_pool : nullptr;
            r.internal = ri;
        }
        GS_CUDA(cudaStreamSynchronize(st));
        for (int i = 0; i < count && download_lines; i++) {
            gsofa_result &r = out[i];
            const int64_t lb = md[i].line_base, n = md[i].n;
            for (int64_t q = 0; q < n; q++) r.line_flags[q] = (uint8_t)(r.line_flags[q] | (lflags[i][q] << 1));
            std::free(lflags[i]);
            lflags[i] = nullptr;
            for (int32_t k = 0; k < r.n_supernodes; k++) r.sn_start[k] -= (int32_t)lb;
            if (pattern_form == 1) {
                const int64_t u0 = r.u_ptr[0], l0 = r.l_ptr[0];
                for (int64_t q = 0; q <= n; q++) { r.u_ptr[q] -= u0; r.l_ptr[q] -= l0; }
            }
            // fills of the processed lines: subtract their original entries
            if (subset) r.fill_count = r.nnz_u + r.nnz_l - processed_orig(i);
        }
        if (host_timing)
            std::fprintf(stderr,
                         "gsofa host: setup %.3f ms, launch..sync %.3f ms (kernel %.3f, traversals %.3f, "
                         "mean CTA %.3f), results %.3f ms\n",
                         t_launch - t_enter, t_done - t_launch, ms, h_misc[16] * 1e-6,
                         h_misc[17] * 1e-6 / std::max(grid, 1), now_ms() - t_done);
        if (subset && !download_lines)
            for (int i = 0; i < count; i++) out[i].fill_count = out[i].nnz_u + out[i].nnz_l - processed_orig(i);
        return GSOFA_OK;
    }
    return GSOFA_ERR_QUEUE_OVERFLOW;
}

}  // namespace

// ============================================================================
// C ABI

extern "C" {

const char *gsofa_status_str(gsofa_status s)
{
    switch (s) {
    case GSOFA_OK: return "ok";
    case GSOFA_ERR_INVALID_INPUT: return "invalid input";
    case GSOFA_ERR_OOM: return "out of memory";
    case GSOFA_ERR_QUEUE_OVERFLOW: return "queue or pattern pool overflow";
    case GSOFA_ERR_TIMEOUT: return "device wait timed out";
    case GSOFA_ERR_CUDA: return "CUDA error";
    case GSOFA_ERR_IO: return "input file error";
    case GSOFA_ERR_UNSUPPORTED: return "unsupported device or size";
    case GSOFA_ERR_BUSY: return "no room for the request now";
    }
    return "unknown status";
}

int gsofa_abi_version(void) { return GSOFA_ABI_VERSION; }

void gsofa_default_params(gsofa_params *p)
{
    if (!p) return;
    std::memset(p, 0, sizeof(*p));
    p->want_pattern = 1;
    p->reuse = -1;
    p->part_count = 1;
}

gsofa_status gsofa_create(gsofa_ctx **out, int device, size_t mem_budget_bytes)
{
    if (!out) return GSOFA_ERR_INVALID_INPUT;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) {
        cudaGetLastError();
        return GSOFA_ERR_UNSUPPORTED;
    }
    if (device < 0 || device >= ndev) return GSOFA_ERR_INVALID_INPUT;
    gsofa_ctx *c = new (std::nothrow) gsofa_ctx();
    if (!c) return GSOFA_ERR_OOM;
    try {
        c->device = device;
        GS_CUDA(cudaSetDevice(device));
        cudaDeviceProp prop;
        GS_CUDA(cudaGetDeviceProperties(&prop, device));
        if (prop.major < 10 || !prop.cooperativeLaunch) {
            delete c;
            return GSOFA_ERR_UNSUPPORTED;
        }
        c->sm_count = prop.multiProcessorCount;
        c->smem_optin = prop.sharedMemPerBlockOptin;
        size_t fr = 0, tot = 0;
        GS_CUDA(cudaMemGetInfo(&fr, &tot));
        c->budget = mem_budget_bytes ? mem_budget_bytes : (size_t)(0.9 * (double)fr);
        GS_CUDA(cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking));
        c->stream = c->own_stream;
        GS_CUDA(cudaEventCreate(&c->ev0));
        GS_CUDA(cudaEventCreate(&c->ev1));
    } catch (CudaFail &f) {
        gsofa_destroy(c);
        return fail_cuda(f.e);
    }
    *out = c;
    return GSOFA_OK;
}

void gsofa_matrix_free(gsofa_matrix *m)
{
    if (!m) return;
    gsofa_ctx *c = m->ctx;
    if (c) {
        cudaSetDevice(c->device);
        auto &v = c->matrices;
        v.erase(std::remove(v.begin(), v.end(), m), v.end());
    }
    if (c) c->slab_give(m->slab, m->slab_bytes);
    else cudaFree(m->slab);
    delete m;
}

void gsofa_destroy(gsofa_ctx *c)
{
    if (!c) return;
    cudaSetDevice(c->device);
    while (!c->matrices.empty()) gsofa_matrix_free(c->matrices.back());
    DevBuf *bufs[] = {&c->queue, &c->cnt, &c->nxt, &c->poff, &c->gptr, &c->lrow, &c->snind,
                      &c->snlist, &c->tiles, &c->misc, &c->pool, &c->out, &c->mats, &c->ranges,
                      &c->st_beg, &c->st_end, &c->st_adj, &c->st_tmp, &c->matinfo, &c->stamp,
                      &c->sn_head, &c->sn_data, &c->gstate, &c->blk, &c->order};
    for (DevBuf *b : bufs) c->release(*b);
    for (DevBuf &b : c->slabs) cudaFree(b.p);
    c->slabs.clear();
    if (c->graph.exec) cudaGraphExecDestroy(c->graph.exec);
    if (c->ev0) cudaEventDestroy(c->ev0);
    if (c->ev1) cudaEventDestroy(c->ev1);
    if (c->own_stream) cudaStreamDestroy(c->own_stream);
    if (c->s_poll) cudaStreamDestroy(c->s_poll);
    if (c->s_copy) cudaStreamDestroy(c->s_copy);
    if (c->h_blk) cudaFreeHost(c->h_blk);
    delete c;
}

gsofa_status gsofa_set_stream(gsofa_ctx *c, void *cuda_stream)
{
    if (!c) return GSOFA_ERR_INVALID_INPUT;
    c->stream = cuda_stream ? (cudaStream_t)cuda_stream : c->own_stream;
    return GSOFA_OK;
}

void gsofa_free(void *p) { std::free(p); }

int32_t gsofa_matrix_n(const gsofa_matrix *m) { return m ? m->n : -1; }

// Binary form of the three input files: the 8-byte magic, little-endian
// int64 counts (csr: nnz then n; colbeg and colend: n), then the int32 ids.
static const char kBinMagic[8] = {'G', 'S', 'O', 'F', 'A', 'B', '0', '1'};

namespace {

// One input file, text or binary (told apart by the magic).  The id count is
// counts[0]: read from the file's header -- text_counts numbers before the ids
// in the text form, bin_counts in the binary one -- or, for a form without a
// header, `want`.  `want` >= 0 is also checked against a header's count.  The
// ids go to a malloc'd array.
gsofa_status read_input_file(const char *path, int text_counts, int bin_counts, long long *counts,
                             long long want, int32_t **ids_out)
{
    *ids_out = nullptr;
    FILE *f = std::fopen(path, "rb");
    if (!f) return GSOFA_ERR_IO;
    char head[8] = {0};
    const bool binary = std::fread(head, 1, 8, f) == 8 && std::memcmp(head, kBinMagic, 8) == 0;
    if (!binary) std::rewind(f);
    const int nc = binary ? bin_counts : text_counts;
    for (int k = 0; k < nc; k++) {
        long long v = -1;
        if (binary) {
            int64_t x = -1;
            if (std::fread(&x, 8, 1, f) != 1) { std::fclose(f); return GSOFA_ERR_IO; }
            v = (long long)x;
        } else if (std::fscanf(f, "%lld", &v) != 1) {
            std::fclose(f);
            return GSOFA_ERR_IO;
        }
        if (v < 0 || v > INT32_MAX) { std::fclose(f); return GSOFA_ERR_IO; }
        counts[k] = v;
    }
    if (nc == 0) counts[0] = want;
    const long long cnt = counts[0];
    if (cnt < 0 || (want >= 0 && cnt != want)) { std::fclose(f); return GSOFA_ERR_IO; }
    int32_t *ids = (int32_t *)std::malloc((size_t)std::max<long long>(cnt, 1) * 4);
    if (!ids) { std::fclose(f); return GSOFA_ERR_OOM; }
    bool ok = true;
    if (binary) {
        ok = std::fread(ids, 4, (size_t)cnt, f) == (size_t)cnt;
    } else {
        for (long long i = 0; i < cnt && ok; i++) {
            long long x;
            ok = std::fscanf(f, "%lld", &x) == 1 && x >= INT32_MIN && x <= INT32_MAX;
            if (ok) ids[i] = (int32_t)x;
        }
    }
    std::fclose(f);
    if (!ok) { std::free(ids); return GSOFA_ERR_IO; }
    *ids_out = ids;
    return GSOFA_OK;
}

}  // namespace

gsofa_status gsofa_read_text(const char *beg_file, const char *end_file, const char *csr_file,
                             int32_t *n_out, int64_t *nnz_out, int32_t **beg_out,
                             int32_t **end_out, int32_t **adj_out)
{
    if (!beg_file || !end_file || !csr_file || !n_out || !nnz_out || !beg_out || !end_out || !adj_out)
        return GSOFA_ERR_INVALID_INPUT;
    *beg_out = *end_out = *adj_out = nullptr;
    // csr: "nnz n" then nnz ids; colbeg / colend: n ids each (their binary
    // form repeats n in its header)
    long long hc[2] = {-1, -1}, cb = -1, ce = -1;
    int32_t *adj = nullptr, *beg = nullptr, *end = nullptr;
    gsofa_status s = read_input_file(csr_file, 2, 2, hc, -1, &adj);
    if (s != GSOFA_OK) return s;
    const long long nnz = hc[0], n = hc[1];
    s = read_input_file(beg_file, 0, 1, &cb, n, &beg);
    if (s == GSOFA_OK) s = read_input_file(end_file, 0, 1, &ce, n, &end);
    if (s != GSOFA_OK) {
        std::free(adj); std::free(beg); std::free(end);
        return s;
    }
    *n_out = (int32_t)n;
    *nnz_out = nnz;
    *beg_out = beg;
    *end_out = end;
    *adj_out = adj;
    return GSOFA_OK;
}

gsofa_status gsofa_write_binary(const char *beg_file, const char *end_file, const char *csr_file,
                                int32_t n, int64_t nnz, const int32_t *beg, const int32_t *end,
                                const int32_t *adj)
{
    if (!beg_file || !end_file || !csr_file || n < 0 || nnz < 0 || nnz > INT32_MAX ||
        (n > 0 && (!beg || !end)) || (nnz > 0 && !adj))
        return GSOFA_ERR_INVALID_INPUT;
    auto put = [](const char *path, const int64_t *hdr, int nh, const int32_t *ids, int64_t cnt) -> bool {
        FILE *f = std::fopen(path, "wb");
        if (!f) return false;
        bool ok = std::fwrite(kBinMagic, 1, 8, f) == 8 && std::fwrite(hdr, 8, (size_t)nh, f) == (size_t)nh &&
                  (cnt == 0 || std::fwrite(ids, 4, (size_t)cnt, f) == (size_t)cnt);
        return (std::fclose(f) == 0) && ok;
    };
    const int64_t hcsr[2] = {nnz, (int64_t)n}, hn[1] = {(int64_t)n};
    if (!put(csr_file, hcsr, 2, adj, nnz) || !put(beg_file, hn, 1, beg, n) || !put(end_file, hn, 1, end, n))
        return GSOFA_ERR_IO;
    return GSOFA_OK;
}

gsofa_status gsofa_upload(gsofa_ctx *c, int32_t n, int64_t nnz, const int32_t *beg,
                          const int32_t *end, const int32_t *adj, gsofa_matrix **out)
{
    if (!c || !out || n < 0 || nnz < 0 || nnz > INT32_MAX) return GSOFA_ERR_INVALID_INPUT;
    if ((n > 0 && (!beg || !end)) || (nnz > 0 && !adj)) return GSOFA_ERR_INVALID_INPUT;
    *out = nullptr;
    gsofa_matrix *m = new (std::nothrow) gsofa_matrix();
    if (!m) return GSOFA_ERR_OOM;
    m->ctx = c;
    m->n = n;
    m->nnz_in = nnz;
    try {
        GS_CUDA(cudaSetDevice(c->device));
        cudaStream_t st = c->stream;
        const size_t nb = (size_t)std::max<int32_t>(n, 1) * 4;
        int32_t *d_beg = (int32_t *)c->grow(c->st_beg, nb);
        int32_t *d_end = (int32_t *)c->grow(c->st_end, nb);
        int32_t *d_adj = (int32_t *)c->grow(c->st_adj, (size_t)std::max<int64_t>(nnz, 1) * 4);
        // tmp: deg[n] | indeg[n+1] | tcursor[n+1] | tile sums | counts | status
        const int64_t scan_tiles = ((int64_t)n + 1 + 255) / 256 + 1;
        const size_t ints_bytes = ((size_t)(3 * ((int64_t)n + 1)) * 4 + 15) / 16 * 16;
        const size_t tmp_bytes = ints_bytes + (size_t)(2 * scan_tiles) * 8 + 64;
        char *tmp = (char *)c->grow(c->st_tmp, tmp_bytes);
        int32_t *d_deg = (int32_t *)tmp;
        int32_t *d_indeg = d_deg + (n + 1);
        int32_t *d_tcur = d_indeg + (n + 1);
        int64_t *d_tsum = (int64_t *)(tmp + ints_bytes);
        unsigned long long *d_counts = (unsigned long long *)(d_tsum + 2 * scan_tiles);
        uint32_t *d_status = (uint32_t *)(d_counts + 4);

        // one slab: G and G^T offsets, per-line counts, and both adjacency
        // arrays (at most nnz entries each: the input minus diagonal and
        // duplicates)
        {
            auto al = [](size_t b) { return (b + 255) / 256 * 256; };
            const size_t pb = al((size_t)(n + 1) * 4), lb = al(nb);
            const size_t ab = al((size_t)std::max<int64_t>(nnz, 1) * 4);
            // row slots only where most rows fit one (mean off-diagonal
            // degree of the input at most SLOT_NB)
            const bool slots = nnz - (int64_t)n <= (int64_t)SLOT_NB * n;
            const size_t sb = slots ? al((size_t)std::max<int32_t>(n, 1) * 32) : 0;
            const size_t total = 2 * pb + 3 * lb + 2 * ab + 2 * sb;
            char *q = (char *)c->slab_take(total, &m->slab_bytes);
            m->slab = q;
            m->d_gptr = (int32_t *)q; q += pb;
            m->d_tptr = (int32_t *)q; q += pb;
            m->d_orig_up = (int32_t *)q; q += lb;
            m->d_orig_lo = (int32_t *)q; q += lb;
            m->d_rawdeg = (int32_t *)q; q += lb;
            m->d_gslot = sb ? (int4 *)q : nullptr; q += sb;
            m->d_tslot = sb ? (int4 *)q : nullptr; q += sb;
            m->d_gadj = (int32_t *)q; q += ab;
            m->d_tadj = (int32_t *)q;
        }
        c->matrices.push_back(m);

        if (n > 0) {
            GS_CUDA(cudaMemcpyAsync(d_beg, beg, (size_t)n * 4, cudaMemcpyHostToDevice, st));
            GS_CUDA(cudaMemcpyAsync(d_end, end, (size_t)n * 4, cudaMemcpyHostToDevice, st));
        }
        if (nnz > 0) GS_CUDA(cudaMemcpyAsync(d_adj, adj, (size_t)nnz * 4, cudaMemcpyHostToDevice, st));
        GS_CUDA(cudaMemsetAsync(d_indeg, 0, (size_t)(n + 1) * 4, st));
        GS_CUDA(cudaMemsetAsync(d_counts, 0, 64, st));
        GS_CUDA(cudaMemsetAsync(m->d_orig_lo, 0, nb, st));
        GS_CUDA(cudaMemsetAsync(d_deg, 0, (size_t)(n + 1) * 4, st));

        UploadArgs u{};
        u.n = n;
        u.nnz = nnz;
        u.beg = d_beg;
        u.end = d_end;
        u.adj = d_adj;
        u.deg = d_deg;
        u.indeg = d_indeg;
        u.orig_up = m->d_orig_up;
        u.orig_lo = m->d_orig_lo;
        u.rawdeg = m->d_rawdeg;
        u.counts = d_counts;
        u.status = d_status;
        const int ub = 256;
        const int ugrid = (int)std::min<int64_t>(std::max<int64_t>(((int64_t)n * 32 + ub - 1) / ub, 1),
                                                 (int64_t)c->sm_count * 16);
        if (n > 0) {
            upload_count_kernel<<<ugrid, ub, 0, st>>>(u);
            GS_CUDA(cudaGetLastError());
        }
        // G offsets (from deg) and G^T offsets (from indeg)
        int64_t tot[2] = {0, 0};
        const int64_t ntl = ((int64_t)n + 255) / 256;
        int32_t *scan_in[2] = {d_deg, d_indeg};
        int32_t *scan_out[2] = {m->d_gptr, m->d_tptr};
        for (int k = 0; k < 2; k++) {
            int64_t *ts = d_tsum + k * scan_tiles;
            int64_t *dt = (int64_t *)(d_counts + 2 + k);
            if (ntl > 0) scan_tiles_kernel<256><<<(unsigned)ntl, 256, 0, st>>>(scan_in[k], n, ts);
            scan_partials_kernel<256><<<1, 256, 0, st>>>(ts, ntl, dt);
            scan_apply_kernel<256><<<(unsigned)std::max<int64_t>(ntl, 1), 256, 0, st>>>(scan_in[k], n, ts,
                                                                                       scan_out[k], dt);
            GS_CUDA(cudaGetLastError());
        }
        unsigned long long hc[5];
        GS_CUDA(cudaMemcpyAsync(hc, d_counts, 5 * 8, cudaMemcpyDeviceToHost, st));
        GS_CUDA(cudaStreamSynchronize(st));
        uint32_t status = (uint32_t)(hc[4] & 0xffffffffu);
        tot[0] = (int64_t)hc[2];
        tot[1] = (int64_t)hc[3];
        if (status & 1u) {
            gsofa_matrix_free(m);
            return GSOFA_ERR_INVALID_INPUT;
        }
        m->orig_up = hc[0];
        m->orig_lo = hc[1];
        m->nnz_g = tot[0];
        if (tot[0] > std::max<int64_t>(nnz, 1) || tot[1] > std::max<int64_t>(nnz, 1))
            throw CudaFail{cudaErrorInvalidValue};   // cannot happen: kept entries <= input entries
        GS_CUDA(cudaMemcpyAsync(d_tcur, m->d_tptr, (size_t)(n + 1) * 4, cudaMemcpyDeviceToDevice, st));
        if (n > 0) {
            upload_fill_kernel<<<ugrid, ub, 0, st>>>(u, m->d_gptr, m->d_gadj, d_tcur, m->d_tadj);
            GS_CUDA(cudaGetLastError());
            if (m->d_gslot != nullptr) {
                const int sgrid = (int)std::min<int64_t>(((int64_t)n + 255) / 256, (int64_t)c->sm_count * 8);
                slot_fill_kernel<<<sgrid, 256, 0, st>>>(n, m->d_gptr, m->d_gadj, m->d_gslot);
                slot_fill_kernel<<<sgrid, 256, 0, st>>>(n, m->d_tptr, m->d_tadj, m->d_tslot);
                GS_CUDA(cudaGetLastError());
            }
        }
        GS_CUDA(cudaStreamSynchronize(st));
    } catch (CudaFail &f) {
        gsofa_matrix_free(m);
        return fail_cuda(f.e);
    }
    *out = m;
    return GSOFA_OK;
}

gsofa_status gsofa_symbfact(gsofa_ctx *c, const gsofa_matrix *m, const gsofa_params *params,
                            gsofa_result *out)
{
    return gsofa_symbfact_batch(c, 1, &m, params, out);
}

gsofa_status gsofa_symbfact_batch(gsofa_ctx *c, int count, const gsofa_matrix *const *mats,
                                  const gsofa_params *params, gsofa_result *out)
{
    if (!c) return GSOFA_ERR_INVALID_INPUT;
    try {
        GS_CUDA(cudaSetDevice(c->device));
        gsofa_status s = run_job(c, count, mats, params, out);
        if (s != GSOFA_OK && out)
            for (int i = 0; i < count; i++) free_result_arrays(&out[i]);
        return s;
    } catch (CudaFail &f) {
        if (out)
            for (int i = 0; i < count; i++) free_result_arrays(&out[i]);
        return fail_cuda(f.e);
    } catch (std::bad_alloc &) {
        if (out)
            for (int i = 0; i < count; i++) free_result_arrays(&out[i]);
        return GSOFA_ERR_OOM;
    }
}

void gsofa_result_free(gsofa_result *r)
{
    if (!r) return;
    free_result_arrays(r);
    delete (ResultInternal *)r->internal;
    r->internal = nullptr;
}

gsofa_status gsofa_result_fetch(gsofa_ctx *c, const gsofa_result *r, int32_t *u_row_count,
                                int32_t *l_col_count, int32_t *l_row_count, int32_t *sn_start,
                                int64_t *u_ptr, int32_t *u_idx, int64_t *l_ptr, int32_t *l_idx)
{
    if (!c || !r || !r->internal) return GSOFA_ERR_INVALID_INPUT;
    const ResultInternal *ri = (const ResultInternal *)r->internal;
    if (ri->job_id != c->job_id) return GSOFA_ERR_INVALID_INPUT;
    try {
        GS_CUDA(cudaSetDevice(c->device));
        cudaStream_t st = c->stream;
        const int64_t L = ri->L, lb = ri->line_base, n = ri->n;
        const int32_t *cnt = (const int32_t *)c->cnt.p;
        const int64_t *gptr = (const int64_t *)c->gptr.p;
        const int32_t *outb = (const int32_t *)c->out.p;
        auto cp = [&](void *dst, const void *src, size_t bytes) {
            if (dst && bytes) GS_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, st));
        };
        if (l_row_count && !ri->pattern) return GSOFA_ERR_INVALID_INPUT;   // counted with the pattern only
        if ((u_ptr || u_idx || l_ptr || l_idx) && (ri->pattern != 1 || !outb))
            return GSOFA_ERR_INVALID_INPUT;   // the CSR form only
        cp(u_row_count, cnt + lb, (size_t)n * 4);
        cp(l_col_count, cnt + L + lb, (size_t)n * 4);
        cp(l_row_count, (const int32_t *)c->lrow.p + lb, (size_t)n * 4);
        cp(u_ptr, gptr + lb, (size_t)(n + 1) * 8);
        cp(l_ptr, gptr + (L + 1) + lb, (size_t)(n + 1) * 8);
        cp(u_idx, outb + ri->u0, (size_t)r->nnz_u * 4);
        cp(l_idx, outb + ri->l0, (size_t)r->nnz_l * 4);
        cp(sn_start, (const int32_t *)c->snlist.p + ri->sn0, (size_t)r->n_supernodes * 4);
        GS_CUDA(cudaStreamSynchronize(st));
        if (sn_start)
            for (int32_t k = 0; k < r->n_supernodes; k++) sn_start[k] -= (int32_t)lb;
        if (u_ptr) {
            const int64_t b = u_ptr[0];
            for (int64_t s = 0; s <= n; s++) u_ptr[s] -= b;
        }
        if (l_ptr) {
            const int64_t b = l_ptr[0];
            for (int64_t s = 0; s <= n; s++) l_ptr[s] -= b;
        }
    } catch (CudaFail &f) {
        return fail_cuda(f.e);
    }
    return GSOFA_OK;
}

gsofa_status gsofa_result_fetch_ranges(gsofa_ctx *c, const gsofa_result *r, int64_t *u_beg,
                                       int64_t *l_beg)
{
    if (!c || !r || !r->internal) return GSOFA_ERR_INVALID_INPUT;
    const ResultInternal *ri = (const ResultInternal *)r->internal;
    if (ri->job_id != c->job_id || ri->pattern != 2) return GSOFA_ERR_INVALID_INPUT;
    try {
        GS_CUDA(cudaSetDevice(c->device));
        cudaStream_t st = c->stream;
        const int64_t *poff = (const int64_t *)c->poff.p;
        if (u_beg && ri->n)
            GS_CUDA(cudaMemcpyAsync(u_beg, poff + ri->line_base, (size_t)ri->n * 8, cudaMemcpyDeviceToHost, st));
        if (l_beg && ri->n)
            GS_CUDA(cudaMemcpyAsync(l_beg, poff + ri->L + ri->line_base, (size_t)ri->n * 8,
                                    cudaMemcpyDeviceToHost, st));
        GS_CUDA(cudaStreamSynchronize(st));
    } catch (CudaFail &f) {
        return fail_cuda(f.e);
    }
    return GSOFA_OK;
}

gsofa_status gsofa_symbfact_ranges(gsofa_ctx *c, int count, const gsofa_matrix *const *mats,
                                   const gsofa_params *params, int32_t *pool, int64_t pool_capacity,
                                   gsofa_result *out)
{
    if (!c || !pool || pool_capacity <= 0 || count <= 0 || !out) return GSOFA_ERR_INVALID_INPUT;
    gsofa_params p;
    resolve_params(params, &p);
    if (p.part_count > 1) return GSOFA_ERR_INVALID_INPUT;
    p.want_pattern = 2;
    try {
        GS_CUDA(cudaSetDevice(c->device));
        // the pool: device memory of this device, or page-locked host memory
        // (written through its device alias while the traversals run)
        cudaPointerAttributes at{};
        if (cudaPointerGetAttributes(&at, pool) != cudaSuccess) {
            cudaGetLastError();
            return GSOFA_ERR_INVALID_INPUT;
        }
        ExtPool ext;
        ext.cap = pool_capacity;
        int32_t *host_dst = nullptr;   // staged: lists go to a device pool, then here
        if (at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged) {
            if (at.type == cudaMemoryTypeDevice && at.device != c->device) return GSOFA_ERR_INVALID_INPUT;
            ext.dev = pool;
        } else if (at.type == cudaMemoryTypeHost) {
            void *d = nullptr;
            if (cudaHostGetDevicePointer(&d, pool, 0) != cudaSuccess) {
                cudaGetLastError();
                return GSOFA_ERR_INVALID_INPUT;
            }
            // Staged through device memory when a device pool of the same
            // capacity fits the budget (the copy engine moves it at full
            // PCIe speed); else, or with GSOFA_FLAG_DIRECT_HOST, the kernel
            // writes the lists into host memory itself, so the pattern needs
            // no device memory at all.
            const size_t bytes = (size_t)pool_capacity * 4;
            const bool staged = !(p.flags & GSOFA_FLAG_DIRECT_HOST) && c->held - c->pool.bytes + bytes <= c->budget / 2;
            if (staged) {
                ext.dev = (int32_t *)c->grow(c->pool, bytes);
                host_dst = pool;
            } else {
                ext.dev = (int32_t *)d;
            }
        } else {
            return GSOFA_ERR_INVALID_INPUT;   // pageable host memory
        }
        // Staged: the kernel counts the entries written into every block of
        // kStreamShift entries; while it runs, this thread reads the counts
        // (a small copy on its own stream) and has the copy engine move each
        // full block to the host, so most of the download overlaps the
        // traversals.  The partly filled blocks follow when the kernel ends.
        constexpr int32_t kStreamShift = 22;   // 4M entries (16 MiB) a block
        std::vector<char> copied;
        if (host_dst) {
            if (!c->s_poll) GS_CUDA(cudaStreamCreateWithFlags(&c->s_poll, cudaStreamNonBlocking));
            if (!c->s_copy) GS_CUDA(cudaStreamCreateWithFlags(&c->s_copy, cudaStreamNonBlocking));
            ext.blk_shift = kStreamShift;
            ext.nblk = ((pool_capacity - 1) >> kStreamShift) + 1;
            ext.blk_done = (unsigned int *)c->grow(c->blk, (size_t)ext.nblk * 4);
            if (c->h_blk_cap < (size_t)ext.nblk) {
                if (c->h_blk) cudaFreeHost(c->h_blk);
                c->h_blk = nullptr;
                c->h_blk_cap = 0;
                GS_CUDA(cudaHostAlloc((void **)&c->h_blk, (size_t)ext.nblk * 4, cudaHostAllocDefault));
                c->h_blk_cap = (size_t)ext.nblk;
            }
            copied.assign((size_t)ext.nblk, 0);
            const int64_t bsz = (int64_t)1 << kStreamShift;
            ext.while_running = [&]() {
                for (;;) {
                    const bool finished = cudaEventQuery(c->ev1) == cudaSuccess;
                    GS_CUDA(cudaMemcpyAsync(c->h_blk, ext.blk_done, (size_t)ext.nblk * 4, cudaMemcpyDeviceToHost,
                                            c->s_poll));
                    GS_CUDA(cudaStreamSynchronize(c->s_poll));
                    for (int64_t b = 0; b < ext.nblk; b++)
                        if (!copied[(size_t)b] && (int64_t)c->h_blk[b] == bsz) {
                            GS_CUDA(cudaMemcpyAsync(host_dst + b * bsz, ext.dev + b * bsz, (size_t)bsz * 4,
                                                    cudaMemcpyDeviceToHost, c->s_copy));
                            copied[(size_t)b] = 1;
                        }
                    if (finished) break;
                    std::this_thread::sleep_for(std::chrono::microseconds(50));
                }
            };
        }
        gsofa_status s = run_job(c, count, mats, &p, out, &ext);
        if (host_dst) {
            if (s == GSOFA_OK) {
                const int64_t bsz = (int64_t)1 << kStreamShift, used = out[0].pool_used;
                for (int64_t b = 0; b < ext.nblk && b * bsz < used; b++)
                    if (!copied[(size_t)b])
                        GS_CUDA(cudaMemcpyAsync(host_dst + b * bsz, ext.dev + b * bsz,
                                                (size_t)(std::min(used, (b + 1) * bsz) - b * bsz) * 4,
                                                cudaMemcpyDeviceToHost, c->s_copy));
            }
            GS_CUDA(cudaStreamSynchronize(c->s_copy));
        }
        if (s != GSOFA_OK)
            for (int i = 0; i < count; i++) free_result_arrays(&out[i]);
        return s;
    } catch (CudaFail &f) {
        for (int i = 0; i < count; i++) free_result_arrays(&out[i]);
        return fail_cuda(f.e);
    } catch (std::bad_alloc &) {
        for (int i = 0; i < count; i++) free_result_arrays(&out[i]);
        return GSOFA_ERR_OOM;
    }
}

static bool valid_lines(int32_t n, int64_t nnz, const int32_t *beg, const int32_t *end, const int32_t *adj)
{
    if (n < 0 || nnz < 0 || (n > 0 && (!beg || !end)) || (nnz > 0 && !adj)) return false;
    for (int32_t v = 0; v < n; v++)
        if (beg[v] < 0 || end[v] < beg[v] || (int64_t)end[v] > nnz) return false;
    for (int32_t v = 0; v < n; v++)
        for (int32_t k = beg[v]; k < end[v]; k++)
            if (adj[k] < 0 || adj[k] >= n) return false;
    return true;
}

gsofa_status gsofa_predict_line_counts(int32_t n, int64_t nnz, const int32_t *beg, const int32_t *end,
                                       const int32_t *adj, int64_t *counts)
{
    if (!counts || !valid_lines(n, nnz, beg, end, adj)) return GSOFA_ERR_INVALID_INPUT;
    try {
        const gsofa::part::Sym sy = gsofa::part::symmetric_structure(n, beg, end, adj);
        const std::vector<int32_t> parent = gsofa::part::etree(n, sy);
        const std::vector<int32_t> post = gsofa::part::postorder(n, parent);
        const std::vector<int64_t> cc = gsofa::part::column_counts(n, sy, parent, post);
        for (int32_t v = 0; v < n; v++) counts[v] = cc[(size_t)v] - 1;
    } catch (std::bad_alloc &) {
        return GSOFA_ERR_OOM;
    }
    return GSOFA_OK;
}

gsofa_status gsofa_partition_lines(int32_t n, int64_t nnz, const int32_t *beg, const int32_t *end,
                                   const int32_t *adj, int32_t parts, int32_t *cuts, double *work)
{
    if (parts <= 0 || !cuts || !valid_lines(n, nnz, beg, end, adj)) return GSOFA_ERR_INVALID_INPUT;
    try {
        gsofa::part::partition(n, beg, end, adj, parts, cuts, work);
    } catch (std::bad_alloc &) {
        return GSOFA_ERR_OOM;
    }
    return GSOFA_OK;
}

gsofa_status gsofa_order_rcm(gsofa_ctx *c, int32_t n, int64_t nnz, const int32_t *beg, const int32_t *end,
                             const int32_t *adj, int32_t *perm)
{
    if (!c || (n > 0 && !perm) || !valid_lines(n, nnz, beg, end, adj)) return GSOFA_ERR_INVALID_INPUT;
    if (n == 0) return GSOFA_OK;
    try {
        GS_CUDA(cudaSetDevice(c->device));
        cudaStream_t st = c->stream;
        // key slots: two per entry of every line's range
        std::vector<int64_t> off((size_t)n + 1);
        off[0] = 0;
        for (int32_t v = 0; v < n; v++) off[(size_t)v + 1] = off[(size_t)v] + 2 * (int64_t)(end[v] - beg[v]);
        const int64_t total = off[(size_t)n];
        if (total > INT32_MAX) return GSOFA_ERR_UNSUPPORTED;   // one radix sort holds at most 2^31 keys
        const int64_t nk = std::max<int64_t>(std::max<int64_t>(total, n), 1);
        size_t sort_tmp = 0, uniq_tmp = 0;
        GS_CUDA(cub::DeviceRadixSort::SortKeys(nullptr, sort_tmp, (unsigned long long *)nullptr,
                                               (unsigned long long *)nullptr, (int)nk, 0, 64, st));
        GS_CUDA(cub::DeviceSelect::Unique(nullptr, uniq_tmp, (unsigned long long *)nullptr,
                                          (unsigned long long *)nullptr, (int *)nullptr, (int)nk, st));
        const size_t tmp_bytes = std::max(sort_tmp, uniq_tmp);
        // one scratch block: every part 256-byte aligned
        size_t at = 0;
        auto take = [&](size_t bytes) { const size_t o = at; at += (bytes + 255) / 256 * 256; return o; };
        const size_t o_beg = take((size_t)n * 4), o_end = take((size_t)n * 4),
                     o_adj = take((size_t)std::max<int64_t>(nnz, 1) * 4), o_off = take(((size_t)n + 1) * 8),
                     o_ka = take((size_t)nk * 8), o_kb = take((size_t)nk * 8), o_sp = take(((size_t)n + 1) * 8),
                     o_sa = take((size_t)nk * 4), o_ord = take((size_t)n * 4), o_pord = take((size_t)n * 4),
                     o_rank = take((size_t)n * 4), o_bykey = take((size_t)n * 4), o_cm = take((size_t)n * 4),
                     o_q = take((size_t)n * 4), o_next = take((size_t)n * 4), o_claim = take((size_t)n * 4),
                     o_gen = take((size_t)n * 4), o_ctr = take(64), o_tmp = take(tmp_bytes);
        char *base = (char *)c->grow(c->order, at);
        int32_t *d_beg = (int32_t *)(base + o_beg), *d_end = (int32_t *)(base + o_end);
        int32_t *d_adj = (int32_t *)(base + o_adj);
        int64_t *d_off = (int64_t *)(base + o_off);
        unsigned long long *ka = (unsigned long long *)(base + o_ka), *kb = (unsigned long long *)(base + o_kb);
        int64_t *d_sp = (int64_t *)(base + o_sp);
        int32_t *d_sa = (int32_t *)(base + o_sa), *d_ord = (int32_t *)(base + o_ord);
        int32_t *d_pord = (int32_t *)(base + o_pord), *d_rank = (int32_t *)(base + o_rank);
        int32_t *d_bykey = (int32_t *)(base + o_bykey), *d_cm = (int32_t *)(base + o_cm);
        int32_t *d_q = (int32_t *)(base + o_q), *d_next = (int32_t *)(base + o_next);
        uint32_t *d_claim = (uint32_t *)(base + o_claim), *d_gen = (uint32_t *)(base + o_gen);
        unsigned long long *d_ctr = (unsigned long long *)(base + o_ctr);   // [0] tail, [1] count
        int32_t *d_small = (int32_t *)(d_ctr + 4);                           // [0] zeros / start / least rank
        void *d_tmp = base + o_tmp;
        const int gridc = c->sm_count * 8;
        auto blocks = [&](int64_t items, int per) {
            return (unsigned)std::max<int64_t>(1, std::min<int64_t>((items + per - 1) / per, gridc));
        };
        auto read_ull = [&](const unsigned long long *d) {
            unsigned long long h = 0;
            GS_CUDA(cudaMemcpyAsync(&h, d, 8, cudaMemcpyDeviceToHost, st));
            GS_CUDA(cudaStreamSynchronize(st));
            return h;
        };
        auto read_i32 = [&](const int32_t *d) {
            int32_t h = 0;
            GS_CUDA(cudaMemcpyAsync(&h, d, 4, cudaMemcpyDeviceToHost, st));
            GS_CUDA(cudaStreamSynchronize(st));
            return h;
        };

        GS_CUDA(cudaMemcpyAsync(d_beg, beg, (size_t)n * 4, cudaMemcpyHostToDevice, st));
        GS_CUDA(cudaMemcpyAsync(d_end, end, (size_t)n * 4, cudaMemcpyHostToDevice, st));
        if (nnz > 0) GS_CUDA(cudaMemcpyAsync(d_adj, adj, (size_t)nnz * 4, cudaMemcpyHostToDevice, st));
        GS_CUDA(cudaMemcpyAsync(d_off, off.data(), ((size_t)n + 1) * 8, cudaMemcpyHostToDevice, st));
        // S = A + A^T: sorted distinct (row, column) keys, the diagonal last
        int64_t count = 0;
        if (total > 0) {
            order_edge_keys_kernel<<<blocks((int64_t)n * 32, 256), 256, 0, st>>>(n, d_beg, d_end, d_adj, d_off, ka);
            GS_CUDA(cudaGetLastError());
            size_t tb = tmp_bytes;
            GS_CUDA(cub::DeviceRadixSort::SortKeys(d_tmp, tb, ka, kb, (int)total, 0, 64, st));
            tb = tmp_bytes;
            GS_CUDA(cub::DeviceSelect::Unique(d_tmp, tb, kb, ka, (int *)(d_ctr + 1), (int)total, st));
            count = (int64_t)(int32_t)(read_ull(d_ctr + 1) & 0xffffffffu);
            if (count > 0 && read_ull(ka + count - 1) == ~0ull) count--;
        }
        order_rows_kernel<<<blocks(count + 1, 256), 256, 0, st>>>(n, ka, count, d_sp, d_sa);
        GS_CUDA(cudaGetLastError());
        // ranks by (degree, id); degree-0 vertices placed first
        order_init_kernel<<<blocks(n, 256), 256, 0, st>>>(n, d_sp, kb, d_ord, d_pord, d_claim, d_gen);
        GS_CUDA(cudaGetLastError());
        {
            size_t tb = tmp_bytes;
            GS_CUDA(cub::DeviceRadixSort::SortKeys(d_tmp, tb, kb, ka, (int)n, 0, 64, st));
        }
        GS_CUDA(cudaMemsetAsync(d_small, 0, 4, st));
        order_ranks_kernel<<<blocks(n, 256), 256, 0, st>>>(n, ka, d_bykey, d_rank, d_ord, d_cm, d_small);
        GS_CUDA(cudaGetLastError());
        std::vector<int32_t> bykey((size_t)n);
        GS_CUDA(cudaMemcpyAsync(bykey.data(), d_bykey, (size_t)n * 4, cudaMemcpyDeviceToHost, st));
        int32_t pos = read_i32(d_small), cursor = pos;
        uint32_t g = 0;

        // breadth-first search from r over the unordered vertices: returns
        // its eccentricity and the vertex of least key in its last level
        auto bfs = [&](int32_t r, int32_t *last_min) -> int32_t {
            ++g;
            GS_CUDA(cudaMemcpyAsync(d_q, &r, 4, cudaMemcpyHostToDevice, st));
            GS_CUDA(cudaMemcpyAsync(d_gen + r, &g, 4, cudaMemcpyHostToDevice, st));
            const unsigned long long one = 1;
            GS_CUDA(cudaMemcpyAsync(d_ctr, &one, 8, cudaMemcpyHostToDevice, st));
            int64_t f0 = 0, f1 = 1;
            int32_t ecc = 0;
            for (;;) {
                order_bfs_kernel<<<blocks((f1 - f0) * 32, 256), 256, 0, st>>>(f0, f1, d_q, d_sp, d_sa, d_ord, d_gen, g,
                                                                           d_ctr);
                GS_CUDA(cudaGetLastError());
                const int64_t t = (int64_t)read_ull(d_ctr);
                if (t == f1) break;
                f0 = f1;
                f1 = t;
                ecc++;
            }
            const int32_t big = INT32_MAX;
            GS_CUDA(cudaMemcpyAsync(d_small, &big, 4, cudaMemcpyHostToDevice, st));
            order_min_rank_kernel<<<blocks(f1 - f0, 256), 256, 0, st>>>(f0, f1, d_q, d_rank, d_small);
            GS_CUDA(cudaGetLastError());
            const int32_t least = read_i32(d_small);
            if (least < 0 || least >= n) throw CudaFail{cudaErrorUnknown};   // cannot happen: the level is not empty
            *last_min = bykey[(size_t)least];
            return ecc;
        };

        while (pos < n) {
            order_find_start_kernel<<<1, 1024, 0, st>>>(n, d_bykey, d_ord, cursor, d_small);
            GS_CUDA(cudaGetLastError());
            cursor = read_i32(d_small);
            if (cursor >= n) throw CudaFail{cudaErrorUnknown};   // cannot happen: pos < n leaves a vertex
            // George-Liu pseudo-peripheral vertex of the component
            int32_t r = bykey[(size_t)cursor], cnd = -1;
            int32_t ecc = bfs(r, &cnd);
            for (;;) {
                int32_t c2 = -1;
                const int32_t ecc_c = bfs(cnd, &c2);
                if (ecc_c <= ecc) break;
                r = cnd;
                ecc = ecc_c;
                cnd = c2;
            }
            // Cuthill-McKee levels from r
            GS_CUDA(cudaMemcpyAsync(d_ord + r, &pos, 4, cudaMemcpyHostToDevice, st));
            GS_CUDA(cudaMemcpyAsync(d_cm + pos, &r, 4, cudaMemcpyHostToDevice, st));
            int32_t l0 = pos, l1 = pos + 1;
            pos++;
            for (;;) {
                GS_CUDA(cudaMemsetAsync(d_ctr, 0, 8, st));
                order_cm_kernel<<<blocks((int64_t)(l1 - l0) * 32, 256), 256, 0, st>>>(l0, l1, d_cm, d_sp, d_sa, d_ord,
                                                                                    d_pord, d_claim, d_next, d_ctr);
                GS_CUDA(cudaGetLastError());
                const int64_t m = (int64_t)read_ull(d_ctr);
                if (m == 0) break;
                if (m > (int64_t)n - pos) throw CudaFail{cudaErrorUnknown};   // cannot happen: each vertex is queued once
                order_level_keys_kernel<<<blocks(m, 256), 256, 0, st>>>(m, d_next, d_pord, d_rank, ka);
                GS_CUDA(cudaGetLastError());
                size_t tb = tmp_bytes;
                GS_CUDA(cub::DeviceRadixSort::SortKeys(d_tmp, tb, ka, kb, (int)m, 0, 64, st));
                order_place_kernel<<<blocks(m, 256), 256, 0, st>>>(m, kb, d_bykey, pos, d_ord, d_cm);
                GS_CUDA(cudaGetLastError());
                l0 = pos;
                pos += (int32_t)m;
                l1 = pos;
            }
        }
        std::vector<int32_t> cm((size_t)n);
        GS_CUDA(cudaMemcpyAsync(cm.data(), d_cm, (size_t)n * 4, cudaMemcpyDeviceToHost, st));
        GS_CUDA(cudaStreamSynchronize(st));
        for (int32_t k = 0; k < n; k++) perm[k] = cm[(size_t)(n - 1 - k)];
    } catch (CudaFail &f) {
        return fail_cuda(f.e);
    } catch (std::bad_alloc &) {
        return GSOFA_ERR_OOM;
    }
    return GSOFA_OK;
}

gsofa_status gsofa_permute_lines(int32_t n, int64_t nnz, const int32_t *beg, const int32_t *end,
                                 const int32_t *adj, const int32_t *perm, int32_t *out_beg, int32_t *out_end,
                                 int32_t *out_adj)
{
    if ((n > 0 && (!perm || !out_beg || !out_end)) || !valid_lines(n, nnz, beg, end, adj))
        return GSOFA_ERR_INVALID_INPUT;
    try {
        std::vector<int32_t> inv((size_t)n, -1);
        for (int32_t k = 0; k < n; k++) {
            if (perm[k] < 0 || perm[k] >= n || inv[(size_t)perm[k]] >= 0) return GSOFA_ERR_INVALID_INPUT;
            inv[(size_t)perm[k]] = k;
        }
        int64_t w = 0;
        for (int32_t k = 0; k < n; k++) {
            const int32_t v = perm[k];
            if (end[v] > beg[v] && !out_adj) return GSOFA_ERR_INVALID_INPUT;
            out_beg[k] = (int32_t)w;
            for (int32_t j = beg[v]; j < end[v]; j++) out_adj[w++] = inv[(size_t)adj[j]];
            std::sort(out_adj + out_beg[k], out_adj + w);
            out_end[k] = (int32_t)w;
        }
    } catch (std::bad_alloc &) {
        return GSOFA_ERR_OOM;
    }
    return GSOFA_OK;
}

int32_t gsofa_supernodes_from_lines(int32_t n, const int32_t *ucnt, const uint8_t *flags,
                                    int32_t max_size, int32_t *sn_start)
{
    if (n < 0 || (n > 0 && (!ucnt || !flags || !sn_start))) return -1;
    int32_t k = 0, run = 0;
    for (int32_t s = 0; s < n; s++) {
        // lines s-1 and s are linked when s-1 is in line s (bit 1 of s-1),
        // s is in line s-1 (bit 0 of s-1) and U row s is U row s-1 minus s
        const bool linked = s > 0 && (flags[s - 1] & 2) && (flags[s - 1] & 1) &&
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

size_t gsofa_predict_scratch_bytes(const gsofa_ctx *c, int32_t n, int64_t nnz,
                                   const gsofa_params *params)
{
    if (!c || n < 0) return 0;
    gsofa_params p;
    resolve_params(params, &p);
    const int block = p.block_size ? p.block_size : pick_block(std::max(n, 1));
    const size_t smem = ((size_t)(n + 31) / 32 * 4 + 15) / 16 * 16;
    int per_sm = p.ctas_per_sm > 0 ? p.ctas_per_sm : std::max(1, (int)(200 * 1024 / std::max<size_t>(smem, 1)));
    per_sm = std::min(per_sm, 2048 / block);
    const size_t grid = (size_t)per_sm * c->sm_count;
    const size_t qcap = (size_t)std::max<int64_t>(p.queue_capacity, n);
    const size_t L = (size_t)n;
    size_t b = grid * qcap * 4;                 // frontier queues
    b += L * (2 * 4 + 2 + 2 * 8 + 4 + 1 + 4);   // cnt, nxt, poff, lrow, snind, sn list
    b += 2 * (L + 1) * 8;                       // gptr
    b += (size_t)(n + 1) * 8 + (size_t)nnz * 8; // G and G^T
    b += (size_t)n * 64;                        // their 32-byte row slots
    if (p.want_pattern)                         // chain stamps, two traversals a CTA
        b += grid * 2 * ((size_t)(n + 4095) / 4096 * 4096) * 2;
    return b;
}

void gsofa_supernodal_free(gsofa_supernodal *s)
{
    if (!s) return;
    std::free(s->xsup);
    std::free(s->supno);
    std::free(s->xlsub);
    std::free(s->lsub);
    std::free(s->xusub);
    std::free(s->usub);
    std::memset(s, 0, sizeof(*s));
}

namespace {

// Arguments of the supernodal kernels for the result r; the head scratch
// (sizes [2][ns] | offsets [2][ns + 1] | supno [n]) is grown to fit.
SupernodalArgs supernodal_args(gsofa_ctx *c, const gsofa_result *r, const ResultInternal *ri)
{
    const int32_t n = (int32_t)ri->n, ns = r->n_supernodes;
    const int64_t L = ri->L, lb = ri->line_base;
    char *head = (char *)c->grow(c->sn_head, (size_t)(4 * (int64_t)ns + 2) * 8 + (size_t)n * 4);
    SupernodalArgs a{};
    a.sn = (const int32_t *)c->snlist.p + ri->sn0;
    a.nsuper = ns;
    a.n = n;
    a.lb = lb;
    a.ucnt = (const int32_t *)c->cnt.p + lb;
    a.lcnt = (const int32_t *)c->cnt.p + L + lb;
    a.uptr = (const int64_t *)c->gptr.p + lb;
    a.lptr = (const int64_t *)c->gptr.p + (L + 1) + lb;
    a.out = ri->pattern == 2 ? ri->pool : (const int32_t *)c->out.p;
    a.u0 = ri->u0;
    a.l0 = ri->l0;
    a.ubeg = ri->pattern == 2 ? (const int64_t *)c->poff.p + lb : nullptr;
    a.lbeg = ri->pattern == 2 ? (const int64_t *)c->poff.p + L + lb : nullptr;
    a.lsize = (int64_t *)head;
    a.usize = a.lsize + ns;
    a.xlsub = a.usize + ns;
    a.xusub = a.xlsub + ns + 1;
    a.supno = (int32_t *)(a.xusub + ns + 1);
    return a;
}

const ResultInternal *supernodal_source(gsofa_ctx *c, const gsofa_result *r)
{
    if (!c || !r) return nullptr;
    const ResultInternal *ri = (const ResultInternal *)r->internal;
    if (!ri || ri->job_id != c->job_id || !ri->pattern) return nullptr;
    if (ri->pattern == 1 ? !c->out.p : !ri->pool) return nullptr;
    const int64_t n = ri->n, ns = r->n_supernodes;
    if (ns < 0 || ns > n || (n > 0 && ns == 0)) return nullptr;
    return ri;
}

}  // namespace

gsofa_status gsofa_result_supernodal_sizes(gsofa_ctx *c, const gsofa_result *r, int32_t *nsuper,
                                           int64_t *nlsub, int64_t *nusub)
{
    const ResultInternal *ri = supernodal_source(c, r);
    if (!ri || !nsuper || !nlsub || !nusub) return GSOFA_ERR_INVALID_INPUT;
    const int32_t ns = r->n_supernodes;
    *nsuper = ns;
    *nlsub = *nusub = 0;
    c->sn_xl.assign((size_t)ns + 1, 0);
    c->sn_xu.assign((size_t)ns + 1, 0);
    c->sn_for = nullptr;
    if (ns == 0) {
        c->sn_for = ri;
        c->sn_job = ri->job_id;
        return GSOFA_OK;
    }
    try {
        GS_CUDA(cudaSetDevice(c->device));
        cudaStream_t st = c->stream;
        SupernodalArgs a = supernodal_args(c, r, ri);
        const int tb = 256;
        const int sgrid = (int)std::min<int64_t>(((int64_t)ns + tb - 1) / tb, (int64_t)c->sm_count * 8);
        supernodal_size_kernel<<<sgrid, tb, 0, st>>>(a);
        GS_CUDA(cudaGetLastError());
        std::vector<int64_t> sz(2 * (size_t)ns);
        GS_CUDA(cudaMemcpyAsync(sz.data(), a.lsize, sz.size() * 8, cudaMemcpyDeviceToHost, st));
        GS_CUDA(cudaStreamSynchronize(st));
        for (int32_t k = 0; k < ns; k++) {
            if (sz[k] < 1 || sz[ns + k] < 0) return GSOFA_ERR_CUDA;   // not a supernode: internal fault
            c->sn_xl[k + 1] = c->sn_xl[k] + sz[k];
            c->sn_xu[k + 1] = c->sn_xu[k] + sz[ns + k];
        }
        GS_CUDA(cudaMemcpyAsync((void *)a.xlsub, c->sn_xl.data(), ((size_t)ns + 1) * 8, cudaMemcpyHostToDevice, st));
        GS_CUDA(cudaMemcpyAsync((void *)a.xusub, c->sn_xu.data(), ((size_t)ns + 1) * 8, cudaMemcpyHostToDevice, st));
        GS_CUDA(cudaStreamSynchronize(st));
    } catch (CudaFail &f) {
        return fail_cuda(f.e);
    }
    *nlsub = c->sn_xl[ns];
    *nusub = c->sn_xu[ns];
    c->sn_for = ri;
    c->sn_job = ri->job_id;
    return GSOFA_OK;
}

gsofa_status gsofa_result_supernodal_fetch(gsofa_ctx *c, const gsofa_result *r, int32_t *xsup,
                                           int32_t *supno, int64_t *xlsub, int32_t *lsub,
                                           int64_t *xusub, int32_t *usub)
{
    const ResultInternal *ri = supernodal_source(c, r);
    if (!ri || c->sn_for != ri || c->sn_job != ri->job_id)   // sizes first, for this result
        return GSOFA_ERR_INVALID_INPUT;
    const int32_t n = (int32_t)ri->n, ns = r->n_supernodes;
    const int64_t lb = ri->line_base;
    if (xlsub) std::memcpy(xlsub, c->sn_xl.data(), ((size_t)ns + 1) * 8);
    if (xusub) std::memcpy(xusub, c->sn_xu.data(), ((size_t)ns + 1) * 8);
    if (ns == 0) {
        if (xsup) xsup[0] = 0;
        return GSOFA_OK;
    }
    try {
        GS_CUDA(cudaSetDevice(c->device));
        cudaStream_t st = c->stream;
        SupernodalArgs a = supernodal_args(c, r, ri);   // same head: sizes and offsets stay
        const int64_t nl = c->sn_xl[ns], nu = c->sn_xu[ns];
        int32_t *data = (int32_t *)c->grow(c->sn_data, (size_t)(nl + nu) * 4);
        a.lsub = data;
        a.usub = data + nl;
        const int tb = 256;
        if (lsub || usub) {
            const int fgrid = (int)std::min<int64_t>(((int64_t)ns * 32 + tb - 1) / tb, (int64_t)c->sm_count * 8);
            supernodal_fill_kernel<<<fgrid, tb, 0, st>>>(a);
            GS_CUDA(cudaGetLastError());
        }
        if (lsub) GS_CUDA(cudaMemcpyAsync(lsub, a.lsub, (size_t)nl * 4, cudaMemcpyDeviceToHost, st));
        if (usub) GS_CUDA(cudaMemcpyAsync(usub, a.usub, (size_t)nu * 4, cudaMemcpyDeviceToHost, st));
        if (supno) GS_CUDA(cudaMemcpyAsync(supno, a.supno, (size_t)n * 4, cudaMemcpyDeviceToHost, st));
        if (xsup) GS_CUDA(cudaMemcpyAsync(xsup, a.sn, (size_t)ns * 4, cudaMemcpyDeviceToHost, st));
        GS_CUDA(cudaStreamSynchronize(st));
        if (xsup) {
            for (int32_t k = 0; k < ns; k++) xsup[k] -= (int32_t)lb;
            xsup[ns] = n;
        }
    } catch (CudaFail &f) {
        return fail_cuda(f.e);
    }
    return GSOFA_OK;
}

gsofa_status gsofa_result_supernodal(gsofa_ctx *c, const gsofa_result *r, gsofa_supernodal *o)
{
    if (!o) return GSOFA_ERR_INVALID_INPUT;
    std::memset(o, 0, sizeof(*o));
    int32_t ns = 0;
    int64_t nl = 0, nu = 0;
    gsofa_status s = gsofa_result_supernodal_sizes(c, r, &ns, &nl, &nu);
    if (s != GSOFA_OK) return s;
    o->n = (int32_t)((const ResultInternal *)r->internal)->n;
    o->nsuper = ns;
    o->nlsub = nl;
    o->nusub = nu;
    o->xsup = (int32_t *)std::malloc(((size_t)ns + 1) * 4);
    o->supno = (int32_t *)std::malloc((size_t)std::max(o->n, 1) * 4);
    o->xlsub = (int64_t *)std::malloc(((size_t)ns + 1) * 8);
    o->xusub = (int64_t *)std::malloc(((size_t)ns + 1) * 8);
    o->lsub = (int32_t *)std::malloc((size_t)std::max<int64_t>(nl, 1) * 4);
    o->usub = (int32_t *)std::malloc((size_t)std::max<int64_t>(nu, 1) * 4);
    if (!o->xsup || !o->supno || !o->xlsub || !o->xusub || !o->lsub || !o->usub) {
        gsofa_supernodal_free(o);
        return GSOFA_ERR_OOM;
    }
    s = gsofa_result_supernodal_fetch(c, r, o->xsup, o->supno, o->xlsub, o->lsub, o->xusub, o->usub);
    if (s != GSOFA_OK) gsofa_supernodal_free(o);
    return s;
}

// ---------------------------------------------------------------------------
// Reference-compatible entry (argv contract of symbfact_min_id).

gsofa_status gsofa_symbfact_min_id(int argc, char **argv, int myrank, uint64_t *fill_count,
                                   double *time_ms)
{
    if (!argv || argc < 5 || argc > 8 || argc == 7) return GSOFA_ERR_INVALID_INPUT;
    const int nparts = std::atoi(argv[4]);
    if (nparts <= 0) return GSOFA_ERR_INVALID_INPUT;
    double mem_gb = argc >= 6 ? std::atof(argv[5]) : 0.0;
    int max_sn = argc >= 8 ? std::atoi(argv[6]) : 0;
    int gpus_per_node = argc >= 8 ? std::atoi(argv[7]) : 1;
    if (gpus_per_node <= 0 || mem_gb < 0) return GSOFA_ERR_INVALID_INPUT;
    int32_t n = 0;
    int64_t nnz = 0;
    int32_t *beg = nullptr, *end = nullptr, *adj = nullptr;
    gsofa_status s = gsofa_read_text(argv[1], argv[2], argv[3], &n, &nnz, &beg, &end, &adj);
    if (s != GSOFA_OK) return s;
    gsofa_ctx *c = nullptr;
    // argv[5] is the device memory pool in GB, as in the reference
    // (with_space_optimization/symbfact.cuh:1683-1686): here the context's
    // budget, which bounds the concurrent traversals (frontier queues) the
    // launch keeps; 0 or absent: 90% of the free memory
    const size_t budget = mem_gb > 0 ? (size_t)(mem_gb * 1073741824.0) : 0;
    s = gsofa_create(&c, myrank % gpus_per_node, budget);
    gsofa_matrix *m = nullptr;
    if (s == GSOFA_OK) s = gsofa_upload(c, n, nnz, beg, end, adj, &m);
    std::free(beg);
    std::free(end);
    std::free(adj);
    uint64_t total = 0;
    double tmax = 0.0, tmin = 1e300, tsum = 0.0;
    for (int g = 0; s == GSOFA_OK && g < nparts; g++) {
        gsofa_params p;
        gsofa_default_params(&p);
        p.want_pattern = 0;
        p.max_supernode_size = max_sn;
        p.part_count = nparts;
        p.part_index = g;
        gsofa_result r;
        s = gsofa_symbfact(c, m, &p, &r);
        if (s == GSOFA_OK) {
            total += r.fill_count;
            tmax = std::max(tmax, r.kernel_ms);
            tmin = std::min(tmin, r.kernel_ms);
            tsum += r.kernel_ms;
            gsofa_result_free(&r);
        }
    }
    if (s == GSOFA_OK) {
        std::printf("Total Number of fill-ins detected: %llu\n", (unsigned long long)total);
        std::printf("\tSlowest virtual GPU takes: %.4f ms\n", tmax);
        std::printf("\tFastest virtual GPU takes: %.4f ms\n", nparts ? tmin : 0.0);
        if (fill_count) *fill_count = total;
        if (time_ms) *time_ms = tsum;
    }
    gsofa_destroy(c);
    return s;
}

}  // extern "C"

// ============================================================================
// Factorization without device allocation (gsofa_symbfact_counts_noalloc).
//
// Every intermediate array of the counts-only factorization sits in one
// file-scope static device array.  Host code cannot use the array's name as a
// device address, so the address is looked up once per device with
// cudaGetSymbolAddress while that device is current.

namespace {

static __device__ __align__(256) unsigned char g_noalloc_scratch[GSOFA_NOALLOC_SCRATCH_BYTES];

constexpr int kNoallocMaxDevices = 64;
std::mutex g_noalloc_mu;
int g_noalloc_sms[kNoallocMaxDevices];     // 0: device not checked yet

// Makes `device` current for the lifetime of the guard and puts the
// caller's current device back on every return path.
struct DeviceGuard {
    int prev = -1;
    cudaError_t err = cudaSuccess;
    explicit DeviceGuard(int device)
    {
        err = cudaGetDevice(&prev);
        if (err == cudaSuccess && prev != device) err = cudaSetDevice(device);
    }
    ~DeviceGuard()
    {
        int cur = -1;
        if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
    }
};

// Carves the static array for an n-line, nnz-entry input: sequential,
// 256-byte aligned slices.
struct NoallocLayout {
    size_t off = 0;
    char *base = nullptr;
    size_t limit = 0;
    bool ok = true;
    template <class T>
    T *take(size_t count)
    {
        off = (off + 255) / 256 * 256;
        T *p = (T *)(base + off);
        off += std::max<size_t>(count, 1) * sizeof(T);
        if (off > limit) ok = false;
        return p;
    }
};

}  // namespace

extern "C" gsofa_status gsofa_symbfact_counts_noalloc(int device, void *cuda_stream, int32_t n,
                                                      int64_t nnz, const int32_t *d_beg,
                                                      const int32_t *d_end, const int32_t *d_adj,
                                                      int32_t max_supernode_size,
                                                      int32_t *d_u_row_count,
                                                      int32_t *d_l_col_count,
                                                      int32_t *d_sn_start, uint64_t *summary)
{
    if (n < 0 || nnz < 0 || !summary) return GSOFA_ERR_INVALID_INPUT;
    if (n > GSOFA_NOALLOC_MAX_N || nnz > GSOFA_NOALLOC_MAX_NNZ) return GSOFA_ERR_UNSUPPORTED;
    if (n > 0 && (!d_beg || !d_end || !d_u_row_count || !d_l_col_count || !d_sn_start))
        return GSOFA_ERR_INVALID_INPUT;
    if (nnz > 0 && !d_adj) return GSOFA_ERR_INVALID_INPUT;
    if (device < 0 || device >= kNoallocMaxDevices) return GSOFA_ERR_INVALID_INPUT;
    summary[0] = summary[1] = summary[2] = 0;
    if (n == 0) return GSOFA_OK;
    DeviceGuard dg(device);   // the caller's current device comes back on return
    if (dg.err != cudaSuccess) return fail_cuda(dg.err);
    try {
        int sms = 0;
        {
            std::lock_guard<std::mutex> lk(g_noalloc_mu);
            if (!g_noalloc_sms[device]) {
                cudaDeviceProp prop;
                GS_CUDA(cudaGetDeviceProperties(&prop, device));
                if (prop.major < 10 || !prop.cooperativeLaunch) return GSOFA_ERR_UNSUPPORTED;
                g_noalloc_sms[device] = prop.multiProcessorCount;
            }
            sms = g_noalloc_sms[device];
        }
        // The array's name is a host-side stand-in; its device address is
        // looked up with this device current, on every call (a cheap lookup
        // once the module is loaded, and never stale after a device reset).
        void *scratch = nullptr;
        GS_CUDA(cudaGetSymbolAddress(&scratch, g_noalloc_scratch));
        cudaStream_t st = (cudaStream_t)cuda_stream;

        // launch shape: 256 threads, one CTA per SM (its queue slice is n ints)
        constexpr int BLOCK = 256;
        void *kfn = factor_kernel_for(BLOCK, false);
        const int32_t bitmap_words = ((n + 31) / 32 + 127) / 128 * 128;
        const int32_t state_words = bitmap_words + bitmap_words / 32 + ((bitmap_words / 32 + 31) / 32 + 3) / 4 * 4;
        const int ring = 4096;
        const size_t smem = (size_t)state_words * 4 + (size_t)ring * 4;
        int occ = 0;
        {
            std::lock_guard<std::mutex> lk(kernel_attr_mutex());
            GS_CUDA(cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            GS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kfn, BLOCK, smem));
        }
        if (occ <= 0) return GSOFA_ERR_UNSUPPORTED;
        const int grid = sms;
        const int64_t L = n;
        const int64_t ntiles = (L + TILE - 1) / TILE;
        const int64_t scan_tiles = ((int64_t)n + 1 + 255) / 256 + 1;

        NoallocLayout lay;
        lay.base = (char *)scratch;
        lay.limit = GSOFA_NOALLOC_SCRATCH_BYTES;
        int32_t *gptr_g = lay.take<int32_t>(n + 1);
        int32_t *gadj = lay.take<int32_t>((size_t)nnz);
        int32_t *tptr = lay.take<int32_t>(n + 1);
        int32_t *tadj = lay.take<int32_t>((size_t)nnz);
        int32_t *deg = lay.take<int32_t>(n + 1);
        int32_t *indeg = lay.take<int32_t>(n + 1);
        int32_t *tcur = lay.take<int32_t>(n + 1);
        int32_t *orig_up = lay.take<int32_t>(n);
        int32_t *orig_lo = lay.take<int32_t>(n);
        int32_t *rawdeg = lay.take<int32_t>(n);
        int4 *gslot = lay.take<int4>((size_t)2 * n);
        int4 *tslot = lay.take<int4>((size_t)2 * n);
        int64_t *tsum = lay.take<int64_t>(2 * scan_tiles);
        unsigned long long *ucounts = lay.take<unsigned long long>(8);
        int32_t *cnt = lay.take<int32_t>(2 * L);
        uint8_t *nxt = lay.take<uint8_t>(2 * L);
        int64_t *gp = lay.take<int64_t>(2 * (L + 1));
        int32_t *lrow = lay.take<int32_t>(L);
        uint8_t *snind = lay.take<uint8_t>(L);
        int64_t *tiles = lay.take<int64_t>(4 * ntiles);
        char *misc = lay.take<char>(256);
        MatDesc *dmat = lay.take<MatDesc>(1);
        Range *drange = lay.take<Range>(1);
        int32_t *queue = lay.take<int32_t>((size_t)grid * n);
        if (!lay.ok) return GSOFA_ERR_UNSUPPORTED;

        // ---- graph build (validation, G without diagonal/duplicates, G^T) ----
        GS_CUDA(cudaMemsetAsync(indeg, 0, (size_t)(n + 1) * 4, st));
        GS_CUDA(cudaMemsetAsync(deg, 0, (size_t)(n + 1) * 4, st));
        GS_CUDA(cudaMemsetAsync(orig_lo, 0, (size_t)n * 4, st));
        GS_CUDA(cudaMemsetAsync(ucounts, 0, 64, st));
        UploadArgs u{};
        u.n = n;
        u.nnz = nnz;
        u.beg = d_beg;
        u.end = d_end;
        u.adj = d_adj;
        u.deg = deg;
        u.indeg = indeg;
        u.orig_up = orig_up;
        u.orig_lo = orig_lo;
        u.rawdeg = rawdeg;
        u.counts = ucounts;
        u.status = (uint32_t *)(ucounts + 4);
        const int ugrid = (int)std::min<int64_t>(((int64_t)n * 32 + 255) / 256, (int64_t)sms * 16);
        upload_count_kernel<<<ugrid, 256, 0, st>>>(u);
        GS_CUDA(cudaGetLastError());
        const int64_t ntl = ((int64_t)n + 255) / 256;
        int32_t *scan_in[2] = {deg, indeg};
        int32_t *scan_out[2] = {gptr_g, tptr};
        for (int k = 0; k < 2; k++) {
            int64_t *ts = tsum + k * scan_tiles;
            int64_t *dt = (int64_t *)(ucounts + 2 + k);
            scan_tiles_kernel<256><<<(unsigned)ntl, 256, 0, st>>>(scan_in[k], n, ts);
            scan_partials_kernel<256><<<1, 256, 0, st>>>(ts, ntl, dt);
            scan_apply_kernel<256><<<(unsigned)ntl, 256, 0, st>>>(scan_in[k], n, ts, scan_out[k], dt);
            GS_CUDA(cudaGetLastError());
        }
        unsigned long long hc[5];
        GS_CUDA(cudaMemcpyAsync(hc, ucounts, sizeof(hc), cudaMemcpyDeviceToHost, st));
        GS_CUDA(cudaStreamSynchronize(st));
        if ((uint32_t)(hc[4] & 0xffffffffu) & 1u) return GSOFA_ERR_INVALID_INPUT;
        if ((int64_t)hc[2] > nnz || (int64_t)hc[3] > nnz) return GSOFA_ERR_INVALID_INPUT;
        GS_CUDA(cudaMemcpyAsync(tcur, tptr, (size_t)(n + 1) * 4, cudaMemcpyDeviceToDevice, st));
        upload_fill_kernel<<<ugrid, 256, 0, st>>>(u, gptr_g, gadj, tcur, tadj);
        slot_fill_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(n, gptr_g, gadj, gslot);
        slot_fill_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(n, tptr, tadj, tslot);
        GS_CUDA(cudaGetLastError());

        // ---- factorization (counts only) ----
        MatDesc md{};
        md.n = n;
        md.line_base = 0;
        md.g[0] = PassGraph{gptr_g, gadj, gslot};
        md.g[1] = PassGraph{tptr, tadj, tslot};
        md.rawdeg = rawdeg;
        Range rg{};
        rg.mat = 0;
        rg.chunk = 32;
        rg.small = 32;
        rg.tail = 0;
        rg.nj = n;
        rg.stride = 1;
        rg.offset = 0;
        rg.piece_base = 0;
        rg.npieces = 2 * (((int64_t)n + 31) / 32);
        GS_CUDA(cudaMemcpyAsync(dmat, &md, sizeof(md), cudaMemcpyHostToDevice, st));
        GS_CUDA(cudaMemcpyAsync(drange, &rg, sizeof(rg), cudaMemcpyHostToDevice, st));
        GS_CUDA(cudaMemsetAsync(misc, 0, 256, st));
        JobArgs a{};
        a.mats = dmat;
        a.nmats = 1;
        a.nranges = 1;
        a.ranges = drange;
        a.npieces = rg.npieces;
        a.piece_counter = (unsigned long long *)misc;
        a.queue = queue;
        a.qcap = n;
        a.bitmap_words = bitmap_words;
        a.state_words = state_words;
        a.ring_size = ring;
        a.lanes = 1;
        a.reuse = 1;
        a.want_pattern = 0;
        a.max_sn = max_supernode_size;
        a.L = L;
        a.cnt = cnt;
        a.nxt = nxt;
        a.poff = nullptr;
        a.pool = nullptr;
        a.pool_cap = 0;
        a.pool_tail = (unsigned long long *)(misc + 8);
        a.gptr = gp;
        a.out = nullptr;
        a.lrow = lrow;
        a.snind = snind;
        a.sn_list = d_sn_start;
        a.ntiles = ntiles;
        a.tile_lo = 0;
        a.tile_hi = ntiles;
        a.tile_sum = tiles;
        a.tile_last = tiles + 2 * ntiles;
        a.tile_sn = tiles + 3 * ntiles;
        a.counters = (unsigned long long *)(misc + 16);
        a.status = (uint32_t *)(misc + 192);
        void *args[] = {&a};
        {
            // the shared-memory attribute is per kernel and process-wide: set
            // it and launch under one lock so no other caller resizes it between
            std::lock_guard<std::mutex> lk(kernel_attr_mutex());
            GS_CUDA(cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            GS_CUDA(cudaLaunchCooperativeKernel(kfn, dim3(grid), dim3(BLOCK), args, smem, st));
        }
        GS_CUDA(cudaMemcpyAsync(d_u_row_count, cnt, (size_t)n * 4, cudaMemcpyDeviceToDevice, st));
        GS_CUDA(cudaMemcpyAsync(d_l_col_count, cnt + L, (size_t)n * 4, cudaMemcpyDeviceToDevice, st));
        unsigned long long hm[25];
        int64_t tot[2];
        GS_CUDA(cudaMemcpyAsync(hm, misc, sizeof(hm), cudaMemcpyDeviceToHost, st));
        GS_CUDA(cudaMemcpyAsync(&tot[0], gp + L, 8, cudaMemcpyDeviceToHost, st));
        GS_CUDA(cudaMemcpyAsync(&tot[1], gp + (L + 1) + L, 8, cudaMemcpyDeviceToHost, st));
        GS_CUDA(cudaStreamSynchronize(st));
        const uint32_t kst = (uint32_t)(hm[24] & 0xffffffffu);
        if (kst & ERR_QUEUE_OVERFLOW) return GSOFA_ERR_QUEUE_OVERFLOW;
        // any other status bit is an internal fault: no result is returned
        if (kst != 0u) return GSOFA_ERR_CUDA;
        summary[0] = (uint64_t)(tot[0] + tot[1]) - hc[0] - hc[1];
        summary[1] = (uint64_t)(tot[0] + tot[1] + n);
        summary[2] = hm[4];
    } catch (CudaFail &f) {
        return fail_cuda(f.e);
    }
    return GSOFA_OK;
}

// ============================================================================
// Serving: persistent kernel fed by the host (gsofa_server_*).

namespace {

// First-fit allocator over [0, size) units, with coalescing frees.
struct RangeAlloc {
    std::map<int64_t, int64_t> free_;   // offset -> length
    void init(int64_t size) { free_.clear(); if (size > 0) free_[0] = size; }
    bool alloc(int64_t len, int64_t *off)
    {
        if (len <= 0) { *off = 0; return true; }
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second >= len) {
                *off = it->first;
                const int64_t rest = it->second - len, at = it->first + len;
                free_.erase(it);
                if (rest > 0) free_[at] = rest;
                return true;
            }
        }
        return false;
    }
    void release(int64_t off, int64_t len)
    {
        if (len <= 0) return;
        auto it = free_.emplace(off, len).first;
        auto nx = std::next(it);
        if (nx != free_.end() && it->first + it->second == nx->first) {
            it->second += nx->second;
            free_.erase(nx);
        }
        if (it != free_.begin()) {
            auto pv = std::prev(it);
            if (pv->first + pv->second == it->first) {
                pv->second += it->second;
                free_.erase(it);
            }
        }
    }
};

constexpr int64_t kArenaUnit = 256;   // bytes
inline int64_t units(int64_t bytes) { return (bytes + kArenaUnit - 1) / kArenaUnit; }

struct ServerReq {
    int slot = -1;
    int32_t n = 0;
    int64_t nnz = 0;
    int64_t lb = 0;                 // first line in the line arena
    int64_t g_off = 0, g_units = 0; // graph region in the arena
    uint64_t npieces = 0;
    uint64_t orig_up = 0, orig_lo = 0;
    int cls = 0;                    // priority class (ring) of its pieces
    bool done = false;
};

constexpr int32_t kSmallRequest = 65536;   // lines below which a request is class 0
// Threads of a serving CTA (12 warps per pass).  With the kernel's 64
// registers a thread, 768 threads leave 16K registers and 1280 thread slots
// per SM: two 256-thread upload blocks still run beside the persistent kernel.
constexpr int kServeBlock = 768;
// Global-state form: 256-thread CTAs, three per SM (768 threads, 48K of the
// 64K registers), six traversals per SM.
constexpr int kServeBlockG = 256;
constexpr int kServeCtasG = 3;

}  // namespace

struct gsofa_server {
    int device = 0, sms = 0;
    size_t optin = 0;
    int32_t max_n = 0;
    int32_t max_sn = 0;
    int32_t chunk = 0;              // sources per piece; 0: from the request's n
    int32_t max_slots = 4096;
    int idle_spins = 10000;
    int block = kServeBlock, ring = 1024, grid = 0;
    bool gbm = false;               // bitmaps in global memory (d_gstate)
    uint32_t *d_gstate = nullptr;
    int32_t bitmap_words = 0, state_words = 0;
    size_t smem = 0;
    cudaStream_t run = nullptr, io = nullptr;
    ServeCtl *d_ctl = nullptr;
    ServePiece *d_pieces = nullptr;
    unsigned long long piece_cap = 1ull << 20;
    MatDesc *d_slots = nullptr;
    unsigned int *d_done = nullptr;
    int32_t *d_cnt = nullptr;
    uint8_t *d_nxt = nullptr;
    int64_t lmax = 0;
    int32_t *d_queue = nullptr;
    uint32_t *d_status = nullptr;
    char *d_arena = nullptr;
    int64_t arena_units = 0;
    RangeAlloc arena, lines;
    std::vector<int> free_slots;
    std::unordered_map<int64_t, ServerReq> reqs;
    std::vector<unsigned int> h_done;
    int64_t next_id = 1;
    unsigned long long published[kServeClasses] = {0, 0};
    unsigned long long taken_seen[kServeClasses] = {0, 0};
};

namespace {

// Bytes of a request's resident graph: G and G^T offsets and ids, per-line
// originals and input degrees.
int64_t server_graph_bytes(int32_t n, int64_t nnz)
{
    const int64_t a = 256;
    auto r = [&](int64_t b) { return (b + a - 1) / a * a; };
    return 2 * r(4 * ((int64_t)n + 1)) + 2 * r(4 * std::max<int64_t>(nnz, 1)) + 3 * r(4 * std::max<int32_t>(n, 1)) +
           2 * r(32 * std::max<int32_t>(n, 1));
}

// Upload staging: input copy, degree arrays, scan partials, counters.
int64_t server_staging_bytes(int32_t n, int64_t nnz)
{
    const int64_t a = 256;
    auto r = [&](int64_t b) { return (b + a - 1) / a * a; };
    const int64_t scan_tiles = ((int64_t)n + 1 + 255) / 256 + 1;
    return 2 * r(4 * std::max<int32_t>(n, 1)) + r(4 * std::max<int64_t>(nnz, 1)) + 3 * r(4 * ((int64_t)n + 1)) +
           r(8 * 2 * scan_tiles) + r(64);
}

// Stops the running launch (its CTAs are idle or finish what they hold) and
// clears the flag so the next launch runs.
void server_stop_kernel(gsofa_server *s)
{
    const int32_t one = 1, zero = 0;
    GS_CUDA(cudaMemcpyAsync(&s->d_ctl->stop, &one, 4, cudaMemcpyHostToDevice, s->io));
    GS_CUDA(cudaStreamSynchronize(s->io));
    GS_CUDA(cudaStreamSynchronize(s->run));
    GS_CUDA(cudaMemcpyAsync(&s->d_ctl->stop, &zero, 4, cudaMemcpyHostToDevice, s->io));
    GS_CUDA(cudaStreamSynchronize(s->io));
}

gsofa_status server_launch_if_idle_impl(gsofa_server *s);

gsofa_status server_launch_if_idle(gsofa_server *s)
{
    try {
        return server_launch_if_idle_impl(s);
    } catch (CudaFail &f) {
        return fail_cuda(f.e);
    }
}

gsofa_status server_launch_if_idle_impl(gsofa_server *s)
{
    cudaError_t q = cudaStreamQuery(s->run);
    if (q == cudaErrorNotReady) {
        // a launch is running: keep it unless some of its CTAs have left
        // (their safety timeout); then let it finish and start a full one
        int32_t exited = 0;
        GS_CUDA(cudaMemcpyAsync(&exited, &s->d_ctl->exited, 4, cudaMemcpyDeviceToHost, s->io));
        GS_CUDA(cudaStreamSynchronize(s->io));
        if (exited == 0) return GSOFA_OK;
        server_stop_kernel(s);
        q = cudaSuccess;
    }
    if (q != cudaSuccess) return fail_cuda(q);
    GS_CUDA(cudaMemsetAsync(&s->d_ctl->exited, 0, 4, s->io));
    GS_CUDA(cudaStreamSynchronize(s->io));
    ServeArgs sa{};
    JobArgs &a = sa.job;
    a.queue = s->d_queue;
    a.qcap = s->max_n;
    a.bitmap_words = s->bitmap_words;
    a.state_words = s->state_words;
    a.ring_size = s->ring;
    a.gbm = s->d_gstate;
    a.lanes = 1;
    a.reuse = 1;
    a.want_pattern = 0;
    a.L = s->lmax;
    a.cnt = s->d_cnt;
    a.nxt = s->d_nxt;
    a.status = s->d_status;
    sa.ctl = s->d_ctl;
    sa.pieces = s->d_pieces;
    sa.piece_cap = s->piece_cap;
    sa.slots = s->d_slots;
    sa.slot_done = s->d_done;
    sa.idle_spins = s->idle_spins;
    if (s->gbm) serve_kernel<kServeBlockG, true><<<s->grid, kServeBlockG, s->smem, s->run>>>(sa);
    else serve_kernel<kServeBlock, false><<<s->grid, kServeBlock, s->smem, s->run>>>(sa);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? GSOFA_OK : fail_cuda(e);
}

void server_release(gsofa_server *s, ServerReq &r)
{
    if (r.slot >= 0) s->free_slots.push_back(r.slot);
    s->lines.release(r.lb, r.n);
    s->arena.release(r.g_off, r.g_units);
    r.slot = -1;
}

}  // namespace

extern "C" {

gsofa_status gsofa_server_create(gsofa_server **out, gsofa_server_config *cfg)
{
    if (!out || !cfg) return GSOFA_ERR_INVALID_INPUT;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) {
        cudaGetLastError();
        return GSOFA_ERR_UNSUPPORTED;
    }
    if (cfg->device < 0 || cfg->device >= ndev) return GSOFA_ERR_INVALID_INPUT;
    gsofa_server *s = new (std::nothrow) gsofa_server();
    if (!s) return GSOFA_ERR_OOM;
    try {
        s->device = cfg->device;
        GS_CUDA(cudaSetDevice(s->device));
        cudaDeviceProp prop;
        GS_CUDA(cudaGetDeviceProperties(&prop, s->device));
        if (prop.major < 10) { delete s; return GSOFA_ERR_UNSUPPORTED; }
        s->sms = prop.multiProcessorCount;
        s->optin = prop.sharedMemPerBlockOptin;
        // Shared memory left free on each SM so the upload kernels (and the
        // runtime's memset kernels) of new requests run beside the serving
        // kernel instead of waiting for it to exit.
        const size_t reserve = 12 * 1024;
        const size_t static_smem = 2 * sizeof(SharedState) + 1024 + reserve;
        if ((cfg->flags & GSOFA_FLAG_GLOBAL_STATE) && (cfg->flags & GSOFA_FLAG_SHARED_STATE)) {
            delete s;
            return GSOFA_ERR_INVALID_INPUT;
        }
        // the global-state form unless shared memory is asked for
        s->gbm = !(cfg->flags & GSOFA_FLAG_SHARED_STATE);
        s->block = s->gbm ? kServeBlockG : kServeBlock;
        const int64_t per_half_words = ((int64_t)(s->optin - static_smem) / 2 - 1024 * 4) / 4;
        const int32_t limit_n =
            s->gbm ? (int32_t)(1 << 26)
                   : (int32_t)std::min<int64_t>((per_half_words - 64) * 32 / 33 / 128 * 128 * 32, INT32_MAX);
        s->max_n = cfg->max_n > 0 ? cfg->max_n : (s->gbm ? (1 << 20) : limit_n);
        if (s->max_n > limit_n || s->max_n <= 0) { delete s; return GSOFA_ERR_UNSUPPORTED; }
        s->max_sn = cfg->max_supernode_size;
        s->chunk = cfg->src_chunk > 0 ? cfg->src_chunk : 0;
        s->max_slots = cfg->max_requests > 0 ? cfg->max_requests : 4096;
        s->idle_spins = std::max(1, (cfg->idle_exit_us > 0 ? cfg->idle_exit_us : 30000000) / 2);
        s->bitmap_words = ((s->max_n + 31) / 32 + 127) / 128 * 128;
        s->state_words = s->bitmap_words + s->bitmap_words / 32 + ((s->bitmap_words / 32 + 31) / 32 + 3) / 4 * 4;
        // frontier ring: the largest that fits beside the two bitmaps (shared
        // state), or beside two more CTAs' rings (global state)
        void *kfn = s->gbm ? (void *)serve_kernel<kServeBlockG, true> : (void *)serve_kernel<kServeBlock, false>;
        const int per_sm = s->gbm ? kServeCtasG : 1;
        const size_t smem_state = s->gbm ? 0 : (size_t)s->state_words * 4;
        s->ring = 0;
        for (int cand = 8192; cand >= 1024; cand >>= 1) {
            const size_t sm = 2 * (smem_state + (size_t)cand * 4);
            if ((sm + static_smem - reserve) * per_sm + reserve <= (size_t)prop.sharedMemPerMultiprocessor &&
                sm + static_smem <= s->optin) {
                s->ring = cand;
                s->smem = sm;
                break;
            }
        }
        if (!s->ring) { delete s; return GSOFA_ERR_UNSUPPORTED; }
        int occ = 0;
        {
            std::lock_guard<std::mutex> lk(kernel_attr_mutex());
            GS_CUDA(cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)s->smem));
            GS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kfn, s->block, s->smem));
        }
        if (occ < per_sm) { delete s; return GSOFA_ERR_UNSUPPORTED; }
        // a fixed number of CTAs per SM leaves room for the upload kernels
        s->grid = s->sms * per_sm;
        GS_CUDA(cudaStreamCreateWithFlags(&s->run, cudaStreamNonBlocking));
        GS_CUDA(cudaStreamCreateWithFlags(&s->io, cudaStreamNonBlocking));
        size_t fr = 0, tot = 0;
        GS_CUDA(cudaMemGetInfo(&fr, &tot));
        const int64_t budget = cfg->mem_budget_bytes > 0 ? cfg->mem_budget_bytes : (int64_t)(0.9 * (double)fr);
        s->lmax = std::max<int64_t>(4 * (int64_t)s->max_n, 1 << 24);
        const int64_t gstate_bytes = s->gbm ? (int64_t)s->grid * 2 * s->state_words * 4 : 0;
        const int64_t fixed = (int64_t)s->grid * 2 * s->max_n * 4 + gstate_bytes +
                              (int64_t)kServeClasses * s->piece_cap * sizeof(ServePiece) +
                              (int64_t)s->max_slots * (sizeof(MatDesc) + 4) + s->lmax * 10 + 4096;
        s->arena_units = (budget - fixed) / kArenaUnit;
        if (s->arena_units < units(server_graph_bytes(s->max_n, 8 * (int64_t)s->max_n))) {
            gsofa_server_destroy(s);
            return GSOFA_ERR_OOM;
        }
        GS_CUDA(cudaMalloc(&s->d_ctl, sizeof(ServeCtl) + 64));
        s->d_status = (uint32_t *)((char *)s->d_ctl + sizeof(ServeCtl));
        GS_CUDA(cudaMalloc(&s->d_pieces, kServeClasses * s->piece_cap * sizeof(ServePiece)));
        GS_CUDA(cudaMalloc(&s->d_slots, (size_t)s->max_slots * sizeof(MatDesc)));
        GS_CUDA(cudaMalloc(&s->d_done, (size_t)s->max_slots * 4));
        GS_CUDA(cudaMalloc(&s->d_cnt, (size_t)2 * s->lmax * 4));
        GS_CUDA(cudaMalloc(&s->d_nxt, (size_t)2 * s->lmax));
        GS_CUDA(cudaMalloc(&s->d_queue, (size_t)s->grid * 2 * s->max_n * 4));
        if (s->gbm) GS_CUDA(cudaMalloc(&s->d_gstate, (size_t)gstate_bytes));
        GS_CUDA(cudaMalloc(&s->d_arena, (size_t)s->arena_units * kArenaUnit));
        GS_CUDA(cudaMemsetAsync(s->d_ctl, 0, sizeof(ServeCtl) + 64, s->io));
        GS_CUDA(cudaMemsetAsync(s->d_done, 0, (size_t)s->max_slots * 4, s->io));
        GS_CUDA(cudaStreamSynchronize(s->io));
        s->arena.init(s->arena_units);
        s->lines.init(s->lmax);
        for (int i = s->max_slots - 1; i >= 0; i--) s->free_slots.push_back(i);
        s->h_done.assign((size_t)s->max_slots, 0u);
    } catch (CudaFail &f) {
        gsofa_server_destroy(s);
        return fail_cuda(f.e);
    }
    cfg->max_n_out = s->max_n;
    *out = s;
    return GSOFA_OK;
}

gsofa_status gsofa_server_drain(gsofa_server *s)
{
    if (!s) return GSOFA_ERR_INVALID_INPUT;
    try {
        GS_CUDA(cudaSetDevice(s->device));
        // every published piece is taken before CTAs go idle, so setting
        // `stop` lets the kernel finish its work and then exit
        const int32_t one = 1, zero = 0;
        GS_CUDA(cudaMemcpyAsync(&s->d_ctl->stop, &one, 4, cudaMemcpyHostToDevice, s->io));
        GS_CUDA(cudaStreamSynchronize(s->io));
        GS_CUDA(cudaStreamSynchronize(s->run));
        GS_CUDA(cudaMemcpyAsync(&s->d_ctl->stop, &zero, 4, cudaMemcpyHostToDevice, s->io));
        GS_CUDA(cudaStreamSynchronize(s->io));
    } catch (CudaFail &f) {
        return fail_cuda(f.e);
    }
    return GSOFA_OK;
}

void gsofa_server_destroy(gsofa_server *s)
{
    if (!s) return;
    cudaSetDevice(s->device);
    if (s->d_ctl && s->io) {
        const int32_t one = 1;
        cudaMemcpyAsync(&s->d_ctl->stop, &one, 4, cudaMemcpyHostToDevice, s->io);
        cudaStreamSynchronize(s->io);
    }
    if (s->run) cudaStreamSynchronize(s->run);   // idle CTAs see `stop` and exit
    cudaFree(s->d_ctl);
    cudaFree(s->d_pieces);
    cudaFree(s->d_slots);
    cudaFree(s->d_done);
    cudaFree(s->d_cnt);
    cudaFree(s->d_nxt);
    cudaFree(s->d_queue);
    cudaFree(s->d_gstate);
    cudaFree(s->d_arena);
    if (s->run) cudaStreamDestroy(s->run);
    if (s->io) cudaStreamDestroy(s->io);
    delete s;
}

size_t gsofa_server_request_bytes(const gsofa_server *s, int32_t n, int64_t nnz)
{
    if (!s || n < 0 || nnz < 0) return 0;
    return (size_t)(server_graph_bytes(n, nnz) + server_staging_bytes(n, nnz) + 10 * (int64_t)n);
}

gsofa_status gsofa_server_submit(gsofa_server *s, int32_t n, int64_t nnz, const int32_t *beg,
                                 const int32_t *end, const int32_t *adj, int64_t *id)
{
    if (!s || !id || n <= 0 || nnz < 0 || nnz > INT32_MAX || !beg || !end || (nnz > 0 && !adj))
        return GSOFA_ERR_INVALID_INPUT;
    if (n > s->max_n) return GSOFA_ERR_UNSUPPORTED;
    ServerReq r;
    r.n = n;
    r.nnz = nnz;
    // long pieces for long requests (a piece's first source cannot reuse
    // state), while keeping about eight pieces per resident CTA
    const int32_t chunk = s->chunk > 0 ? s->chunk
                                       : (int32_t)std::min<int64_t>(
                                             512, std::max<int64_t>(32, (int64_t)n / (8 * std::max(s->grid, 1))));
    const uint64_t npieces = ((uint64_t)n + chunk - 1) / chunk;
    const int cls = n < kSmallRequest ? 0 : 1;
    r.cls = cls;
    if (s->free_slots.empty()) return GSOFA_ERR_BUSY;
    if (s->published[cls] + npieces - s->taken_seen[cls] > s->piece_cap) return GSOFA_ERR_BUSY;
    int64_t st_off = 0;
    const int64_t st_units = units(server_staging_bytes(n, nnz));
    r.g_units = units(server_graph_bytes(n, nnz));
    if (!s->lines.alloc(n, &r.lb)) return GSOFA_ERR_BUSY;
    if (!s->arena.alloc(r.g_units, &r.g_off)) {
        s->lines.release(r.lb, n);
        return GSOFA_ERR_BUSY;
    }
    if (!s->arena.alloc(st_units, &st_off)) {
        s->lines.release(r.lb, n);
        s->arena.release(r.g_off, r.g_units);
        return GSOFA_ERR_BUSY;
    }
    r.slot = s->free_slots.back();
    s->free_slots.pop_back();
    gsofa_status status = GSOFA_OK;
    try {
        GS_CUDA(cudaSetDevice(s->device));
        cudaStream_t st = s->io;
        // carve the graph region and the staging region
        char *gb = s->d_arena + r.g_off * kArenaUnit;
        char *sb = s->d_arena + st_off * kArenaUnit;
        auto take = [](char *&p, int64_t bytes) {
            char *q = p;
            p += (bytes + 255) / 256 * 256;
            return q;
        };
        int32_t *gptr = (int32_t *)take(gb, 4 * ((int64_t)n + 1));
        int32_t *tptr = (int32_t *)take(gb, 4 * ((int64_t)n + 1));
        int32_t *gadj = (int32_t *)take(gb, 4 * std::max<int64_t>(nnz, 1));
        int32_t *tadj = (int32_t *)take(gb, 4 * std::max<int64_t>(nnz, 1));
        int32_t *orig_up = (int32_t *)take(gb, 4 * (int64_t)n);
        int32_t *orig_lo = (int32_t *)take(gb, 4 * (int64_t)n);
        int32_t *rawdeg = (int32_t *)take(gb, 4 * (int64_t)n);
        int4 *gslot = (int4 *)take(gb, 32 * (int64_t)n);
        int4 *tslot = (int4 *)take(gb, 32 * (int64_t)n);
        const int64_t scan_tiles = ((int64_t)n + 1 + 255) / 256 + 1;
        int32_t *d_beg = (int32_t *)take(sb, 4 * (int64_t)n);
        int32_t *d_end = (int32_t *)take(sb, 4 * (int64_t)n);
        int32_t *d_adj = (int32_t *)take(sb, 4 * std::max<int64_t>(nnz, 1));
        int32_t *deg = (int32_t *)take(sb, 4 * ((int64_t)n + 1));
        int32_t *indeg = (int32_t *)take(sb, 4 * ((int64_t)n + 1));
        int32_t *tcur = (int32_t *)take(sb, 4 * ((int64_t)n + 1));
        int64_t *tsum = (int64_t *)take(sb, 8 * 2 * scan_tiles);
        unsigned long long *cnts = (unsigned long long *)take(sb, 64);

        GS_CUDA(cudaMemcpyAsync(d_beg, beg, (size_t)n * 4, cudaMemcpyHostToDevice, st));
        GS_CUDA(cudaMemcpyAsync(d_end, end, (size_t)n * 4, cudaMemcpyHostToDevice, st));
        if (nnz > 0) GS_CUDA(cudaMemcpyAsync(d_adj, adj, (size_t)nnz * 4, cudaMemcpyHostToDevice, st));
        GS_CUDA(cudaMemsetAsync(indeg, 0, (size_t)(n + 1) * 4, st));
        GS_CUDA(cudaMemsetAsync(deg, 0, (size_t)(n + 1) * 4, st));
        GS_CUDA(cudaMemsetAsync(orig_lo, 0, (size_t)n * 4, st));
        GS_CUDA(cudaMemsetAsync(cnts, 0, 64, st));
        UploadArgs u{};
        u.n = n;
        u.nnz = nnz;
        u.beg = d_beg;
        u.end = d_end;
        u.adj = d_adj;
        u.deg = deg;
        u.indeg = indeg;
        u.orig_up = orig_up;
        u.orig_lo = orig_lo;
        u.rawdeg = rawdeg;
        u.counts = cnts;
        u.status = (uint32_t *)(cnts + 4);
        const int ugrid = (int)std::min<int64_t>(((int64_t)n * 32 + 255) / 256, (int64_t)s->sms * 16);
        upload_count_kernel<<<ugrid, 256, 0, st>>>(u);
        GS_CUDA(cudaGetLastError());
        const int64_t ntl = ((int64_t)n + 255) / 256;
        int32_t *scan_in[2] = {deg, indeg};
        int32_t *scan_out[2] = {gptr, tptr};
        for (int k = 0; k < 2; k++) {
            int64_t *ts = tsum + k * scan_tiles;
            int64_t *dt = (int64_t *)(cnts + 2 + k);
            scan_tiles_kernel<256><<<(unsigned)ntl, 256, 0, st>>>(scan_in[k], n, ts);
            scan_partials_kernel<256><<<1, 256, 0, st>>>(ts, ntl, dt);
            scan_apply_kernel<256><<<(unsigned)ntl, 256, 0, st>>>(scan_in[k], n, ts, scan_out[k], dt);
            GS_CUDA(cudaGetLastError());
        }
        unsigned long long hc[5];
        GS_CUDA(cudaMemcpyAsync(hc, cnts, sizeof(hc), cudaMemcpyDeviceToHost, st));
        GS_CUDA(cudaStreamSynchronize(st));
        if ((uint32_t)(hc[4] & 0xffffffffu) & 1u) throw std::invalid_argument("input");
        r.orig_up = hc[0];
        r.orig_lo = hc[1];
        GS_CUDA(cudaMemcpyAsync(tcur, tptr, (size_t)(n + 1) * 4, cudaMemcpyDeviceToDevice, st));
        upload_fill_kernel<<<ugrid, 256, 0, st>>>(u, gptr, gadj, tcur, tadj);
        {
            const int sgrid = (int)std::min<int64_t>(((int64_t)n + 255) / 256, (int64_t)s->sms * 8);
            slot_fill_kernel<<<sgrid, 256, 0, st>>>(n, gptr, gadj, gslot);
            slot_fill_kernel<<<sgrid, 256, 0, st>>>(n, tptr, tadj, tslot);
        }
        GS_CUDA(cudaGetLastError());

        // publish: descriptor, cleared counter, pieces, then the new total
        MatDesc md{};
        md.n = n;
        md.line_base = r.lb;
        md.g[0] = PassGraph{gptr, gadj, gslot};
        md.g[1] = PassGraph{tptr, tadj, tslot};
        md.rawdeg = rawdeg;
        GS_CUDA(cudaMemcpyAsync(s->d_slots + r.slot, &md, sizeof(md), cudaMemcpyHostToDevice, st));
        GS_CUDA(cudaMemsetAsync(s->d_done + r.slot, 0, 4, st));
        std::vector<ServePiece> pcs((size_t)npieces);
        for (uint64_t k = 0; k < npieces; k++) {
            // highest sources first: they carry the largest traversals
            const int64_t hi = (int64_t)n - (int64_t)k * chunk;
            pcs[k] = ServePiece{r.slot, (int32_t)std::max<int64_t>(0, hi - chunk), (int32_t)hi, 0};
        }
        ServePiece *ring = s->d_pieces + (size_t)cls * s->piece_cap;
        const uint64_t at = s->published[cls] % s->piece_cap;
        const uint64_t first = std::min<uint64_t>(npieces, s->piece_cap - at);
        GS_CUDA(cudaMemcpyAsync(ring + at, pcs.data(), first * sizeof(ServePiece), cudaMemcpyHostToDevice, st));
        if (first < npieces)
            GS_CUDA(cudaMemcpyAsync(ring, pcs.data() + first, (npieces - first) * sizeof(ServePiece),
                                    cudaMemcpyHostToDevice, st));
        const unsigned long long newpub = s->published[cls] + npieces;
        GS_CUDA(cudaMemcpyAsync(&s->d_ctl->published[cls], &newpub, 8, cudaMemcpyHostToDevice, st));
        GS_CUDA(cudaStreamSynchronize(st));
        s->published[cls] = newpub;
        r.npieces = npieces;
        s->h_done[(size_t)r.slot] = 0;
    } catch (CudaFail &f) {
        status = fail_cuda(f.e);
    } catch (std::invalid_argument &) {
        status = GSOFA_ERR_INVALID_INPUT;
    }
    s->arena.release(st_off, st_units);
    if (status != GSOFA_OK) {
        server_release(s, r);
        return status;
    }
    const int64_t rid = s->next_id++;
    s->reqs.emplace(rid, r);
    *id = rid;
    return server_launch_if_idle(s);
}

gsofa_status gsofa_server_poll(gsofa_server *s, int64_t *ids, int32_t capacity, int32_t *count)
{
    if (!s || !count || (capacity > 0 && !ids)) return GSOFA_ERR_INVALID_INPUT;
    *count = 0;
    try {
        GS_CUDA(cudaSetDevice(s->device));
        unsigned long long tk[kServeClasses] = {0, 0};
        GS_CUDA(cudaMemcpyAsync(s->h_done.data(), s->d_done, s->h_done.size() * 4, cudaMemcpyDeviceToHost, s->io));
        GS_CUDA(cudaMemcpyAsync(tk, s->d_ctl->taken, sizeof(tk), cudaMemcpyDeviceToHost, s->io));
        GS_CUDA(cudaStreamSynchronize(s->io));
        for (int c = 0; c < kServeClasses; c++) s->taken_seen[c] = tk[c];
        bool pending = false;
        for (auto &kv : s->reqs) {
            ServerReq &r = kv.second;
            if (r.done) continue;
            if (r.slot >= 0 && s->h_done[(size_t)r.slot] >= r.npieces) {
                r.done = true;
                if (*count < capacity) ids[(*count)++] = kv.first;
            } else {
                pending = true;
            }
        }
        if (pending) return server_launch_if_idle(s);
        // nothing in flight: stop the launch so it restarts with every CTA
        if (cudaStreamQuery(s->run) == cudaErrorNotReady) server_stop_kernel(s);
    } catch (CudaFail &f) {
        return fail_cuda(f.e);
    }
    return GSOFA_OK;
}

gsofa_status gsofa_server_result(gsofa_server *s, int64_t id, gsofa_result *out)
{
    if (!s || !out) return GSOFA_ERR_INVALID_INPUT;
    auto it = s->reqs.find(id);
    if (it == s->reqs.end() || !it->second.done) return GSOFA_ERR_INVALID_INPUT;
    ServerReq &r = it->second;
    std::memset(out, 0, sizeof(*out));
    const int64_t n = r.n;
    try {
        GS_CUDA(cudaSetDevice(s->device));
        out->n = r.n;
        out->u_row_count = (int32_t *)std::malloc((size_t)n * 4);
        out->l_col_count = (int32_t *)std::malloc((size_t)n * 4);
        out->line_flags = (uint8_t *)std::malloc((size_t)n);
        std::vector<uint8_t> lf((size_t)n);
        if (!out->u_row_count || !out->l_col_count || !out->line_flags) throw std::bad_alloc();
        GS_CUDA(cudaMemcpyAsync(out->u_row_count, s->d_cnt + r.lb, n * 4, cudaMemcpyDeviceToHost, s->io));
        GS_CUDA(cudaMemcpyAsync(out->l_col_count, s->d_cnt + s->lmax + r.lb, n * 4, cudaMemcpyDeviceToHost, s->io));
        GS_CUDA(cudaMemcpyAsync(out->line_flags, s->d_nxt + r.lb, n, cudaMemcpyDeviceToHost, s->io));
        GS_CUDA(cudaMemcpyAsync(lf.data(), s->d_nxt + s->lmax + r.lb, n, cudaMemcpyDeviceToHost, s->io));
        GS_CUDA(cudaStreamSynchronize(s->io));
        uint64_t su = 0, sl = 0;
        for (int64_t q = 0; q < n; q++) {
            su += (uint64_t)out->u_row_count[q];
            sl += (uint64_t)out->l_col_count[q];
            out->line_flags[q] = (uint8_t)(out->line_flags[q] | (lf[(size_t)q] << 1));
        }
        out->nnz_u = su;
        out->nnz_l = sl;
        out->nnz_lu = su + sl + (uint64_t)n;
        out->fill_count = su + sl - r.orig_up - r.orig_lo;
        std::vector<int32_t> sn((size_t)std::max<int64_t>(n, 1));
        const int32_t k = gsofa_supernodes_from_lines(r.n, out->u_row_count, out->line_flags, s->max_sn, sn.data());
        out->n_supernodes = k;
        out->sn_start = (int32_t *)std::malloc((size_t)std::max(k, 1) * 4);
        if (!out->sn_start) throw std::bad_alloc();
        std::memcpy(out->sn_start, sn.data(), (size_t)k * 4);
        out->sources = 2 * (uint64_t)n;
    } catch (CudaFail &f) {
        free_result_arrays(out);
        return fail_cuda(f.e);
    } catch (std::bad_alloc &) {
        free_result_arrays(out);
        return GSOFA_ERR_OOM;
    }
    server_release(s, r);
    s->reqs.erase(it);
    return GSOFA_OK;
}

}  // extern "C"

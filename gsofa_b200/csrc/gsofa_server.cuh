// gsofa_server.cuh -- persistent serving kernel (continuous batching).
//
// One long-running launch takes work pieces -- (request slot, source range) --
// from a ring in device memory that the host extends while the kernel runs:
// the host writes a request's matrix descriptor and pieces, then raises
// `published`; CTAs claim pieces one at a time with a compare-and-swap on
// `taken`, so requests that arrive while others are being factorized start
// on the next free CTA.  Each finished piece bumps its slot's counter; the
// host polls the counters and finishes a request (totals, supernodes) from
// its per-line arrays.  Idle CTAs wait with a bounded number of sleeps and
// then exit; the host relaunches the kernel when work is pending.
//
// The host reuses device memory of finished requests for new ones while the
// kernel keeps running, so every load of request data goes through L2 only
// (ld.global.cg): no CTA can see a stale L1 copy of a recycled region.
#pragma once

#include "gsofa_device.cuh"

namespace gsofa {
namespace dev {

struct ServePiece {          // sources [s_lo, s_hi) of request slot `slot`
    int32_t slot, s_lo, s_hi, pad;
};

// Two rings: class 0 holds the pieces of small requests and is always served
// first, so they are not queued behind the pieces of a large one.
constexpr int kServeClasses = 2;

struct ServeCtl {            // device memory shared by host and kernel
    unsigned long long published[kServeClasses];  // pieces the kernel may take (host)
    unsigned long long taken[kServeClasses];      // pieces claimed so far (kernel)
    int32_t stop;                  // host: exit as soon as idle
    int32_t exited;                // CTAs of the current launch that have left
    unsigned long long pad[2];
};

struct ServeArgs {
    JobArgs job;                   // per-line arrays, queues, launch shape
    ServeCtl *ctl;
    const ServePiece *pieces;      // kServeClasses rings of piece_cap entries
    unsigned long long piece_cap;
    const MatDesc *slots;          // matrix descriptor of every request slot
    unsigned int *slot_done;       // finished pieces per slot
    int idle_spins;                // sleeps of ~2 us before an idle CTA gives up
                                   // (a safety bound: the host stops the kernel
                                   // itself when nothing is in flight)
};

// Copies a POD through L2-only 8-byte loads.
template <class T>
__device__ __forceinline__ T load_cg(const T *p)
{
    static_assert(sizeof(T) % 8 == 0, "8-byte multiple");
    T out;
    const unsigned long long *src = reinterpret_cast<const unsigned long long *>(p);
    unsigned long long *dst = reinterpret_cast<unsigned long long *>(&out);
#pragma unroll
    for (int i = 0; i < (int)(sizeof(T) / 8); i++) dst[i] = __ldcg(src + i);
    return out;
}

// At most 64 registers a thread, so the upload kernels, which must run beside
// this kernel while it holds every SM, keep registers and thread slots: the
// shared-state form runs one 768-thread CTA per SM (two traversals, their
// bitmaps in shared memory); the global-state form (GBM, bitmaps in global
// memory) three 256-thread CTAs per SM, six traversals of four warps each.
template <int BLOCK, bool GBM>
__global__ void __maxnreg__(64) serve_kernel(ServeArgs sa)
{
    constexpr int GT = BLOCK / 2;
    const JobArgs &a = sa.job;
    extern __shared__ __align__(16) uint32_t smem_dyn[];
    __shared__ SharedState shs[2];
    __shared__ int pair_flag[2][2];
    __shared__ long long s_piece;
    const int tid = threadIdx.x;
    const int half = tid / GT;
    const int gtid = tid % GT;
    const int bar = 1 + half;
    SharedState &sh = shs[half];
    uint32_t *const state = GBM ? a.gbm + ((int64_t)blockIdx.x * 2) * a.state_words : smem_dyn;
    uint32_t *bm = state + (size_t)half * a.state_words;
    uint32_t *summ = bm + a.bitmap_words;
    int32_t *ring = (int32_t *)(GBM ? smem_dyn : smem_dyn + (size_t)2 * a.state_words) + (size_t)half * a.ring_size;
    for (int w = tid; w < 2 * a.state_words; w += BLOCK) state[w] = 0u;
    if (gtid == 0) {
        sh.chain_lo = INT32_MAX; sh.chain_hi = -1; sh.hcount = 0;
        sh.stamp = nullptr;   // counts only: no lists, no stamps
        sh.chain_s0 = 0; sh.chain_len = 0; sh.chain_total = 0;
        for (int q = 0; q < 8; q++) sh.prof[q] = 0;
        sh.nsrc = sh.nreuse = 0;
        sh.tailc[0] = sh.tailc[1] = sh.tailc[2] = 0;
        sh.fetch[0] = sh.fetch[1] = sh.fetch[2] = 0;
        sh.win_lo = sh.win_hi = 0;
    }
    const Frontier fr{ring, a.queue + ((int64_t)blockIdx.x * 2 + half) * a.qcap, a.qcap, a.status,
                      a.ring_size};
    Tally acc;
    __shared__ int s_class;
    __syncthreads();
    for (;;) {
        if (tid == 0) {
            long long got = -1;
            int cls = 0;
            volatile ServeCtl *ctl = sa.ctl;
            for (int it = 0; it < sa.idle_spins && got < 0; it++) {
                bool seen = false;
                for (int c = 0; c < kServeClasses && got < 0; c++) {
                    const unsigned long long pub = ctl->published[c];
                    const unsigned long long tk = ctl->taken[c];
                    if (tk < pub) {
                        seen = true;
                        if (atomicCAS(&sa.ctl->taken[c], tk, tk + 1) == tk) { got = (long long)tk; cls = c; }
                    }
                }
                if (got >= 0 || seen) continue;
                if (ctl->stop) break;     // only once nothing is left to take
                __nanosleep(2000);
            }
            s_piece = got;
            s_class = cls;
        }
        __syncthreads();
        const long long pc = s_piece;
        if (pc < 0) break;
        const ServePiece piece =
            load_cg(sa.pieces + (unsigned long long)s_class * sa.piece_cap + (pc % (long long)sa.piece_cap));
        const MatDesc md = load_cg(sa.slots + piece.slot);
        run_piece<BLOCK, true, true, GBM, false>(a, md, md.g[half], half, piece.s_lo, piece.s_hi, 1, bm, summ, fr, sh,
                                     pair_flag, half, gtid, bar, acc);
        {
            const int clo = sh.chain_lo, chi = sh.chain_hi;
            clear_range<GT>(bm, summ, clo, chi, gtid);
            __syncthreads();
            // the next piece may be another request: no seeding window yet
            if (gtid == 0) { sh.chain_lo = INT32_MAX; sh.chain_hi = -1; sh.hcount = 0; sh.win_lo = sh.win_hi = 0; }
        }
        if (tid == 0) {
            __threadfence();
            atomicAdd(sa.slot_done + piece.slot, 1u);
        }
        __syncthreads();
    }
    if (tid == 0) atomicAdd(&sa.ctl->exited, 1);
}

}  // namespace dev
}  // namespace gsofa

// gsofa_order.cuh -- reverse Cuthill-McKee ordering on the GPU (the step
// before the symbolic factorization: a fill-reducing, bandwidth-reducing
// order of the input pattern; the reference takes its input already ordered).
//
// The order is the one the sequential algorithm gives with every tie broken
// by (degree, vertex id) -- Cuthill and McKee's breadth-first levels, each
// dequeued vertex appending its unordered neighbours by increasing key,
// started at George and Liu's pseudo-peripheral vertex of each component,
// components taken in key order, the whole sequence reversed at the end -- so
// it is compared with the CPU restatement bit for bit.  The GPU computes it
// level by level: a vertex of the next level is appended by the first vertex
// of the current level (in order) that reaches it, so its place is given by
// the key (order of that parent, rank of its own (degree, id)); a level is
// one expansion kernel (atomicMin of the parent's order, one claim per
// vertex) and one radix sort by that key.
#pragma once

#include <cub/cub.cuh>
#include <cstdint>

namespace gsofa {
namespace dev {

// Both directions of every off-diagonal entry of the line ranges as 64-bit
// keys (row << 32 | column); the diagonal becomes the all-ones key, which
// sorts last.  off[v]: first key slot of line v (twice the entries before it).
__global__ void order_edge_keys_kernel(int32_t n, const int32_t *beg, const int32_t *end,
                                       const int32_t *adj, const int64_t *off, unsigned long long *keys)
{
    const int lane = threadIdx.x & 31;
    const int64_t w0 = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t v = w0; v < n; v += nw) {
        const int32_t b = beg[v], e = end[v];
        const int64_t o = off[v];
        for (int32_t k = b + lane; k < e; k += 32) {
            const int32_t u = adj[k];
            const int64_t at = o + 2 * (int64_t)(k - b);
            if (u == (int32_t)v) {
                keys[at] = ~0ull;
                keys[at + 1] = ~0ull;
            } else {
                keys[at] = ((unsigned long long)(uint32_t)v << 32) | (uint32_t)u;
                keys[at + 1] = ((unsigned long long)(uint32_t)u << 32) | (uint32_t)v;
            }
        }
    }
}

// Row offsets and column ids of S from its sorted, distinct keys (count of
// them, the all-ones key excluded); deg[v] and the (degree, id) sort key.
__global__ void order_rows_kernel(int32_t n, const unsigned long long *keys, int64_t count, int64_t *sp,
                                  int32_t *sa)
{
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i <= count; i += stride) {
        const int64_t r = i < count ? (int64_t)(keys[i] >> 32) : (int64_t)n;
        const int64_t rp = i > 0 ? (int64_t)(keys[i - 1] >> 32) : -1;
        for (int64_t row = rp + 1; row <= r; row++) sp[row] = i;   // rows rp+1 .. r start at i
        if (i < count) sa[i] = (int32_t)(keys[i] & 0xffffffffu);
    }
}

__global__ void order_init_kernel(int32_t n, const int64_t *sp, unsigned long long *dkeys, int32_t *ord,
                                  int32_t *pord, uint32_t *claimed, uint32_t *gen)
{
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += stride) {
        const uint32_t d = (uint32_t)(sp[v + 1] - sp[v]);
        dkeys[v] = ((unsigned long long)d << 32) | (uint32_t)v;
        ord[v] = -1;
        pord[v] = INT32_MAX;
        claimed[v] = 0u;
        gen[v] = 0u;
    }
}

// bykey[i] = the vertex of rank i; rank[v] = its position; the vertices of
// degree 0 (ranks 0 .. zeros-1) are each a component of their own and take
// the first places of the Cuthill-McKee sequence in key order.
__global__ void order_ranks_kernel(int32_t n, const unsigned long long *sorted, int32_t *bykey, int32_t *rank,
                                   int32_t *ord, int32_t *cm, int32_t *zeros)
{
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const int32_t v = (int32_t)(sorted[i] & 0xffffffffu);
        bykey[i] = v;
        rank[v] = (int32_t)i;
        if ((sorted[i] >> 32) == 0) {
            ord[v] = (int32_t)i;
            cm[i] = v;
            atomicAdd(zeros, 1);
        }
    }
}

// The first rank >= from whose vertex is still unordered (one block).
__global__ void order_find_start_kernel(int32_t n, const int32_t *bykey, const int32_t *ord, int32_t from,
                                        int32_t *out)
{
    __shared__ int32_t best;
    for (int32_t base = from; base < n; base += blockDim.x) {
        if (threadIdx.x == 0) best = INT32_MAX;
        __syncthreads();
        const int32_t i = base + (int32_t)threadIdx.x;
        if (i < n && ord[bykey[i]] < 0) atomicMin(&best, i);
        __syncthreads();
        const int32_t b = best;
        __syncthreads();
        if (b != INT32_MAX) {
            if (threadIdx.x == 0) out[0] = b;
            return;
        }
    }
    if (threadIdx.x == 0) out[0] = n;
}

// One breadth-first level over the unordered vertices: a warp per frontier
// vertex q[f0 .. f1); a vertex is taken once per search (generation g).
__global__ void order_bfs_kernel(int64_t f0, int64_t f1, int32_t *q, const int64_t *sp, const int32_t *sa,
                                 const int32_t *ord, uint32_t *gen, uint32_t g, unsigned long long *tail)
{
    const int lane = threadIdx.x & 31;
    const int64_t w0 = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t i = f0 + w0; i < f1; i += nw) {
        const int32_t v = q[i];
        for (int64_t k = sp[v] + lane; k < sp[v + 1]; k += 32) {
            const int32_t u = sa[k];
            if (ord[u] >= 0) continue;
            const uint32_t old = gen[u];
            if (old != g && atomicCAS(&gen[u], old, g) == old) q[atomicAdd(tail, 1ull)] = u;
        }
    }
}

// The least rank among q[f0 .. f1) (atomicMin into out).
__global__ void order_min_rank_kernel(int64_t f0, int64_t f1, const int32_t *q, const int32_t *rank, int32_t *out)
{
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    int32_t m = INT32_MAX;
    for (int64_t i = f0 + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < f1; i += stride) m = min(m, rank[q[i]]);
    for (int o = 16; o > 0; o >>= 1) m = min(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0 && m != INT32_MAX) atomicMin(out, m);
}

// One Cuthill-McKee level: the level's vertices are cm[l0 .. l1) (their order
// is their index); every unordered neighbour records the least order among
// the level's vertices that reach it and is queued once.
__global__ void order_cm_kernel(int32_t l0, int32_t l1, const int32_t *cm, const int64_t *sp, const int32_t *sa,
                                const int32_t *ord, int32_t *pord, uint32_t *claimed, int32_t *next,
                                unsigned long long *ntail)
{
    const int lane = threadIdx.x & 31;
    const int64_t w0 = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t i = l0 + w0; i < l1; i += nw) {
        const int32_t v = cm[i];
        for (int64_t k = sp[v] + lane; k < sp[v + 1]; k += 32) {
            const int32_t u = sa[k];
            if (ord[u] >= 0) continue;
            atomicMin(&pord[u], (int32_t)i);
            if (atomicCAS(&claimed[u], 0u, 1u) == 0u) next[atomicAdd(ntail, 1ull)] = u;
        }
    }
}

__global__ void order_level_keys_kernel(int64_t m, const int32_t *next, const int32_t *pord, const int32_t *rank,
                                        unsigned long long *keys)
{
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += stride) {
        const int32_t u = next[i];
        keys[i] = ((unsigned long long)(uint32_t)pord[u] << 32) | (uint32_t)rank[u];
    }
}

// The sorted level takes places pos .. pos + m - 1.
__global__ void order_place_kernel(int64_t m, const unsigned long long *sorted, const int32_t *bykey, int32_t pos,
                                   int32_t *ord, int32_t *cm)
{
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += stride) {
        const int32_t u = bykey[(int32_t)(sorted[i] & 0xffffffffu)];
        ord[u] = pos + (int32_t)i;
        cm[pos + i] = u;
    }
}

}  // namespace dev
}  // namespace gsofa

// gsofa_partition.hpp -- work-predicted contiguous partition of the source
// lines (host code, gsofa_partition_lines).
//
// The reference splits sources over GPUs by interleaving (s = g + t * N_gpu,
// with_space_optimization/symbfact.cuh:1084-1099), which leaves no two
// consecutive sources on one GPU, so no traversal can start from its
// predecessor's state.  Contiguous ranges keep that reuse; their sizes must
// then follow the work, which nested-dissection orders pile up in the last
// (separator) lines.
//
// Work model per line s (both passes): a fixed cost per traversal plus a cost
// per entry of the line's lists.  The list lengths are predicted from the
// symmetric structure S = A + A^T: the column counts of its Cholesky factor
// (an upper bound on |U row s| and |L column s|, which are the counts of the
// unsymmetric factors), computed in near-linear time from the elimination
// tree with the skeleton-matrix method of Gilbert, Ng and Peyton (1994).
// Cuts are then placed on equal shares of the predicted work and moved, within
// a small window, to a line whose predecessor is not in its adjacency (a
// source that would have started from scratch anyway).
#pragma once

#include <algorithm>
#include <cstdint>
#include <vector>

namespace gsofa {
namespace part {

// Per-traversal, per-list-entry and per-edge costs (SM cycles, from the
// factorization kernel's own tallies on the 80^3 nested-dissection matrix:
// ~7K cycles per source and pass, ~2.6 cycles per list entry, ~3.2 cycles per
// inspected edge of a traversal that starts afresh).  A traversal starts
// afresh at the first source of every work piece and then expands all of
// X(s), whose size is bounded by s's descendants in the elimination tree of
// A + A^T.  Work pieces of a range of r lines of an n-line matrix are
// max(r / 8G, min(n / 8G, r / 4G)) sources long on a GPU of G = 148 SMs,
// between 32 and 512.
constexpr double kCostPerSource = 7000.0;
constexpr double kCostPerEntry = 2.6;
constexpr double kCostPerEdge = 3.2;
inline double piece_len(int32_t n, int32_t parts)
{
    const double r = (double)n / (double)std::max(parts, 1), g8 = 8.0 * 148.0;
    return std::min(512.0, std::max(32.0, std::max(r / g8, std::min((double)n / g8, 2.0 * r / g8))));
}

struct Sym {
    std::vector<int64_t> ptr;   // [n+1]
    std::vector<int32_t> idx;   // neighbours of each vertex in S, no diagonal
};

// S = A + A^T without the diagonal (duplicates kept: the counts below
// ignore them).
inline Sym symmetric_structure(int32_t n, const int32_t *beg, const int32_t *end, const int32_t *adj)
{
    Sym s;
    s.ptr.assign((size_t)n + 1, 0);
    for (int32_t v = 0; v < n; v++)
        for (int32_t k = beg[v]; k < end[v]; k++) {
            const int32_t u = adj[k];
            if (u == v) continue;
            s.ptr[(size_t)v + 1]++;
            s.ptr[(size_t)u + 1]++;
        }
    for (int32_t v = 0; v < n; v++) s.ptr[(size_t)v + 1] += s.ptr[(size_t)v];
    s.idx.resize((size_t)s.ptr[(size_t)n]);
    std::vector<int64_t> at(s.ptr.begin(), s.ptr.end() - 1);
    for (int32_t v = 0; v < n; v++)
        for (int32_t k = beg[v]; k < end[v]; k++) {
            const int32_t u = adj[k];
            if (u == v) continue;
            s.idx[(size_t)at[(size_t)v]++] = u;
            s.idx[(size_t)at[(size_t)u]++] = v;
        }
    return s;
}

// Elimination tree of S (Liu's algorithm with path compression): parent[k]
// is the lowest j > k with L(j, k) != 0, or -1.
inline std::vector<int32_t> etree(int32_t n, const Sym &s)
{
    std::vector<int32_t> parent((size_t)n, -1), anc((size_t)n, -1);
    for (int32_t k = 0; k < n; k++) {
        for (int64_t p = s.ptr[(size_t)k]; p < s.ptr[(size_t)k + 1]; p++) {
            int32_t r = s.idx[(size_t)p];
            if (r >= k) continue;
            // climb from r to the root of its current subtree, pointing every
            // visited vertex at k
            while (anc[(size_t)r] != -1 && anc[(size_t)r] != k) {
                const int32_t next = anc[(size_t)r];
                anc[(size_t)r] = k;
                r = next;
            }
            if (anc[(size_t)r] == -1) {
                anc[(size_t)r] = k;
                parent[(size_t)r] = k;
            }
        }
    }
    return parent;
}

// Postorder of the forest (children visited in increasing order).
inline std::vector<int32_t> postorder(int32_t n, const std::vector<int32_t> &parent)
{
    std::vector<int32_t> head((size_t)n, -1), next((size_t)n, -1), post, stack;
    post.reserve((size_t)n);
    for (int32_t j = n - 1; j >= 0; j--) {
        const int32_t p = parent[(size_t)j];
        if (p == -1) continue;
        next[(size_t)j] = head[(size_t)p];
        head[(size_t)p] = j;
    }
    for (int32_t root = 0; root < n; root++) {
        if (parent[(size_t)root] != -1) continue;
        stack.push_back(root);
        while (!stack.empty()) {
            const int32_t v = stack.back();
            const int32_t c = head[(size_t)v];
            if (c == -1) {
                stack.pop_back();
                post.push_back(v);
            } else {
                head[(size_t)v] = next[(size_t)c];   // consume the child
                stack.push_back(c);
            }
        }
    }
    return post;
}

// Column counts of the Cholesky factor of S (diagonal included), by
// accumulating, in postorder, +1 at every leaf of a row subtree and -1 at the
// least common ancestor of consecutive leaves (found with a disjoint-set
// forest that follows the postorder).
inline std::vector<int64_t> column_counts(int32_t n, const Sym &s, const std::vector<int32_t> &parent,
                                          const std::vector<int32_t> &post)
{
    std::vector<int32_t> first((size_t)n, -1), maxfirst((size_t)n, -1), prevleaf((size_t)n, -1), anc((size_t)n);
    std::vector<int64_t> delta((size_t)n, 0);
    for (int32_t k = 0; k < n; k++) {
        int32_t j = post[(size_t)k];
        delta[(size_t)j] = first[(size_t)j] == -1 ? 1 : 0;   // leaves of the tree start at 1
        for (; j != -1 && first[(size_t)j] == -1; j = parent[(size_t)j]) first[(size_t)j] = k;
    }
    for (int32_t i = 0; i < n; i++) anc[(size_t)i] = i;
    for (int32_t k = 0; k < n; k++) {
        const int32_t j = post[(size_t)k];
        if (parent[(size_t)j] != -1) delta[(size_t)parent[(size_t)j]]--;
        for (int64_t p = s.ptr[(size_t)j]; p < s.ptr[(size_t)j + 1]; p++) {
            const int32_t i = s.idx[(size_t)p];
            // is j a leaf of the row subtree of i?  (i > j, and j's subtree
            // starts after every subtree of i's previous leaves)
            if (i <= j || first[(size_t)j] <= maxfirst[(size_t)i]) continue;
            maxfirst[(size_t)i] = first[(size_t)j];
            const int32_t jprev = prevleaf[(size_t)i];
            prevleaf[(size_t)i] = j;
            delta[(size_t)j]++;
            if (jprev == -1) continue;   // first leaf of row i
            // least common ancestor of jprev and j: the root of jprev's set
            int32_t q = jprev;
            while (q != anc[(size_t)q]) q = anc[(size_t)q];
            for (int32_t v = jprev; v != q;) {
                const int32_t up = anc[(size_t)v];
                anc[(size_t)v] = q;
                v = up;
            }
            delta[(size_t)q]--;
        }
        if (parent[(size_t)j] != -1) anc[(size_t)j] = parent[(size_t)j];
    }
    // children before parents: parent[j] > j
    for (int32_t j = 0; j < n; j++)
        if (parent[(size_t)j] != -1) delta[(size_t)parent[(size_t)j]] += delta[(size_t)j];
    return delta;
}

// True when s-1 is in line s of the input (a traversal of s could start from
// the state of s-1 by adjacency).
inline bool has_prev(int32_t s, const int32_t *beg, const int32_t *end, const int32_t *adj)
{
    if (s <= 0) return false;
    for (int32_t k = beg[s]; k < end[s]; k++)
        if (adj[k] == s - 1) return true;
    return false;
}

// Cuts [0 = cuts[0] < ... < cuts[parts] = n] of equal predicted work; the
// predicted work of each part (both passes) goes to work[] when non-null.
inline void partition(int32_t n, const int32_t *beg, const int32_t *end, const int32_t *adj, int32_t parts,
                      int32_t *cuts, double *work)
{
    const Sym s = symmetric_structure(n, beg, end, adj);
    const std::vector<int32_t> parent = etree(n, s);
    const std::vector<int32_t> post = postorder(n, parent);
    const std::vector<int64_t> cc = column_counts(n, s, parent, post);
    // descendants in the elimination tree, with their symmetric degrees: the
    // edges a fresh traversal of v would inspect at most
    std::vector<double> sub((size_t)n, 0.0);
    for (int32_t v = 0; v < n; v++) sub[(size_t)v] = (double)(s.ptr[(size_t)v + 1] - s.ptr[(size_t)v]);
    for (int32_t v = 0; v < n; v++)    // parent[v] > v: children first
        if (parent[(size_t)v] != -1) sub[(size_t)parent[(size_t)v]] += sub[(size_t)v];
    std::vector<double> pre((size_t)n + 1, 0.0);
    const double kPieceLen = piece_len(n, parts);
    for (int32_t v = 0; v < n; v++) {
        const double fresh = (sub[(size_t)v] - (double)(s.ptr[(size_t)v + 1] - s.ptr[(size_t)v])) / 2.0;
        pre[(size_t)v + 1] = pre[(size_t)v] + 2.0 * kCostPerSource +
                             kCostPerEntry * 2.0 * (double)std::max<int64_t>(cc[(size_t)v] - 1, 0) +
                             2.0 * kCostPerEdge * fresh / kPieceLen;
    }
    const double total = pre[(size_t)n];
    cuts[0] = 0;
    for (int32_t p = 1; p < parts; p++) {
        const double target = total * (double)p / (double)parts;
        int32_t c = (int32_t)(std::lower_bound(pre.begin(), pre.end(), target) - pre.begin());
        c = std::max(cuts[p - 1], std::min(c, n));
        // move the cut to a nearby line that does not continue an adjacency
        // chain, when there is one
        for (int32_t t = c; t < std::min(n, c + 64); t++)
            if (!has_prev(t, beg, end, adj)) { c = t; break; }
        cuts[p] = c;
    }
    cuts[parts] = n;
    // no empty part while there are lines for every part
    for (int32_t p = 1; p < parts; p++)
        cuts[p] = std::min(std::max(cuts[p], cuts[p - 1] + 1), std::max(n - (parts - p), cuts[p - 1]));
    for (int32_t p = 1; p <= parts; p++) cuts[p] = std::max(cuts[p], cuts[p - 1]);
    if (work)
        for (int32_t p = 0; p < parts; p++) work[p] = pre[(size_t)cuts[p + 1]] - pre[(size_t)cuts[p]];
}

}  // namespace part
}  // namespace gsofa

// gsofa_supernodal.cuh -- SuperLU-style supernodal structure from a device-
// resident result (the consumer-side format of the symbolic stage).
//
// Supernode k = lines [fst, lst) satisfies, for consecutive lines s-1, s in it:
// s-1 in line s, s in U row s-1 and |U row s| = |U row s-1| - 1.  Hence
//   * U row j = {j+1 .. lst-1} u R for every j in [fst, lst), with R the
//     columns >= lst of U row fst (path concatenation makes U row s contain
//     U row s-1 minus {s}; the count makes them equal), and
//   * L col j minus {j+1} lies inside L col j+1 (a path r -> j through
//     vertices < j continues j -> j+1 through vertices < j, which s in U row
//     s-1 provides), so L col lst-1 holds every row >= lst of the supernode's
//     columns.
// Two passes: sizes per supernode (and supno), then, after the host turns the
// sizes into offsets, one warp per supernode copies its index lists out of
// the pattern (CSR form, or the ranges form's pool and begins).
#pragma once

#include <stdint.h>

namespace gsofa {
namespace dev {

struct SupernodalArgs {
    const int32_t *sn;        // [nsuper] first line of each supernode (job line ids)
    int32_t nsuper;
    int32_t n;
    int64_t lb;               // the matrix's first line in the job
    const int32_t *ucnt;      // [n] |U row s|
    const int32_t *lcnt;      // [n] |L col s|
    const int64_t *uptr;      // [n+1] U row offsets (job-wide, pass 0)
    const int64_t *lptr;      // [n+1] L column offsets (job-wide, pass 1)
    const int32_t *out;       // compacted pattern of the job (CSR form), or the
                              // pool of the ranges form
    int64_t u0, l0;           // where this matrix's U rows / L columns start in out
    const int64_t *ubeg;      // ranges form: [n] where U row s / L column s start
    const int64_t *lbeg;      //   in out (null: the CSR form)
    int64_t *lsize, *usize;   // [nsuper] per-supernode list sizes (first pass)
    const int64_t *xlsub;     // [nsuper+1] offsets (second pass)
    const int64_t *xusub;
    int32_t *lsub, *usub;
    int32_t *supno;           // [n]
};

__device__ __forceinline__ void supernode_range(const SupernodalArgs &a, int32_t k, int32_t *fst, int32_t *lst)
{
    *fst = (int32_t)(a.sn[k] - a.lb);
    *lst = k + 1 < a.nsuper ? (int32_t)(a.sn[k + 1] - a.lb) : a.n;
}

__global__ void supernodal_size_kernel(SupernodalArgs a)
{
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < a.nsuper;
         k += (int64_t)gridDim.x * blockDim.x) {
        int32_t fst, lst;
        supernode_range(a, (int32_t)k, &fst, &lst);
        a.lsize[k] = (int64_t)(lst - fst) + a.lcnt[lst - 1];
        a.usize[k] = (int64_t)a.ucnt[fst] - (lst - fst - 1);
        for (int32_t j = fst; j < lst; j++) a.supno[j] = (int32_t)k;
    }
}

__global__ void supernodal_fill_kernel(SupernodalArgs a)
{
    const int lane = threadIdx.x & 31;
    const int64_t warps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t k = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; k < a.nsuper; k += warps) {
        int32_t fst, lst;
        supernode_range(a, (int32_t)k, &fst, &lst);
        const int32_t w = lst - fst;
        // rows: the diagonal block, then the last column's rows below it
        int32_t *ld = a.lsub + a.xlsub[k];
        for (int32_t i = lane; i < w; i += 32) ld[i] = fst + i;
        const int32_t *lc = a.lbeg ? a.out + a.lbeg[lst - 1] : a.out + a.l0 + (a.lptr[lst - 1] - a.lptr[0]);
        const int32_t nl = a.lcnt[lst - 1];
        for (int32_t i = lane; i < nl; i += 32) ld[w + i] = lc[i];
        // columns right of the block: U row fst past its first w-1 entries
        int32_t *ud = a.usub + a.xusub[k];
        const int32_t *uc = (a.ubeg ? a.out + a.ubeg[fst] : a.out + a.u0 + (a.uptr[fst] - a.uptr[0])) + (w - 1);
        const int64_t nu = a.xusub[k + 1] - a.xusub[k];
        for (int64_t i = lane; i < nu; i += 32) ud[i] = uc[i];
    }
}

}  // namespace dev
}  // namespace gsofa

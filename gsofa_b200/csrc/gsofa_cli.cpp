// gsofa -- command-line driver with the reference's argv contract.
//
//   gsofa colbeg.dat colend.dat csr.dat N_GPU [mem_GB [max_supernode_size GPUs_per_node]]
//   gsofa --to-binary colbeg.dat colend.dat csr.dat out_prefix
//
// The second form writes the three files in the library's binary form
// (out_prefix.colbeg.bin, .colend.bin, .csr.bin), which the first form reads
// without text parsing.
//
// Mirrors without_space_optimization/main.cu:14-50, which calls
// symbfact_min_id(argc, argv, 0, fill_count, time) and prints the result.
// The reference's main prints an MPI-reduced total that is always zero
// (main.cu:19,33,41); this driver prints the real total and exits non-zero on
// any error instead of calling exit() from inside the library.
#include "../../include/gsofa.h"

#include <cstdio>
#include <cstring>
#include <string>

static int to_binary(char **argv)
{
    int32_t n = 0;
    int64_t nnz = 0;
    int32_t *beg = nullptr, *end = nullptr, *adj = nullptr;
    gsofa_status s = gsofa_read_text(argv[2], argv[3], argv[4], &n, &nnz, &beg, &end, &adj);
    if (s == GSOFA_OK) {
        const std::string pre = argv[5];
        const std::string b = pre + ".colbeg.bin", e = pre + ".colend.bin", c = pre + ".csr.bin";
        s = gsofa_write_binary(b.c_str(), e.c_str(), c.c_str(), n, nnz, beg, end, adj);
        if (s == GSOFA_OK) std::printf("wrote %s %s %s (n = %d, nnz = %lld)\n", b.c_str(), e.c_str(), c.c_str(), n,
                                       (long long)nnz);
    }
    gsofa_free(beg);
    gsofa_free(end);
    gsofa_free(adj);
    if (s != GSOFA_OK) {
        std::fprintf(stderr, "gsofa: %s\n", gsofa_status_str(s));
        return 1;
    }
    return 0;
}

int main(int argc, char **argv)
{
    if (argc == 6 && std::strcmp(argv[1], "--to-binary") == 0) return to_binary(argv);
    if (argc < 5) {
        std::fprintf(stderr,
                     "usage: %s colbeg colend csr N_GPU [mem_GB [max_supernode_size GPUs_per_node]]\n"
                     "       %s --to-binary colbeg colend csr out_prefix\n",
                     argv[0], argv[0]);
        return 2;
    }
    std::printf("Number of GPUs used: %s\n", argv[4]);
    uint64_t fills = 0;
    double ms = 0.0;
    gsofa_status s = gsofa_symbfact_min_id(argc, argv, 0, &fills, &ms);
    if (s != GSOFA_OK) {
        std::fprintf(stderr, "gsofa: %s\n", gsofa_status_str(s));
        return 1;
    }
    std::printf("Number of fill-ins detected: %llu\n", (unsigned long long)fills);
    std::printf("Total time over the partitions: %.4f ms\n", ms);
    return 0;
}

// gsofa -- command-line driver with the reference's argv contract.
//
//   gsofa colbeg.dat colend.dat csr.dat N_GPU [mem_GB [max_supernode_size GPUs_per_node]]
//
// Mirrors without_space_optimization/main.cu:14-50, which calls
// symbfact_min_id(argc, argv, 0, fill_count, time) and prints the result.
// The reference's main prints an MPI-reduced total that is always zero
// (main.cu:19,33,41); this driver prints the real total and exits non-zero on
// any error instead of calling exit() from inside the library.
#include "../../include/gsofa.h"

#include <cstdio>

int main(int argc, char **argv)
{
    if (argc < 5) {
        std::fprintf(stderr,
                     "usage: %s colbeg colend csr N_GPU [mem_GB [max_supernode_size GPUs_per_node]]\n",
                     argv[0]);
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

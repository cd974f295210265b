/*
 * gw_ref_convert.cpp -- TEST INFRASTRUCTURE: the reference's own graph
 * preprocessor (convert_if_notexists: convert_to_csr + compute_block,
 * src/preprocess/conversions.hpp:181-404), compiled unmodified from the
 * reference tree, run on one text edge list.  Its output files are the
 * golden vectors of the device converter (tests/golden/make_convert_golden.py).
 *
 * Usage: gw_ref_convert <edge list path> <blocksize_kb>
 * Writes <path>_GraphWalker/... and prints "nblocks <n>".
 */
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "api/graphwalker_basic_includes.hpp"

int main(int argc, char **argv) {
    if (argc < 3) {
        fprintf(stderr, "usage: %s <edge list> <blocksize_kb>\n", argv[0]);
        return 2;
    }
    bid_t nblocks = convert_if_notexists(argv[1], strtoull(argv[2], nullptr, 10));
    printf("nblocks %u\n", (unsigned)nblocks);
    return 0;
}

/*
 * gw_oracle_rmat.c -- BENCHMARK INFRASTRUCTURE ONLY (input preparation for
 * bench.py's reference arm).
 *
 * Writes the seeded R-MAT graph of gw_oracle.c (gwo_rmat_csr) in the
 * reference's preprocessed on-disk layout (src/api/filename.hpp:16-51,
 * written by convert_to_csr, src/preprocess/conversions.hpp:127-141):
 *
 *   <base>_GraphWalker/graphinfo/file_0.beg_pos   uint64 row pointer (nv + 1)
 *   <base>_GraphWalker/graphinfo/file_0.csr       uint32 column ids
 *   <base>_GraphWalker/filesize_1024GB.filerange  "0\n<nv>\n"
 *   <base>_GraphWalker/N.nvertices                "<nv>\n"
 *
 * No block range is written: the reference's own convert_if_notexists
 * (conversions.hpp:371-404) computes and writes it on its first run.
 * It is a separate executable so that the process timing the reference
 * loads no shared library of this repository.
 *
 * Usage: gw_oracle_rmat <scale> <edge_factor> <seed> <a> <b> <c> <base>
 */
#include <errno.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/stat.h>

#include "gw_oracle.h"

static uint32_t prob_to_u32(double x) {
    /* the generator compares a 32-bit word with round(x * 2^32), saturated */
    double t = x * 4294967296.0 + 0.5;
    if (t >= 4294967295.0) return 0xffffffffu;
    if (t <= 0.0) return 0u;
    return (uint32_t)t;
}

static int write_all(const char *path, const void *buf, size_t n) {
    FILE *f = fopen(path, "wb");
    if (!f) return -1;
    size_t w = n ? fwrite(buf, 1, n, f) : 0;
    int rc = fclose(f);
    return (w == n && rc == 0) ? 0 : -1;
}

int main(int argc, char **argv) {
    if (argc != 8) {
        fprintf(stderr, "usage: %s scale edge_factor seed a b c base\n", argv[0]);
        return 2;
    }
    uint32_t scale = (uint32_t)strtoul(argv[1], NULL, 10);
    uint64_t ef = strtoull(argv[2], NULL, 10);
    uint64_t seed = strtoull(argv[3], NULL, 10);
    double a = atof(argv[4]), b = atof(argv[5]), c = atof(argv[6]);
    const char *base = argv[7];
    if (scale == 0 || scale > 31) {
        fprintf(stderr, "scale must be in [1, 31]\n");
        return 2;
    }
    uint64_t nv = 1ull << scale, m = ef * nv;
    uint64_t *rowptr = (uint64_t *)malloc((nv + 1) * sizeof(uint64_t));
    uint32_t *colidx = (uint32_t *)malloc((m ? m : 1) * sizeof(uint32_t));
    if (!rowptr || !colidx) {
        fprintf(stderr, "out of memory\n");
        return 3;
    }
    uint64_t kept = gwo_rmat_csr(scale, m, seed, prob_to_u32(a), prob_to_u32(a + b), prob_to_u32(a + b + c),
                                 rowptr, colidx);

    size_t bl = strlen(base);
    char *path = (char *)malloc(bl + 128);
    sprintf(path, "%s_GraphWalker", base);
    if (mkdir(path, 0777) && errno != EEXIST) { perror(path); return 4; }
    sprintf(path, "%s_GraphWalker/graphinfo", base);
    if (mkdir(path, 0777) && errno != EEXIST) { perror(path); return 4; }
    sprintf(path, "%s_GraphWalker/graphinfo/file_0.beg_pos", base);
    if (write_all(path, rowptr, (nv + 1) * sizeof(uint64_t))) { perror(path); return 4; }
    sprintf(path, "%s_GraphWalker/graphinfo/file_0.csr", base);
    if (write_all(path, colidx, kept * sizeof(uint32_t))) { perror(path); return 4; }
    char txt[64];
    int n = snprintf(txt, sizeof txt, "0\n%llu\n", (unsigned long long)nv);
    sprintf(path, "%s_GraphWalker/filesize_1024GB.filerange", base);
    if (write_all(path, txt, (size_t)n)) { perror(path); return 4; }
    n = snprintf(txt, sizeof txt, "%llu\n", (unsigned long long)nv);
    sprintf(path, "%s_GraphWalker/N.nvertices", base);
    if (write_all(path, txt, (size_t)n)) { perror(path); return 4; }
    printf("nvertices %llu nedges %llu\n", (unsigned long long)nv, (unsigned long long)kept);
    free(path);
    free(rowptr);
    free(colidx);
    return 0;
}

// Replays a list of AddBlock calls through the reference's own
// MultiDomainCCSRBuilder (DBEM1/multidomain.cpp:1101-1210) and writes the
// built block-CCSR matrix (test infrastructure only; linked against the
// unchanged reference objects by oracle/Makefile).
//
//   dbem_ref_builder <calls.bin> <out.bin>
//
// calls.bin: int64 rows, cols, n; then n x (int64 row, int64 col, double
// sign, double block9[9] column-major as the assembly routines produce it).
// out.bin: int64 n_rows, nnz; int32 row_ptr[n_rows + 1]; int32 col[nnz];
// double val[nnz][9] (row-major, as Build stores it).

#include "multidomain.h"

#include <cstdint>
#include <cstdio>
#include <vector>

int main(int argc, char** argv)
{
    if (argc != 3) {
        std::fprintf(stderr, "usage: dbem_ref_builder calls.bin out.bin\n");
        return 2;
    }
    FILE* in = std::fopen(argv[1], "rb");
    if (!in) return 3;
    int64_t head[3];
    if (std::fread(head, sizeof(int64_t), 3, in) != 3) return 4;
    MultiDomainCCSRBuilder b((long)head[0], (long)head[1]);
    for (int64_t i = 0; i < head[2]; ++i) {
        int64_t rc[2];
        double sign, blk[9];
        if (std::fread(rc, sizeof(int64_t), 2, in) != 2 || std::fread(&sign, sizeof(double), 1, in) != 1 ||
            std::fread(blk, sizeof(double), 9, in) != 9)
            return 4;
        b.AddBlock((long)rc[0], (long)rc[1], sign, blk);
    }
    std::fclose(in);
    CCSRMat m;
    b.Build(m);
    FILE* out = std::fopen(argv[2], "wb");
    if (!out) return 5;
    const int64_t nnz = m.n > 0 ? m.row_ptr[m.n] : 0;
    const int64_t hdr[2] = {(int64_t)m.n, nnz};
    std::fwrite(hdr, sizeof(int64_t), 2, out);
    if (m.n > 0) std::fwrite(m.row_ptr, sizeof(int), (size_t)m.n + 1, out);
    if (nnz) {
        std::fwrite(m.col_index, sizeof(int), (size_t)nnz, out);
        std::fwrite(m.value, sizeof(double), 9 * (size_t)nnz, out);
    }
    std::fclose(out);
    return 0;
}

// Reads one block-CCSR matrix at a byte offset of a file with the reference's
// own CCSRMat::ReadBinary and writes it back with CCSRMat::WriteBinary
// (DBEM1/mat_vec.cpp:1690-1730), so a test can check that a matrix section
// of the B200 library's cache file is the reference's binary layout byte for
// byte (test infrastructure only; linked against the unchanged reference
// objects by oracle/Makefile).
//
//   dbem_ref_ccsr <in.bin> <offset> <out.bin>
//
// Prints "n nnz" of the matrix read; exit 5 when ReadBinary refuses it.

#include "mat_vec.h"

#include <cstdio>
#include <cstdlib>

int main(int argc, char** argv)
{
    if (argc != 4) {
        std::fprintf(stderr, "usage: dbem_ref_ccsr in.bin offset out.bin\n");
        return 2;
    }
    FILE* in = std::fopen(argv[1], "rb");
    if (!in) return 3;
    if (std::fseek(in, std::atol(argv[2]), SEEK_SET) != 0) return 4;
    CCSRMat m;
    if (!m.ReadBinary(in)) return 5;
    std::fclose(in);
    FILE* out = std::fopen(argv[3], "wb");
    if (!out) return 6;
    if (!m.WriteBinary(out)) return 7;
    std::fclose(out);
    std::printf("%ld %ld\n", (long)m.n, (long)m.NonZeroBlocks());
    return 0;
}

// wide.h -- contractions whose operand keys need more than 64 bits, relabeled
// onto keys that fit (wide.cu).
#pragma once

#include <memory>

#include "internal.h"

namespace gs {

struct WideMap {
    gsparc_tensor x2, y2;         // X'(F, C), Y'(C, G): 2 modes each, values shared with X, Y
    DBuf<uint64_t> x2idx, y2idx;  // their SoA index arrays
    DBuf<uint64_t> xf, yf;        // rank -> original free part, ascending
    int yb2 = 0;                  // bits of G: output key of X' x Y' is F << yb2 | G
    int nfbits_y = 0;             // original Y free bits: output key x_f << nfbits_y | y_f
    int cx2[1] = {1}, cy2[1] = {0};
};

// Builds X', Y' and the rank tables (one host round trip per operand side).
std::unique_ptr<WideMap> make_wide(Arena &A, const gsparc_tensor *X, const Layout &LX, const gsparc_tensor *Y,
                                   const Layout &LY, cudaStream_t s);
// Output keys of X' x Y' -> output keys of X x Y, in place, on stream s.
void wide_remap_keys(const WideMap &w, uint64_t *keys, uint64_t n, cudaStream_t s);
// The same as 128-bit keys, two words per key (low word first) into out2[2n].
void wide_remap_keys128(const WideMap &w, const uint64_t *keys, uint64_t *out2, uint64_t n, cudaStream_t s);

}  // namespace gs

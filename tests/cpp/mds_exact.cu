// Host check of the Tip5 MDS half-product used by the GPU kernels
// (t5_mds_half in tip5.cuh, compiled here for the CPU: the same IEEE-754 double
// adds and fused multiply-adds as the FP64 pipe).  Each 32-bit half v enters
// as the kernels' biased double 2^52 + v, and every output must equal the exact
// integer circulant product sum_c M[(r - c) mod 16] * v[c] plus the added
// 32-bit value a[r] (a round constant's half in the kernels), plus 2^52.  Inputs:
// all 2^16 patterns of {0, 2^32 - 1} (they reach the extreme value of every
// intermediate of the split convolution), near-extreme and uniform random halves.
#include "../../triton-vm-prover_b200/csrc/tip5.cuh"
#include <cstdio>
#include <cstring>
#include <random>

using namespace tvmc;

static int check(const uint32_t v[16], const uint32_t a[16]) {
    static const long long M[16] = {TVMC_T5_MDS_FIRST_COLUMN};
    double x[16];
    for (int c = 0; c < 16; c++) {
        const uint64_t b = 0x4330000000000000ull | v[c];  // t5_half_biased(v[c])
        memcpy(&x[c], &b, 8);
    }
    double bias[16];
    for (int r = 0; r < 16; r++) bias[r] = T5_MDS_BIAS + (double)a[r];
    t5_mds_half(x, bias);
    int bad = 0;
    for (int r = 0; r < 16; r++) {
        unsigned long long want = 0;
        for (int c = 0; c < 16; c++) want += (unsigned long long)M[(r - c) & 15] * v[c];
        want += a[r];
        uint64_t bits;
        memcpy(&bits, &x[r], 8);
        if ((bits & 0xFFFFFFFFFFFFFull) != want || x[r] != 4503599627370496.0 + (double)want) bad++;
    }
    return bad;
}

int main() {
    long bad = 0, cases = 0;
    uint32_t v[16], a[16], amax[16], azero[16];
    for (int r = 0; r < 16; r++) { amax[r] = 0xFFFFFFFFu; azero[r] = 0; }
    for (uint32_t pat = 0; pat < (1u << 16); pat++, cases++) {
        for (int c = 0; c < 16; c++) v[c] = (pat >> c & 1) ? 0xFFFFFFFFu : 0u;
        bad += check(v, (pat & 1) ? amax : azero);
    }
    std::mt19937_64 rng(7);
    for (int t = 0; t < 200000; t++, cases++) {
        for (int c = 0; c < 16; c++) {
            const uint64_t r = rng();
            v[c] = (t & 1) ? (uint32_t)r : ((r & 1) ? 0xFFFFFFFFu - (uint32_t)(r >> 56) : (uint32_t)(r >> 56));
        }
        for (int r = 0; r < 16; r++) a[r] = (uint32_t)rng();
        bad += check(v, a);
    }
    printf("%ld input vectors, %ld wrong outputs\n", cases, bad);
    return bad != 0;
}

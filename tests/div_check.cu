// GPU check of the Riemann solver's shared-reciprocal division
// (hosono-2dmhd_b200/csrc/physics.cuh, SharedRecipDiv) against IEEE '/':
// for every in-range pair the quotient must have the same bits, and every
// out-of-range operand must clear `ok`.  Operands: random significands and
// exponents, significands of all ones, exact quotients, and quotients next
// to rounding midpoints.  Prints "pairs N mismatches M flagged F"; exit 0
// when M == 0 and every out-of-range case was flagged.
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "physics.cuh"

using namespace hosono;

__device__ __forceinline__ unsigned long long mix(unsigned long long x) {  // splitmix64 finaliser
    x += 0x9e3779b97f4a7c15ull;
    x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ull;
    x = (x ^ (x >> 27)) * 0x94d049bb133111ebull;
    return x ^ (x >> 31);
}
__device__ __forceinline__ double make(unsigned long long sig, int e, bool neg) {
    const unsigned long long bits = ((unsigned long long)(neg ? 1 : 0) << 63) |
                                    ((unsigned long long)(e + 1023) << 52) | (sig & ((1ull << 52) - 1));
    double d;
    memcpy(&d, &bits, 8);
    return d;
}

__global__ void check(unsigned long long seed, long long n, unsigned long long* bad, unsigned long long* missed,
                      unsigned long long* flagged) {
    unsigned long long lbad = 0, lmiss = 0, lflag = 0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const unsigned long long r1 = mix(seed ^ (2 * i)), r2 = mix(seed ^ (2 * i + 1)), r3 = mix(r1 ^ r2);
        const int kind = (int)(r3 & 7);
        const int eb = (int)((r3 >> 8) % 1001) - 500, ea = (int)((r3 >> 20) % 1001) - 500;
        unsigned long long sb = r2;
        if (kind == 1) sb = ~0ull;  // significand of b all ones
        const double b = make(sb, eb, r3 & (1ull << 40));
        double a = make(r1, ea, r3 & (1ull << 41));
        if (kind == 2) a = b * make(r1 >> 20, (int)((r3 >> 32) % 21) - 10, false);  // exact-ish quotients
        if (kind == 3) {  // a/b next to a midpoint between two doubles
            const double m = make(r1, (int)((r3 >> 32) % 21) - 10, false);
            const double up = nextafter(m, 2.0 * m);
            a = fma(b, m, 0.5 * b * (up - m));
        }
        if (kind == 4) a = 0.0 * b;
        SharedRecipDiv dv;
        const auto rr = dv.recip(b);
        const double q = dv.div(a, rr);
        const double ref = a / b;
        const bool in = (fabs(b) >= 0x1p-500 && fabs(b) < 0x1p501) &&
                        (a == 0.0 || (fabs(a) >= 0x1p-500 && fabs(a) < 0x1p501));
        if (dv.ok) {
            unsigned long long x, y;
            memcpy(&x, &q, 8);
            memcpy(&y, &ref, 8);
            if (x != y) lbad++;
            if (!in) lmiss++;
        } else {
            lflag++;
            if (in) lmiss++;
        }
    }
    atomicAdd(bad, lbad);
    atomicAdd(missed, lmiss);
    atomicAdd(flagged, lflag);
}

int main(int argc, char** argv) {
    const long long n = argc > 1 ? atoll(argv[1]) : (1ll << 30);
    const int rounds = argc > 2 ? atoi(argv[2]) : 4;
    unsigned long long* d = nullptr;
    if (cudaMalloc(&d, 3 * sizeof(unsigned long long)) != cudaSuccess) return 2;
    unsigned long long tot[3] = {0, 0, 0};
    for (int r = 0; r < rounds; r++) {
        cudaMemset(d, 0, 3 * sizeof(unsigned long long));
        check<<<148 * 8, 256>>>(0x5eed0000ull + 7919ull * r, n, d, d + 1, d + 2);
        unsigned long long h[3];
        if (cudaMemcpy(h, d, sizeof h, cudaMemcpyDeviceToHost) != cudaSuccess) return 3;
        for (int k = 0; k < 3; k++) tot[k] += h[k];
    }
    cudaFree(d);
    std::printf("pairs %lld mismatches %llu wrongly_flagged_or_missed %llu flagged %llu\n", n * rounds, tot[0], tot[1],
                tot[2]);
    return (tot[0] == 0 && tot[1] == 0) ? 0 : 1;
}

// Randomised check of the server's device-memory arena (csrc/arena.h):
// random alloc/release sequences keep the free and used ranges tiling the
// arena without overlap, merge neighbouring free ranges, and return to one
// free range when everything is released.  Exit status 0 = pass.
#include <cstdio>
#include <random>
#include <vector>

#include "arena.h"

int main(int argc, char** argv) {
    const unsigned seed = argc > 1 ? (unsigned)std::atoi(argv[1]) : 1u;
    std::mt19937_64 rng(seed);
    hosono::Arena a;
    const size_t cap = (size_t)1 << 30;
    a.reset(cap + 100);  // capacity rounds down to the alignment
    if (a.capacity() != cap || !a.check()) return 1;
    std::vector<size_t> live;
    size_t fails = 0;
    for (int op = 0; op < 200000; op++) {
        const bool doAlloc = live.empty() || (rng() % 100) < 55;
        if (doAlloc) {
            const size_t n = 1 + rng() % (cap / 64);
            size_t off = 0;
            const bool fit = a.fits(n);
            if (a.alloc(n, &off)) {
                if (!fit || off % hosono::Arena::kAlign) return 2;
                live.push_back(off);
            } else {
                if (fit) return 3;
                fails++;
            }
        } else {
            const size_t k = rng() % live.size();
            if (!a.release(live[k])) return 4;
            live[k] = live.back();
            live.pop_back();
        }
        if (op % 97 == 0 && !a.check()) return 5;
    }
    if (a.release(12345)) return 6;  // not a block start
    for (size_t off : live)
        if (!a.release(off)) return 7;
    if (!a.check() || a.used() != 0 || a.blocks() != 0 || a.largest_free() != cap) return 8;
    std::printf("ok fails=%zu\n", fails);
    return fails ? 0 : 9;  // the sequence must have filled the arena at least once
}

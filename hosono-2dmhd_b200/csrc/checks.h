// checks.h -- argument checks shared by the C-ABI entry points, done before
// any CUDA call.
#pragma once

#include <cstdlib>

#include "hosono_gpu.h"

namespace hosono {

// the kernels hard-code the stencil order of GP.f90:85-95; check the table
inline bool stencil_ok(int R, const int* stenc) {
    if (!stenc) return true;
    const int nsMax = 1 + 2 * R * (R + 1);
    for (int rr = 1; rr <= R; rr++) {
        int k = 0;
        for (int a = -rr; a <= rr; a++)
            for (int b = -rr; b <= rr; b++)
                if (std::abs(a) + std::abs(b) <= rr) {
                    if (stenc[0 + 2 * (k + nsMax * (rr - 1))] != a || stenc[1 + 2 * (k + nsMax * (rr - 1))] != b)
                        return false;
                    k++;
                }
    }
    return true;
}

// the checks Engine::add repeats
inline bool params_ok(const hosono_params& p) {
    const int R = p.max_radius;
    return R >= 1 && R <= 3 && p.ngc == R + 2 && p.nx >= 2 * p.ngc && p.ny >= 2 * p.ngc &&
           (p.bc == HOSONO_BC_OUTFLOW || p.bc == HOSONO_BC_PERIODIC) && p.riemann_solver == 1 && p.dx > 0 &&
           p.dy > 0;
}

}  // namespace hosono

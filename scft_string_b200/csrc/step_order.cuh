// step_order.cuh -- claim order of the persistent step kernel (k_step_pf).
//
// The (slot, field) groups form blocks of kStepBlock; wave w holds phase p of
// block w - p for p = 3, 2, 1, 0 (the oldest work first).  Phase p of a block
// thus comes one wave after phase p - 1 of the same block, so every item's
// dependencies (all items of the previous phase of its group) come earlier in
// the order, which is what keeps the kernel free of deadlock; and the phases
// of different blocks overlap instead of running one after another over the
// whole batch.  __host__ __device__ so that tests/test_step_order.py checks
// the order on the CPU.
#pragma once
#include <cuda_runtime.h>

#ifndef SCFT_HD
#define SCFT_HD __host__ __device__ __forceinline__
#endif

namespace scft {

constexpr int kStepBlock = 4;

// item `it` of the claim order -> (phase, group, unit); false past the end.
// G groups; per[p] items per group in phase p.
SCFT_HD bool step_item(int it, int G, const int *per, int &phase, int &group, int &unit)
{
    const int nblk = (G + kStepBlock - 1) / kStepBlock;
    for (int w = 0; w < nblk + 3; w++)
        for (int p = 3; p >= 0; p--) {
            const int b = w - p;
            if (b < 0 || b >= nblk) continue;
            const int g0 = b * kStepBlock, ng = (G - g0) < kStepBlock ? (G - g0) : kStepBlock;
            const int n = ng * per[p];
            if (it < n) {
                phase = p;
                group = g0 + it / per[p];
                unit = it - (group - g0) * per[p];
                return true;
            }
            it -= n;
        }
    return false;
}

}  // namespace scft

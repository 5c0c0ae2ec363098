// Grouped launches of the refined solver across a batch of clouds.
//
// A grouped launch runs one kernel over many grids at once: the (cloud, level)
// grids of one step of the batch's V-cycle (every cloud's level-0 sweep, every
// cloud's level-1 residual, ...), clouds of any side.  The host describes each
// grid once in a GridDesc (operand pointers, side, cloud, and the first block
// of the grid in the launch's flattened 1-D block range); a block finds its
// grid by binary search over the descriptors' first blocks and runs the same
// body the single-grid kernel runs, with the grid's own block coordinates.
// Blocks of a cloud whose flags say it has converged return at once, so one
// captured iteration serves every cloud until the last one converges.
#pragma once

#include <cuda.h>

#include "common.cuh"

namespace pb {
namespace batch {

constexpr int kPtrs = 12;

// One grid of a grouped launch (64-byte aligned: the TMA maps are read in place).
struct alignas(64) GridDesc {
    CUtensorMap map[3];   // TMA maps (level-0 sweeps only)
    const void* ptr[kPtrs];  // operands, in the order of the launch kind
    int64_t n;            // grid side
    int64_t cloud;        // cloud index (its flags and scalars)
    int64_t block0;       // first block of this grid in the launch
    int64_t gx, gy, gz;   // the grid's own block grid (x fastest)
    int64_t aux[4];       // kind-specific integers
};

// Per-cloud flags (int[4] per cloud): first step, iterations done, active, unused.
constexpr int kFlagFirst = 0, kFlagIter = 1, kFlagActive = 2, kFlagStride = 4;
// Per-cloud scalars (double[8] per cloud) as the single-cloud FCG uses them.
constexpr int kScalStride = 8;
// Per-cloud loop control (double[2] per cloud): target ||r||^2, iteration cap.
constexpr int kCtrlStride = 2;

// The descriptor of block `b` of a grouped launch, and the block's coordinates
// within its own grid.  descs sorted by block0 ascending, descs[0].block0 == 0.
__device__ __forceinline__ const GridDesc& locate(const GridDesc* __restrict__ descs, int count, int64_t b,
                                                  int& bx, int& by, int& bz) {
    int lo = 0, hi = count - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (descs[mid].block0 <= b) lo = mid;
        else hi = mid - 1;
    }
    const GridDesc& d = descs[lo];
    const int64_t local = b - d.block0;
    bx = (int)(local % d.gx);
    by = (int)((local / d.gx) % d.gy);
    bz = (int)(local / (d.gx * d.gy));
    return d;
}

__device__ __forceinline__ bool cloud_active(const int* __restrict__ flags, int64_t cloud) {
    return flags[cloud * kFlagStride + kFlagActive] != 0;
}

}  // namespace batch
}  // namespace pb

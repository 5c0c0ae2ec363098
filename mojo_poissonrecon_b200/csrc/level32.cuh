// Padded FP32 level layout shared by the FP32 multigrid units.
//
// Side-n grid stored with a one-node ghost layer of zeros on every face, x
// offset 4, row pitch P (a multiple of 8 floats, so every row starts 32-byte
// aligned):
//   index(x, y, z) = ((z+1)*(n+2) + (y+1))*P + (x+4),  x,y,z in [-1, n].
// Ghost entries of every array (solution, right-hand side, residual, operator
// coefficients, prolongation weights) stay zero, so stencil sums and transfer
// operators need no bounds tests: an out-of-grid neighbour contributes zero.
#pragma once

#include <stdint.h>

#include "checked.cuh"

namespace pb {

struct Geom {
    int n;          // grid side
    int P;          // row pitch (floats)
    int64_t plane;  // (n+2)*P
    __host__ __device__ __forceinline__ int64_t at(int x, int y, int z) const {
        return checked_at(((int64_t)(z + 1) * (n + 2) + (y + 1)) * P + (x + 4), (int64_t)(n + 2) * plane,
                          kSitePadded);
    }
};

__host__ __device__ inline int pitch_of(int n) { return ((n + 5) + 7) & ~7; }
__host__ __device__ inline Geom geom(int n) { return Geom{n, pitch_of(n), (int64_t)(n + 2) * pitch_of(n)}; }
__host__ __device__ inline int64_t padded_size(int n) { return (int64_t)(n + 2) * geom(n).plane; }

}  // namespace pb

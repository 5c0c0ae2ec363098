// The checked build (nvcc -DPB_CHECKED -rdc=true; libpoisson_b200_checked.so).
//
// compute-sanitizer is not available where this library is tested, so the
// checked build stands in for its bounds checking: the padded-layout index
// helpers (Geom::at, fcg::Pad::at) and the guarded stores of the hot kernels
// test every index against its array's extent.  An index outside it records
// the first failure in one device word (site << 56 | the index's low 56 bits)
// and is replaced by index 0 or the store is skipped, so the kernel finishes
// without touching memory outside its arrays and the host reads the word
// (pb_check_status).  In the normal build the helpers compile to the plain
// index arithmetic and PB_GUARD to nothing.
#pragma once

#include <stdint.h>

namespace pb {

enum CheckSite : unsigned {
    kSitePadded = 1,      // a padded FP32 level index (Geom::at)
    kSitePad = 2,         // a padded index in the FCG passes (fcg::Pad::at)
    kSiteSweepStore = 3,  // the TMA sweep's output row
    kSiteFcgStore = 4,    // FCG pass 2: p, x (dense) and r32 (padded)
    kSiteProlong = 5,     // the FP32 prolongation's fine store
    kSiteRelax64 = 6,     // the FP64 red-black pass's store
};

#ifdef PB_CHECKED
extern __device__ unsigned long long g_check_word;

__device__ __forceinline__ bool check_index(int64_t i, int64_t size, unsigned site) {
    if (i >= 0 && i < size) return true;
    atomicCAS(&g_check_word, 0ull,
              ((unsigned long long)site << 56) | ((unsigned long long)i & ((1ull << 56) - 1)));
    return false;
}
// Guards the statement that follows: it runs only if i is inside [0, size).
#define PB_GUARD(i, size, site) if (::pb::check_index((int64_t)(i), (int64_t)(size), (site)))
#else
#define PB_GUARD(i, size, site)
#endif

// A padded index checked against the array's extent (device code of the
// checked build); elsewhere the index itself.
__host__ __device__ __forceinline__ int64_t checked_at(int64_t i, int64_t size, unsigned site) {
#if defined(PB_CHECKED) && defined(__CUDA_ARCH__)
    return check_index(i, size, site) ? i : 0;
#else
    (void)size;
    (void)site;
    return i;
#endif
}

}  // namespace pb

// Layout conversion on the device between the BUQ tiles of the C ABI (18x18 per
// block, memloc) and the compact device state (16x16 per block).  Used by
// bgf_set_state / bgf_get_state when the caller's host arrays are pinned: the
// whole tile arrays then cross the host link by DMA and the interior cells are
// picked out here, instead of by the host.
#include <cuda_runtime.h>

#include <algorithm>

#include "bgf_internal.h"

namespace bgf {
namespace layout {

__device__ __forceinline__ int interior18(int c) { return ((c >> 4) + 1) * 18 + (c & 15) + 1; }

// tiles: three fields (h, u, v) of nb tiles each, one after the other.
template <class T> __global__ void tiles_to_compact_kernel(const T* __restrict__ tiles, T* h, T* u, T* v, size_t nb)
{
    const size_t n = nb * 256;
    for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x) {
        const size_t ib = q >> 8;
        const size_t s = ib * 324 + interior18((int)(q & 255));
        h[q] = tiles[s];
        u[q] = tiles[nb * 324 + s];
        v[q] = tiles[2 * nb * 324 + s];
    }
}

// tiles: four fields (zs, h, u, v) of nb tiles each, zero-filled by the caller; the
// interior cells of the active blocks are written, zs = zb + h.
template <class T>
__global__ void compact_to_tiles_kernel(const int* __restrict__ active, const T* __restrict__ h,
                                        const T* __restrict__ u, const T* __restrict__ v, const T* __restrict__ zb,
                                        T* tiles, size_t nb)
{
    const size_t ib = active[blockIdx.x];
    const int c = threadIdx.x;
    const size_t q = ib * 256 + c;
    const size_t d = ib * 324 + interior18(c);
    const T hv = h[q];
    tiles[d] = zb[d] + hv;
    tiles[nb * 324 + d] = hv;
    tiles[2 * nb * 324 + d] = u[q];
    tiles[3 * nb * 324 + d] = v[q];
}

template <class T> void launch_tiles_to_compact(const T* tiles, T* h, T* u, T* v, size_t nb, cudaStream_t st)
{
    const size_t n = nb * 256;
    const int grid = (int)std::min<size_t>((n + 255) / 256, 148 * 16);
    tiles_to_compact_kernel<T><<<grid, 256, 0, st>>>(tiles, h, u, v, nb);
}

template <class T>
void launch_compact_to_tiles(const int* active, int nblk, const T* h, const T* u, const T* v, const T* zb, T* tiles,
                             size_t nb, cudaStream_t st)
{
    if (nblk > 0) compact_to_tiles_kernel<T><<<nblk, 256, 0, st>>>(active, h, u, v, zb, tiles, nb);
}

#define BGF_LAYOUT_INST(T)                                                                                       \
    template void launch_tiles_to_compact<T>(const T*, T*, T*, T*, size_t, cudaStream_t);                      \
    template void launch_compact_to_tiles<T>(const int*, int, const T*, const T*, const T*, const T*, T*, size_t, \
                                             cudaStream_t);
BGF_LAYOUT_INST(float)
BGF_LAYOUT_INST(double)

}  // namespace layout
}  // namespace bgf

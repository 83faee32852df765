// Gauge time series on the device: the reference's time-series output
// (pointoutputstep / storeTSout, src/Mainloop.cu:359-500) records h, zs, u and v at
// every output node after every step into a device store that the host flushes when
// it is full.  Here one launch after each step's corrector records all gauges of a
// handle, or of every scenario of a pool, into a ring of samples; the host drains
// the ring (bgf_read_gauges / bgf_pool_read_gauges) while later steps run.
#include <cuda_runtime.h>

#include "bgf_flow.cuh"
#include "bgf_internal.h"

namespace bgf {

// One sample per launch: gauge g of row k % cap.  A gauge whose scenario did not
// take this step (finished, or not live) records a NaN time.  One CTA, so the
// sample counter advances once per launch after every gauge is written.
template <class T>
__global__ void __launch_bounds__(256) gauge_kernel(DevModel<T> m, GaugeRingDev<T> r, int parity)
{
    const unsigned long long k = *r.count;
    const size_t row = (size_t)(k % (unsigned long long)r.cap) * r.n;
    for (int g = threadIdx.x; g < r.n; g += blockDim.x) {
        const int sc = r.scen ? r.scen[g] : 0;
        const TimeState ts = m.time[2 * sc + parity];
        const TimeState nt = m.time[2 * sc + (parity ^ 1)];
        const bool live = !ts.done && ts.totaltime < ts.endtime && ts.nstep < ts.maxsteps;
        T* o = r.vals + (row + g) * 4;
        if (live) {
            const int c = r.cell[g];  // block slot * 256 + j * 16 + i
            const int ib = c >> 8, j = (c >> 4) & 15, i = c & 15;
            const T hv = m.h[nt.cur][c];
            const T zb = m.zb[(size_t)ib * 324 + hi18(i, j)];
            if (m.datum) {
                // split precision: the state holds deviations from the block's datum
                const double D = (double)m.datum[ib];
                o[0] = (T)(D + (double)hv);
                o[1] = (T)((double)zb + D + (double)hv);
            } else {
                o[0] = hv;
                o[1] = zb + hv;  // zs as RecalculateZs leaves it
            }
            o[2] = m.u[nt.cur][c];
            o[3] = m.v[nt.cur][c];
            r.time[row + g] = nt.totaltime;
        } else {
            r.time[row + g] = __longlong_as_double(0x7ff8000000000000LL);
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) *r.count = k + 1;
}

template <class T> void launch_gauges(const DevModel<T>& m, const GaugeRingDev<T>& r, int parity, cudaStream_t st)
{
    gauge_kernel<T><<<1, 256, 0, st>>>(m, r, parity);
}

template void launch_gauges<float>(const DevModel<float>&, const GaugeRingDev<float>&, int, cudaStream_t);
template void launch_gauges<double>(const DevModel<double>&, const GaugeRingDev<double>&, int, cudaStream_t);

}  // namespace bgf

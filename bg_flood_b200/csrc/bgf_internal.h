// Internal declarations shared by the C-ABI layer and the kernel launchers.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

namespace bgf {

struct TimeState;
struct SegDev;
template <class T> struct DevModel;
template <class T> struct StepParams;
template <class T> struct AmrDev;
template <class T> struct GaugeRingDev;

// Gauge sampling after a step (bgf_gauge.cu), built once: it does no arithmetic
// beyond zs = zb + h.
template <class T> void launch_gauges(const DevModel<T>& m, const GaugeRingDev<T>& r, int parity, cudaStream_t st);

// Kernel launchers, built twice (bgf_flow.cu, bgf_amr.cu): "exact" reproduces the reference
// CPU arithmetic bit for bit, "fast" trades the last bits for speed.
#define BGF_DECLARE_LAUNCHERS                                                                                   \
    template <class T> cudaError_t configure_kernels();                                                        \
    template <class T>                                                                                         \
    void launch_flux(const DevModel<T>& m, const StepParams<T>& p, int engine, int parity, cudaStream_t st,    \
                     int grid);                                                                                \
    template <class T>                                                                                         \
    void launch_update(const DevModel<T>& m, const StepParams<T>& p, int engine, int parity, cudaStream_t st,  \
                       int grid);                                                                              \
    template <class T>                                                                                         \
    void launch_initdt(const DevModel<T>& m, const StepParams<T>& p, int cur, unsigned long long* out,         \
                       cudaStream_t st);                                                                       \
    template <class T> void launch_volume(const DevModel<T>& m, T delta0, int cur, double* out, cudaStream_t st); \
    template <class T> cudaError_t configure_amr_kernels();                                                    \
    template <class T>                                                                                         \
    int launch_amr_stage(const DevModel<T>& m, const AmrDev<T>& a, const StepParams<T>& p, int engine,         \
                         int parity, int stage, int minlev, int maxlev, cudaStream_t st);                      \
    template <class T> int launch_bed_init(const DevModel<T>& m, const StepParams<T>& p, T* zb, T* gx, T* gy,  \
                                           cudaStream_t st);
namespace exact {
BGF_DECLARE_LAUNCHERS
}
namespace fast {
BGF_DECLARE_LAUNCHERS
}

// Refinement-pass kernels (bgf_adapt.cu), built once without FMA contraction.
namespace adapt {
template <class T> struct AdaptDev;
template <class T> void launch_criteria(const DevModel<T>& m, const T* z, int stride324, int kind, T a1, T a2,
                                        uint8_t* flags, cudaStream_t st);
template <class T> void launch_zs(const DevModel<T>& m, T* zs, int cur, cudaStream_t st);
struct TargetMapDev;
template <class T>
void launch_target_level(const DevModel<T>& m, const TargetMapDev& g, double xo, double yo, double dx0,
                         uint8_t* refine, uint8_t* coarsen, cudaStream_t st);
// Old-mesh halos, then the children of refined blocks (refine) and the merged
// quads (nquads > 0, quads[4k..4k+3] on the device); returns the launch count.
template <class T> int launch_children(const DevModel<T>& m, const AdaptDev<T>& a, int cur, T* cf, uint8_t* rainmask,
                                       const int* quads, int nquads, bool refine, cudaStream_t st);
template <class T>
void launch_hgrad(const DevModel<T>& m, const T* zs, int cur, double eps, double hthr, double gthr, double dx0,
                  uint8_t* refine, uint8_t* coarsen, cudaStream_t st);
template <class T> void launch_bed(const DevModel<T>& m, const AdaptDev<T>& a, const StepParams<T>& p, int cur, T* zb,
                                   double xo0, double yo0, const double* bxo, const double* byo, double mask,
                                   uint8_t* rainmask, cudaStream_t st);

// Device side of the sanity pass and the table rebuild (bgf_adapt_dev.cu).
struct DevTables {
    const int* active;
    int nblk, nblkmem;
    const int* level;
    const int* nbr;        // [8][nblkmem]
    const double *xo, *yo;
};
struct DevAdaptScratch {
    int* pos;              // position in the active list, -1 when inactive
    uint8_t *parent, *gone;
    int *fr, *fq, *fk, *ff;  // refine, parent, kept flags per active position; free flag per id
    int *sr, *sq, *sk, *sf;  // their exclusive prefix sums
    int* tiles;            // scan tile totals
    int* counts;           // refined, parents, kept, free
    int* avail;            // free ids in ascending order
    int *nact, *nlev;      // new active list and levels
    double *nxo, *nyo;     // new origins
    int* reflist;          // refined blocks and their children, 4 ids each
    int* grids;            // per-level block index grids
    int *bx, *by;          // block coordinates in the new mesh
    int* nnbr;             // new neighbour tables [8][nblkmem]
};
struct GridSpec {
    int nlev;              // levels 0..nlev-1
    int off[16], w[16], h[16];
    long long total;
};
void scan_excl(const int* in, int* out, int n, int* tile_sum, int* total, cudaStream_t st);
int dev_sanity(const DevTables& t, const DevAdaptScratch& s, uint8_t* refine, uint8_t* coarsen, int minlevel,
               int maxlevel, int allow, int fill_coarsen, double dx, cudaStream_t st);
int dev_tables_count(const DevTables& t, const DevAdaptScratch& s, const uint8_t* refine, const uint8_t* coarsen,
                     cudaStream_t st);
int dev_tables_build(const DevTables& t, const DevAdaptScratch& s, const uint8_t* refine, const uint8_t* coarsen,
                     double dx, int dbl, int nkeep, int nnew, int* child, int* quads, const GridSpec& gs, int* err,
                     cudaStream_t st);
}  // namespace adapt

// Tile <-> compact layout kernels (bgf_layout.cu) for pinned host arrays.
namespace layout {
template <class T> void launch_tiles_to_compact(const T* tiles, T* h, T* u, T* v, size_t nb, cudaStream_t st);
template <class T>
void launch_compact_to_tiles(const int* active, int nblk, const T* h, const T* u, const T* v, const T* zb, T* tiles,
                             size_t nb, cudaStream_t st);
}  // namespace layout

// Records the text returned by bgf_last_error() for this thread.
void set_last_error(const std::string& msg);


}  // namespace bgf

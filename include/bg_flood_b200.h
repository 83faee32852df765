/*
 * bg_flood_b200.h -- C ABI of the B200 implementation of BG_Flood's explicit
 * shallow-water flow step on the block-uniform quadtree (BUQ).
 *
 * The library is a drop-in for the flow step that BG_Flood's time loop calls
 * once per step, FlowGPU / FlowCPU (src/FlowGPU.cu:14-315, src/FlowCPU.cu:15-253,
 * called from src/Mainloop.cu:43-57).  Every entry point takes plain pointers and
 * sizes, returns a status code (BGF_OK == 0) and never exits the process.
 *
 * Data layout at this boundary is the reference's own: each block is an 18x18
 * tile of 16x16 cells plus a one-cell halo, cell (i, j) of block ib at index
 * (i + 1) + (j + 1) * 18 + ib * 324 (memloc, src/MemManagement.cu:37-40).
 * Block tables are the reference BlockP arrays (src/Arrays.h:234-250).
 *
 * Precision follows the reference's "doubleprecision" key: with
 * bgf_param.doubleprecision == 0 all field pointers are float*, otherwise
 * double*.  Simulated time, dt and the output-time clamp are always double.
 *
 * Thread safety: a handle may be used from one host thread at a time; distinct
 * handles are independent.  All work of a handle is ordered on its CUDA stream.
 */
#ifndef BG_FLOOD_B200_H
#define BG_FLOOD_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------ status codes */
enum {
    BGF_OK = 0,
    BGF_EINVAL = 1,        /* bad argument or unsupported configuration        */
    BGF_ECUDA = 2,         /* a CUDA runtime call failed (see bgf_last_error)   */
    BGF_ENOMEM = 3,        /* device allocation failed                          */
    BGF_EDT_UNDERFLOW = 4, /* dt fell below dtmin before endtime (CrashDetection) */
    BGF_ENAN = 5,          /* non-finite h, u or v at the start of a step: the  *
                            * step's dt minimum is zeroed, the scenario stops   */
    BGF_ESTATE = 6,        /* call out of order (e.g. step before state upload) */
    BGF_EBUDGET = 7,       /* serving: request exceeds the HBM budget           */
    BGF_ETIMEOUT = 8,      /* bounded wait gave up                              */
    BGF_ENOKERNEL = 9      /* the CUDA kernels are not available on this device */
};

/* ------------------------------------------------------------ parameters */
/* Subset of the reference Param class (src/Param.h:10-239) used by the flow
 * step, with the reference's member names, meanings and defaults
 * (bgf_param_default fills them). */
typedef struct bgf_param {
    double g;             /* gravity, 9.81                                    */
    double eps;           /* drying height, 1e-4                              */
    double dt;            /* "dt" key (boundary filter/relax factors), 0      */
    double CFL;           /* 0.5                                              */
    double theta;         /* minmod limiter parameter, 1.3                    */
    double cf;            /* uniform friction coefficient, 1e-4               */
    double dx;            /* level-0 resolution                               */
    double delta;         /* resolution used by the solver (== dx, Cartesian) */
    double xo, yo;        /* domain origin                                    */
    double lat;           /* latitude for the Coriolis term, 0                */
    double zsinit;        /* NaN if unset                                     */
    double zsoffset;      /* 0                                                */
    double bndtaper;      /* 0                                                */
    double bndrelaxtime;  /* 3600                                             */
    double bndfiltertime; /* 60                                               */
    double inittime;      /* 0                                                */
    double dtmin;         /* 5e-4                                             */
    double dtinit;        /* -1                                               */
    double mask;          /* 9999                                             */
    int engine;           /* 1 HLLC (Buttinger-Kreuzhuber), 2 Kurganov        */
    int frictionmodel;    /* -1 Manning, 0 quadratic, 1 smart                 */
    int ForceMassConserve;/* 0                                                */
    int wetdryfix;        /* 1                                                */
    int conserveElevation;/* 0 (only 0 is supported)                          */
    int doubleprecision;  /* 0 float state, 1 double state                    */
    int minlevel, maxlevel, initlevel;
    int aoibnd;           /* boundary type of the remainder segment, 0 wall   */
    int rainbnd;          /* 0: no rain on the two outermost cell rows        */
    int GPUDEVICE;        /* CUDA device ordinal                              */
    int fastmath;         /* 0: kernels reproduce the reference CPU arithmetic
                             bit for bit (no FMA contraction, IEEE division and
                             square root); 1: FMA contraction and approximate
                             division / square root (results within the
                             tolerances of the parity tests)                   */
    int splitprecision;   /* 1 (with doubleprecision 0, single-level meshes):
                             FP32 state stored as deviations from a per-block
                             datum depth (whole metres, FP64 on the host), for
                             deep water; field pointers at this boundary are
                             then double*.  No counterpart in the reference.  */
} bgf_param;

/* Reference Loop<T> members the step reads and writes (src/Arrays.h:359-404). */
typedef struct bgf_loop {
    double nextoutputtime;
    double dt;        /* in: previous dt; out: dt of this step               */
    double dtmax;     /* in: previous dt (or initdt); out: dt of this step   */
    double totaltime; /* in: time at the start of the step                   */
} bgf_loop;

/* Reference BlockP<T> tables (src/Arrays.h:234-250).  xo/yo are float when
 * doubleprecision == 0, double otherwise (same rule as the fields). */
typedef struct bgf_blockp {
    int nblk;                   /* active blocks                              */
    const int* active;          /* nblk active block ids                      */
    const int* level;           /* nblkmem                                    */
    const int *BotLeft, *BotRight, *TopLeft, *TopRight;
    const int *LeftBot, *LeftTop, *RightBot, *RightTop;
    const void *xo, *yo;        /* block origins relative to Param.xo/yo     */
} bgf_blockp;

/* Reference EvolvingP<T> (src/Arrays.h:67-77): four BUQ arrays. */
typedef struct bgf_evolving {
    void *zs, *h, *u, *v;
} bgf_evolving;

typedef struct bgf_handle bgf_handle;

/* Fills p with the reference defaults (src/Param.h). */
void bgf_param_default(bgf_param* p);
const char* bgf_strerror(int status);
/* Text of the last CUDA error seen by this thread, or "". */
const char* bgf_last_error(void);
/* 1 when the sm_100a kernels can run on device `dev` (the library was built for sm_100a). */
int bgf_device_supported(int dev);

/* Creates a handle holding device memory for nblkmem blocks.  stream may be
 * NULL (the handle creates its own non-blocking stream). Replaces SetupGPU /
 * AllocateGPU (src/Setup_GPU.cu:15-36, src/MemManagement.cu:804). */
int bgf_create(const bgf_param* p, int nblkmem, void* stream, bgf_handle** out);
int bgf_destroy(bgf_handle* h);

/* Block tables (BlockP).  Replaces the block part of CopytoGPU
 * (src/Setup_GPU.cu:196-375). */
int bgf_set_blocks(bgf_handle* h, const bgf_blockp* blocks);

/* Bed elevation and per-cell inputs in BUQ layout (nblkmem tiles).
 * zb, dzbdx, dzbdy: with dzbdx/dzbdy NULL, only the interior of zb is read and
 *     the library prepares the bed on the device as the reference does at
 *     initialisation (src/Testing.cu:583-588, src/InitialConditions.cu:140-144):
 *     halo fill across levels, gradients, halo gradients, linear refinement of
 *     the halos next to coarser blocks, halo gradients again.  With both given,
 *     zb's halo and the gradients (incl. halo cells) are used as they are.
 * cf: friction coefficient per cell, NULL for the uniform Param.cf.
 * activeCell: rain mask per cell (int), NULL for all ones. */
int bgf_set_bed(bgf_handle* h, const void* zb, const void* dzbdx, const void* dzbdy, const void* cf,
                const int* activeCell);

/* Boundary segment (reference bndsegment, src/Forcing.h:120-144): type 0 wall,
 * 1 Neumann, 2 Dirichlet water level, 3 absorbing 1D; an optional uniform
 * water-level series (n points of time t and level wl); and for each side
 * (0 left, 1 right, 2 top, 3 bot) the blocks it applies to.  Segments are
 * applied in the order they are added, as FlowbndFlux does per segment
 * (src/Boundary.cu:108-195). */
int bgf_add_bnd_segment(bgf_handle* h, int type, int n, const double* t, const double* wl,
                        const int nblk_side[4], const int* const blk_side[4]);

/* Uniform rain series in mm/h (reference Forcing.Rain with unidata). */
int bgf_set_rain_series(bgf_handle* h, int n, const double* t, const double* rain_mmh);

/* Uploads / downloads the evolving state (EvolvingP) in BUQ layout.  zs is
 * ignored on upload (the step recomputes zs = zb + h everywhere, as
 * RecalculateZs does, src/Halo.cu:72-107).  On download the whole nblkmem
 * tiles of each non-NULL field are written: the 16x16 interior of the active
 * blocks holds the state, every other entry is 0.  When all arrays are
 * page-locked (cudaMallocHost / cudaHostRegister), the tiles cross the host
 * link by DMA and the interiors are picked out on the device; otherwise the
 * host converts through a pinned staging buffer. */
int bgf_set_state(bgf_handle* h, const bgf_evolving* ev);
int bgf_get_state(bgf_handle* h, bgf_evolving* ev);

/* initdt (src/Mainloop.cu:515-554): writes loop->dtmax. */
int bgf_init_dt(bgf_handle* h, bgf_loop* loop);

/* One flow step, the equivalent of FlowGPU(XParam, XLoop, XForcing, XModel)
 * (src/FlowGPU.cu:14-315) with the dt reduction of CalctimestepGPU
 * (src/Advection.cu:549-620): reads loop->{totaltime, dt, dtmax,
 * nextoutputtime}, writes loop->dt and loop->dtmax.  Like the reference it
 * leaves loop->totaltime to the caller.  Synchronises the stream (dt is
 * returned to the host). */
int bgf_flow_step(bgf_handle* h, bgf_loop* loop);

/* Device-resident time loop: repeats {flow step; totaltime += dt} while
 * totaltime < endtime, at most maxsteps steps, without host synchronisation
 * between steps (steps are captured in CUDA graphs).  nextoutputtime in loop
 * clamps dt exactly like the reference; it is advanced by outputtimestep
 * (if > 0) each time it is reached.  On return loop holds the final state
 * of the time loop and *nsteps the number of steps taken.
 * Returns BGF_EDT_UNDERFLOW if dt < dtmin before endtime (CrashDetection,
 * src/Mainloop.cu:648-719). */
int bgf_run(bgf_handle* h, bgf_loop* loop, double endtime, double outputtimestep, int maxsteps,
            int* nsteps);

/* Sum of h * delta_l^2 over active interior cells, accumulated in double on the
 * device (the volume total of the reference tests, src/Testing.cu:1111-1129). */
int bgf_volume(bgf_handle* h, double* volume);

/* Number of kernel launches this handle has issued so far. */
int64_t bgf_kernel_launches(bgf_handle* h);
/* Per-kernel timing of bgf_flow_step: when on, CUDA events recorded on the
 * handle's stream around the flux (predictor) and update (corrector) kernels
 * accumulate their device times; turning it on resets the totals. */
int bgf_set_profiling(bgf_handle* h, int on);
int bgf_kernel_timing(bgf_handle* h, double* flux_ms, double* update_ms, int64_t* steps);
/* CTAs of the two fused single-level kernels: 0 (default) launches one per
 * active block; a smaller count makes each CTA loop over blocks (a persistent
 * launch).  Results do not depend on it. */
int bgf_set_grid(bgf_handle* h, int grid);
/* Thread layout of the two fused single-level kernels: 2 (default) gives each
 * thread two vertically adjacent cells of a block (128 threads per block, paired
 * FP32 arithmetic in the fast-math build), 1 one cell per thread (256 threads per
 * block), 3 the two-cell arithmetic in persistent CTAs whose fifth warp stages the
 * next block's tile into shared memory with bulk asynchronous copies while the
 * other four compute (the grid then defaults to the CTAs resident on all SMs).
 * The exact build gives the same results bit for bit with each; split-precision
 * handles always use layout 1.  No counterpart in the reference. */
int bgf_set_kernel_layout(bgf_handle* h, int cells_per_thread);

/* ------------------------------------------------------------ gauges */
/* Gauges, the reference's time-series output nodes (TSnodesout; pointoutputstep /
 * storeTSout, src/Mainloop.cu:359-500): after every step the library records, on
 * the device, the step's time and h, zs, u, v at each gauge cell (block id, i, j,
 * 0 <= i, j < 16, as the reference's TSnodesout block/i/j).  zs is zb + h.  The
 * samples wait in a device ring of 4096 steps; bgf_run drains it after every
 * batch of graphs, bgf_read_gauges drains it and hands out the samples in step
 * order.  After more than 4096 single bgf_flow_step calls without a read the oldest
 * samples are overwritten and counted in *lost.  Setting gauges replaces earlier
 * ones and drops their unread samples; bgf_set_blocks (or a refinement pass) clears
 * them, since they name block ids of the old mesh. */
int bgf_set_gauges(bgf_handle* h, int n, const int* block, const int* i, const int* j);
/* Up to max_samples samples: times[s * n + g], values[(s * n + g) * 4 + q] with q
 * = h, zs, u, v; *nsamples receives the number returned, *lost (optional) the
 * samples overwritten so far. */
int bgf_read_gauges(bgf_handle* h, int max_samples, double* times, double* values, int* nsamples, int64_t* lost);
/* Device time (ms) and kernel launches of the last bgf_run (events around its graphs). */
int bgf_run_timing(bgf_handle* h, double* gpu_ms, int64_t* launches);

/* ------------------------------------------------------------ allocation-free step */
/* No counterpart in the reference.  One flow step (the two kernels of
 * bgf_flow_step) for callers that cannot allocate device memory once they are
 * running -- e.g. a service that reserves its GPU memory pool at start-up and
 * treats any later cudaMalloc as a fault, or a host model that owns all its
 * device arrays (like BG_Flood's Model<T>) and may not trigger the device-wide
 * synchronisation of cudaMalloc / cudaFree.  It calls no allocating routine: the
 * caller passes device pointers to its inputs and outputs, and the kernels'
 * scratch (flux divergence, dt reduction, time slots, boundary running means)
 * lives in one static device array sized for BGF_NOALLOC_MAX_BLOCKS blocks in
 * double precision (about 3.3 MB), which every GPU that loads the library keeps
 * until the process exits.
 * - The first call on a device finds the array's device address, writes its
 *   constant part and clears the boundary running means; make that first call
 *   before any stream capture.  The set-up is cached per device for the life of
 *   the process and does not survive a cudaDeviceReset.  The caller's current
 *   device is restored before the call returns.
 * - Every call shares the array and it keeps the last call's contents.  The time
 *   slot, the dt minimum and the error word are rewritten by each call.  The
 *   absorbing-boundary running means (the reference's per-side qmean, carried
 *   from step to step) persist in the array between calls; set reset_means = 1
 *   on the first step of a run to clear them.  Calls whose GPU work overlaps
 *   (other streams, other threads) race on the array, and two runs interleaved
 *   step by step share one set of running means.
 * - nblkmem > BGF_NOALLOC_MAX_BLOCKS is rejected with BGF_EINVAL.
 * - Single-level meshes only (a cross-level neighbour gives BGF_EINVAL), FP32 or
 *   FP64 state, uniform friction coefficient, no rain, no rivers, no split
 *   precision (splitprecision = 1 and conserveElevation != 0 are rejected).
 *   Boundary sides carry a type (0 wall, 1 Neumann, 2 Dirichlet at the constant
 *   level Param.zsinit, or 0 when zsinit is NaN -- the reference's level for a
 *   segment without a water-level series -- 3 absorbing 1D) or -1 for a side
 *   with a neighbour; time series are not taken.
 * - active must hold nblk distinct ids < nblkmem and nbr ids < nblkmem: the
 *   kernels index with them unchecked.
 * - zb must start on a 16-byte boundary (any cudaMalloc result does): the bed
 *   tiles are copied in 16-byte pieces; BGF_EINVAL otherwise.
 * State layout here is the kernels' own: 256 values per block slot, cell
 * (i, j) at j * 16 + i; the output arrays must not alias the inputs.
 * Synchronises `stream` (dt is returned to the host, as bgf_flow_step does). */
#define BGF_NOALLOC_MAX_BLOCKS 512
typedef struct bgf_noalloc_args {
    int nblk, nblkmem;
    const int* active;    /* device: nblk active block ids                     */
    const int* level;     /* device: nblkmem                                   */
    const int* nbr;       /* device: [8][nblkmem] LeftBot, LeftTop, RightBot,
                             RightTop, BotLeft, BotRight, TopLeft, TopRight    */
    const int* bndtype;   /* device: [nblkmem][4] side type (left, right, top, bot) */
    const void *zb, *dzbdx, *dzbdy; /* device BUQ tiles, 324 per block slot    */
    const void *h_in, *u_in, *v_in; /* device, 256 per block slot              */
    void *h_out, *u_out, *v_out;    /* device, 256 per block slot              */
    int reset_means;      /* 1: clear the absorbing-boundary running means
                             before this step (first step of a run)           */
} bgf_noalloc_args;
int bgf_flow_step_noalloc(const bgf_param* p, const bgf_noalloc_args* args, bgf_loop* loop, void* stream);

/* ------------------------------------------------------------ mesh helpers */
/* Uniform BUQ mesh as InitBlockxoyo / InitBlockneighbours build it
 * (src/Mesh.cu:257-433): nbx*nby candidate blocks in row-major order, blocks
 * whose present[] entry is 0 are skipped (masked), ids are assigned in order,
 * neighbours are matched by position and default to the block itself at the
 * domain edge.  Outputs are sized nbx*nby; returns the block count in *nblk.
 * xo/yo (double) are the block origins (first cell centre) relative to the
 * domain origin, evaluated in the state precision as the reference stores them
 * (float unless doubleprecision). */
int bgf_mesh_uniform(int nbx, int nby, double levdx, const uint8_t* present, int* nblk, int* level,
                     int* nbr8, double* xo, double* yo, int doubleprecision);

/* ------------------------------------------------------------ gridded rain */
/* Rain rate (mm/h) as a gridded series: nt >= 2 frames of nx*ny float nodes from
 * (xo, yo) (absolute coordinates) with spacings dx, dy, frame k at time
 * to + k*dt, frames row-major with row 0 at yo (frames[k*nx*ny + j*nx + i]) --
 * the reference's Rain DynForcingP read from a netCDF file, whose reader is not
 * part of this library.  At the start of each step the two frames around the
 * time (index clamped to [0, nt-2], Forcingthisstep, src/Updateforcing.cu:87-125)
 * are interpolated in time at the grid nodes, then bilinearly at the cell
 * centre as the reference's CPU rain does (interp2BUQ, AddrainforcingImplicitCPU,
 * src/GridManip.cu:540-575, src/Updateforcing.cu:530-580); the reference's GPU
 * path samples a texture instead.  Replaces a uniform series (and
 * bgf_set_rain_series replaces the map).  Not supported in pools. */
int bgf_set_rain_map(bgf_handle* h, int nx, int ny, double xo, double yo, double dx, double dy, int nt, double to,
                     double dt, const float* frames);

/* ------------------------------------------------------------ rivers */
#define BGF_MAX_RIVERS 64
/* A river: discharge q(t) (m^3/s, n >= 2 samples, increasing times) spread over
 * the cells whose box overlaps [xstart, xend] x [ystart, yend] (absolute
 * coordinates, as the reference's "river = file, xstart, xend, ystart, yend").
 * The discharge area is computed from the handle's blocks as InitRivers does
 * (src/InitialConditions.cu:336-420) and written to *area; a river that
 * overlaps no cell (area 0) is not added, as the reference drops it.  Each
 * stage of a step adds q(t)/area to the depth tendency of those cells
 * (AddRiverForcing / InjectManyRiversGPU, src/Updateforcing.cu:146-300), t
 * being the start of the step.  Call after bgf_set_blocks; at most
 * BGF_MAX_RIVERS rivers.  The area is kept when a refinement pass changes the
 * mesh, as in the reference. */
int bgf_add_river(bgf_handle* h, double xstart, double xend, double ystart, double yend, int n, const double* t,
                  const double* q, double* area);

/* ------------------------------------------------------------ input files and set-up */
/* A regular grid of nx*ny nodes from (xo, yo) with spacings dx, dy, values
 * row-major with row 0 at yo: the reference's StaticForcingP<float>
 * (src/Forcing.h), as the bathymetry is held after reading. */
typedef struct bgf_grid {
    int nx, ny;
    double xo, yo, dx, dy, xmax, ymax;
    const float* val;
} bgf_grid;

/* Header of an ESRI ASCII grid, as readbathyASCHead (src/ReadForcing.cu:2067-2176)
 * reads it: the first six non-empty lines, "key value" split on blanks (or tabs),
 * keys ncols, nrows, cellsize, xllcenter, yllcenter, xllcorner, yllcorner
 * (case-sensitive).  When yllcenter or xllcorner is present both origins move
 * by half a cell, as in the reference.  Errors (file missing, header short or
 * unreadable, ncols/nrows/cellsize absent) return BGF_EINVAL with the reason in
 * bgf_last_error; the reference exits or loops there instead. */
int bgf_read_asc_head(const char* path, int* nx, int* ny, double* dx, double* xo, double* yo, double* grdalpha);
/* Values of an ESRI ASCII grid, as readbathyASCzb (src/ReadForcing.cu:2186-2220):
 * six raw lines skipped, then nx*ny numbers, the first file row stored as the
 * last (northern) row of val.  NODATA values are kept as numbers, as in the
 * reference.  Too few values or a non-number return BGF_EINVAL. */
int bgf_read_asc(const char* path, int nx, int ny, float* val);
/* Presence of the nbx*nby candidate blocks of a uniform level mesh with cell
 * size levdx from (xo, yo), as CalcInitnblk / InitBlockxoyo (src/Mesh.cu:36-120,
 * 257-347) decide it: a block is dropped when all its cell centres have a
 * bilinear bed value >= mask.  present is row-major (by, bx); *nblk counts kept. */
int bgf_mask_blocks(const bgf_grid* g, int nbx, int nby, double xo, double yo, double levdx, double mask,
                    uint8_t* present, int* nblk);
/* Bed of every block interpolated from the grid (interp2BUQ,
 * src/GridManip.cu:380-575: bilinear when the block's cells are not coarser than
 * the grid, else the mean of the grid nodes in the cell), then the domain-edge
 * cells set from their inner neighbours (setedges, src/GridManip.cu:222-330).
 * Tables as bgf_set_blocks takes them (blocks 0..nblk-1, nbr8 per block, xo/yo
 * relative to the domain origin (xo, yo)); dx is the level-0 cell size.  The
 * arithmetic follows the model precision (float unless doubleprecision).  zb is
 * nblk*324 doubles: interior cells are written, halo cells are left as given. */
int bgf_interp_bathy(const bgf_grid* g, int nblk, const int* level, const int* nbr8, const double* bxo,
                     const double* byo, double xo, double yo, double dx, int doubleprecision, double* zb);

/* ------------------------------------------------------------ batched scenario pool */
/* No counterpart in the reference, which runs one scenario per process.  A pool
 * holds device memory for nblk_pool block slots shared by up to max_scenarios
 * independent scenarios (same engine, precision and kernel variant; single-level
 * meshes).  Every pool step is one launch pair over all admitted scenarios; each
 * scenario keeps its own parameters, dt (a per-scenario CFL minimum), time,
 * output times, end time and step budget, so its results are those it has when
 * run alone.  Steps run in CUDA graphs. */
typedef struct bgf_pool bgf_pool;
/* track_hmax: keep the running maximum depth of every cell. */
int bgf_pool_create(const bgf_param* p, int nblk_pool, int max_scenarios, int track_hmax, void* stream,
                    bgf_pool** out);
int bgf_pool_destroy(bgf_pool* pool);
/* Copies the scenario prepared in handle h (blocks, bed, state, segments, rain,
 * parameters) into free block slots; loop is its time-loop state (after
 * bgf_init_dt).  BGF_EBUDGET when the pool has too few free block or scenario
 * slots.  *slot identifies the scenario in the pool. */
int bgf_pool_admit(bgf_pool* pool, bgf_handle* h, const bgf_loop* loop, double endtime, double outputtimestep,
                   int maxsteps, int* slot);
/* Copies the scenario's state back into its handle, writes its loop state and
 * step count, and frees its slots. */
int bgf_pool_retire(bgf_pool* pool, int slot, bgf_loop* loop, int* nsteps);
/* Runs pool steps until every admitted scenario has finished or maxsteps steps
 * ran; *nlive receives the number still running. */
int bgf_pool_run(bgf_pool* pool, int maxsteps, int* nlive);
/* status: 0 running, 1 finished (end time or step budget), 2 dt underflow,
 * 3 non-finite state (the scenario stops; see BGF_ENAN). */
int bgf_pool_query(bgf_pool* pool, int slot, bgf_loop* loop, int* status, int64_t* nsteps);
/* Interior depth (and running maximum depth, if tracked) of a scenario's blocks
 * in its active order, 256 values per block. */
int bgf_pool_get_depth(bgf_pool* pool, int slot, void* h, void* hmax);
/* Device time (ms) and pool steps of the last bgf_pool_run; free block slots. */
/* Gauges of a pooled scenario: block is the index in the scenario's active order
 * (0 .. nblk-1), i, j the cell.  Every pool step records them on the device
 * (bgf_set_gauges); bgf_pool_run drains the ring after each batch, and
 * bgf_pool_read_gauges hands out the scenario's samples collected so far, in step
 * order, without touching the device (same layout as bgf_read_gauges).  Unread samples of a retired scenario go with it to
 * its handle (bgf_read_gauges).  No counterpart in the reference. */
int bgf_pool_set_gauges(bgf_pool* P, int slot, int n, const int* block, const int* i, const int* j);
int bgf_pool_read_gauges(bgf_pool* P, int slot, int max_samples, double* times, double* values, int* nsamples);
int bgf_pool_timing(bgf_pool* pool, double* gpu_ms, int64_t* steps, int* free_blocks);
/* bgf_pool_run in two halves, so that the host can work while the pool steps run.
 * bgf_pool_run_async applies pending admissions and retirements and enqueues
 * maxsteps (<= 512) pool steps plus a copy of the time slots, then returns;
 * bgf_pool_wait waits for them, refreshes what bgf_pool_query reports, drains the
 * gauge ring, records the device time and writes the scenarios still running.
 * Between the two, bgf_pool_finish retires finished scenarios, and
 * bgf_pool_admit and bgf_pool_set_gauges queue new scenarios behind the running
 * steps (they join the next run; their index lists come from page-locked
 * staging); retire, run and get_depth return BGF_ESTATE. */
int bgf_pool_run_async(bgf_pool* pool, int maxsteps);
int bgf_pool_wait(bgf_pool* pool, int* nlive);
/* While a run from bgf_pool_run_async is in flight: applies the admissions and
 * retirements made since it started to the pool's tables now, with their uploads
 * queued behind the run, so that the next bgf_pool_run_async launches at once
 * instead of rebuilding the tables after the run.  Does nothing with no run in
 * flight, nothing pending, or gauges set in the pool (the next run then rebuilds).
 * Admissions and retirements after it are applied by the next run.  No counterpart
 * in the reference (its loop steps one model). */
int bgf_pool_prepare(bgf_pool* pool);
/* Retirement of n finished scenarios (bgf_pool_query status != 0) for a caller
 * that needs only their fields: final depth h and maximum depth hmax (either may
 * be NULL; per scenario an array of nblk * 256 values of the field type in the
 * scenario's active order), loop state, step count and status (1 finished, 2 dt
 * underflow, 3 non-finite).  The state is not copied back into the scenarios'
 * handles.  Runs on the pool's own copy stream, also while a run enqueued by
 * bgf_pool_run_async is in flight (finished scenarios are no longer written);
 * the freed slots serve admissions after that run.  BGF_ESTATE for a scenario
 * that is still running. */
int bgf_pool_finish(bgf_pool* pool, int n, const int* slots, void* const* h, void* const* hmax, bgf_loop* loops,
                    int64_t* nsteps, int* status);
/* CTAs of the fused kernels (0: one per block; fewer CTAs loop over the blocks). */
int bgf_pool_set_grid(bgf_pool* pool, int grid);
/* Thread layout of the pool's single-level kernels, as bgf_set_kernel_layout. */
int bgf_pool_set_kernel_layout(bgf_pool* pool, int layout);

/* ------------------------------------------------------------ launch-shape autotuner */
/* Times the fused step kernels on the current mesh from the loop state `loop`
 * (CUDA events; two untimed steps, then `steps` timed ones) for each launch shape -- one CTA per block, and
 * persistent grids of 2, 3, 4, 5, 6 and 8 CTAs per SM smaller than the block count --
 * keeps the fastest (as bgf_set_grid / bgf_pool_set_grid would) and reports it and
 * its time per step.  The state, boundary means, maximum depths and time slots are
 * restored afterwards, so the simulation continues as if no tuning run took place.
 * Multi-level meshes launch one CTA per block: *grid = 0 and nothing is run.
 * Threads per CTA are fixed (256: one per cell of a 16x16 block); the resident
 * CTAs per SM are fixed at compile time (launch bounds). */
int bgf_autotune(bgf_handle* h, const bgf_loop* loop, int steps, int* grid, double* ms_per_step);
int bgf_pool_autotune(bgf_pool* pool, int steps, int* grid, double* ms_per_step);

/* ------------------------------------------------------------ refinement pass */
/* Criterion of the reference's "Adaptation" key (src/AdaptCriteria.cu:20-232):
 * a block is flagged for refinement when any of its cells has var > arg1
 * (Threshold) or arg1 <= var <= arg2 (Inrange), compared in the state precision,
 * or (Targetlevel) when the rounded bilinear value of a target-level map at any of
 * its cells is above the block's level; Targetlevel keeps a block from coarsening
 * when some cell's target equals its level, and each map rewrites the flags of the
 * previous one (the last map decides), as the reference loops over its maps.
 * Threshold and Inrange mark every block that does not refine as a coarsening
 * candidate (coarsen = !refine).
 *
 * Extension (no counterpart key in the reference): BGF_ADAPT_HGRAD flags a block
 * for refinement when some cell has h > arg1 or a wet-surface slope |grad eta| >
 * arg2, and as a coarsening candidate when every cell has h <= arg1/2 and |grad
 * eta| <= arg2/2 (var is not used).  The slope is taken inside the block from wet
 * cells only: along x, (eta(x+1) - eta(x-1)) / (2 dx_l) when both neighbours are
 * wet cells of the block, the one-sided difference to the wet one otherwise, 0
 * with none (likewise along y); a cell is wet when h > eps; |grad eta|^2 =
 * gx^2 + gy^2 is compared with the squared threshold, all in the state precision.
 *
 * allow_coarsen (extension, 0 = the reference's behaviour): the reference's sanity
 * pass cancels every coarsening flag (src/Adaptation.cu:173-175).  With 1 the
 * pass keeps them and applies the reference's coarsening rules instead (see
 * bgf_adapt_sanity), and bgf_adapt merges each complete quad of coarsening blocks
 * into its parent (the reference's coarsen, src/Adaptation.cu:677-1015). */
enum { BGF_ADAPT_THRESHOLD = 1, BGF_ADAPT_INRANGE = 2, BGF_ADAPT_TARGETLEVEL = 3, BGF_ADAPT_HGRAD = 4 };
enum { BGF_VAR_H = 0, BGF_VAR_ZS = 1, BGF_VAR_U = 2, BGF_VAR_V = 3, BGF_VAR_ZB = 4 };
typedef struct bgf_adapt_param {
    int criterion;     /* BGF_ADAPT_*                                          */
    int var;           /* BGF_VAR_* (Threshold, Inrange)                       */
    double arg1, arg2; /* threshold, or zmin and zmax, or h and slope thresholds */
    int maxiteration;  /* adaptmaxiteration, 20 when <= 0                     */
    int allow_coarsen; /* extension: 0 as the reference (no coarsening)       */
} bgf_adapt_param;

/* Bathymetry forcing (the reference's Forcing.Bathy[0]): nx*ny float nodes,
 * row-major, node (0, 0) at (xo, yo), spacing dx in x and y.  bgf_adapt
 * re-interpolates the bed of every block from it, as the reference does
 * (interp2BUQ + setedges, src/GridManip.cu:222-575). */
int bgf_set_bathy(bgf_handle* h, int nx, int ny, double xo, double yo, double dx, const float* val);

/* Target-level maps of the Targetlevel criterion (the reference's
 * Forcing.targetadapt, one per file of "Adaptation = Targetlevel,<file>,..."):
 * nx*ny integer levels, row-major, node (0, 0) at (xo, yo), spacing dx in x and y.
 * Maps are applied in the order they were added. */
int bgf_add_target_level_map(bgf_handle* h, int nx, int ny, double xo, double yo, double dx, const int* levels);
int bgf_clear_target_level_maps(bgf_handle* h);

/* Refine / coarsen flags of one criterion + sanity pass on the current mesh and
 * state, one byte per active block (active order); the mesh is not changed. */
int bgf_adapt_flags(bgf_handle* h, const bgf_adapt_param* a, uint8_t* refine, uint8_t* coarsen);

/* Adaptation (src/Adaptation.cu:17-121) of the handle's mesh and state: up to
 * maxiteration passes of {criterion, sanity pass, refinement with bilinear
 * interpolation of h, zs, u, v into the children, bed re-interpolation from the
 * bathymetry grid, wet/dry fix-up}, stopping when a pass adds no block.  The
 * new blocks take free block slots below nblkmem (BGF_ENOMEM when there are not
 * enough).  Afterwards the bed halo and gradients are prepared for the new mesh
 * and every boundary segment lists the children of its refined blocks on the
 * same side.  Per-cell friction and rain-mask inputs are carried to the children
 * from the covering parent cell.  Writes the new block count and the number of
 * passes.  With allow_coarsen, a pass also merges every quad of coarsening blocks:
 * the parent keeps the lower-left block's id and takes h, zs, u, v (and friction)
 * as T(0.25) * (((c00 + c10) + c01) + c11) of the four cells it covers, its
 * boundary running means restart at zero, the three other ids become free for the
 * next pass, and boundary segments list the parent in their place; passes stop
 * when a pass neither refines nor coarsens. */
int bgf_adapt(bgf_handle* h, const bgf_adapt_param* a, int* nblk, int* niter);
/* Where bgf_adapt does the sanity pass and the new tables: 1 (default) on the
 * device when the mesh allows it (levels 0..15, per-level block grids of at most
 * 64 M entries), else and with 0 in host C++ (bgf_adapt_sanity,
 * bgf_adapt_tables).  Both give the same flags, ids, active list, levels, origins
 * and neighbour tables; the device path copies the tables to the host once per
 * call instead of every pass. */
int bgf_set_adapt_mode(bgf_handle* h, int mode);

/* Host copies of the current block tables: active (nblk entries), level and
 * origins per block slot, neighbours as [nblkmem][8] (LB, LT, RB, RT, BL, BR, TL,
 * TR).  Any output pointer may be NULL. */
int bgf_get_blocks(bgf_handle* h, int* nblk, int* active, int* level, int* nbr8, double* xo, double* yo);
/* The bed on 18x18 tiles of every block slot (nblkmem * 324 values of the state
 * precision), halo included. */
int bgf_get_bed(bgf_handle* h, void* zb);

/* Host-only table work of the reference's adaptation (no device memory involved).
 * Arrays are indexed by block id and sized nblkmem; nbr8 is [nblkmem][8] in the
 * order LeftBot, LeftTop, RightBot, RightTop, BotLeft, BotRight, TopLeft, TopRight.
 *
 * refinesanitycheck (src/Adaptation.cu:157-296): refine/coarsen flags (one byte
 * per block id) corrected in place -- no refinement at maxlevel, coarsening
 * cancelled (as the reference does), coarser first neighbours of a refining block
 * forced to refine until the mesh stays 2:1 balanced. */
int bgf_refine_sanity(int nblk, const int* active, const int* level, const int* nbr8, int nblkmem, int minlevel,
                      int maxlevel, uint8_t* refine, uint8_t* coarsen);
/* CalcAvailblk + refine + Adaptationcleanup (src/Adaptation.cu:535-596,
 * 1017-1876) on the tables: every flagged block becomes four; it keeps its id as
 * the bottom-left child and the k-th flagged block of the active list takes the
 * free ids 3k..3k+2 (ascending) for its bottom-right, top-left and top-right
 * children (children[3*ib..3*ib+2]), which are appended to the active list.
 * Levels, origins (rounded to float unless doubleprecision) and all neighbour
 * tables are updated; *nblk is updated.  BGF_ENOMEM when fewer than 3 free block
 * slots per flagged block exist below nblkmem. */
int bgf_refine_tables(int* nblk, int* active, int* level, int* nbr8, double* xo, double* yo, int nblkmem, double dx,
                      int doubleprecision, const uint8_t* refine, int* children);

/* refinesanitycheck with coarsening kept (extension; allow_coarsen = 0 is
 * bgf_refine_sanity).  The reference's rules without its cancelling line, in its
 * order: (1) no refinement at maxlevel, no coarsening at minlevel; (2) no
 * coarsening of any neighbour entry of a refining block; (3) no coarsening of a
 * block with a finer side neighbour; (4) until nothing changes, every refining
 * block forces its coarser first neighbours to refine and keeps its same-level
 * first neighbours from coarsening (checkneighbourrefine); (5) in active order, a block
 * keeps its flag only when it is the lower-left block of a quad -- its origin
 * xo / dx_l / 16 and yo / dx_l / 16 truncate to even numbers, its right, top and
 * top-right neighbours exist, are on its level and are flagged; every other
 * block's flag is cleared, so that afterwards coarsen[ib] marks the parents.  xo
 * and yo are the block origins as in bgf_get_blocks, dx the level-0 spacing. */
int bgf_adapt_sanity(int nblk, const int* active, const int* level, const int* nbr8, int nblkmem, int minlevel,
                     int maxlevel, const double* xo, const double* yo, double dx, int allow_coarsen, uint8_t* refine,
                     uint8_t* coarsen);
/* bgf_refine_tables with coarsening (extension; coarsen may be NULL): first every
 * flagged quad parent ib (coarsen[ib], after bgf_adapt_sanity) merges its quad
 * (coarsen, src/Adaptation.cu:677-1015): level - 1, origin xo += dx_{l+1} and yo +=
 * dx_{l+1} (the reference's T(calcres(dx, level + 1)) added in T), its right, top
 * and top-right blocks leave the active list (siblings[3*ib..3*ib+2], else -1) and
 * become free for the next pass only; then the refinement as bgf_refine_tables.
 * The active list keeps its order without the removed blocks, followed by the new
 * children.  BGF_EINVAL when a flagged parent is not the lower-left block of a
 * complete quad on its level or also refines. */
int bgf_adapt_tables(int* nblk, int* active, int* level, int* nbr8, double* xo, double* yo, int nblkmem, double dx,
                     int doubleprecision, const uint8_t* refine, const uint8_t* coarsen, int* children,
                     int* siblings);

#ifdef __cplusplus
}
#endif
#endif

/*
 * bgf_oracle -- CPU restatement of BG_Flood's explicit flow step, used ONLY as
 * test infrastructure: tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg call it as the checker.  The product library never links it.
 *
 * It restates, function by function, the reference's FlowCPU path
 * (src/FlowCPU.cu:15-253) on the block-uniform quadtree (BUQ) layout of the
 * reference: every block is an 18x18 tile (16x16 interior cells plus a
 * one-cell halo) addressed by memloc (src/MemManagement.cu:37-40).  Each
 * function cites the reference file:line it follows and keeps the reference's
 * floating-point operation order, so that in single precision its results are
 * bit-identical to the reference CPU build (checked in tests/ against the
 * reference compiled from its own sources, oracle/_ref, and against the
 * reference's golden vector src/Testing.cu:436).
 *
 * Coverage: uniform-level meshes and two-level meshes whose blocks differ by
 * at most one level (the reference's 2:1 balance); engines 1 (HLLC /
 * Buttinger-Kreuzhuber) and 2 (Kurganov); boundary segment types 0 (wall),
 * 1 (Neumann), 2 (Dirichlet) and 3 (absorbing 1D) with uniform water-level
 * series; friction models -1 (Manning), 0 (quadratic), 1 (smart); uniform
 * rain; the CFL reduction with the reference's dt clamps.
 *
 * Everything is exposed twice, for float ("_f") and double ("_d") states.
 */
#ifndef BGF_ORACLE_H
#define BGF_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* Subset of the reference Param class (src/Param.h:10-239) read by the path. */
typedef struct ora_param {
    double g, rho, eps, dt, CFL, theta, cf, delta, dx, xo, yo, lat;
    double zsinit, zsoffset, bndtaper, bndrelaxtime, bndfiltertime, inittime, mask;
    int engine, frictionmodel, ForceMassConserve, wetdryfix, conserveElevation;
    int rainbnd, maxlevel;
    double dtinit;
} ora_param;

void* ora_create(const ora_param* p, int use_double, int nblk);
void ora_destroy(void* m);

/* Block tables, in the reference's BlockP order (src/Arrays.h:234-250): nbr8 holds
 * per block LeftBot, LeftTop, RightBot, RightTop, BotLeft, BotRight, TopLeft, TopRight.
 * Block ib's memory tile is ib (the active list is the identity). */
int ora_set_blocks(void* m, const int* level, const int* nbr8, const double* xo, const double* yo);

/* Fields: "zb","h","u","v","zs","cf","dzbdx","dzbdy","activeCell","dtmax", plus flux and
 * gradient names; layout nblk x 18 x 18 tiles (halo included). */
int ora_set_field(void* m, const char* name, const double* buq);
int ora_get_field(void* m, const char* name, double* buq);

/* Boundary segment: type, optional uniform water-level series, and per side
 * (0 left, 1 right, 2 top, 3 bot) the blocks it applies to (src/Forcing.h:106-144). */
int ora_add_segment(void* m, int type, int n, const double* t, const double* wl,
                    const int* nblk_side, const int* const* blk_side);
int ora_set_rain(void* m, int n, const double* t, const double* r);
/* Gridded rain: nt frames (row-major, row 0 at yo) of nx*ny nodes, frame k at to + k*dt. */
int ora_set_rain_map(void* m, int nx, int ny, double xo, double yo, double dx, double dy, int nt, double to, double dt,
                     const float* frames);
/* A river (box in absolute coordinates, discharge series); returns the discharge area. */
double ora_add_river(void* m, double xs, double xe, double ys, double ye, int n, const double* t, const double* q);

/* Bed halo + bed gradients exactly as src/Testing.cu:583-588. */
int ora_init_bed(void* m);
/* initdt (src/Mainloop.cu:515-554) then sets the loop's dtmax; returns it. */
double ora_init_loop(void* m, double totaltime, double nextoutputtime);
void ora_set_loop(void* m, double totaltime, double nextoutputtime, double dtmax);
/* One full step per iteration: updateforcing (rain) + FlowCPU + totaltime += dt. */
int ora_step(void* m, int nsteps, double* dts);
double ora_totaltime(void* m);

#ifdef __cplusplus
}
#endif
#endif

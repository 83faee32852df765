/* Oracle entry points (see bgf_oracle.h): the precision-generic body in
 * bgf_oracle_impl.inc is instantiated for float and double.  Test
 * infrastructure only; build with -ffp-contract=off so that every float
 * operation rounds like the reference's host build. */
#include "bgf_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define REAL float
#define FN(x) x##_f
#define FMAX fmaxf
#define FMIN fminf
#define FABS fabsf
#define SQRT sqrtf
#define CBRT cbrtf
#define LOG logf
#define SIN sinf
#define NEXTAFTER nextafterf
#define CEIL ceilf
#define FLOOR floorf
#define HUGEPOS FLT_MAX
#include "bgf_oracle_impl.inc"
#undef REAL
#undef FN
#undef FMAX
#undef FMIN
#undef FABS
#undef SQRT
#undef CBRT
#undef LOG
#undef SIN
#undef NEXTAFTER
#undef CEIL
#undef FLOOR
#undef HUGEPOS
#undef ML
#undef BW

#define REAL double
#define FN(x) x##_d
#define FMAX fmax
#define FMIN fmin
#define FABS fabs
#define SQRT sqrt
#define CBRT cbrt
#define LOG log
#define SIN sin
#define NEXTAFTER nextafter
#define CEIL ceil
#define FLOOR floor
#define HUGEPOS DBL_MAX
#include "bgf_oracle_impl.inc"

typedef struct { int dbl; void* m; } ora_handle;

void* ora_create(const ora_param* p, int use_double, int nblk)
{
    ora_handle* h = (ora_handle*)malloc(sizeof(ora_handle));
    h->dbl = use_double;
    h->m = use_double ? api_create_d(p, nblk) : api_create_f(p, nblk);
    return h;
}
#define DISPATCH(call_f, call_d) (((ora_handle*)m)->dbl ? (call_d) : (call_f))
#define MF ((model_t_f*)((ora_handle*)m)->m)
#define MD ((model_t_d*)((ora_handle*)m)->m)
void ora_destroy(void* m)
{
    if (((ora_handle*)m)->dbl) api_destroy_d(MD); else api_destroy_f(MF);
    free(m);
}
int ora_set_blocks(void* m, const int* level, const int* nbr8, const double* xo, const double* yo)
{ return DISPATCH(api_set_blocks_f(MF, level, nbr8, xo, yo), api_set_blocks_d(MD, level, nbr8, xo, yo)); }
int ora_set_field(void* m, const char* name, const double* buq)
{ return DISPATCH(api_set_field_f(MF, name, buq), api_set_field_d(MD, name, buq)); }
int ora_get_field(void* m, const char* name, double* buq)
{ return DISPATCH(api_get_field_f(MF, name, buq), api_get_field_d(MD, name, buq)); }
int ora_add_segment(void* m, int type, int n, const double* t, const double* wl, const int* nblk_side,
                    const int* const* blk_side)
{ return DISPATCH(api_add_segment_f(MF, type, n, t, wl, nblk_side, blk_side),
                  api_add_segment_d(MD, type, n, t, wl, nblk_side, blk_side)); }
int ora_set_rain(void* m, int n, const double* t, const double* r)
{ return DISPATCH(api_set_rain_f(MF, n, t, r), api_set_rain_d(MD, n, t, r)); }
int ora_set_rain_map(void* m, int nx, int ny, double xo, double yo, double dx, double dy, int nt, double to, double dt,
                     const float* frames)
{ return DISPATCH(api_set_rain_map_f(MF, nx, ny, xo, yo, dx, dy, nt, to, dt, frames),
                  api_set_rain_map_d(MD, nx, ny, xo, yo, dx, dy, nt, to, dt, frames)); }
double ora_add_river(void* m, double xs, double xe, double ys, double ye, int n, const double* t, const double* q)
{ return DISPATCH(api_add_river_f(MF, xs, xe, ys, ye, n, t, q), api_add_river_d(MD, xs, xe, ys, ye, n, t, q)); }
int ora_init_bed(void* m) { return DISPATCH(api_init_bed_f(MF), api_init_bed_d(MD)); }
double ora_init_loop(void* m, double totaltime, double nextoutputtime)
{ return DISPATCH(api_init_loop_f(MF, totaltime, nextoutputtime), api_init_loop_d(MD, totaltime, nextoutputtime)); }
void ora_set_loop(void* m, double totaltime, double nextoutputtime, double dtmax)
{
    if (((ora_handle*)m)->dbl) { MD->totaltime = totaltime; MD->nextoutputtime = nextoutputtime; MD->dtmax_loop = dtmax; }
    else { MF->totaltime = totaltime; MF->nextoutputtime = nextoutputtime; MF->dtmax_loop = dtmax; }
}
int ora_step(void* m, int nsteps, double* dts) { return DISPATCH(api_step_f(MF, nsteps, dts), api_step_d(MD, nsteps, dts)); }
double ora_totaltime(void* m) { return DISPATCH(MF->totaltime, MD->totaltime); }

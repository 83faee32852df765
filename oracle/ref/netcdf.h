/*
 * Header-only stand-in for the netCDF-C API, used ONLY to compile the
 * reference BG_Flood sources into the test oracle (oracle/_ref).  netCDF is
 * not installed in this image and none of the reference's netCDF calls lie on
 * the flow-step path the oracle exercises.  The declarations below were
 * written from the reference's own call sites (src/Read_netcdf.cu,
 * src/Write_netcdf.cu, src/InitEvolv.cu, src/ReadForcing.cu); they are not
 * taken from netCDF's header.  Every function is implemented in
 * netcdf_stub.cpp and reports failure, so a reference code path that tried to
 * read or write a file would stop through the reference's own error handler.
 */
#ifndef BGF_NETCDF_SHIM_H
#define BGF_NETCDF_SHIM_H
#include <stddef.h>

typedef int nc_type;

#define NC_NOERR 0
#define NC_EEXIST (-35)
#define NC_GLOBAL (-1)
#define NC_UNLIMITED 0L
#define NC_NOWRITE 0x0000
#define NC_WRITE 0x0001
#define NC_CLOBBER 0x0000
#define NC_NOCLOBBER 0x0004
#define NC_NETCDF4 0x1000
#define NC_MAX_NAME 256
#define NC_MAX_VAR_DIMS 1024
#define NC_SHORT 3
#define NC_INT 4
#define NC_FLOAT 5
#define NC_DOUBLE 6

#ifdef __cplusplus
extern "C" {
#endif
const char* nc_strerror(int status);
int nc_open(...);
int nc_create(...);
int nc_close(...);
int nc_redef(...);
int nc_enddef(...);
int nc_def_dim(...);
int nc_def_var(...);
int nc_def_var_deflate(...);
int nc_inq_varid(...);
int nc_inq_dimid(...);
int nc_inq_dimlen(...);
int nc_inq_dimname(...);
int nc_inq_unlimdim(...);
int nc_inq_varndims(...);
int nc_inq_vardimid(...);
int nc_inq_attid(...);
int nc_inq_attlen(...);
int nc_get_att_double(...);
int nc_get_att_float(...);
int nc_get_att_int(...);
int nc_get_att_text(...);
int nc_get_var_double(...);
int nc_get_var_float(...);
int nc_get_var_int(...);
int nc_get_var1_double(...);
int nc_get_var1_float(...);
int nc_get_vara_double(...);
int nc_get_vara_float(...);
int nc_get_vara_int(...);
int nc_put_att_double(...);
int nc_put_att_float(...);
int nc_put_att_int(...);
int nc_put_att_short(...);
int nc_put_att_text(...);
int nc_put_att_string(...);
int nc_put_var1_double(...);
int nc_put_vara_double(...);
int nc_put_vara_float(...);
int nc_put_vara_int(...);
int nc_put_vara_short(...);
#ifdef __cplusplus
}
#endif
#endif

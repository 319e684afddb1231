/*
 * Declarations of the NetCDF calls that appear in the reference's I/O functions. The reference
 * harness never calls those functions; the definitions in netcdf_stub.c only satisfy the linker
 * and return an error (test infrastructure only).
 */
#ifndef CGFD_REF_SHIM_NETCDF_H
#define CGFD_REF_SHIM_NETCDF_H
#include <stddef.h>
#define NC_NOERR 0
#define NC_CLOBBER 0
#define NC_NOWRITE 0
#define NC_WRITE 1
#define NC_64BIT_OFFSET 0x0200
#define NC_UNLIMITED 0L
#define NC_GLOBAL (-1)
#define NC_INT 4
#define NC_FLOAT 5
#ifdef __cplusplus
extern "C" {
#endif
const char *nc_strerror(int);
int nc_create(const char *, int, int *);
int nc_open(const char *, int, int *);
int nc_close(int);
int nc_enddef(int);
int nc_def_dim(int, const char *, size_t, int *);
int nc_def_var(int, const char *, int, int, const int *, int *);
int nc_put_att_int(int, int, const char *, int, size_t, const int *);
int nc_put_var_float(int, int, const float *);
int nc_put_vara_float(int, int, const size_t *, const size_t *, const float *);
int nc_put_var1_float(int, int, const size_t *, const float *);
int nc_inq_varid(int, const char *, int *);
int nc_get_var(int, int, void *);
int nc_get_vara_float(int, int, const size_t *, const size_t *, float *);
#ifdef __cplusplus
}
#endif
#endif

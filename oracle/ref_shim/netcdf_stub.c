/* Link-only stand-ins for NetCDF (see netcdf.h); every call reports an error. */
#include <stddef.h>
const char *nc_strerror(int e) { (void)e; return "NetCDF is not available in the reference harness"; }
int nc_create(const char *p, int m, int *i) { (void)p; (void)m; (void)i; return -1; }
int nc_open(const char *p, int m, int *i) { (void)p; (void)m; (void)i; return -1; }
int nc_close(int i) { (void)i; return -1; }
int nc_enddef(int i) { (void)i; return -1; }
int nc_def_dim(int i, const char *n, size_t l, int *d) { (void)i; (void)n; (void)l; (void)d; return -1; }
int nc_def_var(int i, const char *n, int t, int nd, const int *d, int *v) { (void)i; (void)n; (void)t; (void)nd; (void)d; (void)v; return -1; }
int nc_put_att_int(int i, int v, const char *n, int t, size_t l, const int *o) { (void)i; (void)v; (void)n; (void)t; (void)l; (void)o; return -1; }
int nc_put_var_float(int i, int v, const float *o) { (void)i; (void)v; (void)o; return -1; }
int nc_put_vara_float(int i, int v, const size_t *s, const size_t *c, const float *o) { (void)i; (void)v; (void)s; (void)c; (void)o; return -1; }
int nc_put_var1_float(int i, int v, const size_t *s, const float *o) { (void)i; (void)v; (void)s; (void)o; return -1; }
int nc_inq_varid(int i, const char *n, int *v) { (void)i; (void)n; (void)v; return -1; }
int nc_get_var(int i, int v, void *o) { (void)i; (void)v; (void)o; return -1; }
int nc_get_vara_float(int i, int v, const size_t *s, const size_t *c, float *o) { (void)i; (void)v; (void)s; (void)c; (void)o; return -1; }

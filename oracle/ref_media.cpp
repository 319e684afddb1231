// ref_media.cpp -- C entry to the reference's own media discretisation code (src/media/, built
// unmodified from the reference tree by oracle/Makefile.ref into oracle/_ref/libref_media.so).
// TEST INFRASTRUCTURE: the checker of cgfd_media_layer_el_iso_gpu and cgfd_media_layer_gpu; nothing in the product
// links it.
#include <cstddef>
#include <set>  // media_grid2model.hpp names std::set without including it

#include "media_bin2model.hpp"
#include "media_grid2model.hpp"
#include "media_layer2model.hpp"

extern "C" int ref_media_layer2model_el_iso(float *lam3d, float *mu3d, float *rho3d, const float *x3d,
                                            const float *y3d, const float *z3d, size_t nx, size_t ny, size_t nz,
                                            const char *in_3lay_file, const char *method) {
  // the curvilinear grid type, as main_curv_col_el_3d.cu:307-313 passes it; rank 1 prints nothing
  return media_layer2model_el_iso(lam3d, mu3d, rho3d, x3d, y3d, z3d, nx, ny, nz, GRID_CURV, in_3lay_file, method, 1);
}

// media_layer2model_ac_iso (media_layer2model.cpp:70-118): rho, kappa
extern "C" int ref_media_layer2model_ac_iso(float *rho3d, float *kappa3d, const float *x3d, const float *y3d,
                                            const float *z3d, size_t nx, size_t ny, size_t nz, const char *in_3lay_file,
                                            const char *method) {
  return media_layer2model_ac_iso(rho3d, kappa3d, x3d, y3d, z3d, nx, ny, nz, GRID_CURV, in_3lay_file, method, 1);
}

// media_layer2model_el_vti (media_layer2model.cpp:173-228): rho, c11, c33, c55, c66, c13
extern "C" int ref_media_layer2model_el_vti(float *rho, float *c11, float *c33, float *c55, float *c66, float *c13,
                                            const float *x3d, const float *y3d, const float *z3d, size_t nx,
                                            size_t ny, size_t nz, const char *in_3lay_file, const char *method) {
  return media_layer2model_el_vti(rho, c11, c33, c55, c66, c13, x3d, y3d, z3d, nx, ny, nz, GRID_CURV, in_3lay_file,
                                  method, 1);
}

// media_layer2model_el_aniso (media_layer2model.cpp:230-398): out[0] rho, out[1..21] c11 c12 c13 c14 c15 c16
// c22 c23 c24 c25 c26 c33 c34 c35 c36 c44 c45 c46 c55 c56 c66
extern "C" int ref_media_layer2model_el_aniso(float *const *out, const float *x3d, const float *y3d, const float *z3d,
                                              size_t nx, size_t ny, size_t nz, const char *in_3lay_file,
                                              const char *method) {
  return media_layer2model_el_aniso(out[0], out[1], out[2], out[3], out[4], out[5], out[6], out[7], out[8], out[9],
                                    out[10], out[11], out[12], out[13], out[14], out[15], out[16], out[17], out[18],
                                    out[19], out[20], out[21], x3d, y3d, z3d, nx, ny, nz, GRID_CURV, in_3lay_file,
                                    method, 1);
}

// media_bin2model_el_iso (media_bin2model.cpp:27-183): rho, lambda, mu from three binary volumes,
// with the grid's x / y range as gd_curv_set_minmax computes it
extern "C" int ref_media_bin2model_el_iso(float *rho3d, float *lam3d, float *mu3d, const float *x3d, const float *y3d,
                                          const float *z3d, size_t nx, size_t ny, size_t nz, float xmin, float xmax,
                                          float ymin, float ymax, int *bin_order, int *bin_size, float *bin_spacing,
                                          float *bin_origin, const char *file_rho, const char *file_vp,
                                          const char *file_vs) {
  return media_bin2model_el_iso(rho3d, lam3d, mu3d, x3d, y3d, z3d, nx, ny, nz, xmin, xmax, ymin, ymax, GRID_CURV,
                                bin_order, bin_size, bin_spacing, bin_origin, file_rho, file_vp, file_vs);
}

// media_grid2model_el_iso (media_grid2model.cpp:133-188): rho, lambda, mu from a grid media file,
// with the grid's x / y range as gd_curv_set_minmax computes it
extern "C" int ref_media_grid2model_el_iso(float *rho3d, float *lam3d, float *mu3d, const float *x3d, const float *y3d,
                                           const float *z3d, int nx, int ny, int nz, float xmin, float xmax,
                                           float ymin, float ymax, const char *in_media_file, const char *method) {
  return media_grid2model_el_iso(rho3d, lam3d, mu3d, x3d, y3d, z3d, nx, ny, nz, xmin, xmax, ymin, ymax, GRID_CURV,
                                 in_media_file, method, 1);
}

// media_grid2model_el_vti (media_grid2model.cpp:190-248): rho, c11, c33, c55, c66, c13
extern "C" int ref_media_grid2model_el_vti(float *const *out, const float *x3d, const float *y3d, const float *z3d,
                                           int nx, int ny, int nz, float xmin, float xmax, float ymin, float ymax,
                                           const char *in_media_file, const char *method) {
  return media_grid2model_el_vti(out[0], out[1], out[2], out[3], out[4], out[5], x3d, y3d, z3d, nx, ny, nz, xmin,
                                 xmax, ymin, ymax, GRID_CURV, in_media_file, method, 1);
}

// media_grid2model_el_aniso (media_grid2model.cpp:250-422): out[0] rho, out[1..21] c11 .. c66
extern "C" int ref_media_grid2model_el_aniso(float *const *out, const float *x3d, const float *y3d, const float *z3d,
                                             int nx, int ny, int nz, float xmin, float xmax, float ymin, float ymax,
                                             const char *in_media_file, const char *method) {
  return media_grid2model_el_aniso(out[0], out[1], out[2], out[3], out[4], out[5], out[6], out[7], out[8], out[9],
                                   out[10], out[11], out[12], out[13], out[14], out[15], out[16], out[17], out[18],
                                   out[19], out[20], out[21], x3d, y3d, z3d, nx, ny, nz, xmin, xmax, ymin, ymax,
                                   GRID_CURV, in_media_file, method, 1);
}

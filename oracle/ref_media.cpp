// ref_media.cpp -- C entry to the reference's own media discretisation code (src/media/, built
// unmodified from the reference tree by oracle/Makefile.ref into oracle/_ref/libref_media.so).
// TEST INFRASTRUCTURE: the checker of cgfd_media_layer_el_iso_gpu; nothing in the product
// links it.
#include <cstddef>

#include "media_layer2model.hpp"

extern "C" int ref_media_layer2model_el_iso(float *lam3d, float *mu3d, float *rho3d, const float *x3d,
                                            const float *y3d, const float *z3d, size_t nx, size_t ny, size_t nz,
                                            const char *in_3lay_file, const char *method) {
  // the curvilinear grid type, as main_curv_col_el_3d.cu:307-313 passes it; rank 1 prints nothing
  return media_layer2model_el_iso(lam3d, mu3d, rho3d, x3d, y3d, z3d, nx, ny, nz, GRID_CURV, in_3lay_file, method, 1);
}

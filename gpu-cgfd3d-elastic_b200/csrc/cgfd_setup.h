// cgfd_setup.h -- host-side (FP64) setup that feeds the time loop.
#pragma once

#include <stdexcept>
#include <string>
#include <vector>

#include "cgfd_b200.h"

namespace cgfd {

struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};

// Reference host layout helpers (3 ghosts).
struct RefGrid {
  int ni, nj, nk, nx, ny, nz;
  size_t siz_iy, siz_iz, siz_icmp;
  explicit RefGrid(int ni_, int nj_, int nk_)
      : ni(ni_), nj(nj_), nk(nk_), nx(ni_ + 6), ny(nj_ + 6), nz(nk_ + 6) {
    siz_iy = nx;
    siz_iz = (size_t)nx * ny;
    siz_icmp = siz_iz * nz;
  }
  // reference index of physical point (i,j,k)
  size_t at(int i, int j, int k) const { return (size_t)(i + 3) + (size_t)(j + 3) * siz_iy + (size_t)(k + 3) * siz_iz; }
};

int medium_ncmp(int medium_type);

struct PmlFaceHost {
  int enable = 0;
  int axis = 0, side = 0;
  int lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
  std::vector<float> A, B, D;
};
void pml_setup(const cgfd_problem_desc *d, PmlFaceHost faces[3][2]);

// [nj][ni][9] matVx2Vz / matVy2Vz at the top layer
void dvh2dvz(const cgfd_problem_desc *d, std::vector<float> &matx, std::vector<float> &maty);
// Visco-elastic media: the GMB fit (cgfd_visco_gmb) and the free-surface frame matrices
// [nj][ni][9] of the stress fix after each time step.
void visco_gmb(const cgfd_visco_desc *v, long long n, const float *lambda, const float *mu, const float *Qp,
               const float *Qs, float *lam_u, float *mu_u, float *Ylam, float *Ymu, float *wl);
void vis_free_matrix(const cgfd_problem_desc *d, std::vector<float> &matD);

// Points given by physical coordinates, located like the reference: global physical index
// (-1000 when outside the grid), fractional shift, and the coordinates after a depth was
// converted to z.
struct Located {
  std::vector<int> idx;
  std::vector<float> inc;
  std::vector<float> xyz;
};
// use_depth[q]: z of point q is a depth below the free surface. Runs on the current device.
void locate_coords(const cgfd_problem_desc *d, int n, const float *xyz, const int *use_depth, Located &out);

struct SrcHost {
  int nsrc = 0, max_ext = 0, max_nt = 0, force = 0, moment = 0;
  std::vector<int> it_begin, ext_num;
  std::vector<int> ext_i, ext_j, ext_k;   // [nsrc][max_ext] physical indices
  std::vector<float> ext_wv, ext_wt;      // coef*(1/rho)/jac, coef/jac
  std::vector<float> stf;                 // [nsrc][max_nt][4][9]
};
// loc: located coordinates of the sources (loc_coord_type 1); nullptr for grid indices, or
// when only sizes are needed (every coordinate source is then taken as inside the grid)
void src_setup(const cgfd_problem_desc *d, SrcHost &s, const Located *loc = nullptr);

struct RecvHost {
  int n = 0;
  std::vector<int> i, j, k;               // corner 0, physical indices
  std::vector<int> input_index;           // position in the station list
  std::vector<float> w8;                  // [n][8]
};
// loc: located coordinates of the stations with flag_coord 1 (indexed like the input list);
// nullptr when only sizes are needed (every such station is then taken as inside the grid)
void recv_setup(const cgfd_problem_desc *d, RecvHost &r, const Located *loc = nullptr);

void validate_desc(const cgfd_problem_desc *d);

// message returned by cgfd_last_error() on this thread
void set_last_error(const std::string &m);

}  // namespace cgfd

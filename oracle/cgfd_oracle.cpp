/*
 * cgfd_oracle.cpp -- CPU restatement of the CGFD3D elastic time-stepping path of
 * hpc-lee/gpu-CGFD3D-elastic, used ONLY as the checker of the CUDA product.
 *
 * TEST INFRASTRUCTURE. Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline /
 * --impl reference legs may load this library. Nothing in the product links or calls it.
 *
 * The code follows the reference function by function, in the reference's host layout
 * (var[cmp][k][j][i], 3 ghosts) and in the reference's order of evaluation, so that the
 * single-precision instantiation reproduces the reference's FP32 arithmetic up to FMA
 * contraction, and the double instantiation is the FP64 oracle of the precision study:
 *   fd tables / pairs / RK coefs ....... src/forward/fd_t.cu:18-310
 *   time loop .......................... src/forward/drv_rk_curv_col.cu:193-541
 *   one stage .......................... sv_curv_col_el_iso_gpu.cu:23-285 (vti :22-287,
 *                                        aniso :23-321)
 *   inner RHS .......................... sv_curv_col_el_iso_gpu.cu:291-452,
 *                                        sv_curv_col_el_vti_gpu.cu:289-459,
 *                                        sv_curv_col_el_aniso_gpu.cu:323-523
 *   traction image ..................... sv_curv_col_el_gpu.cu:19-221
 *   vlow ............................... sv_curv_col_el_iso_gpu.cu:462-603 (vti :461-612,
 *                                        aniso :525-704)
 *   CFS-PML ............................ sv_curv_col_el_iso_gpu.cu:613-1147 (vti :614-1137,
 *                                        aniso :706-1303)
 *   source injection ................... sv_curv_col_el_gpu.cu:227-301
 *   dvh2dvz ............................ sv_curv_col_el_iso_gpu.cu:1152-1261 (vti :1139-1256,
 *                                        aniso :1305-1456), fdlib_math.cu:6-53
 *   PML coefficients ................... bdry_t.cu:85-451
 *   source locate / smooth / STF ....... src_t.cu:143-1009, interp.cu:220-299
 *   station locate / sampling .......... io_funcs.cu:24-299, 1624-1666
 *   metrics + ghost extrapolation ...... gd_t.cu:209-314, 404-502
 *   rho -> 1/rho ....................... md_t.cu:622-637
 */
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <memory>
#include <vector>
#include <stdexcept>

#include "cgfd_b200.h"

namespace {

thread_local std::string g_err;

constexpr int NG = 3;  // fd_t.cu:64-66

// ---------------------------------------------------------------------------------------
// fd_t.cu:56-235 -- MacCormack operators for 4 layers (0: at free surface, 1: 2nd order,
// 2: 4th order, 3: DRP normal op), backward (0) / forward (1), and the 8 pairs.
// ---------------------------------------------------------------------------------------
struct Op {
  int len;
  int idx[5];
  double coef[5];
};

const Op kOps[4][2] = {
  { {2, {-1, 0, 0, 0, 0}, {-1.0, 1.0, 0, 0, 0}},
    {2, { 0, 1, 0, 0, 0}, {-1.0, 1.0, 0, 0, 0}} },
  { {2, {-1, 0, 0, 0, 0}, {-1.0, 1.0, 0, 0, 0}},
    {2, { 0, 1, 0, 0, 0}, {-1.0, 1.0, 0, 0, 0}} },
  { {3, {-2, -1, 0, 0, 0}, {1.0 / 6.0, -8.0 / 6.0, 7.0 / 6.0, 0, 0}},
    {3, { 0, 1, 2, 0, 0}, {-7.0 / 6.0, 8.0 / 6.0, -1.0 / 6.0, 0, 0}} },
  { {5, {-3, -2, -1, 0, 1}, {-0.041686285, 0.333411808, -1.250117713, 0.666745142, 0.291647047}},
    {5, {-1, 0, 1, 2, 3}, {-0.291647047, -0.666745142, 1.250117713, -0.333411808, 0.041686285}} },
};

// fd_t.cu:184-194, 0 = backward, 1 = forward
const int kPairFlags[8][3] = {
  {0, 0, 0}, {1, 1, 0}, {1, 1, 1}, {0, 0, 1}, {0, 1, 0}, {1, 0, 0}, {1, 0, 1}, {0, 1, 1}};

inline int op_dir(int ipair, int istage, int dim) { return (kPairFlags[ipair][dim] + istage) % 2; }

// fd_t.cu:152-170 centered 7-point operator used for the metrics (stored as float).
const int kCenterIdx[7] = {-3, -2, -1, 0, 1, 2, 3};
const double kCenterCoef[7] = {-0.02084, 0.1667, -0.7709, 0.0, 0.7709, -0.1667, 0.02084};

// ---------------------------------------------------------------------------------------
// grid info for one rank (gd_t.cu:1888-2043 with nprocx = nprocy = 1)
// ---------------------------------------------------------------------------------------
struct Grid {
  int ni, nj, nk, nx, ny, nz;
  int ni1, ni2, nj1, nj2, nk1, nk2;
  size_t siz_iy, siz_iz, siz_icmp;
  void set(int ni_, int nj_, int nk_) {
    ni = ni_; nj = nj_; nk = nk_;
    nx = ni + 2 * NG; ny = nj + 2 * NG; nz = nk + 2 * NG;
    ni1 = NG; ni2 = ni1 + ni - 1;
    nj1 = NG; nj2 = nj1 + nj - 1;
    nk1 = NG; nk2 = nk1 + nk - 1;
    siz_iy = nx; siz_iz = (size_t)nx * ny; siz_icmp = siz_iz * nz;
  }
  bool lindx_is_inner(int i, int j, int k) const {  // gd_t.cu:2046-2060
    return i >= ni1 && i <= ni2 && j >= nj1 && j <= nj2 && k >= nk1 && k <= nk2;
  }
};

// geometric_symmetry, gd_t.cu:404-502: ghost values by linear extrapolation.
template <typename T>
void geometric_symmetry(const Grid &g, T *v4d, int ncmp) {
  for (int icmp = 0; icmp < ncmp; icmp++) {
    T *v = v4d + icmp * g.siz_icmp;
    auto at = [&](size_t i, size_t j, size_t k) -> T & { return v[i + j * g.siz_iy + k * g.siz_iz]; };
    for (int k = 0; k < g.nz; k++)
      for (int j = 0; j < g.ny; j++)
        for (int i = 0; i < g.ni1; i++) at(i, j, k) = 2 * at(g.ni1, j, k) - at(2 * g.ni1 - i, j, k);
    for (int k = 0; k < g.nz; k++)
      for (int j = 0; j < g.ny; j++)
        for (int i = g.ni2 + 1; i < g.nx; i++) at(i, j, k) = 2 * at(g.ni2, j, k) - at(2 * g.ni2 - i, j, k);
    for (int k = 0; k < g.nz; k++)
      for (int j = 0; j < g.nj1; j++)
        for (int i = 0; i < g.nx; i++) at(i, j, k) = 2 * at(i, g.nj1, k) - at(i, 2 * g.nj1 - j, k);
    for (int k = 0; k < g.nz; k++)
      for (int j = g.nj2 + 1; j < g.ny; j++)
        for (int i = 0; i < g.nx; i++) at(i, j, k) = 2 * at(i, g.nj2, k) - at(i, 2 * g.nj2 - j, k);
    for (int k = 0; k < g.nk1; k++)
      for (int j = 0; j < g.ny; j++)
        for (int i = 0; i < g.nx; i++) at(i, j, k) = 2 * at(i, j, g.nk1) - at(i, j, 2 * g.nk1 - k);
    for (int k = g.nk2 + 1; k < g.nz; k++)
      for (int j = 0; j < g.ny; j++)
        for (int i = 0; i < g.nx; i++) at(i, j, k) = 2 * at(i, j, g.nk2) - at(i, j, 2 * g.nk2 - k);
  }
}

// gd_curv_metric_cal, gd_t.cu:209-314 (FP32 in the reference).
template <typename T>
void metric_cal(const Grid &g, const T *x3d, const T *y3d, const T *z3d, T *metric) {
  T *jac3d = metric, *xi_x = metric + 1 * g.siz_icmp, *xi_y = metric + 2 * g.siz_icmp,
    *xi_z = metric + 3 * g.siz_icmp, *et_x = metric + 4 * g.siz_icmp, *et_y = metric + 5 * g.siz_icmp,
    *et_z = metric + 6 * g.siz_icmp, *zt_x = metric + 7 * g.siz_icmp, *zt_y = metric + 8 * g.siz_icmp,
    *zt_z = metric + 9 * g.siz_icmp;
  T c[7];
  for (int n = 0; n < 7; n++) c[n] = (T)(float)kCenterCoef[n];
  auto d = [&](const T *v, size_t iptr, size_t shift) {
    T r = c[0] * v[iptr + kCenterIdx[0] * (long)shift];
    for (int n = 1; n < 7; n++) r += c[n] * v[iptr + kCenterIdx[n] * (long)shift];
    return r;
  };
  auto cross = [](const T *a, const T *b, T *o) {
    o[0] = a[1] * b[2] - a[2] * b[1];
    o[1] = a[2] * b[0] - a[0] * b[2];
    o[2] = a[0] * b[1] - a[1] * b[0];
  };
#pragma omp parallel for schedule(static)
  for (int k = g.nk1; k <= g.nk2; k++)
    for (int j = g.nj1; j <= g.nj2; j++)
      for (int i = g.ni1; i <= g.ni2; i++) {
        size_t iptr = i + j * g.siz_iy + k * g.siz_iz;
        T v1[3] = {d(x3d, iptr, 1), d(y3d, iptr, 1), d(z3d, iptr, 1)};
        T v2[3] = {d(x3d, iptr, g.siz_iy), d(y3d, iptr, g.siz_iy), d(z3d, iptr, g.siz_iy)};
        T v3[3] = {d(x3d, iptr, g.siz_iz), d(y3d, iptr, g.siz_iz), d(z3d, iptr, g.siz_iz)};
        T vg[3];
        cross(v1, v2, vg);
        T jac = 0;
        for (int m = 0; m < 3; m++) jac += vg[m] * v3[m];
        jac3d[iptr] = jac;
        cross(v2, v3, vg);
        xi_x[iptr] = vg[0] / jac; xi_y[iptr] = vg[1] / jac; xi_z[iptr] = vg[2] / jac;
        cross(v3, v1, vg);
        et_x[iptr] = vg[0] / jac; et_y[iptr] = vg[1] / jac; et_z[iptr] = vg[2] / jac;
        cross(v1, v2, vg);
        zt_x[iptr] = vg[0] / jac; zt_y[iptr] = vg[1] / jac; zt_z[iptr] = vg[2] / jac;
      }
  geometric_symmetry(g, metric, 10);
}

// fdlib_math.cu:6-36 -- cofactors in the working precision, determinant in double.
template <typename T>
void invert3x3(T m[3][3]) {
  double inv[3][3];
  inv[0][0] = m[1][1] * m[2][2] - m[2][1] * m[1][2];
  inv[0][1] = m[2][1] * m[0][2] - m[0][1] * m[2][2];
  inv[0][2] = m[0][1] * m[1][2] - m[0][2] * m[1][1];
  inv[1][0] = m[1][2] * m[2][0] - m[1][0] * m[2][2];
  inv[1][1] = m[0][0] * m[2][2] - m[2][0] * m[0][2];
  inv[1][2] = m[1][0] * m[0][2] - m[0][0] * m[1][2];
  inv[2][0] = m[1][0] * m[2][1] - m[1][1] * m[2][0];
  inv[2][1] = m[2][0] * m[0][1] - m[0][0] * m[2][1];
  inv[2][2] = m[0][0] * m[1][1] - m[0][1] * m[1][0];
  double det = inv[0][0] * m[0][0] + inv[0][1] * m[1][0] + inv[0][2] * m[2][0];
  det = 1.0 / det;
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) m[i][j] = (T)(inv[i][j] * det);
}

template <typename T>
void matmul3x3(T A[3][3], T B[3][3], T C[3][3]) {  // fdlib_math.cu:38-53
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) {
      C[i][j] = 0;
      for (int k = 0; k < 3; k++) C[i][j] += A[i][k] * B[k][j];
    }
}

// Voigt index of the symmetric pair (a,b), 0-based: xx,yy,zz,yz,xz,xy.
inline int voigt(int a, int b) {
  static const int v[3][3] = {{0, 5, 4}, {5, 1, 3}, {4, 3, 2}};
  return v[a][b];
}

// ---------------------------------------------------------------------------------------
// The oracle state: reference structs flattened.
// ---------------------------------------------------------------------------------------
// Location by physical coordinates (gd_t.cu:949-1835, fdlib_math.cu:168-245), float
// arithmetic as in the reference.
// ---------------------------------------------------------------------------------------
struct Locator {
  const Grid &g;
  const float *x, *y, *z;
  float xmin, xmax, ymin, ymax, zmin, zmax;
  int ts[3][4], te[3][4];
  float tx0[4][4], tx1[4][4], ty0[4][4], ty1[4][4];

  Locator(const Grid &g_, const float *coord) : g(g_), x(coord), y(coord + g_.siz_icmp), z(coord + 2 * g_.siz_icmp) {
    xmin = xmax = x[0]; ymin = ymax = y[0]; zmin = zmax = z[0];
    for (size_t t = 0; t < g.siz_icmp; t++) {  // gd_t.cu:952-969
      xmin = xmin < x[t] ? xmin : x[t]; xmax = xmax > x[t] ? xmax : x[t];
      ymin = ymin < y[t] ? ymin : y[t]; ymax = ymax > y[t] ? ymax : y[t];
      zmin = zmin < z[t] ? zmin : z[t]; zmax = zmax > z[t] ? zmax : z[t];
    }
    const int n[3] = {g.ni, g.nj, g.nk};
    for (int a = 0; a < 3; a++) {  // gd_t.cu:1034-1083
      const int avg = n[a] / 4, left = n[a] % 4;
      for (int t = 0; t < 4; t++) {
        ts[a][t] = t == 0 ? NG : te[a][t - 1] + 1;
        te[a][t] = ts[a][t] + avg - 1;
        if (t < left) te[a][t] += 1;
      }
    }
    for (int jt = 0; jt < 4; jt++)  // tiles of the top k-tile (the only ones depth_to_axis reads)
      for (int it = 0; it < 4; it++) {
        float a0 = 1.0e26f, a1 = -1.0e26f, b0 = 1.0e26f, b1 = -1.0e26f;
        for (int k = ts[2][3]; k <= te[2][3]; k++)
          for (int j = ts[1][jt]; j <= te[1][jt]; j++)
            for (int i = ts[0][it]; i <= te[0][it]; i++) {
              float c0, c1, d0, d1;
              cell_xy(i, j, k, c0, c1, d0, d1);
              a0 = a0 < c0 ? a0 : c0; a1 = a1 > c1 ? a1 : c1;
              b0 = b0 < d0 ? b0 : d0; b1 = b1 > d1 ? b1 : d1;
            }
        tx0[jt][it] = a0; tx1[jt][it] = a1; ty0[jt][it] = b0; ty1[jt][it] = b1;
      }
  }
  size_t at(int i, int j, int k) const { return i + j * g.siz_iy + k * g.siz_iz; }
  // cell_xmin..ymax of gd_t.cu:990-1031 (8 corners)
  void cell_xy(int i, int j, int k, float &a0, float &a1, float &b0, float &b1) const {
    a0 = a1 = x[at(i, j, k)];
    b0 = b1 = y[at(i, j, k)];
    for (int n3 = 0; n3 < 2; n3++)
      for (int n2 = 0; n2 < 2; n2++)
        for (int n1 = 0; n1 < 2; n1++) {
          size_t q = at(i + n1, j + n2, k + n3);
          a0 = a0 < x[q] ? a0 : x[q]; a1 = a1 > x[q] ? a1 : x[q];
          b0 = b0 < y[q] ? b0 : y[q]; b1 = b1 > y[q] ? b1 : y[q];
        }
  }
  // fdlib_math_isPoint2InQuad
  static bool in_quad(float px, float py, const float *vx0, const float *vy0) {
    float vx[4] = {vx0[0], vx0[1], vx0[3], vx0[2]}, vy[4] = {vy0[0], vy0[1], vy0[3], vy0[2]};
    for (int i = 0; i < 4; i++) {
      float ex = i == 3 ? (vx[0] - vx[3]) : (vx[i + 1] - vx[i]);
      float ey = i == 3 ? (vy[0] - vy[3]) : (vy[i + 1] - vy[i]);
      float qx = px - vx[i], qy = py - vy[i];
      float sg = ex * qy - ey * qx;
      sg /= std::sqrt(ex * ex + ey * ey);
      if (sg < -1e-6) return false;
    }
    return true;
  }
  // fdlib_math_rdinterp_2d for 4 points
  static float rdinterp(float xx, float yy, const float *px, const float *py, const float *pv) {
    float w[4] = {0, 0, 0, 0}, tot = 0.0f;
    int atp = -1;
    for (int i = 0; i < 4; i++) {
      float dist = std::sqrt((xx - px[i]) * (xx - px[i]) + (yy - py[i]) * (yy - py[i]));
      if (dist < 1e-9) atp = i;
      else { w[i] = 1.0 / dist; tot += w[i]; }
    }
    if (atp > 0) { tot = 1.0; for (int i = 0; i < 4; i++) w[i] = 0.0; w[atp] = 1.0; }
    float v = 0.0;
    for (int i = 0; i < 4; i++) { w[i] *= 1.0 / tot; v += w[i] * pv[i]; }
    return v;
  }
  // gd_curv_depth_to_axis
  void depth_to_axis(float sx, float sy, float *sz) const {
    if (sx < xmin || sx > xmax || sy < ymin || sy > ymax) return;
    for (int jt = 0; jt < 4; jt++)
      for (int it = 0; it < 4; it++) {
        if (sx < tx0[jt][it] || sx > tx1[jt][it] || sy < ty0[jt][it] || sy > ty1[jt][it]) continue;
        int k = te[2][3];
        for (int j = ts[1][jt]; j <= te[1][jt]; j++)
          for (int i = ts[0][it]; i <= te[0][it]; i++) {
            float c0, c1, d0, d1;
            cell_xy(i, j, k, c0, c1, d0, d1);
            if (sx < c0 || sx > c1 || sy < d0 || sy > d1) continue;
            float px[4], py[4], pz[4];
            for (int n2 = 0; n2 < 2; n2++)
              for (int n1 = 0; n1 < 2; n1++) {
                size_t q = at(i + n1, j + n2, k);
                px[n1 + n2 * 2] = x[q]; py[n1 + n2 * 2] = y[q]; pz[n1 + n2 * 2] = z[q];
              }
            if (in_quad(sx, sy, px, py)) {
              float ztopo = rdinterp(sx, sy, px, py, pz);
              *sz = ztopo - (*sz);
              return;
            }
          }
      }
  }
  static float dot(const float *a, const float *b) {
    float r = 0.0;
    for (int i = 0; i < 3; i++) r += a[i] * b[i];
    return r;
  }
  // isPointInHexahedron_c + point2face + face_normal
  static bool in_hexa(float px, float py, float pz, const float *vx, const float *vy, const float *vz) {
    float pt[3] = {px, py, pz};
    const int fc[6][3] = {{0, 4, 6}, {7, 5, 1}, {5, 4, 0}, {2, 6, 7}, {4, 5, 7}, {3, 1, 0}};
    for (int f = 0; f < 6; f++) {
      float h[3][3];
      for (int c = 0; c < 3; c++) { h[c][0] = vx[fc[f][c]]; h[c][1] = vy[fc[f][c]]; h[c][2] = vz[fc[f][c]]; }
      float p2f[3], A[3], B[3], nrm[3], un[3];
      for (int i = 0; i < 3; i++) p2f[i] = h[0][i] - pt[i];
      for (int i = 0; i < 3; i++) { A[i] = h[1][i] - h[0][i]; B[i] = h[2][i] - h[0][i]; }
      nrm[0] = A[1] * B[2] - A[2] * B[1];
      nrm[1] = A[2] * B[0] - A[0] * B[2];
      nrm[2] = A[0] * B[1] - A[1] * B[0];
      float len = std::sqrt(dot(nrm, nrm));
      for (int i = 0; i < 3; i++) un[i] = nrm[i] / len;
      float sg = dot(p2f, un);
      float lp = std::sqrt(dot(p2f, p2f));
      sg /= lp;
      if (sg < 0.0) return false;
    }
    return true;
  }
  // gd_curv_coord_to_local_indx + gd_curv_coord2index_sample; returns false when not here
  bool locate(float sx, float sy, float sz, int gidx[3], float inc[3]) const {
    gidx[0] = gidx[1] = gidx[2] = -1000;
    inc[0] = inc[1] = inc[2] = 0.0f;
    if (sx < xmin || sx > xmax || sy < ymin || sy > ymax || sz < zmin || sz > zmax) return false;
    float md = std::sqrt((sx - x[0]) * (sx - x[0]) + (sy - y[0]) * (sy - y[0]) + (sz - z[0]) * (sz - z[0]));
    int mi = 0, mj = 0, mk = 0;
    for (int k = 0; k < g.nz; k++)
      for (int j = 0; j < g.ny; j++)
        for (int i = 0; i < g.nx; i++) {
          size_t q = at(i, j, k);
          float dd = std::sqrt((sx - x[q]) * (sx - x[q]) + (sy - y[q]) * (sy - y[q]) + (sz - z[q]) * (sz - z[q]));
          if (md > dd) { md = dd; mi = i; mj = j; mk = k; }
        }
    if (mi < g.ni1 || mi > g.ni2 || mj < g.nj1 || mj > g.nj2 || mk < g.nk1 || mk > g.nk2) return false;
    gidx[0] = mi - NG; gidx[1] = mj - NG; gidx[2] = mk - NG;
    for (int kk = 0; kk < 2; kk++)
      for (int jj = 0; jj < 2; jj++)
        for (int ii = 0; ii < 2; ii++) {
          int ci = mi - 1 + ii, cj = mj - 1 + jj, ck = mk - 1 + kk;
          float vx[8], vy[8], vz[8];
          for (int n3 = 0; n3 < 2; n3++)
            for (int n2 = 0; n2 < 2; n2++)
              for (int n1 = 0; n1 < 2; n1++) {
                size_t q = at(ci + n1, cj + n2, ck + n3);
                int c = n1 + n2 * 2 + n3 * 4;
                vx[c] = x[q]; vy[c] = y[q]; vz[c] = z[q];
              }
          if (!in_hexa(sx, sy, sz, vx, vy, vz)) continue;
          const int ns = 100;
          float m2 = std::sqrt((sx - vx[0]) * (sx - vx[0]) + (sy - vy[0]) * (sy - vy[0]) + (sz - vz[0]) * (sz - vz[0]));
          int b1 = 0, b2 = 0, b3 = 0;
          for (int n3 = 0; n3 < ns + 1; n3++) {
            float Lz[2]; Lz[1] = (float)n3 / (float)ns; Lz[0] = 1.0 - Lz[1];
            for (int n2 = 0; n2 < ns + 1; n2++) {
              float Ly[2]; Ly[1] = (float)n2 / (float)ns; Ly[0] = 1.0 - Ly[1];
              for (int n1 = 0; n1 < ns + 1; n1++) {
                float Lx[2]; Lx[1] = (float)n1 / (float)ns; Lx[0] = 1.0 - Lx[1];
                float xp = 0, yp = 0, zp = 0;
                for (int k2 = 0; k2 < 2; k2++)
                  for (int j2 = 0; j2 < 2; j2++)
                    for (int i2 = 0; i2 < 2; i2++) {
                      int c = i2 + j2 * 2 + k2 * 4;
                      xp += Lx[i2] * Ly[j2] * Lz[k2] * vx[c];
                      yp += Lx[i2] * Ly[j2] * Lz[k2] * vy[c];
                      zp += Lx[i2] * Ly[j2] * Lz[k2] * vz[c];
                    }
                float dd = std::sqrt((sx - xp) * (sx - xp) + (sy - yp) * (sy - yp) + (sz - zp) * (sz - zp));
                if (m2 > dd) { m2 = dd; b1 = n1; b2 = n2; b3 = n3; }
              }
            }
          }
          float si = (float)ci + (float)b1 / (float)ns, sj = (float)cj + (float)b2 / (float)ns,
                sk = (float)ck + (float)b3 / (float)ns;
          inc[0] = si - mi; inc[1] = sj - mj; inc[2] = sk - mk;
          return true;
        }
    return true;  // in no surrounding cell: zero shift (gd_t.cu:1378-1386)
  }
};

// ---------------------------------------------------------------------------------------
template <typename T>
struct Oracle {
  Grid g;
  int medium_type = 0;
  T dt = 0, t0 = 0;
  int nt_total = 0;
  int it_cur = 0;

  std::vector<T> metric;      // [10][siz_icmp]
  std::vector<T> med;         // medium (rho converted to slowness)
  std::vector<T> c6;          // VTI/aniso: [21] upper-triangular Cij per point, Voigt 6x6
  std::vector<T> wave;        // [4 levels][9][siz_icmp]: pre, tmp, rhs, end
  int lvl_pre = 0, lvl_end = 3;

  int free_top = 0;
  std::vector<T> matVx2Vz, matVy2Vz;  // [siz_iz*9]

  struct Face {
    int enable = 0;
    int ni1, ni2, nj1, nj2, nk1, nk2;
    int nx, ny, nz;
    size_t siz_icmp;
    std::vector<T> A, B, D;
    std::vector<T> aux;  // [4 levels][9][box]
    int lvl_pre = 0, lvl_end = 3;
  } face[3][2];

  // src_t (src_t.h:14-53)
  int nsrc = 0, max_nt = 0, max_ext = 0, force_actived = 0, moment_actived = 0;
  std::vector<int> it_begin, it_end, ext_num, ext_indx;
  std::vector<T> ext_coef;
  std::vector<T> F[3], M[6];  // [src][max_nt][4]

  // iorecv_t (io_funcs.h:14-38)
  struct Recv {
    size_t indx1d[8];
    T di, dj, dk;
  };
  std::vector<Recv> recv;
  std::vector<float> seismo;  // [nrecv][9][nt_total]

  // free-surface peak ground motion (PG_calcu_gpu, wav_t.cu:281-360): [15][ny][nx] PGV, PGVh,
  // PGVx..z, PGA, PGAh, PGAx..z, PGD, PGDh, PGDx..z, and the displacement accumulator [3][ny][nx]
  std::vector<T> pg, dis;

  T *lev(int l) { return wave.data() + (size_t)l * 9 * g.siz_icmp; }
  const T *metric_c(int c) const { return metric.data() + (size_t)c * g.siz_icmp; }
  const T *med_c(int c) const { return med.data() + (size_t)c * g.siz_icmp; }

  int ncmp_medium() const {
    if (medium_type == CGFD_MEDIUM_ACOUSTIC_ISO) return 2;  // rho, kappa
    return medium_type == CGFD_MEDIUM_ELASTIC_ISO ? 3 : (medium_type == CGFD_MEDIUM_ELASTIC_VTI ? 6 : 22);
  }

  // full symmetric 6x6 for VTI/aniso at point iptr (VTI mapping: sv_curv_col_el_vti_gpu.cu:401-407)
  void cij(size_t iptr, T C[6][6]) const {
    if (medium_type == CGFD_MEDIUM_ELASTIC_VTI) {
      T c11 = med_c(1)[iptr], c13 = med_c(2)[iptr], c33 = med_c(3)[iptr], c55 = med_c(4)[iptr],
        c66 = med_c(5)[iptr];
      T c12 = (T)(c11 - 2.0 * c66);
      for (int a = 0; a < 6; a++)
        for (int b = 0; b < 6; b++) C[a][b] = 0;
      C[0][0] = c11; C[0][1] = c12; C[0][2] = c13;
      C[1][0] = c12; C[1][1] = c11; C[1][2] = c13;
      C[2][0] = c13; C[2][1] = c13; C[2][2] = c33;
      C[3][3] = c55; C[4][4] = c55; C[5][5] = c66;
    } else {
      int n = 1;
      for (int a = 0; a < 6; a++)
        for (int b = a; b < 6; b++) {
          C[a][b] = med_c(n)[iptr];
          C[b][a] = C[a][b];
          n++;
        }
    }
  }

  // ---- Hooke's law, reference evaluation order --------------------------------------------
  // iso inner/vlow form: sv_curv_col_el_iso_gpu.cu:425-451
  static void hooke_iso_full(T lam, T mu, T lam2mu, const T m[3][3], const T D[3][3], T h[6]) {
    // m[axis][comp] metric, D[axis][vcomp] derivative of V along axis
    T xix = m[0][0], xiy = m[0][1], xiz = m[0][2], etx = m[1][0], ety = m[1][1], etz = m[1][2],
      ztx = m[2][0], zty = m[2][1], ztz = m[2][2];
    T DxVx = D[0][0], DxVy = D[0][1], DxVz = D[0][2], DyVx = D[1][0], DyVy = D[1][1], DyVz = D[1][2],
      DzVx = D[2][0], DzVy = D[2][1], DzVz = D[2][2];
    h[0] = lam2mu * (xix * DxVx + etx * DyVx + ztx * DzVx) +
           lam * (xiy * DxVy + ety * DyVy + zty * DzVy + xiz * DxVz + etz * DyVz + ztz * DzVz);
    h[1] = lam2mu * (xiy * DxVy + ety * DyVy + zty * DzVy) +
           lam * (xix * DxVx + etx * DyVx + ztx * DzVx + xiz * DxVz + etz * DyVz + ztz * DzVz);
    h[2] = lam2mu * (xiz * DxVz + etz * DyVz + ztz * DzVz) +
           lam * (xix * DxVx + etx * DyVx + ztx * DzVx + xiy * DxVy + ety * DyVy + zty * DzVy);
    // Voigt order yz, xz, xy
    h[3] = mu * (xiz * DxVy + xiy * DxVz + etz * DyVy + ety * DyVz + ztz * DzVy + zty * DzVz);
    h[4] = mu * (xiz * DxVx + xix * DxVz + etz * DyVx + etx * DyVz + ztz * DzVx + ztx * DzVz);
    h[5] = mu * (xiy * DxVx + xix * DxVy + ety * DyVx + etx * DyVy + zty * DzVx + ztx * DzVy);
  }
  // iso one-axis form: sv_curv_col_el_iso_gpu.cu:833-841
  static void hooke_iso_axis(T lam, T mu, T lam2mu, const T m[3], const T D[3], T h[6]) {
    h[0] = lam2mu * m[0] * D[0] + lam * m[1] * D[1] + lam * m[2] * D[2];
    h[1] = lam * m[0] * D[0] + lam2mu * m[1] * D[1] + lam * m[2] * D[2];
    h[2] = lam * m[0] * D[0] + lam * m[1] * D[1] + lam2mu * m[2] * D[2];
    h[3] = mu * (m[2] * D[1] + m[1] * D[2]);
    h[4] = mu * (m[2] * D[0] + m[0] * D[2]);
    h[5] = mu * (m[1] * D[0] + m[0] * D[1]);
  }
  // iso free-surface term of the PML faces: sv_curv_col_el_iso_gpu.cu:873-896
  static void hooke_iso_surf(T lam, T mu, T lam2mu, const T z[3], const T D[3], T h[6]) {
    h[0] = lam2mu * (z[0] * D[0]) + lam * (z[1] * D[1] + z[2] * D[2]);
    h[1] = lam2mu * (z[1] * D[1]) + lam * (z[0] * D[0] + z[2] * D[2]);
    h[2] = lam2mu * (z[2] * D[2]) + lam * (z[0] * D[0] + z[1] * D[1]);
    h[3] = mu * (z[2] * D[1] + z[1] * D[2]);
    h[4] = mu * (z[2] * D[0] + z[0] * D[2]);
    h[5] = mu * (z[1] * D[0] + z[0] * D[1]);
  }
  // aniso form: sv_curv_col_el_aniso_gpu.cu:495-518 (VTI is the same with zero entries)
  static void hooke_aniso_axes(const T C[6][6], const T m[][3], const T D[][3], int naxes, T h[6]) {
    for (int I = 0; I < 6; I++) {
      T s = 0;
      bool first = true;
      for (int ax = 0; ax < naxes; ax++)
        for (int vc = 0; vc < 3; vc++) {
          // coefficient of D[ax][vc]: sum_j C[I][voigt(vc,j)] * m[ax][j]
          T cf = C[I][voigt(vc, 0)] * m[ax][0] + C[I][voigt(vc, 1)] * m[ax][1] + C[I][voigt(vc, 2)] * m[ax][2];
          if (first) { s = cf * D[ax][vc]; first = false; }
          else s += cf * D[ax][vc];
        }
      h[I] = s;
    }
  }

  // ---------------------------------------------------------------------------------------
  // setup
  // ---------------------------------------------------------------------------------------
  void setup(const cgfd_problem_desc *d) {
    if (d->ni < 8 || d->nj < 8 || d->nk < 8) throw std::runtime_error("grid too small");
    medium_type = d->medium_type;
    if (medium_type != CGFD_MEDIUM_ELASTIC_ISO && medium_type != CGFD_MEDIUM_ELASTIC_VTI &&
        medium_type != CGFD_MEDIUM_ELASTIC_ANISO && medium_type != CGFD_MEDIUM_ACOUSTIC_ISO)
      throw std::runtime_error("unsupported medium_type");
    g.set(d->ni, d->nj, d->nk);
    dt = (T)d->dt; t0 = (T)d->t0; nt_total = d->nt_total;
    metric.resize(10 * g.siz_icmp);
    for (size_t n = 0; n < metric.size(); n++) metric[n] = (T)d->metric[n];
    int nc = ncmp_medium();
    med.resize((size_t)nc * g.siz_icmp);
    for (size_t n = 0; n < med.size(); n++) med[n] = (T)d->medium[n];
    // md_rho_to_slow (md_t.cu:622-637), done by main before the driver.
    for (size_t n = 0; n < g.siz_icmp; n++) med[n] = med[n] > (T)1e-10 ? (T)(1.0 / med[n]) : (T)0;
    wave.assign(4 * 9 * g.siz_icmp, (T)0);
    free_top = d->free_top;
    if (free_top && medium_type != CGFD_MEDIUM_ACOUSTIC_ISO) dvh2dvz();  // drv_rk_curv_col.cu:89: "not need"
    pml_set(d);
    src_set(d);
    recv_set(d);
  }

  // sv_curv_col_el_{iso,vti,aniso}_dvh2dvz
  void dvh2dvz() {
    matVx2Vz.assign(g.siz_iz * 9, (T)0);
    matVy2Vz.assign(g.siz_iz * 9, (T)0);
    int k = g.nk2;
    for (int j = g.nj1; j <= g.nj2; j++)
      for (int i = g.ni1; i <= g.ni2; i++) {
        size_t iptr = i + j * g.siz_iy + k * g.siz_iz;
        T e[3][3];
        for (int a = 0; a < 3; a++)
          for (int b = 0; b < 3; b++) e[a][b] = metric_c(1 + 3 * a + b)[iptr];
        T A[3][3], B[3][3], C[3][3], AB[3][3], AC[3][3];
        T sign;
        if (medium_type == CGFD_MEDIUM_ELASTIC_ISO) {
          // sv_curv_col_el_iso_gpu.cu:1205-1243
          T lam = med_c(1)[iptr], mu = med_c(2)[iptr];
          T lam2mu = lam + (T)2.0f * mu;
          T e11 = e[0][0], e12 = e[0][1], e13 = e[0][2], e21 = e[1][0], e22 = e[1][1], e23 = e[1][2],
            e31 = e[2][0], e32 = e[2][1], e33 = e[2][2];
          A[0][0] = lam2mu * e31 * e31 + mu * (e32 * e32 + e33 * e33);
          A[0][1] = lam * e31 * e32 + mu * e32 * e31;
          A[0][2] = lam * e31 * e33 + mu * e33 * e31;
          A[1][0] = lam * e32 * e31 + mu * e31 * e32;
          A[1][1] = lam2mu * e32 * e32 + mu * (e31 * e31 + e33 * e33);
          A[1][2] = lam * e32 * e33 + mu * e33 * e32;
          A[2][0] = lam * e33 * e31 + mu * e31 * e33;
          A[2][1] = lam * e33 * e32 + mu * e32 * e33;
          A[2][2] = lam2mu * e33 * e33 + mu * (e31 * e31 + e32 * e32);
          invert3x3(A);
          B[0][0] = -lam2mu * e31 * e11 - mu * (e32 * e12 + e33 * e13);
          B[0][1] = -lam * e31 * e12 - mu * e32 * e11;
          B[0][2] = -lam * e31 * e13 - mu * e33 * e11;
          B[1][0] = -lam * e32 * e11 - mu * e31 * e12;
          B[1][1] = -lam2mu * e32 * e12 - mu * (e31 * e11 + e33 * e13);
          B[1][2] = -lam * e32 * e13 - mu * e33 * e12;
          B[2][0] = -lam * e33 * e11 - mu * e31 * e13;
          B[2][1] = -lam * e33 * e12 - mu * e32 * e13;
          B[2][2] = -lam2mu * e33 * e13 - mu * (e31 * e11 + e32 * e12);
          C[0][0] = -lam2mu * e31 * e21 - mu * (e32 * e22 + e33 * e23);
          C[0][1] = -lam * e31 * e22 - mu * e32 * e21;
          C[0][2] = -lam * e31 * e23 - mu * e33 * e21;
          C[1][0] = -lam * e32 * e21 - mu * e31 * e22;
          C[1][1] = -lam2mu * e32 * e22 - mu * (e31 * e21 + e33 * e23);
          C[1][2] = -lam * e32 * e23 - mu * e33 * e22;
          C[2][0] = -lam * e33 * e21 - mu * e31 * e23;
          C[2][1] = -lam * e33 * e22 - mu * e32 * e23;
          C[2][2] = -lam2mu * e33 * e23 - mu * (e31 * e21 + e32 * e22);
          sign = 1;
        } else {
          // sv_curv_col_el_aniso_gpu.cu:1409-1446 (VTI :1205-1250 is the same with zeros)
          T Cm[6][6];
          cij(iptr, Cm);
          for (int a = 0; a < 3; a++)
            for (int l = 0; l < 3; l++) {
              T sa = 0, sb = 0, sc = 0;
              for (int jj = 0; jj < 3; jj++) {
                int I = voigt(a, jj);
                T ca = Cm[I][voigt(l, 0)] * e[2][0] + Cm[I][voigt(l, 1)] * e[2][1] + Cm[I][voigt(l, 2)] * e[2][2];
                T cb = Cm[I][voigt(l, 0)] * e[0][0] + Cm[I][voigt(l, 1)] * e[0][1] + Cm[I][voigt(l, 2)] * e[0][2];
                T cc = Cm[I][voigt(l, 0)] * e[1][0] + Cm[I][voigt(l, 1)] * e[1][1] + Cm[I][voigt(l, 2)] * e[1][2];
                if (jj == 0) { sa = ca * e[2][jj]; sb = cb * e[2][jj]; sc = cc * e[2][jj]; }
                else { sa += ca * e[2][jj]; sb += cb * e[2][jj]; sc += cc * e[2][jj]; }
              }
              A[a][l] = sa; B[a][l] = sb; C[a][l] = sc;
            }
          invert3x3(A);
          sign = -1;
        }
        matmul3x3(A, B, AB);
        matmul3x3(A, C, AC);
        size_t ij = (j * g.siz_iy + i) * 9;
        for (int r = 0; r < 3; r++)
          for (int c = 0; c < 3; c++) {
            matVx2Vz[ij + r * 3 + c] = sign * AB[r][c];
            matVy2Vz[ij + r * 3 + c] = sign * AC[r][c];
          }
      }
  }

  // bdry_pml_set + bdry_cal_abl_len_dh, bdry_t.cu:85-451
  void pml_set(const cgfd_problem_desc *d) {
    for (int idim = 0; idim < 3; idim++)
      for (int iside = 0; iside < 2; iside++) {
        Face &f = face[idim][iside];
        const cgfd_pml_face &in = d->pml[idim][iside];
        f.enable = in.enable ? 1 : 0;
        if (!f.enable) continue;
        if (idim == 2 && iside == 1 && free_top) throw std::runtime_error("z2 cannot be both PML and free");
        int N = in.num_layers;
        if (N < 1) throw std::runtime_error("pml num_layers < 1");
        f.ni1 = g.ni1; f.ni2 = g.ni2; f.nj1 = g.nj1; f.nj2 = g.nj2; f.nk1 = g.nk1; f.nk2 = g.nk2;
        if (idim == 0 && iside == 0) f.ni2 = g.ni1 + N;
        if (idim == 0 && iside == 1) f.ni1 = g.ni2 - N;
        if (idim == 1 && iside == 0) f.nj2 = g.nj1 + N;
        if (idim == 1 && iside == 1) f.nj1 = g.nj2 - N;
        if (idim == 2 && iside == 0) f.nk2 = g.nk1 + N;
        if (idim == 2 && iside == 1) f.nk1 = g.nk2 - N;
        f.nx = f.ni2 - f.ni1 + 1; f.ny = f.nj2 - f.nj1 + 1; f.nz = f.nk2 - f.nk1 + 1;
        f.siz_icmp = (size_t)f.nx * f.ny * f.nz;
        if (!d->coord) throw std::runtime_error("PML needs coord");
        // bdry_cal_abl_len_dh: average spacing along idim over the face box (double sums)
        const float *x3d = d->coord, *y3d = d->coord + g.siz_icmp, *z3d = d->coord + 2 * g.siz_icmp;
        double L = 0.0;
        long num = 0;
        int lo[3] = {f.ni1, f.nj1, f.nk1}, hi[3] = {f.ni2, f.nj2, f.nk2};
        int a1 = idim == 0 ? 1 : 0, a2 = idim == 2 ? 1 : 2;  // the two other axes, outer = a2
        for (int o2 = lo[a2]; o2 <= hi[a2]; o2++)
          for (int o1 = lo[a1]; o1 <= hi[a1]; o1++) {
            int ijk[3];
            ijk[a1] = o1; ijk[a2] = o2; ijk[idim] = lo[idim];
            size_t p0 = ijk[0] + ijk[1] * g.siz_iy + ijk[2] * g.siz_iz;
            double x0 = x3d[p0], y0 = y3d[p0], z0 = z3d[p0];
            for (int n = lo[idim] + 1; n <= hi[idim]; n++) {
              ijk[idim] = n;
              size_t p = ijk[0] + ijk[1] * g.siz_iy + ijk[2] * g.siz_iz;
              double x1 = x3d[p], y1 = y3d[p], z1 = z3d[p];
              L += sqrt((x1 - x0) * (x1 - x0) + (y1 - y0) * (y1 - y0) + (z1 - z0) * (z1 - z0));
              x0 = x1; y0 = y1; z0 = z1;
              num += 1;
            }
          }
        float avg_dh = (float)(L / num);
        float L0 = avg_dh * (float)(hi[idim] - lo[idim]);
        int npoints = N + 1;
        float num_lay = (float)(npoints - 1);
        // bdry_pml_cal_R / _dmax / _d / _a / _b (bdry_t.cu:297-330), CONSPD=2, CONSPA=1, CONSPB=2
        float Rpp = (float)pow(10, -((log10((double)num_lay) - 1.0) / log10(2.0) + 4.0));
        float dmax = (float)(-in.ref_vel / (2.0 * L0) * log(Rpp) * (2.0f + 1.0));
        float amax = in.alpha_max, bmax = in.beta_max;
        f.A.assign(npoints, 0); f.B.assign(npoints, 0); f.D.assign(npoints, 0);
        for (int n = 0; n < npoints; n++) {
          float Lx = n * avg_dh;
          int i = iside == 0 ? npoints - 1 - n : n;
          float Dv = Lx < 0 ? 0.0f : (float)(dmax * pow(Lx / L0, 2.0f));
          float Av = Lx < 0 ? 0.0f : (float)(amax * (1.0 - pow(Lx / L0, 1.0f)));
          float Bv = Lx < 0 ? 1.0f : (float)(1.0 + (bmax - 1.0) * pow(Lx / L0, 2.0f));
          Dv /= Bv;
          Av += Dv;
          Bv = (float)(1.0 / Bv);
          f.A[i] = Av; f.B[i] = Bv; f.D[i] = Dv;
        }
        f.aux.assign(4 * 9 * f.siz_icmp, (T)0);
      }
  }

  // wavelets: src_t.cu:834-903
  static float wavelet_val(float t, int name, const float *c) {
    const float PIf = (float)3.1415926535897;
    switch (name) {
      case CGFD_WAVELET_RICKER: {
        float u = (float)((t - c[1]) * 2.0 * PIf * c[0]);
        return (float)((1 - u * u / 2.0) * exp(-u * u / 4.0));
      }
      case CGFD_WAVELET_RICKER_DERIV: {
        float u = (float)((t - c[1]) * 2.0 * PIf * c[0]);
        return (float)(u * (-3 + 1.0 / 2.0 * u * u) * exp(-u * u / 4) * PIf * c[0]);
      }
      case CGFD_WAVELET_GAUSSIAN: {
        float a = c[0], t0_ = c[1];
        return (float)(exp(-(t - t0_) * (t - t0_) / (a * a)) / (sqrtf(PIf) * a));
      }
      case CGFD_WAVELET_GAUSSIAN_DERIV: {
        float a = c[0], t0_ = c[1];
        return (float)(exp(-(t - t0_) * (t - t0_) / (a * a)) / (sqrtf(PIf) * a) * (-2 * (t - t0_) / (a * a)));
      }
      case CGFD_WAVELET_KLAUDER: {
        float tt0 = 0.2f, f1 = 1.5f, f2 = 41.5f, T_ = 20.0f;
        float K = (f2 - f1) / T_;
        float fM = (float)((f2 + f1) / 2.0);
        return (float)((sin(PIf * K * t * (T_ - (t - tt0))) * cos(2 * PIf * fM * (t - tt0))) / (PIf * K * (t - tt0)));
      }
    }
    throw std::runtime_error("unknown wavelet");
  }

  static float fun_gauss(float t, float a, float t0_) {  // src_t.cu:852-858
    return (float)(exp(-(t - t0_) * (t - t0_) / (a * a)) / (sqrtf((float)3.1415926535897) * a));
  }

  // angle2moment, src_t.cu:910-950
  static void angle2moment(float strike, float dip, float rake, float *mt) {
    const double PId = 3.1415926535897;
    float dip_pi = (float)(dip / 180.0 * PId), strike_pi = (float)(strike / 180.0 * PId),
          rake_pi = (float)(rake / 180.0 * PId);
    float M11 = (float)(-(sin(dip_pi) * cos(rake_pi) * sin(2.0 * strike_pi) +
                          sin(2.0 * dip_pi) * sin(rake_pi) * sin(strike_pi) * sin(strike_pi)));
    float M22 = (float)(sin(dip_pi) * cos(rake_pi) * sin(2.0 * strike_pi) -
                        sin(2.0 * dip_pi) * sin(rake_pi) * cos(strike_pi) * cos(strike_pi));
    float M33 = -(M11 + M22);
    float M12 = (float)(sin(dip_pi) * cos(rake_pi) * cos(2.0 * strike_pi) +
                        0.5 * sin(2.0 * dip_pi) * sin(rake_pi) * sin(2.0 * strike_pi));
    float M13 = (float)(-(cos(dip_pi) * cos(rake_pi) * cos(strike_pi) +
                          cos(2.0 * dip_pi) * sin(rake_pi) * sin(strike_pi)));
    float M23 = (float)(-(cos(dip_pi) * cos(rake_pi) * sin(strike_pi) -
                          cos(2.0 * dip_pi) * sin(rake_pi) * cos(strike_pi)));
    mt[0] = M22; mt[1] = M11; mt[2] = M33; mt[3] = -M13; mt[4] = -M23; mt[5] = M12;
  }

  // LagInterp_Piecewise_1d, interp.cu:220-299
  static float lag_interp(const float *t, const float *z, int ni, int order, float t_start, float dt_, float ti) {
    float Li = 0.0f;
    int lower, upper;
    if (order % 2 == 0) { lower = order / 2; upper = order / 2; }
    else { lower = order / 2; upper = order / 2 + 1; }
    int indx = (int)((ti - t_start) / dt_ + 0.5);
    if (indx > ni - 1) indx = ni - 1;
    std::vector<float> Lx(order + 1 + 16, 0.0f);
    if ((indx - lower >= 0) && (indx + upper <= ni - 1)) {
      for (int i = indx - lower; i <= indx + upper; i++) {
        Lx[i - indx + lower] = 1;
        for (int j = indx - lower; j <= indx + upper; j++) {
          if (i == j) continue;
          Lx[i - indx + lower] = Lx[i - indx + lower] * (ti - t[j]) / (t[i] - t[j]);
        }
      }
      for (int i = indx - lower; i <= indx + upper; i++) Li = Li + Lx[i - indx + lower] * z[i];
    }
    if (indx - lower < 0) {
      int inc = lower - indx;
      for (int i = 0; i <= indx + upper + inc; i++) {
        Lx[i] = 1;
        for (int j = 0; j <= indx + upper + inc; j++) {
          if (i == j) continue;
          Lx[i] = Lx[i] * (ti - t[j]) / (t[i] - t[j]);
        }
      }
      for (int i = 0; i <= indx + upper + inc; i++) Li = Li + Lx[i] * z[i];
    }
    if (indx + upper > ni - 1) {
      int inc = indx + upper - (ni - 1);
      for (int i = indx - lower - inc; i <= ni - 1; i++) {
        Lx[i - indx + lower + inc] = 1;
        for (int j = indx - lower - inc; j <= ni - 1; j++) {
          if (i == j) continue;
          Lx[i - indx + lower + inc] = Lx[i - indx + lower + inc] * (ti - t[j]) / (t[i] - t[j]);
        }
      }
      for (int i = indx - lower - inc; i <= ni - 1; i++) Li = Li + Lx[i - indx + lower + inc] * z[i];
    }
    return Li;
  }

  // src_read_locate_file (index location), src_t.cu:143-790
  void src_set(const cgfd_problem_desc *d) {
    const cgfd_source_desc &s = d->src;
    nsrc = 0;
    if (s.num <= 0) return;

    const int half = 3;  // fd->fdx_max_half_len
    const int len_ext = 2 * half + 1;
    max_ext = len_ext * len_ext * len_ext;
    std::vector<int> idx(3 * s.num), inthread(s.num, 0), outside(s.num, 0);
    std::vector<float> inc(3 * s.num);
    int gnk2 = g.nk - 1;
    std::unique_ptr<Locator> lc;
    if (s.loc_coord_type == 1) {
      if (!d->coord) throw std::runtime_error("coord is required to locate sources");
      lc.reset(new Locator(g, d->coord));
    }
    for (int is = 0; is < s.num; is++) {
      float c[3] = {s.loc[3 * is], s.loc[3 * is + 1], s.loc[3 * is + 2]};
      if (s.loc_coord_type == 1) {  // src_t.cu:341-398
        if (s.loc_3dim == 1) lc->depth_to_axis(c[0], c[1], &c[2]);
        int gi[3];
        float fi[3];
        lc->locate(c[0], c[1], c[2], gi, fi);
        for (int a = 0; a < 3; a++) { idx[3 * is + a] = gi[a]; inc[3 * is + a] = fi[a]; }
      } else {
        if (s.loc_3dim == 1) c[2] = gnk2 - c[2];
        for (int a = 0; a < 3; a++) {
          int gi = (int)(c[a] + 0.5);
          inc[3 * is + a] = c[a] - gi;
          idx[3 * is + a] = gi;
        }
      }
      // src_t.cu:296-307: an index outside the grid is replaced by -1000, which later
      // leaves the source without any smoothing point inside the grid.
      int tot[3] = {g.ni, g.nj, g.nk};
      for (int a = 0; a < 3; a++)
        if (idx[3 * is + a] < 0 || idx[3 * is + a] > tot[a] - 1) outside[is] = 1;
      // src_glob_ext_ishere, tested with the rounded (unreplaced) index
      int si = idx[3 * is], sj = idx[3 * is + 1], sk = idx[3 * is + 2];
      if (si - half <= g.ni - 1 && si + half >= 0 && sj - half <= g.nj - 1 && sj + half >= 0 &&
          sk - half <= g.nk - 1 && sk + half >= 0) {
        inthread[is] = 1;
        nsrc++;
      }
    }
    if (s.cmp_type == 1 || s.cmp_type == 3) force_actived = 1;
    else if (s.cmp_type == 2 || s.cmp_type == 3) moment_actived = 1;
    if (s.stf_given == 0) max_nt = (int)(s.stf_length / (float)dt + 0.5);
    else max_nt = (int)(((s.stf_nt - 1) * s.stf_dt / (float)dt) + 0.5) + 1;
    const float rk_rhs_time[4] = {0.0f, 0.5f, 0.5f, 1.0f};
    it_begin.assign(nsrc, 0); it_end.assign(nsrc, 0); ext_num.assign(nsrc, 0);
    ext_indx.assign((size_t)nsrc * max_ext, 0); ext_coef.assign((size_t)nsrc * max_ext, 0);
    for (int c = 0; c < 3; c++) F[c].assign(force_actived ? (size_t)nsrc * max_nt * 4 : 0, 0);
    for (int c = 0; c < 6; c++) M[c].assign(moment_actived ? (size_t)nsrc * max_nt * 4 : 0, 0);
    std::vector<float> delt(max_ext), t_in(s.stf_given == 1 ? s.stf_nt : 1);
    int is_local = 0;
    for (int is = 0; is < s.num; is++) {
      if (!inthread[is]) continue;
      int si = idx[3 * is] + NG, sj = idx[3 * is + 1] + NG, sk = idx[3 * is + 2] + NG;
      float cmpv[9];
      for (int c = 0; c < 9; c++) cmpv[c] = s.stf_given == 0 ? s.cmp[9 * is + c] : 0.0f;
      std::vector<float> vals;  // stf by values, [nt][9]
      if (s.stf_given == 1) vals.assign(s.cmp_values + (size_t)is * s.stf_nt * 9, s.cmp_values + (size_t)(is + 1) * s.stf_nt * 9);
      if (moment_actived && s.mechanism_type == 1) {
        size_t iptr = si + sj * g.siz_iy + sk * g.siz_iz;
        auto conv = [&](float *v) {
          float mu = v[6];
          if (mu < 0.0f) {
            if (medium_type != CGFD_MEDIUM_ELASTIC_ISO) throw std::runtime_error("mu<0 needs iso medium");
            mu = (float)med_c(2)[iptr];
          }
          float mt[6];
          angle2moment(v[3], v[4], v[5], mt);
          float M0 = mu * v[7] * v[8];
          for (int c = 0; c < 6; c++) v[3 + c] = M0 * mt[c];
        };
        if (s.stf_given == 0) conv(cmpv);
        else for (int it = 0; it < s.stf_nt; it++) conv(&vals[(size_t)it * 9]);
      }
      // smoothing weights: src_cal_norm_delt3d (src_t.cu:796-827), width = half/2
      float wid = half / 2.0f;
      float x0 = inc[3 * is], y0 = inc[3 * is + 1], z0 = inc[3 * is + 2];
      float SUM = 0.0f;
      int ip = 0;
      for (int k = -half; k <= half; k++)
        for (int j = -half; j <= half; j++)
          for (int i = -half; i <= half; i++) {
            float D1 = fun_gauss(i - x0, wid, 0.0f), D2 = fun_gauss(j - y0, wid, 0.0f), D3 = fun_gauss(k - z0, wid, 0.0f);
            delt[ip] = D1 * D2 * D3;
            SUM += delt[ip];
            ip++;
          }
      for (int n = 0; n < max_ext; n++) delt[n] /= SUM;
      int iext = 0;
      for (int k = sk - half; k <= sk + half; k++)
        for (int j = sj - half; j <= sj + half; j++)
          for (int i = si - half; i <= si + half; i++) {
            if (!outside[is] && g.lindx_is_inner(i, j, k)) {
              int ic = (i - (si - half)) + len_ext * (j - (sj - half)) + len_ext * len_ext * (k - (sk - half));
              ext_indx[(size_t)is_local * max_ext + iext] = (int)(i + j * g.siz_iy + k * g.siz_iz);
              ext_coef[(size_t)is_local * max_ext + iext] = (T)delt[ic];
              iext++;
            }
          }
      ext_num[is_local] = iext;
      float tstart = s.t_start[is];
      int itb = (int)((tstart - (float)t0) / (float)dt);
      it_begin[is_local] = itb;
      it_end[is_local] = itb + max_nt - 1;
      if (s.stf_given == 1)
        for (int it = 0; it < s.stf_nt; it++) t_in[it] = tstart + it * s.stf_dt;
      float t_shift = tstart - (itb * (float)dt + (float)t0);
      for (int it = itb; it <= itb + max_nt - 1; it++) {
        int it1 = it - itb;
        size_t iptr_it = (size_t)is_local * max_nt * 4 + (size_t)it1 * 4;
        for (int istage = 0; istage < 4; istage++) {
          size_t iptr = iptr_it + istage;
          if (s.stf_given == 0) {
            float t = it1 * (float)dt + rk_rhs_time[istage] * (float)dt - t_shift;
            float stf = wavelet_val(t, s.wavelet[is], s.wavelet_coefs + 10 * is);
            if (force_actived) for (int c = 0; c < 3; c++) F[c][iptr] = stf * cmpv[c];
            if (moment_actived) for (int c = 0; c < 6; c++) M[c][iptr] = stf * cmpv[3 + c];
          } else {
            // quirk kept: the by-value branch uses the global step index (src_t.cu:683)
            float t = it * (float)dt + rk_rhs_time[istage] * (float)dt - t_shift;
            std::vector<float> col(s.stf_nt);
            if (force_actived)
              for (int c = 0; c < 3; c++) {
                for (int n = 0; n < s.stf_nt; n++) col[n] = vals[(size_t)n * 9 + c];
                F[c][iptr] = lag_interp(t_in.data(), col.data(), s.stf_nt, 3, tstart, s.stf_dt, t);
              }
            if (moment_actived)
              for (int c = 0; c < 6; c++) {
                for (int n = 0; n < s.stf_nt; n++) col[n] = vals[(size_t)n * 9 + 3 + c];
                M[c][iptr] = lag_interp(t_in.data(), col.data(), s.stf_nt, 3, tstart, s.stf_dt, t);
              }
          }
        }
      }
      is_local++;
    }
  }

  // io_recv_read_locate (index location), io_funcs.cu:24-299
  void recv_set(const cgfd_problem_desc *d) {
    const cgfd_station_desc &s = d->sta;
    recv.clear();
    int gnk2 = g.nk - 1;
    std::unique_ptr<Locator> lc;
    for (int ir = 0; ir < s.num; ir++) {
      int ix, iy, iz;
      float dx, dy, dz;
      if (s.flag_coord[ir] == 1) {  // io_funcs.cu:95-169
        if (!lc) {
          if (!d->coord) throw std::runtime_error("coord is required to locate stations");
          lc.reset(new Locator(g, d->coord));
        }
        float c[3] = {s.loc[3 * ir], s.loc[3 * ir + 1], s.loc[3 * ir + 2]};
        if (s.flag_depth[ir] == 1) lc->depth_to_axis(c[0], c[1], &c[2]);
        int gi[3];
        float fi[3];
        lc->locate(c[0], c[1], c[2], gi, fi);
        for (int a = 0; a < 3; a++)
          if (fi[a] < 0.0) { fi[a] = 1.0 + fi[a]; gi[a] -= 1; }
        ix = gi[0]; iy = gi[1]; iz = gi[2];
        dx = fi[0]; dy = fi[1]; dz = fi[2];
      } else {
        float c[3] = {s.loc[3 * ir] - 1, s.loc[3 * ir + 1] - 1, s.loc[3 * ir + 2]};
        if (s.flag_depth[ir] == 1) c[2] = gnk2 - c[2];
        else c[2] -= 1;
        ix = (int)c[0]; iy = (int)c[1]; iz = (int)c[2];
        dx = c[0] - ix; dy = c[1] - iy; dz = c[2] - iz;
        if (ix < 0 || ix > g.ni) ix = -1000;
        if (iy < 0 || iy > g.nj) iy = -1000;
        if (iz < 0 || iz > g.nk) iz = -1000;
      }
      if (!(ix >= 0 && ix <= g.ni - 1 && iy >= 0 && iy <= g.nj - 1 && iz >= 0 && iz <= g.nk - 1)) continue;
      int il = ix + NG, jl = iy + NG, kl = iz + NG;
      Recv r;
      for (int n = 0; n < 8; n++) {
        int di = n & 1, dj = (n >> 1) & 1, dk = (n >> 2) & 1;
        r.indx1d[n] = (il + di) + (jl + dj) * g.siz_iy + (kl + dk) * g.siz_iz;
      }
      r.di = (T)dx; r.dj = (T)dy; r.dk = (T)dz;
      recv.push_back(r);
    }
    seismo.assign(recv.size() * 9 * (size_t)nt_total, 0.0f);
  }

  // ---------------------------------------------------------------------------------------
  // one stage RHS
  // ---------------------------------------------------------------------------------------
  struct Ops {
    Op x, y, z;          // normal ops for this pair/stage
    Op zlay[4];          // per-layer z ops (vlow)
  };

  Ops make_ops(int ipair, int istage) const {
    Ops o;
    o.x = kOps[3][op_dir(ipair, istage, 0)];
    o.y = kOps[3][op_dir(ipair, istage, 1)];
    o.z = kOps[3][op_dir(ipair, istage, 2)];
    for (int l = 0; l < 4; l++) o.zlay[l] = kOps[l][op_dir(ipair, istage, 2)];
    return o;
  }

  static T fd_apply(const Op &op, const T *v, size_t iptr, long shift) {
    T c0 = (T)(float)op.coef[0];
    T r = c0 * v[iptr + op.idx[0] * shift];
    for (int n = 1; n < op.len; n++) r += (T)(float)op.coef[n] * v[iptr + op.idx[n] * shift];
    return r;
  }

  // wavefield component pointers, reference order Vx,Vy,Vz,Txx,Tyy,Tzz,Tyz,Txz,Txy
  enum { VX, VY, VZ, TXX, TYY, TZZ, TYZ, TXZ, TXY };

  void rhs_inner(const T *w, T *h, const Ops &o) {
    const Grid &G = g;
    long sy = (long)G.siz_iy, sz = (long)G.siz_iz;
#pragma omp parallel for schedule(static)
    for (int k = G.nk1; k <= G.nk2; k++)
      for (int j = G.nj1; j <= G.nj2; j++)
        for (int i = G.ni1; i <= G.ni2; i++) {
          size_t iptr = i + j * G.siz_iy + k * G.siz_iz;
          T Dv[3][3], Dt[3][6];  // [axis][vcomp], [axis][Voigt tcomp]
          const long sh[3] = {1, sy, sz};
          const Op *op[3] = {&o.x, &o.y, &o.z};
          for (int a = 0; a < 3; a++) {
            for (int c = 0; c < 3; c++) Dv[a][c] = fd_apply(*op[a], w + c * G.siz_icmp, iptr, sh[a]);
            // Voigt: xx,yy,zz,yz,xz,xy = cmp 3,4,5,6,7,8
            for (int c = 0; c < 6; c++) Dt[a][c] = fd_apply(*op[a], w + (3 + c) * G.siz_icmp, iptr, sh[a]);
          }
          T m[3][3];
          for (int a = 0; a < 3; a++)
            for (int b = 0; b < 3; b++) m[a][b] = metric_c(1 + 3 * a + b)[iptr];
          T slw = med_c(0)[iptr];
          // momentum: sv_curv_col_el_iso_gpu.cu:414-422
          // hVx: xix*DxTxx + xiy*DxTxy + xiz*DxTxz + ...
          const int tv[3][3] = {{0, 5, 4}, {5, 1, 3}, {4, 3, 2}};  // traction comps for hV_i
          for (int c = 0; c < 3; c++) {
            T s = m[0][0] * Dt[0][tv[c][0]] + m[0][1] * Dt[0][tv[c][1]] + m[0][2] * Dt[0][tv[c][2]] +
                  m[1][0] * Dt[1][tv[c][0]] + m[1][1] * Dt[1][tv[c][1]] + m[1][2] * Dt[1][tv[c][2]] +
                  m[2][0] * Dt[2][tv[c][0]] + m[2][1] * Dt[2][tv[c][1]] + m[2][2] * Dt[2][tv[c][2]];
            h[c * G.siz_icmp + iptr] = slw * s;
          }
          T ht[6];
          hooke_full(iptr, m, Dv, ht);
          for (int c = 0; c < 6; c++) h[(3 + c) * G.siz_icmp + iptr] = ht[c];
        }
  }

  void hooke_full(size_t iptr, const T m[3][3], const T Dv[3][3], T ht[6]) const {
    if (medium_type == CGFD_MEDIUM_ELASTIC_ISO) {
      T lam = med_c(1)[iptr], mu = med_c(2)[iptr];
      T lam2mu = (T)(lam + 2.0 * mu);
      hooke_iso_full(lam, mu, lam2mu, m, Dv, ht);
    } else {
      T C[6][6];
      cij(iptr, C);
      hooke_aniso_axes(C, m, Dv, 3, ht);
    }
  }

  void hooke_axis(size_t iptr, const T m[3], const T D[3], T ht[6], bool surf) const {
    if (medium_type == CGFD_MEDIUM_ELASTIC_ISO) {
      T lam = med_c(1)[iptr], mu = med_c(2)[iptr];
      T lam2mu = (T)(lam + 2.0 * mu);
      if (surf) hooke_iso_surf(lam, mu, lam2mu, m, D, ht);
      else hooke_iso_axis(lam, mu, lam2mu, m, D, ht);
    } else {
      T C[6][6];
      cij(iptr, C);
      T mm[1][3] = {{m[0], m[1], m[2]}};
      T DD[1][3] = {{D[0], D[1], D[2]}};
      hooke_aniso_axes(C, mm, DD, 1, ht);
    }
  }

  // traction image, sv_curv_col_el_gpu.cu:19-221
  void rhs_timg(const T *w, T *h, const Ops &o) {
    const Grid &G = g;
    const T *jac = metric_c(0);
    const T *Tm[6];
    for (int c = 0; c < 6; c++) Tm[c] = w + (3 + c) * G.siz_icmp;  // xx yy zz yz xz xy
    // traction components of row c of the stress tensor, in the reference order:
    // hVx: Txx,Txy,Txz ; hVy: Txy,Tyy,Tyz ; hVz: Txz,Tyz,Tzz
    const int tv[3][3] = {{0, 5, 4}, {5, 1, 3}, {4, 3, 2}};
    int k_min = G.nk2 - o.z.idx[o.z.len - 1];
    for (int k = k_min; k <= G.nk2; k++) {
      int n_free = G.nk2 - k - o.z.idx[0];
#pragma omp parallel for schedule(static)
      for (int j = G.nj1; j <= G.nj2; j++)
        for (int i = G.ni1; i <= G.ni2; i++) {
          size_t iptr = i + j * G.siz_iy + k * G.siz_iz;
          T slwjac = med_c(0)[iptr] / jac[iptr];
          for (int c = 0; c < 3; c++) {
            const T *T1 = Tm[tv[c][0]], *T2 = Tm[tv[c][1]], *T3 = Tm[tv[c][2]];
            T vecxi[5] = {0}, vecet[5] = {0}, veczt[5] = {0};
            auto flux = [&](int axis, size_t p) {
              return jac[p] * (metric_c(1 + 3 * axis)[p] * T1[p] + metric_c(2 + 3 * axis)[p] * T2[p] +
                               metric_c(3 + 3 * axis)[p] * T3[p]);
            };
            for (int n = 0; n < o.x.len; n++) vecxi[n] = flux(0, iptr + o.x.idx[n]);
            for (int n = 0; n < o.y.len; n++) vecet[n] = flux(1, iptr + o.y.idx[n] * (long)G.siz_iy);
            for (int n = 0; n < n_free; n++) veczt[n] = flux(2, iptr + o.z.idx[n] * (long)G.siz_iz);
            veczt[n_free] = 0;
            for (int n = n_free + 1; n < o.z.len; n++) {
              int n_img = o.z.idx[n] - 2 * (n - n_free);
              veczt[n] = -flux(2, iptr + n_img * (long)G.siz_iz);
            }
            auto noindx = [](const Op &op, const T *v) {
              T r = (T)(float)op.coef[0] * v[0];
              for (int n = 1; n < op.len; n++) r += (T)(float)op.coef[n] * v[n];
              return r;
            };
            T DxTx = noindx(o.x, vecxi), DyTy = noindx(o.y, vecet), DzTz = noindx(o.z, veczt);
            h[c * G.siz_icmp + iptr] = (DxTx + DyTy + DzTz) * slwjac;
          }
        }
    }
  }

  // vlow, sv_curv_col_el_iso_gpu.cu:462-603
  void rhs_vlow(const T *w, T *h, const Ops &o) {
    const Grid &G = g;
    for (int n = 0; n < 3; n++) {
      int k = G.nk2 - n;
      const Op &oz = o.zlay[n];
#pragma omp parallel for schedule(static)
      for (int j = G.nj1; j <= G.nj2; j++)
        for (int i = G.ni1; i <= G.ni2; i++) {
          size_t iptr = i + j * G.siz_iy + k * G.siz_iz;
          T m[3][3];
          for (int a = 0; a < 3; a++)
            for (int b = 0; b < 3; b++) m[a][b] = metric_c(1 + 3 * a + b)[iptr];
          T Dv[3][3];
          for (int c = 0; c < 3; c++) {
            Dv[0][c] = fd_apply(o.x, w + c * G.siz_icmp, iptr, 1);
            Dv[1][c] = fd_apply(o.y, w + c * G.siz_icmp, iptr, (long)G.siz_iy);
          }
          if (k == G.nk2) {
            size_t ij = (i + j * G.siz_iy) * 9;
            for (int r = 0; r < 3; r++)
              Dv[2][r] = matVx2Vz[ij + 3 * r + 0] * Dv[0][0] + matVx2Vz[ij + 3 * r + 1] * Dv[0][1] +
                         matVx2Vz[ij + 3 * r + 2] * Dv[0][2] + matVy2Vz[ij + 3 * r + 0] * Dv[1][0] +
                         matVy2Vz[ij + 3 * r + 1] * Dv[1][1] + matVy2Vz[ij + 3 * r + 2] * Dv[1][2];
          } else {
            for (int c = 0; c < 3; c++) Dv[2][c] = fd_apply(oz, w + c * G.siz_icmp, iptr, (long)G.siz_iz);
          }
          T ht[6];
          hooke_full(iptr, m, Dv, ht);
          for (int c = 0; c < 6; c++) h[(3 + c) * G.siz_icmp + iptr] = ht[c];
        }
    }
  }

  // CFS-PML, sv_curv_col_el_iso_gpu.cu:613-1147
  void rhs_cfspml(const T *w, T *h, const Ops &o, int cur_lvl_aux_is_pre) {
    const Grid &G = g;
    const Op *opa[3] = {&o.x, &o.y, &o.z};
    const long sh[3] = {1, (long)G.siz_iy, (long)G.siz_iz};
    const int tv[3][3] = {{0, 5, 4}, {5, 1, 3}, {4, 3, 2}};
    // wave cmp index of Voigt stress c: 3+c ; hT Voigt c -> cmp 3+c
    for (int idim = 0; idim < 3; idim++)
      for (int iside = 0; iside < 2; iside++) {
        Face &f = face[idim][iside];
        if (!f.enable) continue;
        T *aux_cur = f.aux.data() + (size_t)(cur_lvl_aux_is_pre ? f.lvl_pre : 1) * 9 * f.siz_icmp;
        T *aux_rhs = f.aux.data() + (size_t)2 * 9 * f.siz_icmp;
#pragma omp parallel for schedule(static)
        for (int iz = 0; iz < f.nz; iz++)
          for (int iy = 0; iy < f.ny; iy++)
            for (int ix = 0; ix < f.nx; ix++) {
              size_t ia = (size_t)iz * f.ny * f.nx + (size_t)iy * f.nx + ix;
              size_t iptr = (ix + f.ni1) + (iy + f.nj1) * G.siz_iy + (iz + f.nk1) * G.siz_iz;
              int ab = idim == 0 ? ix : (idim == 1 ? iy : iz);
              T cD = f.D[ab], cA = f.A[ab], cB = f.B[ab];
              T cB1 = (T)(cB - 1.0);
              T m[3] = {metric_c(1 + 3 * idim)[iptr], metric_c(2 + 3 * idim)[iptr], metric_c(3 + 3 * idim)[iptr]};
              T slw = med_c(0)[iptr];
              T Dv[3], Dt[6];
              for (int c = 0; c < 3; c++) Dv[c] = fd_apply(*opa[idim], w + c * G.siz_icmp, iptr, sh[idim]);
              for (int c = 0; c < 6; c++) Dt[c] = fd_apply(*opa[idim], w + (3 + c) * G.siz_icmp, iptr, sh[idim]);
              T rhs[9];
              for (int c = 0; c < 3; c++)
                rhs[c] = slw * (m[0] * Dt[tv[c][0]] + m[1] * Dt[tv[c][1]] + m[2] * Dt[tv[c][2]]);
              T ht[6];
              hooke_axis(iptr, m, Dv, ht, false);
              for (int c = 0; c < 6; c++) rhs[3 + c] = ht[c];
              for (int c = 0; c < 9; c++) {
                T a = aux_cur[c * f.siz_icmp + ia];
                h[c * G.siz_icmp + iptr] += cB1 * rhs[c] - cB * a;
                aux_rhs[c * f.siz_icmp + ia] = cD * rhs[c] - cA * a;
              }
              if (free_top && idim < 2 && (iz + f.nk1) == G.nk2) {
                size_t ij = ((ix + f.ni1) + (iy + f.nj1) * G.siz_iy) * 9;
                const T *mat = idim == 0 ? matVx2Vz.data() : matVy2Vz.data();
                T Dz[3];
                for (int r = 0; r < 3; r++)
                  Dz[r] = mat[ij + 3 * r + 0] * Dv[0] + mat[ij + 3 * r + 1] * Dv[1] + mat[ij + 3 * r + 2] * Dv[2];
                T z[3] = {metric_c(7)[iptr], metric_c(8)[iptr], metric_c(9)[iptr]};
                hooke_axis(iptr, z, Dz, ht, true);
                for (int c = 0; c < 6; c++) {
                  h[(3 + c) * G.siz_icmp + iptr] += (T)(cB - 1.0) * ht[c];
                  aux_rhs[(3 + c) * f.siz_icmp + ia] += cD * ht[c];
                }
              }
            }
      }
  }

  // sv_curv_col_el_iso_rhs_src_gpu, sv_curv_col_el_gpu.cu:227-301
  void rhs_src(T *h, int it, int istage) {
    const T *jac = metric_c(0), *slw = med_c(0);
    for (int is = 0; is < nsrc; is++) {
      if (!(it >= it_begin[is] && it <= it_end[is])) continue;
      size_t ip = (size_t)is * max_nt * 4 + (size_t)(it - it_begin[is]) * 4 + istage;
      for (int e = 0; e < ext_num[is]; e++) {
        size_t iptr = ext_indx[(size_t)is * max_ext + e];
        T coef = ext_coef[(size_t)is * max_ext + e];
        if (force_actived) {
          T V = coef * slw[iptr] / jac[iptr];
          for (int c = 0; c < 3; c++) h[c * g.siz_icmp + iptr] += F[c][ip] * V;
        }
        if (moment_actived) {
          T rjac = coef / jac[iptr];
          // M order xx,yy,zz,yz,xz,xy == cmp 3..8
          for (int c = 0; c < 6; c++) h[(3 + c) * g.siz_icmp + iptr] += -M[c][ip] * rjac;
        }
      }
    }
  }

  // ---------------------------------------------------------------------------------------
  // acoustic media, sv_curv_col_ac_iso_gpu.cu: fields Vx Vy Vz P with P in the Txx slot
  // (wav_ac_init, wav_t.cu:190-250), medium slowness and kappa
  // ---------------------------------------------------------------------------------------
  // pressure image of the free surface, in place on the stage input (:376-410)
  void ac_timg(T *w) {
    T *P = w + TXX * g.siz_icmp;
    for (int j = g.nj1; j <= g.nj2; j++)
      for (int i = g.ni1; i <= g.ni2; i++) {
        size_t top = i + j * g.siz_iy + (size_t)g.nk2 * g.siz_iz;
        P[top] = 0;
        for (int k = g.nk2 + 1; k < g.nz; k++)
          P[i + j * g.siz_iy + (size_t)k * g.siz_iz] = -P[i + j * g.siz_iy + (size_t)(2 * g.nk2 - k) * g.siz_iz];
      }
  }

  // inner points (:277-366)
  void ac_inner(const T *w, T *h, const Ops &o) {
    const Grid &G = g;
    const long sy = (long)G.siz_iy, sz = (long)G.siz_iz;
#pragma omp parallel for schedule(static)
    for (int k = G.nk1; k <= G.nk2; k++)
      for (int j = G.nj1; j <= G.nj2; j++)
        for (int i = G.ni1; i <= G.ni2; i++) {
          size_t iptr = i + j * G.siz_iy + k * G.siz_iz;
          const T *Vx = w + VX * G.siz_icmp, *Vy = w + VY * G.siz_icmp, *Vz = w + VZ * G.siz_icmp,
                  *P = w + TXX * G.siz_icmp;
          T DxVx = fd_apply(o.x, Vx, iptr, 1), DyVx = fd_apply(o.y, Vx, iptr, sy), DzVx = fd_apply(o.z, Vx, iptr, sz);
          T DxVy = fd_apply(o.x, Vy, iptr, 1), DyVy = fd_apply(o.y, Vy, iptr, sy), DzVy = fd_apply(o.z, Vy, iptr, sz);
          T DxVz = fd_apply(o.x, Vz, iptr, 1), DyVz = fd_apply(o.y, Vz, iptr, sy), DzVz = fd_apply(o.z, Vz, iptr, sz);
          T DxP = fd_apply(o.x, P, iptr, 1), DyP = fd_apply(o.y, P, iptr, sy), DzP = fd_apply(o.z, P, iptr, sz);
          T xix = metric_c(1)[iptr], xiy = metric_c(2)[iptr], xiz = metric_c(3)[iptr];
          T etx = metric_c(4)[iptr], ety = metric_c(5)[iptr], etz = metric_c(6)[iptr];
          T ztx = metric_c(7)[iptr], zty = metric_c(8)[iptr], ztz = metric_c(9)[iptr];
          T kappa = med_c(1)[iptr], slw = med_c(0)[iptr];
          h[VX * G.siz_icmp + iptr] = -slw * (xix * DxP + etx * DyP + ztx * DzP);
          h[VY * G.siz_icmp + iptr] = -slw * (xiy * DxP + ety * DyP + zty * DzP);
          h[VZ * G.siz_icmp + iptr] = -slw * (xiz * DxP + etz * DyP + ztz * DzP);
          h[TXX * G.siz_icmp + iptr] = -kappa * (xix * DxVx + etx * DyVx + ztx * DzVx + xiy * DxVy + ety * DyVy +
                                                 zty * DzVy + xiz * DxVz + etz * DyVz + ztz * DzVz);
        }
  }

  // low-order pressure rows of the top 3 planes (:413-521): 0 on the surface, 2nd / 4th-order
  // velocity z-derivatives below it
  void ac_vlow(const T *w, T *h, const Ops &o) {
    const Grid &G = g;
    for (int n = 0; n < 3; n++) {
      const int k = G.nk2 - n;
      const Op &oz = o.zlay[n];
#pragma omp parallel for schedule(static)
      for (int j = G.nj1; j <= G.nj2; j++)
        for (int i = G.ni1; i <= G.ni2; i++) {
          size_t iptr = i + j * G.siz_iy + k * G.siz_iz;
          if (k == G.nk2) {
            h[TXX * G.siz_icmp + iptr] = 0;
            continue;
          }
          const T *V[3] = {w + VX * G.siz_icmp, w + VY * G.siz_icmp, w + VZ * G.siz_icmp};
          T Dx[3], Dy[3], Dz[3];
          for (int c = 0; c < 3; c++) {
            Dx[c] = fd_apply(o.x, V[c], iptr, 1);
            Dy[c] = fd_apply(o.y, V[c], iptr, (long)G.siz_iy);
            Dz[c] = fd_apply(oz, V[c], iptr, (long)G.siz_iz);
          }
          T xix = metric_c(1)[iptr], xiy = metric_c(2)[iptr], xiz = metric_c(3)[iptr];
          T etx = metric_c(4)[iptr], ety = metric_c(5)[iptr], etz = metric_c(6)[iptr];
          T ztx = metric_c(7)[iptr], zty = metric_c(8)[iptr], ztz = metric_c(9)[iptr];
          T kappa = med_c(1)[iptr];
          h[TXX * G.siz_icmp + iptr] = -kappa * (xix * Dx[0] + etx * Dy[0] + ztx * Dz[0] + xiy * Dx[1] + ety * Dy[1] +
                                                 zty * Dz[1] + xiz * Dx[2] + etz * Dy[2] + ztz * Dz[2]);
        }
    }
  }

  // CFS-PML (:579-802): per face, the 1-D terms of its axis correct the RHS and drive the 4
  // auxiliary variables
  void ac_cfspml(const T *w, T *h, const Ops &o, int cur_lvl_aux_is_pre) {
    const Grid &G = g;
    const Op *opa[3] = {&o.x, &o.y, &o.z};
    const long sh[3] = {1, (long)G.siz_iy, (long)G.siz_iz};
    const int fld[4] = {VX, VY, VZ, TXX};
    for (int idim = 0; idim < 3; idim++)
      for (int iside = 0; iside < 2; iside++) {
        Face &f = face[idim][iside];
        if (!f.enable) continue;
        T *aux_cur = f.aux.data() + (size_t)(cur_lvl_aux_is_pre ? f.lvl_pre : 1) * 9 * f.siz_icmp;
        T *aux_rhs = f.aux.data() + (size_t)2 * 9 * f.siz_icmp;
#pragma omp parallel for schedule(static)
        for (int iz = 0; iz < f.nz; iz++)
          for (int iy = 0; iy < f.ny; iy++)
            for (int ix = 0; ix < f.nx; ix++) {
              size_t ia = (size_t)iz * f.ny * f.nx + (size_t)iy * f.nx + ix;
              size_t iptr = (ix + f.ni1) + (iy + f.nj1) * G.siz_iy + (iz + f.nk1) * G.siz_iz;
              int ab = idim == 0 ? ix : (idim == 1 ? iy : iz);
              T cD = f.D[ab], cA = f.A[ab], cB = f.B[ab];
              T cB1 = (T)(cB - 1.0);
              T m0 = metric_c(1 + 3 * idim)[iptr], m1 = metric_c(2 + 3 * idim)[iptr], m2 = metric_c(3 + 3 * idim)[iptr];
              T kappa = med_c(1)[iptr], slw = med_c(0)[iptr];
              T D[4];
              for (int c = 0; c < 4; c++) D[c] = fd_apply(*opa[idim], w + fld[c] * G.siz_icmp, iptr, sh[idim]);
              T rhs[4];
              rhs[0] = -slw * (m0 * D[3]);
              rhs[1] = -slw * (m1 * D[3]);
              rhs[2] = -slw * (m2 * D[3]);
              rhs[3] = -kappa * (m0 * D[0] + m1 * D[1] + m2 * D[2]);
              for (int c = 0; c < 4; c++) {
                T a = aux_cur[fld[c] * f.siz_icmp + ia];
                h[fld[c] * G.siz_icmp + iptr] += cB1 * rhs[c] - cB * a;
                aux_rhs[fld[c] * f.siz_icmp + ia] = cD * rhs[c] - cA * a;
              }
            }
      }
  }

  // sources (:823-887): forces on the velocities, Mxx on the pressure
  void ac_src(T *h, int it, int istage) {
    const T *jac = metric_c(0), *slw = med_c(0);
    for (int is = 0; is < nsrc; is++) {
      if (!(it >= it_begin[is] && it <= it_end[is])) continue;
      size_t ip = (size_t)is * max_nt * 4 + (size_t)(it - it_begin[is]) * 4 + istage;
      for (int e = 0; e < ext_num[is]; e++) {
        size_t iptr = ext_indx[(size_t)is * max_ext + e];
        T coef = ext_coef[(size_t)is * max_ext + e];
        if (force_actived) {
          T V = coef * slw[iptr] / jac[iptr];
          for (int c = 0; c < 3; c++) h[c * g.siz_icmp + iptr] += F[c][ip] * V;
        }
        if (moment_actived) {
          T rjac = coef / jac[iptr];
          h[TXX * g.siz_icmp + iptr] += -M[0][ip] * rjac;
        }
      }
    }
  }

  // io_recv_keep, io_funcs.cu:1624-1666 (corner 5 used twice, corner 4 never)
  void recv_keep(const T *w, int it) {
    for (size_t n = 0; n < recv.size(); n++) {
      const Recv &r = recv[n];
      T Lx2 = r.di, Lx1 = (T)(1.0 - Lx2), Ly2 = r.dj, Ly1 = (T)(1.0 - Ly2), Lz2 = r.dk, Lz1 = (T)(1.0 - Lz2);
      for (int c = 0; c < 9; c++) {
        const T *v = w + c * g.siz_icmp;
        T b[8];
        for (int q = 0; q < 8; q++) b[q] = v[r.indx1d[q]];
        T val = b[0] * Lx1 * Ly1 * Lz1 + b[1] * Lx2 * Ly1 * Lz1 + b[2] * Lx1 * Ly2 * Lz1 + b[3] * Lx2 * Ly2 * Lz1 +
                b[5] * Lx1 * Ly1 * Lz2 + b[5] * Lx2 * Ly1 * Lz2 + b[6] * Lx1 * Ly2 * Lz2 + b[7] * Lx2 * Ly2 * Lz2;
        seismo[(n * 9 + c) * (size_t)nt_total + it] = (float)val;
      }
    }
  }

  // PG_calcu_gpu, wav_t.cu:281-360: at the top physical plane, acceleration by the step
  // difference of V, displacement by trapezoidal accumulation (double arithmetic from the
  // 0.5 literal), and running maxima of components and magnitudes.
  void pg_calcu(const T *w_end, const T *w_pre) {
    if (pg.empty()) {
      pg.assign((size_t)15 * g.siz_iz, (T)0);
      dis.assign((size_t)3 * g.siz_iz, (T)0);
    }
    const T dtt = dt;
    for (int iy = 0; iy < g.nj; iy++)
      for (int ix = 0; ix < g.ni; ix++) {
        const size_t iptr1 = (size_t)(ix + 3) + (size_t)(iy + 3) * g.siz_iy;
        const size_t iptr = iptr1 + (size_t)g.nk2 * g.siz_iz;
        T v1[3], v0[3], a[3];
        for (int c = 0; c < 3; c++) {
          v1[c] = w_end[c * g.siz_icmp + iptr];
          v0[c] = w_pre[c * g.siz_icmp + iptr];
          a[c] = std::fabs((v1[c] - v0[c]) / dtt);
          T &d = dis[c * g.siz_iz + iptr1];
          d = (T)((double)d + 0.5 * (double)(T)(v1[c] + v0[c]) * (double)dtt);
        }
        const T *D = &dis[0];
        const T dx = D[iptr1], dy = D[g.siz_iz + iptr1], dz = D[2 * g.siz_iz + iptr1];
        const T V = std::sqrt(v1[0] * v1[0] + v1[1] * v1[1] + v1[2] * v1[2]);
        const T Vh = std::sqrt(v1[0] * v1[0] + v1[1] * v1[1]);
        const T A = std::sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
        const T Ah = std::sqrt(a[0] * a[0] + a[1] * a[1]);
        const T Dm = std::sqrt(dx * dx + dy * dy + dz * dz);
        const T Dh = std::sqrt(dx * dx + dy * dy);
        const T val[15] = {V, Vh, std::fabs(v1[0]), std::fabs(v1[1]), std::fabs(v1[2]),
                           A, Ah, a[0], a[1], a[2],
                           Dm, Dh, std::fabs(dx), std::fabs(dy), std::fabs(dz)};
        for (int q = 0; q < 15; q++) {
          T &m = pg[q * g.siz_iz + iptr1];
          if (m < val[q]) m = val[q];
        }
      }
  }

  // wav_update / wav_update_end, wav_t.cu:362-378
  static void update(size_t n, T coef, T *out, const T *in1, const T *in2) {
#pragma omp parallel for schedule(static)
    for (long i = 0; i < (long)n; i++) out[i] = in1[i] + coef * in2[i];
  }
  static void update_end(size_t n, T coef, T *out, const T *in2) {
#pragma omp parallel for schedule(static)
    for (long i = 0; i < (long)n; i++) out[i] = out[i] + coef * in2[i];
  }

  // drv_rk_curv_col.cu:193-541 (one rank, no halo exchange, no ablexp)
  void run(int nsteps) {
    const float rk_a[3] = {0.5f, 0.5f, 1.0f};
    const float rk_b[4] = {(float)(1.0 / 6.0), (float)(1.0 / 3.0), (float)(1.0 / 3.0), (float)(1.0 / 6.0)};
    size_t lev_n = 9 * g.siz_icmp;
    for (int s = 0; s < nsteps; s++) {
      int it = it_cur;
      T *w_pre = lev(lvl_pre), *w_tmp = lev(1), *w_rhs = lev(2), *w_end = lev(lvl_end);
      if (it < nt_total) recv_keep(w_pre, it);
      int ipair = it % 8;
      for (int istage = 0; istage < 4; istage++) {
        T *w_cur = istage == 0 ? w_pre : w_tmp;
        Ops o = make_ops(ipair, istage);
        if (medium_type == CGFD_MEDIUM_ACOUSTIC_ISO) {  // sv_curv_col_ac_iso_onestage, :21-270
          if (free_top) ac_timg(w_cur);
          ac_inner(w_cur, w_rhs, o);
          if (free_top) ac_vlow(w_cur, w_rhs, o);
          ac_cfspml(w_cur, w_rhs, o, istage == 0);
          ac_src(w_rhs, it, istage);
        } else {
          rhs_inner(w_cur, w_rhs, o);
          if (free_top) {
            rhs_timg(w_cur, w_rhs, o);
            rhs_vlow(w_cur, w_rhs, o);
          }
          rhs_cfspml(w_cur, w_rhs, o, istage == 0);
          rhs_src(w_rhs, it, istage);
        }
        // RK combine (float coefficients as in the reference)
        if (istage == 0) {
          T ca = (T)(rk_a[istage] * (float)dt), cb = (T)(rk_b[istage] * (float)dt);
          if (sizeof(T) == 8) { ca = (T)rk_a[istage] * dt; cb = (T)rk_b[istage] * dt; }
          update(lev_n, ca, w_tmp, w_pre, w_rhs);
          for_faces([&](Face &f) {
            size_t n = 9 * f.siz_icmp;
            T *a = f.aux.data();
            update(n, ca, a + 1 * n, a + f.lvl_pre * n, a + 2 * n);
          });
          update(lev_n, cb, w_end, w_pre, w_rhs);
          for_faces([&](Face &f) {
            size_t n = 9 * f.siz_icmp;
            T *a = f.aux.data();
            update(n, cb, a + f.lvl_end * n, a + f.lvl_pre * n, a + 2 * n);
          });
        } else if (istage < 3) {
          T ca = (T)(rk_a[istage] * (float)dt), cb = (T)(rk_b[istage] * (float)dt);
          if (sizeof(T) == 8) { ca = (T)rk_a[istage] * dt; cb = (T)rk_b[istage] * dt; }
          update(lev_n, ca, w_tmp, w_pre, w_rhs);
          for_faces([&](Face &f) {
            size_t n = 9 * f.siz_icmp;
            T *a = f.aux.data();
            update(n, ca, a + 1 * n, a + f.lvl_pre * n, a + 2 * n);
          });
          update_end(lev_n, cb, w_end, w_rhs);
          for_faces([&](Face &f) {
            size_t n = 9 * f.siz_icmp;
            T *a = f.aux.data();
            update_end(n, cb, a + f.lvl_end * n, a + 2 * n);
          });
        } else {
          T cb = (T)(rk_b[istage] * (float)dt);
          if (sizeof(T) == 8) cb = (T)rk_b[istage] * dt;
          update_end(lev_n, cb, w_end, w_rhs);
          for_faces([&](Face &f) {
            size_t n = 9 * f.siz_icmp;
            T *a = f.aux.data();
            update_end(n, cb, a + f.lvl_end * n, a + 2 * n);
          });
        }
      }
      if (free_top) pg_calcu(w_end, w_pre);  // drv_rk_curv_col.cu:519-527, before the level swap
      std::swap(lvl_pre, lvl_end);
      for_faces([&](Face &f) { std::swap(f.lvl_pre, f.lvl_end); });
      it_cur++;
    }
  }

  template <typename Fn>
  void for_faces(Fn fn) {
    for (int a = 0; a < 3; a++)
      for (int b = 0; b < 2; b++)
        if (face[a][b].enable) fn(face[a][b]);
  }
};

struct Handle {
  int use_double;
  Oracle<float> *f = nullptr;
  Oracle<double> *d = nullptr;
};

template <typename Fn>
int guarded(Fn fn) {
  try {
    fn();
    return 0;
  } catch (std::exception &e) {
    g_err = e.what();
    return -1;
  }
}

template <typename T>
void get_w(Oracle<T> *o, float *out) {
  T *w = o->lev(o->lvl_pre);
  for (size_t n = 0; n < 9 * o->g.siz_icmp; n++) out[n] = (float)w[n];
}
template <typename T>
void set_w(Oracle<T> *o, const float *in) {
  T *w = o->lev(o->lvl_pre);
  const Grid &g = o->g;
  for (int c = 0; c < 9; c++)
    for (int k = 0; k < g.nz; k++)
      for (int j = 0; j < g.ny; j++)
        for (int i = 0; i < g.nx; i++) {
          size_t iptr = c * g.siz_icmp + i + j * g.siz_iy + k * g.siz_iz;
          w[iptr] = g.lindx_is_inner(i, j, k) ? (T)in[iptr] : (T)0;
        }
}

}  // namespace

extern "C" {

const char *orc_error(void) { return g_err.c_str(); }

void *orc_create(const cgfd_problem_desc *d, int use_double) {
  Handle *h = new Handle;
  h->use_double = use_double;
  int rc = guarded([&] {
    if (use_double) { h->d = new Oracle<double>; h->d->setup(d); }
    else { h->f = new Oracle<float>; h->f->setup(d); }
  });
  if (rc) {
    delete h->f; delete h->d; delete h;
    return nullptr;
  }
  return h;
}

void orc_destroy(void *p) {
  Handle *h = (Handle *)p;
  if (!h) return;
  delete h->f;
  delete h->d;
  delete h;
}

int orc_run(void *p, int nsteps) {
  Handle *h = (Handle *)p;
  return guarded([&] {
    if (h->d) { if (nsteps < 0) nsteps = h->d->nt_total - h->d->it_cur; h->d->run(nsteps); }
    else { if (nsteps < 0) nsteps = h->f->nt_total - h->f->it_cur; h->f->run(nsteps); }
  });
}

int orc_set_step(void *p, int it) {
  Handle *h = (Handle *)p;
  if (h->d) h->d->it_cur = it; else h->f->it_cur = it;
  return 0;
}

int orc_num_stations(void *p) {
  Handle *h = (Handle *)p;
  return h->d ? (int)h->d->recv.size() : (int)h->f->recv.size();
}

int orc_get_seismograms(void *p, float *out) {
  Handle *h = (Handle *)p;
  const std::vector<float> &s = h->d ? h->d->seismo : h->f->seismo;
  memcpy(out, s.data(), s.size() * sizeof(float));
  return 0;
}

// Location of n points by physical coordinates (depth_flag: z is a depth below the surface):
// global physical index (-1000 outside) and shift, as src_t.cu:341-398 uses them.
int orc_locate_points(int ni, int nj, int nk, const float *coord, int n, const float *xyz, const int *depth_flag,
                      int *idx, float *inc) {
  return guarded([&] {
    Grid g;
    g.set(ni, nj, nk);
    Locator lc(g, coord);
    for (int q = 0; q < n; q++) {
      float c[3] = {xyz[3 * q], xyz[3 * q + 1], xyz[3 * q + 2]};
      if (depth_flag && depth_flag[q]) lc.depth_to_axis(c[0], c[1], &c[2]);
      lc.locate(c[0], c[1], c[2], idx + 3 * q, inc + 3 * q);
    }
  });
}

// [15][ny][nx] peak ground motion (zeros before the first step or without a free surface)
int orc_get_peak_motion(void *p, float *out) {
  Handle *h = (Handle *)p;
  auto copy = [&](auto *o) {
    const size_t n = (size_t)15 * o->g.siz_iz;
    for (size_t q = 0; q < n; q++) out[q] = o->pg.empty() ? 0.f : (float)o->pg[q];
  };
  if (h->d) copy(h->d); else copy(h->f);
  return 0;
}

int orc_get_wavefield(void *p, float *out) {
  Handle *h = (Handle *)p;
  if (h->d) get_w(h->d, out); else get_w(h->f, out);
  return 0;
}

int orc_set_wavefield(void *p, const float *in) {
  Handle *h = (Handle *)p;
  if (h->d) set_w(h->d, in); else set_w(h->f, in);
  return 0;
}

/* PML coefficients of one face (N+1 values each), for unit checks. */
int orc_pml_coefs(void *p, int idim, int iside, float *A, float *B, float *D) {
  Handle *h = (Handle *)p;
  if (!h->f) return -1;
  auto &f = h->f->face[idim][iside];
  if (!f.enable) return -1;
  for (size_t n = 0; n < f.A.size(); n++) { A[n] = f.A[n]; B[n] = f.B[n]; D[n] = f.D[n]; }
  return (int)f.A.size();
}

/* Free-surface conversion matrices [ny][nx][9] x2, for unit checks. */
int orc_free_mats(void *p, float *mx, float *my) {
  Handle *h = (Handle *)p;
  if (!h->f || !h->f->free_top) return -1;
  for (size_t n = 0; n < h->f->matVx2Vz.size(); n++) { mx[n] = h->f->matVx2Vz[n]; my[n] = h->f->matVy2Vz[n]; }
  return 0;
}

/* Source tables for unit checks: ext_num[nsrc], ext_indx/ext_coef[nsrc][343], it_begin. */
int orc_src_info(void *p, int *nsrc, int *max_nt, int *it_begin, int *ext_num, int *ext_indx, float *ext_coef,
                 float *mxx_stage0) {
  Handle *h = (Handle *)p;
  if (!h->f) return -1;
  auto *o = h->f;
  *nsrc = o->nsrc;
  *max_nt = o->max_nt;
  for (int s = 0; s < o->nsrc; s++) {
    if (it_begin) it_begin[s] = o->it_begin[s];
    if (ext_num) ext_num[s] = o->ext_num[s];
  }
  if (ext_indx) for (size_t n = 0; n < o->ext_indx.size(); n++) ext_indx[n] = o->ext_indx[n];
  if (ext_coef) for (size_t n = 0; n < o->ext_coef.size(); n++) ext_coef[n] = o->ext_coef[n];
  if (mxx_stage0 && o->moment_actived)
    for (int s = 0; s < o->nsrc; s++)
      for (int t = 0; t < o->max_nt; t++) mxx_stage0[(size_t)s * o->max_nt + t] = o->M[0][((size_t)s * o->max_nt + t) * 4];
  return 0;
}

/*
 * Grid helpers used to build test inputs: fill ghost points by linear extrapolation
 * (geometric_symmetry) and compute metrics in FP32 (gd_curv_metric_cal).
 * coord: [3][nz][ny][nx], physical points given; ghosts are overwritten.
 */
int orc_coord_ghosts(int ni, int nj, int nk, float *coord) {
  Grid g;
  g.set(ni, nj, nk);
  geometric_symmetry(g, coord, 3);
  return 0;
}

int orc_metric_calc(int ni, int nj, int nk, const float *coord, float *metric) {
  Grid g;
  g.set(ni, nj, nk);
  metric_cal(g, coord, coord + g.siz_icmp, coord + 2 * g.siz_icmp, metric);
  return 0;
}

int orc_metric_calc_f64(int ni, int nj, int nk, const double *coord, double *metric) {
  Grid g;
  g.set(ni, nj, nk);
  metric_cal(g, coord, coord + g.siz_icmp, coord + 2 * g.siz_icmp, metric);
  return 0;
}

}  // extern "C"

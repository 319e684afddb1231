// cgfd_media.cu -- media discretisation on the GPU: a layered elastic-isotropic model (the
// reference's "elastic_isotropic" interface file) sampled onto the curvilinear grid, ghosts
// included, by the three methods of media_layer2model_el_iso (src/media/media_layer2model.cpp:
// 121-170, 1313-1355 "loc", the "har" and "ari" equivalent-medium averages):
//   loc: every grid point takes the layer below the interfaces above it: value + dz^pow * grad
//        (CalPointValue_layer, media_layer2model.cpp:452-520), averaged with the layer above
//        when the point lies on an interface;
//   har / ari: where the 8 half-grid points around a grid point fall in more than one layer
//        (MarkInterfaceNumber, NumOfValues), the half-grid cell is subdivided 8 x 8 x 8
//        (MeshSubdivide, 729 sample points) and rho is averaged arithmetically, kappa and mu
//        harmonically (har) or lambda and mu arithmetically (ari).
// One thread per grid point (loc, marking, averaging). The float and double steps follow the
// reference's expressions in order with explicit rounding (no fused multiply-add), so the
// result matches the reference's own host code. Kept alike on purpose: the reference's test
// for "on an interface" compares the truncated integer part of dz with 0 (|dz| < 1 in model
// units), because its isEqual() calls the integer abs().
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cuda_runtime.h>

#include <cstring>
#include <string>
#include <vector>

#include "cgfd_b200.h"
#include "cgfd_setup.h"

namespace cgfd {
namespace {

constexpr int kMaxInterfaces = 64;
constexpr int kSub = 8;  // NG, media_utility.hpp:8

struct LayerDev {
  int ni_, nx, ny;
  float x0, y0, dx, dy;
  const float *elev;                       // [NI][ny][nx]
  const float *p[9];                       // rho, rho_grad, rho_pow, vp, vp_grad, vp_pow, vs, vs_grad, vs_pow
  const float *par;                        // general files: [npar][value, grad, pow][NI][ny][nx]
};

struct P3 {
  float x, y, z;
};

// BilinearInterpolation (media_utility.cpp:325-360) on the uniform interface mesh; FLT_MAX
// left of / below the mesh
__device__ float bilinear(const LayerDev &m, const float *v, float xq, float yq) {
  const float x0 = m.x0, x1 = __fadd_rn(m.x0, m.dx);
  const float y0 = m.y0, y1 = __fadd_rn(m.y0, m.dy);
  const int ix = (int)__fdiv_rn(__fsub_rn(xq, x0), __fsub_rn(x1, x0));
  const int iy = (int)__fdiv_rn(__fsub_rn(yq, y0), __fsub_rn(y1, y0));
  // (the reference checks only the lower side here; its callers keep points inside the mesh,
  // and beyond the upper side there is nothing to read)
  if (ix < 0 || iy < 0 || ix > m.nx - 1 || iy > m.ny - 1) return FLT_MAX;
  const int indx = iy * m.nx + ix;
  if (ix == m.nx - 1 || iy == m.ny - 1) return v[indx];
  const float xa = __fadd_rn(m.x0, __fmul_rn(m.dx, (float)ix)), xb = __fadd_rn(m.x0, __fmul_rn(m.dx, (float)(ix + 1)));
  const float ya = __fadd_rn(m.y0, __fmul_rn(m.dy, (float)iy)), yb = __fadd_rn(m.y0, __fmul_rn(m.dy, (float)(iy + 1)));
  const float area = __fmul_rn(__fsub_rn(xb, xa), __fsub_rn(yb, ya));
  float vq = __fmul_rn(__fmul_rn(v[indx], __fsub_rn(xb, xq)), __fsub_rn(yb, yq));
  vq = __fadd_rn(vq, __fmul_rn(__fmul_rn(v[indx + 1], __fsub_rn(xq, xa)), __fsub_rn(yb, yq)));
  vq = __fadd_rn(vq, __fmul_rn(__fmul_rn(v[indx + m.nx], __fsub_rn(xb, xq)), __fsub_rn(yq, ya)));
  vq = __fadd_rn(vq, __fmul_rn(__fmul_rn(v[indx + 1 + m.nx], __fsub_rn(xq, xa)), __fsub_rn(yq, ya)));
  return __fdiv_rn(vq, area);
}

// findLastGreaterEqualIndex (media_utility.cpp:60-81): the last interface of the leading run at
// or above `value`; -1 above the first interface
__device__ int last_ge(float value, const float *e, int n) {
  if (value > e[0]) return -1;
  float dist = FLT_MAX;
  int indx = -1;
  for (int i = 0; i < n; i++) {
    if (e[i] == -FLT_MAX) continue;
    const float nd = __fsub_rn(e[i], value);
    if (nd < 0.f) break;
    if (nd <= dist) { dist = nd; indx = i; }
  }
  return indx;
}

// findFirstGreaterEqualIndex (media_utility.cpp:91-112)
__device__ int first_ge(float value, const float *e, int n) {
  float dist = FLT_MAX;
  int idx = -1;
  for (int i = 0; i < n; i++) {
    if (e[i] == -FLT_MAX) continue;
    const float nd = __fsub_rn(e[i], value);
    if (nd >= 0.f && nd <= dist) {
      if ((double)nd <= 1e-6) return i;
      dist = nd;
      idx = i;
    }
  }
  return idx;
}

// value + dz^pow * grad of layer mi at (x, y): the reference adds in double and stores float
__device__ float layer_val(const LayerDev &m, int q, int mi, float x, float y, float dz) {
  const size_t sl = (size_t)m.nx * m.ny;
  const float v = bilinear(m, m.p[3 * q] + mi * sl, x, y);
  const float g = bilinear(m, m.p[3 * q + 1] + mi * sl, x, y);
  const float pw = bilinear(m, m.p[3 * q + 2] + mi * sl, x, y);
  return (float)__dadd_rn((double)v, __dmul_rn(pow((double)dz, (double)pw), (double)g));
}

// AssignLayerMediaPara2Point + CalPointValue_layer for elastic_isotropic
// (media_layer2model.cpp:401-520): rho, vp, vs at point a. Returns 0, or the error the
// reference exits on: 1 the point is outside the interface mesh (PrintIsPointOutOfInterfaceRange,
// media_utility.cpp:40-51), 2 vp <= sqrt(2) vs.
__device__ int point_value(const LayerDev &m, P3 a, float var[3]) {
  const float maxx = __fadd_rn(m.x0, __fmul_rn(m.dx, (float)(m.nx - 1)));
  const float maxy = __fadd_rn(m.y0, __fmul_rn(m.dy, (float)(m.ny - 1)));
  if (a.x < m.x0 || a.x > maxx || a.y < m.y0 || a.y > maxy) return 1;
  float e[kMaxInterfaces];
  const size_t sl = (size_t)m.nx * m.ny;
  for (int n = 0; n < m.ni_; n++) e[n] = bilinear(m, m.elev + n * sl, a.x, a.y);
  int mi = last_ge(a.z, e, m.ni_);
  if (mi == -1) {  // above the top interface: the top layer's values
    mi = last_ge(e[0], e, m.ni_);
    for (int q = 0; q < 3; q++) var[q] = bilinear(m, m.p[3 * q] + mi * sl, a.x, a.y);
    return 0;
  }
  float dz = __fsub_rn(e[mi], a.z);
  // var[0] rho, var[1] vp, var[2] vs; the reference evaluates vp, vs, then rho
  var[1] = layer_val(m, 1, mi, a.x, a.y, dz);
  var[2] = layer_val(m, 2, mi, a.x, a.y, dz);
  var[0] = layer_val(m, 0, mi, a.x, a.y, dz);
  if ((double)var[1] <= __dmul_rn((double)var[2], 1.4142135623730951)) return 2;
  if ((int)dz == 0) {  // on an interface (the reference's integer-abs test)
    const int mt = first_ge(a.z, e, m.ni_) - 1;
    if (mt >= 0) {
      dz = __fsub_rn(e[mt], a.z);
      const float vpt = layer_val(m, 1, mt, a.x, a.y, dz);
      const float vst = layer_val(m, 2, mt, a.x, a.y, dz);
      const float rhot = layer_val(m, 0, mt, a.x, a.y, dz);
      // (a + b) / 2.0: a float sum, halved in double
      var[0] = (float)__ddiv_rn((double)__fadd_rn(var[0], rhot), 2.0);
      var[1] = (float)__ddiv_rn((double)__fadd_rn(var[1], vpt), 2.0);
      var[2] = (float)__ddiv_rn((double)__fadd_rn(var[2], vst), 2.0);
    }
  }
  return 0;
}

// mu = vs vs rho (float); lambda = vp vp rho - 2.0 mu (double, stored float)
__device__ void lame(const float var[3], float &lam, float &mu) {
  mu = __fmul_rn(__fmul_rn(var[2], var[2]), var[0]);
  lam = (float)__dsub_rn((double)__fmul_rn(__fmul_rn(var[1], var[1]), var[0]), __dmul_rn(2.0, (double)mu));
}

// AssignLayerMediaPara2Point + CalPointValue_layer for acoustic_isotropic
// (media_layer2model.cpp:1177-1207): rho, vp at point a (var[0], var[1]). On an interface the
// layer above is evaluated at the same dz (the branch does not recompute it). Returns 0, or 1
// when the point is outside the interface mesh.
__device__ int point_value_ac(const LayerDev &m, P3 a, float var[2]) {
  const float maxx = __fadd_rn(m.x0, __fmul_rn(m.dx, (float)(m.nx - 1)));
  const float maxy = __fadd_rn(m.y0, __fmul_rn(m.dy, (float)(m.ny - 1)));
  if (a.x < m.x0 || a.x > maxx || a.y < m.y0 || a.y > maxy) return 1;
  float e[kMaxInterfaces];
  const size_t sl = (size_t)m.nx * m.ny;
  for (int n = 0; n < m.ni_; n++) e[n] = bilinear(m, m.elev + n * sl, a.x, a.y);
  int mi = last_ge(a.z, e, m.ni_);
  if (mi == -1) {  // above the top interface: the top layer's values
    mi = last_ge(e[0], e, m.ni_);
    for (int q = 0; q < 2; q++) var[q] = bilinear(m, m.p[3 * q] + mi * sl, a.x, a.y);
    return 0;
  }
  const float dz = __fsub_rn(e[mi], a.z);
  var[0] = layer_val(m, 0, mi, a.x, a.y, dz);
  var[1] = layer_val(m, 1, mi, a.x, a.y, dz);
  if ((int)dz == 0) {  // isEqual(dz, 0.0) with the integer abs()
    const int mt = first_ge(a.z, e, m.ni_) - 1;
    if (mt >= 0) {
      const float rhot = layer_val(m, 0, mt, a.x, a.y, dz), vpt = layer_val(m, 1, mt, a.x, a.y, dz);
      var[0] = (float)__ddiv_rn((double)__fadd_rn(var[0], rhot), 2.0);
      var[1] = (float)__ddiv_rn((double)__fadd_rn(var[1], vpt), 2.0);
    }
  }
  return 0;
}

// kappa = vp vp rho (float, parametrization_layer_ac_iso_loc, media_layer2model.cpp:1302-1305)
__device__ float kappa_of(const float var[2]) { return __fmul_rn(__fmul_rn(var[1], var[1]), var[0]); }

struct GridDev {
  int nx, ny, nz;  // extended grid (ghosts included)
  const float *x, *y, *z;
  float *hx, *hy, *hz;  // half grid
  int *mat;             // material number at the half grid
  float *rho, *lam, *mu;
  int *err;
};

// AC: acoustic files (rho, vp) into rho and kappa (g.lam holds kappa)
template <bool AC>
__global__ void k_media_loc(const __grid_constant__ LayerDev m, const __grid_constant__ GridDev g) {
  const long long n = (long long)g.nx * g.ny * g.nz;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    if constexpr (AC) {
      float var[2];
      const int rc = point_value_ac(m, P3{g.x[t], g.y[t], g.z[t]}, var);
      if (rc) {
        atomicOr(g.err, rc);
        continue;
      }
      g.lam[t] = kappa_of(var);
      g.rho[t] = var[0];
      continue;
    }
    float var[3];
    const int rc = point_value(m, P3{g.x[t], g.y[t], g.z[t]}, var);
    if (rc) {
      atomicOr(g.err, rc);
      continue;
    }
    float lam, mu;
    lame(var, lam, mu);
    g.mu[t] = mu;
    g.lam[t] = lam;
    g.rho[t] = var[0];
  }
}

// GenerateHalfGrid, curvilinear (media_utility.cpp:489-515): the mean of the 8 corners of each
// cell (float sum in order, / 8.0); the last index of any axis keeps the grid point
__global__ void k_half_grid(const __grid_constant__ GridDev g) {
  const long long sl = g.nx, ss = (long long)g.nx * g.ny, n = ss * g.nz;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(t % g.nx), j = (int)((t / g.nx) % g.ny), k = (int)(t / ss);
    const float *G[3] = {g.x, g.y, g.z};
    float *H[3] = {g.hx, g.hy, g.hz};
    for (int a = 0; a < 3; a++) {
      if (i == g.nx - 1 || j == g.ny - 1 || k == g.nz - 1) {
        H[a][t] = G[a][t];
        continue;
      }
      const float *v = G[a];
      float s = v[t];
      s = __fadd_rn(s, v[t + 1]);
      s = __fadd_rn(s, v[t + sl + 1]);
      s = __fadd_rn(s, v[t + sl]);
      s = __fadd_rn(s, v[t + ss]);
      s = __fadd_rn(s, v[t + ss + 1]);
      s = __fadd_rn(s, v[t + ss + sl + 1]);
      s = __fadd_rn(s, v[t + sl + ss]);
      H[a][t] = (float)__ddiv_rn((double)s, 8.0);
    }
  }
}

// MarkInterfaceNumber, curvilinear (media_utility.cpp:1110-1126)
__global__ void k_mark(const __grid_constant__ LayerDev m, const __grid_constant__ GridDev g) {
  const long long n = (long long)g.nx * g.ny * g.nz;
  const size_t sl = (size_t)m.nx * m.ny;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    float e[kMaxInterfaces];
    for (int q = 0; q < m.ni_; q++) e[q] = bilinear(m, m.elev + q * sl, g.hx[t], g.hy[t]);
    int mi = last_ge(g.hz[t], e, m.ni_);
    if (mi == -1) mi = last_ge(e[0], e, m.ni_);
    g.mat[t] = mi;
  }
}

// Equivalent medium where the 8 surrounding half-grid points fall in more than one layer
// (parametrization_layer_el_iso_har / _ari): 9^3 sub-points of the half-grid cell.
// AC: acoustic (parametrization_layer_ac_iso_har / _ari, media_layer2model.cpp:1765-1960): rho
// arithmetically, kappa harmonically (har) or arithmetically (ari); g.lam holds kappa.
template <bool HAR, bool AC>
__global__ void k_media_avg(const __grid_constant__ LayerDev m, const __grid_constant__ GridDev g) {
  const long long sl = g.nx, ss = (long long)g.nx * g.ny;
  const long long n = (long long)(g.nx - 2) * (g.ny - 2) * (g.nz - 2);
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const int i = 1 + (int)(t % (g.nx - 2)), j = 1 + (int)((t / (g.nx - 2)) % (g.ny - 2));
    const int k = 1 + (int)(t / ((long long)(g.nx - 2) * (g.ny - 2)));
    const long long indx = i + j * sl + k * ss;
    const long long c[8] = {indx - 1 - sl - ss, indx - sl - ss, indx - ss, indx - 1 - ss,
                            indx - 1 - sl,      indx - sl,      indx,      indx - 1};
    // NumOfValues (media_utility.cpp:404-418): distinct layers, none if any point is above all
    bool above = false, mixed = false;
    for (int q = 0; q < 8; q++) {
      const int v = g.mat[c[q]];
      if (v == -1) above = true;
      if (v != g.mat[c[0]]) mixed = true;
    }
    if (above || !mixed) continue;
    P3 M[8];
    for (int q = 0; q < 8; q++) M[q] = P3{g.hx[c[q]], g.hy[c[q]], g.hz[c[q]]};
    float acc0 = 0.f, acc1 = 0.f, acc2 = 0.f;  // rho, then kappa^-1 and mu^-1 (har) or lambda and mu (ari)
    int bad = 0;
    auto lerp = [](P3 a, P3 b, int s) {  // a + (b - a) / ng * s, one rounding per step (Point3 operators)
      return P3{__fadd_rn(a.x, __fmul_rn(__fdiv_rn(__fsub_rn(b.x, a.x), (float)kSub), (float)s)),
                __fadd_rn(a.y, __fmul_rn(__fdiv_rn(__fsub_rn(b.y, a.y), (float)kSub), (float)s)),
                __fadd_rn(a.z, __fmul_rn(__fdiv_rn(__fsub_rn(b.z, a.z), (float)kSub), (float)s))};
    };
    // MeshSubdivide (media_utility.cpp:421-448), points in k, j, i order
    for (int kk = 0; kk <= kSub; kk++)
      for (int jj = 0; jj <= kSub; jj++)
        for (int ii = 0; ii <= kSub; ii++) {
          const P3 lx00 = lerp(M[0], M[1], ii), lx10 = lerp(M[3], M[2], ii);
          const P3 lx01 = lerp(M[4], M[5], ii), lx11 = lerp(M[7], M[6], ii);
          const P3 lxy0 = lerp(lx00, lx10, jj), lxy1 = lerp(lx01, lx11, jj);
          float var[3];
          if constexpr (AC) {
            const int rc = point_value_ac(m, lerp(lxy0, lxy1, kk), var);
            if (rc) { bad |= rc; continue; }
            const float kap = kappa_of(var);
            if (HAR) acc1 = (float)__dadd_rn((double)acc1, __ddiv_rn(1.0, (double)kap));
            else acc1 = __fadd_rn(acc1, kap);
            acc0 = __fadd_rn(acc0, var[0]);
            continue;
          }
          const int rc = point_value(m, lerp(lxy0, lxy1, kk), var);
          if (rc) { bad |= rc; continue; }
          float lam, mu;
          lame(var, lam, mu);
          acc0 = __fadd_rn(acc0, var[0]);
          if (HAR) {
            acc1 = (float)__dadd_rn((double)acc1, __ddiv_rn(1.0, __dadd_rn((double)lam, __dmul_rn(2.0 / 3.0, (double)mu))));
            acc2 = (float)__dadd_rn((double)acc2, __ddiv_rn(1.0, (double)mu));
          } else {
            acc1 = __fadd_rn(acc1, lam);
            acc2 = __fadd_rn(acc2, mu);
          }
        }
    if (bad) { atomicOr(g.err, bad); continue; }
    const double nsg = (double)((kSub + 1) * (kSub + 1) * (kSub + 1));
    if constexpr (AC) {
      g.rho[indx] = (float)__ddiv_rn((double)acc0, nsg);
      g.lam[indx] = HAR ? (float)__ddiv_rn(nsg, (double)acc1) : (float)__ddiv_rn((double)acc1, nsg);
      continue;
    }
    if (HAR) {
      const float hmu = (float)__ddiv_rn(nsg, (double)acc2);
      const float hkap = (float)__ddiv_rn(nsg, (double)acc1);
      g.rho[indx] = (float)__ddiv_rn((double)acc0, nsg);
      g.lam[indx] = (float)__dsub_rn((double)hkap, __dmul_rn(2.0 / 3.0, (double)hmu));
      g.mu[indx] = hmu;
    } else {
      g.lam[indx] = (float)__ddiv_rn((double)acc1, nsg);
      g.mu[indx] = (float)__ddiv_rn((double)acc2, nsg);
      g.rho[indx] = (float)__ddiv_rn((double)acc0, nsg);
    }
  }
}


// -----------------------------------------------------------------------------------------
// VTI, TTI and 21-Cij layer files (media_layer2model_el_vti / _el_aniso,
// src/media/media_layer2model.cpp:173-398). The parameters of a file type, in the file's order:
//   22 vti_prem     rho vph vpv vsh vsv eta            25 tti_thomsen rho vp0 vs0 epsilon delta gamma azimuth dip
//   23 vti_thomsen  rho vp0 vs0 epsilon delta gamma    26 tti_bond    rho c11 c33 c55 c66 c13 azimuth dip
//   24 vti_cij      rho c11 c33 c55 c66 c13            27 aniso_cij   rho c11 c12 ... c66 (21)
// Every parameter is value + dz^pow * grad of its layer (CalPointValue_layer,
// media_layer2model.cpp:454-1216), averaged with the layer above on an interface; para2vti /
// para2tti (media_utility.cpp:620-831) turn them into the stiffness: 6 fields (rho c11 c33 c55
// c66 c13) for the VTI files, 22 (rho c11 c12 ... c66) for the others. The har / ari
// averages take c_ij harmonically / arithmetically over the 9^3 sub-points, rho arithmetically.
// NEWDZ: on an interface, the layer above is evaluated at the point's depth below that layer's
// own interface (PREM and Thomsen VTI files, media_layer2model.cpp:596, 669), or, kept alike
// on purpose, at the depth below the point's own interface, as the reference does for the
// VTI-Cij, TTI and 21-Cij files (:721-757, 805-850, 967-1082, 1129-1174 reuse dz).
template <int T> struct LayerFile;
template <> struct LayerFile<22> { static constexpr int NPAR = 6, NOUT = 6; static constexpr bool NEWDZ = true; };
template <> struct LayerFile<23> { static constexpr int NPAR = 6, NOUT = 6; static constexpr bool NEWDZ = true; };
template <> struct LayerFile<24> { static constexpr int NPAR = 6, NOUT = 6; static constexpr bool NEWDZ = false; };
template <> struct LayerFile<25> { static constexpr int NPAR = 8, NOUT = 22; static constexpr bool NEWDZ = false; };
template <> struct LayerFile<26> { static constexpr int NPAR = 8, NOUT = 22; static constexpr bool NEWDZ = false; };
template <> struct LayerFile<27> { static constexpr int NPAR = 22, NOUT = 22; static constexpr bool NEWDZ = false; };

// value + dz^pow * grad of parameter q of layer mi at (x, y)
__device__ float layer_val_par(const LayerDev &m, int q, int mi, float x, float y, float dz) {
  const size_t sl = (size_t)m.nx * m.ny, lv = sl * m.ni_;
  const float *b = m.par + (size_t)q * 3 * lv + (size_t)mi * sl;
  const float v = bilinear(m, b, x, y);
  const float g = bilinear(m, b + lv, x, y);
  const float pw = bilinear(m, b + 2 * lv, x, y);
  return (float)__dadd_rn((double)v, __dmul_rn(pow((double)dz, (double)pw), (double)g));
}

// AssignLayerMediaPara2Point + CalPointValue_layer for the general files; 1: outside the mesh
template <int NPAR, bool NEWDZ>
__device__ int point_params(const LayerDev &m, P3 a, float var[NPAR]) {
  const float maxx = __fadd_rn(m.x0, __fmul_rn(m.dx, (float)(m.nx - 1)));
  const float maxy = __fadd_rn(m.y0, __fmul_rn(m.dy, (float)(m.ny - 1)));
  if (a.x < m.x0 || a.x > maxx || a.y < m.y0 || a.y > maxy) return 1;
  float e[kMaxInterfaces];
  const size_t sl = (size_t)m.nx * m.ny, lv = sl * m.ni_;
  for (int n = 0; n < m.ni_; n++) e[n] = bilinear(m, m.elev + n * sl, a.x, a.y);
  int mi = last_ge(a.z, e, m.ni_);
  if (mi == -1) {  // above the top interface: the top layer's values
    mi = last_ge(e[0], e, m.ni_);
    for (int q = 0; q < NPAR; q++) var[q] = bilinear(m, m.par + (size_t)q * 3 * lv + (size_t)mi * sl, a.x, a.y);
    return 0;
  }
  float dz = __fsub_rn(e[mi], a.z);
  for (int q = 0; q < NPAR; q++) var[q] = layer_val_par(m, q, mi, a.x, a.y, dz);
  if ((int)dz == 0) {  // on an interface (the reference's integer-abs test)
    const int mt = first_ge(a.z, e, m.ni_) - 1;
    if (mt >= 0) {
      if (NEWDZ) dz = __fsub_rn(e[mt], a.z);
      for (int q = 0; q < NPAR; q++) {
        const float top = layer_val_par(m, q, mt, a.x, a.y, dz);
        var[q] = (float)__ddiv_rn((double)__fadd_rn(var[q], top), 2.0);
      }
    }
  }
  return 0;
}

// sqrt(2 delta c33 (c33 - cs) + (c33 - cs)^2) - cs: Thomsen's c13 (the reference's expression,
// double with the float square of the float difference)
__device__ float thomsen_c13(float delta, float c33, float cs) {
  const float dcs = __fsub_rn(c33, cs);
  const double t = __dadd_rn(__dmul_rn(__dmul_rn(__dmul_rn(2.0, (double)delta), (double)c33), (double)dcs),
                             (double)__fmul_rn(dcs, dcs));
  return (float)__dsub_rn(__dsqrt_rn(t), (double)cs);
}

// 2.0 x a * c + c (double, stored float)
__device__ float thomsen_scale(float a, float c) {
  return (float)__dadd_rn(__dmul_rn(__dmul_rn(2.0, (double)a), (double)c), (double)c);
}

// para2vti: o = rho c11 c33 c55 c66 c13
template <int T>
__device__ void para2vti(const float *v, float *o) {
  if constexpr (T == 22) {  // rho vph vpv vsh vsv eta
    const float rho = v[0];
    o[1] = __fmul_rn(__fmul_rn(v[1], v[1]), rho);
    o[2] = __fmul_rn(__fmul_rn(v[2], v[2]), rho);
    o[4] = __fmul_rn(__fmul_rn(v[3], v[3]), rho);
    o[3] = __fmul_rn(__fmul_rn(v[4], v[4]), rho);
    o[0] = rho;
    o[5] = (float)__dmul_rn((double)v[5], __dsub_rn((double)o[1], __dmul_rn(2.0, (double)o[3])));
  } else if constexpr (T == 23) {  // rho vp0 vs0 epsilon delta gamma
    const float rho = v[0];
    const float c33 = __fmul_rn(__fmul_rn(v[1], v[1]), rho), c55 = __fmul_rn(__fmul_rn(v[2], v[2]), rho);
    o[0] = rho;
    o[2] = c33;
    o[3] = c55;
    o[4] = thomsen_scale(v[5], c55);
    o[1] = thomsen_scale(v[3], c33);
    o[5] = thomsen_c13(v[4], c33, c55);
  } else {  // rho c11 c33 c55 c66 c13
    for (int q = 0; q < 6; q++) o[q] = v[q];
  }
}

// BondTransform (media_utility.cpp:683-724): C = R C0 R^T for dip theta and azimuth phi
// (degrees), float matrix products summed in index order. Kept alike on purpose: row 5 of R
// holds a11 a31 + a12 a31 in its last column, as the reference's table does.
__device__ void bond(const float c0[6][6], float theta, float phi, float *o) {
  const double pi = 3.14159265358979311600;  // acos(-1) in double
  theta = (float)__dmul_rn((double)theta, __ddiv_rn(pi, 180.0));
  phi = (float)__dmul_rn((double)phi, __ddiv_rn(pi, 180.0));
  const float ct = cosf(theta), st = sinf(theta), cp = cosf(phi), sp = sinf(phi);
  const float a11 = __fmul_rn(ct, sp), a12 = cp, a13 = __fmul_rn(st, sp);
  const float a21 = -__fmul_rn(ct, cp), a22 = sp, a23 = -__fmul_rn(st, cp);
  const float a31 = -st, a32 = 0.f, a33 = ct;
  auto m2 = [](float a, float b) { return __fmul_rn(__fmul_rn(2.f, a), b); };
  const float R[6][6] = {
      {__fmul_rn(a11, a11), __fmul_rn(a12, a12), __fmul_rn(a13, a13), m2(a12, a13), m2(a13, a11), m2(a11, a12)},
      {__fmul_rn(a21, a21), __fmul_rn(a22, a22), __fmul_rn(a23, a23), m2(a22, a23), m2(a23, a21), m2(a21, a22)},
      {__fmul_rn(a31, a31), __fmul_rn(a32, a32), __fmul_rn(a33, a33), m2(a32, a33), m2(a33, a31), m2(a31, a32)},
      {__fmul_rn(a21, a31), __fmul_rn(a22, a32), __fmul_rn(a23, a33), __fadd_rn(__fmul_rn(a22, a33), __fmul_rn(a23, a32)),
       __fadd_rn(__fmul_rn(a21, a33), __fmul_rn(a23, a31)), __fadd_rn(__fmul_rn(a22, a31), __fmul_rn(a21, a32))},
      {__fmul_rn(a31, a11), __fmul_rn(a32, a12), __fmul_rn(a33, a13), __fadd_rn(__fmul_rn(a12, a33), __fmul_rn(a13, a32)),
       __fadd_rn(__fmul_rn(a13, a31), __fmul_rn(a11, a33)), __fadd_rn(__fmul_rn(a11, a31), __fmul_rn(a12, a31))},
      {__fmul_rn(a11, a21), __fmul_rn(a12, a22), __fmul_rn(a13, a23), __fadd_rn(__fmul_rn(a12, a23), __fmul_rn(a13, a22)),
       __fadd_rn(__fmul_rn(a13, a21), __fmul_rn(a11, a23)), __fadd_rn(__fmul_rn(a11, a22), __fmul_rn(a12, a21))}};
  float RC[6][6];
  for (int i = 0; i < 6; i++)
    for (int j = 0; j < 6; j++) {
      float s = 0.f;
      for (int k = 0; k < 6; k++) s = __fadd_rn(s, __fmul_rn(R[i][k], c0[k][j]));
      RC[i][j] = s;
    }
  int n = 1;
  for (int i = 0; i < 6; i++)
    for (int j = i; j < 6; j++) {
      float s = 0.f;
      for (int k = 0; k < 6; k++) s = __fadd_rn(s, __fmul_rn(RC[i][k], R[j][k]));
      o[n++] = s;
    }
}

// para2tti: o = rho c11 c12 c13 c14 c15 c16 c22 c23 c24 c25 c26 c33 c34 c35 c36 c44 c45 c46 c55 c56 c66
template <int T>
__device__ void para2tti(const float *v, float *o) {
  if constexpr (T == 27) {
    for (int q = 0; q < 22; q++) o[q] = v[q];
  } else {
    float c11, c33, c44, c66, c13;
    if constexpr (T == 25) {  // rho vp0 vs0 epsilon delta gamma azimuth dip
      c33 = __fmul_rn(__fmul_rn(v[1], v[1]), v[0]);
      c44 = __fmul_rn(__fmul_rn(v[2], v[2]), v[0]);
      c66 = thomsen_scale(v[5], c44);
      c11 = thomsen_scale(v[3], c33);
      c13 = thomsen_c13(v[4], c33, c44);
    } else {  // rho c11 c33 c55 c66 c13 azimuth dip
      c11 = v[1]; c33 = v[2]; c44 = v[3]; c66 = v[4]; c13 = v[5];
    }
    o[0] = v[0];
    const float c12 = __fsub_rn(c11, __fmul_rn(2.f, c66));
    const float c0[6][6] = {{c11, c12, c13, 0.f, 0.f, 0.f}, {c12, c11, c13, 0.f, 0.f, 0.f}, {c13, c13, c33, 0.f, 0.f, 0.f},
                            {0.f, 0.f, 0.f, c44, 0.f, 0.f}, {0.f, 0.f, 0.f, 0.f, c44, 0.f}, {0.f, 0.f, 0.f, 0.f, 0.f, c66}};
    bond(c0, v[7], v[6], o);
  }
}

template <int T>
__device__ void para2out(const float *v, float *o) {
  if constexpr (LayerFile<T>::NOUT == 6) para2vti<T>(v, o);
  else para2tti<T>(v, o);
}

struct OutDev {
  long long n;
  float *f;  // [NOUT][n]
  int *err;
};

template <int T>
__global__ void k_media_loc_gen(const __grid_constant__ LayerDev m, const __grid_constant__ GridDev g,
                                const __grid_constant__ OutDev out) {
  constexpr int NP = LayerFile<T>::NPAR, NO = LayerFile<T>::NOUT;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < out.n; t += (long long)gridDim.x * blockDim.x) {
    float var[NP], o[NO];
    if (point_params<NP, LayerFile<T>::NEWDZ>(m, P3{g.x[t], g.y[t], g.z[t]}, var)) {
      atomicOr(out.err, 1);
      continue;
    }
    para2out<T>(var, o);
    for (int q = 0; q < NO; q++) out.f[q * out.n + t] = o[q];
  }
}

// the har / ari equivalent medium of the general files (parametrization_layer_el_vti_har /
// _ari, _el_aniso_har / _ari, media_layer2model.cpp:2176-2793)
template <int T, bool HAR>
__global__ void k_media_avg_gen(const __grid_constant__ LayerDev m, const __grid_constant__ GridDev g,
                                const __grid_constant__ OutDev out) {
  constexpr int NP = LayerFile<T>::NPAR, NO = LayerFile<T>::NOUT;
  const long long sl = g.nx, ss = (long long)g.nx * g.ny;
  const long long n = (long long)(g.nx - 2) * (g.ny - 2) * (g.nz - 2);
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const int i = 1 + (int)(t % (g.nx - 2)), j = 1 + (int)((t / (g.nx - 2)) % (g.ny - 2));
    const int k = 1 + (int)(t / ((long long)(g.nx - 2) * (g.ny - 2)));
    const long long indx = i + j * sl + k * ss;
    const long long c[8] = {indx - 1 - sl - ss, indx - sl - ss, indx - ss, indx - 1 - ss,
                            indx - 1 - sl,      indx - sl,      indx,      indx - 1};
    bool above = false, mixed = false;
    for (int q = 0; q < 8; q++) {
      const int v = g.mat[c[q]];
      if (v == -1) above = true;
      if (v != g.mat[c[0]]) mixed = true;
    }
    if (above || !mixed) continue;
    P3 M[8];
    for (int q = 0; q < 8; q++) M[q] = P3{g.hx[c[q]], g.hy[c[q]], g.hz[c[q]]};
    float acc[NO];
    for (int q = 0; q < NO; q++) acc[q] = 0.f;
    int bad = 0;
    auto lerp = [](P3 a, P3 b, int s) {
      return P3{__fadd_rn(a.x, __fmul_rn(__fdiv_rn(__fsub_rn(b.x, a.x), (float)kSub), (float)s)),
                __fadd_rn(a.y, __fmul_rn(__fdiv_rn(__fsub_rn(b.y, a.y), (float)kSub), (float)s)),
                __fadd_rn(a.z, __fmul_rn(__fdiv_rn(__fsub_rn(b.z, a.z), (float)kSub), (float)s))};
    };
    for (int kk = 0; kk <= kSub; kk++)
      for (int jj = 0; jj <= kSub; jj++)
        for (int ii = 0; ii <= kSub; ii++) {
          const P3 lx00 = lerp(M[0], M[1], ii), lx10 = lerp(M[3], M[2], ii);
          const P3 lx01 = lerp(M[4], M[5], ii), lx11 = lerp(M[7], M[6], ii);
          const P3 lxy0 = lerp(lx00, lx10, jj), lxy1 = lerp(lx01, lx11, jj);
          float var[NP], o[NO];
          if (point_params<NP, LayerFile<T>::NEWDZ>(m, lerp(lxy0, lxy1, kk), var)) { bad = 1; continue; }
          para2out<T>(var, o);
          acc[0] = __fadd_rn(acc[0], o[0]);
          for (int q = 1; q < NO; q++)
            acc[q] = HAR ? (float)__dadd_rn((double)acc[q], __ddiv_rn(1.0, (double)o[q])) : __fadd_rn(acc[q], o[q]);
        }
    if (bad) { atomicOr(out.err, 1); continue; }
    constexpr int nsg = (kSub + 1) * (kSub + 1) * (kSub + 1);
    out.f[indx] = __fdiv_rn(acc[0], (float)nsg);
    for (int q = 1; q < NO; q++)
      out.f[q * out.n + indx] = HAR ? (float)__ddiv_rn((double)nsg, (double)acc[q]) : __fdiv_rn(acc[q], (float)nsg);
  }
}

template <int T>
void launch_media_gen(const LayerDev &m, const GridDev &g, const OutDev &o, int method, cudaStream_t st) {
  k_media_loc_gen<T><<<148 * 8, 256, 0, st>>>(m, g, o);
  if (method == CGFD_MEDIA_LOC) return;
  k_half_grid<<<148 * 8, 256, 0, st>>>(g);
  k_mark<<<148 * 8, 256, 0, st>>>(m, g);
  if (method == CGFD_MEDIA_HAR) k_media_avg_gen<T, true><<<148 * 8, 128, 0, st>>>(m, g, o);
  else k_media_avg_gen<T, false><<<148 * 8, 128, 0, st>>>(m, g, o);
}

}  // namespace
}  // namespace cgfd

namespace cgfd {
namespace {
// The isotropic families on the GPU: elastic_isotropic files (hp: rho, vp, vs with gradient and
// power each, 9 arrays) into rho, lambda, mu, or acoustic_isotropic files (ac; rho, vp: 6 arrays)
// into rho, kappa; medium gets 3 or 2 fields of (ni+6)(nj+6)(nk+6) points.
int layer_iso_family(int device, int ni, int nj, int nk, const float *coord, int num_interfaces, int mnx, int mny,
                     float x0, float y0, float dx, float dy, const float *elevation, const float *const *hp, bool ac,
                     int method, float *medium) {
  const int nq = ac ? 6 : 9, nout = ac ? 2 : 3;
  const size_t nx = ni + 6, ny = nj + 6, nz = nk + 6, n = nx * ny * nz;
  const size_t msz = (size_t)num_interfaces * mnx * mny;
  std::vector<void *> owned;
  cudaStream_t st = nullptr;
  auto cleanup = [&] {
    for (void *q : owned) cudaFree(q);
    if (st) cudaStreamDestroy(st);
  };
  auto fail = [&](cudaError_t e, const char *what) {
    cleanup();
    set_last_error(std::string(what) + ": " + cudaGetErrorString(e));
    return e == cudaErrorMemoryAllocation ? CGFD_ERR_NOMEM : CGFD_ERR_CUDA;
  };
  auto dalloc = [&](size_t bytes, void **out) {
    cudaError_t e = cudaMalloc(out, bytes);
    if (e == cudaSuccess) owned.push_back(*out);
    return e;
  };
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) return fail(e, "cudaSetDevice");
  if ((e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking)) != cudaSuccess) return fail(e, "cudaStreamCreate");
  LayerDev m{};
  m.ni_ = num_interfaces; m.nx = mnx; m.ny = mny;
  m.x0 = x0; m.y0 = y0; m.dx = dx; m.dy = dy;
  float *dm = nullptr;
  if ((e = dalloc((1 + nq) * msz * sizeof(float), (void **)&dm)) != cudaSuccess) return fail(e, "cudaMalloc");
  if ((e = cudaMemcpyAsync(dm, elevation, msz * sizeof(float), cudaMemcpyHostToDevice, st)) != cudaSuccess)
    return fail(e, "cudaMemcpy");
  m.elev = dm;
  for (int q = 0; q < nq; q++) {
    if ((e = cudaMemcpyAsync(dm + (1 + q) * msz, hp[q], msz * sizeof(float), cudaMemcpyHostToDevice, st)) != cudaSuccess)
      return fail(e, "cudaMemcpy");
    m.p[q] = dm + (1 + q) * msz;
  }
  GridDev g;
  g.nx = (int)nx; g.ny = (int)ny; g.nz = (int)nz;
  float *dc = nullptr, *dout = nullptr;
  int *derr = nullptr;
  if ((e = dalloc(3 * n * sizeof(float), (void **)&dc)) != cudaSuccess) return fail(e, "cudaMalloc");
  if ((e = dalloc((size_t)nout * n * sizeof(float), (void **)&dout)) != cudaSuccess) return fail(e, "cudaMalloc");
  if ((e = dalloc(sizeof(int), (void **)&derr)) != cudaSuccess) return fail(e, "cudaMalloc");
  if ((e = cudaMemcpyAsync(dc, coord, 3 * n * sizeof(float), cudaMemcpyHostToDevice, st)) != cudaSuccess)
    return fail(e, "cudaMemcpy");
  cudaMemsetAsync(derr, 0, sizeof(int), st);
  g.x = dc; g.y = dc + n; g.z = dc + 2 * n;
  // the medium order: rho, lambda, mu (elastic) or rho, kappa (acoustic, kappa in g.lam)
  g.rho = dout; g.lam = dout + n; g.mu = ac ? nullptr : dout + 2 * n;
  g.err = derr;
  g.hx = g.hy = g.hz = nullptr;
  g.mat = nullptr;
  if (ac) k_media_loc<true><<<148 * 8, 256, 0, st>>>(m, g);
  else k_media_loc<false><<<148 * 8, 256, 0, st>>>(m, g);
  if (method != CGFD_MEDIA_LOC) {
    float *dh = nullptr;
    int *dmat = nullptr;
    if ((e = dalloc(3 * n * sizeof(float), (void **)&dh)) != cudaSuccess) return fail(e, "cudaMalloc");
    if ((e = dalloc(n * sizeof(int), (void **)&dmat)) != cudaSuccess) return fail(e, "cudaMalloc");
    g.hx = dh; g.hy = dh + n; g.hz = dh + 2 * n;
    g.mat = dmat;
    k_half_grid<<<148 * 8, 256, 0, st>>>(g);
    k_mark<<<148 * 8, 256, 0, st>>>(m, g);
    if (method == CGFD_MEDIA_HAR) {
      if (ac) k_media_avg<true, true><<<148 * 8, 128, 0, st>>>(m, g);
      else k_media_avg<true, false><<<148 * 8, 128, 0, st>>>(m, g);
    } else {
      if (ac) k_media_avg<false, true><<<148 * 8, 128, 0, st>>>(m, g);
      else k_media_avg<false, false><<<148 * 8, 128, 0, st>>>(m, g);
    }
  }
  if ((e = cudaGetLastError()) != cudaSuccess) return fail(e, "media kernels");
  int herr = 0;
  if ((e = cudaMemcpyAsync(&herr, derr, sizeof(int), cudaMemcpyDeviceToHost, st)) != cudaSuccess)
    return fail(e, "cudaMemcpy");
  if ((e = cudaMemcpyAsync(medium, dout, (size_t)nout * n * sizeof(float), cudaMemcpyDeviceToHost, st)) !=
      cudaSuccess)
    return fail(e, "cudaMemcpy");
  if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return fail(e, "cudaStreamSynchronize");
  cleanup();
  if (herr) {
    set_last_error((herr & 1) ? "a grid point lies outside the interface mesh"
                              : "vp must be larger than sqrt(2) vs in every layer");
    return CGFD_ERR_INVALID;
  }
  return CGFD_OK;
}
}  // namespace
}  // namespace cgfd

extern "C" int cgfd_media_layer_el_iso_gpu(int device, int ni, int nj, int nk, const float *coord,
                                           const cgfd_layer_model *lm, int method, float *medium) {
  using namespace cgfd;
  if (!coord || !lm || !medium || ni < 4 || nj < 4 || nk < 4 || method < CGFD_MEDIA_LOC || method > CGFD_MEDIA_ARI) {
    set_last_error("invalid argument");
    return CGFD_ERR_INVALID;
  }
  if (lm->num_interfaces < 1 || lm->num_interfaces > kMaxInterfaces || lm->nx < 2 || lm->ny < 2 || !lm->elevation) {
    set_last_error("layer model: 1 to 64 interfaces on a mesh of at least 2 x 2 points are required");
    return CGFD_ERR_INVALID;
  }
  const float *hp[9] = {lm->rho, lm->rho_grad, lm->rho_pow, lm->vp, lm->vp_grad, lm->vp_pow, lm->vs, lm->vs_grad, lm->vs_pow};
  for (const float *q : hp)
    if (!q) { set_last_error("layer model: a parameter array is missing"); return CGFD_ERR_INVALID; }
  return layer_iso_family(device, ni, nj, nk, coord, lm->num_interfaces, lm->nx, lm->ny, lm->x0, lm->y0, lm->dx, lm->dy,
                          lm->elevation, hp, false, method, medium);
}

namespace cgfd {
namespace {
// The family's fields (iso rho lambda mu | VTI rho c11 c33 c55 c66 c13 | 22 Cij) into the
// cgfd_problem_desc medium of medium_type; iso and VTI families into a 21-Cij medium by the
// reference's expansion (media_layer2model_el_aniso / media_grid2model_el_aniso).
int family_to_medium(const std::vector<float> &fam, int nfam, int medium_type, size_t n, float *medium) {
  const int nout_med = medium_type == CGFD_MEDIUM_ELASTIC_ISO ? 3 : (medium_type == CGFD_MEDIUM_ELASTIC_VTI ? 6 : 22);
  auto M = [&](int f) { return medium + (size_t)f * n; };
  if (medium_type == CGFD_MEDIUM_ELASTIC_ISO) {
    std::memcpy(medium, fam.data(), 3 * n * sizeof(float));
    return CGFD_OK;
  }
  auto F = [&](int f) { return fam.data() + (size_t)f * n; };
  if (medium_type == CGFD_MEDIUM_ELASTIC_VTI) {  // rho c11 c33 c55 c66 c13 -> rho c11 c13 c33 c55 c66
    const int from[6] = {0, 1, 5, 2, 3, 4};
    for (int f = 0; f < 6; f++) std::memcpy(M(f), F(from[f]), n * sizeof(float));
    return CGFD_OK;
  }
  // 21-Cij medium (desc order rho c11 c12 c13 c14 c15 c16 c22 c23 c24 c25 c26 c33 c34 c35 c36 c44
  // c45 c46 c55 c56 c66)
  if (nfam == 22) {
    std::memcpy(medium, fam.data(), 22 * n * sizeof(float));
    return CGFD_OK;
  }
  std::memset(medium, 0, (size_t)nout_med * n * sizeof(float));
  enum { RHO = 0, C11 = 1, C12 = 2, C13 = 3, C22 = 7, C23 = 8, C33 = 12, C44 = 16, C55 = 19, C66 = 21 };
  const bool iso = nfam == 3;
#pragma omp parallel for schedule(static)
  for (long long t = 0; t < (long long)n; t++) {
    if (iso) {  // el_aniso's elastic_isotropic branch: lambda -> c13, mu -> c44
      const float c13 = F(1)[t], c44 = F(2)[t];
      const float c11 = (float)((double)c13 + 2.0 * (double)c44);
      M(RHO)[t] = F(0)[t];
      M(C11)[t] = c11; M(C22)[t] = c11; M(C33)[t] = c11;
      M(C12)[t] = c13; M(C13)[t] = c13; M(C23)[t] = c13;
      M(C44)[t] = c44; M(C55)[t] = c44; M(C66)[t] = c44;
    } else {  // its VTI branch
      const float c11 = F(1)[t], c33 = F(2)[t], c55 = F(3)[t], c66 = F(4)[t], c13 = F(5)[t];
      M(RHO)[t] = F(0)[t];
      M(C11)[t] = c11; M(C22)[t] = c11; M(C33)[t] = c33;
      M(C12)[t] = (float)((double)c11 - 2.0 * (double)c66);
      M(C13)[t] = c13; M(C23)[t] = c13;
      M(C44)[t] = c55; M(C55)[t] = c55; M(C66)[t] = c66;
    }
  }
  return CGFD_OK;
}
}  // namespace
}  // namespace cgfd

extern "C" int cgfd_media_layer_gpu(int device, int ni, int nj, int nk, const float *coord, const cgfd_layer_media *lm,
                                    int medium_type, int method, float *medium) {
  using namespace cgfd;
  if (!coord || !lm || !medium || !lm->elevation || !lm->param || ni < 4 || nj < 4 || nk < 4 ||
      method < CGFD_MEDIA_LOC || method > CGFD_MEDIA_ARI) {
    set_last_error("invalid argument");
    return CGFD_ERR_INVALID;
  }
  if (lm->num_interfaces < 1 || lm->num_interfaces > kMaxInterfaces || lm->nx < 2 || lm->ny < 2) {
    set_last_error("layer model: 1 to 64 interfaces on a mesh of at least 2 x 2 points are required");
    return CGFD_ERR_INVALID;
  }
  const int T = lm->type;
  // acoustic_isotropic files into acoustic media (media_layer2model_ac_iso, media_layer2model.cpp:70-118)
  if (T == CGFD_LAYER_ACOUSTIC_ISO || medium_type == CGFD_MEDIUM_ACOUSTIC_ISO) {
    if (T != CGFD_LAYER_ACOUSTIC_ISO || medium_type != CGFD_MEDIUM_ACOUSTIC_ISO) {
      set_last_error("layer file type not usable for this medium type");
      return CGFD_ERR_INVALID;
    }
    const size_t lv = (size_t)lm->num_interfaces * lm->nx * lm->ny;
    const float *hp[6];
    for (int q = 0; q < 6; q++) hp[q] = lm->param + (size_t)q * lv;  // rho, rho_grad, rho_pow, vp, vp_grad, vp_pow
    return layer_iso_family(device, ni, nj, nk, coord, lm->num_interfaces, lm->nx, lm->ny, lm->x0, lm->y0, lm->dx,
                            lm->dy, lm->elevation, hp, true, method, medium);
  }
  // the file types each target medium accepts (media_layer2model_el_iso / _el_vti / _el_aniso)
  const bool ok = (medium_type == CGFD_MEDIUM_ELASTIC_ISO && T == CGFD_LAYER_ELASTIC_ISO) ||
                  (medium_type == CGFD_MEDIUM_ELASTIC_VTI && T >= CGFD_LAYER_VTI_PREM && T <= CGFD_LAYER_VTI_CIJ) ||
                  (medium_type == CGFD_MEDIUM_ELASTIC_ANISO && T >= CGFD_LAYER_ELASTIC_ISO && T <= CGFD_LAYER_ANISO_CIJ);
  if (!ok) {
    set_last_error("layer file type not usable for this medium type");
    return CGFD_ERR_INVALID;
  }
  const size_t nx = ni + 6, ny = nj + 6, nz = nk + 6, n = nx * ny * nz;
  const size_t lv = (size_t)lm->num_interfaces * lm->nx * lm->ny;

  // the family's fields on the device: iso (rho lambda mu), VTI (rho c11 c33 c55 c66 c13), 22 Cij
  std::vector<float> fam;
  int nfam = 0;
  if (T == CGFD_LAYER_ELASTIC_ISO) {
    cgfd_layer_model m{};
    m.num_interfaces = lm->num_interfaces; m.nx = lm->nx; m.ny = lm->ny;
    m.x0 = lm->x0; m.y0 = lm->y0; m.dx = lm->dx; m.dy = lm->dy;
    m.elevation = lm->elevation;
    const float **pp[9] = {&m.rho, &m.rho_grad, &m.rho_pow, &m.vp, &m.vp_grad, &m.vp_pow, &m.vs, &m.vs_grad, &m.vs_pow};
    for (int q = 0; q < 9; q++) *pp[q] = lm->param + (size_t)q * lv;
    if (medium_type == CGFD_MEDIUM_ELASTIC_ISO)
      return cgfd_media_layer_el_iso_gpu(device, ni, nj, nk, coord, &m, method, medium);
    fam.resize(3 * n);
    nfam = 3;
    const int rc = cgfd_media_layer_el_iso_gpu(device, ni, nj, nk, coord, &m, method, fam.data());
    if (rc) return rc;
  } else {
    nfam = T <= CGFD_LAYER_VTI_CIJ ? 6 : 22;
    const int npar = T <= CGFD_LAYER_VTI_CIJ ? 6 : (T == CGFD_LAYER_ANISO_CIJ ? 22 : 8);
    std::vector<void *> owned;
    cudaStream_t st = nullptr;
    auto cleanup = [&] {
      for (void *q : owned) cudaFree(q);
      if (st) cudaStreamDestroy(st);
    };
    auto fail = [&](cudaError_t e, const char *what) {
      cleanup();
      set_last_error(std::string(what) + ": " + cudaGetErrorString(e));
      return e == cudaErrorMemoryAllocation ? CGFD_ERR_NOMEM : CGFD_ERR_CUDA;
    };
    auto dalloc = [&](size_t bytes, void **out) {
      cudaError_t e = cudaMalloc(out, bytes);
      if (e == cudaSuccess) owned.push_back(*out);
      return e;
    };
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return fail(e, "cudaSetDevice");
    if ((e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking)) != cudaSuccess) return fail(e, "cudaStreamCreate");
    LayerDev m{};
    m.ni_ = lm->num_interfaces; m.nx = lm->nx; m.ny = lm->ny;
    m.x0 = lm->x0; m.y0 = lm->y0; m.dx = lm->dx; m.dy = lm->dy;
    float *dm = nullptr, *dc = nullptr, *dout = nullptr, *dh = nullptr;
    int *derr = nullptr, *dmat = nullptr;
    if ((e = dalloc((1 + 3 * (size_t)npar) * lv * sizeof(float), (void **)&dm)) != cudaSuccess) return fail(e, "cudaMalloc");
    if ((e = cudaMemcpyAsync(dm, lm->elevation, lv * sizeof(float), cudaMemcpyHostToDevice, st)) != cudaSuccess ||
        (e = cudaMemcpyAsync(dm + lv, lm->param, 3 * (size_t)npar * lv * sizeof(float), cudaMemcpyHostToDevice, st)) !=
            cudaSuccess)
      return fail(e, "cudaMemcpy");
    m.elev = dm;
    m.par = dm + lv;
    if ((e = dalloc(3 * n * sizeof(float), (void **)&dc)) != cudaSuccess) return fail(e, "cudaMalloc");
    if ((e = dalloc((size_t)nfam * n * sizeof(float), (void **)&dout)) != cudaSuccess) return fail(e, "cudaMalloc");
    if ((e = dalloc(sizeof(int), (void **)&derr)) != cudaSuccess) return fail(e, "cudaMalloc");
    if ((e = cudaMemcpyAsync(dc, coord, 3 * n * sizeof(float), cudaMemcpyHostToDevice, st)) != cudaSuccess)
      return fail(e, "cudaMemcpy");
    cudaMemsetAsync(derr, 0, sizeof(int), st);
    GridDev g{};
    g.nx = (int)nx; g.ny = (int)ny; g.nz = (int)nz;
    g.x = dc; g.y = dc + n; g.z = dc + 2 * n;
    if (method != CGFD_MEDIA_LOC) {
      if ((e = dalloc(3 * n * sizeof(float), (void **)&dh)) != cudaSuccess) return fail(e, "cudaMalloc");
      if ((e = dalloc(n * sizeof(int), (void **)&dmat)) != cudaSuccess) return fail(e, "cudaMalloc");
      g.hx = dh; g.hy = dh + n; g.hz = dh + 2 * n;
      g.mat = dmat;
    }
    OutDev o{(long long)n, dout, derr};
    switch (T) {
      case CGFD_LAYER_VTI_PREM: launch_media_gen<22>(m, g, o, method, st); break;
      case CGFD_LAYER_VTI_THOMSEN: launch_media_gen<23>(m, g, o, method, st); break;
      case CGFD_LAYER_VTI_CIJ: launch_media_gen<24>(m, g, o, method, st); break;
      case CGFD_LAYER_TTI_THOMSEN: launch_media_gen<25>(m, g, o, method, st); break;
      case CGFD_LAYER_TTI_BOND: launch_media_gen<26>(m, g, o, method, st); break;
      default: launch_media_gen<27>(m, g, o, method, st); break;
    }
    if ((e = cudaGetLastError()) != cudaSuccess) return fail(e, "media kernels");
    int herr = 0;
    fam.resize((size_t)nfam * n);
    if ((e = cudaMemcpyAsync(&herr, derr, sizeof(int), cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
        (e = cudaMemcpyAsync(fam.data(), dout, (size_t)nfam * n * sizeof(float), cudaMemcpyDeviceToHost, st)) !=
            cudaSuccess)
      return fail(e, "cudaMemcpy");
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return fail(e, "cudaStreamSynchronize");
    cleanup();
    if (herr) {
      set_last_error("a grid point lies outside the interface mesh");
      return CGFD_ERR_INVALID;
    }
  }
  return family_to_medium(fam, nfam, medium_type, n, medium);
}

// -----------------------------------------------------------------------------------------
// Binary models (media_bin2model_el_iso, src/media/media_bin2model.cpp:27-233): the model cut to
// the grid's x / y range is sampled at every grid point by TrilinearInterpolation
// (src/media/media_utility.cpp:189-283), float arithmetic in the reference's order. The volumes
// stay in file order on the device; the cut model is addressed through the file strides of its
// x, y and z samples, which reads the same values as the reference's re-ordered copy.
// -----------------------------------------------------------------------------------------
namespace cgfd {
namespace {

struct BinDev {
  int n[3];                    // samples of the cut model along x, y, z
  long long st[3];             // file strides of one sample along x, y, z
  long long off;               // file offset of the cut model's first sample
  const float *xv, *yv, *zv;   // sample coordinates of the cut model
  const float *rho, *vp, *vs;  // file-order volumes
};

__device__ __forceinline__ float lerp_rn(float a, float b, float w) { return __fadd_rn(a, __fmul_rn(w, __fsub_rn(b, a))); }

// floor / ceil sample indices of q on the axis (first sample v0, spacing d), clamped to [0, n-1]
__device__ __forceinline__ void bracket(float q, float v0, float d, int n, int &i0, int &i2) {
  const float f = __fdiv_rn(__fsub_rn(q, v0), d);
  i0 = (int)floorf(f);
  i2 = (int)ceilf(f);
  i0 = i0 < 0 ? 0 : (i0 > n - 1 ? n - 1 : i0);
  i2 = i2 < 0 ? 0 : (i2 > n - 1 ? n - 1 : i2);
}

__device__ float trilinear(const BinDev &b, const float *v, float xq, float yq, float zq) {
  int ix0, ix2, iy0, iy2, iz0, iz2;
  bracket(xq, b.xv[0], __fsub_rn(b.xv[1], b.xv[0]), b.n[0], ix0, ix2);
  bracket(yq, b.yv[0], __fsub_rn(b.yv[1], b.yv[0]), b.n[1], iy0, iy2);
  bracket(zq, b.zv[0], __fsub_rn(b.zv[1], b.zv[0]), b.n[2], iz0, iz2);
  auto at = [&](int ix, int iy, int iz) { return __ldg(v + b.off + ix * b.st[0] + iy * b.st[1] + iz * b.st[2]); };
  if (ix0 == ix2 && iy0 == iy2 && iz0 == iz2) return at(ix0, iy0, iz0);
  const float v000 = at(ix0, iy0, iz0), v002 = at(ix0, iy0, iz2), v200 = at(ix2, iy0, iz0), v202 = at(ix2, iy0, iz2);
  const float v020 = at(ix0, iy2, iz0), v022 = at(ix0, iy2, iz2), v220 = at(ix2, iy2, iz0), v222 = at(ix2, iy2, iz2);
  float v100 = v000, v102 = v002, v122 = v022, v120 = v020;
  if (ix0 != ix2) {
    const float w = __fdiv_rn(__fsub_rn(xq, b.xv[ix0]), __fsub_rn(b.xv[ix2], b.xv[ix0]));
    v100 = lerp_rn(v000, v200, w);
    v102 = lerp_rn(v002, v202, w);
    v122 = lerp_rn(v022, v222, w);
    v120 = lerp_rn(v020, v220, w);
  }
  float v110 = v100, v112 = v102;
  if (iy0 != iy2) {
    const float w = __fdiv_rn(__fsub_rn(yq, b.yv[iy0]), __fsub_rn(b.yv[iy2], b.yv[iy0]));
    v110 = lerp_rn(v100, v120, w);
    v112 = lerp_rn(v102, v122, w);
  }
  if (iz0 == iz2) return v110;
  const float w = __fdiv_rn(__fsub_rn(zq, b.zv[iz0]), __fsub_rn(b.zv[iz2], b.zv[iz0]));
  return __fadd_rn(v110, __fmul_rn(w, __fsub_rn(v112, v110)));
}

// parameterization_bin_el_iso_loc (media_bin2model.cpp:185-233): every grid point, ghosts included
__global__ void k_media_bin(const __grid_constant__ BinDev b, const __grid_constant__ GridDev g) {
  const long long n = (long long)g.nx * g.ny * g.nz;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const float xq = g.x[t], yq = g.y[t], zq = g.z[t];
    float var[3];
    var[0] = trilinear(b, b.rho, xq, yq, zq);
    var[1] = trilinear(b, b.vp, xq, yq, zq);
    var[2] = trilinear(b, b.vs, xq, yq, zq);
    float lam, mu;
    lame(var, lam, mu);
    g.mu[t] = mu;
    g.lam[t] = lam;
    g.rho[t] = var[0];
  }
}

}  // namespace
}  // namespace cgfd

extern "C" int cgfd_media_bin_el_iso_gpu(int device, int ni, int nj, int nk, const float *coord,
                                         const cgfd_bin_model *bm, float *medium) {
  using namespace cgfd;
  if (!coord || !bm || !medium || !bm->rho || !bm->vp || !bm->vs || ni < 4 || nj < 4 || nk < 4) {
    set_last_error("invalid argument");
    return CGFD_ERR_INVALID;
  }
  // the grid axis of each file dimension (bin_order): dim[a] = the file dimension of axis a
  int dim[3] = {-1, -1, -1};
  for (int d = 0; d < 3; d++) {
    const int o = bm->order[d];
    if (o < 0 || o > 2 || dim[o] != -1) {
      set_last_error("binary model: order must name x (0), y (1) and z (2) once each");
      return CGFD_ERR_INVALID;
    }
    dim[o] = d;
    if (bm->size[d] < 2) {
      set_last_error("binary model: every dimension needs at least 2 samples");
      return CGFD_ERR_INVALID;
    }
  }
  const size_t nx = ni + 6, ny = nj + 6, nz = nk + 6, n = nx * ny * nz;
  const float *X = coord, *Y = coord + n, *Z = coord + 2 * n;
  // gd_curv_set_minmax (gd_t.cu:949-970): every point, ghosts included
  float xmin = X[0], xmax = X[0], ymin = Y[0], ymax = Y[0], zmin = FLT_MAX, zmax = -FLT_MAX;
  for (size_t t = 0; t < n; t++) {
    xmin = std::min(xmin, X[t]); xmax = std::max(xmax, X[t]);
    ymin = std::min(ymin, Y[t]); ymax = std::max(ymax, Y[t]);
    zmin = std::min(zmin, Z[t]); zmax = std::max(zmax, Z[t]);
  }
  // the read range along x and y (media_bin2model.cpp:82-110), float arithmetic as there
  const float x0 = bm->origin[dim[0]], y0 = bm->origin[dim[1]], z0 = bm->origin[dim[2]];
  const float dxb = bm->spacing[dim[0]], dyb = bm->spacing[dim[1]], dzb = bm->spacing[dim[2]];
  const int sx = bm->size[dim[0]], sy = bm->size[dim[1]], sz = bm->size[dim[2]];
  const int ix_start = xmin < x0 ? 0 : (int)((xmin - x0) / dxb);
  const int iy_start = ymin < y0 ? 0 : (int)((ymin - y0) / dyb);
  const float zn = z0 + dzb * (float)(sz - 1);
  if (ix_start >= sx || xmax < x0 || iy_start >= sy || ymax < y0 || zmin >= std::max(zn, z0) ||
      zmax <= std::min(z0, zn)) {
    set_last_error("binary model: the model does not coincide with the calculation area");
    return CGFD_ERR_INVALID;
  }
  const int ix_end = std::min((int)std::ceil((xmax - x0) / dxb), sx - 1);
  const int iy_end = std::min((int)std::ceil((ymax - y0) / dyb), sy - 1);
  const int bnx = ix_end - ix_start + 1, bny = iy_end - iy_start + 1;
  if (bnx < 2 || bny < 2) {
    set_last_error("binary model: the cut model needs at least 2 samples along x and y");
    return CGFD_ERR_INVALID;
  }
  std::vector<float> xv(bnx), yv(bny), zv(sz);
  for (int q = 0; q < bnx; q++) xv[q] = x0 + (float)(ix_start + q) * dxb;
  for (int q = 0; q < bny; q++) yv[q] = y0 + (float)(iy_start + q) * dyb;
  for (int q = 0; q < sz; q++) zv[q] = z0 + (float)q * dzb;
  const long long fst[3] = {1, (long long)bm->size[0], (long long)bm->size[0] * bm->size[1]};
  const size_t nvol = (size_t)bm->size[0] * bm->size[1] * bm->size[2];

  std::vector<void *> owned;
  cudaStream_t st = nullptr;
  auto cleanup = [&] {
    for (void *q : owned) cudaFree(q);
    if (st) cudaStreamDestroy(st);
  };
  auto fail = [&](cudaError_t e, const char *what) {
    cleanup();
    set_last_error(std::string(what) + ": " + cudaGetErrorString(e));
    return e == cudaErrorMemoryAllocation ? CGFD_ERR_NOMEM : CGFD_ERR_CUDA;
  };
  auto dalloc = [&](size_t bytes, void **out) {
    cudaError_t e = cudaMalloc(out, bytes);
    if (e == cudaSuccess) owned.push_back(*out);
    return e;
  };
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) return fail(e, "cudaSetDevice");
  if ((e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking)) != cudaSuccess) return fail(e, "cudaStreamCreate");
  float *dvol = nullptr, *dvec = nullptr, *dc = nullptr, *dout = nullptr;
  if ((e = dalloc(3 * nvol * sizeof(float), (void **)&dvol)) != cudaSuccess) return fail(e, "cudaMalloc");
  if ((e = dalloc((size_t)(bnx + bny + sz) * sizeof(float), (void **)&dvec)) != cudaSuccess) return fail(e, "cudaMalloc");
  if ((e = dalloc(3 * n * sizeof(float), (void **)&dc)) != cudaSuccess) return fail(e, "cudaMalloc");
  if ((e = dalloc(3 * n * sizeof(float), (void **)&dout)) != cudaSuccess) return fail(e, "cudaMalloc");
  const float *src[3] = {bm->rho, bm->vp, bm->vs};
  for (int q = 0; q < 3 && e == cudaSuccess; q++)
    e = cudaMemcpyAsync(dvol + q * nvol, src[q], nvol * sizeof(float), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dvec, xv.data(), bnx * sizeof(float), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dvec + bnx, yv.data(), bny * sizeof(float), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dvec + bnx + bny, zv.data(), sz * sizeof(float), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dc, coord, 3 * n * sizeof(float), cudaMemcpyHostToDevice, st);
  if (e != cudaSuccess) return fail(e, "cudaMemcpy");
  BinDev b;
  b.n[0] = bnx; b.n[1] = bny; b.n[2] = sz;
  for (int a = 0; a < 3; a++) b.st[a] = fst[dim[a]];
  b.off = (long long)ix_start * b.st[0] + (long long)iy_start * b.st[1];
  b.xv = dvec; b.yv = dvec + bnx; b.zv = dvec + bnx + bny;
  b.rho = dvol; b.vp = dvol + nvol; b.vs = dvol + 2 * nvol;
  GridDev g{};
  g.nx = (int)nx; g.ny = (int)ny; g.nz = (int)nz;
  g.x = dc; g.y = dc + n; g.z = dc + 2 * n;
  g.rho = dout; g.lam = dout + n; g.mu = dout + 2 * n;  // the medium order rho, lambda, mu
  k_media_bin<<<148 * 8, 256, 0, st>>>(b, g);
  if ((e = cudaGetLastError()) != cudaSuccess) return fail(e, "media kernel");
  if ((e = cudaMemcpyAsync(medium, dout, 3 * n * sizeof(float), cudaMemcpyDeviceToHost, st)) != cudaSuccess)
    return fail(e, "cudaMemcpy");
  if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return fail(e, "cudaStreamSynchronize");
  cleanup();
  return CGFD_OK;
}

// -----------------------------------------------------------------------------------------
// Grid models (media_grid2model_el_iso, src/media/media_grid2model.cpp:133-188, the par file's
// "infile_grid"): NL layers, layer l described by ngz[l] surfaces (elevation and rho vp vs on the
// mesh, top first). A point takes the values of the surfaces above and below it, interpolated
// linearly in elevation (CalPointValue_grid, :486-957); a point within the reference's isEqual of
// a layer top takes the average of the two layers there. har / ari: where the 8 surrounding
// half-grid points fall in more than one layer (MarkLayerNumber, :1269-1355), 9^3 sub-points of
// the half-grid cell are averaged (:1819-2078), those on a layer top left out.
// -----------------------------------------------------------------------------------------
namespace cgfd {
namespace {

constexpr int kMaxGridLayers = 64;

struct GridMediaDev {
  LayerDev m;             // mesh (x0 .. dy of the cut mesh), elev [NI][ny][nx], p[0..2] rho vp vs [NI][ny][nx]
  int nl;                 // layers
  int tops[kMaxGridLayers];  // surface index of each layer's top (tops[0] = 0)
};

// last_ge over the NI surfaces with the elevations evaluated on the fly (no per-point array)
__device__ int last_ge_grid(const LayerDev &m, float value, float x, float y) {
  const size_t sl = (size_t)m.nx * m.ny;
  if (value > bilinear(m, m.elev, x, y)) return -1;
  float dist = FLT_MAX;
  int indx = -1;
  for (int i = 0; i < m.ni_; i++) {
    const float e = bilinear(m, m.elev + i * sl, x, y);
    if (e == -FLT_MAX) continue;
    const float nd = __fsub_rn(e, value);
    if (nd < 0.f) break;
    if (nd <= dist) { dist = nd; indx = i; }
  }
  return indx;
}

__device__ __forceinline__ bool is_layer_top(const GridMediaDev &g, int mi) {
  for (int l = 1; l < g.nl; l++)
    if (g.tops[l] == mi) return true;
  return false;
}

// AssignGridMediaPara2Point + CalPointValue_grid (elastic_isotropic): rho, vp, vs at a; on_inter:
// the point lies on a layer top. Returns 0, 1 outside the mesh, or 2 vp <= sqrt(2) vs.
__device__ int grid_point_value(const GridMediaDev &g, P3 a, float var[3], bool &on_inter) {
  const LayerDev &m = g.m;
  const float maxx = __fadd_rn(m.x0, __fmul_rn(m.dx, (float)(m.nx - 1)));
  const float maxy = __fadd_rn(m.y0, __fmul_rn(m.dy, (float)(m.ny - 1)));
  if (a.x < m.x0 || a.x > maxx || a.y < m.y0 || a.y > maxy) return 1;
  const size_t sl = (size_t)m.nx * m.ny;
  int mi = last_ge_grid(m, a.z, a.x, a.y);
  const float em = mi >= 0 ? bilinear(m, m.elev + mi * sl, a.x, a.y) : 0.f;
  on_inter = mi >= 0 && is_layer_top(g, mi) && (int)__fsub_rn(a.z, em) == 0;  // isEqual, integer abs
  auto val = [&](int q, int s) { return bilinear(m, m.p[q] + s * sl, a.x, a.y); };
  if (mi == -1) {
    mi = last_ge_grid(m, bilinear(m, m.elev, a.x, a.y), a.x, a.y);
    for (int q = 0; q < 3; q++) var[q] = val(q, mi);
    return 0;
  }
  if (mi == m.ni_ - 1) {
    for (int q = 0; q < 3; q++) var[q] = val(q, mi);
    return 0;
  }
  const float ep = bilinear(m, m.elev + (mi + 1) * sl, a.x, a.y);
  float dis_r = 0.5f;
  if ((double)fabsf(__fsub_rn(ep, em)) > 1e-6) dis_r = __fdiv_rn(__fsub_rn(a.z, em), __fsub_rn(ep, em));
  if (mi > 0 && (int)__fsub_rn(em, a.z) == 0 && is_layer_top(g, mi)) {
    mi--;
    dis_r = 0.5f;
  }
  for (int q = 0; q < 3; q++) {
    const float v0 = val(q, mi), v1 = val(q, mi + 1);
    var[q] = __fadd_rn(v0, __fmul_rn(__fsub_rn(v1, v0), dis_r));
  }
  if ((double)var[1] <= __dmul_rn(1.4142135623730951, (double)var[2])) return 2;
  return 0;
}

// LayerNumberAtPoint (:1269-1310): the layer whose top is the last at or above the point
__device__ int grid_layer_at(const GridMediaDev &g, float x, float y, float z) {
  const size_t sl = (size_t)g.m.nx * g.m.ny;
  float e[kMaxGridLayers];
  for (int l = 0; l < g.nl; l++) e[l] = bilinear(g.m, g.m.elev + g.tops[l] * sl, x, y);
  int mi = last_ge(z, e, g.nl);
  if (mi == -1) mi = last_ge(e[0], e, g.nl);
  return mi;
}

}  // namespace
}  // namespace cgfd

namespace cgfd {
namespace {

// parametrization_grid_el_iso_loc (:1067-1125)
__global__ void k_grid_loc(const __grid_constant__ GridMediaDev gm, const __grid_constant__ GridDev g) {
  const long long n = (long long)g.nx * g.ny * g.nz;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    float var[3];
    bool on;
    const int rc = grid_point_value(gm, P3{g.x[t], g.y[t], g.z[t]}, var, on);
    if (rc) {
      atomicOr(g.err, rc);
      continue;
    }
    float lam, mu;
    lame(var, lam, mu);
    g.mu[t] = mu;
    g.lam[t] = lam;
    g.rho[t] = var[0];
  }
}

// MarkLayerNumber, curvilinear: the layer of every half-grid point
__global__ void k_grid_mark(const __grid_constant__ GridMediaDev gm, const __grid_constant__ GridDev g) {
  const long long n = (long long)g.nx * g.ny * g.nz;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x)
    g.mat[t] = grid_layer_at(gm, g.hx[t], g.hy[t], g.hz[t]);
}

// parametrization_grid_el_iso_har / _ari (:1819-2078): sub-points on a layer top are left out
// (num_dis); har: rho arithmetic (float mean), kappa and mu harmonic; ari: rho, lambda, mu
// arithmetic (double means)
template <bool HAR>
__global__ void k_grid_avg(const __grid_constant__ GridMediaDev gm, const __grid_constant__ GridDev g) {
  const long long sl = g.nx, ss = (long long)g.nx * g.ny;
  const long long n = (long long)(g.nx - 2) * (g.ny - 2) * (g.nz - 2);
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const int i = 1 + (int)(t % (g.nx - 2)), j = 1 + (int)((t / (g.nx - 2)) % (g.ny - 2));
    const int k = 1 + (int)(t / ((long long)(g.nx - 2) * (g.ny - 2)));
    const long long indx = i + j * sl + k * ss;
    const long long c[8] = {indx - 1 - sl - ss, indx - sl - ss, indx - ss, indx - 1 - ss,
                            indx - 1 - sl,      indx - sl,      indx,      indx - 1};
    bool above = false, mixed = false;  // NumOfValues (media_utility.cpp:404-418) > 1
    for (int q = 0; q < 8; q++) {
      const int v = g.mat[c[q]];
      if (v == -1) above = true;
      if (v != g.mat[c[0]]) mixed = true;
    }
    if (above || !mixed) continue;
    P3 M[8];
    for (int q = 0; q < 8; q++) M[q] = P3{g.hx[c[q]], g.hy[c[q]], g.hz[c[q]]};
    float acc0 = 0.f, acc1 = 0.f, acc2 = 0.f;  // rho; kappa^-1 and mu^-1 (har) or lambda and mu (ari)
    int num_dis = (kSub + 1) * (kSub + 1) * (kSub + 1), bad = 0;
    auto lerp = [](P3 a, P3 b, int s) {  // a + (b - a) / ng * s, one rounding per step (Point3 operators)
      return P3{__fadd_rn(a.x, __fmul_rn(__fdiv_rn(__fsub_rn(b.x, a.x), (float)kSub), (float)s)),
                __fadd_rn(a.y, __fmul_rn(__fdiv_rn(__fsub_rn(b.y, a.y), (float)kSub), (float)s)),
                __fadd_rn(a.z, __fmul_rn(__fdiv_rn(__fsub_rn(b.z, a.z), (float)kSub), (float)s))};
    };
    for (int kk = 0; kk <= kSub; kk++)
      for (int jj = 0; jj <= kSub; jj++)
        for (int ii = 0; ii <= kSub; ii++) {
          const P3 lx00 = lerp(M[0], M[1], ii), lx10 = lerp(M[3], M[2], ii);
          const P3 lx01 = lerp(M[4], M[5], ii), lx11 = lerp(M[7], M[6], ii);
          const P3 lxy0 = lerp(lx00, lx10, jj), lxy1 = lerp(lx01, lx11, jj);
          float var[3];
          bool on = false;
          const int rc = grid_point_value(gm, lerp(lxy0, lxy1, kk), var, on);
          if (rc) { bad |= rc; continue; }
          if (on) { num_dis--; continue; }
          float lam, mu;
          lame(var, lam, mu);
          acc0 = __fadd_rn(acc0, var[0]);
          if (HAR) {
            acc1 = (float)__dadd_rn((double)acc1, __ddiv_rn(1.0, __dadd_rn((double)lam, __dmul_rn(2.0 / 3.0, (double)mu))));
            acc2 = (float)__dadd_rn((double)acc2, __ddiv_rn(1.0, (double)mu));
          } else {
            acc1 = __fadd_rn(acc1, lam);
            acc2 = __fadd_rn(acc2, mu);
          }
        }
    if (bad) { atomicOr(g.err, bad); continue; }
    if (HAR) {
      const float hmu = (float)__ddiv_rn((double)num_dis, (double)acc2);
      const float hkap = (float)__ddiv_rn((double)num_dis, (double)acc1);
      g.rho[indx] = __fdiv_rn(acc0, (float)num_dis);
      g.lam[indx] = (float)__dsub_rn((double)hkap, __dmul_rn(2.0 / 3.0, (double)hmu));
      g.mu[indx] = hmu;
    } else {
      g.lam[indx] = (float)__ddiv_rn((double)acc1, (double)num_dis);
      g.mu[indx] = (float)__ddiv_rn((double)acc2, (double)num_dis);
      g.rho[indx] = (float)__ddiv_rn((double)acc0, (double)num_dis);
    }
  }
}

}  // namespace
}  // namespace cgfd

namespace cgfd {
namespace {

// CalPointValue_grid for the VTI / TTI / Cij file types: the NPAR parameters of the surfaces
// around a, interpolated in elevation (par: [NPAR][NI][ny][nx]); on_inter as grid_point_value.
template <int NPAR>
__device__ int grid_point_params(const GridMediaDev &g, P3 a, float var[NPAR], bool &on_inter) {
  const LayerDev &m = g.m;
  const float maxx = __fadd_rn(m.x0, __fmul_rn(m.dx, (float)(m.nx - 1)));
  const float maxy = __fadd_rn(m.y0, __fmul_rn(m.dy, (float)(m.ny - 1)));
  if (a.x < m.x0 || a.x > maxx || a.y < m.y0 || a.y > maxy) return 1;
  const size_t sl = (size_t)m.nx * m.ny, ps = (size_t)m.ni_ * sl;
  int mi = last_ge_grid(m, a.z, a.x, a.y);
  const float em = mi >= 0 ? bilinear(m, m.elev + mi * sl, a.x, a.y) : 0.f;
  on_inter = mi >= 0 && is_layer_top(g, mi) && (int)__fsub_rn(a.z, em) == 0;
  auto val = [&](int q, int s) { return bilinear(m, m.par + q * ps + s * sl, a.x, a.y); };
  if (mi == -1 || mi == m.ni_ - 1) {
    if (mi == -1) mi = last_ge_grid(m, bilinear(m, m.elev, a.x, a.y), a.x, a.y);
    for (int q = 0; q < NPAR; q++) var[q] = val(q, mi);
    return 0;
  }
  const float ep = bilinear(m, m.elev + (mi + 1) * sl, a.x, a.y);
  float dis_r = 0.5f;
  if ((double)fabsf(__fsub_rn(ep, em)) > 1e-6) dis_r = __fdiv_rn(__fsub_rn(a.z, em), __fsub_rn(ep, em));
  if (mi > 0 && (int)__fsub_rn(em, a.z) == 0 && is_layer_top(g, mi)) {
    mi--;
    dis_r = 0.5f;
  }
  for (int q = 0; q < NPAR; q++) {
    const float v0 = val(q, mi), v1 = val(q, mi + 1);
    var[q] = __fadd_rn(v0, __fmul_rn(__fsub_rn(v1, v0), dis_r));
  }
  return 0;
}

// parametrization_grid_el_{vti,aniso}_loc (:1127-1267)
template <int T>
__global__ void k_grid_loc_gen(const __grid_constant__ GridMediaDev gm, const __grid_constant__ GridDev g,
                               const __grid_constant__ OutDev out) {
  constexpr int NP = LayerFile<T>::NPAR, NO = LayerFile<T>::NOUT;
  const long long n = (long long)g.nx * g.ny * g.nz;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    float var[NP], o[NO];
    bool on;
    if (grid_point_params<NP>(gm, P3{g.x[t], g.y[t], g.z[t]}, var, on)) {
      atomicOr(out.err, 1);
      continue;
    }
    para2out<T>(var, o);
    for (int q = 0; q < NO; q++) out.f[q * out.n + t] = o[q];
  }
}

// parametrization_grid_el_{vti,aniso}_{har,ari} (:2080-2793): every c_ij harmonically (double
// sum of 1/c into a float, num_dis / sum in double) or arithmetically (float sum / num_dis), rho
// arithmetically; the sub-points on a layer top left out
template <int T, bool HAR>
__global__ void k_grid_avg_gen(const __grid_constant__ GridMediaDev gm, const __grid_constant__ GridDev g,
                               const __grid_constant__ OutDev out) {
  constexpr int NP = LayerFile<T>::NPAR, NO = LayerFile<T>::NOUT;
  const long long sl = g.nx, ss = (long long)g.nx * g.ny;
  const long long n = (long long)(g.nx - 2) * (g.ny - 2) * (g.nz - 2);
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const int i = 1 + (int)(t % (g.nx - 2)), j = 1 + (int)((t / (g.nx - 2)) % (g.ny - 2));
    const int k = 1 + (int)(t / ((long long)(g.nx - 2) * (g.ny - 2)));
    const long long indx = i + j * sl + k * ss;
    const long long c[8] = {indx - 1 - sl - ss, indx - sl - ss, indx - ss, indx - 1 - ss,
                            indx - 1 - sl,      indx - sl,      indx,      indx - 1};
    bool above = false, mixed = false;
    for (int q = 0; q < 8; q++) {
      const int v = g.mat[c[q]];
      if (v == -1) above = true;
      if (v != g.mat[c[0]]) mixed = true;
    }
    if (above || !mixed) continue;
    P3 M[8];
    for (int q = 0; q < 8; q++) M[q] = P3{g.hx[c[q]], g.hy[c[q]], g.hz[c[q]]};
    float acc[NO];
    for (int q = 0; q < NO; q++) acc[q] = 0.f;
    int num_dis = (kSub + 1) * (kSub + 1) * (kSub + 1), bad = 0;
    auto lerp = [](P3 a, P3 b, int s) {
      return P3{__fadd_rn(a.x, __fmul_rn(__fdiv_rn(__fsub_rn(b.x, a.x), (float)kSub), (float)s)),
                __fadd_rn(a.y, __fmul_rn(__fdiv_rn(__fsub_rn(b.y, a.y), (float)kSub), (float)s)),
                __fadd_rn(a.z, __fmul_rn(__fdiv_rn(__fsub_rn(b.z, a.z), (float)kSub), (float)s))};
    };
    for (int kk = 0; kk <= kSub; kk++)
      for (int jj = 0; jj <= kSub; jj++)
        for (int ii = 0; ii <= kSub; ii++) {
          const P3 lx00 = lerp(M[0], M[1], ii), lx10 = lerp(M[3], M[2], ii);
          const P3 lx01 = lerp(M[4], M[5], ii), lx11 = lerp(M[7], M[6], ii);
          const P3 lxy0 = lerp(lx00, lx10, jj), lxy1 = lerp(lx01, lx11, jj);
          float var[NP], o[NO];
          bool on = false;
          if (grid_point_params<NP>(gm, lerp(lxy0, lxy1, kk), var, on)) { bad = 1; continue; }
          if (on) { num_dis--; continue; }
          para2out<T>(var, o);
          acc[0] = __fadd_rn(acc[0], o[0]);
          for (int q = 1; q < NO; q++)
            acc[q] = HAR ? (float)__dadd_rn((double)acc[q], __ddiv_rn(1.0, (double)o[q])) : __fadd_rn(acc[q], o[q]);
        }
    if (bad) { atomicOr(out.err, 1); continue; }
    out.f[indx] = __fdiv_rn(acc[0], (float)num_dis);
    for (int q = 1; q < NO; q++)
      out.f[q * out.n + indx] =
          HAR ? (float)__ddiv_rn((double)num_dis, (double)acc[q]) : __fdiv_rn(acc[q], (float)num_dis);
  }
}

// The part of the grid file's mesh read_grid_file keeps (media_read_file.cpp:774-800), float
// arithmetic as there: cut[0] elevation, cut[1 ..] the npar parameters, each [NI][cny][cnx];
// gm gets the cut mesh. A grid beyond the mesh is refused (where the reference's check lets it
// through, it reads values it never stored).
int grid_setup(const cgfd_grid_media *gmd, int npar, const float *coord, size_t n, std::vector<float> &cut,
               GridMediaDev &gm) {
  const int NL = gmd->num_layers;
  if (NL < 1 || NL > kMaxGridLayers || gmd->nx < 2 || gmd->ny < 2 || !gmd->ngz || !gmd->elevation || !gmd->param) {
    set_last_error("grid model: 1 to 64 layers on a mesh of at least 2 x 2 points are required");
    return CGFD_ERR_INVALID;
  }
  gm = GridMediaDev{};
  gm.nl = NL;
  int NI = 0;
  for (int l = 0; l < NL; l++) {
    if (gmd->ngz[l] < 1) {
      set_last_error("grid model: every layer needs at least one surface");
      return CGFD_ERR_INVALID;
    }
    gm.tops[l] = NI;
    NI += gmd->ngz[l];
  }
  const float *X = coord, *Y = coord + n;
  float xmin = X[0], xmax = X[0], ymin = Y[0], ymax = Y[0];  // gd_curv_set_minmax
  for (size_t t = 0; t < n; t++) {
    xmin = std::min(xmin, X[t]); xmax = std::max(xmax, X[t]);
    ymin = std::min(ymin, Y[t]); ymax = std::max(ymax, Y[t]);
  }
  const float MINX = gmd->x0, MINY = gmd->y0, DX = gmd->dx, DY = gmd->dy;
  if (xmin < MINX || ymin < MINY) {
    set_last_error("grid model: the given media range is smaller than the calculation grid range");
    return CGFD_ERR_INVALID;
  }
  const size_t ix0 = (size_t)((xmin - MINX) / DX), iy0 = (size_t)((ymin - MINY) / DY);
  const size_t ix1 = (size_t)std::ceil((xmax - MINX) / DX), iy1 = (size_t)std::ceil((ymax - MINY) / DY);
  if (ix1 > (size_t)gmd->nx - 1 || iy1 > (size_t)gmd->ny - 1) {
    set_last_error("grid model: the given media range is smaller than the calculation grid range");
    return CGFD_ERR_INVALID;
  }
  const size_t cnx = ix1 - ix0 + 1, cny = iy1 - iy0 + 1, csl = cnx * cny, fsl = (size_t)gmd->nx * gmd->ny;
  cut.assign((size_t)(1 + npar) * NI * csl, 0.f);
  for (int q = 0; q <= npar; q++) {
    const float *src = q == 0 ? gmd->elevation : gmd->param + (size_t)(q - 1) * NI * fsl;
    for (int sfc = 0; sfc < NI; sfc++)
      for (size_t iy = 0; iy < cny; iy++)
        for (size_t ix = 0; ix < cnx; ix++)
          cut[((size_t)q * NI + sfc) * csl + iy * cnx + ix] = src[sfc * fsl + (iy0 + iy) * gmd->nx + ix0 + ix];
  }
  gm.m.ni_ = NI; gm.m.nx = (int)cnx; gm.m.ny = (int)cny;
  gm.m.x0 = (float)ix0 * DX + MINX;
  gm.m.y0 = (float)iy0 * DY + MINY;
  gm.m.dx = DX; gm.m.dy = DY;
  return CGFD_OK;
}

}  // namespace
}  // namespace cgfd

extern "C" int cgfd_media_grid_el_iso_gpu(int device, int ni, int nj, int nk, const float *coord,
                                          const cgfd_grid_media *gmd, int method, float *medium) {
  using namespace cgfd;
  if (!coord || !gmd || !medium || !gmd->ngz || !gmd->elevation || !gmd->param || ni < 4 || nj < 4 || nk < 4 ||
      method < CGFD_MEDIA_LOC || method > CGFD_MEDIA_ARI) {
    set_last_error("invalid argument");
    return CGFD_ERR_INVALID;
  }
  if (gmd->type != CGFD_LAYER_ELASTIC_ISO) {
    set_last_error("grid model: an elastic_isotropic file is required");
    return CGFD_ERR_INVALID;
  }
  const size_t nx = ni + 6, ny = nj + 6, nz = nk + 6, n = nx * ny * nz;
  GridMediaDev gm;
  std::vector<float> cut;
  if (const int rc = grid_setup(gmd, 3, coord, n, cut, gm)) return rc;
  const int NL = gm.nl, NI = gm.m.ni_;
  const size_t csl = (size_t)gm.m.nx * gm.m.ny;

  std::vector<void *> owned;
  cudaStream_t st = nullptr;
  auto cleanup = [&] {
    for (void *q : owned) cudaFree(q);
    if (st) cudaStreamDestroy(st);
  };
  auto fail = [&](cudaError_t e, const char *what) {
    cleanup();
    set_last_error(std::string(what) + ": " + cudaGetErrorString(e));
    return e == cudaErrorMemoryAllocation ? CGFD_ERR_NOMEM : CGFD_ERR_CUDA;
  };
  auto dalloc = [&](size_t bytes, void **out) {
    cudaError_t e = cudaMalloc(out, bytes);
    if (e == cudaSuccess) owned.push_back(*out);
    return e;
  };
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) return fail(e, "cudaSetDevice");
  if ((e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking)) != cudaSuccess) return fail(e, "cudaStreamCreate");
  float *dm = nullptr, *dc = nullptr, *dout = nullptr;
  int *derr = nullptr;
  if ((e = dalloc(cut.size() * sizeof(float), (void **)&dm)) != cudaSuccess) return fail(e, "cudaMalloc");
  if ((e = dalloc(3 * n * sizeof(float), (void **)&dc)) != cudaSuccess) return fail(e, "cudaMalloc");
  if ((e = dalloc(3 * n * sizeof(float), (void **)&dout)) != cudaSuccess) return fail(e, "cudaMalloc");
  if ((e = dalloc(sizeof(int), (void **)&derr)) != cudaSuccess) return fail(e, "cudaMalloc");
  if ((e = cudaMemcpyAsync(dm, cut.data(), cut.size() * sizeof(float), cudaMemcpyHostToDevice, st)) != cudaSuccess ||
      (e = cudaMemcpyAsync(dc, coord, 3 * n * sizeof(float), cudaMemcpyHostToDevice, st)) != cudaSuccess)
    return fail(e, "cudaMemcpy");
  cudaMemsetAsync(derr, 0, sizeof(int), st);
  gm.m.elev = dm;
  for (int q = 0; q < 3; q++) gm.m.p[q] = dm + (size_t)(1 + q) * NI * csl;  // rho, vp, vs
  GridDev g{};
  g.nx = (int)nx; g.ny = (int)ny; g.nz = (int)nz;
  g.x = dc; g.y = dc + n; g.z = dc + 2 * n;
  g.rho = dout; g.lam = dout + n; g.mu = dout + 2 * n;  // the medium order rho, lambda, mu
  g.err = derr;
  k_grid_loc<<<148 * 8, 256, 0, st>>>(gm, g);
  if (method != CGFD_MEDIA_LOC && NL >= 2) {  // one layer: the local values (the reference does the same)
    float *dh = nullptr;
    int *dmat = nullptr;
    if ((e = dalloc(3 * n * sizeof(float), (void **)&dh)) != cudaSuccess) return fail(e, "cudaMalloc");
    if ((e = dalloc(n * sizeof(int), (void **)&dmat)) != cudaSuccess) return fail(e, "cudaMalloc");
    g.hx = dh; g.hy = dh + n; g.hz = dh + 2 * n;
    g.mat = dmat;
    k_half_grid<<<148 * 8, 256, 0, st>>>(g);
    k_grid_mark<<<148 * 8, 256, 0, st>>>(gm, g);
    if (method == CGFD_MEDIA_HAR) k_grid_avg<true><<<148 * 8, 128, 0, st>>>(gm, g);
    else k_grid_avg<false><<<148 * 8, 128, 0, st>>>(gm, g);
  }
  if ((e = cudaGetLastError()) != cudaSuccess) return fail(e, "media kernels");
  int herr = 0;
  if ((e = cudaMemcpyAsync(&herr, derr, sizeof(int), cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
      (e = cudaMemcpyAsync(medium, dout, 3 * n * sizeof(float), cudaMemcpyDeviceToHost, st)) != cudaSuccess)
    return fail(e, "cudaMemcpy");
  if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return fail(e, "cudaStreamSynchronize");
  cleanup();
  if (herr) {
    set_last_error((herr & 1) ? "a grid point lies outside the media grid mesh"
                              : "vp must be larger than sqrt(2) vs in every layer");
    return CGFD_ERR_INVALID;
  }
  return CGFD_OK;
}

extern "C" int cgfd_media_grid_gpu(int device, int ni, int nj, int nk, const float *coord,
                                   const cgfd_grid_media *gmd, int medium_type, int method, float *medium) {
  using namespace cgfd;
  if (!coord || !gmd || !medium || ni < 4 || nj < 4 || nk < 4 || method < CGFD_MEDIA_LOC || method > CGFD_MEDIA_ARI) {
    set_last_error("invalid argument");
    return CGFD_ERR_INVALID;
  }
  const int T = gmd->type;
  // the file types each target medium accepts (media_grid2model_el_iso / _el_vti / _el_aniso; the
  // grid reader has no TTI-Bond branch)
  const bool vti_file = T >= CGFD_LAYER_VTI_PREM && T <= CGFD_LAYER_VTI_CIJ;
  const bool ok = (medium_type == CGFD_MEDIUM_ELASTIC_ISO && T == CGFD_LAYER_ELASTIC_ISO) ||
                  (medium_type == CGFD_MEDIUM_ELASTIC_VTI && vti_file) ||
                  (medium_type == CGFD_MEDIUM_ELASTIC_ANISO &&
                   (T == CGFD_LAYER_ELASTIC_ISO || vti_file || T == CGFD_LAYER_TTI_THOMSEN || T == CGFD_LAYER_ANISO_CIJ));
  if (!ok) {
    set_last_error("grid file type not usable for this medium type");
    return CGFD_ERR_INVALID;
  }
  if (medium_type == CGFD_MEDIUM_ELASTIC_ISO) return cgfd_media_grid_el_iso_gpu(device, ni, nj, nk, coord, gmd, method, medium);
  const size_t nx = ni + 6, ny = nj + 6, nz = nk + 6, n = nx * ny * nz;
  std::vector<float> fam;
  int nfam = 0;
  if (T == CGFD_LAYER_ELASTIC_ISO) {
    fam.resize(3 * n);
    nfam = 3;
    if (const int rc = cgfd_media_grid_el_iso_gpu(device, ni, nj, nk, coord, gmd, method, fam.data())) return rc;
    return family_to_medium(fam, nfam, medium_type, n, medium);
  }
  nfam = vti_file ? 6 : 22;
  const int npar = vti_file ? 6 : (T == CGFD_LAYER_ANISO_CIJ ? 22 : 8);
  GridMediaDev gm;
  std::vector<float> cut;
  if (const int rc = grid_setup(gmd, npar, coord, n, cut, gm)) return rc;
  const size_t ps = (size_t)gm.m.ni_ * gm.m.nx * gm.m.ny;

  std::vector<void *> owned;
  cudaStream_t st = nullptr;
  auto cleanup = [&] {
    for (void *q : owned) cudaFree(q);
    if (st) cudaStreamDestroy(st);
  };
  auto fail = [&](cudaError_t e, const char *what) {
    cleanup();
    set_last_error(std::string(what) + ": " + cudaGetErrorString(e));
    return e == cudaErrorMemoryAllocation ? CGFD_ERR_NOMEM : CGFD_ERR_CUDA;
  };
  auto dalloc = [&](size_t bytes, void **out) {
    cudaError_t e = cudaMalloc(out, bytes);
    if (e == cudaSuccess) owned.push_back(*out);
    return e;
  };
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) return fail(e, "cudaSetDevice");
  if ((e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking)) != cudaSuccess) return fail(e, "cudaStreamCreate");
  float *dm = nullptr, *dc = nullptr, *dout = nullptr, *dh = nullptr;
  int *derr = nullptr, *dmat = nullptr;
  if ((e = dalloc(cut.size() * sizeof(float), (void **)&dm)) != cudaSuccess) return fail(e, "cudaMalloc");
  if ((e = dalloc(3 * n * sizeof(float), (void **)&dc)) != cudaSuccess) return fail(e, "cudaMalloc");
  if ((e = dalloc((size_t)nfam * n * sizeof(float), (void **)&dout)) != cudaSuccess) return fail(e, "cudaMalloc");
  if ((e = dalloc(sizeof(int), (void **)&derr)) != cudaSuccess) return fail(e, "cudaMalloc");
  if ((e = cudaMemcpyAsync(dm, cut.data(), cut.size() * sizeof(float), cudaMemcpyHostToDevice, st)) != cudaSuccess ||
      (e = cudaMemcpyAsync(dc, coord, 3 * n * sizeof(float), cudaMemcpyHostToDevice, st)) != cudaSuccess)
    return fail(e, "cudaMemcpy");
  cudaMemsetAsync(derr, 0, sizeof(int), st);
  gm.m.elev = dm;
  gm.m.par = dm + ps;
  GridDev g{};
  g.nx = (int)nx; g.ny = (int)ny; g.nz = (int)nz;
  g.x = dc; g.y = dc + n; g.z = dc + 2 * n;
  const bool avg = method != CGFD_MEDIA_LOC && gm.nl >= 2;
  if (avg) {
    if ((e = dalloc(3 * n * sizeof(float), (void **)&dh)) != cudaSuccess) return fail(e, "cudaMalloc");
    if ((e = dalloc(n * sizeof(int), (void **)&dmat)) != cudaSuccess) return fail(e, "cudaMalloc");
    g.hx = dh; g.hy = dh + n; g.hz = dh + 2 * n;
    g.mat = dmat;
  }
  OutDev o{(long long)n, dout, derr};
  auto run = [&](auto tag) {
    constexpr int TT = decltype(tag)::value;
    k_grid_loc_gen<TT><<<148 * 8, 256, 0, st>>>(gm, g, o);
    if (!avg) return;
    k_half_grid<<<148 * 8, 256, 0, st>>>(g);
    k_grid_mark<<<148 * 8, 256, 0, st>>>(gm, g);
    if (method == CGFD_MEDIA_HAR) k_grid_avg_gen<TT, true><<<148 * 8, 128, 0, st>>>(gm, g, o);
    else k_grid_avg_gen<TT, false><<<148 * 8, 128, 0, st>>>(gm, g, o);
  };
  switch (T) {
    case CGFD_LAYER_VTI_PREM: run(std::integral_constant<int, 22>()); break;
    case CGFD_LAYER_VTI_THOMSEN: run(std::integral_constant<int, 23>()); break;
    case CGFD_LAYER_VTI_CIJ: run(std::integral_constant<int, 24>()); break;
    case CGFD_LAYER_TTI_THOMSEN: run(std::integral_constant<int, 25>()); break;
    default: run(std::integral_constant<int, 27>()); break;
  }
  if ((e = cudaGetLastError()) != cudaSuccess) return fail(e, "media kernels");
  int herr = 0;
  fam.resize((size_t)nfam * n);
  if ((e = cudaMemcpyAsync(&herr, derr, sizeof(int), cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
      (e = cudaMemcpyAsync(fam.data(), dout, (size_t)nfam * n * sizeof(float), cudaMemcpyDeviceToHost, st)) != cudaSuccess)
    return fail(e, "cudaMemcpy");
  if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return fail(e, "cudaStreamSynchronize");
  cleanup();
  if (herr) {
    set_last_error("a grid point lies outside the media grid mesh");
    return CGFD_ERR_INVALID;
  }
  return family_to_medium(fam, nfam, medium_type, n, medium);
}

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
#include <cfloat>
#include <cuda_runtime.h>

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

struct GridDev {
  int nx, ny, nz;  // extended grid (ghosts included)
  const float *x, *y, *z;
  float *hx, *hy, *hz;  // half grid
  int *mat;             // material number at the half grid
  float *rho, *lam, *mu;
  int *err;
};

__global__ void k_media_loc(const __grid_constant__ LayerDev m, const __grid_constant__ GridDev g) {
  const long long n = (long long)g.nx * g.ny * g.nz;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
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
template <bool HAR>
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
  const size_t nx = ni + 6, ny = nj + 6, nz = nk + 6, n = nx * ny * nz;
  const size_t msz = (size_t)lm->num_interfaces * lm->nx * lm->ny;
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
  LayerDev m;
  m.ni_ = lm->num_interfaces; m.nx = lm->nx; m.ny = lm->ny;
  m.x0 = lm->x0; m.y0 = lm->y0; m.dx = lm->dx; m.dy = lm->dy;
  float *dm = nullptr;
  if ((e = dalloc(10 * msz * sizeof(float), (void **)&dm)) != cudaSuccess) return fail(e, "cudaMalloc");
  if ((e = cudaMemcpyAsync(dm, lm->elevation, msz * sizeof(float), cudaMemcpyHostToDevice, st)) != cudaSuccess)
    return fail(e, "cudaMemcpy");
  m.elev = dm;
  for (int q = 0; q < 9; q++) {
    if ((e = cudaMemcpyAsync(dm + (1 + q) * msz, hp[q], msz * sizeof(float), cudaMemcpyHostToDevice, st)) != cudaSuccess)
      return fail(e, "cudaMemcpy");
    m.p[q] = dm + (1 + q) * msz;
  }
  GridDev g;
  g.nx = (int)nx; g.ny = (int)ny; g.nz = (int)nz;
  float *dc = nullptr, *dout = nullptr;
  int *derr = nullptr;
  if ((e = dalloc(3 * n * sizeof(float), (void **)&dc)) != cudaSuccess) return fail(e, "cudaMalloc");
  if ((e = dalloc(3 * n * sizeof(float), (void **)&dout)) != cudaSuccess) return fail(e, "cudaMalloc");
  if ((e = dalloc(sizeof(int), (void **)&derr)) != cudaSuccess) return fail(e, "cudaMalloc");
  if ((e = cudaMemcpyAsync(dc, coord, 3 * n * sizeof(float), cudaMemcpyHostToDevice, st)) != cudaSuccess)
    return fail(e, "cudaMemcpy");
  cudaMemsetAsync(derr, 0, sizeof(int), st);
  g.x = dc; g.y = dc + n; g.z = dc + 2 * n;
  g.rho = dout; g.lam = dout + n; g.mu = dout + 2 * n;  // the medium order rho, lambda, mu
  g.err = derr;
  g.hx = g.hy = g.hz = nullptr;
  g.mat = nullptr;
  k_media_loc<<<148 * 8, 256, 0, st>>>(m, g);
  if (method != CGFD_MEDIA_LOC) {
    float *dh = nullptr;
    int *dmat = nullptr;
    if ((e = dalloc(3 * n * sizeof(float), (void **)&dh)) != cudaSuccess) return fail(e, "cudaMalloc");
    if ((e = dalloc(n * sizeof(int), (void **)&dmat)) != cudaSuccess) return fail(e, "cudaMalloc");
    g.hx = dh; g.hy = dh + n; g.hz = dh + 2 * n;
    g.mat = dmat;
    k_half_grid<<<148 * 8, 256, 0, st>>>(g);
    k_mark<<<148 * 8, 256, 0, st>>>(m, g);
    if (method == CGFD_MEDIA_HAR) k_media_avg<true><<<148 * 8, 128, 0, st>>>(m, g);
    else k_media_avg<false><<<148 * 8, 128, 0, st>>>(m, g);
  }
  if ((e = cudaGetLastError()) != cudaSuccess) return fail(e, "media kernels");
  int herr = 0;
  if ((e = cudaMemcpyAsync(&herr, derr, sizeof(int), cudaMemcpyDeviceToHost, st)) != cudaSuccess)
    return fail(e, "cudaMemcpy");
  if ((e = cudaMemcpyAsync(medium, dout, 3 * n * sizeof(float), cudaMemcpyDeviceToHost, st)) != cudaSuccess)
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

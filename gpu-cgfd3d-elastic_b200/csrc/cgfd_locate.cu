// cgfd_locate.cu -- sources and stations given by physical coordinates: grid index and
// fractional shift, as the reference locates them (gd_t.cu:1189-1500, 1570-1655,
// 1766-1835; src_t.cu:341-398, 952-995; io_funcs.cu:95-170, 1700-1745).
//
//   depth -> z      the top physical plane's quad containing (x, y), searched tile by tile
//                   in the reference's order, z interpolated by inverse distance (host);
//   nearest point   over every grid point, ghosts included, first minimum in memory order
//                   (device: one block row per point, 64-bit (distance, index) minimum);
//   shift           the first of the 8 cells around the nearest point that contains the
//                   point (convex-hexahedron test), then the nearest of 101^3 trilinear
//                   samples of that cell (device: one block per point).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "cgfd_b200.h"
#include "cgfd_setup.h"

namespace cgfd {
namespace {

#define LCK(call)                                                                                 \
  do {                                                                                            \
    cudaError_t e_ = (call);                                                                      \
    if (e_ != cudaSuccess) throw Error(CGFD_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

constexpr int kTiles = 4;       // GD_TILE_NX/NY/NZ (gd_t.h:9-11)
constexpr int kSamples = 100;   // samples per cell edge (gd_t.cu:1354-1360)

struct HostGrid {
  int ni, nj, nk, nx, ny, nz;
  size_t siz_iy, siz_iz, siz_icmp;
  const float *x, *y, *z;
  size_t at(int i, int j, int k) const { return (size_t)i + (size_t)j * siz_iy + (size_t)k * siz_iz; }
};

// fdlib_math_isPoint2InQuad (fdlib_math.cu:168-194): corners 0,1,3,2 walked in order
bool point_in_quad(float px, float py, const float *vx0, const float *vy0) {
  const float vx[4] = {vx0[0], vx0[1], vx0[3], vx0[2]}, vy[4] = {vy0[0], vy0[1], vy0[3], vy0[2]};
  for (int i = 0; i < 4; i++) {
    const float ex = i == 3 ? (vx[0] - vx[3]) : (vx[i + 1] - vx[i]);
    const float ey = i == 3 ? (vy[0] - vy[3]) : (vy[i + 1] - vy[i]);
    const float qx = px - vx[i], qy = py - vy[i];
    float s = ex * qy - ey * qx;
    s /= std::sqrt(ex * ex + ey * ey);
    if (s < -1e-6) return false;
  }
  return true;
}

// fdlib_math_rdinterp_2d (fdlib_math.cu:201-245), 4 points: inverse-distance weights with the
// reference's arithmetic (double reciprocals stored in float)
float idw4(float x, float y, const float *px, const float *py, const float *pv) {
  float w[4] = {0.f, 0.f, 0.f, 0.f}, tot = 0.f;
  int at_point = -1;
  for (int i = 0; i < 4; i++) {
    const float dist = std::sqrt((x - px[i]) * (x - px[i]) + (y - py[i]) * (y - py[i]));
    if (dist < 1e-9) at_point = i;
    else {
      w[i] = (float)(1.0 / dist);
      tot += w[i];
    }
  }
  if (at_point > 0) {  // the reference tests > 0 (a hit on corner 0 keeps the distance weights)
    tot = 1.0f;
    for (int i = 0; i < 4; i++) w[i] = 0.f;
    w[at_point] = 1.0f;
  }
  float v = 0.f;
  for (int i = 0; i < 4; i++) {
    w[i] = (float)(w[i] * (1.0 / tot));
    v += w[i] * pv[i];
  }
  return v;
}

// Tiles of physical points (gd_t.cu:1034-1115): average size plus the remainder spread over
// the first tiles; the x-y bounds of the top k-tile's tiles over their cells' 8 corners.
struct SurfaceTiles {
  int ts[3][kTiles], te[3][kTiles];
  float x0[kTiles][kTiles], x1[kTiles][kTiles], y0[kTiles][kTiles], y1[kTiles][kTiles];  // [j_tile][i_tile]
};

void cell_xy(const HostGrid &g, int i, int j, int k, float &x0, float &x1, float &y0, float &y1) {
  x0 = x1 = g.x[g.at(i, j, k)];
  y0 = y1 = g.y[g.at(i, j, k)];
  for (int n3 = 0; n3 < 2; n3++)
    for (int n2 = 0; n2 < 2; n2++)
      for (int n1 = 0; n1 < 2; n1++) {
        const size_t q = g.at(i + n1, j + n2, k + n3);
        x0 = x0 < g.x[q] ? x0 : g.x[q]; x1 = x1 > g.x[q] ? x1 : g.x[q];
        y0 = y0 < g.y[q] ? y0 : g.y[q]; y1 = y1 > g.y[q] ? y1 : g.y[q];
      }
}

SurfaceTiles surface_tiles(const HostGrid &g) {
  SurfaceTiles t;
  const int n[3] = {g.ni, g.nj, g.nk};
  for (int a = 0; a < 3; a++) {
    const int avg = n[a] / kTiles, left = n[a] % kTiles;
    for (int q = 0; q < kTiles; q++) {
      t.ts[a][q] = q == 0 ? 3 : t.te[a][q - 1] + 1;
      t.te[a][q] = t.ts[a][q] + avg - 1 + (q < left ? 1 : 0);
    }
  }
  const int kt = kTiles - 1;
  for (int jt = 0; jt < kTiles; jt++)
    for (int it = 0; it < kTiles; it++) {
      float tx0 = 1.0e26f, tx1 = -1.0e26f, ty0 = 1.0e26f, ty1 = -1.0e26f;
      for (int k = t.ts[2][kt]; k <= t.te[2][kt]; k++)
        for (int j = t.ts[1][jt]; j <= t.te[1][jt]; j++)
          for (int i = t.ts[0][it]; i <= t.te[0][it]; i++) {
            float a0, a1, b0, b1;
            cell_xy(g, i, j, k, a0, a1, b0, b1);
            tx0 = tx0 < a0 ? tx0 : a0; tx1 = tx1 > a1 ? tx1 : a1;
            ty0 = ty0 < b0 ? ty0 : b0; ty1 = ty1 > b1 ? ty1 : b1;
          }
      t.x0[jt][it] = tx0; t.x1[jt][it] = tx1; t.y0[jt][it] = ty0; t.y1[jt][it] = ty1;
    }
  return t;
}

// gd_curv_depth_to_axis (gd_t.cu:1393-1491): z = surface height at (x, y) - depth, the first
// top-plane quad containing (x, y) in tile order
void depth_to_axis(const HostGrid &g, const SurfaceTiles &t, float xmin, float xmax, float ymin, float ymax, float sx,
                   float sy, float *sz) {
  if (sx < xmin || sx > xmax || sy < ymin || sy > ymax) return;
  const int kt = kTiles - 1;
  for (int jt = 0; jt < kTiles; jt++)
    for (int it = 0; it < kTiles; it++) {
      if (sx < t.x0[jt][it] || sx > t.x1[jt][it] || sy < t.y0[jt][it] || sy > t.y1[jt][it]) continue;
      const int k = t.te[2][kt];
      for (int j = t.ts[1][jt]; j <= t.te[1][jt]; j++)
        for (int i = t.ts[0][it]; i <= t.te[0][it]; i++) {
          float a0, a1, b0, b1;
          cell_xy(g, i, j, k, a0, a1, b0, b1);
          if (sx < a0 || sx > a1 || sy < b0 || sy > b1) continue;
          float px[4], py[4], pz[4];
          for (int n2 = 0; n2 < 2; n2++)
            for (int n1 = 0; n1 < 2; n1++) {
              const size_t q = g.at(i + n1, j + n2, k);
              px[n1 + 2 * n2] = g.x[q];
              py[n1 + 2 * n2] = g.y[q];
              pz[n1 + 2 * n2] = g.z[q];
            }
          if (point_in_quad(sx, sy, px, py)) {
            *sz = idw4(sx, sy, px, py, pz) - *sz;
            return;
          }
        }
    }
}

// ---- device side ----------------------------------------------------------------------

__device__ __forceinline__ unsigned long long dist_key(float d, unsigned int idx) {
  return ((unsigned long long)__float_as_uint(d) << 32) | idx;  // d >= 0: bit order = value order
}

__device__ __forceinline__ unsigned long long block_min(unsigned long long v) {
  __shared__ unsigned long long red[32];
  for (int o = 16; o; o >>= 1) {
    const unsigned long long u = __shfl_xor_sync(0xffffffffu, v, o);
    v = u < v ? u : v;
  }
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x < 32) {
    v = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : ~0ull;
    for (int o = 16; o; o >>= 1) {
      const unsigned long long u = __shfl_xor_sync(0xffffffffu, v, o);
      v = u < v ? u : v;
    }
  }
  return v;
}

// nearest grid point (all points, ghosts included) of query blockIdx.y
__global__ void k_nearest(const float *__restrict__ x, const float *__restrict__ y, const float *__restrict__ z,
                          unsigned long long n, const float *__restrict__ q, unsigned long long *key) {
  const float sx = q[3 * blockIdx.y], sy = q[3 * blockIdx.y + 1], sz = q[3 * blockIdx.y + 2];
  unsigned long long best = ~0ull;
  for (unsigned long long t = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; t < n;
       t += (unsigned long long)gridDim.x * blockDim.x) {
    const float d = sqrtf((sx - x[t]) * (sx - x[t]) + (sy - y[t]) * (sy - y[t]) + (sz - z[t]) * (sz - z[t]));
    const unsigned long long k = dist_key(d, (unsigned int)t);
    best = k < best ? k : best;
  }
  best = block_min(best);
  if (threadIdx.x == 0) atomicMin(&key[blockIdx.y], best);
}

struct DevGrid {
  const float *x, *y, *z;
  int nx, ny, nz, ni1, ni2, nj1, nj2, nk1, nk2;
  unsigned long long siz_iy, siz_iz;
};

__device__ __forceinline__ float dot3(const float *a, const float *b) {
  float r = 0.0f;
  for (int i = 0; i < 3; i++) r += a[i] * b[i];
  return r;
}

// isPointInHexahedron_c (gd_t.cu:1766-1803) with face_normal (gd_t.cu:1814-1835)
__device__ bool point_in_hexahedron(float px, float py, float pz, const float *vx, const float *vy, const float *vz) {
  const float point[3] = {px, py, pz};
  const int faces[6][3] = {{0, 4, 6}, {7, 5, 1}, {5, 4, 0}, {2, 6, 7}, {4, 5, 7}, {3, 1, 0}};
  for (int f = 0; f < 6; f++) {
    float h[3][3];
    for (int c = 0; c < 3; c++) {
      h[c][0] = vx[faces[f][c]];
      h[c][1] = vy[faces[f][c]];
      h[c][2] = vz[faces[f][c]];
    }
    float p2f[3], A[3], B[3], nrm[3], un[3];
    for (int i = 0; i < 3; i++) p2f[i] = h[0][i] - point[i];
    for (int i = 0; i < 3; i++) {
      A[i] = h[1][i] - h[0][i];
      B[i] = h[2][i] - h[0][i];
    }
    nrm[0] = A[1] * B[2] - A[2] * B[1];
    nrm[1] = A[2] * B[0] - A[0] * B[2];
    nrm[2] = A[0] * B[1] - A[1] * B[0];
    const float len = sqrtf(dot3(nrm, nrm));
    for (int i = 0; i < 3; i++) un[i] = nrm[i] / len;
    float sign = dot3(p2f, un);
    const float lp = sqrtf(dot3(p2f, p2f));
    sign /= lp;
    if (sign < 0.0f) return false;
  }
  return true;
}

// shift of query blockIdx.x inside the cell that contains it (gd_t.cu:1303-1389, 1570-1655)
__global__ void k_shift(DevGrid g, const float *__restrict__ q, const unsigned long long *__restrict__ key, int *idx,
                        float *inc) {
  const int qi = blockIdx.x;
  const float sx = q[3 * qi], sy = q[3 * qi + 1], sz = q[3 * qi + 2];
  const unsigned int p = (unsigned int)(key[qi] & 0xffffffffu);
  const int mk = (int)(p / g.siz_iz), mj = (int)((p % g.siz_iz) / g.siz_iy), mi = (int)(p % g.siz_iy);
  __shared__ int cell[4];  // found, cur_i, cur_j, cur_k
  __shared__ float cx[8], cy[8], cz[8];
  if (threadIdx.x == 0) {
    cell[0] = -1;
    if (mi < g.ni1 || mi > g.ni2 || mj < g.nj1 || mj > g.nj2 || mk < g.nk1 || mk > g.nk2) {
      cell[0] = -2;  // nearest point is a ghost: not in this grid
    } else {
      for (int kk = 0; kk < 2 && cell[0] < 0; kk++)
        for (int jj = 0; jj < 2 && cell[0] < 0; jj++)
          for (int ii = 0; ii < 2 && cell[0] < 0; ii++) {
            const int ci = mi - 1 + ii, cj = mj - 1 + jj, ck = mk - 1 + kk;
            float vx[8], vy[8], vz[8];
            for (int n3 = 0; n3 < 2; n3++)
              for (int n2 = 0; n2 < 2; n2++)
                for (int n1 = 0; n1 < 2; n1++) {
                  const unsigned long long a = (ci + n1) + (cj + n2) * g.siz_iy + (ck + n3) * g.siz_iz;
                  vx[n1 + 2 * n2 + 4 * n3] = g.x[a];
                  vy[n1 + 2 * n2 + 4 * n3] = g.y[a];
                  vz[n1 + 2 * n2 + 4 * n3] = g.z[a];
                }
            if (point_in_hexahedron(sx, sy, sz, vx, vy, vz)) {
              cell[0] = 1; cell[1] = ci; cell[2] = cj; cell[3] = ck;
              for (int c = 0; c < 8; c++) { cx[c] = vx[c]; cy[c] = vy[c]; cz[c] = vz[c]; }
            }
          }
    }
  }
  __syncthreads();
  if (cell[0] == -2) {
    if (threadIdx.x == 0) {
      for (int a = 0; a < 3; a++) { idx[3 * qi + a] = -1000; inc[3 * qi + a] = 0.f; }
    }
    return;
  }
  if (cell[0] < 0) {  // in no cell around the nearest point: the reference keeps a zero shift
    if (threadIdx.x == 0) {
      idx[3 * qi] = mi - g.ni1; idx[3 * qi + 1] = mj - g.nj1; idx[3 * qi + 2] = mk - g.nk1;
      inc[3 * qi] = inc[3 * qi + 1] = inc[3 * qi + 2] = 0.f;
    }
    return;
  }
  // nearest of the (kSamples+1)^3 trilinear samples, first in (n3, n2, n1) order
  const int ns = kSamples + 1;
  unsigned long long best = ~0ull;
  for (int t = threadIdx.x; t < ns * ns * ns; t += blockDim.x) {
    const int n1 = t % ns, n2 = (t / ns) % ns, n3 = t / (ns * ns);
    float Lx[2], Ly[2], Lz[2];
    Lz[1] = (float)(n3) / (float)(kSamples);
    Lz[0] = 1.0 - Lz[1];
    Ly[1] = (float)(n2) / (float)(kSamples);
    Ly[0] = 1.0 - Ly[1];
    Lx[1] = (float)(n1) / (float)(kSamples);
    Lx[0] = 1.0 - Lx[1];
    float xp = 0, yp = 0, zp = 0;
    for (int kk = 0; kk < 2; kk++)
      for (int jj = 0; jj < 2; jj++)
        for (int ii = 0; ii < 2; ii++) {
          const int c = ii + jj * 2 + kk * 4;
          xp += Lx[ii] * Ly[jj] * Lz[kk] * cx[c];
          yp += Lx[ii] * Ly[jj] * Lz[kk] * cy[c];
          zp += Lx[ii] * Ly[jj] * Lz[kk] * cz[c];
        }
    const float d = sqrtf((sx - xp) * (sx - xp) + (sy - yp) * (sy - yp) + (sz - zp) * (sz - zp));
    const unsigned long long k = dist_key(d, (unsigned int)t);
    best = k < best ? k : best;
  }
  best = block_min(best);
  if (threadIdx.x == 0) {
    const int t = (int)(best & 0xffffffffu);
    const int n1 = t % ns, n2 = (t / ns) % ns, n3 = t / (ns * ns);
    const float si = (float)cell[1] + (float)n1 / (float)kSamples;
    const float sj = (float)cell[2] + (float)n2 / (float)kSamples;
    const float sk = (float)cell[3] + (float)n3 / (float)kSamples;
    idx[3 * qi] = mi - g.ni1; idx[3 * qi + 1] = mj - g.nj1; idx[3 * qi + 2] = mk - g.nk1;
    inc[3 * qi] = si - mi; inc[3 * qi + 1] = sj - mj; inc[3 * qi + 2] = sk - mk;
  }
}

}  // namespace

void locate_coords(const cgfd_problem_desc *d, int n, const float *xyz, const int *use_depth, Located &out) {
  out.idx.assign(3 * (size_t)n, -1000);
  out.inc.assign(3 * (size_t)n, 0.f);
  out.xyz.assign(xyz, xyz + 3 * (size_t)n);
  if (n <= 0) return;
  if (!d->coord) throw Error(CGFD_ERR_INVALID, "coord is required to locate sources/stations by coordinates");
  HostGrid g;
  g.ni = d->ni; g.nj = d->nj; g.nk = d->nk;
  g.nx = g.ni + 6; g.ny = g.nj + 6; g.nz = g.nk + 6;
  g.siz_iy = g.nx; g.siz_iz = (size_t)g.nx * g.ny; g.siz_icmp = g.siz_iz * g.nz;
  g.x = d->coord; g.y = d->coord + g.siz_icmp; g.z = d->coord + 2 * g.siz_icmp;
  // coordinate range over every point, ghosts included (gd_t.cu:952-969)
  float mn[3] = {g.x[0], g.y[0], g.z[0]}, mx[3] = {g.x[0], g.y[0], g.z[0]};
  const float *c3[3] = {g.x, g.y, g.z};
  for (int a = 0; a < 3; a++)
    for (size_t t = 0; t < g.siz_icmp; t++) {
      mn[a] = mn[a] < c3[a][t] ? mn[a] : c3[a][t];
      mx[a] = mx[a] > c3[a][t] ? mx[a] : c3[a][t];
    }
  bool any_depth = false;
  for (int q = 0; q < n; q++) any_depth |= use_depth && use_depth[q];
  if (any_depth) {
    const SurfaceTiles tiles = surface_tiles(g);
    for (int q = 0; q < n; q++)
      if (use_depth[q])
        depth_to_axis(g, tiles, mn[0], mx[0], mn[1], mx[1], out.xyz[3 * q], out.xyz[3 * q + 1], &out.xyz[3 * q + 2]);
  }
  // points inside the coordinate range go to the device
  std::vector<int> which;
  std::vector<float> qs;
  for (int q = 0; q < n; q++) {
    const float *p = &out.xyz[3 * q];
    if (p[0] < mn[0] || p[0] > mx[0] || p[1] < mn[1] || p[1] > mx[1] || p[2] < mn[2] || p[2] > mx[2]) continue;
    which.push_back(q);
    qs.insert(qs.end(), p, p + 3);
  }
  if (which.empty()) return;
  if (g.siz_icmp >= 0xffffffffull) throw Error(CGFD_ERR_UNSUPPORTED, "grid too large to locate by coordinates");
  const int m = (int)which.size();
  float *dx = nullptr, *dq = nullptr, *dinc = nullptr;
  unsigned long long *dkey = nullptr;
  int *didx = nullptr;
  auto release = [&] { cudaFree(dx); cudaFree(dq); cudaFree(dinc); cudaFree(dkey); cudaFree(didx); };
  try {
    LCK(cudaMalloc(&dx, 3 * g.siz_icmp * sizeof(float)));
    LCK(cudaMalloc(&dq, qs.size() * sizeof(float)));
    LCK(cudaMalloc(&dkey, m * sizeof(unsigned long long)));
    LCK(cudaMalloc(&didx, 3 * m * sizeof(int)));
    LCK(cudaMalloc(&dinc, 3 * m * sizeof(float)));
    LCK(cudaMemcpy(dx, d->coord, 3 * g.siz_icmp * sizeof(float), cudaMemcpyHostToDevice));
    LCK(cudaMemcpy(dq, qs.data(), qs.size() * sizeof(float), cudaMemcpyHostToDevice));
    LCK(cudaMemset(dkey, 0xff, m * sizeof(unsigned long long)));
    k_nearest<<<dim3(296, m), 256>>>(dx, dx + g.siz_icmp, dx + 2 * g.siz_icmp, g.siz_icmp, dq, dkey);
    LCK(cudaGetLastError());
    DevGrid dg{dx, dx + g.siz_icmp, dx + 2 * g.siz_icmp, g.nx, g.ny, g.nz, 3, g.ni + 2, 3, g.nj + 2, 3, g.nk + 2,
               (unsigned long long)g.siz_iy, (unsigned long long)g.siz_iz};
    k_shift<<<m, 256>>>(dg, dq, dkey, didx, dinc);
    LCK(cudaGetLastError());
    std::vector<int> hidx(3 * m);
    std::vector<float> hinc(3 * m);
    LCK(cudaMemcpy(hidx.data(), didx, hidx.size() * sizeof(int), cudaMemcpyDeviceToHost));
    LCK(cudaMemcpy(hinc.data(), dinc, hinc.size() * sizeof(float), cudaMemcpyDeviceToHost));
    for (int w = 0; w < m; w++)
      for (int a = 0; a < 3; a++) {
        out.idx[3 * which[w] + a] = hidx[3 * w + a];
        out.inc[3 * which[w] + a] = hinc[3 * w + a];
      }
  } catch (...) {
    release();
    throw;
  }
  release();
}

}  // namespace cgfd

// cgfd_grid.cu -- grid metrics in FP64 on the GPU (gd_curv_metric_cal, gd_t.cu:209-314, and the
// ghost extrapolation geometric_symmetry, gd_t.cu:404-502).
//
// The reference computes the metrics once per run on the host in FP32. Here they are computed
// in FP64 on the device from the coordinates: one thread per physical point (7-point centered
// derivatives of x, y, z along the three axes, the Jacobian as the triple product, the
// contravariant metrics as cofactors over the Jacobian), rounded to float, then the three ghost
// layers of every field by linear extrapolation, axis by axis (x, then y over all x, then z
// over all x and y, so corners follow the host order). The double arithmetic uses explicit
// round-to-nearest products and sums (no fused multiply-add), so the results equal the host
// FP64 version (cgfd_metric_calc) bitwise.
#include <cuda_runtime.h>

#include <string>

#include "cgfd_b200.h"
#include "cgfd_launch.h"
#include "cgfd_setup.h"

namespace cgfd {

// fd_t.cu:162, the centered metric operator
__constant__ double c_metric_op[7] = {-0.02084, 0.1667, -0.7709, 0.0, 0.7709, -0.1667, 0.02084};

// Metrics of the physical points from coordinates with ghosts. Both arrays use one layout:
// element (i, j, k) of field f (physical 0-based i, j, k; ghosts at -3..-1 and n..n+2) at
// f * fstride + off0 + k * sz + j * sx + i. Outputs: jac, then 9 fields xi_x .. zeta_z, written
// through out[0..9] (separate arrays, same layout).
struct MetricP {
  int ni, nj, nk;
  long long sx, sz, off0;
  const float *x, *y, *z;
  float *out[10];
};

__device__ __forceinline__ double dmad(double a, double b, double c) { return __dadd_rn(__dmul_rn(a, b), c); }

__global__ void k_metric(const __grid_constant__ MetricP q) {
  const long long n = (long long)q.ni * q.nj * q.nk;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(t % q.ni), j = (int)((t / q.ni) % q.nj), k = (int)(t / ((long long)q.ni * q.nj));
    const long long p = q.off0 + (long long)k * q.sz + (long long)j * q.sx + i;
    const long long sh[3] = {1, q.sx, q.sz};
    double v[3][3];  // v[axis][xyz]
#pragma unroll
    for (int a = 0; a < 3; a++) {
      double sx = 0.0, sy = 0.0, sz = 0.0;
#pragma unroll
      for (int m = 0; m < 7; m++) {
        const long long r = p + (long long)(m - 3) * sh[a];
        sx = dmad(c_metric_op[m], (double)q.x[r], sx);
        sy = dmad(c_metric_op[m], (double)q.y[r], sy);
        sz = dmad(c_metric_op[m], (double)q.z[r], sz);
      }
      v[a][0] = sx; v[a][1] = sy; v[a][2] = sz;
    }
    auto cross = [](const double *a, const double *b, double *o) {
      o[0] = __dsub_rn(__dmul_rn(a[1], b[2]), __dmul_rn(a[2], b[1]));
      o[1] = __dsub_rn(__dmul_rn(a[2], b[0]), __dmul_rn(a[0], b[2]));
      o[2] = __dsub_rn(__dmul_rn(a[0], b[1]), __dmul_rn(a[1], b[0]));
    };
    double g1[3], g2[3], g3[3];
    cross(v[0], v[1], g3);
    const double jac = __dadd_rn(__dadd_rn(__dmul_rn(g3[0], v[2][0]), __dmul_rn(g3[1], v[2][1])), __dmul_rn(g3[2], v[2][2]));
    cross(v[1], v[2], g1);
    cross(v[2], v[0], g2);
    q.out[0][p] = (float)jac;
#pragma unroll
    for (int b = 0; b < 3; b++) {
      q.out[1 + b][p] = (float)__ddiv_rn(g1[b], jac);
      q.out[4 + b][p] = (float)__ddiv_rn(g2[b], jac);
      q.out[7 + b][p] = (float)__ddiv_rn(g3[b], jac);
    }
  }
}

// Ghost layers of one field along `axis` by v(ghost) = 2 v(edge) - v(mirror), over the full
// extent (ghosts included) of the other two axes (geometric_symmetry, gd_t.cu:404-502).
__global__ void k_ghost_axis(float *v, int ni, int nj, int nk, long long sx, long long sz, long long off0, int axis) {
  const int n[3] = {ni, nj, nk};
  const int e0 = n[(axis + 1) % 3] + 6, e1 = n[(axis + 2) % 3] + 6;
  const long long total = 6LL * e0 * e1;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    const int g = (int)(t % 6);  // ghost layer: 0-2 low side (-3..-1), 3-5 high side (n..n+2)
    const int a = (int)((t / 6) % e0) - 3, b = (int)(t / (6LL * e0)) - 3;
    const int na = n[axis];
    const int gi = g < 3 ? g - 3 : na + (g - 3);
    const int edge = g < 3 ? 0 : na - 1;
    const int mir = 2 * edge - gi;
    int c[3];
    c[(axis + 1) % 3] = a;
    c[(axis + 2) % 3] = b;
    auto at = [&](int s) {
      c[axis] = s;
      return off0 + (long long)c[2] * sz + (long long)c[1] * sx + c[0];
    };
    const float ve = v[at(edge)], vm = v[at(mir)];
    v[at(gi)] = 2 * ve - vm;
  }
}

void launch_metric(const float *x, const float *y, const float *z, float *const out[10], int ni, int nj, int nk,
                   long long sx, long long sz, long long off0, cudaStream_t st) {
  MetricP q;
  q.ni = ni; q.nj = nj; q.nk = nk; q.sx = sx; q.sz = sz; q.off0 = off0;
  q.x = x; q.y = y; q.z = z;
  for (int f = 0; f < 10; f++) q.out[f] = out[f];
  k_metric<<<148 * 8, 256, 0, st>>>(q);
  // axis order x, y, z: each pass reads the edge and mirror points the previous passes filled
  for (int axis = 0; axis < 3; axis++)
    for (int f = 0; f < 10; f++) k_ghost_axis<<<148 * 4, 256, 0, st>>>(out[f], ni, nj, nk, sx, sz, off0, axis);
}

}  // namespace cgfd

extern "C" int cgfd_metric_calc_gpu(int device, int ni, int nj, int nk, const float *coord, float *metric) {
  if (!coord || !metric || ni < 4 || nj < 4 || nk < 4) {
    cgfd::set_last_error("invalid argument");
    return CGFD_ERR_INVALID;
  }
  cgfd::RefGrid g(ni, nj, nk);
  const size_t siz = g.siz_icmp;
  float *dc = nullptr, *dm = nullptr;
  cudaStream_t st = nullptr;
  auto fail = [&](cudaError_t e, const char *what) {
    if (dc) cudaFree(dc);
    if (dm) cudaFree(dm);
    if (st) cudaStreamDestroy(st);
    cgfd::set_last_error(std::string(what) + ": " + cudaGetErrorString(e));
    return e == cudaErrorMemoryAllocation ? CGFD_ERR_NOMEM : CGFD_ERR_CUDA;
  };
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) return fail(e, "cudaSetDevice");
  if ((e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking)) != cudaSuccess) return fail(e, "cudaStreamCreate");
  if ((e = cudaMalloc(&dc, 3 * siz * sizeof(float))) != cudaSuccess) return fail(e, "cudaMalloc");
  if ((e = cudaMalloc(&dm, 10 * siz * sizeof(float))) != cudaSuccess) return fail(e, "cudaMalloc");
  if ((e = cudaMemcpyAsync(dc, coord, 3 * siz * sizeof(float), cudaMemcpyHostToDevice, st)) != cudaSuccess)
    return fail(e, "cudaMemcpy");
  if ((e = cudaMemsetAsync(dm, 0, 10 * siz * sizeof(float), st)) != cudaSuccess) return fail(e, "cudaMemset");
  // the reference layout is the device layout with sx = nx, sz = nx ny and the origin at (3,3,3)
  const long long sx = g.nx, sz = (long long)g.nx * g.ny, off0 = 3 + 3 * sx + 3 * sz;
  float *out[10];
  for (int f = 0; f < 10; f++) out[f] = dm + f * siz;
  cgfd::launch_metric(dc, dc + siz, dc + 2 * siz, out, ni, nj, nk, sx, sz, off0, st);
  if ((e = cudaGetLastError()) != cudaSuccess) return fail(e, "metric kernels");
  if ((e = cudaMemcpyAsync(metric, dm, 10 * siz * sizeof(float), cudaMemcpyDeviceToHost, st)) != cudaSuccess)
    return fail(e, "cudaMemcpy");
  if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return fail(e, "cudaStreamSynchronize");
  cudaFree(dc);
  cudaFree(dm);
  cudaStreamDestroy(st);
  return CGFD_OK;
}

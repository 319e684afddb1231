// cgfd_visco.cu -- visco-elastic media (generalized Maxwell body, nmax relaxation mechanisms).
//
// A stage of a visco-elastic medium runs the elastic iso kernels in their right-hand-side mode
// (the bulk planes and the surface slab write the 9-field right-hand side, CFS-PML and the free
// surface included, to one array), then k_vis_atten below: per physical point the strain rate
// recovered from the stress right-hand side, the memory-variable right-hand side
// wl_n (strain rate - J_n), the anelastic stress sum_n (lambda Ylam_n tr J_n + 2 mu Ymu_n J_n)
// taken off the stress right-hand side, and the RK combine of the 9 wave fields and the 6 nmax
// memory variables. Sources are added afterwards, as for elastic media. After the last stage,
// k_vis_free rotates the surface stress of w_end into the local frame, zeroes its normal part and
// rotates it back.
//
// Reference: sv_curv_col_vis_iso_gpu.cu (onestage :21-283, atten :285-433, free :435-531),
// drv_rk_curv_col.cu:317-331 and :479-490.
#include <cuda_runtime.h>

#include "cgfd_dev.cuh"
#include "cgfd_launch.h"

namespace cgfd {

// Stress rows of the wave fields (components 3..8): xx yy zz yz xz xy. One thread per physical
// point: x from the block's x index, one block row per (j, k); NM mechanisms unrolled so that
// every load of a point is issued before its arithmetic.
template <int NM>
__global__ void __launch_bounds__(128) k_vis_atten(const __grid_constant__ VisP q) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= q.ni) return;
  const int j = blockIdx.y, k = blockIdx.z;
  const long long sf = q.sf;
  {
    const long long id = q.off0 + (long long)k * q.sz + (long long)j * q.sx + i;
    float h[9];
#pragma unroll
    for (int f = 0; f < 9; f++) h[f] = q.rhs[f * sf + id];
    const float lam = __ldg(q.coef + (long long)CF_MED * sf + id);
    const float mu = __ldg(q.coef + (long long)(CF_MED + 1) * sf + id);
    // strain rate from the stress rate (isotropic compliance); the diagonal in double, as the
    // reference's double literals make it
    const float tr = (h[3] + h[4] + h[5]) / (3.f * lam + 2.f * mu);
    float ev[6];
    ev[0] = (float)(((2.0 * h[3] - h[4] - h[5]) / (double)(2.f * mu) + tr) / 3.0);
    ev[1] = (float)(((2.0 * h[4] - h[3] - h[5]) / (double)(2.f * mu) + tr) / 3.0);
    ev[2] = (float)(((2.0 * h[5] - h[3] - h[4]) / (double)(2.f * mu) + tr) / 3.0);
    ev[3] = (float)((double)(h[6] / mu) * 0.5);
    ev[4] = (float)((double)(h[7] / mu) * 0.5);
    ev[5] = (float)((double)(h[8] / mu) * 0.5);
    float sl = 0.f, sm[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
#pragma unroll
    for (int m = 0; m < NM; m++) {
      const float ylam = __ldg(q.y + (long long)m * sf + id);
      const float ymu = __ldg(q.y + (long long)(NM + m) * sf + id);
      float jc[6], hj[6];
#pragma unroll
      for (int c = 0; c < 6; c++) jc[c] = q.jcur[(long long)(6 * m + c) * sf + id];
#pragma unroll
      for (int c = 0; c < 6; c++) hj[c] = q.wl[m] * (ev[c] - jc[c]);
      sl += ylam * (jc[0] + jc[1] + jc[2]);
#pragma unroll
      for (int c = 0; c < 6; c++) sm[c] += ymu * jc[c];
      // RK combine of the memory variables
#pragma unroll
      for (int c = 0; c < 6; c++) {
        const long long o = (long long)(6 * m + c) * sf + id;
        if (q.stage == 0) {
          q.jtmp[o] = jc[c] + q.ca * hj[c];
          q.jend[o] = jc[c] + q.cb * hj[c];
        } else if (q.stage < 3) {
          q.jtmp[o] = q.jpre[o] + q.ca * hj[c];
          q.jend[o] = q.jend[o] + q.cb * hj[c];
        } else {
          q.jend[o] = q.jend[o] + q.cb * hj[c];
        }
      }
    }
    const float ls = lam * sl;
    const double mu2 = 2.0 * (double)mu;
#pragma unroll
    for (int c = 0; c < 3; c++) h[3 + c] -= (float)((double)ls + mu2 * (double)sm[c]);
#pragma unroll
    for (int c = 3; c < 6; c++) h[3 + c] -= (float)(mu2 * (double)sm[c]);
    // RK combine of the wave fields
    if (q.stage == 0) {
#pragma unroll
      for (int f = 0; f < 9; f++) {
        const float c0 = q.cur[f * sf + id];
        q.tmp_out[f * sf + id] = c0 + q.ca * h[f];
        q.end[f * sf + id] = c0 + q.cb * h[f];
      }
    } else if (q.stage < 3) {
#pragma unroll
      for (int f = 0; f < 9; f++) {
        q.tmp_out[f * sf + id] = __ldg(q.pre + f * sf + id) + q.ca * h[f];
        q.end[f * sf + id] = q.end[f * sf + id] + q.cb * h[f];
      }
    } else {
      bool bad = false;
#pragma unroll
      for (int f = 0; f < 9; f++) {
        const float e = q.end[f * sf + id] + q.cb * h[f];
        q.end[f * sf + id] = e;
        bad |= nonfinite(e);
      }
      if (bad && q.err) atomicOr(q.err, kErrWaveNonfinite);
    }
  }
}

__global__ void __launch_bounds__(256) k_vis_free(const __grid_constant__ VisFreeP q) {
  const long long n = (long long)q.ni * q.nj;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(t % q.ni), j = (int)(t / q.ni);
    const long long id = q.off_top + (long long)j * q.sx + i;
    float D[3][3];
#pragma unroll
    for (int a = 0; a < 9; a++) D[a / 3][a % 3] = __ldg(q.matD + t * 9 + a);
    float *w = q.w_end;
    const long long sf = q.sf;
    const float txx = w[3 * sf + id], tyy = w[4 * sf + id], tzz = w[5 * sf + id];
    const float tyz = w[6 * sf + id], txz = w[7 * sf + id], txy = w[8 * sf + id];
    // the stress in the local frame: only the tangential block (rows 0-1) is kept
    float L[2][2];
    L[0][0] = D[0][0] * D[0][0] * txx + D[0][1] * D[0][1] * tyy + D[0][2] * D[0][2] * tzz +
              2.f * (D[0][0] * D[0][1] * txy + D[0][0] * D[0][2] * txz + D[0][1] * D[0][2] * tyz);
    L[0][1] = D[0][0] * D[1][0] * txx + D[0][1] * D[1][1] * tyy + D[0][2] * D[1][2] * tzz +
              (D[0][0] * D[1][1] + D[0][1] * D[1][0]) * txy + (D[0][0] * D[1][2] + D[1][0] * D[0][2]) * txz +
              (D[0][1] * D[1][2] + D[1][1] * D[0][2]) * tyz;
    L[1][1] = D[1][0] * D[1][0] * txx + D[1][1] * D[1][1] * tyy + D[1][2] * D[1][2] * tzz +
              2.f * (D[1][0] * D[1][1] * txy + D[1][0] * D[1][2] * txz + D[1][1] * D[1][2] * tyz);
    L[1][0] = L[0][1];
    // back to the grid frame: D^T L D
    float DL[3][2];
#pragma unroll
    for (int a = 0; a < 3; a++)
#pragma unroll
      for (int d = 0; d < 2; d++) DL[a][d] = D[0][a] * L[0][d] + D[1][a] * L[1][d];
    auto g = [&](int a, int b) { return DL[a][0] * D[0][b] + DL[a][1] * D[1][b]; };
    w[3 * sf + id] = g(0, 0);
    w[4 * sf + id] = g(1, 1);
    w[5 * sf + id] = g(2, 2);
    w[6 * sf + id] = g(1, 2);
    w[7 * sf + id] = g(0, 2);
    w[8 * sf + id] = g(0, 1);
  }
}

static unsigned grid_for(long long n) {
  long long b = (n + 255) / 256;
  return (unsigned)std::max(1LL, std::min(b, 148LL * 16));
}

int launch_vis_atten(const VisP &q, cudaStream_t st) {
  const dim3 grid((q.ni + 127) / 128, q.nj, q.nk);
  switch (q.nmax) {
    case 1: k_vis_atten<1><<<grid, 128, 0, st>>>(q); break;
    case 2: k_vis_atten<2><<<grid, 128, 0, st>>>(q); break;
    case 3: k_vis_atten<3><<<grid, 128, 0, st>>>(q); break;
    case 4: k_vis_atten<4><<<grid, 128, 0, st>>>(q); break;
    case 5: k_vis_atten<5><<<grid, 128, 0, st>>>(q); break;
    case 6: k_vis_atten<6><<<grid, 128, 0, st>>>(q); break;
    case 7: k_vis_atten<7><<<grid, 128, 0, st>>>(q); break;
    case 8: k_vis_atten<8><<<grid, 128, 0, st>>>(q); break;
    case 9: k_vis_atten<9><<<grid, 128, 0, st>>>(q); break;
    default: k_vis_atten<10><<<grid, 128, 0, st>>>(q); break;
  }
  return 1;
}

int launch_vis_free(const VisFreeP &q, cudaStream_t st) {
  k_vis_free<<<grid_for((long long)q.ni * q.nj), 256, 0, st>>>(q);
  return 1;
}

}  // namespace cgfd

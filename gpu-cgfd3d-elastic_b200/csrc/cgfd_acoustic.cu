// cgfd_acoustic.cu -- acoustic RK stage of the CGFD3D path for sm_100a
// (sv_curv_col_ac_iso_gpu.cu: fields Vx Vy Vz P, P stored in the Txx slot as wav_ac_init
// does, wav_t.cu:190-250; medium 1/rho and kappa).
//
// k_ac_image: the pressure image of the free surface, in place on the stage input before the
//   stage (sv_curv_col_ac_iso_rhs_timg_z2_gpu, sv_curv_col_ac_iso_gpu.cu:376-410): P = 0 on the
//   top plane, P of the 3 ghost planes above = -P of the planes mirrored below it.
// k_stage_ac: every cell of the grid in one launch: the inner RHS (:277-366), the low-order
//   pressure rows of the top 3 planes (vlow, :413-521), the CFS-PML corrections and auxiliary
//   updates of every face (:579-802) and the RK combine of wavefield and auxiliaries
//   (wav_update / wav_update_end, wav_t.cu:362-378), the RHS kept in registers. A block owns a
//   TX x TY column tile and marches along z: the x-y tile of the current plane with its operator
//   halo in shared memory (double-buffered, one barrier per plane), the 5 planes of the z
//   operator in a per-thread register queue. 4 fields: 16 B of wavefield per cell.
#include <algorithm>

#include "cgfd_dev.cuh"
#include "cgfd_launch.h"

namespace cgfd {

constexpr int kAcF = 4;  // Vx Vy Vz P
constexpr int kAcP = 3;  // field index of P (the Txx slot)

// Pressure image of the top plane for every (i, j, shot). end_ghost (stage 0 only, may be
// null): the end level, whose ghost planes the reference's whole-level RK combine fills with
// the stage-0 input's ghost values (end = pre + b * rhs, rhs = 0 there).
template <typename R>
__global__ void k_ac_image(R *cur, R *end_ghost, int ni, int nj, int nk, long long sx, long long sz, long long sf,
                           long long off0) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= ni || j >= nj) return;
  const long long fP = ((long long)blockIdx.z * 9 + kAcP) * sf;
  const long long top = fP + off0 + (long long)(nk - 1) * sz + (long long)j * sx + i;
  cur[top] = R(0);
#pragma unroll
  for (int g = 1; g <= 3; g++) {
    const R v = -cur[top - g * sz];
    cur[top + g * sz] = v;
    if (end_ghost) end_ghost[top + g * sz] = v;
  }
}

// CFS-PML work of one face for one acoustic cell (sv_curv_col_ac_iso_gpu.cu:647-802): the 1-D
// terms of this axis rhs_d; h += (B-1) rhs_d - B aux; aux' = D rhs_d - A aux; RK combine of the
// 4 auxiliary variables (component stride n, shot stride 9 n as for the elastic faces).
template <typename R>
__device__ __forceinline__ void ac_pml_face(const StagePT<R> &p, const FacePT<R> &f, int i, int j, int k, int shot,
                                            R slw, R kappa, const R m[3], const R dv[3], R dp, R hc[kAcF]) {
  const int ab = f.axis == 0 ? i - f.lo[0] : (f.axis == 1 ? j - f.lo[1] : k - f.lo[2]);
  const R cA = __ldg(f.A + ab), cB = __ldg(f.B + ab), cD = __ldg(f.D + ab);
  const R cB1 = cB - R(1);
  const long long ia =
      (long long)shot * 9 * f.n + ((long long)(k - f.lo[2]) * f.ny + (j - f.lo[1])) * f.nx + (i - f.lo[0]);
  R rhs[kAcF];
  rhs[0] = -slw * (m[0] * dp);
  rhs[1] = -slw * (m[1] * dp);
  rhs[2] = -slw * (m[2] * dp);
  rhs[3] = -kappa * (m[0] * dv[0] + m[1] * dv[1] + m[2] * dv[2]);
  R aux[kAcF], arhs[kAcF];
#pragma unroll
  for (int c = 0; c < kAcF; c++) {
    aux[c] = f.aux_cur[c * f.n + ia];
    hc[c] += cB1 * rhs[c] - cB * aux[c];
    arhs[c] = cD * rhs[c] - cA * aux[c];
  }
  rk_store<kAcF>(p.stage, p.ca, p.cb, f.n, ia, aux, arhs, f.aux_pre, f.aux_tmp, f.aux_end);
}

template <typename R>
struct AcTile {
  static constexpr int SW = TX + 4, SH = TY + 4;
  static constexpr int MINB = sizeof(R) == 8 ? 1 : 2;
};

template <int DX, int DY, int DZ, typename R>
__global__ void __launch_bounds__(TX *TY, AcTile<R>::MINB)
    k_stage_ac(const __grid_constant__ StagePT<R> p, int nzc, int nchunk) {
  constexpr int LX = op_left(DX), LY = op_left(DY), LZ = op_left(DZ);
  constexpr int SW = AcTile<R>::SW, SH = AcTile<R>::SH;
  __shared__ R s[2][kAcF][SH][SW];

  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
  const int bx = blockIdx.x, by = blockIdx.y;
  const int i = bx * TX + tx, j = by * TY + ty;
  const bool act = (i < p.ni) && (j < p.nj);
  const long long sf = p.sf;
  const R *__restrict__ p_coef = static_cast<const R *>(p.coef);  // FP32 (FP64 build: double) coefficients

  // halo slot of this thread (x halo: 4 columns per tile row, y halo: 4 rows per tile column)
  int h_i = 0, h_j = 0, h_sx = 0, h_sy = 0;
  bool h_on = false;
  if (tid < 4 * TY) {
    const int row = tid >> 2, hh = tid & 3;
    h_j = by * TY + row;
    h_sy = row + LY;
    if (hh < LX) { h_i = bx * TX - LX + hh; h_sx = hh; }
    else { h_i = bx * TX + TX + (hh - LX); h_sx = TX + hh; }
    h_on = true;
  } else if (tid < 4 * TY + 4 * TX) {
    const int q = tid - 4 * TY;
    const int col = q % TX, hh = q / TX;
    h_i = bx * TX + col;
    h_sx = col + LX;
    h_j = hh < LY ? by * TY - LY + hh : by * TY + TY + (hh - LY);
    h_sy = LY + (h_j - by * TY);
    h_on = true;
  }
  // points beyond the 3 ghost layers are never needed; they read as 0 without a load
  const bool h_ld = h_on && h_i <= p.ni + 2 && h_j <= p.nj + 2;

  for (int bz = blockIdx.z; bz < nchunk * p.nshot; bz += gridDim.z) {
    const int shot = bz / nchunk, kb = (bz % nchunk) * nzc;
    const int ke = min(kb + nzc, p.nk);
    const long long woff = (long long)shot * 9 * sf;
    const R *__restrict__ cur = p.cur + woff;
    R *tmp_out = p.tmp_out ? p.tmp_out + woff : nullptr;

    const R *__restrict__ pre = p.pre + woff;
    R *end = p.end + woff;

    // z register queue: q[f][n] holds plane k - LZ + n
    R q[kAcF][5];
#pragma unroll
    for (int f = 0; f < kAcF; f++)
#pragma unroll
      for (int n = 0; n < 5; n++) q[f][n] = R(0);
    if (act) {
#pragma unroll
      for (int n = 0; n < 4; n++) {
        const long long id = didx(p, i, j, kb - LZ + n);
#pragma unroll
        for (int f = 0; f < kAcF; f++) q[f][n] = __ldg(cur + f * sf + id);
      }
    }
    // Loads of a plane are issued one plane ahead (the barrier and the arithmetic of the current
    // plane cover their latency): the top of the z queue, this thread's halo value, the 11
    // coefficients and the RK levels the combine reads.
    R nq[kAcF], nh[kAcF], ncf[11], npr[kAcF], nen[kAcF];
    auto fetch = [&](int kk) {
      if (act) {
        const long long iq = didx(p, i, j, kk + 4 - LZ), id = didx(p, i, j, kk);
#pragma unroll
        for (int f = 0; f < kAcF; f++) nq[f] = __ldg(cur + f * sf + iq);
#pragma unroll
        for (int c = 0; c < 11; c++) ncf[c] = __ldg(p_coef + c * sf + id);
        if (p.stage == 1 || p.stage == 2) {
#pragma unroll
          for (int f = 0; f < kAcF; f++) npr[f] = __ldg(pre + f * sf + id);
        }
        if (p.stage >= 1) {  // end is read and written by this thread only
#pragma unroll
          for (int f = 0; f < kAcF; f++) nen[f] = end[f * sf + id];
        }
      }
      if (h_on) {
        const long long id = h_ld ? didx(p, h_i, h_j, kk) : 0;
#pragma unroll
        for (int f = 0; f < kAcF; f++) nh[f] = h_ld ? __ldg(cur + f * sf + id) : R(0);
      }
    };
#pragma unroll
    for (int f = 0; f < kAcF; f++) { nq[f] = nh[f] = npr[f] = nen[f] = R(0); }
#pragma unroll
    for (int c = 0; c < 11; c++) ncf[c] = R(0);
    fetch(kb);

    for (int k = kb; k < ke; k++) {
      const int buf = k & 1;
      R cf[11], pr[kAcF], en[kAcF];
#pragma unroll
      for (int f = 0; f < kAcF; f++) {
        q[f][4] = nq[f];
        pr[f] = npr[f];
        en[f] = nen[f];
        s[buf][f][ty + LY][tx + LX] = q[f][LZ];
        if (h_on) s[buf][f][h_sy][h_sx] = nh[f];
      }
#pragma unroll
      for (int c = 0; c < 11; c++) cf[c] = ncf[c];
      if (k + 1 < ke) fetch(k + 1);
      __syncthreads();

      if (act) {
        const long long id = didx(p, i, j, k);
        R m[3][3];
#pragma unroll
        for (int a = 0; a < 3; a++)
#pragma unroll
          for (int b = 0; b < 3; b++) m[a][b] = cf[3 * a + b];
        const R slw = cf[CF_SLW], kappa = cf[CF_MED];
        // derivatives along x, y, z of Vx Vy Vz (dv[axis][comp]) and of P (dp[axis])
        R dv[3][3], dp[3];
#pragma unroll
        for (int f = 0; f < kAcF; f++) {
          const R *r = &s[buf][f][ty + LY][tx];
          const R dx = drp5<DX>(r[0], r[1], r[2], r[3], r[4]);
          const R dy = drp5<DY>(s[buf][f][ty][tx + LX], s[buf][f][ty + 1][tx + LX], s[buf][f][ty + 2][tx + LX],
                                s[buf][f][ty + 3][tx + LX], s[buf][f][ty + 4][tx + LX]);
          const R dz = drp5<DZ>(q[f][0], q[f][1], q[f][2], q[f][3], q[f][4]);
          if (f < 3) { dv[0][f] = dx; dv[1][f] = dy; dv[2][f] = dz; }
          else { dp[0] = dx; dp[1] = dy; dp[2] = dz; }
        }
        R h[kAcF];
        // moment equation (:351-354)
#pragma unroll
        for (int c = 0; c < 3; c++) h[c] = -slw * (m[0][c] * dp[0] + m[1][c] * dp[1] + m[2][c] * dp[2]);
        // Hooke (:357-359); on the top 3 planes of a free surface the velocity z-derivative is
        // of 2nd (second plane) or 4th order (third plane), and the top plane's value is 0
        // (vlow, :459-518, with the one-sided operators of fd_t.cu:82-89, 103-110)
        R dvz[3] = {dv[2][0], dv[2][1], dv[2][2]};
        const int nl = p.free_top ? p.nk - 1 - k : 3;
        if (nl == 1) {
#pragma unroll
          for (int c = 0; c < 3; c++) {
            if constexpr (DZ) dvz[c] = -q[c][1] + q[c][2];  // planes k, k+1 (LZ = 1)
            else dvz[c] = -q[c][2] + q[c][3];               // planes k-1, k (LZ = 3)
          }
        } else if (nl == 2) {
#pragma unroll
          for (int c = 0; c < 3; c++) {
            if constexpr (DZ)
              dvz[c] = R(-7.0f / 6.0f) * q[c][1] + R(8.0f / 6.0f) * q[c][2] - R(1.0f / 6.0f) * q[c][3];
            else
              dvz[c] = R(1.0f / 6.0f) * q[c][1] - R(8.0f / 6.0f) * q[c][2] + R(7.0f / 6.0f) * q[c][3];
          }
        }
        h[kAcP] = nl == 0 ? R(0)
                          : -kappa * (m[0][0] * dv[0][0] + m[1][0] * dv[1][0] + m[2][0] * dvz[0] +
                                      m[0][1] * dv[0][1] + m[1][1] * dv[1][1] + m[2][1] * dvz[1] +
                                      m[0][2] * dv[0][2] + m[1][2] * dv[1][2] + m[2][2] * dvz[2]);
        // CFS-PML of every face the cell lies in (full-order derivatives of the face's axis)
        R hc[kAcF] = {R(0), R(0), R(0), R(0)};
        for (int fi = 0; fi < p.nface; fi++) {
          const FacePT<R> &fc = p.face[fi];
          if (in_face(fc, i, j, k)) ac_pml_face(p, fc, i, j, k, shot, slw, kappa, m[fc.axis], dv[fc.axis], dp[fc.axis], hc);
        }
#pragma unroll
        for (int c = 0; c < kAcF; c++) h[c] += hc[c];
        // RK combine (rk_store's arithmetic on the prefetched levels)
        if (p.stage == 0) {
#pragma unroll
          for (int f = 0; f < kAcF; f++) {
            tmp_out[f * sf + id] = q[f][LZ] + p.ca * h[f];
            end[f * sf + id] = q[f][LZ] + p.cb * h[f];
          }
        } else if (p.stage < 3) {
#pragma unroll
          for (int f = 0; f < kAcF; f++) {
            tmp_out[f * sf + id] = pr[f] + p.ca * h[f];
            end[f * sf + id] = en[f] + p.cb * h[f];
          }
        } else {
          bool bad = false;
#pragma unroll
          for (int f = 0; f < kAcF; f++) {
            const R v = en[f] + p.cb * h[f];
            end[f * sf + id] = v;
            bad |= nonfinite(v);
          }
          if (bad) atomicOr(p.err, kErrWaveNonfinite);
        }
      }
#pragma unroll
      for (int f = 0; f < kAcF; f++)
#pragma unroll
        for (int n = 0; n < 4; n++) q[f][n] = q[f][n + 1];
    }
    __syncthreads();  // the next chunk's first plane reuses buffer kb & 1
  }
}

template <typename R>
int launch_ac_image(const StagePT<R> &p, cudaStream_t st) {
  if (!p.free_top) return 0;
  const dim3 block(32, 8), grid((p.ni + 31) / 32, (p.nj + 7) / 8, p.nshot);
  k_ac_image<R><<<grid, block, 0, st>>>(const_cast<R *>(p.cur), p.stage == 0 ? p.end : nullptr, p.ni, p.nj, p.nk,
                                        p.sx, p.sz, p.sf, p.off0);
  return 1;
}

template <typename R>
int launch_stage_ac(const StagePT<R> &p, int nzc, cudaStream_t st) {
  nzc = std::max(1, std::min(nzc, p.nk));
  const int nchunk = (p.nk + nzc - 1) / nzc;
  const dim3 block(TX, TY);
  const dim3 grid((p.ni + TX - 1) / TX, (p.nj + TY - 1) / TY, (unsigned)std::min(nchunk * p.nshot, 65535));
  switch (p.dir[0] | (p.dir[1] << 1) | (p.dir[2] << 2)) {
#define CASE(c)                                                                                         \
  case c:                                                                                               \
    k_stage_ac<(c)&1, ((c) >> 1) & 1, ((c) >> 2) & 1, R><<<grid, block, 0, st>>>(p, nzc, nchunk);       \
    break;
    CASE(0) CASE(1) CASE(2) CASE(3) CASE(4) CASE(5) CASE(6) CASE(7)
#undef CASE
  }
  return 1;
}

template int launch_ac_image<float>(const StagePT<float> &, cudaStream_t);
template int launch_ac_image<double>(const StagePT<double> &, cudaStream_t);
template int launch_stage_ac<float>(const StagePT<float> &, int, cudaStream_t);
template int launch_stage_ac<double>(const StagePT<double> &, int, cudaStream_t);

}  // namespace cgfd

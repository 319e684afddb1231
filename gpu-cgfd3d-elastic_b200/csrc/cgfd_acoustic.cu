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
#include "cgfd_tma.cuh"

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

// -----------------------------------------------------------------------------------------
// TMA-pipelined form (FP32): thread 0 streams, with mbarrier completion and one plane ahead of the
// computation, the stage input of one plane with its x-y halo (4 fields, one 4-D box of
// 40 x (TYT+4) x 1 x 4, x halo 16 bytes on both sides for the TMA alignment) into a 3-slot ring,
// and the 11 coefficients plus the w_pre / w_end values the RK combine reads (centre boxes) into
// a 2-slot ring. The z march runs upwards for backward z operators and downwards for forward
// ones, so that the one-sided operator needs exactly one plane ahead: the current plane and the
// one ahead come from the ring, the 3 planes behind from a per-thread register queue. The
// stage-input map covers the physical cells and the 3 ghost planes above the top (the pressure
// image); the halo beyond the grid's sides and bottom is zero fill, as the ghosts hold 0 there.
// -----------------------------------------------------------------------------------------
struct AcSmem {
  static constexpr int TYT = TY;
  static constexpr int XO = 4;             // x halo of the box: 16 bytes of floats
  static constexpr int WX = TX + 2 * XO;   // x box [-XO, 32+XO) around the tile
  static constexpr int WY = TYT + 4;       // y box [-1, TYT+3) (forward) or [-3, TYT+1) (backward)
  static constexpr int CELLS = TX * TYT;
  static constexpr int WAVE_ELEMS = kAcF * WY * WX;
  static constexpr int WAVE_SLOT = ((WAVE_ELEMS * 4 + 127) / 128) * 128;  // bytes
  static constexpr int COEF_BYTES = 11 * CELLS * 4;
  static constexpr int FLD_BYTES = kAcF * CELLS * 4;
  static constexpr int OFF_PRE = COEF_BYTES, OFF_END = COEF_BYTES + FLD_BYTES;  // within a cpe slot
  static constexpr int CPE_SLOT = COEF_BYTES + 2 * FLD_BYTES;
  static constexpr int NW = 3;  // wave ring slots: this plane, the one ahead, one in flight
  static constexpr int OFF_CPE = NW * WAVE_SLOT;
  static constexpr int OFF_BAR = OFF_CPE + 2 * CPE_SLOT;
  static constexpr int BYTES = OFF_BAR + 8 * 8;
  static constexpr int MINB = 3;
  static_assert(COEF_BYTES % 128 == 0 && FLD_BYTES % 128 == 0, "TMA destinations stay 128-byte aligned");
  static_assert(MINB * (BYTES + 1024) <= 228 * 1024, "MINB blocks must fit one SM's shared memory");
};

template <int DX, int DY, int DZ>
__global__ void __launch_bounds__(TX *AcSmem::TYT, AcSmem::MINB)
    k_stage_ac_tma(const __grid_constant__ StageP p, const __grid_constant__ TmaP tm, int nzc, int nchunk) {
  using S = AcSmem;
  constexpr int TYT = S::TYT;
  constexpr int LX = op_left(DX), LY = op_left(DY);
  constexpr int SD = DZ ? -1 : 1;  // march direction
  extern __shared__ __align__(128) unsigned char smem[];
  float *wave = reinterpret_cast<float *>(smem);
  unsigned char *cpe = smem + S::OFF_CPE;
  uint64_t *bar = reinterpret_cast<uint64_t *>(smem + S::OFF_BAR);  // NW wave, then 2 cpe

  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
  const int bx = blockIdx.x, by = blockIdx.y;
  const int shot = blockIdx.z / nchunk, kb = (blockIdx.z % nchunk) * nzc;
  const int ke = min(kb + nzc, p.nk);
  if (kb >= ke) return;
  const int n = ke - kb;
  const int i = bx * TX + tx, j = by * TYT + ty;
  const bool act = i < p.ni && j < p.nj;
  const int k0 = SD > 0 ? kb : ke - 1;
  const long long sf = p.sf;
  const long long woff = (long long)shot * 9 * sf;
  const float *__restrict__ cur = p.cur + woff;
  float *__restrict__ tmp_out = p.tmp_out ? p.tmp_out + woff : nullptr;
  float *__restrict__ endw = p.end + woff;
  const int stage = p.stage;
  const bool need_pre = stage == 1 || stage == 2;
  const bool need_end = stage >= 1;
  const uint32_t wave_bytes = S::WAVE_ELEMS * 4;
  const uint32_t cpe_bytes = S::COEF_BYTES + (need_pre ? S::FLD_BYTES : 0) + (need_end ? S::FLD_BYTES : 0);
  // box origins (x a multiple of 4 floats): the stage-input map counts physical cells from
  // (0, 0, 0); the centre-box maps count device-layout (padded) coordinates
  const int xw = bx * TX - S::XO, yw = by * TYT - LY;  // box row r = tile row r - LY
  const int xc = GX + bx * TX, yc = 3 + by * TYT;

  if (tid == 0) {
    for (int b = 0; b < S::NW + 2; b++) mbar_init(&bar[b], 1);
    fence_barrier_init();
  }
  __syncthreads();

  auto issue_wave = [&](int m) {
    const int kk = k0 + m * SD;
    uint64_t *b = &bar[m % S::NW];
    mbar_expect_tx(b, wave_bytes);
    tma_load_4d(wave + (m % S::NW) * (S::WAVE_SLOT / 4), &tm.cur, xw, yw, kk, 9 * shot, b);
  };
  auto issue_cpe = [&](int m) {
    const int kk = k0 + m * SD;
    const int sl = m & 1;
    uint64_t *b = &bar[S::NW + sl];
    unsigned char *base = cpe + sl * S::CPE_SLOT;
    mbar_expect_tx(b, cpe_bytes);
    tma_load_4d(base, &tm.coef, xc, yc, kk + 3, 0, b);
    if (need_pre) tma_load_4d(base + S::OFF_PRE, &tm.pre, xc, yc, kk + 3, 9 * shot, b);
    if (need_end) tma_load_4d(base + S::OFF_END, &tm.end, xc, yc, kk + 3, 9 * shot, b);
  };
  if (tid == 0) {
    for (int m = 0; m + 1 < S::NW && m <= n; m++) issue_wave(m);  // planes 0..n exist
    issue_cpe(0);
  }

  // PML faces that intersect this block (uniform)
  unsigned fmask = 0;
  for (int fi = 0; fi < p.nface; fi++) {
    const FaceP &f = p.face[fi];
    const bool xo = f.lo[0] <= bx * TX + TX - 1 && f.hi[0] >= bx * TX;
    const bool yo = f.lo[1] <= by * TYT + TYT - 1 && f.hi[1] >= by * TYT;
    const bool zo = f.lo[2] <= ke - 1 && f.hi[2] >= kb;
    if (xo && yo && zo) fmask |= 1u << fi;
  }

  // register queue of the planes behind, in march order: q[f][n] = plane k + (n - 3) * SD
  float q[kAcF][3];
#pragma unroll
  for (int f = 0; f < kAcF; f++)
#pragma unroll
    for (int m = 0; m < 3; m++) q[f][m] = 0.f;
  if (act) {
#pragma unroll
    for (int m = 0; m < 3; m++) {
      const long long id = didx(p, i, j, k0 + (m - 3) * SD);
#pragma unroll
      for (int f = 0; f < kAcF; f++) q[f][m] = __ldg(cur + f * sf + id);
    }
  }
  const int wc = (ty + LY) * S::WX + tx + S::XO;  // centre of this thread in a wave slot (per field)
  mbar_wait(&bar[0], 0, p.err);
  bool bad = false;  // stage 3: a new solution value is NaN/Inf

  const int cell = ty * TX + tx;
  for (int m = 0; m < n; m++) {
    const int k = k0 + m * SD;
    if (tid == 0) {
      if (m + S::NW - 1 <= n) issue_wave(m + S::NW - 1);
      if (m + 1 < n) issue_cpe(m + 1);
    }
    const int ws = m % S::NW, wn = (m + 1) % S::NW, cs = m & 1;
    mbar_wait(&bar[wn], ((m + 1) / S::NW) & 1, p.err);
    mbar_wait(&bar[S::NW + cs], (m >> 1) & 1, p.err);
    const float *W = wave + ws * (S::WAVE_SLOT / 4);
    const float *Wn = wave + wn * (S::WAVE_SLOT / 4);

    if (act) {
      const float *Cc = reinterpret_cast<const float *>(cpe + cs * S::CPE_SLOT) + cell;
      float mt[3][3];
#pragma unroll
      for (int a = 0; a < 3; a++)
#pragma unroll
        for (int b = 0; b < 3; b++) mt[a][b] = Cc[(3 * a + b) * S::CELLS];
      const float slw = Cc[CF_SLW * S::CELLS], kappa = Cc[CF_MED * S::CELLS];
      // derivatives along x, y, z of Vx Vy Vz (dv[axis][comp]) and of P (dp[axis])
      float dv[3][3], dp[3];
#pragma unroll
      for (int f = 0; f < kAcF; f++) {
        const float *r = W + f * S::WY * S::WX + (ty + LY) * S::WX + tx + S::XO - LX;
        const float dx = drp5<DX>(r[0], r[1], r[2], r[3], r[4]);
        const float *c = W + f * S::WY * S::WX + ty * S::WX + tx + S::XO;
        const float dy = drp5<DY>(c[0], c[S::WX], c[2 * S::WX], c[3 * S::WX], c[4 * S::WX]);
        const float c0 = W[f * S::WY * S::WX + wc], c1 = Wn[f * S::WY * S::WX + wc];
        const float dz = SD > 0 ? drp5<DZ>(q[f][0], q[f][1], q[f][2], c0, c1) : drp5<DZ>(c1, c0, q[f][2], q[f][1], q[f][0]);
        if (f < 3) { dv[0][f] = dx; dv[1][f] = dy; dv[2][f] = dz; }
        else { dp[0] = dx; dp[1] = dy; dp[2] = dz; }
      }
      float h[kAcF];
#pragma unroll
      for (int c = 0; c < 3; c++) h[c] = -slw * (mt[0][c] * dp[0] + mt[1][c] * dp[1] + mt[2][c] * dp[2]);
      // vlow rows of the top 3 planes (as k_stage_ac): planes k, k+1, k+2 are c0, q[2], q[1] when
      // marching down (forward operators), k-2, k-1, k are q[1], q[2], c0 when marching up
      float dvz[3] = {dv[2][0], dv[2][1], dv[2][2]};
      const int nl = p.free_top ? p.nk - 1 - k : 3;
      if (nl == 1 || nl == 2) {
#pragma unroll
        for (int c = 0; c < 3; c++) {
          const float c0 = W[c * S::WY * S::WX + wc];
          if constexpr (DZ) {
            dvz[c] = nl == 1 ? -c0 + q[c][2]
                             : -7.0f / 6.0f * c0 + 8.0f / 6.0f * q[c][2] - 1.0f / 6.0f * q[c][1];
          } else {
            dvz[c] = nl == 1 ? -q[c][2] + c0
                             : 1.0f / 6.0f * q[c][1] - 8.0f / 6.0f * q[c][2] + 7.0f / 6.0f * c0;
          }
        }
      }
      h[kAcP] = nl == 0 ? 0.f
                        : -kappa * (mt[0][0] * dv[0][0] + mt[1][0] * dv[1][0] + mt[2][0] * dvz[0] +
                                    mt[0][1] * dv[0][1] + mt[1][1] * dv[1][1] + mt[2][1] * dvz[1] +
                                    mt[0][2] * dv[0][2] + mt[1][2] * dv[1][2] + mt[2][2] * dvz[2]);
      if (fmask) {
        float hc[kAcF] = {0.f, 0.f, 0.f, 0.f};
        for (int fi = 0; fi < p.nface; fi++) {
          const FaceP &fc = p.face[fi];
          if ((fmask >> fi & 1) && in_face(fc, i, j, k))
            ac_pml_face(p, fc, i, j, k, shot, slw, kappa, mt[fc.axis], dv[fc.axis], dp[fc.axis], hc);
        }
#pragma unroll
        for (int c = 0; c < kAcF; c++) h[c] += hc[c];
      }
      // RK combine (wav_update / wav_update_end)
      const long long id = didx(p, i, j, k);
      const float *PR = reinterpret_cast<const float *>(cpe + cs * S::CPE_SLOT + S::OFF_PRE) + cell;
      const float *EN = reinterpret_cast<const float *>(cpe + cs * S::CPE_SLOT + S::OFF_END) + cell;
      const float ca = p.ca, cb = p.cb;
      if (stage == 0) {
#pragma unroll
        for (int f = 0; f < kAcF; f++) {
          const float c0 = W[f * S::WY * S::WX + wc];  // stage input = w_pre at stage 0
          tmp_out[f * sf + id] = c0 + ca * h[f];
          endw[f * sf + id] = c0 + cb * h[f];
        }
      } else if (stage < 3) {
#pragma unroll
        for (int f = 0; f < kAcF; f++) {
          tmp_out[f * sf + id] = PR[f * S::CELLS] + ca * h[f];
          endw[f * sf + id] = EN[f * S::CELLS] + cb * h[f];
        }
      } else {
#pragma unroll
        for (int f = 0; f < kAcF; f++) {
          const float e = EN[f * S::CELLS] + cb * h[f];
          endw[f * sf + id] = e;
          bad |= nonfinite(e);
        }
      }
    }
#pragma unroll
    for (int f = 0; f < kAcF; f++) {
      q[f][0] = q[f][1];
      q[f][1] = q[f][2];
      q[f][2] = W[f * S::WY * S::WX + wc];
    }
    // the slots read in this plane are refilled by TMA after the barrier
    fence_proxy_async_smem();
    __syncthreads();
  }
  if (bad) atomicOr(p.err, kErrWaveNonfinite);
}

int launch_stage_ac_tma(const StageP &p, const TmaP &tm, int nzc, cudaStream_t st) {
  nzc = std::max(1, std::min(nzc, p.nk));
  const int nchunk = (p.nk + nzc - 1) / nzc;
  if ((long long)nchunk * p.nshot > 65535) return -1;  // the caller runs the direct-load kernel
  const dim3 block(TX, AcSmem::TYT);
  const dim3 grid((p.ni + TX - 1) / TX, (p.nj + AcSmem::TYT - 1) / AcSmem::TYT, nchunk * p.nshot);
  static bool attr_done[8] = {};  // the opt-in above 48 KB of dynamic shared memory, once per instantiation
  switch (p.dir[0] | (p.dir[1] << 1) | (p.dir[2] << 2)) {
#define CASE(c)                                                                                           \
  case c:                                                                                                 \
    if (!attr_done[c]) {                                                                                  \
      cudaFuncSetAttribute(k_stage_ac_tma<(c)&1, ((c) >> 1) & 1, ((c) >> 2) & 1>,                         \
                           cudaFuncAttributeMaxDynamicSharedMemorySize, AcSmem::BYTES);                   \
      attr_done[c] = true;                                                                                \
    }                                                                                                     \
    k_stage_ac_tma<(c)&1, ((c) >> 1) & 1, ((c) >> 2) & 1><<<grid, block, AcSmem::BYTES, st>>>(p, tm, nzc, nchunk); \
    break;
    CASE(0) CASE(1) CASE(2) CASE(3) CASE(4) CASE(5) CASE(6) CASE(7)
#undef CASE
  }
  return 1;
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

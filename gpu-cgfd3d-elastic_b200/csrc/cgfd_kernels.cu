// cgfd_kernels.cu -- fused RK-stage kernels of the CGFD3D elastic path for sm_100a.
//
// k_stage_bulk: all planes below the surface slab. A thread block owns a TX x TY column
//   tile and marches along z: the x-y tile of the current plane (with the 3/1-point halo of
//   the one-sided MacCormack operators) sits in shared memory, double-buffered so that each
//   plane needs one barrier, and the 5 planes the z operator needs sit in a per-thread
//   register queue. Every wavefield value is read from HBM once per stage (halo re-reads hit
//   L2), the RHS is combined into tmp/end in registers and never stored.
//   Replaces sv_curv_col_el_{iso,vti,aniso}_rhs_inner_gpu, _rhs_cfspml_gpu and the
//   wav_update/wav_update_end launches for these cells.
// k_stage_surface: the top NSURF planes when the free surface is on: inner RHS, traction
//   image (sv_curv_col_el_gpu.cu:19-221), vlow (sv_curv_col_el_iso_gpu.cu:462-603), PML
//   with the free-surface terms, RK combine.
// k_source: moment/force injection over the smoothed points (sv_curv_col_el_gpu.cu:227-301),
//   applied to tmp/end with the stage's RK weights.
// k_recv: trilinear station sampling of w_pre for all stations (io_funcs.cu:1624-1666).
#include <algorithm>

#include "cgfd_dev.cuh"
#include "cgfd_launch.h"
#include "cgfd_tma.cuh"

namespace cgfd {

// Shared memory of the direct-load kernel: the double-buffered x-y tile with its halo, 9 fields
// (31 KB in FP32; 62 KB in the FP64 build, one block per SM).
template <typename R> struct DirectTile {
  static constexpr int SW = TX + 4, SH = TY + 4;
  static constexpr int BYTES = 2 * 9 * SH * SW * (int)sizeof(R);
  static constexpr int MINB = sizeof(R) == 8 ? 1 : 2;
};

template <int MED, int DX, int DY, int DZ, typename R = float>
__global__ void __launch_bounds__(TX *TY, DirectTile<R>::MINB)
    k_stage_bulk(const __grid_constant__ StagePT<R> p, int nzc) {
  constexpr int LX = op_left(DX), LY = op_left(DY), LZ = op_left(DZ);
  constexpr int SW = DirectTile<R>::SW, SH = DirectTile<R>::SH;
  extern __shared__ __align__(16) unsigned char dsm[];
  R(*s)[9][SH][SW] = reinterpret_cast<R(*)[9][SH][SW]>(dsm);

  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
  const int bx = blockIdx.x, by = blockIdx.y;
  const int i = bx * TX + tx, j = by * TY + ty;
  const int kb = blockIdx.z * nzc;
  const int ke = min(kb + nzc, p.nbulk);
  if (kb >= ke) return;
  const bool act = (i < p.ni) && (j < p.nj);
  const long long sf = p.sf;
  const R *__restrict__ cur = p.cur;

  // halo slot of this thread (x halo: 4 columns per tile row, y halo: 4 rows per tile column)
  int h_i = 0, h_j = 0, h_sx = 0, h_sy = 0;
  bool h_on = false;
  if (tid < 4 * TY) {
    int row = tid >> 2, hh = tid & 3;
    h_j = by * TY + row;
    h_sy = row + LY;
    if (hh < LX) { h_i = bx * TX - LX + hh; h_sx = hh; }
    else { h_i = bx * TX + TX + (hh - LX); h_sx = TX + hh; }
    h_on = true;
  } else if (tid < 4 * TY + 4 * TX) {
    int q = tid - 4 * TY;
    int col = q % TX, hh = q / TX;
    h_i = bx * TX + col;
    h_sx = col + LX;
    h_j = hh < LY ? by * TY - LY + hh : by * TY + TY + (hh - LY);
    h_sy = LY + (h_j - by * TY);
    h_on = true;
  }
  // points beyond the 3 ghost layers are never needed; they read as 0 without a load
  const bool h_ld = h_on && h_i <= p.ni + 2 && h_j <= p.nj + 2;

  // z register queue: q[f][n] holds plane k - LZ + n
  R q[9][5];
#pragma unroll
  for (int f = 0; f < 9; f++)
#pragma unroll
    for (int n = 0; n < 5; n++) q[f][n] = R(0);
  if (act) {
#pragma unroll
    for (int n = 0; n < 4; n++) {
      long long id = didx(p, i, j, kb - LZ + n);
#pragma unroll
      for (int f = 0; f < 9; f++) q[f][n] = __ldg(cur + f * sf + id);
    }
  }

  for (int k = kb; k < ke; k++) {
    const int buf = k & 1;
    if (act) {
      long long id = didx(p, i, j, k + 4 - LZ);
#pragma unroll
      for (int f = 0; f < 9; f++) q[f][4] = __ldg(cur + f * sf + id);
    }
#pragma unroll
    for (int f = 0; f < 9; f++) s[buf][f][ty + LY][tx + LX] = q[f][LZ];
    if (h_on) {
      long long id = h_ld ? didx(p, h_i, h_j, k) : 0;
#pragma unroll
      for (int f = 0; f < 9; f++) s[buf][f][h_sy][h_sx] = h_ld ? __ldg(cur + f * sf + id) : R(0);
    }
    __syncthreads();

    if (act) {
      const long long id = didx(p, i, j, k);
      const CoefView<R> cv(p);
      R m[3][3];
#pragma unroll
      for (int a = 0; a < 3; a++)
#pragma unroll
        for (int b = 0; b < 3; b++) m[a][b] = cv(3 * a + b, id);
      const R slw = cv(CF_SLW, id);
      Medium<MED, R> md;
      md.load([&](int c) { return cv(c, id); });
      CellAcc<R> acc;
      acc.zero();
      // ---- x
      {
        R d[9];
#pragma unroll
        for (int f = 0; f < 9; f++) {
          const R *r = &s[buf][f][ty + LY][tx];
          d[f] = drp5<DX>(r[0], r[1], r[2], r[3], r[4]);
        }
        acc.add_axis(m[0], d, d + 3);
        for (int fi = 0; fi < p.nface; fi++) {
          const FacePT<R> &fc = p.face[fi];
          if (fc.axis == 0 && i >= fc.lo[0] && i <= fc.hi[0] && j >= fc.lo[1] && j <= fc.hi[1] && k >= fc.lo[2] &&
              k <= fc.hi[2])
            pml_face<MED>(p, fc, i, j, k, md, slw, m[0], d, d + 3, nullptr, nullptr, acc.hc);
        }
      }
      // ---- y
      {
        R d[9];
#pragma unroll
        for (int f = 0; f < 9; f++)
          d[f] = drp5<DY>(s[buf][f][ty][tx + LX], s[buf][f][ty + 1][tx + LX], s[buf][f][ty + 2][tx + LX],
                          s[buf][f][ty + 3][tx + LX], s[buf][f][ty + 4][tx + LX]);
        acc.add_axis(m[1], d, d + 3);
        for (int fi = 0; fi < p.nface; fi++) {
          const FacePT<R> &fc = p.face[fi];
          if (fc.axis == 1 && i >= fc.lo[0] && i <= fc.hi[0] && j >= fc.lo[1] && j <= fc.hi[1] && k >= fc.lo[2] &&
              k <= fc.hi[2])
            pml_face<MED>(p, fc, i, j, k, md, slw, m[1], d, d + 3, nullptr, nullptr, acc.hc);
        }
      }
      // ---- z
      {
        R d[9];
#pragma unroll
        for (int f = 0; f < 9; f++) d[f] = drp5<DZ>(q[f][0], q[f][1], q[f][2], q[f][3], q[f][4]);
        acc.add_axis(m[2], d, d + 3);
        for (int fi = 0; fi < p.nface; fi++) {
          const FacePT<R> &fc = p.face[fi];
          if (fc.axis == 2 && i >= fc.lo[0] && i <= fc.hi[0] && j >= fc.lo[1] && j <= fc.hi[1] && k >= fc.lo[2] &&
              k <= fc.hi[2])
            pml_face<MED>(p, fc, i, j, k, md, slw, m[2], d, d + 3, nullptr, nullptr, acc.hc);
        }
      }
      R h[9];
      h[0] = slw * acc.mom[0] + acc.hc[0];
      h[1] = slw * acc.mom[1] + acc.hc[1];
      h[2] = slw * acc.mom[2] + acc.hc[2];
      md.hooke(acc.G, h + 3);
#pragma unroll
      for (int c = 3; c < 9; c++) h[c] += acc.hc[c];
      if (p.rhs) {
#pragma unroll
        for (int f = 0; f < 9; f++) p.rhs[f * sf + id] = h[f];
      } else {
        R cc[9];
#pragma unroll
        for (int f = 0; f < 9; f++) cc[f] = q[f][LZ];
        rk_store(p.stage, p.ca, p.cb, sf, id, cc, h, p.pre, p.tmp_out, p.end, p.err);
      }
    }
#pragma unroll
    for (int f = 0; f < 9; f++)
#pragma unroll
      for (int n = 0; n < 4; n++) q[f][n] = q[f][n + 1];
  }
}

// -----------------------------------------------------------------------------------------
// surface slab
// -----------------------------------------------------------------------------------------
// Stage input of the surface kernel: FP32, or scaled FP16 (value = scale[f] * stored).
template <typename TW>
struct WaveIn {
  const TW *w;
  long long sf;
  const float *sc;
  __device__ __forceinline__ real_of<TW> operator()(int f, long long q) const {
    const real_of<TW> v = to_f(__ldg(w + f * sf + q));
    if constexpr (std::is_same<TW, float>::value || std::is_same<TW, double>::value) return v;
    else return v * __ldg(sc + f);
  }
};

template <typename TW>
__device__ __forceinline__ void ld5(int dir, const WaveIn<TW> &cur, int f, long long id, long long off,
                                    real_of<TW> (&o)[5]) {
  int L = op_left(dir);
#pragma unroll
  for (int n = 0; n < 5; n++) o[n] = cur(f, id + (n - L) * off);
}

// Surface slab: one thread per cell of the top NSURF planes; a block holds the NSURF planes of
// 32 x 2 columns, so that the z-stencil loads of one column hit in the SM's L1. WP is the wave
// policy of the bulk kernel (0 FP32 stage levels; 1 FP32 input, FP16 output; 2 FP16 input and
// output). The kernel is latency-bound on its many cached loads: registers are capped at 128 so
// that 16 warps share each SM (a few spills are cheaper than 8 warps).
// The operator directions of the stage (DX, DY, DZ: 0 backward, 1 forward) are template
// parameters, so that every stencil offset is a compile-time constant.
// Traction-image fluxes of the stage input at the top kFluxPlanes planes, every column of the
// extended x-y range (ghosts give 0: the wavefield is 0 there): for stress row c (Txx Txy Txz /
// Txy Tyy Tyz / Txz Tyz Tzz) and metric row a (xi, eta, zeta), jac (m_a . T_c) -- the
// J (grad xi_a . T) terms sv_curv_col_el_gpu.cu:53-217 differentiates. Computed once per point
// here instead of once per stencil use in the surface slab.
template <typename TC, int WP>
__global__ void __launch_bounds__(256) k_timg_flux(const __grid_constant__ StagePT<real_of<TC>> p) {
  using R = real_of<TC>;
  using TW = typename std::conditional<WP == 2, __half, R>::type;
  const int nxe = p.ni + 6, nye = p.nj + 6;
  const long long plane = (long long)nxe * nye, per_shot = 9 * kFluxPlanes * plane;
  const long long total = plane * kFluxPlanes * p.nshot;
  const CoefView<TC> cv(p);
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    const int ii = (int)(t % nxe), jj = (int)((t / nxe) % nye);
    const int pl = (int)((t / plane) % kFluxPlanes), shot = (int)(t / (plane * kFluxPlanes));
    const int k = p.nk - kFluxPlanes + pl;
    const long long q = didx(p, ii - 3, jj - 3, k);
    const WaveIn<TW> cur{reinterpret_cast<const TW *>(p.cur) + (long long)shot * 9 * p.sf, p.sf,
                         p.wsc + shot * 18};
    const int tr[3][3] = {{3, 8, 7}, {8, 4, 6}, {7, 6, 5}};
    const R jc = __ldg(p.jac + q);
    R *out = p.flux + shot * per_shot + (long long)pl * plane + (long long)jj * nxe + ii;
#pragma unroll
    for (int c = 0; c < 3; c++) {
      const R t1 = cur(tr[c][0], q), t2 = cur(tr[c][1], q), t3 = cur(tr[c][2], q);
#pragma unroll
      for (int a = 0; a < 3; a++)
        out[(3 * c + a) * kFluxPlanes * plane] = jc * (cv(3 * a, q) * t1 + cv(3 * a + 1, q) * t2 + cv(3 * a + 2, q) * t3);
    }
  }
}

template <int MED, typename TC, int WP, int DX, int DY, int DZ>
__global__ void __launch_bounds__(32 * 2 * NSURF, 2) k_stage_surface(const __grid_constant__ StagePT<real_of<TC>> p) {
  constexpr int DIR[3] = {DX, DY, DZ};
  using R = real_of<TC>;  // double in the FP64 build (TC double, WP 0), float otherwise
  using TW = typename std::conditional<WP == 2, __half, R>::type;
  using TT = typename std::conditional<WP >= 1, __half, R>::type;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= p.ni || j >= p.nj) return;
  const long long sf = p.sf;
  const int shot = blockIdx.z;
  const long long woff = (long long)shot * 9 * sf;
  const float *wsc = p.wsc + shot * 18;  // FP16 stage levels: this shot's scale
  const WaveIn<TW> cur{reinterpret_cast<const TW *>(p.cur) + woff, sf, wsc};
  const long long offs[3] = {1, p.sx, p.sz};
  const int nk2 = p.nk - 1;

  {
    const int k = p.nbulk + threadIdx.z;  // one thread per cell of the slab (nk - nbulk == NSURF)
    const long long id = didx(p, i, j, k);
    const CoefView<TC> cv(p);
    R m[3][3];
#pragma unroll
    for (int a = 0; a < 3; a++)
#pragma unroll
      for (int b = 0; b < 3; b++) m[a][b] = cv(3 * a + b, id);
    const R slw = cv(CF_SLW, id);
    Medium<MED, R> md;
    md.load([&](int c) { return cv(c, id); });

    // normal derivatives of all 9 fields along the 3 axes
    R dv[3][3], dtt[3][6];
#pragma unroll
    for (int a = 0; a < 3; a++) {
#pragma unroll
      for (int f = 0; f < 9; f++) {
        R v[5];
        ld5(DIR[a], cur, f, id, offs[a], v);
        R d = drp5r(DIR[a], v[0], v[1], v[2], v[3], v[4]);
        if (f < 3) dv[a][f] = d; else dtt[a][f - 3] = d;
      }
    }
    R hc[9];
#pragma unroll
    for (int c = 0; c < 9; c++) hc[c] = R(0);

    // momentum: normal form, or the traction image near the free surface
    R h[9];
    {
      R mom[3] = {R(0), R(0), R(0)};
#pragma unroll
      for (int a = 0; a < 3; a++) {
        R mm[3];
        momentum_axis(m[a], dtt[a], mm);
        mom[0] += mm[0]; mom[1] += mm[1]; mom[2] += mm[2];
      }
      h[0] = slw * mom[0]; h[1] = slw * mom[1]; h[2] = slw * mom[2];
    }
    constexpr int dzr = DZ;
    if (p.free_top) {
      constexpr int idx_last = dzr ? 3 : 1, idx_first = dzr ? -1 : -3;
      if (k >= nk2 - idx_last) {
        // sv_curv_col_el_gpu.cu:53-217, on the fluxes k_timg_flux computed for this stage
        const int n_free = nk2 - k - idx_first;
        const R jc = __ldg(p.jac + id);
        const R slwjac = slw / jc;
        constexpr int LXo = op_left(DX), LYo = op_left(DY), LZo = op_left(dzr);
        const int nxe = p.ni + 6;
        const long long fpl = (long long)nxe * (p.nj + 6), fcs = kFluxPlanes * fpl;
        const R *F = p.flux + (long long)shot * 9 * fcs + (long long)(j + 3) * nxe + (i + 3);
        const int pk = k - (p.nk - kFluxPlanes);  // flux plane of this cell
#pragma unroll
        for (int c = 0; c < 3; c++) {
          R vx[5], vy[5], vz[5];
          const R *Fx = F + (3 * c + 0) * fcs + pk * fpl, *Fy = F + (3 * c + 1) * fcs + pk * fpl;
          const R *Fz = F + (3 * c + 2) * fcs;
#pragma unroll
          for (int n = 0; n < 5; n++) {
            vx[n] = __ldg(Fx + (n - LXo));
            vy[n] = __ldg(Fy + (long long)(n - LYo) * nxe);
            int off;
            R sgn;
            if (n < n_free) { off = n - LZo; sgn = R(1); }
            else if (n == n_free) { off = 0; sgn = R(0); }
            else { off = (n - LZo) - 2 * (n - n_free); sgn = R(-1); }
            vz[n] = sgn * __ldg(Fz + (long long)(pk + off) * fpl);
          }
          R DxTx = drp5<DX>(vx[0], vx[1], vx[2], vx[3], vx[4]);
          R DyTy = drp5<DY>(vy[0], vy[1], vy[2], vy[3], vy[4]);
          R DzTz = drp5<DZ>(vz[0], vz[1], vz[2], vz[3], vz[4]);
          h[c] = (DxTx + DyTy + DzTz) * slwjac;
        }
      }
    }
    // Hooke: normal, or vlow with low-order / converted dzV in the top 3 layers
    {
      R dz[3] = {dv[2][0], dv[2][1], dv[2][2]};
      if (p.free_top && k >= nk2 - 2) {
        const int nl = nk2 - k;
        if (nl == 0) {
          const long long ij = ((long long)j * p.ni + i) * 9;
#pragma unroll
          for (int r = 0; r < 3; r++)
            dz[r] = __ldg(p.matx + ij + 3 * r) * dv[0][0] + __ldg(p.matx + ij + 3 * r + 1) * dv[0][1] +
                    __ldg(p.matx + ij + 3 * r + 2) * dv[0][2] + __ldg(p.maty + ij + 3 * r) * dv[1][0] +
                    __ldg(p.maty + ij + 3 * r + 1) * dv[1][1] + __ldg(p.maty + ij + 3 * r + 2) * dv[1][2];
        } else {
#pragma unroll
          for (int c = 0; c < 3; c++) {
            if (nl == 1) {  // 2nd order (fd_t.cu:82-85, 103-106)
              dz[c] = dzr ? (-cur(c, id) + cur(c, id + p.sz)) : (-cur(c, id - p.sz) + cur(c, id));
            } else {        // 4th order (fd_t.cu:86-89, 107-110)
              dz[c] = dzr ? (-7.0f / 6.0f * cur(c, id) + 8.0f / 6.0f * cur(c, id + p.sz) -
                             1.0f / 6.0f * cur(c, id + 2 * p.sz))
                          : (1.0f / 6.0f * cur(c, id - 2 * p.sz) - 8.0f / 6.0f * cur(c, id - p.sz) +
                             7.0f / 6.0f * cur(c, id));
            }
          }
        }
      }
      R G[3][3];
#pragma unroll
      for (int vi = 0; vi < 3; vi++)
#pragma unroll
        for (int xj = 0; xj < 3; xj++) G[vi][xj] = m[0][xj] * dv[0][vi] + m[1][xj] * dv[1][vi] + m[2][xj] * dz[vi];
      md.hooke(G, h + 3);
    }
    // CFS-PML faces, with the free-surface terms on x/y faces at the top layer
    for (int fi = 0; fi < p.nface; fi++) {
      const FacePT<R> &fc = p.face[fi];
      if (!(i >= fc.lo[0] && i <= fc.hi[0] && j >= fc.lo[1] && j <= fc.hi[1] && k >= fc.lo[2] && k <= fc.hi[2])) continue;
      const int a = fc.axis;
      const R *smat = nullptr;
      if (p.free_top && a < 2 && k == nk2) smat = (a == 0 ? p.matx : p.maty) + ((long long)j * p.ni + i) * 9;
      pml_face<MED>(p, fc, i, j, k, md, slw, m[a], dv[a], dtt[a], smat, m[2], hc, shot);
    }
#pragma unroll
    for (int c = 0; c < 9; c++) h[c] += hc[c];
    if (WP == 0 && p.rhs) {
#pragma unroll
      for (int f = 0; f < 9; f++) p.rhs[woff + f * sf + id] = h[f];
    } else if constexpr (WP == 0) {
      R cc[9];
#pragma unroll
      for (int f = 0; f < 9; f++) cc[f] = cur(f, id);
      rk_store(p.stage, p.ca, p.cb, sf, id, cc, h, p.pre + woff, p.tmp_out ? p.tmp_out + woff : nullptr, p.end + woff,
               p.err);
    } else {
      // FP16 stage levels: the RK combine of rk_store with the stage output scaled to FP16
      TT *tout = reinterpret_cast<TT *>(p.tmp_out) + woff;
      float *endw = p.end + woff;
      const float *prw = p.pre + woff;
      if (p.stage == 0) {
#pragma unroll
        for (int f = 0; f < 9; f++) {
          const float c0 = cur(f, id);
          tout[f * sf + id] = from_f<TT>((c0 + p.ca * h[f]) * __ldg(wsc + 9 + f));
          endw[f * sf + id] = c0 + p.cb * h[f];
        }
      } else if (p.stage < 3) {
#pragma unroll
        for (int f = 0; f < 9; f++) {
          tout[f * sf + id] = from_f<TT>((__ldg(prw + f * sf + id) + p.ca * h[f]) * __ldg(wsc + 9 + f));
          endw[f * sf + id] = endw[f * sf + id] + p.cb * h[f];
        }
      } else {
        float vmax = 0.f, smax = 0.f;
        bool bad = false;
#pragma unroll
        for (int f = 0; f < 9; f++) {
          const float e = endw[f * sf + id] + p.cb * h[f];
          endw[f * sf + id] = e;
          bad |= nonfinite(e);
          if (f < 3) vmax = fmaxf(vmax, fabsf(e));
          else smax = fmaxf(smax, fabsf(e));
        }
        if (bad) atomicOr(p.err, kErrWaveNonfinite);
        atomic_max_abs(&p.amax[2 * shot + 0], vmax);
        atomic_max_abs(&p.amax[2 * shot + 1], smax);
      }
    }
  }
}

// -----------------------------------------------------------------------------------------
// sources, stations, step counter
// -----------------------------------------------------------------------------------------
template <typename R>
__global__ void k_source(const __grid_constant__ SrcPT<R> s) {
  const int is = blockIdx.y;
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (is >= s.nsrc || e >= s.ext_num[is]) return;
  const int it = *s.d_it;
  const int ib = s.it_begin[is];
  if (it < ib || it > ib + s.max_nt - 1) return;
  const float *v = s.stf + (((long long)is * s.max_nt + (it - ib)) * 4 + s.stage) * 9;
  const int shot = s.src_shot[is];
  const long long id = s.ext_idx[(long long)is * s.max_ext + e] + (long long)shot * 9 * s.sf;
  const R wv = s.ext_wv[(long long)is * s.max_ext + e];
  const R wt = s.ext_wt[(long long)is * s.max_ext + e];
  for (int c = 0; c < 9; c++) {
    R h;
    if (c < 3) { if (!s.force) continue; h = R(v[c]) * wv; }
    else { if (!s.moment) continue; h = -R(v[c]) * wt; }
    if (s.stage < 3) {
      if constexpr (std::is_same<R, float>::value) {
        if (s.wave16)
          atomicAdd(reinterpret_cast<__half *>(s.tmp_out) + c * s.sf + id,
                    __float2half_rn(s.ca * h * s.wsc[18 * shot + 9 + c]));
        else atomicAdd(s.tmp_out + c * s.sf + id, s.ca * h);
      } else {
        atomicAdd(s.tmp_out + c * s.sf + id, s.ca * h);
      }
    }
    const R old = atomicAdd(s.end + c * s.sf + id, s.cb * h);
    if constexpr (std::is_same<R, float>::value)
      if (s.wave16 && s.stage == 3) atomic_max_abs(&s.amax[2 * shot + wgroup(c)], old + s.cb * h);
  }
}

template <typename R>
__global__ void k_recv(const __grid_constant__ RecvPT<R> r) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= r.nshot * r.nsta * 9) return;
  const int it = *r.d_it;
  if (it < 0 || it >= r.nt_total) return;
  const int shot = t / (r.nsta * 9), sidx = (t / 9) % r.nsta, c = t % 9;
  const R *pre = r.pre + (long long)shot * 9 * r.sf;
  R v = R(0);
#pragma unroll
  for (int qn = 0; qn < 8; qn++) {
    const R w = r.w8[sidx * 8 + qn];
    if (w != R(0)) v += w * __ldg(pre + c * r.sf + r.idx8[sidx * 8 + qn]);
  }
  if (nonfinite(v)) atomicOr(r.d_flag, kErrStationNonfinite);
  r.seis[(((long long)shot * r.nsta + sidx) * 9 + c) * r.nt_total + it] = (float)v;
}

// PG_calcu_gpu (wav_t.cu:281-360) on the top physical plane, every shot: acceleration from the
// step difference of V, displacement accumulated by the trapezoid rule in double (the
// reference's 0.5 literal), running maxima of the components and magnitudes.
template <typename R>
__global__ void k_peak_motion(const __grid_constant__ PgPT<R> q) {
  const long long nij = (long long)q.ni * q.nj;
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= nij * q.nshot) return;
  const int shot = (int)(t / nij);
  const long long ij = t % nij;
  const int j = (int)(ij / q.ni), i = (int)(ij % q.ni);
  const long long idx = (long long)shot * 9 * q.sf + q.off_top + (long long)j * q.sx + i;
  R v1[3], v0[3], a[3], d[3];
  R *dis = q.dis + (long long)shot * 3 * nij + ij;
#pragma unroll
  for (int c = 0; c < 3; c++) {
    v1[c] = q.w_end[c * q.sf + idx];
    v0[c] = q.w_pre[c * q.sf + idx];
    a[c] = fabs((v1[c] - v0[c]) / R(q.dt));
    d[c] = (R)((double)dis[c * nij] + 0.5 * (double)(v1[c] + v0[c]) * (double)q.dt);
    dis[c * nij] = d[c];
  }
  const R val[15] = {sqrt(v1[0] * v1[0] + v1[1] * v1[1] + v1[2] * v1[2]),
                     sqrt(v1[0] * v1[0] + v1[1] * v1[1]),
                     fabs(v1[0]), fabs(v1[1]), fabs(v1[2]),
                     sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]),
                     sqrt(a[0] * a[0] + a[1] * a[1]),
                     a[0], a[1], a[2],
                     sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]),
                     sqrt(d[0] * d[0] + d[1] * d[1]),
                     fabs(d[0]), fabs(d[1]), fabs(d[2])};
  float *pg = q.pg + (long long)shot * 15 * nij + ij;
#pragma unroll
  for (int n = 0; n < 15; n++)
    if (pg[n * nij] < (float)val[n]) pg[n * nij] = (float)val[n];
}

template <typename R>
int launch_peak_motion(const PgPT<R> &q, cudaStream_t st) {
  const long long n = (long long)q.ni * q.nj * q.nshot;
  k_peak_motion<R><<<(unsigned)((n + 255) / 256), 256, 0, st>>>(q);
  return 1;
}
template int launch_peak_motion<float>(const PgPT<float> &, cudaStream_t);
template int launch_peak_motion<double>(const PgPT<double> &, cudaStream_t);

template <typename R>
__global__ void k_gather_box(const R *__restrict__ w, long long sf, long long sx, long long sz, long long off0,
                             int3 start, int3 count, int3 stride, float *__restrict__ dst) {
  const long long per = (long long)count.x * count.y * count.z;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < 9 * per; t += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(t / per);
    const long long r = t % per;
    const int i = start.x + (int)(r % count.x) * stride.x;
    const int j = start.y + (int)((r / count.x) % count.y) * stride.y;
    const int k = start.z + (int)(r / ((long long)count.x * count.y)) * stride.z;
    dst[t] = (float)w[c * sf + off0 + (long long)k * sz + (long long)j * sx + i];
  }
}

template <typename R>
void launch_gather_box(const R *w, long long sf, long long sx, long long sz, long long off0, const int start[3],
                       const int count[3], const int stride[3], float *dst, cudaStream_t st) {
  k_gather_box<R><<<592, 256, 0, st>>>(w, sf, sx, sz, off0, make_int3(start[0], start[1], start[2]),
                                       make_int3(count[0], count[1], count[2]),
                                       make_int3(stride[0], stride[1], stride[2]), dst);
}
template void launch_gather_box<float>(const float *, long long, long long, long long, long long, const int[3],
                                       const int[3], const int[3], float *, cudaStream_t);
template void launch_gather_box<double>(const double *, long long, long long, long long, long long, const int[3],
                                        const int[3], const int[3], float *, cudaStream_t);

template <typename R>
__global__ void k_slices(const __grid_constant__ SliceP<R> q) {
  const int it = *q.d_it;
  const long long total = q.per_shot * q.nshot;
  const long long px = (long long)q.nk * q.nj, py = (long long)q.nk * q.ni, pz = (long long)q.nj * q.ni;
  const long long ex = 9 * px * q.nxs, ey = 9 * py * q.nys;
  float *out = q.ring + (long long)(it % q.ring_steps) * total;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    const int shot = (int)(t / q.per_shot);
    long long r = t % q.per_shot;
    int i, j, k, c;
    if (r < ex) {  // x slice: [s][c][k][j]
      const int s = (int)(r / (9 * px));
      r %= 9 * px;
      c = (int)(r / px);
      k = (int)((r % px) / q.nj);
      j = (int)(r % q.nj);
      i = q.idx[s];
    } else if (r < ex + ey) {  // y slice: [s][c][k][i]
      r -= ex;
      const int s = (int)(r / (9 * py));
      r %= 9 * py;
      c = (int)(r / py);
      k = (int)((r % py) / q.ni);
      i = (int)(r % q.ni);
      j = q.idx[q.nxs + s];
    } else {  // z slice: [s][c][j][i]
      r -= ex + ey;
      const int s = (int)(r / (9 * pz));
      r %= 9 * pz;
      c = (int)(r / pz);
      j = (int)((r % pz) / q.ni);
      i = (int)(r % q.ni);
      k = q.idx[q.nxs + q.nys + s];
    }
    out[t] = (float)q.pre[((long long)shot * 9 + c) * q.sf + q.off0 + (long long)k * q.sz + (long long)j * q.sx + i];
  }
}

template <typename R>
int launch_slices(const SliceP<R> &q, cudaStream_t st) {
  if (q.per_shot <= 0) return 0;
  const long long total = q.per_shot * q.nshot;
  const int blocks = (int)std::min<long long>((total + 255) / 256, 148 * 8);
  k_slices<R><<<blocks, 256, 0, st>>>(q);
  return 1;
}
template int launch_slices<float>(const SliceP<float> &, cudaStream_t);
template int launch_slices<double>(const SliceP<double> &, cudaStream_t);

__global__ void k_advance(int *d_it) {
  if (threadIdx.x == 0 && blockIdx.x == 0) *d_it += 1;
}

// Repack one field from the reference host layout (3 ghosts, nx = ni+6) into the device
// layout. mode 1 converts density to 1/rho (md_rho_to_slow, md_t.cu:622-637).
template <typename R>
__global__ void k_repack_in(const float *__restrict__ src, R *__restrict__ dst, int ni, int nj, int nk,
                            long long sx, long long sz, long long off0, int mode, int ghosts) {
  const long long nxr = ni + 6, nyr = nj + 6;
  const long long total = nxr * nyr * (nk + 6);
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    int ir = (int)(t % nxr), jr = (int)((t / nxr) % nyr), kr = (int)(t / (nxr * nyr));
    int i = ir - 3, j = jr - 3, k = kr - 3;
    bool inner = i >= 0 && i < ni && j >= 0 && j < nj && k >= 0 && k < nk;
    if (!ghosts && !inner) continue;
    float v = src[t];
    if (mode == 1) v = v > 1e-10f ? 1.0f / v : 0.0f;  // 1/rho in float, as md_rho_to_slow
    dst[off0 + (long long)k * sz + (long long)j * sx + i] = (R)v;
  }
}

template <typename R>
__global__ void k_repack_out(const R *__restrict__ src, float *__restrict__ dst, int ni, int nj, int nk,
                             long long sx, long long sz, long long off0) {
  const long long nxr = ni + 6, nyr = nj + 6;
  const long long total = nxr * nyr * (nk + 6);
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    int ir = (int)(t % nxr), jr = (int)((t / nxr) % nyr), kr = (int)(t / (nxr * nyr));
    int i = ir - 3, j = jr - 3, k = kr - 3;
    bool inner = i >= 0 && i < ni && j >= 0 && j < nj && k >= 0 && k < nk;
    dst[t] = inner ? (float)src[off0 + (long long)k * sz + (long long)j * sx + i] : 0.0f;
  }
}

// -----------------------------------------------------------------------------------------
// launch tables
// -----------------------------------------------------------------------------------------
template <int MED, typename R>
static void launch_bulk_med(const StagePT<R> &p, int nzc, dim3 grid, cudaStream_t st) {
  const int code = p.dir[0] | (p.dir[1] << 1) | (p.dir[2] << 2);
  dim3 block(TX, TY);
  constexpr int B = DirectTile<R>::BYTES;
  // above 48 KB of dynamic shared memory each instantiation needs the opt-in once
  static bool attr_done[8] = {};
  switch (code) {
#define CASE(c)                                                                                          \
  case c:                                                                                                \
    if (B > 48 * 1024 && !attr_done[c]) {                                                                \
      cudaFuncSetAttribute(k_stage_bulk<MED, (c)&1, ((c) >> 1) & 1, ((c) >> 2) & 1, R>,                  \
                           cudaFuncAttributeMaxDynamicSharedMemorySize, B);                              \
      attr_done[c] = true;                                                                               \
    }                                                                                                    \
    k_stage_bulk<MED, (c)&1, ((c) >> 1) & 1, ((c) >> 2) & 1, R><<<grid, block, B, st>>>(p, nzc);       \
    break;
    CASE(0) CASE(1) CASE(2) CASE(3) CASE(4) CASE(5) CASE(6) CASE(7)
#undef CASE
  }
}

template <typename R>
int launch_stage_bulk(int med, const StagePT<R> &p, int nzc, cudaStream_t st) {
  if (p.nbulk <= 0) return 0;
  dim3 grid((p.ni + TX - 1) / TX, (p.nj + TY - 1) / TY, (p.nbulk + nzc - 1) / nzc);
  if (med == MED_ISO) launch_bulk_med<MED_ISO>(p, nzc, grid, st);
  else if (med == MED_VTI) launch_bulk_med<MED_VTI>(p, nzc, grid, st);
  else launch_bulk_med<MED_ANISO>(p, nzc, grid, st);
  return 1;
}
template int launch_stage_bulk<float>(int, const StagePT<float> &, int, cudaStream_t);
template int launch_stage_bulk<double>(int, const StagePT<double> &, int, cudaStream_t);

template <int MED, typename TC, int WP>
static void launch_surface_med(const StagePT<real_of<TC>> &p, dim3 grid, dim3 block, cudaStream_t st) {
  switch (p.dir[0] | (p.dir[1] << 1) | (p.dir[2] << 2)) {
#define CASE(c)                                                                                          \
  case c:                                                                                                \
    k_stage_surface<MED, TC, WP, (c)&1, ((c) >> 1) & 1, ((c) >> 2) & 1><<<grid, block, 0, st>>>(p);      \
    break;
    CASE(0) CASE(1) CASE(2) CASE(3) CASE(4) CASE(5) CASE(6) CASE(7)
#undef CASE
  }
}

template <typename TC, int WP>
static void launch_surface_tc(int med, const StagePT<real_of<TC>> &p, dim3 grid, dim3 block, cudaStream_t st) {
  if (med == MED_ISO) launch_surface_med<MED_ISO, TC, WP>(p, grid, block, st);
  else if (med == MED_VTI) launch_surface_med<MED_VTI, TC, WP>(p, grid, block, st);
  else launch_surface_med<MED_ANISO, TC, WP>(p, grid, block, st);
}

template <typename TC, int WP>
static void launch_flux_tc(const StagePT<real_of<TC>> &p, cudaStream_t st) {
  const long long total = (long long)(p.ni + 6) * (p.nj + 6) * kFluxPlanes * p.nshot;
  const int blocks = (int)std::min<long long>((total + 255) / 256, 148 * 8);
  k_timg_flux<TC, WP><<<blocks, 256, 0, st>>>(p);
}

int launch_timg_flux(int coef_type, int wave16, const StageP &p, cudaStream_t st) {
  if (!p.free_top || !p.flux) return 0;
  if (wave16) {
    if (p.stage == 0) launch_flux_tc<uint16_t, 1>(p, st);
    else launch_flux_tc<uint16_t, 2>(p, st);
  } else if (coef_type == COEF_U16) launch_flux_tc<uint16_t, 0>(p, st);
  else if (coef_type == COEF_F16) launch_flux_tc<__half, 0>(p, st);
  else if (coef_type == COEF_BF16) launch_flux_tc<__nv_bfloat16, 0>(p, st);
  else launch_flux_tc<float, 0>(p, st);
  return 1;
}

int launch_timg_flux64(const StagePT<double> &p, cudaStream_t st) {
  if (!p.free_top || !p.flux) return 0;
  launch_flux_tc<double, 0>(p, st);
  return 1;
}

int launch_stage_surface(int med, int coef_type, int wave16, const StageP &p, cudaStream_t st) {
  if (p.nbulk >= p.nk) return 0;
  dim3 block(32, 2, NSURF);
  dim3 grid((p.ni + 31) / 32, (p.nj + 1) / 2, p.nshot);
  if (wave16) {
    if (p.stage == 0) launch_surface_tc<uint16_t, 1>(med, p, grid, block, st);
    else launch_surface_tc<uint16_t, 2>(med, p, grid, block, st);
  } else if (coef_type == COEF_U16) launch_surface_tc<uint16_t, 0>(med, p, grid, block, st);
  else if (coef_type == COEF_F16) launch_surface_tc<__half, 0>(med, p, grid, block, st);
  else if (coef_type == COEF_BF16) launch_surface_tc<__nv_bfloat16, 0>(med, p, grid, block, st);
  else launch_surface_tc<float, 0>(med, p, grid, block, st);
  return 1;
}

int launch_stage_surface64(int med, const StagePT<double> &p, cudaStream_t st) {
  if (p.nbulk >= p.nk) return 0;
  dim3 block(32, 2, NSURF);
  dim3 grid((p.ni + 31) / 32, (p.nj + 1) / 2, p.nshot);
  launch_surface_tc<double, 0>(med, p, grid, block, st);
  return 1;
}

// Scale of the FP16 stage levels for this step: max |w| at the step's start (collected by
// the last step's stage 3) and the largest source increment of this step, mapped by a power
// of two into [2^12, 2^13); FP16 then holds 8x-16x growth within the step before its
// largest finite value. Then clears the collector for this step's stage 3.
// One scale per shot and group: shots of a batch round exactly as when run alone.
__global__ void k_wave_scale(unsigned int *amax, const float *srcb, const int *d_it, int nt_total, int nshot,
                             float *wsc_all) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 2 * nshot) return;
  const int shot = t >> 1, g = t & 1;
  float *wsc = wsc_all + 18 * shot;
  const int it = *d_it;
  float m = __uint_as_float(amax[t]);
  if (srcb && it >= 0 && it < nt_total) m = fmaxf(m, srcb[((long long)it * nshot + shot) * 2 + g]);
  int e = 0;
  if (m > 0.f && m <= 3.0e38f) {
    e = (int)((__float_as_uint(m) >> 23) & 0xff) - 127 - 12;  // exponent of m (m normal)
    if (m < 1.1754944e-38f) e = -126 - 12;
  }
  e = max(-100, min(100, e));
  const float sc = __uint_as_float((unsigned)(e + 127) << 23), inv = __uint_as_float((unsigned)(127 - e) << 23);
  for (int f = g ? 3 : 0; f < (g ? 9 : 3); f++) {
    wsc[f] = sc;
    wsc[9 + f] = inv;
  }
  amax[t] = 0u;
}

int launch_wave_scale(unsigned int *amax, const float *srcb, const int *d_it, int nt_total, int nshot, float *wsc,
                      cudaStream_t st) {
  k_wave_scale<<<(2 * nshot + 127) / 128, 128, 0, st>>>(amax, srcb, d_it, nt_total, nshot, wsc);
  return 1;
}

__global__ void k_wave_absmax(const float *__restrict__ w, long long sf, unsigned int *amax) {
  const long long n = 9 * sf;
  float vm = 0.f, sm = 0.f;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const int f = (int)((t / sf) % 9);
    if (f < 3) vm = fmaxf(vm, fabsf(w[t]));
    else sm = fmaxf(sm, fabsf(w[t]));
  }
  for (int o = 16; o; o >>= 1) {
    vm = fmaxf(vm, __shfl_xor_sync(0xffffffffu, vm, o));
    sm = fmaxf(sm, __shfl_xor_sync(0xffffffffu, sm, o));
  }
  if ((threadIdx.x & 31) == 0) {
    atomic_max_abs(&amax[0], vm);
    atomic_max_abs(&amax[1], sm);
  }
}

// One mbarrier wait that no transfer completes, bounded by `polls`: the stage kernels' wait
// path on a lost TMA transfer (records the pipeline-timeout bit in *err and returns).
__global__ void k_wait_bound_check(int *err, int polls) {
  __shared__ __align__(8) uint64_t bar;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    fence_barrier_init();
  }
  __syncthreads();
  if (threadIdx.x == 0) mbar_wait(&bar, 0, err, polls);
}

int launch_wait_bound_check(int *err, int polls, cudaStream_t st) {
  k_wait_bound_check<<<1, 32, 0, st>>>(err, polls);
  return 1;
}

void launch_wave_absmax(const float *w, long long sf, int nshot, unsigned int *amax, cudaStream_t st) {
  for (int s = 0; s < nshot; s++) k_wave_absmax<<<1184, 256, 0, st>>>(w + (size_t)s * 9 * sf, sf, amax + 2 * s);
}

// Convert one FP32 coefficient field to 16 bits (value = scale * stored + offset) by
// stochastic rounding: each cell rounds up or down with the probabilities that make the
// stored value exact on average, the draw a fixed hash of (field, cell). Round-to-nearest
// would give every cell of a homogeneous layer the same error, i.e. a systematic shift of
// the layer's wave speed whose phase error grows with travel time; stochastic rounding
// leaves zero-mean cell-scale noise that the wave averages over a wavelength.
__device__ __forceinline__ unsigned int mix32(unsigned int h) {  // murmur3 finaliser
  h ^= h >> 16;
  h *= 0x85ebca6bu;
  h ^= h >> 13;
  h *= 0xc2b2ae35u;
  h ^= h >> 16;
  return h;
}

template <typename TC>
__global__ void k_coef_to16(const float *__restrict__ src, TC *__restrict__ dst, long long n, float scale,
                            float offset, unsigned int field) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const unsigned int hsh = mix32((unsigned int)t ^ mix32((unsigned int)(t >> 32) + 0x9e3779b9u * (field + 1)));
    const float u = (float)(hsh >> 8) * (1.0f / 16777216.0f);  // [0, 1)
    if constexpr (std::is_same<TC, uint16_t>::value) {
      // fixed point over the field's [min, max]; cells outside it (padding) clamp
      const float q = (src[t] - offset) / scale;
      float fl = floorf(q);
      if (u < q - fl) fl += 1.f;
      dst[t] = (uint16_t)fminf(fmaxf(fl, 0.f), 65535.f);
    } else {
      const float v = src[t] / scale;
      TC lo;
      if constexpr (std::is_same<TC, __half>::value) lo = __float2half_rz(v);
      else lo = __float2bfloat16_rz(v);
      const float flo = to_f(lo);
      if (flo != v && isfinite(v)) {
        TC hi;
        unsigned short bits;
        memcpy(&bits, &lo, 2);
        bits += 1;  // next representable value away from zero (sign-magnitude)
        memcpy(&hi, &bits, 2);
        const float fhi = to_f(hi);
        if (u < (v - flo) / (fhi - flo)) lo = hi;
      }
      dst[t] = lo;
    }
  }
}

// order-preserving key of a float (unsigned compare of keys = float compare)
__device__ __forceinline__ unsigned int fkey(float f) {
  const unsigned int b = __float_as_uint(f);
  return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}

float coef_key_to_float(unsigned int k) {
  unsigned int b = (k & 0x80000000u) ? (k & 0x7fffffffu) : ~k;
  float f;
  memcpy(&f, &b, 4);
  return f;
}

__global__ void k_coef_minmax(const float *__restrict__ src, int ni, int nj, int nk, long long sx, long long sz,
                              long long off0, unsigned int *out) {
  const int nx = ni + 6, ny = nj + 6;
  const long long n = (long long)nx * ny * (nk + 6);
  unsigned int mn = 0xffffffffu, mx = 0u;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(t % nx) - 3, j = (int)((t / nx) % ny) - 3, k = (int)(t / ((long long)nx * ny)) - 3;
    const unsigned int key = fkey(src[off0 + (long long)k * sz + (long long)j * sx + i]);
    mn = min(mn, key);
    mx = max(mx, key);
  }
  for (int o = 16; o; o >>= 1) {
    mn = min(mn, __shfl_xor_sync(0xffffffffu, mn, o));
    mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMin(&out[0], mn);
    atomicMax(&out[1], mx);
  }
}

void launch_coef_minmax(const float *src, int ni, int nj, int nk, long long sx, long long sz, long long off0,
                        unsigned int *out, cudaStream_t st) {
  k_coef_minmax<<<592, 256, 0, st>>>(src, ni, nj, nk, sx, sz, off0, out);
}

__global__ void k_absmax(const float *__restrict__ src, long long n, unsigned int *out) {
  float m = 0.f;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x)
    m = fmaxf(m, fabsf(src[t]));
  for (int o = 16; o; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, __float_as_uint(m));  // non-negative floats order as uints
}

void launch_absmax(const float *src, long long n, unsigned int *out, cudaStream_t st) {
  k_absmax<<<592, 256, 0, st>>>(src, n, out);
}

void launch_coef_to16(int coef_type, const float *src, void *dst, long long n, float scale, float offset, int field,
                      cudaStream_t st) {
  if (coef_type == COEF_U16)
    k_coef_to16<uint16_t><<<1184, 256, 0, st>>>(src, (uint16_t *)dst, n, scale, offset, field);
  else if (coef_type == COEF_F16)
    k_coef_to16<__half><<<1184, 256, 0, st>>>(src, (__half *)dst, n, scale, offset, field);
  else
    k_coef_to16<__nv_bfloat16><<<1184, 256, 0, st>>>(src, (__nv_bfloat16 *)dst, n, scale, offset, field);
}

template <typename R>
int launch_source(const SrcPT<R> &s, cudaStream_t st) {
  if (s.nsrc <= 0) return 0;
  dim3 block(128);
  dim3 grid((s.max_ext + 127) / 128, s.nsrc);
  k_source<R><<<grid, block, 0, st>>>(s);
  return 1;
}
template int launch_source<float>(const SrcPT<float> &, cudaStream_t);
template int launch_source<double>(const SrcPT<double> &, cudaStream_t);

template <typename R>
int launch_recv(const RecvPT<R> &r, cudaStream_t st) {
  if (r.nsta <= 0) return 0;
  int n = r.nshot * r.nsta * 9;
  k_recv<R><<<(n + 127) / 128, 128, 0, st>>>(r);
  return 1;
}
template int launch_recv<float>(const RecvPT<float> &, cudaStream_t);
template int launch_recv<double>(const RecvPT<double> &, cudaStream_t);

int launch_advance(int *d_it, cudaStream_t st) {
  k_advance<<<1, 32, 0, st>>>(d_it);
  return 1;
}

template <typename R>
void launch_repack_in(const float *src, R *dst, int ni, int nj, int nk, long long sx, long long sz, long long off0,
                      int mode, int ghosts, cudaStream_t st) {
  k_repack_in<R><<<1184, 256, 0, st>>>(src, dst, ni, nj, nk, sx, sz, off0, mode, ghosts);
}
template void launch_repack_in<float>(const float *, float *, int, int, int, long long, long long, long long, int, int,
                                      cudaStream_t);
template void launch_repack_in<double>(const float *, double *, int, int, int, long long, long long, long long, int,
                                       int, cudaStream_t);

template <typename R>
void launch_repack_out(const R *src, float *dst, int ni, int nj, int nk, long long sx, long long sz, long long off0,
                       cudaStream_t st) {
  k_repack_out<R><<<1184, 256, 0, st>>>(src, dst, ni, nj, nk, sx, sz, off0);
}
template void launch_repack_out<float>(const float *, float *, int, int, int, long long, long long, long long,
                                       cudaStream_t);
template void launch_repack_out<double>(const double *, float *, int, int, int, long long, long long, long long,
                                        cudaStream_t);

}  // namespace cgfd

// cgfd_dev.cuh -- device-side building blocks of the fused RK-stage kernels.
//
// One RK stage of the reference (sv_curv_col_el_*_onestage + wav_update/wav_update_end,
// drv_rk_curv_col.cu:263-491) becomes, per grid cell and in one pass over HBM:
//   27 one-sided 5-point MacCormack derivatives (fd_t.cu:90-114 coefficients),
//   momentum + Hooke (iso / VTI / 21-Cij), the CFS-PML correction and auxiliary-variable
//   update of every face that contains the cell, and the RK4 combine of the wavefield and
//   of the PML auxiliaries (tmp = pre + a*dt*rhs, end (+)= b*dt*rhs).
// The RHS itself never reaches HBM.
#pragma once

#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <type_traits>

namespace cgfd {

// Planes below the top whose traction-image fluxes the surface slab reads (the image's z
// stencil reaches 4 planes below the top one).
constexpr int kFluxPlanes = 5;

// Thread-block tile of the z-marching kernel (x fastest).
constexpr int TX = 32;
constexpr int TY = 8;
// Ghost offset along x in the device layout: the physical row starts on a 128-byte line.
constexpr int GX = 32;
// Planes below the top processed by the surface-slab kernel when the free surface is on:
// the traction image rewrites up to 4 layers, vlow 3 (sv_curv_col_el_iso_gpu.cu:212-249).
constexpr int NSURF = 4;

// elastic media; MED_AC: acoustic (fields Vx Vy Vz P, P in the Txx slot; cgfd_acoustic.cu)
enum { MED_ISO = 0, MED_VTI = 1, MED_ANISO = 2, MED_AC = 3 };

// Coefficient fields in the device coefficient array, in this order:
//   0..8  xi_x xi_y xi_z eta_x eta_y eta_z zeta_x zeta_y zeta_z
//   9     1/rho
//   10..  iso: lambda mu | vti: c11 c13 c33 c55 c66 | aniso: c11 c12 .. c66 (21, row-major upper)
//         | acoustic: kappa
constexpr int CF_SLW = 9;
constexpr int CF_MED = 10;
template <int MED> struct MedInfo;
template <> struct MedInfo<MED_ISO>   { static constexpr int NCOEF = 12; };
template <> struct MedInfo<MED_VTI>   { static constexpr int NCOEF = 15; };
template <> struct MedInfo<MED_ANISO> { static constexpr int NCOEF = 31; };
template <> struct MedInfo<MED_AC>    { static constexpr int NCOEF = 11; };

// Real type R of the stored solution, coefficients and arithmetic: float (the reference's
// precision, every production mode) or double (the FP64 build, CGFD_PREC_FP64).

// One CFS-PML face (bdry_t.cu:85-257): box [lo,hi] in physical indices, 1-D A/B/D along the
// face normal, and the 9-component auxiliary variables (component stride n) at the levels
// this stage reads and writes.
template <typename R>
struct FacePT {
  int enable;
  int axis;           // 0 x, 1 y, 2 z
  int lo[3], hi[3];   // inclusive box, physical 0-based indices
  int nx, ny;         // box extents along x, y
  long long n;        // points in the box
  const R *A, *B, *D;
  // each level holds nshot x 9 components (shot stride 9 n)
  const R *aux_cur;   // level read by the RHS (pre at stage 0, tmp otherwise)
  const R *aux_pre;   // pre level (stages 1-2)
  R *aux_tmp;         // tmp level written at stages 0-2 (== aux_cur at stages 1-2)
  R *aux_end;         // end level
};
using FaceP = FacePT<float>;

template <typename R>
struct StagePT {
  int ni, nj, nk;
  int stage;              // 0..3
  int dir[3];             // 0 backward, 1 forward (fd_t.cu:184-235)
  long long sx, sz, sf;   // row, plane and field strides of the device layout (floats)
  long long off0;         // offset of physical point (0,0,0)
  const R *cur;           // wavefield read by the stencils (9 fields); __half when the
                          // FP16 stage levels are the input (stages 1-3)
  const R *pre;           // w_pre (stages 1-2)
  R *tmp_out;             // next stage input (stages 0-2); __half in FP16-stage mode
  R *end;                 // accumulator (written at every stage)
  R *rhs;                 // non-null (visco-elastic media): the wave fields' right-hand side
                          // [9][sf] is written here instead of the RK combine (PML auxiliaries
                          // are still combined); the attenuation pass combines them
  R ca, cb;               // rk_a[stage]*dt, rk_b[stage]*dt
  const void *coef;       // [ncoef][sf] of R, __half, __nv_bfloat16 or uint16_t
  float cscale[32];       // 16-bit coefficients: value = cscale[f] * stored + coffset[f]
  float coffset[32];
  const R *jac;           // [sf]
  const R *matx;          // free surface: [nj][ni][9] matVx2Vz (row-major 3x3)
  const R *maty;          //                [nj][ni][9] matVy2Vz
  int free_top;
  // traction-image fluxes of the stage input (free surface): flux[shot][9][kFluxPlanes][nj+6][ni+6],
  // component 3c + a = jac (metric row a . stress row c) at planes nk-kFluxPlanes .. nk-1,
  // ghost columns included
  R *flux;
  int nbulk;              // planes [0, nbulk) belong to the bulk kernel
  int nface;
  FacePT<R> face[6];
  int *err;               // device error word: kErrStationNonfinite, kErrPipelineTimeout, kErrWaveNonfinite
  int nshot;              // wavefields sharing this grid (batched sources); 1 = plain
  // FP16 stage levels, per shot s: wsc[18s + 0..8] scale (value = scale * stored),
  // wsc[18s + 9..17] its inverse, fixed for one time step; amax[2s + 0..1] collects max |w|
  // of the velocity / stress fields written at stage 3 (the next step's scale)
  const float *wsc;
  unsigned int *amax;
};
using StageP = StagePT<float>;

// max |w| groups of the FP16 stage levels: velocity (fields 0-2) and stress (3-8)
__host__ __device__ constexpr int wgroup(int f) { return f < 3 ? 0 : 1; }

// Tensor maps of the arrays one stage streams through TMA: the stage input (4-D box with
// the x-y halo, all 9 fields), w_pre / w_end (centre boxes, 9 fields), coefficients.
struct TmaP {
  CUtensorMap cur, pre, end, coef;
};

// ---------------------------------------------------------------------------------------
// MacCormack DRP operator (fd_t.cu:90-93, 111-114): backward uses offsets -3..+1,
// forward -1..+3. The 5 samples are passed in increasing position.
// ---------------------------------------------------------------------------------------
// (the coefficients are the reference's float values, in either real type)
template <int DIR, typename R>
__device__ __forceinline__ R drp5(R a0, R a1, R a2, R a3, R a4) {
  if (DIR == 0)
    return R(-0.041686285f) * a0 + R(0.333411808f) * a1 - R(1.250117713f) * a2 + R(0.666745142f) * a3 +
           R(0.291647047f) * a4;
  else
    return R(-0.291647047f) * a0 - R(0.666745142f) * a1 + R(1.250117713f) * a2 - R(0.333411808f) * a3 +
           R(0.041686285f) * a4;
}
template <typename R>
__device__ __forceinline__ R drp5r(int dir, R a0, R a1, R a2, R a3, R a4) {
  return dir ? drp5<1>(a0, a1, a2, a3, a4) : drp5<0>(a0, a1, a2, a3, a4);
}
// left extent of the operator
__host__ __device__ constexpr int op_left(int dir) { return dir ? 1 : 3; }

// Voigt index of (a,b): xx yy zz yz xz xy == wavefield components 3..8 minus 3.
__host__ __device__ constexpr int voigt(int a, int b) {
  return a == b ? a : (a + b == 3 ? 3 : (a + b == 2 ? 4 : 5));
}

// ---------------------------------------------------------------------------------------
// Hooke's law from the velocity gradient G[vi][xj] = dV_vi/dx_j, per medium.
// ---------------------------------------------------------------------------------------
template <int MED, typename R = float>
struct Medium;

template <typename R>
struct Medium<MED_ISO, R> {
  R lam, mu, lam2mu;
  template <typename G>
  __device__ __forceinline__ void load(G get) {  // get(c): coefficient field c at the cell
    lam = get(CF_MED + 0);
    mu = get(CF_MED + 1);
    lam2mu = lam + R(2) * mu;
  }
  __device__ __forceinline__ void hooke(const R G[3][3], R h[6]) const {
    h[0] = lam2mu * G[0][0] + lam * (G[1][1] + G[2][2]);
    h[1] = lam2mu * G[1][1] + lam * (G[0][0] + G[2][2]);
    h[2] = lam2mu * G[2][2] + lam * (G[0][0] + G[1][1]);
    h[3] = mu * (G[1][2] + G[2][1]);
    h[4] = mu * (G[0][2] + G[2][0]);
    h[5] = mu * (G[0][1] + G[1][0]);
  }
};

template <typename R>
struct Medium<MED_VTI, R> {
  R c11, c12, c13, c33, c55, c66;
  template <typename G>
  __device__ __forceinline__ void load(G get) {
    c11 = get(CF_MED + 0);
    c13 = get(CF_MED + 1);
    c33 = get(CF_MED + 2);
    c55 = get(CF_MED + 3);
    c66 = get(CF_MED + 4);
    c12 = c11 - R(2) * c66;  // sv_curv_col_el_vti_gpu.cu:407
  }
  __device__ __forceinline__ void hooke(const R G[3][3], R h[6]) const {
    h[0] = c11 * G[0][0] + c12 * G[1][1] + c13 * G[2][2];
    h[1] = c12 * G[0][0] + c11 * G[1][1] + c13 * G[2][2];
    h[2] = c13 * (G[0][0] + G[1][1]) + c33 * G[2][2];
    h[3] = c55 * (G[1][2] + G[2][1]);
    h[4] = c55 * (G[0][2] + G[2][0]);
    h[5] = c66 * (G[0][1] + G[1][0]);
  }
};

template <typename R>
struct Medium<MED_ANISO, R> {
  R c[21];  // c11 c12 c13 c14 c15 c16 c22 .. c66 (upper triangle, row-major)
  template <typename G>
  __device__ __forceinline__ void load(G get) {
#pragma unroll
    for (int n = 0; n < 21; n++) c[n] = get(CF_MED + n);
  }
  __device__ __forceinline__ static constexpr int up(int a, int b) {
    // index of C[a][b] (a<=b) in the packed upper triangle
    return a * 6 - a * (a - 1) / 2 + (b - a);
  }
  __device__ __forceinline__ R C(int a, int b) const { return a <= b ? c[up(a, b)] : c[up(b, a)]; }
  __device__ __forceinline__ void hooke(const R G[3][3], R h[6]) const {
    R e[6] = {G[0][0], G[1][1], G[2][2], G[1][2] + G[2][1], G[0][2] + G[2][0], G[0][1] + G[1][0]};
#pragma unroll
    for (int I = 0; I < 6; I++) {
      R s = C(I, 0) * e[0];
#pragma unroll
      for (int J = 1; J < 6; J++) s += C(I, J) * e[J];
      h[I] = s;
    }
  }
};

// 16-bit storage: value = per-field scale x stored value (FP32 arithmetic)
__device__ __forceinline__ float to_f(float x) { return x; }
__device__ __forceinline__ double to_f(double x) { return x; }
__device__ __forceinline__ float to_f(__half x) { return __half2float(x); }
__device__ __forceinline__ float to_f(__nv_bfloat16 x) { return __bfloat162float(x); }
__device__ __forceinline__ float to_f(uint16_t x) { return (float)x; }
template <typename T>
__device__ __forceinline__ T from_f(float x);
template <>
__device__ __forceinline__ float from_f<float>(float x) { return x; }
template <>
__device__ __forceinline__ __half from_f<__half>(float x) { return __float2half_rn(x); }

// non-negative float maximum through the integer atomic (order of non-negative floats is
// the order of their bit patterns)
__device__ __forceinline__ void atomic_max_abs(unsigned int *a, float v) {
  atomicMax(a, __float_as_uint(fabsf(v)));
}

// Real type the kernels compute in for coefficient storage TC: double for the FP64 build,
// float otherwise.
template <typename TC>
using real_of = typename std::conditional<std::is_same<TC, double>::value, double, float>::type;

// decode of one stored coefficient of field c
template <typename TC, typename P>
__device__ __forceinline__ real_of<TC> coef_decode(TC v, const P &p, int c) {
  if constexpr (std::is_same<TC, float>::value || std::is_same<TC, double>::value) return v;
  else return fmaf(p.cscale[c], to_f(v), p.coffset[c]);
}

template <typename TC>
struct CoefView {
  using P = StagePT<real_of<TC>>;
  const TC *base;
  long long stride;
  const P &p;
  __device__ __forceinline__ CoefView(const P &p_) : base(static_cast<const TC *>(p_.coef)), stride(p_.sf), p(p_) {}
  __device__ __forceinline__ real_of<TC> operator()(int c, long long idx) const {
    return coef_decode<TC>(__ldg(base + c * stride + idx), p, c);
  }
};

// momentum of one axis: sum_j m[j] * dT_(vi,j) / d(axis)
template <typename R>
__device__ __forceinline__ void momentum_axis(const R m[3], const R dt[6], R mom[3]) {
  mom[0] = m[0] * dt[0] + m[1] * dt[5] + m[2] * dt[4];
  mom[1] = m[0] * dt[5] + m[1] * dt[1] + m[2] * dt[3];
  mom[2] = m[0] * dt[4] + m[1] * dt[3] + m[2] * dt[2];
}

// ---------------------------------------------------------------------------------------
// Per-cell state carried from the derivative phase to the store phase.
// ---------------------------------------------------------------------------------------
template <typename R = float>
struct CellAcc {
  R G[3][3];   // velocity gradient
  R mom[3];    // divergence of stress (before 1/rho)
  R hc[9];     // sum of PML corrections
  __device__ __forceinline__ void zero() {
#pragma unroll
    for (int a = 0; a < 3; a++) {
      mom[a] = R(0);
#pragma unroll
      for (int b = 0; b < 3; b++) G[a][b] = R(0);
    }
#pragma unroll
    for (int c = 0; c < 9; c++) hc[c] = R(0);
  }
  // accumulate the derivatives of one axis with metric row m
  __device__ __forceinline__ void add_axis(const R m[3], const R dv[3], const R dt[6]) {
#pragma unroll
    for (int vi = 0; vi < 3; vi++)
#pragma unroll
      for (int xj = 0; xj < 3; xj++) G[vi][xj] += m[xj] * dv[vi];
    R mm[3];
    momentum_axis(m, dt, mm);
    mom[0] += mm[0]; mom[1] += mm[1]; mom[2] += mm[2];
  }
};

// Bits of the problem's device error word (reported by cgfd_synchronize).
constexpr int kErrStationNonfinite = 1;  // a station sample is NaN/Inf
constexpr int kErrWaveNonfinite = 4;     // the RK combine produced a NaN/Inf solution value

// true when v is NaN or +-Inf (a NaN compares false)
__device__ __forceinline__ bool nonfinite(float v) { return !(fabsf(v) <= 3.402823466e38f); }
__device__ __forceinline__ bool nonfinite(double v) { return !(fabs(v) <= 1.7976931348623157e308); }

// RK combine of N values at one point (wav_update / wav_update_end, wav_t.cu:362-378): the 9
// elastic components, or the 4 acoustic ones (Vx Vy Vz P).
// cur_c: the stage input at the point (== pre at stage 0). err (may be null): at stage 3,
// a non-finite new solution value sets kErrWaveNonfinite there -- the blow-up sentinel the
// reference leaves stubbed (drv_rk_curv_col.cu:507-510, wav_check_value wav_t.cu:260-279).
template <int N = 9, typename R>
__device__ __forceinline__ void rk_store(int stage, R ca, R cb, long long comp_stride, long long idx,
                                         const R cur_c[N], const R h[N], const R *pre,
                                         R *tmp_out, R *end, int *err = nullptr) {
  if (stage == 0) {
#pragma unroll
    for (int c = 0; c < N; c++) {
      tmp_out[c * comp_stride + idx] = cur_c[c] + ca * h[c];
      end[c * comp_stride + idx] = cur_c[c] + cb * h[c];
    }
  } else if (stage < 3) {
    R p[N], e[N];
#pragma unroll
    for (int c = 0; c < N; c++) {
      p[c] = __ldg(pre + c * comp_stride + idx);
      e[c] = end[c * comp_stride + idx];
    }
#pragma unroll
    for (int c = 0; c < N; c++) {
      tmp_out[c * comp_stride + idx] = p[c] + ca * h[c];
      end[c * comp_stride + idx] = e[c] + cb * h[c];
    }
  } else {
    R e[N];
    bool bad = false;
#pragma unroll
    for (int c = 0; c < N; c++) e[c] = end[c * comp_stride + idx];
#pragma unroll
    for (int c = 0; c < N; c++) {
      const R v = e[c] + cb * h[c];
      end[c * comp_stride + idx] = v;
      bad |= nonfinite(v);
    }
    if (err && bad) atomicOr(err, kErrWaveNonfinite);
  }
}

// CFS-PML work of one face for one cell (sv_curv_col_el_iso_gpu.cu:680-1147):
//   rhs_d = the 1-D terms of this axis; h += (B-1) rhs_d - B aux; aux' = D rhs_d - A aux,
//   plus the free-surface-converted zeta terms on x/y faces at the top (surf != nullptr),
//   followed by the RK combine of the auxiliary variables.
template <typename T> struct nondeduced { using type = T; };  // keeps nullptr arguments out of deduction

template <int MED, typename R>
__device__ __forceinline__ void pml_face(const StagePT<R> &p, const FacePT<R> &f, int i, int j, int k,
                                         const Medium<MED, R> &md, R slw, const R m[3],
                                         const R dv[3], const R dt[6], const typename nondeduced<R>::type *surf_mat,
                                         const typename nondeduced<R>::type *zeta, R hc[9], int shot = 0) {
  int ab = f.axis == 0 ? i - f.lo[0] : (f.axis == 1 ? j - f.lo[1] : k - f.lo[2]);
  R cA = __ldg(f.A + ab), cB = __ldg(f.B + ab), cD = __ldg(f.D + ab);
  R cB1 = cB - R(1);
  long long ia = (long long)shot * 9 * f.n + ((long long)(k - f.lo[2]) * f.ny + (j - f.lo[1])) * f.nx + (i - f.lo[0]);
  R rhs[9];
  momentum_axis(m, dt, rhs);
  rhs[0] *= slw; rhs[1] *= slw; rhs[2] *= slw;
  {
    R Ga[3][3];
#pragma unroll
    for (int vi = 0; vi < 3; vi++)
#pragma unroll
      for (int xj = 0; xj < 3; xj++) Ga[vi][xj] = m[xj] * dv[vi];
    md.hooke(Ga, rhs + 3);
  }
  R aux[9], arhs[9];
#pragma unroll
  for (int c = 0; c < 9; c++) {
    aux[c] = f.aux_cur[c * f.n + ia];
    hc[c] += cB1 * rhs[c] - cB * aux[c];
    arhs[c] = cD * rhs[c] - cA * aux[c];
  }
  if (surf_mat) {
    // dzV converted from this axis' derivative (sv_curv_col_el_iso_gpu.cu:855-915)
    R dz[3];
#pragma unroll
    for (int r = 0; r < 3; r++) dz[r] = surf_mat[3 * r] * dv[0] + surf_mat[3 * r + 1] * dv[1] + surf_mat[3 * r + 2] * dv[2];
    R Gs[3][3], hs[6];
#pragma unroll
    for (int vi = 0; vi < 3; vi++)
#pragma unroll
      for (int xj = 0; xj < 3; xj++) Gs[vi][xj] = zeta[xj] * dz[vi];
    md.hooke(Gs, hs);
#pragma unroll
    for (int c = 0; c < 6; c++) {
      hc[3 + c] += cB1 * hs[c];
      arhs[3 + c] += cD * hs[c];
    }
  }
  rk_store(p.stage, p.ca, p.cb, f.n, ia, aux, arhs, f.aux_pre, f.aux_tmp, f.aux_end);
}

template <typename R>
__device__ __forceinline__ bool in_face(const FacePT<R> &f, int i, int j, int k) {
  return i >= f.lo[0] && i <= f.hi[0] && j >= f.lo[1] && j <= f.hi[1] && k >= f.lo[2] && k <= f.hi[2];
}


// Index helpers for the device layout.
template <typename R>
__device__ __forceinline__ long long didx(const StagePT<R> &p, int i, int j, int k) {
  return p.off0 + (long long)k * p.sz + (long long)j * p.sx + i;
}

}  // namespace cgfd

// cgfd_setup.cpp -- FP64 host setup of the CGFD3D time loop: CFS-PML coefficients,
// free-surface velocity-gradient conversion, source smoothing and time functions, station
// location, grid metrics and the CFL time-step bound. The results are stored as float for
// the FP32 device path.
#include "cgfd_setup.h"

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <utility>

namespace cgfd {

static const double kPi = 3.1415926535897;  // constants.h:14

int medium_ncmp(int medium_type) {
  switch (medium_type) {
    case CGFD_MEDIUM_ACOUSTIC_ISO: return 2;
    case CGFD_MEDIUM_ELASTIC_ISO: return 3;
    case CGFD_MEDIUM_ELASTIC_VTI: return 6;
    case CGFD_MEDIUM_ELASTIC_ANISO: return 22;
    case CGFD_MEDIUM_VISCO_ISO: return 5;  // rho lambda mu Qp Qs
  }
  return -1;
}

void validate_desc(const cgfd_problem_desc *d) {
  if (!d) throw Error(CGFD_ERR_INVALID, "desc is NULL");
  if (d->ni < 8 || d->nj < 8 || d->nk < 8) throw Error(CGFD_ERR_INVALID, "grid must have at least 8 points per axis");
  if (medium_ncmp(d->medium_type) < 0)
    throw Error(CGFD_ERR_UNSUPPORTED, "medium_type must be acoustic iso, elastic iso/vti/aniso or visco-elastic iso");
  if (d->medium_type == CGFD_MEDIUM_ACOUSTIC_ISO && d->precision != CGFD_PREC_FP32 && d->precision != CGFD_PREC_FP64)
    throw Error(CGFD_ERR_UNSUPPORTED, "acoustic media run in FP32 or FP64 (CGFD_PREC_FP32 / CGFD_PREC_FP64)");
  if (d->medium_type == CGFD_MEDIUM_VISCO_ISO && d->precision != CGFD_PREC_FP32)
    throw Error(CGFD_ERR_UNSUPPORTED, "visco-elastic media run in FP32 (CGFD_PREC_FP32)");
  if (d->medium_type == CGFD_MEDIUM_VISCO_ISO && !d->visco)
    throw Error(CGFD_ERR_INVALID, "visco-elastic media need desc->visco");
  if (!d->medium) throw Error(CGFD_ERR_INVALID, "the medium array is required");
  if (!d->metric && !d->coord) throw Error(CGFD_ERR_INVALID, "coordinates are required when no metric is given");
  if (!(d->dt > 0.0f)) throw Error(CGFD_ERR_INVALID, "dt must be > 0");
  if (d->nt_total < 1) throw Error(CGFD_ERR_INVALID, "nt_total must be >= 1");
  if (d->precision < CGFD_PREC_FP32 || d->precision > CGFD_PREC_FP64)
    throw Error(CGFD_ERR_INVALID, "unknown precision");
  if (d->free_top && d->pml[2][1].enable) throw Error(CGFD_ERR_INVALID, "the top face cannot be both free and PML");
  for (int a = 0; a < 3; a++)
    for (int s = 0; s < 2; s++) {
      const cgfd_pml_face &f = d->pml[a][s];
      if (!f.enable) continue;
      int n = a == 0 ? d->ni : (a == 1 ? d->nj : d->nk);
      if (f.num_layers < 1 || f.num_layers >= n) throw Error(CGFD_ERR_INVALID, "pml num_layers out of range");
      if (!d->coord) throw Error(CGFD_ERR_INVALID, "coord is required when a PML face is enabled");
    }
  if (d->src.num < 0 || d->sta.num < 0) throw Error(CGFD_ERR_INVALID, "negative source/station count");
  if (d->src.num > 0) {
    if (!d->src.loc || !d->src.t_start) throw Error(CGFD_ERR_INVALID, "source loc/t_start missing");
    if (d->src.loc_coord_type != 0 && d->src.loc_coord_type != 1)
      throw Error(CGFD_ERR_INVALID, "loc_coord_type must be 0 (grid index) or 1 (physical coordinates)");
    if (d->src.loc_coord_type == 1 && !d->coord)
      throw Error(CGFD_ERR_INVALID, "coord is required to locate sources by physical coordinates");
    if (d->src.stf_given == 0 && (!d->src.wavelet || !d->src.wavelet_coefs || !d->src.cmp))
      throw Error(CGFD_ERR_INVALID, "wavelet source needs wavelet, wavelet_coefs and cmp");
    if (d->src.stf_given == 1 && (!d->src.cmp_values || d->src.stf_nt < 1 || !(d->src.stf_dt > 0)))
      throw Error(CGFD_ERR_INVALID, "sampled source needs cmp_values, stf_nt and stf_dt");
    if (d->src.stf_given != 0 && d->src.stf_given != 1) throw Error(CGFD_ERR_INVALID, "stf_given must be 0 or 1");
    if (d->src.cmp_type < 1 || d->src.cmp_type > 3) throw Error(CGFD_ERR_INVALID, "cmp_type must be 1, 2 or 3");
  }
  if (d->sta.num > 0) {
    if (!d->sta.loc || !d->sta.flag_coord || !d->sta.flag_depth) throw Error(CGFD_ERR_INVALID, "station arrays missing");
    for (int r = 0; r < d->sta.num; r++) {
      if (d->sta.flag_coord[r] != 0 && d->sta.flag_coord[r] != 1)
        throw Error(CGFD_ERR_INVALID, "station flag_coord must be 0 (grid index) or 1 (physical coordinates)");
      if (d->sta.flag_coord[r] == 1 && !d->coord)
        throw Error(CGFD_ERR_INVALID, "coord is required to locate stations by physical coordinates");
    }
  }
}

// ---------------------------------------------------------------------------------------
// CFS-PML (bdry_t.cu:85-451): face boxes of N+1 points along the normal spanning the other
// axes, d(x)=dmax (x/L)^2, alpha(x)=amax (1-x/L), beta(x)=1+(bmax-1)(x/L)^2 stored as
// D=d/beta, A=alpha+d/beta, B=1/beta, index 0 at the outer edge of side 0.
// ---------------------------------------------------------------------------------------
void pml_setup(const cgfd_problem_desc *d, PmlFaceHost faces[3][2]) {
  RefGrid g(d->ni, d->nj, d->nk);
  int n[3] = {d->ni, d->nj, d->nk};
  for (int a = 0; a < 3; a++)
    for (int s = 0; s < 2; s++) {
      PmlFaceHost &f = faces[a][s];
      const cgfd_pml_face &in = d->pml[a][s];
      f = PmlFaceHost();
      f.axis = a;
      f.side = s;
      if (!in.enable) continue;
      f.enable = 1;
      int N = in.num_layers;
      for (int b = 0; b < 3; b++) { f.lo[b] = 0; f.hi[b] = n[b] - 1; }
      if (s == 0) f.hi[a] = N;
      else f.lo[a] = n[a] - 1 - N;
      // average spacing along the normal over the face box: one partial sum per line of the
      // outer axis (threads take lines), added in line order, so the result does not depend on
      // the thread count
      const float *x = d->coord, *y = d->coord + g.siz_icmp, *z = d->coord + 2 * g.siz_icmp;
      const int a1 = a == 0 ? 1 : 0, a2 = a == 2 ? 1 : 2;
      const int n2 = f.hi[a2] - f.lo[a2] + 1;
      std::vector<double> part(n2, 0.0);
#pragma omp parallel for schedule(static)
      for (int q = 0; q < n2; q++) {
        const int o2 = f.lo[a2] + q;
        double Lq = 0.0;
        for (int o1 = f.lo[a1]; o1 <= f.hi[a1]; o1++) {
          int ijk[3];
          ijk[a1] = o1; ijk[a2] = o2; ijk[a] = f.lo[a];
          size_t p0 = g.at(ijk[0], ijk[1], ijk[2]);
          for (int m = f.lo[a] + 1; m <= f.hi[a]; m++) {
            ijk[a] = m;
            size_t p1 = g.at(ijk[0], ijk[1], ijk[2]);
            double dx = (double)x[p1] - x[p0], dy = (double)y[p1] - y[p0], dz = (double)z[p1] - z[p0];
            Lq += std::sqrt(dx * dx + dy * dy + dz * dz);
            p0 = p1;
          }
        }
        part[q] = Lq;
      }
      double L = 0.0;
      for (double v : part) L += v;
      const long long num = (long long)n2 * (f.hi[a1] - f.lo[a1] + 1) * (f.hi[a] - f.lo[a]);
      double dh = L / (double)num;
      double L0 = dh * N;
      double Rpp = std::pow(10.0, -((std::log10((double)N) - 1.0) / std::log10(2.0) + 4.0));
      double dmax = -(double)in.ref_vel / (2.0 * L0) * std::log(Rpp) * 3.0;
      f.A.assign(N + 1, 0.f); f.B.assign(N + 1, 0.f); f.D.assign(N + 1, 0.f);
      for (int m = 0; m <= N; m++) {
        double xr = m * dh / L0;
        int idx = s == 0 ? N - m : m;
        double dd = dmax * xr * xr;
        double aa = in.alpha_max * (1.0 - xr);
        double bb = 1.0 + (in.beta_max - 1.0) * xr * xr;
        dd /= bb;
        f.A[idx] = (float)(aa + dd);
        f.B[idx] = (float)(1.0 / bb);
        f.D[idx] = (float)dd;
      }
    }
}

// ---------------------------------------------------------------------------------------
// Free surface (sv_curv_col_el_{iso,vti,aniso}_dvh2dvz): zero traction t_i = C_ijkl zeta_j
// dV_k/dx_l at the top gives dzeta V = -A^-1 (B dxi V + C deta V) with
//   A_ik = zeta_j C_ijkl zeta_l, B_ik = zeta_j C_ijkl xi_l, C_ik = zeta_j C_ijkl eta_l.
// Solved in FP64 per surface column.
// ---------------------------------------------------------------------------------------
static void cij_at(const cgfd_problem_desc *d, size_t iptr, size_t siz, double C[6][6]) {
  const float *m = d->medium;
  for (int a = 0; a < 6; a++)
    for (int b = 0; b < 6; b++) C[a][b] = 0.0;
  if (d->medium_type == CGFD_MEDIUM_ELASTIC_ISO) {
    double lam = m[1 * siz + iptr], mu = m[2 * siz + iptr];
    for (int a = 0; a < 3; a++)
      for (int b = 0; b < 3; b++) C[a][b] = lam;
    for (int a = 0; a < 3; a++) C[a][a] = lam + 2.0 * mu;
    for (int a = 3; a < 6; a++) C[a][a] = mu;
  } else if (d->medium_type == CGFD_MEDIUM_ELASTIC_VTI) {
    double c11 = m[1 * siz + iptr], c13 = m[2 * siz + iptr], c33 = m[3 * siz + iptr], c55 = m[4 * siz + iptr],
           c66 = m[5 * siz + iptr];
    double c12 = c11 - 2.0 * c66;
    C[0][0] = C[1][1] = c11;
    C[0][1] = C[1][0] = c12;
    C[0][2] = C[2][0] = C[1][2] = C[2][1] = c13;
    C[2][2] = c33;
    C[3][3] = C[4][4] = c55;
    C[5][5] = c66;
  } else {
    int n = 1;
    for (int a = 0; a < 6; a++)
      for (int b = a; b < 6; b++) {
        C[a][b] = C[b][a] = m[(size_t)n * siz + iptr];
        n++;
      }
  }
}

static inline int voigt(int a, int b) {
  static const int v[3][3] = {{0, 5, 4}, {5, 1, 3}, {4, 3, 2}};
  return v[a][b];
}

void dvh2dvz(const cgfd_problem_desc *d, std::vector<float> &matx, std::vector<float> &maty) {
  RefGrid g(d->ni, d->nj, d->nk);
  matx.assign((size_t)d->ni * d->nj * 9, 0.f);
  maty.assign((size_t)d->ni * d->nj * 9, 0.f);
  const int k = d->nk - 1;
  int singular = 0;
  // one independent 3x3 solve per surface column
#pragma omp parallel for schedule(static) reduction(| : singular)
  for (int j = 0; j < d->nj; j++)
    for (int i = 0; i < d->ni; i++) {
      size_t iptr = g.at(i, j, k);
      double e[3][3];
      for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++) e[a][b] = d->metric[(size_t)(1 + 3 * a + b) * g.siz_icmp + iptr];
      double C[6][6];
      cij_at(d, iptr, g.siz_icmp, C);
      double A[3][3], B[3][3], Cm[3][3];
      for (int ii = 0; ii < 3; ii++)
        for (int kk = 0; kk < 3; kk++) {
          double sa = 0, sb = 0, sc = 0;
          for (int jj = 0; jj < 3; jj++)
            for (int ll = 0; ll < 3; ll++) {
              double c = C[voigt(ii, jj)][voigt(kk, ll)];
              sa += e[2][jj] * c * e[2][ll];
              sb += e[2][jj] * c * e[0][ll];
              sc += e[2][jj] * c * e[1][ll];
            }
          A[ii][kk] = sa; B[ii][kk] = sb; Cm[ii][kk] = sc;
        }
      double inv[3][3];
      inv[0][0] = A[1][1] * A[2][2] - A[2][1] * A[1][2];
      inv[0][1] = A[2][1] * A[0][2] - A[0][1] * A[2][2];
      inv[0][2] = A[0][1] * A[1][2] - A[0][2] * A[1][1];
      inv[1][0] = A[1][2] * A[2][0] - A[1][0] * A[2][2];
      inv[1][1] = A[0][0] * A[2][2] - A[2][0] * A[0][2];
      inv[1][2] = A[1][0] * A[0][2] - A[0][0] * A[1][2];
      inv[2][0] = A[1][0] * A[2][1] - A[1][1] * A[2][0];
      inv[2][1] = A[2][0] * A[0][1] - A[0][0] * A[2][1];
      inv[2][2] = A[0][0] * A[1][1] - A[0][1] * A[1][0];
      double det = inv[0][0] * A[0][0] + inv[0][1] * A[1][0] + inv[0][2] * A[2][0];
      if (det == 0.0 || !std::isfinite(det)) {
        singular = 1;
        continue;
      }
      for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++) inv[a][b] /= det;
      size_t ij = ((size_t)j * d->ni + i) * 9;
      for (int r = 0; r < 3; r++)
        for (int c = 0; c < 3; c++) {
          double ab = 0, ac = 0;
          for (int q = 0; q < 3; q++) { ab += inv[r][q] * B[q][c]; ac += inv[r][q] * Cm[q][c]; }
          matx[ij + r * 3 + c] = (float)(-ab);
          maty[ij + r * 3 + c] = (float)(-ac);
        }
    }
  if (singular) throw Error(CGFD_ERR_INVALID, "singular free-surface traction matrix");
}

// ---------------------------------------------------------------------------------------
// Visco-elastic media: the generalized-Maxwell-body fit (md_vis_GMB_cal_Y, md_t.cu:657-781).
// Frequencies wk[m] = wmin (wmax/wmin)^(m/(kmax-1)), m < kmax = 2 nmax - 1 (angular), the
// relaxation frequencies wl[n] = wk[2n]. For Q^-1 = 1/round(Q) the weights Y solve, in the least-
// squares sense, sum_n G[m][n] Y[n] = Q^-1 with G[m][n] = (wl_n wk_m + wl_n^2 Q^-1) /
// (wl_n^2 + wk_m^2) (md_visco_LS: the normal equations). At wr = 2 pi fr,
// theta1 = 1 - sum_n Y_n / (1 + (wr/wl_n)^2), theta2 = sum_n Y_n (wr/wl_n) / (1 + (wr/wl_n)^2),
// R = |theta|, and a modulus M given at fr is unrelaxed as M (R + theta1) / (2 R^2): the P modulus
// lambda + 2 mu with Y of Qp, mu with Y of Qs. Ylam = (1 + 2 mu_u / lam_u) YP - 2 mu_u / lam_u YS,
// Ymu = YS. Y and the factor depend on Q alone, so they are solved once per distinct Q.
// ---------------------------------------------------------------------------------------
namespace {
struct GmbQ {
  double y[10];
  double fac;
};

GmbQ gmb_solve(double qinv, int nmax, const double *wl, const double *wk, int kmax, double wr) {
  double A[10][10] = {}, r[10] = {};
  for (int m = 0; m < kmax; m++) {
    double g[10];
    for (int n = 0; n < nmax; n++) g[n] = (wl[n] * wk[m] + wl[n] * wl[n] * qinv) / (wl[n] * wl[n] + wk[m] * wk[m]);
    for (int a = 0; a < nmax; a++) {
      r[a] += g[a] * qinv;
      for (int b = 0; b < nmax; b++) A[a][b] += g[a] * g[b];
    }
  }
  // Gauss-Jordan elimination with partial pivoting on the normal equations
  for (int c = 0; c < nmax; c++) {
    int piv = c;
    for (int a = c + 1; a < nmax; a++)
      if (std::fabs(A[a][c]) > std::fabs(A[piv][c])) piv = a;
    if (A[piv][c] == 0.0) throw Error(CGFD_ERR_INVALID, "singular GMB least-squares system");
    if (piv != c) {
      for (int b = 0; b < nmax; b++) std::swap(A[c][b], A[piv][b]);
      std::swap(r[c], r[piv]);
    }
    for (int a = 0; a < nmax; a++) {
      if (a == c) continue;
      const double f = A[a][c] / A[c][c];
      for (int b = c; b < nmax; b++) A[a][b] -= f * A[c][b];
      r[a] -= f * r[c];
    }
  }
  GmbQ o;
  double t1 = 0, t2 = 0;
  for (int n = 0; n < nmax; n++) {
    o.y[n] = r[n] / A[n][n];
    const double x = wr / wl[n], den = 1.0 + x * x;
    t1 += o.y[n] / den;
    t2 += o.y[n] * x / den;
  }
  t1 = 1.0 - t1;
  const double R = std::sqrt(t1 * t1 + t2 * t2);
  o.fac = (R + t1) / (2.0 * R * R);
  return o;
}
}  // namespace

void visco_gmb(const cgfd_visco_desc *v, long long n, const float *lambda, const float *mu, const float *Qp,
               const float *Qs, float *lam_u, float *mu_u, float *Ylam, float *Ymu, float *wl_out) {
  if (!v) throw Error(CGFD_ERR_INVALID, "visco parameters are required");
  if (v->nmaxwell < 1 || v->nmaxwell > 10) throw Error(CGFD_ERR_INVALID, "nmaxwell must be in [1, 10]");
  if (!(v->fmin > 0.f) || !(v->fmax > v->fmin) || !(v->fr > 0.f))
    throw Error(CGFD_ERR_INVALID, "visco frequencies must satisfy 0 < fmin < fmax and fr > 0");
  const int nmax = v->nmaxwell, kmax = 2 * nmax - 1;
  const double wmin = 2 * kPi * v->fmin, wmax = 2 * kPi * v->fmax, wr = 2 * kPi * v->fr;
  double wk[19], wl[10];
  for (int m = 0; m < kmax; m++) wk[m] = kmax > 1 ? wmin * std::pow(wmax / wmin, m / (double)(kmax - 1)) : wmin;
  for (int q = 0; q < nmax; q++) {
    wl[q] = wk[2 * q];
    if (wl_out) wl_out[q] = (float)wl[q];
  }
  std::map<long long, GmbQ> cache;
  auto fit = [&](float Q) -> const GmbQ & {
    const double rq = std::round((double)Q);
    if (!(rq >= 1.0)) throw Error(CGFD_ERR_INVALID, "Q values must round to >= 1");
    auto it = cache.find((long long)rq);
    if (it == cache.end()) it = cache.emplace((long long)rq, gmb_solve(1.0 / rq, nmax, wl, wk, kmax, wr)).first;
    return it->second;
  };
  for (long long t = 0; t < n; t++) {
    const GmbQ &P = fit(Qp[t]);
    const GmbQ &S = fit(Qs[t]);
    const double m_u = (double)mu[t] * S.fac;
    const double l_u = ((double)lambda[t] + 2.0 * mu[t]) * P.fac - 2.0 * m_u;
    lam_u[t] = (float)l_u;
    mu_u[t] = (float)m_u;
    const double r = l_u != 0.0 ? 2.0 * m_u / l_u : 0.0;
    for (int q = 0; q < nmax; q++) {
      Ylam[(size_t)q * n + t] = (float)((1.0 + r) * P.y[q] - r * S.y[q]);
      Ymu[(size_t)q * n + t] = (float)S.y[q];
    }
  }
}

// Local frame of the free surface for the visco-elastic stress fix
// (sv_curv_col_vis_iso_dvh2dvz, sv_curv_col_vis_iso_gpu.cu:632-706): with the surface normal
// zeta / |zeta| and the tangent r_eta / |r_eta| (the centered operator along j on the
// coordinates), D = [tangent x normal scaled by 1/(|r_eta||zeta|) ; r_eta / |r_eta| ;
// zeta / |zeta|], row-major per surface column.
void vis_free_matrix(const cgfd_problem_desc *d, std::vector<float> &matD) {
  if (!d->coord) throw Error(CGFD_ERR_INVALID, "visco-elastic media with a free surface need the coordinates");
  static const double c7[7] = {-0.02084, 0.1667, -0.7709, 0.0, 0.7709, -0.1667, 0.02084};  // fd_t.cu:162
  RefGrid g(d->ni, d->nj, d->nk);
  matD.assign((size_t)d->ni * d->nj * 9, 0.f);
  const int k = d->nk - 1;
  for (int j = 0; j < d->nj; j++)
    for (int i = 0; i < d->ni; i++) {
      const size_t iptr = g.at(i, j, k);
      double r[3] = {0, 0, 0};
      for (int a = 0; a < 3; a++)
        for (int t = 0; t < 7; t++)
          r[a] += c7[t] * d->coord[(size_t)a * g.siz_icmp + iptr + (size_t)((long long)(t - 3) * (long long)g.siz_iy)];
      double e[3];
      for (int a = 0; a < 3; a++) e[a] = d->metric[(size_t)(7 + a) * g.siz_icmp + iptr];
      const double en = 1.0 / std::sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
      const double em = 1.0 / std::sqrt(e[0] * e[0] + e[1] * e[1] + e[2] * e[2]);
      const double enm = en * em;
      const double D[9] = {(r[1] * e[2] - r[2] * e[1]) * enm, (r[2] * e[0] - r[0] * e[2]) * enm,
                           (r[0] * e[1] - r[1] * e[0]) * enm, r[0] * en, r[1] * en, r[2] * en,
                           e[0] * em, e[1] * em, e[2] * em};
      for (int q = 0; q < 9; q++) matD[((size_t)j * d->ni + i) * 9 + q] = (float)D[q];
    }
}

// ---------------------------------------------------------------------------------------
// Sources (src_t.cu:143-1009): nearest-index location, 7^3 Gaussian smoothing normalised to
// a unit sum (kept only on physical points, not renormalised), STF per (step, RK stage).
// ---------------------------------------------------------------------------------------
static double wavelet(double t, int name, const float *c) {
  switch (name) {
    case CGFD_WAVELET_RICKER: {
      double u = (t - c[1]) * 2.0 * kPi * c[0];
      return (1 - u * u / 2.0) * std::exp(-u * u / 4.0);
    }
    case CGFD_WAVELET_RICKER_DERIV: {
      double u = (t - c[1]) * 2.0 * kPi * c[0];
      return u * (-3 + 0.5 * u * u) * std::exp(-u * u / 4) * kPi * c[0];
    }
    case CGFD_WAVELET_GAUSSIAN: {
      double a = c[0], t0 = c[1];
      return std::exp(-(t - t0) * (t - t0) / (a * a)) / (std::sqrt(kPi) * a);
    }
    case CGFD_WAVELET_GAUSSIAN_DERIV: {
      double a = c[0], t0 = c[1];
      return std::exp(-(t - t0) * (t - t0) / (a * a)) / (std::sqrt(kPi) * a) * (-2 * (t - t0) / (a * a));
    }
    case CGFD_WAVELET_KLAUDER: {  // fixed parameters as in src_cal_wavelet
      double tt0 = 0.2, f1 = 1.5, f2 = 41.5, T = 20;
      double K = (f2 - f1) / T, fM = (f2 + f1) / 2.0;
      return (std::sin(kPi * K * t * (T - (t - tt0))) * std::cos(2 * kPi * fM * (t - tt0))) / (kPi * K * (t - tt0));
    }
  }
  throw Error(CGFD_ERR_INVALID, "unknown wavelet id");
}

static void angle2moment(double strike, double dip, double rake, double mt[6]) {
  double d = dip / 180.0 * kPi, s = strike / 180.0 * kPi, r = rake / 180.0 * kPi;
  double M11 = -(std::sin(d) * std::cos(r) * std::sin(2 * s) + std::sin(2 * d) * std::sin(r) * std::sin(s) * std::sin(s));
  double M22 = std::sin(d) * std::cos(r) * std::sin(2 * s) - std::sin(2 * d) * std::sin(r) * std::cos(s) * std::cos(s);
  double M33 = -(M11 + M22);
  double M12 = std::sin(d) * std::cos(r) * std::cos(2 * s) + 0.5 * std::sin(2 * d) * std::sin(r) * std::sin(2 * s);
  double M13 = -(std::cos(d) * std::cos(r) * std::cos(s) + std::cos(2 * d) * std::sin(r) * std::sin(s));
  double M23 = -(std::cos(d) * std::cos(r) * std::sin(s) - std::cos(2 * d) * std::sin(r) * std::cos(s));
  // x east / y north / z up (src_t.cu:936-945)
  mt[0] = M22; mt[1] = M11; mt[2] = M33; mt[3] = -M13; mt[4] = -M23; mt[5] = M12;
}

// piecewise Lagrange interpolation of order 3 on a uniform series (interp.cu:220-299)
static double lag_interp(const std::vector<double> &t, const std::vector<double> &z, double t_start, double dt,
                         double ti) {
  const int order = 3, lower = 1, upper = 2;
  int ni = (int)t.size();
  int indx = (int)((ti - t_start) / dt + 0.5);
  if (indx > ni - 1) indx = ni - 1;
  auto window = [&](int a, int b) {
    double Li = 0;
    for (int i = a; i <= b; i++) {
      double Lx = 1;
      for (int j = a; j <= b; j++)
        if (i != j) Lx = Lx * (ti - t[j]) / (t[i] - t[j]);
      Li += Lx * z[i];
    }
    return Li;
  };
  (void)order;
  double Li = 0;
  if (indx - lower >= 0 && indx + upper <= ni - 1) Li += window(indx - lower, indx + upper);
  if (indx - lower < 0) Li += window(0, indx + upper + (lower - indx));
  if (indx + upper > ni - 1) Li += window(indx - lower - (indx + upper - (ni - 1)), ni - 1);
  return Li;
}

void src_setup(const cgfd_problem_desc *d, SrcHost &s, const Located *loc) {
  s = SrcHost();
  const cgfd_source_desc &in = d->src;
  if (in.num <= 0) return;
  RefGrid g(d->ni, d->nj, d->nk);
  const int half = 3, len = 7;
  s.max_ext = len * len * len;
  s.force = (in.cmp_type == 1 || in.cmp_type == 3) ? 1 : 0;
  s.moment = (!s.force && in.cmp_type == 2) ? 1 : 0;  // src_t.cu:437-441 (3 -> force only)
  const double dt = d->dt, t0 = d->t0;
  if (in.stf_given == 0) s.max_nt = (int)(in.stf_length / d->dt + 0.5);
  else s.max_nt = (int)(((in.stf_nt - 1) * in.stf_dt / d->dt) + 0.5) + 1;
  if (s.max_nt < 1) throw Error(CGFD_ERR_INVALID, "source time function shorter than one step");
  const double rk_time[4] = {0.0, 0.5, 0.5, 1.0};
  const int n[3] = {d->ni, d->nj, d->nk};
  for (int is = 0; is < in.num; is++) {
    int gi[3];
    double inc[3];
    bool outside = false;
    if (in.loc_coord_type == 1) {
      // located by coordinates: nearest grid point and shift (src_t.cu:341-398); without the
      // location (sizing only) the source counts as inside
      for (int a = 0; a < 3; a++) {
        gi[a] = loc ? loc->idx[3 * is + a] : n[a] / 2;
        inc[a] = loc ? loc->inc[3 * is + a] : 0.0f;
        if (gi[a] < 0 || gi[a] > n[a] - 1) outside = true;
      }
    } else {
      double c[3] = {in.loc[3 * is], in.loc[3 * is + 1], in.loc[3 * is + 2]};
      if (in.loc_3dim == 1) c[2] = (d->nk - 1) - (float)c[2];
      for (int a = 0; a < 3; a++) {
        gi[a] = (int)((float)c[a] + 0.5f);
        inc[a] = (float)c[a] - gi[a];
        if (gi[a] < 0 || gi[a] > n[a] - 1) outside = true;
      }
    }
    bool here = true;
    for (int a = 0; a < 3; a++)
      if (gi[a] - half > n[a] - 1 || gi[a] + half < 0) here = false;
    if (!here) continue;
    // component values (F and M), possibly from strike/dip/rake + mu D A
    int nt_in = in.stf_given == 0 ? 1 : in.stf_nt;
    std::vector<double> vals((size_t)nt_in * 9);
    for (int t = 0; t < nt_in; t++)
      for (int q = 0; q < 9; q++)
        vals[(size_t)t * 9 + q] = in.stf_given == 0 ? in.cmp[9 * is + q] : in.cmp_values[((size_t)is * in.stf_nt + t) * 9 + q];
    if (s.moment && in.mechanism_type == 1) {
      for (int t = 0; t < nt_in; t++) {
        double *v = &vals[(size_t)t * 9];
        double mu = v[6];
        if (mu < 0.0) {
          if (d->medium_type != CGFD_MEDIUM_ELASTIC_ISO || outside)
            throw Error(CGFD_ERR_INVALID, "mu < 0 needs an isotropic medium at the source point");
          mu = d->medium[2 * g.siz_icmp + g.at(gi[0], gi[1], gi[2])];
        }
        double mt[6];
        angle2moment(v[3], v[4], v[5], mt);
        double M0 = mu * v[7] * v[8];
        for (int q = 0; q < 6; q++) v[3 + q] = M0 * mt[q];
      }
    }
    // smoothing weights
    double wid = half / 2.0;
    std::vector<double> delt(s.max_ext);
    double sum = 0;
    int ip = 0;
    for (int kk = -half; kk <= half; kk++)
      for (int jj = -half; jj <= half; jj++)
        for (int ii = -half; ii <= half; ii++) {
          auto gs = [&](double x) { return std::exp(-x * x / (wid * wid)) / (std::sqrt(kPi) * wid); };
          delt[ip] = gs(ii - inc[0]) * gs(jj - inc[1]) * gs(kk - inc[2]);
          sum += delt[ip++];
        }
    int is_local = s.nsrc++;
    s.ext_i.resize((size_t)s.nsrc * s.max_ext, 0);
    s.ext_j.resize((size_t)s.nsrc * s.max_ext, 0);
    s.ext_k.resize((size_t)s.nsrc * s.max_ext, 0);
    s.ext_wv.resize((size_t)s.nsrc * s.max_ext, 0.f);
    s.ext_wt.resize((size_t)s.nsrc * s.max_ext, 0.f);
    int ne = 0;
    if (!outside) {
      for (int kk = -half; kk <= half; kk++)
        for (int jj = -half; jj <= half; jj++)
          for (int ii = -half; ii <= half; ii++) {
            int i = gi[0] + ii, j = gi[1] + jj, k = gi[2] + kk;
            if (i < 0 || i >= d->ni || j < 0 || j >= d->nj || k < 0 || k >= d->nk) continue;
            double w = delt[(ii + half) + len * (jj + half) + len * len * (kk + half)] / sum;
            size_t p = g.at(i, j, k);
            // (no metric: only the sizes are wanted, cgfd_problem_bytes before the metric exists)
            double jac = d->metric ? (double)d->metric[p] : 1.0;
            double rho = d->medium[p];
            double slw = rho > 1e-10 ? 1.0 / rho : 0.0;
            size_t e = (size_t)is_local * s.max_ext + ne;
            s.ext_i[e] = i; s.ext_j[e] = j; s.ext_k[e] = k;
            s.ext_wv[e] = (float)(w * slw / jac);
            s.ext_wt[e] = (float)(w / jac);
            ne++;
          }
    }
    s.ext_num.push_back(ne);
    double tstart = in.t_start[is];
    int itb = (int)(((float)tstart - (float)t0) / (float)dt);
    s.it_begin.push_back(itb);
    double t_shift = tstart - (itb * dt + t0);
    s.stf.resize((size_t)s.nsrc * s.max_nt * 36, 0.f);
    std::vector<double> t_in, col;
    if (in.stf_given == 1) {
      t_in.resize(in.stf_nt);
      col.resize(in.stf_nt);
      for (int t = 0; t < in.stf_nt; t++) t_in[t] = tstart + t * (double)in.stf_dt;
    }
    for (int it1 = 0; it1 < s.max_nt; it1++)
      for (int st = 0; st < 4; st++) {
        float *out = &s.stf[(((size_t)is_local * s.max_nt + it1) * 4 + st) * 9];
        if (in.stf_given == 0) {
          double t = it1 * dt + rk_time[st] * dt - t_shift;
          double v = wavelet(t, in.wavelet[is], in.wavelet_coefs + 10 * is);
          for (int q = 0; q < 9; q++) out[q] = (float)(v * vals[q]);
        } else {
          // the sampled branch evaluates at the global step index (src_t.cu:683)
          double t = (itb + it1) * dt + rk_time[st] * dt - t_shift;
          for (int q = 0; q < 9; q++) {
            for (int m = 0; m < in.stf_nt; m++) col[m] = vals[(size_t)m * 9 + q];
            out[q] = (float)lag_interp(t_in, col, tstart, in.stf_dt, t);
          }
        }
        if (!s.force) out[0] = out[1] = out[2] = 0.f;
        if (!s.moment) for (int q = 3; q < 9; q++) out[q] = 0.f;
      }
  }
}

// ---------------------------------------------------------------------------------------
// Stations (io_funcs.cu:24-299, 1624-1666): 1-based grid index, floor location, trilinear
// weights with the reference's corner usage (corner 5 counted twice, corner 4 never).
// ---------------------------------------------------------------------------------------
void recv_setup(const cgfd_problem_desc *d, RecvHost &r, const Located *loc) {
  r = RecvHost();
  const cgfd_station_desc &in = d->sta;
  for (int ir = 0; ir < in.num; ir++) {
    int ix, iy, iz;
    double dx, dy, dz;
    if (in.flag_coord[ir] == 1) {
      // located by coordinates; a negative shift moves to the lower neighbour (io_funcs.cu:150-169)
      int id[3];
      float inc[3];
      const int n[3] = {d->ni, d->nj, d->nk};
      for (int a = 0; a < 3; a++) {
        id[a] = loc ? loc->idx[3 * ir + a] : n[a] / 2;
        inc[a] = loc ? loc->inc[3 * ir + a] : 0.0f;
        if (id[a] != -1000 && inc[a] < 0.0) {
          inc[a] = (float)(1.0 + inc[a]);
          id[a] -= 1;
        }
      }
      ix = id[0]; iy = id[1]; iz = id[2];
      dx = inc[0]; dy = inc[1]; dz = inc[2];
    } else {
      float c[3] = {in.loc[3 * ir] - 1, in.loc[3 * ir + 1] - 1, in.loc[3 * ir + 2]};
      if (in.flag_depth[ir] == 1) c[2] = (d->nk - 1) - c[2];
      else c[2] -= 1;
      ix = (int)c[0]; iy = (int)c[1]; iz = (int)c[2];
      dx = c[0] - ix; dy = c[1] - iy; dz = c[2] - iz;
    }
    if (!(ix >= 0 && ix <= d->ni - 1 && iy >= 0 && iy <= d->nj - 1 && iz >= 0 && iz <= d->nk - 1)) continue;
    r.i.push_back(ix); r.j.push_back(iy); r.k.push_back(iz);
    r.input_index.push_back(ir);
    double x1 = 1.0 - dx, y1 = 1.0 - dy, z1 = 1.0 - dz;
    double w[8] = {x1 * y1 * z1, dx * y1 * z1, x1 * dy * z1, dx * dy * z1,
                   0.0, x1 * y1 * dz + dx * y1 * dz, x1 * dy * dz, dx * dy * dz};
    for (int q = 0; q < 8; q++) r.w8.push_back((float)w[q]);
    r.n++;
  }
}

}  // namespace cgfd

// ---------------------------------------------------------------------------------------
// C ABI grid helpers
// ---------------------------------------------------------------------------------------
namespace {
thread_local std::string g_setup_err;
}

extern "C" {

int cgfd_visco_gmb(const cgfd_visco_desc *v, long long n, const float *lambda, const float *mu, const float *Qp,
                   const float *Qs, float *lam_u, float *mu_u, float *Ylam, float *Ymu, float *wl) {
  if (n < 0 || (n > 0 && (!lambda || !mu || !Qp || !Qs || !lam_u || !mu_u || !Ylam || !Ymu))) {
    cgfd::set_last_error("invalid argument");
    return CGFD_ERR_INVALID;
  }
  try {
    cgfd::visco_gmb(v, n, lambda, mu, Qp, Qs, lam_u, mu_u, Ylam, Ymu, wl);
  } catch (const cgfd::Error &e) {
    cgfd::set_last_error(e.what());
    return e.code;
  }
  return CGFD_OK;
}

// Fill the 3 ghost layers of ncmp fields by linear extrapolation (gd_t.cu:404-502).
int cgfd_fill_ghosts(int ni, int nj, int nk, int ncmp, float *v4d) {
  if (!v4d || ni < 4 || nj < 4 || nk < 4 || ncmp < 1) return CGFD_ERR_INVALID;
  cgfd::RefGrid g(ni, nj, nk);
  int ni1 = 3, ni2 = ni + 2, nj1 = 3, nj2 = nj + 2, nk1 = 3, nk2 = nk + 2;
  for (int c = 0; c < ncmp; c++) {
    float *v = v4d + (size_t)c * g.siz_icmp;
    auto at = [&](int i, int j, int k) -> float & { return v[i + (size_t)j * g.siz_iy + (size_t)k * g.siz_iz]; };
    for (int k = 0; k < g.nz; k++)
      for (int j = 0; j < g.ny; j++) {
        for (int i = 0; i < ni1; i++) at(i, j, k) = 2 * at(ni1, j, k) - at(2 * ni1 - i, j, k);
        for (int i = ni2 + 1; i < g.nx; i++) at(i, j, k) = 2 * at(ni2, j, k) - at(2 * ni2 - i, j, k);
      }
    for (int k = 0; k < g.nz; k++) {
      for (int j = 0; j < nj1; j++)
        for (int i = 0; i < g.nx; i++) at(i, j, k) = 2 * at(i, nj1, k) - at(i, 2 * nj1 - j, k);
      for (int j = nj2 + 1; j < g.ny; j++)
        for (int i = 0; i < g.nx; i++) at(i, j, k) = 2 * at(i, nj2, k) - at(i, 2 * nj2 - j, k);
    }
    for (int k = 0; k < nk1; k++)
      for (int j = 0; j < g.ny; j++)
        for (int i = 0; i < g.nx; i++) at(i, j, k) = 2 * at(i, j, nk1) - at(i, j, 2 * nk1 - k);
    for (int k = nk2 + 1; k < g.nz; k++)
      for (int j = 0; j < g.ny; j++)
        for (int i = 0; i < g.nx; i++) at(i, j, k) = 2 * at(i, j, nk2) - at(i, j, 2 * nk2 - k);
  }
  return CGFD_OK;
}

// Grid metrics in FP64 from coordinates with filled ghosts (gd_t.cu:209-314), stored as
// float [10][nz][ny][nx] (jac, xi_*, eta_*, zeta_*), ghosts by linear extrapolation.
int cgfd_metric_calc(int ni, int nj, int nk, const float *coord, float *metric) {
  if (!coord || !metric || ni < 4 || nj < 4 || nk < 4) return CGFD_ERR_INVALID;
  cgfd::RefGrid g(ni, nj, nk);
  static const double c7[7] = {-0.02084, 0.1667, -0.7709, 0.0, 0.7709, -0.1667, 0.02084};  // fd_t.cu:162
  const float *x = coord, *y = coord + g.siz_icmp, *z = coord + 2 * g.siz_icmp;
  std::memset(metric, 0, sizeof(float) * 10 * g.siz_icmp);
#pragma omp parallel for schedule(static)
  for (int k = 0; k < nk; k++)
    for (int j = 0; j < nj; j++)
      for (int i = 0; i < ni; i++) {
        size_t p = g.at(i, j, k);
        double v[3][3];  // v[axis][xyz]
        const size_t sh[3] = {1, g.siz_iy, g.siz_iz};
        for (int a = 0; a < 3; a++) {
          double sx = 0, sy = 0, sz = 0;
          for (int n = 0; n < 7; n++) {
            size_t q = p + (long long)(n - 3) * (long long)sh[a];
            sx += c7[n] * x[q]; sy += c7[n] * y[q]; sz += c7[n] * z[q];
          }
          v[a][0] = sx; v[a][1] = sy; v[a][2] = sz;
        }
        auto cross = [](const double *a, const double *b, double *o) {
          o[0] = a[1] * b[2] - a[2] * b[1];
          o[1] = a[2] * b[0] - a[0] * b[2];
          o[2] = a[0] * b[1] - a[1] * b[0];
        };
        double g1[3], g2[3], g3[3];
        cross(v[0], v[1], g3);
        double jac = g3[0] * v[2][0] + g3[1] * v[2][1] + g3[2] * v[2][2];
        cross(v[1], v[2], g1);
        cross(v[2], v[0], g2);
        metric[p] = (float)jac;
        for (int b = 0; b < 3; b++) {
          metric[(size_t)(1 + b) * g.siz_icmp + p] = (float)(g1[b] / jac);
          metric[(size_t)(4 + b) * g.siz_icmp + p] = (float)(g2[b] / jac);
          metric[(size_t)(7 + b) * g.siz_icmp + p] = (float)(g3[b] / jac);
        }
      }
  return cgfd_fill_ghosts(ni, nj, nk, 10, metric);
}

// Largest stable time step in FP64 (blk_t.cu:673-763): CFL * (min distance from a point
// to the 8 planes through its neighbours) / Vp, over physical points except the last
// index of each axis. Vp: iso sqrt((lambda+2mu)/rho), VTI max(sqrt(c11/rho),
// sqrt(c33/rho)), aniso sqrt(c11/rho), acoustic sqrt(kappa/rho).
int cgfd_dt_estimate(const cgfd_problem_desc *d, double cfl, double *dtmax) {
  if (!d || !d->coord || !d->medium || !dtmax) return CGFD_ERR_INVALID;
  cgfd::RefGrid g(d->ni, d->nj, d->nk);
  const float *x = d->coord, *y = d->coord + g.siz_icmp, *z = d->coord + 2 * g.siz_icmp;
  const float *m = d->medium;
  double best = 1e300;
#pragma omp parallel for reduction(min : best) schedule(static)
  for (int k = 0; k < d->nk - 1; k++)
    for (int j = 0; j < d->nj - 1; j++)
      for (int i = 0; i < d->ni - 1; i++) {
        size_t p = g.at(i, j, k);
        double rho = m[p], vp;
        if (d->medium_type == CGFD_MEDIUM_ACOUSTIC_ISO) vp = std::sqrt(m[g.siz_icmp + p] / rho);
        else if (d->medium_type == CGFD_MEDIUM_ELASTIC_ISO) vp = std::sqrt((m[g.siz_icmp + p] + 2.0 * m[2 * g.siz_icmp + p]) / rho);
        else if (d->medium_type == CGFD_MEDIUM_ELASTIC_VTI)
          vp = std::fmax(std::sqrt(m[g.siz_icmp + p] / rho), std::sqrt(m[3 * g.siz_icmp + p] / rho));
        else vp = std::sqrt(m[g.siz_icmp + p] / rho);
        double p0[3] = {x[p], y[p], z[p]};
        double L = 1e300;
        for (int kk = -1; kk <= 1; kk += 2)
          for (int jj = -1; jj <= 1; jj += 2)
            for (int ii = -1; ii <= 1; ii += 2) {
              size_t q1 = p - ii, q2 = p - (long long)jj * (long long)g.siz_iy, q3 = p - (long long)kk * (long long)g.siz_iz;
              double a[3] = {x[q1], y[q1], z[q1]}, b[3] = {x[q2], y[q2], z[q2]}, c[3] = {x[q3], y[q3], z[q3]};
              double u[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]}, w[3] = {c[0] - a[0], c[1] - a[1], c[2] - a[2]};
              double n[3] = {u[1] * w[2] - u[2] * w[1], u[2] * w[0] - u[0] * w[2], u[0] * w[1] - u[1] * w[0]};
              double nn = std::sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
              double dist = std::fabs(n[0] * (p0[0] - a[0]) + n[1] * (p0[1] - a[1]) + n[2] * (p0[2] - a[2])) / nn;
              if (dist < L) L = dist;
            }
        double dtp = cfl / vp * L;
        if (dtp < best) best = dtp;
      }
  *dtmax = best;
  return CGFD_OK;
}

// Keep three significant digits (blk_t.cu:765-780).
double cgfd_keep_three_digits(double dt) {
  char s[64];
  snprintf(s, sizeof(s), "%9.7e", dt);
  for (int i = 3; i < 9; i++) s[i] = '0';
  return atof(s);
}

}  // extern "C"

// cgfd_launch.h -- host-visible launch entry points of the device kernels.
#pragma once

#include <cuda_runtime.h>

namespace cgfd {

template <typename R> struct StagePT;
using StageP = StagePT<float>;
struct TmaP;

// storage type of the coefficient array
// (16-bit types: value = scale * stored + offset, one scale/offset per field)
enum { COEF_F32 = 0, COEF_F16 = 1, COEF_BF16 = 2, COEF_U16 = 3 };

// Source injection of one stage (sv_curv_col_el_gpu.cu:227-301), applied to tmp/end.
// R: real type of the wavefield levels (float; double in the FP64 build).
template <typename R>
struct SrcPT {
  int nsrc, max_ext, max_nt;
  int force, moment;
  int stage;
  R ca, cb;
  const int *it_begin;         // [nsrc]
  const int *ext_num;          // [nsrc]
  const long long *ext_idx;    // [nsrc][max_ext] device-layout index
  const float *ext_wv;         // [nsrc][max_ext] coef * (1/rho) / jac
  const float *ext_wt;         // [nsrc][max_ext] coef / jac
  const float *stf;            // [nsrc][max_nt][4][9]: fx fy fz mxx myy mzz myz mxz mxy
  const int *src_shot;         // [nsrc] wavefield (shot) each source acts on
  R *tmp_out;                  // __half when wave16
  R *end;
  long long sf;
  const int *d_it;
  int wave16;                  // FP16 stage levels: tmp_out holds scaled __half
  const float *wsc;            // [nshot][18] scale / inverse scale of this step (wave16)
  unsigned int *amax;          // [nshot][2] max |w_end| per group, collected at stage 3 (wave16)
};
using SrcP = SrcPT<float>;

// Strided sub-box of the 9 wavefield components into dst[9][count_k][count_j][count_i]
// (io_snap_pack_buff, io_funcs.cu:1569-1595, all components in one launch).
template <typename R>
void launch_gather_box(const R *w, long long sf, long long sx, long long sz, long long off0, const int start[3],
                       const int count[3], const int stride[3], float *dst, cudaStream_t st);

// Free-surface peak ground motion after each time step (PG_calcu_gpu, wav_t.cu:281-360).
template <typename R>
struct PgPT {
  int ni, nj, nshot;
  long long sx, sf, off_top;   // off_top: device index of physical (0, 0, nk-1)
  const R *w_end, *w_pre;      // the step's new and old state
  float *pg;                   // [nshot][15][nj][ni]
  R *dis;                      // [nshot][3][nj][ni] displacement accumulator
  float dt;
};
using PgP = PgPT<float>;
template <typename R>
int launch_peak_motion(const PgPT<R> &q, cudaStream_t st);

// Visco-elastic media (generalized Maxwell body), cgfd_visco.cu. The attenuation pass of one
// RK stage (sv_curv_col_vis_iso_atten_gpu, sv_curv_col_vis_iso_gpu.cu:285-433) on the elastic
// right-hand side `rhs`, then the RK combine of the 9 wave fields and the 6 nmax memory variables.
struct VisP {
  int ni, nj, nk, nmax, stage;
  long long sx, sz, sf, off0;
  const float *rhs;                   // [9][sf] elastic right-hand side (no sources)
  const float *cur, *pre;             // wave levels: stage input, w_pre
  float *tmp_out, *end;               // next stage input (stages 0-2), w_end
  const float *jcur, *jpre;           // memory variables [nmax][6][sf], xx yy zz yz xz xy
  float *jtmp, *jend;
  const float *coef;                  // coefficient fields: lambda at 10, mu at 11 (unrelaxed)
  const float *y;                     // [2 nmax][sf]: Ylam[n], then Ymu[n]
  float wl[10];                       // relaxation angular frequencies
  float ca, cb;
  int *err;                           // kErrWaveNonfinite when w_end turns non-finite (stage 3)
};
int launch_vis_atten(const VisP &q, cudaStream_t st);
// The stress rotation of w_end at the free surface after the last stage
// (sv_curv_col_vis_iso_free_gpu, sv_curv_col_vis_iso_gpu.cu:435-531): the stress in the local
// frame D (rows: tangent x normal, tangent along eta, normal), its normal components zeroed.
struct VisFreeP {
  int ni, nj;
  long long sx, sf, off_top;          // off_top: device index of physical (0, 0, nk-1)
  float *w_end;
  const float *matD;                  // [nj][ni][9] row-major
};
int launch_vis_free(const VisFreeP &q, cudaStream_t st);

// Station sampling of w_pre (io_funcs.cu:1624-1666).
template <typename R>
struct RecvPT {
  int nsta;
  int nshot;                   // every shot is sampled at the same stations
  int nt_total;
  const long long *idx8;       // [nsta][8] device-layout corner index
  const float *w8;             // [nsta][8] trilinear weights (reference corner usage)
  const R *pre;
  long long sf;
  float *seis;                 // [nshot][nsta][9][nt_total]
  const int *d_it;
  int *d_flag;
};
using RecvP = RecvPT<float>;

// Slices: full x / y / z planes of the 9 components of w_pre at the start of every step
// (io_slice_nc_put, io_funcs.cu:667-788, pack kernels io_funcs.cu:1528-1567), written into a
// device ring of ring_steps steps: ring[(it % ring_steps) * nshot + shot][per_shot] with, per
// shot, the x slices [nxs][9][nk][nj], then the y slices [nys][9][nk][ni], then the z slices
// [nzs][9][nj][ni] (physical points only).
template <typename R>
struct SliceP {
  int ni, nj, nk, nshot;
  long long sx, sz, sf, off0;
  const R *pre;
  int nxs, nys, nzs;
  const int *idx;              // [nxs + nys + nzs] physical 0-based plane index
  float *ring;
  int ring_steps;
  long long per_shot;          // 9 * (nxs nk nj + nys nk ni + nzs nj ni)
  const int *d_it;
};
template <typename R>
int launch_slices(const SliceP<R> &q, cudaStream_t st);

// Grid metrics in FP64 from coordinates x, y, z (ghosts filled) into out[10] (jac, xi_x ..
// zeta_z), all in one layout (off0 + k sz + j sx + i), ghosts by linear extrapolation.
void launch_metric(const float *x, const float *y, const float *z, float *const out[10], int ni, int nj, int nk,
                   long long sx, long long sz, long long off0, cudaStream_t st);

// Each launcher returns the number of kernels it launched (0 or 1).
template <typename R>
int launch_stage_bulk(int med, const StagePT<R> &p, int nzc, cudaStream_t st);
int launch_stage_surface(int med, int coef_type, int wave16, const StageP &p, cudaStream_t st);
// Acoustic media (cgfd_acoustic.cu), R float or double: the free-surface pressure image of the
// stage input (before the stage; no launch without a free surface), and the fused stage of
// every cell in z chunks of nzc planes.
template <typename R>
int launch_ac_image(const StagePT<R> &p, cudaStream_t st);
template <typename R>
int launch_stage_ac(const StagePT<R> &p, int nzc, cudaStream_t st);
// the TMA-pipelined acoustic stage (FP32; tm: the acoustic maps of the stage input, w_pre,
// w_end and the coefficients); -1 when the grid does not fit one launch (run launch_stage_ac)
int launch_stage_ac_tma(const StageP &p, const TmaP &tm, int nzc, cudaStream_t st);
// FP64 build: the surface slab with double storage and arithmetic
int launch_stage_surface64(int med, const StagePT<double> &p, cudaStream_t st);
// traction-image fluxes of the stage input for the surface slab (before it, same stream)
int launch_timg_flux(int coef_type, int wave16, const StageP &p, cudaStream_t st);
int launch_timg_flux64(const StagePT<double> &p, cudaStream_t st);
// TMA-pipelined bulk kernel: tile height, one-time function attributes, launch.
// wave16: FP16 stage levels (requires COEF_F16).
// shape: tile shape index (0 default, 1 the alternative; cgfd_bulk_tma.cuh TileShape)
int tma_tile_y(int med, int shape);
int tma_blocks_per_sm(int med, int shape);  // resident blocks per SM the tile shape is built for
cudaError_t tma_prepare(int med, int coef_type, int wave16, int shape);
// Tile list of the TMA bulk kernel (device array, one int4 per block in launch order:
// bx + kTilePml if a CFS-PML face meets the tile + (shot << 16), by, first and end z plane).
constexpr int kTilePml = 0x8000;     // bit 15 of x
constexpr int kTileBxMask = 0x7fff;  // bits 0-14 of x: bx (bits 16-30: the shot)
struct BulkTiles {
  const int4 *list = nullptr;
  int n = 0, npml = 0;  // entries, of which PML tiles
};
int launch_stage_bulk_tma(int med, int coef_type, int wave16, int shape, const StageP &p, const TmaP &tm,
                          const BulkTiles &t, cudaStream_t st);
// FP16 stage levels: per-step scale from the last step's max |w| and the step's source bound
int launch_wave_scale(unsigned int *amax, const float *srcb, const int *d_it, int nt_total, int nshot, float *wsc,
                      cudaStream_t st);
// one bounded mbarrier wait that nothing completes (failure-path check)
int launch_wait_bound_check(int *err, int polls, cudaStream_t st);
// max |w| of the velocity / stress groups of each of `nshot` wavefields into amax[nshot][2]
void launch_wave_absmax(const float *w, long long sf, int nshot, unsigned int *amax, cudaStream_t st);
// 16-bit coefficient storage
void launch_absmax(const float *src, long long n, unsigned int *out, cudaStream_t st);
// min / max of one field over the cells any kernel reads (physical box + 3 ghosts per side),
// as order-preserving keys out[0] (min), out[1] (max); decode with coef_key_to_float
void launch_coef_minmax(const float *src, int ni, int nj, int nk, long long sx, long long sz, long long off0,
                        unsigned int *out, cudaStream_t st);
float coef_key_to_float(unsigned int key);
void launch_coef_to16(int coef_type, const float *src, void *dst, long long n, float scale, float offset, int field,
                      cudaStream_t st);
template <typename R>
int launch_source(const SrcPT<R> &s, cudaStream_t st);
template <typename R>
int launch_recv(const RecvPT<R> &r, cudaStream_t st);
int launch_advance(int *d_it, cudaStream_t st);
// reference layout (float, 3 ghosts) -> device layout of real type R, and back
template <typename R>
void launch_repack_in(const float *src, R *dst, int ni, int nj, int nk, long long sx, long long sz,
                      long long off0, int mode, int ghosts, cudaStream_t st);
template <typename R>
void launch_repack_out(const R *src, float *dst, int ni, int nj, int nk, long long sx, long long sz,
                       long long off0, cudaStream_t st);

}  // namespace cgfd

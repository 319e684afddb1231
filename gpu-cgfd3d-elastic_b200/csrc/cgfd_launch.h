// cgfd_launch.h -- host-visible launch entry points of the device kernels.
#pragma once

#include <cuda_runtime.h>

namespace cgfd {

struct StageP;
struct TmaP;

// Source injection of one stage (sv_curv_col_el_gpu.cu:227-301), applied to tmp/end.
struct SrcP {
  int nsrc, max_ext, max_nt;
  int force, moment;
  int stage;
  float ca, cb;
  const int *it_begin;         // [nsrc]
  const int *ext_num;          // [nsrc]
  const long long *ext_idx;    // [nsrc][max_ext] device-layout index
  const float *ext_wv;         // [nsrc][max_ext] coef * (1/rho) / jac
  const float *ext_wt;         // [nsrc][max_ext] coef / jac
  const float *stf;            // [nsrc][max_nt][4][9]: fx fy fz mxx myy mzz myz mxz mxy
  const int *src_shot;         // [nsrc] wavefield (shot) each source acts on
  float *tmp_out;
  float *end;
  long long sf;
  const int *d_it;
};

// Station sampling of w_pre (io_funcs.cu:1624-1666).
struct RecvP {
  int nsta;
  int nshot;                   // every shot is sampled at the same stations
  int nt_total;
  const long long *idx8;       // [nsta][8] device-layout corner index
  const float *w8;             // [nsta][8] trilinear weights (reference corner usage)
  const float *pre;
  long long sf;
  float *seis;                 // [nshot][nsta][9][nt_total]
  const int *d_it;
  int *d_flag;
};

// Each launcher returns the number of kernels it launched (0 or 1).
int launch_stage_bulk(int med, const StageP &p, int nzc, cudaStream_t st);
int launch_stage_surface(int med, const StageP &p, cudaStream_t st);
// TMA-pipelined bulk kernel: tile height, one-time function attributes, launch.
int tma_tile_y(int med);
cudaError_t tma_prepare(int med);
int launch_stage_bulk_tma(int med, const StageP &p, const TmaP &tm, int nzc, cudaStream_t st);
int launch_source(const SrcP &s, cudaStream_t st);
int launch_recv(const RecvP &r, cudaStream_t st);
int launch_advance(int *d_it, cudaStream_t st);
void launch_repack_in(const float *src, float *dst, int ni, int nj, int nk, long long sx, long long sz,
                      long long off0, int mode, int ghosts, cudaStream_t st);
void launch_repack_out(const float *src, float *dst, int ni, int nj, int nk, long long sx, long long sz,
                       long long off0, cudaStream_t st);

}  // namespace cgfd

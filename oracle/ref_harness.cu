/*
 * ref_harness.cu -- runs the reference's own CGFD3D solver code (compiled unmodified from the
 * reference sources) on one GPU for a problem written by tests/golden/ref_io.py, and dumps the
 * seismograms, the final wavefield and the reference-computed metrics.
 *
 * TEST INFRASTRUCTURE: it pins the CPU oracle (oracle/cgfd_oracle.cpp) and the product to the
 * reference. Setup follows main_curv_col_el_3d.cu:22-797 (grid import -> geometric_symmetry ->
 * gd_curv_metric_cal -> media -> src_read_locate_file -> wav_init -> io_recv_read_locate ->
 * bdry_pml_set -> bdry_free_set -> md_rho_to_slow), and the time loop restates
 * drv_rk_curv_col.cu:75-541 for one rank without halo exchange, slices, snapshots, PGV or the
 * exponential sponge, calling the reference's sv_curv_col_el_*_onestage (sv_curv_col_ac_iso_onestage
 * for acoustic media; sv_curv_col_vis_iso_onestage, md_vis_GMB_cal_Y, sv_curv_col_vis_iso_dvh2dvz and
 * sv_curv_col_vis_iso_free_gpu for visco-elastic media), wav_update and io_recv_keep.
 *
 * usage: ref_harness <dir>   (dir holds params.txt, coord.bin, medium.bin, src.src, station.list)
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "alloc.h"
#include "bdry_t.h"
#include "constants.h"
#include "cuda_common.h"
#include "fd_t.h"
#include "gd_t.h"
#include "io_funcs.h"
#include "md_t.h"
#include "src_t.h"
#include "sv_curv_col_ac_iso_gpu.h"
#include "sv_curv_col_el_aniso_gpu.h"
#include "sv_curv_col_el_gpu.h"
#include "sv_curv_col_el_iso_gpu.h"
#include "sv_curv_col_el_vti_gpu.h"
#include "sv_curv_col_vis_iso_gpu.h"
#include "wav_t.h"

static void die(const char *m) {
  fprintf(stderr, "ref_harness: %s\n", m);
  exit(2);
}

static void read_bin(const char *path, float *dst, size_t n) {
  FILE *f = fopen(path, "rb");
  if (!f) die(path);
  if (fread(dst, sizeof(float), n, f) != n) die("short read");
  fclose(f);
}

static void write_bin(const char *path, const float *src, size_t n) {
  FILE *f = fopen(path, "wb");
  if (!f) die(path);
  fwrite(src, sizeof(float), n, f);
  fclose(f);
}

int main(int argc, char **argv) {
  if (argc < 2) die("usage: ref_harness <dir>");
  char path[4096];
  const char *dir = argv[1];

  // ---- parameters
  int ni, nj, nk, medium_type, nt_total, nsteps, free_top;
  float dt, t0;
  int pml_on[3][2], pml_n[3][2];
  float pml_a[3][2], pml_b[3][2], pml_v[3][2];
  snprintf(path, sizeof(path), "%s/params.txt", dir);
  FILE *fp = fopen(path, "r");
  if (!fp) die("params.txt");
  if (fscanf(fp, "%d %d %d %d %d %d %d %f %f", &ni, &nj, &nk, &medium_type, &nt_total, &nsteps, &free_top, &dt, &t0) != 9)
    die("params header");
  for (int a = 0; a < 3; a++)
    for (int s = 0; s < 2; s++)
      if (fscanf(fp, "%d %d %f %f %f", &pml_on[a][s], &pml_n[a][s], &pml_a[a][s], &pml_b[a][s], &pml_v[a][s]) != 5)
        die("params pml");
  // visco-elastic media (CONST_MEDIUM_VISCOELASTIC_ISO, GMB): an extra line
  // "nmaxwell fr fmin fmax" (par_t.cu:736-770)
  int nmaxwell = 0;
  float vis_fr = 0.f, vis_fmin = 0.f, vis_fmax = 0.f;
  const bool visco = medium_type == CONST_MEDIUM_VISCOELASTIC_ISO;
  if (visco && fscanf(fp, "%d %f %f %f", &nmaxwell, &vis_fr, &vis_fmin, &vis_fmax) != 4) die("params visco");
  fclose(fp);

  int myid = 0;
  MPI_Comm comm = MPI_COMM_WORLD;

  fd_t fd;
  fd_set_macdrp(&fd);

  mympi_t mympi;
  memset(&mympi, 0, sizeof(mympi));
  mympi.nprocx = 1; mympi.nprocy = 1; mympi.nprocz = 1;
  mympi.myid = 0; mympi.comm = comm; mympi.topocomm = comm;
  for (int n = 0; n < CONST_NDIM_2; n++) mympi.neighid[n] = MPI_PROC_NULL;

  int abs_layers[3][2];
  for (int a = 0; a < 3; a++)
    for (int s = 0; s < 2; s++) abs_layers[a][s] = pml_on[a][s] ? pml_n[a][s] : 0;

  gd_t gd;
  memset(&gd, 0, sizeof(gd));
  gd_info_set(&gd, &mympi, ni, nj, nk, abs_layers, fd.fdx_nghosts, fd.fdy_nghosts, fd.fdz_nghosts);
  gd_curv_init(&gd);
  gd_metric_t metric;
  memset(&metric, 0, sizeof(metric));
  gd_curv_metric_init(&gd, &metric);

  // grid: physical points from coord.bin (reference layout, ghosts ignored), ghosts by
  // geometric_symmetry as in gd_curv_coord_import (gd_t.cu:727-796)
  {
    std::vector<float> c(3 * gd.siz_icmp);
    snprintf(path, sizeof(path), "%s/coord.bin", dir);
    read_bin(path, c.data(), c.size());
    float *dst[3] = {gd.x3d, gd.y3d, gd.z3d};
    for (int q = 0; q < 3; q++)
      for (int k = gd.nk1; k <= gd.nk2; k++)
        for (int j = gd.nj1; j <= gd.nj2; j++)
          for (int i = gd.ni1; i <= gd.ni2; i++) {
            size_t p = i + j * gd.siz_iy + k * gd.siz_iz;
            dst[q][p] = c[q * gd.siz_icmp + p];
          }
    geometric_symmetry(&gd, gd.v4d, gd.ncmp);
  }
  gd_curv_set_minmax(&gd);
  gd_curv_metric_cal(&gd, &metric, fd.fdc_len, fd.fdc_indx, fd.fdc_coef);

  // medium: physical points as md_import does (md_t.cu:269-326), ghosts left at 0
  md_t md;
  memset(&md, 0, sizeof(md));
  md_init(&gd, &md, medium_type, visco ? CONST_VISCO_GMB : 0, nmaxwell);
  {
    // visco-elastic: rho lambda mu Qp Qs (the first five of md_init's components); the Ylam /
    // Ymu components come from md_vis_GMB_cal_Y below
    const int nread = visco ? 5 : md.ncmp;
    std::vector<float> m((size_t)nread * gd.siz_icmp);
    snprintf(path, sizeof(path), "%s/medium.bin", dir);
    read_bin(path, m.data(), m.size());
    for (int c = 0; c < nread; c++) {
      float *ptr = md.v4d + md.cmp_pos[c];
      for (int k = gd.nk1; k <= gd.nk2; k++)
        for (int j = gd.nj1; j <= gd.nj2; j++)
          for (int i = gd.ni1; i <= gd.ni2; i++) {
            size_t p = i + j * gd.siz_iy + k * gd.siz_iz;
            ptr[p] = m[c * gd.siz_icmp + p];
          }
    }
  }

  if (visco) {  // main_curv_col_el_3d.cu:558-561
    md_vis_GMB_cal_Y(&md, vis_fr, vis_fmin, vis_fmax);
    // the fitted medium: lambda, mu (unrelaxed), Ylam[n], Ymu[n], then wl[n] (relaxation
    // frequencies)
    std::vector<float> fit((size_t)(2 + 2 * nmaxwell) * gd.siz_icmp + nmaxwell);
    memcpy(fit.data(), md.lambda, sizeof(float) * gd.siz_icmp);
    memcpy(fit.data() + gd.siz_icmp, md.mu, sizeof(float) * gd.siz_icmp);
    for (int n = 0; n < nmaxwell; n++) {
      memcpy(fit.data() + (2 + n) * gd.siz_icmp, md.Ylam[n], sizeof(float) * gd.siz_icmp);
      memcpy(fit.data() + (2 + nmaxwell + n) * gd.siz_icmp, md.Ymu[n], sizeof(float) * gd.siz_icmp);
    }
    memcpy(fit.data() + (2 + 2 * nmaxwell) * gd.siz_icmp, md.wl, sizeof(float) * nmaxwell);
    snprintf(path, sizeof(path), "%s/ref_gmb.bin", dir);
    write_bin(path, fit.data(), fit.size());
  }

  src_t src;
  memset(&src, 0, sizeof(src));
  snprintf(path, sizeof(path), "%s/src.src", dir);
  src_read_locate_file(&gd, &md, &src, path, t0, dt, fd.num_rk_stages, fd.rk_rhs_time, fd.fdx_max_half_len, comm,
                       myid);

  wav_t wav;
  memset(&wav, 0, sizeof(wav));
  if (medium_type == CONST_MEDIUM_ACOUSTIC_ISO) wav_ac_init(&gd, &wav, fd.num_rk_stages);  // main:676-681
  else wav_init(&gd, &wav, fd.num_rk_stages, visco ? CONST_VISCO_GMB : 0, nmaxwell);

  iorecv_t iorecv;
  memset(&iorecv, 0, sizeof(iorecv));
  snprintf(path, sizeof(path), "%s/station.list", dir);
  io_recv_read_locate(&gd, &iorecv, nt_total, wav.ncmp, path, comm, myid);

  bdrypml_t bdrypml;
  memset(&bdrypml, 0, sizeof(bdrypml));
  bdry_pml_set(&gd, &wav, &bdrypml, mympi.neighid, pml_on, abs_layers, pml_a, pml_b, pml_v);
  bdryfree_t bdryfree;
  memset(&bdryfree, 0, sizeof(bdryfree));
  int free_sides[3][2] = {{0, 0}, {0, 0}, {0, free_top}};
  bdry_free_set(&gd, &bdryfree, mympi.neighid, free_sides);

  // export the reference metrics (before anything else touches them)
  snprintf(path, sizeof(path), "%s/ref_metric.bin", dir);
  write_bin(path, metric.v4d, (size_t)10 * gd.siz_icmp);

  md_rho_to_slow(md.rho, md.siz_icmp);

  // ---- time loop: drv_rk_curv_col.cu:75-541 on one rank
  if (bdryfree.is_sides_free[CONST_NDIM - 1][1] == 1 && md.medium_type != CONST_MEDIUM_ACOUSTIC_ISO) {  // :73-95
    if (md.medium_type == CONST_MEDIUM_ELASTIC_ISO) sv_curv_col_el_iso_dvh2dvz(&gd, &metric, &md, &bdryfree);
    else if (md.medium_type == CONST_MEDIUM_ELASTIC_VTI) sv_curv_col_el_vti_dvh2dvz(&gd, &metric, &md, &bdryfree);
    else if (visco)
      sv_curv_col_vis_iso_dvh2dvz(&gd, &metric, &md, &bdryfree, fd.fdc_len, fd.fdc_indx, fd.fdc_coef);
    else sv_curv_col_el_aniso_dvh2dvz(&gd, &metric, &md, &bdryfree);
  }
  gd_t gd_d;
  md_t md_d;
  src_t src_d;
  wav_t wav_d;
  gd_metric_t metric_d;
  fd_wav_t fd_wav_d;
  bdryfree_t bdryfree_d;
  bdrypml_t bdrypml_d;
  init_gdinfo_device(&gd, &gd_d);
  init_md_device(&md, &md_d);
  init_fd_device(&fd, &fd_wav_d, &gd);
  init_src_device(&src, &src_d);
  init_metric_device(&metric, &metric_d);
  init_wave_device(&wav, &wav_d);
  init_bdryfree_device(&gd, &bdryfree, &bdryfree_d);
  init_bdrypml_device(&gd, &bdrypml, &bdrypml_d);

  float *w_buff = wav.v5d;
  float *w_pre_d = wav_d.v5d + wav_d.siz_ilevel * 0;
  float *w_tmp_d = wav_d.v5d + wav_d.siz_ilevel * 1;
  float *w_rhs_d = wav_d.v5d + wav_d.siz_ilevel * 2;
  float *w_end_d = wav_d.v5d + wav_d.siz_ilevel * 3;
  float *w_cur_d;
  if (bdrypml_d.is_enable_pml == 1)
    for (int a = 0; a < CONST_NDIM; a++)
      for (int s = 0; s < 2; s++)
        if (bdrypml_d.is_sides_pml[a][s] == 1) {
          bdrypml_auxvar_t *x = &(bdrypml_d.auxvar[a][s]);
          x->pre = x->var + x->siz_ilevel * 0;
          x->tmp = x->var + x->siz_ilevel * 1;
          x->rhs = x->var + x->siz_ilevel * 2;
          x->end = x->var + x->siz_ilevel * 3;
        }

  // free-surface peak ground motion, as drv_rk_curv_col.cu:174-186 allocates it
  float *PG_d = nullptr, *Dis_accu_d = nullptr;
  if (free_top) {
    PG_d = init_PGVAD_device(&gd);
    Dis_accu_d = init_Dis_accu_device(&gd);
  }

  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0);
  // Statement by statement against drv_rk_curv_col.cu (line numbers of that file). Left out:
  // io_line_keep / io_slice_nc_put / io_snap_nc_put (:203-215; outputs the harness does not
  // write), the MPI message pack / start / wait / unpack (:336, :353-355, :407-408, :461-462,
  // :492-501; one rank, no neighbours), the
  // stubbed NaN check (:507-510) and the exponential sponge (:513-515, not enabled by the cases). The per-stage cudaDeviceSynchronize (:333) is implied by the
  // default stream's ordering.
  for (int it = 0; it < nsteps; it++) {  // :193
    io_recv_keep(&iorecv, w_pre_d, w_buff, it, wav.ncmp, wav.siz_icmp);  // :200
    int ipair = it % fd.num_of_pairs;                                     // :221
    for (int istage = 0; istage < fd.num_rk_stages; istage++) {         // :224
      w_cur_d = istage == 0 ? w_pre_d : w_tmp_d;                          // :237-257
      if (bdrypml_d.is_enable_pml == 1)
        for (int a = 0; a < CONST_NDIM; a++)
          for (int s = 0; s < 2; s++)
            bdrypml_d.auxvar[a][s].cur = istage == 0 ? bdrypml_d.auxvar[a][s].pre : bdrypml_d.auxvar[a][s].tmp;
      src_set_time(&src_d, it, istage);  // :260
      // :263-315, the acoustic and the three elastic media
      if (md_d.medium_type == CONST_MEDIUM_ACOUSTIC_ISO)
        sv_curv_col_ac_iso_onestage(w_cur_d, w_rhs_d, wav_d, fd_wav_d, gd_d, metric_d, md_d, bdrypml_d, bdryfree_d, src_d,
                                    fd.num_of_fdx_op, fd.pair_fdx_op[ipair][istage], fd.num_of_fdy_op,
                                    fd.pair_fdy_op[ipair][istage], fd.num_of_fdz_op, fd.pair_fdz_op[ipair][istage],
                                    fd.fdz_max_len, myid);
      else if (md_d.medium_type == CONST_MEDIUM_ELASTIC_ISO)
        sv_curv_col_el_iso_onestage(w_cur_d, w_rhs_d, wav_d, fd_wav_d, gd_d, metric_d, md_d, bdrypml_d, bdryfree_d, src_d,
                                    fd.num_of_fdx_op, fd.pair_fdx_op[ipair][istage], fd.num_of_fdy_op,
                                    fd.pair_fdy_op[ipair][istage], fd.num_of_fdz_op, fd.pair_fdz_op[ipair][istage],
                                    fd.fdz_max_len, myid);
      else if (visco)  // :317-331
        sv_curv_col_vis_iso_onestage(w_cur_d, w_rhs_d, wav_d, fd_wav_d, gd_d, metric_d, md_d, bdrypml_d, bdryfree_d, src_d,
                                     fd.num_of_fdx_op, fd.pair_fdx_op[ipair][istage], fd.num_of_fdy_op,
                                     fd.pair_fdy_op[ipair][istage], fd.num_of_fdz_op, fd.pair_fdz_op[ipair][istage],
                                     fd.fdz_max_len, myid);
      else if (md_d.medium_type == CONST_MEDIUM_ELASTIC_VTI)
        sv_curv_col_el_vti_onestage(w_cur_d, w_rhs_d, wav_d, fd_wav_d, gd_d, metric_d, md_d, bdrypml_d, bdryfree_d, src_d,
                                    fd.num_of_fdx_op, fd.pair_fdx_op[ipair][istage], fd.num_of_fdy_op,
                                    fd.pair_fdy_op[ipair][istage], fd.num_of_fdz_op, fd.pair_fdz_op[ipair][istage],
                                    fd.fdz_max_len, myid);
      else
        sv_curv_col_el_aniso_onestage(w_cur_d, w_rhs_d, wav_d, fd_wav_d, gd_d, metric_d, md_d, bdrypml_d, bdryfree_d,
                                      src_d, fd.num_of_fdx_op, fd.pair_fdx_op[ipair][istage], fd.num_of_fdy_op,
                                      fd.pair_fdy_op[ipair][istage], fd.num_of_fdz_op, fd.pair_fdz_op[ipair][istage],
                                      fd.fdz_max_len, myid);
      dim3 block(256);
      dim3 grid((wav_d.siz_ilevel + block.x - 1) / block.x);
      auto aux_update = [&](int kind, float coef) {
        if (bdrypml_d.is_enable_pml != 1) return;
        for (int a = 0; a < CONST_NDIM; a++)
          for (int s = 0; s < 2; s++)
            if (bdrypml_d.is_sides_pml[a][s] == 1) {
              bdrypml_auxvar_t *x = &(bdrypml_d.auxvar[a][s]);
              dim3 g2((x->siz_ilevel + block.x - 1) / block.x);
              if (kind == 0) wav_update<<<g2, block>>>(x->siz_ilevel, coef, x->tmp, x->pre, x->rhs);
              else if (kind == 1) wav_update<<<g2, block>>>(x->siz_ilevel, coef, x->end, x->pre, x->rhs);
              else wav_update_end<<<g2, block>>>(x->siz_ilevel, coef, x->end, x->rhs);
            }
      };
      if (istage == 0) {  // :339-395
        float ca = fd.rk_a[istage] * dt, cb = fd.rk_b[istage] * dt;
        wav_update<<<grid, block>>>(wav_d.siz_ilevel, ca, w_tmp_d, w_pre_d, w_rhs_d);  // :349
        aux_update(0, ca);                                                              // :358-372
        wav_update<<<grid, block>>>(wav_d.siz_ilevel, cb, w_end_d, w_pre_d, w_rhs_d);  // :378
        aux_update(1, cb);                                                              // :381-395
      } else if (istage < fd.num_rk_stages - 1) {  // :396-447
        float ca = fd.rk_a[istage] * dt, cb = fd.rk_b[istage] * dt;
        wav_update<<<grid, block>>>(wav_d.siz_ilevel, ca, w_tmp_d, w_pre_d, w_rhs_d);  // :403
        aux_update(0, ca);                                                              // :410-424
        wav_update_end<<<grid, block>>>(wav_d.siz_ilevel, cb, w_end_d, w_rhs_d);       // :430
        aux_update(2, cb);                                                              // :433-447
      } else {  // :448-478
        float cb = fd.rk_b[istage] * dt;
        wav_update_end<<<grid, block>>>(wav_d.siz_ilevel, cb, w_end_d, w_rhs_d);  // :456
        aux_update(2, cb);                                                         // :464-478
        if (visco && free_top) {                                                   // :479-490
          dim3 fb(32, 16), fg((ni + fb.x - 1) / fb.x, (nj + fb.y - 1) / fb.y);
          sv_curv_col_vis_iso_free_gpu<<<fg, fb>>>(w_end_d, wav_d, gd_d, metric_d, md_d, bdryfree_d, myid);
        }
      }
    }
    if (free_top) {  // drv_rk_curv_col.cu:519-527
      dim3 pb(8, 8), pgr((ni + 7) / 8, (nj + 7) / 8);
      PG_calcu_gpu<<<pgr, pb>>>(w_end_d, w_pre_d, gd_d, PG_d, Dis_accu_d, dt);
    }
    float *t = w_pre_d;  // :529
    w_pre_d = w_end_d;
    w_end_d = t;
    if (bdrypml_d.is_enable_pml == 1)  // :531-541
      for (int a = 0; a < CONST_NDIM; a++)
        for (int s = 0; s < 2; s++) {
          bdrypml_auxvar_t *x = &(bdrypml_d.auxvar[a][s]);
          x->cur = x->pre;
          x->pre = x->end;
          x->end = x->cur;
        }
  }
  cudaEventRecord(e1);
  cudaEventSynchronize(e1);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaError_t err = cudaGetLastError();
  if (err != cudaSuccess) die(cudaGetErrorString(err));

  // ---- outputs, in the 9-component layout (acoustic: Vx Vy Vz P, components 4-8 left 0)
  std::vector<float> seis((size_t)iorecv.total_number * 9 * nt_total, 0.f);
  // samples of steps that were not run stay 0 (the reference leaves them uninitialised)
  for (int r = 0; r < iorecv.total_number; r++)
    for (int c = 0; c < wav.ncmp && c < 9; c++)
      for (int t = 0; t < nsteps && t < nt_total; t++)
        seis[((size_t)r * 9 + c) * nt_total + t] = iorecv.recvone[r].seismo[(size_t)c * nt_total + t];
  snprintf(path, sizeof(path), "%s/ref_seismo.bin", dir);
  write_bin(path, seis.data(), seis.size());
  std::vector<float> w((size_t)9 * gd.siz_icmp, 0.f);
  // (visco-elastic: the 9 wave fields; the memory variables follow them in the level)
  cudaMemcpy(w.data(), w_pre_d, sizeof(float) * std::min(wav.ncmp, 9) * gd.siz_icmp, cudaMemcpyDeviceToHost);
  snprintf(path, sizeof(path), "%s/ref_wave.bin", dir);
  write_bin(path, w.data(), w.size());
  if (free_top) {
    std::vector<float> pg((size_t)15 * gd.nx * gd.ny);
    cudaMemcpy(pg.data(), PG_d, sizeof(float) * pg.size(), cudaMemcpyDeviceToHost);
    snprintf(path, sizeof(path), "%s/ref_pg.bin", dir);
    write_bin(path, pg.data(), pg.size());
  }
  snprintf(path, sizeof(path), "%s/ref_info.txt", dir);
  fp = fopen(path, "w");
  fprintf(fp, "nrecv %d\nnsrc %d\nloop_ms %.4f\ncell_stages %lld\n", iorecv.total_number, src.total_number, ms,
          (long long)ni * nj * nk * 4 * nsteps);
  fclose(fp);
  return 0;
}

/*
 * cgfd_b200.h -- C ABI of the B200-native CGFD3D elastic time-stepping path.
 *
 * The library (libcgfd_b200.so) replaces the time loop of hpc-lee/gpu-CGFD3D-elastic:
 *   drv_rk_curv_col_allstep()          src/forward/drv_rk_curv_col.cu:28-567
 *   sv_curv_col_el_{iso,vti,aniso}_onestage()  sv_curv_col_el_*_gpu.cu (RHS of one RK stage)
 *   wav_update / wav_update_end         src/forward/wav_t.cu:362-378 (RK combine)
 *   io_recv_keep                        src/forward/io_funcs.cu:1624-1666 (station sampling)
 * together with the setup steps whose results that loop consumes (CFS-PML coefficients,
 * free-surface velocity-gradient conversion matrices, source smoothing and source time
 * functions, station location).
 *
 * Conventions shared with the reference:
 *  - Host arrays use the reference layout var[cmp][k][j][i] with i fastest and CGFD_NGHOST
 *    ghost points on every side: nx = ni+6, ny = nj+6, nz = nk+6 (gd_t.cu:1888-2043).
 *  - Wavefield components are ordered Vx,Vy,Vz,Txx,Tyy,Tzz,Tyz,Txz,Txy (wav_t.cu:100-143).
 *    Acoustic media (sv_curv_col_ac_iso_gpu.cu, wav_ac_init wav_t.cu:190-250) use Vx,Vy,Vz,P:
 *    P takes the Txx slot (component 3) and components 4-8 stay 0, so every wavefield,
 *    seismogram, slice and snapshot array keeps the 9-component layout. Acoustic sources use
 *    the force and the Mxx moment component (the pressure source of
 *    sv_curv_col_ac_iso_rhs_src_gpu); acoustic problems run in CGFD_PREC_FP32 or CGFD_PREC_FP64.
 *  - Metric components are ordered jac,xi_x,xi_y,xi_z,eta_x,eta_y,eta_z,zeta_x,zeta_y,zeta_z
 *    (gd_t.cu:140-200, gd_curv_metric_init).
 *  - Medium components are ordered as the media_*.nc variables (md_t.cu:16-268):
 *      acoustic_iso : rho, kappa
 *      elastic_iso  : rho, lambda, mu
 *      elastic_vti  : rho, c11, c13, c33, c55, c66
 *      elastic_aniso: rho, c11,c12,c13,c14,c15,c16, c22,c23,c24,c25,c26, c33,c34,c35,c36,
 *                     c44,c45,c46, c55,c56, c66
 *    rho is the density; the library converts it to 1/rho like md_rho_to_slow (md_t.cu:622-637).
 *
 * Error convention: every entry point returns 0 on success and a negative CGFD_ERR_* code
 * on failure; cgfd_last_error() then returns a message for the calling thread. Nothing in
 * the library calls exit() or abort() (the reference aborts via MPI_Abort / exit).
 */
#ifndef CGFD_B200_H
#define CGFD_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CGFD_NGHOST 3
#define CGFD_NCMP   9

/* medium ids: src/forward/constants.h:20-24 */
#define CGFD_MEDIUM_ACOUSTIC_ISO  1
#define CGFD_MEDIUM_ELASTIC_ISO   2
#define CGFD_MEDIUM_ELASTIC_VTI   3
#define CGFD_MEDIUM_ELASTIC_ANISO 4
#define CGFD_MEDIUM_VISCO_ISO     5  /* visco-elastic iso, generalized Maxwell body (CONST_VISCO_GMB) */

/* wavelet names accepted in .src files: src_t.cu:873-903 (src_cal_wavelet) */
#define CGFD_WAVELET_RICKER         0
#define CGFD_WAVELET_GAUSSIAN       1
#define CGFD_WAVELET_RICKER_DERIV   2
#define CGFD_WAVELET_GAUSSIAN_DERIV 3
#define CGFD_WAVELET_KLAUDER        4

/* Storage precision of the device state; arithmetic is FP32 in every mode. The 16-bit
   coefficient modes store the 9 metric fields, 1/rho and the moduli (the Jacobian, read only
   at the free surface, stays FP32) with one scale and offset per field, stochastically
   rounded (zero-mean per-cell error, so a homogeneous layer keeps its wave speed). */
#define CGFD_PREC_FP32       0  /* everything FP32 (the reference's arithmetic)              */
#define CGFD_PREC_BF16_COEF  1  /* coefficients BF16 (power-of-two scale), wavefield FP32     */
#define CGFD_PREC_FP16_COEF  2  /* coefficients FP16 (power-of-two scale), wavefield FP32     */
#define CGFD_PREC_U16_COEF   3  /* coefficients 16-bit fixed point over each field's range    */
#define CGFD_PREC_FP16_WAVE  4  /* U16 coefficients + RK stage wavefields FP16 (dynamic per-
                                   step scale); the solution levels stay FP32                */
#define CGFD_PREC_FP64       5  /* FP64 build of the same kernels: wavefield, coefficients, PML
                                   auxiliaries and all arithmetic in double (the reference
                                   each precision mode's seismogram error is measured against;
                                   direct-load bulk kernel, not a production mode)            */

/* status codes */
#define CGFD_OK               0
#define CGFD_ERR_INVALID     -1   /* malformed description or argument                     */
#define CGFD_ERR_CUDA        -2   /* CUDA runtime error                                     */
#define CGFD_ERR_NOMEM       -3   /* device memory budget exceeded                          */
#define CGFD_ERR_NONFINITE   -4   /* NaN/Inf detected in the wavefield                      */
#define CGFD_ERR_UNSUPPORTED -5   /* option recognised but not implemented                  */
#define CGFD_ERR_IO          -6   /* file could not be read or written                      */
#define CGFD_ERR_BUSY        -7   /* serving queue full / request not finished              */

/* One CFS-PML face (par_t.cu:230-371 "cfspml" block; bdry_t.cu:85-257 bdry_pml_set). */
typedef struct cgfd_pml_face {
  int   enable;       /* 1: CFS-PML on this face                                           */
  int   num_layers;   /* N; the face box spans N+1 grid points (bdry_t.cu:138-155)          */
  float alpha_max;
  float beta_max;
  float ref_vel;
} cgfd_pml_face;

/*
 * Sources, as read from a .src file (src_t.cu:143-790, src_read_locate_file), located by grid
 * index (loc_coord_type 0) or by physical coordinates (1; gd_curv_coord_to_glob_indx_gpu and
 * gd_curv_depth_to_axis, gd_t.cu:1189-1500; desc->coord required).
 */
typedef struct cgfd_source_desc {
  int   num;              /* in_num_source                                                 */
  int   stf_given;        /* 0: wavelet by name, 1: sampled values                         */
  float stf_length;       /* stf_given 0: length of the source time function (s)           */
  float stf_dt;           /* stf_given 1: sample interval                                  */
  int   stf_nt;           /* stf_given 1: number of samples                                */
  int   cmp_type;         /* 1 force, 2 moment, 3 force+moment (quirk kept: 3 = force only) */
  int   mechanism_type;   /* 0 moment tensor, 1 strike/dip/rake + mu,D,A                   */
  int   loc_coord_type;   /* 0 grid index, 1 physical coordinates                          */
  int   loc_3dim;         /* 0: z is a grid index / coordinate, 1: z is the depth below the
                             free surface (index count or length)                           */
  const float *loc;       /* [num][3] x,y,z (0-based index, or coordinates)                */
  const float *t_start;   /* [num] wavelet_tstart                                          */
  const int   *wavelet;   /* [num] CGFD_WAVELET_* (stf_given 0)                             */
  const float *wavelet_coefs; /* [num][10]                                                 */
  const float *cmp;       /* stf_given 0: [num][9] = fx,fy,fz,mxx,myy,mzz,myz,mxz,mxy       */
  const float *cmp_values;/* stf_given 1: [num][stf_nt][9], same order                      */
} cgfd_source_desc;

/* Stations, as read from a station list (io_funcs.cu:24-299, io_recv_read_locate). */
typedef struct cgfd_station_desc {
  int          num;
  const int   *flag_coord; /* [num] 0: grid index, 1: physical coordinates                 */
  const int   *flag_depth; /* [num] 1: z is the depth below the free surface               */
  const float *loc;        /* [num][3] x,y 1-based index (or coordinates), z per flags      */
} cgfd_station_desc;

/*
 * Everything drv_rk_curv_col_allstep() consumes, in the reference's host layout.
 */
/*
 * Visco-elastic media (CGFD_MEDIUM_VISCO_ISO; the par file's visco_config, par_t.cu:728-770):
 * a generalized Maxwell body of nmaxwell relaxation mechanisms fitted to the per-point Qp and Qs
 * over [fmin, fmax] with the moduli given at the reference frequency fr (md_vis_GMB_cal_Y).
 */
typedef struct cgfd_visco_desc {
  int   nmaxwell;           /* 1..10                                                          */
  float fr, fmin, fmax;     /* Hz; 0 < fmin < fmax                                           */
} cgfd_visco_desc;

typedef struct cgfd_problem_desc {
  int ni, nj, nk;           /* physical points incl. PML layers (ghosts excluded)          */
  int medium_type;          /* CGFD_MEDIUM_ACOUSTIC_ISO, CGFD_MEDIUM_ELASTIC_* or _VISCO_ISO   */
  const float *coord;       /* [3][nz][ny][nx] x,y,z with ghosts filled; used for the PML
                               length/spacing average (bdry_t.cu:334-451). May be NULL when
                               no PML face is enabled and metric is given.                   */
  const float *metric;      /* [10][nz][ny][nx] jac, xi_x..zeta_z with ghosts filled; or
                               NULL: computed on the device from coord (the "calculate"
                               metric method: gd_curv_metric_cal + geometric_symmetry, here
                               in FP64, equal to cgfd_metric_calc bitwise), so that only the
                               coordinates cross the host link                               */
  const float *medium;      /* [ncmp][nz][ny][nx]                                           */
  cgfd_pml_face pml[3][2];  /* [x,y,z][left/bottom, right/top]                              */
  int   free_top;           /* 1: traction-image free surface at the top (z2)              */
  float dt;
  float t0;
  int   nt_total;           /* number_of_time_steps + 1 (main_curv_col_el_3d.cu:589)        */
  cgfd_source_desc  src;
  cgfd_station_desc sta;
  int   precision;          /* CGFD_PREC_*                                                  */
  int   device;             /* CUDA device ordinal                                          */
  const cgfd_visco_desc *visco; /* CGFD_MEDIUM_VISCO_ISO: the GMB parameters (medium [5] = rho,
                               lambda, mu, Qp, Qs); NULL for the other media                 */
} cgfd_problem_desc;

typedef struct cgfd_problem cgfd_problem;

/* Library version (major*10000 + minor*100 + patch). */
int cgfd_version(void);

/* Message for the last failed call on this thread ("" if none). */
const char *cgfd_last_error(void);

/*
 * Build device-resident state for one forward simulation: the setup work that precedes
 * drv_rk_curv_col_allstep() (bdry_pml_set, the dvh2dvz matrices, src_read_locate_file's
 * smoothing and STF tables, io_recv_read_locate) plus the device mirrors of alloc.cu.
 * Replaces: the init_*_device calls at drv_rk_curv_col.cu:109-117.
 */
int cgfd_problem_create(const cgfd_problem_desc *desc, cgfd_problem **out);

/*
 * Batched sources on one grid: nshot (1..32767) independent wavefields share the grid,
 * metrics, medium, boundaries and stations (desc->src is ignored); shots[s] holds the sources
 * of wavefield s. One launch per kernel and RK stage covers every shot; the shots of a group
 * (cgfd_set_shot_group) run side by side, so that the coefficient tiles of a grid tile are
 * read once from HBM for the group. Seismograms come back as [nshot][nsta][9][nt_total].
 * No counterpart in the reference (one source set per run there).
 */
int cgfd_batch_create(const cgfd_problem_desc *desc, int nshot, const cgfd_source_desc *shots,
                      cgfd_problem **out);
int cgfd_num_shots(const cgfd_problem *p);

/*
 * Advance nsteps time steps (4 RK stages each), sampling the stations at the start of
 * every step like io_recv_keep. nsteps < 0 runs to nt_total.
 * Replaces: the time loop drv_rk_curv_col.cu:193-541.
 */
int cgfd_run(cgfd_problem *p, int nsteps);

/* Index of the next time step to run (0 after create). */
int cgfd_current_step(const cgfd_problem *p);

/* Set the step counter (selects the MacCormack pair it%8 and the source time). */
int cgfd_set_step(cgfd_problem *p, int it);

/*
 * Seismograms, [nshot][nsta][9][nt_total] in component order Vx..Txy (nshot = 1 unless
 * created by cgfd_batch_create); entries for steps not yet run are 0. Replaces: iorecv->recvone[r].seismo (io_funcs.cu:283-288, 1651-1659).
 */
int cgfd_get_seismograms(cgfd_problem *p, float *out);

/* Number of stations located inside the grid (io_recv_read_locate's total_number). */
int cgfd_num_stations(const cgfd_problem *p);

/*
 * For each located station (seismogram order): its position in the input list
 * (input_index[nsta], may be NULL) and the physical 0-based grid index of its interpolation
 * corner 0 (ijk[nsta][3], may be NULL). Replaces: iorecv->recvone[r].i/j/k (io_funcs.cu:250-260).
 */
int cgfd_station_info(const cgfd_problem *p, int *input_index, int *ijk);

/*
 * Current wavefield w_pre in the reference layout [9][nz][ny][nx] (ghosts are 0), e.g.
 * for a final snapshot. Replaces: the device-to-host copy of io_snap_nc_put.
 */
int cgfd_get_wavefield(cgfd_problem *p, float *out);

/* Overwrite w_pre (physical points only; ghosts stay 0; acoustic media take components 0-3). */
int cgfd_set_wavefield(cgfd_problem *p, const float *in);

/*
 * Strided sub-box of the current wavefield w_pre (the state at the start of the next step),
 * all 9 components: out[9][count[2]][count[1]][count[0]] with point (n0,n1,n2) at physical
 * index start[a] + n_a * stride[a] (0-based, x,y,z order). Replaces: the per-component
 * io_snap_pack_buff launches + copies of io_snap_nc_put (io_funcs.cu:1049-1256, 1569-1595).
 */
int cgfd_get_wavefield_box(cgfd_problem *p, int shot, const int *start, const int *count, const int *stride,
                           float *out);

/*
 * Free-surface peak ground motion accumulated over the steps run so far, [15][ny][nx] in the
 * order PGV, PGVh, PGVx, PGVy, PGVz, PGA, PGAh, PGAx, PGAy, PGAz, PGD, PGDh, PGDx, PGDy, PGDz
 * (ghost points 0), i.e. the array PG_slice_output writes (io_funcs.cu:2065-2124), updated
 * after every time step like PG_calcu_gpu (wav_t.cu:281-360, drv_rk_curv_col.cu:519-527).
 * CGFD_ERR_UNSUPPORTED when the problem has no free surface.
 */
int cgfd_get_peak_motion(cgfd_problem *p, int shot, float *out);

/*
 * Line receivers: the 9 components of w_pre at grid points (no interpolation) at the start of
 * every step, like io_line_keep (io_funcs.cu:1669-1700) on the points io_line_locate
 * (io_funcs.cu:300-414) builds from the "receiver_line" entries (point n of a line at
 * start + n * incre; the caller drops points outside the grid as io_line_locate does, this
 * call refuses them). ijk[npts][3] are physical 0-based indices. Replaces the receiver set of
 * any earlier call; steps run before the call hold zeros. Samples go to a device buffer and
 * come back with cgfd_get_line_seismograms as [nshot][npts][9][nt_total] (the array
 * io_line_output_sac writes, io_funcs.cu:1943-1985). The buffers count in cgfd_device_bytes.
 */
int cgfd_set_line_receivers(cgfd_problem *p, int npts, const int *ijk);
int cgfd_get_line_seismograms(cgfd_problem *p, float *out);

/*
 * Slices: the full x, y and z planes (physical 0-based indices ix[nx], iy[ny], iz[nz]) of the
 * 9 components of w_pre at the start of every step, like io_slice_nc_put
 * (io_funcs.cu:667-788, called every step at drv_rk_curv_col.cu:206) on the planes
 * io_slice_locate (io_funcs.cu:418-528) keeps. The planes are packed on the device into a ring
 * of ring_steps steps (no host round trip inside the time loop); cgfd_get_slices returns the
 * planes of one step `it` still in the ring (current_step - ring_steps <= it < current_step)
 * as the x slices [nx][9][nk][nj], then the y slices [ny][9][nk][ni], then the z slices
 * [nz][9][nj][ni]. Replaces any earlier slice set; the ring counts in cgfd_device_bytes.
 */
int cgfd_set_slices(cgfd_problem *p, int nx, const int *ix, int ny, const int *iy, int nz, const int *iz,
                    int ring_steps);
int cgfd_get_slices(cgfd_problem *p, int shot, int it, float *out);

/* Per-shot variants of cgfd_get_wavefield / cgfd_set_wavefield for batched problems. */
int cgfd_get_wavefield_shot(cgfd_problem *p, int shot, float *out);
int cgfd_set_wavefield_shot(cgfd_problem *p, int shot, const float *in);

/*
 * Same result as cgfd_get_wavefield_shot, but allocates no device memory: the repack goes
 * through one static 4 MiB device array (2^20 floats) shared by every call, a chunk of
 * reference-layout z planes at a time. For callers that cannot allocate: a server that holds
 * the device at its memory budget with resident problems, where the temporary buffer of
 * cgfd_get_wavefield_shot (one full wavefield component, (ni+6)(nj+6)(nk+6) floats, from the
 * device's memory pool) may not fit and a snapshot must not fail for lack of memory.
 * Limit: one plane, (ni+6)*(nj+6) floats, must fit the array; larger grids get
 * CGFD_ERR_INVALID. The array and its repack kernel are loaded on a device when the first
 * problem is created there (cgfd_problem_create / cgfd_batch_create look up the array's
 * address, with that device current), and stay until the process exits; the call itself
 * takes no device memory. Nothing in the array needs to start at zero (each chunk is fully
 * written before it is copied). Calls that overlap on one device (other threads, other
 * problems) race on the shared array and must be serialised by the caller.
 * No counterpart in the reference.
 */
int cgfd_get_wavefield_shot_noalloc(cgfd_problem *p, int shot, float *out);

/* Device bytes held by the problem (including the staging buffer of cgfd_get_wavefield_box
   once it has been used: it grows to the largest box asked for and stays with the problem). */
size_t cgfd_device_bytes(const cgfd_problem *p);

/*
 * Device bytes cgfd_batch_create(desc, nshot, shots) (shots NULL and nshot 1: the plain
 * cgfd_problem_create) will hold once built (*resident, = cgfd_device_bytes) and at its
 * high-water mark during the build (*peak); host work only, no device call.
 * No counterpart in the reference.
 */
int cgfd_problem_bytes(const cgfd_problem_desc *desc, int nshot, const cgfd_source_desc *shots,
                       size_t *resident, size_t *peak);

/* Release all device and host state. Replaces: drv_rk_curv_col.cu:546-556. */
int cgfd_problem_destroy(cgfd_problem *p);

/*
 * Stream the library launches on (a cudaStream_t, returned as void* so that the header
 * needs no CUDA include).
 */
void *cgfd_stream(cgfd_problem *p);

/*
 * Enqueue n time steps on the problem's stream without synchronising (benchmarks and
 * overlapping host work). cgfd_synchronize() waits and reports device-side errors:
 * CGFD_ERR_NONFINITE when a step produced a NaN/Inf solution value anywhere in the grid
 * (checked by the RK combine of the last stage of every step; the reference's check,
 * drv_rk_curv_col.cu:507-510 / wav_check_value wav_t.cu:260-279, is stubbed out) or sampled
 * one at a station; CGFD_ERR_CUDA when a stage kernel's pipeline wait timed out.
 */
int cgfd_enqueue_steps(cgfd_problem *p, int nsteps);
int cgfd_synchronize(cgfd_problem *p);

/*
 * Failure-path check: runs, on the problem's stream, one device-side pipeline wait that no
 * transfer completes, bounded like the stage kernels' waits (2^16 polls), and reports it the
 * way a lost transfer in a stage would be reported: CGFD_ERR_CUDA with the pipeline-timeout
 * message. The device error word is cleared afterwards, so the problem stays usable.
 * No counterpart in the reference.
 */
int cgfd_check_wait_bound(cgfd_problem *p);

/* ---- tuning knobs -------------------------------------------------------------------- */

/* Disable (0) or enable (1, default) CUDA-graph replay of the time steps. */
int cgfd_set_graph_mode(cgfd_problem *p, int on);

/* z planes per thread block of the bulk stage kernel (autotuner knob). */
int cgfd_set_zchunk(cgfd_problem *p, int nzc);
int cgfd_get_zchunk(const cgfd_problem *p);

/*
 * Tile shape of the TMA bulk kernel, 0 or 1, per medium
 *   iso, VTI: 32x8 columns at two blocks per SM | 32x4 at three blocks per SM
 *   21-Cij:   32x4 at three blocks per SM      | 32x8 at one block per SM (w_pre staged too).
 * Default: 1 for iso media, 0 otherwise (with z chunks of about 12 planes). Results do not
 * depend on the shape (the per-cell arithmetic is the same).
 */
int cgfd_set_tile_shape(cgfd_problem *p, int shape);
int cgfd_get_tile_shape(const cgfd_problem *p);

/*
 * Block order of a batch's bulk kernel: the shots come in groups of `group` (default 8; values
 * above the batch's shot count mean every shot), each group's blocks cover every tile before
 * the next group's start, and within a group the shot is the fastest block index. The blocks
 * of one tile then share its coefficient tiles through L2 while a tile's x-y neighbours of the
 * same shot stay resident beside it. Results do not depend on the group. Graphs are rebuilt.
 * cgfd_get_shot_group returns the group in effect (at most the shot count). No counterpart in
 * the reference.
 */
int cgfd_set_shot_group(cgfd_problem *p, int group);
int cgfd_get_shot_group(const cgfd_problem *p);

/*
 * Autotuner of the bulk kernel's tile: times `steps` graph-replayed time steps for each tile
 * shape (cgfd_set_tile_shape) and z-chunk length (planes per thread block column: 8, 10, 12,
 * 14, 16, 20, 24, 32, 48, 64, 96 and all bulk planes; the shapes interleaved) on this problem,
 * times the three fastest and the default tiling twice more over 2 x `steps` steps in a
 * palindromic order and keeps the pair of lowest mean (*chosen:
 * the z chunk; cgfd_get_tile_shape: the shape) and returns the problem to its freshly created
 * state (zero wavefield, step 0). For a batch it then times the shot groups 4, 8, 16 and every
 * shot at the chosen pair and keeps the fastest (cgfd_get_shot_group). Only on a problem that
 * has not stepped yet. Results do not depend on the choice. No counterpart in the reference.
 */
int cgfd_autotune(cgfd_problem *p, int steps, int *chosen);

/* Bulk stage kernel variant: 1 = TMA-pipelined (default), 0 = direct global loads. Acoustic
   media: their stage kernel in the same two forms (FP32; the FP64 build runs direct loads). */
int cgfd_set_bulk_variant(cgfd_problem *p, int tma);

/* Per-kernel CUDA-event timing of subsequent steps (uses direct launches while on). */
int cgfd_set_timing(cgfd_problem *p, int on);

/*
 * Accumulated kernel times (ms[8]) and launch counts (count[8]) for the kernel kinds
 * {bulk stage of RK stage 0, 1, 2, 3, surface slab, source, stations, FP16 stage scale}, and the
 * number of kernels the library launched (*launches); reset != 0 clears them.
 */
int cgfd_get_timing(cgfd_problem *p, double *ms, long long *count, long long *launches, int reset);

/* ---- serving ------------------------------------------------------------------------- */
/*
 * A request loop on one GPU (no counterpart in the reference, which runs one simulation per
 * process). Requests are forward simulations of any grid size, medium type and precision,
 * each with its own sources; a scheduler thread admits them in submission order whenever a
 * slot and the HBM budget allow (sized by cgfd_problem_bytes), builds queued requests that
 * share a grid (same coord/metric/medium arrays, boundaries, time stepping, stations and
 * precision) as ONE batched problem, and advances every resident problem in slices of
 * time steps on its own stream, so admitted work overlaps on the device and a new request
 * starts while others are mid-run. Results are bitwise those of the request run alone.
 * The caller's coord/metric/medium arrays must stay valid until the request completes
 * (sources and stations are copied at submit).
 */
typedef struct cgfd_server cgfd_server;

typedef struct cgfd_server_opts {
  int    device;            /* CUDA device ordinal of every request                          */
  size_t hbm_budget;        /* device bytes the server may hold; 0: 85% of free memory       */
  int    max_active;        /* resident problems (streams) at once; <= 0: 4                  */
  int    max_batch;         /* same-grid requests per batched problem; <= 0: 8               */
  int    steps_per_slice;   /* time steps enqueued per problem per scheduling pass; <= 0: 50 */
} cgfd_server_opts;

typedef struct cgfd_server_stats {
  long long submitted, completed, failed, pending, active, batches;
  double    p50_ms, p99_ms, mean_ms;      /* submit -> results ready, completed requests      */
  double    cell_stages_per_s;          /* completed grid-cell x RK-stage updates per second
                                           between the first admission and the last result  */
  double    source_steps_per_s;         /* completed source x time steps per second          */
  size_t    hbm_budget, hbm_in_use, hbm_peak;
} cgfd_server_stats;

int cgfd_server_create(const cgfd_server_opts *opts, cgfd_server **out);
/* Validate and queue one request; *request_id identifies it. */
int cgfd_server_submit(cgfd_server *s, const cgfd_problem_desc *desc, long long *request_id);
/*
 * CGFD_ERR_BUSY while queued or running; CGFD_OK when done (*nsta stations; with seismo_out
 * non-NULL the [nsta][9][nt_total] seismograms are copied there and the request's results are
 * released); the request's error code if it failed (cgfd_last_error() says why).
 */
int cgfd_server_poll(cgfd_server *s, long long request_id, float *seismo_out, int *nsta);
/* Block until the request finishes (timeout_s < 0: no limit); CGFD_ERR_BUSY on timeout. */
int cgfd_server_wait(cgfd_server *s, long long request_id, double timeout_s);
int cgfd_server_get_stats(cgfd_server *s, cgfd_server_stats *out);
/* Stop the scheduler: queued requests fail with CGFD_ERR_BUSY, device state is released. */
int cgfd_server_destroy(cgfd_server *s);

/* ---- grid helpers (host, FP64) ------------------------------------------------------- */

/*
 * The generalized-Maxwell-body fit of visco-elastic media for n points (md_vis_GMB_cal_Y,
 * md_t.cu:657-781, with its least-squares solve md_visco_LS): relaxation frequencies wl[nmaxwell]
 * spread log-uniformly over [fmin, fmax], per point the anelastic weights Ylam[nmaxwell][n] /
 * Ymu[nmaxwell][n] fitted to 1/round(Qp), 1/round(Qs), and the unrelaxed moduli lam_u[n], mu_u[n]
 * that give lambda, mu at the reference frequency fr. cgfd_problem_create runs the same fit for a
 * CGFD_MEDIUM_VISCO_ISO medium. Solved in FP64 (the reference solves in float).
 * Returns CGFD_ERR_INVALID for Q values that round below 1 or parameters out of range.
 */
int cgfd_visco_gmb(const cgfd_visco_desc *v, long long n, const float *lambda, const float *mu, const float *Qp,
                   const float *Qs, float *lam_u, float *mu_u, float *Ylam, float *Ymu, float *wl);

/*
 * Fill the 3 ghost layers of ncmp fields [ncmp][nz][ny][nx] by linear extrapolation.
 * Replaces: geometric_symmetry, gd_t.cu:404-502.
 */
int cgfd_fill_ghosts(int ni, int nj, int nk, int ncmp, float *v4d);

/*
 * Metrics from coordinates (ghosts filled), computed in FP64 with the 7-point centered
 * operator and stored as float [10][nz][ny][nx].
 * Replaces: gd_curv_metric_cal, gd_t.cu:209-314 (FP32 in the reference).
 */
int cgfd_metric_calc(int ni, int nj, int nk, const float *coord, float *metric);

/*
 * The same metrics computed on the GPU `device` (FP64 arithmetic without fused multiply-add,
 * so the result equals cgfd_metric_calc bitwise): host arrays in and out, one thread per
 * point, ghost layers by linear extrapolation on the device (the host version is one pass of
 * OpenMP threads over the grid; a large model's setup no longer waits on it).
 * Replaces: gd_curv_metric_cal + geometric_symmetry, gd_t.cu:209-314, 404-502.
 */
int cgfd_metric_calc_gpu(int device, int ni, int nj, int nk, const float *coord, float *metric);

/*
 * Layered elastic-isotropic model: the contents of the reference's "elastic_isotropic"
 * interface file (read_interface_file, src/media/media_read_file.cpp:22-210; the par-file
 * medium input_way "infile_layer"). num_interfaces interfaces, each on a uniform mesh of
 * nx * ny points at x0 + i dx, y0 + j dy, top interface first; per interface and mesh point the
 * elevation and, for the layer below it, rho, vp, vs as value, gradient and power
 * (v(z) = value + (elevation - z)^power * gradient). Arrays [num_interfaces][ny][nx].
 */
typedef struct cgfd_layer_model {
  int   num_interfaces, nx, ny;
  float x0, y0, dx, dy;
  const float *elevation;
  const float *rho, *rho_grad, *rho_pow;
  const float *vp, *vp_grad, *vp_pow;
  const float *vs, *vs_grad, *vs_pow;
} cgfd_layer_model;

/* equivalent_medium_method of the par file */
#define CGFD_MEDIA_LOC 0  /* the layer at each grid point                                   */
#define CGFD_MEDIA_HAR 1  /* volume averaging at interfaces: rho arithmetic, kappa and mu
                             harmonic                                                        */
#define CGFD_MEDIA_ARI 2  /* volume averaging at interfaces: rho, lambda and mu arithmetic    */

/*
 * Media discretisation on the GPU `device`: samples the layered model onto the curvilinear
 * grid coord [3][nz][ny][nx] (ghosts filled) at every point, ghosts included, into
 * medium [3][nz][ny][nx] = rho, lambda, mu (the cgfd_problem_desc medium of elastic_iso).
 * One thread per grid point; at interfaces the har / ari methods average 9^3 sample points of
 * the surrounding half-grid cell. CGFD_ERR_INVALID when a grid point lies outside the
 * interface mesh or vp <= sqrt(2) vs (the reference exits there).
 * Replaces: media_layer2model_el_iso, src/media/media_layer2model.cpp:121-170 with
 * parametrization_layer_el_iso_loc / _har / _ari (:1313-1355 and the averaging loops).
 */
int cgfd_media_layer_el_iso_gpu(int device, int ni, int nj, int nk, const float *coord, const cgfd_layer_model *model,
                                int method, float *medium);

/*
 * Layer files of the acoustic and every elastic media type (read_interface_file,
 * media_read_file.cpp:22-560), by the reference's type numbers; the parameters of each, in the
 * file's order:
 */
#define CGFD_LAYER_ACOUSTIC_ISO  10  /* rho vp (into CGFD_MEDIUM_ACOUSTIC_ISO: rho, kappa)     */
#define CGFD_LAYER_ELASTIC_ISO   21  /* rho vp vs                                              */
#define CGFD_LAYER_VTI_PREM      22  /* rho vph vpv vsh vsv eta                                */
#define CGFD_LAYER_VTI_THOMSEN   23  /* rho vp0 vs0 epsilon delta gamma                        */
#define CGFD_LAYER_VTI_CIJ       24  /* rho c11 c33 c55 c66 c13                                */
#define CGFD_LAYER_TTI_THOMSEN   25  /* rho vp0 vs0 epsilon delta gamma azimuth dip (degrees)  */
#define CGFD_LAYER_TTI_BOND      26  /* rho c11 c33 c55 c66 c13 azimuth dip (degrees)          */
#define CGFD_LAYER_ANISO_CIJ     27  /* rho c11 c12 c13 c14 c15 c16 c22 c23 c24 c25 c26 c33 c34
                                        c35 c36 c44 c45 c46 c55 c56 c66                        */
typedef struct cgfd_layer_media {
  int   type;                    /* CGFD_LAYER_*                                            */
  int   num_interfaces, nx, ny;  /* as cgfd_layer_model                                     */
  float x0, y0, dx, dy;
  const float *elevation;        /* [num_interfaces][ny][nx]                                */
  const float *param;            /* [npar][3][num_interfaces][ny][nx]: value, gradient and
                                    power of each parameter of the type, in the order above  */
} cgfd_layer_media;

/*
 * Media discretisation of any layer file on the GPU `device` into the cgfd_problem_desc medium
 * of medium_type: acoustic [rho kappa] from an acoustic_isotropic file (kappa = vp vp rho; har
 * averages kappa harmonically, ari arithmetically, rho arithmetically: media_layer2model_ac_iso,
 * media_layer2model.cpp:70-118, 1263-1310, 1765-1960); iso from an elastic_isotropic file (as
 * cgfd_media_layer_el_iso_gpu); VTI [rho c11 c13 c33 c55 c66] from the three VTI files; 21-Cij
 * [rho c11 c12 ... c66] from any of the seven (iso and VTI files expanded to the full tensor).
 * method CGFD_MEDIA_LOC / _HAR / _ARI; har and ari average every c_ij harmonically /
 * arithmetically over the 9^3 sub-points of a half-grid cell an interface crosses (rho
 * arithmetically), the VTI files' in VTI form before the expansion. CGFD_ERR_INVALID for a
 * file type the medium type does not take or a grid point outside the interface mesh.
 * Replaces: media_layer2model_el_vti / _el_aniso (src/media/media_layer2model.cpp:173-398) with
 * parametrization_layer_el_{vti,aniso}_{loc,har,ari} (:1365-1492, 2176-2793), para2vti,
 * BondTransform, para2tti (src/media/media_utility.cpp:620-831).
 */
int cgfd_media_layer_gpu(int device, int ni, int nj, int nk, const float *coord, const cgfd_layer_media *model,
                         int medium_type, int method, float *medium);

/*
 * A 3-D binary model (the par file's medium input_way "binfile", par_t.cu:495-600): raw float32
 * volumes of rho, Vp and Vs, size[0] x size[1] x size[2] samples with file dimension 0 fastest.
 * order[d] is the grid axis of file dimension d (0 x, 1 y, 2 z: the par file's dim1..dim3);
 * spacing and origin are per file dimension (z may decrease).
 */
typedef struct cgfd_bin_model {
  int   order[3];
  int   size[3];
  float spacing[3], origin[3];
  const float *rho, *vp, *vs;  /* size[0] * size[1] * size[2] values each, in file order */
} cgfd_bin_model;

/*
 * Media discretisation of a binary model on the GPU `device` into the elastic_iso medium
 * [3][nz][ny][nx] = rho, lambda, mu (ghosts included): the model is cut to the grid's x / y range
 * (all points, ghosts included) and sampled at every grid point by the reference's trilinear
 * interpolation (samples clamped to the cut model), mu = vs vs rho, lambda = vp vp rho - 2 mu.
 * CGFD_ERR_INVALID when order is not a permutation of 0, 1, 2, a dimension has fewer than 2
 * samples, or the model does not coincide with the grid in x, y or z (the reference exits there).
 * Replaces: media_bin2model_el_iso, src/media/media_bin2model.cpp:27-233, with
 * TrilinearInterpolation (src/media/media_utility.cpp:189-283).
 */
int cgfd_media_bin_el_iso_gpu(int device, int ni, int nj, int nk, const float *coord, const cgfd_bin_model *model,
                              float *medium);

/*
 * A grid model (the par file's medium input_way "infile_grid", read_grid_file,
 * media_read_file.cpp:670-1266): num_layers layers, layer l described by ngz[l] surfaces (NI = sum
 * of ngz) on a uniform nx x ny mesh, top first; per surface and mesh point the elevation and the
 * parameters of the file type (CGFD_LAYER_ELASTIC_ISO, _VTI_PREM, _VTI_THOMSEN, _VTI_CIJ,
 * _TTI_THOMSEN or _ANISO_CIJ: the parameters listed above, values only, no gradients).
 */
typedef struct cgfd_grid_media {
  int   type;                    /* CGFD_LAYER_*                                            */
  int   num_layers;
  const int *ngz;                /* [num_layers] */
  int   nx, ny;
  float x0, y0, dx, dy;
  const float *elevation;        /* [NI][ny][nx] */
  const float *param;            /* [npar][NI][ny][nx], the type's parameters in file order */
} cgfd_grid_media;

/*
 * Media discretisation of a grid model on the GPU `device` into the elastic_iso medium
 * [3][nz][ny][nx] = rho, lambda, mu (ghosts included). A point takes the values of the two
 * surfaces around it interpolated linearly in elevation, the average of the two layers on a layer
 * top; har / ari average the 9^3 sub-points of a half-grid cell that a layer top crosses (those on
 * the top left out): rho arithmetically, kappa and mu harmonically (har) or lambda and mu
 * arithmetically (ari). CGFD_ERR_INVALID when the mesh does not cover the grid, a point falls
 * outside it or vp <= sqrt(2) vs (the reference exits there).
 * Replaces: media_grid2model_el_iso, src/media/media_grid2model.cpp:133-188 with
 * parametrization_grid_el_iso_loc / _har / _ari (:1067-1125, 1819-2078).
 */
int cgfd_media_grid_el_iso_gpu(int device, int ni, int nj, int nk, const float *coord, const cgfd_grid_media *model,
                               int method, float *medium);

/*
 * A grid model of any type on the GPU `device` into the cgfd_problem_desc medium of medium_type:
 * iso from an elastic_isotropic file (as cgfd_media_grid_el_iso_gpu); VTI [rho c11 c13 c33 c55
 * c66] from the PREM, Thomsen and Cij VTI files; 21-Cij from any of the six file types (iso and VTI
 * results expanded to the full tensor). The surfaces' parameters are interpolated in elevation,
 * then converted to stiffness as for layer files; har / ari average every c_ij harmonically /
 * arithmetically over the sub-points off the layer tops (rho arithmetically).
 * Replaces: media_grid2model_el_vti / _el_aniso (src/media/media_grid2model.cpp:190-422) with
 * parametrization_grid_el_{vti,aniso}_{loc,har,ari} (:1127-1267, 2080-2793).
 */
int cgfd_media_grid_gpu(int device, int ni, int nj, int nk, const float *coord, const cgfd_grid_media *model,
                        int medium_type, int method, float *medium);

/*
 * Largest stable time step (FP64): CFL * min distance to the 8 neighbour planes / Vp.
 * Uses desc->coord and desc->medium (density form). The reference's CFL is 1.3.
 * Replaces: blk_dt_esti_curv, blk_t.cu:673-763.
 */
int cgfd_dt_estimate(const cgfd_problem_desc *desc, double cfl, double *dtmax);

/* Keep three significant digits. Replaces: blk_keep_three_digi, blk_t.cu:765-780. */
double cgfd_keep_three_digits(double dt);

#ifdef __cplusplus
}
#endif

#endif /* CGFD_B200_H */

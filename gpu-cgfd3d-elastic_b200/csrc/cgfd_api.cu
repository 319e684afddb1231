// cgfd_api.cu -- host runtime and C ABI of the B200 CGFD3D time loop.
//
// A cgfd_problem holds everything drv_rk_curv_col_allstep() keeps on the device
// (drv_rk_curv_col.cu:98-184) in a layout chosen for sm_100a:
//   wavefield: 4 levels (w_pre/w_end pair that swaps every step + tmpA/tmpB ping-pong of
//              the stage input) x 9 fields; no rhs level (the RHS lives in registers).
//   fields:    [k][j][i] with 3 ghost planes in y/z and a 32-float ghost offset in x, so that
//              every physical row starts on a 128-byte line.
//   PML:       per enabled face, 3 levels (pre/end pair + tmp updated in place) x 9 fields.
// One time step = station sampling, then per RK stage the bulk and surface-slab stage
// kernels and the source kernel, then the step-counter advance. The 8 MacCormack pairs and
// the 2 buffer parities give 8 distinct steps; each is captured once as a CUDA graph.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "cgfd_b200.h"
#include "cgfd_dev.cuh"
#include "cgfd_launch.h"
#include "cgfd_setup.h"
#include "cgfd_tma.cuh"

namespace {

thread_local std::string g_err;

void set_err(const std::string &m) { g_err = m; }

#define CK(call)                                                                                 \
  do {                                                                                           \
    cudaError_t e_ = (call);                                                                     \
    if (e_ != cudaSuccess)                                                                       \
      throw cgfd::Error(CGFD_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));      \
  } while (0)

// 8 pairs of forward/backward flags (fd_t.cu:184-194), direction = (flag + stage) % 2
const int kPairFlags[8][3] = {{0, 0, 0}, {1, 1, 0}, {1, 1, 1}, {0, 0, 1},
                              {0, 1, 0}, {1, 0, 0}, {1, 0, 1}, {0, 1, 1}};
const float kRkA[3] = {0.5f, 0.5f, 1.0f};                                          // fd_t.cu:35-37
const float kRkB[4] = {1.0f / 6.0f, 1.0f / 3.0f, 1.0f / 3.0f, 1.0f / 6.0f};        // fd_t.cu:39-42

// Device memory of a problem comes from the device's stream-ordered memory pool, allocated and
// freed in the order of the problem's own stream: freeing a problem (cudaFreeAsync) does not
// synchronise the device, so the serving loop retires one problem while others keep running
// (cudaFree waits for all work on the device). The pool keeps freed memory for the next
// problem (release threshold raised once per device).
void keep_pool_memory(int device) {
  static std::mutex mu;
  static std::vector<int> done;
  std::lock_guard<std::mutex> lk(mu);
  if (std::find(done.begin(), done.end(), device) != done.end()) return;
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
    uint64_t keep = UINT64_MAX;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    // reuse memory another stream freed only once that free has completed (no hidden
    // dependency on the other problem's stream)
    int no = 0;
    cudaMemPoolSetAttribute(pool, cudaMemPoolReuseAllowInternalDependencies, &no);
  }
  done.push_back(device);
}

template <typename T>
T *dmalloc(size_t n, size_t &acc, cudaStream_t st) {
  void *p = nullptr;
  if (n == 0) return nullptr;
  cudaError_t e = cudaMallocAsync(&p, n * sizeof(T), st);
  if (e == cudaErrorMemoryAllocation) {
    cudaGetLastError();
    throw cgfd::Error(CGFD_ERR_NOMEM, "device allocation of " + std::to_string(n * sizeof(T)) + " bytes failed");
  }
  if (e != cudaSuccess) throw cgfd::Error(CGFD_ERR_CUDA, std::string("cudaMallocAsync: ") + cudaGetErrorString(e));
  // the allocation is usable by the host's synchronous copies and by every stream from here on
  e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) throw cgfd::Error(CGFD_ERR_CUDA, std::string("cudaStreamSynchronize: ") + cudaGetErrorString(e));
  acc += n * sizeof(T);
  return (T *)p;
}

// frees memory from dmalloc in the order of stream st (nullptr is ignored)
inline void dfree(void *ptr, cudaStream_t st) {
  if (ptr) cudaFreeAsync(ptr, st);
}

PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (!fn) {
    void *ptr = nullptr;
    cudaDriverEntryPointQueryResult q;
    CK(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &ptr, cudaEnableDefault, &q));
    if (q != cudaDriverEntryPointSuccess || !ptr)
      throw cgfd::Error(CGFD_ERR_CUDA, "cuTensorMapEncodeTiled is not available");
    fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(ptr);
  }
  return fn;
}

// 4-D map (x, y, z, field) over one device-layout array of nf fields of `esize`-byte elements
// (4: FP32, 2: FP16 or BF16 as `dtype` says).
// 4-D map (x, y, z, field) of extents nx, ny, nz, nf over rows of sx, planes of sz and fields of
// sf elements from `base`; a box that reaches beyond an extent reads zeros there without
// touching memory.
void make_map(CUtensorMap *m, const void *base, long long nx, long long ny, long long nz, int nf, long long sx,
              long long sz, long long sf, int boxx, int boxy, int boxf,
              CUtensorMapDataType dtype = CU_TENSOR_MAP_DATA_TYPE_FLOAT32, int esize = 4) {
  cuuint64_t dims[4] = {(cuuint64_t)nx, (cuuint64_t)ny, (cuuint64_t)nz, (cuuint64_t)nf};
  cuuint64_t strides[3] = {(cuuint64_t)(sx * esize), (cuuint64_t)(sz * esize), (cuuint64_t)(sf * esize)};
  cuuint32_t box[4] = {(cuuint32_t)boxx, (cuuint32_t)boxy, 1, (cuuint32_t)boxf};
  cuuint32_t es[4] = {1, 1, 1, 1};
  // L2 fills at 128-byte lines: 256-byte promotion drags half a chunk of the x-neighbour (or of
  // the row padding) into L2 with every row of a box, which the tiles at the grid's x edges, whose
  // neighbours run in the other launch, never use (measured: 128 B and no promotion both 0.9%
  // faster than 256 B on 480x480x240)
  CUresult r = tensor_map_encoder()(m, dtype, 4, const_cast<void *>(base), dims, strides,
                                    box, es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                                    CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) throw cgfd::Error(CGFD_ERR_CUDA, "cuTensorMapEncodeTiled failed: " + std::to_string((int)r));
}

}  // namespace

struct cgfd_problem {
  int device = 0;
  cudaStream_t stream = nullptr;
  int ni = 0, nj = 0, nk = 0, med = 0, ncoef = 0, nt_total = 0, free_top = 0;
  int nbulk = 0;  // planes [0, nbulk) of the bulk kernel (elastic: below the surface slab; acoustic: all)
  int nshot = 1;  // wavefields sharing the grid, coefficients and stations
  int shot_group = 8;  // bulk kernel: shots per block group of a batch (cgfd_set_shot_group)
  // FP64 build (CGFD_PREC_FP64): every real-typed device array below holds doubles (esz 8)
  int fp64 = 0;
  size_t esz = 4;
  float dt = 0.f;
  long long sx = 0, sz = 0, sf = 0, off0 = 0;
  size_t bytes = 0;
  int nzc = 16;
  int shape = 0;  // tile shape of the bulk kernel (cgfd_set_tile_shape; set per medium at creation)

  float *wbuf[4] = {nullptr, nullptr, nullptr, nullptr};  // [0],[1]: pre/end by parity; [2],[3]: tmpA/tmpB
  // visco-elastic media (CGFD_MEDIUM_VISCO_ISO, run as iso media plus the attenuation pass):
  // memory variables [nmax][6][sf] per level (same roles as wbuf), the anelastic weights
  // [2 nmax][sf] (Ylam, then Ymu), the stage right-hand side [9][sf], the surface frame [nj][ni][9]
  int vis = 0, nmax = 0;
  float wl[10] = {};
  float *jbuf[4] = {nullptr, nullptr, nullptr, nullptr};
  float *d_y = nullptr, *d_rhs = nullptr, *d_matD = nullptr;
  // (real-typed arrays -- wbuf, coef, jac, matx/maty, PML A/B/D/aux, d_dis -- are held as float*
  // and hold doubles in the FP64 build; rptr() gives the typed, element-offset pointer)
  float *coef = nullptr, *jac = nullptr, *matx = nullptr, *maty = nullptr;
  float *d_flux = nullptr;  // traction-image fluxes of the current stage input (free surface)
  // 16-bit coefficient storage (replaces `coef` when coef_type != COEF_F32):
  // value = cscale[field] * stored + coffset[field]
  int precision = CGFD_PREC_FP32;
  int coef_type = cgfd::COEF_F32;
  void *coef16 = nullptr;
  float cscale[32] = {}, coffset[32] = {};
  // FP16 stage levels (CGFD_PREC_FP16_WAVE): wbuf[2], wbuf[3] hold __half; per-step scale
  // d_wsc[18] from d_amax[2] (max |w| of velocity / stress) and d_srcb[nt_total][2] (largest
  // source increment of each step)
  int wave16 = 0;
  // TMA bulk kernel tile lists for the current z chunk (interior tiles, then PML tiles)
  int4 *d_tiles = nullptr, *d_tiles_dn = nullptr;
  cgfd::BulkTiles tiles, tiles_dn;  // z layers upwards (backward z operators) / downwards
  // the flux pass and surface slab run on `side`, forked from and joined back into `stream`
  // at every stage
  cudaStream_t side = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  float *d_wsc = nullptr, *d_srcb = nullptr;
  unsigned int *d_amax = nullptr;

  struct Face {
    cgfd::PmlFaceHost h;
    float *A = nullptr, *B = nullptr, *D = nullptr;
    float *aux = nullptr;  // [3][9][n]
    long long n = 0;
  };
  std::vector<Face> faces;

  cgfd::SrcHost src;
  std::vector<int> src_shot;
  int *d_it_begin = nullptr, *d_ext_num = nullptr, *d_src_shot = nullptr;
  long long *d_ext_idx = nullptr;
  float *d_ext_wv = nullptr, *d_ext_wt = nullptr, *d_stf = nullptr;

  cgfd::RecvHost rec;
  long long *d_idx8 = nullptr;
  float *d_w8 = nullptr, *d_seis = nullptr;
  // line receivers (grid points sampled like stations, weight 1 at corner 0)
  int nline = 0;
  long long *d_line_idx8 = nullptr;
  float *d_line_w8 = nullptr, *d_line_seis = nullptr;
  // slices: plane indices (x, then y, then z), device ring of ring steps
  int nslx = 0, nsly = 0, nslz = 0, slice_ring = 0;
  long long slice_per_shot = 0;
  int *d_slice_idx = nullptr;
  float *d_slices = nullptr;

  int *d_it = nullptr, *d_flag = nullptr;
  int it = 0;
  // free-surface peak ground motion [nshot][15][nj][ni] and displacement [nshot][3][nj][ni]
  float *d_pg = nullptr, *d_dis = nullptr;
  // staging buffer of cgfd_get_wavefield_box (grows to the largest box asked for)
  float *d_box = nullptr;
  size_t box_cap = 0;

  bool use_graph = true;
  bool use_tma = true;
  CUtensorMap map_halo[4], map_ctr[4], map_coef;  // acoustic media: the 4-field forms (make_ac_maps)
  bool ac_tma = false;  // acoustic FP32: the TMA-pipelined stage kernel (else the direct-load one)
  cudaGraphExec_t graph[8] = {};
  bool graph_ok[8] = {};
  int graph_launches[8] = {};

  // per-kernel CUDA-event timing (direct launches only): kinds 0-3 bulk stage 0..3,
  // 4 surface slab, 5 source, 6 stations, 7 FP16 stage scale
  bool timing = false;
  std::vector<cudaEvent_t> ev_free;
  struct TimedLaunch { int kind; cudaEvent_t a, b; };
  std::vector<TimedLaunch> pending;
  double t_ms[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  long long t_n[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  long long launches = 0;

  cudaEvent_t get_event() {
    if (ev_free.empty()) {
      cudaEvent_t e;
      CK(cudaEventCreate(&e));
      return e;
    }
    cudaEvent_t e = ev_free.back();
    ev_free.pop_back();
    return e;
  }

  template <typename Fn>
  int timed(int kind, Fn fn) {
    if (!timing) return fn();
    cudaEvent_t a = get_event(), b = get_event();
    CK(cudaEventRecord(a, stream));
    int n = fn();
    CK(cudaEventRecord(b, stream));
    pending.push_back({kind, a, b});
    return n;
  }

  void collect_timing() {
    for (auto &t : pending) {
      float ms = 0.f;
      CK(cudaEventElapsedTime(&ms, t.a, t.b));
      t_ms[t.kind] += ms;
      t_n[t.kind] += 1;
      ev_free.push_back(t.a);
      ev_free.push_back(t.b);
    }
    pending.clear();
  }

  long long didx(int i, int j, int k) const { return off0 + (long long)k * sz + (long long)j * sx + i; }

  // element `off` of a real-typed array held as float* (doubles in the FP64 build)
  template <typename R>
  static R *rptr(const float *base, size_t off = 0) {
    return base ? reinterpret_cast<R *>(const_cast<float *>(base)) + off : nullptr;
  }
  void *rvoid(const float *base, size_t off) const {
    return base ? (void *)((char *)base + off * esz) : nullptr;
  }

  cgfd::StageP stage_params(int step, int stage) const { return stage_params_t<float>(step, stage); }

  template <typename R>
  cgfd::StagePT<R> stage_params_t(int step, int stage) const {
    cgfd::StagePT<R> p;
    memset(&p, 0, sizeof(p));
    p.ni = ni; p.nj = nj; p.nk = nk;
    p.stage = stage;
    int ipair = step % 8;
    for (int a = 0; a < 3; a++) p.dir[a] = (kPairFlags[ipair][a] + stage) % 2;
    p.sx = sx; p.sz = sz; p.sf = sf; p.off0 = off0;
    R *pre = rptr<R>(wbuf[step & 1]), *end = rptr<R>(wbuf[(step + 1) & 1]);
    R *tA = rptr<R>(wbuf[2]), *tB = rptr<R>(wbuf[3]);
    const R *curs[4] = {pre, tA, tB, tA};
    R *outs[4] = {tA, tB, tA, nullptr};
    p.cur = curs[stage];
    p.pre = pre;
    p.tmp_out = outs[stage];
    p.end = end;
    // RK weights x dt: float as in the reference; in double from the same float constants
    p.ca = stage < 3 ? R(kRkA[stage]) * R(dt) : R(0);
    p.cb = R(kRkB[stage]) * R(dt);
    p.coef = coef_type == cgfd::COEF_F32 ? (const void *)coef : (const void *)coef16;
    for (int c = 0; c < 32; c++) { p.cscale[c] = cscale[c]; p.coffset[c] = coffset[c]; }
    p.jac = rptr<R>(jac); p.matx = rptr<R>(matx); p.maty = rptr<R>(maty);
    p.flux = rptr<R>(d_flux);
    p.free_top = free_top;
    p.nbulk = nbulk;
    p.err = d_flag;
    p.nshot = nshot;
    p.wsc = d_wsc;
    p.amax = d_amax;
    p.nface = 0;
    for (const Face &f : faces) {
      cgfd::FacePT<R> &o = p.face[p.nface++];
      o.enable = 1;
      o.axis = f.h.axis;
      for (int b = 0; b < 3; b++) { o.lo[b] = f.h.lo[b]; o.hi[b] = f.h.hi[b]; }
      o.nx = f.h.hi[0] - f.h.lo[0] + 1;
      o.ny = f.h.hi[1] - f.h.lo[1] + 1;
      o.n = f.n;
      o.A = rptr<R>(f.A); o.B = rptr<R>(f.B); o.D = rptr<R>(f.D);
      const size_t L = (size_t)nshot * 9 * f.n;
      R *apre = rptr<R>(f.aux, (size_t)(step & 1) * L), *aend = rptr<R>(f.aux, (size_t)((step + 1) & 1) * L);
      R *atmp = rptr<R>(f.aux, (size_t)2 * L);
      o.aux_cur = stage == 0 ? apre : atmp;
      o.aux_pre = apre;
      o.aux_tmp = atmp;
      o.aux_end = aend;
    }
    return p;
  }

  // Line receivers and slices: samples of w_pre at the start of the step, after the stations
  // (io_line_keep and io_slice_nc_put follow io_recv_keep, drv_rk_curv_col.cu:199-206).
  template <typename R>
  int enqueue_outputs(int step) {
    int n = 0;
    if (nline > 0) {
      cgfd::RecvPT<R> r;
      r.nsta = nline; r.nshot = nshot; r.nt_total = nt_total; r.idx8 = d_line_idx8; r.w8 = d_line_w8;
      r.pre = rptr<R>(wbuf[step & 1]); r.sf = sf; r.seis = d_line_seis; r.d_it = d_it; r.d_flag = d_flag;
      n += timed(6, [&] { return cgfd::launch_recv(r, stream); });
    }
    if (slice_per_shot > 0) {
      cgfd::SliceP<R> q;
      q.ni = ni; q.nj = nj; q.nk = nk; q.nshot = nshot;
      q.sx = sx; q.sz = sz; q.sf = sf; q.off0 = off0;
      q.pre = rptr<R>(wbuf[step & 1]);
      q.nxs = nslx; q.nys = nsly; q.nzs = nslz; q.idx = d_slice_idx;
      q.ring = d_slices; q.ring_steps = slice_ring; q.per_shot = slice_per_shot; q.d_it = d_it;
      n += timed(6, [&] { return cgfd::launch_slices(q, stream); });
    }
    return n;
  }

  // One time step of the FP64 build: the same kernels instantiated in double (direct-load bulk
  // kernel, surface slab, sources, stations, peak motion), launched in the same order.
  int enqueue_step64(int step) {
    cudaStream_t st = stream;
    int n = 0;
    if (rec.n > 0) {
      cgfd::RecvPT<double> r;
      r.nsta = rec.n; r.nshot = nshot; r.nt_total = nt_total; r.idx8 = d_idx8; r.w8 = d_w8;
      r.pre = rptr<double>(wbuf[step & 1]); r.sf = sf; r.seis = d_seis; r.d_it = d_it; r.d_flag = d_flag;
      n += timed(6, [&] { return cgfd::launch_recv(r, st); });
    }
    n += enqueue_outputs<double>(step);
    for (int s = 0; s < 4; s++) {
      const cgfd::StagePT<double> p = stage_params_t<double>(step, s);
      n += timed(s, [&] { return cgfd::launch_stage_bulk(med, p, nzc, st); });
      n += timed(4, [&] { return cgfd::launch_timg_flux64(p, st) + cgfd::launch_stage_surface64(med, p, st); });
      if (src.nsrc > 0) {
        cgfd::SrcPT<double> q;
        memset(&q, 0, sizeof(q));
        q.nsrc = src.nsrc; q.max_ext = src.max_ext; q.max_nt = src.max_nt;
        q.force = src.force; q.moment = src.moment; q.stage = s;
        q.ca = p.ca; q.cb = p.cb;
        q.it_begin = d_it_begin; q.ext_num = d_ext_num; q.ext_idx = d_ext_idx;
        q.ext_wv = d_ext_wv; q.ext_wt = d_ext_wt; q.stf = d_stf; q.src_shot = d_src_shot;
        q.tmp_out = p.tmp_out; q.end = p.end; q.sf = sf; q.d_it = d_it;
        n += timed(5, [&] { return cgfd::launch_source(q, st); });
      }
    }
    if (free_top) {
      cgfd::PgPT<double> q;
      q.ni = ni; q.nj = nj; q.nshot = nshot; q.sx = sx; q.sf = sf;
      q.off_top = off0 + (long long)(nk - 1) * sz;
      q.w_end = rptr<double>(wbuf[(step + 1) & 1]); q.w_pre = rptr<double>(wbuf[step & 1]);
      q.pg = d_pg; q.dis = rptr<double>(d_dis); q.dt = dt;
      n += cgfd::launch_peak_motion(q, st);
    }
    n += cgfd::launch_advance(d_it, st);
    return n;
  }

  // One time step of a visco-elastic problem (drv_rk_curv_col.cu:193-541 with
  // sv_curv_col_vis_iso_onestage): per stage the iso kernels write the right-hand side (bulk
  // planes, then the traction-image fluxes and the surface slab), the attenuation pass combines it
  // with the memory variables, then the sources; after the last stage the surface stress fix.
  int enqueue_step_vis(int step) {
    cudaStream_t st = stream;
    int n = 0;
    if (rec.n > 0) {
      cgfd::RecvPT<float> r;
      r.nsta = rec.n; r.nshot = nshot; r.nt_total = nt_total; r.idx8 = d_idx8; r.w8 = d_w8;
      r.pre = wbuf[step & 1]; r.sf = sf; r.seis = d_seis; r.d_it = d_it; r.d_flag = d_flag;
      n += timed(6, [&] { return cgfd::launch_recv(r, st); });
    }
    n += enqueue_outputs<float>(step);
    float *jpre = jbuf[step & 1], *jend = jbuf[(step + 1) & 1];
    const float *jcurs[4] = {jpre, jbuf[2], jbuf[3], jbuf[2]};
    float *jouts[4] = {jbuf[2], jbuf[3], jbuf[2], nullptr};
    for (int s = 0; s < 4; s++) {
      cgfd::StagePT<float> p = stage_params_t<float>(step, s);
      p.rhs = d_rhs;
      n += timed(s, [&] { return cgfd::launch_stage_bulk(cgfd::MED_ISO, p, nzc, st); });
      if (free_top)
        n += timed(4, [&] {
          return cgfd::launch_timg_flux(coef_type, 0, p, st) + cgfd::launch_stage_surface(cgfd::MED_ISO, coef_type, 0, p, st);
        });
      cgfd::VisP v;
      memset(&v, 0, sizeof(v));
      v.ni = ni; v.nj = nj; v.nk = nk; v.nmax = nmax; v.stage = s;
      v.sx = sx; v.sz = sz; v.sf = sf; v.off0 = off0;
      v.rhs = d_rhs; v.cur = p.cur; v.pre = p.pre; v.tmp_out = p.tmp_out; v.end = p.end;
      v.jcur = jcurs[s]; v.jpre = jpre; v.jtmp = jouts[s]; v.jend = jend;
      v.coef = coef; v.y = d_y;
      for (int m = 0; m < nmax; m++) v.wl[m] = wl[m];
      v.ca = p.ca; v.cb = p.cb; v.err = d_flag;
      n += timed(s, [&] { return cgfd::launch_vis_atten(v, st); });
      if (src.nsrc > 0) {
        cgfd::SrcPT<float> q;
        memset(&q, 0, sizeof(q));
        q.nsrc = src.nsrc; q.max_ext = src.max_ext; q.max_nt = src.max_nt;
        q.force = src.force; q.moment = src.moment; q.stage = s;
        q.ca = p.ca; q.cb = p.cb;
        q.it_begin = d_it_begin; q.ext_num = d_ext_num; q.ext_idx = d_ext_idx;
        q.ext_wv = d_ext_wv; q.ext_wt = d_ext_wt; q.stf = d_stf; q.src_shot = d_src_shot;
        q.tmp_out = p.tmp_out; q.end = p.end; q.sf = sf; q.d_it = d_it;
        n += timed(5, [&] { return cgfd::launch_source(q, st); });
      }
    }
    if (free_top) {
      cgfd::VisFreeP f;
      f.ni = ni; f.nj = nj; f.sx = sx; f.sf = sf; f.off_top = off0 + (long long)(nk - 1) * sz;
      f.w_end = wbuf[(step + 1) & 1]; f.matD = d_matD;
      n += timed(4, [&] { return cgfd::launch_vis_free(f, st); });
      cgfd::PgPT<float> q;
      q.ni = ni; q.nj = nj; q.nshot = nshot; q.sx = sx; q.sf = sf;
      q.off_top = off0 + (long long)(nk - 1) * sz;
      q.w_end = wbuf[(step + 1) & 1]; q.w_pre = wbuf[step & 1];
      q.pg = d_pg; q.dis = d_dis; q.dt = dt;
      n += cgfd::launch_peak_motion(q, st);
    }
    n += cgfd::launch_advance(d_it, st);
    return n;
  }

  // One time step of an acoustic problem (drv_rk_curv_col.cu:193-541 with
  // sv_curv_col_ac_iso_onestage): per stage the free-surface pressure image of the stage input,
  // then the fused stage of every cell, then the sources; R float, or double in the FP64 build.
  template <typename R>
  int enqueue_step_ac(int step) {
    cudaStream_t st = stream;
    int n = 0;
    if (rec.n > 0) {
      cgfd::RecvPT<R> r;
      r.nsta = rec.n; r.nshot = nshot; r.nt_total = nt_total; r.idx8 = d_idx8; r.w8 = d_w8;
      r.pre = rptr<R>(wbuf[step & 1]); r.sf = sf; r.seis = d_seis; r.d_it = d_it; r.d_flag = d_flag;
      n += timed(6, [&] { return cgfd::launch_recv(r, st); });
    }
    n += enqueue_outputs<R>(step);
    for (int s = 0; s < 4; s++) {
      const cgfd::StagePT<R> p = stage_params_t<R>(step, s);
      n += timed(s, [&] {
        int k = cgfd::launch_ac_image(p, st);
        int t = -1;
        if constexpr (std::is_same<R, float>::value) {
          if (ac_tma) {
            cgfd::TmaP tm;
            const int pre = step & 1, end = (step + 1) & 1;
            const int curs[4] = {pre, 2, 3, 2};
            tm.cur = map_halo[curs[s]];
            tm.pre = map_ctr[pre];
            tm.end = map_ctr[end];
            tm.coef = map_coef;
            t = cgfd::launch_stage_ac_tma(p, tm, nzc, st);
          }
        }
        return k + (t >= 0 ? t : cgfd::launch_stage_ac(p, nzc, st));
      });
      if (src.nsrc > 0) {
        cgfd::SrcPT<R> q;
        memset(&q, 0, sizeof(q));
        q.nsrc = src.nsrc; q.max_ext = src.max_ext; q.max_nt = src.max_nt;
        q.force = src.force; q.moment = src.moment; q.stage = s;
        q.ca = p.ca; q.cb = p.cb;
        q.it_begin = d_it_begin; q.ext_num = d_ext_num; q.ext_idx = d_ext_idx;
        q.ext_wv = d_ext_wv; q.ext_wt = d_ext_wt; q.stf = d_stf; q.src_shot = d_src_shot;
        q.tmp_out = p.tmp_out; q.end = p.end; q.sf = sf; q.d_it = d_it;
        n += timed(5, [&] { return cgfd::launch_source(q, st); });
      }
    }
    if (free_top) {
      cgfd::PgPT<R> q;
      q.ni = ni; q.nj = nj; q.nshot = nshot; q.sx = sx; q.sf = sf;
      q.off_top = off0 + (long long)(nk - 1) * sz;
      q.w_end = rptr<R>(wbuf[(step + 1) & 1]); q.w_pre = rptr<R>(wbuf[step & 1]);
      q.pg = d_pg; q.dis = rptr<R>(d_dis); q.dt = dt;
      n += cgfd::launch_peak_motion(q, st);
    }
    n += cgfd::launch_advance(d_it, st);
    return n;
  }

  int enqueue_step(int step) {
    if (vis) return enqueue_step_vis(step);
    if (med == cgfd::MED_AC) return fp64 ? enqueue_step_ac<double>(step) : enqueue_step_ac<float>(step);
    if (fp64) return enqueue_step64(step);
    cudaStream_t st = stream;
    int n = 0;
    if (rec.n > 0) {
      cgfd::RecvP r;
      r.nsta = rec.n; r.nshot = nshot; r.nt_total = nt_total; r.idx8 = d_idx8; r.w8 = d_w8;
      r.pre = wbuf[step & 1]; r.sf = sf; r.seis = d_seis; r.d_it = d_it; r.d_flag = d_flag;
      n += timed(6, [&] { return cgfd::launch_recv(r, st); });
    }
    n += enqueue_outputs<float>(step);
    if (wave16)
      n += timed(7, [&] { return cgfd::launch_wave_scale(d_amax, d_srcb, d_it, nt_total, nshot, d_wsc, st); });
    for (int s = 0; s < 4; s++) {
      cgfd::StageP p = stage_params(step, s);
      bool surface_done = false;
      if (use_tma) {
        cgfd::TmaP tm;
        const int pre = step & 1, end = (step + 1) & 1;
        const int curs[4] = {pre, 2, 3, 2};
        tm.cur = map_halo[curs[s]];
        tm.pre = map_ctr[pre];
        tm.end = map_ctr[end];
        tm.coef = map_coef;
        // Outside per-kernel timing, the flux pass and the surface slab (latency-bound, top
        // planes only) run on a side stream beside the bulk tiles: they write only the top
        // planes of the stage outputs, which no bulk tile reads or writes in this stage.
        const bool fork = free_top && tiles.n > 0 && !timing;
        surface_done = fork;
        n += timed(s, [&] {
          if (fork) {
            CK(cudaEventRecord(ev_fork, st));
            CK(cudaStreamWaitEvent(side, ev_fork, 0));
          }
          int k = cgfd::launch_stage_bulk_tma(med, coef_type, wave16, shape, p, tm, p.dir[2] ? tiles_dn : tiles, st);
          if (surface_done)
            k += cgfd::launch_timg_flux(coef_type, wave16, p, side) +
                 cgfd::launch_stage_surface(med, coef_type, wave16, p, side);
          if (fork) {
            CK(cudaEventRecord(ev_join, side));
            CK(cudaStreamWaitEvent(st, ev_join, 0));
          }
          return k;
        });
      } else {
        n += timed(s, [&] { return cgfd::launch_stage_bulk(med, p, nzc, st); });
      }
      if (!surface_done)
        n += timed(4, [&] {
          return cgfd::launch_timg_flux(coef_type, wave16, p, st) +
                 cgfd::launch_stage_surface(med, coef_type, wave16, p, st);
        });
      if (src.nsrc > 0) {
        cgfd::SrcP q;
        q.nsrc = src.nsrc; q.max_ext = src.max_ext; q.max_nt = src.max_nt;
        q.force = src.force; q.moment = src.moment; q.stage = s;
        q.ca = p.ca; q.cb = p.cb;
        q.it_begin = d_it_begin; q.ext_num = d_ext_num; q.ext_idx = d_ext_idx;
        q.ext_wv = d_ext_wv; q.ext_wt = d_ext_wt; q.stf = d_stf; q.src_shot = d_src_shot;
        q.tmp_out = p.tmp_out; q.end = p.end; q.sf = sf; q.d_it = d_it;
        q.wave16 = wave16; q.wsc = d_wsc; q.amax = d_amax;
        n += timed(5, [&] { return cgfd::launch_source(q, st); });
      }
    }
    if (free_top) {  // drv_rk_curv_col.cu:519-527: after the last stage, before the level swap
      cgfd::PgP q;
      q.ni = ni; q.nj = nj; q.nshot = nshot; q.sx = sx; q.sf = sf;
      q.off_top = off0 + (long long)(nk - 1) * sz;
      q.w_end = wbuf[(step + 1) & 1]; q.w_pre = wbuf[step & 1];
      q.pg = d_pg; q.dis = d_dis; q.dt = dt;
      n += cgfd::launch_peak_motion(q, st);
    }
    n += cgfd::launch_advance(d_it, st);
    return n;
  }

  void run_steps(int n) {
    for (int s = 0; s < n; s++) {
      int step = it;
      int slot = step % 8;
      if (use_graph && !timing) {
        if (!graph_ok[slot]) {
          cudaGraph_t g;
          CK(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
          graph_launches[slot] = enqueue_step(step);
          CK(cudaStreamEndCapture(stream, &g));
          CK(cudaGraphInstantiate(&graph[slot], g, 0));
          CK(cudaGraphDestroy(g));
          graph_ok[slot] = true;
        }
        CK(cudaGraphLaunch(graph[slot], stream));
        launches += graph_launches[slot];
      } else {
        launches += enqueue_step(step);
        CK(cudaGetLastError());
      }
      it++;
    }
  }

  void release() {
    if (device >= 0) cudaSetDevice(device);
    for (int s = 0; s < 8; s++)
      if (graph_ok[s]) cudaGraphExecDestroy(graph[s]);
    for (auto &t : pending) { ev_free.push_back(t.a); ev_free.push_back(t.b); }
    for (auto e : ev_free) cudaEventDestroy(e);
    if (stream) {  // everything below was allocated in the order of this stream
      const cudaStream_t st = stream;
      for (auto *p : wbuf) dfree(p, st);
      for (auto *p : jbuf) dfree(p, st);
      dfree(d_y, st); dfree(d_rhs, st); dfree(d_matD, st);
      dfree(coef, st); dfree(coef16, st); dfree(jac, st); dfree(matx, st); dfree(maty, st); dfree(d_flux, st);
      for (Face &f : faces) { dfree(f.A, st); dfree(f.B, st); dfree(f.D, st); dfree(f.aux, st); }
      dfree(d_it_begin, st); dfree(d_ext_num, st); dfree(d_src_shot, st); dfree(d_ext_idx, st); dfree(d_ext_wv, st);
      dfree(d_ext_wt, st); dfree(d_wsc, st); dfree(d_srcb, st); dfree(d_amax, st); dfree(d_tiles, st);
      dfree(d_tiles_dn, st); dfree(d_pg, st);
      dfree(d_dis, st); dfree(d_box, st); dfree(d_stf, st); dfree(d_idx8, st); dfree(d_w8, st); dfree(d_seis, st);
      dfree(d_line_idx8, st); dfree(d_line_w8, st); dfree(d_line_seis, st); dfree(d_slice_idx, st); dfree(d_slices, st);
      dfree(d_it, st); dfree(d_flag, st);
      cudaStreamSynchronize(st);
    }
    if (stream) cudaStreamDestroy(stream);
    if (side) cudaStreamDestroy(side);
    if (ev_fork) cudaEventDestroy(ev_fork);
    if (ev_join) cudaEventDestroy(ev_join);
  }
};

namespace {

template <typename Fn>
int guarded(Fn fn) {
  try {
    fn();
    return CGFD_OK;
  } catch (cgfd::Error &e) {
    set_err(e.what());
    return e.code;
  } catch (std::exception &e) {
    set_err(e.what());
    return CGFD_ERR_INVALID;
  }
}

// Host -> device copies of the caller's model arrays (pageable memory) through two pinned
// chunks: host threads fill one chunk while the copy engine drains the other, so the upload
// runs at the slower of a parallel host memcpy and the host link instead of the driver's
// serial pageable path. One stager per device, allocated on first use and kept for the life
// of the process (2 x 64 MiB of pinned host memory): allocating and freeing pinned memory per
// problem would synchronise the device under the serving loop's concurrent problems. Users
// hold its lock for a whole upload; each chunk is refilled only after the copy out of it
// has completed (per-chunk events), so no device-wide synchronisation is involved.
class PinnedStager {
 public:
  static constexpr size_t kChunk = size_t(64) << 20;
  // fields below this size go through the plain pageable copy
  static constexpr size_t kMinBytes = size_t(16) << 20;

  static PinnedStager &for_device(int device) {
    static std::mutex mu;
    static std::vector<PinnedStager *> all;
    std::lock_guard<std::mutex> lk(mu);
    if ((int)all.size() <= device) all.resize(device + 1, nullptr);
    if (!all[device]) all[device] = new PinnedStager();  // device is current
    return *all[device];
  }
  std::mutex &mutex() { return mu_; }

  // device -> caller's (pageable) host memory, the reverse pipeline: the copy engine fills one
  // chunk while host threads empty the other
  void copy_out(void *dst, const void *src, size_t n, cudaStream_t st) {
    const size_t nch = (n + kChunk - 1) / kChunk;
    auto issue = [&](size_t c) {
      const size_t o = c * kChunk, m = std::min(kChunk, n - o);
      CK(cudaEventSynchronize(done_[c & 1]));
      CK(cudaMemcpyAsync(buf_[c & 1], static_cast<const char *>(src) + o, m, cudaMemcpyDeviceToHost, st));
      CK(cudaEventRecord(done_[c & 1], st));
    };
    if (nch > 0) issue(0);
    for (size_t c = 0; c < nch; c++) {
      if (c + 1 < nch) issue(c + 1);
      CK(cudaEventSynchronize(done_[c & 1]));
      const size_t o = c * kChunk, m = std::min(kChunk, n - o);
      char *out = static_cast<char *>(dst) + o;
      const long long pieces = (long long)((m + kPiece - 1) / kPiece);
#pragma omp parallel for schedule(static)
      for (long long q = 0; q < pieces; q++) {
        const size_t a = (size_t)q * kPiece;
        std::memcpy(out + a, buf_[c & 1] + a, std::min(kPiece, m - a));
      }
    }
    next_ = (int)(nch & 1);
  }

  void copy(void *dst, const void *src, size_t n, cudaStream_t st) {
    for (size_t o = 0; o < n; o += kChunk) {
      const size_t m = std::min(kChunk, n - o);
      const int b = next_;
      next_ ^= 1;
      CK(cudaEventSynchronize(done_[b]));  // the previous copy out of this chunk has finished
      const char *in = static_cast<const char *>(src) + o;
      const long long pieces = (long long)((m + kPiece - 1) / kPiece);
#pragma omp parallel for schedule(static)
      for (long long q = 0; q < pieces; q++) {
        const size_t a = (size_t)q * kPiece;
        std::memcpy(buf_[b] + a, in + a, std::min(kPiece, m - a));
      }
      CK(cudaMemcpyAsync(static_cast<char *>(dst) + o, buf_[b], m, cudaMemcpyHostToDevice, st));
      CK(cudaEventRecord(done_[b], st));
    }
  }

 private:
  PinnedStager() {
    for (int b = 0; b < 2; b++) {
      CK(cudaHostAlloc(reinterpret_cast<void **>(&buf_[b]), kChunk, cudaHostAllocPortable));
      CK(cudaEventCreateWithFlags(&done_[b], cudaEventDisableTiming));
    }
  }
  static constexpr size_t kPiece = size_t(1) << 20;
  std::mutex mu_;
  char *buf_[2] = {nullptr, nullptr};
  cudaEvent_t done_[2] = {nullptr, nullptr};
  int next_ = 0;
};

// One model field (reference layout) into its device array, through stage_buf. ps: the
// device's pinned stager, its lock held by the caller (nullptr: plain pageable copy).
// dst: the device field (float, or double in the FP64 build).
void upload_field(cgfd_problem *p, const float *host_ref, void *dst, float *stage_buf, int mode, int ghosts,
                  PinnedStager *ps = nullptr) {
  size_t n = (size_t)(p->ni + 6) * (p->nj + 6) * (p->nk + 6);
  if (ps && n * sizeof(float) >= PinnedStager::kMinBytes) ps->copy(stage_buf, host_ref, n * sizeof(float), p->stream);
  else CK(cudaMemcpyAsync(stage_buf, host_ref, n * sizeof(float), cudaMemcpyHostToDevice, p->stream));
  if (p->fp64)
    cgfd::launch_repack_in(stage_buf, (double *)dst, p->ni, p->nj, p->nk, p->sx, p->sz, p->off0, mode, ghosts, p->stream);
  else
    cgfd::launch_repack_in(stage_buf, (float *)dst, p->ni, p->nj, p->nk, p->sx, p->sz, p->off0, mode, ghosts, p->stream);
  CK(cudaGetLastError());
}

// Metrics computed on the device from the caller's coordinates (desc->metric NULL): the FP64
// kernel of cgfd_metric_calc_gpu (bitwise equal to cgfd_metric_calc, ghosts included) in the
// reference layout, each field then repacked into the problem's layout like an uploaded
// metric. `view` (host, 10 fields in the reference layout, zero-initialised) receives what the
// host-side setup reads: the Jacobian (source weights) and the top plane of the other fields
// (free-surface matrices). ps: the device's pinned stager, its lock held by the caller.
void metric_from_coords(cgfd_problem *p, const cgfd_problem_desc *d, PinnedStager &ps, float *view) {
  cgfd::RefGrid g(p->ni, p->nj, p->nk);
  const size_t siz = g.siz_icmp;
  size_t acc = 0;
  float *dc = dmalloc<float>(3 * siz, acc, p->stream);
  float *dm = dmalloc<float>(10 * siz, acc, p->stream);
  for (int c = 0; c < 3; c++) ps.copy(dc + c * siz, d->coord + c * siz, siz * sizeof(float), p->stream);
  CK(cudaMemsetAsync(dm, 0, 10 * siz * sizeof(float), p->stream));
  const long long sx = g.nx, sz = (long long)g.nx * g.ny, off0 = 3 + 3 * sx + 3 * sz;
  float *out[10];
  for (int f = 0; f < 10; f++) out[f] = dm + f * siz;
  cgfd::launch_metric(dc, dc + siz, dc + 2 * siz, out, p->ni, p->nj, p->nk, sx, sz, off0, p->stream);
  CK(cudaGetLastError());
  for (int f = 0; f < 10; f++) {
    void *dst = f == 0 ? (void *)p->jac : p->rvoid(p->coef, (size_t)(f - 1) * p->sf);
    if (p->fp64)
      cgfd::launch_repack_in(out[f], (double *)dst, p->ni, p->nj, p->nk, p->sx, p->sz, p->off0, 0, 1, p->stream);
    else
      cgfd::launch_repack_in(out[f], (float *)dst, p->ni, p->nj, p->nk, p->sx, p->sz, p->off0, 0, 1, p->stream);
  }
  CK(cudaGetLastError());
  ps.copy_out(view, dm, siz * sizeof(float), p->stream);
  const size_t top = (size_t)(p->nk - 1 + 3) * g.nx * g.ny, plane = (size_t)g.nx * g.ny;
  for (int f = 1; f < 10; f++)
    CK(cudaMemcpyAsync(view + f * siz + top, dm + f * siz + top, plane * sizeof(float), cudaMemcpyDeviceToHost,
                       p->stream));
  CK(cudaStreamSynchronize(p->stream));
  dfree(dc, p->stream);
  dfree(dm, p->stream);
}

// a real-typed device array of n elements (doubles in the FP64 build), held as float*
float *dalloc_real(cgfd_problem *p, size_t n, size_t &acc) {
  return (float *)dmalloc<uint16_t>(n * p->esz / 2, acc, p->stream);
}

// host floats -> device real-typed array (converted to double in the FP64 build)
void upload_real(cgfd_problem *p, float *dst, const std::vector<float> &v) {
  if (p->fp64) {
    std::vector<double> d(v.begin(), v.end());
    CK(cudaMemcpy(dst, d.data(), d.size() * sizeof(double), cudaMemcpyHostToDevice));
  } else {
    CK(cudaMemcpy(dst, v.data(), v.size() * sizeof(float), cudaMemcpyHostToDevice));
  }
}

// Replace the FP32 coefficient array by a 16-bit copy (stochastically rounded), one
// scale/offset per field chosen in FP64 from the field's exact extremes over the cells the
// kernels read (physical box + 3 ghosts):
//   FP16 / BF16: offset 0, power-of-two scale putting max |value| in [2^13, 2^14) (FP16
//                keeps 11 significant bits for values down to 2^-27 of the maximum);
//   U16 (fixed point): offset = min, scale = (max - min) / 65535, i.e. 16 bits across the
//                field's range -- for the bounded ranges of metrics, 1/rho and moduli this
//                is 20-30x finer than FP16.
void to_16bit_coefficients(cgfd_problem *p) {
  unsigned int *d_mm = dmalloc<unsigned int>(2 * p->ncoef, p->bytes, p->stream);
  std::vector<unsigned int> mm(2 * p->ncoef);
  for (int c = 0; c < p->ncoef; c++) { mm[2 * c] = 0xffffffffu; mm[2 * c + 1] = 0u; }
  CK(cudaMemcpyAsync(d_mm, mm.data(), sizeof(unsigned int) * mm.size(), cudaMemcpyHostToDevice, p->stream));
  for (int c = 0; c < p->ncoef; c++)
    cgfd::launch_coef_minmax(p->coef + (size_t)c * p->sf, p->ni, p->nj, p->nk, p->sx, p->sz, p->off0, d_mm + 2 * c,
                             p->stream);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(mm.data(), d_mm, sizeof(unsigned int) * mm.size(), cudaMemcpyDeviceToHost, p->stream));
  CK(cudaStreamSynchronize(p->stream));
  dfree(d_mm, p->stream);
  p->bytes -= sizeof(unsigned int) * 2 * p->ncoef;
  p->coef16 = dmalloc<uint16_t>((size_t)p->ncoef * p->sf, p->bytes, p->stream);
  for (int c = 0; c < p->ncoef; c++) {
    const double lo = cgfd::coef_key_to_float(mm[2 * c]), hi = cgfd::coef_key_to_float(mm[2 * c + 1]);
    if (!std::isfinite(lo) || !std::isfinite(hi))
      throw cgfd::Error(CGFD_ERR_NONFINITE, "coefficient field " + std::to_string(c) + " is not finite");
    double scale = 1.0, offset = 0.0;
    if (p->coef_type == cgfd::COEF_U16) {
      offset = lo;
      scale = hi > lo ? (hi - lo) / 65535.0 : 1.0;
    } else {
      const double m = std::max(std::fabs(lo), std::fabs(hi));
      if (m > 0.0) scale = std::ldexp(1.0, std::ilogb(m) - 13);
    }
    p->cscale[c] = (float)scale;
    p->coffset[c] = (float)offset;
    cgfd::launch_coef_to16(p->coef_type, p->coef + (size_t)c * p->sf, (uint16_t *)p->coef16 + (size_t)c * p->sf, p->sf,
                           p->cscale[c], p->coffset[c], c, p->stream);
  }
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(p->stream));
  dfree(p->coef, p->stream);
  p->coef = nullptr;
  p->bytes -= sizeof(float) * p->ncoef * p->sf;
}

// Device layout [k][j][i] of one field: rows padded to 32 floats with the physical x origin
// at GX (128-byte aligned rows), 3 ghost rows/planes in y/z, fields 256-byte aligned.
void layout(int ni, int nj, int nk, long long &sx, long long &sz, long long &sf, long long &off0) {
  sx = ((cgfd::GX + ni + 3 + 31) / 32) * 32;
  sz = sx * (nj + 6);
  sf = ((sz * (nk + 6) + 63) / 64) * 64;
  off0 = 3 * sz + 3 * sx + cgfd::GX;
}

// Device bytes build() holds once done (*resident) and at its high-water mark (*peak), from
// the description alone (host work only: PML, source and station setup).
void problem_bytes(const cgfd_problem_desc *d, int nshot, const cgfd_source_desc *shots, size_t *resident,
                   size_t *peak) {
  cgfd::validate_desc(d);
  if (nshot < 1 || nshot > 32767) throw cgfd::Error(CGFD_ERR_INVALID, "nshot must be in [1, 32767]");
  long long sx, sz, sf, off0;
  layout(d->ni, d->nj, d->nk, sx, sz, sf, off0);
  const bool ac = d->medium_type == CGFD_MEDIUM_ACOUSTIC_ISO;
  const bool vis = d->medium_type == CGFD_MEDIUM_VISCO_ISO;
  const int ncoef = ac ? 11 : (d->medium_type == CGFD_MEDIUM_ELASTIC_ISO || vis ? 12 : (d->medium_type == CGFD_MEDIUM_ELASTIC_VTI ? 15 : 31));
  const bool f64 = d->precision == CGFD_PREC_FP64;
  const bool c16 = d->precision != CGFD_PREC_FP32 && !f64, w16 = d->precision == CGFD_PREC_FP16_WAVE;
  const size_t F = f64 ? sizeof(double) : sizeof(float);  // real-typed arrays
  const size_t waves = (size_t)9 * sf * nshot * (2 * F + 2 * (w16 ? 2 : F));
  const size_t coef32 = (size_t)ncoef * sf * F, coef16 = (size_t)ncoef * sf * 2, jac = (size_t)sf * F;
  const size_t stage_buf = (size_t)(d->ni + 6) * (d->nj + 6) * (d->nk + 6) * sizeof(float);
  size_t r = waves + (c16 ? coef16 : coef32) + jac;
  // metric computed on the device (no metric given): coordinates and the 10 metric fields in the
  // reference layout are held beside the staging buffer while the metric is repacked
  const size_t upload = stage_buf * (d->metric ? 1 : 14);
  const size_t high = waves + jac + coef32 + (c16 ? std::max(upload, coef16 + 8 * (size_t)ncoef) : upload);
  if (d->free_top && !ac)  // conversion matrices and traction-image fluxes (elastic media)
    r += (size_t)2 * 9 * d->ni * d->nj * F + (size_t)9 * cgfd::kFluxPlanes * (d->ni + 6) * (d->nj + 6) * nshot * F;
  if (vis)  // memory variables (4 levels), anelastic weights, stage right-hand side, surface frame
    r += (size_t)(4 * 6 + 2) * d->visco->nmaxwell * sf * F + (size_t)9 * sf * F + (size_t)9 * d->ni * d->nj * F;
  cgfd::PmlFaceHost fh[3][2];
  cgfd::pml_setup(d, fh);
  for (int a = 0; a < 3; a++)
    for (int s = 0; s < 2; s++) {
      if (!fh[a][s].enable) continue;
      const cgfd::PmlFaceHost &h = fh[a][s];
      const size_t n = (size_t)(h.hi[0] - h.lo[0] + 1) * (h.hi[1] - h.lo[1] + 1) * (h.hi[2] - h.lo[2] + 1);
      r += 3 * h.A.size() * F + (size_t)3 * 9 * n * nshot * F;
    }
  size_t nsrc = 0, max_ext = 0, max_nt = 0;
  for (int sh = 0; sh < (shots ? nshot : 1); sh++) {
    cgfd_problem_desc ds = *d;
    if (shots) ds.src = shots[sh];
    cgfd::SrcHost q;
    cgfd::validate_desc(&ds);
    cgfd::src_setup(&ds, q);
    nsrc += q.nsrc;
    max_ext = std::max(max_ext, (size_t)q.max_ext);
    max_nt = std::max(max_nt, (size_t)q.max_nt);
  }
  if (nsrc > 0)
    r += nsrc * 3 * sizeof(int) + nsrc * max_ext * (sizeof(long long) + 2 * sizeof(float)) +
         nsrc * max_nt * 36 * sizeof(float);
  cgfd::RecvHost rec;
  cgfd::recv_setup(d, rec);
  if (rec.n > 0)
    r += (size_t)rec.n * 8 * (sizeof(long long) + sizeof(float)) + (size_t)rec.n * 9 * d->nt_total * nshot * sizeof(float);
  r += 2 * sizeof(int);
  if (d->free_top) r += (size_t)(15 * sizeof(float) + 3 * F) * d->ni * d->nj * nshot;
  if (w16) r += (size_t)nshot * (18 * F + 2 * sizeof(unsigned int) + (size_t)d->nt_total * 2 * F);
  if (resident) *resident = r;
  if (peak) *peak = std::max(r, high);
}

// Largest source increment added to an RK stage input in each step, per shot and group
// (velocity: forces, stress: moments): max over the shot's sources, stages 0-2 and spread
// points of |rk_a[s] dt * value * weight|; [nt_total][nshot][2]. Part of the FP16
// stage-level scale of that step.
std::vector<float> source_bounds(const cgfd_problem *p) {
  std::vector<float> sb((size_t)p->nt_total * p->nshot * 2, 0.f);
  const cgfd::SrcHost &s = p->src;
  for (int is = 0; is < s.nsrc; is++) {
    float wv = 0.f, wt = 0.f;
    for (int e = 0; e < s.ext_num[is]; e++) {
      wv = std::max(wv, std::fabs(s.ext_wv[(size_t)is * s.max_ext + e]));
      wt = std::max(wt, std::fabs(s.ext_wt[(size_t)is * s.max_ext + e]));
    }
    for (int t = 0; t < s.max_nt; t++) {
      const int it = s.it_begin[is] + t;
      if (it < 0 || it >= p->nt_total) continue;
      for (int st = 0; st < 3; st++) {
        const float ca = std::fabs(kRkA[st] * p->dt);
        const float *v = &s.stf[(((size_t)is * s.max_nt + t) * 4 + st) * 9];
        for (int c = 0; c < 9; c++) {
          if (c < 3 && !s.force) continue;
          if (c >= 3 && !s.moment) continue;
          const float b = ca * std::fabs(v[c]) * (c < 3 ? wv : wt);
          float &o = sb[((size_t)it * p->nshot + p->src_shot[is]) * 2 + (c < 3 ? 0 : 1)];
          o = std::max(o, b);
        }
      }
    }
  }
  return sb;
}

void make_tiles(cgfd_problem *p);
void make_maps(cgfd_problem *p);
void make_ac_maps(cgfd_problem *p);
float *noalloc_scratch(int device);

// sources given by physical coordinates: located on the current device (nullptr otherwise)
const cgfd::Located *locate_sources(const cgfd_problem_desc *d, cgfd::Located &out) {
  if (d->src.num <= 0 || d->src.loc_coord_type != 1) return nullptr;
  std::vector<int> depth(d->src.num, d->src.loc_3dim == 1 ? 1 : 0);
  cgfd::locate_coords(d, d->src.num, d->src.loc, depth.data(), out);
  return &out;
}

void build(cgfd_problem *p, const cgfd_problem_desc *d, int nshot, const cgfd_source_desc *shots) {
  cgfd::validate_desc(d);
  if (nshot < 1 || nshot > 32767) throw cgfd::Error(CGFD_ERR_INVALID, "nshot must be in [1, 32767]");
  p->nshot = nshot;
  // visco-elastic media: the GMB fit of the physical points on the host (cgfd_visco_gmb); the
  // kernels then see the iso medium of the unrelaxed moduli plus the anelastic weights
  cgfd_problem_desc dvis;
  std::vector<float> vis_med, vis_y;
  if (d->medium_type == CGFD_MEDIUM_VISCO_ISO) {
    if (nshot != 1) throw cgfd::Error(CGFD_ERR_UNSUPPORTED, "visco-elastic media run one shot per problem");
    if (d->nj > 65535 || d->nk > 65535)  // the attenuation pass runs one block row per (j, k)
      throw cgfd::Error(CGFD_ERR_UNSUPPORTED, "visco-elastic media take nj, nk <= 65535");
    cgfd::RefGrid g(d->ni, d->nj, d->nk);
    const size_t N = g.siz_icmp;
    const int nm = d->visco->nmaxwell;
    const long long np = (long long)d->ni * d->nj * d->nk;
    std::vector<float> l(np), m(np), qp(np), qs(np), lu(np), mu(np), yl((size_t)np * std::max(nm, 1)),
        ym((size_t)np * std::max(nm, 1));
    long long t = 0;
    for (int k = 0; k < d->nk; k++)
      for (int j = 0; j < d->nj; j++)
        for (int i = 0; i < d->ni; i++, t++) {
          const size_t ip = g.at(i, j, k);
          l[t] = d->medium[N + ip]; m[t] = d->medium[2 * N + ip];
          qp[t] = d->medium[3 * N + ip]; qs[t] = d->medium[4 * N + ip];
        }
    cgfd::visco_gmb(d->visco, np, l.data(), m.data(), qp.data(), qs.data(), lu.data(), mu.data(), yl.data(),
                    ym.data(), p->wl);
    p->vis = 1;
    p->nmax = nm;
    vis_med.assign(d->medium, d->medium + 3 * N);  // rho, lambda, mu; ghosts as given
    vis_y.assign((size_t)2 * nm * N, 0.f);
    t = 0;
    for (int k = 0; k < d->nk; k++)
      for (int j = 0; j < d->nj; j++)
        for (int i = 0; i < d->ni; i++, t++) {
          const size_t ip = g.at(i, j, k);
          vis_med[N + ip] = lu[t];
          vis_med[2 * N + ip] = mu[t];
          for (int q = 0; q < nm; q++) {
            vis_y[(size_t)q * N + ip] = yl[(size_t)q * np + t];
            vis_y[(size_t)(nm + q) * N + ip] = ym[(size_t)q * np + t];
          }
        }
    dvis = *d;
    dvis.medium_type = CGFD_MEDIUM_ELASTIC_ISO;
    dvis.medium = vis_med.data();
    dvis.visco = nullptr;
    d = &dvis;
  }
  p->precision = d->precision;
  switch (d->precision) {
    case CGFD_PREC_BF16_COEF: p->coef_type = cgfd::COEF_BF16; break;
    case CGFD_PREC_FP16_COEF: p->coef_type = cgfd::COEF_F16; break;
    case CGFD_PREC_U16_COEF:
    case CGFD_PREC_FP16_WAVE: p->coef_type = cgfd::COEF_U16; break;
    default: p->coef_type = cgfd::COEF_F32;
  }
  p->wave16 = d->precision == CGFD_PREC_FP16_WAVE ? 1 : 0;
  p->fp64 = d->precision == CGFD_PREC_FP64 ? 1 : 0;
  p->esz = p->fp64 ? sizeof(double) : sizeof(float);
  if (p->fp64 || p->vis) p->use_tma = false;  // the FP64 build and visco-elastic media run the direct-load bulk kernel
  p->device = d->device;
  CK(cudaSetDevice(p->device));
  keep_pool_memory(p->device);
  // the no-allocation snapshot path's static scratch is loaded here, with the problem's own
  // memory, so that cgfd_get_wavefield_shot_noalloc itself never takes device memory
  noalloc_scratch(p->device);
  CK(cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking));
  CK(cudaStreamCreateWithFlags(&p->side, cudaStreamNonBlocking));
  CK(cudaEventCreateWithFlags(&p->ev_fork, cudaEventDisableTiming));
  CK(cudaEventCreateWithFlags(&p->ev_join, cudaEventDisableTiming));
  p->ni = d->ni; p->nj = d->nj; p->nk = d->nk;
  p->med = d->medium_type == CGFD_MEDIUM_ACOUSTIC_ISO ? cgfd::MED_AC
           : d->medium_type == CGFD_MEDIUM_ELASTIC_ISO ? cgfd::MED_ISO
           : (d->medium_type == CGFD_MEDIUM_ELASTIC_VTI ? cgfd::MED_VTI : cgfd::MED_ANISO);
  p->ncoef = p->med == cgfd::MED_AC ? 11 : (p->med == cgfd::MED_ISO ? 12 : (p->med == cgfd::MED_VTI ? 15 : 31));
  if (p->med == cgfd::MED_AC) {  // acoustic media run their own stage kernel (TMA-pipelined in FP32)
    p->use_tma = false;
    p->ac_tma = !p->fp64;
  }
  p->nt_total = d->nt_total;
  p->dt = d->dt;
  p->free_top = d->free_top ? 1 : 0;
  if (p->free_top && p->nk < cgfd::NSURF + 4) throw cgfd::Error(CGFD_ERR_INVALID, "nk too small for the free surface");
  p->nbulk = p->med == cgfd::MED_AC || !p->free_top ? p->nk : p->nk - cgfd::NSURF;
  // device layout
  layout(p->ni, p->nj, p->nk, p->sx, p->sz, p->sf, p->off0);
  // default tiling (cgfd_set_tile_shape / cgfd_set_zchunk / the autotuner refine it): 32x4
  // tiles at three blocks per SM for iso media, the shape-0 tiles otherwise, and z chunks of
  // about 12 planes (with strip-ordered tile lists a chunk's 3-plane prologue comes from L2, and
  // short chunks keep the resident blocks on neighbouring planes)
  p->shape = p->med == cgfd::MED_ISO ? 1 : 0;
  {
    int chunks = std::max(1, (p->nbulk + 11) / 12);
    p->nzc = (p->nbulk + chunks - 1) / chunks;
  }

  size_t &B = p->bytes;
  // levels 0-1 (w_pre / w_end) FP32; 2-3 (RK stage inputs) FP32 or FP16
  const size_t E = p->esz;
  const size_t lev_bytes[4] = {E, E, p->wave16 ? 2u : E, p->wave16 ? 2u : E};
  for (int l = 0; l < 4; l++)
    p->wbuf[l] = (float *)dmalloc<uint16_t>((size_t)9 * p->sf * nshot * (lev_bytes[l] / 2), B, p->stream);
  p->coef = dalloc_real(p, (size_t)p->ncoef * p->sf, B);
  p->jac = dalloc_real(p, (size_t)p->sf, B);
  for (int l = 0; l < 4; l++) CK(cudaMemsetAsync(p->wbuf[l], 0, lev_bytes[l] * 9 * p->sf * nshot, p->stream));
  CK(cudaMemsetAsync(p->coef, 0, E * p->ncoef * p->sf, p->stream));
  CK(cudaMemsetAsync(p->jac, 0, E * p->sf, p->stream));

  // coefficients: metric (ghosts kept for the traction image), 1/rho, medium
  cgfd::RefGrid g(p->ni, p->nj, p->nk);
  float *stage_buf = dmalloc<float>(g.siz_icmp, B, p->stream);
  // desc->metric NULL: metrics computed on the device from the coordinates; the host-side
  // setup below then reads the description with `view` as its metric
  std::unique_ptr<float, void (*)(void *)> view(nullptr, std::free);
  cgfd_problem_desc dv;
  {
    PinnedStager &ps = PinnedStager::for_device(p->device);
    std::lock_guard<std::mutex> lk(ps.mutex());
    if (d->metric) {
      upload_field(p, d->metric, p->jac, stage_buf, 0, 1, &ps);
      for (int c = 0; c < 9; c++)
        upload_field(p, d->metric + (size_t)(1 + c) * g.siz_icmp, p->rvoid(p->coef, (size_t)c * p->sf), stage_buf, 0,
                     1, &ps);
    } else {
      view.reset(static_cast<float *>(std::calloc((size_t)10 * g.siz_icmp, sizeof(float))));
      if (!view) throw cgfd::Error(CGFD_ERR_NOMEM, "host memory for the metric view");
      metric_from_coords(p, d, ps, view.get());
      dv = *d;
      dv.metric = view.get();
      d = &dv;
    }
    upload_field(p, d->medium, p->rvoid(p->coef, (size_t)cgfd::CF_SLW * p->sf), stage_buf, 1, 0, &ps);
    int nmed = cgfd::medium_ncmp(d->medium_type) - 1;
    for (int c = 0; c < nmed; c++)
      upload_field(p, d->medium + (size_t)(1 + c) * g.siz_icmp, p->rvoid(p->coef, (size_t)(cgfd::CF_MED + c) * p->sf),
                   stage_buf, 0, 0, &ps);
    if (p->vis) {
      p->d_y = dalloc_real(p, (size_t)2 * p->nmax * p->sf, B);
      CK(cudaMemsetAsync(p->d_y, 0, sizeof(float) * 2 * p->nmax * p->sf, p->stream));
      for (int c = 0; c < 2 * p->nmax; c++)
        upload_field(p, vis_y.data() + (size_t)c * g.siz_icmp, p->d_y + (size_t)c * p->sf, stage_buf, 0, 0, &ps);
    }
  }
  CK(cudaStreamSynchronize(p->stream));
  dfree(stage_buf, p->stream);
  B -= g.siz_icmp * sizeof(float);
  if (p->coef_type != cgfd::COEF_F32) to_16bit_coefficients(p);

  // TMA tensor maps of the four wavefield levels and of the coefficients
  if (p->use_tma) make_maps(p);
  if (p->ac_tma) make_ac_maps(p);
  // free surface of elastic media: velocity-gradient conversion and traction-image fluxes
  if (p->free_top && p->med != cgfd::MED_AC) {
    std::vector<float> mx, my;
    cgfd::dvh2dvz(d, mx, my);
    p->matx = dalloc_real(p, mx.size(), B);
    p->maty = dalloc_real(p, my.size(), B);
    upload_real(p, p->matx, mx);
    upload_real(p, p->maty, my);
    p->d_flux = dalloc_real(p, (size_t)9 * cgfd::kFluxPlanes * (p->ni + 6) * (p->nj + 6) * nshot, B);
  }
  if (p->vis) {
    for (int l = 0; l < 4; l++) {
      p->jbuf[l] = dalloc_real(p, (size_t)6 * p->nmax * p->sf, B);
      CK(cudaMemsetAsync(p->jbuf[l], 0, sizeof(float) * 6 * p->nmax * p->sf, p->stream));
    }
    p->d_rhs = dalloc_real(p, (size_t)9 * p->sf, B);
    CK(cudaMemsetAsync(p->d_rhs, 0, sizeof(float) * 9 * p->sf, p->stream));
    if (p->free_top) {
      std::vector<float> md;
      cgfd::vis_free_matrix(d, md);
      p->d_matD = dalloc_real(p, md.size(), B);
      upload_real(p, p->d_matD, md);
    }
  }
  // PML
  cgfd::PmlFaceHost fh[3][2];
  cgfd::pml_setup(d, fh);
  for (int a = 0; a < 3; a++)
    for (int s = 0; s < 2; s++) {
      if (!fh[a][s].enable) continue;
      cgfd_problem::Face f;
      f.h = fh[a][s];
      f.n = (long long)(f.h.hi[0] - f.h.lo[0] + 1) * (f.h.hi[1] - f.h.lo[1] + 1) * (f.h.hi[2] - f.h.lo[2] + 1);
      size_t N1 = f.h.A.size();
      f.A = dalloc_real(p, N1, B); f.B = dalloc_real(p, N1, B); f.D = dalloc_real(p, N1, B);
      upload_real(p, f.A, f.h.A);
      upload_real(p, f.B, f.h.B);
      upload_real(p, f.D, f.h.D);
      f.aux = dalloc_real(p, (size_t)3 * 9 * f.n * nshot, B);
      CK(cudaMemset(f.aux, 0, E * 3 * 9 * f.n * nshot));
      p->faces.push_back(f);
    }
  // sources: one set per shot, concatenated (each source knows its shot)
  if (!shots) {
    cgfd::Located sl;
    cgfd::src_setup(d, p->src, locate_sources(d, sl));
    p->src_shot.assign(p->src.nsrc, 0);
  } else {
    cgfd::SrcHost &all = p->src;
    all = cgfd::SrcHost();
    std::vector<cgfd::SrcHost> per(nshot);
    for (int sh = 0; sh < nshot; sh++) {
      cgfd_problem_desc ds = *d;
      ds.src = shots[sh];
      cgfd::validate_desc(&ds);
      cgfd::Located sl;
      cgfd::src_setup(&ds, per[sh], locate_sources(&ds, sl));
      all.max_nt = std::max(all.max_nt, per[sh].max_nt);
      all.max_ext = std::max(all.max_ext, per[sh].max_ext);
      all.force |= per[sh].force;
      all.moment |= per[sh].moment;
    }
    for (int sh = 0; sh < nshot; sh++) {
      const cgfd::SrcHost &q = per[sh];
      for (int is = 0; is < q.nsrc; is++) {
        all.it_begin.push_back(q.it_begin[is]);
        all.ext_num.push_back(q.ext_num[is]);
        for (int e = 0; e < all.max_ext; e++) {
          bool ok = e < q.max_ext;
          size_t qe = (size_t)is * q.max_ext + e;
          all.ext_i.push_back(ok ? q.ext_i[qe] : 0);
          all.ext_j.push_back(ok ? q.ext_j[qe] : 0);
          all.ext_k.push_back(ok ? q.ext_k[qe] : 0);
          all.ext_wv.push_back(ok ? q.ext_wv[qe] : 0.f);
          all.ext_wt.push_back(ok ? q.ext_wt[qe] : 0.f);
        }
        for (int t = 0; t < all.max_nt; t++)
          for (int c = 0; c < 36; c++)
            all.stf.push_back(t < q.max_nt ? q.stf[((size_t)is * q.max_nt + t) * 36 + c] : 0.f);
        p->src_shot.push_back(sh);
        all.nsrc++;
      }
    }
  }
  if (p->med == cgfd::MED_AC) {
    // the acoustic source term takes the force and Mxx only (sv_curv_col_ac_iso_rhs_src_gpu,
    // sv_curv_col_ac_iso_gpu.cu:823-887); the other moment components would land in the unused
    // fields 4-8
    for (size_t q = 0; q < p->src.stf.size(); q += 9)
      for (int c = 4; c < 9; c++) p->src.stf[q + c] = 0.f;
  }
  if (p->src.nsrc > 0) {
    cgfd::SrcHost &s = p->src;
    size_t ne = (size_t)s.nsrc * s.max_ext;
    std::vector<long long> idx(ne, p->off0);
    for (size_t e = 0; e < ne; e++) idx[e] = p->didx(s.ext_i[e], s.ext_j[e], s.ext_k[e]);
    p->d_it_begin = dmalloc<int>(s.nsrc, B, p->stream);
    p->d_ext_num = dmalloc<int>(s.nsrc, B, p->stream);
    p->d_ext_idx = dmalloc<long long>(ne, B, p->stream);
    p->d_ext_wv = dmalloc<float>(ne, B, p->stream);
    p->d_ext_wt = dmalloc<float>(ne, B, p->stream);
    p->d_stf = dmalloc<float>(s.stf.size(), B, p->stream);
    p->d_src_shot = dmalloc<int>(s.nsrc, B, p->stream);
    CK(cudaMemcpy(p->d_src_shot, p->src_shot.data(), s.nsrc * sizeof(int), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(p->d_it_begin, s.it_begin.data(), s.nsrc * sizeof(int), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(p->d_ext_num, s.ext_num.data(), s.nsrc * sizeof(int), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(p->d_ext_idx, idx.data(), ne * sizeof(long long), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(p->d_ext_wv, s.ext_wv.data(), ne * sizeof(float), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(p->d_ext_wt, s.ext_wt.data(), ne * sizeof(float), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(p->d_stf, s.stf.data(), s.stf.size() * sizeof(float), cudaMemcpyHostToDevice));
  }
  // stations (those given by physical coordinates located on the device first)
  {
    const cgfd_station_desc &st = d->sta;
    std::vector<int> which;
    std::vector<float> xyz;
    std::vector<int> depth;
    for (int r = 0; r < st.num; r++)
      if (st.flag_coord[r] == 1) {
        which.push_back(r);
        xyz.insert(xyz.end(), st.loc + 3 * r, st.loc + 3 * r + 3);
        depth.push_back(st.flag_depth[r] == 1);
      }
    cgfd::Located rl;
    if (!which.empty()) {
      cgfd::Located part;
      cgfd::locate_coords(d, (int)which.size(), xyz.data(), depth.data(), part);
      rl.idx.assign(3 * (size_t)st.num, -1000);
      rl.inc.assign(3 * (size_t)st.num, 0.f);
      rl.xyz.assign(3 * (size_t)st.num, 0.f);
      for (size_t w = 0; w < which.size(); w++)
        for (int a = 0; a < 3; a++) {
          rl.idx[3 * which[w] + a] = part.idx[3 * w + a];
          rl.inc[3 * which[w] + a] = part.inc[3 * w + a];
          rl.xyz[3 * which[w] + a] = part.xyz[3 * w + a];
        }
    }
    cgfd::recv_setup(d, p->rec, which.empty() ? nullptr : &rl);
  }
  if (p->rec.n > 0) {
    std::vector<long long> idx8((size_t)p->rec.n * 8);
    for (int r = 0; r < p->rec.n; r++)
      for (int q = 0; q < 8; q++)
        idx8[(size_t)r * 8 + q] = p->didx(p->rec.i[r] + (q & 1), p->rec.j[r] + ((q >> 1) & 1), p->rec.k[r] + ((q >> 2) & 1));
    p->d_idx8 = dmalloc<long long>(idx8.size(), B, p->stream);
    p->d_w8 = dmalloc<float>(p->rec.w8.size(), B, p->stream);
    p->d_seis = dmalloc<float>((size_t)p->rec.n * 9 * p->nt_total * nshot, B, p->stream);
    CK(cudaMemcpy(p->d_idx8, idx8.data(), idx8.size() * sizeof(long long), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(p->d_w8, p->rec.w8.data(), p->rec.w8.size() * sizeof(float), cudaMemcpyHostToDevice));
    CK(cudaMemset(p->d_seis, 0, sizeof(float) * p->rec.n * 9 * p->nt_total * nshot));
  }
  make_tiles(p);
  if (p->free_top) {
    const size_t nij = (size_t)p->ni * p->nj * nshot;
    p->d_pg = dmalloc<float>(15 * nij, B, p->stream);
    p->d_dis = dalloc_real(p, 3 * nij, B);
    CK(cudaMemset(p->d_pg, 0, sizeof(float) * 15 * nij));
    CK(cudaMemset(p->d_dis, 0, E * 3 * nij));
  }
  p->d_it = dmalloc<int>(1, B, p->stream);
  p->d_flag = dmalloc<int>(1, B, p->stream);
  CK(cudaMemset(p->d_it, 0, sizeof(int)));
  CK(cudaMemset(p->d_flag, 0, sizeof(int)));
  if (p->wave16) {
    p->d_wsc = dmalloc<float>(18 * (size_t)nshot, B, p->stream);
    p->d_amax = dmalloc<unsigned int>(2 * (size_t)nshot, B, p->stream);
    CK(cudaMemset(p->d_wsc, 0, sizeof(float) * 18 * nshot));
    CK(cudaMemset(p->d_amax, 0, sizeof(unsigned int) * 2 * nshot));  // the wavefield starts at zero
    std::vector<float> sb = source_bounds(p);
    p->d_srcb = dmalloc<float>(sb.size(), B, p->stream);
    CK(cudaMemcpy(p->d_srcb, sb.data(), sb.size() * sizeof(float), cudaMemcpyHostToDevice));
  }
  CK(cudaDeviceSynchronize());
}

// TMA tensor maps of the four wavefield levels and of the coefficients for the current tile
// shape (box heights follow the tile), and the bulk kernels' shared-memory attributes.
void make_maps(cgfd_problem *p) {
  const int nshot = p->nshot;
  {
    const int ty = cgfd::tma_tile_y(p->med, p->shape);
    // The stage-input (halo) maps cover the physical cells only, from (0, 0, 0): the halo columns,
    // rows and planes beyond the grid, which hold zeros in memory, come as the boxes' zero fill
    // instead of as DRAM lines of row padding and ghost cells. The centre-box maps cover the
    // whole allocation (padded coordinates).
    const long long nx = p->ni, ny = p->nj, nz = p->nk;
    for (int l = 0; l < 4; l++) {
      if (p->wave16 && l >= 2) {  // FP16 stage level: x halo of 8 elements keeps the box 16-byte aligned
        make_map(&p->map_halo[l], reinterpret_cast<const __half *>(p->wbuf[l]) + p->off0, nx, ny, nz, 9 * nshot, p->sx,
                 p->sz, p->sf, cgfd::TX + 16, ty + 4, 9, CU_TENSOR_MAP_DATA_TYPE_FLOAT16, 2);
        make_map(&p->map_ctr[l], p->wbuf[l], p->sx, p->nj + 6, p->nk + 6, 9 * nshot, p->sx, p->sz, p->sf, cgfd::TX, ty,
                 9, CU_TENSOR_MAP_DATA_TYPE_FLOAT16, 2);
        continue;
      }
      make_map(&p->map_halo[l], p->wbuf[l] + p->off0, nx, ny, nz, 9 * nshot, p->sx, p->sz, p->sf, cgfd::TX + 8, ty + 4,
               9);
      make_map(&p->map_ctr[l], p->wbuf[l], p->sx, p->nj + 6, p->nk + 6, 9 * nshot, p->sx, p->sz, p->sf, cgfd::TX, ty, 9);
    }
    if (p->coef_type == cgfd::COEF_F32)
      make_map(&p->map_coef, p->coef, p->sx, p->nj + 6, p->nk + 6, p->ncoef, p->sx, p->sz, p->sf, cgfd::TX, ty,
               p->ncoef);
    else
      make_map(&p->map_coef, p->coef16, p->sx, p->nj + 6, p->nk + 6, p->ncoef, p->sx, p->sz, p->sf, cgfd::TX, ty,
               p->ncoef,
               p->coef_type == cgfd::COEF_F16    ? CU_TENSOR_MAP_DATA_TYPE_FLOAT16
               : p->coef_type == cgfd::COEF_BF16 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16
                                                 : CU_TENSOR_MAP_DATA_TYPE_UINT16,
               2);
    CK(cgfd::tma_prepare(p->med, p->coef_type, p->wave16, p->shape));
  }
}

// TMA tensor maps of the acoustic stage kernel: the stage input of each level (physical cells and
// the 3 ghost planes above the top, which hold the free surface's pressure image; 4 fields of a
// shot), w_pre / w_end centre boxes (levels 0-1, 4 fields) and the 11 coefficient fields.
void make_ac_maps(cgfd_problem *p) {
  const int nshot = p->nshot;
  for (int l = 0; l < 4; l++) {
    make_map(&p->map_halo[l], p->wbuf[l] + p->off0, p->ni, p->nj, p->nk + 3, 9 * nshot, p->sx, p->sz, p->sf,
             cgfd::TX + 8, cgfd::TY + 4, 4);
    make_map(&p->map_ctr[l], p->wbuf[l], p->sx, p->nj + 6, p->nk + 6, 9 * nshot, p->sx, p->sz, p->sf, cgfd::TX,
             cgfd::TY, 4);
  }
  make_map(&p->map_coef, p->coef, p->sx, p->nj + 6, p->nk + 6, p->ncoef, p->sx, p->sz, p->sf, cgfd::TX, cgfd::TY,
           p->ncoef);
}

// Tile lists of the TMA bulk kernel: 32 x TY columns, split along z into chunks of about
// nzc planes that never straddle a z-face boundary of the CFS-PML (so planes above the
// bottom absorbing layer run as tiles without face code); a tile that any PML face box meets
// carries the kTilePml flag. Entries (bx [+ kTilePml] [+ shot << 16], by, first plane, end plane).
// Order: strips of tile rows, each strip z layer by z layer, x fastest. A strip's layer holds
// about as many blocks as the GPU keeps resident, so that a tile's x-y neighbours run beside it
// at the same planes (their halo lines are read from DRAM once), and the tile's next chunk
// starts as this one ends (the 3 planes its register queue starts from are still in L2). The
// layers run in the march direction of the stage's z operator: upwards for backward operators
// (tiles), downwards for forward ones (tiles_dn).
void make_tiles(cgfd_problem *p) {
  if (p->med == cgfd::MED_AC) return;  // no TMA kernel for acoustic media
  const int ty = cgfd::tma_tile_y(p->med, p->shape), nbulk = p->nbulk;
  const int nbx = (p->ni + cgfd::TX - 1) / cgfd::TX, nby = (p->nj + ty - 1) / ty;
  if (nbx > cgfd::kTileBxMask + 1) throw cgfd::Error(CGFD_ERR_INVALID, "grid too wide for the bulk tile list");
  std::vector<int> cuts = {0, nbulk};
  for (const auto &f : p->faces)
    if (f.h.axis == 2)
      for (int c : {f.h.lo[2], f.h.hi[2] + 1})
        if (c > 0 && c < nbulk) cuts.push_back(c);
  std::sort(cuts.begin(), cuts.end());
  cuts.erase(std::unique(cuts.begin(), cuts.end()), cuts.end());
  std::vector<std::pair<int, int>> zr;
  for (size_t s = 0; s + 1 < cuts.size(); s++) {
    const int len = cuts[s + 1] - cuts[s], nch = std::max(1, (len + p->nzc - 1) / p->nzc);
    for (int c = 0; c < nch; c++) zr.emplace_back(cuts[s] + len * c / nch, cuts[s] + len * (c + 1) / nch);
  }
  int nsm = 148;
  CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, p->device));
  const int group = std::max(1, std::min(p->shot_group, p->nshot));
  const long long resident = (long long)nsm * cgfd::tma_blocks_per_sm(p->med, p->shape);
  const int strip = (int)std::max<long long>(1, (resident + (long long)nbx * group - 1) / ((long long)nbx * group));
  for (int dn = 0; dn < 2; dn++) {
    std::vector<int4> list;
    int npml = 0;
    for (int s0 = 0; s0 < nby; s0 += strip)
      for (size_t zi = 0; zi < zr.size(); zi++) {
        const auto &z = zr[dn ? zr.size() - 1 - zi : zi];
        for (int by = s0; by < std::min(nby, s0 + strip); by++)
          for (int bx = 0; bx < nbx; bx++) {
            bool touch = false;
            for (const auto &f : p->faces) {
              const bool xo = f.h.lo[0] <= bx * cgfd::TX + cgfd::TX - 1 && f.h.hi[0] >= bx * cgfd::TX;
              const bool yo = f.h.lo[1] <= by * ty + ty - 1 && f.h.hi[1] >= by * ty;
              const bool zo = f.h.lo[2] <= z.second - 1 && f.h.hi[2] >= z.first;
              touch |= xo && yo && zo;
            }
            npml += touch;
            list.push_back(make_int4(bx + (touch ? cgfd::kTilePml : 0), by, z.first, z.second));
          }
      }
    // batches: one entry per tile and shot, the shots in groups of `group`; a group's entries
    // cover every tile before the next group's, the shot fastest within a group (the group's
    // blocks of one tile share its coefficient tiles through L2, and a tile's x-y neighbours of
    // the same shot stay resident beside it)
    if (p->nshot > 1) {
      std::vector<int4> ex;
      ex.reserve(list.size() * p->nshot);
      for (int g0 = 0; g0 < p->nshot; g0 += group)
        for (const int4 &e : list)
          for (int sh = g0; sh < std::min(p->nshot, g0 + group); sh++)
            ex.push_back(make_int4(e.x + (sh << 16), e.y, e.z, e.w));
      list.swap(ex);
      npml *= p->nshot;
    }
    int4 *&dt = dn ? p->d_tiles_dn : p->d_tiles;
    cgfd::BulkTiles &tl = dn ? p->tiles_dn : p->tiles;
    dfree(dt, p->stream);
    dt = nullptr;
    size_t acc = 0;
    dt = dmalloc<int4>(std::max<size_t>(list.size(), 1), acc, p->stream);
    if (!list.empty()) CK(cudaMemcpy(dt, list.data(), list.size() * sizeof(int4), cudaMemcpyHostToDevice));
    tl.list = dt;
    tl.n = (int)list.size();
    tl.npml = npml;
  }
}

// Back to the state right after cgfd_problem_create: zero wavefield levels, PML auxiliaries,
// seismograms, peak motion, scale collectors, error word; step 0.
void reset_state(cgfd_problem *p) {
  const size_t E = p->esz;
  const size_t lev_bytes[4] = {E, E, p->wave16 ? 2u : E, p->wave16 ? 2u : E};
  for (int l = 0; l < 4; l++) CK(cudaMemsetAsync(p->wbuf[l], 0, lev_bytes[l] * 9 * p->sf * p->nshot, p->stream));
  for (auto &f : p->faces) CK(cudaMemsetAsync(f.aux, 0, E * 3 * 9 * f.n * p->nshot, p->stream));
  for (auto *jb : p->jbuf)
    if (jb) CK(cudaMemsetAsync(jb, 0, sizeof(float) * 6 * p->nmax * p->sf, p->stream));
  if (p->rec.n > 0)
    CK(cudaMemsetAsync(p->d_seis, 0, sizeof(float) * p->rec.n * 9 * p->nt_total * p->nshot, p->stream));
  if (p->nline > 0)
    CK(cudaMemsetAsync(p->d_line_seis, 0, sizeof(float) * p->nline * 9 * p->nt_total * p->nshot, p->stream));
  if (p->d_pg) {
    const size_t nij = (size_t)p->ni * p->nj * p->nshot;
    CK(cudaMemsetAsync(p->d_pg, 0, sizeof(float) * 15 * nij, p->stream));
    CK(cudaMemsetAsync(p->d_dis, 0, p->esz * 3 * nij, p->stream));
  }
  if (p->d_amax) CK(cudaMemsetAsync(p->d_amax, 0, sizeof(unsigned int) * 2 * p->nshot, p->stream));
  p->it = 0;
  CK(cudaMemsetAsync(p->d_it, 0, sizeof(int), p->stream));
  CK(cudaMemsetAsync(p->d_flag, 0, sizeof(int), p->stream));
  CK(cudaStreamSynchronize(p->stream));
  p->collect_timing();
}

// FP16 stage levels: recompute max |w_pre| after the host replaced or re-labelled levels.
void refresh_wave_max(cgfd_problem *p) {
  if (!p->wave16) return;
  CK(cudaMemsetAsync(p->d_amax, 0, sizeof(unsigned int) * 2 * p->nshot, p->stream));
  cgfd::launch_wave_absmax(p->wbuf[p->it & 1], p->sf, p->nshot, p->d_amax, p->stream);
  CK(cudaGetLastError());
}

}  // namespace

void cgfd::set_last_error(const std::string &m) { set_err(m); }

extern "C" {

int cgfd_version(void) { return 100; }

const char *cgfd_last_error(void) { return g_err.c_str(); }

int cgfd_problem_bytes(const cgfd_problem_desc *desc, int nshot, const cgfd_source_desc *shots, size_t *resident,
                       size_t *peak) {
  if (!desc) { set_err("desc is NULL"); return CGFD_ERR_INVALID; }
  return guarded([&] { problem_bytes(desc, nshot, shots, resident, peak); });
}

int cgfd_problem_create(const cgfd_problem_desc *desc, cgfd_problem **out) {
  if (!out) { set_err("out is NULL"); return CGFD_ERR_INVALID; }
  *out = nullptr;
  cgfd_problem *p = new cgfd_problem;
  int rc = guarded([&] { build(p, desc, 1, nullptr); });
  if (rc != CGFD_OK) {
    p->release();
    delete p;
    return rc;
  }
  *out = p;
  return CGFD_OK;
}

int cgfd_batch_create(const cgfd_problem_desc *desc, int nshot, const cgfd_source_desc *shots, cgfd_problem **out) {
  if (!out || !shots) { set_err("out/shots is NULL"); return CGFD_ERR_INVALID; }
  *out = nullptr;
  cgfd_problem *p = new cgfd_problem;
  int rc = guarded([&] { build(p, desc, nshot, shots); });
  if (rc != CGFD_OK) {
    p->release();
    delete p;
    return rc;
  }
  *out = p;
  return CGFD_OK;
}

int cgfd_num_shots(const cgfd_problem *p) { return p ? p->nshot : -1; }

int cgfd_problem_destroy(cgfd_problem *p) {
  if (!p) return CGFD_OK;
  p->release();
  delete p;
  return CGFD_OK;
}

int cgfd_enqueue_steps(cgfd_problem *p, int nsteps) {
  if (!p) { set_err("problem is NULL"); return CGFD_ERR_INVALID; }
  return guarded([&] {
    CK(cudaSetDevice(p->device));
    if (nsteps < 0) nsteps = p->nt_total - p->it;
    p->run_steps(nsteps);
  });
}

int cgfd_synchronize(cgfd_problem *p) {
  if (!p) { set_err("problem is NULL"); return CGFD_ERR_INVALID; }
  return guarded([&] {
    CK(cudaSetDevice(p->device));
    CK(cudaStreamSynchronize(p->stream));
    p->collect_timing();
    int flag = 0;
    CK(cudaMemcpy(&flag, p->d_flag, sizeof(int), cudaMemcpyDeviceToHost));
    if (flag & cgfd::kErrPipelineTimeout)
      throw cgfd::Error(CGFD_ERR_CUDA, "a TMA pipeline wait timed out in the stage kernel");
    if (flag & cgfd::kErrWaveNonfinite)
      throw cgfd::Error(CGFD_ERR_NONFINITE, "non-finite value in the wavefield (RK combine of stage 3)");
    if (flag) throw cgfd::Error(CGFD_ERR_NONFINITE, "non-finite value sampled at a station");
  });
}

int cgfd_check_wait_bound(cgfd_problem *p) {
  if (!p) { set_err("problem is NULL"); return CGFD_ERR_INVALID; }
  int rc = guarded([&] {
    CK(cudaSetDevice(p->device));
    CK(cudaStreamSynchronize(p->stream));
    cgfd::launch_wait_bound_check(p->d_flag, 1 << 16, p->stream);
    CK(cudaGetLastError());
  });
  if (rc != CGFD_OK) return rc;
  rc = cgfd_synchronize(p);  // reports the timeout like a stage kernel's
  std::string msg = g_err;
  int zero = 0;
  if (cudaMemcpy(p->d_flag, &zero, sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess) {
    set_err("could not clear the device error word");
    return CGFD_ERR_CUDA;
  }
  set_err(msg);
  return rc;
}

int cgfd_run(cgfd_problem *p, int nsteps) {
  int rc = cgfd_enqueue_steps(p, nsteps);
  if (rc) return rc;
  return cgfd_synchronize(p);
}

int cgfd_current_step(const cgfd_problem *p) { return p ? p->it : -1; }

int cgfd_set_step(cgfd_problem *p, int it) {
  if (!p || it < 0) { set_err("invalid argument"); return CGFD_ERR_INVALID; }
  return guarded([&] {
    CK(cudaSetDevice(p->device));
    CK(cudaStreamSynchronize(p->stream));
    // the buffer roles follow the step parity: move w_pre / PML pre to the new parity
    if ((it & 1) != (p->it & 1)) {
      std::swap(p->wbuf[0], p->wbuf[1]);
      std::swap(p->map_halo[0], p->map_halo[1]);
      std::swap(p->map_ctr[0], p->map_ctr[1]);
      for (auto &f : p->faces) {
        size_t n = (size_t)9 * f.n * p->nshot;
        void *l0 = p->rvoid(f.aux, 0), *l1 = p->rvoid(f.aux, n), *l2 = p->rvoid(f.aux, 2 * n);
        CK(cudaMemcpyAsync(l2, l0, n * p->esz, cudaMemcpyDeviceToDevice, p->stream));
        CK(cudaMemcpyAsync(l0, l1, n * p->esz, cudaMemcpyDeviceToDevice, p->stream));
        CK(cudaMemcpyAsync(l1, l2, n * p->esz, cudaMemcpyDeviceToDevice, p->stream));
      }
      for (int s = 0; s < 8; s++)
        if (p->graph_ok[s]) { cudaGraphExecDestroy(p->graph[s]); p->graph_ok[s] = false; }
    }
    p->it = it;
    CK(cudaMemcpyAsync(p->d_it, &p->it, sizeof(int), cudaMemcpyHostToDevice, p->stream));
    refresh_wave_max(p);
    CK(cudaStreamSynchronize(p->stream));
  });
}

int cgfd_num_stations(const cgfd_problem *p) { return p ? p->rec.n : -1; }

int cgfd_station_info(const cgfd_problem *p, int *input_index, int *ijk) {
  if (!p) { set_err("problem is NULL"); return CGFD_ERR_INVALID; }
  for (int r = 0; r < p->rec.n; r++) {
    if (input_index) input_index[r] = p->rec.input_index[r];
    if (ijk) { ijk[3 * r] = p->rec.i[r]; ijk[3 * r + 1] = p->rec.j[r]; ijk[3 * r + 2] = p->rec.k[r]; }
  }
  return CGFD_OK;
}

int cgfd_get_seismograms(cgfd_problem *p, float *out) {
  if (!p || !out) { set_err("invalid argument"); return CGFD_ERR_INVALID; }
  return guarded([&] {
    CK(cudaSetDevice(p->device));
    CK(cudaStreamSynchronize(p->stream));
    if (p->rec.n > 0)
      CK(cudaMemcpy(out, p->d_seis, sizeof(float) * p->rec.n * 9 * p->nt_total * p->nshot, cudaMemcpyDeviceToHost));
  });
}

int cgfd_get_wavefield_shot(cgfd_problem *p, int shot, float *out) {
  if (!p || !out || shot < 0 || shot >= p->nshot) { set_err("invalid argument"); return CGFD_ERR_INVALID; }
  return guarded([&] {
    CK(cudaSetDevice(p->device));
    cgfd::RefGrid g(p->ni, p->nj, p->nk);
    size_t acc = 0;
    float *tmp = dmalloc<float>(g.siz_icmp, acc, p->stream);
    for (int c = 0; c < 9; c++) {
      const size_t off = ((size_t)shot * 9 + c) * p->sf;
      if (p->fp64)
        cgfd::launch_repack_out(p->rptr<double>(p->wbuf[p->it & 1], off), tmp, p->ni, p->nj, p->nk, p->sx, p->sz,
                                p->off0, p->stream);
      else
        cgfd::launch_repack_out(p->rptr<float>(p->wbuf[p->it & 1], off), tmp, p->ni, p->nj, p->nk, p->sx, p->sz,
                                p->off0, p->stream);
      CK(cudaMemcpyAsync(out + (size_t)c * g.siz_icmp, tmp, g.siz_icmp * sizeof(float), cudaMemcpyDeviceToHost, p->stream));
    }
    CK(cudaStreamSynchronize(p->stream));
    dfree(tmp, p->stream);
  });
}

int cgfd_get_wavefield(cgfd_problem *p, float *out) { return cgfd_get_wavefield_shot(p, 0, out); }

int cgfd_get_wavefield_box(cgfd_problem *p, int shot, const int *start, const int *count, const int *stride,
                           float *out) {
  if (!p || !out || !start || !count || !stride || shot < 0 || shot >= p->nshot) {
    set_err("invalid argument");
    return CGFD_ERR_INVALID;
  }
  const int n[3] = {p->ni, p->nj, p->nk};
  for (int a = 0; a < 3; a++)
    if (count[a] < 1 || stride[a] < 1 || start[a] < 0 || start[a] + (long long)(count[a] - 1) * stride[a] >= n[a]) {
      set_err("box outside the physical grid");
      return CGFD_ERR_INVALID;
    }
  return guarded([&] {
    CK(cudaSetDevice(p->device));
    const size_t cnt = (size_t)9 * count[0] * count[1] * count[2];
    if (cnt > p->box_cap) {  // the staging buffer stays with the problem and counts in its bytes
      CK(cudaStreamSynchronize(p->stream));
      dfree(p->d_box, p->stream);
      p->d_box = nullptr;
      p->bytes -= p->box_cap * sizeof(float);
      p->box_cap = 0;
      p->d_box = dmalloc<float>(cnt, p->bytes, p->stream);
      p->box_cap = cnt;
    }
    const size_t off = (size_t)shot * 9 * p->sf;
    if (p->fp64)
      cgfd::launch_gather_box(p->rptr<double>(p->wbuf[p->it & 1], off), p->sf, p->sx, p->sz, p->off0, start, count,
                              stride, p->d_box, p->stream);
    else
      cgfd::launch_gather_box(p->rptr<float>(p->wbuf[p->it & 1], off), p->sf, p->sx, p->sz, p->off0, start, count,
                              stride, p->d_box, p->stream);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(out, p->d_box, cnt * sizeof(float), cudaMemcpyDeviceToHost, p->stream));
    CK(cudaStreamSynchronize(p->stream));
  });
}

int cgfd_get_peak_motion(cgfd_problem *p, int shot, float *out) {
  if (!p || !out || shot < 0 || shot >= p->nshot) { set_err("invalid argument"); return CGFD_ERR_INVALID; }
  if (!p->free_top) { set_err("peak ground motion is computed at a free surface only"); return CGFD_ERR_UNSUPPORTED; }
  return guarded([&] {
    CK(cudaSetDevice(p->device));
    CK(cudaStreamSynchronize(p->stream));
    const size_t nij = (size_t)p->ni * p->nj, nx = p->ni + 6, ny = p->nj + 6;
    std::vector<float> pg(15 * nij);
    CK(cudaMemcpy(pg.data(), p->d_pg + (size_t)shot * 15 * nij, pg.size() * sizeof(float), cudaMemcpyDeviceToHost));
    std::fill(out, out + 15 * nx * ny, 0.f);  // ghost points stay 0 (PG_slice_output writes nx x ny)
    for (int q = 0; q < 15; q++)
      for (int j = 0; j < p->nj; j++)
        memcpy(out + (size_t)q * nx * ny + (size_t)(j + 3) * nx + 3, pg.data() + (size_t)q * nij + (size_t)j * p->ni,
               p->ni * sizeof(float));
  });
}

}  // extern "C"

// ---- wavefield read-back without device allocation -------------------------------------
// cgfd_get_wavefield_shot stages one wavefield component in a temporary device buffer taken
// from the stream-ordered pool ((ni+6)(nj+6)(nk+6) floats for the call's duration). Some
// callers cannot afford that: a serving process that keeps the device filled to its memory
// budget with resident problems, where the temporary may not fit and a snapshot must not fail
// for lack of memory. This variant stages through one fixed static device array instead, a
// few z planes at a time. The array (and the repack kernel's code) is loaded when a problem
// is created on the device, so the entry point itself takes no device memory.
namespace {

constexpr size_t kNoAllocScratchFloats = (size_t)1 << 20;  // 4 MiB: one chunk of reference planes
constexpr int kNoAllocMaxDevices = 64;
static __device__ __align__(256) float g_noalloc_scratch[kNoAllocScratchFloats];
std::mutex g_noalloc_mu;
float *g_noalloc_ptr[kNoAllocMaxDevices] = {};

// planes [kr0, kr0 + nplanes) of one field in the reference layout (3 ghosts, 0 there)
template <typename R>
__global__ void k_repack_out_planes(const R *__restrict__ src, float *__restrict__ dst, int ni, int nj, int nk,
                                    long long sx, long long sz, long long off0, int kr0, int nplanes) {
  const long long nxr = ni + 6, nyr = nj + 6;
  const long long total = nxr * nyr * nplanes;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    const int ir = (int)(t % nxr), jr = (int)((t / nxr) % nyr), kr = kr0 + (int)(t / (nxr * nyr));
    const int i = ir - 3, j = jr - 3, k = kr - 3;
    const bool inner = i >= 0 && i < ni && j >= 0 && j < nj && k >= 0 && k < nk;
    dst[t] = inner ? (float)src[off0 + (long long)k * sz + (long long)j * sx + i] : 0.0f;
  }
}

// Device address of the scratch array on `device` (current): looked up once per device, by
// the first problem created there. The lookup loads this file's device module (the 4 MiB array
// and the repack kernel, whose code cudaFuncGetAttributes loads as well under lazy loading).
float *noalloc_scratch(int device) {
  if (device < 0 || device >= kNoAllocMaxDevices) throw cgfd::Error(CGFD_ERR_INVALID, "device ordinal out of range");
  std::lock_guard<std::mutex> g(g_noalloc_mu);
  if (!g_noalloc_ptr[device]) {
    float *ptr = nullptr;
    cudaError_t e = cudaGetSymbolAddress((void **)&ptr, g_noalloc_scratch);
    if (e != cudaSuccess || !ptr)
      throw cgfd::Error(CGFD_ERR_CUDA, std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
    cudaFuncAttributes fa;
    e = cudaFuncGetAttributes(&fa, k_repack_out_planes<float>);
    if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, k_repack_out_planes<double>);
    if (e != cudaSuccess)
      throw cgfd::Error(CGFD_ERR_CUDA, std::string("cudaFuncGetAttributes(repack): ") + cudaGetErrorString(e));
    g_noalloc_ptr[device] = ptr;
  }
  return g_noalloc_ptr[device];
}

}  // namespace

extern "C" {

int cgfd_get_wavefield_shot_noalloc(cgfd_problem *p, int shot, float *out) {
  if (!p || !out || shot < 0 || shot >= p->nshot) { set_err("invalid argument"); return CGFD_ERR_INVALID; }
  return guarded([&] {
    const size_t nxr = (size_t)p->ni + 6, nyr = (size_t)p->nj + 6, nzr = (size_t)p->nk + 6;
    const size_t plane = nxr * nyr;
    if (plane > kNoAllocScratchFloats)
      throw cgfd::Error(CGFD_ERR_INVALID, "one reference-layout plane (" + std::to_string(plane) +
                                              " floats) exceeds the no-allocation scratch of " +
                                              std::to_string(kNoAllocScratchFloats) + " floats");
    CK(cudaSetDevice(p->device));
    float *scratch = noalloc_scratch(p->device);
    const int per = (int)(kNoAllocScratchFloats / plane);
    for (int c = 0; c < 9; c++)
      for (int k0 = 0; k0 < (int)nzr; k0 += per) {
        const int np = std::min(per, (int)nzr - k0);
        const size_t off = ((size_t)shot * 9 + c) * p->sf;
        // stream order keeps the copy of one chunk ahead of the kernel that refills the scratch
        if (p->fp64)
          k_repack_out_planes<<<592, 256, 0, p->stream>>>(p->rptr<double>(p->wbuf[p->it & 1], off), scratch, p->ni,
                                                           p->nj, p->nk, p->sx, p->sz, p->off0, k0, np);
        else
          k_repack_out_planes<<<592, 256, 0, p->stream>>>(p->rptr<float>(p->wbuf[p->it & 1], off), scratch, p->ni,
                                                           p->nj, p->nk, p->sx, p->sz, p->off0, k0, np);
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(out + (size_t)c * plane * nzr + (size_t)k0 * plane, scratch, (size_t)np * plane * sizeof(float),
                           cudaMemcpyDeviceToHost, p->stream));
      }
    CK(cudaStreamSynchronize(p->stream));
  });
}

int cgfd_set_line_receivers(cgfd_problem *p, int npts, const int *ijk) {
  if (!p || npts < 0 || (npts > 0 && !ijk)) { set_err("invalid argument"); return CGFD_ERR_INVALID; }
  for (int r = 0; r < npts; r++)
    if (ijk[3 * r] < 0 || ijk[3 * r] >= p->ni || ijk[3 * r + 1] < 0 || ijk[3 * r + 1] >= p->nj || ijk[3 * r + 2] < 0 ||
        ijk[3 * r + 2] >= p->nk) {
      set_err("line receiver " + std::to_string(r) + " lies outside the physical grid");
      return CGFD_ERR_INVALID;
    }
  return guarded([&] {
    CK(cudaSetDevice(p->device));
    CK(cudaStreamSynchronize(p->stream));
    dfree(p->d_line_idx8, p->stream); dfree(p->d_line_w8, p->stream); dfree(p->d_line_seis, p->stream);
    p->d_line_idx8 = nullptr; p->d_line_w8 = nullptr; p->d_line_seis = nullptr;
    p->bytes -= (size_t)p->nline * (8 * (sizeof(long long) + sizeof(float)) + 9 * p->nt_total * p->nshot * sizeof(float));
    p->nline = 0;
    if (npts > 0) {
      std::vector<long long> idx((size_t)npts * 8);
      std::vector<float> w((size_t)npts * 8, 0.f);
      for (int r = 0; r < npts; r++) {
        const long long id = p->didx(ijk[3 * r], ijk[3 * r + 1], ijk[3 * r + 2]);
        for (int q = 0; q < 8; q++) idx[(size_t)r * 8 + q] = id;
        w[(size_t)r * 8] = 1.f;
      }
      p->d_line_idx8 = dmalloc<long long>(idx.size(), p->bytes, p->stream);
      p->d_line_w8 = dmalloc<float>(w.size(), p->bytes, p->stream);
      p->d_line_seis = dmalloc<float>((size_t)npts * 9 * p->nt_total * p->nshot, p->bytes, p->stream);
      CK(cudaMemcpy(p->d_line_idx8, idx.data(), idx.size() * sizeof(long long), cudaMemcpyHostToDevice));
      CK(cudaMemcpy(p->d_line_w8, w.data(), w.size() * sizeof(float), cudaMemcpyHostToDevice));
      CK(cudaMemset(p->d_line_seis, 0, sizeof(float) * npts * 9 * p->nt_total * p->nshot));
      p->nline = npts;
    }
    for (int s = 0; s < 8; s++)
      if (p->graph_ok[s]) { cudaGraphExecDestroy(p->graph[s]); p->graph_ok[s] = false; }
  });
}

int cgfd_get_line_seismograms(cgfd_problem *p, float *out) {
  if (!p || !out) { set_err("invalid argument"); return CGFD_ERR_INVALID; }
  return guarded([&] {
    CK(cudaSetDevice(p->device));
    CK(cudaStreamSynchronize(p->stream));
    if (p->nline > 0)
      CK(cudaMemcpy(out, p->d_line_seis, sizeof(float) * p->nline * 9 * p->nt_total * p->nshot, cudaMemcpyDeviceToHost));
  });
}

int cgfd_set_slices(cgfd_problem *p, int nx, const int *ix, int ny, const int *iy, int nz, const int *iz,
                    int ring_steps) {
  if (!p || nx < 0 || ny < 0 || nz < 0 || (nx && !ix) || (ny && !iy) || (nz && !iz) ||
      (nx + ny + nz > 0 && ring_steps < 1)) {
    set_err("invalid argument");
    return CGFD_ERR_INVALID;
  }
  for (int s = 0; s < nx; s++)
    if (ix[s] < 0 || ix[s] >= p->ni) { set_err("x slice index outside the physical grid"); return CGFD_ERR_INVALID; }
  for (int s = 0; s < ny; s++)
    if (iy[s] < 0 || iy[s] >= p->nj) { set_err("y slice index outside the physical grid"); return CGFD_ERR_INVALID; }
  for (int s = 0; s < nz; s++)
    if (iz[s] < 0 || iz[s] >= p->nk) { set_err("z slice index outside the physical grid"); return CGFD_ERR_INVALID; }
  return guarded([&] {
    CK(cudaSetDevice(p->device));
    CK(cudaStreamSynchronize(p->stream));
    dfree(p->d_slice_idx, p->stream); dfree(p->d_slices, p->stream);
    p->d_slice_idx = nullptr; p->d_slices = nullptr;
    p->bytes -= (size_t)(p->nslx + p->nsly + p->nslz) * sizeof(int) +
                (size_t)p->slice_ring * p->nshot * p->slice_per_shot * sizeof(float);
    p->nslx = p->nsly = p->nslz = p->slice_ring = 0;
    p->slice_per_shot = 0;
    const long long per = 9LL * ((long long)nx * p->nk * p->nj + (long long)ny * p->nk * p->ni + (long long)nz * p->nj * p->ni);
    if (per > 0) {
      std::vector<int> idx;
      idx.insert(idx.end(), ix, ix + nx);
      idx.insert(idx.end(), iy, iy + ny);
      idx.insert(idx.end(), iz, iz + nz);
      p->d_slice_idx = dmalloc<int>(idx.size(), p->bytes, p->stream);
      CK(cudaMemcpy(p->d_slice_idx, idx.data(), idx.size() * sizeof(int), cudaMemcpyHostToDevice));
      p->d_slices = dmalloc<float>((size_t)ring_steps * p->nshot * per, p->bytes, p->stream);
      p->nslx = nx; p->nsly = ny; p->nslz = nz;
      p->slice_ring = ring_steps;
      p->slice_per_shot = per;
    }
    for (int s = 0; s < 8; s++)
      if (p->graph_ok[s]) { cudaGraphExecDestroy(p->graph[s]); p->graph_ok[s] = false; }
  });
}

int cgfd_get_slices(cgfd_problem *p, int shot, int it, float *out) {
  if (!p || !out || shot < 0 || shot >= p->nshot) { set_err("invalid argument"); return CGFD_ERR_INVALID; }
  if (p->slice_per_shot <= 0) { set_err("no slices are set"); return CGFD_ERR_INVALID; }
  if (it < 0 || it >= p->it || it < p->it - p->slice_ring) {
    set_err("step " + std::to_string(it) + " is not in the slice ring (steps " +
            std::to_string(std::max(0, p->it - p->slice_ring)) + " .. " + std::to_string(p->it - 1) + ")");
    return CGFD_ERR_INVALID;
  }
  return guarded([&] {
    CK(cudaSetDevice(p->device));
    CK(cudaStreamSynchronize(p->stream));
    const size_t off = ((size_t)(it % p->slice_ring) * p->nshot + shot) * p->slice_per_shot;
    CK(cudaMemcpy(out, p->d_slices + off, sizeof(float) * p->slice_per_shot, cudaMemcpyDeviceToHost));
  });
}

int cgfd_set_wavefield_shot(cgfd_problem *p, int shot, const float *in) {
  if (!p || !in || shot < 0 || shot >= p->nshot) { set_err("invalid argument"); return CGFD_ERR_INVALID; }
  return guarded([&] {
    CK(cudaSetDevice(p->device));
    cgfd::RefGrid g(p->ni, p->nj, p->nk);
    size_t acc = 0;
    float *tmp = dmalloc<float>(g.siz_icmp, acc, p->stream);
    {
      PinnedStager &ps = PinnedStager::for_device(p->device);
      std::lock_guard<std::mutex> lk(ps.mutex());
      // acoustic media: Vx Vy Vz P; components 4-8 are not part of the state and stay 0
      const int nf = p->med == cgfd::MED_AC ? 4 : 9;
      for (int c = 0; c < nf; c++)
        upload_field(p, in + (size_t)c * g.siz_icmp, p->rvoid(p->wbuf[p->it & 1], ((size_t)shot * 9 + c) * p->sf), tmp, 0,
                     0, &ps);
    }
    refresh_wave_max(p);
    CK(cudaStreamSynchronize(p->stream));
    dfree(tmp, p->stream);
  });
}

int cgfd_set_wavefield(cgfd_problem *p, const float *in) { return cgfd_set_wavefield_shot(p, 0, in); }

size_t cgfd_device_bytes(const cgfd_problem *p) { return p ? p->bytes : 0; }

void *cgfd_stream(cgfd_problem *p) { return p ? (void *)p->stream : nullptr; }

/* Disable (0) or enable (1) CUDA-graph replay of the time steps. */
int cgfd_set_graph_mode(cgfd_problem *p, int on) {
  if (!p) return CGFD_ERR_INVALID;
  p->use_graph = on != 0;
  return CGFD_OK;
}

/* z planes per thread block of the bulk stage kernel (autotuner knob; graphs are rebuilt). */
int cgfd_set_zchunk(cgfd_problem *p, int nzc) {
  if (!p || nzc < 1) return CGFD_ERR_INVALID;
  return guarded([&] {
    CK(cudaSetDevice(p->device));
    CK(cudaStreamSynchronize(p->stream));
    p->nzc = nzc;
    make_tiles(p);
    for (int s = 0; s < 8; s++)
      if (p->graph_ok[s]) { cudaGraphExecDestroy(p->graph[s]); p->graph_ok[s] = false; }
  });
}

int cgfd_get_zchunk(const cgfd_problem *p) { return p ? p->nzc : -1; }

/* Tile shape of the TMA bulk kernel (0 default, 1 alternative); maps, tiles and graphs are rebuilt. */
int cgfd_set_tile_shape(cgfd_problem *p, int shape) {
  if (!p || shape < 0 || shape > 1) { set_err("invalid argument"); return CGFD_ERR_INVALID; }
  if (!p->use_tma) { set_err("tile shapes belong to the TMA bulk kernel"); return CGFD_ERR_UNSUPPORTED; }
  return guarded([&] {
    CK(cudaSetDevice(p->device));
    CK(cudaStreamSynchronize(p->stream));
    p->shape = shape;
    make_maps(p);
    make_tiles(p);
    for (int s = 0; s < 8; s++)
      if (p->graph_ok[s]) { cudaGraphExecDestroy(p->graph[s]); p->graph_ok[s] = false; }
  });
}

int cgfd_get_tile_shape(const cgfd_problem *p) { return p ? p->shape : -1; }

/* Shots per block group of a batch's bulk kernel; graphs are rebuilt. */
int cgfd_set_shot_group(cgfd_problem *p, int group) {
  if (!p || group < 1) { set_err("invalid argument"); return CGFD_ERR_INVALID; }
  return guarded([&] {
    CK(cudaSetDevice(p->device));
    CK(cudaStreamSynchronize(p->stream));
    p->shot_group = group;
    if (p->use_tma) make_tiles(p);  // the strip height follows the group
    for (int s = 0; s < 8; s++)
      if (p->graph_ok[s]) { cudaGraphExecDestroy(p->graph[s]); p->graph_ok[s] = false; }
  });
}

int cgfd_get_shot_group(const cgfd_problem *p) { return p ? std::max(1, std::min(p->shot_group, p->nshot)) : -1; }

int cgfd_autotune(cgfd_problem *p, int steps, int *chosen) {
  if (!p || steps < 1) { set_err("invalid argument"); return CGFD_ERR_INVALID; }
  if (p->it != 0) { set_err("autotuning runs on a problem that has not stepped yet (step 0)"); return CGFD_ERR_INVALID; }
  return guarded([&] {
    CK(cudaSetDevice(p->device));
    const int nbulk = p->nbulk;
    std::vector<int> zc;
    for (int c : {8, 10, 12, 14, 16, 20, 24, 32, 48, 64, 96, nbulk})
      if (c >= 1 && c <= nbulk && std::find(zc.begin(), zc.end(), c) == zc.end()) zc.push_back(c);
    // (tile shape, z chunk), the shapes interleaved so that a clock drifting during the tuning
    // (power cap, temperature) does not favour one of them; the FP64 build has no TMA kernel
    std::vector<std::pair<int, int>> cand;
    for (int c : zc)
      for (int sh = 0; sh < (p->use_tma ? 2 : 1); sh++) cand.emplace_back(sh, c);
    const std::pair<int, int> dflt(p->shape, p->nzc);
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    int best = p->nzc, best_shape = p->shape;
    float best_ms = 1e30f;
    const bool timing = p->timing;
    p->timing = false;
    // graph-replayed steps of the current choice, after the 8 captures
    auto time_choice = [&]() {
      for (int s = 0; s < 8; s++)
        if (p->graph_ok[s]) { cudaGraphExecDestroy(p->graph[s]); p->graph_ok[s] = false; }
      p->run_steps(8);
      CK(cudaEventRecord(e0, p->stream));
      p->run_steps(steps);
      CK(cudaEventRecord(e1, p->stream));
      CK(cudaEventSynchronize(e1));
      float ms = 0.f;
      CK(cudaEventElapsedTime(&ms, e0, e1));
      return ms;
    };
    auto use = [&](const std::pair<int, int> &sc) {
      CK(cudaStreamSynchronize(p->stream));
      if (p->use_tma && sc.first != p->shape) {
        p->shape = sc.first;
        make_maps(p);
      }
      p->nzc = sc.second;
      make_tiles(p);
    };
    // every candidate once; then the three fastest and the default tiling again, twice each
    // over twice the steps in a palindromic order (a b c d d c b a: a clock drifting linearly
    // during the tuning adds the same to every finalist), keeping the lowest mean (close
    // candidates differ by less than a short run's spread)
    std::vector<std::pair<float, std::pair<int, int>>> timed;
    for (const auto &sc : cand) {
      use(sc);
      timed.emplace_back(time_choice(), sc);
    }
    std::stable_sort(timed.begin(), timed.end(),
                     [](const auto &a, const auto &b) { return a.first < b.first; });
    std::vector<std::pair<int, int>> fin;
    for (size_t r = 0; r < std::min<size_t>(3, timed.size()); r++) fin.push_back(timed[r].second);
    if (std::find(fin.begin(), fin.end(), dflt) == fin.end()) fin.push_back(dflt);
    std::vector<float> sum(fin.size(), 0.f);
    const int steps1 = steps;
    steps = 2 * steps1;
    for (int pass = 0; pass < 2; pass++)
      for (size_t r = 0; r < fin.size(); r++) {
        const size_t q = pass ? fin.size() - 1 - r : r;
        use(fin[q]);
        sum[q] += time_choice();
      }
    steps = steps1;
    for (size_t q = 0; q < fin.size(); q++)
      if (sum[q] < best_ms) { best_ms = sum[q]; best = fin[q].second; best_shape = fin[q].first; }
    CK(cudaStreamSynchronize(p->stream));
    if (p->use_tma && best_shape != p->shape) {
      p->shape = best_shape;
      make_maps(p);
    }
    p->nzc = best;
    make_tiles(p);
    // batches: the shot group at the chosen tiling (4, 8, 16 or every shot)
    if (p->use_tma && p->nshot > 1) {
      int best_g = std::max(1, std::min(p->shot_group, p->nshot));
      float best_gms = 1e30f;
      std::vector<int> gc;
      for (int g : {4, 8, 16, p->nshot})
        if (g <= p->nshot && std::find(gc.begin(), gc.end(), g) == gc.end()) gc.push_back(g);
      for (int g : gc) {
        CK(cudaStreamSynchronize(p->stream));
        p->shot_group = g;
        make_tiles(p);
        const float ms = time_choice();
        if (ms < best_gms) { best_gms = ms; best_g = g; }
      }
      CK(cudaStreamSynchronize(p->stream));
      p->shot_group = best_g;
      make_tiles(p);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    p->timing = timing;
    for (int s = 0; s < 8; s++)
      if (p->graph_ok[s]) { cudaGraphExecDestroy(p->graph[s]); p->graph_ok[s] = false; }
    reset_state(p);
    if (chosen) *chosen = best;
  });
}

/* Bulk kernel variant: 1 = TMA-pipelined (default), 0 = direct loads. */
int cgfd_set_bulk_variant(cgfd_problem *p, int tma) {
  if (!p) return CGFD_ERR_INVALID;
  if (!tma && p->nshot > 1 && p->med != cgfd::MED_AC) {
    set_err("the direct-load bulk kernel handles one shot");
    return CGFD_ERR_UNSUPPORTED;
  }
  if (tma && p->fp64) {
    set_err("the FP64 build runs the direct-load bulk kernel");
    return CGFD_ERR_UNSUPPORTED;
  }
  if (tma && p->vis) {
    set_err("visco-elastic media run the direct-load bulk kernel");
    return CGFD_ERR_UNSUPPORTED;
  }
  if (p->med == cgfd::MED_AC) {  // acoustic: the TMA-pipelined (1) or direct-load (0) stage kernel
    p->ac_tma = tma != 0;
    for (int s = 0; s < 8; s++)
      if (p->graph_ok[s]) { cudaGraphExecDestroy(p->graph[s]); p->graph_ok[s] = false; }
    return CGFD_OK;
  }
  if (!tma && p->precision != CGFD_PREC_FP32 && !p->fp64) {
    set_err("the direct-load bulk kernel handles FP32 storage only");
    return CGFD_ERR_UNSUPPORTED;
  }
  p->use_tma = tma != 0;
  for (int s = 0; s < 8; s++)
    if (p->graph_ok[s]) { cudaGraphExecDestroy(p->graph[s]); p->graph_ok[s] = false; }
  return CGFD_OK;
}

/* Per-kernel CUDA-event timing of subsequent steps (forces direct launches while on). */
int cgfd_set_timing(cgfd_problem *p, int on) {
  if (!p) return CGFD_ERR_INVALID;
  p->timing = on != 0;
  return CGFD_OK;
}

int cgfd_get_timing(cgfd_problem *p, double *ms, long long *count, long long *launches, int reset) {
  if (!p) return CGFD_ERR_INVALID;
  for (int k = 0; k < 8; k++) {
    if (ms) ms[k] = p->t_ms[k];
    if (count) count[k] = p->t_n[k];
  }
  if (launches) *launches = p->launches;
  if (reset) {
    for (int k = 0; k < 8; k++) { p->t_ms[k] = 0; p->t_n[k] = 0; }
    p->launches = 0;
  }
  return CGFD_OK;
}

}  // extern "C"

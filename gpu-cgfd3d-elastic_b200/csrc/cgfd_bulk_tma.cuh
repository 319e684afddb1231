// cgfd_bulk_tma.cuh -- TMA-pipelined bulk RK-stage kernel for sm_100a (template; instantiated
// per medium by cgfd_bulk_tma_{iso,vti,aniso}.cu, dispatched by cgfd_bulk_tma.cu).
//
// Each thread block owns a 32 x TYT column tile and marches along z through its chunk of
// planes. Thread 0 streams, two planes ahead of the computation and with mbarrier
// completion:
//   - the stage input of one plane with its x-y halo, all 9 fields, as ONE 4-D TMA box
//     (40 x (TYT+4) x 1 x 9) into a 3-slot ring (plane k for the x/y operators, plane k+-1
//     for the z look-ahead, one in flight). The one-sided y operator of the stage reads one
//     row on one side and three on the other, so the box holds rows [-1, TYT+3) for forward
//     and [-3, TYT+1) for backward y operators; the x halo is 16 bytes on both sides (TMA
//     alignment);
//   - the coefficients (metrics, 1/rho, moduli) and, when the stage needs them, w_end and
//     (at one block per SM) w_pre of the same plane (centre boxes) into a 2-slot ring; with
//     two blocks per SM w_pre is read directly by each thread.
// The z march runs upwards for backward z operators and downwards for forward ones, so the
// one-sided operator always needs exactly one plane ahead; the current plane and the one
// ahead are read from the ring, the 3 planes behind live in a per-thread register queue.
// No thread computes an address for a stencil or coefficient load.
#pragma once

#include "cgfd_dev.cuh"
#include "cgfd_launch.h"
#include "cgfd_tma.cuh"

namespace cgfd {

// Wave policies: stage input / next-stage output storage.
//   WP 0: FP32 in, FP32 out (plain)      WP 1: FP32 in, FP16 out (stage 0 of FP16 mode)
//   WP 2: FP16 in, FP16 out (stages 1-3 of FP16 mode; stage 3 has no stage output)
template <int WP> struct WavePolicy {
  using TW = typename std::conditional<WP == 2, __half, float>::type;
  using TT = typename std::conditional<WP >= 1, __half, float>::type;
};

// Tile shapes (columns x rows of one thread block, resident blocks per SM), two per medium; the
// autotuner (cgfd_autotune) picks one per problem (default: shape 1 for iso, 0 otherwise):
//   iso, VTI: 32x8 at two blocks per SM (two independent barrier domains hide each other's
//             pipeline waits; <= 128 registers), or 32x4 at three blocks per SM;
//   21-Cij:   32x4 at three blocks per SM (its 31 coefficient fields do not fit twice at 32x8),
//             or 32x8 at one block per SM with w_pre staged by TMA as well.
template <int MED, int SHAPE> struct TileShape;
template <> struct TileShape<MED_ISO, 0> { static constexpr int TYT = 8, MINB = 2; };
template <> struct TileShape<MED_ISO, 1> { static constexpr int TYT = 4, MINB = 3; };
template <> struct TileShape<MED_VTI, 0> { static constexpr int TYT = 8, MINB = 2; };
template <> struct TileShape<MED_VTI, 1> { static constexpr int TYT = 4, MINB = 3; };
template <> struct TileShape<MED_ANISO, 0> { static constexpr int TYT = 4, MINB = 3; };
template <> struct TileShape<MED_ANISO, 1> { static constexpr int TYT = 8, MINB = 1; };

template <int MED, int TYT, typename TC, typename TW, int MINB>
struct BulkSmem {
  static constexpr int XO = 16 / (int)sizeof(TW);  // x halo of the box: 16 bytes, TMA-aligned
  static constexpr int WX = TX + 2 * XO;  // x box [-XO, 32+XO) around the tile
  static constexpr int WY = TYT + 4;      // y box [-1, TYT+3) (forward) or [-3, TYT+1) (backward)
  static constexpr int NC = MedInfo<MED>::NCOEF;
  static constexpr int CELLS = TX * TYT;
  static constexpr int WAVE_ELEMS = 9 * WY * WX;
  static constexpr int WAVE_SLOT = ((WAVE_ELEMS * (int)sizeof(TW) + 127) / 128) * 128;  // bytes
  static constexpr int COEF_BYTES = NC * CELLS * (int)sizeof(TC);  // multiple of 128 for every medium
  static constexpr int FLD_BYTES = 9 * CELLS * 4;
  // w_pre staged by TMA at one block per SM; with two blocks per SM it is read directly
  // (measured faster on 480x480x240: the smaller ring leaves the SM more L1)
  static constexpr bool PT = MINB == 1;
  static constexpr int OFF_END = COEF_BYTES + (PT ? FLD_BYTES : 0);  // within a cpe slot
  static constexpr int CPE_SLOT = OFF_END + FLD_BYTES;
  static constexpr int NW = 3;  // wave ring slots: this plane, the one ahead, one in flight
  static constexpr int OFF_CPE = NW * WAVE_SLOT;
  static constexpr int OFF_BAR = OFF_CPE + 2 * CPE_SLOT;
  static constexpr int BYTES = OFF_BAR + 8 * 8;
  static_assert(NW + 2 <= 8, "mbarrier area");
  static_assert(COEF_BYTES % 128 == 0, "w_pre/w_end boxes must stay 128-byte aligned");
  static_assert(MINB == 1 || MINB * (BYTES + 1024) <= 228 * 1024, "MINB blocks must fit one SM's shared memory");
};

// one cell's coefficients from a shared-memory tile (stride = cells per tile)
template <typename TC, int STRIDE>
struct CoefTile {
  const TC *c;  // field 0 of this cell
  const StageP &p;
  __device__ __forceinline__ float operator()(int f) const { return coef_decode<TC>(c[f * STRIDE], p, f); }
};

// One tile (a block) of the stage; PML false: the tile meets no CFS-PML face and the face code
// is compiled out.
template <int MED, int DX, int DY, int DZ, int TYT, int MINB, typename TC, int WP, bool PML>
__device__ __forceinline__ void bulk_tile(const StageP &p, const TmaP &tm, const int4 tl) {
  using TW = typename WavePolicy<WP>::TW;
  using TT = typename WavePolicy<WP>::TT;
  using S = BulkSmem<MED, TYT, TC, TW, MINB>;
  constexpr int LX = op_left(DX), LY = op_left(DY);
  constexpr int SD = DZ ? -1 : 1;  // march direction
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ float s_wsc[18];  // FP16 stage levels: scale, inverse scale
  TW *wave = reinterpret_cast<TW *>(smem);
  unsigned char *cpe = smem + S::OFF_CPE;
  uint64_t *bar = reinterpret_cast<uint64_t *>(smem + S::OFF_BAR);  // NW wave, then 2 cpe

  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
  const int bx = tl.x & kTileBxMask, by = tl.y, shot = tl.x >> 16;
  const int i = bx * TX + tx, j = by * TYT + ty;
  const int kb = tl.z, ke = tl.w;
  if (kb >= ke) return;
  const int n = ke - kb;
  const bool act = i < p.ni && j < p.nj;
  const int k0 = SD > 0 ? kb : ke - 1;
  const long long sf = p.sf;
  const long long woff = (long long)shot * 9 * sf;
  const TW *__restrict__ cur = reinterpret_cast<const TW *>(p.cur) + woff;
  TT *__restrict__ tmp_out = reinterpret_cast<TT *>(p.tmp_out) + woff;
  float *__restrict__ endw = p.end + woff;
  const int stage = p.stage;
  const bool need_pre = stage == 1 || stage == 2;
  const bool need_end = stage >= 1;
  const uint32_t wave_bytes = S::WAVE_ELEMS * sizeof(TW);
  const uint32_t cpe_bytes = S::COEF_BYTES + (need_pre && S::PT ? S::FLD_BYTES : 0) + (need_end ? S::FLD_BYTES : 0);
  // box origins (x * element size a multiple of 16 bytes): the stage-input map counts physical
  // cells from (0, 0, 0), so the halo beyond the grid is zero fill; the centre-box maps count
  // device-layout (padded) coordinates
  const int xw = bx * TX - S::XO, yw = by * TYT - LY;  // box row r = tile row r - LY
  const int xc = GX + bx * TX, yc = 3 + by * TYT;

  if (tid == 0) {
    for (int b = 0; b < S::NW + 2; b++) mbar_init(&bar[b], 1);
    fence_barrier_init();
  }
  if constexpr (WP != 0) {
    if (tid < 18) s_wsc[tid] = p.wsc[shot * 18 + tid];  // this shot's scale
  }
  __syncthreads();

  auto issue_wave = [&](int m) {
    const int kk = k0 + m * SD;
    uint64_t *b = &bar[m % S::NW];
    mbar_expect_tx(b, wave_bytes);
    tma_load_4d(wave + (m % S::NW) * (S::WAVE_SLOT / (int)sizeof(TW)), &tm.cur, xw, yw, kk, 9 * shot, b);
  };
  auto issue_cpe = [&](int m) {
    const int kk = k0 + m * SD;
    const int sl = m & 1;
    uint64_t *b = &bar[S::NW + sl];
    unsigned char *base = cpe + sl * S::CPE_SLOT;
    mbar_expect_tx(b, cpe_bytes);
    tma_load_4d(base, &tm.coef, xc, yc, kk + 3, 0, b);
    if (S::PT && need_pre) tma_load_4d(base + S::COEF_BYTES, &tm.pre, xc, yc, kk + 3, 9 * shot, b);
    if (need_end) tma_load_4d(base + S::OFF_END, &tm.end, xc, yc, kk + 3, 9 * shot, b);
  };
  if (tid == 0) {
    for (int m = 0; m + 1 < S::NW && m <= n; m++) issue_wave(m);  // planes 0..n exist
    issue_cpe(0);
  }

  // PML faces that intersect this block (uniform)
  unsigned fmask = 0;
  for (int fi = 0; PML && fi < p.nface; fi++) {
    const FaceP &f = p.face[fi];
    const bool xo = f.lo[0] <= bx * TX + TX - 1 && f.hi[0] >= bx * TX;
    const bool yo = f.lo[1] <= by * TYT + TYT - 1 && f.hi[1] >= by * TYT;
    const bool zo = f.lo[2] <= ke - 1 && f.hi[2] >= kb;
    if (xo && yo && zo) fmask |= 1u << fi;
  }

  // register queue of the planes behind, in march order: q[f][n] = plane k + (n - 3) * SD
  float q[9][3];
#pragma unroll
  for (int f = 0; f < 9; f++)
#pragma unroll
    for (int m = 0; m < 3; m++) q[f][m] = 0.f;
  if (act) {
#pragma unroll
    for (int m = 0; m < 3; m++) {
      const long long id = didx(p, i, j, k0 + (m - 3) * SD);
#pragma unroll
      for (int f = 0; f < 9; f++) q[f][m] = to_f(__ldg(cur + f * sf + id));
    }
  }
  const int wc = (ty + LY) * S::WX + tx + S::XO;  // centre of this thread in a wave slot (per field)
  mbar_wait(&bar[0], 0, p.err);
  float vmax = 0.f, smax = 0.f;  // FP16 mode, stage 3: max |w_end| of this thread
  bool bad = false;              // stage 3: a new solution value is NaN/Inf

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
    const TW *W = wave + ws * (S::WAVE_SLOT / (int)sizeof(TW));
    const TW *Wn = wave + wn * (S::WAVE_SLOT / (int)sizeof(TW));

    if (act) {
      const CoefTile<TC, S::CELLS> Cc{reinterpret_cast<const TC *>(cpe + cs * S::CPE_SLOT) + cell, p};
      float mt[3][3];
#pragma unroll
      for (int a = 0; a < 3; a++)
#pragma unroll
        for (int b = 0; b < 3; b++) mt[a][b] = Cc(3 * a + b);
      const float slw = Cc(CF_SLW);
      Medium<MED> md;
      md.load(Cc);
      // the 9 derivatives of the stage input along one axis at this cell
      auto deriv_x = [&](float d[9]) {
#pragma unroll
        for (int f = 0; f < 9; f++) {
          const TW *r = W + f * S::WY * S::WX + (ty + LY) * S::WX + tx + S::XO - LX;
          d[f] = drp5<DX>(to_f(r[0]), to_f(r[1]), to_f(r[2]), to_f(r[3]), to_f(r[4]));
          if constexpr (WP == 2) d[f] *= s_wsc[f];  // the operator is linear: scale once
        }
      };
      auto deriv_y = [&](float d[9]) {
#pragma unroll
        for (int f = 0; f < 9; f++) {
          const TW *r = W + f * S::WY * S::WX + ty * S::WX + tx + S::XO;
          d[f] = drp5<DY>(to_f(r[0]), to_f(r[S::WX]), to_f(r[2 * S::WX]), to_f(r[3 * S::WX]), to_f(r[4 * S::WX]));
          if constexpr (WP == 2) d[f] *= s_wsc[f];
        }
      };
      auto deriv_z = [&](float d[9]) {  // queue, this plane and the one ahead, in increasing k
#pragma unroll
        for (int f = 0; f < 9; f++) {
          const float c0 = to_f(W[f * S::WY * S::WX + wc]), c1 = to_f(Wn[f * S::WY * S::WX + wc]);
          d[f] = SD > 0 ? drp5<DZ>(q[f][0], q[f][1], q[f][2], c0, c1) : drp5<DZ>(c1, c0, q[f][2], q[f][1], q[f][0]);
          if constexpr (WP == 2) d[f] *= s_wsc[f];
        }
      };
      CellAcc acc;
      acc.zero();
      {
        float d[9];
        deriv_x(d);
        acc.add_axis(mt[0], d, d + 3);
        deriv_y(d);
        acc.add_axis(mt[1], d, d + 3);
        deriv_z(d);
        acc.add_axis(mt[2], d, d + 3);
      }
      float h[9];
      h[0] = slw * acc.mom[0];
      h[1] = slw * acc.mom[1];
      h[2] = slw * acc.mom[2];
      md.hooke(acc.G, h + 3);
      if constexpr (PML) {
        // CFS-PML corrections added to the full right-hand side face by face, in face order
        // (x1 x2 y1 y2 z1), as the reference applies its face kernels after the inner one;
        // the face axis' derivatives are recomputed here, when the accumulators above are
        // dead, to keep the face code's registers free
        if (fmask)
          for (int fi = 0; fi < p.nface; fi++) {
            const FaceP &fc = p.face[fi];
            if (!(fmask >> fi & 1) || !in_face(fc, i, j, k)) continue;
            float d[9];
            if (fc.axis == 0) {
              deriv_x(d);
              pml_face<MED>(p, fc, i, j, k, md, slw, mt[0], d, d + 3, nullptr, nullptr, h, shot);
            } else if (fc.axis == 1) {
              deriv_y(d);
              pml_face<MED>(p, fc, i, j, k, md, slw, mt[1], d, d + 3, nullptr, nullptr, h, shot);
            } else {
              deriv_z(d);
              pml_face<MED>(p, fc, i, j, k, md, slw, mt[2], d, d + 3, nullptr, nullptr, h, shot);
            }
          }
      }
      // RK combine (wav_update / wav_update_end)
      const long long id = didx(p, i, j, k);
      const float *PR = reinterpret_cast<const float *>(cpe + cs * S::CPE_SLOT + S::COEF_BYTES) + cell;
      const float *EN = reinterpret_cast<const float *>(cpe + cs * S::CPE_SLOT + S::OFF_END) + cell;
      const float *prg = p.pre + woff + id;  // w_pre in HBM when it is not staged
      const float ca = p.ca, cb = p.cb;
      if (stage == 0) {
#pragma unroll
        for (int f = 0; f < 9; f++) {
          const float c0 = to_f(W[f * S::WY * S::WX + wc]);  // stage input = w_pre at stage 0
          const float t = c0 + ca * h[f];
          tmp_out[f * sf + id] = from_f<TT>(WP != 0 ? t * s_wsc[9 + f] : t);
          endw[f * sf + id] = c0 + cb * h[f];
        }
      } else if (stage < 3) {
#pragma unroll
        for (int f = 0; f < 9; f++) {
          const float t = (S::PT ? PR[f * S::CELLS] : __ldg(prg + f * sf)) + ca * h[f];
          tmp_out[f * sf + id] = from_f<TT>(WP != 0 ? t * s_wsc[9 + f] : t);
          endw[f * sf + id] = EN[f * S::CELLS] + cb * h[f];
        }
      } else {
#pragma unroll
        for (int f = 0; f < 9; f++) {
          const float e = EN[f * S::CELLS] + cb * h[f];
          endw[f * sf + id] = e;
          bad |= nonfinite(e);
          if constexpr (WP == 2) {
            if (f < 3) vmax = fmaxf(vmax, fabsf(e));
            else smax = fmaxf(smax, fabsf(e));
          }
        }
      }
    }
#pragma unroll
    for (int f = 0; f < 9; f++) {
      q[f][0] = q[f][1];
      q[f][1] = q[f][2];
      q[f][2] = to_f(W[f * S::WY * S::WX + wc]);
    }
    // the slots read in this plane are refilled by TMA after the barrier: every read of them
    // (the queue load above may still be in flight) must be ordered before those writes
    fence_proxy_async_smem();
    __syncthreads();
  }
  if (bad) atomicOr(p.err, kErrWaveNonfinite);  // blow-up sentinel (drv_rk_curv_col.cu:507-510)
  if constexpr (WP == 2) {
    if (stage == 3) {  // the next step's FP16 scale
      for (int o = 16; o; o >>= 1) {
        vmax = fmaxf(vmax, __shfl_xor_sync(0xffffffffu, vmax, o));
        smax = fmaxf(smax, __shfl_xor_sync(0xffffffffu, smax, o));
      }
      if (tx == 0) {
        atomic_max_abs(&p.amax[2 * shot + 0], vmax);
        atomic_max_abs(&p.amax[2 * shot + 1], smax);
      }
    }
  }
}


// The bulk stage: one block per tile-list entry, in list order. An entry is (bx + PML flag
// (kTilePml) + (shot << 16), by, first plane, end plane); a PML tile runs the face code, the
// others its compiled-out form. Both kinds in one launch keep a tile's x-y neighbours, PML or
// not, resident beside it, so that the halo lines they share are read from DRAM once.
template <int MED, int DX, int DY, int DZ, int TYT, int MINB, typename TC, int WP>
__global__ void __launch_bounds__(TX *TYT, MINB)
    k_stage_bulk_tma(const __grid_constant__ StageP p, const __grid_constant__ TmaP tm,
                     const int4 *__restrict__ tiles) {
  const int4 tl = __ldg(tiles + blockIdx.x);
  if (tl.x & kTilePml) bulk_tile<MED, DX, DY, DZ, TYT, MINB, TC, WP, true>(p, tm, tl);
  else bulk_tile<MED, DX, DY, DZ, TYT, MINB, TC, WP, false>(p, tm, tl);
}

// -----------------------------------------------------------------------------------------
template <int MED, int SH, typename TC, int WP>
static int launch_tma_shape(const StageP &p, const TmaP &tm, const BulkTiles &t, cudaStream_t st) {
  constexpr int TYT = TileShape<MED, SH>::TYT, MINB = TileShape<MED, SH>::MINB;
  using S = BulkSmem<MED, TYT, TC, typename WavePolicy<WP>::TW, MINB>;
  if (t.n <= 0) return 0;
  const int code = p.dir[0] | (p.dir[1] << 1) | (p.dir[2] << 2);
  dim3 block(TX, TYT);
  dim3 grid(t.n);
  switch (code) {
#define CASE(c)                                                                                              \
  case c:                                                                                                    \
    k_stage_bulk_tma<MED, (c)&1, ((c) >> 1) & 1, ((c) >> 2) & 1, TYT, MINB, TC, WP>                          \
        <<<grid, block, S::BYTES, st>>>(p, tm, t.list);                                                      \
    break;
    CASE(0) CASE(1) CASE(2) CASE(3) CASE(4) CASE(5) CASE(6) CASE(7)
#undef CASE
  }
  return 1;
}

template <int MED, int SH, typename TC, int WP>
static cudaError_t set_attr_shape() {
  constexpr int TYT = TileShape<MED, SH>::TYT, MINB = TileShape<MED, SH>::MINB;
  using S = BulkSmem<MED, TYT, TC, typename WavePolicy<WP>::TW, MINB>;
  cudaError_t e = cudaSuccess;
#define ATTR(c)                                                                                               \
  if (e == cudaSuccess)                                                                                       \
    e = cudaFuncSetAttribute(k_stage_bulk_tma<MED, (c)&1, ((c) >> 1) & 1, ((c) >> 2) & 1, TYT, MINB, TC, WP>,     \
                             cudaFuncAttributeMaxDynamicSharedMemorySize, S::BYTES);
  ATTR(0) ATTR(1) ATTR(2) ATTR(3) ATTR(4) ATTR(5) ATTR(6) ATTR(7)
#undef ATTR
  return e;
}

template <int MED, typename TC, int WP>
static int launch_tc(int shape, const StageP &p, const TmaP &tm, const BulkTiles &t, cudaStream_t st) {
  return shape ? launch_tma_shape<MED, 1, TC, WP>(p, tm, t, st) : launch_tma_shape<MED, 0, TC, WP>(p, tm, t, st);
}

template <int MED, typename TC, int WP>
static cudaError_t prepare_tc(int shape) {
  return shape ? set_attr_shape<MED, 1, TC, WP>() : set_attr_shape<MED, 0, TC, WP>();
}

// One medium: every coefficient storage type and wave policy, both tile shapes.
template <int MED>
int launch_bulk_tma_med(int coef_type, int wave16, int shape, const StageP &p, const TmaP &tm, const BulkTiles &t,
                        cudaStream_t st) {
  if (wave16) {  // 16-bit fixed-point coefficients with FP16 stage levels
    if (p.stage == 0) return launch_tc<MED, uint16_t, 1>(shape, p, tm, t, st);
    return launch_tc<MED, uint16_t, 2>(shape, p, tm, t, st);
  }
  if (coef_type == COEF_U16) return launch_tc<MED, uint16_t, 0>(shape, p, tm, t, st);
  if (coef_type == COEF_F16) return launch_tc<MED, __half, 0>(shape, p, tm, t, st);
  if (coef_type == COEF_BF16) return launch_tc<MED, __nv_bfloat16, 0>(shape, p, tm, t, st);
  return launch_tc<MED, float, 0>(shape, p, tm, t, st);
}

template <int MED>
cudaError_t prepare_bulk_tma_med(int coef_type, int wave16, int shape) {
  if (wave16) {
    if (coef_type != COEF_U16) return cudaErrorInvalidValue;
    cudaError_t e = prepare_tc<MED, uint16_t, 1>(shape);
    return e == cudaSuccess ? prepare_tc<MED, uint16_t, 2>(shape) : e;
  }
  if (coef_type == COEF_U16) return prepare_tc<MED, uint16_t, 0>(shape);
  if (coef_type == COEF_F16) return prepare_tc<MED, __half, 0>(shape);
  if (coef_type == COEF_BF16) return prepare_tc<MED, __nv_bfloat16, 0>(shape);
  return prepare_tc<MED, float, 0>(shape);
}

}  // namespace cgfd

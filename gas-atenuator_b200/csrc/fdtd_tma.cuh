// fdtd_tma.cuh - the field sub-cycle of the resident simulation (fdtd_ratio 1):
// one warp per patch, the patch staged by TMA, the sub-cycle in registers.
//
// One launch advances the fields by one particle step: H(dt/4), E(dt/2),
// H(dt/2), E(dt/2), H(dt/4) (EM3_1.cu:2-17 and EM3.cu:2-43, called as the
// sub-cycle of electricmagneticfield6.m:146-151), with the same arithmetic as
// the reference-layout kernels of fdtd.cuh.
//
// Work: the grid (n_r + 1 columns x n_z + 1 rows of Yee points) is cut into
// tiles of 26 columns x (R - 6) rows.  A warp owns a patch of 32 columns x R
// rows around its tile (3 halo columns and rows on each side: the five
// sub-updates need two on the low side and three on the high side, and one
// more on the low side lets the warp assemble every gather quad of its tile
// from values it computed).  Lane l holds column l of the patch - Er, Ez, H
// and the two current terms of all R rows - in registers: vertical
// neighbours are registers, horizontal ones are warp shuffles, so the warps
// never wait on one another (no block barrier) and the halo is recomputed by
// each warp instead of exchanged.
//
// Staging: one lane of each warp issues five 2D tensor copies (Er, Ez, H as
// stored, Jr, Jz as 64-bit fixed point) of its patch into the warp's own
// staging area, completing on the warp's mbarrier.  Once the lanes hold the
// patch in registers the area is free, and the copies of the warp's next
// patch go out before the current one is computed.  Warps walk the work items
// warp-stride.  The tiles are written to a second set of fields: a patch
// staged after its neighbours' tiles were written still reads the old fields
// in its halo.
//
// TMA copies want 16-byte aligned starting columns: each box starts at the
// patch's first column rounded down to a 16-byte boundary and is wide enough
// (36 floats, 34 doubles or 64-bit counters) to cover the 32 patch columns
// from there; a lane reads its column at that offset.  Points outside the
// grid (negative or beyond the extent) arrive as zeros and are never updated.
//
// Every wait on an mbarrier is bounded; a warp whose copy has not completed
// after the bound sets the cell's *err, waits (bounded) once more for that
// copy and returns.
#pragma once
#include <cuda.h>
#include "fdtd.cuh"

namespace gasatt {

constexpr int kTmaTileW = 26;                 // output columns per tile
constexpr int kTmaPatchW = 32;                // patch columns (one per lane)
constexpr int kTmaHalo = 3;                   // halo columns / rows on each side
constexpr int kTmaWarps = 1;                  // warps per block (each on its own patches)
constexpr unsigned kTmaWaitLimit = 1u << 22;  // try_wait rounds before giving up

// staging box widths (elements): 32 columns from an aligned start below the
// patch's first column
template <typename T> struct TmaBox { static constexpr int w = sizeof(T) == 4 ? 36 : 34; };

// ------------------------------------------------------------ PTX wrappers
__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("{\n\t.reg .b64 st;\n\t"
               "mbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n\t}" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}
// true once the phase with the given parity has completed; false after the bound
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity) {
  for (unsigned it = 0; it < kTmaWaitLimit; ++it) {
    uint32_t done;
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                 "selp.u32 %0, 1, 0, p;\n\t}"
                 : "=r"(done)
                 : "r"(smem_u32(bar)), "r"(parity)
                 : "memory");
    if (done) return true;
  }
  return false;
}
// 2D tiled tensor copy global -> shared (no multicast), completion on bar
__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map, int x, int y,
                                            uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3}], [%4];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
      : "memory");
}

// ------------------------------------------------------------ layout
// One warp's staging area for R patch rows (Er, Ez, H in T, Jr, Jz in 64 bits;
// each 128-byte aligned).  A block holds kTmaWarps areas, then one mbarrier
// per warp.
template <typename T, int R>
struct TmaStage {
  static constexpr size_t up(size_t b) { return (b + 127) & ~(size_t)127; }
  static constexpr size_t field_bytes = up((size_t)TmaBox<T>::w * R * sizeof(T));
  static constexpr size_t cur_bytes = up((size_t)34 * R * 8);
  static constexpr size_t bytes = 3 * field_bytes + 2 * cur_bytes;
  static constexpr size_t block_bytes = kTmaWarps * bytes + 128;
  // bytes one patch's five copies deliver (whole boxes, out-of-bounds fill included)
  static constexpr uint32_t tx_bytes =
      (uint32_t)(3 * (size_t)TmaBox<T>::w * R * sizeof(T) + 2 * (size_t)34 * R * 8);
};

struct TmaMaps {
  CUtensorMap er, ez, h, jr, jz;
};

// One gas cell's field update as the kernel sees it: its tensor maps (the
// field and current buffers read in this step), where the tile is written
// (the other field buffer in T, the other current buffer cleared, FP32 gather
// quads),
// the coefficients and its tile grid.  A single cell passes it as a kernel
// parameter; a batch keeps one per cell in global memory.
struct FdtdInst {
  TmaMaps maps;
  void *Er, *Ez, *H;
  unsigned long long *Jr_next, *Jz_next;
  // per column i in [0, n_r]: {1/V scaled from fixed point, coefficient of
  // H(i) and of H(i-1) in the Ez update} (FdtdColumn), precomputed on the host
  // with the expressions the kernels of fdtd.cuh evaluate per thread
  const double *colc;
  ExtraCurrent xj;
  FieldQuads q;
  FdtdCoef c;
  double chr4, chz4, chr2, chz2;   // H update factors h/(mu dr), h/(mu dz) for h = dt/4, dt/2
  int nr, nz, ldf, ldj;
  unsigned flags;
  int tiles_x, ntiles;
  unsigned *err;              // set when a tile copy of this cell did not complete
};

// Work of a launch: tile t of one cell, or entry t of a table of (cell, tile)
// pairs over the cells of a batch.
struct FdtdWork {
  const FdtdInst *inst;       // one cell, or the batch's cells
  const int2 *table;          // null for one cell; else (cell, tile) per work item
  int ntiles;                 // work items
  __device__ __forceinline__ const FdtdInst &at(int t, int &lt) const {
    if (!table) { lt = t; return *inst; }
    const int2 e = table[t];
    lt = e.y;
    return inst[e.x];
  }
};

// tile t of a tiles_x-wide row-major tile grid -> the patch origin (x0, y0)
__device__ __forceinline__ void tma_patch_origin(int t, int tiles_x, int rows, int &x0, int &y0) {
  const int ty = t / tiles_x, tx = t - ty * tiles_x;
  x0 = tx * kTmaTileW - kTmaHalo;
  y0 = ty * (rows - 2 * kTmaHalo) - kTmaHalo;
}

// issue the copies of work item t into a warp's staging area (one lane)
template <typename T, int R>
__device__ __forceinline__ void tma_issue_item(const FdtdWork &W, int t, unsigned char *stage,
                                               uint64_t *bar) {
  using S = TmaStage<T, R>;
  constexpr int al = 16 / (int)sizeof(T);
  int lt, x0, y0;
  const FdtdInst &I = W.at(t, lt);
  tma_patch_origin(lt, I.tiles_x, R, x0, y0);
  const int xf = x0 & ~(al - 1), xj = x0 & ~1;       // floor to a 16-byte column
  const TmaMaps &M = I.maps;
  mbar_expect_tx(bar, S::tx_bytes);
  tma_load_2d(stage, &M.er, xf, y0, bar);
  tma_load_2d(stage + S::field_bytes, &M.ez, xf, y0, bar);
  tma_load_2d(stage + 2 * S::field_bytes, &M.h, xf, y0, bar);
  tma_load_2d(stage + 3 * S::field_bytes, &M.jr, xj, y0, bar);
  tma_load_2d(stage + 3 * S::field_bytes + S::cur_bytes, &M.jz, xj, y0, bar);
}

// The sub-cycle on the work items of W (cells on the padded layout: row
// strides ldf for the fields, ldj for the currents), R patch rows per warp.
// The field arithmetic is that of fdtd_tiled (fdtd.cuh); the per-column
// coefficients come from the cell's table, the current terms of the two E
// updates are formed once per patch.
template <typename T, int R>
__device__ __forceinline__ void fdtd_warp_body(const FdtdWork &W) {
  using S = TmaStage<T, R>;
  static_assert(R > 2 * kTmaHalo && R <= 32, "patch rows");
  constexpr int BW = TmaBox<T>::w, al = 16 / (int)sizeof(T);
  constexpr unsigned FULL = 0xFFFFFFFFu;
  extern __shared__ __align__(128) unsigned char smem[];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  unsigned char *stage = smem + wib * S::bytes;
  uint64_t *bar = reinterpret_cast<uint64_t *>(smem + kTmaWarps * S::bytes) + wib;
  const int ntiles = W.ntiles, stride = gridDim.x * kTmaWarps;
  int t = blockIdx.x * kTmaWarps + wib;
  if (lane == 0) {
    mbar_init(bar, 1);
    mbar_fence_init();
  }
  __syncwarp();
  if (lane == 0 && t < ntiles) tma_issue_item<T, R>(W, t, stage, bar);
  for (int k = 0; t < ntiles; t += stride, ++k) {
    int lt, x0, y0;
    const FdtdInst &I = W.at(t, lt);
    tma_patch_origin(lt, I.tiles_x, R, x0, y0);
    const int nr = I.nr, nz = I.nz;
    const unsigned flags = I.flags;
    const bool endcopy = (flags & GASATT_Q_ER_END_COPY) != 0;
    const bool jsign = (flags & GASATT_Q_EZ_AXIS_JSIGN) != 0;
    const double dt_eps = I.c.dt_eps, dt_eps_dz = I.c.dt_eps_dz, axis = I.c.axis;
    const int col = x0 + lane;
    const int of = x0 - (x0 & ~(al - 1)), oj = x0 - (x0 & ~1);
    const bool colH = col >= 0 && col < nr;
    // Every point of the patch is updated by the same expression: no in-grid
    // update reads a point outside the grid (the boundary rules never reach
    // past the edge), so the values those points take do not matter.  The
    // rules that keep an in-grid point from the interior expression become
    // coefficients: Ez on the axis (col 0) takes (+J term, axis factor, 0),
    // Ez at col n_r and beyond is left as it is (0, 0, 0); Er rows 0 and n_z
    // are fixed up after each E update.  (Read while the copies are in flight.)
    double iv = 0.0, ezp = 0.0, ezm = 0.0;
    if (colH) {
      iv = I.colc[3 * col];
      ezp = col == 0 ? axis : I.colc[3 * col + 1];
      ezm = I.colc[3 * col + 2];            // 0 on the axis
    }
    const bool ok = __all_sync(FULL, mbar_wait(bar, (uint32_t)(k & 1)));
    if (!ok) {
      if (lane == 0) {
        atomicOr(I.err, 1u);
        mbar_wait(bar, (uint32_t)(k & 1));          // the copy still owns the area
      }
      break;
    }
    // the column's patch: fields, and the current terms of the E updates
    // (jr: dt/eps (J_r(j-1) + J_r(j)) / 2; jz: the same over columns i-1, i,
    // or on the axis minus the signed dt/eps J_z term)
    double er[R], ez[R], h[R], jr[R], jz[R];
    {
      const T *gEr = reinterpret_cast<const T *>(stage);
      const T *gEz = reinterpret_cast<const T *>(stage + S::field_bytes);
      const T *gH = reinterpret_cast<const T *>(stage + 2 * S::field_bytes);
      const long long *gJr = reinterpret_cast<const long long *>(stage + 3 * S::field_bytes);
      const long long *gJz = reinterpret_cast<const long long *>(stage + 3 * S::field_bytes + S::cur_bytes);
      const ExtraCurrent xj = I.xj;
      double below = 0.0;
      if (xj.Jr) {
#pragma unroll
        for (int r = 0; r < R; ++r) {
          const int sf = lane + of + r * BW, sj = lane + oj + r * 34, row = y0 + r;
          er[r] = (double)gEr[sf];
          ez[r] = (double)gEz[sf];
          h[r] = (double)gH[sf];
          double a = (double)gJr[sj], b = (double)gJz[sj];
          if (colH && row >= 0 && row < nz) {
            const int64_t g = col + (int64_t)row * I.ldj;
            a = a + (double)(long long)xj.Jr[g] * xj.rel;
            b = b + (double)(long long)xj.Jz[g] * xj.rel;
          }
          a = a * iv;
          b = b * iv;
          jr[r] = dt_eps * (below + a) / 2;
          below = a;
          jz[r] = b;
        }
      } else {
#pragma unroll
        for (int r = 0; r < R; ++r) {
          const int sf = lane + of + r * BW, sj = lane + oj + r * 34;
          er[r] = (double)gEr[sf];
          ez[r] = (double)gEz[sf];
          h[r] = (double)gH[sf];
          const double a = (double)gJr[sj] * iv;
          jr[r] = dt_eps * (below + a) / 2;
          below = a;
          jz[r] = (double)gJz[sj] * iv;
        }
      }
    }
    __syncwarp();
    // the area is free: the warp's next patch is fetched while this one is computed
    if (lane == 0 && t + stride < ntiles) {
      fence_proxy_async_smem();
      tma_issue_item<T, R>(W, t + stride, stage, bar);
    }
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const double left = __shfl_up_sync(FULL, jz[r], 1);
      const double jt = jsign ? dt_eps * jz[r] : -(dt_eps * jz[r]);
      jz[r] = col == 0 ? -jt : (colH ? dt_eps * (left + jz[r]) / 2 : 0.0);
    }
    // patch rows of grid rows 0 and n_z (Er there: zero, or the end copies)
    const int r0 = -y0, rn = nz - y0;
    const bool edge_rows = (r0 >= 0 && r0 < R) || (rn >= 0 && rn < R);
    auto h_update = [&](double chr, double chz) {
#pragma unroll
      for (int r = 0; r + 1 < R; ++r) {
        const double ezr = __shfl_down_sync(FULL, ez[r], 1);
        h[r] = h[r] + (chr * (ezr - ez[r]) - chz * (er[r + 1] - er[r]));
      }
    };
    auto e_update = [&]() {
      double ne[R];
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const int rm = r > 0 ? r - 1 : 0;
        const double hl = __shfl_up_sync(FULL, h[r], 1);
        ne[r] = er[r] - jr[r] - dt_eps_dz * (h[r] - h[rm]);
        ez[r] = ez[r] - jz[r] + ezp * h[r] + ezm * hl;
      }
      if (edge_rows) {
#pragma unroll
        for (int r = 0; r < R; ++r) {
          const int rm = r > 0 ? r - 1 : r, rp = r + 1 < R ? r + 1 : r;
          if (r == r0) ne[r] = endcopy ? er[rp] : 0.0;
          if (r == rn) ne[r] = endcopy ? er[rm] : 0.0;
        }
      }
#pragma unroll
      for (int r = 0; r < R; ++r) er[r] = ne[r];
    };
    h_update(I.chr4, I.chz4);
    e_update();
    h_update(I.chr2, I.chz2);
    e_update();
    h_update(I.chr4, I.chz4);
    // write back the tile: columns [3, 29) and rows [3, R - 3) of the patch
    T *Er = reinterpret_cast<T *>(I.Er), *Ez = reinterpret_cast<T *>(I.Ez), *H = reinterpret_cast<T *>(I.H);
    unsigned long long *Jr_next = I.Jr_next, *Jz_next = I.Jz_next;
    const int ldf = I.ldf, ldj = I.ldj;
    const bool out_col = lane >= kTmaHalo && lane < kTmaHalo + kTmaTileW && col <= nr;
    if (sizeof(T) == 4) {
      // FP32 form: the fields rounded to float once; whole gather quads (when
      // the cell has them) from those floats, corner columns from the lane
      // below by shuffle
      const FieldQuads q = I.q;
      float fe[R], fz[R], fh[R];
#pragma unroll
      for (int r = kTmaHalo - 1; r <= R - kTmaHalo; ++r) {
        fe[r] = (float)er[r];
        fz[r] = (float)ez[r];
        fh[r] = (float)h[r];
      }
      const bool lo0 = col > 0, hi0 = col > nr - 1;   // corner column c0 = col - 1, c1 = col - 1
#pragma unroll
      for (int r = kTmaHalo; r < R - kTmaHalo; ++r) {
        const int row = y0 + r;
        const float eu0 = __shfl_up_sync(FULL, fe[r], 1), eu1 = __shfl_up_sync(FULL, fe[r + 1], 1);
        const float zd0 = __shfl_down_sync(FULL, fz[r - 1], 1), zd1 = __shfl_down_sync(FULL, fz[r], 1);
        const float hu0 = __shfl_up_sync(FULL, fh[r - 1], 1), hu1 = __shfl_up_sync(FULL, fh[r], 1);
        if (!out_col || row > nz) continue;
        if (col < nr) reinterpret_cast<float *>(Er)[col + (int64_t)row * ldf] = fe[r];
        if (row < nz) reinterpret_cast<float *>(Ez)[col + (int64_t)row * ldf] = fz[r];
        if (col < nr && row < nz) {
          reinterpret_cast<float *>(H)[col + (int64_t)row * ldf] = fh[r];
          const int64_t g = col + (int64_t)row * ldj;
          Jr_next[g] = 0;
          Jz_next[g] = 0;
        }
        if (!q.er) continue;                                 // no gather quads in this cell
        const bool ra_lo = row > 0, rb_lo = row > nz - 1;   // quad rows ra = row - 1, rb = row - 1
        if (row < nz)
          q.er[col + (int64_t)row * (nr + 1)] =
              make_float4(lo0 ? eu0 : fe[r], hi0 ? eu0 : fe[r], lo0 ? eu1 : fe[r + 1], hi0 ? eu1 : fe[r + 1]);
        if (col < nr)
          q.ez[col + (int64_t)row * nr] =
              make_float4(ra_lo ? fz[r - 1] : fz[r], ra_lo ? zd0 : zd1, rb_lo ? fz[r - 1] : fz[r],
                          rb_lo ? zd0 : zd1);
        const float ha0 = ra_lo ? hu0 : hu1, ha = ra_lo ? fh[r - 1] : fh[r];
        const float hb0 = rb_lo ? hu0 : hu1, hb = rb_lo ? fh[r - 1] : fh[r];
        q.h[col + (int64_t)row * (nr + 1)] =
            make_float4(lo0 ? ha0 : ha, hi0 ? ha0 : ha, lo0 ? hb0 : hb, hi0 ? hb0 : hb);
      }
    } else if (out_col) {
#pragma unroll
      for (int r = kTmaHalo; r < R - kTmaHalo; ++r) {
        const int row = y0 + r;
        if (row > nz) continue;
        if (col < nr) Er[col + (int64_t)row * ldf] = (T)er[r];
        if (row < nz) Ez[col + (int64_t)row * ldf] = (T)ez[r];
        if (col < nr && row < nz) {
          H[col + (int64_t)row * ldf] = (T)h[r];
          const int64_t g = col + (int64_t)row * ldj;
          Jr_next[g] = 0;
          Jz_next[g] = 0;
        }
      }
    }
  }
}

// the per-column table of FdtdInst::colc for n_r columns: {1/V scaled, Ez
// coefficients of H(i) and H(i-1)} (the expressions fdtd_tiled evaluates)
inline void fdtd_column_table(int nr, const FdtdCoef &c, const double *invV, unsigned flags,
                              double *out) {
  const double inv_dr = 1 / c.dr;
  for (int i = 0; i < nr; ++i) {
    const double ri = ((flags & GASATT_Q_EZ_RSHIFT) ? (i + 1) : i) * c.dr;
    out[3 * i] = invV[i];
    out[3 * i + 1] = i > 0 ? c.dt_eps * (1 / (2 * ri) + inv_dr) : 0.0;
    out[3 * i + 2] = i > 0 ? c.dt_eps * (1 / (2 * ri) - inv_dr) : 0.0;
  }
}

}  // namespace gasatt

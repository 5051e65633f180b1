// fdtd_tma.cuh - the field sub-cycle of the resident simulation (fdtd_ratio 1)
// as a persistent kernel fed by TMA tile copies.
//
// One launch advances the fields by one particle step: H(dt/4), E(dt/2),
// H(dt/2), E(dt/2), H(dt/4) (EM3_1.cu:2-17 and EM3.cu:2-43, called as the
// sub-cycle of electricmagneticfield6.m:146-151), with the same arithmetic as
// the reference-layout kernels of fdtd.cuh.
//
// Work: the grid (n_r + 1 columns x n_z + 1 rows of Yee points) is cut into
// tiles of 26 columns x (PH - 6) rows.  A block owns a patch of 32 columns x
// PH rows around its tile (3 halo columns and rows on each side: the five
// sub-updates need two on the low side and three on the high side, and one
// more on the low side lets the block assemble every gather quad of its tile
// from values it computed).  Blocks are persistent and walk the tiles
// block-stride; for each tile one thread issues five 2D tensor copies (Er,
// Ez, H as stored, Jr, Jz as 64-bit fixed point) into a staging buffer in
// shared memory, completing on an mbarrier.  The copies of the next tile go
// out before the current one is computed (two staging buffers), so a block's
// loads overlap its arithmetic.  The staged values are widened into double
// working arrays (the current scaled by 1 / shell volume), the five
// sub-updates run there, and the tile is written back: the fields in their
// storage type, zeros into the other current buffer, and - FP32 form - the
// whole gather quads of the tile.
//
// TMA copies want 16-byte aligned starting columns: each box starts at the
// patch's first column rounded down to a 16-byte boundary and is wide enough
// (36 floats, 34 doubles or 64-bit counters) to cover the 32 patch columns
// from there; a thread reads its column at that offset.  Points outside the
// grid (negative or beyond the extent) arrive as zeros and are never updated.
//
// Every wait on an mbarrier is bounded; a block whose copy has not completed
// after the bound sets the cell's *err, waits (bounded) for its other copy in
// flight and returns.
#pragma once
#include <cuda.h>
#include "fdtd.cuh"

namespace gasatt {

constexpr int kTmaTileW = 26;                 // output columns per tile
constexpr int kTmaPatchW = 32;                // patch columns (one per lane)
constexpr int kTmaRows = 16;                  // blockDim = (32, kTmaRows)
constexpr int kTmaHalo = 3;                   // halo columns / rows on each side
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
// Byte offsets of the dynamic shared memory of k_fdtd_tma for PH patch rows:
// two staging buffers (Er, Ez, H in T, Jr, Jz in 64 bits; each 128-byte
// aligned), the double working arrays, two mbarriers.
template <typename T>
struct TmaSmem {
  int ph;
  __host__ __device__ explicit TmaSmem(int ph_) : ph(ph_) {}
  __host__ __device__ static size_t up(size_t b) { return (b + 127) & ~(size_t)127; }
  __host__ __device__ size_t field_bytes() const { return up((size_t)TmaBox<T>::w * ph * sizeof(T)); }
  __host__ __device__ size_t cur_bytes() const { return up((size_t)34 * ph * 8); }
  __host__ __device__ size_t stage_bytes() const { return 3 * field_bytes() + 2 * cur_bytes(); }
  __host__ __device__ size_t work_bytes() const { return (size_t)ph * kTmaPatchW * 8; }
  __host__ __device__ size_t work_off() const { return 2 * stage_bytes(); }
  __host__ __device__ size_t bar_off() const { return work_off() + 5 * work_bytes(); }
  __host__ __device__ size_t total() const { return bar_off() + 16; }
  // bytes one tile's five copies deliver (whole boxes, out-of-bounds fill included)
  __host__ __device__ uint32_t tx_bytes() const {
    return (uint32_t)(3 * (size_t)TmaBox<T>::w * ph * sizeof(T) + 2 * (size_t)34 * ph * 8);
  }
};

struct TmaMaps {
  CUtensorMap er, ez, h, jr, jz;
};

// One gas cell's field update as the kernel sees it: its tensor maps (the
// fields and the current buffer read in this step), where the tile is written
// back (fields in T, the other current buffer cleared, FP32 gather quads),
// the coefficients and its tile grid.  A single cell passes it as a kernel
// parameter; a batch keeps one per cell in global memory.
struct FdtdInst {
  TmaMaps maps;
  void *Er, *Ez, *H;
  unsigned long long *Jr_next, *Jz_next;
  const double *invV;
  ExtraCurrent xj;
  FieldQuads q;
  FdtdCoef c;
  double mu, dt;
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
__device__ __forceinline__ void tma_patch_origin(int t, int tiles_x, int ph, int &x0, int &y0) {
  const int ty = t / tiles_x, tx = t - ty * tiles_x;
  x0 = tx * kTmaTileW - kTmaHalo;
  y0 = ty * (ph - 2 * kTmaHalo) - kTmaHalo;
}

template <typename T>
__device__ __forceinline__ void tma_issue(const TmaMaps &M, unsigned char *stage, uint64_t *bar,
                                          const TmaSmem<T> &L, int x0, int y0) {
  constexpr int al = 16 / (int)sizeof(T);
  const int xf = x0 & ~(al - 1), xj = x0 & ~1;       // floor to a 16-byte column
  mbar_expect_tx(bar, L.tx_bytes());
  tma_load_2d(stage, &M.er, xf, y0, bar);
  tma_load_2d(stage + L.field_bytes(), &M.ez, xf, y0, bar);
  tma_load_2d(stage + 2 * L.field_bytes(), &M.h, xf, y0, bar);
  tma_load_2d(stage + 3 * L.field_bytes(), &M.jr, xj, y0, bar);
  tma_load_2d(stage + 3 * L.field_bytes() + L.cur_bytes(), &M.jz, xj, y0, bar);
}

// issue the copies of work item t (thread 0)
template <typename T>
__device__ __forceinline__ void tma_issue_item(const FdtdWork &W, int t, unsigned char *stage,
                                               uint64_t *bar, const TmaSmem<T> &L) {
  int lt, x0, y0;
  const FdtdInst &I = W.at(t, lt);
  tma_patch_origin(lt, I.tiles_x, L.ph, x0, y0);
  tma_issue<T>(I.maps, stage, bar, L, x0, y0);
}

// The sub-cycle on the work items of W (cells on the padded layout: row
// strides ldf for the fields, ldj for the currents).  The field arithmetic is
// that of fdtd_tiled1 (fdtd.cuh).
template <typename T>
__device__ __forceinline__ void fdtd_tma_body(const FdtdWork &W, int ph) {
  constexpr int PW = kTmaPatchW;
  constexpr int al = 16 / (int)sizeof(T);
  extern __shared__ __align__(1024) unsigned char smem[];
  const TmaSmem<T> L(ph);
  unsigned char *stage[2] = {smem, smem + L.stage_bytes()};
  double *sEr = reinterpret_cast<double *>(smem + L.work_off());
  double *sEz = sEr + ph * PW, *sH = sEz + ph * PW, *sJr = sH + ph * PW, *sJz = sJr + ph * PW;
  uint64_t *bar = reinterpret_cast<uint64_t *>(smem + L.bar_off());
  const int li = threadIdx.x, tid = threadIdx.y * PW + threadIdx.x;
  const int nrow_t = ph / kTmaRows;                  // patch rows per thread
  const int ntiles = W.ntiles;
  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    mbar_fence_init();
  }
  __syncthreads();
  int t = blockIdx.x;
  bool issued0 = false, issued1 = false;             // thread 0: a copy of buffer 0 / 1 in flight
  if (tid == 0 && t < ntiles) {
    tma_issue_item<T>(W, t, stage[0], &bar[0], L);
    issued0 = true;
  }
  for (int k = 0; t < ntiles; t += gridDim.x, ++k) {
    const int b = k & 1;
    // the next item's copies go out now, into the buffer the previous item
    // has finished with (every thread read it before the barriers below)
    if (tid == 0 && t + (int)gridDim.x < ntiles) {
      fence_proxy_async_smem();
      tma_issue_item<T>(W, t + gridDim.x, stage[b ^ 1], &bar[b ^ 1], L);
      if (b) issued0 = true; else issued1 = true;
    }
    const bool ok = mbar_wait(&bar[b], (uint32_t)((k >> 1) & 1));
    if (tid == 0 && ok) { if (b) issued1 = false; else issued0 = false; }
    if (__syncthreads_or(!ok)) {
      int lt;
      if (tid == 0) atomicOr(W.at(t, lt).err, 1u);
      break;
    }
    int lt, x0, y0;
    const FdtdInst &I = W.at(t, lt);
    tma_patch_origin(lt, I.tiles_x, ph, x0, y0);
    const int nr = I.nr, nz = I.nz;
    const FdtdCoef &c = I.c;
    const unsigned flags = I.flags;
    const bool endcopy = (flags & GASATT_Q_ER_END_COPY) != 0;
    const bool jsign = (flags & GASATT_Q_EZ_AXIS_JSIGN) != 0;
    const double dt_eps = c.dt_eps, dt_eps_dz = c.dt_eps_dz, axis = c.axis, inv_dr = 1 / c.dr;
    const double mu = I.mu, dt = I.dt;
    const int col = x0 + li;
    const int of = x0 - (x0 & ~(al - 1)), oj = x0 - (x0 & ~1);
    // widen the staged tile into the working arrays
    {
      const T *gEr = reinterpret_cast<const T *>(stage[b]);
      const T *gEz = reinterpret_cast<const T *>(stage[b] + L.field_bytes());
      const T *gH = reinterpret_cast<const T *>(stage[b] + 2 * L.field_bytes());
      const long long *gJr = reinterpret_cast<const long long *>(stage[b] + 3 * L.field_bytes());
      const long long *gJz =
          reinterpret_cast<const long long *>(stage[b] + 3 * L.field_bytes() + L.cur_bytes());
      const double iv = (col >= 0 && col < nr) ? I.invV[col] : 0.0;
      const ExtraCurrent xj = I.xj;
      for (int m = 0; m < nrow_t; ++m) {
        const int r = threadIdx.y + kTmaRows * m, s = li + r * PW;
        const int sf = li + of + r * TmaBox<T>::w, sj = li + oj + r * 34;
        sEr[s] = (double)gEr[sf];
        sEz[s] = (double)gEz[sf];
        sH[s] = (double)gH[sf];
        const int jrow = y0 + r;
        if (xj.Jr && col >= 0 && col < nr && jrow >= 0 && jrow < nz) {
          const int64_t g = col + (int64_t)jrow * I.ldj;
          sJr[s] = ((double)gJr[sj] + (double)(long long)xj.Jr[g] * xj.rel) * iv;
          sJz[s] = ((double)gJz[sj] + (double)(long long)xj.Jz[g] * xj.rel) * iv;
        } else {
          sJr[s] = (double)gJr[sj] * iv;
          sJz[s] = (double)gJz[sj] * iv;
        }
      }
    }
    // which updates each cell takes (the grid's boundary rules; the patch's
    // last column and row have no upper neighbours and are left alone)
    const double ri = ((flags & GASATT_Q_EZ_RSHIFT) ? (col + 1) : col) * c.dr;
    const double ezp = col > 0 ? dt_eps * (1 / (2 * ri) + inv_dr) : 0.0;   // coefficient of H(i)
    const double ezm = col > 0 ? dt_eps * (1 / (2 * ri) - inv_dr) : 0.0;   // coefficient of H(i-1)
    const bool colH = col >= 0 && col < nr;
    __syncthreads();
    auto h_update = [&](double h) {
      const double chr = h / (mu * c.dr), chz = h / (mu * c.dz);
      for (int m = 0; m < nrow_t; ++m) {
        const int r = threadIdx.y + kTmaRows * m, s = li + r * PW, row = y0 + r;
        if (colH && li + 1 < PW && row >= 0 && row < nz && r + 1 < ph)
          sH[s] = sH[s] + (chr * (sEz[s + 1] - sEz[s]) - chz * (sEr[s + PW] - sEr[s]));
      }
    };
    auto e_update = [&]() {
      for (int m = 0; m < nrow_t; ++m) {
        const int r = threadIdx.y + kTmaRows * m, s = li + r * PW, row = y0 + r;
        if (colH) {
          if (row >= 1 && row < nz) {
            if (r >= 1) {
              const double old = sEr[s];
              sEr[s] = old - dt_eps * (sJr[s - PW] + sJr[s]) / 2 - dt_eps_dz * (sH[s] - sH[s - PW]);
              if (endcopy) {
                if (row == 1) sEr[s - PW] = old;
                if (row == nz - 1 && r + 1 < ph) sEr[s + PW] = old;
              }
            }
          } else if (!endcopy && (row == 0 || row == nz)) {
            sEr[s] = 0.0;
          }
        }
        if (row >= 0 && row < nz) {
          if (col == 0) {
            const double jz0 = sJz[s];
            const double jterm = jsign ? dt_eps * jz0 : -(dt_eps * jz0);
            sEz[s] = sEz[s] + jterm + axis * sH[s];
          } else if (col > 0 && col < nr && li >= 1) {
            sEz[s] = sEz[s] - dt_eps * (sJz[s - 1] + sJz[s]) / 2 + ezp * sH[s] + ezm * sH[s - 1];
          }
        }
      }
    };
    h_update(dt / 4);
    __syncthreads();
    e_update();
    __syncthreads();
    h_update(dt / 2);
    __syncthreads();
    e_update();
    __syncthreads();
    h_update(dt / 4);
    __syncthreads();
    // write back the tile: columns [3, 29) and rows [3, ph - 3) of the patch
    T *Er = reinterpret_cast<T *>(I.Er), *Ez = reinterpret_cast<T *>(I.Ez), *H = reinterpret_cast<T *>(I.H);
    unsigned long long *Jr_next = I.Jr_next, *Jz_next = I.Jz_next;
    const int ldf = I.ldf, ldj = I.ldj;
    const FieldQuads q = I.q;
    if (li >= kTmaHalo && li < kTmaHalo + kTmaTileW && col <= nr) {
      const int c0 = col > 0 ? li - 1 : li, c1 = col > nr - 1 ? li - 1 : li;   // quad columns
      for (int m = 0; m < nrow_t; ++m) {
        const int r = threadIdx.y + kTmaRows * m, row = y0 + r;
        if (r < kTmaHalo || r >= ph - kTmaHalo || row > nz) continue;
        const int s = li + r * PW;
        if (col < nr) Er[col + (int64_t)row * ldf] = (T)sEr[s];
        if (row < nz) Ez[col + (int64_t)row * ldf] = (T)sEz[s];
        if (col < nr && row < nz) {
          H[col + (int64_t)row * ldf] = (T)sH[s];
          const int64_t g = col + (int64_t)row * ldj;
          Jr_next[g] = 0;
          Jz_next[g] = 0;
        }
        if (q.er) {
          const int ra = row > 0 ? r - 1 : r, rb = row > nz - 1 ? r - 1 : r;   // quad rows
          if (row < nz)
            q.er[col + (int64_t)row * (nr + 1)] =
                make_float4((float)sEr[c0 + r * PW], (float)sEr[c1 + r * PW],
                            (float)sEr[c0 + (r + 1) * PW], (float)sEr[c1 + (r + 1) * PW]);
          if (col < nr)
            q.ez[col + (int64_t)row * nr] =
                make_float4((float)sEz[li + ra * PW], (float)sEz[li + 1 + ra * PW],
                            (float)sEz[li + rb * PW], (float)sEz[li + 1 + rb * PW]);
          q.h[col + (int64_t)row * (nr + 1)] =
              make_float4((float)sH[c0 + ra * PW], (float)sH[c1 + ra * PW], (float)sH[c0 + rb * PW],
                          (float)sH[c1 + rb * PW]);
        }
      }
    }
    __syncthreads();
  }
  // a block that gave up still owns copies in flight: let them land first
  if (tid == 0) {
    // the parity of a buffer's outstanding phase is not tracked here: waiting
    // for both (bounded) covers the copy in flight
    if (issued0) { mbar_wait(&bar[0], 0u); mbar_wait(&bar[0], 1u); }
    if (issued1) { mbar_wait(&bar[1], 0u); mbar_wait(&bar[1], 1u); }
  }
}

}  // namespace gasatt

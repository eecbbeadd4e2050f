// hpccg_iter_tma.cuh -- one whole iteration of the FP32 matrix-free inner CG
// in a single pass over the grid.
//
// The three-kernel iteration (p = r + beta p with d += alpha p; Ap = A p with
// p.Ap; r -= alpha Ap with r.r) moves 40 bytes per row.  This pass moves 24:
// it reads r, p and d and writes r, p and d.  The product A p of the previous
// iteration is not stored; each tile recomputes it from p with a two-deep halo.
// For iteration k (k >= 1), with alpha = alpha_{k-1} and beta = beta_k:
//
//   Ap_old = 28 p - box27(p)                 (A p_{k-1}; p is p_{k-1})
//   r'     = r - alpha Ap_old                (r_k)
//   p'     = r' + beta p                     (p_k)
//   d     += alpha p                         (the correction gains alpha_{k-1} p_{k-1})
//   Ap'    = 28 p' - box27(p')               (A p_k, reduced into the dots only)
//   dots   = p'.Ap', r'.Ap', Ap'.Ap', r'.r'
//
// The first pass of an inner solve (k = 0) sets p' = r' = r / ||r|| (the
// refinement residual arrives unscaled) and d = 0.  From the dots the
// last block forms alpha_k = r'.r' / p'.Ap' and the next beta from the
// recurrence ||r_k - alpha_k Ap_k||^2 = r'.r' - 2 alpha_k r'.Ap' +
// alpha_k^2 Ap'.Ap', which the next pass needs before it can build p_{k+1}.
// r and p are double-buffered (the halo of a tile is another tile's rows).
//
// A CTA of 512 threads owns a 64 x 64 tile of grid columns (4 x 2 per thread)
// and a chunk of z planes, one CTA per SM (128 registers a thread, 199 KB of
// shared memory).  Step s receives by TMA plane s of p (box 72 x 68 from
// (x0-4, y0-2)), plane s-1 of r (box 72 x 66 from (x0-4, y0-1)) and plane s-1
// of d (box 64 x 64) into a ring of kItStages slots; zeros arrive outside the
// grid.  Phase A of step s forms p'(s-1) on the tile and its one-wide ring (the
// ring by 260 threads, one position each) into a shared p' plane, and stores
// r', p' and d of the tile's own rows; phase B forms Ap'(s-3) from the shared
// p' planes s-4 .. s-2 and accumulates the dots.  The loop is unrolled by two
// so that values kept for one or two steps alternate between two register sets.
// Against 32 x 64 tiles of 256 threads, two CTAs per SM, the 64 x 64 tile
// recomputes fewer ring positions and halo lines per row (260 ring positions
// per 4096 rows instead of 196 per 2048; p box 1.20 instead of 1.33 floats per
// row) and passes half as many CTA barriers per row: 0.079 against 0.087 ms a
// pass at 256^3, same iterates.
//
// Every stencil sum has one association, fixed by the position: a 3-point line
// sum at even x is x[x-1] + (x[x] + x[x+1]) and at odd x (x[x-1] + x[x]) +
// x[x+1] (neighbouring columns share the pair); the 3-line box sum likewise by
// the parity of y; the 3-plane sum is (box(z-1) + box(z)) + box(z+1).  So a
// ring position equals, bit for bit, the value its owning tile stores, and Ap'
// here equals the A p the next pass recomputes.
//
// Waits on the ring's mbarriers are bounded: on expiry the CTA records
// HPCCG_ERR_TIMEOUT in the caller's status word, waits (bounded) for its own
// loads in flight and finishes without the remaining rows.
#pragma once
#include "hpccg_stencil_tma.cuh"

namespace hpccg {

constexpr int kItTileX = 64, kItTileY = 64;                   // 64 x 64 columns per CTA
constexpr int kItBlock = 512;                                 // threads per CTA
constexpr int kItTX = kItTileX / 4;                           // threads along x
constexpr int kItBoxX = kItTileX + 8;                         // x0-4 .. x0+67
constexpr int kItPBoxY = kItTileY + 4;                        // p box: y0-2 .. y0+65
constexpr int kItRBoxY = kItTileY + 2;                        // r box, p' plane: y0-1 .. y0+64
constexpr uint32_t kItPBytes = kItBoxX * kItPBoxY * 4;        // 19584
constexpr uint32_t kItRBytes = kItBoxX * kItRBoxY * 4;        // 19008
constexpr uint32_t kItDBytes = kItTileX * kItTileY * 4;       // 16384
constexpr int kItRSlot = ((kItRBytes + 127) / 128) * 128;     // 19072
constexpr int kItStageBytes = kItPBytes + kItRSlot + kItDBytes;  // 55040
constexpr int kItStages = 3;
constexpr int kItNFloats = kItRSlot / 4;                      // one shared p' plane
constexpr int kItHalo = 2 * kItRBoxY + 2 * kItTileX;          // ring positions of a p' plane (260)
constexpr int kItSmemBytes = kItStages * kItStageBytes + 2 * kItRSlot;  // dynamic shared memory
constexpr int kItMaxGrid = (kMaxPartials - 1) / 4;           // four partials per CTA
static_assert(kItPBytes % 128 == 0 && kItDBytes % 128 == 0 && kItHalo <= kItBlock, "layout");
static_assert(kItBlock == (kItTileX / 4) * (kItTileY / 2), "one thread per 4 x 2 columns");

struct IterScalars {
  float alpha, nalpha, beta;
  float inv;  // first pass: r arrives unscaled and is multiplied by inv = 1/||r||
};

// 3-point line sums of the four columns at r[0..3] (r[-1] and r[4] are the
// neighbours; r[0] sits at an even x).
__device__ __forceinline__ float4 it_line4(const float *r, float ls[4]) {
  const float4 m = *reinterpret_cast<const float4 *>(r);
  const float l = r[-1], rr = r[4];
  const float a = m.x + m.y, b = m.z + m.w;
  ls[0] = l + a;
  ls[1] = a + m.z;
  ls[2] = m.y + b;
  ls[3] = b + rr;
  return m;
}
// the same for one column at r[0]
__device__ __forceinline__ float it_line1(const float *r, bool odd_x) {
  return odd_x ? (r[-1] + r[0]) + r[1] : r[-1] + (r[0] + r[1]);
}
// 3-line box sums of rows y (even) and y+1 from the line sums of y-1 .. y+2
__device__ __forceinline__ void it_box2(const float ls[4][4], float b[2][4]) {
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const float m = ls[1][i] + ls[2][i];
    b[0][i] = ls[0][i] + m;
    b[1][i] = m + ls[3][i];
  }
}

__device__ __forceinline__ float &f4(float4 &v, int i) { return reinterpret_cast<float *>(&v)[i]; }
__device__ __forceinline__ float f4(const float4 &v, int i) { return reinterpret_cast<const float *>(&v)[i]; }

// Per-thread constants of a pass.
struct ItCta {
  int nz, z0, z1, s_lo, s_hi;
  int plane, nx, xc, yc;   // row offsets fit in int: the grid has fewer than 2^31 rows
  int txo, tyo, dofs;      // own columns in the boxes; own rows (r box, p' plane); d slot offset
  int hofs;                // ring position in the r box / p' plane
  bool in_r[2], has_h, h_in, h_oddx, h_oddy;
};
// Values kept one or two steps: two sets, used by even and odd steps in turn.
struct ItGen {
  float b2[2][4];  // box sums of p, plane s (step s)
  float4 pc[2];    // p of the own rows, plane s
  float n2[2][4];  // box sums of p', plane s-2
  float4 rn[2];    // r' of the own rows, plane s-1 (read back two steps later)
  float b2h, pch;  // the ring position's box sum and p, plane s
};
struct ItRun {
  float T[2][4];   // box(s-2) + box(s-1) of p
  float Tn[2][4];  // box(s-4) + box(s-3) of p'
  float Th;
  double dacc[4];  // the dots; each step's FP32 partials are added in double
};

template <bool FIRST>
__device__ __forceinline__ bool it_step(const int s, const ItCta &c, unsigned char *smem, uint64_t *full,
                                        ItGen &cur, const ItGen &prv, ItRun &run, float *r_out, float *p_out,
                                        float *d, const IterScalars &sc, int *status) {
  float *const nbuf = reinterpret_cast<float *>(smem + kItStages * kItStageBytes);
  // ---- phase B: Ap'(s-3) from p' planes s-4 .. s-2 (plane s-2 made last step);
  // nothing at s = z1 + 3, the extra step of an odd count under the two-step loop
  if (s >= c.z0 + 1 && s <= c.z1 + 2) {
    float ls[4][4];
    const float *nb = nbuf + (s & 1) * kItNFloats + c.tyo - kItBoxX + c.txo;  // N(s-2), line yc-1
#pragma unroll
    for (int k = 0; k < 4; ++k) it_line4(nb + k * kItBoxX, ls[k]);
    it_box2(ls, cur.n2);
    if (s - 3 >= c.z0 && s - 3 < c.z1) {
      const float *nc = nbuf + ((s + 1) & 1) * kItNFloats + c.tyo + c.txo;  // N(s-3), row yc
      float fpa = 0.f, fra = 0.f, faa = 0.f;
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        if (!c.in_r[j]) continue;
        const float4 pn = *reinterpret_cast<const float4 *>(nc + j * kItBoxX);
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          const float ap = fmaf(28.f, f4(pn, i), -(run.Tn[j][i] + cur.n2[j][i]));
          fpa = fmaf(f4(pn, i), ap, fpa);
          fra = fmaf(f4(cur.rn[j], i), ap, fra);
          faa = fmaf(ap, ap, faa);
        }
      }
      run.dacc[0] += (double)fpa;
      run.dacc[1] += (double)fra;
      run.dacc[2] += (double)faa;
    }
#pragma unroll
    for (int j = 0; j < 2; ++j)
#pragma unroll
      for (int i = 0; i < 4; ++i) run.Tn[j][i] = prv.n2[j][i] + cur.n2[j][i];
  }
  // ---- phase A: p'(s-1) on the tile and its ring; r', p', d of the own rows
  if (s > c.s_hi) return true;
  const int k = (s - c.s_lo) % kItStages;
  const uint32_t parity = (uint32_t)((s - c.s_lo) / kItStages) & 1u;
  for (uint32_t i = 0;; ++i) {
    if (tc::mbar_try_wait(&full[k], parity)) break;
    if (i >= tc::kSpinLimit) {
      if (status) atomicCAS(status, 0, HPCCG_ERR_TIMEOUT);
      return false;
    }
  }
  const float *P = reinterpret_cast<const float *>(smem + k * kItStageBytes);
  const float *R = P + kItPBytes / 4;
  const float *D = P + (kItPBytes + kItRSlot) / 4;
  if (!FIRST) {
    float ls[4][4];
    const float *pr = P + c.tyo + c.txo;  // p box row of line yc-1
#pragma unroll
    for (int kk = 0; kk < 4; ++kk) {
      const float4 m = it_line4(pr + kk * kItBoxX, ls[kk]);
      if (kk == 1) cur.pc[0] = m;
      if (kk == 2) cur.pc[1] = m;
    }
    it_box2(ls, cur.b2);
    if (c.has_h) {
      const float *hp = P + c.hofs;  // p box row of the ring position's y-1
      const float l0 = it_line1(hp, c.h_oddx), l1 = it_line1(hp + kItBoxX, c.h_oddx),
                  l2 = it_line1(hp + 2 * kItBoxX, c.h_oddx);
      cur.b2h = c.h_oddy ? (l0 + l1) + l2 : l0 + (l1 + l2);
      cur.pch = hp[kItBoxX];
    }
  }
  if (s >= c.z0) {  // p'(s-1), s-1 in [z0-1, z1]
    const bool pin = (unsigned)(s - 1) < (unsigned)c.nz;
    const bool own = s - 1 >= c.z0 && s - 1 < c.z1;
    float *N = nbuf + ((s + 1) & 1) * kItNFloats;  // N(s-1)
    const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
    float frr = 0.f;
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      const float4 ro = *reinterpret_cast<const float4 *>(R + c.tyo + j * kItBoxX + c.txo);
      float4 rn, pn;
      if (FIRST) {
#pragma unroll
        for (int i = 0; i < 4; ++i) f4(rn, i) = f4(ro, i) * sc.inv;
        pn = rn;
      } else {
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          const float ap = fmaf(28.f, f4(prv.pc[j], i), -(run.T[j][i] + cur.b2[j][i]));
          f4(rn, i) = fmaf(sc.nalpha, ap, f4(ro, i));
          f4(pn, i) = fmaf(sc.beta, f4(prv.pc[j], i), f4(rn, i));
        }
      }
      if (!(pin && c.in_r[j])) rn = pn = z4;
      *reinterpret_cast<float4 *>(N + c.tyo + j * kItBoxX + c.txo) = pn;
      cur.rn[j] = rn;
      if (own && c.in_r[j]) {
        const int gi = (s - 1) * c.plane + (c.yc + j) * c.nx + c.xc;
        *reinterpret_cast<float4 *>(r_out + gi) = rn;
        *reinterpret_cast<float4 *>(p_out + gi) = pn;
        if (FIRST) {
          *reinterpret_cast<float4 *>(d + gi) = z4;  // the correction of a new inner solve starts at 0
        } else {
          float4 dv = *reinterpret_cast<const float4 *>(D + c.dofs + j * kItTileX);
#pragma unroll
          for (int i = 0; i < 4; ++i) f4(dv, i) = fmaf(sc.alpha, f4(prv.pc[j], i), f4(dv, i));
          *reinterpret_cast<float4 *>(d + gi) = dv;
        }
#pragma unroll
        for (int i = 0; i < 4; ++i) frr = fmaf(f4(rn, i), f4(rn, i), frr);
      }
    }
    run.dacc[3] += (double)frr;
    if (c.has_h) {
      const float ro = R[c.hofs];
      float pn;
      if (FIRST) {
        pn = ro * sc.inv;
      } else {
        const float ap = fmaf(28.f, prv.pch, -(run.Th + cur.b2h));
        pn = fmaf(sc.beta, prv.pch, fmaf(sc.nalpha, ap, ro));
      }
      N[c.hofs] = (pin && c.h_in) ? pn : 0.f;
    }
  }
  if (!FIRST) {
#pragma unroll
    for (int j = 0; j < 2; ++j)
#pragma unroll
      for (int i = 0; i < 4; ++i) run.T[j][i] = prv.b2[j][i] + cur.b2[j][i];
    run.Th = prv.b2h + cur.b2h;
  }
  return true;
}

// Rows of the calling CTA.  dots[0..3] receive this thread's p'.Ap', r'.Ap',
// Ap'.Ap', r'.r'.  Every thread of the CTA must call it (it has barriers).
template <bool FIRST>
__device__ __forceinline__ void iter_rows_tma(const TmaTile &t, const CUtensorMap *pmap, const CUtensorMap *rmap,
                                              const CUtensorMap *dmap, float *r_out, float *p_out, float *d,
                                              const IterScalars &sc, double dots[4], int *status) {
  extern __shared__ __align__(128) unsigned char it_smem[];  // kItSmemBytes
  __shared__ uint64_t full[kItStages];
  const int tid = threadIdx.x, tx = tid % kItTX, ty = tid / kItTX;
  const int per_plane = t.tiles_x * t.tiles_y;
  const int q = blockIdx.x / per_plane, tile = blockIdx.x - q * per_plane;
  const int x0 = (tile % t.tiles_x) * kItTileX, y0 = (tile / t.tiles_x) * kItTileY;
  ItCta c;
  c.nz = t.nz;
  c.z0 = q * t.zc;
  c.z1 = min(t.nz, c.z0 + t.zc);
  c.s_lo = c.z0 - 2;  // planes of p this CTA loads: s_lo .. s_hi
  c.s_hi = c.z1 + 1;
  c.plane = t.nx * t.ny;
  c.nx = t.nx;
  c.xc = x0 + 4 * tx;
  c.yc = y0 + 2 * ty;
  c.txo = 4 * tx + 4;
  c.tyo = (2 * ty + 1) * kItBoxX;
  c.dofs = (2 * ty) * kItTileX + 4 * tx;
  c.in_r[0] = c.xc < t.nx && c.yc < t.ny;
  c.in_r[1] = c.xc < t.nx && c.yc + 1 < t.ny;
  // ring position of this thread (r box coordinates hbx, hby)
  c.has_h = tid < kItHalo;
  int hbx, hby;
  if (tid < kItRBoxY) {
    hbx = 3, hby = tid;  // column x0-1
  } else if (tid < 2 * kItRBoxY) {
    hbx = kItBoxX - 4, hby = tid - kItRBoxY;  // column x0+kItTileX
  } else if (tid < 2 * kItRBoxY + kItTileX) {
    hbx = 4 + tid - 2 * kItRBoxY, hby = 0;  // row y0-1
  } else {
    hbx = 4 + min(tid - 2 * kItRBoxY - kItTileX, kItTileX - 1), hby = kItRBoxY - 1;  // row y0+64
  }
  const int hx = x0 - 4 + hbx, hy = y0 - 1 + hby;
  c.h_in = c.has_h && hx >= 0 && hx < t.nx && hy >= 0 && hy < t.ny;
  c.h_oddx = hx & 1;
  c.h_oddy = hy & 1;
  c.hofs = hby * kItBoxX + hbx;  // also the p box row of y-1 (the p box starts one row higher)

  if (tid == 0) {
    for (int k = 0; k < kItStages; ++k) tc::mbar_init(&full[k], 1);
    tc::fence_mbar_init();
  }
  __syncthreads();
  // The first pass of an inner solve reads r alone: p' = r' = r / ||r|| needs no
  // p, and d is written as 0 without being read.
  auto issue = [&](int s) {  // thread 0
    const int k = (s - c.s_lo) % kItStages;
    unsigned char *st = it_smem + k * kItStageBytes;
    tc::mbar_expect_tx(&full[k], FIRST ? kItRBytes : kItPBytes + kItRBytes + kItDBytes);
    if (!FIRST) tma_load_3d(st, pmap, &full[k], x0 - 4, y0 - 2, s);
    tma_load_3d(st + kItPBytes, rmap, &full[k], x0 - 4, y0 - 1, s - 1);
    if (!FIRST) tma_load_3d(st + kItPBytes + kItRSlot, dmap, &full[k], x0, y0, s - 1);
  };
  int next = c.s_lo;  // next plane to load (thread 0's view)
  if (tid == 0)
    for (; next <= c.s_hi && next < c.s_lo + kItStages; ++next) issue(next);

  ItGen A, B;
  ItRun run;
#pragma unroll
  for (int j = 0; j < 2; ++j) {
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      A.b2[j][i] = B.b2[j][i] = A.n2[j][i] = B.n2[j][i] = run.T[j][i] = run.Tn[j][i] = 0.f;
    }
    A.pc[j] = B.pc[j] = A.rn[j] = B.rn[j] = make_float4(0.f, 0.f, 0.f, 0.f);
  }
  A.b2h = B.b2h = A.pch = B.pch = run.Th = 0.f;
#pragma unroll
  for (int k = 0; k < 4; ++k) run.dacc[k] = 0.0;
  int consumed = c.s_lo - 1;
  bool failed = false;
  // after each step every thread is done with its slot and with N(s-3), and N(s-1) is complete
  auto end_step = [&](int s, bool ok) -> bool {
    if (__syncthreads_or(!ok)) return false;
    if (s <= c.s_hi) consumed = s;
    if (tid == 0 && next <= c.s_hi) {
      issue(next);
      ++next;
    }
    return true;
  };
  for (int s = c.s_lo; s <= c.z1 + 2; s += 2) {  // s = z1 + 3 is a step without effect
    if (!end_step(s, it_step<FIRST>(s, c, it_smem, full, A, B, run, r_out, p_out, d, sc, status))) {
      failed = true;
      break;
    }
    if (!end_step(s + 1, it_step<FIRST>(s + 1, c, it_smem, full, B, A, run, r_out, p_out, d, sc, status))) {
      failed = true;
      break;
    }
  }
  if (failed && tid == 0) {  // loads still in flight land before the CTA exits
    for (int s = consumed + 1; s < next; ++s) {
      const int k = (s - c.s_lo) % kItStages;
      const uint32_t parity = (uint32_t)((s - c.s_lo) / kItStages) & 1u;
      for (uint32_t i = 0; i < tc::kSpinLimit; ++i)
        if (tc::mbar_try_wait(&full[k], parity)) break;
    }
  }
#pragma unroll
  for (int k = 0; k < 4; ++k) dots[k] = run.dacc[k];
}

// Sums v[0..3] over the block (fixed order); valid in thread 0.
template <int BLOCK>
__device__ __forceinline__ void block_sum4(double v[4], double *smem /* [4 * 32] */) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    v[k] = warp_sum(v[k]);
    if (lane == 0) smem[k * 32 + wid] = v[k];
  }
  __syncthreads();
  if (wid == 0) {
#pragma unroll
    for (int k = 0; k < 4; ++k) v[k] = warp_sum(lane < BLOCK / 32 ? smem[k * 32 + lane] : 0.0);
  }
  __syncthreads();
}

// Four partials per block at partials[k * gridDim.x + block]; true in every
// thread of the last block to arrive, whose thread 0 then holds the totals
// summed in block order.
template <int BLOCK>
__device__ __forceinline__ bool reduce4_last(const Reduction &red, double v[4], double *smem) {
  __shared__ bool s_last;
  block_sum4<BLOCK>(v, smem);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < 4; ++k) red.partials[k * gridDim.x + blockIdx.x] = v[k];
    __threadfence();
    s_last = atomicAdd(red.counter, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!s_last) return false;
  __threadfence();
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    double a = 0.0;
    for (int i = threadIdx.x; i < (int)gridDim.x; i += BLOCK)
      a = __dadd_rn(a, ((volatile double *)red.partials)[k * gridDim.x + i]);
    v[k] = a;
  }
  block_sum4<BLOCK>(v, smem);
  if (threadIdx.x == 0) *red.counter = 0u;
  return true;
}

}  // namespace hpccg

// hpccg_slab.cu -- multi-rank CG over z slabs of the weak-scaled problem.
//
// With P ranks the reference gives rank r the rows local_nrow*r+1 ..
// local_nrow*(r+1) of the nx x ny x (nz*P) grid (MPI/src/SparseMatrix.F90:
// 68-185), renumbers each rank's columns into its own rows followed by
// "externals" owned by other ranks (make_local_matrix, :235-627), fills the
// externals of p before every SpMV (exchange_externals, :630-680) and sums
// every dot product over the ranks (MPI/src/vector_operations.F90:64-65,
// 96-97).  This file holds:
//
//  - the halo plan (host): a rank's renumbering and the lists that say which
//    of its externals come from which rank, in either form the reference
//    has: HPCCG_HALO_MPI -- externals grouped by owner, a send list of local
//    indices per neighbour, pack and send (MPI variant); HPCCG_HALO_GET --
//    externals in order of first appearance, blocks of one owner, each filled
//    from one contiguous range of the owner's vector (CAF-V2 variant,
//    CAF-V2/src/SparseMatrix.F90:205-370);
//  - the device part of a rank (hpccg_slab): the local matrix as a column-
//    major ELL whose columns index [own rows | externals], the pack and
//    scatter kernels of the two exchanges, and the CG steps of one rank, each
//    leaving its local dot product in a caller-owned state array so that any
//    transport can sum it over the ranks;
//  - hpccg_slab_group_cg: all ranks of the communicator in this process (on
//    one GPU or several), the exchange done by device copies and the sums by
//    a fixed-order fold over ranks.
//
// The MPI variant's block lengths: make_local_matrix's counting loop
// (:533-545) comes out one too large for every neighbour block but the last,
// which would shift the halo of ranks with two neighbours.  The plan here uses
// the block sizes themselves, the routine's evident intent; with two ranks
// the two agree.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <unordered_map>
#include <vector>

#include "hpccg_internal.cuh"

namespace hpccg {

constexpr int kSlabMaxBlocks = 1024;  // partial sums of the local dot products
enum SlabState { kLocal = 0, kGlobal = 1, kRtrans = 2, kNormr = 3, kAlpha = 4, kBeta = 5, kDone = 6, kTol = 7 };

}  // namespace hpccg

struct hpccg_slab_plan {
  int32_t nrow = 0, nranks = 1, rank = 0, mode = HPCCG_HALO_MPI;
  int64_t nnz = 0;
  std::vector<int32_t> rowindex;      // 1-based, nrow+1
  std::vector<int32_t> col_local;     // 1-based local columns: 1..nrow own, nrow+1.. externals
  std::vector<int32_t> ext_global;    // global id (1-based) of local external i (0-based i)
  std::vector<int32_t> ext_owner;     // owning rank of local external i
  // HPCCG_HALO_MPI
  std::vector<int32_t> neighbors, recv_length, send_length, elements_to_send;  // elements_to_send: 1-based local
  bool sends_set = false;
  // HPCCG_HALO_GET: per block owner, first external (1-based), inmin, inmax (owner-local, 1-based)
  std::vector<int32_t> blocks;  // 4 per block
  std::vector<int32_t> remote_index;  // owner-local index (1-based) of each external
  int32_t first_row = 1;              // this rank's first global row
};

struct hpccg_slab {
  int device = 0, num_sms = 0;
  cudaStream_t stream = nullptr;
  int32_t nrow = 0, ncol = 0, npad = 0, width = 0, mode = HPCCG_HALO_MPI, rank = 0, nranks = 1;
  int32_t *d_col = nullptr;   // [width][npad], 0-based into [0, ncol)
  double *d_val = nullptr;
  int32_t *d_send = nullptr;  // elements_to_send, 0-based
  int32_t nsend = 0;
  std::vector<int32_t> neighbors, recv_length, send_length;
  int32_t *d_remote = nullptr;  // GET: per external, offset into its block's range (remote_index - inmin)
  std::vector<int32_t> blocks;
  double *d_partials = nullptr;
  unsigned *d_counter = nullptr;
  double *d_stage = nullptr;  // GET: one block's remote range; MPI: the send buffer (group CG)
  int64_t stage_len = 0;
  int grid = 0;
};

namespace hpccg {

// ---- the plan: make_local_matrix's per-rank work -------------------------

// Renumbers the rank's columns.  MPI form (MPI/src/SparseMatrix.F90:285-389):
// externals numbered in order of first appearance, then renumbered so that
// the externals of one owner are consecutive, owners in order of their first
// external.  GET form (CAF-V2/src/SparseMatrix.F90:234-306): externals keep
// their order of first appearance; runs with one owner form blocks.
static int build_plan(hpccg_slab_plan *P, const int32_t *colindex, const int32_t *first_rows) {
  const int32_t n = P->nrow, first = first_rows[P->rank], last = first_rows[P->rank + 1] - 1;
  const int32_t total = first_rows[P->nranks] - 1;
  P->first_row = first;
  auto owner_of = [&](int32_t g) {  // last rank whose first row is <= g (:330-343)
    int32_t q = P->nranks - 1;
    while (q > 0 && first_rows[q] > g) --q;
    return q;
  };
  // first appearance order (the reference keeps a table over all global ids,
  // :283-286; a map over the externals alone holds the same information)
  std::unordered_map<int32_t, int32_t> seen;
  std::vector<int32_t> order;  // global ids in order of first appearance
  P->col_local.assign(colindex, colindex + P->nnz);
  for (int64_t k = 0; k < P->nnz; ++k) {
    const int32_t g = colindex[k];
    if (g < 1 || g > total) return HPCCG_ERR_INVALID_ARG;
    if (g >= first && g <= last) continue;
    if (seen.emplace(g, (int32_t)order.size()).second) order.push_back(g);
  }
  const int32_t ne = (int32_t)order.size();
  std::vector<int32_t> local_of(ne);  // first-appearance number -> local external number (0-based)
  if (P->mode == HPCCG_HALO_MPI) {
    std::vector<int32_t> owner(ne);
    for (int32_t i = 0; i < ne; ++i) owner[i] = owner_of(order[i]);
    std::vector<char> done(ne, 0);
    int32_t next = 0;
    for (int32_t i = 0; i < ne; ++i) {
      if (done[i]) continue;
      for (int32_t j = i; j < ne; ++j)
        if (!done[j] && owner[j] == owner[i]) {
          local_of[j] = next++;
          done[j] = 1;
        }
    }
    P->ext_global.assign(ne, 0);
    P->ext_owner.assign(ne, 0);
    for (int32_t i = 0; i < ne; ++i) {
      P->ext_global[local_of[i]] = order[i];
      P->ext_owner[local_of[i]] = owner[i];
    }
    P->neighbors.clear();
    P->recv_length.clear();
    for (int32_t i = 0; i < ne; ++i) {
      if (i == 0 || P->ext_owner[i] != P->ext_owner[i - 1]) {
        P->neighbors.push_back(P->ext_owner[i]);
        P->recv_length.push_back(0);
      }
      P->recv_length.back() += 1;
    }
  } else {
    for (int32_t i = 0; i < ne; ++i) local_of[i] = i;
    P->ext_global = order;
    P->ext_owner.assign(ne, 0);
    P->remote_index.assign(ne, 0);
    P->blocks.clear();
    for (int32_t i = 0; i < ne; ++i) {
      const int32_t q = owner_of(order[i]);
      const int32_t ind = order[i] - first_rows[q] + 1;
      P->ext_owner[i] = q;
      P->remote_index[i] = ind;
      if (i == 0 || q != P->ext_owner[i - 1]) {
        P->blocks.insert(P->blocks.end(), {q, i + 1, ind, ind});
      } else {
        int32_t *b = &P->blocks[P->blocks.size() - 4];
        b[2] = std::min(b[2], ind);
        b[3] = std::max(b[3], ind);
      }
    }
    if (P->nranks == 1) P->blocks.clear();
  }
  for (int64_t k = 0; k < P->nnz; ++k) {
    const int32_t g = colindex[k];
    P->col_local[k] = (g >= first && g <= last) ? g - first + 1 : n + 1 + local_of[seen.find(g)->second];
  }
  return HPCCG_OK;
}

// ---- device kernels -------------------------------------------------------

// y = A x over the local ELL, the reference's k order with separately rounded
// terms (MPI/src/SparseMatrix.F90:213-232); optionally the local x.y (dot_x
// non-null: the dot of y with dot_x's own rows), reduced in a fixed order.
template <bool DOT>
__global__ void __launch_bounds__(kBlock) k_slab_spmv(int32_t n, int32_t npad, int32_t width,
                                                      const int32_t *__restrict__ col,
                                                      const double *__restrict__ val,
                                                      const double *__restrict__ x, double *__restrict__ y,
                                                      Reduction red, double *out, const double *state) {
  __shared__ double smem[32];
  if (state && state[kDone] != 0.0) return;
  double part = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int k = 0; k < width; ++k) {
      const int64_t o = (int64_t)k * npad + i;
      s = __dadd_rn(s, __dmul_rn(__ldg(val + o), __ldg(x + __ldg(col + o))));
    }
    y[i] = s;
    if (DOT) part = __dadd_rn(part, __dmul_rn(x[i], s));
  }
  if (DOT) {
    const double t = block_sum<kBlock>(part, smem);
    if (arrive_last(red, t)) {
      const double v = finish_sum<kBlock>(red, smem);
      if (threadIdx.x == 0) *out = v;
    }
  }
}

// Local dot of a vector with itself, fixed order (MPI/src/vector_operations.F90:73-103, one rank's part).
__global__ void __launch_bounds__(kBlock) k_slab_dot1(int32_t n, const double *__restrict__ x, Reduction red,
                                                      double *out, const double *state) {
  __shared__ double smem[32];
  if (state && state[kDone] != 0.0) return;
  double part = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    part = __dadd_rn(part, __dmul_rn(x[i], x[i]));
  const double t = block_sum<kBlock>(part, smem);
  if (arrive_last(red, t)) {
    const double v = finish_sum<kBlock>(red, smem);
    if (threadIdx.x == 0) *out = v;
  }
}

// send_buffer(i) = x(elements_to_send(i)) (MPI/src/SparseMatrix.F90:664-666)
__global__ void k_slab_pack(int32_t m, const int32_t *__restrict__ idx, const double *__restrict__ x,
                            double *__restrict__ buf, const double *state) {
  if (state && state[kDone] != 0.0) return;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) buf[i] = x[idx[i]];
}

// x(nrow + i) = xl(remote_index(i) - inmin + 1) for the block's externals
// (CAF-V2/src/SparseMatrix.F90:362-366); rel[i] = remote_index(i) - inmin.
__global__ void k_slab_scatter(int32_t first, int32_t count, const int32_t *__restrict__ rel,
                               const double *__restrict__ xl, double *__restrict__ xext, const double *state) {
  if (state && state[kDone] != 0.0) return;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x)
    xext[first + i] = xl[rel[first + i]];
}

// ---- CG steps of one rank (MPI/src/numerics.F90:41-162) --------------------
// start: p = x
__global__ void k_slab_start(int32_t n, const double *__restrict__ x, double *__restrict__ p) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) p[i] = x[i];
}
// prepare: r = b - Ap (waxpby with alpha = 1, beta = -1; :96)
__global__ void k_slab_residual(int32_t n, const double *__restrict__ b, const double *__restrict__ Ap,
                                double *__restrict__ r) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    r[i] = __dadd_rn(__dmul_rn(1.0, b[i]), __dmul_rn(-1.0, Ap[i]));
}
// after the sum of r.r over ranks: rtrans, normr (:97-98); hist[0]
__global__ void k_slab_prepared(double *state, double *hist) {
  state[kRtrans] = state[kGlobal];
  state[kNormr] = sqrt(state[kRtrans]);
  state[kDone] = 0.0;
  if (hist) hist[0] = state[kNormr];
}
// top of iteration k (:109-126): stop test on the previous normr; k == 1: p = r,
// else beta from the new r.r (summed over ranks) and p = r + beta p.
__global__ void k_slab_begin(int32_t n, int32_t k, const double *__restrict__ r, double *__restrict__ p,
                             double *state, double *hist, int32_t *niters) {
  const double normr = state[kNormr];
  if (state[kDone] != 0.0) return;
  if (normr < state[kTol]) {  // every block sees the same normr: all return
    if (blockIdx.x == 0 && threadIdx.x == 0) state[kDone] = 1.0;
    return;
  }
  double beta = 0.0, rtrans = state[kRtrans];
  if (k > 1) {
    rtrans = state[kGlobal];
    beta = rtrans / state[kRtrans];
  }
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    p[i] = k == 1 ? r[i] : __dadd_rn(r[i], __dmul_rn(beta, p[i]));
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    state[kBeta] = beta;
    if (niters) *niters = k;
    if (hist) hist[k] = sqrt(rtrans);
  }
}
// The block-0 bookkeeping of begin must not race the other blocks' reads of
// kRtrans / kGlobal: it runs as a separate one-thread kernel after begin.
__global__ void k_slab_begin_scalars(int32_t k, double *state) {
  if (state[kDone] != 0.0) return;
  if (k > 1) state[kRtrans] = state[kGlobal];
  state[kNormr] = sqrt(state[kRtrans]);
}
// after the sum of p.Ap over ranks: alpha = rtrans / p.Ap (:136-138); r -= alpha Ap,
// x += alpha p (:139-140); then the local r.r for the next iteration's beta.
__global__ void k_slab_update(int32_t n, const double *__restrict__ p, const double *__restrict__ Ap,
                              double *__restrict__ r, double *__restrict__ x, const double *state) {
  if (state[kDone] != 0.0) return;
  const double alpha = state[kRtrans] / state[kGlobal];
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    r[i] = __dadd_rn(r[i], __dmul_rn(-alpha, Ap[i]));
    x[i] = __dadd_rn(x[i], __dmul_rn(alpha, p[i]));
  }
}
// fixed-order fold of the ranks' local values into the global sum (rank order)
__global__ void k_slab_fold(const double *gathered, int32_t nranks, double *state) {
  double s = gathered[0];
  for (int q = 1; q < nranks; ++q) s = __dadd_rn(s, gathered[q]);
  state[kGlobal] = s;
}

}  // namespace hpccg

using namespace hpccg;

// ===========================================================================
// C-ABI: plan
// ===========================================================================

extern "C" int hpccg_generate_matrix_rank(int32_t nx, int32_t ny, int32_t nz, int32_t rank, int32_t nranks,
                                          int32_t *rowindex, int32_t *colindex, double *values, double *x,
                                          double *b, double *xexact, int64_t *nnz) {
  if (nx < 1 || ny < 1 || nz < 1 || nranks < 1 || rank < 0 || rank >= nranks || !rowindex || !colindex ||
      !values || !nnz)
    return HPCCG_ERR_INVALID_ARG;
  const int64_t local = (int64_t)nx * ny * nz;
  if (local * nranks > INT32_MAX || 27 * local > INT32_MAX) return HPCCG_ERR_TOO_LARGE;
  const int32_t plane = nx * ny, nrow = (int32_t)local, total = (int32_t)(local * nranks);
  const int32_t start = nrow * rank + 1;
  int32_t cursor = 1;
  // rows in iz -> iy -> ix order, stencil sz -> sy -> sx; kept when the
  // neighbour is inside the x and y faces and its global id inside
  // [1, total_nrow] (the z truncation at the global ends, :151-153)
  for (int32_t iz = 0; iz < nz; ++iz)
    for (int32_t iy = 0; iy < ny; ++iy)
      for (int32_t ix = 0; ix < nx; ++ix) {
        const int32_t li = iz * plane + iy * nx + ix, row = start + li;
        rowindex[li] = cursor;
        int32_t cnt = 0;
        for (int32_t sz = -1; sz <= 1; ++sz)
          for (int32_t sy = -1; sy <= 1; ++sy) {
            if (iy + sy < 0 || iy + sy >= ny) continue;
            for (int32_t sx = -1; sx <= 1; ++sx) {
              if (ix + sx < 0 || ix + sx >= nx) continue;
              const int32_t col = row + sz * plane + sy * nx + sx;
              if (col < 1 || col > total) continue;
              colindex[cursor - 1] = col;
              values[cursor - 1] = col == row ? 27.0 : -1.0;
              ++cursor;
              ++cnt;
            }
          }
        if (x) x[li] = 0.0;
        if (b) b[li] = 27.0 - (double)(cnt - 1);
        if (xexact) xexact[li] = 1.0;
      }
  rowindex[nrow] = cursor;
  *nnz = cursor - 1;
  return HPCCG_OK;
}

extern "C" int hpccg_slab_plan_create(int32_t nrow, int64_t nnz, const int32_t *rowindex, const int32_t *colindex,
                                      int32_t nranks, int32_t rank, const int32_t *first_rows, int32_t halo_mode,
                                      hpccg_slab_plan **plan) {
  if (!plan || !rowindex || !colindex || !first_rows || nrow < 1 || nnz < 1 || nranks < 1 || rank < 0 ||
      rank >= nranks || (halo_mode != HPCCG_HALO_MPI && halo_mode != HPCCG_HALO_GET))
    return HPCCG_ERR_INVALID_ARG;
  *plan = nullptr;
  if (rowindex[0] != 1 || (int64_t)rowindex[nrow] - 1 != nnz) return HPCCG_ERR_INVALID_ARG;
  for (int32_t i = 0; i < nrow; ++i)
    if (rowindex[i + 1] < rowindex[i]) return HPCCG_ERR_INVALID_ARG;
  for (int32_t q = 0; q < nranks; ++q)
    if (first_rows[q + 1] <= first_rows[q]) return HPCCG_ERR_INVALID_ARG;
  if (first_rows[0] != 1 || first_rows[rank + 1] - first_rows[rank] != nrow) return HPCCG_ERR_INVALID_ARG;
  auto *P = new (std::nothrow) hpccg_slab_plan;
  if (!P) return HPCCG_ERR_OOM;
  P->nrow = nrow, P->nnz = nnz, P->nranks = nranks, P->rank = rank, P->mode = halo_mode;
  P->rowindex.assign(rowindex, rowindex + nrow + 1);
  const int rc = build_plan(P, colindex, first_rows);
  if (rc) {
    delete P;
    return rc;
  }
  P->sends_set = halo_mode == HPCCG_HALO_GET || P->neighbors.empty();
  if (P->neighbors.empty()) P->send_length.clear();
  *plan = P;
  return HPCCG_OK;
}

extern "C" void hpccg_slab_plan_destroy(hpccg_slab_plan *plan) { delete plan; }

extern "C" int hpccg_slab_plan_info(const hpccg_slab_plan *P, int32_t *num_external, int32_t *num_neighbors,
                                    int32_t *num_blocks, int32_t *total_to_send) {
  if (!P) return HPCCG_ERR_INVALID_ARG;
  if (num_external) *num_external = (int32_t)P->ext_global.size();
  if (num_neighbors) *num_neighbors = (int32_t)P->neighbors.size();
  if (num_blocks) *num_blocks = (int32_t)(P->blocks.size() / 4);
  if (total_to_send) *total_to_send = P->sends_set ? (int32_t)P->elements_to_send.size() : -1;
  return HPCCG_OK;
}

extern "C" int hpccg_slab_plan_neighbors(const hpccg_slab_plan *P, int32_t *neighbors, int32_t *recv_length) {
  if (!P) return HPCCG_ERR_INVALID_ARG;
  if (neighbors) std::copy(P->neighbors.begin(), P->neighbors.end(), neighbors);
  if (recv_length) std::copy(P->recv_length.begin(), P->recv_length.end(), recv_length);
  return HPCCG_OK;
}

extern "C" int hpccg_slab_plan_externals(const hpccg_slab_plan *P, int32_t *global_ids, int32_t *owners) {
  if (!P) return HPCCG_ERR_INVALID_ARG;
  if (global_ids) std::copy(P->ext_global.begin(), P->ext_global.end(), global_ids);
  if (owners) std::copy(P->ext_owner.begin(), P->ext_owner.end(), owners);
  return HPCCG_OK;
}

extern "C" int hpccg_slab_plan_set_sends(hpccg_slab_plan *P, const int32_t *send_length, const int32_t *global_ids) {
  if (!P || P->mode != HPCCG_HALO_MPI || (!P->neighbors.empty() && (!send_length || !global_ids)))
    return HPCCG_ERR_INVALID_ARG;
  std::vector<int32_t> lens(P->neighbors.size()), idx;
  for (size_t i = 0; i < P->neighbors.size(); ++i) {
    if (send_length[i] < 0) return HPCCG_ERR_INVALID_ARG;
    lens[i] = send_length[i];
  }
  const int32_t first = P->first_row, last = P->first_row + P->nrow - 1;
  size_t pos = 0;
  for (size_t i = 0; i < lens.size(); ++i)
    for (int32_t k = 0; k < lens[i]; ++k, ++pos) {
      const int32_t g = global_ids[pos];
      if (g < first || g > last) return HPCCG_ERR_INVALID_ARG;  // a rank sends only rows it owns
      idx.push_back(g - first + 1);  // local index (:605-607)
    }
  P->send_length = lens;
  P->elements_to_send = idx;
  P->sends_set = true;
  return HPCCG_OK;
}

extern "C" int hpccg_slab_plan_colindex(const hpccg_slab_plan *P, int32_t *colindex_local) {
  if (!P || !colindex_local) return HPCCG_ERR_INVALID_ARG;
  std::copy(P->col_local.begin(), P->col_local.end(), colindex_local);
  return HPCCG_OK;
}

extern "C" int hpccg_slab_plan_sends(const hpccg_slab_plan *P, int32_t *send_length, int32_t *elements_to_send) {
  if (!P || !P->sends_set) return HPCCG_ERR_INVALID_ARG;
  if (send_length) std::copy(P->send_length.begin(), P->send_length.end(), send_length);
  if (elements_to_send) std::copy(P->elements_to_send.begin(), P->elements_to_send.end(), elements_to_send);
  return HPCCG_OK;
}

extern "C" int hpccg_slab_plan_blocks(const hpccg_slab_plan *P, int32_t *blocks, int32_t *remote_index) {
  if (!P) return HPCCG_ERR_INVALID_ARG;
  if (blocks) std::copy(P->blocks.begin(), P->blocks.end(), blocks);
  if (remote_index) std::copy(P->remote_index.begin(), P->remote_index.end(), remote_index);
  return HPCCG_OK;
}

// ===========================================================================
// C-ABI: device part of a rank
// ===========================================================================

extern "C" void hpccg_slab_destroy(hpccg_slab *S) {
  if (!S) return;
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(S->device);
  if (S->stream) cudaStreamSynchronize(S->stream);
  cudaFree(S->d_col);
  cudaFree(S->d_val);
  cudaFree(S->d_send);
  cudaFree(S->d_remote);
  cudaFree(S->d_partials);
  cudaFree(S->d_counter);
  cudaFree(S->d_stage);
  if (S->stream) cudaStreamDestroy(S->stream);
  cudaSetDevice(prev);
  delete S;
}

extern "C" int hpccg_slab_create(const hpccg_slab_plan *P, const double *values, hpccg_slab **out) {
  if (!P || !values || !out) return HPCCG_ERR_INVALID_ARG;
  *out = nullptr;
  if (!P->sends_set) return HPCCG_ERR_INVALID_ARG;  // MPI form: the neighbours' requests are not in yet
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) {
    cudaGetLastError();
    return HPCCG_ERR_NO_DEVICE;
  }
  auto *S = new (std::nothrow) hpccg_slab;
  if (!S) return HPCCG_ERR_OOM;
  int rc = HPCCG_OK;
  auto fail = [&](int code) {
    hpccg_slab_destroy(S);
    return code;
  };
  cudaGetDevice(&S->device);
  cudaDeviceGetAttribute(&S->num_sms, cudaDevAttrMultiProcessorCount, S->device);
  S->nrow = P->nrow;
  S->ncol = P->nrow + (int32_t)P->ext_global.size();
  S->mode = P->mode, S->rank = P->rank, S->nranks = P->nranks;
  S->neighbors = P->neighbors, S->recv_length = P->recv_length, S->send_length = P->send_length;
  S->blocks = P->blocks;
  S->npad = (S->nrow + kEllAlign - 1) / kEllAlign * kEllAlign;
  for (int32_t i = 0; i < S->nrow; ++i) S->width = std::max(S->width, P->rowindex[i + 1] - P->rowindex[i]);
  S->grid = std::min(kSlabMaxBlocks, std::max(1, std::min(S->num_sms * 8, (S->nrow + kBlock - 1) / kBlock)));
  // column-major ELL over local columns; padding slots read x(own row) * 0
  std::vector<int32_t> col((size_t)S->width * S->npad);
  std::vector<double> val((size_t)S->width * S->npad, 0.0);
  for (int32_t i = 0; i < S->npad; ++i)
    for (int32_t k = 0; k < S->width; ++k) col[(size_t)k * S->npad + i] = i < S->nrow ? i : 0;
  for (int32_t i = 0; i < S->nrow; ++i)
    for (int32_t k = P->rowindex[i] - 1, s = 0; k < P->rowindex[i + 1] - 1; ++k, ++s) {
      col[(size_t)s * S->npad + i] = P->col_local[k] - 1;
      val[(size_t)s * S->npad + i] = values[k];
    }
  auto cu = [&](cudaError_t e, const char *what) {
    if (e == cudaSuccess) return HPCCG_OK;
    return set_cuda_error(e, what, __FILE__, __LINE__);
  };
  if ((rc = cu(cudaStreamCreateWithFlags(&S->stream, cudaStreamNonBlocking), "cudaStreamCreate"))) return fail(rc);
  if (cudaMalloc(&S->d_col, col.size() * sizeof(int32_t)) != cudaSuccess ||
      cudaMalloc(&S->d_val, val.size() * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&S->d_partials, kSlabMaxBlocks * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&S->d_counter, sizeof(unsigned)) != cudaSuccess) {
    cudaGetLastError();
    return fail(HPCCG_ERR_OOM);
  }
  if ((rc = cu(cudaMemcpy(S->d_col, col.data(), col.size() * sizeof(int32_t), cudaMemcpyHostToDevice), "upload")) ||
      (rc = cu(cudaMemcpy(S->d_val, val.data(), val.size() * sizeof(double), cudaMemcpyHostToDevice), "upload")) ||
      (rc = cu(cudaMemset(S->d_counter, 0, sizeof(unsigned)), "cudaMemset")))
    return fail(rc);
  if (P->mode == HPCCG_HALO_MPI) {
    S->nsend = (int32_t)P->elements_to_send.size();
    std::vector<int32_t> idx(P->elements_to_send);
    for (auto &v : idx) v -= 1;
    S->stage_len = S->nsend;
    if (S->nsend > 0) {
      if (cudaMalloc(&S->d_send, idx.size() * sizeof(int32_t)) != cudaSuccess) {
        cudaGetLastError();
        return fail(HPCCG_ERR_OOM);
      }
      if ((rc = cu(cudaMemcpy(S->d_send, idx.data(), idx.size() * sizeof(int32_t), cudaMemcpyHostToDevice),
                   "upload")))
        return fail(rc);
    }
  } else {
    const int32_t ne = (int32_t)P->ext_global.size();
    std::vector<int32_t> rel(std::max(ne, 1), 0);
    for (size_t b = 0; b < P->blocks.size() / 4; ++b) {
      const int32_t first = P->blocks[4 * b + 1] - 1, inmin = P->blocks[4 * b + 2], inmax = P->blocks[4 * b + 3];
      const int32_t end = b + 1 < P->blocks.size() / 4 ? P->blocks[4 * (b + 1) + 1] - 1 : ne;
      for (int32_t i = first; i < end; ++i) rel[i] = P->remote_index[i] - inmin;
      S->stage_len = std::max<int64_t>(S->stage_len, inmax - inmin + 1);
    }
    if (cudaMalloc(&S->d_remote, rel.size() * sizeof(int32_t)) != cudaSuccess) {
      cudaGetLastError();
      return fail(HPCCG_ERR_OOM);
    }
    if ((rc = cu(cudaMemcpy(S->d_remote, rel.data(), rel.size() * sizeof(int32_t), cudaMemcpyHostToDevice),
                 "upload")))
      return fail(rc);
  }
  if (S->stage_len > 0 && cudaMalloc(&S->d_stage, S->stage_len * sizeof(double)) != cudaSuccess) {
    cudaGetLastError();
    return fail(HPCCG_ERR_OOM);
  }
  *out = S;
  return HPCCG_OK;
}

extern "C" int hpccg_slab_info(const hpccg_slab *S, int32_t *nrow, int32_t *ncol, int32_t *total_to_send,
                               int32_t *num_blocks) {
  if (!S) return HPCCG_ERR_INVALID_ARG;
  if (nrow) *nrow = S->nrow;
  if (ncol) *ncol = S->ncol;
  if (total_to_send) *total_to_send = S->nsend;
  if (num_blocks) *num_blocks = (int32_t)(S->blocks.size() / 4);
  return HPCCG_OK;
}

namespace {

struct DevGuard {
  int prev = 0;
  explicit DevGuard(int dev) {
    cudaGetDevice(&prev);
    cudaSetDevice(dev);
  }
  ~DevGuard() { cudaSetDevice(prev); }
};

int small_grid(const hpccg_slab *S, int64_t n) {
  return (int)std::max<int64_t>(1, std::min<int64_t>(S->num_sms * 4, (n + kBlock - 1) / kBlock));
}

// Enqueues one step of a rank's CG on the slab's stream (no synchronisation).
int enqueue_step(hpccg_slab *S, int32_t step, int32_t k, const double *b, double *x, double *p, double *r,
                 double *Ap, double *state, double *hist, int32_t *niters) {
  const Reduction red{S->d_partials, S->d_counter};
  const int g = small_grid(S, S->nrow);
  switch (step) {
    case HPCCG_SLAB_START:
      k_slab_start<<<g, kBlock, 0, S->stream>>>(S->nrow, x, p);
      break;
    case HPCCG_SLAB_PREPARE:  // Ap = A p, r = b - Ap, local r.r
      k_slab_spmv<false><<<S->grid, kBlock, 0, S->stream>>>(S->nrow, S->npad, S->width, S->d_col, S->d_val, p, Ap,
                                                             red, nullptr, nullptr);
      k_slab_residual<<<g, kBlock, 0, S->stream>>>(S->nrow, b, Ap, r);
      k_slab_dot1<<<S->grid, kBlock, 0, S->stream>>>(S->nrow, r, red, state + kLocal, nullptr);
      break;
    case HPCCG_SLAB_PREPARED:
      k_slab_prepared<<<1, 1, 0, S->stream>>>(state, hist);
      break;
    case HPCCG_SLAB_BEGIN:
      k_slab_begin<<<g, kBlock, 0, S->stream>>>(S->nrow, k, r, p, state, hist, niters);
      k_slab_begin_scalars<<<1, 1, 0, S->stream>>>(k, state);
      break;
    case HPCCG_SLAB_SPMV:  // Ap = A p and the local p.Ap
      k_slab_spmv<true><<<S->grid, kBlock, 0, S->stream>>>(S->nrow, S->npad, S->width, S->d_col, S->d_val, p, Ap,
                                                            red, state + kLocal, state);
      break;
    case HPCCG_SLAB_UPDATE:  // r -= alpha Ap, x += alpha p, local r.r
      k_slab_update<<<g, kBlock, 0, S->stream>>>(S->nrow, p, Ap, r, x, state);
      k_slab_dot1<<<S->grid, kBlock, 0, S->stream>>>(S->nrow, r, red, state + kLocal, state);
      break;
    default:
      return HPCCG_ERR_INVALID_ARG;
  }
  HPCCG_CUDA(cudaGetLastError());
  return HPCCG_OK;
}

}  // namespace

extern "C" int hpccg_slab_spmv(hpccg_slab *S, const double *d_x, double *d_y) {
  if (!S || !d_x || !d_y) return HPCCG_ERR_INVALID_ARG;
  DevGuard dg(S->device);
  const Reduction red{S->d_partials, S->d_counter};
  k_slab_spmv<false><<<S->grid, kBlock, 0, S->stream>>>(S->nrow, S->npad, S->width, S->d_col, S->d_val, d_x, d_y,
                                                         red, nullptr, nullptr);
  HPCCG_CUDA(cudaGetLastError());
  HPCCG_CUDA(cudaStreamSynchronize(S->stream));
  return HPCCG_OK;
}

extern "C" int hpccg_slab_pack(hpccg_slab *S, const double *d_x, double *d_sendbuf) {
  if (!S || !d_x || (S->nsend > 0 && !d_sendbuf) || S->mode != HPCCG_HALO_MPI) return HPCCG_ERR_INVALID_ARG;
  if (S->nsend == 0) return HPCCG_OK;
  DevGuard dg(S->device);
  k_slab_pack<<<small_grid(S, S->nsend), kBlock, 0, S->stream>>>(S->nsend, S->d_send, d_x, d_sendbuf, nullptr);
  HPCCG_CUDA(cudaGetLastError());
  HPCCG_CUDA(cudaStreamSynchronize(S->stream));
  return HPCCG_OK;
}

extern "C" int hpccg_slab_scatter_block(hpccg_slab *S, int32_t block, const double *d_range, double *d_x) {
  const int32_t nb = S ? (int32_t)(S->blocks.size() / 4) : 0;
  if (!S || S->mode != HPCCG_HALO_GET || block < 0 || block >= nb || !d_range || !d_x) return HPCCG_ERR_INVALID_ARG;
  DevGuard dg(S->device);
  const int32_t first = S->blocks[4 * block + 1] - 1;
  const int32_t end = block + 1 < nb ? S->blocks[4 * (block + 1) + 1] - 1 : S->ncol - S->nrow;
  k_slab_scatter<<<small_grid(S, end - first), kBlock, 0, S->stream>>>(first, end - first, S->d_remote, d_range,
                                                                      d_x + S->nrow, nullptr);
  HPCCG_CUDA(cudaGetLastError());
  HPCCG_CUDA(cudaStreamSynchronize(S->stream));
  return HPCCG_OK;
}

extern "C" int hpccg_slab_cg_step(hpccg_slab *S, int32_t step, int32_t k, const double *d_b, double *d_x,
                                  double *d_p, double *d_r, double *d_Ap, double *d_state, double *d_hist) {
  if (!S || !d_state || !d_p || !d_r || !d_Ap || !d_x || (step == HPCCG_SLAB_PREPARE && !d_b))
    return HPCCG_ERR_INVALID_ARG;
  DevGuard dg(S->device);
  const int rc = enqueue_step(S, step, k, d_b, d_x, d_p, d_r, d_Ap, d_state, d_hist, nullptr);
  if (rc) return rc;
  HPCCG_CUDA(cudaStreamSynchronize(S->stream));
  return HPCCG_OK;
}

// ===========================================================================
// All ranks in this process
// ===========================================================================

namespace {

struct GroupRank {
  hpccg_slab *S;
  double *p = nullptr, *r = nullptr, *Ap = nullptr, *state = nullptr, *gather = nullptr, *hist = nullptr;
  int32_t *niters = nullptr;
  cudaEvent_t ev = nullptr;
};

// make every rank's stream wait for everything enqueued so far on all streams
int all_wait_all(std::vector<GroupRank> &R) {
  if (R.size() == 1) return HPCCG_OK;
  for (auto &g : R) {
    DevGuard dg(g.S->device);
    HPCCG_CUDA(cudaEventRecord(g.ev, g.S->stream));
  }
  for (auto &g : R) {
    DevGuard dg(g.S->device);
    for (auto &h : R)
      if (&g != &h) HPCCG_CUDA(cudaStreamWaitEvent(g.S->stream, h.ev, 0));
  }
  return HPCCG_OK;
}

// exchange_externals of p on every rank, by device copies
int group_exchange(std::vector<GroupRank> &R) {
  const int32_t P = (int32_t)R.size();
  if (R[0].S->mode == HPCCG_HALO_MPI) {
    for (auto &g : R) {  // pack each rank's send buffer (:664-666)
      hpccg_slab *S = g.S;
      if (S->nsend == 0) continue;
      DevGuard dg(S->device);
      k_slab_pack<<<small_grid(S, S->nsend), kBlock, 0, S->stream>>>(S->nsend, S->d_send, g.p, S->d_stage, g.state);
      HPCCG_CUDA(cudaGetLastError());
    }
    if (int rc = all_wait_all(R)) return rc;
    for (int32_t q = 0; q < P; ++q) {  // the receives of rank q (:647-653)
      hpccg_slab *S = R[q].S;
      DevGuard dg(S->device);
      int64_t off = 0;
      for (size_t i = 0; i < S->neighbors.size(); ++i) {
        const hpccg_slab *N = R[S->neighbors[i]].S;
        int64_t soff = 0;
        size_t slot = 0;
        for (; slot < N->neighbors.size() && N->neighbors[slot] != q; ++slot) soff += N->send_length[slot];
        if (slot == N->neighbors.size() || N->send_length[slot] != S->recv_length[i]) return HPCCG_ERR_INVALID_ARG;
        HPCCG_CUDA(cudaMemcpyPeerAsync(R[q].p + S->nrow + off, S->device, N->d_stage + soff, N->device,
                                       S->recv_length[i] * sizeof(double), S->stream));
        off += S->recv_length[i];
      }
    }
  } else {
    if (int rc = all_wait_all(R)) return rc;
    for (int32_t q = 0; q < P; ++q) {  // one contiguous get per block, then the scatter (:360-367)
      hpccg_slab *S = R[q].S;
      DevGuard dg(S->device);
      const int32_t nb = (int32_t)(S->blocks.size() / 4);
      for (int32_t b = 0; b < nb; ++b) {
        const int32_t owner = S->blocks[4 * b], inmin = S->blocks[4 * b + 2], inmax = S->blocks[4 * b + 3];
        const hpccg_slab *N = R[owner].S;
        HPCCG_CUDA(cudaMemcpyPeerAsync(S->d_stage, S->device, R[owner].p + (inmin - 1), N->device,
                                       (size_t)(inmax - inmin + 1) * sizeof(double), S->stream));
        const int32_t first = S->blocks[4 * b + 1] - 1;
        const int32_t end = b + 1 < nb ? S->blocks[4 * (b + 1) + 1] - 1 : S->ncol - S->nrow;
        k_slab_scatter<<<small_grid(S, end - first), kBlock, 0, S->stream>>>(first, end - first, S->d_remote,
                                                                            S->d_stage, R[q].p + S->nrow,
                                                                            R[q].state);
        HPCCG_CUDA(cudaGetLastError());
      }
    }
  }
  return all_wait_all(R);  // p complete everywhere before any SpMV reads it, and stage free again
}

// state[kGlobal] on every rank = the ranks' state[kLocal] folded in rank order
int group_allreduce(std::vector<GroupRank> &R) {
  const int32_t P = (int32_t)R.size();
  if (int rc = all_wait_all(R)) return rc;
  GroupRank &g0 = R[0];
  {
    DevGuard dg(g0.S->device);
    for (int32_t q = 0; q < P; ++q)
      HPCCG_CUDA(cudaMemcpyPeerAsync(g0.gather + q, g0.S->device, R[q].state + kLocal, R[q].S->device,
                                     sizeof(double), g0.S->stream));
    k_slab_fold<<<1, 1, 0, g0.S->stream>>>(g0.gather, P, g0.state);
    HPCCG_CUDA(cudaGetLastError());
  }
  if (int rc = all_wait_all(R)) return rc;
  for (int32_t q = 1; q < P; ++q) {
    DevGuard dg(R[q].S->device);
    HPCCG_CUDA(cudaMemcpyPeerAsync(R[q].state + kGlobal, R[q].S->device, g0.state + kGlobal, g0.S->device,
                                   sizeof(double), R[q].S->stream));
  }
  return all_wait_all(R);
}

}  // namespace

extern "C" int hpccg_slab_group_cg(hpccg_slab *const *slabs, int32_t nslabs, const double *const *d_b,
                                   double *const *d_x, int32_t max_iter, double tolerance, int32_t *niters,
                                   double *normr, double *resid_hist) {
  if (!slabs || nslabs < 1 || !d_b || !d_x || max_iter < 0 || !niters || !normr) return HPCCG_ERR_INVALID_ARG;
  for (int32_t q = 0; q < nslabs; ++q)
    if (!slabs[q] || slabs[q]->rank != q || slabs[q]->nranks != nslabs || slabs[q]->mode != slabs[0]->mode ||
        !d_b[q] || !d_x[q])
      return HPCCG_ERR_INVALID_ARG;
  std::vector<GroupRank> R(nslabs);
  int rc = HPCCG_OK;
  auto cleanup = [&]() {
    for (auto &g : R) {
      if (!g.S) continue;
      DevGuard dg(g.S->device);
      cudaStreamSynchronize(g.S->stream);
      cudaFree(g.p);
      cudaFree(g.r);
      cudaFree(g.Ap);
      cudaFree(g.state);
      if (g.ev) cudaEventDestroy(g.ev);
    }
  };
  for (int32_t q = 0; q < nslabs && !rc; ++q) {
    GroupRank &g = R[q];
    g.S = slabs[q];
    DevGuard dg(g.S->device);
    // p (ncol) | r | Ap; state (8) | gather (nslabs) | niters | hist (max_iter + 1)
    if (cudaMalloc(&g.p, (size_t)g.S->ncol * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&g.r, (size_t)g.S->nrow * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&g.Ap, (size_t)g.S->nrow * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&g.state, (size_t)(8 + nslabs + 1 + max_iter + 1) * sizeof(double)) != cudaSuccess) {
      cudaGetLastError();
      rc = HPCCG_ERR_OOM;
      break;
    }
    g.gather = g.state + 8;
    g.niters = reinterpret_cast<int32_t *>(g.state + 8 + nslabs);
    g.hist = g.state + 8 + nslabs + 1;
    if (cudaMemset(g.p, 0, (size_t)g.S->ncol * sizeof(double)) != cudaSuccess ||
        cudaMemset(g.state, 0, (size_t)(8 + nslabs + 1 + max_iter + 1) * sizeof(double)) != cudaSuccess ||
        cudaEventCreateWithFlags(&g.ev, cudaEventDisableTiming) != cudaSuccess) {
      rc = set_cuda_error(cudaGetLastError(), "slab group set-up", __FILE__, __LINE__);
      break;
    }
    const double tol_done[2] = {tolerance, 0.0};
    if (cudaMemcpy(g.state + kTol, &tol_done[0], sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess) {
      rc = set_cuda_error(cudaGetLastError(), "slab group set-up", __FILE__, __LINE__);
      break;
    }
  }
  auto each = [&](int32_t step, int32_t k) -> int {
    for (int32_t q = 0; q < nslabs; ++q) {
      DevGuard dg(R[q].S->device);
      const int e = enqueue_step(R[q].S, step, k, d_b[q], d_x[q], R[q].p, R[q].r, R[q].Ap, R[q].state,
                                 q == 0 ? R[q].hist : nullptr, q == 0 ? R[q].niters : nullptr);
      if (e) return e;
    }
    return HPCCG_OK;
  };
  // prepare (:91-98)
  if (!rc) rc = each(HPCCG_SLAB_START, 0);
  if (!rc) rc = group_exchange(R);
  if (!rc) rc = each(HPCCG_SLAB_PREPARE, 0);
  if (!rc) rc = group_allreduce(R);
  if (!rc) rc = each(HPCCG_SLAB_PREPARED, 0);
  // the loop (:108-147); every step becomes a no-op once rank 0's begin has
  // seen normr < tolerance (all ranks hold the same normr); the host checks
  // the flag every 16 iterations
  for (int32_t k = 1; k <= max_iter && !rc; ++k) {
    rc = each(HPCCG_SLAB_BEGIN, k);
    if (!rc) rc = group_exchange(R);
    if (!rc) rc = each(HPCCG_SLAB_SPMV, k);
    if (!rc) rc = group_allreduce(R);
    if (!rc) rc = each(HPCCG_SLAB_UPDATE, k);
    if (!rc) rc = group_allreduce(R);
    if (!rc && (k % 16 == 0 || k == max_iter)) {
      double done = 0.0;
      DevGuard dg(R[0].S->device);
      if (cudaMemcpyAsync(&done, R[0].state + kDone, sizeof(double), cudaMemcpyDeviceToHost, R[0].S->stream) !=
              cudaSuccess ||
          cudaStreamSynchronize(R[0].S->stream) != cudaSuccess) {
        rc = set_cuda_error(cudaGetLastError(), "slab group loop", __FILE__, __LINE__);
        break;
      }
      if (done != 0.0) break;
    }
  }
  if (!rc) {
    DevGuard dg(R[0].S->device);
    double st[8];
    int32_t it = 0;
    if (cudaStreamSynchronize(R[0].S->stream) != cudaSuccess ||
        cudaMemcpy(st, R[0].state, sizeof st, cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(&it, R[0].niters, sizeof it, cudaMemcpyDeviceToHost) != cudaSuccess ||
        (resid_hist && cudaMemcpy(resid_hist, R[0].hist, (size_t)(it + 1) * sizeof(double),
                                  cudaMemcpyDeviceToHost) != cudaSuccess)) {
      rc = set_cuda_error(cudaGetLastError(), "slab group result", __FILE__, __LINE__);
    } else {
      *niters = it;
      *normr = st[kNormr];
      if (!std::isfinite(st[kNormr])) rc = HPCCG_ERR_BREAKDOWN;
    }
  }
  for (auto &g : R)
    if (g.S) {
      DevGuard dg(g.S->device);
      cudaStreamSynchronize(g.S->stream);
    }
  cleanup();
  return rc;
}

extern "C" int hpccg_slab_group_cg_host(hpccg_slab *const *slabs, int32_t nslabs, const double *const *b,
                                        double *const *x, int32_t max_iter, double tolerance, int32_t *niters,
                                        double *normr, double *resid_hist) {
  if (!slabs || nslabs < 1 || !b || !x) return HPCCG_ERR_INVALID_ARG;
  for (int32_t q = 0; q < nslabs; ++q)
    if (!slabs[q] || !b[q] || !x[q]) return HPCCG_ERR_INVALID_ARG;
  std::vector<double *> db(nslabs, nullptr), dx(nslabs, nullptr);
  int rc = HPCCG_OK;
  for (int32_t q = 0; q < nslabs && !rc; ++q) {
    DevGuard dg(slabs[q]->device);
    const size_t bytes = (size_t)slabs[q]->nrow * sizeof(double);
    if (cudaMalloc(&db[q], bytes) != cudaSuccess || cudaMalloc(&dx[q], bytes) != cudaSuccess) {
      cudaGetLastError();
      rc = HPCCG_ERR_OOM;
    } else if (cudaMemcpy(db[q], b[q], bytes, cudaMemcpyHostToDevice) != cudaSuccess ||
               cudaMemcpy(dx[q], x[q], bytes, cudaMemcpyHostToDevice) != cudaSuccess) {
      rc = set_cuda_error(cudaGetLastError(), "slab group upload", __FILE__, __LINE__);
    }
  }
  if (!rc) {
    rc = hpccg_slab_group_cg(slabs, nslabs, db.data(), dx.data(), max_iter, tolerance, niters, normr, resid_hist);
    if (rc == HPCCG_OK || rc == HPCCG_ERR_BREAKDOWN)
      for (int32_t q = 0; q < nslabs; ++q) {
        DevGuard dg(slabs[q]->device);
        if (cudaMemcpy(x[q], dx[q], (size_t)slabs[q]->nrow * sizeof(double), cudaMemcpyDeviceToHost) !=
            cudaSuccess) {
          rc = set_cuda_error(cudaGetLastError(), "slab group download", __FILE__, __LINE__);
          break;
        }
      }
  }
  for (int32_t q = 0; q < nslabs; ++q) {
    DevGuard dg(slabs[q]->device);
    cudaFree(db[q]);
    cudaFree(dx[q]);
  }
  return rc;
}

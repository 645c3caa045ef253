// Device-side construction of the evaluation work lists of a geometry
// (fmmb_set_geometry): the tensor-core M2L's pair tiles and the CSR of its
// per-box reduction, the near-field work items, the inverse target
// permutation.  Scans and stable radix sorts (tree.cu) over the device lists
// the tree build produced, so that none of it is copied to the host; the
// results are the ones the former host loops gave (same orders, ties kept in
// input order).
//
// The lists restate the work of the reference's fmm() driver
// (fmm/fmm.cxx:29-152: ijbox's lists per level, kernel/m2l.cxx:13-93 over
// them) in the order the kernels want it.
#include <cuda_runtime.h>

#include <vector>

#include "internal.h"
#include "kernels.h"

namespace fmmb {
namespace {

constexpr int kT = 256;
constexpr int kMaxLev = 12;

inline unsigned nblk(long long n, int t) { return (unsigned)((n + t - 1) / t); }
inline int bits_for(long long n) {  // bits to hold values in [0, n)
  int b = 1;
  while ((1LL << b) < n) b++;
  return b;
}

// The (level, box, slot) enumeration of the M2L pairs: levels 2..lmax
// ascending, boxes of a level in order, the 189 slots of a box in order.
struct LevTab {
  int nlev;                // levels 2..lmax
  int vstart[kMaxLev + 1]; // first virtual index of level lev - 2 (vstart[nlev] = total)
  int boxoff[kMaxLev];     // first box of the level in the all-level target arrays
  int srcoff[kMaxLev];     // first box of the level in the all-level source arrays
  int set[kMaxLev];        // operator set of the level
};

__device__ __forceinline__ void lev_of(const LevTab& T, int v, int& l, int& b, int& sl) {
  l = 0;
  while (l + 1 < T.nlev && T.vstart[l + 1] <= v) l++;
  const int r = v - T.vstart[l];
  b = r / kM2LSlots;
  sl = r - b * kM2LSlots;
}

__global__ void m2l_pair_flags(int V, LevTab T, const int* __restrict__ lst, int* __restrict__ flag) {
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= V) return;
  int l, b, sl;
  lev_of(T, v, l, b, sl);
  flag[v] = lst[(size_t)(T.boxoff[l] + b) * kM2LSlots + sl] >= 0 ? 1 : 0;
}

// pair k (in enumeration order) -> operator key, source row, target row
__global__ void m2l_pair_emit(int V, LevTab T, const int* __restrict__ lst, const int* __restrict__ key_i,
                              const int* __restrict__ slot_rel, const int* __restrict__ rel_to_op,
                              const int* __restrict__ pos, int* __restrict__ opk, int* __restrict__ ord,
                              int* __restrict__ src, int* __restrict__ dst) {
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= V) return;
  int l, b, sl;
  lev_of(T, v, l, b, sl);
  const int box = T.boxoff[l] + b;
  const int s = lst[(size_t)box * kM2LSlots + sl];
  if (s < 0) return;
  const int k = pos[v];
  opk[k] = T.set[l] * 316 + rel_to_op[slot_rel[(key_i[box] & 7) * kM2LSlots + sl]];
  ord[k] = k;
  src[k] = T.srcoff[l] + s;
  dst[k] = box;
}

__global__ void count_keys(int n, const int* __restrict__ key, int* __restrict__ cnt) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j < n) atomicAdd(&cnt[key[j]], 1);
}

__global__ void tiles_per_key(int nk, const int* __restrict__ cnt, int* __restrict__ tiles) {
  const int o = blockIdx.x * blockDim.x + threadIdx.x;
  if (o < nk) tiles[o] = (cnt[o] + 127) / 128;
}

// sorted pair j -> tile tile_base[op] + r / 128, column r % 128 (r = its rank
// among the pairs of its operator)
__global__ void fill_tiles(int n, const int* __restrict__ opk, const int* __restrict__ ord,
                           const int* __restrict__ src, const int* __restrict__ dst, const int* __restrict__ op_start,
                           const int* __restrict__ tile_base, int* __restrict__ tile_op, int* __restrict__ tile_src,
                           int* __restrict__ tdst) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  const int op = opk[j], r = j - op_start[op];
  const int t = tile_base[op] + r / 128, c = r % 128;
  tile_src[(size_t)t * 128 + c] = src[ord[j]];
  tdst[(size_t)t * 128 + c] = dst[ord[j]];
  if (c == 0) tile_op[t] = op;
}

__global__ void fill_tile_y(int ntile, int* __restrict__ ty) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= ntile) return;
  ty[2 * t] = t * 128;
  ty[2 * t + 1] = 0;
}

__global__ void nonneg_flags(int n, const int* __restrict__ a, int* __restrict__ flag) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n) flag[k] = a[k] >= 0 ? 1 : 0;
}

// column k of the tiles with a target -> (target row, k), in k order
__global__ void compact_cols(int n, const int* __restrict__ tdst, const int* __restrict__ pos,
                             int* __restrict__ rowk, int* __restrict__ colk) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n || tdst[k] < 0) return;
  rowk[pos[k]] = tdst[k];
  colk[pos[k]] = k;
}

__global__ void run_starts(int n, const int* __restrict__ key, int* __restrict__ flag) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m < n) flag[m] = (m == 0 || key[m] != key[m - 1]) ? 1 : 0;
}

__global__ void emit_runs(int n, const int* __restrict__ key, const int* __restrict__ pos, int* __restrict__ rows,
                          int* __restrict__ ptr) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= n) return;
  const bool st = m == 0 || key[m] != key[m - 1];  // pos[m]: the runs started before m
  if (st) {
    rows[pos[m]] = key[m];
    ptr[pos[m]] = m;
  }
  if (m == n - 1) ptr[pos[m] + (st ? 1 : 0)] = n;
}

// ---- near-field work items ----
__global__ void leaf_item_counts(int nleaf, const int2* __restrict__ leaf_i, const int2* __restrict__ leaf_j,
                                 const int* __restrict__ list, int* __restrict__ cnt, long long* __restrict__ nsrc) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nleaf) return;
  long long s = 0;
  for (int sl = 0; sl < kP2PSlots; sl++) {
    const int jl = list[(size_t)b * kP2PSlots + sl];
    if (jl >= 0) s += leaf_j[jl].y;
  }
  nsrc[b] = s > 0 ? s : 1;
  cnt[b] = (leaf_i[b].y + 127) / 128;
}

// items of leaf b in leaf order; the sort key puts the heaviest first
__global__ void leaf_items(int nleaf, const int2* __restrict__ leaf_i, const long long* __restrict__ nsrc,
                           const int* __restrict__ base, int2* __restrict__ work, int* __restrict__ skey,
                           int* __restrict__ sval) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nleaf) return;
  const int n = leaf_i[b].y;
  for (int t = 0, k = base[b]; t < n; t += 128, k++) {
    const long long cost = (long long)min(128, n - t) * nsrc[b];
    const long long cap = (1LL << 30) - 1;
    work[k] = make_int2(b, t);
    skey[k] = (int)(cap - (cost < cap ? cost : cap));
    sval[k] = k;
  }
}

// ---- P2M work items: pieces of up to `per` sources of a source leaf ----
__global__ void src_item_counts(int nleaf, int per, const int2* __restrict__ leaf_j, int* __restrict__ cnt) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b < nleaf) cnt[b] = (leaf_j[b].y + per - 1) / per;
}

__global__ void src_items(int nleaf, int per, const int2* __restrict__ leaf_j, const int* __restrict__ base,
                          int2* __restrict__ work) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nleaf) return;
  const int n = leaf_j[b].y;
  for (int t = 0, k = base[b]; t < n; t += per, k++) work[k] = make_int2(b, t);
}

// sorted item j -> launch (j & 1), position j >> 1 within it
__global__ void deal_items(int n, int n0, const int* __restrict__ sorted, const int2* __restrict__ work,
                           int2* __restrict__ out) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  out[(j & 1) ? n0 + (j >> 1) : (j >> 1)] = work[sorted[j]];
}

__global__ void invert_perm(int n, const int* __restrict__ perm, int* __restrict__ inv) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) inv[perm[i]] = i;
}

int d2h_int(const int* p, cudaStream_t s) {
  int h = 0;
  FMMB_CUDA(cudaMemcpyAsync(&h, p, sizeof(int), cudaMemcpyDeviceToHost, s));
  FMMB_CUDA(cudaStreamSynchronize(s));
  return h;
}

}  // namespace

bool build_m2l_job_dev(fmmb_plan* pl, fmmb_plan::TcJob& job, int ys, cudaStream_t s) {
  const int lmax = pl->lmax;
  if (lmax - 1 > kMaxLev) return false;
  LevTab T{};
  long long V = 0;
  T.nlev = 0;
  for (int lev = 2; lev <= lmax; lev++) {
    const int l = T.nlev++;
    T.vstart[l] = (int)V;
    T.boxoff[l] = pl->off_i[lev];
    T.srcoff[l] = pl->off_j[lev];
    T.set[l] = pl->ops.m2l_sets > 1 ? lev - 2 : 0;
    V += (long long)pl->nbox_i[lev] * kM2LSlots;
  }
  if (V >= (1LL << 31) - 1) return false;  // the host loops take such sizes
  T.vstart[T.nlev] = (int)V;
  const int nv = (int)V;
  const int nops = pl->ops.m2l_sets * 316;
  TmpBuf<int> pos(s);
  pos.alloc((size_t)nv + 1);
  m2l_pair_flags<<<nblk(nv, kT), kT, 0, s>>>(nv, T, pl->m2l_list.get(), pos.get());
  FMMB_CHECK_LAUNCH();
  FMMB_CUDA(cudaMemsetAsync(pos.get() + nv, 0, sizeof(int), s));
  exclusive_scan(pos.get(), nv + 1, s);
  const int npair = d2h_int(pos.get() + nv, s);
  TmpBuf<int> opk(s), ord(s), src(s), dst(s);
  opk.alloc(npair);
  ord.alloc(npair);
  src.alloc(npair);
  dst.alloc(npair);
  m2l_pair_emit<<<nblk(nv, kT), kT, 0, s>>>(nv, T, pl->m2l_list.get(), pl->key_i.get(), pl->d_slot_rel.get(),
                                           pl->d_rel_to_op.get(), pos.get(), opk.get(), ord.get(), src.get(),
                                           dst.get());
  FMMB_CHECK_LAUNCH();
  radix_sort(opk.get(), ord.get(), npair, bits_for(nops), s);  // stable: enumeration order within an operator
  // tiles of 128 pairs per operator
  TmpBuf<int> cnt(s), op_start(s), tile_base(s);
  cnt.alloc(nops + 1);
  op_start.alloc(nops + 1);
  tile_base.alloc(nops + 1);
  FMMB_CUDA(cudaMemsetAsync(cnt.get(), 0, (nops + 1) * sizeof(int), s));
  if (npair > 0) {
    count_keys<<<nblk(npair, kT), kT, 0, s>>>(npair, opk.get(), cnt.get());
    FMMB_CHECK_LAUNCH();
  }
  FMMB_CUDA(cudaMemcpyAsync(op_start.get(), cnt.get(), (nops + 1) * sizeof(int), cudaMemcpyDeviceToDevice, s));
  tiles_per_key<<<nblk(nops + 1, kT), kT, 0, s>>>(nops + 1, cnt.get(), tile_base.get());
  FMMB_CHECK_LAUNCH();
  exclusive_scan(op_start.get(), nops + 1, s);
  exclusive_scan(tile_base.get(), nops + 1, s);
  const int ntile = d2h_int(tile_base.get() + nops, s);
  job.ntile = ntile;
  job.tile_op.alloc(std::max(ntile, 1));
  job.tile_src.alloc((size_t)std::max(ntile, 1) * 128);
  job.tile_y.alloc((size_t)std::max(ntile, 1) * 2);
  TmpBuf<int> tdst(s);
  tdst.alloc((size_t)std::max(ntile, 1) * 128);
  FMMB_CUDA(cudaMemsetAsync(job.tile_src.get(), 0xff, (size_t)ntile * 128 * sizeof(int), s));
  FMMB_CUDA(cudaMemsetAsync(tdst.get(), 0xff, (size_t)ntile * 128 * sizeof(int), s));
  if (npair > 0) {
    fill_tiles<<<nblk(npair, kT), kT, 0, s>>>(npair, opk.get(), ord.get(), src.get(), dst.get(), op_start.get(),
                                             tile_base.get(), job.tile_op.get(), job.tile_src.get(), tdst.get());
    FMMB_CHECK_LAUNCH();
  }
  if (ntile > 0) {
    fill_tile_y<<<nblk(ntile, kT), kT, 0, s>>>(ntile, job.tile_y.get());
    FMMB_CHECK_LAUNCH();
  }
  // per output box, its pair rows (tile * 128 + column) in increasing order
  const int ncol = ntile * 128;
  TmpBuf<int> cpos(s);
  cpos.alloc((size_t)ncol + 1);
  if (ncol > 0) {
    nonneg_flags<<<nblk(ncol, kT), kT, 0, s>>>(ncol, tdst.get(), cpos.get());
    FMMB_CHECK_LAUNCH();
  }
  FMMB_CUDA(cudaMemsetAsync(cpos.get() + ncol, 0, sizeof(int), s));
  exclusive_scan(cpos.get(), ncol + 1, s);
  TmpBuf<int> rowk(s), colk(s);
  rowk.alloc(std::max(npair, 1));
  colk.alloc(std::max(npair, 1));
  if (ncol > 0) {
    compact_cols<<<nblk(ncol, kT), kT, 0, s>>>(ncol, tdst.get(), cpos.get(), rowk.get(), colk.get());
    FMMB_CHECK_LAUNCH();
  }
  radix_sort(rowk.get(), colk.get(), npair, bits_for(pl->tot_i), s);
  TmpBuf<int> rpos(s);
  rpos.alloc((size_t)npair + 1);
  if (npair > 0) {
    run_starts<<<nblk(npair, kT), kT, 0, s>>>(npair, rowk.get(), rpos.get());
    FMMB_CHECK_LAUNCH();
  }
  FMMB_CUDA(cudaMemsetAsync(rpos.get() + npair, 0, sizeof(int), s));
  exclusive_scan(rpos.get(), npair + 1, s);
  const int nred = d2h_int(rpos.get() + npair, s);
  job.nred = nred;
  job.red_rows.alloc(std::max(nred, 1));
  job.red_ptr.alloc((size_t)nred + 1);
  if (npair > 0) {
    emit_runs<<<nblk(npair, kT), kT, 0, s>>>(npair, rowk.get(), rpos.get(), job.red_rows.get(), job.red_ptr.get());
    FMMB_CHECK_LAUNCH();
  } else {
    FMMB_CUDA(cudaMemsetAsync(job.red_ptr.get(), 0, sizeof(int), s));
  }
  job.red_idx.alloc(std::max(npair, 1));
  if (npair > 0)
    FMMB_CUDA(cudaMemcpyAsync(job.red_idx.get(), colk.get(), (size_t)npair * sizeof(int), cudaMemcpyDeviceToDevice, s));
  job.ys = ys;
  pl->tc_y.alloc((size_t)std::max(ntile, 1) * 128 * ys);
  FMMB_CUDA(cudaStreamSynchronize(s));
  return true;
}

void build_p2p_work_dev(fmmb_plan* pl, cudaStream_t s) {
  const int nleaf = pl->nbox_i[pl->lmax];
  TmpBuf<int> cnt(s);
  TmpBuf<long long> nsrc(s);
  cnt.alloc((size_t)nleaf + 1);
  nsrc.alloc(std::max(nleaf, 1));
  FMMB_CUDA(cudaMemsetAsync(cnt.get() + nleaf, 0, sizeof(int), s));
  if (nleaf > 0) {
    leaf_item_counts<<<nblk(nleaf, kT), kT, 0, s>>>(nleaf, pl->leaf_i.get(), pl->leaf_j.get(), pl->p2p_list.get(),
                                                   cnt.get(), nsrc.get());
    FMMB_CHECK_LAUNCH();
  }
  exclusive_scan(cnt.get(), nleaf + 1, s);
  const int n = d2h_int(cnt.get() + nleaf, s);
  pl->m_p2p_work.alloc(std::max(n, 1));
  pl->m_p2p_nwork = n;
  TmpBuf<int> skey(s), sval(s);
  skey.alloc(std::max(n, 1));
  sval.alloc(std::max(n, 1));
  if (nleaf > 0) {
    leaf_items<<<nblk(nleaf, kT), kT, 0, s>>>(nleaf, pl->leaf_i.get(), nsrc.get(), cnt.get(), pl->m_p2p_work.get(),
                                             skey.get(), sval.get());
    FMMB_CHECK_LAUNCH();
  }
  radix_sort(skey.get(), sval.get(), n, 30, s);  // stable: leaf order among equal costs
  const int n0 = (n + 1) / 2;
  pl->p2p_work.alloc(std::max(n, 1));
  if (n > 0) {
    deal_items<<<nblk(n, kT), kT, 0, s>>>(n, n0, sval.get(), pl->m_p2p_work.get(), pl->p2p_work.get());
    FMMB_CHECK_LAUNCH();
  }
  pl->p2p_nwork = n;
  pl->p2p_nwork0 = n0;
  FMMB_CUDA(cudaStreamSynchronize(s));
}

void build_p2m_work_dev(fmmb_plan* pl, cudaStream_t s) {
  const int nleaf = pl->nbox_j[pl->lmax], per = kP2MItem;
  TmpBuf<int> cnt(s);
  cnt.alloc((size_t)nleaf + 1);
  FMMB_CUDA(cudaMemsetAsync(cnt.get() + nleaf, 0, sizeof(int), s));
  if (nleaf > 0) {
    src_item_counts<<<nblk(nleaf, kT), kT, 0, s>>>(nleaf, per, pl->leaf_j.get(), cnt.get());
    FMMB_CHECK_LAUNCH();
  }
  exclusive_scan(cnt.get(), nleaf + 1, s);
  const int n = d2h_int(cnt.get() + nleaf, s);
  pl->p2m_work.alloc(std::max(n, 1));
  pl->p2m_nwork = n;
  if (nleaf > 0) {
    src_items<<<nblk(nleaf, kT), kT, 0, s>>>(nleaf, per, pl->leaf_j.get(), cnt.get(), pl->p2m_work.get());
    FMMB_CHECK_LAUNCH();
  }
  FMMB_CUDA(cudaStreamSynchronize(s));
}

void build_inverse_perm_dev(fmmb_plan* pl, cudaStream_t s) {
  pl->inv_i.alloc(std::max(pl->ni, 1));
  if (pl->ni > 0) {
    invert_perm<<<nblk(pl->ni, kT), kT, 0, s>>>(pl->ni, pl->perm_i.get(), pl->inv_i.get());
    FMMB_CHECK_LAUNCH();
  }
}

}  // namespace fmmb

// Octree construction on the GPU.
//
// Replaces the reference's serial tree build: box keys (fmm/boxn.cxx:5-31),
// the stable counting sort and the particle permutation (sort/csort.cxx:5-17,
// sort/sorti.cxx:12-35, sort/sortj.cxx:12-36), leaf ranges
// (fmm/boxdatai.cxx:10-34, fmm/boxdataj.cxx:10-36), parent levels
// (fmm/boxm2mi.cxx:6-24, fmm/boxm2mj.cxx:6-26) and the neighbour and
// interaction lists (fmm/ijbox.cxx:9-117).  The result is bit-identical to the
// reference: same keys (same float/double rounding), same stable order, same
// list entries in the same order.
//
// Lists are stored densely: 27 slots per target leaf for the near field and
// 189 slots per target box for M2L, -1 where the source box is empty.  The
// slot order is the reference's loop order, so dropping the -1 entries gives
// the reference lists.
//
// Forest (many independent problems in one plan): the problem index of a
// point sits above its 3*lmax Morton bits, so the sort groups the points by
// problem, every box belongs to one problem (its key at level l is
// (problem << 3l) | morton), and a neighbour or interaction-list lookup only
// finds boxes of the same problem.  With one problem the keys are the
// reference's.
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <cstring>
#include <mutex>

#include "internal.h"

namespace fmmb {

namespace {

constexpr int kScanThreads = 256;
constexpr int kScanItems = 4;
constexpr int kScanTile = kScanThreads * kScanItems;

// Exclusive scan of each tile; tile sums to `sums`.
__global__ void scan_tiles(int* data, int n, int* sums) {
  __shared__ int s[kScanThreads];
  const int base = blockIdx.x * kScanTile + threadIdx.x * kScanItems;
  int v[kScanItems];
  int t = 0;
#pragma unroll
  for (int i = 0; i < kScanItems; i++) {
    v[i] = (base + i < n) ? data[base + i] : 0;
    t += v[i];
  }
  s[threadIdx.x] = t;
  __syncthreads();
  for (int off = 1; off < kScanThreads; off <<= 1) {
    int x = (threadIdx.x >= off) ? s[threadIdx.x - off] : 0;
    __syncthreads();
    s[threadIdx.x] += x;
    __syncthreads();
  }
  int run = s[threadIdx.x] - t;
#pragma unroll
  for (int i = 0; i < kScanItems; i++) {
    if (base + i < n) data[base + i] = run;
    run += v[i];
  }
  if (threadIdx.x == kScanThreads - 1 && sums) sums[blockIdx.x] = s[threadIdx.x];
}

__global__ void scan_add(int* data, int n, const int* offs) {
  const int i = blockIdx.x * kScanTile + threadIdx.x;
  const int b = blockIdx.x;
  for (int k = 0; k < kScanItems; k++) {
    int j = i + k * kScanThreads;
    if (j < n) data[j] += offs[b];
  }
}

}  // namespace

// In-place exclusive scan (multi-level).
void exclusive_scan(int* data, int n, cudaStream_t s) {
  if (n <= 0) return;
  int nb = (n + kScanTile - 1) / kScanTile;
  if (nb == 1) {
    scan_tiles<<<1, kScanThreads, 0, s>>>(data, n, nullptr);
    FMMB_CHECK_LAUNCH();
    return;
  }
  TmpBuf<int> sums(s);  // freed in stream order
  sums.alloc(nb);
  scan_tiles<<<nb, kScanThreads, 0, s>>>(data, n, sums.get());
  FMMB_CHECK_LAUNCH();
  exclusive_scan(sums.get(), nb, s);
  scan_add<<<nb, kScanThreads, 0, s>>>(data, n, sums.get());
  FMMB_CHECK_LAUNCH();
}

cudaMemPool_t scratch_pool() {
  static std::mutex mu;
  static cudaMemPool_t pools[64] = {};
  int dev = 0;
  FMMB_CUDA(cudaGetDevice(&dev));
  FMMB_REQUIRE(dev >= 0 && dev < 64, FMMB_ERR_ARG, "device ordinal out of range");
  std::lock_guard<std::mutex> lk(mu);
  if (!pools[dev]) {
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t pool = nullptr;
    FMMB_CUDA(cudaMemPoolCreate(&pool, &props));
    uint64_t keep = kScratchPoolKeep;
    FMMB_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
    pools[dev] = pool;
  }
  return pools[dev];
}

namespace {

// ---- stable LSD radix sort of (key, index) ----
constexpr int kRsWarps = 8;
constexpr int kRsThreads = kRsWarps * 32;
constexpr int kRsRounds = 8;
constexpr int kRsTile = kRsThreads * kRsRounds;  // 2048

__global__ void rs_hist(const int* keys, int n, int shift, int nblocks, int* counts) {
  __shared__ int h[256];
  for (int d = threadIdx.x; d < 256; d += blockDim.x) h[d] = 0;
  __syncthreads();
  const int base = blockIdx.x * kRsTile;
  for (int i = threadIdx.x; i < kRsTile; i += blockDim.x)
    if (base + i < n) atomicAdd(&h[(keys[base + i] >> shift) & 255], 1);
  __syncthreads();
  for (int d = threadIdx.x; d < 256; d += blockDim.x) counts[d * nblocks + blockIdx.x] = h[d];
}

// Each warp owns a contiguous run of kRsRounds*32 elements, processed 32 at a
// time in order; ranks among equal digits come from __match_any_sync, so the
// scatter keeps the input order of equal keys (stable).
__global__ void rs_scatter(const int* kin, const int* vin, int* kout, int* vout, int n, int shift, int nblocks,
                           const int* offsets) {
  __shared__ int wc[kRsWarps][256];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int d = threadIdx.x; d < 256 * kRsWarps; d += blockDim.x) (&wc[0][0])[d] = 0;
  __syncthreads();
  const int base = blockIdx.x * kRsTile + w * (kRsRounds * 32);
  const unsigned lt = (1u << lane) - 1;
  int rank[kRsRounds], dig[kRsRounds], key[kRsRounds], val[kRsRounds];
#pragma unroll
  for (int r = 0; r < kRsRounds; r++) {
    const int i = base + r * 32 + lane;
    const bool ok = i < n;
    key[r] = ok ? kin[i] : 0;
    val[r] = ok ? vin[i] : 0;
    const int d = ok ? ((key[r] >> shift) & 255) : (256 + lane);
    dig[r] = d;
    const unsigned peers = __match_any_sync(0xffffffffu, d);
    const int before = __popc(peers & lt);
    const int prior = ok ? wc[w][d] : 0;
    __syncwarp();
    if (ok && before == 0) wc[w][d] = prior + __popc(peers);
    __syncwarp();
    rank[r] = prior + before;
  }
  __syncthreads();
  if (threadIdx.x < 256) {
    int run = 0;
    for (int ww = 0; ww < kRsWarps; ww++) {
      int t = wc[ww][threadIdx.x];
      wc[ww][threadIdx.x] = run;
      run += t;
    }
  }
  __syncthreads();
#pragma unroll
  for (int r = 0; r < kRsRounds; r++) {
    const int d = dig[r];
    if (d < 256) {
      const int pos = offsets[d * nblocks + blockIdx.x] + wc[w][d] + rank[r];
      kout[pos] = key[r];
      vout[pos] = val[r];
    }
  }
}

}  // namespace

void radix_sort(int* keys, int* vals, int n, int bits, cudaStream_t s) {
  if (n <= 1 || bits <= 0) return;
  const int nb = (n + kRsTile - 1) / kRsTile;
  TmpBuf<int> k2(s), v2(s), counts(s);
  k2.alloc(n);
  v2.alloc(n);
  counts.alloc((size_t)256 * nb);
  int *ka = keys, *va = vals, *kb = k2.get(), *vb = v2.get();
  int passes = 0;
  for (int shift = 0; shift < bits; shift += 8, passes++) {
    rs_hist<<<nb, kRsThreads, 0, s>>>(ka, n, shift, nb, counts.get());
    FMMB_CHECK_LAUNCH();
    exclusive_scan(counts.get(), 256 * nb, s);
    rs_scatter<<<nb, kRsThreads, 0, s>>>(ka, va, kb, vb, n, shift, nb, counts.get());
    FMMB_CHECK_LAUNCH();
    std::swap(ka, kb);
    std::swap(va, vb);
  }
  if (passes & 1) {
    FMMB_CUDA(cudaMemcpyAsync(keys, ka, n * sizeof(int), cudaMemcpyDeviceToDevice, s));
    FMMB_CUDA(cudaMemcpyAsync(vals, va, n * sizeof(int), cudaMemcpyDeviceToDevice, s));
  }
}

namespace {

// ---- keys (fmm/boxn.cxx:5-31) ----
__device__ __forceinline__ int morton(int cx, int cy, int cz, int lev) {
  int k = 0;
  for (int i = 0; i < lev; i++)
    k |= (((cx >> i) & 1) << (3 * i + 1)) | (((cy >> i) & 1) << (3 * i)) | (((cz >> i) & 1) << (3 * i + 2));
  return k;
}
__device__ __forceinline__ void demorton(int k, int& cx, int& cy, int& cz) {
  cx = cy = cz = 0;
  for (int i = 0; i < 10; i++) {
    cy |= ((k >> (3 * i)) & 1) << i;
    cx |= ((k >> (3 * i + 1)) & 1) << i;
    cz |= ((k >> (3 * i + 2)) & 1) << i;
  }
}

// The reference truncates (x - xmin) [float] * rb [double, from the float
// division kl/rd] and moves the last boundary back by one box.  Points below
// the root corner are clamped to box 0 (the reference leaves them undefined).
__device__ __forceinline__ int box_coord(float x, float xmin, double rb, int kl) {
  const float d = __fsub_rn(x, xmin);
  int c = (int)__dmul_rn((double)d, rb);
  if (c >= kl) c--;
  if (c >= kl) c = kl - 1;
  if (c < 0) c = 0;
  return c;
}

// off[0..nprob]: first point of each problem (off[nprob] = n)
__global__ void keys_kernel(int n, const float* x, const float* y, const float* z, float xmin, float ymin, float zmin,
                            double rb, int lmax, int nprob, const int* off, int* key, int* idx) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int kl = 1 << lmax;
  int pid = 0;
  if (nprob > 1) {  // last problem whose first point is <= i
    int lo = 0, hi = nprob - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (off[mid] <= i) lo = mid;
      else hi = mid - 1;
    }
    pid = lo;
  }
  key[i] = (pid << (3 * lmax)) |
           morton(box_coord(x[i], xmin, rb, kl), box_coord(y[i], ymin, rb, kl), box_coord(z[i], zmin, rb, kl), lmax);
  idx[i] = i;
}

// spatial part of the keys (problem bits removed)
__global__ void mask_keys(int n, const int* key, int mask, int* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = key[i] & mask;
}

__global__ void gather_points(int n, const int* perm, const float* x, const float* y, const float* z, const float* nx,
                              const float* ny, const float* nz, float4* pos, float4* nrm) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int o = perm[i];
  pos[i] = make_float4(x[o], y[o], z[o], 0.f);
  nrm[i] = nx ? make_float4(nx[o], ny[o], nz[o], 0.f) : make_float4(0.f, 0.f, 0.f, 0.f);
}

// flag[i] = 1 where a new run of (key >> shift) starts
__global__ void run_flags(int n, const int* key, int shift, int* flag, int* flag_copy) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int f = (i == 0 || (key[i] >> shift) != (key[i - 1] >> shift)) ? 1 : 0;
  flag[i] = f;
  flag_copy[i] = f;
}

// runs of a level = last scanned flag + last flag
__global__ void run_count(int n, const int* scanned, const int* flag_copy, int* count) {
  *count = n > 0 ? scanned[n - 1] + flag_copy[n - 1] : 0;
}

// After the exclusive scan of the flags: write compact keys, run starts and
// the run index of every element.
__global__ void run_compact(int n, const int* key, int shift, const int* scanned, const int* flag_copy, int* out_key,
                            int* out_first, int* elem_run) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int r = scanned[i] + flag_copy[i] - 1;
  if (elem_run) elem_run[i] = r;
  if (flag_copy[i]) {
    out_key[r] = key[i] >> shift;
    if (out_first) out_first[r] = i;
  }
}

__global__ void leaf_ranges(int nleaf, int n, const int* first, int2* leaf) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nleaf) return;
  const int f = first[b];
  const int e = (b + 1 < nleaf) ? first[b + 1] : n;
  leaf[b] = make_int2(f, e - f);
}

// child ranges of each parent (children of one parent are contiguous and
// every parent has at least one child): first the starts, then (next launch)
// the counts from consecutive starts.
__global__ void child_starts(int nchild, const int* parent, int* start) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nchild) return;
  const int p = parent[c];
  if (c == 0 || parent[c - 1] != p) start[p] = c;
}
__global__ void child_counts(int nparent, int nchild, const int* start, int* count) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= nparent) return;
  count[p] = ((p + 1 < nparent) ? start[p + 1] : nchild) - start[p];
}

__device__ __forceinline__ int find_key(const int* keys, int n, int k) {
  int lo = 0, hi = n;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (keys[mid] < k) lo = mid + 1;
    else hi = mid;
  }
  return (lo < n && keys[lo] == k) ? lo : -1;
}

// Near-field slots (fmm/ijbox.cxx:30-53): jx, jy, jz ascending over the 3x3x3
// neighbourhood, self included.
__global__ void p2p_lists(int nleaf_i, const int* key_i, int nleaf_j, const int* key_j, int lev, int* list) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nleaf_i) return;
  int ix, iy, iz;
  const int smask = (1 << (3 * lev)) - 1, prob = key_i[b] & ~smask;
  demorton(key_i[b] & smask, ix, iy, iz);
  const int kl = 1 << lev;
  int s = 0;
  for (int jx = ix - 1; jx <= ix + 1; jx++)
    for (int jy = iy - 1; jy <= iy + 1; jy++)
      for (int jz = iz - 1; jz <= iz + 1; jz++) {
        int v = -1;
        if (jx >= 0 && jx < kl && jy >= 0 && jy < kl && jz >= 0 && jz < kl)
          v = find_key(key_j, nleaf_j, prob | morton(jx, jy, jz, lev));
        list[(size_t)b * kP2PSlots + s++] = v;
      }
}

// Interaction-list slots (fmm/ijbox.cxx:74-109), relative offsets per octant
// from slot_rel.
__global__ void m2l_lists(int nbox_i, const int* key_i, int nbox_j, const int* key_j, int lev, const int* slot_rel,
                          int* list) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nbox_i * kM2LSlots) return;
  const int b = t / kM2LSlots, s = t % kM2LSlots;
  const int key = key_i[b];
  const int smask = (1 << (3 * lev)) - 1, prob = key & ~smask;
  int ix, iy, iz;
  demorton(key & smask, ix, iy, iz);
  const int code = slot_rel[(key & 7) * kM2LSlots + s];
  const int jx = ix - (code / 49 - 3), jy = iy - ((code / 7) % 7 - 3), jz = iz - (code % 7 - 3);
  const int kl = 1 << lev;
  int v = -1;
  if (jx >= 0 && jx < kl && jy >= 0 && jy < kl && jz >= 0 && jz < kl)
    v = find_key(key_j, nbox_j, prob | morton(jx, jy, jz, lev));
  list[t] = v;
}

__global__ void count_p2p_pairs(int nleaf_i, const int2* leaf_i, const int2* leaf_j, const int* list,
                                unsigned long long* out) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nleaf_i) return;
  unsigned long long acc = 0;
  for (int s = 0; s < kP2PSlots; s++) {
    const int j = list[(size_t)b * kP2PSlots + s];
    if (j >= 0) acc += (unsigned long long)leaf_i[b].y * (unsigned long long)leaf_j[j].y;
  }
  atomicAdd(out, acc);
}

__global__ void count_nonneg(size_t n, const int* list, unsigned long long* out) {
  size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  unsigned long long acc = 0;
  for (; i < n; i += (size_t)gridDim.x * blockDim.x) acc += list[i] >= 0;
  atomicAdd(out, acc);
}

__global__ void minmax_kernel(int n, const float* x, float* out /*[2] min,max*/) {
  float lo = FLT_MAX, hi = -FLT_MAX;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    lo = fminf(lo, x[i]);
    hi = fmaxf(hi, x[i]);
  }
  for (int o = 16; o; o >>= 1) {
    lo = fminf(lo, __shfl_xor_sync(0xffffffffu, lo, o));
    hi = fmaxf(hi, __shfl_xor_sync(0xffffffffu, hi, o));
  }
  if ((threadIdx.x & 31) == 0) {
    // order-preserving int encoding for atomics on floats
    int ilo = __float_as_int(lo), ihi = __float_as_int(hi);
    ilo = ilo >= 0 ? ilo : ilo ^ 0x7fffffff;
    ihi = ihi >= 0 ? ihi : ihi ^ 0x7fffffff;
    atomicMin((int*)&out[0], ilo);
    atomicMax((int*)&out[1], ihi);
  }
}

inline int blocks(size_t n, int t) { return (int)((n + t - 1) / t); }

__global__ void gather_int(int n, const int* idx, const int* src, int* dst) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) dst[i] = src[idx[i]];
}

struct Side {
  const float *x, *y, *z, *nx, *ny, *nz;
  int n;
  const int* off;  // device [nprob + 1] first point of each problem
};

int prob_bits(int nprob) {
  int b = 0;
  while ((1 << b) < nprob) b++;
  return b;
}

// Builds keys, order, sorted points and all levels of one point set.
void build_side(fmmb_plan* pl, const Side& sd, bool is_target, cudaStream_t s) {
  const int n = sd.n, lmax = pl->lmax;
  TmpBuf<int> key(s), idx(s), flag(s), flag2(s), nbd(s);
  key.alloc(n);
  idx.alloc(n);
  const double rb = (double)((float)(1 << lmax) / pl->bbox[3]);  // kl/rd: float division, as the reference
  keys_kernel<<<blocks(n, 256), 256, 0, s>>>(n, sd.x, sd.y, sd.z, pl->bbox[0], pl->bbox[1], pl->bbox[2], rb, lmax,
                                              pl->nprob, sd.off, key.get(), idx.get());
  FMMB_CHECK_LAUNCH();
  radix_sort(key.get(), idx.get(), n, 3 * lmax + prob_bits(pl->nprob), s);
  DevBuf<int>& perm = is_target ? pl->perm_i : pl->perm_j;
  DevBuf<float4>& pos = is_target ? pl->tpos : pl->spos;
  DevBuf<float4>& nrm = is_target ? pl->tnrm : pl->snrm;
  perm.alloc(n);
  pos.alloc(n);
  nrm.alloc(n);
  FMMB_CUDA(cudaMemcpyAsync(perm.get(), idx.get(), n * sizeof(int), cudaMemcpyDeviceToDevice, s));
  gather_points<<<blocks(n, 256), 256, 0, s>>>(n, idx.get(), sd.x, sd.y, sd.z, sd.nx, sd.ny, sd.nz, pos.get(), nrm.get());
  FMMB_CHECK_LAUNCH();

  // Levels lmax..2: runs of key >> 3(lmax-lev) over the sorted points.  Level
  // lmax's runs are the leaves; parents come from the run index of the
  // first point of each child.
  std::vector<int>& nbox = is_target ? pl->nbox_i : pl->nbox_j;
  nbox.assign(lmax + 1, 0);
  // every level's runs at once (arrays of n, the bound), the counts read
  // back with one synchronisation
  std::vector<TmpBuf<int>> kstore, fstore, rstore;
  for (int lev = 0; lev <= lmax; lev++) {
    kstore.emplace_back(s);
    fstore.emplace_back(s);
    rstore.emplace_back(s);
  }
  flag.alloc(n);
  flag2.alloc(n);
  nbd.alloc(lmax + 1);
  for (int lev = lmax; lev >= 2; lev--) {
    const int shift = 3 * (lmax - lev);
    if (n > 0) {
      run_flags<<<blocks(n, 256), 256, 0, s>>>(n, key.get(), shift, flag.get(), flag2.get());
      FMMB_CHECK_LAUNCH();
    }
    exclusive_scan(flag.get(), n, s);
    run_count<<<1, 1, 0, s>>>(n, flag.get(), flag2.get(), nbd.get() + lev);
    FMMB_CHECK_LAUNCH();
    kstore[lev].alloc(n);
    fstore[lev].alloc(n);
    rstore[lev].alloc(n);
    if (n > 0) {
      run_compact<<<blocks(n, 256), 256, 0, s>>>(n, key.get(), shift, flag.get(), flag2.get(), kstore[lev].get(),
                                                 fstore[lev].get(), rstore[lev].get());
      FMMB_CHECK_LAUNCH();
    }
  }
  FMMB_CUDA(cudaMemcpyAsync(nbox.data(), nbd.get(), (lmax + 1) * sizeof(int), cudaMemcpyDeviceToHost, s));
  FMMB_CUDA(cudaStreamSynchronize(s));
  nbox[0] = nbox[1] = 0;
  // concatenated per-level arrays, lmax first (the reference's nlbi/nlbj layout)
  std::vector<int>& off = is_target ? pl->off_i : pl->off_j;
  off.assign(lmax + 1, 0);
  int tot = 0;
  for (int lev = lmax; lev >= 2; lev--) {
    off[lev] = tot;
    tot += nbox[lev];
  }
  (is_target ? pl->tot_i : pl->tot_j) = tot;
  DevBuf<int>& keys_all = is_target ? pl->key_i : pl->key_j;
  DevBuf<int>& parent_all = is_target ? pl->parent_i : pl->parent_j;
  keys_all.alloc(tot);
  parent_all.alloc(tot);
  FMMB_CUDA(cudaMemsetAsync(parent_all.get(), 0xff, tot * sizeof(int), s));
  for (int lev = lmax; lev >= 2; lev--) {
    FMMB_CUDA(cudaMemcpyAsync(keys_all.get() + off[lev], kstore[lev].get(), nbox[lev] * sizeof(int),
                              cudaMemcpyDeviceToDevice, s));
    if (lev > 2) {
      // parent of box b at lev = run index (at lev-1) of its first point
      const int nb = nbox[lev];
      gather_int<<<blocks(nb, 256), 256, 0, s>>>(nb, fstore[lev].get(), rstore[lev - 1].get(),
                                                 parent_all.get() + off[lev]);
      FMMB_CHECK_LAUNCH();
    }
  }
  // leaves
  DevBuf<int2>& leaf = is_target ? pl->leaf_i : pl->leaf_j;
  leaf.alloc(nbox[lmax]);
  leaf_ranges<<<blocks(nbox[lmax], 256), 256, 0, s>>>(nbox[lmax], n, fstore[lmax].get(), leaf.get());
  FMMB_CHECK_LAUNCH();
  // leaf keys without the problem bits (box centres of P2M / L2P)
  DevBuf<int>& lk = is_target ? pl->leafkey_i : pl->leafkey_j;
  lk.alloc(nbox[lmax]);
  mask_keys<<<blocks(nbox[lmax], 256), 256, 0, s>>>(nbox[lmax], keys_all.get() + off[lmax], (1 << (3 * lmax)) - 1,
                                                    lk.get());
  FMMB_CHECK_LAUNCH();
  if (!is_target) {
    pl->child_start_j.alloc(tot);
    pl->child_count_j.alloc(tot);
    FMMB_CUDA(cudaMemsetAsync(pl->child_count_j.get(), 0, tot * sizeof(int), s));
    for (int lev = lmax; lev >= 3; lev--) {
      // children at lev, parents at lev-1 (indices within the level)
      child_starts<<<blocks(nbox[lev], 256), 256, 0, s>>>(nbox[lev], parent_all.get() + off[lev],
                                                         pl->child_start_j.get() + off[lev - 1]);
      FMMB_CHECK_LAUNCH();
      child_counts<<<blocks(nbox[lev - 1], 256), 256, 0, s>>>(nbox[lev - 1], nbox[lev], pl->child_start_j.get() + off[lev - 1],
                                                             pl->child_count_j.get() + off[lev - 1]);
      FMMB_CHECK_LAUNCH();
    }
  }
  {
    // cheap host checks that keep a broken tree from reaching the expansion
    // kernels: every parent owns 1..8 children, every parent index is in range
    std::vector<int> pa(tot), cc;
    FMMB_CUDA(cudaMemcpyAsync(pa.data(), parent_all.get(), tot * sizeof(int), cudaMemcpyDeviceToHost, s));
    if (!is_target) {
      cc.resize(tot);
      FMMB_CUDA(cudaMemcpyAsync(cc.data(), pl->child_count_j.get(), tot * sizeof(int), cudaMemcpyDeviceToHost, s));
    }
    FMMB_CUDA(cudaStreamSynchronize(s));
    if (!is_target)
      for (int lev = lmax - 1; lev >= 2; lev--)
        for (int b = 0; b < nbox[lev]; b++) {
          const int c = cc[off[lev] + b];
          FMMB_REQUIRE(c >= 1 && c <= 8, FMMB_ERR_STATE, "tree build: inconsistent child count");
        }
    for (int lev = lmax; lev >= 3; lev--)
      for (int b = 0; b < nbox[lev]; b++) {
        const int q = pa[off[lev] + b];
        FMMB_REQUIRE(q >= 0 && q < nbox[lev - 1], FMMB_ERR_STATE, "tree build: parent index out of range");
      }
  }
}

}  // namespace

void build_tree(fmmb_plan* pl, int ni, const float* tx, const float* ty, const float* tz, const float* tnx,
                const float* tny, const float* tnz, int nj, const float* sx, const float* sy, const float* sz,
                const float* snx, const float* sny, const float* snz, const float* bbox_in) {
  cudaStream_t s = pl->st.main;
  FMMB_REQUIRE(3 * pl->cfg.lmax + prob_bits(pl->nprob) <= 30, FMMB_ERR_CAPACITY,
               "box keys: 3*lmax + ceil(log2(problems)) must stay within 30 bits");
  pl->ni = ni;
  pl->nj = nj;
  pl->lmax = pl->cfg.lmax;
  if (bbox_in) {
    for (int k = 0; k < 4; k++) pl->bbox[k] = bbox_in[k];
  } else {
    // root cube from the extent of all points, as the BEM drivers do
    // (biobem/fmm_matmult.h:29-114): corner at the minimum, side = largest
    // extent * (1 + 1e-5).
    TmpBuf<float> mm(s);
    mm.alloc(6 * 2);
    float init[12];
    for (int k = 0; k < 6; k++) {
      init[2 * k] = FLT_MAX;
      init[2 * k + 1] = -FLT_MAX;
    }
    // encode initial values like minmax_kernel does
    int enc[12];
    for (int k = 0; k < 12; k++) {
      int v;
      std::memcpy(&v, &init[k], 4);
      enc[k] = v >= 0 ? v : v ^ 0x7fffffff;
    }
    FMMB_CUDA(cudaMemcpyAsync(mm.get(), enc, sizeof(enc), cudaMemcpyHostToDevice, s));
    const float* arr[6] = {tx, ty, tz, sx, sy, sz};
    for (int k = 0; k < 6; k++) {
      int n = k < 3 ? ni : nj;
      if (n > 0) minmax_kernel<<<std::min(blocks(n, 256), 1024), 256, 0, s>>>(n, arr[k], mm.get() + 2 * k);
      FMMB_CHECK_LAUNCH();
    }
    int res[12];
    FMMB_CUDA(cudaMemcpyAsync(res, mm.get(), sizeof(res), cudaMemcpyDeviceToHost, s));
    FMMB_CUDA(cudaStreamSynchronize(s));
    float v[12];
    for (int k = 0; k < 12; k++) {
      int e = res[k] >= 0 ? res[k] : res[k] ^ 0x7fffffff;
      std::memcpy(&v[k], &e, 4);
    }
    float lo[3], hi[3];
    for (int d = 0; d < 3; d++) {
      lo[d] = std::min(ni ? v[2 * d] : FLT_MAX, nj ? v[6 + 2 * d] : FLT_MAX);
      hi[d] = std::max(ni ? v[2 * d + 1] : -FLT_MAX, nj ? v[6 + 2 * d + 1] : -FLT_MAX);
    }
    float rd = 0;
    for (int d = 0; d < 3; d++) rd = std::max(rd, (hi[d] - lo[d]) * (1 + 1e-5f));
    if (!(rd > 0)) rd = 1;
    pl->bbox[0] = lo[0];
    pl->bbox[1] = lo[1];
    pl->bbox[2] = lo[2];
    pl->bbox[3] = rd;
  }
  FMMB_REQUIRE(pl->bbox[3] > 0, FMMB_ERR_ARG, "root box side must be positive");
  build_side(pl, Side{tx, ty, tz, tnx, tny, tnz, ni, pl->d_prob_off.get()}, true, s);
  build_side(pl, Side{sx, sy, sz, snx, sny, snz, nj, pl->d_prob_off.get() + pl->nprob + 1}, false, s);

  const int lmax = pl->lmax;
  const int nleaf_i = pl->nbox_i[lmax], nleaf_j = pl->nbox_j[lmax];
  pl->p2p_list.alloc((size_t)nleaf_i * kP2PSlots);
  p2p_lists<<<blocks(nleaf_i, 128), 128, 0, s>>>(nleaf_i, pl->key_i.get() + pl->off_i[lmax], nleaf_j,
                                                 pl->key_j.get() + pl->off_j[lmax], lmax, pl->p2p_list.get());
  FMMB_CHECK_LAUNCH();
  pl->m2l_list.alloc((size_t)pl->tot_i * kM2LSlots);
  for (int lev = 2; lev <= lmax; lev++) {
    const int nb = pl->nbox_i[lev];
    m2l_lists<<<blocks((size_t)nb * kM2LSlots, 256), 256, 0, s>>>(
        nb, pl->key_i.get() + pl->off_i[lev], pl->nbox_j[lev], pl->key_j.get() + pl->off_j[lev], lev,
        pl->d_slot_rel.get(), pl->m2l_list.get() + (size_t)pl->off_i[lev] * kM2LSlots);
    FMMB_CHECK_LAUNCH();
  }
  TmpBuf<unsigned long long> cnt(s);
  cnt.alloc(2);
  FMMB_CUDA(cudaMemsetAsync(cnt.get(), 0, 2 * sizeof(unsigned long long), s));
  count_p2p_pairs<<<blocks(nleaf_i, 128), 128, 0, s>>>(nleaf_i, pl->leaf_i.get(), pl->leaf_j.get(), pl->p2p_list.get(),
                                                       cnt.get());
  FMMB_CHECK_LAUNCH();
  count_nonneg<<<256, 256, 0, s>>>((size_t)pl->tot_i * kM2LSlots, pl->m2l_list.get(), cnt.get() + 1);
  FMMB_CHECK_LAUNCH();
  unsigned long long h[2];
  FMMB_CUDA(cudaMemcpyAsync(h, cnt.get(), sizeof(h), cudaMemcpyDeviceToHost, s));
  FMMB_CUDA(cudaStreamSynchronize(s));
  pl->p2p_pairs = (long long)h[0];
  pl->m2l_pairs = (long long)h[1];
}

}  // namespace fmmb

// Box-to-box translations (M2L, M2M, L2L) on the 5th-generation tensor
// cores (tcgen05, TMEM accumulators) in TF32x3, for the mixed-precision form.
//
// Every translation is a dense real K x K operator (operators.cpp: the
// reference's rotate / z-translate / rotate-back steps of kernel/m2l.cxx:30-83,
// kernel/m2m.cxx:28-62 and kernel/l2l.cxx:44-78 composed into one matrix per
// relative position).  The work is a list of box pairs (output row, input
// row, operator), grouped by operator and cut into tiles of 128 pairs: one
// tile is one GEMM  D (128 coefficients x 128 pairs) = T_op . X[inputs],
// X being the TF32 (hi, lo) split of the input expansions, and its columns
// are added into the FP64 output rows in the epilogue by reductions at the L2
// (an output row receives several pairs in M2L and M2M).  Grouping by
// operator keeps the tiles full whatever the geometry (on a surface most of
// the 189 interaction positions of a box are empty, so tiles of output boxes
// would be mostly zero columns).  Each product is split into three TF32 MMAs,
// A_hi.B_hi + A_hi.B_lo + A_lo.B_hi (about 2^-21 relative error per product
// instead of 2^-11 for plain TF32), accumulated in FP32 in tensor memory over
// the K coefficients of one pair only; the sum over pairs is FP64.
//
// A persistent CTA takes a contiguous range of tiles, so consecutive tiles
// mostly share their operator, which stays resident and is reloaded by the
// epilogue warps only when it changes: its hi part in shared memory (4
// K-blocks, 64 KB, one bulk copy each), its lo part in tensor memory (lane =
// output coefficient, 128 columns), so the A_lo.B_hi product reads A from
// tensor memory and shared memory keeps room for a 5-stage ring of input
// K-blocks (hi + lo, 32 KB each).  Five producer groups (group s fills ring
// slot s) gather the input rows with cp.async, so up to five stages are in
// flight while the tensor core works.  Tensor memory (512 columns): three
// alternating FP32 accumulators (MMA warp / four epilogue warps) and A_lo.
#include <cuda_runtime.h>

#include <cstdint>

#include "internal.h"
#include "kernels.h"


namespace fmmb {
namespace tc {

constexpr int kTile = 128;        // pairs per tile (MMA N)
constexpr int kRows = 128;        // output coefficients per work item (MMA M)
constexpr int kKB = 32;           // TF32 values per K-block (128 bytes)
constexpr int kHalf = kTile * 128;                  // one 128 x 128-byte K-block tile (16 KB)
constexpr int kStageBytes = 2 * kHalf;              // input K-block, hi and lo (32 KB)
constexpr int kBarBytes = 256;                      // <= 18 mbarriers + the TMEM address
constexpr int kGroupWarps = 2;                      // producer warps per ring slot
constexpr int kGroupThreads = 32 * kGroupWarps;
constexpr int kTmemCols = 512;
constexpr int kMaxNKB = 8;                          // K <= 256 (p <= 15)
constexpr unsigned kSpinLimit = 1u << 22;           // bounded waits (seconds at most)

// Layout for operators of NKB K-blocks (K padded to 32 NKB): the hi part is
// resident in shared memory (NKB x 16 KB), the input ring takes what is left
// of 224 KB; the lo part takes the last 32 NKB tensor-memory columns and the
// accumulators (128 columns each) the rest.
template <int NKB>
struct Cfg {
  static constexpr int kKPad = NKB * kKB;
  static constexpr int kABytes = NKB * kHalf;
  static constexpr int kStages = (224 * 1024 - kABytes) / kStageBytes;
  static constexpr int kSmemBytes = kABytes + kStages * kStageBytes + kBarBytes + 1024;
  static constexpr int kThreads = 32 * (5 + kStages * kGroupWarps);  // 4 epilogue + 1 MMA + producers
  static constexpr int kColAlo = kTmemCols - NKB * kKB;
  static constexpr int kNAcc = kColAlo / kTile < 3 ? kColAlo / kTile : 3;
  static constexpr int kImgFloats = 2 * kRows * kKPad;  // hi image (swizzled K-blocks) + lo rows
  static_assert(kStages >= 2 && kNAcc >= 2, "operator too large for the tensor-core layout");
};

// instruction descriptor: F32 accumulate, TF32 A and B, both K-major,
// N = 128 (bits 17..22 hold N>>3), M = 128 (bits 24..28 hold M>>4)
constexpr uint32_t kIdesc = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(kTile >> 3) << 17) |
                            ((uint32_t)(kRows >> 4) << 24);

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// K-major SWIZZLE_128B shared-memory matrix descriptor: start address, LBO
// (unused for this layout, 1), SBO = 1024 bytes between 8-row groups,
// descriptor version 1, layout type 2.
__device__ __forceinline__ uint64_t make_desc(uint32_t saddr) {
  return (uint64_t)((saddr >> 4) & 0x3FFF) | ((uint64_t)1 << 16) | ((uint64_t)(1024 >> 4) << 32) |
         ((uint64_t)1 << 46) | ((uint64_t)2 << 61);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void mbar_arrive_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
// Bounded wait on a phase parity; false on timeout.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  const uint32_t a = smem_u32(bar);
  for (unsigned it = 0; it < kSpinLimit; it++) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void mma_tf32(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(kIdesc), "r"(accumulate)
      : "memory");
}

// D (+)= A . B with A read from tensor memory (lane = row, one TF32 per column).
__device__ __forceinline__ void mma_tf32_ta(uint32_t tmem_d, uint32_t tmem_a, uint64_t db, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], [%1], %2, %3, p;\n\t}" ::"r"(tmem_d),
      "r"(tmem_a), "l"(db), "r"(kIdesc), "r"(accumulate)
      : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.expect_tx.relaxed.cta.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ void prefetch_l2(const void* p, uint32_t bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

// 32 consecutive accumulator columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float* v) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]),
        "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
        "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; i++) v[i] = __uint_as_float(r[i]);
}

// 32 consecutive accumulator columns of this thread's TMEM lane, raw (no wait).
__device__ __forceinline__ void tmem_ld32_nowait(uint32_t taddr, uint32_t* r) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]),
        "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
        "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ void tmem_st32(uint32_t taddr, const uint32_t* r) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x32.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,"
      "%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31,%32};" ::"r"(taddr),
      "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7]), "r"(r[8]), "r"(r[9]),
      "r"(r[10]), "r"(r[11]), "r"(r[12]), "r"(r[13]), "r"(r[14]), "r"(r[15]), "r"(r[16]), "r"(r[17]), "r"(r[18]),
      "r"(r[19]), "r"(r[20]), "r"(r[21]), "r"(r[22]), "r"(r[23]), "r"(r[24]), "r"(r[25]), "r"(r[26]), "r"(r[27]),
      "r"(r[28]), "r"(r[29]), "r"(r[30]), "r"(r[31])
      : "memory");
}
__device__ __forceinline__ void tmem_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }

__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// Swizzled byte offset of 16-byte chunk c of row r in a K-block tile.
__device__ __forceinline__ uint32_t swz(int r, int c) { return (uint32_t)(r * 128 + ((c ^ (r & 7)) << 4)); }

struct Params {
  int ntile;              // work items: (pair tile, row block of the operator)
  const int* tile_op;     // [ntile] operator image of each work item (sorted)
  const int* tile_src;    // [ntile][128] input row of each pair (-1 = empty column)
  const int2* tile_y;     // [ntile] (first pair row in y, coefficient offset in the row)
  const float* opimg;     // operator images [ops][Cfg::kImgFloats]: hi K-block images, then lo rows [128][kKPad]
  const float* xin;       // TF32 split of the inputs [rows][2][kKPad] (hi, lo)
  float* y;               // pair rows: column j of work item g goes to y[(tile_y.x + j)*ys + tile_y.y + row]
  int ys;                 // floats per pair row of y
  int* err;               // set to a nonzero code on timeout
};

// The epilogue warps make operator image `op` resident: thread 0 bulk-copies
// the hi images into shared memory (their bytes counted on a_full), every
// thread writes its row of the lo part into tensor memory, then arrives.
template <int NKB>
__device__ __forceinline__ void load_operator(const Params& P, int op, int row, uint32_t lane_base,
                                              unsigned char* sA, uint64_t* a_full) {
  using C = Cfg<NKB>;
  const float* img = P.opimg + (size_t)op * C::kImgFloats;
  if (row == 0) {
    mbar_expect_tx(a_full, C::kABytes);
    for (int c = 0; c < NKB; c++) bulk_g2s(sA + c * kHalf, img + (size_t)c * (kRows * kKB), kHalf, a_full);
  }
  const float4* lo = reinterpret_cast<const float4*>(img + NKB * kRows * kKB + (size_t)row * C::kKPad);
#pragma unroll 1
  for (int c = 0; c < NKB; c += 2) {  // two chunks of 32 columns per batch of loads
    uint32_t r[2][32];
#pragma unroll
    for (int u = 0; u < 2; u++)
#pragma unroll
      for (int q = 0; q < 8; q++) {
        const float4 v = c + u < NKB ? __ldg(lo + (c + u) * 8 + q) : make_float4(0.f, 0.f, 0.f, 0.f);
        r[u][4 * q] = __float_as_uint(v.x);
        r[u][4 * q + 1] = __float_as_uint(v.y);
        r[u][4 * q + 2] = __float_as_uint(v.z);
        r[u][4 * q + 3] = __float_as_uint(v.w);
      }
#pragma unroll
    for (int u = 0; u < 2; u++)
      if (c + u < NKB) tmem_st32(lane_base + (uint32_t)(C::kColAlo + (c + u) * 32), r[u]);
  }
  tmem_wait_st();
  tc_fence_before();
  mbar_arrive(a_full);
}

template <int NKB>
__global__ void __launch_bounds__(Cfg<NKB>::kThreads, 1) translate_tc(Params P) {
  using C = Cfg<NKB>;
  constexpr int kStages = C::kStages, kNAcc = C::kNAcc;
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char* smem = (unsigned char*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  unsigned char* sA = smem;                       // resident operator, hi part
  unsigned char* sB = smem + C::kABytes;          // input ring
  uint64_t* full = (uint64_t*)(sB + kStages * kStageBytes);
  uint64_t* empty = full + kStages;
  uint64_t* accf = empty + kStages;  // [kNAcc] accumulator b holds a finished tile
  uint64_t* acce = accf + kNAcc;     // [kNAcc] accumulator b read out by the epilogue
  uint64_t* a_full = acce + kNAcc;   // operator resident (hi bytes landed, lo rows written)
  uint64_t* drain = a_full + 1;      // all MMAs done (before tensor memory is freed)
  uint32_t* tmem_slot = (uint32_t*)(drain + 1);
  __shared__ int sh_fail;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int t_begin = (int)((long long)P.ntile * blockIdx.x / gridDim.x);
  const int t_end = (int)((long long)P.ntile * (blockIdx.x + 1) / gridDim.x);
  const int ntile = t_end - t_begin;
  const int nstage_total = ntile * NKB;

  if (threadIdx.x == 0) {
    sh_fail = 0;
    for (int s = 0; s < kStages; s++) {
      mbar_init(&full[s], kGroupThreads);  // the producers of ring slot s
      mbar_init(&empty[s], 1);             // one tcgen05.commit
    }
    for (int b = 0; b < kNAcc; b++) {
      mbar_init(&accf[b], 1);    // tcgen05.commit after a tile's MMAs
      mbar_init(&acce[b], 128);  // every epilogue thread after reading the tile
    }
    mbar_init(a_full, 128);      // every epilogue thread (+ the hi bytes)
    mbar_init(drain, 1);         // tcgen05.commit
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    // this CTA's pair lists and operator images, into L2 ahead of their use
    prefetch_l2(P.tile_src + (size_t)t_begin * kTile, (uint32_t)(ntile * kTile * sizeof(int)));
    for (int i = 0, prev = -1; i < ntile; i++) {
      const int op = P.tile_op[t_begin + i];
      if (op != prev) prefetch_l2(P.opimg + (size_t)op * C::kImgFloats, (uint32_t)(C::kImgFloats * sizeof(float)));
      prev = op;
    }
  }
  if (warp == 4) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(kTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp >= 5) {
    // ------------------------------------------------ producers
    // group s (2 warps) fills ring slot s for stages s, s+kStages, ...  A
    // stage is 128 input rows x (hi, lo) x 128 bytes; one warp instruction
    // copies two rows: lanes 0-7 the hi line of the first row, 8-15 its lo
    // line, 16-31 the same for the second, so it touches four whole lines.
    const int grp = (warp - 5) / kGroupWarps;
    const int gw = (warp - 5) % kGroupWarps;
    const int part = (lane >> 3) & 1, chunk = lane & 7;
    constexpr int kRowsPerThread = kTile / (2 * kGroupWarps);  // 32
    unsigned char* bdst = sB + grp * kStageBytes + part * kHalf;
    for (int st = grp; st < nstage_total; st += kStages) {
      const uint32_t ph = (st / kStages) & 1;
      bool ok = true;
      if (st >= kStages && lane == 0) ok = mbar_wait(&empty[grp], ph ^ 1);
      ok = __shfl_sync(0xffffffffu, ok ? 1 : 0, 0) != 0;
      if (!ok) atomicExch(&sh_fail, 1);
      if (!ok || *(volatile int*)&sh_fail) break;
      const int g = t_begin + st / NKB;
      const int kb = st % NKB;
      const int* tsrc = P.tile_src + (size_t)g * kTile;
      int src[kRowsPerThread];
#pragma unroll
      for (int k = 0; k < kRowsPerThread; k++) src[k] = __ldg(tsrc + k * 2 * kGroupWarps + gw * 2 + (lane >> 4));
#pragma unroll
      for (int k = 0; k < kRowsPerThread; k++) {
        const int r = k * 2 * kGroupWarps + gw * 2 + (lane >> 4);
        unsigned char* d = bdst + swz(r, chunk);
        if (src[k] >= 0)
          cp_async16(d, P.xin + (size_t)src[k] * (2 * C::kKPad) + part * C::kKPad + kb * kKB + 4 * chunk);
        else
          *reinterpret_cast<float4*>(d) = make_float4(0.f, 0.f, 0.f, 0.f);
      }
      cp_async_commit();
      cp_async_wait<0>();
      fence_async_smem();
      mbar_arrive(&full[grp]);
    }
    cp_async_wait<0>();
  } else if (warp == 4) {
    // ------------------------------------------------ MMA issuer
    bool ok = true;
    int cur_op = -1, nload = 0;
    for (int i = 0; i < ntile && ok; i++) {
      const int g = t_begin + i;
      const int buf = i % kNAcc;
      const uint32_t dcol = tmem + (uint32_t)(buf * kTile);
      const int op = P.tile_op[g];
      if (op != cur_op) {  // the epilogue makes each new operator resident once the MMAs using the old one are done
        if (lane == 0) ok = mbar_wait(a_full, nload & 1);
        ok = __shfl_sync(0xffffffffu, ok ? 1 : 0, 0) != 0;
        if (!ok) break;
        cur_op = op;
        nload++;
      }
      if (i >= kNAcc) {  // wait until the epilogue has read this accumulator
        if (lane == 0) ok = mbar_wait(&acce[buf], (i / kNAcc - 1) & 1);
        ok = __shfl_sync(0xffffffffu, ok ? 1 : 0, 0) != 0;
        if (!ok) break;
      }
      tc_fence_after();
      for (int kb = 0; kb < NKB && ok; kb++) {
        const int st = i * NKB + kb;
        const int s = st % kStages;
        if (lane == 0) ok = mbar_wait(&full[s], (st / kStages) & 1);
        ok = __shfl_sync(0xffffffffu, ok ? 1 : 0, 0) != 0;
        if (!ok) break;
        tc_fence_after();
        if (lane == 0) {
          const uint32_t ahi = smem_u32(sA + kb * kHalf);
          const uint32_t alo = tmem + (uint32_t)(C::kColAlo + kb * kKB);
          const uint32_t bhi = smem_u32(sB + s * kStageBytes), blo = bhi + kHalf;
#pragma unroll
          for (int k = 0; k < kKB / 8; k++) {  // 4 MMAs of K=8 per 32-wide block
            const uint32_t o = k * 32;           // 8 TF32 = 32 bytes along K in shared memory
            mma_tf32(dcol, make_desc(ahi + o), make_desc(bhi + o), (kb | k) ? 1u : 0u);
            mma_tf32(dcol, make_desc(ahi + o), make_desc(blo + o), 1u);
            mma_tf32_ta(dcol, alo + k * 8, make_desc(bhi + o), 1u);
          }
          mma_commit(&empty[s]);  // frees the ring slot when these MMAs are done
          if (kb == NKB - 1) mma_commit(&accf[buf]);
        }
        __syncwarp();
      }
    }
    if (!ok && lane == 0) atomicExch(&sh_fail, 2);
    // drain: every MMA issued above completes before tensor memory is freed
    if (lane == 0) {
      mma_commit(drain);
      mbar_wait(drain, 0);
    }
    __syncwarp();
  } else {
    // ------------------------------------------------ epilogue (warps 0..3)
    // thread `row` owns output coefficient row (tensor memory lane `row`): it
    // makes each new operator resident, then stores column j of every tile to
    // its pair row of y (plain coalesced FP32 stores; reduce_pairs sums the
    // pair rows of each output box in FP64).
    const int row = warp * 32 + lane;
    const uint32_t lane_base = tmem + ((uint32_t)(warp * 32) << 16);
    bool ok = true;
    if (ntile > 0) load_operator<NKB>(P, P.tile_op[t_begin], row, lane_base, sA, a_full);
    for (int i = 0; i < ntile; i++) {
      const int g = t_begin + i;
      const int buf = i % kNAcc;
      const int2 ty = P.tile_y[g];
      const bool w = mbar_wait(&accf[buf], (i / kNAcc) & 1);
      ok = __all_sync(0xffffffffu, w && *(volatile int*)&sh_fail == 0) != 0;
      if (!ok) break;
      tc_fence_after();
      if (i + 1 < ntile && P.tile_op[g + 1] != P.tile_op[g])  // every MMA up to tile i is done
        load_operator<NKB>(P, P.tile_op[g + 1], row, lane_base, sA, a_full);
#pragma unroll
      for (int h = 0; h < kTile / 32; h++) {
        uint32_t v[32];
        tmem_ld32_nowait(lane_base + (uint32_t)(buf * kTile + h * 32), v);
        tmem_wait_ld();
        if (h == kTile / 32 - 1) {  // the accumulator is free once read
          tc_fence_before();
          mbar_arrive(&acce[buf]);
        }
        float* yb = P.y + ((size_t)ty.x + h * 32) * P.ys + ty.y + row;
#pragma unroll
        for (int j = 0; j < 32; j++) yb[(size_t)j * P.ys] = __uint_as_float(v[j]);
      }
    }
    if (!ok) atomicExch(&sh_fail, 3);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 4) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols));
  }
  if (threadIdx.x == 0 && sh_fail) atomicExch(P.err, sh_fail);
}

// TF32 round-to-nearest (ties away) of an FP32 value, as cvt.rna.tf32.f32.
__device__ __forceinline__ float tf32_rna(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}

// M (FP64, [nbox][K]) -> Mtf ([nbox][2][kpad] FP32: TF32 hi, TF32 lo, zero padded)
__global__ void split_tf32(int nbox, int K, int kpad, const double* __restrict__ M, float* __restrict__ Mtf) {
  const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i >= (size_t)nbox * kpad) return;
  const size_t b = i / kpad;
  const int k = (int)(i % kpad);
  float hi = 0.f, lo = 0.f;
  if (k < K) {
    const double x = M[b * K + k];
    hi = tf32_rna((float)x);
    lo = tf32_rna((float)(x - (double)hi));
  }
  Mtf[b * 2 * kpad + k] = hi;
  Mtf[b * 2 * kpad + kpad + k] = lo;
}

// out[rows[w]][0..K) += sum over e in [ptr[w], ptr[w+1]) of y[idx[e]][0..K)
// (pair rows of ys floats, ys >= K a multiple of 4), in FP64 and in list
// order (deterministic); one warp per output row, lane l holding coefficients
// 128c + 4l .. 128c + 4l + 3 of each 128-coefficient chunk c (K <= 256), the
// lanes past the row reading nothing; for K <= 128 eight rows in flight.
__global__ void reduce_pairs(int nrow, const int* __restrict__ rows, const int* __restrict__ ptr,
                             const int* __restrict__ idx, const float* __restrict__ y, int ys, int K,
                             double* __restrict__ out) {
  const int w = (int)((blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5);
  const int lane = threadIdx.x & 31;
  if (w >= nrow) return;
  const int nch = (K + 127) / 128;
  double a[2][4] = {{0, 0, 0, 0}, {0, 0, 0, 0}};
  const int e0 = ptr[w], e1 = ptr[w + 1];
  const bool live0 = 4 * lane < ys, live1 = nch > 1 && 128 + 4 * lane < ys;
  const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
  int e = e0;
  if (nch == 1) {  // K <= 128: one read of up to 512 bytes per pair row, 8 rows in flight
    for (; e + 8 <= e1; e += 8) {
      int r8[8];
#pragma unroll
      for (int u = 0; u < 8; u++) r8[u] = idx[e + u];
      float4 v[8];
#pragma unroll
      for (int u = 0; u < 8; u++) v[u] = live0 ? __ldcs(reinterpret_cast<const float4*>(y + (size_t)r8[u] * ys) + lane) : z4;
#pragma unroll
      for (int u = 0; u < 8; u++) {
        a[0][0] += v[u].x;
        a[0][1] += v[u].y;
        a[0][2] += v[u].z;
        a[0][3] += v[u].w;
      }
    }
  }
  for (; e + 4 <= e1; e += 4) {
    float4 v[4][2];
#pragma unroll
    for (int u = 0; u < 4; u++) {
      const float4* yr = reinterpret_cast<const float4*>(y + (size_t)idx[e + u] * ys);
      v[u][0] = live0 ? __ldcs(yr + lane) : z4;
      v[u][1] = live1 ? __ldcs(yr + 32 + lane) : z4;
    }
#pragma unroll
    for (int u = 0; u < 4; u++)
#pragma unroll
      for (int c = 0; c < 2; c++) {
        a[c][0] += v[u][c].x;
        a[c][1] += v[u][c].y;
        a[c][2] += v[u][c].z;
        a[c][3] += v[u][c].w;
      }
  }
  for (; e < e1; e++) {
    const float4* yr = reinterpret_cast<const float4*>(y + (size_t)idx[e] * ys);
#pragma unroll
    for (int c = 0; c < 2; c++) {
      if (c >= nch || !(c ? live1 : live0)) break;
      const float4 v = __ldcs(yr + 32 * c + lane);
      a[c][0] += v.x;
      a[c][1] += v.y;
      a[c][2] += v.z;
      a[c][3] += v.w;
    }
  }
  // each output row has one warp: its single atomic addition is the value of
  // a read-modify-write, without the warp waiting for the read
  double* o = out + (size_t)rows[w] * K;
#pragma unroll
  for (int c = 0; c < 2; c++)
#pragma unroll
    for (int u = 0; u < 4; u++) {
      const int k = 128 * c + 4 * lane + u;
      if (k < K) atomicAdd(o + k, a[c][u]);
    }
}

}  // namespace tc

int tc_tile() { return tc::kTile; }
int tc_kpad(int K) { return K <= 128 ? 128 : ((K + tc::kKB - 1) / tc::kKB) * tc::kKB; }
int tc_max_k() { return tc::kMaxNKB * tc::kKB; }

void launch_reduce_pairs(int nrow, const int* rows, const int* ptr, const int* idx, const float* y, int ys, int K,
                         double* out, cudaStream_t st) {
  if (nrow <= 0) return;
  const size_t threads = (size_t)nrow * 32;
  tc::reduce_pairs<<<(unsigned)((threads + 255) / 256), 256, 0, st>>>(nrow, rows, ptr, idx, y, ys, K, out);
  FMMB_CHECK_LAUNCH();
}

void launch_split_tf32(int nbox, int K, int kpad, const double* M, float* Mtf, cudaStream_t st) {
  if (nbox <= 0) return;
  const size_t n = (size_t)nbox * kpad;
  tc::split_tf32<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(nbox, K, kpad, M, Mtf);
  FMMB_CHECK_LAUNCH();
}

namespace {
template <int NKB>
void prepare_nkb() {
  FMMB_CUDA(cudaFuncSetAttribute(tc::translate_tc<NKB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 tc::Cfg<NKB>::kSmemBytes));
}
template <int NKB>
void launch_nkb(const tc::Params& P, int grid, cudaStream_t st) {
  tc::translate_tc<NKB><<<grid, tc::Cfg<NKB>::kThreads, tc::Cfg<NKB>::kSmemBytes, st>>>(P);
}
}  // namespace

void prepare_translate_tc() {
  prepare_nkb<4>();
  prepare_nkb<5>();
  prepare_nkb<6>();
  prepare_nkb<7>();
  prepare_nkb<8>();
}

void launch_translate_tc(const TcJobArgs& a, int nsm, cudaStream_t st) {
  if (a.ntile <= 0) return;
  tc::Params P{};
  P.ntile = a.ntile;
  P.tile_op = a.tile_op;
  P.tile_src = a.tile_src;
  P.tile_y = a.tile_y;
  P.opimg = a.opimg;
  P.xin = a.xin;
  P.y = a.y;
  P.ys = a.ys;
  P.err = a.err;
  const int grid = a.ntile < nsm ? a.ntile : nsm;
  switch (tc_kpad(a.K) / tc::kKB) {
    case 4: launch_nkb<4>(P, grid, st); break;
    case 5: launch_nkb<5>(P, grid, st); break;
    case 6: launch_nkb<6>(P, grid, st); break;
    case 7: launch_nkb<7>(P, grid, st); break;
    default: launch_nkb<8>(P, grid, st); break;
  }
  FMMB_CHECK_LAUNCH();
}

}  // namespace fmmb

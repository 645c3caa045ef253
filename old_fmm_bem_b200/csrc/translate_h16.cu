// M2L on the 5th-generation tensor cores (tcgen05, TMEM accumulators) in
// FP16x3, for the mixed-precision form with K = (p+1)^2 <= 176 (p <= 12).
//
// The translation of a box pair is the dense real K x K operator of its
// relative position (operators.cpp: the rotate / z-translate / rotate-back
// steps of kernel/m2l.cxx:30-83 composed into one matrix).  Work is the list of
// box pairs grouped by operator and cut into tiles of 128 pairs; one tile is
// one GEMM with the pairs as the M dimension:
//
//   D (128 pairs x N coefficients) = X (128 pairs x K inputs) . T^T
//
// so the output coefficients are the N dimension, padded only to a multiple of
// 16 (N = 176 for K = 169), and the operator is the B operand, resident in
// shared memory while consecutive tiles share it.  Each product is split into
// three FP16 MMAs, X_hi.T_hi + X_hi.T_lo + X_lo.T_hi, accumulated in FP32 in
// tensor memory over the K inputs of one pair (hi + lo keep 22 bits of each
// value; FP16 products are exact in FP32), at twice the tensor-core rate of the
// TF32 form.  FP16 has a narrow exponent range, so both operands are scaled by
// powers of two that put the largest value of every input expansion (per
// box) and of every operator in [2^14, 2^15), just below the FP16 maximum: hi
// and lo then keep 22 bits of every value down to 2^-18 of the largest (a lo
// part below FP16's normal range loses bits only under that), and what is
// smaller still is exact to 2^-40 of the largest -- an absolute error far
// below that of the largest products (the entries that small are the
// high-degree terms of distant boxes); the FP32 products stay far from
// overflow (2^30 each).  The epilogue undoes both scalings exactly (powers of
// two) and stores each pair's K coefficients as an FP32 row for the FP64
// segmented sum per output box (reduce_pairs in translate_tc.cu): the four
// epilogue warps transpose their rows through shared memory, so that every
// global store writes whole 128-byte lines.
//
// A persistent CTA takes a contiguous range of tiles.  Warps 0-3: epilogue
// (thread = tensor-memory lane = pair of the tile; the next tile's pair and
// scale data loaded ahead) and operator loads; warp 4:
// MMA issue; the rest: producer groups gathering the input rows of the tile
// with cp.async into a ring of K-blocks (64 FP16 of 128 pairs, hi and lo,
// K-major SWIZZLE_128B).  Two FP32 accumulators of N columns alternate
// between the MMA warp and the epilogue.  All mbarrier waits are bounded; a
// timeout sets a device error code and tensor memory is always freed.
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "internal.h"
#include "kernels.h"

namespace fmmb {
namespace h16 {

constexpr int kTile = 128;                  // pairs per tile (MMA M)
constexpr int kKB = 64;                     // FP16 values per K-block (128 bytes)
constexpr int kRowBytes = 128;
constexpr int kAHalf = kTile * kRowBytes;   // one K-block of the tile's inputs (16 KB)
constexpr int kStageBytes = 2 * kAHalf;     // hi and lo (32 KB)
constexpr int kBarBytes = 256;
constexpr int kTmemCols = 512;
constexpr int kAccStride = 256;             // accumulator b starts at tensor-memory column 256 b
// Bounded waits: each try_wait may suspend the thread for up to kSuspendNs
// (it resumes as soon as the phase completes), so a waiting warp polls the
// barrier rarely instead of keeping the load/store pipe busy; kSpinLimit
// tries bound a wait to a few seconds.
constexpr unsigned kSpinLimit = 1u << 18;
constexpr unsigned kSuspendNs = 16384;

// NKB K-blocks of 64 inputs (K <= 64 NKB); operators of up to kNMax output
// rows; the input ring takes what the resident operator leaves.
constexpr int kStgStride = 36;              // floats per row of an epilogue warp's transpose buffer
constexpr int kStgBytes = 4 * 32 * kStgStride * 4;

template <int NKB>
struct Cfg {
  static constexpr int kNMax = NKB == 2 ? 128 : 176;
  static constexpr int kOpBytes = 2 * NKB * kNMax * kRowBytes;  // hi and lo K-blocks
  static constexpr int kStages = NKB == 2 ? 4 : 2;
  static constexpr int kGroupWarps = NKB == 2 ? 2 : 4;           // producer warps per ring slot
  static constexpr int kGroupThreads = 32 * kGroupWarps;
  static constexpr int kSmemBytes = kOpBytes + kStages * kStageBytes + kStgBytes + kBarBytes + 1024;
  static constexpr int kThreads = 32 * (5 + kStages * kGroupWarps);
  static_assert(kSmemBytes <= 227 * 1024, "shared memory");
};

// instruction descriptor of kind::f16: F32 accumulator, F16 A and B, both
// K-major, N (bits 17..22 hold N >> 3), M = 128 (bits 24..28 hold M >> 4)
__host__ __device__ constexpr uint32_t idesc_f16(int n) {
  return (1u << 4) | (0u << 7) | (0u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(kTile >> 4) << 24);
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
// K-major SWIZZLE_128B shared-memory matrix descriptor (start address, LBO 1,
// SBO = 1024 bytes between 8-row groups, descriptor version 1, layout 2)
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
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.expect_tx.relaxed.cta.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  const uint32_t a = smem_u32(bar);
  for (unsigned it = 0; it < kSpinLimit; it++) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(a), "r"(parity), "n"(kSuspendNs)
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
__device__ __forceinline__ void prefetch_l2(const void* p, uint32_t bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void mma_f16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc,
                                        uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(idesc), "r"(accumulate)
      : "memory");
}
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t* r) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]),
        "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
        "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

// byte offset of 16-byte chunk c of row r in a K-block tile (K-major SWIZZLE_128B)
__device__ __forceinline__ uint32_t swz(int r, int c) { return (uint32_t)(r * kRowBytes + ((c ^ (r & 7)) << 4)); }

// 2^e as a float for |e| within the normal range
__device__ __forceinline__ float pow2f(int e) {
  e = e < -126 ? -126 : (e > 127 ? 127 : e);
  return __int_as_float((127 + e) << 23);
}

struct Params {
  int ntile;                  // tiles (128 pairs of one operator each)
  int n;                      // output rows of the operators (MMA N: K rounded up to 16)
  int K, ys;                  // coefficients per expansion, floats per pair row of y
  const int* tile_op;         // [ntile] operator of each tile (sorted)
  const int* tile_src;        // [ntile][128] input row of each pair (-1 = empty)
  const int2* tile_y;         // [ntile] (first pair row in y, 0)
  const unsigned char* opimg; // operator images, img_bytes each: hi K-blocks, lo K-blocks, the scale 2^f
  size_t img_bytes;
  const __half* xin;          // scaled FP16 split of the inputs [rows][2][64 NKB] (hi, lo)
  const int* xexp;            // [rows] e of each input (its coefficients were scaled by 2^-e)
  float* y;                   // pair rows: pair j of tile g -> y[(tile_y[g].x + j) * ys + k]
  int* err;                   // set to a nonzero code on timeout
};

// The epilogue warps make operator `op` resident: thread 0 bulk-copies its hi
// and lo K-blocks (their bytes counted on a_full), then every epilogue thread
// arrives.  The operator's scale 2^f is read from global memory by the
// epilogue with the tile's other data.
template <int NKB>
__device__ __forceinline__ void load_operator(const Params& P, int op, int row, unsigned char* sOp,
                                              uint64_t* a_full) {
  if (row == 0) {
    const unsigned char* img = P.opimg + (size_t)op * P.img_bytes;
    const uint32_t kb_bytes = (uint32_t)P.n * kRowBytes;
    mbar_expect_tx(a_full, 2 * NKB * kb_bytes);
    for (int c = 0; c < 2 * NKB; c++) bulk_g2s(sOp + (size_t)c * kb_bytes, img + (size_t)c * kb_bytes, kb_bytes, a_full);
  }
  mbar_arrive(a_full);
}

template <int NKB>
__global__ void __launch_bounds__(Cfg<NKB>::kThreads, 1) translate_h16(Params P) {
  using C = Cfg<NKB>;
  constexpr int kStages = C::kStages, kGW = C::kGroupWarps;
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char* smem = (unsigned char*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  unsigned char* sOp = smem;                    // resident operator: hi K-blocks then lo K-blocks (n rows each)
  unsigned char* sB = smem + C::kOpBytes;       // input ring
  float* sStg = (float*)(sB + kStages * kStageBytes);  // [4 warps][32][kStgStride] transpose buffers
  uint64_t* full = (uint64_t*)((unsigned char*)sStg + kStgBytes);
  uint64_t* empty = full + kStages;
  uint64_t* accf = empty + kStages;  // [2] accumulator b holds a finished tile
  uint64_t* acce = accf + 2;         // [2] accumulator b read out by the epilogue
  uint64_t* a_full = acce + 2;       // operator resident
  uint64_t* drain = a_full + 1;      // every MMA done (before tensor memory is freed)
  uint32_t* tmem_slot = (uint32_t*)(drain + 1);
  __shared__ int sh_fail;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int t_begin = (int)((long long)P.ntile * blockIdx.x / gridDim.x);
  const int t_end = (int)((long long)P.ntile * (blockIdx.x + 1) / gridDim.x);
  const int ntile = t_end - t_begin;
  const int nstage_total = ntile * NKB;
  const uint32_t kb_bytes = (uint32_t)P.n * kRowBytes;

  if (threadIdx.x == 0) {
    sh_fail = 0;
    for (int s = 0; s < kStages; s++) {
      mbar_init(&full[s], C::kGroupThreads);  // the producers of ring slot s
      mbar_init(&empty[s], 1);                // one tcgen05.commit
    }
    for (int b = 0; b < 2; b++) {
      mbar_init(&accf[b], 1);    // tcgen05.commit after a tile's MMAs
      mbar_init(&acce[b], 128);  // every epilogue thread after reading the tile
    }
    mbar_init(a_full, 128);      // every epilogue thread (+ the operator bytes)
    mbar_init(drain, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    prefetch_l2(P.tile_src + (size_t)t_begin * kTile, (uint32_t)(ntile * kTile * sizeof(int)));
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
    // group s fills ring slot s for stages s, s + kStages, ...  A stage is the
    // tile's 128 input rows x (hi, lo) x 128 bytes of one K-block; one warp
    // instruction copies two rows (lanes 0-7: the hi line of the first row,
    // 8-15: its lo line, 16-31: the same for the second row).
    const int grp = (warp - 5) / kGW;
    const int gw = (warp - 5) % kGW;
    const int part = (lane >> 3) & 1, chunk = lane & 7;
    constexpr int kRowsPerThread = kTile / (2 * kGW);
    const int kpad = NKB * kKB;
    unsigned char* bdst = sB + grp * kStageBytes + part * kAHalf;
    const int rsel = gw * 2 + (lane >> 4);  // this thread's rows: k * 2 kGW + rsel
    int src[kRowsPerThread];                // input rows of the stage about to be filled
    if (grp < nstage_total) {
      const int* tsrc = P.tile_src + (size_t)(t_begin + grp / NKB) * kTile;
#pragma unroll
      for (int k = 0; k < kRowsPerThread; k++) src[k] = __ldg(tsrc + k * 2 * kGW + rsel);
    }
    for (int st = grp; st < nstage_total; st += kStages) {
      const uint32_t ph = (st / kStages) & 1;
      bool ok = true;
      if (st >= kStages && lane == 0) ok = mbar_wait(&empty[grp], ph ^ 1);
      ok = __shfl_sync(0xffffffffu, ok ? 1 : 0, 0) != 0;
      if (!ok) atomicExch(&sh_fail, 1);
      if (!ok || *(volatile int*)&sh_fail) break;
      const int kb = st % NKB;
#pragma unroll
      for (int k = 0; k < kRowsPerThread; k++) {
        const int r = k * 2 * kGW + rsel;
        unsigned char* d = bdst + swz(r, chunk);
        if (src[k] >= 0)
          cp_async16(d, P.xin + (size_t)src[k] * (2 * kpad) + part * kpad + kb * kKB + 8 * chunk);
        else
          *reinterpret_cast<float4*>(d) = make_float4(0.f, 0.f, 0.f, 0.f);
      }
      cp_async_commit();
      // the next stage's input rows, loaded while this stage's copies land
      const int st2 = st + kStages;
      if (st2 < nstage_total && st2 / NKB != st / NKB) {
        const int* tsrc = P.tile_src + (size_t)(t_begin + st2 / NKB) * kTile;
#pragma unroll
        for (int k = 0; k < kRowsPerThread; k++) src[k] = __ldg(tsrc + k * 2 * kGW + rsel);
      }
      cp_async_wait_all();
      fence_async_smem();
      mbar_arrive(&full[grp]);
    }
    cp_async_wait_all();
  } else if (warp == 4) {
    // ------------------------------------------------ MMA issuer
    // first the operator images of this CTA's tiles into L2 (the lanes in
    // parallel, one prefetch per operator run)
    for (int i = lane; i < ntile; i += 32) {
      const int op = P.tile_op[t_begin + i];
      if (i == 0 || P.tile_op[t_begin + i - 1] != op)
        prefetch_l2(P.opimg + (size_t)op * P.img_bytes, (uint32_t)(P.img_bytes & ~(size_t)15));
    }
    __syncwarp();
    const uint32_t idesc = idesc_f16(P.n);
    bool ok = true;
    int cur_op = -1, nload = 0;
    for (int i = 0; i < ntile && ok; i++) {
      const int g = t_begin + i;
      const int buf = i & 1;
      const uint32_t dcol = tmem + (uint32_t)(buf * kAccStride);
      const int op = P.tile_op[g];
      if (op != cur_op) {  // the epilogue loads each new operator once the MMAs using the old one are done
        if (lane == 0) ok = mbar_wait(a_full, nload & 1);
        ok = __shfl_sync(0xffffffffu, ok ? 1 : 0, 0) != 0;
        if (!ok) break;
        cur_op = op;
        nload++;
      }
      if (i >= 2) {  // the epilogue has read this accumulator
        if (lane == 0) ok = mbar_wait(&acce[buf], ((i >> 1) - 1) & 1);
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
          const uint32_t ahi = smem_u32(sB + s * kStageBytes), alo = ahi + kAHalf;
          const uint32_t bhi = smem_u32(sOp + (size_t)kb * kb_bytes);
          const uint32_t blo = smem_u32(sOp + (size_t)(NKB + kb) * kb_bytes);
#pragma unroll
          for (int k = 0; k < kKB / 16; k++) {  // 4 MMAs of K = 16 per K-block
            const uint32_t o = k * 32;            // 16 FP16 = 32 bytes along K
            mma_f16(dcol, make_desc(ahi + o), make_desc(bhi + o), idesc, (kb | k) ? 1u : 0u);
            mma_f16(dcol, make_desc(ahi + o), make_desc(blo + o), idesc, 1u);
            mma_f16(dcol, make_desc(alo + o), make_desc(bhi + o), idesc, 1u);
          }
          mma_commit(&empty[s]);  // frees the ring slot once these MMAs are done
          if (kb == NKB - 1) mma_commit(&accf[buf]);
        }
        __syncwarp();
      }
    }
    if (!ok && lane == 0) atomicExch(&sh_fail, 2);
    if (lane == 0) {
      mma_commit(drain);
      mbar_wait(drain, 0);
    }
    __syncwarp();
  } else {
    // ------------------------------------------------ epilogue (warps 0..3)
    // thread `row` owns pair `row` of each tile (tensor-memory lane `row`):
    // it loads each new operator and undoes the scalings; each warp then
    // writes its 32 pair rows, 32 coefficients at a time, through its
    // transpose buffer (lane l of a store covers 16 bytes of row 4 k + l / 8)
    const int row = warp * 32 + lane;
    const uint32_t lane_base = tmem + ((uint32_t)(warp * 32) << 16);
    const int nch = (P.n + 31) / 32;
    float* stg = sStg + warp * 32 * kStgStride;
    bool ok = true;
    if (ntile > 0) load_operator<NKB>(P, P.tile_op[t_begin], row, sOp, a_full);
    // this tile's data (the next tile's is loaded while this one is stored)
    int src = -1, xe = 0;
    float osc = 0.f;
    int2 ty = make_int2(0, 0);
    if (ntile > 0) {
      src = __ldg(P.tile_src + (size_t)t_begin * kTile + row);
      xe = src >= 0 ? __ldg(P.xexp + src) : 0;
      osc = __ldg(reinterpret_cast<const float*>(P.opimg + (size_t)P.tile_op[t_begin] * P.img_bytes +
                                                 (size_t)2 * NKB * kb_bytes));
      ty = P.tile_y[t_begin];
    }
    for (int i = 0; i < ntile; i++) {
      const int g = t_begin + i;
      const int buf = i & 1;
      const int nsrc = i + 1 < ntile ? __ldg(P.tile_src + (size_t)(g + 1) * kTile + row) : -1;
      const int nop = i + 1 < ntile ? P.tile_op[g + 1] : -1;
      const float nosc = i + 1 < ntile ? __ldg(reinterpret_cast<const float*>(
                                             P.opimg + (size_t)nop * P.img_bytes + (size_t)2 * NKB * kb_bytes))
                                       : 0.f;
      const int2 nty = i + 1 < ntile ? P.tile_y[g + 1] : make_int2(0, 0);
      const bool w = mbar_wait(&accf[buf], (i >> 1) & 1);
      ok = __all_sync(0xffffffffu, w && *(volatile int*)&sh_fail == 0) != 0;
      if (!ok) break;
      tc_fence_after();
      if (i + 1 < ntile && nop != P.tile_op[g])  // every MMA up to tile i is done
        load_operator<NKB>(P, nop, row, sOp, a_full);
      const int nxe = nsrc >= 0 ? __ldg(P.xexp + nsrc) : 0;
      const float f = src >= 0 ? osc * pow2f(xe) : 0.f;
      const unsigned live = __ballot_sync(0xffffffffu, src >= 0);  // pairs of this warp with a source
      float* ybase = P.y + ((size_t)ty.x + warp * 32) * P.ys;
      for (int c = 0; c < nch; c++) {
        uint32_t v[32];
        tmem_ld32(lane_base + (uint32_t)(buf * kAccStride + c * 32), v);
        if (c == nch - 1) {  // the accumulator is free once read
          tc_fence_before();
          mbar_arrive(&acce[buf]);
        }
        __syncwarp();
#pragma unroll
        for (int q = 0; q < 8; q++) {
          float4 o;
          o.x = __uint_as_float(v[4 * q + 0]) * f;
          o.y = __uint_as_float(v[4 * q + 1]) * f;
          o.z = __uint_as_float(v[4 * q + 2]) * f;
          o.w = __uint_as_float(v[4 * q + 3]) * f;
          *reinterpret_cast<float4*>(stg + lane * kStgStride + 4 * q) = o;
        }
        __syncwarp();
        const int k = c * 32 + 4 * (lane & 7);  // this lane's 4 coefficients
#pragma unroll
        for (int rr = 0; rr < 8; rr++) {
          const int r = 4 * rr + (lane >> 3);  // row of the warp's 32
          if (k < P.ys && ((live >> r) & 1u)) {
            float4 o = *reinterpret_cast<const float4*>(stg + r * kStgStride + 4 * (lane & 7));
            if (k + 3 >= P.K) {  // zero the padding of the row past K
              if (k + 0 >= P.K) o.x = 0.f;
              if (k + 1 >= P.K) o.y = 0.f;
              if (k + 2 >= P.K) o.z = 0.f;
              if (k + 3 >= P.K) o.w = 0.f;
            }
            __stcs(reinterpret_cast<float4*>(ybase + (size_t)r * P.ys + k), o);  // streamed: keep L2 for the inputs
          }
        }
      }
      src = nsrc;
      xe = nxe;
      osc = nosc;
      ty = nty;
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

// M (FP64, [nbox][K]) -> xh ([nbox][2][kpad] FP16: hi, lo of M * 2^-e, zero
// padded) and xexp[box] = e with the box's largest |coefficient| * 2^-e in
// [2^14, 2^15) (e = 0 for an all-zero box).  One warp per box.
__global__ void split_h16(int nbox, int K, int kpad, const double* __restrict__ M, __half* __restrict__ xh,
                          int* __restrict__ xexp) {
  const int w = (int)((blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5);
  const int lane = threadIdx.x & 31;
  if (w >= nbox) return;
  const double* m = M + (size_t)w * K;
  double mx = 0.0;
  for (int k = lane; k < K; k += 32) mx = fmax(mx, fabs(m[k]));
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  int e = 0;
  if (mx > 0.0) {
    frexp(mx, &e);  // mx = f 2^e, f in [0.5, 1)
    e -= 15;
  }
  __half* hi = xh + (size_t)w * 2 * kpad;
  __half* lo = hi + kpad;
  for (int k = lane; k < kpad; k += 32) {
    __half h = __float2half(0.f), l = __float2half(0.f);
    if (k < K) {
      const double x = ldexp(m[k], -e);
      h = __double2half(x);
      l = __double2half(x - (double)__half2float(h));
    }
    hi[k] = h;
    lo[k] = l;
  }
  if (lane == 0) xexp[w] = e;
}

}  // namespace h16

int h16_max_k() { return h16::Cfg<3>::kNMax; }
int h16_n(int K) { return (K + 15) / 16 * 16; }
int h16_kpad(int K) { return K <= 2 * h16::kKB ? 2 * h16::kKB : 3 * h16::kKB; }
size_t h16_img_bytes(int K) { return (size_t)2 * (h16_kpad(K) / h16::kKB) * h16_n(K) * h16::kRowBytes + 16; }

void prepare_translate_h16() {
  FMMB_CUDA(cudaFuncSetAttribute(h16::translate_h16<2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 h16::Cfg<2>::kSmemBytes));
  FMMB_CUDA(cudaFuncSetAttribute(h16::translate_h16<3>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 h16::Cfg<3>::kSmemBytes));
}

void launch_split_h16(int nbox, int K, const double* M, void* xh, int* xexp, cudaStream_t st) {
  if (nbox <= 0) return;
  const size_t threads = (size_t)nbox * 32;
  h16::split_h16<<<(unsigned)((threads + 255) / 256), 256, 0, st>>>(nbox, K, h16_kpad(K), M, (__half*)xh, xexp);
  FMMB_CHECK_LAUNCH();
}

void launch_translate_h16(const H16JobArgs& a, int nsm, cudaStream_t st) {
  if (a.ntile <= 0) return;
  h16::Params P{};
  P.ntile = a.ntile;
  P.n = h16_n(a.K);
  P.K = a.K;
  P.ys = a.ys;
  P.tile_op = a.tile_op;
  P.tile_src = a.tile_src;
  P.tile_y = a.tile_y;
  P.opimg = (const unsigned char*)a.opimg;
  P.img_bytes = h16_img_bytes(a.K);
  P.xin = (const __half*)a.xin;
  P.xexp = a.xexp;
  P.y = a.y;
  P.err = a.err;
  const int grid = a.ntile < nsm ? a.ntile : nsm;
  if (h16_kpad(a.K) == 2 * h16::kKB)
    h16::translate_h16<2><<<grid, h16::Cfg<2>::kThreads, h16::Cfg<2>::kSmemBytes, st>>>(P);
  else
    h16::translate_h16<3><<<grid, h16::Cfg<3>::kThreads, h16::Cfg<3>::kSmemBytes, st>>>(P);
  FMMB_CHECK_LAUNCH();
}

}  // namespace fmmb

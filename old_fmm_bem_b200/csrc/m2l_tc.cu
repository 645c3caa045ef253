// M2L on the 5th-generation tensor cores (tcgen05, TMEM accumulators), TF32x3.
//
// Same operator as kernels_fp64.cu's m2l_f64 (the reference's
// rotate / z-translate / rotate-back M2L of kernel/m2l.cxx:30-83 composed into
// one real K x K matrix per relative position, operators.cpp), applied as
//
//   L[:, tile] += sum over active slots d of  T_d (128 x 128) . M[src(tile, d)] (128 x 128)
//
// for a tile of 64 target boxes of one octant at one level (they share the
// slot -> operator map).  Each product is split into three TF32 MMAs,
// A_hi.B_hi + A_hi.B_lo + A_lo.B_hi, where hi/lo are the TF32 rounding of a
// value and of its remainder (about 2^-21 relative error per product instead
// of 2^-11 for plain TF32).  One slot's product (128 coefficients x 64
// targets, 48 MMAs) is accumulated in FP32 in tensor memory; two such
// accumulators alternate, and while the tensor core fills one the epilogue
// warps drain the other into FP64 registers, so the FP32 accumulation depth
// is one slot instead of ~100.
//
// Operands use the K-major SWIZZLE_128B shared-memory layout: per K-block of
// 32 TF32 values a tile row is 128 bytes, 8-row groups are 1024 bytes apart,
// and the 16-byte chunk c of row r sits at chunk c ^ (r & 7).  The operator
// K-blocks are stored in global memory as exactly that image, so one
// cp.async.bulk per K-block loads them; the source multipoles are gathered by
// the producer warps with 16-byte loads and swizzled stores.
//
// Warp roles (288 threads): warps 0..3 drain the accumulators (tcgen05.ld
// 32x32b: warp w sees TMEM lanes 32w..32w+31 = coefficients) and own the FP64
// sums; warp 4 owns the tensor memory and one lane issues the MMAs; warps 5..8
// produce the pipeline stages.  Every mbarrier wait is bounded: on timeout the
// kernel records an error code, skips the remaining work and still frees its
// tensor memory.
#include <cuda_runtime.h>

#include <cstdint>

#include "internal.h"
#include "kernels.h"

namespace fmmb {
namespace tc {

constexpr int kTile = 64;         // target boxes per tile (MMA N)
constexpr int kRows = 128;        // output coefficients (MMA M), K <= 128
constexpr int kKB = 32;           // TF32 values per K-block (128 bytes)
constexpr int kNKB = 4;           // K-blocks (K padded to 128)
constexpr int kStages = 4;
constexpr int kOpBytes = kRows * 128;               // operator K-block image (16 KB)
constexpr int kBBytes = kTile * 128;                // gathered multipole K-block (8 KB)
constexpr int kStageBytes = 2 * kOpBytes + 2 * kBBytes;  // A_hi, A_lo, B_hi, B_lo
constexpr int kSmemBytes = kStages * kStageBytes + 1024 + 256;
constexpr int kThreads = 288;
constexpr int kTmemCols = 2 * kTile;                // two alternating accumulators
constexpr unsigned kSpinLimit = 1u << 22;           // bounded waits (seconds at most)

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

// Swizzled byte offset of 16-byte chunk c of row r in a K-block tile.
__device__ __forceinline__ uint32_t swz(int r, int c) { return (uint32_t)(r * 128 + ((c ^ (r & 7)) << 4)); }

struct Params {
  int K;                        // real coefficients per expansion (<= 128)
  const int* tile_boxes;        // [ntile][128] global target box index or -1
  const int* tile_oct;          // [ntile] octant shared by the tile's boxes
  const int* tile_level;        // [ntile]
  const int* work_tile;         // [nwork] tile of each work item (a tile may be split over its slots)
  const int* slot_off;          // [nwork + 1] CSR of the active slots of each work item
  const int* slots;             // active slot numbers
  const int* list;              // [tot_i][189] source box within the level or -1
  const int* slot_rel;          // [8][189]
  const int* rel_to_op;         // [343]
  const float* opimg;           // operator images [sets][316][4][2][128*32]
  long long op_set_off[11];     // float offset of each level's operator set
  const float* Mtf;             // all-level source multipoles [tot_j][2][128] (hi, lo)
  int mtf_box_off[11];          // first box of each level in Mtf
  double* L;                    // all-level locals [tot_i][K]
  int atomic;                   // 1 when a tile is split over several work items
  int* err;                     // set to a nonzero code on timeout
};

__global__ void __launch_bounds__(kThreads, 1) m2l_tc_kernel(Params P) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char* smem = (unsigned char*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  uint64_t* full = (uint64_t*)(smem + kStages * kStageBytes);
  uint64_t* empty = full + kStages;
  uint64_t* accf = empty + kStages;  // [2] accumulator b complete
  uint64_t* acce = accf + 2;         // [2] accumulator b drained
  uint32_t* tmem_slot = (uint32_t*)(acce + 2);
  __shared__ int sh_boxes[kTile];
  __shared__ int sh_fail;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int work = blockIdx.x;
  const int tile = P.work_tile[work];
  const int oct = P.tile_oct[tile];
  const int lev = P.tile_level[tile];
  const float* opimg = P.opimg + P.op_set_off[lev];
  const float* Mtf = P.Mtf + (size_t)P.mtf_box_off[lev] * 256;
  const int s_begin = P.slot_off[work], s_end = P.slot_off[work + 1];
  const int nslot = s_end - s_begin;
  const int nstage_total = nslot * kNKB;

  if (threadIdx.x < kTile) sh_boxes[threadIdx.x] = P.tile_boxes[tile * kTile + threadIdx.x];
  if (threadIdx.x == 0) {
    sh_fail = 0;
    for (int s = 0; s < kStages; s++) {
      mbar_init(&full[s], 129);  // 128 producer arrivals + 1 expect_tx arrival
      mbar_init(&empty[s], 1);   // one tcgen05.commit
    }
    for (int b = 0; b < 2; b++) {
      mbar_init(&accf[b], 1);    // tcgen05.commit after a slot's MMAs
      mbar_init(&acce[b], 128);  // every epilogue thread after its tcgen05.ld
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
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
    // ------------------------------------------------ producers (128 threads)
    const int pt = threadIdx.x - 160;        // 0..127
    const int row = pt >> 1, part = pt & 1;  // one 128-byte row of B_hi or B_lo
    for (int st = 0; st < nstage_total; st++) {
      const int s = st % kStages;
      const uint32_t ph = (st / kStages) & 1;
      if (st >= kStages) {
        if (!mbar_wait(&empty[s], ph ^ 1)) {
          atomicExch(&sh_fail, 1);
          break;
        }
      }
      if (*(volatile int*)&sh_fail) break;
      const int slot = P.slots[s_begin + st / kNKB];
      const int kb = st % kNKB;
      unsigned char* stage = smem + s * kStageBytes;
      if (pt == 0) {
        const int op = P.rel_to_op[P.slot_rel[oct * kM2LSlots + slot]];
        const float* img = opimg + ((size_t)op * kNKB + kb) * 2 * (kRows * kKB);
        mbar_arrive_tx(&full[s], 2 * kOpBytes);
        bulk_g2s(stage, img, kOpBytes, &full[s]);
        bulk_g2s(stage + kOpBytes, img + kRows * kKB, kOpBytes, &full[s]);
      }
      const int box = sh_boxes[row];
      const int src = box >= 0 ? P.list[(size_t)box * kM2LSlots + slot] : -1;
      unsigned char* dst = stage + 2 * kOpBytes + part * kBBytes;
      if (src >= 0) {
        const float4* g = reinterpret_cast<const float4*>(Mtf + (size_t)src * 256 + part * 128 + kb * kKB);
#pragma unroll
        for (int c = 0; c < 8; c++) *reinterpret_cast<float4*>(dst + swz(row, c)) = __ldg(g + c);
      } else {
        const float4 z = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
        for (int c = 0; c < 8; c++) *reinterpret_cast<float4*>(dst + swz(row, c)) = z;
      }
      fence_async_smem();
      mbar_arrive(&full[s]);
    }
  } else if (warp == 4) {
    // ------------------------------------------------ MMA issuer
    bool ok = true;
    for (int g = 0; g < nslot && ok; g++) {
      const int buf = g & 1;
      const uint32_t dcol = tmem + (uint32_t)(buf * kTile);
      if (g >= 2) {  // wait until the epilogue has drained this accumulator
        if (lane == 0) ok = mbar_wait(&acce[buf], ((g >> 1) - 1) & 1);
        ok = __shfl_sync(0xffffffffu, ok ? 1 : 0, 0) != 0;
        if (!ok) break;
        tc_fence_after();
      }
      for (int kb = 0; kb < kNKB && ok; kb++) {
        const int st = g * kNKB + kb;
        const int s = st % kStages;
        const uint32_t ph = (st / kStages) & 1;
        if (lane == 0) ok = mbar_wait(&full[s], ph);
        ok = __shfl_sync(0xffffffffu, ok ? 1 : 0, 0) != 0;
        if (!ok) break;
        tc_fence_after();
        if (lane == 0) {
          const uint32_t base = smem_u32(smem + s * kStageBytes);
          const uint32_t ahi = base, alo = base + kOpBytes, bhi = base + 2 * kOpBytes, blo = bhi + kBBytes;
#pragma unroll
          for (int k = 0; k < kKB / 8; k++) {  // 4 MMAs of K=8 per 32-wide block
            const uint32_t o = k * 32;           // 8 TF32 = 32 bytes along K
            mma_tf32(dcol, make_desc(ahi + o), make_desc(bhi + o), (kb | k) ? 1u : 0u);
            mma_tf32(dcol, make_desc(ahi + o), make_desc(blo + o), 1u);
            mma_tf32(dcol, make_desc(alo + o), make_desc(bhi + o), 1u);
          }
          mma_commit(&empty[s]);  // frees the stage when these MMAs are done
          if (kb == kNKB - 1) mma_commit(&accf[buf]);
        }
        __syncwarp();
      }
    }
    if (!ok && lane == 0) atomicExch(&sh_fail, 2);
  } else {
    // ------------------------------------------------ epilogue (warps 0..3)
    const int row = warp * 32 + lane;  // output coefficient of this thread
    double acc[kTile];
#pragma unroll
    for (int j = 0; j < kTile; j++) acc[j] = 0.0;
    bool ok = true;
    for (int g = 0; g < nslot; g++) {
      const int buf = g & 1;
      bool w = mbar_wait(&accf[buf], (g >> 1) & 1);
      ok = __all_sync(0xffffffffu, w && *(volatile int*)&sh_fail == 0) != 0;
      if (!ok) break;
      tc_fence_after();
      float v[32];
#pragma unroll
      for (int h = 0; h < kTile / 32; h++) {
        tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(buf * kTile + h * 32), v);
#pragma unroll
        for (int j = 0; j < 32; j++) acc[h * 32 + j] += (double)v[j];
      }
      tc_fence_before();
      mbar_arrive(&acce[buf]);
    }
    if (!ok) atomicExch(&sh_fail, 3);
    if (ok && row < P.K) {
#pragma unroll
      for (int j = 0; j < kTile; j++) {
        const int box = sh_boxes[j];
        if (box >= 0) {
          double* dst = P.L + (size_t)box * P.K + row;
          if (P.atomic) atomicAdd(dst, acc[j]);
          else *dst += acc[j];
        }
      }
    }
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

// M (FP64, [nbox][K]) -> Mtf ([nbox][2][128] FP32: TF32 hi, TF32 lo, zero padded)
__global__ void split_tf32(int nbox, int K, const double* __restrict__ M, float* __restrict__ Mtf) {
  const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i >= (size_t)nbox * 128) return;
  const size_t b = i / 128;
  const int k = (int)(i % 128);
  float hi = 0.f, lo = 0.f;
  if (k < K) {
    const double x = M[b * K + k];
    hi = tf32_rna((float)x);
    lo = tf32_rna((float)(x - (double)hi));
  }
  Mtf[b * 256 + k] = hi;
  Mtf[b * 256 + 128 + k] = lo;
}

}  // namespace tc

int m2l_tc_tile() { return tc::kTile; }

void launch_split_tf32(int nbox, int K, const double* M, float* Mtf, cudaStream_t st) {
  if (nbox <= 0) return;
  const size_t n = (size_t)nbox * 128;
  tc::split_tf32<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(nbox, K, M, Mtf);
  FMMB_CHECK_LAUNCH();
}

void launch_m2l_tc(const M2LTcArgs& a, cudaStream_t st) {
  if (a.nwork <= 0) return;
  FMMB_CUDA(cudaFuncSetAttribute(tc::m2l_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, tc::kSmemBytes));
  tc::Params P{};
  P.K = a.K;
  P.tile_boxes = a.tile_boxes;
  P.tile_oct = a.tile_oct;
  P.tile_level = a.tile_level;
  P.work_tile = a.work_tile;
  P.slot_off = a.slot_off;
  P.slots = a.slots;
  P.list = a.list;
  P.slot_rel = a.slot_rel;
  P.rel_to_op = a.rel_to_op;
  P.opimg = a.opimg;
  P.Mtf = a.Mtf;
  for (int l = 0; l < 11; l++) {
    P.op_set_off[l] = a.op_set_off[l];
    P.mtf_box_off[l] = a.mtf_box_off[l];
  }
  P.L = a.L;
  P.atomic = a.atomic;
  P.err = a.err;
  tc::m2l_tc_kernel<<<a.nwork, tc::kThreads, tc::kSmemBytes, st>>>(P);
  FMMB_CHECK_LAUNCH();
}

}  // namespace fmmb

// Near-field P2P in FP32 with compensated per-target accumulation.
//
// Same sums as the reference's P2P kernels (kernel/G_p2p.cxx:12-37,
// kernel/Gni_p2p.cxx:12-28, kernel/Gnj_p2p.cxx:12-28) over the 27-slot
// neighbour lists of the GPU tree.  Pair arithmetic is FP32 (hardware rsqrt);
// each thread sums 32 sources at a time in FP32 and promotes every partial sum
// into FP64 accumulators, so the accumulated rounding stays at the FP32 level
// of one 32-term sum whatever the number of sources.
//
// Layout: one block of 4 warps per target leaf.  The sources of all
// neighbour leaves are staged once into shared memory as one list -- the
// leaf's own source leaf first, padded to a multiple of 32 with far,
// zero-charge points, then the other neighbours, padded likewise -- so that
// every run of 32 sources needs no bounds check, and only runs of the own leaf
// test for coincident points (points at zero distance share a leaf).  A pass
// covers NT columns of 32 targets (NT = 1..4, as many as the leaf needs, so
// a leaf of 53 targets fills 83% of its lanes); each lane holds the NT
// targets of its column position, so one shared-memory read of a source
// serves NT pairs; warp w takes runs w, w+4, ... and the four warps' FP64
// partial sums are added through shared memory at the end of a pass.
#include <cuda_runtime.h>

#include "internal.h"
#include "kernels.h"

namespace fmmb {
namespace {

constexpr int kThreads = 128;
constexpr int kWarps = kThreads / 32;
constexpr int kMaxNT = 4;     // target columns of 32 per pass
constexpr int kCap = 1024;    // staged sources per chunk (multiple of 32)
constexpr int kSelfSlot = 13; // offset (0, 0, 0) in the 27-slot list
constexpr float kFar = 1e18f; // padding sources: r^2 ~ 3e36 stays finite in FP32

__device__ __forceinline__ int pad32(int n) { return (n + 31) & ~31; }

// 1/sqrt(x) from the hardware approximation, subnormal inputs flushed to zero
// (r^2 is either 0 -- coincident points, handled by the caller -- or far
// above the subnormal range for any pair of distinct float positions in
// neighbouring leaves), so no subnormal fix-up instructions are emitted.
__device__ __forceinline__ float rsqrt_ftz(float x) {
  float y;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

template <int KER>
struct Acc {
  float p, fx, fy, fz;
};

// One run of 32 staged sources against the thread's NT targets.
template <int KER, bool EXCL, int NT>
__device__ __forceinline__ void run32(const float4* __restrict__ sp, const float4* __restrict__ sm, const float4* xt,
                                      const float4* nt, float eps2, Acc<KER>* acc) {
#pragma unroll 4
  for (int k = 0; k < 32; k++) {
    const float4 xj = sp[k];
    float4 mj = make_float4(0.f, 0.f, 0.f, 0.f);
    if (KER == FMMB_LAPLACE_GNJ) mj = sm[k];
#pragma unroll
    for (int t = 0; t < NT; t++) {
      const float4 xi = xt[t];
      Acc<KER>& c = acc[t];
      const float dx = xi.x - xj.x, dy = xi.y - xj.y, dz = xi.z - xj.z;
      const float r2 = fmaf(dx, dx, fmaf(dy, dy, fmaf(dz, dz, eps2)));
      float rinv = rsqrt_ftz(r2);
      if (EXCL) rinv = (r2 > 0.f) ? rinv : 0.f;
      if (KER == FMMB_LAPLACE_G) {
        const float qr = xj.w * rinv;
        const float qr3 = qr * rinv * rinv;
        c.p += qr;
        c.fx = fmaf(dx, qr3, c.fx);
        c.fy = fmaf(dy, qr3, c.fy);
        c.fz = fmaf(dz, qr3, c.fz);
      } else if (KER == FMMB_LAPLACE_GNI) {
        const float4 nv = nt[t];
        const float qr3 = xj.w * rinv * rinv * rinv;
        c.p = fmaf(fmaf(dx, nv.x, fmaf(dy, nv.y, dz * nv.z)), qr3, c.p);
      } else {
        const float r3 = rinv * rinv * rinv;
        c.p = fmaf(fmaf(dx, mj.x, fmaf(dy, mj.y, dz * mj.z)), r3, c.p);
      }
    }
  }
}

// Shared state of one block (one target leaf).
template <int KER>
struct Smem {
  static constexpr int NC = KER == FMMB_LAPLACE_G ? 4 : 1;  // accumulated components
  float4 sp[kCap];                                          // x, y, z, q (Gnj: q unused)
  float4 sm[KER == FMMB_LAPLACE_GNJ ? kCap : 1];            // q * n_j (Gnj)
  double red[kWarps - 1][NC][kMaxNT * 32];
  int2 seg[kP2PSlots];                                      // (first source, count), own leaf first
  int nseg;
};

// Stages virtual sources [c0, c1): far zero-charge points, then every
// segment's part of the chunk.
template <int KER>
__device__ void stage(Smem<KER>& S, int c0, int c1, int self_end, const float4* __restrict__ spos,
                      const float4* __restrict__ snrm, const float* __restrict__ qs) {
  __syncthreads();
  for (int e = threadIdx.x; e < c1 - c0; e += kThreads) {
    S.sp[e] = make_float4(kFar, kFar, kFar, 0.f);
    if (KER == FMMB_LAPLACE_GNJ) S.sm[e] = make_float4(0.f, 0.f, 0.f, 0.f);
  }
  __syncthreads();
  int v0 = 0;  // virtual start of the segment
  for (int s = 0; s < S.nseg; s++) {
    const int2 sg = S.seg[s];
    const int lo = max(v0, c0), hi = min(v0 + sg.y, c1);
    for (int v = lo + (int)threadIdx.x; v < hi; v += kThreads) {
      const int j = sg.x + (v - v0);
      float4 x = spos[j];
      const float q = qs[j];
      x.w = q;
      S.sp[v - c0] = x;
      if (KER == FMMB_LAPLACE_GNJ) {
        const float4 nj = snrm[j];
        S.sm[v - c0] = make_float4(q * nj.x, q * nj.y, q * nj.z, 0.f);
      }
    }
    v0 = (s == 0) ? self_end : v0 + sg.y;
  }
  __syncthreads();
}

// One pass over target columns [t0, t0 + 32*NT) of the leaf.
template <int KER, bool EXCL, int NT>
__device__ void pass(Smem<KER>& S, int2 li, int t0, bool restage, int self_end, int vlen,
                     const float4* __restrict__ tpos, const float4* __restrict__ tnrm,
                     const float4* __restrict__ spos, const float4* __restrict__ snrm, const float* __restrict__ qs,
                     float eps2, double coef, double* __restrict__ pot, double* __restrict__ grad, int ni) {
  constexpr int NC = Smem<KER>::NC;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
  float4 xt[NT], nt[NT];
  double P[NT][NC];
#pragma unroll
  for (int t = 0; t < NT; t++) {
    const int it = t0 + t * 32 + lane;
    xt[t] = it < li.y ? tpos[li.x + it] : z4;
    nt[t] = (KER == FMMB_LAPLACE_GNI && it < li.y) ? tnrm[li.x + it] : z4;
#pragma unroll
    for (int c = 0; c < NC; c++) P[t][c] = 0.0;
  }
  const int nchunk = (vlen + kCap - 1) / kCap;
  for (int ch = 0; ch < nchunk; ch++) {
    const int c0 = ch * kCap, c1 = min(vlen, c0 + kCap);
    if (restage || nchunk > 1) stage<KER>(S, c0, c1, self_end, spos, snrm, qs);
    // runs of 32 sources: warp w takes runs w, w + 4, ...
    for (int r0 = c0 + warp * 32; r0 < c1; r0 += kWarps * 32) {
      Acc<KER> acc[NT];
#pragma unroll
      for (int t = 0; t < NT; t++) acc[t] = Acc<KER>{0.f, 0.f, 0.f, 0.f};
      const float4* sp = S.sp + (r0 - c0);
      const float4* sm = S.sm + (KER == FMMB_LAPLACE_GNJ ? r0 - c0 : 0);
      if (EXCL && r0 < self_end)
        run32<KER, true, NT>(sp, sm, xt, nt, eps2, acc);
      else
        run32<KER, false, NT>(sp, sm, xt, nt, eps2, acc);
#pragma unroll
      for (int t = 0; t < NT; t++) {
        P[t][0] += (double)acc[t].p;
        if (KER == FMMB_LAPLACE_G) {
          P[t][1] += (double)acc[t].fx;
          P[t][2] += (double)acc[t].fy;
          P[t][3] += (double)acc[t].fz;
        }
      }
    }
  }
  // add the warps' partial sums
  if (warp > 0) {
#pragma unroll
    for (int t = 0; t < NT; t++)
#pragma unroll
      for (int c = 0; c < NC; c++) S.red[warp - 1][c][t * 32 + lane] = P[t][c];
  }
  __syncthreads();
  if (warp == 0) {
#pragma unroll
    for (int t = 0; t < NT; t++) {
#pragma unroll
      for (int w = 0; w < kWarps - 1; w++)
#pragma unroll
        for (int c = 0; c < NC; c++) P[t][c] += S.red[w][c][t * 32 + lane];
      const int it = t0 + t * 32 + lane;
      if (it < li.y) {
        const int i = li.x + it;
        pot[i] = coef * P[t][0];
        if (KER == FMMB_LAPLACE_G && grad) {
          grad[i] = -coef * P[t][1];
          grad[ni + i] = -coef * P[t][2];
          grad[2 * (size_t)ni + i] = -coef * P[t][3];
        }
      }
    }
  }
  __syncthreads();
}

template <int KER, bool EXCL>
__global__ void __launch_bounds__(kThreads) p2p_mixed(const int2* __restrict__ leaf_i, const int2* __restrict__ leaf_j,
                                                      const int* __restrict__ list, const float4* __restrict__ tpos,
                                                      const float4* __restrict__ tnrm, const float4* __restrict__ spos,
                                                      const float4* __restrict__ snrm, const float* __restrict__ qs,
                                                      float eps2, double coef, double* __restrict__ pot,
                                                      double* __restrict__ grad, int ni) {
  __shared__ Smem<KER> S;
  const int b = blockIdx.x;
  const int2 li = leaf_i[b];
  if (threadIdx.x == 0) {
    int n = 0;
    const int self = list[(size_t)b * kP2PSlots + kSelfSlot];
    S.seg[n++] = self >= 0 ? leaf_j[self] : make_int2(0, 0);
    for (int s = 0; s < kP2PSlots; s++) {
      const int jl = list[(size_t)b * kP2PSlots + s];
      if (s != kSelfSlot && jl >= 0) S.seg[n++] = leaf_j[jl];
    }
    S.nseg = n;
  }
  __syncthreads();
  int n_other = 0;
  for (int s = 1; s < S.nseg; s++) n_other += S.seg[s].y;
  const int self_end = pad32(S.seg[0].y);                // virtual list: [own | pad | others | pad]
  const int vlen = self_end + pad32(n_other);
  for (int t0 = 0; t0 < li.y; t0 += kMaxNT * 32) {
    const int nt = min(kMaxNT, (li.y - t0 + 31) / 32);
    const bool restage = t0 == 0;
    switch (nt) {
      case 1:
        pass<KER, EXCL, 1>(S, li, t0, restage, self_end, vlen, tpos, tnrm, spos, snrm, qs, eps2, coef, pot, grad, ni);
        break;
      case 2:
        pass<KER, EXCL, 2>(S, li, t0, restage, self_end, vlen, tpos, tnrm, spos, snrm, qs, eps2, coef, pot, grad, ni);
        break;
      case 3:
        pass<KER, EXCL, 3>(S, li, t0, restage, self_end, vlen, tpos, tnrm, spos, snrm, qs, eps2, coef, pot, grad, ni);
        break;
      default:
        pass<KER, EXCL, 4>(S, li, t0, restage, self_end, vlen, tpos, tnrm, spos, snrm, qs, eps2, coef, pot, grad, ni);
        break;
    }
  }
}

template <int KER>
void launch_k(int nleaf, bool excl, const int2* leaf_i, const int2* leaf_j, const int* list, const float4* tpos,
              const float4* tnrm, const float4* spos, const float4* snrm, const float* qs, float eps2, double coef,
              double* pot, double* grad, int ni, cudaStream_t st) {
  if (excl)
    p2p_mixed<KER, true><<<nleaf, kThreads, 0, st>>>(leaf_i, leaf_j, list, tpos, tnrm, spos, snrm, qs, eps2, coef, pot, grad, ni);
  else
    p2p_mixed<KER, false><<<nleaf, kThreads, 0, st>>>(leaf_i, leaf_j, list, tpos, tnrm, spos, snrm, qs, eps2, coef, pot, grad, ni);
}

}  // namespace

void launch_p2p_mixed(int kernel, int nleaf, const int2* leaf_i, const int2* leaf_j, const int* list, const float4* tpos,
                      const float4* tnrm, const float4* spos, const float4* snrm, const float* qs, const Sem& s,
                      double* pot, double* grad, int ni, cudaStream_t st) {
  if (nleaf <= 0) return;
  const float eps2 = (float)s.eps2;
  const bool excl = s.excl_self != 0;
  if (kernel == FMMB_LAPLACE_G)
    launch_k<FMMB_LAPLACE_G>(nleaf, excl, leaf_i, leaf_j, list, tpos, tnrm, spos, snrm, qs, eps2, s.coef, pot, grad, ni, st);
  else if (kernel == FMMB_LAPLACE_GNI)
    launch_k<FMMB_LAPLACE_GNI>(nleaf, excl, leaf_i, leaf_j, list, tpos, tnrm, spos, snrm, qs, eps2, s.coef, pot, grad, ni, st);
  else
    launch_k<FMMB_LAPLACE_GNJ>(nleaf, excl, leaf_i, leaf_j, list, tpos, tnrm, spos, snrm, qs, eps2, s.coef, pot, grad, ni, st);
  FMMB_CHECK_LAUNCH();
}

}  // namespace fmmb

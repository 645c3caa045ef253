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
// test for coincident points (points at zero distance share a leaf).  Each
// lane holds two targets (a pass covers 64), so one shared-memory read of a
// source serves two pairs; warp w takes runs w, w+4, ... and the four warps'
// FP64 partial sums are added through shared memory at the end of a pass.
#include <cuda_runtime.h>

#include "internal.h"
#include "kernels.h"

namespace fmmb {
namespace {

constexpr int kThreads = 128;
constexpr int kWarps = kThreads / 32;
constexpr int kPass = 64;     // targets per pass (two per lane)
constexpr int kCap = 1024;    // staged sources per chunk (multiple of 32)
constexpr int kSelfSlot = 13; // offset (0, 0, 0) in the 27-slot list
constexpr float kFar = 1e18f; // padding sources: r^2 ~ 3e36 stays finite in FP32

__device__ __forceinline__ int pad32(int n) { return (n + 31) & ~31; }

template <int KER>
struct Acc {
  float p, fx, fy, fz;
};

// One run of 32 staged sources against the thread's two targets.
template <int KER, bool EXCL>
__device__ __forceinline__ void run32(const float4* __restrict__ sp, const float4* __restrict__ sm, float4 xa,
                                      float4 xb, float4 na, float4 nb, float eps2, Acc<KER>& a, Acc<KER>& b) {
#pragma unroll 8
  for (int k = 0; k < 32; k++) {
    const float4 xj = sp[k];
    float4 mj = make_float4(0.f, 0.f, 0.f, 0.f);
    if (KER == FMMB_LAPLACE_GNJ) mj = sm[k];
#pragma unroll
    for (int t = 0; t < 2; t++) {
      const float4 xi = t ? xb : xa;
      Acc<KER>& c = t ? b : a;
      const float dx = xi.x - xj.x, dy = xi.y - xj.y, dz = xi.z - xj.z;
      const float r2 = fmaf(dx, dx, fmaf(dy, dy, fmaf(dz, dz, eps2)));
      float rinv = rsqrtf(r2);
      if (EXCL) rinv = (r2 > 0.f) ? rinv : 0.f;
      if (KER == FMMB_LAPLACE_G) {
        const float qr = xj.w * rinv;
        const float qr3 = qr * rinv * rinv;
        c.p += qr;
        c.fx = fmaf(dx, qr3, c.fx);
        c.fy = fmaf(dy, qr3, c.fy);
        c.fz = fmaf(dz, qr3, c.fz);
      } else if (KER == FMMB_LAPLACE_GNI) {
        const float4 nv = t ? nb : na;
        const float qr3 = xj.w * rinv * rinv * rinv;
        c.p = fmaf(fmaf(dx, nv.x, fmaf(dy, nv.y, dz * nv.z)), qr3, c.p);
      } else {
        const float r3 = rinv * rinv * rinv;
        c.p = fmaf(fmaf(dx, mj.x, fmaf(dy, mj.y, dz * mj.z)), r3, c.p);
      }
    }
  }
}

template <int KER, bool EXCL>
__global__ void __launch_bounds__(kThreads) p2p_mixed(const int2* __restrict__ leaf_i, const int2* __restrict__ leaf_j,
                                                      const int* __restrict__ list, const float4* __restrict__ tpos,
                                                      const float4* __restrict__ tnrm, const float4* __restrict__ spos,
                                                      const float4* __restrict__ snrm, const float* __restrict__ qs,
                                                      float eps2, double coef, double* __restrict__ pot,
                                                      double* __restrict__ grad, int ni) {
  constexpr int NC = KER == FMMB_LAPLACE_G ? 4 : 1;  // accumulated components
  __shared__ float4 sp[kCap];                                   // x, y, z, q (Gnj: q unused)
  __shared__ float4 sm[KER == FMMB_LAPLACE_GNJ ? kCap : 1];     // q * n_j (Gnj)
  __shared__ double red[kWarps - 1][NC][kPass];
  __shared__ int2 seg[kP2PSlots];                               // (first source, count), own leaf first
  __shared__ int nseg_sh;

  const int b = blockIdx.x;
  const int2 li = leaf_i[b];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    int n = 0;
    const int self = list[(size_t)b * kP2PSlots + kSelfSlot];
    seg[n++] = self >= 0 ? leaf_j[self] : make_int2(0, 0);
    for (int s = 0; s < kP2PSlots; s++) {
      const int jl = list[(size_t)b * kP2PSlots + s];
      if (s != kSelfSlot && jl >= 0) seg[n++] = leaf_j[jl];
    }
    nseg_sh = n;
  }
  __syncthreads();
  const int nseg = nseg_sh;
  int n_other = 0;
  for (int s = 1; s < nseg; s++) n_other += seg[s].y;
  const int self_end = pad32(seg[0].y);                  // virtual list: [own | pad | others | pad]
  const int vlen = self_end + pad32(n_other);
  const int nchunk = (vlen + kCap - 1) / kCap;

  for (int t0 = 0; t0 < li.y; t0 += kPass) {
    const int ia = t0 + lane, ib = t0 + 32 + lane;
    const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
    const float4 xa = ia < li.y ? tpos[li.x + ia] : z4;
    const float4 xb = ib < li.y ? tpos[li.x + ib] : z4;
    float4 na = z4, nb = z4;
    if (KER == FMMB_LAPLACE_GNI) {
      if (ia < li.y) na = tnrm[li.x + ia];
      if (ib < li.y) nb = tnrm[li.x + ib];
    }
    double PA[NC], PB[NC];
#pragma unroll
    for (int c = 0; c < NC; c++) PA[c] = PB[c] = 0.0;

    for (int ch = 0; ch < nchunk; ch++) {
      const int c0 = ch * kCap, c1 = min(vlen, c0 + kCap);
      if (nchunk > 1 || t0 == 0) {
        // stage virtual sources [c0, c1): far zero-charge points, then every
        // segment's part of the chunk
        __syncthreads();
        for (int e = threadIdx.x; e < c1 - c0; e += kThreads) {
          sp[e] = make_float4(kFar, kFar, kFar, 0.f);
          if (KER == FMMB_LAPLACE_GNJ) sm[e] = z4;
        }
        __syncthreads();
        int v0 = 0;  // virtual start of the segment
        for (int s = 0; s < nseg; s++) {
          const int2 sg = seg[s];
          const int lo = max(v0, c0), hi = min(v0 + sg.y, c1);
          for (int v = lo + threadIdx.x; v < hi; v += kThreads) {
            const int j = sg.x + (v - v0);
            float4 x = spos[j];
            const float q = qs[j];
            x.w = q;
            sp[v - c0] = x;
            if (KER == FMMB_LAPLACE_GNJ) {
              const float4 nj = snrm[j];
              sm[v - c0] = make_float4(q * nj.x, q * nj.y, q * nj.z, 0.f);
            }
          }
          v0 = (s == 0) ? self_end : v0 + sg.y;
        }
        __syncthreads();
      }
      // runs of 32 sources: warp w takes runs w, w + 4, ...
      for (int r0 = c0 + warp * 32; r0 < c1; r0 += kWarps * 32) {
        Acc<KER> a{0.f, 0.f, 0.f, 0.f}, bb{0.f, 0.f, 0.f, 0.f};
        if (EXCL && r0 < self_end)
          run32<KER, true>(sp + (r0 - c0), sm + (KER == FMMB_LAPLACE_GNJ ? r0 - c0 : 0), xa, xb, na, nb, eps2, a, bb);
        else
          run32<KER, false>(sp + (r0 - c0), sm + (KER == FMMB_LAPLACE_GNJ ? r0 - c0 : 0), xa, xb, na, nb, eps2, a, bb);
        PA[0] += (double)a.p;
        PB[0] += (double)bb.p;
        if (KER == FMMB_LAPLACE_G) {
          PA[1] += (double)a.fx;
          PA[2] += (double)a.fy;
          PA[3] += (double)a.fz;
          PB[1] += (double)bb.fx;
          PB[2] += (double)bb.fy;
          PB[3] += (double)bb.fz;
        }
      }
    }
    // add the warps' partial sums
    if (warp > 0) {
#pragma unroll
      for (int c = 0; c < NC; c++) {
        red[warp - 1][c][lane] = PA[c];
        red[warp - 1][c][32 + lane] = PB[c];
      }
    }
    __syncthreads();
    if (warp == 0) {
#pragma unroll
      for (int w = 0; w < kWarps - 1; w++)
#pragma unroll
        for (int c = 0; c < NC; c++) {
          PA[c] += red[w][c][lane];
          PB[c] += red[w][c][32 + lane];
        }
#pragma unroll
      for (int t = 0; t < 2; t++) {
        const int it = t ? ib : ia;
        if (it < li.y) {
          const int i = li.x + it;
          const double* P = t ? PB : PA;
          pot[i] = coef * P[0];
          if (KER == FMMB_LAPLACE_G && grad) {
            grad[i] = -coef * P[1];
            grad[ni + i] = -coef * P[2];
            grad[2 * (size_t)ni + i] = -coef * P[3];
          }
        }
      }
    }
    __syncthreads();
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

// Near-field P2P in FP32 with compensated per-target accumulation.
//
// Same sums as the reference's P2P kernels (kernel/G_p2p.cxx:12-37,
// kernel/Gni_p2p.cxx:12-28, kernel/Gnj_p2p.cxx:12-28) over the 27-slot
// neighbour lists of the GPU tree.  Pair arithmetic is FP32 (hardware rsqrt);
// each thread sums 32 sources at a time in FP32 and promotes every partial sum
// into FP64 accumulators, so the accumulated rounding stays at the FP32 level
// of one 32-term sum whatever the number of sources.
//
// Layout: one block of 128 threads per target leaf.  Threads 0..63 and
// 64..127 take the same 64 targets and split each staged source chunk in two
// halves; the halves are combined through shared memory at the end (leaves are
// ~64 points, so one thread per target would idle half the block).
#include <cuda_runtime.h>

#include "internal.h"
#include "kernels.h"

namespace fmmb {
namespace {

constexpr int kThreads = 128;
constexpr int kTeam = 64;      // targets per pass
constexpr int kChunk = 256;    // sources staged per pass

template <int KER, bool EXCL>
__global__ void __launch_bounds__(kThreads) p2p_mixed(const int2* __restrict__ leaf_i, const int2* __restrict__ leaf_j,
                                                      const int* __restrict__ list, const float4* __restrict__ tpos,
                                                      const float4* __restrict__ tnrm, const float4* __restrict__ spos,
                                                      const float4* __restrict__ snrm, const float* __restrict__ qs,
                                                      float eps2, double coef, double* __restrict__ pot,
                                                      double* __restrict__ grad, int ni) {
  __shared__ float4 sp[kChunk];
  __shared__ float4 sn[KER == FMMB_LAPLACE_GNJ ? kChunk : 1];
  __shared__ double red[4][kTeam];
  const int b = blockIdx.x;
  const int2 li = leaf_i[b];
  const int t = threadIdx.x & (kTeam - 1);
  const int half = threadIdx.x / kTeam;
  int slots[kP2PSlots];
  int nslot = 0;
  for (int s = 0; s < kP2PSlots; s++) {
    const int jl = list[(size_t)b * kP2PSlots + s];
    if (jl >= 0) slots[nslot++] = jl;
  }
  for (int t0 = 0; t0 < li.y; t0 += kTeam) {
    const bool act = t0 + t < li.y;
    const int i = li.x + t0 + t;
    const float4 xi = act ? tpos[i] : make_float4(0.f, 0.f, 0.f, 0.f);
    const float4 nv = (KER == FMMB_LAPLACE_GNI && act) ? tnrm[i] : make_float4(0.f, 0.f, 0.f, 0.f);
    double P = 0, FX = 0, FY = 0, FZ = 0;
    for (int s = 0; s < nslot; s++) {
      const int2 lj = leaf_j[slots[s]];
      for (int j0 = 0; j0 < lj.y; j0 += kChunk) {
        const int nld = min(kChunk, lj.y - j0);
        __syncthreads();
        for (int e = threadIdx.x; e < nld; e += kThreads) {
          const int j = lj.x + j0 + e;
          float4 v = spos[j];
          v.w = qs[j];
          sp[e] = v;
          if (KER == FMMB_LAPLACE_GNJ) sn[e] = snrm[j];
        }
        __syncthreads();
        // this half's share of the chunk, in runs of 32
        const int mid = (nld + 1) >> 1;
        const int jb = half ? mid : 0, je = half ? nld : mid;
        for (int r0 = jb; r0 < je; r0 += 32) {
          const int r1 = min(je, r0 + 32);
          float p = 0.f, fx = 0.f, fy = 0.f, fz = 0.f;
#pragma unroll 8
          for (int jj = r0; jj < r1; jj++) {
            const float4 xj = sp[jj];
            const float dx = xi.x - xj.x, dy = xi.y - xj.y, dz = xi.z - xj.z;
            const float r2 = fmaf(dx, dx, fmaf(dy, dy, fmaf(dz, dz, eps2)));
            float rinv = rsqrtf(r2);
            if (EXCL) rinv = (r2 > 0.f) ? rinv : 0.f;
            if (KER == FMMB_LAPLACE_G) {
              const float qr = xj.w * rinv;
              const float qr3 = qr * rinv * rinv;
              p += qr;
              fx = fmaf(dx, qr3, fx);
              fy = fmaf(dy, qr3, fy);
              fz = fmaf(dz, qr3, fz);
            } else if (KER == FMMB_LAPLACE_GNI) {
              const float qr3 = xj.w * rinv * rinv * rinv;
              p = fmaf(fmaf(dx, nv.x, fmaf(dy, nv.y, dz * nv.z)), qr3, p);
            } else {
              const float4 nj = sn[jj];
              const float qr3 = xj.w * rinv * rinv * rinv;
              p = fmaf(fmaf(dx, nj.x, fmaf(dy, nj.y, dz * nj.z)), qr3, p);
            }
          }
          P += (double)p;
          if (KER == FMMB_LAPLACE_G) {
            FX += (double)fx;
            FY += (double)fy;
            FZ += (double)fz;
          }
        }
      }
    }
    // combine the two halves
    __syncthreads();
    if (half) {
      red[0][t] = P;
      if (KER == FMMB_LAPLACE_G) {
        red[1][t] = FX;
        red[2][t] = FY;
        red[3][t] = FZ;
      }
    }
    __syncthreads();
    if (!half && act) {
      pot[i] = coef * (P + red[0][t]);
      if (KER == FMMB_LAPLACE_G && grad) {
        grad[i] = -coef * (FX + red[1][t]);
        grad[ni + i] = -coef * (FY + red[2][t]);
        grad[2 * ni + i] = -coef * (FZ + red[3][t]);
      }
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

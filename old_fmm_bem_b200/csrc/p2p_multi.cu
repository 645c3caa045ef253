// Near field for many right-hand sides at once (mixed form, Laplace kernels).
//
// The same sums as p2p_mixed.cu (kernel/G_p2p.cxx:12-37, Gni_p2p.cxx:12-28,
// Gnj_p2p.cxx:12-28) for R charge vectors in one pass: the pair geometry --
// distance, inverse distance, the kernel value -- is computed once per pair
// and applied to the R charges of the source, so a GMRES block of R iterates
// costs little more than one.  One block (128 threads, one target each) per
// work item of up to 128 targets of a leaf; the sources of the 27 neighbour
// slots are staged through shared memory in chunks of 128 with their R
// charges; FP32 pair terms, summed per chunk in FP32 and promoted to FP64.
// Zero-distance pairs are skipped (their inverse distance is taken as 0) when
// the plan excludes them.
#include <cuda_runtime.h>

#include "internal.h"
#include "kernels.h"

namespace fmmb {
namespace {

constexpr int kT = 128;

__device__ __forceinline__ float rsqrt_ftz(float x) {
  float y;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

template <int KER, int R>
__global__ void __launch_bounds__(kT) p2p_multi(const int2* __restrict__ work, const int2* __restrict__ leaf_i,
                                                const int2* __restrict__ leaf_j, const int* __restrict__ list,
                                                const float4* __restrict__ tpos, const float4* __restrict__ tnrm,
                                                const float4* __restrict__ spos, const float4* __restrict__ snrm,
                                                const float* __restrict__ qs, int nj, float eps2, int excl, double coef,
                                                double* __restrict__ pot, double* __restrict__ grad, int ni) {
  constexpr int NC = KER == FMMB_LAPLACE_G ? 4 : 1;  // accumulated components per right-hand side
  constexpr int RV = R % 4 == 0 ? R / 4 : 0;          // charges of a source as float4 vectors (R = 4, 8)
  __shared__ float4 sx[kT];
  __shared__ float4 sn[KER == FMMB_LAPLACE_GNJ ? kT : 1];
  __shared__ float4 sq4[RV > 0 ? kT : 1][RV > 0 ? RV : 1];
  __shared__ float sq[RV > 0 ? 1 : R][kT];
  const int2 wk = work[blockIdx.x];
  const int b = wk.x;
  const int2 li = leaf_i[b];
  const int it = wk.y + threadIdx.x;
  const bool on = it < li.y;
  const float4 xi = on ? tpos[li.x + it] : make_float4(0.f, 0.f, 0.f, 0.f);
  const float4 ni4 = (KER == FMMB_LAPLACE_GNI && on) ? tnrm[li.x + it] : make_float4(0.f, 0.f, 0.f, 0.f);
  double P[R][NC];
#pragma unroll
  for (int r = 0; r < R; r++)
#pragma unroll
    for (int c = 0; c < NC; c++) P[r][c] = 0.0;
  for (int sl = 0; sl < kP2PSlots; sl++) {
    const int jl = list[(size_t)b * kP2PSlots + sl];
    if (jl < 0) continue;
    const int2 lj = leaf_j[jl];
    for (int c0 = 0; c0 < lj.y; c0 += kT) {
      __syncthreads();
      if (c0 + (int)threadIdx.x < lj.y) {
        const int j = lj.x + c0 + threadIdx.x;
        sx[threadIdx.x] = spos[j];
        if (KER == FMMB_LAPLACE_GNJ) sn[threadIdx.x] = snrm[j];
        if (RV > 0) {
#pragma unroll
          for (int v = 0; v < (RV > 0 ? RV : 1); v++)
            sq4[threadIdx.x][v] = make_float4(qs[(size_t)(4 * v) * nj + j], qs[(size_t)(4 * v + 1) * nj + j],
                                              qs[(size_t)(4 * v + 2) * nj + j], qs[(size_t)(4 * v + 3) * nj + j]);
        } else {
#pragma unroll
          for (int r = 0; r < R; r++) sq[r][threadIdx.x] = qs[(size_t)r * nj + j];
        }
      }
      __syncthreads();
      if (!on) continue;
      const int nc = min(kT, lj.y - c0);
      float A[R][NC];
#pragma unroll
      for (int r = 0; r < R; r++)
#pragma unroll
        for (int c = 0; c < NC; c++) A[r][c] = 0.f;
      // Gni / Gnj with 4 or 8 right-hand sides: the sums of right-hand sides
      // 2h, 2h + 1 side by side for the two-lane FP32 FMA
      constexpr bool PK = KER != FMMB_LAPLACE_G && RV > 0;
      float2 A2[PK ? R / 2 : 1];
#pragma unroll
      for (int h = 0; h < (PK ? R / 2 : 1); h++) A2[h] = make_float2(0.f, 0.f);
#pragma unroll 2
      for (int jj = 0; jj < nc; jj++) {
        float qv[R];  // the source's charges, vector loads when R is a multiple of 4
        if (RV > 0) {
#pragma unroll
          for (int v = 0; v < (RV > 0 ? RV : 1); v++) {
            const float4 t4 = sq4[jj][v];
            qv[4 * v] = t4.x;
            qv[4 * v + 1] = t4.y;
            qv[4 * v + 2] = t4.z;
            qv[4 * v + 3] = t4.w;
          }
        } else {
#pragma unroll
          for (int r = 0; r < R; r++) qv[r] = sq[r][jj];
        }
        const float4 xj = sx[jj];
        const float dx = xi.x - xj.x, dy = xi.y - xj.y, dz = xi.z - xj.z;
        const float r2 = fmaf(dx, dx, fmaf(dy, dy, fmaf(dz, dz, eps2)));
        float rinv = rsqrt_ftz(r2);
        if (excl) rinv = r2 > 0.f ? rinv : 0.f;
        if (KER == FMMB_LAPLACE_G) {
          const float r3 = rinv * rinv * rinv;
#pragma unroll
          for (int r = 0; r < R; r++) {
            const float q = qv[r];
            const float qr3 = q * r3;
            A[r][0] = fmaf(q, rinv, A[r][0]);
            A[r][1] = fmaf(dx, qr3, A[r][1]);
            A[r][2] = fmaf(dy, qr3, A[r][2]);
            A[r][3] = fmaf(dz, qr3, A[r][3]);
          }
        } else {
          float kv;
          if (KER == FMMB_LAPLACE_GNI) {
            kv = fmaf(dx, ni4.x, fmaf(dy, ni4.y, dz * ni4.z)) * (rinv * rinv * rinv);
          } else {
            const float4 nj4 = sn[jj];
            kv = fmaf(dx, nj4.x, fmaf(dy, nj4.y, dz * nj4.z)) * (rinv * rinv * rinv);
          }
          if (PK) {
            const float2 kv2 = make_float2(kv, kv);
#pragma unroll
            for (int h = 0; h < (PK ? R / 2 : 1); h++)
              A2[h] = __ffma2_rn(make_float2(qv[2 * h], qv[2 * h + 1]), kv2, A2[h]);
          } else {
#pragma unroll
            for (int r = 0; r < R; r++) A[r][0] = fmaf(qv[r], kv, A[r][0]);
          }
        }
      }
      if (PK) {
#pragma unroll
        for (int h = 0; h < (PK ? R / 2 : 1); h++) {
          A[2 * h][0] = A2[h].x;
          A[2 * h + 1][0] = A2[h].y;
        }
      }
#pragma unroll
      for (int r = 0; r < R; r++)
#pragma unroll
        for (int c = 0; c < NC; c++) P[r][c] += (double)A[r][c];
    }
  }
  if (!on) return;
  const int i = li.x + it;
#pragma unroll
  for (int r = 0; r < R; r++) {
    pot[(size_t)r * ni + i] = coef * P[r][0];
    if (KER == FMMB_LAPLACE_G && grad) {
      double* g = grad + (size_t)r * 3 * ni;
      g[i] = -coef * P[r][1];
      g[ni + i] = -coef * P[r][2];
      g[2 * (size_t)ni + i] = -coef * P[r][3];
    }
  }
}

template <int KER, int R>
void launch_r(int nwork, const int2* work, const int2* leaf_i, const int2* leaf_j, const int* list, const float4* tpos,
              const float4* tnrm, const float4* spos, const float4* snrm, const float* qs, int nj, const Sem& s,
              double* pot, double* grad, int ni, cudaStream_t st) {
  p2p_multi<KER, R><<<nwork, kT, 0, st>>>(work, leaf_i, leaf_j, list, tpos, tnrm, spos, snrm, qs, nj, (float)s.eps2,
                                           s.excl_self, s.coef, pot, grad, ni);
}

template <int KER>
void launch_k(int nrhs, int nwork, const int2* work, const int2* leaf_i, const int2* leaf_j, const int* list,
              const float4* tpos, const float4* tnrm, const float4* spos, const float4* snrm, const float* qs, int nj,
              const Sem& s, double* pot, double* grad, int ni, cudaStream_t st) {
  // right-hand sides in groups of 8, 4, 2, 1
  for (int r0 = 0; r0 < nrhs;) {
    const int left = nrhs - r0;
    const float* q = qs + (size_t)r0 * nj;
    double* p = pot + (size_t)r0 * ni;
    double* g = grad ? grad + (size_t)r0 * 3 * ni : nullptr;
    if (left >= 8) {
      launch_r<KER, 8>(nwork, work, leaf_i, leaf_j, list, tpos, tnrm, spos, snrm, q, nj, s, p, g, ni, st);
      r0 += 8;
    } else if (left >= 4) {
      launch_r<KER, 4>(nwork, work, leaf_i, leaf_j, list, tpos, tnrm, spos, snrm, q, nj, s, p, g, ni, st);
      r0 += 4;
    } else if (left >= 2) {
      launch_r<KER, 2>(nwork, work, leaf_i, leaf_j, list, tpos, tnrm, spos, snrm, q, nj, s, p, g, ni, st);
      r0 += 2;
    } else {
      launch_r<KER, 1>(nwork, work, leaf_i, leaf_j, list, tpos, tnrm, spos, snrm, q, nj, s, p, g, ni, st);
      r0 += 1;
    }
    FMMB_CHECK_LAUNCH();
  }
}

}  // namespace

int launch_p2p_multi(int kernel, int nrhs, int nwork, const int2* work, const int2* leaf_i, const int2* leaf_j,
                     const int* list, const float4* tpos, const float4* tnrm, const float4* spos, const float4* snrm,
                     const float* qs, int nj, const Sem& s, double* pot, double* grad, int ni, cudaStream_t st) {
  if (nwork <= 0 || nrhs <= 0) return 0;
  if (kernel == FMMB_LAPLACE_G)
    launch_k<FMMB_LAPLACE_G>(nrhs, nwork, work, leaf_i, leaf_j, list, tpos, tnrm, spos, snrm, qs, nj, s, pot, grad,
                             ni, st);
  else if (kernel == FMMB_LAPLACE_GNI)
    launch_k<FMMB_LAPLACE_GNI>(nrhs, nwork, work, leaf_i, leaf_j, list, tpos, tnrm, spos, snrm, qs, nj, s, pot,
                               nullptr, ni, st);
  else
    launch_k<FMMB_LAPLACE_GNJ>(nrhs, nwork, work, leaf_i, leaf_j, list, tpos, tnrm, spos, snrm, qs, nj, s, pot,
                               nullptr, ni, st);
  return nrhs / 8 + ((nrhs % 8) >= 4) + ((nrhs % 4) >= 2) + (nrhs % 2);  // launches
}

}  // namespace fmmb

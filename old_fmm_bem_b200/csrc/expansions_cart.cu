// P2M and L2P from Cartesian solid-harmonic recurrences (accurate semantics).
//
// The reference evaluates r^n fac(n,m) P_n^m(cos a) e^{-i m b} through
// spherical angles (acos, atan, exp; kernel/multipole.cxx:7-35,
// kernel/G_p2m.cxx:28-55) and the local-expansion gradient through spherical
// derivatives with a 1/sin(theta) (kernel/G_l2p.cxx:44-70).  In exact
// arithmetic the same quantities follow from the homogeneous polynomials
//   S_n^m(x) = r^n P_n^m(cos theta) e^{i m phi}   (Condon-Shortley phase)
// without any trigonometric function:
//   S_m^m = -(2m-1) (x + i y) S_{m-1}^{m-1},   S_{m+1}^m = (2m+1) z S_m^m,
//   (n-m) S_n^m = (2n-1) z S_{n-1}^m - (n+m-1) r^2 S_{n-2}^m,
// with the ladder identities
//   d/dz S_n^m = (n+m) S_{n-1}^m,  (d/dx + i d/dy) S_n^m = S_{n-1}^{m+1},
//   (d/dx - i d/dy) S_n^m = -(n+m)(n+m-1) S_{n-1}^{m-1},
//   S_{n}^{-1} = -conj(S_n^1) / (n (n+1)).
// Multipole basis: fac(n,m) conj(S_n^m); local evaluation: Re sum w_m
// fac(n,m) L_n^m S_n^m with w_0 = 1, w_m = 2.  This form has no singular
// points (a target on a box axis or at a box centre is fine), so it is used
// for accurate semantics; reference semantics keep the spherical kernels
// of kernels_fp64.cu, which reproduce the reference's eps-shifted radius and
// single-precision angles.
#include <cuda_runtime.h>

#include <cmath>

#include "internal.h"
#include "kernels.h"

namespace fmmb {
namespace {

struct cplx {
  double re, im;
};

// 1/k for the Legendre-type recurrences (k = n - m <= 40): avoids FP64 divides
__constant__ double c_inv[41] = {0.0,      1.0 / 1,  1.0 / 2,  1.0 / 3,  1.0 / 4,  1.0 / 5,  1.0 / 6,  1.0 / 7,
                                 1.0 / 8,  1.0 / 9,  1.0 / 10, 1.0 / 11, 1.0 / 12, 1.0 / 13, 1.0 / 14, 1.0 / 15,
                                 1.0 / 16, 1.0 / 17, 1.0 / 18, 1.0 / 19, 1.0 / 20, 1.0 / 21, 1.0 / 22, 1.0 / 23,
                                 1.0 / 24, 1.0 / 25, 1.0 / 26, 1.0 / 27, 1.0 / 28, 1.0 / 29, 1.0 / 30, 1.0 / 31,
                                 1.0 / 32, 1.0 / 33, 1.0 / 34, 1.0 / 35, 1.0 / 36, 1.0 / 37, 1.0 / 38, 1.0 / 39,
                                 1.0 / 40};
__device__ __forceinline__ cplx cmul(cplx a, cplx b) { return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
__device__ __forceinline__ cplx cscale(cplx a, double s) { return {a.re * s, a.im * s}; }

__device__ __forceinline__ void box_center(int key, float xmin, float ymin, float zmin, double rb, double& xc, double& yc,
                                           double& zc) {
  int cx = 0, cy = 0, cz = 0;
  for (int i = 0; i < 10; i++) {
    cy |= ((key >> (3 * i)) & 1) << i;
    cx |= ((key >> (3 * i + 1)) & 1) << i;
    cz |= ((key >> (3 * i + 2)) & 1) << i;
  }
  xc = (double)xmin + (cx + 0.5) * rb;
  yc = (double)ymin + (cy + 0.5) * rb;
  zc = (double)zmin + (cz + 0.5) * rb;
}

// ------------------------------------------------------------------ P2M
// One block (128 threads) per source leaf.  Lanes are grouped in segments of
// SEG; lane m of a segment owns order m (column m of S) of one point, so a
// block processes 128/SEG points at a time.  The dipole needs the neighbouring
// columns m-1 and m+1 of the previous degree, which come from the adjacent
// lanes by shuffles.  Each segment accumulates into its own shared-memory
// copy of the multipole; the copies are summed at the end.
template <int KER, int SEG>
__global__ void __launch_bounds__(128) p2m_cart(int p, int K, const int* __restrict__ keys, const int2* __restrict__ leaf,
                                                const float4* __restrict__ spos, const float4* __restrict__ snrm,
                                                const float* __restrict__ qs, const double* __restrict__ fac, float xmin,
                                                float ymin, float zmin, double rb, double* __restrict__ M) {
  constexpr int G = 128 / SEG;
  extern __shared__ double acc[];  // [G][K]
  const int g = threadIdx.x / SEG, m = threadIdx.x % SEG;
  for (int k = threadIdx.x; k < G * K; k += blockDim.x) acc[k] = 0.0;
  __syncthreads();
  const int b = blockIdx.x;
  double xc, yc, zc;
  box_center(keys[b], xmin, ymin, zmin, rb, xc, yc, zc);
  const int2 lf = leaf[b];
  double* my = acc + g * K;
  const double inv_rb = 1.0 / rb;
  const unsigned segmask = 0xffffffffu;  // every lane of the warp runs the same loop trip counts
  const int rounds = (lf.y + G - 1) / G;
  for (int it = 0; it < rounds; it++) {
    const int jj = it * G + g;
    const bool act = jj < lf.y;
    const int j = lf.x + (act ? jj : 0);
    const float4 xs = spos[j];
    const double q = act ? (double)qs[j] : 0.0;
    const double x = ((double)xs.x - xc) * inv_rb, y = ((double)xs.y - yc) * inv_rb, z = ((double)xs.z - zc) * inv_rb;
    const double r2 = x * x + y * y + z * z;
    // S_m^m = prod_{k<m} -(2k+1) (x + i y)
    cplx smm = {1.0, 0.0};
    for (int k = 0; k < m; k++) smm = cscale(cmul(smm, cplx{x, y}), -(2.0 * k + 1.0));
    cplx s1 = {0.0, 0.0}, s2 = {0.0, 0.0};  // S_{n-1}^m, S_{n-2}^m
    double qnx = 0, qny = 0, qnz = 0;
    if (KER == FMMB_LAPLACE_GNJ) {
      const float4 nv = snrm[j];
      const float qf = act ? qs[j] : 0.f;
      qnx = (double)(qf * nv.x) * inv_rb;
      qny = (double)(qf * nv.y) * inv_rb;
      qnz = (double)(qf * nv.z) * inv_rb;
    }
    for (int n = 0; n <= p; n++) {
      cplx sn;
      if (n < m) sn = {0.0, 0.0};
      else if (n == m) sn = smm;
      else if (n == m + 1) sn = cscale(s1, (2.0 * m + 1.0) * z);
      else {
        const double inv = c_inv[n - m];
        const double a = (2.0 * n - 1.0) * z * inv, c = (n + m - 1.0) * r2 * inv;
        sn = {a * s1.re - c * s2.re, a * s1.im - c * s2.im};
      }
      if (KER != FMMB_LAPLACE_GNJ) {
        if (n >= m && m <= p) {
          const double f = q * fac[ifull_d(n, m)];
          if (m == 0) my[n * n] += f * sn.re;
          else {
            my[n * n + 2 * m - 1] += f * sn.re;
            my[n * n + 2 * m] -= f * sn.im;
          }
        }
      } else {
        // n . grad S_n^m from degree n-1 (s1): columns m+1 (lane above) and
        // m-1 (lane below; for m = 0 the conjugate of column 1)
        cplx up, dn;
        up.re = __shfl_down_sync(segmask, s1.re, 1, SEG);
        up.im = __shfl_down_sync(segmask, s1.im, 1, SEG);
        dn.re = __shfl_up_sync(segmask, s1.re, 1, SEG);
        dn.im = __shfl_up_sync(segmask, s1.im, 1, SEG);
        if (m == SEG - 1) up = {0.0, 0.0};
        double cm;
        if (m == 0) {
          dn = {up.re, -up.im};
          cm = 1.0;
        } else {
          cm = -(double)(n + m) * (double)(n + m - 1);
        }
        if (n >= 1 && n >= m && m <= p) {
          // D = 1/2 (nx - i ny) up + 1/2 (nx + i ny) cm dn + nz (n+m) s1
          const cplx a = cmul(cplx{0.5 * qnx, -0.5 * qny}, up);
          const cplx c = cmul(cplx{0.5 * qnx * cm, 0.5 * qny * cm}, dn);
          const double d = qnz * (n + m);
          const double Dre = a.re + c.re + d * s1.re, Dim = a.im + c.im + d * s1.im;
          const double f = fac[ifull_d(n, m)];
          if (m == 0) my[n * n] += f * Dre;
          else {
            my[n * n + 2 * m - 1] += f * Dre;
            my[n * n + 2 * m] -= f * Dim;
          }
        }
      }
      s2 = s1;
      s1 = sn;
    }
  }
  __syncthreads();
  for (int k = threadIdx.x; k < K; k += blockDim.x) {
    double t = 0.0;
#pragma unroll
    for (int gg = 0; gg < G; gg++) t += acc[gg * K + k];
    M[(size_t)b * K + k] = t;
  }
}

// ------------------------------------------------------------------ P2M (FP32)
// Mixed-precision P2M: one thread per source point evaluates every S_n^m of
// its point in FP32 with the degree rows held in registers (order P fixed at
// compile time, runtime order p <= P), writes its contributions to shared
// memory, and the block reduces the columns in FP64.  The multipole of a leaf
// carries FP32 rounding of each point's terms (relative 1e-7) -- below the
// tensor-core error of the translations that consume it.  A block is one work
// item of up to kP2MItem sources of a leaf, so that the dense leaves of
// clustered points (a thousand points and more) spread over many SMs; a leaf
// of several items is summed with FP64 atomics into zeroed rows.
__constant__ float c_fac32[21 * 21 + 21];  // fac(n, m) at n*n+n+m, n <= 20

constexpr int kP2MThreads = kP2MItem;

template <int KER, int P>
__global__ void __launch_bounds__(kP2MThreads) p2m_f32(int p, int K, const int2* __restrict__ work,
                                                       const int* __restrict__ keys,
                                                       const int2* __restrict__ leaf, const float4* __restrict__ spos,
                                                       const float4* __restrict__ snrm, const float* __restrict__ qs,
                                                       float xmin, float ymin, float zmin, double rb,
                                                       double* __restrict__ M) {
  extern __shared__ float contrib[];  // [kP2MThreads][K]
  const int2 wk = work[blockIdx.x];
  const int b = wk.x;
  double xc, yc, zc;
  box_center(keys[b], xmin, ymin, zmin, rb, xc, yc, zc);
  const int2 leaf_b = leaf[b];
  const bool shared_leaf = leaf_b.y > kP2MThreads;  // summed by several items
  const int2 lf = make_int2(leaf_b.x + wk.y, min(kP2MThreads, leaf_b.y - wk.y));
  const double inv_rb = 1.0 / rb;
  double acc0 = 0.0, acc1 = 0.0;  // columns threadIdx.x and threadIdx.x + 64 (K <= 128 per pass)
  double acc[(P + 1) * (P + 1) / kP2MThreads + 1];
#pragma unroll
  for (int i = 0; i < (P + 1) * (P + 1) / kP2MThreads + 1; i++) acc[i] = 0.0;
  (void)acc0;
  (void)acc1;
  float* my = contrib + threadIdx.x * K;
  for (int j0 = 0; j0 < lf.y; j0 += kP2MThreads) {
    const int jj = j0 + threadIdx.x;
    const bool act = jj < lf.y;
    const int j = lf.x + (act ? jj : 0);
    const float4 xs = spos[j];
    const float q = act ? qs[j] : 0.f;
    const float x = (float)(((double)xs.x - xc) * inv_rb), y = (float)(((double)xs.y - yc) * inv_rb),
                z = (float)(((double)xs.z - zc) * inv_rb);
    const float r2 = x * x + y * y + z * z;
    float qnx = 0.f, qny = 0.f, qnz = 0.f;
    if (KER == FMMB_LAPLACE_GNJ) {
      const float4 nv = snrm[j];
      const float s = q * (float)inv_rb;
      qnx = s * nv.x;
      qny = s * nv.y;
      qnz = s * nv.z;
    }
    float r1re[P + 1], r1im[P + 1], r2re[P + 1], r2im[P + 1];
#pragma unroll
    for (int m = 0; m <= P; m++) r1re[m] = r1im[m] = r2re[m] = r2im[m] = 0.f;
#pragma unroll
    for (int n = 0; n <= P; n++) {
      float cre[P + 1], cim[P + 1];
#pragma unroll
      for (int m = 0; m <= P; m++) {
        cre[m] = cim[m] = 0.f;
        if (m > n) continue;
        if (n == 0) {
          cre[0] = 1.f;
        } else if (m == n) {  // S_n^n = -(2n-1) (x + i y) S_{n-1}^{n-1}
          const float a = -(2.f * n - 1.f);
          cre[m] = a * (x * r1re[n - 1] - y * r1im[n - 1]);
          cim[m] = a * (x * r1im[n - 1] + y * r1re[n - 1]);
        } else if (m == n - 1) {
          const float a = (2.f * n - 1.f) * z;
          cre[m] = a * r1re[m];
          cim[m] = a * r1im[m];
        } else {
          const float inv = 1.f / (float)(n - m);
          const float a = (2.f * n - 1.f) * z * inv, c = (float)(n + m - 1) * r2 * inv;
          cre[m] = a * r1re[m] - c * r2re[m];
          cim[m] = a * r1im[m] - c * r2im[m];
        }
        if (n > p) continue;
        float vre, vim;
        if (KER != FMMB_LAPLACE_GNJ) {
          const float f = q * c_fac32[n * n + n + m];
          vre = f * cre[m];
          vim = -f * cim[m];
        } else {
          if (n == 0) {
            vre = vim = 0.f;
          } else {
            // n . grad S_n^m from degree n-1
            const float upr = (m + 1 <= n - 1) ? r1re[m + 1 <= P ? m + 1 : P] : 0.f;
            const float upi = (m + 1 <= n - 1) ? r1im[m + 1 <= P ? m + 1 : P] : 0.f;
            float dnr, dni, cm;
            if (m == 0) {  // conj(S_{n-1}^1)
              dnr = (n - 1 >= 1) ? r1re[1 <= P ? 1 : P] : 0.f;
              dni = (n - 1 >= 1) ? -r1im[1 <= P ? 1 : P] : 0.f;
              cm = 1.f;
            } else {
              dnr = r1re[m - 1 >= 0 ? m - 1 : 0];
              dni = r1im[m - 1 >= 0 ? m - 1 : 0];
              cm = -(float)(n + m) * (float)(n + m - 1);
            }
            const float s1r = (m <= n - 1) ? r1re[m] : 0.f, s1i = (m <= n - 1) ? r1im[m] : 0.f;
            // D = 1/2 (nx - i ny) up + 1/2 cm (nx + i ny) dn + nz (n+m) s1
            const float Dre = 0.5f * (qnx * upr + qny * upi) + 0.5f * cm * (qnx * dnr - qny * dni) + qnz * (n + m) * s1r;
            const float Dim = 0.5f * (qnx * upi - qny * upr) + 0.5f * cm * (qnx * dni + qny * dnr) + qnz * (n + m) * s1i;
            const float f = c_fac32[n * n + n + m];
            vre = f * Dre;
            vim = -f * Dim;
          }
        }
        if (m == 0) my[n * n] = vre;
        else {
          my[n * n + 2 * m - 1] = vre;
          my[n * n + 2 * m] = vim;
        }
      }
#pragma unroll
      for (int m = 0; m <= P; m++) {
        r2re[m] = r1re[m];
        r2im[m] = r1im[m];
        r1re[m] = cre[m];
        r1im[m] = cim[m];
      }
    }
    __syncthreads();
    // column sums over the chunk's points (inactive points contributed zeros)
#pragma unroll
    for (int i = 0; i < (P + 1) * (P + 1) / kP2MThreads + 1; i++) {
      const int k = threadIdx.x + i * kP2MThreads;
      if (k < K) {
        float t = 0.f;
        const int npt = min(kP2MThreads, lf.y - j0);
        for (int pt = 0; pt < npt; pt++) t += contrib[pt * K + k];
        acc[i] += (double)t;
      }
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < (P + 1) * (P + 1) / kP2MThreads + 1; i++) {
    const int k = threadIdx.x + i * kP2MThreads;
    if (k < K) {
      if (shared_leaf) atomicAdd(M + (size_t)b * K + k, acc[i]);
      else M[(size_t)b * K + k] = acc[i];
    }
  }
}

// ------------------------------------------------------------------ L2P
// One block (64 threads) per target leaf.  The leaf's local expansion is
// turned once into the coefficients of the potential and of the three
// derivative expansions (ladder identities above), then each thread walks
// the S_n^m of its point column by column.
constexpr int kL2PThreads = 64;

template <int KER>
__global__ void __launch_bounds__(kL2PThreads) l2p_cart(int p, int K, const int* __restrict__ keys,
                                                        const int2* __restrict__ leaf, const float4* __restrict__ tpos,
                                                        const float4* __restrict__ tnrm, const double* __restrict__ fac,
                                                        float xmin, float ymin, float zmin, double rb, double coef,
                                                        const double* __restrict__ L, double* __restrict__ pot,
                                                        double* __restrict__ grad, int ni) {
  extern __shared__ double sm[];
  const int P = (p + 1) * (p + 2) / 2;
  cplx* Cphi = reinterpret_cast<cplx*>(sm);
  cplx* Cz = Cphi + P;
  cplx* Cp = Cz + P;
  cplx* Cm = Cp + P;
  double* Cs = reinterpret_cast<double*>(Cm + P);  // [p+1]
  const int b = blockIdx.x;
  const double* Lb = L + (size_t)b * K;
  auto Lnm = [&](int n, int m) -> cplx {
    if (m == 0) return {Lb[n * n], 0.0};
    return {Lb[n * n + 2 * m - 1], Lb[n * n + 2 * m]};
  };
  for (int idx = threadIdx.x; idx < P; idx += blockDim.x) {
    int n = 0;
    while ((n + 1) * (n + 2) / 2 <= idx) n++;
    const int m = idx - n * (n + 1) / 2;
    const double wm = m ? 2.0 : 1.0;
    Cphi[idx] = cscale(Lnm(n, m), wm * fac[ifull_d(n, m)]);
    if (n < p) {
      Cz[idx] = cscale(Lnm(n + 1, m), wm * fac[ifull_d(n + 1, m)] * (n + 1 + m));
      Cp[idx] = (m >= 1) ? cscale(Lnm(n + 1, m - 1), (m - 1 ? 2.0 : 1.0) * fac[ifull_d(n + 1, m - 1)]) : cplx{0.0, 0.0};
      Cm[idx] = cscale(Lnm(n + 1, m + 1), -2.0 * fac[ifull_d(n + 1, m + 1)] * (double)(n + m + 2) * (double)(n + m + 1));
    } else {
      Cz[idx] = Cp[idx] = Cm[idx] = cplx{0.0, 0.0};
    }
  }
  for (int n = threadIdx.x; n <= p; n += blockDim.x) Cs[n] = (n < p) ? fac[ifull_d(n + 1, 0)] * Lb[(n + 1) * (n + 1)] : 0.0;
  __syncthreads();
  double xc, yc, zc;
  box_center(keys[b], xmin, ymin, zmin, rb, xc, yc, zc);
  const int2 lf = leaf[b];
  const double inv_rb = 1.0 / rb;
  for (int ii = threadIdx.x; ii < lf.y; ii += blockDim.x) {
    const int i = lf.x + ii;
    const float4 xt = tpos[i];
    const double x = ((double)xt.x - xc) * inv_rb, y = ((double)xt.y - yc) * inv_rb, z = ((double)xt.z - zc) * inv_rb;
    const double r2 = x * x + y * y + z * z;
    double F = 0, dzr = 0, dpr = 0, dpi = 0, dmr = 0, dmi = 0;
    cplx smm = {1.0, 0.0};
    for (int m = 0; m <= p; m++) {
      if (m > 0) smm = cscale(cmul(smm, cplx{x, y}), -(2.0 * m - 1.0));
      cplx s1 = {0.0, 0.0}, s2 = {0.0, 0.0};
      for (int n = m; n <= p; n++) {
        cplx sn;
        if (n == m) sn = smm;
        else if (n == m + 1) sn = cscale(s1, (2.0 * m + 1.0) * z);
        else {
          const double inv = c_inv[n - m];
        const double a = (2.0 * n - 1.0) * z * inv, c = (n + m - 1.0) * r2 * inv;
          sn = {a * s1.re - c * s2.re, a * s1.im - c * s2.im};
        }
        const int idx = n * (n + 1) / 2 + m;
        const cplx cf = Cphi[idx];
        F += cf.re * sn.re - cf.im * sn.im;  // Re(C S)
        if (n < p) {
          const cplx cz = Cz[idx], cp = Cp[idx], cmm = Cm[idx];
          dzr += cz.re * sn.re - cz.im * sn.im;
          dpr += cp.re * sn.re - cp.im * sn.im;
          dpi += cp.re * sn.im + cp.im * sn.re;
          dmr += cmm.re * sn.re - cmm.im * sn.im;
          dmi += cmm.re * sn.im + cmm.im * sn.re;
          if (m == 1) {  // Cs[n] * conj(S_n^1)
            dmr += Cs[n] * sn.re;
            dmi -= Cs[n] * sn.im;
          }
        }
        s2 = s1;
        s1 = sn;
      }
    }
    const double gx = 0.5 * (dpr + dmr), gy = 0.5 * (dpi - dmi), gz = dzr;
    const double c1 = coef * inv_rb, c2 = coef * inv_rb * inv_rb;
    if (KER == FMMB_LAPLACE_GNI) {
      const float4 nv = tnrm[i];
      pot[i] = -c2 * ((double)nv.x * gx + (double)nv.y * gy + (double)nv.z * gz);
    } else {
      pot[i] = c1 * F;
      if (grad) {  // G and Gnj: the local expansion is the potential itself
        grad[i] = c2 * gx;
        grad[ni + i] = c2 * gy;
        grad[2 * ni + i] = c2 * gz;
      }
    }
  }
}

// ------------------------------------------------------------------ L2P, Hessian
// The gradient w.r.t. the target position of the far-field Gni potential
// -(1/4pi) n . grad(phi) (normal held fixed): -(1/4pi) H n, H the Hessian of
// the local expansion.  One block (64 threads) per target leaf.  With F the
// real potential of L in scaled coordinates written over all orders,
// F = sum_{n, |m| <= n} b_n^m S_n^m (b_n^m = fac(n,m) L_n^m for m >= 0,
// b_n^{-m} = (-1)^m (n+m)!/(n-m)! conj(b_n^m)), the ladder identities give its
// derivatives as expansions of one degree less:
//   d/dx F: c_{n-1}^k = (b_n^{k-1} - (n+k+1)(n+k) b_n^{k+1}) / 2
//   d/dy F: c_{n-1}^k = (b_n^{k-1} + (n+k+1)(n+k) b_n^{k+1}) / (2i)
//   d/dz F: c_{n-1}^k = (n+k) b_n^k
// i.e. local expansions L^D = c / fac of the same form (real potentials); the
// gradient of each, evaluated like l2p_cart's, is one row of H.
constexpr int kL2PHThreads = 64;

__global__ void __launch_bounds__(kL2PHThreads) l2p_hess_gni(int p, int K, const int* __restrict__ keys,
                                                             const int2* __restrict__ leaf,
                                                             const float4* __restrict__ tpos,
                                                             const float4* __restrict__ tnrm,
                                                             const double* __restrict__ fac, float xmin, float ymin,
                                                             float zmin, double rb, double coef,
                                                             const double* __restrict__ L, double* __restrict__ grad,
                                                             int ni) {
  extern __shared__ double sm[];
  const int P = (p + 1) * (p + 2) / 2;
  cplx* Ld = reinterpret_cast<cplx*>(sm);  // [3][P] derivative expansions (m >= 0)
  cplx* Cz = Ld + 3 * P;                   // [3][P] their gradient coefficient sets
  cplx* Cp = Cz + 3 * P;
  cplx* Cm = Cp + 3 * P;
  double* Cs = reinterpret_cast<double*>(Cm + 3 * P);  // [3][p+1]
  const int b = blockIdx.x;
  const double* Lb = L + (size_t)b * K;
  auto bnm = [&](int n, int m) -> cplx {  // b_n^m for -1 <= m
    if (n < 0 || m > n || n > p) return {0.0, 0.0};
    if (m == -1) {
      if (n < 1) return {0.0, 0.0};
      const double f = fac[ifull_d(n, 1)];
      return {-(double)n * (n + 1) * f * Lb[n * n + 1], (double)n * (n + 1) * f * Lb[n * n + 2]};
    }
    if (m == 0) return {fac[ifull_d(n, 0)] * Lb[n * n], 0.0};
    const double f = fac[ifull_d(n, m)];
    return {f * Lb[n * n + 2 * m - 1], f * Lb[n * n + 2 * m]};
  };
  for (int idx = threadIdx.x; idx < P; idx += blockDim.x) {
    int n1 = 0;
    while ((n1 + 1) * (n1 + 2) / 2 <= idx) n1++;
    const int k = idx - n1 * (n1 + 1) / 2;  // degree n1 = n - 1, order k
    cplx cx = {0.0, 0.0}, cy = {0.0, 0.0}, cz = {0.0, 0.0};
    if (n1 < p) {
      const int n = n1 + 1;
      const cplx lo = bnm(n, k - 1), hi = bnm(n, k + 1), mid = bnm(n, k);
      const double a = (double)(n + k + 1) * (double)(n + k);
      cx = {0.5 * (lo.re - a * hi.re), 0.5 * (lo.im - a * hi.im)};
      const cplx t = {lo.re + a * hi.re, lo.im + a * hi.im};
      cy = {0.5 * t.im, -0.5 * t.re};  // t / (2i)
      cz = {(n + k) * mid.re, (n + k) * mid.im};
    }
    const double inv = 1.0 / fac[ifull_d(n1, k)];
    Ld[idx] = cscale(cx, inv);
    Ld[P + idx] = cscale(cy, inv);
    Ld[2 * P + idx] = cscale(cz, inv);
    if (k == 0) {  // real by construction; drop the rounding residue
      Ld[idx].im = Ld[P + idx].im = Ld[2 * P + idx].im = 0.0;
    }
  }
  __syncthreads();
  // gradient coefficient sets of each derivative expansion (as l2p_cart's of L)
  for (int e = threadIdx.x; e < 3 * P; e += blockDim.x) {
    const int d = e / P, idx = e % P;
    const cplx* Lx = Ld + d * P;
    auto Lnm = [&](int n, int m) -> cplx { return Lx[n * (n + 1) / 2 + m]; };
    int n = 0;
    while ((n + 1) * (n + 2) / 2 <= idx) n++;
    const int m = idx - n * (n + 1) / 2;
    const double wm = m ? 2.0 : 1.0;
    if (n < p) {
      Cz[e] = cscale(Lnm(n + 1, m), wm * fac[ifull_d(n + 1, m)] * (n + 1 + m));
      Cp[e] = (m >= 1) ? cscale(Lnm(n + 1, m - 1), (m - 1 ? 2.0 : 1.0) * fac[ifull_d(n + 1, m - 1)]) : cplx{0.0, 0.0};
      Cm[e] = (m + 1 <= n + 1) ? cscale(Lnm(n + 1, m + 1), -2.0 * fac[ifull_d(n + 1, m + 1)] * (double)(n + m + 2) *
                                                                (double)(n + m + 1))
                               : cplx{0.0, 0.0};
    } else {
      Cz[e] = Cp[e] = Cm[e] = cplx{0.0, 0.0};
    }
  }
  for (int e = threadIdx.x; e < 3 * (p + 1); e += blockDim.x) {
    const int d = e / (p + 1), n = e % (p + 1);
    Cs[e] = (n < p) ? fac[ifull_d(n + 1, 0)] * Ld[d * P + (n + 1) * (n + 2) / 2].re : 0.0;
  }
  __syncthreads();
  double xc, yc, zc;
  box_center(keys[b], xmin, ymin, zmin, rb, xc, yc, zc);
  const int2 lf = leaf[b];
  const double inv_rb = 1.0 / rb;
  for (int ii = threadIdx.x; ii < lf.y; ii += blockDim.x) {
    const int i = lf.x + ii;
    const float4 xt = tpos[i];
    const double x = ((double)xt.x - xc) * inv_rb, y = ((double)xt.y - yc) * inv_rb, z = ((double)xt.z - zc) * inv_rb;
    const double r2 = x * x + y * y + z * z;
    double dzr[3] = {0, 0, 0}, dpr[3] = {0, 0, 0}, dpi[3] = {0, 0, 0}, dmr[3] = {0, 0, 0}, dmi[3] = {0, 0, 0};
    cplx smm = {1.0, 0.0};
    for (int m = 0; m <= p; m++) {
      if (m > 0) smm = cscale(cmul(smm, cplx{x, y}), -(2.0 * m - 1.0));
      cplx s1 = {0.0, 0.0}, s2 = {0.0, 0.0};
      for (int n = m; n < p; n++) {  // the derivative expansions stop at degree p - 1
        cplx sn;
        if (n == m) sn = smm;
        else if (n == m + 1) sn = cscale(s1, (2.0 * m + 1.0) * z);
        else {
          const double inv = c_inv[n - m];
          const double a = (2.0 * n - 1.0) * z * inv, c = (n + m - 1.0) * r2 * inv;
          sn = {a * s1.re - c * s2.re, a * s1.im - c * s2.im};
        }
        const int idx = n * (n + 1) / 2 + m;
#pragma unroll
        for (int d = 0; d < 3; d++) {
          const cplx cz = Cz[d * P + idx], cp = Cp[d * P + idx], cmm = Cm[d * P + idx];
          dzr[d] += cz.re * sn.re - cz.im * sn.im;
          dpr[d] += cp.re * sn.re - cp.im * sn.im;
          dpi[d] += cp.re * sn.im + cp.im * sn.re;
          dmr[d] += cmm.re * sn.re - cmm.im * sn.im;
          dmi[d] += cmm.re * sn.im + cmm.im * sn.re;
          if (m == 1) {
            dmr[d] += Cs[d * (p + 1) + n] * sn.re;
            dmi[d] -= Cs[d * (p + 1) + n] * sn.im;
          }
        }
        s2 = s1;
        s1 = sn;
      }
    }
    const float4 nv = tnrm[i];
    const double nn[3] = {(double)nv.x, (double)nv.y, (double)nv.z};
    double hn[3] = {0, 0, 0};  // H n in scaled coordinates (H symmetric: row d of H is grad(d/dd F))
#pragma unroll
    for (int d = 0; d < 3; d++) {
      hn[0] += nn[d] * 0.5 * (dpr[d] + dmr[d]);
      hn[1] += nn[d] * 0.5 * (dpi[d] - dmi[d]);
      hn[2] += nn[d] * dzr[d];
    }
    const double c3 = -coef * inv_rb * inv_rb * inv_rb;
    grad[i] = c3 * hn[0];
    grad[ni + i] = c3 * hn[1];
    grad[2 * ni + i] = c3 * hn[2];
  }
}

// FP32 L2P for the mixed form: the same coefficient arrays as l2p_cart
// (computed in FP64, stored as FP32 pairs), the solid harmonics S_n^m of a
// point by the P2M recurrence in FP32 registers (fully unrolled to order P),
// each degree's partial sums in FP32 and promoted to FP64 accumulators.
constexpr int kL2PF32Threads = 128;  // one work item of up to 128 targets per block

// Shared-memory coefficient reads.  A thread evaluates one point (a block is
// one work item of up to 128 targets), so the compiler is free to schedule
// these loads ahead of their use in the unrolled degree / order loops.
__device__ __forceinline__ float2 lds2(const float2* p) { return *p; }
__device__ __forceinline__ float lds1(const float* p) { return *p; }

template <int KER, int P>
__global__ void __launch_bounds__(kL2PF32Threads) l2p_f32(int p, int K, const int2* __restrict__ work,
                                                          const int* __restrict__ keys,
                                                          const int2* __restrict__ leaf, const float4* __restrict__ tpos,
                                                          const float4* __restrict__ tnrm, const double* __restrict__ fac,
                                                          float xmin, float ymin, float zmin, double rb, double coef,
                                                          const double* __restrict__ L, double* __restrict__ pot,
                                                          double* __restrict__ grad, int ni) {
  constexpr int NT = (P + 1) * (P + 2) / 2;
  constexpr bool DER = KER != FMMB_LAPLACE_GNJ;  // derivative sums needed
  __shared__ float2 Cphi[NT], Cz[DER ? NT : 1], Cp[DER ? NT : 1], Cm[DER ? NT : 1];
  __shared__ float Cs[P + 1];
  // the derivative sums in pairs for the two-lane FP32 FMAs: (fn, zn) from
  // CA = (Cphi.re, Cz.re, -Cphi.im, -Cz.im), (pr, mr) and (pi, mi) from
  // CB = (Cp.re, Cm.re, -Cp.im, -Cm.im) and CC = (Cp.im, Cm.im); the same
  // per-lane operations, in the same order, as the scalar sums
  __shared__ float4 CA[DER ? NT : 1], CB[DER ? NT : 1];
  __shared__ float2 CC[DER ? NT : 1];
  const int2 wk = work[blockIdx.x];
  const int b = wk.x;
  const double* Lb = L + (size_t)b * K;
  auto Lnm = [&](int n, int m) -> cplx {
    if (m == 0) return {Lb[n * n], 0.0};
    return {Lb[n * n + 2 * m - 1], Lb[n * n + 2 * m]};
  };
  auto f2 = [](cplx c) { return make_float2((float)c.re, (float)c.im); };
  for (int idx = threadIdx.x; idx < NT; idx += blockDim.x) {
    int n = 0;
    while ((n + 1) * (n + 2) / 2 <= idx) n++;
    const int m = idx - n * (n + 1) / 2;
    const double wm = m ? 2.0 : 1.0;
    Cphi[idx] = n <= p ? f2(cscale(Lnm(n, m), wm * fac[ifull_d(n, m)])) : make_float2(0.f, 0.f);
    if (DER) {
      if (n < p) {
        Cz[idx] = f2(cscale(Lnm(n + 1, m), wm * fac[ifull_d(n + 1, m)] * (n + 1 + m)));
        Cp[idx] = (m >= 1) ? f2(cscale(Lnm(n + 1, m - 1), (m - 1 ? 2.0 : 1.0) * fac[ifull_d(n + 1, m - 1)]))
                           : make_float2(0.f, 0.f);
        Cm[idx] = f2(cscale(Lnm(n + 1, m + 1), -2.0 * fac[ifull_d(n + 1, m + 1)] * (double)(n + m + 2) * (double)(n + m + 1)));
      } else {
        Cz[idx] = Cp[idx] = Cm[idx] = make_float2(0.f, 0.f);
      }
    }
  }
  for (int n = threadIdx.x; n <= P; n += blockDim.x) Cs[n] = (n < p) ? (float)(fac[ifull_d(n + 1, 0)] * Lb[(n + 1) * (n + 1)]) : 0.f;
  if (DER) {
    __syncthreads();
    for (int idx = threadIdx.x; idx < NT; idx += blockDim.x) {
      const float2 f = Cphi[idx], zz = Cz[idx], pp = Cp[idx], mm = Cm[idx];
      CA[idx] = make_float4(f.x, zz.x, -f.y, -zz.y);
      CB[idx] = make_float4(pp.x, mm.x, -pp.y, -mm.y);
      CC[idx] = make_float2(pp.y, mm.y);
    }
  }
  __syncthreads();
  double xc, yc, zc;
  box_center(keys[b], xmin, ymin, zmin, rb, xc, yc, zc);
  const int2 leaf_b = leaf[b];
  const int2 lf = make_int2(leaf_b.x + wk.y, min(kL2PF32Threads, leaf_b.y - wk.y));  // this item's targets
  const double inv_rb = 1.0 / rb;
  if ((int)threadIdx.x < lf.y) {  // one target per thread
    const int i = lf.x + threadIdx.x;
    const float4 xt = tpos[i];
    const float x = (float)(((double)xt.x - xc) * inv_rb), y = (float)(((double)xt.y - yc) * inv_rb),
                z = (float)(((double)xt.z - zc) * inv_rb);
    const float r2 = x * x + y * y + z * z;
    double F = 0, dzr = 0, dpr = 0, dpi = 0, dmr = 0, dmi = 0;
    float r1re[P + 1], r1im[P + 1], r2re[P + 1], r2im[P + 1];
#pragma unroll
    for (int m = 0; m <= P; m++) r1re[m] = r1im[m] = r2re[m] = r2im[m] = 0.f;
#pragma unroll
    for (int n = 0; n <= P; n++) {
      float cre[P + 1], cim[P + 1];
      float fn = 0.f;
      float2 fz = make_float2(0.f, 0.f), pmr = fz, pmi = fz;  // (fn, zn), (pr, mr), (pi, mi)
#pragma unroll
      for (int m = 0; m <= P; m++) {
        cre[m] = cim[m] = 0.f;
        if (m > n) continue;
        if (n == 0) {
          cre[0] = 1.f;
        } else if (m == n) {  // S_n^n = -(2n-1) (x + i y) S_{n-1}^{n-1}
          const float a = -(2.f * n - 1.f);
          cre[m] = a * (x * r1re[n - 1] - y * r1im[n - 1]);
          cim[m] = a * (x * r1im[n - 1] + y * r1re[n - 1]);
        } else if (m == n - 1) {
          const float a = (2.f * n - 1.f) * z;
          cre[m] = a * r1re[m];
          cim[m] = a * r1im[m];
        } else {
          const float inv = 1.f / (float)(n - m);
          const float a = (2.f * n - 1.f) * z * inv, c = (float)(n + m - 1) * r2 * inv;
          cre[m] = a * r1re[m] - c * r2re[m];
          cim[m] = a * r1im[m] - c * r2im[m];
        }
        const int idx = n * (n + 1) / 2 + m;
        if (DER) {
          const float4 a = CA[idx], bq = CB[idx];
          const float2 cc = CC[idx];
          const float2 re2 = make_float2(cre[m], cre[m]), im2 = make_float2(cim[m], cim[m]);
          fz = __ffma2_rn(make_float2(a.x, a.y), re2, __ffma2_rn(make_float2(a.z, a.w), im2, fz));
          pmr = __ffma2_rn(make_float2(bq.x, bq.y), re2, __ffma2_rn(make_float2(bq.z, bq.w), im2, pmr));
          pmi = __ffma2_rn(make_float2(bq.x, bq.y), im2, __ffma2_rn(cc, re2, pmi));
          if (m == 1) {  // Cs[n] * conj(S_n^1)
            const float cs = lds1(Cs + n);
            pmr.y = fmaf(cs, cre[m], pmr.y);
            pmi.y = fmaf(-cs, cim[m], pmi.y);
          }
        } else {
          const float2 cf = lds2(Cphi + idx);
          fn = fmaf(cf.x, cre[m], fmaf(-cf.y, cim[m], fn));
        }
      }
      if (DER) {
        F += (double)fz.x;
        dzr += (double)fz.y;
        dpr += (double)pmr.x;
        dpi += (double)pmi.x;
        dmr += (double)pmr.y;
        dmi += (double)pmi.y;
      } else {
        F += (double)fn;
      }
#pragma unroll
      for (int m = 0; m <= P; m++) {
        r2re[m] = r1re[m];
        r2im[m] = r1im[m];
        r1re[m] = cre[m];
        r1im[m] = cim[m];
      }
    }
    const double gx = 0.5 * (dpr + dmr), gy = 0.5 * (dpi - dmi), gz = dzr;
    const double c1 = coef * inv_rb, c2 = coef * inv_rb * inv_rb;
    if (KER == FMMB_LAPLACE_GNI) {
      const float4 nv = tnrm[i];
      pot[i] = -c2 * ((double)nv.x * gx + (double)nv.y * gy + (double)nv.z * gz);
    } else {
      pot[i] = c1 * F;
      if (KER == FMMB_LAPLACE_G && grad) {
        grad[i] = c2 * gx;
        grad[ni + i] = c2 * gy;
        grad[2 * ni + i] = c2 * gz;
      }
    }
  }
}

template <int P>
void l2p_f32_launch(int kernel, int nwork, const int2* work, int p, int K, const int* keys, const int2* leaf,
                    const float4* tpos, const float4* tnrm, const double* fac, const float* bbox, double rb,
                    double coef, const double* L, double* pot, double* grad, int ni, cudaStream_t st) {
  if (kernel == FMMB_LAPLACE_G)
    l2p_f32<FMMB_LAPLACE_G, P><<<nwork, kL2PF32Threads, 0, st>>>(p, K, work, keys, leaf, tpos, tnrm, fac, bbox[0], bbox[1], bbox[2], rb, coef, L, pot, grad, ni);
  else if (kernel == FMMB_LAPLACE_GNI)
    l2p_f32<FMMB_LAPLACE_GNI, P><<<nwork, kL2PF32Threads, 0, st>>>(p, K, work, keys, leaf, tpos, tnrm, fac, bbox[0], bbox[1], bbox[2], rb, coef, L, pot, grad, ni);
  else
    l2p_f32<FMMB_LAPLACE_GNJ, P><<<nwork, kL2PF32Threads, 0, st>>>(p, K, work, keys, leaf, tpos, tnrm, fac, bbox[0], bbox[1], bbox[2], rb, coef, L, pot, grad, ni);
}

}  // namespace

void launch_p2m_cart(int kernel, int nleaf, int p, int K, const int* keys, const int2* leaf, const float4* spos,
                     const float4* snrm, const float* qs, const double* fac, const float* bbox, double rb, double* M,
                     cudaStream_t st) {
  if (nleaf <= 0) return;
  if (p <= 14) {
    const size_t sm = (size_t)(128 / 16) * K * sizeof(double);
    if (kernel == FMMB_LAPLACE_GNJ)
      p2m_cart<FMMB_LAPLACE_GNJ, 16><<<nleaf, 128, sm, st>>>(p, K, keys, leaf, spos, snrm, qs, fac, bbox[0], bbox[1], bbox[2], rb, M);
    else
      p2m_cart<FMMB_LAPLACE_G, 16><<<nleaf, 128, sm, st>>>(p, K, keys, leaf, spos, snrm, qs, fac, bbox[0], bbox[1], bbox[2], rb, M);
  } else {
    const size_t sm = (size_t)(128 / 32) * K * sizeof(double);
    if (kernel == FMMB_LAPLACE_GNJ)
      p2m_cart<FMMB_LAPLACE_GNJ, 32><<<nleaf, 128, sm, st>>>(p, K, keys, leaf, spos, snrm, qs, fac, bbox[0], bbox[1], bbox[2], rb, M);
    else
      p2m_cart<FMMB_LAPLACE_G, 32><<<nleaf, 128, sm, st>>>(p, K, keys, leaf, spos, snrm, qs, fac, bbox[0], bbox[1], bbox[2], rb, M);
  }
  FMMB_CHECK_LAUNCH();
}

namespace {
template <int P>
void p2m_f32_launch(int kernel, int nwork, const int2* work, int p, int K, const int* keys, const int2* leaf,
                    const float4* spos, const float4* snrm, const float* qs, const float* bbox, double rb, double* M,
                    cudaStream_t st) {
  const size_t sm = (size_t)kP2MThreads * K * sizeof(float);
  if (kernel == FMMB_LAPLACE_GNJ)
    p2m_f32<FMMB_LAPLACE_GNJ, P><<<nwork, kP2MThreads, sm, st>>>(p, K, work, keys, leaf, spos, snrm, qs, bbox[0], bbox[1], bbox[2], rb, M);
  else
    p2m_f32<FMMB_LAPLACE_G, P><<<nwork, kP2MThreads, sm, st>>>(p, K, work, keys, leaf, spos, snrm, qs, bbox[0], bbox[1], bbox[2], rb, M);
}
}  // namespace

void init_fac32() {
  static bool done[64] = {};
  int dev = 0;
  FMMB_CUDA(cudaGetDevice(&dev));
  if (dev < 64 && done[dev]) return;
  float h[21 * 21 + 21] = {};
  for (int n = 0; n <= 20; n++)
    for (int m = 0; m <= n; m++) {
      double f = 1.0;  // sqrt((n-m)!/(n+m)!)
      for (int k = n - m + 1; k <= n + m; k++) f /= k;
      h[n * n + n + m] = (float)std::sqrt(f);
    }
  FMMB_CUDA(cudaMemcpyToSymbol(c_fac32, h, sizeof(h)));
  if (dev < 64) done[dev] = true;
}

bool launch_p2m_f32(int kernel, int nwork, const int2* work, int p, int K, const int* keys, const int2* leaf,
                    const float4* spos, const float4* snrm, const float* qs, const float* bbox, double rb, double* M,
                    cudaStream_t st) {
  if ((size_t)kP2MThreads * K * sizeof(float) > 48 * 1024) return false;  // per-point rows staged in shared memory
  if (p > 16) return false;
  if (nwork <= 0) return true;
  if (p <= 8) p2m_f32_launch<8>(kernel, nwork, work, p, K, keys, leaf, spos, snrm, qs, bbox, rb, M, st);
  else if (p <= 10) p2m_f32_launch<10>(kernel, nwork, work, p, K, keys, leaf, spos, snrm, qs, bbox, rb, M, st);
  else if (p <= 12) p2m_f32_launch<12>(kernel, nwork, work, p, K, keys, leaf, spos, snrm, qs, bbox, rb, M, st);
  else p2m_f32_launch<16>(kernel, nwork, work, p, K, keys, leaf, spos, snrm, qs, bbox, rb, M, st);
  FMMB_CHECK_LAUNCH();
  return true;
}

void launch_l2p_cart(int kernel, int nleaf, int p, int K, const int* keys, const int2* leaf, const float4* tpos,
                     const float4* tnrm, const double* fac, const float* bbox, double rb, double coef, const double* L,
                     double* pot, double* grad, int ni, cudaStream_t st) {
  if (nleaf <= 0) return;
  const int P = (p + 1) * (p + 2) / 2;
  const size_t sm = (size_t)4 * P * 2 * sizeof(double) + (p + 1) * sizeof(double);
  if (kernel == FMMB_LAPLACE_G)
    l2p_cart<FMMB_LAPLACE_G><<<nleaf, kL2PThreads, sm, st>>>(p, K, keys, leaf, tpos, tnrm, fac, bbox[0], bbox[1], bbox[2], rb, coef, L, pot, grad, ni);
  else if (kernel == FMMB_LAPLACE_GNI)
    l2p_cart<FMMB_LAPLACE_GNI><<<nleaf, kL2PThreads, sm, st>>>(p, K, keys, leaf, tpos, tnrm, fac, bbox[0], bbox[1], bbox[2], rb, coef, L, pot, grad, ni);
  else
    l2p_cart<FMMB_LAPLACE_GNJ><<<nleaf, kL2PThreads, sm, st>>>(p, K, keys, leaf, tpos, tnrm, fac, bbox[0], bbox[1], bbox[2], rb, coef, L, pot, grad, ni);
  FMMB_CHECK_LAUNCH();
}

void launch_l2p_hess_gni(int nleaf, int p, int K, const int* keys, const int2* leaf, const float4* tpos,
                         const float4* tnrm, const double* fac, const float* bbox, double rb, double coef,
                         const double* L, double* grad, int ni, cudaStream_t st) {
  if (nleaf <= 0) return;
  const int P = (p + 1) * (p + 2) / 2;
  const size_t sm = (size_t)12 * P * sizeof(cplx) + 3 * (p + 1) * sizeof(double);
  l2p_hess_gni<<<nleaf, kL2PHThreads, sm, st>>>(p, K, keys, leaf, tpos, tnrm, fac, bbox[0], bbox[1], bbox[2], rb, coef,
                                                L, grad, ni);
  FMMB_CHECK_LAUNCH();
}

bool launch_l2p_f32(int kernel, int nwork, const int2* work, int p, int K, const int* keys, const int2* leaf,
                    const float4* tpos, const float4* tnrm, const double* fac, const float* bbox, double rb,
                    double coef, const double* L, double* pot, double* grad, int ni, cudaStream_t st) {
  if (p > 16) return false;
  if (nwork <= 0) return true;
  if (p <= 8) l2p_f32_launch<8>(kernel, nwork, work, p, K, keys, leaf, tpos, tnrm, fac, bbox, rb, coef, L, pot, grad, ni, st);
  else if (p <= 10) l2p_f32_launch<10>(kernel, nwork, work, p, K, keys, leaf, tpos, tnrm, fac, bbox, rb, coef, L, pot, grad, ni, st);
  else if (p <= 12) l2p_f32_launch<12>(kernel, nwork, work, p, K, keys, leaf, tpos, tnrm, fac, bbox, rb, coef, L, pot, grad, ni, st);
  else l2p_f32_launch<16>(kernel, nwork, work, p, K, keys, leaf, tpos, tnrm, fac, bbox, rb, coef, L, pot, grad, ni, st);
  FMMB_CHECK_LAUNCH();
  return true;
}

}  // namespace fmmb

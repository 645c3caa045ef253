// Complex Helmholtz kernel e^{ikr} / (4 pi r) (FMMB_HELMHOLTZ_G).
//
// The reference's "Helmholtz" is the Yukawa kernel (kernel/Helmholtz_*.cxx);
// the oscillatory kernel has no counterpart there, so this family is written
// from the mathematics:
//
//   e^{ik|x-y|} / (4 pi |x-y|) = ik sum_n j_n(k|y|) h_n(k|x|) sum_m Y_n^m(x^) conj(Y_n^m(y^)),  |x| > |y|
//
// with h_n = j_n + i y_n the spherical Hankel function of the first kind and
// Y_n^m = Ybar_n^|m|(cos t) e^{i m p} the orthonormal spherical harmonics
// (no Condon-Shortley phase; Ybar by the standard fully normalised
// three-term recurrence).  Expansions hold K = (p+1)^2 complex coefficients
// per box, index n^2 + n + m, stored as [re(K) | im(K)]:
//   multipole  phi(x) = sum M_n^m h_n(k r) Y_n^m,  M_n^m = ik sum_j q_j j_n(k rho_j) conj(Y_n^m)
//   local      phi(x) = sum L_n^m j_n(k r) Y_n^m
// Spherical Bessel functions: j_n by Miller's backward recurrence (upward
// when x > n, the power series near 0), y_n by the upward recurrence -- the
// standard methods (e.g. Abramowitz & Stegun 10.1.19, Press et al. 6.7).
//
// Translations (M2M, M2L, L2L) are dense complex K x K operators per level
// and relative position, built here on the GPU by projection: the field of
// one source basis function is sampled on a sphere around the target centre
// (Gauss-Legendre nodes in cos(theta) x equispaced in phi, 2p+8 x 4p+16
// points) and projected on the target basis, conj(Y) and a division by the
// target radial function at the sphere's radius.  The operators are stored in
// the real 2K x 2K form acting on [re | im] (transposed, row stride 2K) and
// applied by the FP64 pair kernel of kernels_fp64.cu.
//
// The same code serves the Yukawa kernel (FMMB_YUKAWA, the reference's neq 10,
// kernel/Helmholtz_G_p2p.cxx:18-23: (pi/2) e^{-lambda r} / (lambda r)) through
//   e^{-l|x-y|} / (4 pi |x-y|) = (2l/pi) sum_n i_n(l|y|) k_n(l|x|) sum_m Y_n^m(x^) conj(Y_n^m(y^))
// with the modified spherical Bessel functions i_n (Miller's backward
// recurrence normalised by i_0 = sinh(x)/x) and k_n (k_0 = (pi/2) e^{-x}/x,
// upward recurrence): real radial functions in place of j_n and h_n, the
// factor 2l/pi in place of ik; the result is scaled by 2 pi^2 / l on output.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>

#include "internal.h"
#include "kernels.h"

namespace fmmb {
namespace {

constexpr int kMaxP = 20;

// j_n(x), n = 0..nmax, x >= 0
__device__ void sph_j(int nmax, double x, double* j) {
  if (x < 1e-6) {  // x^n / (2n+1)!! (1 - x^2 / (2 (2n+3)))
    double t = 1.0;
    for (int n = 0; n <= nmax; n++) {
      j[n] = t * (1.0 - x * x / (2.0 * (2 * n + 3)));
      t *= x / (2 * n + 3);
    }
    return;
  }
  double s, c;
  sincos(x, &s, &c);
  const double j0 = s / x, j1 = s / (x * x) - c / x;
  j[0] = j0;
  if (nmax == 0) return;
  if (x > (double)nmax) {  // upward recurrence is stable
    j[1] = j1;
    for (int n = 1; n < nmax; n++) j[n + 1] = (2 * n + 1) / x * j[n] - j[n - 1];
    return;
  }
  // Miller: backward from N with arbitrary start, rescaled on the way, then
  // normalised by the larger of j0, j1
  const int N = nmax + 24 + (int)x;
  double jp1 = 0.0, jn = 1e-250;
  for (int n = N; n >= 1; n--) {
    const double jm1 = (2 * n + 1) / x * jn - jp1;
    jp1 = jn;
    jn = jm1;
    if (n - 1 <= nmax) j[n - 1] = jm1;
    if (fabs(jn) > 1e250) {
      jn *= 1e-250;
      jp1 *= 1e-250;
      for (int k = max(n - 1, 0); k <= nmax; k++) j[k] *= 1e-250;
    }
  }
  const double sc = fabs(j0) >= fabs(j1) ? j0 / j[0] : j1 / j[1];
  for (int n = 0; n <= nmax; n++) j[n] *= sc;
}

// y_n(x), n = 0..nmax, x > 0 (upward recurrence)
__device__ void sph_y(int nmax, double x, double* y) {
  double s, c;
  sincos(x, &s, &c);
  y[0] = -c / x;
  if (nmax >= 1) y[1] = -c / (x * x) - s / x;
  for (int n = 1; n < nmax; n++) y[n + 1] = (2 * n + 1) / x * y[n] - y[n - 1];
}

// i_n(x), n = 0..nmax, x >= 0: Miller's backward recurrence
// i_{n-1} = i_{n+1} + (2n+1)/x i_n, normalised by i_0 = sinh(x)/x
__device__ void sph_i(int nmax, double x, double* v) {
  if (x < 1e-6) {  // x^n / (2n+1)!! (1 + x^2 / (2 (2n+3)))
    double t = 1.0;
    for (int n = 0; n <= nmax; n++) {
      v[n] = t * (1.0 + x * x / (2.0 * (2 * n + 3)));
      t *= x / (2 * n + 3);
    }
    return;
  }
  const int N = nmax + 24 + (int)x;
  double ip1 = 0.0, in = 1e-250;
  for (int n = N; n >= 1; n--) {
    const double im1 = (2 * n + 1) / x * in + ip1;
    ip1 = in;
    in = im1;
    if (n - 1 <= nmax) v[n - 1] = im1;
    if (fabs(in) > 1e250) {
      in *= 1e-250;
      ip1 *= 1e-250;
      for (int q = max(n - 1, 0); q <= nmax; q++) v[q] *= 1e-250;
    }
  }
  const double sc = (sinh(x) / x) / v[0];
  for (int n = 0; n <= nmax; n++) v[n] *= sc;
}

// k_n(x), n = 0..nmax, x > 0, normalised k_0 = (pi/2) e^{-x} / x (upward recurrence)
__device__ void sph_k(int nmax, double x, double* v) {
  const double e = 0.5 * M_PI * exp(-x);
  v[0] = e / x;
  if (nmax >= 1) v[1] = e * (1.0 / x + 1.0 / (x * x));
  for (int n = 1; n < nmax; n++) v[n + 1] = v[n - 1] + (2 * n + 1) / x * v[n];
}

// regular radial functions: j_n (Helmholtz) or i_n (Yukawa)
__device__ __forceinline__ void radial_reg(int yuk, int nmax, double x, double* v) {
  if (yuk) sph_i(nmax, x, v);
  else sph_j(nmax, x, v);
}

// direction of v: cos(theta), and e^{i phi} (1 on the axis)
__device__ __forceinline__ void direction(double vx, double vy, double vz, double r, double& ct, double& st, double& cp,
                                          double& sp) {
  const double rxy = sqrt(vx * vx + vy * vy);
  if (r > 0) {
    ct = vz / r;
    st = rxy / r;
  } else {
    ct = 1.0;
    st = 0.0;
  }
  if (rxy > 0) {
    cp = vx / rxy;
    sp = vy / rxy;
  } else {
    cp = 1.0;
    sp = 0.0;
  }
}

// Ybar_m^m from Ybar_{m-1}^{m-1}
__device__ __forceinline__ double ybar_mm_next(int m, double st, double prev) {
  return sqrt((2.0 * m + 1.0) / (2.0 * m)) * st * prev;
}
// Ybar_n^m from Ybar_{n-1}^m, Ybar_{n-2}^m (n >= m+2)
__device__ __forceinline__ double ybar_next(int n, int m, double ct, double y1, double y2) {
  const double a = sqrt((4.0 * n * n - 1.0) / ((double)n * n - (double)m * m));
  const double b = sqrt((((double)n - 1) * (n - 1) - (double)m * m) / (4.0 * (n - 1) * (n - 1) - 1.0));
  return a * (ct * y1 - b * y2);
}

// Ybar_n^m(ct) for one (n, m), m >= 0
__device__ double ybar_one(int n, int m, double ct, double st) {
  double ymm = 0.28209479177387814;  // 1 / sqrt(4 pi)
  for (int k = 1; k <= m; k++) ymm = ybar_mm_next(k, st, ymm);
  if (n == m) return ymm;
  double y2 = ymm, y1 = sqrt(2.0 * m + 3.0) * ct * ymm;
  for (int l = m + 2; l <= n; l++) {
    const double y = ybar_next(l, m, ct, y1, y2);
    y2 = y1;
    y1 = y;
  }
  return y1;
}

struct Corner {  // root-cube corner (passed by value: the plan keeps it on the host)
  double x, y, z;
};

__device__ __forceinline__ void box_centre(int key, Corner bbox, double w, double& x, double& y, double& z) {
  int cx = 0, cy = 0, cz = 0;
  for (int i = 0; i < 10; i++) {
    cy |= ((key >> (3 * i)) & 1) << i;
    cx |= ((key >> (3 * i + 1)) & 1) << i;
    cz |= ((key >> (3 * i + 2)) & 1) << i;
  }
  x = bbox.x + (cx + 0.5) * w;
  y = bbox.y + (cy + 0.5) * w;
  z = bbox.z + (cz + 0.5) * w;
}

__device__ __forceinline__ double warp_sum(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// ---------------------------------------------------------------- P2M
// One block (4 warps) per source leaf; a warp takes 32 points at a time, each
// lane streams its point's terms over (m, n), warp sums go to shared FP64
// accumulators; M = ik * sum.
__global__ void __launch_bounds__(128) helm_p2m(int p, int K, double k, int yuk, const int* __restrict__ keys,
                                                const int2* __restrict__ leaf, const float4* __restrict__ spos,
                                                const float2* __restrict__ q, Corner bbox, double w,
                                                double* __restrict__ M) {
  extern __shared__ double acc[];  // [2K]
  const int b = blockIdx.x;
  for (int c = threadIdx.x; c < 2 * K; c += blockDim.x) acc[c] = 0.0;
  __syncthreads();
  double xc, yc, zc;
  box_centre(keys[b], bbox, w, xc, yc, zc);
  const int2 lf = leaf[b];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  double jv[kMaxP + 1];
  for (int base = warp * 32; base < lf.y; base += 128) {
    const int i = base + lane;
    const bool on = i < lf.y;
    double vx = 0, vy = 0, vz = 0, qr = 0, qi = 0;
    if (on) {
      const float4 s = spos[lf.x + i];
      const float2 qq = q[lf.x + i];
      vx = (double)s.x - xc;
      vy = (double)s.y - yc;
      vz = (double)s.z - zc;
      qr = qq.x;
      qi = qq.y;
    }
    const double r = sqrt(vx * vx + vy * vy + vz * vz);
    double ct, st, cp, sp;
    direction(vx, vy, vz, r, ct, st, cp, sp);
    radial_reg(yuk, p, k * r, jv);
    double ymm = 0.28209479177387814, er = 1.0, ei = 0.0;  // Ybar_m^m, e^{i m phi}
    for (int m = 0; m <= p; m++) {
      if (m > 0) {
        ymm = ybar_mm_next(m, st, ymm);
        const double t = er * cp - ei * sp;
        ei = er * sp + ei * cp;
        er = t;
      }
      double y2 = 0.0, y1 = ymm;
      for (int n = m; n <= p; n++) {
        double y;
        if (n == m) y = ymm;
        else if (n == m + 1) y = sqrt(2.0 * m + 3.0) * ct * ymm;
        else y = ybar_next(n, m, ct, y1, y2);
        if (n > m) {
          y2 = y1;
          y1 = y;
        }
        const double a = on ? jv[n] * y : 0.0;
        // conj(Y_n^m) = Ybar e^{-i m phi}: q a (er - i ei)
        double tr = warp_sum(a * (qr * er + qi * ei));
        double ti = warp_sum(a * (qi * er - qr * ei));
        if (lane == 0) {
          atomicAdd(&acc[n * n + n + m], tr);
          atomicAdd(&acc[K + n * n + n + m], ti);
        }
        if (m > 0) {  // conj(Y_n^{-m}) = Ybar e^{+i m phi}
          tr = warp_sum(a * (qr * er - qi * ei));
          ti = warp_sum(a * (qi * er + qr * ei));
          if (lane == 0) {
            atomicAdd(&acc[n * n + n - m], tr);
            atomicAdd(&acc[K + n * n + n - m], ti);
          }
        }
      }
    }
  }
  __syncthreads();
  double* out = M + (size_t)b * 2 * K;
  for (int c = threadIdx.x; c < K; c += blockDim.x) {
    if (yuk) {  // (2 l / pi) (a + ib)
      out[c] = 2.0 * k / M_PI * acc[c];
      out[K + c] = 2.0 * k / M_PI * acc[K + c];
    } else {  // ik (a + ib) = -k b + i k a
      out[c] = -k * acc[K + c];
      out[K + c] = k * acc[c];
    }
  }
}

// ---------------------------------------------------------------- L2P
// One block per target leaf, one thread per target: phi = sum L j_n(kr) Y_n^m.
__global__ void __launch_bounds__(128) helm_l2p(int p, int K, double k, int yuk, const int* __restrict__ keys,
                                                const int2* __restrict__ leaf, const float4* __restrict__ tpos,
                                                Corner bbox, double w, const double* __restrict__ L,
                                                double2* __restrict__ pot) {
  extern __shared__ double Ls[];  // [2K]
  const int b = blockIdx.x;
  for (int c = threadIdx.x; c < 2 * K; c += blockDim.x) Ls[c] = L[(size_t)b * 2 * K + c];
  __syncthreads();
  double xc, yc, zc;
  box_centre(keys[b], bbox, w, xc, yc, zc);
  const int2 lf = leaf[b];
  double jv[kMaxP + 1];
  for (int i = threadIdx.x; i < lf.y; i += blockDim.x) {
    const float4 t = tpos[lf.x + i];
    const double vx = (double)t.x - xc, vy = (double)t.y - yc, vz = (double)t.z - zc;
    const double r = sqrt(vx * vx + vy * vy + vz * vz);
    double ct, st, cp, sp;
    direction(vx, vy, vz, r, ct, st, cp, sp);
    radial_reg(yuk, p, k * r, jv);
    double pr = 0, pi = 0;
    double ymm = 0.28209479177387814, er = 1.0, ei = 0.0;
    for (int m = 0; m <= p; m++) {
      if (m > 0) {
        ymm = ybar_mm_next(m, st, ymm);
        const double tt = er * cp - ei * sp;
        ei = er * sp + ei * cp;
        er = tt;
      }
      double y2 = 0.0, y1 = ymm;
      for (int n = m; n <= p; n++) {
        double y;
        if (n == m) y = ymm;
        else if (n == m + 1) y = sqrt(2.0 * m + 3.0) * ct * ymm;
        else y = ybar_next(n, m, ct, y1, y2);
        if (n > m) {
          y2 = y1;
          y1 = y;
        }
        const double a = jv[n] * y;
        const int c = n * n + n + m;
        // L_n^m e^{i m phi}
        pr += a * (Ls[c] * er - Ls[K + c] * ei);
        pi += a * (Ls[c] * ei + Ls[K + c] * er);
        if (m > 0) {  // L_n^{-m} e^{-i m phi}
          const int c2 = n * n + n - m;
          pr += a * (Ls[c2] * er + Ls[K + c2] * ei);
          pi += a * (Ls[K + c2] * er - Ls[c2] * ei);
        }
      }
    }
    pot[lf.x + i] = make_double2(pr, pi);
  }
}

// ---------------------------------------------------------------- P2P
// Pairs at zero distance are skipped when the plan excludes them; eps2 (the
// plan's softening) is added to r^2.
// One block (128 threads) per work item = up to 256 targets of one leaf, two
// per thread (one shared-memory read of a source serves both); the sources of
// the leaf's 27 neighbour slots are staged through shared memory in chunks of
// 128.  Work items split large leaves, so the launch is not bound by the
// densest leaf.  Mixed form: FP32 terms (hardware sine / cosine of the
// phase reduced to [-pi, pi]), summed over 32 sources, then added in FP64;
// FP64 form: everything in FP64.  Zero-distance pairs
// contribute nothing (their inverse distance is taken as 0).
template <bool YUK, bool REDUCE>
__device__ __forceinline__ void helm_pair(float k, float eps2, bool excl, const float4 x, const float4 s,
                                          const float2 q, float& fr, float& fi) {
  const float dx = x.x - s.x, dy = x.y - s.y, dz = x.z - s.z;
  const float d2 = dx * dx + dy * dy + dz * dz, r2 = d2 + eps2;
  const float rinv = (excl && d2 == 0.f) || r2 == 0.f ? 0.f : rsqrtf(r2);
  if (YUK) {  // real kernel e^{-l r} / r
    const float e = __expf(-k * (r2 * rinv)) * rinv;
    fr = fmaf(q.x, e, fr);
    fi = fmaf(q.y, e, fi);
    return;
  }
  // phase k r reduced to [-pi, pi] (the identity for k r < pi, the usual
  // near-field range), then the hardware sine / cosine (absolute error ~4e-7
  // there)
  const float ph = k * (r2 * rinv);
  const float red = REDUCE ? fmaf(-6.28318530717958647f, rintf(ph * 0.159154943091895336f), ph) : ph;
  float sn, cs;
  __sincosf(red, &sn, &cs);
  fr += (q.x * cs - q.y * sn) * rinv;
  fi += (q.x * sn + q.y * cs) * rinv;
}
template <bool YUK>
__device__ __forceinline__ void helm_pair64(double k, double eps2, bool excl, const float4 x, const float4 s,
                                            const float2 q, double& ar, double& ai) {
  const double dx = (double)x.x - s.x, dy = (double)x.y - s.y, dz = (double)x.z - s.z;
  const double d2 = dx * dx + dy * dy + dz * dz, r2 = d2 + eps2;
  if ((excl && d2 == 0.0) || r2 == 0.0) return;
  const double r = sqrt(r2);
  if (YUK) {
    const double e = exp(-k * r) / r;
    ar += q.x * e;
    ai += q.y * e;
    return;
  }
  double sn, cs;
  sincos(k * r, &sn, &cs);
  ar += (q.x * cs - q.y * sn) / r;
  ai += (q.x * sn + q.y * cs) / r;
}

// Near field.  A block of 128 threads takes a work item of up to 256 targets
// of one leaf (2 per thread).  The sources of its (up to 27) neighbour leaves
// are staged into shared memory as one list in chunks of kHC (warp 0 lays the
// leaves end to end with one lane per neighbour slot: ballot + scan), so a
// chunk costs two barriers whatever the leaf sizes -- the former per-leaf
// staging paid two barriers per 128 sources of every leaf.  Each thread sums
// runs of 32 sources in FP32 (mixed form) and promotes each run's partial sum
// to FP64.  REDUCE: reduce the phase k r to [-pi, pi] before the hardware sine
// and cosine; the launcher leaves it out when every near-field distance is
// below pi / k (then the reduction is the identity: same values).
constexpr int kHC = 1024;

template <bool F32, bool YUK, bool REDUCE>
__global__ void __launch_bounds__(128) helm_p2p(float k, float eps2, int excl, const int2* __restrict__ work,
                                                const int2* __restrict__ leaf_i,
                                                const int2* __restrict__ leaf_j, const int* __restrict__ list,
                                                const float4* __restrict__ tpos, const float4* __restrict__ spos,
                                                const float2* __restrict__ q, double2* __restrict__ pot) {
  __shared__ float4 sp[kHC];
  __shared__ float2 sq[kHC];
  __shared__ int2 seg[32];  // (first source, count) of each non-empty neighbour leaf
  __shared__ int vst[33];   // start of each leaf in the staged list, then the total
  __shared__ int nseg_s;
  const int2 wk = work[blockIdx.x];
  const int b = wk.x;
  const int2 li = leaf_i[b];
  const int i0 = wk.y + threadIdx.x, i1 = i0 + 128;
  const bool on0 = i0 < li.y, on1 = i1 < li.y;
  const float4 x0 = on0 ? tpos[li.x + i0] : make_float4(0.f, 0.f, 0.f, 0.f);
  const float4 x1 = on1 ? tpos[li.x + i1] : make_float4(0.f, 0.f, 0.f, 0.f);
  if (threadIdx.x < 32) {
    const int lane = threadIdx.x;
    int2 sg = make_int2(0, 0);
    if (lane < kP2PSlots) {
      const int jl = list[(size_t)b * kP2PSlots + lane];
      if (jl >= 0) sg = leaf_j[jl];
    }
    const bool has = sg.y > 0;
    const unsigned mask = __ballot_sync(0xffffffffu, has);
    const int pos = __popc(mask & ((1u << lane) - 1u));
    int incl = has ? sg.y : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += t;
    }
    if (has) {
      seg[pos] = sg;
      vst[pos] = incl - sg.y;
    }
    if (lane == 31) {
      vst[__popc(mask)] = incl;  // the total
      nseg_s = __popc(mask);
    }
  }
  __syncthreads();
  const int nseg = nseg_s, ntot = vst[nseg];
  double ar0 = 0, ai0 = 0, ar1 = 0, ai1 = 0;
  for (int c0 = 0; c0 < ntot; c0 += kHC) {
    const int nc = min(kHC, ntot - c0);
    __syncthreads();  // the previous chunk's readers are done
    for (int u = threadIdx.x; u < nc; u += 128) {
      const int v = c0 + u;
      int sgi = 0;
      while (sgi + 1 < nseg && vst[sgi + 1] <= v) sgi++;
      const int j = seg[sgi].x + (v - vst[sgi]);
      sp[u] = spos[j];
      sq[u] = q[j];
    }
    __syncthreads();
    if (!on0) continue;
    for (int r0 = 0; r0 < nc; r0 += 32) {
      const int re = min(nc, r0 + 32);
      if (F32) {
        float fr0 = 0.f, fi0 = 0.f, fr1 = 0.f, fi1 = 0.f;
        if (on1) {
          for (int jj = r0; jj < re; jj++) {
            const float4 sv = sp[jj];
            const float2 qq = sq[jj];
            helm_pair<YUK, REDUCE>(k, eps2, excl, x0, sv, qq, fr0, fi0);
            helm_pair<YUK, REDUCE>(k, eps2, excl, x1, sv, qq, fr1, fi1);
          }
        } else {
          for (int jj = r0; jj < re; jj++) helm_pair<YUK, REDUCE>(k, eps2, excl, x0, sp[jj], sq[jj], fr0, fi0);
        }
        ar0 += fr0;
        ai0 += fi0;
        ar1 += fr1;
        ai1 += fi1;
      } else {
        for (int jj = r0; jj < re; jj++) {
          const float4 sv = sp[jj];
          const float2 qq = sq[jj];
          helm_pair64<YUK>((double)k, (double)eps2, excl, x0, sv, qq, ar0, ai0);
          if (on1) helm_pair64<YUK>((double)k, (double)eps2, excl, x1, sv, qq, ar1, ai1);
        }
      }
    }
  }
  const double coef = 0.25 / M_PI;
  if (on0) pot[li.x + i0] = make_double2(coef * ar0, coef * ai0);
  if (on1) pot[li.x + i1] = make_double2(coef * ar1, coef * ai1);
}

// ---------------------------------------------------------------- direct
__global__ void __launch_bounds__(128) helm_direct(int i0, int i1, const int* __restrict__ inv_i,
                                                   const float4* __restrict__ tpos, int nj,
                                                   const float4* __restrict__ spos, const float2* __restrict__ q,
                                                   double k, int yuk, double eps2, int excl,
                                                   double2* __restrict__ out) {
  __shared__ float4 sp[128];
  __shared__ float2 sq[128];
  const int i = i0 + blockIdx.x * blockDim.x + threadIdx.x;
  const bool act = i < i1;
  const float4 xi = tpos[act ? inv_i[i] : 0];
  double ar = 0, ai = 0;
  for (int j0 = 0; j0 < nj; j0 += 128) {
    __syncthreads();
    if (j0 + threadIdx.x < nj) {
      sp[threadIdx.x] = spos[j0 + threadIdx.x];
      sq[threadIdx.x] = q[j0 + threadIdx.x];
    }
    __syncthreads();
    const int nl = min(128, nj - j0);
    for (int jj = 0; jj < nl; jj++) {
      const double dx = (double)xi.x - sp[jj].x, dy = (double)xi.y - sp[jj].y, dz = (double)xi.z - sp[jj].z;
      const double d2 = dx * dx + dy * dy + dz * dz, r2 = d2 + eps2;
      if ((excl && d2 == 0.0) || r2 == 0.0) continue;
      const double r = sqrt(r2);
      double sn, cs;
      if (yuk) {
        sn = 0.0;
        cs = exp(-k * r);
      } else {
        sincos(k * r, &sn, &cs);
      }
      ar += (sq[jj].x * cs - sq[jj].y * sn) / r;
      ai += (sq[jj].x * sn + sq[jj].y * cs) / r;
    }
  }
  if (act) out[i - i0] = make_double2(0.25 / M_PI * ar, 0.25 / M_PI * ai);
}

// ---------------------------------------------------------------- operators
// One block per (operator, source coefficient).  f = source basis function
// R_n(k|v|) Y_n^m(v^) at v = D + rad * s_q over the quadrature points s_q;
// g[i][m'] = sum_j f[i][j] e^{-i m' phi_j} 2 pi / NP;
// T[n'm'] = sum_i w_i g[i][m'] Ybar_n'^|m'|(x_i) / R'_n'(k rad).
__global__ void __launch_bounds__(256) helm_build_ops(int p, int K, double k, int yuk, const HelmOp* __restrict__ ops,
                                                      int NQ, int NP, const double* __restrict__ gl_x,
                                                      const double* __restrict__ gl_w,
                                                      const double* __restrict__ ybar_q,  // [NQ][P] Ybar at the nodes
                                                      double* __restrict__ opT, size_t ostride) {
  extern __shared__ double sm[];
  double2* f = (double2*)sm;                   // [NQ * NP]
  double2* g = f + (size_t)NQ * NP;            // [NQ][2p+1]
  double2* rt = g + (size_t)NQ * (2 * p + 1);  // [p+1] target radial values at rad
  const int o = blockIdx.y, c = blockIdx.x;
  const HelmOp op = ops[o];
  int n = 0;
  while ((n + 1) * (n + 1) <= c) n++;
  const int m = c - n * n - n;
  const int am = m < 0 ? -m : m;
  double rad[kMaxP + 1], rad2[kMaxP + 1];
  // 1. samples of the source basis function
  for (int t = threadIdx.x; t < NQ * NP; t += blockDim.x) {
    const int iq = t / NP, jq = t % NP;
    const double x = gl_x[iq], s = sqrt(fmax(0.0, 1.0 - x * x));
    double sphi, cphi;
    sincospi(2.0 * jq / NP, &sphi, &cphi);
    const double vx = op.dx + op.rad * s * cphi, vy = op.dy + op.rad * s * sphi, vz = op.dz + op.rad * x;
    const double r = sqrt(vx * vx + vy * vy + vz * vz);
    double ct, st, cp, sp;
    direction(vx, vy, vz, r, ct, st, cp, sp);
    const double yb = ybar_one(n, am, ct, st);
    // e^{i m phi}
    double er = 1.0, ei = 0.0;
    for (int l = 0; l < am; l++) {
      const double tt = er * cp - ei * sp;
      ei = er * sp + ei * cp;
      er = tt;
    }
    if (m < 0) ei = -ei;
    double rr, ri = 0.0;
    if (yuk) {  // k_n outgoing, i_n regular
      if (op.src_out) sph_k(n, k * r, rad);
      else sph_i(n, k * r, rad);
      rr = rad[n];
    } else {  // h_n = j_n + i y_n outgoing, j_n regular
      sph_j(n, k * r, rad);
      rr = rad[n];
      if (op.src_out) {
        sph_y(n, k * r, rad2);
        ri = rad2[n];
      }
    }
    // (rr + i ri) yb (er + i ei)
    f[t] = make_double2(yb * (rr * er - ri * ei), yb * (rr * ei + ri * er));
  }
  if (threadIdx.x == 0) {
    if (yuk) {
      if (op.tgt_out) sph_k(p, k * op.rad, rad);
      else sph_i(p, k * op.rad, rad);
      for (int l = 0; l <= p; l++) rt[l] = make_double2(rad[l], 0.0);
    } else {
      sph_j(p, k * op.rad, rad);
      if (op.tgt_out) sph_y(p, k * op.rad, rad2);
      for (int l = 0; l <= p; l++) rt[l] = make_double2(rad[l], op.tgt_out ? rad2[l] : 0.0);
    }
  }
  __syncthreads();
  // 2. azimuthal transform
  const int nm = 2 * p + 1;
  for (int t = threadIdx.x; t < NQ * nm; t += blockDim.x) {
    const int iq = t / nm, mp = t % nm - p;
    double sr = 0, si = 0;
    for (int jq = 0; jq < NP; jq++) {
      double sn, cs;
      sincospi(-2.0 * mp * jq / NP, &sn, &cs);
      const double2 v = f[iq * NP + jq];
      sr += v.x * cs - v.y * sn;
      si += v.x * sn + v.y * cs;
    }
    g[t] = make_double2(sr * (2.0 * M_PI / NP), si * (2.0 * M_PI / NP));
  }
  __syncthreads();
  // 3. polar transform, division by the target radial function, real form
  double* col_re = opT + (size_t)o * ostride + (size_t)c * (2 * K);        // input re[c]
  double* col_im = opT + (size_t)o * ostride + (size_t)(K + c) * (2 * K);  // input im[c]
  for (int t = threadIdx.x; t < K; t += blockDim.x) {
    int n2 = 0;
    while ((n2 + 1) * (n2 + 1) <= t) n2++;
    const int m2 = t - n2 * n2 - n2;
    const int am2 = m2 < 0 ? -m2 : m2;
    double sr = 0, si = 0;
    for (int iq = 0; iq < NQ; iq++) {
      const double wy = gl_w[iq] * ybar_q[(size_t)iq * ((p + 1) * (p + 2) / 2) + n2 * (n2 + 1) / 2 + am2];
      const double2 v = g[iq * nm + m2 + p];
      sr += wy * v.x;
      si += wy * v.y;
    }
    const double2 d = rt[n2];
    const double den = d.x * d.x + d.y * d.y;
    const double tr = (sr * d.x + si * d.y) / den, ti = (si * d.x - sr * d.y) / den;
    col_re[t] = tr;
    col_re[K + t] = ti;
    col_im[t] = -ti;
    col_im[K + t] = tr;
  }
}

// ---------------------------------------------------------------- glue
__global__ void helm_gather(int n, int nrhs, const int* __restrict__ perm, const float2* __restrict__ q,
                            float2* __restrict__ qs) {
  const size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (t >= (size_t)n * nrhs) return;
  const int r = (int)(t / n), i = (int)(t % n);
  qs[t] = q[(size_t)r * n + perm[i]];
}

__global__ void helm_gather_real(int n, int nrhs, const int* __restrict__ perm, const float* __restrict__ q,
                                 float2* __restrict__ qs) {
  const size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (t >= (size_t)n * nrhs) return;
  const int r = (int)(t / n), i = (int)(t % n);
  qs[t] = make_float2(q[(size_t)r * n + perm[i]], 0.f);
}

// real part of near + far, scaled, to caller order (Yukawa)
template <typename T>
__global__ void helm_finalize_real(int n, const int* __restrict__ perm, const double2* __restrict__ near,
                                   const double2* __restrict__ far, double scale, T* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  out[perm[i]] = (T)(scale * (near[i].x + (far ? far[i].x : 0.0)));
}

template <typename T>
__global__ void helm_finalize(int n, const int* __restrict__ perm, const double2* __restrict__ near,
                              const double2* __restrict__ far, T* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double2 a = near[i], b = far ? far[i] : make_double2(0.0, 0.0);
  const int o = perm[i];
  out[2 * (size_t)o] = (T)(a.x + b.x);
  out[2 * (size_t)o + 1] = (T)(a.y + b.y);
}

unsigned nb(size_t n, int t) { return (unsigned)((n + t - 1) / t); }

}  // namespace

void launch_helm_gather(int n, int nrhs, const int* perm, const float* q, float* qs, cudaStream_t st) {
  if (n <= 0) return;
  helm_gather<<<nb((size_t)n * nrhs, 256), 256, 0, st>>>(n, nrhs, perm, (const float2*)q, (float2*)qs);
  FMMB_CHECK_LAUNCH();
}

void launch_helm_p2p(bool f32, bool yuk, float k, float eps2, bool excl, float leaf_side, int nwork,
                     const int2* work, const int2* leaf_i, const int2* leaf_j, const int* list, const float4* tpos,
                     const float4* spos, const float* qs, double* pot, cudaStream_t st) {
  if (nwork <= 0) return;
  const float2* q2 = (const float2*)qs;
  double2* p2 = (double2*)pot;
  const int ex = excl ? 1 : 0;
  // points of neighbouring leaves lie at most 2 sqrt(3) leaf sides apart:
  // below pi / k (with a margin for the float phase) no reduction is needed
  const double rmax = std::sqrt(12.0 * (double)leaf_side * leaf_side + (double)eps2);
  const bool reduce = !((double)k * rmax < 0.999 * M_PI);
  if (f32 && !yuk && reduce)
    helm_p2p<true, false, true><<<nwork, 128, 0, st>>>(k, eps2, ex, work, leaf_i, leaf_j, list, tpos, spos, q2, p2);
  else if (f32 && !yuk)
    helm_p2p<true, false, false><<<nwork, 128, 0, st>>>(k, eps2, ex, work, leaf_i, leaf_j, list, tpos, spos, q2, p2);
  else if (f32)
    helm_p2p<true, true, false><<<nwork, 128, 0, st>>>(k, eps2, ex, work, leaf_i, leaf_j, list, tpos, spos, q2, p2);
  else if (!yuk)
    helm_p2p<false, false, false><<<nwork, 128, 0, st>>>(k, eps2, ex, work, leaf_i, leaf_j, list, tpos, spos, q2, p2);
  else
    helm_p2p<false, true, false><<<nwork, 128, 0, st>>>(k, eps2, ex, work, leaf_i, leaf_j, list, tpos, spos, q2, p2);
  FMMB_CHECK_LAUNCH();
}

void launch_helm_gather_real(int n, int nrhs, const int* perm, const float* q, float* qs, cudaStream_t st) {
  if (n <= 0) return;
  helm_gather_real<<<nb((size_t)n * nrhs, 256), 256, 0, st>>>(n, nrhs, perm, q, (float2*)qs);
  FMMB_CHECK_LAUNCH();
}

template <typename T>
void launch_helm_finalize_real(int n, const int* perm, const double* near, const double* far, double scale, T* out,
                               cudaStream_t st) {
  if (n <= 0) return;
  helm_finalize_real<T><<<nb(n, 256), 256, 0, st>>>(n, perm, (const double2*)near, (const double2*)far, scale, out);
  FMMB_CHECK_LAUNCH();
}
template void launch_helm_finalize_real<float>(int, const int*, const double*, const double*, double, float*,
                                               cudaStream_t);
template void launch_helm_finalize_real<double>(int, const int*, const double*, const double*, double, double*,
                                                cudaStream_t);

void launch_helm_p2m(int nleaf, int p, double k, bool yuk, const int* keys, const int2* leaf, const float4* spos,
                     const float* qs, const float* bbox, double w, double* M, cudaStream_t st) {
  if (nleaf <= 0) return;
  const int K = (p + 1) * (p + 1);
  const Corner c{bbox[0], bbox[1], bbox[2]};  // host array
  helm_p2m<<<nleaf, 128, 2 * K * sizeof(double), st>>>(p, K, k, yuk ? 1 : 0, keys, leaf, spos, (const float2*)qs, c,
                                                        w, M);
  FMMB_CHECK_LAUNCH();
}

void launch_helm_l2p(int nleaf, int p, double k, bool yuk, const int* keys, const int2* leaf, const float4* tpos,
                     const float* bbox, double w, const double* L, double* pot, cudaStream_t st) {
  if (nleaf <= 0) return;
  const int K = (p + 1) * (p + 1);
  const Corner c{bbox[0], bbox[1], bbox[2]};  // host array
  helm_l2p<<<nleaf, 128, 2 * K * sizeof(double), st>>>(p, K, k, yuk ? 1 : 0, keys, leaf, tpos, c, w, L,
                                                        (double2*)pot);
  FMMB_CHECK_LAUNCH();
}

void launch_helm_direct(int i0, int i1, const int* inv_i, const float4* tpos, int nj, const float4* spos,
                        const float* qs, double k, bool yuk, double eps2, bool excl, double* out, cudaStream_t st) {
  if (i1 <= i0) return;
  helm_direct<<<nb(i1 - i0, 128), 128, 0, st>>>(i0, i1, inv_i, tpos, nj, spos, (const float2*)qs, k, yuk ? 1 : 0,
                                                eps2, excl ? 1 : 0, (double2*)out);
  FMMB_CHECK_LAUNCH();
}

template <typename T>
void launch_helm_finalize(int n, const int* perm, const double* near, const double* far, T* out, cudaStream_t st) {
  if (n <= 0) return;
  helm_finalize<T><<<nb(n, 256), 256, 0, st>>>(n, perm, (const double2*)near, (const double2*)far, out);
  FMMB_CHECK_LAUNCH();
}
template void launch_helm_finalize<float>(int, const int*, const double*, const double*, float*, cudaStream_t);
template void launch_helm_finalize<double>(int, const int*, const double*, const double*, double*, cudaStream_t);

size_t helm_build_smem(int p) {
  const int NQ = 2 * p + 8, NP = 2 * NQ;
  return ((size_t)NQ * NP + (size_t)NQ * (2 * p + 1) + (p + 1)) * sizeof(double2);
}

void launch_helm_build_ops(int p, double k, bool yuk, int nops, const HelmOp* ops, const double* gl_x,
                           const double* gl_w, const double* ybar_q, double* opT, cudaStream_t st) {
  if (nops <= 0) return;
  const int K = (p + 1) * (p + 1), NQ = 2 * p + 8, NP = 2 * NQ;
  const size_t smem = helm_build_smem(p);
  FMMB_CUDA(cudaFuncSetAttribute(helm_build_ops, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const size_t ostride = (size_t)4 * K * K;
  for (int o0 = 0; o0 < nops; o0 += 65535) {
    dim3 grid(K, std::min(65535, nops - o0));
    helm_build_ops<<<grid, 256, smem, st>>>(p, K, k, yuk ? 1 : 0, ops + o0, NQ, NP, gl_x, gl_w, ybar_q,
                                            opT + (size_t)o0 * ostride, ostride);
    FMMB_CHECK_LAUNCH();
  }
}

}  // namespace fmmb

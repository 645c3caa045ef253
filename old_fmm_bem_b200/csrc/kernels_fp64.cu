// FP64 evaluation kernels: the plain-FP64 form of every FMM phase, and the
// P2M/M2M/L2L/L2P phases of the mixed-precision form (they are a few percent
// of the work, so they stay FP64 there too).
//
// Expansions are real-packed and scaled by the box size (operators.cpp).  P2M
// and L2P follow the reference's spherical formulation -- the same radius,
// angles, Legendre recurrences and Cartesian gradient conversion
// (kernel/multipole.cxx:7-35, kernel/multipoled.cxx:7-34,
// kernel/G_p2m.cxx:19-55, kernel/Gn_p2m.cxx:19-63, kernel/G_l2p.cxx:19-76,
// kernel/Gn_l2p.cxx:19-68) -- so that reference semantics can be reproduced
// to rounding.
#include <cuda_runtime.h>

#include <algorithm>

#include "internal.h"
#include "kernels.h"

namespace fmmb {

namespace {

inline int nblk(size_t n, int t) { return (int)((n + t - 1) / t); }

__device__ __forceinline__ double azimuth(double x, double y, const Sem& s) {
  if (!s.ref) return (x == 0.0 && y == 0.0) ? 0.0 : atan2(y, x);
  if (fabs(x) + fabs(y) < s.ang_eps) return 0.0;
  if (fabs(x) < s.ang_eps) return y / fabs(y) * s.pi_ang * 0.5;
  if (x > 0) return atan(y / x);
  return atan(y / x) + s.pi_ang;
}

// ---------------------------------------------------------------- charges
__global__ void gather_charges(int n, int nrhs, const int* perm, const float* q, float* qs) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int o = perm[i];
  for (int r = 0; r < nrhs; r++) qs[(size_t)r * n + i] = q[(size_t)r * n + o];
}

// ---------------------------------------------------------------- P2P (FP64)
// kernel/G_p2p.cxx:12-37, Gni_p2p.cxx:12-28, Gnj_p2p.cxx:12-28: one block per
// work item (up to 128 targets of a target leaf), its 27 neighbour slots
// staged through shared memory.
constexpr int kP2PThreads = 128;

template <int KER>
__global__ void __launch_bounds__(kP2PThreads) p2p_f64(const int2* __restrict__ work, const int2* __restrict__ leaf_i,
                                                       const int2* __restrict__ leaf_j,
                                                       const int* __restrict__ list, const float4* __restrict__ tpos,
                                                       const float4* __restrict__ tnrm, const float4* __restrict__ spos,
                                                       const float4* __restrict__ snrm, const float* __restrict__ qs,
                                                       Sem s, double* __restrict__ pot, double* __restrict__ grad,
                                                       int ni) {
  __shared__ float4 sp[kP2PThreads];
  __shared__ float4 sn[kP2PThreads];
  __shared__ float sq[kP2PThreads];
  const int2 wk = work[blockIdx.x];
  const int b = wk.x;
  int2 li = leaf_i[b];
  li.x += wk.y;
  li.y = min(kP2PThreads, li.y - wk.y);
  for (int t0 = 0; t0 < li.y; t0 += kP2PThreads) {
    const int i = li.x + t0 + threadIdx.x;
    const bool act = (t0 + threadIdx.x) < li.y;
    float4 xi = act ? tpos[i] : make_float4(0, 0, 0, 0);
    float4 ni4 = (KER == FMMB_LAPLACE_GNI && act) ? tnrm[i] : make_float4(0, 0, 0, 0);
    double p = 0, fx = 0, fy = 0, fz = 0;
    for (int slot = 0; slot < kP2PSlots; slot++) {
      const int jl = list[(size_t)b * kP2PSlots + slot];
      if (jl < 0) continue;
      const int2 lj = leaf_j[jl];
      for (int j0 = 0; j0 < lj.y; j0 += kP2PThreads) {
        const int nld = min(kP2PThreads, lj.y - j0);
        __syncthreads();
        if (threadIdx.x < nld) {
          const int j = lj.x + j0 + threadIdx.x;
          sp[threadIdx.x] = spos[j];
          sq[threadIdx.x] = qs[j];
          if (KER == FMMB_LAPLACE_GNJ) sn[threadIdx.x] = snrm[j];
        }
        __syncthreads();
        for (int jj = 0; jj < nld; jj++) {
          const float4 xj = sp[jj];
          double dx, dy, dz;
          if (s.ref) {  // float differences, as the reference (kernel/G_p2p.cxx:21-23)
            dx = (double)__fsub_rn(xi.x, xj.x);
            dy = (double)__fsub_rn(xi.y, xj.y);
            dz = (double)__fsub_rn(xi.z, xj.z);
          } else {
            dx = (double)xi.x - (double)xj.x;
            dy = (double)xi.y - (double)xj.y;
            dz = (double)xi.z - (double)xj.z;
          }
          if (s.excl_self && dx == 0.0 && dy == 0.0 && dz == 0.0) continue;
          const double r2 = dx * dx + dy * dy + dz * dz + s.eps2;
          const double rinv = 1.0 / sqrt(r2);
          const double qr = s.coef * (double)sq[jj] * rinv;
          if (KER == FMMB_LAPLACE_G) {
            const double qr3 = qr * rinv * rinv;
            p += qr;
            fx -= dx * qr3;
            fy -= dy * qr3;
            fz -= dz * qr3;
          } else {
            // Gni: n = the target's normal; Gnj: the source's.  With a gradient
            // (accurate semantics): d/dx_i of q (d.n) / r^3 = q n / r^3 - 3 q (d.n) d / r^5
            double nx, ny, nz;
            if (KER == FMMB_LAPLACE_GNI) {
              nx = ni4.x;
              ny = ni4.y;
              nz = ni4.z;
            } else {
              const float4 nj = sn[jj];
              nx = nj.x;
              ny = nj.y;
              nz = nj.z;
            }
            const double qr3 = qr * rinv * rinv, dot = dx * nx + dy * ny + dz * nz;
            p += dot * qr * rinv * rinv;  // the potential's operation order as without the gradient
            if (grad) {
              const double c = -3.0 * dot * qr3 * rinv * rinv;
              fx += qr3 * nx + c * dx;
              fy += qr3 * ny + c * dy;
              fz += qr3 * nz + c * dz;
            }
          }
        }
      }
    }
    if (act) {
      pot[i] = p;
      if (grad) {
        grad[i] = fx;
        grad[ni + i] = fy;
        grad[2 * ni + i] = fz;
      }
    }
  }
}

// ---------------------------------------------------------------- P2M
// One block per source leaf: 4 groups of 32 lanes, lane m owns the order-m
// coefficients; groups take every 4th point and are summed at the end.
template <int KER>
__global__ void __launch_bounds__(128) p2m_f64(int p, int K, const int* __restrict__ keys, const int2* __restrict__ leaf,
                                               const float4* __restrict__ spos, const float4* __restrict__ snrm,
                                               const float* __restrict__ qs, const double* __restrict__ fac, Sem s,
                                               float xmin, float ymin, float zmin, double rb, double* __restrict__ M) {
  extern __shared__ double acc[];  // [4][K]
  const int g = threadIdx.x >> 5, m = threadIdx.x & 31;
  for (int k = threadIdx.x; k < 4 * K; k += blockDim.x) acc[k] = 0.0;
  __syncthreads();
  const int b = blockIdx.x;
  int cx, cy, cz;
  {
    const int key = keys[b];
    cx = cy = cz = 0;
    for (int i = 0; i < 10; i++) {
      cy |= ((key >> (3 * i)) & 1) << i;
      cx |= ((key >> (3 * i + 1)) & 1) << i;
      cz |= ((key >> (3 * i + 2)) & 1) << i;
    }
  }
  const double xc = (double)xmin + (cx + 0.5) * rb, yc = (double)ymin + (cy + 0.5) * rb, zc = (double)zmin + (cz + 0.5) * rb;
  const int2 lf = leaf[b];
  double* my = acc + g * K;
  if (m <= p) {
    for (int jj = g; jj < lf.y; jj += 4) {
      const int j = lf.x + jj;
      const float4 xs = spos[j];
      const double x = (double)xs.x - xc, y = (double)xs.y - yc, z = (double)xs.z - zc;
      const double rh = sqrt(x * x + y * y + z * z) + s.rho_eps;
      const double al = rh == 0.0 ? 0.0 : acos(z / rh);
      const double be = azimuth(x, y, s);
      const double rs = rh / rb;  // radius in units of the leaf size
      const double xx = cos(al), s2 = sqrt((1 - xx) * (1 + xx));
      double pmm = 1.0;
      for (int i = 0; i < m; i++) pmm = -pmm * (2 * i + 1) * s2;
      double sb, cb;
      sincos(m * be, &sb, &cb);
      double rm1 = 1.0;  // rs^(m-1) for m >= 1
      for (int i = 1; i < m; i++) rm1 *= rs;
      const double rm = (m == 0) ? 1.0 : rm1 * rs;
      if (KER != FMMB_LAPLACE_GNJ) {
        // M^_n^m += q r^n fac P_n^m(cos al) e^{-i m be}
        const double q = (double)qs[j];
        double pv = pmm, p1 = pmm, p2 = 0.0;
        double rn = rm;
        for (int n = m; n <= p; n++) {
          if (n > m) {
            const double pn = (n == m + 1) ? xx * (2 * m + 1) * p1 : (xx * (2 * n - 1) * p1 - (n - 1 + m) * p2) / (n - m);
            p2 = p1;
            p1 = pn;
            pv = pn;
          }
          const double bnm = rn * fac[ifull_d(n, m)] * pv;
          if (m == 0) {
            my[n * n] += q * bnm;
          } else {
            my[n * n + 2 * m - 1] += q * bnm * cb;
            my[n * n + 2 * m] -= q * bnm * sb;
          }
          rn *= rs;
        }
      } else {
        // dipole: sum (q n) . grad R(x - c), in scaled form (1/rb) x the
        // reference's expression with the scaled radius (kernel/Gn_p2m.cxx:42-57)
        const float4 nv = snrm[j];
        const float qf = qs[j];
        const double qx = (double)(qf * nv.x), qy = (double)(qf * nv.y), qz = (double)(qf * nv.z);
        const double sa = sin(al), ca = cos(al), sbe = sin(be), cbe = cos(be);
        const double yy = sa;
        double p_n = pmm, p_np1 = xx * (2 * m + 1) * pmm;  // P_m^m, P_{m+1}^m
        double rn = rm, rn1 = (m == 0) ? 0.0 : rm1;        // rs^n, rs^(n-1)
        for (int n = m; n <= p; n++) {
          const double f = fac[ifull_d(n, m)];
          const double bnm = f * p_n;
          const double bth = (n == m) ? f * (p_np1 - (m + 1) * xx * p_n) / yy
                                      : f * ((n - m + 1) * p_np1 - (n + 1) * xx * p_n) / yy;
          // e = e^{-i m be} = (cb, -sb)
          const double brh_re = n * rn1 * bnm * cb, brh_im = -n * rn1 * bnm * sb;
          const double bal_re = rn * bth * cb, bal_im = -rn * bth * sb;
          // bbe = -m rn bnm e i = -m rn bnm (sb, cb)
          const double bbe_re = -m * rn * bnm * sb, bbe_im = -m * rn * bnm * cb;
          const double c1x = sa * cbe, c2x = ca * cbe / rs, c3x = sbe / rs / sa;
          const double c1y = sa * sbe, c2y = ca * sbe / rs, c3y = cbe / rs / sa;
          const double c1z = ca, c2z = sa / rs;
          const double bx_re = c1x * brh_re + c2x * bal_re - c3x * bbe_re;
          const double bx_im = c1x * brh_im + c2x * bal_im - c3x * bbe_im;
          const double by_re = c1y * brh_re + c2y * bal_re + c3y * bbe_re;
          const double by_im = c1y * brh_im + c2y * bal_im + c3y * bbe_im;
          const double bz_re = c1z * brh_re - c2z * bal_re;
          const double bz_im = c1z * brh_im - c2z * bal_im;
          const double vre = (qx * bx_re + qy * by_re + qz * bz_re) / rb;
          const double vim = (qx * bx_im + qy * by_im + qz * bz_im) / rb;
          if (m == 0) {
            my[n * n] += vre;
          } else {
            my[n * n + 2 * m - 1] += vre;
            my[n * n + 2 * m] += vim;
          }
          // advance the Legendre recurrence (kernel/multipoled.cxx:23-30)
          const double pn2 = (xx * (2 * (n + 1) + 1) * p_np1 - (n + 1 + m) * p_n) / (n + 1 - m + 1);
          p_n = p_np1;
          p_np1 = pn2;
          rn1 = rn;
          rn *= rs;
        }
      }
    }
  }
  __syncthreads();
  for (int k = threadIdx.x; k < K; k += blockDim.x) M[(size_t)b * K + k] = acc[k] + acc[K + k] + acc[2 * K + k] + acc[3 * K + k];
}

// ---------------------------------------------------------------- translations (FP64)
// One kernel for the three box-to-box translations (M2L, M2M, L2L): a block
// owns a tile of up to 32 output boxes and walks `nslots` slots; slot s of
// output box b reads input box list[b*nslots + s] (an index into `in`, or
// -1) through operator tile_ops[tile*nslots + s] (-1: no box of the tile uses
// the slot).  Per slot the K x K operator is streamed through shared memory
// in column panels and applied to the tile's gathered inputs -- a batched
// K x K x 32 DGEMM whose operator is shared by the whole tile.  grid.y
// splits the slots when there are few tiles; the shares are then added with
// FP64 atomics.
//   M2L: tiles of target boxes of one octant, 189 interaction slots
//        (kernel/m2l.cxx:30-83);
//   M2M: tiles of parent boxes, 8 child slots (kernel/m2m.cxx:28-62);
//   L2L: tiles of child boxes of one octant, 1 parent slot (kernel/l2l.cxx:44-78).
constexpr int kXTile = 32;    // output boxes per block
constexpr int kXPanel = 16;   // operator columns per shared-memory panel
constexpr int kXThreads = 256;

__global__ void __launch_bounds__(kXThreads) translate_f64(int K, int nslots, const int* __restrict__ tile_boxes,
                                                           const int* __restrict__ tile_ops, const int* __restrict__ list,
                                                           const double* __restrict__ ops, const double* __restrict__ in,
                                                           double* __restrict__ out) {
  constexpr int RPT = 8;  // rows per thread: ty + 16*r covers 128 rows
  __shared__ double sT[kXPanel][128 + 1];
  __shared__ double sB[kXPanel][kXTile + 1];
  __shared__ int sSrc[kXTile];
  __shared__ int sBox[kXTile];
  const int tile = blockIdx.x;
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;  // 16 x 16 threads
  if (threadIdx.x < kXTile) sBox[threadIdx.x] = tile_boxes[tile * kXTile + threadIdx.x];
  __syncthreads();
  const int s0 = (blockIdx.y * nslots) / gridDim.y, s1 = ((blockIdx.y + 1) * nslots) / gridDim.y;
  for (int rb0 = 0; rb0 < K; rb0 += 128) {
    double acc[RPT][2];
#pragma unroll
    for (int r = 0; r < RPT; r++) acc[r][0] = acc[r][1] = 0.0;
    for (int slot = s0; slot < s1; slot++) {
      const int op = tile_ops[(size_t)tile * nslots + slot];
      if (op < 0) continue;
      __syncthreads();
      if (threadIdx.x < kXTile) {
        const int box = sBox[threadIdx.x];
        sSrc[threadIdx.x] = box >= 0 ? list[(size_t)box * nslots + slot] : -1;
      }
      const double* T = ops + (size_t)op * K * K;
      for (int k0 = 0; k0 < K; k0 += kXPanel) {
        __syncthreads();
        for (int e = threadIdx.x; e < kXPanel * 128; e += kXThreads) {
          const int row = e / kXPanel, kk = e % kXPanel;
          const int gr = rb0 + row, gk = k0 + kk;
          sT[kk][row] = (gr < K && gk < K) ? T[(size_t)gr * K + gk] : 0.0;
        }
        for (int e = threadIdx.x; e < kXPanel * kXTile; e += kXThreads) {
          const int t = e / kXPanel, kk = e % kXPanel;
          const int src = sSrc[t], gk = k0 + kk;
          sB[kk][t] = (src >= 0 && gk < K) ? in[(size_t)src * K + gk] : 0.0;
        }
        __syncthreads();
#pragma unroll 4
        for (int kk = 0; kk < kXPanel; kk++) {
          const double b0 = sB[kk][tx], b1 = sB[kk][tx + 16];
#pragma unroll
          for (int r = 0; r < RPT; r++) {
            const double a = sT[kk][ty + 16 * r];
            acc[r][0] += a * b0;
            acc[r][1] += a * b1;
          }
        }
      }
    }
#pragma unroll
    for (int r = 0; r < RPT; r++) {
      const int row = rb0 + ty + 16 * r;
      if (row < K) {
        const int b0 = sBox[tx], b1 = sBox[tx + 16];
        if (gridDim.y > 1) {
          if (b0 >= 0) atomicAdd(&out[(size_t)b0 * K + row], acc[r][0]);
          if (b1 >= 0) atomicAdd(&out[(size_t)b1 * K + row], acc[r][1]);
        } else {
          if (b0 >= 0) out[(size_t)b0 * K + row] += acc[r][0];
          if (b1 >= 0) out[(size_t)b1 * K + row] += acc[r][1];
        }
      }
    }
  }
}

// ---------------------------------------------------------------- L2P
constexpr int kL2PThreads = 64;

template <int KER>
__global__ void __launch_bounds__(kL2PThreads) l2p_f64(int p, int K, const int* __restrict__ keys, const int2* __restrict__ leaf,
                                                       const float4* __restrict__ tpos, const float4* __restrict__ tnrm,
                                                       const double* __restrict__ fac, Sem s, float xmin, float ymin,
                                                       float zmin, double rb, const double* __restrict__ L,
                                                       double* __restrict__ pot, double* __restrict__ grad, int ni) {
  extern __shared__ double sl[];
  const int b = blockIdx.x;
  for (int k = threadIdx.x; k < K; k += blockDim.x) sl[k] = L[(size_t)b * K + k];
  __syncthreads();
  int cx = 0, cy = 0, cz = 0;
  {
    const int key = keys[b];
    for (int i = 0; i < 10; i++) {
      cy |= ((key >> (3 * i)) & 1) << i;
      cx |= ((key >> (3 * i + 1)) & 1) << i;
      cz |= ((key >> (3 * i + 2)) & 1) << i;
    }
  }
  const double xc = (double)xmin + (cx + 0.5) * rb, yc = (double)ymin + (cy + 0.5) * rb, zc = (double)zmin + (cz + 0.5) * rb;
  const int2 lf = leaf[b];
  for (int ii = threadIdx.x; ii < lf.y; ii += blockDim.x) {
    const int i = lf.x + ii;
    const float4 xt = tpos[i];
    const double x = (double)xt.x - xc, y = (double)xt.y - yc, z = (double)xt.z - zc;
    const double r = sqrt(x * x + y * y + z * z) + s.rho_eps;
    const double th = r == 0.0 ? 0.0 : acos(z / r);
    const double ph = azimuth(x, y, s);
    const double rs = r / rb;
    const double xx = cos(th), yy = sin(th), s2 = sqrt((1 - xx) * (1 + xx));
    double g = 0, gr = 0, gth = 0, gph = 0;
    double pmm = 1.0, fact = 1.0, rm = 1.0, rm1 = 0.0;  // P_m^m, (2m+1), rs^m, rs^(m-1)
    for (int m = 0; m <= p; m++) {
      double sm, cm;
      sincos(m * ph, &sm, &cm);
      double p_n = pmm, p_np1 = xx * (2 * m + 1) * pmm;
      double rn = rm, rn1 = rm1;
      for (int n = m; n <= p; n++) {
        const double f = fac[ifull_d(n, m)];
        const double bnm = f * p_n;
        const double bth = (n == m) ? f * (p_np1 - (m + 1) * xx * p_n) / yy
                                    : f * ((n - m + 1) * p_np1 - (n + 1) * xx * p_n) / yy;
        if (m == 0) {
          const double a = sl[n * n];
          g += rn * bnm * a;
          gr += n * rn1 * bnm * a;
          gth += rn * bth * a;
        } else {
          const double are = sl[n * n + 2 * m - 1], aim = sl[n * n + 2 * m];
          const double re = cm * are - sm * aim;  // Re(e^{i m ph} L)
          const double im = sm * are + cm * aim;  // Im(e^{i m ph} L)
          g += 2 * rn * bnm * re;
          gr += 2 * n * rn1 * bnm * re;
          gth += 2 * rn * bth * re;
          gph += -2 * m * rn * bnm * im;
        }
        const double pn2 = (xx * (2 * (n + 1) + 1) * p_np1 - (n + 1 + m) * p_n) / (n + 1 - m + 1);
        p_n = p_np1;
        p_np1 = pn2;
        rn1 = rn;
        rn *= rs;
      }
      pmm = -pmm * fact * s2;
      fact += 2;
      rm1 = rm;
      rm *= rs;
    }
    const double st = sin(th), ct = cos(th), sp = sin(ph), cp = cos(ph);
    const double ex = st * cp * gr + ct * cp / rs * gth - sp / rs / st * gph;
    const double ey = st * sp * gr + ct * sp / rs * gth + cp / rs / st * gph;
    const double ez = ct * gr - st / rs * gth;
    const double c1 = s.coef / rb, c2 = s.coef / (rb * rb);
    if (KER == FMMB_LAPLACE_GNI) {
      const float4 nv = tnrm[i];
      pot[i] = -c2 * ((double)nv.x * ex + (double)nv.y * ey + (double)nv.z * ez);
    } else {
      pot[i] = c1 * g;
      if (KER == FMMB_LAPLACE_G && grad) {
        grad[i] = c2 * ex;
        grad[ni + i] = c2 * ey;
        grad[2 * ni + i] = c2 * ez;
      }
    }
  }
}

// ---------------------------------------------------------------- outputs
template <typename T>
__global__ void finalize(int n, const int* perm, const double* pn, const double* pf, const double* gn, const double* gf,
                         T* pot, T* grad) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int o = perm[i];
  pot[o] = (T)(pn[i] + pf[i]);
  if (grad) {
    grad[o] = (T)(gn[i] + gf[i]);
    grad[n + o] = (T)(gn[n + i] + gf[n + i]);
    grad[2 * n + o] = (T)(gn[2 * n + i] + gf[2 * n + i]);
  }
}

// ---------------------------------------------------------------- direct
template <int KER>
__global__ void __launch_bounds__(128) direct_f64(int i0, int i1, const int* __restrict__ inv_i, const float4* __restrict__ tpos,
                                                  const float4* __restrict__ tnrm, int nj, const float4* __restrict__ spos,
                                                  const float4* __restrict__ snrm, const float* __restrict__ qs, Sem s,
                                                  double* __restrict__ pot, double* __restrict__ grad) {
  __shared__ float4 sp[128], sn[128];
  __shared__ float sq[128];
  const int i = i0 + blockIdx.x * blockDim.x + threadIdx.x;
  const bool act = i < i1;
  const int si = act ? inv_i[i] : 0;
  const float4 xi = tpos[si];
  const float4 nv = tnrm[si];
  double p = 0, fx = 0, fy = 0, fz = 0;
  for (int j0 = 0; j0 < nj; j0 += 128) {
    __syncthreads();
    if (j0 + threadIdx.x < nj) {
      sp[threadIdx.x] = spos[j0 + threadIdx.x];
      sn[threadIdx.x] = snrm[j0 + threadIdx.x];
      sq[threadIdx.x] = qs[j0 + threadIdx.x];
    }
    __syncthreads();
    const int nl = min(128, nj - j0);
    for (int jj = 0; jj < nl; jj++) {
      const float4 xj = sp[jj];
      double dx, dy, dz;
      if (s.ref) {
        dx = (double)__fsub_rn(xi.x, xj.x);
        dy = (double)__fsub_rn(xi.y, xj.y);
        dz = (double)__fsub_rn(xi.z, xj.z);
      } else {
        dx = (double)xi.x - (double)xj.x;
        dy = (double)xi.y - (double)xj.y;
        dz = (double)xi.z - (double)xj.z;
      }
      if (s.excl_self && dx == 0.0 && dy == 0.0 && dz == 0.0) continue;
      const double r2 = dx * dx + dy * dy + dz * dz + s.eps2;
      const double rinv = 1.0 / sqrt(r2);
      const double qr = s.coef * (double)sq[jj] * rinv;
      if (KER == FMMB_LAPLACE_G) {
        p += qr;
        const double qr3 = qr * rinv * rinv;
        fx -= dx * qr3;
        fy -= dy * qr3;
        fz -= dz * qr3;
      } else {
        // Gni: the target's normal, Gnj: the source's; gradient w.r.t. the
        // target position with the normal fixed: q n / r^3 - 3 q (d.n) d / r^5
        double nx = nv.x, ny = nv.y, nz = nv.z;
        if (KER == FMMB_LAPLACE_GNJ) {
          const float4 nj4 = sn[jj];
          nx = nj4.x;
          ny = nj4.y;
          nz = nj4.z;
        }
        const double qr3 = qr * rinv * rinv, dot = dx * nx + dy * ny + dz * nz;
        p += dot * qr * rinv * rinv;  // the potential's operation order as without the gradient
        const double c = -3.0 * dot * qr3 * rinv * rinv;
        fx += qr3 * nx + c * dx;
        fy += qr3 * ny + c * dy;
        fz += qr3 * nz + c * dz;
      }
    }
  }
  if (act) {
    pot[i - i0] = p;
    if (grad) {
      const int m = i1 - i0;
      grad[i - i0] = fx;
      grad[m + i - i0] = fy;
      grad[2 * m + i - i0] = fz;
    }
  }
}

}  // namespace

// ---------------------------------------------------------------- launchers
void launch_gather_charges(int n, int nrhs, const int* perm, const float* q, float* qs, cudaStream_t st) {
  gather_charges<<<nblk(n, 256), 256, 0, st>>>(n, nrhs, perm, q, qs);
  FMMB_CHECK_LAUNCH();
}

void launch_p2p_f64(int kernel, int nwork, const int2* work, const int2* leaf_i, const int2* leaf_j, const int* list,
                    const float4* tpos, const float4* tnrm, const float4* spos, const float4* snrm, const float* qs,
                    const Sem& s, double* pot, double* grad, int ni, cudaStream_t st) {
  if (nwork <= 0) return;
  if (kernel == FMMB_LAPLACE_G)
    p2p_f64<FMMB_LAPLACE_G><<<nwork, kP2PThreads, 0, st>>>(work, leaf_i, leaf_j, list, tpos, tnrm, spos, snrm, qs, s,
                                                           pot, grad, ni);
  else if (kernel == FMMB_LAPLACE_GNI)
    p2p_f64<FMMB_LAPLACE_GNI><<<nwork, kP2PThreads, 0, st>>>(work, leaf_i, leaf_j, list, tpos, tnrm, spos, snrm, qs, s,
                                                             pot, grad, ni);
  else
    p2p_f64<FMMB_LAPLACE_GNJ><<<nwork, kP2PThreads, 0, st>>>(work, leaf_i, leaf_j, list, tpos, tnrm, spos, snrm, qs, s,
                                                             pot, grad, ni);
  FMMB_CHECK_LAUNCH();
}

void launch_p2m(int kernel, int nleaf, int p, int K, const int* keys, const int2* leaf, const float4* spos, const float4* snrm,
                const float* qs, const double* fac, const Sem& s, const float* bbox, double rb, double* M, cudaStream_t st) {
  if (nleaf <= 0) return;
  const size_t sm = 4 * (size_t)K * sizeof(double);
  if (kernel == FMMB_LAPLACE_GNJ)
    p2m_f64<FMMB_LAPLACE_GNJ><<<nleaf, 128, sm, st>>>(p, K, keys, leaf, spos, snrm, qs, fac, s, bbox[0], bbox[1], bbox[2], rb, M);
  else
    p2m_f64<FMMB_LAPLACE_G><<<nleaf, 128, sm, st>>>(p, K, keys, leaf, spos, snrm, qs, fac, s, bbox[0], bbox[1], bbox[2], rb, M);
  FMMB_CHECK_LAUNCH();
}

int translate_tile_size() { return kXTile; }

void launch_translate_f64(int ntile, int nsplit, int K, int nslots, const int* tile_boxes, const int* tile_ops,
                          const int* list, const double* ops, const double* in, double* out, cudaStream_t st) {
  if (ntile <= 0) return;
  translate_f64<<<dim3(ntile, std::max(1, nsplit)), kXThreads, 0, st>>>(K, nslots, tile_boxes, tile_ops, list, ops, in, out);
  FMMB_CHECK_LAUNCH();
}

void launch_l2p(int kernel, int nleaf, int p, int K, const int* keys, const int2* leaf, const float4* tpos, const float4* tnrm,
                const double* fac, const Sem& s, const float* bbox, double rb, const double* L, double* pot, double* grad,
                int ni, cudaStream_t st) {
  if (nleaf <= 0) return;
  const size_t sm = (size_t)K * sizeof(double);
  if (kernel == FMMB_LAPLACE_G)
    l2p_f64<FMMB_LAPLACE_G><<<nleaf, kL2PThreads, sm, st>>>(p, K, keys, leaf, tpos, tnrm, fac, s, bbox[0], bbox[1], bbox[2], rb, L, pot, grad, ni);
  else if (kernel == FMMB_LAPLACE_GNI)
    l2p_f64<FMMB_LAPLACE_GNI><<<nleaf, kL2PThreads, sm, st>>>(p, K, keys, leaf, tpos, tnrm, fac, s, bbox[0], bbox[1], bbox[2], rb, L, pot, grad, ni);
  else
    l2p_f64<FMMB_LAPLACE_GNJ><<<nleaf, kL2PThreads, sm, st>>>(p, K, keys, leaf, tpos, tnrm, fac, s, bbox[0], bbox[1], bbox[2], rb, L, pot, grad, ni);
  FMMB_CHECK_LAUNCH();
}

void launch_finalize_f32(int n, const int* perm, const double* pn, const double* pf, const double* gn, const double* gf, float* pot,
                         float* grad, cudaStream_t st) {
  finalize<float><<<nblk(n, 256), 256, 0, st>>>(n, perm, pn, pf, gn, gf, pot, grad);
  FMMB_CHECK_LAUNCH();
}
void launch_finalize_f64(int n, const int* perm, const double* pn, const double* pf, const double* gn, const double* gf, double* pot,
                         double* grad, cudaStream_t st) {
  finalize<double><<<nblk(n, 256), 256, 0, st>>>(n, perm, pn, pf, gn, gf, pot, grad);
  FMMB_CHECK_LAUNCH();
}

namespace {

// Box-pair translations (M2M, L2L, and every dense translation of the
// Helmholtz-family kernels) in FP64 on the FP64 tensor cores: a tile holds up
// to 32 pairs sharing one operator T, and
//   out[dst[p]][r] (+)= sum_c T[r][c] in[src[p]][c]
// added atomically when an output row receives several pairs (M2M, M2L) and
// also for L2L, although each of its output rows receives one pair: the
// single atomic addition gives the value of a read-modify-write without the
// warp waiting for the read.
constexpr int kGN = 32;  // pairs per tile (at most)

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src, int bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(bytes) : "memory");
}

__device__ __forceinline__ void cp_async8(uint32_t dst, const void* src, int bytes) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(dst), "l"(src), "r"(bytes) : "memory");
}

// Grouped GEMM on the FP64 tensor cores (mma.sync m8n8k4 .f64, 256 FMA per
// warp instruction): a block of 8 warps computes 128 output rows x the
// tile's 32 pairs, warp w rows 32 (w % 4) .. + 31 x pairs 16 (w / 4) .. + 15
// (4 x 2 MMA tiles of 8 x 8, 16 FP64 accumulators per thread).  Operator
// chunks of 8 columns and the inputs go through a 4-stage cp.async ring (43 KB:
// three blocks per SM; 16-column chunks with one block fewer ran 10 % slower);
// the shared-memory rows are padded (132 and 36 doubles) so that the
// fragment reads of the four k-rows of an MMA fall in different banks.
constexpr int kDM = 128, kDN = 32, kDK = 8, kDT = 256, kDS = 4;
constexpr int kDAs = kDM + 4;  // operator chunk row stride (doubles)
constexpr int kDXs = kDN + 4;  // input chunk row stride
constexpr size_t kDSmem = kDS * (size_t)kDK * (kDAs + kDXs) * sizeof(double);  // 43 KB: 3 blocks per SM

__device__ __forceinline__ void dmma884(double (&c)[2], double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
               : "+d"(c[0]), "+d"(c[1])
               : "d"(a), "d"(b));
}

__global__ void __launch_bounds__(kDT) pairs_dmma_f64(PairArgs P) {
  extern __shared__ __align__(16) double dsm2[];
  double* As = dsm2;                     // [kDS][kDK][kDAs]: operator T[r][c] at [c][r]
  double* Xs = dsm2 + kDS * kDK * kDAs;  // [kDS][kDK][kDXs]: inputs x_p[c] at [c][p]
  __shared__ int ssrc[kDN], sdst[kDN];
  const int g = blockIdx.x, r0 = blockIdx.y * kDM, K = P.K, KP = (K + 1) & ~1, tp = P.tp;
  const double* T = P.opT + (size_t)P.tile_op[g] * P.ostride;
  if (threadIdx.x < kDN) {
    const bool on = (int)threadIdx.x < tp;
    ssrc[threadIdx.x] = on ? P.tile_src[(size_t)g * tp + threadIdx.x] : -1;
    sdst[threadIdx.x] = on ? P.tile_dst[(size_t)g * tp + threadIdx.x] : -1;
  }
  __syncthreads();
  auto issue = [&](int kc, int st) {
    const int k0 = kc * kDK;
#pragma unroll
    for (int i = 0; i < kDK * kDM / 2 / kDT; i++) {  // operator: 16-byte pieces of 2 rows
      const int e = (int)threadIdx.x + i * kDT;
      const int c = e / (kDM / 2), rr = 2 * (e % (kDM / 2));
      const int col = k0 + c, row = r0 + rr;
      const bool ok = col < K && row < KP;
      cp_async16(smem_addr(As + (st * kDK + c) * kDAs + rr), ok ? T + (size_t)col * KP + row : T, ok ? 16 : 0);
    }
#pragma unroll
    for (int i = 0; i < kDK * kDN / kDT; i++) {  // inputs: 8 bytes each, a pair's kDK columns from adjacent lanes
      const int e = (int)threadIdx.x + i * kDT;
      const int pi = e / kDK, c = e % kDK;
      const int sj = ssrc[pi], col = k0 + c;
      const bool ok = sj >= 0 && col < K;
      cp_async8(smem_addr(Xs + (st * kDK + c) * kDXs + pi), ok ? P.xin + (size_t)sj * K + col : P.xin, ok ? 8 : 0);
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
  };
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int gq = lane >> 2, tq = lane & 3;             // MMA fragment coordinates
  const int wr = 32 * (warp & 3), wp = 16 * (warp >> 2);  // the warp's rows and pairs in the block
  double acc[4][2][2];
#pragma unroll
  for (int i = 0; i < 4; i++)
#pragma unroll
    for (int j = 0; j < 2; j++) acc[i][j][0] = acc[i][j][1] = 0.0;
  // this block's column chunks [kc0, kc1): blockIdx.z of gridDim.z parts of
  // the columns (the parts' sums are added atomically)
  const int nk = (K + kDK - 1) / kDK;
  const int kc0 = (int)(blockIdx.z * (unsigned)nk / gridDim.z), kc1 = (int)((blockIdx.z + 1) * (unsigned)nk / gridDim.z);
  const int nkb = kc1 - kc0;
#pragma unroll
  for (int st = 0; st < kDS - 1; st++) {
    if (st < nkb)
      issue(kc0 + st, st);
    else
      asm volatile("cp.async.commit_group;" ::: "memory");
  }
  for (int kb = 0; kb < nkb; kb++) {
    if (kb + kDS - 1 < nkb)
      issue(kc0 + kb + kDS - 1, (kb + kDS - 1) % kDS);
    else
      asm volatile("cp.async.commit_group;" ::: "memory");
    asm volatile("cp.async.wait_group %0;" ::"n"(kDS - 1) : "memory");
    __syncthreads();
    const double* a = As + (kb % kDS) * kDK * kDAs + wr + gq;
    const double* x = Xs + (kb % kDS) * kDK * kDXs + wp + gq;
#pragma unroll
    for (int k4 = 0; k4 < kDK; k4 += 4) {
      const int kr = k4 + tq;  // the k-row of this lane's A column / B row
      double af[4], bf[2];
#pragma unroll
      for (int i = 0; i < 4; i++) af[i] = a[kr * kDAs + 8 * i];
#pragma unroll
      for (int j = 0; j < 2; j++) bf[j] = x[kr * kDXs + 8 * j];
#pragma unroll
      for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 2; j++) dmma884(acc[i][j], af[i], bf[j]);
    }
    __syncthreads();  // the stage is refilled by the next iteration's copies
  }
  // accumulator (i, j): rows wr + 8 i + gq, pairs wp + 8 j + 2 tq + {0, 1}
#pragma unroll
  for (int j = 0; j < 2; j++)
#pragma unroll
    for (int h = 0; h < 2; h++) {
      const int d = sdst[wp + 8 * j + 2 * tq + h];
      if (d < 0) continue;
#pragma unroll
      for (int i = 0; i < 4; i++) {
        const int r = r0 + wr + 8 * i + gq;
        if (r >= K) continue;
        double* o = P.out + (size_t)d * K + r;
        if (P.atomic || gridDim.z > 1)
          atomicAdd(o, acc[i][j][h]);
        else
          *o += acc[i][j][h];
      }
    }
}
}  // namespace

// One operator's tiles of up to 32 pairs (the tensor-core kernel's block
// width); a tile of fewer pairs leaves the rest of the block's columns idle.
int pairs_f64_tile(int, int, int) { return kGN; }

void prepare_translate_pairs_f64() {
  FMMB_CUDA(cudaFuncSetAttribute(pairs_dmma_f64, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kDSmem));
}

void launch_translate_pairs_f64(const PairArgs& a, cudaStream_t st) {
  if (a.ntile <= 0) return;
  FMMB_REQUIRE(a.tp >= 1 && a.tp <= kGN, FMMB_ERR_ARG, "pair tile larger than 32");
  // the columns split into parts (added atomically) when the tiles alone give
  // fewer than four blocks per SM: the small levels' launches are one block's
  // chain of column chunks long, so a part of the chain per block shortens them
  // (a target of 2 or 8 blocks per SM ran the surface matvec 2 % / 1 % slower)
  const int nrb = (a.K + kDM - 1) / kDM, nk = (a.K + kDK - 1) / kDK;
  int kz = 1;
  if (a.atomic) {
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    const long long blocks = (long long)a.ntile * nrb;
    while (kz < 8 && 2 * kz <= nk && blocks * kz < 4LL * nsm) kz *= 2;
  }
  const dim3 grid((unsigned)a.ntile, (unsigned)nrb, (unsigned)kz);
  pairs_dmma_f64<<<grid, kDT, kDSmem, st>>>(a);
  FMMB_CHECK_LAUNCH();
}

namespace {
template <typename T>
__global__ void scale_kernel(T* p, size_t n, T s) {
  const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i < n) p[i] *= s;
}
__global__ void weight_field_kernel(int n, const float* __restrict__ w, const double* __restrict__ f,
                                    double* __restrict__ out) {
  const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i < 3 * (size_t)n) out[i] = (double)w[i % n] * f[i];
}
}  // namespace

void launch_scale(float* p, size_t n, float s, cudaStream_t st) {
  if (n == 0) return;
  scale_kernel<float><<<(unsigned)((n + 255) / 256), 256, 0, st>>>(p, n, s);
  FMMB_CHECK_LAUNCH();
}
void launch_scale(double* p, size_t n, double s, cudaStream_t st) {
  if (n == 0) return;
  scale_kernel<double><<<(unsigned)((n + 255) / 256), 256, 0, st>>>(p, n, s);
  FMMB_CHECK_LAUNCH();
}
void launch_weight_field(int n, const float* w, const double* field, double* out, cudaStream_t st) {
  if (n <= 0) return;
  const size_t t = 3 * (size_t)n;
  weight_field_kernel<<<(unsigned)((t + 255) / 256), 256, 0, st>>>(n, w, field, out);
  FMMB_CHECK_LAUNCH();
}

void launch_direct_f64(int kernel, int i0, int i1, const int* inv_i, const float4* tpos, const float4* tnrm, int nj,
                       const float4* spos, const float4* snrm, const float* qs, const Sem& s, double* pot, double* grad,
                       cudaStream_t st) {
  const int m = i1 - i0;
  if (m <= 0) return;
  if (kernel == FMMB_LAPLACE_G)
    direct_f64<FMMB_LAPLACE_G><<<nblk(m, 128), 128, 0, st>>>(i0, i1, inv_i, tpos, tnrm, nj, spos, snrm, qs, s, pot, grad);
  else if (kernel == FMMB_LAPLACE_GNI)
    direct_f64<FMMB_LAPLACE_GNI><<<nblk(m, 128), 128, 0, st>>>(i0, i1, inv_i, tpos, tnrm, nj, spos, snrm, qs, s, pot, grad);
  else
    direct_f64<FMMB_LAPLACE_GNJ><<<nblk(m, 128), 128, 0, st>>>(i0, i1, inv_i, tpos, tnrm, nj, spos, snrm, qs, s, pot, grad);
  FMMB_CHECK_LAUNCH();
}

}  // namespace fmmb

// Translation operators of the FMM, built once per plan on the host in FP64.
//
// The reference applies M2M, M2L and L2L as three steps per box pair:
// rotate the expansion so the translation vector lies on the z axis
// (kernel/spharot.cxx:3-24 with the Wigner tables of kernel/precalc.cxx:78-203),
// translate along z (kernel/m2m.cxx:43-57, kernel/m2l.cxx:56-77,
// kernel/l2l.cxx:59-73), rotate back.  All three steps are linear, so here they
// are composed once per relative position into a dense real matrix that the GPU
// applies as a batched contraction.
//
// Representation.  An expansion of order p holds complex coefficients E_n^m,
// 0 <= m <= n <= p, with E_n^{-m} = conj(E_n^m) implied (the convention of
// kernel/spharot.cxx).  The GPU stores it "real-packed" as K = (p+1)^2 reals:
// for each degree n, [Re E_n^0, Re E_n^1, Im E_n^1, ..., Re E_n^n, Im E_n^n]
// (Im E_n^0 is zero for real charges and is not stored).
//
// Scaling.  Expansions are stored scaled by the box size rb of their level:
// multipoles M^_n = M_n / rb^n, locals L^_n = L_n * rb^(n+1).  With that, M2M
// and L2L are the same matrices on every level and M2L depends only on the
// relative position in box units -- except in reference semantics, where the
// reference adds eps=1e-6 to the M2L distance in absolute units
// (kernel/m2l.cxx:54), so one M2L set per level is built.
#include <cuda_fp16.h>
#include <cmath>
#include <complex>
#include <cstring>
#include <thread>
#include <vector>

#include "internal.h"

namespace fmmb {
namespace {

typedef std::complex<double> cd;
const double kPiF = (double)(float)M_PI;
const double kEpsF = (double)1e-6f;

inline double to_ref_float(double v, bool ref) { return ref ? (double)(float)v : v; }

double factorial(int n) {
  double f = 1;
  for (int i = 1; i <= n; i++) f *= i;
  return f;
}

// Morton decode/encode with the reference's bit order (fmm/boxc.cxx:3-24,
// fmm/boxn1.cxx:3-19): x on bit 3i+1, y on bit 3i, z on bit 3i+2.
void decode3(int key, int c[3]) {
  c[0] = c[1] = c[2] = 0;
  for (int i = 0; i < 10; i++) {
    c[1] |= ((key >> (3 * i)) & 1) << i;
    c[0] |= ((key >> (3 * i + 1)) & 1) << i;
    c[2] |= ((key >> (3 * i + 2)) & 1) << i;
  }
}
int encode3(const int c[3], int lev) {
  int k = 0;
  for (int i = 0; i < lev; i++)
    k |= (((c[0] >> i) & 1) << (3 * i + 1)) | (((c[1] >> i) & 1) << (3 * i)) | (((c[2] >> i) & 1) << (3 * i + 2));
  return k;
}

double azimuth(double x, double y, bool ref) {
  if (!ref) return (x == 0 && y == 0) ? 0.0 : std::atan2(y, x);
  if (std::abs(x) + std::abs(y) < kEpsF) return 0;
  if (std::abs(x) < kEpsF) return y / std::abs(y) * kPiF * 0.5;
  if (x > 0) return std::atan(y / x);
  return std::atan(y / x) + kPiF;
}

// Wigner rotation table for one direction: W[n][m*(2n+1) + k+n] for
// 0 <= m <= n, -n <= k <= n, equal to s_k d^n_{k m}(al) e^{i(m+k) be} with
// s_k = (-1)^k for k < 0 (the tables of kernel/precalc.cxx:100-146, built by
// the same recurrence in k then m).  A rotation by pi, where the recurrence
// divides 0/0, uses its closed form (-1)^n [k == -m].
void wigner(double al, double be, int p, std::vector<std::vector<cd>>& W) {
  W.assign(p + 1, {});
  const bool flip = (1 + std::cos(al)) == 0;
  const double sc = std::sin(al) / (1 + std::cos(al));
  std::vector<double> d;
  for (int n = 0; n <= p; n++) {
    const int w = 2 * n + 1;
    W[n].assign((size_t)(n + 1) * w, cd(0, 0));
    if (flip) {
      for (int m = 0; m <= n; m++) W[n][m * w + (-m + n)] = std::pow(-1.0, n) * std::exp(cd(0, 0 * be));
      continue;
    }
    d.assign((size_t)w * w, 0.0);
    auto D = [&](int m, int k) -> double& { return d[(size_t)(m + n) * w + (k + n)]; };
    D(n, n) = std::pow(std::cos(0.5 * al), 2 * n);
    for (int k = n; k >= 1 - n; k--) D(n, k - 1) = std::sqrt(((double)n + k) / (n - k + 1)) * std::tan(0.5 * al) * D(n, k);
    for (int m = n; m >= 1; m--)
      for (int k = m - 1; k >= 1 - m; k--) {
        const double den = n * (n + 1) - m * (m - 1);
        D(m - 1, k) = std::sqrt((n * (n + 1) - k * (k + 1)) / den) * D(m, k + 1) - (m + k) / std::sqrt(den) * sc * D(m, k);
      }
    for (int m = 0; m <= n && n >= 1; m++) {
      for (int k = -m; k <= -1; k++) {
        D(m, k) *= std::pow(-1.0, k);
        D(-k, -m) = std::pow(-1.0, m + k) * D(m, k);
      }
      for (int k = 0; k <= m; k++) {
        D(k, m) = std::pow(-1.0, m + k) * D(m, k);
        D(-k, -m) = D(k, m);
      }
    }
    for (int m = 0; m <= n; m++)
      for (int k = -n; k <= n; k++) W[n][m * w + (k + n)] = D(m, k) * std::exp(cd(0, (k + m) * be));
  }
}

// Rotation of one degree (kernel/spharot.cxx:7-23): out[m] = sum_{k<0}
// W[m][k] conj(in[-k]) + sum_{k>=0} W[m][k] in[k].
void rotate_degree(const std::vector<cd>& Wn, int n, const cd* in, cd* out) {
  const int w = 2 * n + 1;
  for (int m = 0; m <= n; m++) {
    cd acc = 0;
    for (int k = -n; k <= -1; k++) acc += Wn[m * w + k + n] * std::conj(in[-k]);
    for (int k = 0; k <= n; k++) acc += Wn[m * w + k + n] * in[k];
    out[m] = acc;
  }
}

// Direction of a relative-position code pos in [0, 512): decoded box offset
// minus 3 (kernel/precalc.cxx:78-93).
void direction(int pos, double rho_eps, bool ref, double& al, double& be) {
  int c[3];
  decode3(pos, c);
  double x = c[0] - 3, y = c[1] - 3, z = c[2] - 3;
  double rh = std::sqrt(x * x + y * y + z * z) + rho_eps;
  al = rh == 0 ? 0.0 : std::acos(z / rh);
  be = azimuth(x, y, ref);
}

// Composes rotate(pos) -> z-translation Z -> rotate back into a K x K
// real-packed matrix.  Z(j, n, k) gives the coefficient from (n,k) to (j,k).
template <typename ZF>
void compose(int p, const std::vector<std::vector<cd>>& Wf, const std::vector<std::vector<cd>>& Wb, ZF Z,
             const double* col_scale, double* T) {
  const int K = (p + 1) * (p + 1);
  std::vector<cd> in(p + 1), rot(p + 1), mid((p + 1) * (p + 2) / 2), out(p + 1), tmp(p + 1);
  for (int n0 = 0; n0 <= p; n0++) {
    for (int pc = 0; pc < 2 * n0 + 1; pc++) {
      const int col = n0 * n0 + pc;
      std::fill(in.begin(), in.end(), cd(0, 0));
      if (pc == 0) in[0] = 1;
      else in[(pc + 1) / 2] = (pc & 1) ? cd(1, 0) : cd(0, 1);
      rotate_degree(Wf[n0], n0, in.data(), rot.data());
      // translate: degree n0 feeds every degree j through Z(j, n0, k)
      for (int j = 0; j <= p; j++) {
        for (int k = 0; k <= j; k++) tmp[k] = (k <= n0) ? Z(j, n0, k) * rot[k] : cd(0, 0);
        rotate_degree(Wb[j], j, tmp.data(), out.data());
        const double s = col_scale ? col_scale[n0] : 1.0;
        T[(size_t)(j * j) * K + col] = out[0].real() * s;
        for (int m = 1; m <= j; m++) {
          T[(size_t)(j * j + 2 * m - 1) * K + col] = out[m].real() * s;
          T[(size_t)(j * j + 2 * m) * K + col] = out[m].imag() * s;
        }
      }
    }
  }
}

template <typename F>
void parallel_for(int n, F f) {
  int nt = (int)std::thread::hardware_concurrency();
  if (nt < 1) nt = 1;
  if (nt > 32) nt = 32;
  std::vector<std::thread> th;
  for (int t = 0; t < nt; t++)
    th.emplace_back([=, &f] {
      for (int i = t; i < n; i += nt) f(i);
    });
  for (auto& x : th) x.join();
}

}  // namespace

namespace {
std::vector<double> anm_table(int p, bool ref) {
  const int mp = p + 1;
  std::vector<double> anm(4 * mp * mp);
  for (int n = 0; n < 2 * mp; n++)
    for (int m = -n; m <= n; m++)
      anm[ifull(n, m)] = to_ref_float(std::pow(-1.0, n) / std::sqrt(factorial(n - m) * factorial(n + m)), ref);
  return anm;
}
}  // namespace

void build_static_operators(Operators& ops, int p, bool ref) {
  const int mp = p + 1, K = mp * mp;
  ops.p = p;
  ops.K = K;
  ops.ref = ref;
  // fac and anm as kernel/precalc.cxx:19-31 stores them (float in the reference).
  ops.fac.assign(4 * mp * mp, 0.0);
  for (int n = 0; n < 2 * mp; n++)
    for (int m = -n; m <= n; m++) {
      int a = std::abs(m);
      ops.fac[ifull(n, m)] = to_ref_float(std::sqrt(factorial(n - a) / factorial(n + a)), ref);
    }
  const std::vector<double> anm = anm_table(p, ref);
  auto A = [&](int n, int m) { return anm[ifull(n, m)]; };

  const double rho_eps = ref ? kEpsF : 0.0;
  // Rotation tables for the 512 relative positions and their inverses.
  auto& Wf = ops.Wf;
  auto& Wb = ops.Wb;
  Wf.assign(512, {});
  Wb.assign(512, {});
  parallel_for(512, [&](int pos) {
    double al, be;
    direction(pos, rho_eps, ref, al, be);
    wigner(al, be, p, Wf[pos]);
    wigner(-al, -be, p, Wb[pos]);
  });

  // M2M: child octant c -> parent, rho = sqrt(3)/4 in parent units
  // (kernel/m2m.cxx:28-61); input degree n' scaled by 2^-n'.
  std::vector<double> scale_m2m(mp), scale_l2l(mp);
  for (int n = 0; n <= p; n++) {
    scale_m2m[n] = std::ldexp(1.0, -n);
    scale_l2l[n] = std::ldexp(1.0, -(n + 1));
  }
  ops.m2m.assign((size_t)8 * K * K, 0.0);
  ops.l2l.assign((size_t)8 * K * K, 0.0);
  for (int oct = 0; oct < 8; oct++) {
    int c[3];
    decode3(oct, c);
    int nc[3] = {4 - 2 * c[0], 4 - 2 * c[1], 4 - 2 * c[2]};
    int je = encode3(nc, 3);
    const double rh = std::sqrt(3.0) / 4;
    auto Zm = [&](int j, int n0, int k) -> double {  // from degree n0 = j - n
      int n = j - n0;
      if (n < 0 || n0 < k) return 0.0;
      return std::pow(-1.0, n) * A(n, 0) * A(j - n, k) / A(j, k) * std::pow(rh, n);
    };
    compose(p, Wf[je], Wb[je], Zm, scale_m2m.data(), &ops.m2m[(size_t)oct * K * K]);
    // L2L: parent -> child octant c, rho = sqrt(3)/2 in child units
    // (kernel/l2l.cxx:44-77); input degree n scaled by 2^-(n+1).
    int nl[3] = {2 * c[0] + 2, 2 * c[1] + 2, 2 * c[2] + 2};
    int jl = encode3(nl, 3);
    const double rl = std::sqrt(3.0) / 2;
    auto Zl = [&](int j, int n, int k) -> double {
      if (n < j || n < k) return 0.0;
      return A(n - j, 0) * A(j, k) / A(n, k) * std::pow(rl, n - j);
    };
    compose(p, Wf[jl], Wb[jl], Zl, scale_l2l.data(), &ops.l2l[(size_t)oct * K * K]);
  }

  // M2L slot structure: for a target box in octant c, the reference's
  // interaction-list loop (fmm/ijbox.cxx:85-104) visits parent-neighbour
  // offsets (ax,ay,az), then children (bx,by,bz), skipping adjacent boxes.
  ops.slot_rel.assign(8 * kM2LSlots, -1);
  ops.rel_to_op.assign(kRelCodes, -1);
  std::vector<int>& op_rel = ops.op_rel;
  op_rel.clear();
  for (int dx = -3; dx <= 3; dx++)
    for (int dy = -3; dy <= 3; dy++)
      for (int dz = -3; dz <= 3; dz++) {
        if (std::abs(dx) <= 1 && std::abs(dy) <= 1 && std::abs(dz) <= 1) continue;
        int code = (dx + 3) * 49 + (dy + 3) * 7 + (dz + 3);
        ops.rel_to_op[code] = (int)op_rel.size();
        op_rel.push_back(code);
      }
  for (int oct = 0; oct < 8; oct++) {
    int c[3];
    decode3(oct, c);
    int s = 0;
    for (int ax = -1; ax <= 1; ax++)
      for (int ay = -1; ay <= 1; ay++)
        for (int az = -1; az <= 1; az++)
          for (int bx = 0; bx <= 1; bx++)
            for (int by = 0; by <= 1; by++)
              for (int bz = 0; bz <= 1; bz++) {
                int dx = c[0] - 2 * ax - bx, dy = c[1] - 2 * ay - by, dz = c[2] - 2 * az - bz;
                if (std::abs(dx) <= 1 && std::abs(dy) <= 1 && std::abs(dz) <= 1) continue;
                ops.slot_rel[oct * kM2LSlots + s++] = (dx + 3) * 49 + (dy + 3) * 7 + (dz + 3);
              }
  }

  ops.m2l.clear();
  ops.m2l_sets = 0;
  ops.m2l_lmax = 0;
}

// M2L operators (kernel/m2l.cxx:43-78): one set, or one per level when the
// distance carries the reference's absolute eps.
void build_m2l_operators(Operators& ops, int lmax, float rd) {
  const int p = ops.p, K = ops.K;
  const bool ref = ops.ref;
  const std::vector<double> anm = anm_table(p, ref);
  auto A = [&](int n, int m) { return anm[ifull(n, m)]; };
  // sr of kernel/precalc.cxx:33-43
  auto SR = [&](int j, int k, int n) { return to_ref_float(std::pow(-1.0, j + k) * A(n, k) * A(j, k) / A(j + n, 0), ref); };
  const double rho_eps = ref ? kEpsF : 0.0;
  const auto& op_rel = ops.op_rel;
  const auto& Wf = ops.Wf;
  const auto& Wb = ops.Wb;
  const int nops = (int)op_rel.size();  // 316
  ops.m2l_sets = ref ? (lmax - 1) : 1;
  ops.m2l_lmax = lmax;
  ops.m2l_rd = rd;
  ops.m2l.assign((size_t)ops.m2l_sets * nops * K * K, 0.0);
  parallel_for(ops.m2l_sets * nops, [&](int w) {
    const int set = w / nops, o = w % nops;
    const int code = op_rel[o];
    const int dx = code / 49 - 3, dy = (code / 7) % 7 - 3, dz = code % 7 - 3;
    int nc[3] = {dx + 3, dy + 3, dz + 3};
    const int je = encode3(nc, 3);
    double rho = std::sqrt((double)(dx * dx + dy * dy + dz * dz));
    if (ref) {
      const int lev = 2 + set;
      const double rb = (double)(rd / (float)(1 << lev));
      rho = (rb * rho + rho_eps) / rb;  // (|d| rb + eps) in units of rb
    }
    auto Z = [&](int j, int n, int k) -> double {
      if (n < k) return 0.0;
      return SR(j, k, n) / std::pow(rho, j + n + 1);
    };
    compose(p, Wf[je], Wb[je], Z, nullptr, &ops.m2l[((size_t)set * nops + o) * K * K]);
  });
}

}  // namespace fmmb

namespace fmmb {

// TF32 round-to-nearest (ties away from zero) of an FP32 value, the rounding
// of cvt.rna.tf32.f32: keep 10 mantissa bits.
static float tf32_rna_host(float x) {
  uint32_t b;
  std::memcpy(&b, &x, 4);
  if ((b & 0x7f800000u) != 0x7f800000u) b = (b + 0x1000u) & 0xffffe000u;
  float y;
  std::memcpy(&y, &b, 4);
  return y;
}

// Translation operators as TF32 (hi, lo) pairs for the tensor-core kernel,
// zero padded to kpad columns; one image per operator and block of 128 output
// rows (nrb = ceil(K / 128) blocks, image index op * nrb + block), each of
// 2 x 128 x kpad floats:
//  * hi (TF32 rounding of the FP64 entry) laid out like the kernel's
//    shared-memory operand tiles: per K-block of 32 columns, 128 rows of 128
//    bytes with the 16-byte chunk c of row r stored at chunk c ^ (r & 7)
//    (K-major SWIZZLE_128B), kpad / 32 K-blocks;
//  * lo (TF32 rounding of the remainder) row-major, 128 rows of kpad values,
//    which the kernel writes into tensor-memory lane r.
void build_tc_images(const std::vector<double>& mats, int nmat, int K, int kpad, std::vector<float>& img) {
  const int nrb = (K + 127) / 128, nkb = kpad / 32;
  const size_t per_img = (size_t)2 * 128 * kpad;
  img.assign((size_t)nmat * nrb * per_img, 0.0f);
  parallel_for(nmat, [&](int w) {
    const double* T = &mats[(size_t)w * K * K];
    for (int blk = 0; blk < nrb; blk++) {
      float* out = &img[((size_t)w * nrb + blk) * per_img];
      for (int rr = 0; rr < 128; rr++) {
        const int r = blk * 128 + rr;
        if (r >= K) break;
        for (int col = 0; col < K; col++) {
          const double v = T[(size_t)r * K + col];
          const float hi = tf32_rna_host((float)v);
          const float lo = tf32_rna_host((float)(v - (double)hi));
          const int kb = col / 32, j = col % 32;
          out[(size_t)kb * 4096 + (size_t)rr * 32 + (size_t)(((j >> 2) ^ (rr & 7)) << 2) + (j & 3)] = hi;
          out[(size_t)nkb * 4096 + (size_t)rr * kpad + col] = lo;
        }
      }
    }
  });
}

// Translation operators for the FP16x3 tensor-core M2L (translate_h16.cu),
// one image of img_bytes per operator:
//  * the operator scaled by 2^-f so that its largest |entry| lies in
//    [2^14, 2^15), just below the FP16 maximum; hi = FP16 rounding of the
//    scaled entry, lo = FP16 rounding of the remainder;
//  * hi then lo as kpad / 64 K-blocks each of n rows (n = K rounded up to 16)
//    of 128 bytes, 16-byte chunk c of row r stored at chunk c ^ (r & 7)
//    (K-major SWIZZLE_128B, the kernel's B operand), zero padded;
//  * then the factor 2^f as a float, padded to 16 bytes.
void build_h16_images(const std::vector<double>& mats, int nmat, int K, int n, int kpad, size_t img_bytes,
                      std::vector<unsigned char>& img) {
  const int nkb = kpad / 64;
  const size_t kb_bytes = (size_t)n * 128;
  img.assign((size_t)nmat * img_bytes, 0);
  parallel_for(nmat, [&](int w) {
    const double* T = &mats[(size_t)w * K * K];
    unsigned char* base = &img[(size_t)w * img_bytes];
    double mx = 0.0;
    for (size_t i = 0; i < (size_t)K * K; i++) mx = std::max(mx, std::fabs(T[i]));
    int f = 0;
    if (mx > 0.0) {
      std::frexp(mx, &f);  // mx = g 2^f, g in [0.5, 1)
      f -= 15;
    }
    const float scale = std::ldexp(1.0f, f);
    std::memcpy(base + 2 * nkb * kb_bytes, &scale, 4);
    for (int r = 0; r < K; r++)
      for (int c = 0; c < K; c++) {
        const double v = std::ldexp(T[(size_t)r * K + c], -f);
        const __half hi = __double2half(v);
        const __half lo = __double2half(v - (double)__half2float(hi));
        const int kb = c / 64, j = c % 64;
        const size_t off = (size_t)r * 128 + (size_t)((((j >> 3) ^ (r & 7)) << 4) + (j & 7) * 2);
        std::memcpy(base + (size_t)kb * kb_bytes + off, &hi, 2);
        std::memcpy(base + (size_t)(nkb + kb) * kb_bytes + off, &lo, 2);
      }
  });
}

}  // namespace fmmb

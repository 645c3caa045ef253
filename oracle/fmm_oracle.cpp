// CPU restatement of the reference FMM -- TEST INFRASTRUCTURE ONLY.
//
// This file is the oracle: tests/, __graft_entry__.smoke() and bench.py's CPU
// baseline use it as the checker.  The product (old_fmm_bem_b200, libfmmb.so)
// never links or calls it.
//
// It restates, function by function, the reference's serial FMM path
// (fmm/fmm.cxx:29-152 and the fmm/, sort/ and kernel/ files it calls) with two
// generalisations: the expansion order is a run-time parameter, and the
// arithmetic conventions are switchable.  With ref_semantics=1 it keeps every
// numerical convention of the reference (tables fac/anm/sr rounded to float as
// kernel/precalc.cxx stores them, the single-precision pi in azimuths and in
// 1/(4 pi), eps=1e-6f added to every expansion radius, outputs accumulated in
// float); with ref_semantics=0 it computes the same algorithm in plain FP64
// with exact angles.  The level-2 M2L uses every non-adjacent box (the fix of
// fmm/fmm.cxx:104, see oracle/refshim/src/ref_driver.cpp).
//
// Parity is pinned against the reference itself: tests/test_oracle_pin.py runs
// the reference compiled from source (oracle/_ref) and this restatement on the
// same inputs and requires identical trees/lists and matching potentials.
#include "fmm_oracle.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <complex>
#include <cstring>
#include <vector>

typedef std::complex<double> cd;

namespace {

const double kPiF = (double)(float)M_PI;   // reference include/constants.h:35
const double kEpsF = (double)1e-6f;        // reference include/constants.h:34

struct Sem {
  bool ref;
  double rho_eps;  // added to every expansion radius (reference: eps)
  double ang_eps;  // azimuth branch threshold (reference: eps)
  double pi_ang;   // pi used in azimuth branches
  double coef;     // 1/(4 pi) factor of the kernels
  double eps2;     // P2P softening
  bool excl_self;
};

inline int isym(int n, int m) { return n * (n + 1) / 2 + m; }
inline int ifull(int n, int m) { return n * n + n + m; }

// kernel/factorial.cxx:1-10
double factorial(int n) {
  double f = 1;
  for (int i = 1; i <= n; i++) f = f * i;
  return f;
}

// fmm/boxc.cxx:3-24 -- Morton key -> box coordinates (x from bit 3i+1,
// y from bit 3i, z from bit 3i+2).
void key_decode(int key, int* c) {
  c[0] = c[1] = c[2] = 0;
  for (int i = 0; key >> (3 * i); i++) {
    c[1] |= ((key >> (3 * i)) & 1) << i;
    c[0] |= ((key >> (3 * i + 1)) & 1) << i;
    c[2] |= ((key >> (3 * i + 2)) & 1) << i;
  }
}

// fmm/boxn1.cxx:3-19 -- box coordinates -> Morton key over `lev` levels.
int key_encode(const int* c, int lev) {
  int k = 0;
  for (int i = 0; i < lev; i++) {
    k += ((c[0] >> i) & 1) << (3 * i + 1);
    k += ((c[1] >> i) & 1) << (3 * i);
    k += ((c[2] >> i) & 1) << (3 * i + 2);
  }
  return k;
}

// Azimuth with the reference's branches (kernel/G_p2m.cxx:33-41,
// kernel/G_l2p.cxx:31-39, kernel/precalc.cxx:85-93) or atan2.
double azimuth(double x, double y, const Sem& s) {
  if (!s.ref) return (x == 0 && y == 0) ? 0.0 : std::atan2(y, x);
  if (std::abs(x) + std::abs(y) < s.ang_eps) return 0;
  if (std::abs(x) < s.ang_eps) return y / std::abs(y) * s.pi_ang * 0.5;
  if (x > 0) return std::atan(y / x);
  return std::atan(y / x) + s.pi_ang;
}

inline double polar(double z, double rh) { return rh == 0 ? 0.0 : std::acos(z / rh); }

struct Tables {
  int mp = 0;
  std::vector<double> fac, anm;  // index n*n+n+m, n < 2mp
  std::vector<double> sr;        // [(j*j+j+k)*mp*mp + n*n+n+k]
  std::vector<cd> dnm;           // [((pos*mp)+m)*mp*mp + n*n+n+k], pos < 1024
  const cd* rot(int pos) const { return &dnm[(size_t)pos * mp * mp * mp]; }
};

inline double maybe_float(double v, bool ref) { return ref ? (double)(float)v : v; }

// kernel/precalc.cxx:104-146 -- Wigner d^n_{mk}(al) e^{i(m+k) be} for one
// relative position, by the reference's recurrence in k then m.
// The recurrence divides by 1+cos(al), which vanishes for a rotation by pi
// (relative positions straight down the z axis).  The reference never meets
// it because its radius carries +eps; for exact angles the closed form
// D(m,k) = (-1)^n [k == -m] of that rotation is used.
void rotation_table(double al, double be, int mp, cd* out) {
  std::vector<double> d;
  const bool flip = (1 + std::cos(al)) == 0;
  double sc = std::sin(al) / (1 + std::cos(al));
  for (int n = 0; n < mp; n++) {
    int w = 2 * n + 1;
    d.assign((size_t)w * w, 0.0);
    auto D = [&](int m, int k) -> double& { return d[(size_t)(m + n) * w + (k + n)]; };
    if (flip) {
      for (int m = 0; m <= n; m++)
        for (int k = -n; k <= n; k++)
          out[(size_t)m * mp * mp + ifull(n, k)] =
              (k == -m ? std::pow(-1.0, n) : 0.0) * std::exp(cd(0, (k + m) * be));
      continue;
    }
    D(n, n) = std::pow(std::cos(al * 0.5), 2 * n);
    for (int k = n; k >= 1 - n; k--) {
      double ank = ((double)n + k) / (n - k + 1);
      D(n, k - 1) = std::sqrt(ank) * std::tan(al * 0.5) * D(n, k);
    }
    for (int m = n; m >= 1; m--) {
      for (int k = m - 1; k >= 1 - m; k--) {
        double anmd = n * (n + 1) - m * (m - 1);
        double a0 = -(m + k) / std::sqrt(anmd);
        double a1 = std::sqrt(((double)(n * (n + 1) - k * (k + 1))) / (n * (n + 1) - m * (m - 1)));
        D(m - 1, k) = a1 * D(m, k + 1) + a0 * sc * D(m, k);
      }
    }
    // kernel/precalc.cxx:119-136 -- fill the rest by symmetry
    if (n >= 1) {
      for (int m = 0; m <= n; m++) {
        for (int k = -m; k <= -1; k++) {
          D(m, k) = std::pow(-1.0, k) * D(m, k);
          D(-k, -m) = std::pow(-1.0, m + k) * D(m, k);
        }
        for (int k = 0; k <= m; k++) {
          D(k, m) = std::pow(-1.0, m + k) * D(m, k);
          D(-k, -m) = D(k, m);
        }
      }
    }
    for (int m = 0; m <= n; m++)
      for (int k = -n; k <= n; k++) {
        double ang = (k + m) * be;
        out[(size_t)m * mp * mp + ifull(n, k)] = D(m, k) * std::exp(cd(0, ang));
      }
  }
}

// kernel/precalc.cxx:10-213 (fac, anm, sr, rotation tables; ynm(n,m) is 1 for
// m=0 and 0 otherwise -- the Legendre recurrence at x=1 of precalc.cxx:45-64 --
// so it is folded into the translation formulas below).
void build_tables(int mp, const Sem& s, Tables& t) {
  t.mp = mp;
  int nt = 4 * mp * mp;
  t.fac.assign(nt, 0.0);
  t.anm.assign(nt, 0.0);
  for (int n = 0; n < 2 * mp; n++)
    for (int m = -n; m <= n; m++) {
      int a = std::abs(m);
      t.fac[ifull(n, m)] = maybe_float(std::sqrt(factorial(n - a) / factorial(n + a)), s.ref);
      t.anm[ifull(n, m)] = maybe_float(std::pow(-1.0, n) / std::sqrt(factorial(n - m) * factorial(n + m)), s.ref);
    }
  t.sr.assign((size_t)mp * mp * mp * mp, 0.0);
  for (int j = 0; j < mp; j++)
    for (int k = -j; k <= j; k++)
      for (int n = std::abs(k); n < mp; n++) {
        int jk = ifull(j, k), nk = ifull(n, k), jn = ifull(j + n, 0);
        t.sr[(size_t)jk * mp * mp + nk] =
            maybe_float(std::pow(-1.0, j + k) * t.anm[nk] * t.anm[jk] / t.anm[jn], s.ref);
      }
  t.dnm.assign((size_t)1024 * mp * mp * mp, cd(0, 0));
  for (int i = 0; i < 512; i++) {
    int c[3];
    key_decode(i, c);
    double x = c[0] - 3, y = c[1] - 3, z = c[2] - 3;
    double rh = std::sqrt(x * x + y * y + z * z) + s.rho_eps;
    double al = polar(z, rh);
    double be = azimuth(x, y, s);
    rotation_table(al, be, mp, &t.dnm[(size_t)i * mp * mp * mp]);
    rotation_table(-al, -be, mp, &t.dnm[(size_t)(i + 512) * mp * mp * mp]);
  }
}

// kernel/spharot.cxx:3-24
void spharot(const cd* yx, cd* yxr, int mp, const cd* dnm) {
  for (int n = 0; n < mp; n++)
    for (int m = 0; m <= n; m++) {
      const cd* row = dnm + (size_t)m * mp * mp;
      cd acc = 0;
      for (int k = -n; k <= -1; k++) acc += row[ifull(n, k)] * std::conj(yx[isym(n, -k)]);
      for (int k = 0; k <= n; k++) acc += row[ifull(n, k)] * yx[isym(n, k)];
      yxr[isym(n, m)] = acc;
    }
}

// kernel/multipole.cxx:7-35 -- rh^n fac P_n^m(cos al), m >= 0.
void multipole(double rh, double al, int mp, const double* fac, double* bnm) {
  double xx = std::cos(al), s2 = std::sqrt((1 - xx) * (1 + xx));
  double fact = 1, pn = 1, rhm = 1;
  for (int m = 0; m < mp; m++) {
    double p = pn;
    bnm[ifull(m, m)] = rhm * fac[ifull(m, m)] * p;
    double p1 = p, p2;
    p = xx * (2 * m + 1) * p;
    rhm *= rh;
    double rhn = rhm;
    for (int n = m + 1; n < mp; n++) {
      bnm[ifull(n, m)] = rhn * fac[ifull(n, m)] * p;
      p2 = p1;
      p1 = p;
      p = (xx * (2 * n + 1) * p1 - (n + m) * p2) / (n - m + 1);
      rhn *= rh;
    }
    pn = -pn * fact * s2;
    fact += 2;
  }
}

// kernel/multipoled.cxx:7-34 -- fac P_n^m(cos th) and fac dP_n^m/dth.
void multipoled(double th, int mp, const double* fac, double* bnm, double* bth) {
  double xx = std::cos(th), yy = std::sin(th), s2 = std::sqrt((1 - xx) * (1 + xx));
  double fact = 1, pn = 1;
  for (int m = 0; m < mp; m++) {
    double p = pn;
    int nm = ifull(m, m);
    bnm[nm] = fac[nm] * p;
    double p1 = p, p2;
    p = xx * (2 * m + 1) * p;
    bth[nm] = fac[nm] * (p - (m + 1) * xx * p1) / yy;
    for (int n = m + 1; n < mp; n++) {
      nm = ifull(n, m);
      bnm[nm] = fac[nm] * p;
      p2 = p1;
      p1 = p;
      p = (xx * (2 * n + 1) * p1 - (n + m) * p2) / (n - m + 1);
      bth[nm] = fac[nm] * ((n - m + 1) * p - (n + 1) * xx * p1) / yy;
    }
    pn = -pn * fact * s2;
    fact += 2;
  }
}

struct Tree {
  // per level lev (index lev, 2..lmax): sorted distinct box keys
  std::vector<std::vector<int>> ki, kj;
  std::vector<int> li0, li1, lj0, lj1;  // leaf ranges (first, last) in sorted order
  std::vector<int> perm_i, perm_j;
};

// fmm/boxn.cxx:5-31 -- leaf key of each point (float box offset times a
// float scale, truncated, clamped to the last box).
void box_keys(int n, const float* x, const float* y, const float* z, int lmax, float xmin,
              float ymin, float zmin, float rd, std::vector<int>& key) {
  int kl = 1 << lmax;
  double rb = (float)kl / rd;  // int / float is a float division in the reference
  key.resize(n);
  for (int j = 0; j < n; j++) {
    int c[3] = {int((x[j] - xmin) * rb), int((y[j] - ymin) * rb), int((z[j] - zmin) * rb)};
    for (int i = 0; i < 3; i++)
      if (c[i] >= kl) c[i]--;
    key[j] = key_encode(c, lmax);
  }
}

// sort/csort.cxx:5-17 -- stable sort of keys; perm[pos] = original index.
void stable_order(const std::vector<int>& key, std::vector<int>& perm) {
  perm.resize(key.size());
  for (size_t i = 0; i < key.size(); i++) perm[i] = (int)i;
  std::stable_sort(perm.begin(), perm.end(), [&](int a, int b) { return key[a] < key[b]; });
}

// fmm/boxdatai.cxx:10-34 / boxdataj.cxx:10-36 (leaf keys and ranges) and
// fmm/boxm2mi.cxx:6-24 / boxm2mj.cxx:6-26 (parent levels by key/8, unique).
void build_levels(const std::vector<int>& sorted_key, int lmax, std::vector<std::vector<int>>& lev_keys,
                  std::vector<int>& first, std::vector<int>& last) {
  lev_keys.assign(lmax + 1, {});
  first.clear();
  last.clear();
  int n = (int)sorted_key.size();
  for (int i = 0; i < n; i++) {
    if (i == 0 || sorted_key[i] != sorted_key[i - 1]) {
      lev_keys[lmax].push_back(sorted_key[i]);
      first.push_back(i);
      if (i > 0) last.push_back(i - 1);
    }
  }
  if (n > 0) last.push_back(n - 1);
  for (int lev = lmax - 1; lev >= 2; lev--) {
    for (size_t b = 0; b < lev_keys[lev + 1].size(); b++) {
      int pk = lev_keys[lev + 1][b] / 8;
      if (lev_keys[lev].empty() || lev_keys[lev].back() != pk) lev_keys[lev].push_back(pk);
    }
  }
}

int find_box(const std::vector<int>& keys, int key) {
  auto it = std::lower_bound(keys.begin(), keys.end(), key);
  return (it != keys.end() && *it == key) ? (int)(it - keys.begin()) : -1;
}

// fmm/ijbox.cxx:9-117 -- lists of source boxes (compact indices at `lev`)
// for each target box.  mode 0: 3x3x3 neighbourhood incl. self; mode 1: all
// non-adjacent boxes; mode 2: children of the parent's neighbours that are not
// adjacent.  Loops are in the reference order; the clip to the source
// bounding box only skips boxes that cannot exist.
void build_lists(const std::vector<int>& ti, const std::vector<int>& tj, int lev, int mode,
                 std::vector<std::vector<int>>& lists) {
  int lo[3] = {1000000, 1000000, 1000000}, hi[3] = {-1000000, -1000000, -1000000};
  std::vector<std::array<int, 3>> cj(tj.size());
  for (size_t jj = 0; jj < tj.size(); jj++) {
    int c[3];
    key_decode(tj[jj], c);
    for (int d = 0; d < 3; d++) {
      cj[jj][d] = c[d];
      lo[d] = std::min(lo[d], c[d]);
      hi[d] = std::max(hi[d], c[d]);
    }
  }
  lists.assign(ti.size(), {});
  for (size_t ii = 0; ii < ti.size(); ii++) {
    int c[3];
    key_decode(ti[ii], c);
    int ix = c[0], iy = c[1], iz = c[2];
    auto& L = lists[ii];
    if (mode == 0) {
      for (int jx = std::max(ix - 1, lo[0]); jx <= std::min(ix + 1, hi[0]); jx++)
        for (int jy = std::max(iy - 1, lo[1]); jy <= std::min(iy + 1, hi[1]); jy++)
          for (int jz = std::max(iz - 1, lo[2]); jz <= std::min(iz + 1, hi[2]); jz++) {
            int cc[3] = {jx, jy, jz};
            int jj = find_box(tj, key_encode(cc, lev));
            if (jj != -1) L.push_back(jj);
          }
    } else if (mode == 1) {
      for (size_t jj = 0; jj < tj.size(); jj++) {
        int jx = cj[jj][0], jy = cj[jj][1], jz = cj[jj][2];
        if (jx < ix - 1 || ix + 1 < jx || jy < iy - 1 || iy + 1 < jy || jz < iz - 1 || iz + 1 < jz)
          L.push_back((int)jj);
      }
    } else {
      int px = (ix + 2) / 2, py = (iy + 2) / 2, pz = (iz + 2) / 2;
      for (int qx = px - 1; qx <= px + 1; qx++)
        for (int qy = py - 1; qy <= py + 1; qy++)
          for (int qz = pz - 1; qz <= pz + 1; qz++)
            for (int jx = std::max(2 * qx - 2, lo[0]); jx <= std::min(2 * qx - 1, hi[0]); jx++)
              for (int jy = std::max(2 * qy - 2, lo[1]); jy <= std::min(2 * qy - 1, hi[1]); jy++)
                for (int jz = std::max(2 * qz - 2, lo[2]); jz <= std::min(2 * qz - 1, hi[2]); jz++) {
                  if (jx < ix - 1 || ix + 1 < jx || jy < iy - 1 || iy + 1 < jy || jz < iz - 1 ||
                      iz + 1 < jz) {
                    int cc[3] = {jx, jy, jz};
                    int jj = find_box(tj, key_encode(cc, lev));
                    if (jj != -1) L.push_back(jj);
                  }
                }
    }
  }
}

// Records of the last run.
std::vector<int> rec[9];
std::vector<double> exp_rec[2];
int g_np = 0;

}  // namespace

extern "C" {

int oracle_fmm(const oracle_config* cfg, int ni, int nj, const float* tx, const float* ty,
               const float* tz, const float* tnx, const float* tny, const float* tnz,
               const float* sx, const float* sy, const float* sz, const float* snx,
               const float* sny, const float* snz, const float* q, double* pot, double* gx,
               double* gy, double* gz) {
  const int mp = cfg->p + 1, lmax = cfg->lmax, neq = cfg->neq;
  if (mp < 2 || lmax < 2 || lmax > 10 || (neq != 0 && neq != 1 && neq != 2)) return -1;
  Sem s;
  s.ref = cfg->ref_semantics != 0;
  s.rho_eps = s.ref ? kEpsF : 0.0;
  s.ang_eps = s.ref ? kEpsF : 0.0;
  s.pi_ang = s.ref ? kPiF : M_PI;
  s.coef = s.ref ? 0.25 / kPiF : 0.25 / M_PI;
  s.eps2 = cfg->eps2;
  s.excl_self = cfg->exclude_self != 0;
  const int nmp = mp * (mp + 1) / 2;

  Tables tb;
  build_tables(mp, s, tb);

  // Tree: keys, stable order, sorted copies (sort/sorti.cxx:12-35, sortj.cxx:12-36).
  Tree tr;
  std::vector<int> key_i, key_j;
  box_keys(ni, tx, ty, tz, lmax, cfg->xmin, cfg->ymin, cfg->zmin, cfg->rd, key_i);
  box_keys(nj, sx, sy, sz, lmax, cfg->xmin, cfg->ymin, cfg->zmin, cfg->rd, key_j);
  stable_order(key_i, tr.perm_i);
  stable_order(key_j, tr.perm_j);
  std::vector<int> ski(ni), skj(nj);
  std::vector<float> X(ni), Y(ni), Z(ni), NX(ni), NY(ni), NZ(ni);
  std::vector<float> XJ(nj), YJ(nj), ZJ(nj), NXJ(nj), NYJ(nj), NZJ(nj), QJ(nj);
  for (int i = 0; i < ni; i++) {
    int o = tr.perm_i[i];
    ski[i] = key_i[o];
    X[i] = tx[o]; Y[i] = ty[o]; Z[i] = tz[o];
    NX[i] = tnx ? tnx[o] : 0.f; NY[i] = tny ? tny[o] : 0.f; NZ[i] = tnz ? tnz[o] : 0.f;
  }
  for (int j = 0; j < nj; j++) {
    int o = tr.perm_j[j];
    skj[j] = key_j[o];
    XJ[j] = sx[o]; YJ[j] = sy[o]; ZJ[j] = sz[o];
    NXJ[j] = snx ? snx[o] : 0.f; NYJ[j] = sny ? sny[o] : 0.f; NZJ[j] = snz ? snz[o] : 0.f;
    QJ[j] = q[o];
  }
  build_levels(ski, lmax, tr.ki, tr.li0, tr.li1);
  build_levels(skj, lmax, tr.kj, tr.lj0, tr.lj1);

  for (auto& r : rec) r.clear();
  rec[0] = tr.perm_i;
  rec[1] = tr.perm_j;
  rec[4].assign(lmax + 1, 0);
  rec[5].assign(lmax + 1, 0);
  for (int lev = lmax; lev >= 2; lev--) {
    rec[2].insert(rec[2].end(), tr.ki[lev].begin(), tr.ki[lev].end());
    rec[3].insert(rec[3].end(), tr.kj[lev].begin(), tr.kj[lev].end());
    rec[4][lev] = (int)tr.ki[lev].size();
    rec[5][lev] = (int)tr.kj[lev].size();
  }
  for (size_t b = 0; b < tr.li0.size(); b++) { rec[6].push_back(tr.li0[b]); rec[6].push_back(tr.li1[b]); }
  for (size_t b = 0; b < tr.lj0.size(); b++) { rec[7].push_back(tr.lj0[b]); rec[7].push_back(tr.lj1[b]); }
  auto record_lists = [&](int lev, int mode, const std::vector<std::vector<int>>& L) {
    rec[8].push_back(lev);
    rec[8].push_back(mode);
    rec[8].push_back((int)tr.ki[lev].size());
    rec[8].push_back((int)tr.kj[lev].size());
    for (auto& l : L) rec[8].push_back((int)l.size());
    for (auto& l : L) rec[8].insert(rec[8].end(), l.begin(), l.end());
  };

  // Outputs: float accumulation (reference) or double.
  std::vector<double> V(ni, 0.0), GX(ni, 0.0), GY(ni, 0.0), GZ(ni, 0.0);
  std::vector<float> Vf(ni, 0.f), GXf(ni, 0.f), GYf(ni, 0.f), GZf(ni, 0.f);
  auto add_out = [&](int i, double v, double a, double b, double c) {
    if (s.ref) {
      Vf[i] += v; GXf[i] += a; GYf[i] += b; GZf[i] += c;
    } else {
      V[i] += v; GX[i] += a; GY[i] += b; GZ[i] += c;
    }
  };

  // Step 1. P2P at lmax (fmm/fmm.cxx:44-65; kernel/G_p2p.cxx:12-37,
  // Gni_p2p.cxx:12-28, Gnj_p2p.cxx:12-28).
  std::vector<std::vector<int>> near;
  build_lists(tr.ki[lmax], tr.kj[lmax], lmax, 0, near);
  record_lists(lmax, 0, near);
  for (size_t ii = 0; ii < near.size(); ii++) {
    for (int jj : near[ii]) {
      for (int i = tr.li0[ii]; i <= tr.li1[ii]; i++) {
        double pij = 0, fx = 0, fy = 0, fz = 0;
        for (int j = tr.lj0[jj]; j <= tr.lj1[jj]; j++) {
          // float differences as the reference (kernel/G_p2p.cxx:21-23);
          // exact FP64 differences in accurate semantics
          double dx, dy, dz;
          if (s.ref) {
            dx = X[i] - XJ[j]; dy = Y[i] - YJ[j]; dz = Z[i] - ZJ[j];
          } else {
            dx = (double)X[i] - XJ[j]; dy = (double)Y[i] - YJ[j]; dz = (double)Z[i] - ZJ[j];
          }
          if (s.excl_self && dx == 0 && dy == 0 && dz == 0) continue;
          double r2 = dx * dx + dy * dy + dz * dz + s.eps2;
          if (neq == 0) {
            double rs = s.coef * QJ[j] / r2 / std::sqrt(r2);
            pij += s.coef * QJ[j] / std::sqrt(r2);
            fx -= dx * rs; fy -= dy * rs; fz -= dz * rs;
          } else {
            double rs = s.coef * QJ[j] / std::sqrt(r2) / r2;
            if (neq == 1) pij += (dx * NX[i] + dy * NY[i] + dz * NZ[i]) * rs;
            else pij += (dx * NXJ[j] + dy * NYJ[j] + dz * NZJ[j]) * rs;
          }
        }
        add_out(i, pij, fx, fy, fz);
      }
    }
  }

  // Expansion storage: every level, reference order (lmax first).
  std::vector<std::vector<cd>> M(lmax + 1), L(lmax + 1);
  for (int lev = 2; lev <= lmax; lev++) {
    M[lev].assign(tr.kj[lev].size() * nmp, cd(0, 0));
    L[lev].assign(tr.ki[lev].size() * nmp, cd(0, 0));
  }
  std::vector<double> bnm(4 * mp * mp), bth(4 * mp * mp);
  const double* fac = tb.fac.data();
  const double* anm = tb.anm.data();

  // Step 2. P2M at lmax (kernel/G_p2m.cxx:11-59, kernel/Gn_p2m.cxx:11-67).
  const double rbl = (double)(cfg->rd / (float)(1 << lmax));  // rd/kl: float division
  for (size_t jj = 0; jj < tr.kj[lmax].size(); jj++) {
    int c[3];
    key_decode(tr.kj[lmax][jj], c);
    double xc = cfg->xmin + (c[0] + 0.5) * rbl;
    double yc = cfg->ymin + (c[1] + 0.5) * rbl;
    double zc = cfg->zmin + (c[2] + 0.5) * rbl;
    cd* bx = &M[lmax][jj * nmp];
    for (int j = tr.lj0[jj]; j <= tr.lj1[jj]; j++) {
      double x = XJ[j] - xc, y = YJ[j] - yc, z = ZJ[j] - zc;
      double rh = std::sqrt(x * x + y * y + z * z) + s.rho_eps;
      double al = polar(z, rh);
      double be = azimuth(x, y, s);
      if (neq != 2) {
        multipole(rh, al, mp, fac, bnm.data());
        for (int n = 0; n < mp; n++)
          for (int m = 0; m <= n; m++) {
            cd eim = std::exp(cd(0, -m * be));
            bx[isym(n, m)] += ((cd)QJ[j]) * bnm[ifull(n, m)] * eim;
          }
      } else {
        multipoled(al, mp, fac, bnm.data(), bth.data());
        double sa = std::sin(al), ca = std::cos(al), sb = std::sin(be), cb = std::cos(be);
        cd qx = (double)(QJ[j] * NXJ[j]), qy = (double)(QJ[j] * NYJ[j]), qz = (double)(QJ[j] * NZJ[j]);
        for (int n = 0; n < mp; n++)
          for (int m = 0; m <= n; m++) {
            int nm = ifull(n, m);
            cd eim = std::exp(cd(0, -m * be));
            cd brh = n * std::pow(rh, n - 1) * bnm[nm] * eim;
            cd bal = std::pow(rh, n) * bth[nm] * eim;
            cd bbe = -m * std::pow(rh, n) * bnm[nm] * eim * cd(0, 1);
            cd bxd = sa * cb * brh + ca * cb / rh * bal - sb / rh / sa * bbe;
            cd byd = sa * sb * brh + ca * sb / rh * bal + cb / rh / sa * bbe;
            cd bzd = ca * brh - sa / rh * bal;
            bx[isym(n, m)] += qx * bxd;
            bx[isym(n, m)] += qy * byd;
            bx[isym(n, m)] += qz * bzd;
          }
      }
    }
  }

  std::vector<cd> t1(nmp), t2(nmp);
  // Step 3. M2M lmax-1..2 (kernel/m2m.cxx:13-66): rotate, shift along z by
  // rh = rb sqrt(3)/4 (rb = parent box size), rotate back, add to parent.
  for (int lev = lmax - 1; lev >= 2; lev--) {
    double rb = (double)(cfg->rd / (float)(1 << lev));
    double rh = rb * std::sqrt(3.0) / 4;
    for (size_t jj = 0; jj < tr.kj[lev + 1].size(); jj++) {
      int ck = tr.kj[lev + 1][jj];
      int ib = find_box(tr.kj[lev], ck / 8);
      int c[3];
      key_decode(ck % 8, c);
      int nc[3] = {4 - 2 * c[0], 4 - 2 * c[1], 4 - 2 * c[2]};
      int je = key_encode(nc, 3);
      spharot(&M[lev + 1][jj * nmp], t1.data(), mp, tb.rot(je));
      for (int j = 0; j < mp; j++)
        for (int k = 0; k <= j; k++) {
          cd acc = 0;
          for (int n = 0; n <= j - std::abs(k); n++) {
            double cnm = std::pow(-1.0, n) * anm[ifull(n, 0)] * anm[ifull(j - n, k)] / anm[ifull(j, k)] *
                         std::pow(rh, n);
            acc += t1[isym(j - n, k)] * cnm;
          }
          t2[isym(j, k)] = acc;
        }
      spharot(t2.data(), t1.data(), mp, tb.rot(je + 512));
      for (int j = 0; j < nmp; j++) M[lev][ib * nmp + j] += t1[j];
    }
  }

  // Steps 4-6. M2L at level 2 (all non-adjacent boxes), then for
  // lev = 3..lmax: L2L from the parent (kernel/l2l.cxx:13-84) and M2L over
  // the interaction list (kernel/m2l.cxx:13-93).
  auto m2l_level = [&](int lev, const std::vector<std::vector<int>>& lists) {
    double rb = (double)(cfg->rd / (float)(1 << lev));
    for (size_t ii = 0; ii < lists.size(); ii++) {
      int ci[3];
      key_decode(tr.ki[lev][ii], ci);
      for (int jj : lists[ii]) {
        int cj[3];
        key_decode(tr.kj[lev][jj], cj);
        double x = (ci[0] - cj[0]) * rb, y = (ci[1] - cj[1]) * rb, z = (ci[2] - cj[2]) * rb;
        int nc[3] = {ci[0] - cj[0] + 3, ci[1] - cj[1] + 3, ci[2] - cj[2] + 3};
        int je = key_encode(nc, 3);
        double rh = std::sqrt(x * x + y * y + z * z) + s.rho_eps;
        spharot(&M[lev][jj * nmp], t1.data(), mp, tb.rot(je));
        for (int j = 0; j < mp; j++)
          for (int k = 0; k <= j; k++) {
            cd acc = 0;
            for (int n = k; n < mp; n++) {
              double cnm = tb.sr[(size_t)ifull(j, k) * mp * mp + ifull(n, k)] / std::pow(rh, j + n + 1);
              acc += t1[isym(n, k)] * cnm;
            }
            t2[isym(j, k)] = acc;
          }
        spharot(t2.data(), t1.data(), mp, tb.rot(je + 512));
        for (int j = 0; j < nmp; j++) L[lev][ii * nmp + j] += t1[j];
      }
    }
  };
  {
    std::vector<std::vector<int>> lists;
    build_lists(tr.ki[2], tr.kj[2], 2, 1, lists);
    record_lists(2, 1, lists);
    m2l_level(2, lists);
  }
  for (int lev = 3; lev <= lmax; lev++) {
    double rb = (double)(cfg->rd / (float)(1 << lev));
    double rh = rb * std::sqrt(3.0) / 2;
    for (size_t ii = 0; ii < tr.ki[lev].size(); ii++) {
      int ck = tr.ki[lev][ii];
      int ip = find_box(tr.ki[lev - 1], ck / 8);
      int c[3];
      key_decode(ck % 8, c);
      int nc[3] = {2 * c[0] + 2, 2 * c[1] + 2, 2 * c[2] + 2};
      int je = key_encode(nc, 3);
      spharot(&L[lev - 1][ip * nmp], t1.data(), mp, tb.rot(je));
      for (int j = 0; j < mp; j++)
        for (int k = 0; k <= j; k++) {
          cd acc = 0;
          for (int n = j; n < mp; n++) {
            double cnm = anm[ifull(n - j, 0)] * anm[ifull(j, k)] / anm[ifull(n, k)] * std::pow(rh, n - j);
            acc += t1[isym(n, k)] * cnm;
          }
          t2[isym(j, k)] = acc;
        }
      spharot(t2.data(), t1.data(), mp, tb.rot(je + 512));
      for (int j = 0; j < nmp; j++) L[lev][ii * nmp + j] = t1[j];
    }
    std::vector<std::vector<int>> lists;
    build_lists(tr.ki[lev], tr.kj[lev], lev, 2, lists);
    record_lists(lev, 2, lists);
    m2l_level(lev, lists);
  }

  // Step 7. L2P at lmax (kernel/G_l2p.cxx:11-80, kernel/Gn_l2p.cxx:11-72).
  for (size_t ii = 0; ii < tr.ki[lmax].size(); ii++) {
    int c[3];
    key_decode(tr.ki[lmax][ii], c);
    double xc = cfg->xmin + (c[0] + 0.5) * rbl;
    double yc = cfg->ymin + (c[1] + 0.5) * rbl;
    double zc = cfg->zmin + (c[2] + 0.5) * rbl;
    const cd* ax = &L[lmax][ii * nmp];
    for (int i = tr.li0[ii]; i <= tr.li1[ii]; i++) {
      double x = X[i] - xc, y = Y[i] - yc, z = Z[i] - zc;
      double r = std::sqrt(x * x + y * y + z * z) + s.rho_eps;
      double th = polar(z, r);
      double ph = azimuth(x, y, s);
      multipoled(th, mp, fac, bnm.data(), bth.data());
      double g = 0, gr = 0, gth = 0, gph = 0;
      for (int n = 0; n < mp; n++) {
        int nm = ifull(n, 0), ns = isym(n, 0);
        double rn = std::pow(r, n), rn1 = n * std::pow(r, n - 1);
        g += std::real(rn * bnm[nm] * ax[ns]);
        gr += std::real(rn1 * bnm[nm] * ax[ns]);
        gth += std::real(rn * bth[nm] * ax[ns]);
        for (int m = 1; m <= n; m++) {
          nm = ifull(n, m);
          ns = isym(n, m);
          cd eim = std::exp(cd(0, m * ph));
          cd rs = rn * bnm[nm] * eim;
          cd rr = rn1 * bnm[nm] * eim;
          cd rt = rn * bth[nm] * eim;
          cd rp = m * rn * bnm[nm] * eim * cd(0, 1);
          g += 2 * std::real(rs * ax[ns]);
          gr += 2 * std::real(rr * ax[ns]);
          gth += 2 * std::real(rt * ax[ns]);
          gph += 2 * std::real(rp * ax[ns]);
        }
      }
      double st = std::sin(th), ct = std::cos(th), sp = std::sin(ph), cp = std::cos(ph);
      double ex = st * cp * gr + ct * cp / r * gth - sp / r / st * gph;
      double ey = st * sp * gr + ct * sp / r * gth + cp / r / st * gph;
      double ez = ct * gr - st / r * gth;
      if (neq == 1) {
        add_out(i, -s.coef * (NX[i] * ex + NY[i] * ey + NZ[i] * ez), 0, 0, 0);
      } else {
        add_out(i, s.coef * g, s.coef * ex, s.coef * ey, s.coef * ez);
      }
    }
  }

  for (int i = 0; i < ni; i++) {
    int o = tr.perm_i[i];
    double v = s.ref ? (double)Vf[i] : V[i];
    pot[o] = v;
    if (neq == 0) {
      if (gx) gx[o] = s.ref ? (double)GXf[i] : GX[i];
      if (gy) gy[o] = s.ref ? (double)GYf[i] : GY[i];
      if (gz) gz[o] = s.ref ? (double)GZf[i] : GZ[i];
    }
  }
  g_np = nmp;
  for (int w = 0; w < 2; w++) exp_rec[w].clear();
  for (int lev = lmax; lev >= 2; lev--) {
    for (const cd& v : M[lev]) { exp_rec[0].push_back(v.real()); exp_rec[0].push_back(v.imag()); }
    for (const cd& v : L[lev]) { exp_rec[1].push_back(v.real()); exp_rec[1].push_back(v.imag()); }
  }
  return 0;
}

long oracle_record_size(int kind) { return (kind >= 0 && kind < 9) ? (long)rec[kind].size() : -1; }
int oracle_record_copy(int kind, int* dst) {
  if (kind < 0 || kind >= 9) return -1;
  if (!rec[kind].empty()) std::memcpy(dst, rec[kind].data(), rec[kind].size() * sizeof(int));
  return 0;
}
long oracle_expansion_size(int which) { return (which == 0 || which == 1) ? (long)exp_rec[which].size() : -1; }
int oracle_expansion_copy(int which, double* dst) {
  if (which != 0 && which != 1) return -1;
  if (!exp_rec[which].empty()) std::memcpy(dst, exp_rec[which].data(), exp_rec[which].size() * sizeof(double));
  return 0;
}

int oracle_direct(int neq, double eps2, int exclude_self, int coef_ref_pi, int ni, int nj, int i0,
                  int i1, const float* tx, const float* ty, const float* tz, const float* tnx,
                  const float* tny, const float* tnz, const float* sx, const float* sy,
                  const float* sz, const float* snx, const float* sny, const float* snz,
                  const float* q, double* pot, double* gx, double* gy, double* gz) {
  (void)ni;
  if (neq != 0 && neq != 1 && neq != 2) return -1;
  const double coef = coef_ref_pi ? 0.25 / kPiF : 0.25 / M_PI;
  for (int i = i0; i < i1; i++) {
    double p = 0, fx = 0, fy = 0, fz = 0;
    for (int j = 0; j < nj; j++) {
      double dx, dy, dz;
      if (coef_ref_pi) {  // float differences, as kernel/G_dir.cxx:15-17
        dx = tx[i] - sx[j]; dy = ty[i] - sy[j]; dz = tz[i] - sz[j];
      } else {
        dx = (double)tx[i] - sx[j]; dy = (double)ty[i] - sy[j]; dz = (double)tz[i] - sz[j];
      }
      if (exclude_self && dx == 0 && dy == 0 && dz == 0) continue;
      double r2 = dx * dx + dy * dy + dz * dz + eps2;
      double rinv = 1.0 / std::sqrt(r2);
      double r3 = coef * q[j] * rinv * rinv * rinv;
      if (neq == 0) {
        p += coef * q[j] * rinv;
        fx -= dx * r3; fy -= dy * r3; fz -= dz * r3;
      } else if (neq == 1) {
        p += (dx * tnx[i] + dy * tny[i] + dz * tnz[i]) * r3;
      } else {
        p += (dx * snx[j] + dy * sny[j] + dz * snz[j]) * r3;
      }
    }
    pot[i - i0] = p;
    if (neq == 0) {
      if (gx) gx[i - i0] = fx;
      if (gy) gy[i - i0] = fy;
      if (gz) gz[i - i0] = fz;
    }
  }
  return 0;
}

}  // extern "C"

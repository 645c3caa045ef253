// C-ABI driver around the reference's own CPU FMM, built from the reference's
// sources by oracle/Makefile into oracle/_ref/libfmmref_mp<mp>.so (test
// infrastructure: used only by tests/ and by bench.py's CPU baseline).
//
// It reproduces the call sequence of the reference's test driver
// (test/test.cxx:106-116: boxpart, sorti, sortj, boxallocate, alloc(1), fmm,
// unsorti, unsortj, dealloc(1)) on caller-supplied arrays, and records the
// tree (permutations, box keys, leaf ranges) and every list ijbox() builds so
// that the GPU tree can be compared with it bit for bit.
//
// One deliberate change, made at link time the way the reference swaps its own
// kernels (test/Makefile:27-41): this file supplies ifbox() instead of
// fmm/ifbox.cxx.  The shipped fmm() asks for neighbour mode 3 at level 2
// (fmm/fmm.cxx:104), which ijbox() does not implement (fmm/ijbox.cxx:30,54,74),
// so the stale near-field list is reused for the level-2 M2L and the result is
// inf.  Here mode 3 is mapped to mode 1 (every non-adjacent box at level 2),
// which is what the level-2 step needs.
//
// A second link-time replacement: multipoleh() instead of
// kernel/multipoleh.cxx, whose Bessel buffer (kernel/multipoleh.cxx:10,
// double inr[mpcmp], mp entries) is one entry short of what in() writes
// (nb + 1 = mp + 1, kernel/in.cxx:34) -- a stack overflow that crashes the
// reference's Yukawa FMM (neq 10).  The replacement below has the longer
// buffer and otherwise the same recurrences in the same order.
#define MAIN
#include "../include/constants.h"
#include <arrays.h>
#undef MAIN

#include <vector>

extern void nlevel(int);
extern void boxpart(int, int);
extern void sorti(int&);
extern void sortj(int&);
extern void unsorti(int&);
extern void unsortj(int&);
extern void boxallocate(int, int, int, int);
extern void alloc(int);
extern void dealloc(int);
extern void fmm(int, int, int);
extern void ijbox(int, int, int, int);
extern void G_dir(int, int, int, int);
extern void Gni_dir(int, int, int, int);
extern void Gnj_dir(int, int, int, int);
extern void Helmholtz_G_dir(int, int, int, int);

static std::vector<int> g_lists;   // [lev, neib, lbi, lbj, nij[lbi], entries...] per ifbox call
static std::vector<int> g_perm_i, g_perm_j, g_nfi, g_nfj, g_nlbi, g_nlbj, g_ndi, g_ndj;
static int g_nbnet_i = 0, g_nbnet_j = 0;

// Replacement for fmm/ifbox.cxx:7-13 (see the header comment for why).
void ifbox(int mi, int mj, int nmp, int lbi, int lbj, int& lbjr, int lev, int neib) {
  (void)mi; (void)mj; (void)nmp;
  if (neib == 3) neib = 1;
  ijbox(lbi, lbj, lev, neib);
  lbjr = lbj;
  g_lists.push_back(lev);
  g_lists.push_back(neib);
  g_lists.push_back(lbi);
  g_lists.push_back(lbj);
  for (int ii = 0; ii < lbi; ii++) g_lists.push_back(nij[ii]);
  for (int ii = 0; ii < lbi; ii++)
    for (int k = 0; k < nij[ii]; k++) g_lists.push_back(neij[ii][k]);
}

extern void in(double, double, const int, double*, int);

// Replacement for kernel/multipoleh.cxx:8-33 (see the header comment): the
// scaled modified spherical Bessel values i_n(lambda rh) (n = 0..mp, one entry
// more than the reference's buffer holds) times (2n + 1) fac(n,m)^2
// P_n^m(cos al) into bnm[n n + n + m], with the associated Legendre functions
// by the upward recurrence in n from P_m^m = (-1)^m (2m-1)!! sin^m(al) --
// operation for operation as the reference, so that the outputs are bit
// identical; `be` is unused there too.
void multipoleh(double rh, double al, double be, int mpx) {
  (void)be;
  double inr[mpcmp + 1];
  in(scale, rh * lambda, mpx, inr, 0);
  const double c = cos(al);
  const double s = sqrt((1 - c) * (1 + c));
  double pmm = 1, odd = 1;
  for (int m = 0; m < mpx; m++) {
    double pcur = pmm;  // P_m^m
    int k = m * m + 2 * m;
    bnm[k] = inr[m] * (2 * m + 1) * fac[k] * fac[k] * pcur;
    double pprev = pcur;
    pcur = c * (2 * m + 1) * pcur;  // P_{m+1}^m
    for (int n = m + 1; n < mpx; n++) {
      k = n * n + n + m;
      bnm[k] = inr[n] * (2 * n + 1) * fac[k] * fac[k] * pcur;
      const double pp = pprev;
      pprev = pcur;
      pcur = (c * (2 * n + 1) * pprev - (n + m) * pp) / (n - m + 1);
    }
    pmm = -pmm * odd * s;
    odd += 2;
  }
}

static void alloc_points(int n, int nbox) {
  int m = n > 0 ? n : 1;
  int mc = m > nbox ? m : nbox;
  xi = new float[m]; yi = new float[m]; zi = new float[m];
  gxi = new float[m]; gyi = new float[m]; gzi = new float[m]; vi = new float[m];
  xj = new float[m]; yj = new float[m]; zj = new float[m];
  gxj = new float[m]; gyj = new float[m]; gzj = new float[m]; vj = new float[m];
  nfn = new int[m]; na = new int[m]; nb = new int[m]; nd = new int[m];
  nc = new int[mc];     // csort uses nc[0..nbmax) (sort/csort.cxx:8)
  nbi = new int[m]; nbj = new int[m];
  sortd = new float[m];
  tfmm = new double[100];
  for (int i = 0; i < 100; i++) tfmm[i] = 0;
}

static void free_points() {
  delete[] xi; delete[] yi; delete[] zi; delete[] gxi; delete[] gyi; delete[] gzi; delete[] vi;
  delete[] xj; delete[] yj; delete[] zj; delete[] gxj; delete[] gyj; delete[] gzj; delete[] vj;
  delete[] nfn; delete[] na; delete[] nb; delete[] nc; delete[] nd; delete[] nbi; delete[] nbj;
  delete[] sortd; delete[] tfmm;
}

extern "C" {

int ref_mp(void) { return mp; }

// Runs the reference fmm(ni,nj,neq) on unsorted inputs.  Outputs are written in
// the caller's (unsorted) order.  neq: 0 G (potential+gradient), 1 Gni, 2 Gnj,
// 10 Yukawa.  For neq 1 the target normals are (tnx,tny,tnz); for neq 2 the
// source normals are (snx,sny,snz).  lmax_in <= 0 picks lmax with nlevel().
// timings (nullable) receives the 100 tfmm buckets.
int ref_fmm(int ni, int nj, int neq, int lmax_in,
            float xmin_in, float ymin_in, float zmin_in, float rd_in, double lambda_in,
            const float* tx, const float* ty, const float* tz,
            const float* tnx, const float* tny, const float* tnz,
            const float* sx, const float* sy, const float* sz,
            const float* snx, const float* sny, const float* snz, const float* sq,
            float* v_out, float* gx_out, float* gy_out, float* gz_out, double* timings) {
  nprocs = 1; myrank = 0; umem = 0; ncheck = 0;
  static double tfmm_nlevel[100];  // nlevel() adds its time to tfmm[0] before the arrays exist
  if (lmax_in > 0) {
    lmax = lmax_in;
  } else {
    tfmm = tfmm_nlevel;
    nlevel(nj);
  }
  nbmax = 1 << 3 * lmax;
  xmin = xmin_in; ymin = ymin_in; zmin = zmin_in; rd = rd_in;
  lambda = lambda_in;
  int n = ni > nj ? ni : nj;
  alloc_points(n, nbmax);
  for (int i = 0; i < ni; i++) {
    xi[i] = tx[i]; yi[i] = ty[i]; zi[i] = tz[i];
    gxi[i] = tnx ? tnx[i] : 0.f; gyi[i] = tny ? tny[i] : 0.f; gzi[i] = tnz ? tnz[i] : 0.f;
    vi[i] = 0.f;
  }
  for (int j = 0; j < nj; j++) {
    xj[j] = sx[j]; yj[j] = sy[j]; zj[j] = sz[j];
    gxj[j] = snx ? snx[j] : 0.f; gyj[j] = sny ? sny[j] : 0.f; gzj[j] = snz ? snz[j] : 0.f;
    vj[j] = sq[j];
  }
  if (neq == 10) {  // scale choice of test/testh.cxx:119-123
    scale = (rd * lambda > 1) ? 1 / rd : lambda;
  }
  g_lists.clear();
  boxpart(ni, nj);
  sorti(ni);
  sortj(nj);
  g_perm_i.assign(nbi, nbi + ni);
  g_perm_j.assign(nbj, nbj + nj);
  boxallocate(0, ni, 0, nj);
  alloc(1);
  fmm(ni, nj, neq);
  g_nbnet_i = nbnet; g_nbnet_j = nbnet;
  g_nlbi.assign(nlbi, nlbi + lmax);
  g_nlbj.assign(nlbj, nlbj + lmax);
  g_nfi.assign(nfi, nfi + nbnet);
  g_nfj.assign(nfj, nfj + nbnet);
  // Leaf ranges are the level-lmax part written by boxdatai/boxdataj; the
  // first ifbox call (P2P list at lmax) carries the leaf counts.
  g_ndi.clear(); g_ndj.clear();
  if (g_lists.size() >= 4) {
    int lbi_leaf = g_lists[2], lbj_leaf = g_lists[3];
    for (int i = 0; i < lbi_leaf; i++) { g_ndi.push_back(ndi[0][i]); g_ndi.push_back(ndi[1][i]); }
    for (int i = 0; i < lbj_leaf; i++) { g_ndj.push_back(ndj[0][i]); g_ndj.push_back(ndj[1][i]); }
  }
  unsorti(ni);
  unsortj(nj);
  for (int i = 0; i < ni; i++) {
    v_out[i] = vi[i];
    if (gx_out) gx_out[i] = gxi[i];
    if (gy_out) gy_out[i] = gyi[i];
    if (gz_out) gz_out[i] = gzi[i];
  }
  if (timings) for (int i = 0; i < 100; i++) timings[i] = tfmm[i];
  dealloc(1);
  free_points();
  return lmax;
}

// Record accessors (valid after ref_fmm).  kind: 0 perm_i, 1 perm_j, 2 nfi,
// 3 nfj, 4 nlbi, 5 nlbj, 6 ndi pairs, 7 ndj pairs, 8 list stream.
static const std::vector<int>* rec(int kind) {
  switch (kind) {
    case 0: return &g_perm_i; case 1: return &g_perm_j; case 2: return &g_nfi;
    case 3: return &g_nfj; case 4: return &g_nlbi; case 5: return &g_nlbj;
    case 6: return &g_ndi; case 7: return &g_ndj; case 8: return &g_lists;
  }
  return 0;
}
long ref_record_size(int kind) { const std::vector<int>* v = rec(kind); return v ? (long)v->size() : -1; }
int ref_record_copy(int kind, int* dst) {
  const std::vector<int>* v = rec(kind);
  if (!v) return -1;
  for (size_t i = 0; i < v->size(); i++) dst[i] = (*v)[i];
  return 0;
}

// The reference direct sums (kernel/G_dir.cxx:6-30, Gni_dir.cxx:6-21,
// Gnj_dir.cxx:6-21, Helmholtz_G_dir.cxx) over all targets and sources.
int ref_direct(int ni, int nj, int neq, double lambda_in,
               const float* tx, const float* ty, const float* tz,
               const float* tnx, const float* tny, const float* tnz,
               const float* sx, const float* sy, const float* sz,
               const float* snx, const float* sny, const float* snz, const float* sq,
               float* v_out, float* gx_out, float* gy_out, float* gz_out) {
  lambda = lambda_in;
  int n = ni > nj ? ni : nj;
  alloc_points(n, 1);
  for (int i = 0; i < ni; i++) {
    xi[i] = tx[i]; yi[i] = ty[i]; zi[i] = tz[i];
    gxi[i] = tnx ? tnx[i] : 0.f; gyi[i] = tny ? tny[i] : 0.f; gzi[i] = tnz ? tnz[i] : 0.f;
    vi[i] = 0.f;
  }
  for (int j = 0; j < nj; j++) {
    xj[j] = sx[j]; yj[j] = sy[j]; zj[j] = sz[j];
    gxj[j] = snx ? snx[j] : 0.f; gyj[j] = sny ? sny[j] : 0.f; gzj[j] = snz ? snz[j] : 0.f;
    vj[j] = sq[j];
  }
  if (neq == 0) G_dir(0, ni - 1, 0, nj - 1);
  else if (neq == 1) Gni_dir(0, ni - 1, 0, nj - 1);
  else if (neq == 2) Gnj_dir(0, ni - 1, 0, nj - 1);
  else if (neq == 10) Helmholtz_G_dir(0, ni - 1, 0, nj - 1);
  for (int i = 0; i < ni; i++) {
    v_out[i] = vi[i];
    if (gx_out) gx_out[i] = gxi[i];
    if (gy_out) gy_out[i] = gyi[i];
    if (gz_out) gz_out[i] = gzi[i];
  }
  free_points();
  return 0;
}

}  // extern "C"

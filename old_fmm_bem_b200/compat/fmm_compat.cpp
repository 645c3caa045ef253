// Reference-compatible entry points over libfmmb's C ABI.
//
// A reference application (test/test.cxx, bio/main.cxx, biobem/main.cxx) calls
//   void fmm(int mi, int mj, int neq);                       // fmm/fmm.cxx:29
//   void G_dir(int n0, int n1, int n2, int n3);              // kernel/G_dir.cxx:6
//   void Gni_dir(int n0, int n1, int n2, int n3);            // kernel/Gni_dir.cxx:6
//   void Gnj_dir(int n0, int n1, int n2, int n3);            // kernel/Gnj_dir.cxx:6
// over the global particle arrays of include/arrays.h:5-12 and the geometry
// globals of include/constants.h:57-62 (lmax, xmin, ymin, zmin, rd).  Linking
// this file (and libfmmb.so) in place of fmm/fmm.o and the kernel objects --
// the link-time substitution the reference's Makefiles already use to switch
// between CPU and GPU kernels (test/Makefile:27-41) -- sends those calls to
// the GPU.  The application keeps defining the globals; this file only
// declares them.
//
// Behaviour matches the reference:
//   * fmm: vi is overwritten with the result; for neq 0 gxi/gyi/gzi are
//     overwritten with the gradient (fmm/fmm.cxx:46-53); for neq 1 gxi.. are
//     read as target normals, for neq 2 gxj.. as source normals, and neither
//     is modified.  Inputs may be in any order (the reference requires
//     sorti/sortj first; the GPU tree sorts internally and returns results in
//     the caller's order, so presorted inputs work unchanged).
//   * *_dir: overwrite vi (and gx.. for G) on targets n0..n1 (inclusive) from
//     sources n2..n3 (inclusive).
// The expansion order is the reference's compile-time mp - 1; here it is
// fmmb_compat_set_order(p) (default 8, the shipped mp = 9).  Reference
// semantics (eps = 1e-6f, single-precision pi, float tables) are used so that
// results are those of the reference (to its float output rounding).
// Errors: the reference aborts through CUDA_SAFE_CALL; here a failing call
// prints fmmb_last_error() to stderr and leaves the outputs unchanged.
#include <cstdio>

#include "../../include/fmmb.h"

extern float *xi, *yi, *zi, *gxi, *gyi, *gzi, *vi;
extern float *xj, *yj, *zj, *gxj, *gyj, *gzj, *vj;
extern int lmax;
extern float xmin, ymin, zmin, rd;
extern double lambda;  // Yukawa screening (include/constants.h:60)

namespace {
int g_order = 8;
int g_precision = FMMB_FP64;

bool report(int rc, const char* where) {
  if (rc == FMMB_OK) return true;
  std::fprintf(stderr, "fmmb (%s): %s\n", where, fmmb_last_error());
  return false;
}

// The Yukawa kernel has no reference-semantics mode: its near field takes the
// reference's conventions through the plan's eps2 (1e-6f added to r^2,
// kernel/Helmholtz_G_p2p.cxx:21) and self pairs included; wavenumber = lambda.
void yukawa_config(fmmb_config& cfg) {
  cfg.semantics = FMMB_SEM_ACCURATE;
  cfg.eps2 = (double)1e-6f;
  cfg.exclude_self = 0;
  cfg.wavenumber = lambda;
}

// One plan per (kernel, order, depth, precision, Yukawa lambda), rebuilt when they change.
struct Cached {
  fmmb_plan* plan = nullptr;
  int kernel = -1, p = -1, lmax = -1, precision = -1;
  double lam = 0;
};
Cached g_fmm[4];  // neq 0, 1, 2, 10

fmmb_plan* plan_for(int kernel, int levels) {
  Cached& c = g_fmm[kernel == FMMB_YUKAWA ? 3 : kernel];
  const double lam = kernel == FMMB_YUKAWA ? lambda : 0.0;
  if (c.plan && c.p == g_order && c.lmax == levels && c.precision == g_precision && c.lam == lam) return c.plan;
  if (c.plan) fmmb_plan_destroy(c.plan);
  c.plan = nullptr;
  fmmb_config cfg;
  fmmb_config_init(&cfg);
  cfg.kernel = kernel;
  cfg.p = g_order;
  cfg.lmax = levels;
  cfg.precision = g_precision;
  cfg.semantics = FMMB_SEM_REFERENCE;
  if (kernel == FMMB_YUKAWA) yukawa_config(cfg);
  if (!report(fmmb_plan_create(&cfg, &c.plan), "plan_create")) return nullptr;
  c.kernel = kernel;
  c.p = g_order;
  c.lmax = levels;
  c.precision = g_precision;
  c.lam = lam;
  return c.plan;
}

void direct(int neq, int n0, int n1, int n2, int n3) {
  const int ni = n1 - n0 + 1, nj = n3 - n2 + 1;
  if (ni <= 0 || nj <= 0) return;
  fmmb_config cfg;
  fmmb_config_init(&cfg);
  cfg.kernel = neq;
  cfg.lmax = 2;
  cfg.semantics = FMMB_SEM_REFERENCE;
  if (neq == FMMB_YUKAWA) yukawa_config(cfg);
  fmmb_plan* pl = nullptr;
  if (!report(fmmb_plan_create(&cfg, &pl), "plan_create")) return;
  if (report(fmmb_set_geometry(pl, ni, xi + n0, yi + n0, zi + n0, neq == 1 ? gxi + n0 : nullptr,
                               neq == 1 ? gyi + n0 : nullptr, neq == 1 ? gzi + n0 : nullptr, nj, xj + n2, yj + n2,
                               zj + n2, neq == 2 ? gxj + n2 : nullptr, neq == 2 ? gyj + n2 : nullptr,
                               neq == 2 ? gzj + n2 : nullptr, nullptr),
             "set_geometry")) {
    double* pot = new double[ni];
    double* grad = neq == 0 ? new double[3 * (size_t)ni] : nullptr;
    if (report(fmmb_direct_f64(pl, vj + n2, 0, ni, pot, grad), "direct")) {
      for (int i = 0; i < ni; i++) {
        vi[n0 + i] = (float)pot[i];
        if (grad) {
          gxi[n0 + i] = (float)grad[i];
          gyi[n0 + i] = (float)grad[ni + i];
          gzi[n0 + i] = (float)grad[2 * (size_t)ni + i];
        }
      }
    }
    delete[] pot;
    delete[] grad;
  }
  fmmb_plan_destroy(pl);
}
}  // namespace

extern "C" void fmmb_compat_set_order(int p) { g_order = p; }
extern "C" void fmmb_compat_set_precision(int precision) { g_precision = precision; }

void fmm(int mi, int mj, int neq) {
  if (neq != FMMB_LAPLACE_G && neq != FMMB_LAPLACE_GNI && neq != FMMB_LAPLACE_GNJ && neq != FMMB_YUKAWA) {
    std::fprintf(stderr, "fmmb: fmm(neq=%d) not supported (0, 1, 2, 10)\n", neq);
    return;
  }
  fmmb_plan* pl = plan_for(neq, lmax);
  if (!pl) return;
  const float bbox[4] = {xmin, ymin, zmin, rd};
  if (!report(fmmb_set_geometry(pl, mi, xi, yi, zi, neq == 1 ? gxi : nullptr, neq == 1 ? gyi : nullptr,
                                neq == 1 ? gzi : nullptr, mj, xj, yj, zj, neq == 2 ? gxj : nullptr,
                                neq == 2 ? gyj : nullptr, neq == 2 ? gzj : nullptr, bbox),
              "set_geometry"))
    return;
  if (neq == FMMB_LAPLACE_G) {
    float* grad = new float[3 * (size_t)mi];
    if (report(fmmb_evaluate(pl, vj, vi, grad), "evaluate"))
      for (int i = 0; i < mi; i++) {
        gxi[i] = grad[i];
        gyi[i] = grad[mi + i];
        gzi[i] = grad[2 * (size_t)mi + i];
      }
    delete[] grad;
  } else {
    report(fmmb_evaluate(pl, vj, vi, nullptr), "evaluate");
    if (neq == FMMB_YUKAWA)  // the reference zeroes the gradient outputs for neq 10 (fmm/fmm.cxx:46-53)
      for (int i = 0; i < mi; i++) gxi[i] = gyi[i] = gzi[i] = 0.f;
  }
}

void G_dir(int n0, int n1, int n2, int n3) { direct(FMMB_LAPLACE_G, n0, n1, n2, n3); }
void Gni_dir(int n0, int n1, int n2, int n3) { direct(FMMB_LAPLACE_GNI, n0, n1, n2, n3); }
void Gnj_dir(int n0, int n1, int n2, int n3) { direct(FMMB_LAPLACE_GNJ, n0, n1, n2, n3); }

// kernel/Helmholtz_G_dir.cxx:6: the Yukawa direct sum on targets n0..n1 from
// sources n2..n3 (inclusive), eps = 1e-6 on r^2, self pairs included
void Helmholtz_G_dir(int n0, int n1, int n2, int n3) { direct(FMMB_YUKAWA, n0, n1, n2, n3); }

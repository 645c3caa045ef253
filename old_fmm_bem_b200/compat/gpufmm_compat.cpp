// Link-time replacement of the reference's GPU library entry points p2pgpu_,
// p2mgpu_, m2lgpu_ and l2pgpu_ (libgpu/gpufmm.cu:57, 200, 336, 481) over
// libfmmb's fmmb_gpu_p2p / _p2m / _m2l / _l2p.
//
// The reference builds its GPU variant from the host-side kernel files
// (kernel/G_p2p_gpu.cxx, Gni_p2p_gpu.cxx, Gnj_p2p_gpu.cxx, G_p2m_gpu.cxx,
// Gn_p2m_gpu.cxx, m2m_gpu.cxx, m2l_gpu.cxx, l2l_gpu.cxx, G_l2p_gpu.cxx,
// Gn_l2p_gpu.cxx: they pack targets, sources and coefficients in blocks and
// describe them in the record array nvecd) linked against libgpu
// (test/Makefile:37-41, 75-76).  Linking this file and libfmmb.so in place of
// libgpu keeps those host files unchanged: same symbols (C++ linkage, as
// libgpu/gpufmm.cu defines them), same arguments, same record formats, same
// outputs.  Not used: `op` (the caller's flop estimate) and the table
// arguments (fac; ynm and the rotation tables dnm of m2lgpu_): the library
// builds the same operators itself.  The reference's GPU translations are
// valid only for mp <= 5 (libgpu/var.h:2, libgpu/m2l.cu:69); these are valid
// for every mp with mp (mp+1) / 2 <= 64, the record block size.
//
// Errors: libgpu exits through CUDA_SAFE_CALL; so does this shim, after
// printing fmmb_last_error().
#include <cstdio>
#include <cstdlib>

#include "../../include/fmmb.h"

void p2pgpu_(int nvecd[], double* op, float xi[], float yi[], float zi[], float gxi[], float gyi[], float gzi[],
             float vi[], float xj[], float yj[], float zj[], float gxj[], float gyj[], float gzj[], float vj[]) {
  (void)op;
  const int rc = fmmb_gpu_p2p(nvecd, xi, yi, zi, gxi, gyi, gzi, vi, xj, yj, zj, gxj, gyj, gzj, vj);
  if (rc != FMMB_OK) {
    std::fprintf(stderr, "p2pgpu_: %s\n", fmmb_last_error());
    std::exit(EXIT_FAILURE);
  }
}

void p2mgpu_(int nvecd[], double* op, double* rb, double* xmin, double* ymin, double* zmin, float xjg[], float yjg[],
             float zjg[], float gxjg[], float gyjg[], float gzjg[], float vjg[], float brex[], float bimx[],
             float fac[]) {
  (void)op;
  (void)fac;
  const int rc = fmmb_gpu_p2m(nvecd, rb, xmin, ymin, zmin, xjg, yjg, zjg, gxjg, gyjg, gzjg, vjg, brex, bimx);
  if (rc != FMMB_OK) {
    std::fprintf(stderr, "p2mgpu_: %s\n", fmmb_last_error());
    std::exit(EXIT_FAILURE);
  }
}

void l2pgpu_(int nvecd[], double* op, double* rb, double* xmin, double* ymin, double* zmin, float xig[], float yig[],
             float zig[], float gxig[], float gyig[], float gzig[], float vig[], float arex[], float aimx[],
             float fac[]) {
  (void)op;
  (void)fac;
  const int rc = fmmb_gpu_l2p(nvecd, rb, xmin, ymin, zmin, xig, yig, zig, gxig, gyig, gzig, vig, arex, aimx);
  if (rc != FMMB_OK) {
    std::fprintf(stderr, "l2pgpu_: %s\n", fmmb_last_error());
    std::exit(EXIT_FAILURE);
  }
}

void m2lgpu_(int nvecd[], double* op, double* rb, float arex[], float aimx[], float brex[], float bimx[],
             float ynmre[], float ynmim[], float dnmre[], float dnmim[]) {
  (void)op;
  (void)ynmre;
  (void)ynmim;
  (void)dnmre;
  (void)dnmim;
  const int rc = fmmb_gpu_m2l(nvecd, rb, arex, aimx, brex, bimx);
  if (rc != FMMB_OK) {
    std::fprintf(stderr, "m2lgpu_: %s\n", fmmb_last_error());
    std::exit(EXIT_FAILURE);
  }
}

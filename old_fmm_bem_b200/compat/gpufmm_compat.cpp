// Link-time replacement of the reference's GPU library entry point for the
// near field, p2pgpu_ (libgpu/gpufmm.cu:57-197), over libfmmb's
// fmmb_gpu_p2p.
//
// The reference builds its GPU variant from the host-side kernel files
// (kernel/G_p2p_gpu.cxx, Gni_p2p_gpu.cxx, Gnj_p2p_gpu.cxx: they pack targets
// in blocks of 128 and source ranges in the record array nvecd) linked
// against libgpu (test/Makefile:37-41, 75-76).  Linking this file and
// libfmmb.so in place of libgpu's p2pgpu_ keeps those host files unchanged:
// same symbol (C++ linkage, as libgpu/gpufmm.cu defines it), same arguments,
// same record format, same outputs (vi, gxi, gyi, gzi of every packed target
// overwritten: potential and gradient for neq 0, potential and zeros for
// neq 1 and 2).  `op` (the caller's flop estimate) is not used.
//
// The expansion entry points p2mgpu_, m2lgpu_ and l2pgpu_ are not provided:
// their float record formats feed the reference's 2010 kernels, whose M2L is
// valid only for mp <= 5 (libgpu/var.h:2, libgpu/m2l.cu:69); a GPU far field
// is reached through fmm() (fmm_compat.cpp) or the plan API instead.
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

// The reference's batch near-field entry point, p2pgpu_ (libgpu/gpufmm.cu:57-197
// over the kernels of libgpu/G_p2p.cu, Gni_p2p.cu, Gnj_p2p.cu and the record
// walk of libgpu/kernel.cu:1-48), behind fmmb_gpu_p2p.  Its callers
// (kernel/G_p2p_gpu.cxx, Gni_p2p_gpu.cxx, Gnj_p2p_gpu.cxx) pack the targets of
// each leaf in blocks of 128 and describe, per block, the source ranges of its
// neighbour leaves in the integer record array nvecd:
//   nvecd[1] blocks, nvecd[2] record stride, nvecd[3] sources, nvecd[4] kernel (neq)
//   block b: nvecd[b*stride + 10] ranges; range r: first source
//   nvecd[b*stride + 2r + 11], count nvecd[b*stride + 2r + 12]
// Outputs per target: (v, gx, gy, gz) overwritten -- the gradient for neq 0,
// zeros for the normal-derivative kernels, like the reference's kernels.
// Arithmetic as there: eps = 1e-6 added to r^2, FP32 pair terms with 1/(4 pi)
// in float; here each range's FP32 sum over 128 sources is added in FP64.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>

#include "internal.h"

namespace fmmb {
namespace {

constexpr int kBlk = 128;  // targets per block record (the reference's NBLOK0)

template <int NEQ>
__global__ void __launch_bounds__(kBlk) p2p_blocks(const int* __restrict__ rec, const float* __restrict__ tgt,
                                                   const float* __restrict__ src, int nj, float* __restrict__ out) {
  __shared__ float s[7][kBlk];
  const int b = blockIdx.x, t = threadIdx.x, stride = rec[2];
  const int i = b * kBlk + t;
  const float xi = tgt[i], yi = tgt[(size_t)gridDim.x * kBlk + i], zi = tgt[2 * (size_t)gridDim.x * kBlk + i];
  const float nx = tgt[3 * (size_t)gridDim.x * kBlk + i], ny = tgt[4 * (size_t)gridDim.x * kBlk + i],
              nz = tgt[5 * (size_t)gridDim.x * kBlk + i];
  const float eps = 1e-6f, pi14 = (float)(0.25 / M_PI);
  double v = 0, gx = 0, gy = 0, gz = 0;
  const int nr = rec[(size_t)b * stride + 10];
  for (int r = 0; r < nr; r++) {
    const int jb = rec[(size_t)b * stride + 2 * r + 11], js = rec[(size_t)b * stride + 2 * r + 12];
    for (int c0 = 0; c0 < js; c0 += kBlk) {
      __syncthreads();
      const int j = jb + c0 + t;
      if (c0 + t < js && j >= 0 && j < nj)
        for (int k = 0; k < 7; k++) s[k][t] = src[(size_t)k * nj + j];
      else
        for (int k = 0; k < 7; k++) s[k][t] = 0.f;
      __syncthreads();
      const int n = min(kBlk, js - c0);
      float fv = 0, fx = 0, fy = 0, fz = 0;
      for (int jj = 0; jj < n; jj++) {
        const float dx = xi - s[0][jj], dy = yi - s[1][jj], dz = zi - s[2][jj];
        const float rinv = rsqrtf(dx * dx + dy * dy + dz * dz + eps);
        const float rs = pi14 * s[6][jj] * rinv * rinv * rinv;
        if (NEQ == 0) {
          fv += pi14 * s[6][jj] * rinv;
          fx -= dx * rs;
          fy -= dy * rs;
          fz -= dz * rs;
        } else if (NEQ == 1) {
          fv += (dx * nx + dy * ny + dz * nz) * rs;
        } else {
          fv += (dx * s[3][jj] + dy * s[4][jj] + dz * s[5][jj]) * rs;
        }
      }
      v += fv;
      gx += fx;
      gy += fy;
      gz += fz;
    }
  }
  const size_t nt = (size_t)gridDim.x * kBlk;
  out[i] = (float)v;
  out[nt + i] = (float)gx;
  out[2 * nt + i] = (float)gy;
  out[3 * nt + i] = (float)gz;
}

// per-process device buffers of the batch entry point (the reference keeps
// static ones too, libgpu/var.h:11-28)
DevBuf<int> g_rec;
DevBuf<float> g_tgt, g_src, g_out;

}  // namespace
}  // namespace fmmb

using namespace fmmb;

extern "C" int fmmb_gpu_p2p(const int* nvecd, float* xi, float* yi, float* zi, float* gxi, float* gyi, float* gzi,
                            float* vi, const float* xj, const float* yj, const float* zj, const float* gxj,
                            const float* gyj, const float* gzj, const float* vj) {
  try {
    FMMB_REQUIRE(nvecd, FMMB_ERR_ARG, "null record array");
    const int nblock = nvecd[1], stride = nvecd[2], nj = nvecd[3], neq = nvecd[4];
    FMMB_REQUIRE(nblock >= 0 && stride >= 1 && nj >= 0, FMMB_ERR_ARG, "bad block records");
    FMMB_REQUIRE(neq == 0 || neq == 1 || neq == 2, FMMB_ERR_ARG, "p2pgpu_ handles neq 0, 1, 2");
    if (nblock == 0) return FMMB_OK;
    FMMB_REQUIRE(xi && yi && zi && gxi && gyi && gzi && vi && xj && yj && zj && gxj && gyj && gzj && vj, FMMB_ERR_ARG,
                 "null particle array");
    // every range must lie inside the source arrays (checked here, on the host)
    const size_t nrec = (size_t)nblock * stride + 10;
    for (int b = 0; b < nblock; b++) {
      const int nr = nvecd[(size_t)b * stride + 10];
      FMMB_REQUIRE(nr >= 0 && 2 * nr < stride, FMMB_ERR_ARG, "too many source ranges for the record stride");
      for (int r = 0; r < nr; r++) {
        const long long jb = nvecd[(size_t)b * stride + 2 * r + 11], js = nvecd[(size_t)b * stride + 2 * r + 12];
        FMMB_REQUIRE(jb >= 0 && js >= 0 && jb + js <= nj, FMMB_ERR_ARG, "source range outside the source arrays");
      }
    }
    const size_t nt = (size_t)nblock * kBlk;
    g_rec.alloc(nrec);
    g_tgt.alloc(6 * nt);
    g_src.alloc(7 * (size_t)std::max(nj, 1));
    g_out.alloc(4 * nt);
    cudaStream_t st = cudaStreamLegacy;
    FMMB_CUDA(cudaMemcpyAsync(g_rec.get(), nvecd, nrec * sizeof(int), cudaMemcpyHostToDevice, st));
    const float* tin[6] = {xi, yi, zi, gxi, gyi, gzi};
    for (int k = 0; k < 6; k++)
      FMMB_CUDA(cudaMemcpyAsync(g_tgt.get() + k * nt, tin[k], nt * sizeof(float), cudaMemcpyHostToDevice, st));
    const float* sin_[7] = {xj, yj, zj, gxj, gyj, gzj, vj};
    for (int k = 0; k < 7 && nj > 0; k++)
      FMMB_CUDA(cudaMemcpyAsync(g_src.get() + (size_t)k * nj, sin_[k], nj * sizeof(float), cudaMemcpyHostToDevice, st));
    if (neq == 0) p2p_blocks<0><<<nblock, kBlk, 0, st>>>(g_rec.get(), g_tgt.get(), g_src.get(), nj, g_out.get());
    else if (neq == 1) p2p_blocks<1><<<nblock, kBlk, 0, st>>>(g_rec.get(), g_tgt.get(), g_src.get(), nj, g_out.get());
    else p2p_blocks<2><<<nblock, kBlk, 0, st>>>(g_rec.get(), g_tgt.get(), g_src.get(), nj, g_out.get());
    FMMB_CHECK_LAUNCH();
    float* outs[4] = {vi, gxi, gyi, gzi};
    for (int k = 0; k < 4; k++)
      FMMB_CUDA(cudaMemcpyAsync(outs[k], g_out.get() + k * nt, nt * sizeof(float), cudaMemcpyDeviceToHost, st));
    FMMB_CUDA(cudaStreamSynchronize(st));
    return FMMB_OK;
  } catch (const Error& e) {
    set_error(e.msg);
    return e.code;
  }
}

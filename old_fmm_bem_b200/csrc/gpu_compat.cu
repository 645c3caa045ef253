// The reference's batch GPU entry points behind fmmb_gpu_p2p / _p2m / _l2p.
//
// p2pgpu_ (libgpu/gpufmm.cu:57-197 over the kernels of libgpu/G_p2p.cu,
// Gni_p2p.cu, Gnj_p2p.cu and the record walk of libgpu/kernel.cu:1-48).  Its callers
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

#include <map>
#include <memory>
#include <vector>

#include "internal.h"
#include "kernels.h"

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

// per-process device buffers of the batch entry points (the reference keeps
// static ones too, libgpu/var.h:11-28)
DevBuf<int> g_rec;
DevBuf<float> g_tgt, g_src, g_out;

// p2mgpu_ / l2pgpu_: the reference-semantics FP64 P2M / L2P kernels of the plan
// path (kernels_fp64.cu) on the reference's block records.  Their tables (fac,
// rounded to float as the reference stores them) per order, built once.
struct RefTables {
  DevBuf<double> fac;
};
RefTables& ref_tables(int p) {
  static std::map<int, std::unique_ptr<RefTables>> cache;
  auto& t = cache[p];
  if (!t) {
    Operators ops;
    build_static_operators(ops, p, true);
    std::unique_ptr<RefTables> n(new RefTables());
    n->fac.alloc(ops.fac.size());
    FMMB_CUDA(cudaMemcpy(n->fac.get(), ops.fac.data(), ops.fac.size() * sizeof(double), cudaMemcpyHostToDevice));
    t = std::move(n);
  }
  return *t;
}
// reference conventions (eps = 1e-6f on r^2 and radii, single-precision pi)
Sem ref_sem() {
  Sem s;
  s.eps2 = (double)1e-6f;
  s.coef = 0.25 / (double)(float)M_PI;
  s.rho_eps = (double)1e-6f;
  s.ang_eps = (double)1e-6f;
  s.pi_ang = (double)(float)M_PI;
  s.ref = 1;
  s.excl_self = 0;
  return s;
}
constexpr int kBlk1 = 64;  // coefficients / targets per block record (the reference's NBLOK1)

int isym_h(int n, int m) { return n * (n + 1) / 2 + m; }

DevBuf<int> g_keys;
DevBuf<int2> g_leaf;
DevBuf<float4> g_pos, g_nrm;
DevBuf<float> g_q;
DevBuf<double> g_exp, g_pot;

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

namespace {
template <typename F>
int guarded_c(F f) {
  try {
    f();
    return FMMB_OK;
  } catch (const Error& e) {
    set_error(e.msg);
    return e.code;
  }
}
}  // namespace

extern "C" int fmmb_gpu_p2m(const int* nvecd, const double* rb, const double* xmin, const double* ymin,
                            const double* zmin, const float* xj, const float* yj, const float* zj, const float* gxj,
                            const float* gyj, const float* gzj, const float* vj, float* brex, float* bimx) {
  return guarded_c([&] {
    FMMB_REQUIRE(nvecd && rb && xmin && ymin && zmin, FMMB_ERR_ARG, "null argument");
    const int nblock = nvecd[1], stride = nvecd[2], nj = nvecd[3], neq = nvecd[4], mp = nvecd[6];
    FMMB_REQUIRE(neq == 0 || neq == 1, FMMB_ERR_ARG, "p2mgpu_ handles neq 0 (G) and 1 (Gn)");
    FMMB_REQUIRE(mp >= 1 && mp * (mp + 1) / 2 <= kBlk1, FMMB_ERR_ARG, "p2mgpu_ takes mp (mp + 1) / 2 <= 64");
    FMMB_REQUIRE(nblock >= 0 && stride >= 3 && nj >= 0, FMMB_ERR_ARG, "bad block records");
    if (nblock == 0) return;
    FMMB_REQUIRE(xj && yj && zj && gxj && gyj && gzj && vj && brex && bimx, FMMB_ERR_ARG, "null array");
    const int p = mp - 1, K = mp * mp;
    std::vector<int> keys(nblock);
    std::vector<int2> leaf(nblock);
    for (int b = 0; b < nblock; b++) {
      keys[b] = nvecd[(size_t)b * stride + 10];
      leaf[b] = make_int2(nvecd[(size_t)b * stride + 11], nvecd[(size_t)b * stride + 12]);
      FMMB_REQUIRE(keys[b] >= 0 && leaf[b].x >= 0 && leaf[b].y >= 0 && (long long)leaf[b].x + leaf[b].y <= nj,
                   FMMB_ERR_ARG, "block record outside the source arrays");
    }
    std::vector<float4> pos(std::max(nj, 1)), nrm(std::max(nj, 1));
    for (int j = 0; j < nj; j++) {
      pos[j] = make_float4(xj[j], yj[j], zj[j], 0.f);
      nrm[j] = make_float4(gxj[j], gyj[j], gzj[j], 0.f);
    }
    const RefTables& tb = ref_tables(p);
    g_keys.alloc(nblock);
    g_leaf.alloc(nblock);
    g_pos.alloc(pos.size());
    g_nrm.alloc(nrm.size());
    g_q.alloc(std::max(nj, 1));
    g_exp.alloc((size_t)nblock * K);
    FMMB_CUDA(cudaMemcpy(g_keys.get(), keys.data(), nblock * sizeof(int), cudaMemcpyHostToDevice));
    FMMB_CUDA(cudaMemcpy(g_leaf.get(), leaf.data(), nblock * sizeof(int2), cudaMemcpyHostToDevice));
    FMMB_CUDA(cudaMemcpy(g_pos.get(), pos.data(), pos.size() * sizeof(float4), cudaMemcpyHostToDevice));
    FMMB_CUDA(cudaMemcpy(g_nrm.get(), nrm.data(), nrm.size() * sizeof(float4), cudaMemcpyHostToDevice));
    if (nj) FMMB_CUDA(cudaMemcpy(g_q.get(), vj, nj * sizeof(float), cudaMemcpyHostToDevice));
    const float bbox[4] = {(float)*xmin, (float)*ymin, (float)*zmin, 0.f};
    launch_p2m(neq == 0 ? FMMB_LAPLACE_G : FMMB_LAPLACE_GNJ, nblock, p, K, g_keys.get(), g_leaf.get(), g_pos.get(),
               g_nrm.get(), g_q.get(), tb.fac.get(), ref_sem(), bbox, *rb, g_exp.get(), cudaStreamLegacy);
    std::vector<double> M((size_t)nblock * K);
    FMMB_CUDA(cudaMemcpy(M.data(), g_exp.get(), M.size() * sizeof(double), cudaMemcpyDeviceToHost));
    // scaled real-packed [Re M_n^0, Re M_n^1, Im M_n^1, ...] / rb^n -> the
    // reference's complex coefficients at n (n+1) / 2 + m of each block
    for (int b = 0; b < nblock; b++) {
      float* re = brex + (size_t)b * kBlk1;
      float* im = bimx + (size_t)b * kBlk1;
      for (int k = 0; k < kBlk1; k++) re[k] = im[k] = 0.f;
      const double* v = &M[(size_t)b * K];
      double sc = 1.0;
      for (int n = 0; n <= p; n++, sc *= *rb) {
        re[isym_h(n, 0)] = (float)(v[n * n] * sc);
        for (int m = 1; m <= n; m++) {
          re[isym_h(n, m)] = (float)(v[n * n + 2 * m - 1] * sc);
          im[isym_h(n, m)] = (float)(v[n * n + 2 * m] * sc);
        }
      }
    }
  });
}

extern "C" int fmmb_gpu_l2p(const int* nvecd, const double* rb, const double* xmin, const double* ymin,
                            const double* zmin, const float* xi, const float* yi, const float* zi, float* gxi,
                            float* gyi, float* gzi, float* vi, const float* arex, const float* aimx) {
  return guarded_c([&] {
    FMMB_REQUIRE(nvecd && rb && xmin && ymin && zmin, FMMB_ERR_ARG, "null argument");
    const int nblock = nvecd[1], stride = nvecd[2], nc = nvecd[3], neq = nvecd[4], mp = nvecd[6];
    FMMB_REQUIRE(neq == 0 || neq == 1, FMMB_ERR_ARG, "l2pgpu_ handles neq 0 (G) and 1 (Gn)");
    FMMB_REQUIRE(mp >= 1 && mp <= 21, FMMB_ERR_ARG, "l2pgpu_ takes mp <= 21");
    FMMB_REQUIRE(nblock >= 0 && stride >= 3 && nc >= 0, FMMB_ERR_ARG, "bad block records");
    if (nblock == 0) return;
    FMMB_REQUIRE(xi && yi && zi && gxi && gyi && gzi && vi && arex && aimx, FMMB_ERR_ARG, "null array");
    const int p = mp - 1, K = mp * mp, P = mp * (mp + 1) / 2;
    const int nt = nblock * kBlk1;
    std::vector<int> keys(nblock);
    std::vector<int2> leaf(nblock);
    std::vector<double> L((size_t)nblock * K);
    for (int b = 0; b < nblock; b++) {
      keys[b] = nvecd[(size_t)b * stride + 10];
      const int jb = nvecd[(size_t)b * stride + 11];
      FMMB_REQUIRE(keys[b] >= 0 && jb >= 0 && jb + P <= nc, FMMB_ERR_ARG, "block record outside the coefficients");
      leaf[b] = make_int2(b * kBlk1, kBlk1);
      // the reference's complex L_n^m -> scaled real-packed L_n rb^(n+1)
      double* v = &L[(size_t)b * K];
      double sc = *rb;
      for (int n = 0; n <= p; n++, sc *= *rb) {
        v[n * n] = arex[jb + isym_h(n, 0)] * sc;
        for (int m = 1; m <= n; m++) {
          v[n * n + 2 * m - 1] = arex[jb + isym_h(n, m)] * sc;
          v[n * n + 2 * m] = aimx[jb + isym_h(n, m)] * sc;
        }
      }
    }
    std::vector<float4> pos(nt), nrm(nt);
    for (int i = 0; i < nt; i++) {
      pos[i] = make_float4(xi[i], yi[i], zi[i], 0.f);
      nrm[i] = make_float4(gxi[i], gyi[i], gzi[i], 0.f);
    }
    const RefTables& tb = ref_tables(p);
    g_keys.alloc(nblock);
    g_leaf.alloc(nblock);
    g_pos.alloc(nt);
    g_nrm.alloc(nt);
    g_exp.alloc(L.size());
    g_pot.alloc((size_t)4 * nt);
    FMMB_CUDA(cudaMemcpy(g_keys.get(), keys.data(), nblock * sizeof(int), cudaMemcpyHostToDevice));
    FMMB_CUDA(cudaMemcpy(g_leaf.get(), leaf.data(), nblock * sizeof(int2), cudaMemcpyHostToDevice));
    FMMB_CUDA(cudaMemcpy(g_pos.get(), pos.data(), nt * sizeof(float4), cudaMemcpyHostToDevice));
    FMMB_CUDA(cudaMemcpy(g_nrm.get(), nrm.data(), nt * sizeof(float4), cudaMemcpyHostToDevice));
    FMMB_CUDA(cudaMemcpy(g_exp.get(), L.data(), L.size() * sizeof(double), cudaMemcpyHostToDevice));
    FMMB_CUDA(cudaMemset(g_pot.get(), 0, (size_t)4 * nt * sizeof(double)));
    const float bbox[4] = {(float)*xmin, (float)*ymin, (float)*zmin, 0.f};
    launch_l2p(neq == 0 ? FMMB_LAPLACE_G : FMMB_LAPLACE_GNI, nblock, p, K, g_keys.get(), g_leaf.get(), g_pos.get(),
               g_nrm.get(), tb.fac.get(), ref_sem(), bbox, *rb, g_exp.get(), g_pot.get(), g_pot.get() + nt, nt,
               cudaStreamLegacy);
    std::vector<double> out((size_t)4 * nt);
    FMMB_CUDA(cudaMemcpy(out.data(), g_pot.get(), out.size() * sizeof(double), cudaMemcpyDeviceToHost));
    for (int i = 0; i < nt; i++) {
      vi[i] = (float)out[i];
      gxi[i] = neq == 0 ? (float)out[nt + i] : 0.f;
      gyi[i] = neq == 0 ? (float)out[2 * (size_t)nt + i] : 0.f;
      gzi[i] = neq == 0 ? (float)out[3 * (size_t)nt + i] : 0.f;
    }
  });
}

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
#include <array>
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

// ---------------------------------------------------------------- m2lgpu_
// The reference's batch translation call (libgpu/gpufmm.cu:336-480 over
// kernel/m2m_gpu.cxx, m2l_gpu.cxx, l2l_gpu.cxx): nvecd[4] = 0 M2M, 1 M2L,
// 2 L2L; per block b the number of inputs nvecd[b*stride + 10] and per input
// r the offset of its coefficients in brex/bimx (nvecd[..+2r+11]) and its
// relative-position code + 1 (nvecd[..+2r+12]): the Morton encoding
// (fmm/boxn1.cxx) of (4 - 2c) per axis for the child octant c of an M2M, of
// (2c + 2) for an L2L, of (target - source + 3) for an M2L.  rb is the box
// side of the parents (M2M), of both boxes (M2L), of the children (L2L).
// Here the same dense operators as the plan path (reference semantics,
// operators.cpp) are applied by the FP64 pair kernel to the inputs in the
// scaled real-packed form, and the block sums are written back as the
// reference's complex coefficients.
namespace fmmb {
namespace {

struct TransTables {
  DevBuf<double> m2m_t, l2l_t, m2l_t;  // transposed, [op][column][row], row stride even(K)
  std::vector<int> rel_to_op;
  float m2l_rb = -1.f;
};

std::vector<double> transpose_ops(const std::vector<double>& a, int K) {
  const int KP = (K + 1) & ~1;
  const size_t nop = a.size() / ((size_t)K * K), os = (size_t)K * KP;
  std::vector<double> t(nop * os, 0.0);
  for (size_t op = 0; op < nop; op++)
    for (int r = 0; r < K; r++)
      for (int c = 0; c < K; c++) t[op * os + (size_t)c * KP + r] = a[(op * K + r) * K + c];
  return t;
}

TransTables& trans_tables(int p, double rb) {
  static std::map<int, std::unique_ptr<TransTables>> cache;
  auto& t = cache[p];
  const int K = (p + 1) * (p + 1);
  auto up = [&](DevBuf<double>& d, const std::vector<double>& h) {
    d.alloc(h.size());
    FMMB_CUDA(cudaMemcpy(d.get(), h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice));
  };
  if (!t) {
    Operators ops;
    build_static_operators(ops, p, true);
    t.reset(new TransTables());
    up(t->m2m_t, transpose_ops(ops.m2m, K));
    up(t->l2l_t, transpose_ops(ops.l2l, K));
    t->rel_to_op = ops.rel_to_op;
  }
  if (t->m2l_rb != (float)rb) {  // reference semantics: the M2L set depends on the box side
    Operators ops;
    build_static_operators(ops, p, true);
    build_m2l_operators(ops, 2, (float)(4.0 * rb));  // level 2 of a root of side 4 rb has side rb
    up(t->m2l_t, transpose_ops(ops.m2l, K));
    t->m2l_rb = (float)rb;
  }
  return *t;
}

int morton3_decode(int code, int* c) {  // (x, y, z) of a 3-level key, bit order of fmm/boxn1.cxx
  c[0] = c[1] = c[2] = 0;
  for (int i = 0; i < 3; i++) {
    c[1] |= ((code >> (3 * i)) & 1) << i;
    c[0] |= ((code >> (3 * i + 1)) & 1) << i;
    c[2] |= ((code >> (3 * i + 2)) & 1) << i;
  }
  return 0;
}

DevBuf<int> g_top, g_tsrc, g_tdst;
DevBuf<double> g_in, g_tout;

}  // namespace
}  // namespace fmmb

extern "C" int fmmb_gpu_m2l(const int* nvecd, const double* rb, float* arex, float* aimx, const float* brex,
                            const float* bimx) {
  return guarded_c([&] {
    FMMB_REQUIRE(nvecd && rb && arex && aimx && brex && bimx, FMMB_ERR_ARG, "null argument");
    const int nblock = nvecd[1], stride = nvecd[2], nin = nvecd[3], var = nvecd[4], mp = nvecd[6];
    FMMB_REQUIRE(var >= 0 && var <= 2, FMMB_ERR_ARG, "m2lgpu_ takes nvecd[4] = 0 (M2M), 1 (M2L), 2 (L2L)");
    FMMB_REQUIRE(mp >= 1 && mp * (mp + 1) / 2 <= kBlk1, FMMB_ERR_ARG, "m2lgpu_ takes mp (mp + 1) / 2 <= 64");
    FMMB_REQUIRE(nblock >= 0 && stride >= 3 && nin >= 0 && *rb > 0, FMMB_ERR_ARG, "bad block records");
    if (nblock == 0) return;
    const int p = mp - 1, K = mp * mp, P = mp * (mp + 1) / 2;
    TransTables& tt = trans_tables(p, *rb);
    // input rows: one per distinct coefficient offset, scaled real-packed
    const double r_in = var == 0 ? *rb / 2 : (var == 1 ? *rb : 2 * *rb);
    std::map<int, int> row_of;
    std::vector<double> in;
    std::vector<std::array<int, 3>> pairs;  // {operator, input row, block}
    for (int b = 0; b < nblock; b++) {
      const int nr = nvecd[(size_t)b * stride + 10];
      FMMB_REQUIRE(nr >= 0 && 2 * nr < stride, FMMB_ERR_ARG, "too many inputs for the record stride");
      for (int r = 0; r < nr; r++) {
        const int jb = nvecd[(size_t)b * stride + 2 * r + 11], code = nvecd[(size_t)b * stride + 2 * r + 12] - 1;
        FMMB_REQUIRE(jb >= 0 && jb + P <= nin && code >= 0 && code < 512, FMMB_ERR_ARG, "bad input record");
        int c[3];
        morton3_decode(code, c);
        int op;
        if (var == 1) {
          FMMB_REQUIRE(c[0] <= 6 && c[1] <= 6 && c[2] <= 6, FMMB_ERR_ARG, "M2L offset outside the 7^3 cube");
          op = tt.rel_to_op[c[0] * 49 + c[1] * 7 + c[2]];
          FMMB_REQUIRE(op >= 0, FMMB_ERR_ARG, "M2L between adjacent boxes");
        } else {
          int oc[3];
          for (int d = 0; d < 3; d++) {
            oc[d] = var == 0 ? (4 - c[d]) / 2 : (c[d] - 2) / 2;
            FMMB_REQUIRE(oc[d] == 0 || oc[d] == 1, FMMB_ERR_ARG, "bad octant code");
          }
          op = (oc[0] << 1) | oc[1] | (oc[2] << 2);  // key bits: x 1, y 0, z 2
        }
        auto it = row_of.find(jb);
        int row;
        if (it == row_of.end()) {
          row = (int)row_of.size();
          row_of[jb] = row;
          in.resize(in.size() + K);
          double* v = &in[(size_t)row * K];
          for (int n = 0; n <= p; n++) {
            const double sc = var == 2 ? std::pow(r_in, n + 1) : 1.0 / std::pow(r_in, n);
            v[n * n] = brex[jb + isym_h(n, 0)] * sc;
            for (int m = 1; m <= n; m++) {
              v[n * n + 2 * m - 1] = brex[jb + isym_h(n, m)] * sc;
              v[n * n + 2 * m] = bimx[jb + isym_h(n, m)] * sc;
            }
          }
        } else {
          row = it->second;
        }
        pairs.push_back({op, row, b});
      }
    }
    // tiles of same-operator pairs for the pair kernel
    std::stable_sort(pairs.begin(), pairs.end(),
                     [](const std::array<int, 3>& a, const std::array<int, 3>& b) { return a[0] < b[0]; });
    int nsm = 148;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, 0);
    const int tp = pairs_f64_tile(K, (int)pairs.size(), nsm);
    std::vector<int> top, tsrc, tdst;
    for (size_t i = 0; i < pairs.size();) {
      size_t j = i;
      while (j < pairs.size() && pairs[j][0] == pairs[i][0]) j++;
      for (size_t k = i; k < j; k += tp) {
        top.push_back(pairs[i][0]);
        for (int c = 0; c < tp; c++) {
          tsrc.push_back(k + c < j ? pairs[k + c][1] : -1);
          tdst.push_back(k + c < j ? pairs[k + c][2] : -1);
        }
      }
      i = j;
    }
    auto upi = [&](DevBuf<int>& d, const std::vector<int>& h) {
      d.alloc(std::max<size_t>(h.size(), 1));
      if (!h.empty()) FMMB_CUDA(cudaMemcpy(d.get(), h.data(), h.size() * sizeof(int), cudaMemcpyHostToDevice));
    };
    upi(g_top, top);
    upi(g_tsrc, tsrc);
    upi(g_tdst, tdst);
    g_in.alloc(std::max<size_t>(in.size(), 1));
    if (!in.empty()) FMMB_CUDA(cudaMemcpy(g_in.get(), in.data(), in.size() * sizeof(double), cudaMemcpyHostToDevice));
    g_tout.alloc((size_t)nblock * K);
    FMMB_CUDA(cudaMemset(g_tout.get(), 0, (size_t)nblock * K * sizeof(double)));
    prepare_translate_pairs_f64();
    PairArgs a{};
    a.ntile = (int)top.size();
    a.tp = tp;
    a.K = K;
    a.atomic = 1;
    a.tile_op = g_top.get();
    a.tile_src = g_tsrc.get();
    a.tile_dst = g_tdst.get();
    a.opT = (var == 0 ? tt.m2m_t : var == 1 ? tt.m2l_t : tt.l2l_t).get();
    a.ostride = (size_t)K * ((K + 1) & ~1);
    a.xin = g_in.get();
    a.out = g_tout.get();
    launch_translate_pairs_f64(a, cudaStreamLegacy);
    std::vector<double> out((size_t)nblock * K);
    FMMB_CUDA(cudaMemcpy(out.data(), g_tout.get(), out.size() * sizeof(double), cudaMemcpyDeviceToHost));
    // scaled outputs -> the reference's complex coefficients of each block
    const double r_out = *rb;  // side of the output boxes: parents (M2M), the level (M2L), children (L2L)
    for (int b = 0; b < nblock; b++) {
      float* re = arex + (size_t)b * kBlk1;
      float* im = aimx + (size_t)b * kBlk1;
      for (int k = 0; k < kBlk1; k++) re[k] = im[k] = 0.f;
      const double* v = &out[(size_t)b * K];
      for (int n = 0; n <= p; n++) {
        const double sc = var == 0 ? std::pow(r_out, n) : 1.0 / std::pow(r_out, n + 1);
        re[isym_h(n, 0)] = (float)(v[n * n] * sc);
        for (int m = 1; m <= n; m++) {
          re[isym_h(n, m)] = (float)(v[n * n + 2 * m - 1] * sc);
          im[isym_h(n, m)] = (float)(v[n * n + 2 * m] * sc);
        }
      }
    }
  });
}

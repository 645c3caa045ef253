// C ABI of libfmmb (include/fmmb.h): plan lifetime, geometry, evaluation.
//
// The evaluation is the reference's seven-step driver (fmm/fmm.cxx:29-152)
// recast for one GPU: the near field (P2P) runs on a side stream while the far
// field runs P2M -> M2M (lmax-1..2) -> M2L at level 2 -> for each level
// 3..lmax: L2L then M2L -> L2P on the main stream; the two halves meet in the
// final scatter to caller order.
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "internal.h"
#include "kernels.h"

namespace fmmb {

thread_local std::string g_last_error;
void set_error(const std::string& m) { g_last_error = m; }

namespace {

const double kPiF = (double)(float)M_PI;
const double kEpsF = (double)1e-6f;

bool is_device_ptr(const void* p) {
  if (!p) return false;
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

template <typename F>
int guarded(F f) {
  try {
    f();
    return FMMB_OK;
  } catch (const Error& e) {
    set_error(e.msg);
    return e.code;
  } catch (const std::exception& e) {
    set_error(e.what());
    return FMMB_ERR_ARG;
  }
}

Sem make_sem(const fmmb_plan* pl) {
  Sem s;
  s.eps2 = pl->eps2;
  s.coef = pl->coef;
  s.rho_eps = pl->rho_eps;
  s.ang_eps = pl->ang_eps;
  s.pi_ang = pl->pi_ang;
  s.ref = pl->ref ? 1 : 0;
  s.excl_self = (!pl->ref && pl->cfg.exclude_self) ? 1 : 0;
  return s;
}

// Copies a host or device float array of n elements to a device pointer
// (staging when needed).  Returns the device pointer to use.
const float* to_device(const float* src, size_t n, DevBuf<float>& stage, cudaStream_t s) {
  if (!src) return nullptr;
  if (is_device_ptr(src)) return src;
  stage.alloc(n);
  FMMB_CUDA(cudaMemcpyAsync(stage.get(), src, n * sizeof(float), cudaMemcpyHostToDevice, s));
  return stage.get();
}

void upload(DevBuf<double>& d, const std::vector<double>& h, cudaStream_t s) {
  d.alloc(h.size());
  FMMB_CUDA(cudaMemcpyAsync(d.get(), h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice, s));
  FMMB_CUDA(cudaStreamSynchronize(s));
}

// Doubles per operator in the transposed M2M/L2L arrays: K columns of KP = K
// rounded up to even rows (16-byte aligned row pairs; a 16-byte multiple in
// all, so each operator can be bulk-copied).
size_t pair_op_stride(int K) { return (size_t)K * (size_t)((K + 1) & ~1); }

void upload_static_ops(fmmb_plan* pl) {
  const Operators& o = pl->ops;
  cudaStream_t s = pl->st.main;
  upload(pl->d_fac, o.fac, s);
  const int K = pl->K;
  const size_t ostride = pair_op_stride(K);
  const int KP = (K + 1) & ~1;
  auto transposed = [&](const std::vector<double>& a) {  // [op][r][c] -> [op][c][r], row stride KP
    const size_t nop = a.size() / ((size_t)K * K);
    std::vector<double> t(nop * ostride, 0.0);
    for (size_t op = 0; op < nop; op++)
      for (int r = 0; r < K; r++)
        for (int c = 0; c < K; c++) t[op * ostride + (size_t)c * KP + r] = a[(op * K + r) * K + c];
    return t;
  };
  upload(pl->d_m2m_t, transposed(o.m2m), s);
  upload(pl->d_l2l_t, transposed(o.l2l), s);
  pl->d_slot_rel.alloc(o.slot_rel.size());
  FMMB_CUDA(cudaMemcpyAsync(pl->d_slot_rel.get(), o.slot_rel.data(), o.slot_rel.size() * sizeof(int), cudaMemcpyHostToDevice, s));
  pl->d_rel_to_op.alloc(o.rel_to_op.size());
  FMMB_CUDA(cudaMemcpyAsync(pl->d_rel_to_op.get(), o.rel_to_op.data(), o.rel_to_op.size() * sizeof(int), cudaMemcpyHostToDevice, s));
  FMMB_CUDA(cudaStreamSynchronize(s));
}

// The tensor-core M2L's operator images (mixed form), rebuilt when the
// operator set changed: FP16 (hi, lo) for K <= h16_max_k(), TF32 above.
void m2l_images(fmmb_plan* pl) {
  const int K = pl->K;
  if (pl->cfg.precision != FMMB_MIXED || K > tc_max_k() || helm_family(pl->cfg.kernel) || pl->ops.m2l.empty()) return;
  const bool stale = pl->opimg_sets != pl->ops.m2l_sets || pl->opimg_rd != pl->ops.m2l_rd;
  if (K > h16_max_k() && (stale || pl->d_img_m2l.get() == nullptr)) {
    std::vector<float> img;
    build_tc_images(pl->ops.m2l, pl->ops.m2l_sets * 316, K, tc_kpad(K), img);
    pl->d_img_m2l.alloc(img.size());
    FMMB_CUDA(cudaMemcpy(pl->d_img_m2l.get(), img.data(), img.size() * sizeof(float), cudaMemcpyHostToDevice));
  } else if (K <= h16_max_k() && (stale || pl->d_img_h16.get() == nullptr)) {
    std::vector<unsigned char> img;
    build_h16_images(pl->ops.m2l, pl->ops.m2l_sets * 316, K, h16_n(K), h16_kpad(K), h16_img_bytes(K), img);
    pl->d_img_h16.alloc(img.size());
    FMMB_CUDA(cudaMemcpy(pl->d_img_h16.get(), img.data(), img.size(), cudaMemcpyHostToDevice));
  }
  pl->opimg_sets = pl->ops.m2l_sets;
  pl->opimg_rd = pl->ops.m2l_rd;
}

}  // namespace
}  // namespace fmmb

using namespace fmmb;

extern "C" {

const char* fmmb_last_error(void) { return g_last_error.c_str(); }

int fmmb_config_init(fmmb_config* cfg) {
  if (!cfg) return FMMB_ERR_ARG;
  std::memset(cfg, 0, sizeof(*cfg));
  cfg->kernel = FMMB_LAPLACE_G;
  cfg->p = 8;
  cfg->lmax = 3;
  cfg->precision = FMMB_FP64;
  cfg->semantics = FMMB_SEM_REFERENCE;
  cfg->eps2 = 0.0;
  cfg->exclude_self = 0;
  cfg->nrhs = 1;
  return FMMB_OK;
}

int fmmb_plan_create(const fmmb_config* cfg, fmmb_plan** out) {
  return guarded([&] {
    FMMB_REQUIRE(cfg && out, FMMB_ERR_ARG, "null argument");
    FMMB_REQUIRE(cfg->kernel == FMMB_LAPLACE_G || cfg->kernel == FMMB_LAPLACE_GNI || cfg->kernel == FMMB_LAPLACE_GNJ ||
                     helm_family(cfg->kernel),
                 FMMB_ERR_ARG, "unknown kernel");
    FMMB_REQUIRE(!helm_family(cfg->kernel) || (cfg->wavenumber > 0 && std::isfinite(cfg->wavenumber)),
                 FMMB_ERR_ARG, "the Helmholtz and Yukawa kernels need a finite wavenumber > 0");
    FMMB_REQUIRE(!helm_family(cfg->kernel) || cfg->semantics == FMMB_SEM_ACCURATE, FMMB_ERR_ARG,
                 "the Helmholtz and Yukawa kernels take FMMB_SEM_ACCURATE");
    FMMB_REQUIRE(cfg->p >= 1 && cfg->p <= 20, FMMB_ERR_ARG, "p must be in 1..20");
    FMMB_REQUIRE(cfg->lmax >= 2 && cfg->lmax <= 10, FMMB_ERR_ARG, "lmax must be in 2..10");
    FMMB_REQUIRE(cfg->precision == FMMB_FP64 || cfg->precision == FMMB_MIXED, FMMB_ERR_ARG, "unknown precision");
    FMMB_REQUIRE(cfg->semantics == FMMB_SEM_REFERENCE || cfg->semantics == FMMB_SEM_ACCURATE, FMMB_ERR_ARG,
                 "unknown semantics");
    FMMB_REQUIRE(cfg->nrhs >= 1 && cfg->nrhs <= 4096, FMMB_ERR_ARG, "nrhs must be in 1..4096");
    FMMB_REQUIRE(cfg->eps2 >= 0 && std::isfinite(cfg->eps2), FMMB_ERR_ARG, "eps2 must be finite and >= 0");
    int ndev = 0;
    FMMB_CUDA(cudaGetDeviceCount(&ndev));
    FMMB_REQUIRE(ndev > 0, FMMB_ERR_CUDA, "no CUDA device");
    auto* pl = new fmmb_plan();
    try {
      pl->cfg = *cfg;
      pl->p = cfg->p;
      pl->K = (cfg->p + 1) * (cfg->p + 1);
      pl->P = (cfg->p + 1) * (cfg->p + 2) / 2;
      pl->ref = cfg->semantics == FMMB_SEM_REFERENCE;
      pl->eps2 = pl->ref ? kEpsF : cfg->eps2;
      pl->coef = pl->ref ? 0.25 / kPiF : 0.25 / M_PI;
      pl->rho_eps = pl->ref ? kEpsF : 0.0;
      pl->ang_eps = pl->ref ? kEpsF : 0.0;
      pl->pi_ang = pl->ref ? kPiF : M_PI;
      FMMB_CUDA(cudaGetDevice(&pl->device));
      // the far field (main / capture stream) outranks the near field (side
      // stream): its short dependent launches take SMs first and the P2P
      // blocks fill the rest
      int prio_low = 0, prio_high = 0;
      FMMB_CUDA(cudaDeviceGetStreamPriorityRange(&prio_low, &prio_high));
      FMMB_CUDA(cudaStreamCreateWithPriority(&pl->st.main, cudaStreamNonBlocking, prio_high));
      FMMB_CUDA(cudaStreamCreateWithPriority(&pl->st.side, cudaStreamNonBlocking, prio_low));
      FMMB_CUDA(cudaStreamCreateWithPriority(&pl->st.cap, cudaStreamNonBlocking, prio_high));
      FMMB_CUDA(cudaEventCreateWithFlags(&pl->st.fork, cudaEventDisableTiming));
      FMMB_CUDA(cudaEventCreateWithFlags(&pl->st.join, cudaEventDisableTiming));
      FMMB_CUDA(cudaEventCreateWithFlags(&pl->st.near_done, cudaEventDisableTiming));
      for (auto& e : pl->ev) FMMB_CUDA(cudaEventCreate(&e));
      for (auto& e : pl->evp) FMMB_CUDA(cudaEventCreate(&e));
      pl->d_err.alloc(1);
      FMMB_CUDA(cudaMemset(pl->d_err.get(), 0, sizeof(int)));
      FMMB_CUDA(cudaHostAlloc((void**)&pl->h_err, sizeof(int), cudaHostAllocDefault));
      *pl->h_err = 0;
      build_static_operators(pl->ops, pl->p, pl->ref);
      upload_static_ops(pl);
      if (!pl->ref && !helm_family(cfg->kernel)) {  // geometry-independent M2L set
        build_m2l_operators(pl->ops, 2, 1.0f);
        upload(pl->d_m2l, pl->ops.m2l, pl->st.main);
        m2l_images(pl);
      }
    } catch (...) {
      fmmb_plan_destroy(pl);
      throw;
    }
    *out = pl;
  });
}

int fmmb_plan_destroy(fmmb_plan* pl) {
  if (!pl) return FMMB_OK;
  cudaDeviceSynchronize();
  for (auto& g : pl->gexec)
    if (g) cudaGraphExecDestroy(g);
  if (pl->tplan && pl->tplan != pl) fmmb_plan_destroy(pl->tplan);
  if (pl->own_stream && pl->st.main) cudaStreamDestroy(pl->st.main);
  if (pl->st.side) cudaStreamDestroy(pl->st.side);
  if (pl->st.cap) cudaStreamDestroy(pl->st.cap);
  if (pl->st.fork) cudaEventDestroy(pl->st.fork);
  if (pl->st.join) cudaEventDestroy(pl->st.join);
  if (pl->st.near_done) cudaEventDestroy(pl->st.near_done);
  if (pl->st.copy) cudaStreamDestroy(pl->st.copy);
  for (auto& e : pl->st.copy_ev)
    if (e) cudaEventDestroy(e);
  for (auto& e : pl->ev)
    if (e) cudaEventDestroy(e);
  for (auto& e : pl->evp)
    if (e) cudaEventDestroy(e);
  if (pl->h_err) cudaFreeHost(pl->h_err);
  delete pl;
  return FMMB_OK;
}

int fmmb_set_stream(fmmb_plan* pl, void* stream) {
  return guarded([&] {
    FMMB_REQUIRE(pl, FMMB_ERR_ARG, "null plan");
    if (!stream) return;
    if (pl->own_stream && pl->st.main) FMMB_CUDA(cudaStreamDestroy(pl->st.main));
    pl->st.main = (cudaStream_t)stream;
    pl->own_stream = false;
    if (pl->tplan && pl->tplan != pl) {
      const int rc = fmmb_set_stream(pl->tplan, stream);
      if (rc != FMMB_OK) throw Error{rc, std::string(fmmb_last_error())};
    }
  });
}

}  // extern "C"

namespace {

// fmmb_set_geometry (nprob = 1, no offsets) and fmmb_set_geometry_batch
// (nprob problems, host or device offsets toff / soff of nprob + 1 entries)
int geometry_impl(fmmb_plan* pl, int nprob, const int* toff, const int* soff, int ni, const float* tx, const float* ty,
                  const float* tz, const float* tnx, const float* tny, const float* tnz, int nj, const float* sx,
                  const float* sy, const float* sz, const float* snx, const float* sny, const float* snz,
                  const float* bbox) {
  const auto t_setup = std::chrono::steady_clock::now();
  const int rc = guarded([&] {
    FMMB_REQUIRE(pl, FMMB_ERR_ARG, "null plan");
    FMMB_REQUIRE(ni >= 1 && nj >= 1, FMMB_ERR_ARG, "need at least one target and one source");
    FMMB_REQUIRE(nprob >= 1 && nprob <= (1 << 20), FMMB_ERR_ARG, "number of problems must be in 1..2^20");
    std::vector<int> to(nprob + 1), so(nprob + 1);
    if (nprob == 1) {
      to = {0, ni};
      so = {0, nj};
    } else {
      FMMB_REQUIRE(toff && soff, FMMB_ERR_ARG, "null problem offsets");
      for (int w = 0; w < 2; w++) {
        const int* src = w ? soff : toff;
        std::vector<int>& dst = w ? so : to;
        if (is_device_ptr(src)) FMMB_CUDA(cudaMemcpy(dst.data(), src, (nprob + 1) * sizeof(int), cudaMemcpyDeviceToHost));
        else std::memcpy(dst.data(), src, (nprob + 1) * sizeof(int));
      }
      for (int b = 0; b < nprob; b++)
        FMMB_REQUIRE(to[b] <= to[b + 1] && so[b] <= so[b + 1], FMMB_ERR_ARG, "problem offsets must not decrease");
      FMMB_REQUIRE(to[0] == 0 && so[0] == 0 && to[nprob] == ni && so[nprob] == nj, FMMB_ERR_ARG,
                   "problem offsets must run from 0 to the point counts");
    }
    for (int w = 0; w < 4; w++) {  // captured evaluates refer to the old buffers
      if (pl->gexec[w]) {
        FMMB_CUDA(cudaStreamSynchronize(pl->st.main));
        cudaGraphExecDestroy(pl->gexec[w]);
        pl->gexec[w] = nullptr;
      }
    }
    if (pl->tplan) {  // its geometry is the old one
      if (pl->tplan != pl) fmmb_plan_destroy(pl->tplan);
      pl->tplan = nullptr;
    }
    // one set of points as both targets and sources (the same arrays): the
    // transpose of a symmetric kernel is then this plan itself
    pl->same_sets = nprob == 1 && ni == nj && tx == sx && ty == sy && tz == sz;
    FMMB_REQUIRE(tx && ty && tz && sx && sy && sz, FMMB_ERR_ARG, "null coordinates");
    FMMB_REQUIRE(pl->cfg.kernel != FMMB_LAPLACE_GNI || (tnx && tny && tnz), FMMB_ERR_ARG, "Gni needs target normals");
    FMMB_REQUIRE(pl->cfg.kernel != FMMB_LAPLACE_GNJ || (snx && sny && snz), FMMB_ERR_ARG, "Gnj needs source normals");
    FMMB_REQUIRE((long long)ni * pl->cfg.nrhs < (1LL << 31) && (long long)nj * pl->cfg.nrhs < (1LL << 31),
                 FMMB_ERR_CAPACITY, "n * nrhs must stay below 2^31");
    float bb[4];
    if (bbox) {
      if (is_device_ptr(bbox)) FMMB_CUDA(cudaMemcpy(bb, bbox, sizeof(bb), cudaMemcpyDeviceToHost));
      else std::memcpy(bb, bbox, sizeof(bb));
      FMMB_REQUIRE(bb[3] > 0 && std::isfinite(bb[3]), FMMB_ERR_ARG, "bbox side must be positive");
    }
    cudaStream_t s = pl->st.main;
    pl->have_geometry = false;
    pl->have_expansions = false;
    DevBuf<float> st[12];
    const float* d[12] = {to_device(tx, ni, st[0], s),  to_device(ty, ni, st[1], s),  to_device(tz, ni, st[2], s),
                          to_device(tnx, ni, st[3], s), to_device(tny, ni, st[4], s), to_device(tnz, ni, st[5], s),
                          to_device(sx, nj, st[6], s),  to_device(sy, nj, st[7], s),  to_device(sz, nj, st[8], s),
                          to_device(snx, nj, st[9], s), to_device(sny, nj, st[10], s), to_device(snz, nj, st[11], s)};
    pl->nprob = nprob;
    pl->prob_toff = to;
    pl->prob_soff = so;
    pl->d_prob_off.alloc(2 * (size_t)(nprob + 1));
    FMMB_CUDA(cudaMemcpyAsync(pl->d_prob_off.get(), to.data(), (nprob + 1) * sizeof(int), cudaMemcpyHostToDevice, s));
    FMMB_CUDA(cudaMemcpyAsync(pl->d_prob_off.get() + nprob + 1, so.data(), (nprob + 1) * sizeof(int),
                              cudaMemcpyHostToDevice, s));
    const auto t_tree = std::chrono::steady_clock::now();
    build_tree(pl, ni, d[0], d[1], d[2], d[3], d[4], d[5], nj, d[6], d[7], d[8], d[9], d[10], d[11], bbox ? bb : nullptr);
    FMMB_CUDA(cudaStreamSynchronize(s));
    pl->tree_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_tree).count();
    // caller-order copy of the geometry for the transposed plan
    pl->geo.alloc((size_t)6 * ni + 6 * (size_t)nj);
    pl->geo_tn = d[3] && d[4] && d[5];
    pl->geo_sn = d[9] && d[10] && d[11];
    for (int k = 0; k < 12; k++) {
      const size_t n = k < 6 ? ni : nj;
      float* dst = pl->geo.get() + (k < 6 ? (size_t)k * ni : (size_t)6 * ni + (size_t)(k - 6) * nj);
      if (d[k]) FMMB_CUDA(cudaMemcpyAsync(dst, d[k], n * sizeof(float), cudaMemcpyDeviceToDevice, s));
    }
    if (helm_family(pl->cfg.kernel)) {  // its own operators and jobs
      helm_setup(pl);
      pl->have_geometry = true;
      return;
    }
    // reference semantics: the M2L distance carries an absolute eps, so the
    // operator set depends on the level sizes (rebuilt when they change)
    if (pl->ref && (pl->ops.m2l_lmax != pl->lmax || pl->ops.m2l_rd != pl->bbox[3])) {
      build_m2l_operators(pl->ops, pl->lmax, pl->bbox[3]);
      upload(pl->d_m2l, pl->ops.m2l, s);
    }
    // FP64 translation tiles (M2L, M2M, L2L) per level
    std::vector<int> keys(pl->tot_i), keys_j(pl->tot_j), par_j(pl->tot_j), lst;
    FMMB_CUDA(cudaMemcpy(keys.data(), pl->key_i.get(), pl->tot_i * sizeof(int), cudaMemcpyDeviceToHost));
    FMMB_CUDA(cudaMemcpy(keys_j.data(), pl->key_j.get(), pl->tot_j * sizeof(int), cudaMemcpyDeviceToHost));
    FMMB_CUDA(cudaMemcpy(par_j.data(), pl->parent_j.get(), pl->tot_j * sizeof(int), cudaMemcpyDeviceToHost));
    // the M2L lists on the host only for the work lists built there: the FP64
    // M2L's box tiles and the TF32 form's tiles (the FP16 form's are built on
    // the device, setup.cu)
    const bool tc_m2l = pl->cfg.precision == FMMB_MIXED && pl->K <= tc_max_k();
    const bool h16_m2l = pl->cfg.precision == FMMB_MIXED && pl->K <= h16_max_k();
    if (!h16_m2l) {
      lst.resize((size_t)pl->tot_i * kM2LSlots);
      FMMB_CUDA(cudaMemcpy(lst.data(), pl->m2l_list.get(), lst.size() * sizeof(int), cudaMemcpyDeviceToHost));
    }
    const int XT = translate_tile_size();
    auto make_tiles = [&](const std::vector<std::vector<int>>& groups, int nslots, auto op_of) {
      std::unique_ptr<fmmb_plan::TileSet> ts(new fmmb_plan::TileSet());
      std::vector<int> tb, to;
      for (const auto& g : groups)
        for (size_t k = 0; k < g.size(); k += XT) {
          const size_t e = std::min(g.size(), k + XT);
          std::vector<int> ops_row(nslots, -1);
          bool any_slot = false;
          for (int sl = 0; sl < nslots; sl++)
            for (size_t t = k; t < e; t++) {
              const int o = op_of(g[t], sl);
              if (o >= 0) {
                ops_row[sl] = o;
                any_slot = true;
                break;
              }
            }
          if (!any_slot) continue;
          for (int t = 0; t < XT; t++) tb.push_back(k + t < e ? g[k + t] : -1);
          to.insert(to.end(), ops_row.begin(), ops_row.end());
        }
      ts->ntile = (int)tb.size() / XT;
      ts->boxes.alloc(tb.size());
      ts->ops.alloc(to.size());
      if (!tb.empty()) {
        FMMB_CUDA(cudaMemcpy(ts->boxes.get(), tb.data(), tb.size() * sizeof(int), cudaMemcpyHostToDevice));
        FMMB_CUDA(cudaMemcpy(ts->ops.get(), to.data(), to.size() * sizeof(int), cudaMemcpyHostToDevice));
      }
      return ts;
    };
    // M2M child lists: [parent][octant] -> child within the child level
    std::vector<int> m2m_list((size_t)pl->tot_j * 8, -1);
    for (int lev = pl->lmax; lev >= 3; lev--)
      for (int c = 0; c < pl->nbox_j[lev]; c++) {
        const int par = par_j[pl->off_j[lev] + c];
        m2m_list[(size_t)(pl->off_j[lev - 1] + par) * 8 + (keys_j[pl->off_j[lev] + c] & 7)] = c;
      }
    pl->m2m_list.alloc(m2m_list.size());
    FMMB_CUDA(cudaMemcpy(pl->m2m_list.get(), m2m_list.data(), m2m_list.size() * sizeof(int), cudaMemcpyHostToDevice));
    pl->m2l_tiles.clear();
    // the FP64 M2L's box tiles (the tensor-core forms use the pair tiles below)
    const bool fp64_m2l = !tc_m2l;
    for (int lev = 0; lev <= pl->lmax; lev++) {
      std::vector<std::vector<int>> by_oct(8);
      if (lev >= 2 && fp64_m2l)
        for (int b = 0; b < pl->nbox_i[lev]; b++) by_oct[keys[pl->off_i[lev] + b] & 7].push_back(pl->off_i[lev] + b);
      pl->m2l_tiles.push_back(make_tiles(by_oct, kM2LSlots, [&](int box, int sl) {
        if (lst[(size_t)box * kM2LSlots + sl] < 0) return -1;
        return pl->ops.rel_to_op[pl->ops.slot_rel[(keys[box] & 7) * kM2LSlots + sl]];
      }));
    }
    int dev_sms = 148;
    cudaDeviceGetAttribute(&dev_sms, cudaDevAttrMultiProcessorCount, pl->device);
    pl->nsm = dev_sms;
    // M2M / L2L pair tiles: {operator = child octant, input row, output row},
    // grouped by operator, tiles of tp pairs
    {
      using P3 = std::array<int, 3>;
      auto pair_job = [&](std::vector<P3>& pairs) {
        std::unique_ptr<fmmb_plan::PairJob> job(new fmmb_plan::PairJob());
        std::stable_sort(pairs.begin(), pairs.end(), [](const P3& x, const P3& y) { return x[0] < y[0]; });
        const int tp = pairs_f64_tile(pl->K, (int)pairs.size(), dev_sms);
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
        job->ntile = (int)top.size();
        job->tp = tp;
        auto up = [&](DevBuf<int>& d, const std::vector<int>& h) {
          d.alloc(h.size());
          if (!h.empty()) FMMB_CUDA(cudaMemcpy(d.get(), h.data(), h.size() * sizeof(int), cudaMemcpyHostToDevice));
        };
        up(job->tile_op, top);
        up(job->tile_src, tsrc);
        up(job->tile_dst, tdst);
        return job;
      };
      std::vector<int> par_i(pl->tot_i);
      FMMB_CUDA(cudaMemcpy(par_i.data(), pl->parent_i.get(), pl->tot_i * sizeof(int), cudaMemcpyDeviceToHost));
      pl->m2m_pairs.clear();
      pl->l2l_pairs.clear();
      for (int lev = 0; lev <= pl->lmax; lev++) {
        std::vector<P3> up_pairs, down_pairs;
        if (lev >= 2 && lev < pl->lmax)
          for (int b = 0; b < pl->nbox_j[lev]; b++) {
            const int box = pl->off_j[lev] + b;
            for (int sl = 0; sl < 8; sl++) {
              const int c = m2m_list[(size_t)box * 8 + sl];
              if (c >= 0) up_pairs.push_back({sl, pl->off_j[lev + 1] + c, box});
            }
          }
        if (lev >= 3)
          for (int b = 0; b < pl->nbox_i[lev]; b++) {
            const int box = pl->off_i[lev] + b;
            down_pairs.push_back({keys[box] & 7, pl->off_i[lev - 1] + par_i[box], box});
          }
        pl->m2m_pairs.push_back(pair_job(up_pairs));
        pl->l2l_pairs.push_back(pair_job(down_pairs));
      }
    }
    // tensor-core M2L (mixed precision, K <= tc_max_k()): operator images (one
    // per operator and block of 128 output rows), the TF32 split of M, and
    // the work items over the pair tiles of all levels
    // M2L on the tensor cores in the mixed form: FP16x3 for K <= h16_max_k()
    // (p <= 12), TF32x3 above
    const bool mixed = pl->cfg.precision == FMMB_MIXED;
    pl->use_h16 = mixed && pl->K <= h16_max_k();
    pl->use_tc = mixed && !pl->use_h16 && pl->K <= tc_max_k();
    init_fac32();
    prepare_translate_pairs_f64();
    if (pl->use_tc) prepare_translate_tc();
    if (pl->use_h16) prepare_translate_h16();
    if (pl->use_tc || pl->use_h16) {
      const int K = pl->K, kpad = tc_kpad(K), nrb = pl->use_h16 ? 1 : (K + 127) / 128;
      m2l_images(pl);  // built once at plan creation in accurate semantics
      if (pl->use_tc) pl->Mtf.alloc((size_t)pl->tot_j * 2 * kpad);
      if (pl->use_h16) {
        pl->Xh.alloc((size_t)pl->tot_j * 2 * h16_kpad(K));
        pl->xexp.alloc(pl->tot_j);
      }
      const int TT = tc_tile();
      auto up = [&](DevBuf<int>& d, const std::vector<int>& h) {
        d.alloc(h.size());
        if (!h.empty()) FMMB_CUDA(cudaMemcpy(d.get(), h.data(), h.size() * sizeof(int), cudaMemcpyHostToDevice));
      };
      // box pairs {operator, input row, output row} -> tiles of TT pairs of one
      // operator each (operators ascending, pairs in output order within one);
      // a work item is a tile and a block of 128 output rows (operator image
      // op * nrb + block), items of one operator and block consecutive
      using Pair = std::array<int, 3>;
      auto build_job = [&](fmmb_plan::TcJob& job, std::vector<Pair>& pairs) {
        std::stable_sort(pairs.begin(), pairs.end(), [](const Pair& x, const Pair& y) { return x[0] < y[0]; });
        std::vector<int> wop, wsrc, wy, tdst;
        int ntile = 0;
        for (size_t i = 0; i < pairs.size();) {
          size_t j = i;
          while (j < pairs.size() && pairs[j][0] == pairs[i][0]) j++;
          const int t0 = ntile;
          for (size_t k = i; k < j; k += TT, ntile++)
            for (int c = 0; c < TT; c++) tdst.push_back(k + c < j ? pairs[k + c][2] : -1);
          for (int h = 0; h < nrb; h++)
            for (int t = t0; t < ntile; t++) {
              const size_t k = i + (size_t)(t - t0) * TT;
              wop.push_back(pairs[i][0] * nrb + h);
              for (int c = 0; c < TT; c++) wsrc.push_back(k + c < j ? pairs[k + c][1] : -1);
              wy.push_back(t * TT);
              wy.push_back(128 * h);
            }
          i = j;
        }
        job.ntile = (int)wop.size();
        up(job.tile_op, wop);
        up(job.tile_src, wsrc);
        up(job.tile_y, wy);
        // per output row, its pair rows (tile * TT + column)
        std::vector<std::array<int, 2>> pos;
        for (size_t k = 0; k < tdst.size(); k++)
          if (tdst[k] >= 0) pos.push_back({tdst[k], (int)k});
        std::sort(pos.begin(), pos.end());
        std::vector<int> rows, ptr, idx;
        for (size_t k = 0; k < pos.size(); k++) {
          if (k == 0 || pos[k][0] != pos[k - 1][0]) {
            rows.push_back(pos[k][0]);
            ptr.push_back((int)k);
          }
          idx.push_back(pos[k][1]);
        }
        ptr.push_back((int)pos.size());
        job.nred = (int)rows.size();
        up(job.red_rows, rows);
        up(job.red_ptr, ptr);
        up(job.red_idx, idx);
        job.ys = pl->use_h16 ? (K + 3) / 4 * 4 : 128 * nrb;
        pl->tc_y.alloc((size_t)ntile * TT * job.ys);
      };
      // M2L, all levels in one job: operator = set(level)*316 + relative position
      if (!(pl->use_h16 && build_m2l_job_dev(pl, pl->tc_m2l, (K + 3) / 4 * 4, s))) {
        if (lst.empty()) {
          lst.resize((size_t)pl->tot_i * kM2LSlots);
          FMMB_CUDA(cudaMemcpy(lst.data(), pl->m2l_list.get(), lst.size() * sizeof(int), cudaMemcpyDeviceToHost));
        }
        std::vector<Pair> pairs;
        for (int lev = 2; lev <= pl->lmax; lev++) {
          const int set = pl->ops.m2l_sets > 1 ? lev - 2 : 0;
          for (int b = 0; b < pl->nbox_i[lev]; b++) {
            const int box = pl->off_i[lev] + b;
            for (int sl = 0; sl < kM2LSlots; sl++) {
              const int src = lst[(size_t)box * kM2LSlots + sl];
              if (src < 0) continue;
              const int op = set * 316 + pl->ops.rel_to_op[pl->ops.slot_rel[(keys[box] & 7) * kM2LSlots + sl]];
              pairs.push_back({op, pl->off_j[lev] + src, box});
            }
          }
        }
        build_job(pl->tc_m2l, pairs);
      }
    }
    // inverse target permutation (caller -> sorted) for the direct sum, and the
    // near-field work items: pieces of up to 128 targets of a leaf (the
    // many-right-hand-side pass takes them in leaf order; the one-right-hand-
    // side kernels heaviest first -- targets x sources of the 27 neighbour
    // leaves -- dealt alternately to the two near-field launches of an
    // evaluate, so that each launch starts with its longest blocks), on the
    // device (setup.cu)
    build_inverse_perm_dev(pl, s);
    build_p2p_work_dev(pl, s);
    build_p2m_work_dev(pl, s);
    // evaluation buffers
    const int nr = pl->cfg.nrhs;
    pl->qs.alloc((size_t)nj * nr);
    pl->M.alloc((size_t)pl->tot_j * pl->K);
    pl->L.alloc((size_t)pl->tot_i * pl->K);
    pl->pot_s.alloc((size_t)ni * 2);          // near, far
    pl->grad_s.alloc((size_t)ni * 6);         // near xyz, far xyz
    FMMB_CUDA(cudaMemsetAsync(pl->grad_s.get(), 0, (size_t)ni * 6 * sizeof(double), s));
    FMMB_CUDA(cudaStreamSynchronize(s));
    pl->have_geometry = true;
  });
  if (rc == FMMB_OK && pl)
    pl->setup_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_setup).count();
  return rc;
}

}  // namespace

extern "C" {

int fmmb_set_geometry(fmmb_plan* pl, int ni, const float* tx, const float* ty, const float* tz, const float* tnx,
                      const float* tny, const float* tnz, int nj, const float* sx, const float* sy, const float* sz,
                      const float* snx, const float* sny, const float* snz, const float* bbox) {
  return geometry_impl(pl, 1, nullptr, nullptr, ni, tx, ty, tz, tnx, tny, tnz, nj, sx, sy, sz, snx, sny, snz, bbox);
}

int fmmb_set_geometry_batch(fmmb_plan* pl, int nprob, const int* t_off, const float* tx, const float* ty,
                            const float* tz, const float* tnx, const float* tny, const float* tnz, const int* s_off,
                            const float* sx, const float* sy, const float* sz, const float* snx, const float* sny,
                            const float* snz, const float* bbox) {
  int ni = 0, nj = 0;
  const int rc = guarded([&] {
    FMMB_REQUIRE(pl && t_off && s_off, FMMB_ERR_ARG, "null argument");
    FMMB_REQUIRE(nprob >= 1, FMMB_ERR_ARG, "need at least one problem");
    for (int w = 0; w < 2; w++) {
      const int* src = (w ? s_off : t_off) + nprob;
      int& dst = w ? nj : ni;
      if (is_device_ptr(src)) FMMB_CUDA(cudaMemcpy(&dst, src, sizeof(int), cudaMemcpyDeviceToHost));
      else dst = *src;
    }
  });
  if (rc != FMMB_OK) return rc;
  return geometry_impl(pl, nprob, t_off, s_off, ni, tx, ty, tz, tnx, tny, tnz, nj, sx, sy, sz, snx, sny, snz, bbox);
}

}  // extern "C"

namespace {

// Slot split of a translation launch: enough blocks for ~8 per SM on 148 SMs.
int split_for(int ntile, int nslots) {
  if (ntile <= 0) return 1;
  return std::max(1, std::min(std::min(nslots, 27), (8 * 148 + ntile - 1) / ntile));
}

// Brackets one launch with a pair of pool events (phase 0..5 as in
// fmmb_get_timings); silently stops timing when the pool is exhausted.
// Records a timing event; while the evaluate is being captured into a graph,
// as an event-record node (a plain record would only become a dependency).
cudaError_t time_mark(const fmmb_plan* pl, cudaEvent_t e, cudaStream_t s) {
  return cudaEventRecordWithFlags(e, s, pl->capturing ? cudaEventRecordExternal : cudaEventRecordDefault);
}

struct PhaseTimer {
  fmmb_plan* pl;
  int phase, idx;
  cudaStream_t s;
  PhaseTimer(fmmb_plan* p, int ph, cudaStream_t st) : pl(p), phase(ph), idx(-1), s(st) {
    if (pl->ev_used + 2 <= fmmb_plan::kEvPool) {
      idx = pl->ev_used;
      pl->ev_used += 2;
      FMMB_CUDA(time_mark(pl, pl->evp[idx], s));
    }
    pl->launches++;
  }
  ~PhaseTimer() {
    if (idx >= 0) {
      time_mark(pl, pl->evp[idx + 1], s);
      pl->ev_phase.push_back({phase, idx});
    }
  }
};

// One right-hand side of the complex Helmholtz kernel: qs (sorted complex
// charges) -> near / far sorted complex potentials.  P2P on the side stream;
// P2M, M2M, M2L (all levels), L2L and L2P on the main stream, the dense
// translations through the FP64 pair kernel.
void run_one_helm(fmmb_plan* pl, const float* qs) {
  const int K = pl->K, p = pl->p, lmax = pl->lmax;
  const double k = pl->cfg.wavenumber;
  const bool yuk = pl->cfg.kernel == FMMB_YUKAWA;
  cudaStream_t m = pl->st.main, side = pl->serial ? m : pl->st.side;
  double* pot_near = pl->pot_s.get();
  double* pot_far = pl->pot_s.get() + 2 * (size_t)pl->ni;
  const int nleaf_i = pl->nbox_i[lmax], nleaf_j = pl->nbox_j[lmax];
  const double wleaf = (double)pl->bbox[3] / (double)(1 << lmax);
  FMMB_CUDA(cudaEventRecord(pl->st.fork, m));
  FMMB_CUDA(cudaStreamWaitEvent(side, pl->st.fork, 0));
  FMMB_CUDA(time_mark(pl, pl->ev[0], side));
  {
    PhaseTimer tm(pl, 0, side);
    launch_helm_p2p(pl->cfg.precision == FMMB_MIXED, yuk, (float)k, (float)pl->cfg.eps2, pl->cfg.exclude_self != 0,
                    (float)wleaf, pl->h_p2p_nwork, pl->h_p2p_work.get(),
                    pl->leaf_i.get(), pl->leaf_j.get(), pl->p2p_list.get(), pl->tpos.get(), pl->spos.get(), qs,
                    pot_near, side);
  }
  FMMB_CUDA(time_mark(pl, pl->ev[1], side));
  FMMB_CUDA(cudaEventRecord(pl->st.join, side));
  FMMB_CUDA(time_mark(pl, pl->ev[2], m));
  {
    PhaseTimer tm(pl, 1, m);
    launch_helm_p2m(nleaf_j, p, k, yuk, pl->leafkey_j.get(), pl->leaf_j.get(), pl->spos.get(), qs, pl->bbox, wleaf,
                    pl->M.get() + (size_t)pl->off_j[lmax] * 2 * K, m);
  }
  FMMB_CUDA(time_mark(pl, pl->ev[3], m));
  auto pairs_run = [&](const fmmb_plan::PairJob& job, double* xin, double* out, int atomic, int phase) {
    if (job.ntile <= 0) return;
    PhaseTimer tm(pl, phase, m);
    PairArgs a{};
    a.ntile = job.ntile;
    a.tp = job.tp;
    a.K = 2 * K;
    a.atomic = atomic;
    a.tile_op = job.tile_op.get();
    a.tile_src = job.tile_src.get();
    a.tile_dst = job.tile_dst.get();
    a.opT = pl->d_hops.get();
    a.ostride = (size_t)4 * K * K;
    a.xin = xin;
    a.out = out;
    launch_translate_pairs_f64(a, m);
  };
  // parents are accumulated from their children, level by level
  const size_t above = (size_t)(pl->tot_j - pl->nbox_j[lmax]) * 2 * K;
  if (above) FMMB_CUDA(cudaMemsetAsync(pl->M.get() + (size_t)pl->off_j[lmax - 1] * 2 * K, 0, above * sizeof(double), m));
  for (int lev = lmax - 1; lev >= 2; lev--) pairs_run(*pl->m2m_pairs[lev], pl->M.get(), pl->M.get(), 1, 2);
  FMMB_CUDA(time_mark(pl, pl->ev[4], m));
  FMMB_CUDA(cudaMemsetAsync(pl->L.get(), 0, (size_t)pl->tot_i * 2 * K * sizeof(double), m));
  pairs_run(*pl->h_m2l, pl->M.get(), pl->L.get(), 1, 3);
  for (int lev = 3; lev <= lmax; lev++) pairs_run(*pl->l2l_pairs[lev], pl->L.get(), pl->L.get(), 1, 4);
  FMMB_CUDA(time_mark(pl, pl->ev[5], m));
  {
    PhaseTimer tm(pl, 5, m);
    launch_helm_l2p(nleaf_i, p, k, yuk, pl->leafkey_i.get(), pl->leaf_i.get(), pl->tpos.get(), pl->bbox, wleaf,
                    pl->L.get() + (size_t)pl->off_i[lmax] * 2 * K, pot_far, m);
  }
  FMMB_CUDA(time_mark(pl, pl->ev[6], m));
  FMMB_CUDA(cudaStreamWaitEvent(m, pl->st.join, 0));
}

// Runs one right-hand side: qs (sorted, device) -> near/far sorted outputs.
void run_one(fmmb_plan* pl, const float* qs, bool want_grad) {
  if (helm_family(pl->cfg.kernel)) {
    run_one_helm(pl, qs);
    return;
  }
  const int K = pl->K, p = pl->p, lmax = pl->lmax, ker = pl->cfg.kernel;
  const Sem s = make_sem(pl);
  cudaStream_t m = pl->st.main, side = pl->serial ? m : pl->st.side;
  double* pot_near = pl->pot_s.get();
  double* pot_far = pl->pot_s.get() + pl->ni;
  double* g_near = want_grad ? pl->grad_s.get() : nullptr;
  double* g_far = want_grad ? pl->grad_s.get() + 3 * (size_t)pl->ni : nullptr;
  const int nleaf_i = pl->nbox_i[lmax], nleaf_j = pl->nbox_j[lmax];
  // Near field on the low-priority side stream, in two halves of the work
  // items: the first overlaps the upward pass (P2M / M2M, short dependent
  // launches that leave SMs idle), the second the downward tail (L2L / L2P);
  // the tensor-core M2L, which needs whole SMs, runs between them.
  auto near_field = [&](int l0, int l1, bool last) {
    if (pl->far_only) {  // the near field of this evaluate runs elsewhere
      if (last) FMMB_CUDA(cudaEventRecord(pl->st.join, m));
      return;
    }
    if (l1 <= l0) {
      if (last) FMMB_CUDA(cudaEventRecord(pl->st.join, side));
      return;
    }
    FMMB_CUDA(cudaEventRecord(pl->st.fork, m));
    FMMB_CUDA(cudaStreamWaitEvent(side, pl->st.fork, 0));
    if (l0 == 0) FMMB_CUDA(time_mark(pl, pl->ev[0], side));
    {
      PhaseTimer tm(pl, 0, side);
      const int2* wk = pl->p2p_work.get() + l0;
      if (pl->cfg.precision == FMMB_MIXED)
        launch_p2p_mixed(ker, l1 - l0, wk, pl->leaf_i.get(), pl->leaf_j.get(), pl->p2p_list.get(), pl->tpos.get(),
                         pl->tnrm.get(), pl->spos.get(), pl->snrm.get(), qs, s, pot_near, g_near, pl->ni, side);
      else
        launch_p2p_f64(ker, l1 - l0, wk, pl->leaf_i.get(), pl->leaf_j.get(), pl->p2p_list.get(), pl->tpos.get(),
                       pl->tnrm.get(), pl->spos.get(), pl->snrm.get(), qs, s, pot_near, g_near, pl->ni, side);
    }
    if (last) {
      FMMB_CUDA(time_mark(pl, pl->ev[1], side));
      FMMB_CUDA(cudaEventRecord(pl->st.join, side));
    }
  };
  const int p2p_split = pl->p2p_nwork0;
  near_field(0, p2p_split, false);

  // far field on the main stream
  FMMB_CUDA(time_mark(pl, pl->ev[2], m));
  const double rb_leaf = (double)(pl->bbox[3] / (float)(1 << lmax));
  {
    PhaseTimer tm(pl, 1, m);
    if (pl->ref)  // the reference's spherical formulation, quirks included
      launch_p2m(ker, nleaf_j, p, K, pl->leafkey_j.get(), pl->leaf_j.get(), pl->spos.get(), pl->snrm.get(),
                 qs, pl->d_fac.get(), s, pl->bbox, rb_leaf, pl->M.get() + (size_t)pl->off_j[lmax] * K, m);
    else {
      double* Mleaf = pl->M.get() + (size_t)pl->off_j[lmax] * K;
      bool done = false;
      if (pl->cfg.precision == FMMB_MIXED) {
        if (pl->p2m_nwork > nleaf_j)  // some leaf is summed by several items: its rows start at zero
          FMMB_CUDA(cudaMemsetAsync(Mleaf, 0, (size_t)nleaf_j * K * sizeof(double), m));
        done = launch_p2m_f32(ker, pl->p2m_nwork, pl->p2m_work.get(), p, K, pl->leafkey_j.get(), pl->leaf_j.get(),
                              pl->spos.get(), pl->snrm.get(), qs, pl->bbox, rb_leaf, Mleaf, m);
      }
      if (!done)
        launch_p2m_cart(ker, nleaf_j, p, K, pl->leafkey_j.get(), pl->leaf_j.get(), pl->spos.get(), pl->snrm.get(), qs,
                        pl->d_fac.get(), pl->bbox, rb_leaf, Mleaf, m);
    }
  }
  FMMB_CUDA(time_mark(pl, pl->ev[3], m));
  // upward pass: parents accumulate their children (levels below lmax start at zero)
  if (lmax > 2)
    FMMB_CUDA(cudaMemsetAsync(pl->M.get() + (size_t)pl->off_j[lmax - 1] * K, 0,
                              (size_t)(pl->tot_j - pl->off_j[lmax - 1]) * K * sizeof(double), m));
  auto tc_run = [&](const fmmb_plan::TcJob& job, const float* img, const float* xin, double* out, int phase) {
    PhaseTimer tm(pl, phase, m);
    TcJobArgs a{};
    a.ntile = job.ntile;
    a.K = K;
    a.tile_op = job.tile_op.get();
    a.tile_src = job.tile_src.get();
    a.tile_y = reinterpret_cast<const int2*>(job.tile_y.get());
    a.opimg = img;
    a.xin = xin;
    a.y = pl->tc_y.get();
    a.ys = job.ys;
    a.err = pl->d_err.get();
    launch_translate_tc(a, pl->nsm, m);
    launch_reduce_pairs(job.nred, job.red_rows.get(), job.red_ptr.get(), job.red_idx.get(), pl->tc_y.get(), job.ys, K,
                        out, m);
    pl->launches++;
  };
  auto split = [&](const double* X, float* Xtf, int off, int n, int phase) {
    PhaseTimer tm(pl, phase, m);
    launch_split_tf32(n, K, tc_kpad(K), X + (size_t)off * K, Xtf + (size_t)off * 2 * tc_kpad(K), m);
  };
  auto pairs_run = [&](const fmmb_plan::PairJob& job, const double* opT, const double* xin, double* out, int atomic,
                       int phase) {
    if (job.ntile <= 0) return;
    PhaseTimer tm(pl, phase, m);
    PairArgs a{};
    a.ntile = job.ntile;
    a.tp = job.tp;
    a.K = K;
    a.atomic = atomic;
    a.tile_op = job.tile_op.get();
    a.tile_src = job.tile_src.get();
    a.tile_dst = job.tile_dst.get();
    a.opT = opT;
    a.ostride = pair_op_stride(K);
    a.xin = xin;
    a.out = out;
    launch_translate_pairs_f64(a, m);
  };
  for (int lev = lmax - 1; lev >= 2; lev--)  // parents at lev from their children (several per parent)
    pairs_run(*pl->m2m_pairs[lev], pl->d_m2m_t.get(), pl->M.get(), pl->M.get(), 1, 2);
  if (pl->use_tc) split(pl->M.get(), pl->Mtf.get(), 0, pl->tot_j, 2);  // every level, for the M2L
  if (pl->use_h16) {
    PhaseTimer tm(pl, 2, m);
    launch_split_h16(pl->tot_j, K, pl->M.get(), pl->Xh.get(), pl->xexp.get(), m);
  }
  FMMB_CUDA(time_mark(pl, pl->ev[4], m));
  // downward pass: M2L of every level into zeroed locals, then each level
  // adds its parent's translated local (L2L), top down
  FMMB_CUDA(cudaMemsetAsync(pl->L.get(), 0, (size_t)pl->tot_i * K * sizeof(double), m));
  if (pl->use_tc) {
    tc_run(pl->tc_m2l, pl->d_img_m2l.get(), pl->Mtf.get(), pl->L.get(), 3);
  } else if (pl->use_h16) {
    PhaseTimer tm(pl, 3, m);
    const fmmb_plan::TcJob& job = pl->tc_m2l;
    H16JobArgs a{};
    a.ntile = job.ntile;
    a.K = K;
    a.ys = job.ys;
    a.tile_op = job.tile_op.get();
    a.tile_src = job.tile_src.get();
    a.tile_y = reinterpret_cast<const int2*>(job.tile_y.get());
    a.opimg = pl->d_img_h16.get();
    a.xin = pl->Xh.get();
    a.xexp = pl->xexp.get();
    a.y = pl->tc_y.get();
    a.err = pl->d_err.get();
    launch_translate_h16(a, pl->nsm, m);
    launch_reduce_pairs(job.nred, job.red_rows.get(), job.red_ptr.get(), job.red_idx.get(), pl->tc_y.get(), job.ys, K,
                        pl->L.get(), m);
    pl->launches++;
  } else {
    const size_t opsz = (size_t)316 * K * K;
    for (int lev = 2; lev <= lmax; lev++) {
      PhaseTimer tm(pl, 3, m);
      const int set = pl->ops.m2l_sets > 1 ? lev - 2 : 0;
      const auto& ts = *pl->m2l_tiles[lev];
      launch_translate_f64(ts.ntile, split_for(ts.ntile, kM2LSlots), K, kM2LSlots, ts.boxes.get(), ts.ops.get(),
                           pl->m2l_list.get(), pl->d_m2l.get() + set * opsz, pl->M.get() + (size_t)pl->off_j[lev] * K,
                           pl->L.get(), m);
    }
  }
  near_field(p2p_split, pl->p2p_nwork, true);
  for (int lev = 3; lev <= lmax; lev++)  // children at lev from their parent (one pair each, added by one atomic)
    pairs_run(*pl->l2l_pairs[lev], pl->d_l2l_t.get(), pl->L.get(), pl->L.get(), 1, 4);
  FMMB_CUDA(time_mark(pl, pl->ev[5], m));
  {
    PhaseTimer tm(pl, 5, m);
    if (pl->ref)
      launch_l2p(ker, nleaf_i, p, K, pl->leafkey_i.get(), pl->leaf_i.get(), pl->tpos.get(), pl->tnrm.get(),
                 pl->d_fac.get(), s, pl->bbox, rb_leaf, pl->L.get() + (size_t)pl->off_i[lmax] * K, pot_far, g_far, pl->ni, m);
    else if (!(pl->cfg.precision == FMMB_MIXED && (ker == FMMB_LAPLACE_G || !want_grad) &&
               launch_l2p_f32(ker, pl->m_p2p_nwork, pl->m_p2p_work.get(), p, K, pl->leafkey_i.get(), pl->leaf_i.get(), pl->tpos.get(),
                              pl->tnrm.get(), pl->d_fac.get(), pl->bbox, rb_leaf, s.coef,
                              pl->L.get() + (size_t)pl->off_i[lmax] * K, pot_far, g_far, pl->ni, m)))
      launch_l2p_cart(ker, nleaf_i, p, K, pl->leafkey_i.get(), pl->leaf_i.get(), pl->tpos.get(),
                      pl->tnrm.get(), pl->d_fac.get(), pl->bbox, rb_leaf, s.coef, pl->L.get() + (size_t)pl->off_i[lmax] * K,
                      pot_far, ker == FMMB_LAPLACE_GNI ? nullptr : g_far, pl->ni, m);
    if (want_grad && ker == FMMB_LAPLACE_GNI && !pl->ref)  // its gradient needs the Hessian of the local expansion
      launch_l2p_hess_gni(nleaf_i, p, K, pl->leafkey_i.get(), pl->leaf_i.get(), pl->tpos.get(), pl->tnrm.get(),
                          pl->d_fac.get(), pl->bbox, rb_leaf, s.coef, pl->L.get() + (size_t)pl->off_i[lmax] * K, g_far,
                          pl->ni, m);
  }
  FMMB_CUDA(time_mark(pl, pl->ev[6], m));
  FMMB_CUDA(cudaStreamWaitEvent(m, pl->st.join, 0));
}

// One right-hand side through its captured graph: captured on first use
// after each fmmb_set_geometry (run_one with the plan's private capture stream
// standing in for the main stream, in thread-local capture mode, the side
// stream joining through the fork/join events), then replayed with one launch
// on the main stream (which may be a legacy default stream, where capture is
// not possible).  A graph that fails to instantiate turns graphs off for the
// plan and runs the evaluate directly.
void run_graph(fmmb_plan* pl, bool want_grad, bool far_only = false) {
  const int w = (want_grad ? 1 : 0) + (far_only ? 2 : 0);
  const float* qin = far_only ? pl->qs_far.get() : pl->qs.get();
  cudaStream_t m = pl->st.main;
  if (!pl->gexec[w]) {
    cudaStream_t c = pl->st.cap;
    FMMB_CUDA(cudaStreamBeginCapture(c, cudaStreamCaptureModeThreadLocal));
    cudaGraph_t graph = nullptr;
    pl->st.main = c;
    pl->capturing = true;
    pl->far_only = far_only;
    try {
      run_one(pl, qin, want_grad);
    } catch (...) {
      pl->st.main = m;
      pl->capturing = false;
      pl->far_only = false;
      cudaStreamEndCapture(c, &graph);
      if (graph) cudaGraphDestroy(graph);
      cudaGetLastError();
      throw;
    }
    pl->st.main = m;
    pl->capturing = false;
    pl->far_only = false;
    FMMB_CUDA(cudaStreamEndCapture(c, &graph));
    cudaGraphExec_t exec = nullptr;
    const cudaError_t e = cudaGraphInstantiate(&exec, graph, cudaGraphInstantiateFlagUseNodePriority);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) {
      cudaGetLastError();
      pl->use_graph = false;
      pl->ev_used = 0;
      pl->ev_phase.clear();
      pl->far_only = far_only;
      run_one(pl, qin, want_grad);
      pl->far_only = false;
      return;
    }
    pl->gexec[w] = exec;
    pl->gphase[w] = pl->ev_phase;
    pl->glaunches[w] = pl->launches;
  }
  pl->ev_phase = pl->gphase[w];
  pl->launches = pl->glaunches[w];
  FMMB_CUDA(cudaGraphLaunch(pl->gexec[w], m));
}

template <typename T>
int evaluate_impl(fmmb_plan* pl, const float* q, T* pot, T* grad) {
  return guarded([&] {
    FMMB_REQUIRE(pl && q && pot, FMMB_ERR_ARG, "null argument");
    FMMB_REQUIRE(pl->have_geometry, FMMB_ERR_STATE, "fmmb_set_geometry must come first");
    cudaStream_t m = pl->st.main;
    const int ni = pl->ni, nj = pl->nj, nr = pl->cfg.nrhs;
    // gradient output: G, and the normal-derivative kernels in accurate
    // semantics (the gradient w.r.t. the target position, normals fixed)
    const bool gn = pl->cfg.kernel == FMMB_LAPLACE_GNI || pl->cfg.kernel == FMMB_LAPLACE_GNJ;
    FMMB_REQUIRE(!(grad && gn && pl->ref), FMMB_ERR_ARG,
                 "gradients of the normal-derivative kernels need FMMB_SEM_ACCURATE");
    const bool want_grad = grad && (pl->cfg.kernel == FMMB_LAPLACE_G || gn);
    if (*pl->h_err) {  // reported by the tensor-core kernel of an earlier call
      const int e = *pl->h_err;
      *pl->h_err = 0;
      FMMB_CUDA(cudaMemsetAsync(pl->d_err.get(), 0, sizeof(int), pl->st.main));
      throw Error{FMMB_ERR_CUDA, "tensor-core M2L pipeline wait timed out (code " + std::to_string(e) + ")"};
    }
    pl->ev_used = 0;
    pl->ev_phase.clear();
    pl->launches = 0;
    FMMB_CUDA(cudaEventRecord(pl->ev[7], m));
    if (helm_family(pl->cfg.kernel)) {
      // Helmholtz: complex charges and potentials, interleaved; Yukawa: real
      // ones, run through the same complex pipeline with zero imaginary parts
      const bool yuk = pl->cfg.kernel == FMMB_YUKAWA;
      const size_t cw = yuk ? 1 : 2;
      const float* qd = to_device(q, cw * nj * nr, pl->stage_f, m);
      if (yuk) launch_helm_gather_real(nj, nr, pl->perm_j.get(), qd, pl->qs.get(), m);
      else launch_helm_gather(nj, nr, pl->perm_j.get(), qd, pl->qs.get(), m);
      pl->launches++;
      const bool pot_dev = is_device_ptr(pot);
      T* pd = pot;
      if (!pot_dev) {
        pl->stage_out.alloc(cw * ni * nr * sizeof(T));
        pd = (T*)pl->stage_out.get();
      }
      for (int r = 0; r < nr; r++) {
        if (pl->use_graph) {
          if (r > 0)
            FMMB_CUDA(cudaMemcpyAsync(pl->qs.get(), pl->qs.get() + (size_t)2 * r * nj, (size_t)2 * nj * sizeof(float),
                                      cudaMemcpyDeviceToDevice, m));
          run_graph(pl, false);
        } else {
          run_one(pl, pl->qs.get() + (size_t)2 * r * nj, false);
        }
        if (yuk)  // (pi/2) e^{-l r}/(l r) = (2 pi^2 / l) e^{-l r}/(4 pi r)
          launch_helm_finalize_real<T>(ni, pl->perm_i.get(), pl->pot_s.get(), pl->pot_s.get() + 2 * (size_t)ni,
                                       2.0 * M_PI * M_PI / pl->cfg.wavenumber, pd + (size_t)r * ni, m);
        else
          launch_helm_finalize<T>(ni, pl->perm_i.get(), pl->pot_s.get(), pl->pot_s.get() + 2 * (size_t)ni,
                                  pd + (size_t)2 * r * ni, m);
        pl->launches++;
      }
      FMMB_CUDA(cudaEventRecord(pl->ev[6], m));
      FMMB_CUDA(cudaMemcpyAsync(pl->h_err, pl->d_err.get(), sizeof(int), cudaMemcpyDeviceToHost, m));
      if (!pot_dev) FMMB_CUDA(cudaMemcpyAsync(pot, pd, cw * ni * nr * sizeof(T), cudaMemcpyDeviceToHost, m));
      if (!pot_dev || !is_device_ptr(q)) FMMB_CUDA(cudaStreamSynchronize(m));
      pl->have_expansions = true;
      pl->timings_valid = true;
      return;
    }
    const float* qd = to_device(q, (size_t)nj * nr, pl->stage_f, m);
    launch_gather_charges(nj, nr, pl->perm_j.get(), qd, pl->qs.get(), m);
    pl->launches++;
    const bool pot_dev = is_device_ptr(pot);
    const bool grad_dev = want_grad && is_device_ptr(grad);
    // device destinations (staged through the plan when the caller gave host memory)
    T* pd = pot_dev ? pot : nullptr;
    T* gd = grad_dev ? grad : nullptr;
    size_t need = 0;
    if (!pot_dev) need += (size_t)ni * nr;
    if (want_grad && !grad_dev) need += (size_t)3 * ni * nr;
    if (need) {
      pl->stage_out.alloc(need * sizeof(T));
      char* base = (char*)pl->stage_out.get();
      if (!pot_dev) {
        pd = (T*)base;
        base += (size_t)ni * nr * sizeof(T);
      }
      if (want_grad && !grad_dev) gd = (T*)base;
    }
    // several right-hand sides in the mixed form: the near field of all of
    // them in one pass on the side stream (sources read once for every
    // right-hand side), the far field of each through the far-field graph
    const bool multi = nr > 1 && pl->cfg.precision == FMMB_MIXED && pl->use_graph && !(want_grad && gn);
    if (multi) {
      pl->near_all.alloc((size_t)nr * ni * (want_grad ? 4 : 1));
      pl->qs_far.alloc(nj);
      cudaStream_t ns = pl->serial ? m : pl->st.side;
      FMMB_CUDA(cudaEventRecord(pl->st.fork, m));
      FMMB_CUDA(cudaStreamWaitEvent(ns, pl->st.fork, 0));
      pl->launches += launch_p2p_multi(pl->cfg.kernel, nr, pl->m_p2p_nwork, pl->m_p2p_work.get(), pl->leaf_i.get(),
                                       pl->leaf_j.get(), pl->p2p_list.get(), pl->tpos.get(), pl->tnrm.get(),
                                       pl->spos.get(), pl->snrm.get(), pl->qs.get(), nj, make_sem(pl),
                                       pl->near_all.get(), want_grad ? pl->near_all.get() + (size_t)nr * ni : nullptr,
                                       ni, ns);
      FMMB_CUDA(cudaEventRecord(pl->st.near_done, ns));
    }
    for (int r = 0; r < nr; r++) {
      if (multi) {
        FMMB_CUDA(cudaMemcpyAsync(pl->qs_far.get(), pl->qs.get() + (size_t)r * nj, (size_t)nj * sizeof(float),
                                  cudaMemcpyDeviceToDevice, m));
        run_graph(pl, want_grad, true);
        if (r == 0) FMMB_CUDA(cudaStreamWaitEvent(m, pl->st.near_done, 0));
      } else if (pl->use_graph) {
        // the graph reads the charges of the first block: move right-hand
        // side r there once the previous one is consumed (stream order)
        if (r > 0)
          FMMB_CUDA(cudaMemcpyAsync(pl->qs.get(), pl->qs.get() + (size_t)r * nj, (size_t)nj * sizeof(float),
                                    cudaMemcpyDeviceToDevice, m));
        run_graph(pl, want_grad);
      } else {
        run_one(pl, pl->qs.get() + (size_t)r * nj, want_grad);
      }
      // near and far parts of right-hand side r
      const double* pnear = multi ? pl->near_all.get() + (size_t)r * ni : pl->pot_s.get();
      const double* gnear = multi ? pl->near_all.get() + (size_t)nr * ni + (size_t)3 * r * ni : pl->grad_s.get();
      const double* pfar = pl->pot_s.get() + ni;
      const double* gfar = pl->grad_s.get() + 3 * (size_t)ni;
      if (sizeof(T) == 4)
        launch_finalize_f32(ni, pl->perm_i.get(), pnear, pfar, want_grad ? gnear : nullptr, want_grad ? gfar : nullptr,
                            (float*)(pd + (size_t)r * ni), want_grad ? (float*)(gd + (size_t)3 * r * ni) : nullptr, m);
      else
        launch_finalize_f64(ni, pl->perm_i.get(), pnear, pfar, want_grad ? gnear : nullptr, want_grad ? gfar : nullptr,
                            (double*)(pd + (size_t)r * ni), want_grad ? (double*)(gd + (size_t)3 * r * ni) : nullptr, m);
      pl->launches++;
    }
    FMMB_CUDA(cudaEventRecord(pl->ev[6], m));
    FMMB_CUDA(cudaMemcpyAsync(pl->h_err, pl->d_err.get(), sizeof(int), cudaMemcpyDeviceToHost, m));
    if (!pot_dev) FMMB_CUDA(cudaMemcpyAsync(pot, pd, (size_t)ni * nr * sizeof(T), cudaMemcpyDeviceToHost, m));
    if (want_grad && !grad_dev) FMMB_CUDA(cudaMemcpyAsync(grad, gd, (size_t)3 * ni * nr * sizeof(T), cudaMemcpyDeviceToHost, m));
    if (!pot_dev || (want_grad && !grad_dev) || !is_device_ptr(q)) FMMB_CUDA(cudaStreamSynchronize(m));
    pl->have_expansions = true;
    pl->timings_valid = true;
  });
}

}  // namespace

extern "C" {

int fmmb_evaluate(fmmb_plan* pl, const float* q, float* pot, float* grad) { return evaluate_impl<float>(pl, q, pot, grad); }
int fmmb_evaluate_f64(fmmb_plan* pl, const float* q, double* pot, double* grad) {
  return evaluate_impl<double>(pl, q, pot, grad);
}

}  // extern "C"

namespace {

// Times one evaluate per octree depth in [lmin, lmax_hi] on the geometry that
// set_geo gives a fresh plan, and returns the fastest depth.
template <typename SetGeo>
int autotune_impl(const fmmb_config* cfg, int ni, int nj, int lmin, int lmax_hi, int reps, int* best, float* ms_out,
                  SetGeo set_geo) {
  return guarded([&] {
    FMMB_REQUIRE(cfg && best, FMMB_ERR_ARG, "null argument");
    FMMB_REQUIRE(ni >= 1 && nj >= 1, FMMB_ERR_ARG, "need at least one target and one source");
    if (lmin <= 0 || lmax_hi <= 0) {  // around 64 points per leaf of a uniform cloud, then one coarser / two finer
      int l = 2;
      while (l < 10 && (double)std::max(ni, nj) / std::pow(8.0, l) > 64.0) l++;
      lmin = std::max(2, l - 1);
      lmax_hi = std::min(10, l + 2);
    }
    FMMB_REQUIRE(2 <= lmin && lmin <= lmax_hi && lmax_hi <= 10, FMMB_ERR_ARG, "lmax range must lie in [2, 10]");
    reps = std::max(1, reps);
    // random charges on the device (caller order), one FP64 output buffer
    const size_t cw = cfg->kernel == FMMB_HELMHOLTZ_G ? 2 : 1;  // complex: interleaved (Yukawa is real)
    std::vector<float> hq(cw * nj * std::max(1, cfg->nrhs));
    uint64_t st = 0x9E3779B97F4A7C15ull;
    for (auto& v : hq) {
      st = st * 6364136223846793005ull + 1442695040888963407ull;
      v = (float)((st >> 40) * (2.0 / 16777216.0) - 1.0);
    }
    DevBuf<float> dq;
    dq.alloc(hq.size());
    FMMB_CUDA(cudaMemcpy(dq.get(), hq.data(), hq.size() * sizeof(float), cudaMemcpyHostToDevice));
    DevBuf<float> dpot, dgrad;
    dpot.alloc(cw * ni * std::max(1, cfg->nrhs));
    dgrad.alloc((size_t)3 * ni * std::max(1, cfg->nrhs));
    cudaEvent_t e0, e1;
    FMMB_CUDA(cudaEventCreate(&e0));
    FMMB_CUDA(cudaEventCreate(&e1));
    float best_ms = 0.f;
    *best = -1;
    for (int l = lmin; l <= lmax_hi; l++) {
      fmmb_config c = *cfg;
      c.lmax = l;
      fmmb_plan* pl = nullptr;
      int rc = fmmb_plan_create(&c, &pl);
      if (rc == FMMB_OK) rc = set_geo(pl);
      float ms = -1.f;
      if (rc == FMMB_OK) {
        float* g = cfg->kernel == FMMB_LAPLACE_G ? dgrad.get() : nullptr;
        rc = fmmb_evaluate(pl, dq.get(), dpot.get(), g);  // warm-up (captures the graph)
        if (rc == FMMB_OK) {
          FMMB_CUDA(cudaEventRecord(e0, pl->st.main));
          for (int r = 0; r < reps && rc == FMMB_OK; r++) rc = fmmb_evaluate(pl, dq.get(), dpot.get(), g);
          FMMB_CUDA(cudaEventRecord(e1, pl->st.main));
          FMMB_CUDA(cudaEventSynchronize(e1));
          FMMB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
          ms /= reps;
        }
      }
      const std::string err = rc == FMMB_OK ? std::string() : std::string(fmmb_last_error());
      if (pl) fmmb_plan_destroy(pl);
      if (rc == FMMB_ERR_NOMEM || rc == FMMB_ERR_CAPACITY) ms = -1.f;  // this depth does not fit: skip it
      else if (rc != FMMB_OK) {
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        throw Error{rc, "autotune at lmax " + std::to_string(l) + ": " + err};
      }
      if (ms_out) ms_out[l - lmin] = ms;
      if (ms >= 0.f && (*best < 0 || ms < best_ms)) {
        best_ms = ms;
        *best = l;
      }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    FMMB_REQUIRE(*best >= 0, FMMB_ERR_NOMEM, "no octree depth in the range fits on the device");
  });
}

}  // namespace

extern "C" {

int fmmb_autotune_lmax(const fmmb_config* cfg, int ni, const float* tx, const float* ty, const float* tz,
                       const float* tnx, const float* tny, const float* tnz, int nj, const float* sx, const float* sy,
                       const float* sz, const float* snx, const float* sny, const float* snz, const float* bbox,
                       int lmin, int lmax_hi, int reps, int* best, float* ms_out) {
  return autotune_impl(cfg, ni, nj, lmin, lmax_hi, reps, best, ms_out, [&](fmmb_plan* pl) {
    return fmmb_set_geometry(pl, ni, tx, ty, tz, tnx, tny, tnz, nj, sx, sy, sz, snx, sny, snz, bbox);
  });
}

int fmmb_autotune_order(const fmmb_config* cfg, int ni, const float* tx, const float* ty, const float* tz,
                        const float* tnx, const float* tny, const float* tnz, int nj, const float* sx, const float* sy,
                        const float* sz, const float* snx, const float* sny, const float* snz, const float* bbox,
                        double tol, int p_lo, int p_hi, int nsample, int reps, int* p_out, int* lmax_out,
                        double* err_out, float* ms_out) {
  return guarded([&] {
    FMMB_REQUIRE(cfg && p_out && lmax_out, FMMB_ERR_ARG, "null argument");
    FMMB_REQUIRE(!helm_family(cfg->kernel), FMMB_ERR_ARG, "order autotuning takes the Laplace kernels");
    FMMB_REQUIRE(tol > 0.0 && 1 <= p_lo && p_lo <= p_hi && p_hi <= 20, FMMB_ERR_ARG,
                 "need tol > 0 and 1 <= p_lo <= p_hi <= 20");
    FMMB_REQUIRE(ni >= 1 && nj >= 1, FMMB_ERR_ARG, "need at least one target and one source");
    nsample = std::max(1, std::min(nsample > 0 ? nsample : 1024, ni));
    // pseudo-random charges (caller order) and the FP64 direct sums on the
    // sample: 16 runs of consecutive targets spread over [0, ni)
    std::vector<float> hq(nj);
    uint64_t st = 0x2545F4914F6CDD1Dull;
    for (auto& v : hq) {
      st = st * 6364136223846793005ull + 1442695040888963407ull;
      v = (float)((st >> 40) * (2.0 / 16777216.0) - 1.0);
    }
    DevBuf<float> dq;
    dq.alloc(nj);
    FMMB_CUDA(cudaMemcpy(dq.get(), hq.data(), nj * sizeof(float), cudaMemcpyHostToDevice));
    const int nrun = std::min(16, nsample), per = nsample / nrun;
    std::vector<std::pair<int, int>> runs;
    for (int r = 0; r < nrun; r++) {
      const int a = (int)((long long)ni * r / nrun);
      runs.push_back({a, std::min(ni, a + per)});
    }
    std::vector<double> ref;
    {
      fmmb_config c = *cfg;
      c.nrhs = 1;
      c.lmax = 2;
      fmmb_plan* pl = nullptr;
      int rc = fmmb_plan_create(&c, &pl);
      if (rc == FMMB_OK) rc = fmmb_set_geometry(pl, ni, tx, ty, tz, tnx, tny, tnz, nj, sx, sy, sz, snx, sny, snz, bbox);
      for (const auto& r : runs) {
        std::vector<double> h(r.second - r.first);
        if (rc == FMMB_OK) rc = fmmb_direct_f64(pl, dq.get(), r.first, r.second, h.data(), nullptr);
        ref.insert(ref.end(), h.begin(), h.end());
      }
      const std::string err = rc == FMMB_OK ? std::string() : std::string(fmmb_last_error());
      if (pl) fmmb_plan_destroy(pl);
      if (rc != FMMB_OK) throw Error{rc, "order autotune, direct sum: " + err};
    }
    double rn = 0.0;
    for (double v : ref) rn += v * v;
    DevBuf<double> dpot;
    dpot.alloc(ni);
    std::vector<double> pot(ni);
    *p_out = -1;
    for (int p = p_lo; p <= p_hi; p++) {
      fmmb_config c = *cfg;
      c.p = p;
      c.nrhs = 1;
      int best = -1;
      std::vector<float> ms(16, -1.f);
      int rc = fmmb_autotune_lmax(&c, ni, tx, ty, tz, tnx, tny, tnz, nj, sx, sy, sz, snx, sny, snz, bbox, 0, 0, reps,
                                  &best, ms.data());
      if (rc != FMMB_OK) throw Error{rc, "order autotune at p " + std::to_string(p) + ": " + fmmb_last_error()};
      c.lmax = best;
      fmmb_plan* pl = nullptr;
      rc = fmmb_plan_create(&c, &pl);
      if (rc == FMMB_OK) rc = fmmb_set_geometry(pl, ni, tx, ty, tz, tnx, tny, tnz, nj, sx, sy, sz, snx, sny, snz, bbox);
      if (rc == FMMB_OK) rc = fmmb_evaluate_f64(pl, dq.get(), dpot.get(), nullptr);
      const std::string err = rc == FMMB_OK ? std::string() : std::string(fmmb_last_error());
      if (pl) fmmb_plan_destroy(pl);
      if (rc != FMMB_OK) throw Error{rc, "order autotune at p " + std::to_string(p) + ": " + err};
      FMMB_CUDA(cudaMemcpy(pot.data(), dpot.get(), ni * sizeof(double), cudaMemcpyDeviceToHost));
      double dn = 0.0;
      size_t k = 0;
      for (const auto& r : runs)
        for (int i = r.first; i < r.second; i++, k++) dn += (pot[i] - ref[k]) * (pot[i] - ref[k]);
      const double e = rn > 0.0 ? std::sqrt(dn / rn) : std::sqrt(dn);
      *p_out = p;
      *lmax_out = best;
      if (err_out) *err_out = e;
      if (ms_out) {
        // the chosen depth's time: autotune_lmax's range starts at its own estimate
        int l = 2;
        while (l < 10 && (double)std::max(ni, nj) / std::pow(8.0, l) > 64.0) l++;
        *ms_out = ms[best - std::max(2, l - 1)];
      }
      if (e <= tol) break;
    }
  });
}

int fmmb_autotune_lmax_batch(const fmmb_config* cfg, int nprob, const int* t_off, const float* tx, const float* ty,
                             const float* tz, const float* tnx, const float* tny, const float* tnz, const int* s_off,
                             const float* sx, const float* sy, const float* sz, const float* snx, const float* sny,
                             const float* snz, const float* bbox, int lmin, int lmax_hi, int reps, int* best,
                             float* ms_out) {
  int ni = 0, nj = 0;
  const int rc = guarded([&] {
    FMMB_REQUIRE(t_off && s_off && nprob >= 1, FMMB_ERR_ARG, "null problem offsets");
    for (int w = 0; w < 2; w++) {
      const int* src = (w ? s_off : t_off) + nprob;
      int& dst = w ? nj : ni;
      if (is_device_ptr(src)) FMMB_CUDA(cudaMemcpy(&dst, src, sizeof(int), cudaMemcpyDeviceToHost));
      else dst = *src;
    }
  });
  if (rc != FMMB_OK) return rc;
  return autotune_impl(cfg, ni, nj, lmin, lmax_hi, reps, best, ms_out, [&](fmmb_plan* pl) {
    return fmmb_set_geometry_batch(pl, nprob, t_off, tx, ty, tz, tnx, tny, tnz, s_off, sx, sy, sz, snx, sny, snz,
                                   bbox);
  });
}

}  // extern "C"

namespace {

// The plan with targets and sources swapped (G -> G, Gni -> Gnj, Gnj -> Gni),
// on the same root cube and stream, built on first use.
fmmb_plan* transposed_plan(fmmb_plan* pl) {
  if (pl->tplan) return pl->tplan;
  FMMB_REQUIRE(pl->have_geometry, FMMB_ERR_STATE, "fmmb_set_geometry must come first");
  if (pl->same_sets && (pl->cfg.kernel == FMMB_LAPLACE_G || helm_family(pl->cfg.kernel))) {
    pl->tplan = pl;  // G(x_i - x_j) = G(x_j - x_i) on one point set: A^T = A
    return pl;
  }
  fmmb_config c = pl->cfg;
  c.kernel = pl->cfg.kernel == FMMB_LAPLACE_GNI ? FMMB_LAPLACE_GNJ
             : pl->cfg.kernel == FMMB_LAPLACE_GNJ ? FMMB_LAPLACE_GNI : pl->cfg.kernel;  // G, Helmholtz: symmetric
  fmmb_plan* t = nullptr;
  int rc = fmmb_plan_create(&c, &t);
  if (rc == FMMB_OK) rc = fmmb_set_stream(t, pl->st.main);
  const int ni = pl->ni, nj = pl->nj;
  const float* g = pl->geo.get();
  const float* tg = g;                    // this plan's targets: the transposed sources
  const float* sg = g + (size_t)6 * ni;   // this plan's sources: the transposed targets
  const bool tn = c.kernel == FMMB_LAPLACE_GNI, sn = c.kernel == FMMB_LAPLACE_GNJ;
  if (rc == FMMB_OK)
    rc = geometry_impl(t, pl->nprob, pl->prob_soff.data(), pl->prob_toff.data(), nj, sg, sg + nj, sg + 2 * (size_t)nj,
                       tn ? sg + 3 * (size_t)nj : nullptr, tn ? sg + 4 * (size_t)nj : nullptr,
                       tn ? sg + 5 * (size_t)nj : nullptr, ni, tg, tg + ni, tg + 2 * (size_t)ni,
                       sn ? tg + 3 * (size_t)ni : nullptr, sn ? tg + 4 * (size_t)ni : nullptr,
                       sn ? tg + 5 * (size_t)ni : nullptr, pl->bbox);
  if (rc != FMMB_OK) {
    const std::string msg = fmmb_last_error();
    if (t) fmmb_plan_destroy(t);
    throw Error{rc, "transposed plan: " + msg};
  }
  pl->tplan = t;
  return t;
}

template <typename T>
void negate(T* p, size_t n, cudaStream_t s) {
  if (is_device_ptr(p)) {
    launch_scale(p, n, T(-1), s);
  } else {
    FMMB_CUDA(cudaStreamSynchronize(s));
    for (size_t i = 0; i < n; i++) p[i] = -p[i];
  }
}

template <typename T>
int transpose_impl(fmmb_plan* pl, const float* w, T* out, T* grad) {
  return guarded([&] {
    FMMB_REQUIRE(pl && w && out, FMMB_ERR_ARG, "null argument");
    FMMB_REQUIRE(!helm_family(pl->cfg.kernel) || grad == nullptr, FMMB_ERR_ARG,
                 "the complex kernels' transpose has no gradient output");
    fmmb_plan* t = transposed_plan(pl);
    const int rc = sizeof(T) == 4 ? fmmb_evaluate(t, w, (float*)out, (float*)grad)
                                  : fmmb_evaluate_f64(t, w, (double*)out, (double*)grad);
    if (rc != FMMB_OK) throw Error{rc, std::string(fmmb_last_error())};
    if (pl->cfg.kernel == FMMB_LAPLACE_GNI || pl->cfg.kernel == FMMB_LAPLACE_GNJ) {  // A^T = -(swapped plan)
      negate(out, (size_t)pl->nj * pl->cfg.nrhs, t->st.main);
      if (grad) negate(grad, (size_t)3 * pl->nj * pl->cfg.nrhs, t->st.main);
    }
  });
}

}  // namespace

extern "C" {

int fmmb_evaluate_transpose(fmmb_plan* pl, const float* w, float* out, float* grad) {
  return transpose_impl<float>(pl, w, out, grad);
}
int fmmb_evaluate_transpose_f64(fmmb_plan* pl, const float* w, double* out, double* grad) {
  return transpose_impl<double>(pl, w, out, grad);
}

int fmmb_position_grad(fmmb_plan* pl, const float* q, const float* w, double* dxt, double* dxs) {
  return guarded([&] {
    FMMB_REQUIRE(pl && q && w && (dxt || dxs), FMMB_ERR_ARG, "null argument");
    FMMB_REQUIRE(!helm_family(pl->cfg.kernel), FMMB_ERR_ARG, "position gradients are for the Laplace kernels");
    FMMB_REQUIRE(pl->cfg.kernel == FMMB_LAPLACE_G || !pl->ref, FMMB_ERR_ARG,
                 "position gradients of the normal-derivative kernels need FMMB_SEM_ACCURATE");
    FMMB_REQUIRE(pl->cfg.nrhs == 1, FMMB_ERR_ARG, "position gradients take one right-hand side");
    FMMB_REQUIRE(pl->have_geometry, FMMB_ERR_STATE, "fmmb_set_geometry must come first");
    const int ni = pl->ni, nj = pl->nj;
    cudaStream_t m = pl->st.main;
    // work space: pot[ni], field_t[3 ni], adj[nj], field_s[3 nj], out staging[3 ni + 3 nj]
    pl->pg_tmp.alloc((size_t)4 * ni + 4 * (size_t)nj + 3 * (size_t)ni + 3 * (size_t)nj);
    double* pot = pl->pg_tmp.get();
    double* ft = pot + ni;
    double* adj = ft + 3 * (size_t)ni;
    double* fs = adj + nj;
    double* stage = fs + 3 * (size_t)nj;
    int rc = FMMB_OK;
    if (dxt) rc = fmmb_evaluate_f64(pl, q, pot, ft);
    if (rc == FMMB_OK && dxs) rc = fmmb_evaluate_transpose_f64(pl, w, adj, fs);
    if (rc != FMMB_OK) throw Error{rc, std::string(fmmb_last_error())};
    DevBuf<float> sw, sq;
    const float* wd = to_device(w, ni, sw, m);
    const float* qd = to_device(q, nj, sq, m);
    double* ot = dxt ? (is_device_ptr(dxt) ? dxt : stage) : nullptr;
    double* os = dxs ? (is_device_ptr(dxs) ? dxs : stage + 3 * (size_t)ni) : nullptr;
    if (ot) launch_weight_field(ni, wd, ft, ot, m);   // dL/dx_t = w * grad(pot)(x_t)
    if (os) launch_weight_field(nj, qd, fs, os, m);   // dL/dx_s = q * grad(psi)(x_s)
    if (dxt && ot != dxt) FMMB_CUDA(cudaMemcpyAsync(dxt, ot, 3 * (size_t)ni * sizeof(double), cudaMemcpyDeviceToHost, m));
    if (dxs && os != dxs) FMMB_CUDA(cudaMemcpyAsync(dxs, os, 3 * (size_t)nj * sizeof(double), cudaMemcpyDeviceToHost, m));
    FMMB_CUDA(cudaStreamSynchronize(m));
  });
}

int fmmb_adjoint_f64(fmmb_plan* pl, const float* q, const float* w, const double* field_t, double* dq, double* dxt,
                     double* dxs) {
  return guarded([&] {
    FMMB_REQUIRE(pl && w && (dq || dxt || dxs), FMMB_ERR_ARG, "null argument");
    FMMB_REQUIRE((!dxt && !dxs) || pl->cfg.kernel == FMMB_LAPLACE_G || !pl->ref, FMMB_ERR_ARG,
                 "position gradients of the normal-derivative kernels need FMMB_SEM_ACCURATE");
    FMMB_REQUIRE(!dxt || field_t, FMMB_ERR_ARG, "dxt needs the forward field");
    FMMB_REQUIRE(!dxs || q, FMMB_ERR_ARG, "dxs needs the charges");
    FMMB_REQUIRE(pl->cfg.nrhs == 1 || (!dxt && !dxs), FMMB_ERR_ARG, "position gradients take one right-hand side");
    FMMB_REQUIRE(pl->have_geometry, FMMB_ERR_STATE, "fmmb_set_geometry must come first");
    FMMB_REQUIRE(!helm_family(pl->cfg.kernel), FMMB_ERR_ARG, "the complex kernels use fmmb_evaluate_transpose");
    const int ni = pl->ni, nj = pl->nj;
    const size_t nadj = (size_t)nj * pl->cfg.nrhs;
    cudaStream_t m = pl->st.main;
    // plan-owned work space (allocated on first use): adj[nadj] | field_s[3 nj]
    // | dxs[3 nj] | field_t[3 ni] | dxt[3 ni], and the staged charges / weights
    pl->adj_tmp.alloc(nadj + 6 * (size_t)nj + 6 * (size_t)ni);
    double* adj = pl->adj_tmp.get();
    double* fs = adj + nadj;
    double* os = fs + 3 * (size_t)nj;
    double* ft = os + 3 * (size_t)nj;
    double* ot = ft + 3 * (size_t)ni;
    // host copies that need not wait for the transposed matvec go on a copy
    // stream beside it: dL/dx_t (it needs only w and the forward field) to the
    // host, and q to the device
    const bool host_q = dxs && !is_device_ptr(q), host_dxt = dxt && !is_device_ptr(dxt);
    cudaStream_t cs = m;
    if (host_q || host_dxt) {
      if (!pl->st.copy) {
        FMMB_CUDA(cudaStreamCreateWithFlags(&pl->st.copy, cudaStreamNonBlocking));
        for (auto& e : pl->st.copy_ev) FMMB_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
      }
      cs = pl->st.copy;
      FMMB_CUDA(cudaEventRecord(pl->st.copy_ev[0], m));  // the plan's earlier work on its buffers is done
      FMMB_CUDA(cudaStreamWaitEvent(cs, pl->st.copy_ev[0], 0));
    }
    // w (ni nrhs) and q (nj) staged once when they are host arrays
    const float* wd = to_device(w, (size_t)ni * pl->cfg.nrhs, pl->adj_ws, m);
    const float* qd = dxs ? to_device(q, nj, pl->adj_qs, cs) : nullptr;
    if (dxt) {  // dL/dx_t = w * grad(pot)(x_t)
      const double* fd = field_t;
      if (!is_device_ptr(field_t)) {
        FMMB_CUDA(cudaMemcpyAsync(ft, field_t, 3 * (size_t)ni * sizeof(double), cudaMemcpyHostToDevice, m));
        fd = ft;
      }
      if (!host_dxt) ot = dxt;
      launch_weight_field(ni, wd, fd, ot, m);
      if (host_dxt) {
        FMMB_CUDA(cudaEventRecord(pl->st.copy_ev[0], m));
        FMMB_CUDA(cudaStreamWaitEvent(cs, pl->st.copy_ev[0], 0));
        FMMB_CUDA(cudaMemcpyAsync(dxt, ot, 3 * (size_t)ni * sizeof(double), cudaMemcpyDeviceToHost, cs));
      }
    }
    if (dq || dxs) {
      if (is_device_ptr(dq)) adj = dq;
      const int rc = fmmb_evaluate_transpose_f64(pl, wd, adj, dxs ? fs : nullptr);
      if (rc != FMMB_OK) {
        const std::string msg(fmmb_last_error());
        if (cs != m) cudaStreamSynchronize(cs);  // no copy into the caller's memory after the error returns
        throw Error{rc, msg};
      }
      if (dq && adj != dq) FMMB_CUDA(cudaMemcpyAsync(dq, adj, nadj * sizeof(double), cudaMemcpyDeviceToHost, m));
      if (dxs) {  // dL/dx_s = q * grad(psi)(x_s)
        if (host_q) {
          FMMB_CUDA(cudaEventRecord(pl->st.copy_ev[1], cs));
          FMMB_CUDA(cudaStreamWaitEvent(m, pl->st.copy_ev[1], 0));
        }
        if (is_device_ptr(dxs)) os = dxs;
        launch_weight_field(nj, qd, fs, os, m);
        if (os != dxs) FMMB_CUDA(cudaMemcpyAsync(dxs, os, 3 * (size_t)nj * sizeof(double), cudaMemcpyDeviceToHost, m));
      }
    }
    // host outputs are complete on return; device outputs are ordered on the
    // plan's stream (the copy stream carries host-side work only)
    if (!is_device_ptr(w) || (q && !is_device_ptr(q)) || (dq && !is_device_ptr(dq)) || (dxt && !is_device_ptr(dxt)) ||
        (dxs && !is_device_ptr(dxs)) || (field_t && !is_device_ptr(field_t))) {
      FMMB_CUDA(cudaStreamSynchronize(m));
      if (cs != m) FMMB_CUDA(cudaStreamSynchronize(cs));
    }
  });
}

int fmmb_direct_f64(fmmb_plan* pl, const float* q, int i0, int i1, double* pot, double* grad) {
  return guarded([&] {
    FMMB_REQUIRE(pl && q && pot, FMMB_ERR_ARG, "null argument");
    FMMB_REQUIRE(pl->have_geometry, FMMB_ERR_STATE, "fmmb_set_geometry must come first");
    FMMB_REQUIRE(0 <= i0 && i0 <= i1 && i1 <= pl->ni, FMMB_ERR_ARG, "target range out of bounds");
    cudaStream_t m = pl->st.main;
    const int nj = pl->nj, cnt = i1 - i0;
    if (helm_family(pl->cfg.kernel)) {  // Helmholtz: pot holds 2 cnt doubles (re, im); Yukawa: cnt
      const bool yuk = pl->cfg.kernel == FMMB_YUKAWA;
      const float* qd = to_device(q, (size_t)(yuk ? 1 : 2) * nj, pl->stage_f, m);
      if (yuk) launch_helm_gather_real(nj, 1, pl->perm_j.get(), qd, pl->qs.get(), m);
      else launch_helm_gather(nj, 1, pl->perm_j.get(), qd, pl->qs.get(), m);
      DevBuf<double> out;
      out.alloc((size_t)2 * cnt + 2);
      const std::vector<int>&to = pl->prob_toff, &so = pl->prob_soff;
      for (int b = 0; b < pl->nprob; b++) {
        const int a0 = std::max(i0, to[b]), a1 = std::min(i1, to[b + 1]);
        if (a0 >= a1) continue;
        launch_helm_direct(a0, a1, pl->inv_i.get(), pl->tpos.get(), so[b + 1] - so[b], pl->spos.get() + so[b],
                           pl->qs.get() + (size_t)2 * so[b], pl->cfg.wavenumber, yuk, pl->cfg.eps2,
                           pl->cfg.exclude_self != 0, out.get() + (size_t)2 * (a0 - i0), m);
      }
      if (yuk) {
        std::vector<double> h((size_t)2 * cnt);
        FMMB_CUDA(cudaMemcpyAsync(h.data(), out.get(), h.size() * sizeof(double), cudaMemcpyDeviceToHost, m));
        FMMB_CUDA(cudaStreamSynchronize(m));
        std::vector<double> r(cnt);
        for (int i = 0; i < cnt; i++) r[i] = 2.0 * M_PI * M_PI / pl->cfg.wavenumber * h[2 * (size_t)i];
        FMMB_CUDA(cudaMemcpy(pot, r.data(), cnt * sizeof(double), cudaMemcpyDefault));
        return;
      }
      FMMB_CUDA(cudaMemcpyAsync(pot, out.get(), (size_t)2 * cnt * sizeof(double),
                                is_device_ptr(pot) ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, m));
      FMMB_CUDA(cudaStreamSynchronize(m));
      return;
    }
    const float* qd = to_device(q, nj, pl->stage_f, m);
    launch_gather_charges(nj, 1, pl->perm_j.get(), qd, pl->qs.get(), m);
    const bool want_grad = grad != nullptr;  // every Laplace kernel (w.r.t. the target position, normals fixed)
    DevBuf<double> out;
    out.alloc((size_t)cnt * 4 + 1);
    if (pl->nprob == 1) {
      launch_direct_f64(pl->cfg.kernel, i0, i1, pl->inv_i.get(), pl->tpos.get(), pl->tnrm.get(), nj, pl->spos.get(),
                        pl->snrm.get(), pl->qs.get(), make_sem(pl), out.get(), want_grad ? out.get() + cnt : nullptr, m);
    } else {
      // one launch per problem over its own sources (sorted source positions
      // of problem b are [soff[b], soff[b+1]) like the caller's), then the
      // [pot | gx | gy | gz] blocks of each problem moved into place
      DevBuf<double> tmp;
      tmp.alloc((size_t)cnt * 4 + 1);
      const std::vector<int>&to = pl->prob_toff, &so = pl->prob_soff;
      for (int b = 0; b < pl->nprob; b++) {
        const int a0 = std::max(i0, to[b]), a1 = std::min(i1, to[b + 1]);
        if (a0 >= a1) continue;
        const int mb = a1 - a0;
        double* tb = tmp.get() + (size_t)4 * (a0 - i0);
        launch_direct_f64(pl->cfg.kernel, a0, a1, pl->inv_i.get(), pl->tpos.get(), pl->tnrm.get(), so[b + 1] - so[b],
                          pl->spos.get() + so[b], pl->snrm.get() + so[b], pl->qs.get() + so[b], make_sem(pl), tb,
                          want_grad ? tb + mb : nullptr, m);
        for (int c = 0; c < (want_grad ? 4 : 1); c++)
          FMMB_CUDA(cudaMemcpyAsync(out.get() + (size_t)c * cnt + (a0 - i0), tb + (size_t)c * mb, mb * sizeof(double),
                                    cudaMemcpyDeviceToDevice, m));
      }
    }
    FMMB_CUDA(cudaMemcpyAsync(pot, out.get(), cnt * sizeof(double), is_device_ptr(pot) ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, m));
    if (want_grad)
      FMMB_CUDA(cudaMemcpyAsync(grad, out.get() + cnt, 3 * (size_t)cnt * sizeof(double),
                                is_device_ptr(grad) ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, m));
    FMMB_CUDA(cudaStreamSynchronize(m));
  });
}

}  // extern "C"

namespace {
int tree_record(fmmb_plan* pl, int k, std::vector<int>& v) {
  return guarded([&] {
    FMMB_REQUIRE(pl, FMMB_ERR_ARG, "null plan");
    FMMB_REQUIRE(pl->have_geometry, FMMB_ERR_STATE, "no geometry");
    FMMB_REQUIRE(k >= 0 && k <= 8, FMMB_ERR_ARG, "unknown tree record");
    const int lmax = pl->lmax;
    v.clear();
    auto d2h = [&](const int* src, size_t n) {
      std::vector<int> h(n);
      if (n) FMMB_CUDA(cudaMemcpy(h.data(), src, n * sizeof(int), cudaMemcpyDeviceToHost));
      return h;
    };
    if (k == 0) v = d2h(pl->perm_i.get(), pl->ni);
    else if (k == 1) v = d2h(pl->perm_j.get(), pl->nj);
    else if (k == 2) v = d2h(pl->key_i.get(), pl->tot_i);
    else if (k == 3) v = d2h(pl->key_j.get(), pl->tot_j);
    else if (k == 4 || k == 5) {
      v.assign(lmax + 1, 0);
      for (int l = 2; l <= lmax; l++) v[l] = (k == 4 ? pl->nbox_i : pl->nbox_j)[l];
    } else if (k == 6 || k == 7) {
      const int nl = (k == 6 ? pl->nbox_i : pl->nbox_j)[lmax];
      std::vector<int2> lf(nl);
      FMMB_CUDA(cudaMemcpy(lf.data(), (k == 6 ? pl->leaf_i : pl->leaf_j).get(), nl * sizeof(int2), cudaMemcpyDeviceToHost));
      for (auto& x : lf) {
        v.push_back(x.x);
        v.push_back(x.x + x.y - 1);
      }
    } else {
      // lists in the order fmm() builds them: near field at lmax, level 2, levels 3..lmax
      const int nli = pl->nbox_i[lmax];
      std::vector<int> near = d2h(pl->p2p_list.get(), (size_t)nli * kP2PSlots);
      std::vector<int> far = d2h(pl->m2l_list.get(), (size_t)pl->tot_i * kM2LSlots);
      auto emit = [&](int lev, int mode, int nbi, int nbj, const std::vector<std::vector<int>>& L) {
        v.push_back(lev);
        v.push_back(mode);
        v.push_back(nbi);
        v.push_back(nbj);
        for (auto& l : L) v.push_back((int)l.size());
        for (auto& l : L) v.insert(v.end(), l.begin(), l.end());
      };
      std::vector<std::vector<int>> L(nli);
      for (int b = 0; b < nli; b++)
        for (int s = 0; s < kP2PSlots; s++)
          if (near[(size_t)b * kP2PSlots + s] >= 0) L[b].push_back(near[(size_t)b * kP2PSlots + s]);
      emit(lmax, 0, nli, pl->nbox_j[lmax], L);
      for (int lev = 2; lev <= lmax; lev++) {
        std::vector<std::vector<int>> F(pl->nbox_i[lev]);
        for (int b = 0; b < pl->nbox_i[lev]; b++) {
          const size_t g = (size_t)(pl->off_i[lev] + b) * kM2LSlots;
          for (int s = 0; s < kM2LSlots; s++)
            if (far[g + s] >= 0) F[b].push_back(far[g + s]);
          // level 2 visits every source box in index order (fmm/ijbox.cxx:62-72)
          if (lev == 2) std::sort(F[b].begin(), F[b].end());
        }
        emit(lev, lev == 2 ? 1 : 2, pl->nbox_i[lev], pl->nbox_j[lev], F);
      }
    }
  });
}
}  // namespace

extern "C" {

long fmmb_get_tree_size(fmmb_plan* pl, int kind) {
  std::vector<int> v;
  const int rc = tree_record(pl, kind, v);
  return rc != FMMB_OK ? rc : (long)v.size();
}

int fmmb_get_tree(fmmb_plan* pl, int kind, int* out) {
  std::vector<int> v;
  const int rc = tree_record(pl, kind, v);
  if (rc == FMMB_OK && out && !v.empty()) std::memcpy(out, v.data(), v.size() * sizeof(int));
  return rc;
}

long fmmb_get_expansion_size(fmmb_plan* pl, int which) {
  if (!pl || !pl->have_geometry || (which != 0 && which != 1)) return FMMB_ERR_ARG;
  return (long)(which == 0 ? pl->tot_j : pl->tot_i) * pl->P * 2;
}

int fmmb_get_expansions(fmmb_plan* pl, int which, double* out) {
  return guarded([&] {
    FMMB_REQUIRE(pl && out && (which == 0 || which == 1), FMMB_ERR_ARG, "bad argument");
    FMMB_REQUIRE(pl->have_expansions, FMMB_ERR_STATE, "no evaluate yet");
    FMMB_CUDA(cudaStreamSynchronize(pl->st.main));
    const int tot = which == 0 ? pl->tot_j : pl->tot_i;
    const int K = pl->K, p = pl->p, P = pl->P;
    std::vector<double> h((size_t)tot * K);
    FMMB_CUDA(cudaMemcpy(h.data(), (which == 0 ? pl->M : pl->L).get(), h.size() * sizeof(double), cudaMemcpyDeviceToHost));
    const std::vector<int>& off = which == 0 ? pl->off_j : pl->off_i;
    for (int lev = pl->lmax; lev >= 2; lev--) {
      const double rb = (double)(pl->bbox[3] / (float)(1 << lev));
      const int nb = (which == 0 ? pl->nbox_j : pl->nbox_i)[lev];
      for (int b = 0; b < nb; b++) {
        const double* v = &h[(size_t)(off[lev] + b) * K];
        double* o = out + (size_t)(off[lev] + b) * P * 2;
        for (int n = 0; n <= p; n++) {
          // undo the scaling: M_n = M^_n rb^n, L_n = L^_n / rb^(n+1)
          const double sc = which == 0 ? std::pow(rb, n) : std::pow(rb, -(n + 1));
          o[2 * isym(n, 0)] = v[n * n] * sc;
          o[2 * isym(n, 0) + 1] = 0.0;
          for (int mm = 1; mm <= n; mm++) {
            o[2 * isym(n, mm)] = v[n * n + 2 * mm - 1] * sc;
            o[2 * isym(n, mm) + 1] = v[n * n + 2 * mm] * sc;
          }
        }
      }
    }
  });
}

int fmmb_get_timings(fmmb_plan* pl, float* ms) {
  return guarded([&] {
    FMMB_REQUIRE(pl && ms, FMMB_ERR_ARG, "null argument");
    FMMB_REQUIRE(pl->timings_valid, FMMB_ERR_STATE, "no evaluate yet");
    FMMB_CUDA(cudaStreamSynchronize(pl->st.main));
    FMMB_CUDA(cudaStreamSynchronize(pl->st.side));
    FMMB_REQUIRE(*pl->h_err == 0, FMMB_ERR_CUDA, "tensor-core M2L pipeline wait timed out");
    for (int k = 0; k < 7; k++) ms[k] = 0.0f;
    for (auto& ph : pl->ev_phase) {
      float t = 0;
      FMMB_CUDA(cudaEventElapsedTime(&t, pl->evp[ph.second], pl->evp[ph.second + 1]));
      ms[ph.first] += t;
    }
    float tot = 0;
    FMMB_CUDA(cudaEventElapsedTime(&tot, pl->ev[7], pl->ev[6]));
    ms[6] = tot;
  });
}

int fmmb_set_overlap(fmmb_plan* pl, int on) {
  return guarded([&] {
    FMMB_REQUIRE(pl, FMMB_ERR_ARG, "null plan");
    if (pl->serial == (on == 0)) return;
    for (int w = 0; w < 4; w++) {  // captured with the other stream layout
      if (pl->gexec[w]) {
        FMMB_CUDA(cudaStreamSynchronize(pl->st.main));
        cudaGraphExecDestroy(pl->gexec[w]);
        pl->gexec[w] = nullptr;
      }
    }
    pl->serial = on == 0;
  });
}

int fmmb_get_setup_times(fmmb_plan* pl, double* ms) {
  return guarded([&] {
    FMMB_REQUIRE(pl && ms, FMMB_ERR_ARG, "null argument");
    FMMB_REQUIRE(pl->have_geometry, FMMB_ERR_STATE, "no geometry");
    ms[0] = pl->tree_ms;
    ms[1] = pl->setup_ms;
  });
}

int fmmb_get_stats(fmmb_plan* pl, long long* o) {
  return guarded([&] {
    FMMB_REQUIRE(pl && o, FMMB_ERR_ARG, "null argument");
    FMMB_REQUIRE(pl->have_geometry, FMMB_ERR_STATE, "no geometry");
    o[0] = pl->ni;
    o[1] = pl->nj;
    o[2] = pl->nbox_i[pl->lmax];
    o[3] = pl->nbox_j[pl->lmax];
    o[4] = pl->p2p_pairs;
    o[5] = pl->m2l_pairs;
    o[6] = pl->lmax;
    o[7] = pl->launches;
  });
}

}  // extern "C"

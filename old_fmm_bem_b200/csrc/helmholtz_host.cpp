// Host side of the complex Helmholtz kernel (FMMB_HELMHOLTZ_G): the per-level
// translation operators (built on the GPU by helmholtz.cu) and the pair jobs
// that apply them with the FP64 pair kernel.  Called by fmmb_set_geometry
// after the octree is built; the evaluation itself is in api.cpp.
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <vector>

#include "internal.h"
#include "kernels.h"

namespace fmmb {
namespace {

// Gauss-Legendre nodes and weights on [-1, 1] (Newton on P_n from the
// Chebyshev guesses)
void gauss_legendre(int n, std::vector<double>& x, std::vector<double>& w) {
  x.assign(n, 0.0);
  w.assign(n, 0.0);
  for (int i = 0; i < n; i++) {
    double z = std::cos(M_PI * (i + 0.75) / (n + 0.5)), dp = 1.0;
    for (int it = 0; it < 100; it++) {
      double p0 = 1.0, p1 = z;
      for (int k = 2; k <= n; k++) {
        const double p2 = ((2.0 * k - 1.0) * z * p1 - (k - 1.0) * p0) / k;
        p0 = p1;
        p1 = p2;
      }
      dp = n * (z * p1 - p0) / (z * z - 1.0);
      const double dz = p1 / dp;
      z -= dz;
      if (std::fabs(dz) < 1e-16) break;
    }
    {
      double p0 = 1.0, p1 = z;
      for (int k = 2; k <= n; k++) {
        const double p2 = ((2.0 * k - 1.0) * z * p1 - (k - 1.0) * p0) / k;
        p0 = p1;
        p1 = p2;
      }
      dp = n * (z * p1 - p0) / (z * z - 1.0);
    }
    x[i] = z;
    w[i] = 2.0 / ((1.0 - z * z) * dp * dp);
  }
}

// Ybar_n^m(x), m >= 0, the fully normalised recurrence of helmholtz.cu,
// [n (n+1) / 2 + m]
void ybar_table(int p, double x, double* out) {
  const double s = std::sqrt(std::max(0.0, 1.0 - x * x));
  double ymm = 0.28209479177387814;
  for (int m = 0; m <= p; m++) {
    if (m > 0) ymm = std::sqrt((2.0 * m + 1.0) / (2.0 * m)) * s * ymm;
    double y2 = 0.0, y1 = ymm;
    for (int n = m; n <= p; n++) {
      double y;
      if (n == m) {
        y = ymm;
      } else if (n == m + 1) {
        y = std::sqrt(2.0 * m + 3.0) * x * ymm;
      } else {
        const double a = std::sqrt((4.0 * n * n - 1.0) / ((double)n * n - (double)m * m));
        const double b = std::sqrt((((double)n - 1) * (n - 1) - (double)m * m) / (4.0 * (n - 1) * (n - 1) - 1.0));
        y = a * (x * y1 - b * y2);
      }
      if (n > m) {
        y2 = y1;
        y1 = y;
      }
      out[n * (n + 1) / 2 + m] = y;
    }
  }
}

template <typename T>
void upload_vec(DevBuf<T>& d, const std::vector<T>& h) {
  d.alloc(h.size());
  if (!h.empty()) FMMB_CUDA(cudaMemcpy(d.get(), h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice));
}

// {operator, input row, output row} -> tiles of tp pairs of one operator
std::unique_ptr<fmmb_plan::PairJob> pair_job(std::vector<std::array<int, 3>>& pairs, int Kreal, int nsm) {
  std::unique_ptr<fmmb_plan::PairJob> job(new fmmb_plan::PairJob());
  std::stable_sort(pairs.begin(), pairs.end(),
                   [](const std::array<int, 3>& a, const std::array<int, 3>& b) { return a[0] < b[0]; });
  const int tp = pairs_f64_tile(Kreal, (int)pairs.size(), nsm);
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
  upload_vec(job->tile_op, top);
  upload_vec(job->tile_src, tsrc);
  upload_vec(job->tile_dst, tdst);
  return job;
}

}  // namespace

void helm_setup(fmmb_plan* pl) {
  const int p = pl->p, K = pl->K, lmax = pl->lmax;
  const double k = pl->cfg.wavenumber, rd = pl->bbox[3];
  cudaStream_t s = pl->st.main;
  auto width = [&](int l) { return rd / (double)(1 << l); };
  // operators: M2M for child levels 3..lmax (8 octants each), L2L likewise,
  // M2L for levels 2..lmax (316 relative positions each)
  std::vector<HelmOp> ops;
  auto octant_offset = [&](int oct, double wc, double* o) {  // child centre - parent centre
    o[0] = (((oct >> 1) & 1) - 0.5) * wc;  // key bit 1: x
    o[1] = ((oct & 1) - 0.5) * wc;         // key bit 0: y
    o[2] = (((oct >> 2) & 1) - 0.5) * wc;  // key bit 2: z
  };
  const bool yuk = pl->cfg.kernel == FMMB_YUKAWA;
  // Helmholtz: keeps k * rad below the first zero of j_0 (i_n of Yukawa has no zeros)
  const double rad_cap = yuk ? 1e300 : 2.5 / k;
  pl->hop_m2m0 = 0;
  for (int lc = 3; lc <= lmax; lc++)
    for (int oct = 0; oct < 8; oct++) {
      double o[3];
      octant_offset(oct, width(lc), o);
      ops.push_back({-o[0], -o[1], -o[2], 2.0 * width(lc - 1), 1, 1});
    }
  pl->hop_l2l0 = (int)ops.size();
  for (int lc = 3; lc <= lmax; lc++)
    for (int oct = 0; oct < 8; oct++) {
      double o[3];
      octant_offset(oct, width(lc), o);
      ops.push_back({o[0], o[1], o[2], std::min(0.8660254037844386 * width(lc), rad_cap), 0, 0});
    }
  pl->hop_m2l0 = (int)ops.size();
  for (int l = 2; l <= lmax; l++)
    for (int slot = 0; slot < 316; slot++) {
      const int code = pl->ops.op_rel[slot];
      const double w = width(l);
      ops.push_back({(code / 49 - 3) * w, ((code / 7) % 7 - 3) * w, (code % 7 - 3) * w,
                     std::min(0.8660254037844386 * w, rad_cap), 1, 0});
    }
  const int nops = (int)ops.size();
  const size_t ostride = (size_t)4 * K * K;
  pl->d_hops.alloc((size_t)nops * ostride);
  {
    const int NQ = 2 * p + 8, P = (p + 1) * (p + 2) / 2;
    std::vector<double> gx, gw;
    gauss_legendre(NQ, gx, gw);
    std::vector<double> yb((size_t)NQ * P);
    for (int i = 0; i < NQ; i++) ybar_table(p, gx[i], yb.data() + (size_t)i * P);
    DevBuf<double> d_gx, d_gw, d_yb;
    DevBuf<HelmOp> d_ops;
    upload_vec(d_gx, gx);
    upload_vec(d_gw, gw);
    upload_vec(d_yb, yb);
    upload_vec(d_ops, ops);
    launch_helm_build_ops(p, k, yuk, nops, d_ops.get(), d_gx.get(), d_gw.get(), d_yb.get(), pl->d_hops.get(), s);
    FMMB_CUDA(cudaStreamSynchronize(s));
  }
  // pair jobs (rows are indices into the all-level M / L arrays)
  std::vector<int> par_i(pl->tot_i), par_j(pl->tot_j), key_i(pl->tot_i), key_j(pl->tot_j),
      lst((size_t)pl->tot_i * kM2LSlots);
  FMMB_CUDA(cudaMemcpy(par_i.data(), pl->parent_i.get(), pl->tot_i * sizeof(int), cudaMemcpyDeviceToHost));
  FMMB_CUDA(cudaMemcpy(par_j.data(), pl->parent_j.get(), pl->tot_j * sizeof(int), cudaMemcpyDeviceToHost));
  FMMB_CUDA(cudaMemcpy(key_i.data(), pl->key_i.get(), pl->tot_i * sizeof(int), cudaMemcpyDeviceToHost));
  FMMB_CUDA(cudaMemcpy(key_j.data(), pl->key_j.get(), pl->tot_j * sizeof(int), cudaMemcpyDeviceToHost));
  FMMB_CUDA(cudaMemcpy(lst.data(), pl->m2l_list.get(), lst.size() * sizeof(int), cudaMemcpyDeviceToHost));
  int nsm = 148;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, pl->device);
  pl->nsm = nsm;
  prepare_translate_pairs_f64();
  using P3 = std::array<int, 3>;
  pl->m2m_pairs.clear();
  pl->l2l_pairs.clear();
  for (int lev = 0; lev <= lmax; lev++) {
    std::vector<P3> up, down;
    if (lev >= 2 && lev < lmax)  // children at lev + 1 into their parents at lev
      for (int c = 0; c < pl->nbox_j[lev + 1]; c++) {
        const int box = pl->off_j[lev + 1] + c;
        up.push_back({pl->hop_m2m0 + (lev + 1 - 3) * 8 + (key_j[box] & 7), box, pl->off_j[lev] + par_j[box]});
      }
    if (lev >= 3)  // parents at lev - 1 into their children at lev
      for (int b = 0; b < pl->nbox_i[lev]; b++) {
        const int box = pl->off_i[lev] + b;
        down.push_back({pl->hop_l2l0 + (lev - 3) * 8 + (key_i[box] & 7), pl->off_i[lev - 1] + par_i[box], box});
      }
    pl->m2m_pairs.push_back(pair_job(up, 2 * K, nsm));
    pl->l2l_pairs.push_back(pair_job(down, 2 * K, nsm));
  }
  std::vector<P3> m2l;
  for (int lev = 2; lev <= lmax; lev++)
    for (int b = 0; b < pl->nbox_i[lev]; b++) {
      const int box = pl->off_i[lev] + b;
      for (int sl = 0; sl < kM2LSlots; sl++) {
        const int src = lst[(size_t)box * kM2LSlots + sl];
        if (src < 0) continue;
        const int slot = pl->ops.rel_to_op[pl->ops.slot_rel[(key_i[box] & 7) * kM2LSlots + sl]];
        m2l.push_back({pl->hop_m2l0 + (lev - 2) * 316 + slot, pl->off_j[lev] + src, box});
      }
    }
  pl->h_m2l = pair_job(m2l, 2 * K, nsm);
  // P2P work items: every target leaf in pieces of 256 targets
  {
    const int nleaf = pl->nbox_i[lmax];
    std::vector<int2> leaf(nleaf), work;
    FMMB_CUDA(cudaMemcpy(leaf.data(), pl->leaf_i.get(), nleaf * sizeof(int2), cudaMemcpyDeviceToHost));
    for (int b = 0; b < nleaf; b++)
      for (int t = 0; t < leaf[b].y; t += 256) work.push_back(make_int2(b, t));
    upload_vec(pl->h_p2p_work, work);
    pl->h_p2p_nwork = (int)work.size();
  }
  // inverse target permutation (caller -> sorted) for the direct sum
  {
    std::vector<int> perm(pl->ni), inv(pl->ni);
    FMMB_CUDA(cudaMemcpy(perm.data(), pl->perm_i.get(), pl->ni * sizeof(int), cudaMemcpyDeviceToHost));
    for (int i = 0; i < pl->ni; i++) inv[perm[i]] = i;
    upload_vec(pl->inv_i, inv);
  }
  const int nr = pl->cfg.nrhs;
  pl->qs.alloc((size_t)2 * pl->nj * nr);
  pl->M.alloc((size_t)pl->tot_j * 2 * K);
  pl->L.alloc((size_t)pl->tot_i * 2 * K);
  pl->pot_s.alloc((size_t)4 * pl->ni);  // near, far (complex)
  pl->use_tc = false;
  pl->use_h16 = false;
  FMMB_CUDA(cudaStreamSynchronize(s));
}

}  // namespace fmmb

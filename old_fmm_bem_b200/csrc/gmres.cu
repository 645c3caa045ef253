// Batched GMRES on the device for the BEM systems of a plan (fmmb_gmres).
//
// The reference solves one boundary-integral system per run with PETSc's
// KSP GMRES over a shell matrix whose matvec is one fmm() call
// (bio/main.cxx:27-53 mymatmult, :55-70 mypcshell, :377-413 KSPSolve):
//     A x = c x + K (w .* x),   preconditioner  y = d x,
// K the plan's kernel (Gni in the reference), w the panel weights (are/e1),
// c = (e1+e2)/(2 e1 (e1-e2)) and d = 1/c.  Here every (right-hand side,
// problem) pair of a plan -- nrhs x nprob independent systems -- runs GMRES
// in lockstep: one FMM evaluate per iteration serves all of them, and the
// Krylov work (Gram-Schmidt, norms, Givens rotations, the update of x) runs
// as device kernels over per-system segments.  Left preconditioning and a
// restart length as in PETSc's KSPGMRES; classical Gram-Schmidt with one
// reorthogonalisation pass (CGS2).  Dot products are deterministic: fixed
// chunks of each system's segment, block tree sums, then the chunk partials
// added in chunk order.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "internal.h"
#include "kernels.h"

namespace fmmb {
namespace {

constexpr int kChunk = 4096;   // elements of one system segment per block
constexpr int kThreads = 256;
constexpr int kMaxRestart = 64;

__device__ __forceinline__ double block_sum(double v, double* red) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) red[w] = v;
  __syncthreads();
  double t = 0;
  if (threadIdx.x == 0)
    for (int k = 0; k < (int)(blockDim.x >> 5); k++) t += red[k];
  return t;  // valid in thread 0
}

struct ChunkArgs {
  const int* sys;    // system of each chunk
  const int* start;  // first element (within the nrhs x n vector)
  const int* len;
};

// partial[c][i] = <V_i, w> over chunk c, i < nv (V_i = V + i*ld)
__global__ void __launch_bounds__(kThreads) k_dots(ChunkArgs ch, const double* __restrict__ V, size_t ld, int nv,
                                                   const double* __restrict__ w, double* __restrict__ partial,
                                                   int pstride) {
  __shared__ double red[32];
  const int c = blockIdx.x, st = ch.start[c], len = ch.len[c];
  for (int i = 0; i < nv; i++) {
    const double* v = V + (size_t)i * ld + st;
    double a = 0;
    for (int e = threadIdx.x; e < len; e += blockDim.x) a += v[e] * w[st + e];
    a = block_sum(a, red);
    if (threadIdx.x == 0) partial[(size_t)c * pstride + i] = a;
  }
}

// out[s][i] (+)= sum over the chunks of system s of partial[c][i]
__global__ void k_sum(int nsys, const int* __restrict__ sptr, const double* __restrict__ partial, int pstride, int nv,
                      double* __restrict__ out, int ostride) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nsys * nv) return;
  const int s = t / nv, i = t % nv;
  double a = 0;
  for (int c = sptr[s]; c < sptr[s + 1]; c++) a += partial[(size_t)c * pstride + i];
  out[(size_t)s * ostride + i] = a;
}

// w -= sum_i h[s][i] V_i   (or, with add = true, x += sum_i h[s][i] V_i over i < cnt[s])
__global__ void __launch_bounds__(kThreads) k_combine(ChunkArgs ch, const double* __restrict__ V, size_t ld, int nv,
                                                      const double* __restrict__ h, int hstride,
                                                      const int* __restrict__ cnt, double sign, double* __restrict__ w) {
  __shared__ double hs[kMaxRestart + 1];
  const int c = blockIdx.x, s = ch.sys[c], st = ch.start[c], len = ch.len[c];
  const int n = cnt ? min(nv, cnt[s]) : nv;
  for (int i = threadIdx.x; i < n; i += blockDim.x) hs[i] = h[(size_t)s * hstride + i];
  __syncthreads();
  for (int e = threadIdx.x; e < len; e += blockDim.x) {
    double a = w[st + e];
    for (int i = 0; i < n; i++) a += sign * hs[i] * V[(size_t)i * ld + st + e];
    w[st + e] = a;
  }
}

// q = (float)(weight .* v) for active systems, 0 otherwise
__global__ void __launch_bounds__(kThreads) k_charges(ChunkArgs ch, int n, const double* __restrict__ v,
                                                      const float* __restrict__ weight, const int* __restrict__ active,
                                                      float* __restrict__ q) {
  const int c = blockIdx.x, s = ch.sys[c], st = ch.start[c], len = ch.len[c];
  const bool on = active == nullptr || active[s];
  for (int e = threadIdx.x; e < len; e += blockDim.x) {
    const int g = st + e;
    const double wt = weight ? (double)weight[g % n] : 1.0;
    q[g] = on ? (float)(wt * v[g]) : 0.f;
  }
}

// out = d (pot + c v)                  (mode 0: the preconditioned A v)
// out = d (b - (pot + c v))            (mode 1: the preconditioned residual)
__global__ void __launch_bounds__(kThreads) k_apply(ChunkArgs ch, const double* __restrict__ pot,
                                                    const double* __restrict__ v, const double* __restrict__ b,
                                                    double c, double d, int mode, double* __restrict__ out) {
  const int blk = blockIdx.x, st = ch.start[blk], len = ch.len[blk];
  for (int e = threadIdx.x; e < len; e += blockDim.x) {
    const int g = st + e;
    const double av = pot[g] + c * v[g];
    out[g] = mode ? d * (b[g] - av) : d * av;
  }
}

// v = w * inv[s]
__global__ void __launch_bounds__(kThreads) k_scale_into(ChunkArgs ch, const double* __restrict__ w,
                                                         const double* __restrict__ inv, double* __restrict__ v) {
  const int c = blockIdx.x, st = ch.start[c], len = ch.len[c];
  const double f = inv[ch.sys[c]];
  for (int e = threadIdx.x; e < len; e += blockDim.x) v[st + e] = w[st + e] * f;
}

struct State {
  double *H, *cs, *sn, *g, *beta0, *inv, *resid, *y;
  int *active, *kact;
  int m;
};

// start of a cycle: beta = ||r||, g = (beta, 0, ...); first cycle fixes beta0
__global__ void k_start(int nsys, State S, const double* __restrict__ nrm2, int first, double rtol) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nsys) return;
  const int m = S.m;
  const double beta = sqrt(fmax(nrm2[s], 0.0));
  if (first) {
    S.beta0[s] = beta;
    S.active[s] = beta > 0.0;
  }
  if (beta <= rtol * S.beta0[s]) S.active[s] = 0;
  for (int k = 0; k <= m; k++) S.g[(size_t)s * (m + 1) + k] = 0.0;
  S.g[(size_t)s * (m + 1)] = S.active[s] ? beta : 0.0;
  S.kact[s] = 0;
  S.resid[s] = beta;
  S.inv[s] = S.active[s] ? 1.0 / beta : 0.0;
}

// column j of the Hessenberg matrix (h1 + h2 from the two Gram-Schmidt
// passes, ||w|| below), the previous rotations applied, a new rotation, the
// residual estimate |g[j+1]|; breakdown or convergence freezes the system
__global__ void k_givens(int nsys, int j, State S, const double* __restrict__ h1, const double* __restrict__ h2,
                         const double* __restrict__ nrm2, double rtol) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nsys) return;
  const int m = S.m;
  if (!S.active[s]) {
    S.inv[s] = 0.0;
    return;
  }
  double* col = S.H + (size_t)s * (m + 1) * m + (size_t)j * (m + 1);
  double* cs = S.cs + (size_t)s * m;
  double* sn = S.sn + (size_t)s * m;
  double* g = S.g + (size_t)s * (m + 1);
  double cn = 0;
  for (int i = 0; i <= j; i++) {
    col[i] = h1[(size_t)s * (m + 1) + i] + h2[(size_t)s * (m + 1) + i];
    cn += col[i] * col[i];
  }
  const double hn = sqrt(fmax(nrm2[s], 0.0));
  col[j + 1] = hn;
  for (int i = 0; i < j; i++) {
    const double t = cs[i] * col[i] + sn[i] * col[i + 1];
    col[i + 1] = -sn[i] * col[i] + cs[i] * col[i + 1];
    col[i] = t;
  }
  const double a = col[j], b = col[j + 1];
  const double r = hypot(a, b);
  const double c = r > 0 ? a / r : 1.0, sv = r > 0 ? b / r : 0.0;
  cs[j] = c;
  sn[j] = sv;
  col[j] = r;
  col[j + 1] = 0.0;
  const double gj = g[j];
  g[j] = c * gj;
  g[j + 1] = -sv * gj;
  S.kact[s] = j + 1;
  S.resid[s] = fabs(g[j + 1]);
  const bool breakdown = !(hn > 1e-14 * sqrt(cn + hn * hn));
  if (breakdown || S.resid[s] <= rtol * S.beta0[s]) {
    S.active[s] = 0;
    S.inv[s] = 0.0;
  } else {
    S.inv[s] = 1.0 / hn;
  }
}

// y = R^{-1} g over the kact columns of the cycle (back substitution)
__global__ void k_trisolve(int nsys, State S) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nsys) return;
  const int m = S.m, k = S.kact[s];
  const double* H = S.H + (size_t)s * (m + 1) * m;
  const double* g = S.g + (size_t)s * (m + 1);
  double* y = S.y + (size_t)s * (m + 1);
  for (int i = k - 1; i >= 0; i--) {
    double a = g[i];
    for (int l = i + 1; l < k; l++) a -= H[(size_t)l * (m + 1) + i] * y[l];
    const double d = H[(size_t)i * (m + 1) + i];
    y[i] = d != 0.0 ? a / d : 0.0;
  }
}

__global__ void k_count_active(int nsys, const int* __restrict__ active, int* __restrict__ out) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s < nsys && active[s]) atomicAdd(out, 1);
}

unsigned nblk(long long n, int t) { return (unsigned)((n + t - 1) / t); }

bool is_dev(const void* p) {
  if (!p) return false;
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

}  // namespace
}  // namespace fmmb

using namespace fmmb;

extern "C" {

int fmmb_gmres_config_init(fmmb_gmres_config* c) {
  if (!c) return FMMB_ERR_ARG;
  std::memset(c, 0, sizeof(*c));
  c->restart = 30;
  c->max_iter = 20;
  c->rtol = 0.0;
  c->diag = 0.0;
  c->precond = 1.0;
  return FMMB_OK;
}

int fmmb_gmres(fmmb_plan* pl, const fmmb_gmres_config* cfg, const float* weight, const double* b, double* x,
               int* iters_out, double* resid_out) {
  try {
    FMMB_REQUIRE(pl && cfg && b && x, FMMB_ERR_ARG, "null argument");
    FMMB_REQUIRE(pl->have_geometry, FMMB_ERR_STATE, "fmmb_set_geometry must come first");
    FMMB_REQUIRE(cfg->restart >= 1 && cfg->restart <= kMaxRestart, FMMB_ERR_ARG, "restart must be in 1..64");
    FMMB_REQUIRE(cfg->max_iter >= 0, FMMB_ERR_ARG, "max_iter must be >= 0");
    FMMB_REQUIRE(cfg->rtol >= 0 && std::isfinite(cfg->diag) && std::isfinite(cfg->precond), FMMB_ERR_ARG,
                 "rtol must be >= 0, diag and precond finite");
    FMMB_REQUIRE(!helm_family(pl->cfg.kernel), FMMB_ERR_ARG, "GMRES takes the Laplace kernels");
    FMMB_REQUIRE(pl->ni == pl->nj && pl->prob_toff == pl->prob_soff, FMMB_ERR_ARG,
                 "GMRES needs a square system: the targets are the sources, problem by problem");
    const int n = pl->ni, nrhs = pl->cfg.nrhs, nprob = pl->nprob, m = cfg->restart;
    const int nsys = nrhs * nprob;
    const size_t L = (size_t)n * nrhs;
    cudaStream_t st = pl->st.main;

    // chunks of every system's segment: system s = r * nprob + p covers
    // [r n + toff[p], r n + toff[p+1])
    std::vector<int> csys, cstart, clen, sptr(nsys + 1, 0);
    for (int r = 0; r < nrhs; r++)
      for (int p = 0; p < nprob; p++) {
        const int s = r * nprob + p;
        sptr[s] = (int)csys.size();
        for (int e = pl->prob_toff[p]; e < pl->prob_toff[p + 1]; e += kChunk) {
          csys.push_back(s);
          cstart.push_back(r * n + e);
          clen.push_back(std::min(kChunk, pl->prob_toff[p + 1] - e));
        }
      }
    sptr[nsys] = (int)csys.size();
    const int nch = (int)csys.size();
    DevBuf<int>& d_ci = pl->gm_ci;  // workspaces kept by the plan (grown, never shrunk)
    d_ci.alloc(3 * (size_t)nch + nsys + 1 + 1);
    FMMB_CUDA(cudaMemcpyAsync(d_ci.get(), csys.data(), nch * sizeof(int), cudaMemcpyHostToDevice, st));
    FMMB_CUDA(cudaMemcpyAsync(d_ci.get() + nch, cstart.data(), nch * sizeof(int), cudaMemcpyHostToDevice, st));
    FMMB_CUDA(cudaMemcpyAsync(d_ci.get() + 2 * nch, clen.data(), nch * sizeof(int), cudaMemcpyHostToDevice, st));
    FMMB_CUDA(cudaMemcpyAsync(d_ci.get() + 3 * nch, sptr.data(), (nsys + 1) * sizeof(int), cudaMemcpyHostToDevice, st));
    const ChunkArgs ch{d_ci.get(), d_ci.get() + nch, d_ci.get() + 2 * nch};
    const int* d_sptr = d_ci.get() + 3 * nch;
    int* d_count = d_ci.get() + 3 * nch + nsys + 1;

    // vectors: V[0..m], w, b, x, pot (FP64), q (FP32)
    DevBuf<double>& vec = pl->gm_vec;
    vec.alloc((size_t)(m + 5) * L);
    double* V = vec.get();
    double* W = V + (size_t)(m + 1) * L;
    double* B = W + L;
    double* X = B + L;
    double* POT = X + L;
    DevBuf<float>& qbuf = pl->gm_q;
    DevBuf<float>& wbuf = pl->gm_w;
    qbuf.alloc(L);
    const float* wt = nullptr;
    if (weight) {
      if (is_dev(weight)) {
        wt = weight;
      } else {
        wbuf.alloc(n);
        FMMB_CUDA(cudaMemcpyAsync(wbuf.get(), weight, n * sizeof(float), cudaMemcpyHostToDevice, st));
        wt = wbuf.get();
      }
    }
    FMMB_CUDA(cudaMemcpyAsync(B, b, L * sizeof(double), cudaMemcpyDefault, st));
    FMMB_CUDA(cudaMemcpyAsync(X, x, L * sizeof(double), cudaMemcpyDefault, st));

    // per-system state
    const int pst = m + 1;
    DevBuf<double>& sd = pl->gm_sd;
    // H [(m+1) m], cs, sn [m], g, y, h1, h2 [m+1], beta0, inv, resid, nrm2 per
    // system, then the chunk partials
    sd.alloc((size_t)nsys * ((m + 1) * m + 2 * m + 4 * (m + 1) + 4) + (size_t)nch * pst);
    State S;
    S.m = m;
    S.H = sd.get();
    S.cs = S.H + (size_t)nsys * (m + 1) * m;
    S.sn = S.cs + (size_t)nsys * m;
    S.g = S.sn + (size_t)nsys * m;
    S.y = S.g + (size_t)nsys * (m + 1);
    double* h1 = S.y + (size_t)nsys * (m + 1);
    double* h2 = h1 + (size_t)nsys * (m + 1);
    S.beta0 = h2 + (size_t)nsys * (m + 1);
    S.inv = S.beta0 + nsys;
    S.resid = S.inv + nsys;
    double* nrm2 = S.resid + nsys;
    double* partial = nrm2 + nsys;
    DevBuf<int>& si = pl->gm_si;
    si.alloc(2 * (size_t)nsys);
    S.active = si.get();
    S.kact = si.get() + nsys;
    FMMB_CUDA(cudaMemsetAsync(S.H, 0, (size_t)nsys * (m + 1) * m * sizeof(double), st));

    const double c = cfg->diag, d = cfg->precond;
    auto check = [&](int rc) {
      if (rc != FMMB_OK) throw Error{rc, std::string(fmmb_last_error())};
    };
    // w = d (K (weight .* v) + c v)  (mode 0)  or  w = d (b - A v)  (mode 1)
    auto matvec = [&](const double* v, const int* act, int mode, double* out) {
      k_charges<<<nch, kThreads, 0, st>>>(ch, n, v, wt, act, qbuf.get());
      FMMB_CHECK_LAUNCH();
      check(fmmb_evaluate_f64(pl, qbuf.get(), POT, nullptr));
      k_apply<<<nch, kThreads, 0, st>>>(ch, POT, v, B, c, d, mode, out);
      FMMB_CHECK_LAUNCH();
    };
    auto dots = [&](const double* Vb, int nv, const double* w, double* out, int ostride) {
      k_dots<<<nch, kThreads, 0, st>>>(ch, Vb, L, nv, w, partial, pst);
      FMMB_CHECK_LAUNCH();
      k_sum<<<nblk((long long)nsys * nv, 128), 128, 0, st>>>(nsys, d_sptr, partial, pst, nv, out, ostride);
      FMMB_CHECK_LAUNCH();
    };
    auto any_active = [&]() {
      FMMB_CUDA(cudaMemsetAsync(d_count, 0, sizeof(int), st));
      k_count_active<<<nblk(nsys, 128), 128, 0, st>>>(nsys, S.active, d_count);
      FMMB_CHECK_LAUNCH();
      int h = 0;
      FMMB_CUDA(cudaMemcpyAsync(&h, d_count, sizeof(int), cudaMemcpyDeviceToHost, st));
      FMMB_CUDA(cudaStreamSynchronize(st));
      return h > 0;
    };

    int it = 0;
    bool first = true;
    while (true) {
      // V_0 = d (b - A x), beta = ||V_0||, g = (beta, 0, ...), V_0 /= beta
      matvec(X, nullptr, 1, V);
      dots(V, 1, V, nrm2, 1);
      k_start<<<nblk(nsys, 128), 128, 0, st>>>(nsys, S, nrm2, first ? 1 : 0, cfg->rtol);
      FMMB_CHECK_LAUNCH();
      k_scale_into<<<nch, kThreads, 0, st>>>(ch, V, S.inv, V);
      FMMB_CHECK_LAUNCH();
      first = false;
      bool stop = cfg->rtol > 0 && !any_active();
      for (int j = 0; !stop && j < m && it < cfg->max_iter; j++) {
        matvec(V + (size_t)j * L, S.active, 0, W);
        // CGS2: two passes of h = V^T w, w -= V h
        dots(V, j + 1, W, h1, m + 1);
        k_combine<<<nch, kThreads, 0, st>>>(ch, V, L, j + 1, h1, m + 1, nullptr, -1.0, W);
        FMMB_CHECK_LAUNCH();
        dots(V, j + 1, W, h2, m + 1);
        k_combine<<<nch, kThreads, 0, st>>>(ch, V, L, j + 1, h2, m + 1, nullptr, -1.0, W);
        FMMB_CHECK_LAUNCH();
        dots(W, 1, W, nrm2, 1);
        k_givens<<<nblk(nsys, 128), 128, 0, st>>>(nsys, j, S, h1, h2, nrm2, cfg->rtol);
        FMMB_CHECK_LAUNCH();
        k_scale_into<<<nch, kThreads, 0, st>>>(ch, W, S.inv, V + (size_t)(j + 1) * L);
        FMMB_CHECK_LAUNCH();
        it++;
        if (cfg->rtol > 0 && !any_active()) stop = true;
      }
      // x += V y, y = R^{-1} g over each system's columns of this cycle
      k_trisolve<<<nblk(nsys, 128), 128, 0, st>>>(nsys, S);
      FMMB_CHECK_LAUNCH();
      k_combine<<<nch, kThreads, 0, st>>>(ch, V, L, m, S.y, m + 1, S.kact, 1.0, X);
      FMMB_CHECK_LAUNCH();
      if (stop || it >= cfg->max_iter) break;
    }
    if (resid_out) {
      // the residual of the returned iterate itself, ||d (b - A x)||, by one
      // more matvec (the Givens estimate |g| keeps falling below what the
      // matvec's own rounding lets A x reach, in the mixed form by orders)
      matvec(X, nullptr, 1, V);
      dots(V, 1, V, nrm2, 1);
      std::vector<double> r(nsys), b0(nsys);
      FMMB_CUDA(cudaMemcpyAsync(r.data(), nrm2, nsys * sizeof(double), cudaMemcpyDeviceToHost, st));
      FMMB_CUDA(cudaMemcpyAsync(b0.data(), S.beta0, nsys * sizeof(double), cudaMemcpyDeviceToHost, st));
      FMMB_CUDA(cudaStreamSynchronize(st));
      for (int k = 0; k < nsys; k++) r[k] = b0[k] > 0 ? std::sqrt(std::max(r[k], 0.0)) / b0[k] : 0.0;
      if (is_dev(resid_out)) FMMB_CUDA(cudaMemcpy(resid_out, r.data(), nsys * sizeof(double), cudaMemcpyHostToDevice));
      else std::memcpy(resid_out, r.data(), nsys * sizeof(double));
    }
    FMMB_CUDA(cudaMemcpyAsync(x, X, L * sizeof(double), cudaMemcpyDefault, st));
    FMMB_CUDA(cudaStreamSynchronize(st));
    if (iters_out) *iters_out = it;
    return FMMB_OK;
  } catch (const Error& e) {
    set_error(e.msg);
    return e.code;
  }
}

}  // extern "C"

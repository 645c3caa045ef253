// Near-field P2P in FP32 with compensated per-target accumulation.
//
// Same sums as the reference's P2P kernels (kernel/G_p2p.cxx:12-37,
// kernel/Gni_p2p.cxx:12-28, kernel/Gnj_p2p.cxx:12-28) over the 27-slot
// neighbour lists of the GPU tree.  Pair arithmetic is FP32 (hardware rsqrt);
// each lane sums up to 128 sources at a time in FP32 (two lanes of 64, added
// before the conversion) and promotes every partial sum into FP64
// accumulators, so the accumulated rounding stays at the FP32 level of one
// 128-term sum whatever the number of sources.
//
// Layout: one block of 4 warps per work item, up to 128 targets of one
// target leaf (a leaf of more targets is several items, so that the dense
// leaves of clustered points spread over many SMs; the items come heaviest
// first).  The sources of all
// neighbour leaves are staged into shared memory as one list -- the leaf's
// own source leaf first, padded to a multiple of 32 with far, zero-charge
// points, then the other neighbours, padded likewise -- so that no run of 32
// sources needs a bounds check, and only the own leaf's runs test for
// coincident points (points at zero distance share a leaf).  Warp 0 builds
// the segment list with one lane per neighbour slot (ballot + scan), and the
// staging issues four sources' loads per thread before storing any.
//
// A warp is 8 target lanes x 4 source streams: lane (g, s) = (lane % 8,
// lane / 8) holds target g of each of its NT groups of 8 targets and takes
// source pairs s, s + 4, s + 8, s + 12 of a run of 32 sources, so one
// shared-memory read (four consecutive pairs per warp, one bank wavefront)
// serves 2 NT pairs and a leaf occupies its lanes in steps of 8 targets
// rather than 32 (leaves of a surface hold tens of points).  The pair
// arithmetic uses the two-lane FP32 instructions (add / mul / fma .f32x2) on
// the two sources of a pair: half the FP32 instructions of the scalar form,
// the same values.  The warps form teams that share a tile of up
// to 4 groups and split its runs: 1 team of 4 warps for leaves of up to 4
// groups, 2 teams of 2 for up to 8, else 4 one-warp teams (with more rounds of
// tiles for big leaves).  The 4 streams' FP64 sums of a target are added by
// two shuffles, the warps of a team through shared memory.
#include <cuda_runtime.h>

#include <climits>

#include "internal.h"
#include "kernels.h"

namespace fmmb {
namespace {

constexpr int kThreads = 128;
constexpr int kWarps = kThreads / 32;
constexpr int kG = 8;          // targets of a group (lanes g = lane % 8)
constexpr int kS = 32 / kG;    // source streams of a warp (s = lane / 8)
constexpr int kMaxNT = 4;      // groups of a tile
constexpr int kCap = 1024;     // staged sources per chunk (multiple of 32 * 4)
constexpr int kSelfSlot = 13;  // offset (0, 0, 0) in the 27-slot list
constexpr float kFar = 1e18f;  // padding sources: r^2 ~ 3e36 stays finite in FP32

__device__ __forceinline__ int pad32(int n) { return (n + 31) & ~31; }

// 1/sqrt(x) from the hardware approximation, subnormal inputs flushed to zero
// (r^2 is either 0 -- coincident points, handled by the caller -- or far
// above the subnormal range for any pair of distinct float positions in
// neighbouring leaves), so no subnormal fix-up instructions are emitted.
__device__ __forceinline__ float rsqrt_ftz(float x) {
  float y;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

template <int KER>
struct Acc {
  float p, fx, fy, fz;
};

// Kernel selector of the templates: a Laplace kernel, plus kWithGrad for the
// normal-derivative kernels with the gradient of the potential w.r.t. the
// target position (normals held fixed) as well.
constexpr int kWithGrad = 16;
constexpr int base(int KER) { return KER & (kWithGrad - 1); }
constexpr bool with_grad(int KER) { return KER == FMMB_LAPLACE_G || (KER & kWithGrad) != 0; }

template <int KER>
constexpr int ncomp() {
  return with_grad(KER) ? 4 : 1;  // accumulated components: potential (and gradient)
}

// Negated positions of sources j, j + 1 (even j) of the staged list, packed
// for the two-lane FP32 instructions: (-x_j, -x_j+1, -y_j, -y_j+1) and
// (-z_j, -z_j+1, q_j, q_j+1) (G, Gni; for Gnj the charge slots hold
// q_j n_z, q_j+1 n_z and M the x, y components of q n): one 16-byte read per
// quantity pair.  Pair values
// are bit-identical to the scalar forms (x_i + (-x_j) = x_i - x_j, the same
// operation order after it); each lane keeps two FP32 partial sums, over the
// even and the odd sources.
template <int KER>
struct Smem {
  static constexpr int NC = ncomp<KER>();
  static constexpr int NP = kCap / 2;
  float4 A[NP];
  float4 BQ[NP];                                      // (-z j, j+1, q j, j+1) or (-z j, j+1, qn_z j, j+1)
  float4 M[base(KER) == FMMB_LAPLACE_GNJ ? NP : 1];   // (qn_x j, j+1, qn_y j, j+1)
  double red[kWarps][kMaxNT][NC][kG];           // team partial sums
  int2 seg[32];                                 // (first source, count), own leaf first
  int vst[32];                                  // virtual start of each segment, then INT_MAX
};

struct Tgt {
  float2 x, y, z;     // the target's coordinates, duplicated in both lanes
  float2 nx, ny, nz;  // Gni: its normal, duplicated
};

__device__ __forceinline__ float2 dup(float v) { return make_float2(v, v); }

// The lane's 4 source pairs of one run of 32 (pairs pb, pb + 4, pb + 8,
// pb + 12 of the chunk) against its NT targets.
template <int KER, bool EXCL, int NT>
__device__ __forceinline__ void run16(const Smem<KER>& S, int pb, const Tgt (&tg)[kMaxNT], float2 e2,
                                      float2 (&acc)[NT][ncomp<KER>()]) {
#pragma unroll (EXCL ? 1 : 4)
  for (int u = 0; u < 4; u++) {
    const int pi = pb + 4 * u;
    const float4 a = S.A[pi], bq = S.BQ[pi];
    const float2 sx = make_float2(a.x, a.y), sy = make_float2(a.z, a.w), sz = make_float2(bq.x, bq.y);
    float2 q2 = make_float2(0.f, 0.f), mx = q2, my = q2, mz = q2;
    if (base(KER) == FMMB_LAPLACE_GNJ) {
      const float4 m = S.M[pi];
      mx = make_float2(m.x, m.y);
      my = make_float2(m.z, m.w);
      mz = make_float2(bq.z, bq.w);
    } else {
      q2 = make_float2(bq.z, bq.w);
    }
#pragma unroll
    for (int t = 0; t < NT; t++) {
      const float2 dx = __fadd2_rn(tg[t].x, sx), dy = __fadd2_rn(tg[t].y, sy), dz = __fadd2_rn(tg[t].z, sz);
      const float2 r2 = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __ffma2_rn(dz, dz, e2)));
      float2 ri = make_float2(rsqrt_ftz(r2.x), rsqrt_ftz(r2.y));
      if (EXCL) {
        ri.x = r2.x > 0.f ? ri.x : 0.f;
        ri.y = r2.y > 0.f ? ri.y : 0.f;
      }
      if (KER == FMMB_LAPLACE_G) {
        const float2 qr = __fmul2_rn(q2, ri);
        const float2 qr3 = __fmul2_rn(__fmul2_rn(qr, ri), ri);
        acc[t][0] = __fadd2_rn(acc[t][0], qr);
        acc[t][1] = __ffma2_rn(dx, qr3, acc[t][1]);
        acc[t][2] = __ffma2_rn(dy, qr3, acc[t][2]);
        acc[t][3] = __ffma2_rn(dz, qr3, acc[t][3]);
      } else if (base(KER) == FMMB_LAPLACE_GNI) {
        const float2 qr3 = __fmul2_rn(__fmul2_rn(__fmul2_rn(q2, ri), ri), ri);
        const float2 dot = __ffma2_rn(dx, tg[t].nx, __ffma2_rn(dy, tg[t].ny, __fmul2_rn(dz, tg[t].nz)));
        acc[t][0] = __ffma2_rn(dot, qr3, acc[t][0]);
        if (with_grad(KER)) {  // d/dx_i of (d.n_i) q / r^3 = q n_i / r^3 - 3 (d.n_i) q d / r^5
          const float2 c = __fmul2_rn(__fmul2_rn(dot, qr3), __fmul2_rn(__fmul2_rn(ri, ri), dup(-3.f)));
          acc[t][1] = __ffma2_rn(qr3, tg[t].nx, __ffma2_rn(c, dx, acc[t][1]));
          acc[t][2] = __ffma2_rn(qr3, tg[t].ny, __ffma2_rn(c, dy, acc[t][2]));
          acc[t][3] = __ffma2_rn(qr3, tg[t].nz, __ffma2_rn(c, dz, acc[t][3]));
        }
      } else {
        const float2 r3 = __fmul2_rn(__fmul2_rn(ri, ri), ri);
        const float2 dot = __ffma2_rn(dx, mx, __ffma2_rn(dy, my, __fmul2_rn(dz, mz)));
        acc[t][0] = __ffma2_rn(dot, r3, acc[t][0]);
        if (with_grad(KER)) {  // d/dx_i of (d.m) / r^3 = m / r^3 - 3 (d.m) d / r^5, m = q n_j
          const float2 c = __fmul2_rn(__fmul2_rn(dot, r3), __fmul2_rn(__fmul2_rn(ri, ri), dup(-3.f)));
          acc[t][1] = __ffma2_rn(mx, r3, __ffma2_rn(c, dx, acc[t][1]));
          acc[t][2] = __ffma2_rn(my, r3, __ffma2_rn(c, dy, acc[t][2]));
          acc[t][3] = __ffma2_rn(mz, r3, __ffma2_rn(c, dz, acc[t][3]));
        }
      }
    }
  }
}

// Stages virtual sources [c0, c1) of the list [own | pad | others | pad] as
// packed pairs: each thread locates four sources (two pairs; binary search
// over the segment starts), issues their loads, then stores them.
template <int KER>
__device__ __forceinline__ int locate(const Smem<KER>& S, int v, int c1) {
  int sgi = 0;
#pragma unroll
  for (int st = 16; st > 0; st >>= 1)
    if (S.vst[sgi + st] <= v) sgi += st;
  const int2 sg = S.seg[sgi];
  const int off = v - S.vst[sgi];
  return (v < c1 && off < sg.y) ? sg.x + off : -1;
}

template <int KER>
__device__ void stage(Smem<KER>& S, int c0, int c1, const float4* __restrict__ spos,
                      const float4* __restrict__ snrm, const float* __restrict__ qs) {
  __syncthreads();  // the previous chunk's readers are done
  const int np = (c1 - c0) >> 1;
  for (int pb = threadIdx.x; pb < np; pb += 2 * kThreads) {
    int jj[4];
#pragma unroll
    for (int u = 0; u < 4; u++) jj[u] = locate(S, c0 + 2 * (pb + (u >> 1) * kThreads) + (u & 1), c1);
    float4 x[4], n[4];
    float q[4];
#pragma unroll
    for (int u = 0; u < 4; u++) {
      x[u] = make_float4(kFar, kFar, kFar, 0.f);
      n[u] = make_float4(0.f, 0.f, 0.f, 0.f);
      q[u] = 0.f;
      if (jj[u] >= 0) {
        x[u] = spos[jj[u]];
        q[u] = qs[jj[u]];
        if (base(KER) == FMMB_LAPLACE_GNJ) n[u] = snrm[jj[u]];
      }
    }
#pragma unroll
    for (int h = 0; h < 2; h++) {
      const int pi = pb + h * kThreads;
      if (pi < np) {
        const float4 x0 = x[2 * h], x1 = x[2 * h + 1];
        const float q0 = q[2 * h], q1 = q[2 * h + 1];
        S.A[pi] = make_float4(-x0.x, -x1.x, -x0.y, -x1.y);
        if (base(KER) == FMMB_LAPLACE_GNJ) {
          const float4 n0 = n[2 * h], n1 = n[2 * h + 1];
          S.M[pi] = make_float4(q0 * n0.x, q1 * n1.x, q0 * n0.y, q1 * n1.y);
          S.BQ[pi] = make_float4(-x0.z, -x1.z, q0 * n0.z, q1 * n1.z);
        } else {
          S.BQ[pi] = make_float4(-x0.z, -x1.z, q0, q1);
        }
      }
    }
  }
  __syncthreads();
}

// The team tile's runs of the chunk [c0, c1): runs k, k + m, ... (global run
// index), the own leaf's runs (below self_end) with the coincident-point test.
template <int KER, bool EXCL, int NT>
__device__ __forceinline__ void tile_runs(const Smem<KER>& S, int c0, int c1, int self_end, int s, int k, int m,
                                          const Tgt (&tg)[kMaxNT], float eps2, double (&P)[kMaxNT][ncomp<KER>()]) {
  constexpr int NC = ncomp<KER>();
  const float2 e2 = dup(eps2);
  const int rend = c1 >> 5;
  int r = (c0 >> 5) + k;  // c0 / 32 is a multiple of m
  while (r < rend) {
    float2 acc[NT][NC];
#pragma unroll
    for (int t = 0; t < NT; t++)
#pragma unroll
      for (int c = 0; c < NC; c++) acc[t][c] = make_float2(0.f, 0.f);
    for (int i = 0; i < 16 && r < rend; i++, r += m) {  // 16 runs: 64 sources in each lane's two sums
      const int pb = ((r * 32 - c0) >> 1) + s;
      if (EXCL && r * 32 < self_end)
        run16<KER, true, NT>(S, pb, tg, e2, acc);
      else
        run16<KER, false, NT>(S, pb, tg, e2, acc);
    }
#pragma unroll
    for (int t = 0; t < NT; t++)
#pragma unroll
      for (int c = 0; c < NC; c++) {
        P[t][c] += (double)(acc[t][c].x + acc[t][c].y);
      }
  }
}

template <int KER, bool EXCL>
__global__ void __launch_bounds__(kThreads) p2p_mixed(const int2* __restrict__ work, const int2* __restrict__ leaf_i,
                                                      const int2* __restrict__ leaf_j,
                                                      const int* __restrict__ list, const float4* __restrict__ tpos,
                                                      const float4* __restrict__ tnrm, const float4* __restrict__ spos,
                                                      const float4* __restrict__ snrm, const float* __restrict__ qs,
                                                      float eps2, double coef, double* __restrict__ pot,
                                                      double* __restrict__ grad, int ni) {
  constexpr int NC = ncomp<KER>();
  __shared__ Smem<KER> S;
  const int2 wk = work[blockIdx.x];
  const int b = wk.x;  // target leaf; this item's targets: [li.x, li.x + li.y)
  int2 li = leaf_i[b];
  li.x += wk.y;
  li.y = min(kThreads, li.y - wk.y);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane & (kG - 1), s = lane / kG;
  // segment list: lane l of warp 0 reads neighbour slot l; the own leaf goes
  // first, the non-empty others after it in slot order
  if (warp == 0) {
    int2 sg = make_int2(0, 0);
    if (lane < kP2PSlots) {
      const int jl = list[(size_t)b * kP2PSlots + lane];
      if (jl >= 0) sg = leaf_j[jl];
    }
    const int self_end = pad32(__shfl_sync(0xffffffffu, sg.y, kSelfSlot));
    const bool oth = lane != kSelfSlot && sg.y > 0;
    const unsigned mask = __ballot_sync(0xffffffffu, oth);
    const int pos = 1 + __popc(mask & ((1u << lane) - 1u));
    const int cnt = oth ? sg.y : 0;
    int incl = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += t;
    }
    const int nseg = 1 + __popc(mask);
    if (lane == kSelfSlot) {
      S.seg[0] = sg;
      S.vst[0] = 0;
    }
    if (oth) {
      S.seg[pos] = sg;
      S.vst[pos] = self_end + incl - cnt;
    }
    if (lane >= nseg) S.vst[lane] = INT_MAX;
    const int n_other = __shfl_sync(0xffffffffu, incl, 31);
    if (lane == 0) S.seg[31] = make_int2(0, n_other);  // slot 31 is never a segment: it holds n_other
  }
  __syncthreads();
  const int own = S.seg[0].y;
  const int self_end = pad32(own);
  const int n_other = S.seg[31].y;
  const int vlen = self_end + pad32(n_other);
  const int nchunk = (vlen + kCap - 1) / kCap;
  // teams of m warps share a tile and split its runs
  const int ng = (li.y + kG - 1) / kG;
  const int m = ng <= kMaxNT ? 4 : ng <= 2 * kMaxNT ? 2 : 1;  // block-uniform
  const int nteam = kWarps / m, team = warp / m, k = warp % m;
  const int g0 = team * ng / nteam, g1 = (team + 1) * ng / nteam;
  const int rounds = ((ng + nteam - 1) / nteam + kMaxNT - 1) / kMaxNT;
  const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
  for (int tr = 0; tr < rounds; tr++) {
    const int ga = g0 + tr * kMaxNT;
    const int ntl = max(0, min(kMaxNT, g1 - ga));  // warp-uniform
    Tgt tg[kMaxNT];
    double P[kMaxNT][NC];
#pragma unroll
    for (int t = 0; t < kMaxNT; t++) {
      const int it = (ga + t) * kG + g;
      const bool on = t < ntl && it < li.y;
      const float4 x = on ? tpos[li.x + it] : z4;
      const float4 n = (base(KER) == FMMB_LAPLACE_GNI && on) ? tnrm[li.x + it] : z4;
      tg[t] = Tgt{dup(x.x), dup(x.y), dup(x.z), dup(n.x), dup(n.y), dup(n.z)};
#pragma unroll
      for (int c = 0; c < NC; c++) P[t][c] = 0.0;
    }
    for (int ch = 0; ch < nchunk; ch++) {
      const int c0 = ch * kCap, c1 = min(vlen, c0 + kCap);
      if (nchunk > 1 || tr == 0) stage<KER>(S, c0, c1, spos, snrm, qs);
      switch (ntl) {
        case 0: break;
        case 1: tile_runs<KER, EXCL, 1>(S, c0, c1, self_end, s, k, m, tg, eps2, P); break;
        case 2: tile_runs<KER, EXCL, 2>(S, c0, c1, self_end, s, k, m, tg, eps2, P); break;
        case 3: tile_runs<KER, EXCL, 3>(S, c0, c1, self_end, s, k, m, tg, eps2, P); break;
        default: tile_runs<KER, EXCL, 4>(S, c0, c1, self_end, s, k, m, tg, eps2, P); break;
      }
    }
    // add the 4 streams' sums of each target (lanes g, g + 8, g + 16, g + 24)
#pragma unroll
    for (int t = 0; t < kMaxNT; t++)
#pragma unroll
      for (int c = 0; c < NC; c++) {
        P[t][c] += __shfl_xor_sync(0xffffffffu, P[t][c], 8);
        P[t][c] += __shfl_xor_sync(0xffffffffu, P[t][c], 16);
      }
    if (m > 1) {  // block-uniform (rounds == 1): the team's warps through shared memory
      if (s == 0 && k > 0) {
#pragma unroll
        for (int t = 0; t < kMaxNT; t++)
#pragma unroll
          for (int c = 0; c < NC; c++) S.red[warp][t][c][g] = P[t][c];
      }
      __syncthreads();
      if (k == 0 && s == 0) {
        for (int w = 1; w < m; w++)
#pragma unroll
          for (int t = 0; t < kMaxNT; t++)
#pragma unroll
            for (int c = 0; c < NC; c++) P[t][c] += S.red[warp + w][t][c][g];
      }
    }
    if (k == 0 && s == 0) {
#pragma unroll
      for (int t = 0; t < kMaxNT; t++) {
        const int it = (ga + t) * kG + g;
        if (t < ntl && it < li.y) {
          const int i = li.x + it;
          pot[i] = coef * P[t][0];
          if (KER == FMMB_LAPLACE_G) {  // grad(1/r) = -d / r^3; G's gradient is optional
            if (grad) {
              grad[i] = -coef * P[t][1];
              grad[ni + i] = -coef * P[t][2];
              grad[2 * (size_t)ni + i] = -coef * P[t][3];
            }
          } else if (with_grad(KER)) {
            grad[i] = coef * P[t][1];
            grad[ni + i] = coef * P[t][2];
            grad[2 * (size_t)ni + i] = coef * P[t][3];
          }
        }
      }
    }
  }
}

template <int KER>
void launch_k(int nwork, bool excl, const int2* work, const int2* leaf_i, const int2* leaf_j, const int* list,
              const float4* tpos, const float4* tnrm, const float4* spos, const float4* snrm, const float* qs,
              float eps2, double coef, double* pot, double* grad, int ni, cudaStream_t st) {
  if (excl)
    p2p_mixed<KER, true><<<nwork, kThreads, 0, st>>>(work, leaf_i, leaf_j, list, tpos, tnrm, spos, snrm, qs, eps2,
                                                     coef, pot, grad, ni);
  else
    p2p_mixed<KER, false><<<nwork, kThreads, 0, st>>>(work, leaf_i, leaf_j, list, tpos, tnrm, spos, snrm, qs, eps2,
                                                      coef, pot, grad, ni);
}

}  // namespace

void launch_p2p_mixed(int kernel, int nwork, const int2* work, const int2* leaf_i, const int2* leaf_j, const int* list,
                      const float4* tpos, const float4* tnrm, const float4* spos, const float4* snrm, const float* qs,
                      const Sem& s, double* pot, double* grad, int ni, cudaStream_t st) {
  if (nwork <= 0) return;
  const float eps2 = (float)s.eps2;
  const bool excl = s.excl_self != 0;
  if (kernel == FMMB_LAPLACE_G)
    launch_k<FMMB_LAPLACE_G>(nwork, excl, work, leaf_i, leaf_j, list, tpos, tnrm, spos, snrm, qs, eps2, s.coef, pot,
                             grad, ni, st);
  else if (kernel == FMMB_LAPLACE_GNI && grad)
    launch_k<FMMB_LAPLACE_GNI | kWithGrad>(nwork, excl, work, leaf_i, leaf_j, list, tpos, tnrm, spos, snrm, qs, eps2,
                                           s.coef, pot, grad, ni, st);
  else if (kernel == FMMB_LAPLACE_GNJ && grad)
    launch_k<FMMB_LAPLACE_GNJ | kWithGrad>(nwork, excl, work, leaf_i, leaf_j, list, tpos, tnrm, spos, snrm, qs, eps2,
                                           s.coef, pot, grad, ni, st);
  else if (kernel == FMMB_LAPLACE_GNI)
    launch_k<FMMB_LAPLACE_GNI>(nwork, excl, work, leaf_i, leaf_j, list, tpos, tnrm, spos, snrm, qs, eps2, s.coef, pot,
                               grad, ni, st);
  else
    launch_k<FMMB_LAPLACE_GNJ>(nwork, excl, work, leaf_i, leaf_j, list, tpos, tnrm, spos, snrm, qs, eps2, s.coef, pot,
                               grad, ni, st);
  FMMB_CHECK_LAUNCH();
}

}  // namespace fmmb

// Kernel launchers shared by the API layer (not part of the C ABI).
#pragma once

#include <cuda_runtime.h>

namespace fmmb {

// Arithmetic conventions of a plan (reference or accurate semantics).
struct Sem {
  double eps2;     // P2P softening added to r^2
  double coef;     // 1/(4 pi)
  double rho_eps;  // added to expansion radii (reference: 1e-6)
  double ang_eps;  // azimuth branch threshold (reference: 1e-6)
  double pi_ang;   // pi in azimuth branches
  int ref;         // reference semantics
  int excl_self;   // skip zero-distance pairs
};

__host__ __device__ __forceinline__ int ifull_d(int n, int m) { return n * n + n + m; }

// device primitives of the tree build (tree.cu), also used by the set-up of
// the evaluation work lists (setup.cu); both synchronise the stream on return
void exclusive_scan(int* data, int n, cudaStream_t s);  // in place
void radix_sort(int* keys, int* vals, int n, int bits, cudaStream_t s);  // stable, keys >= 0 below 2^bits
void launch_gather_charges(int n, int nrhs, const int* perm, const float* q, float* qs, cudaStream_t st);
// Near field of one right-hand side over work items (target leaf, first
// target) of up to 128 targets of a leaf against its 27 neighbour slots
// (list[leaf][27]); one block per item.
void launch_p2p_f64(int kernel, int nwork, const int2* work, const int2* leaf_i, const int2* leaf_j, const int* list,
                    const float4* tpos, const float4* tnrm, const float4* spos, const float4* snrm, const float* qs,
                    const Sem& s, double* pot, double* grad, int ni, cudaStream_t st);
void launch_p2p_mixed(int kernel, int nwork, const int2* work, const int2* leaf_i, const int2* leaf_j, const int* list,
                      const float4* tpos, const float4* tnrm, const float4* spos, const float4* snrm, const float* qs,
                      const Sem& s, double* pot, double* grad, int ni, cudaStream_t st);
void launch_p2m(int kernel, int nleaf, int p, int K, const int* keys, const int2* leaf, const float4* spos, const float4* snrm,
                const float* qs, const double* fac, const Sem& s, const float* bbox, double rb, double* M, cudaStream_t st);
// trig-free Cartesian P2M / L2P (accurate semantics), expansions_cart.cu
void launch_p2m_cart(int kernel, int nleaf, int p, int K, const int* keys, const int2* leaf, const float4* spos,
                     const float4* snrm, const float* qs, const double* fac, const float* bbox, double rb, double* M,
                     cudaStream_t st);
void launch_l2p_cart(int kernel, int nleaf, int p, int K, const int* keys, const int2* leaf, const float4* tpos,
                     const float4* tnrm, const double* fac, const float* bbox, double rb, double coef, const double* L,
                     double* pot, double* grad, int ni, cudaStream_t st);
// far-field gradient of the Gni potential w.r.t. the target position
// (normal fixed), -(1/4pi) H n from the local expansions (accurate semantics)
void launch_l2p_hess_gni(int nleaf, int p, int K, const int* keys, const int2* leaf, const float4* tpos,
                         const float4* tnrm, const double* fac, const float* bbox, double rb, double coef,
                         const double* L, double* grad, int ni, cudaStream_t st);
// mixed-form near field of nrhs right-hand sides in one pass (p2p_multi.cu):
// qs [nrhs][nj] sorted charges, pot [nrhs][ni], grad [nrhs][3][ni] (G only,
// may be null); work items (target leaf, first target) of up to 128 targets.
// Returns the number of launches.
int launch_p2p_multi(int kernel, int nrhs, int nwork, const int2* work, const int2* leaf_i, const int2* leaf_j,
                     const int* list, const float4* tpos, const float4* tnrm, const float4* spos, const float4* snrm,
                     const float* qs, int nj, const Sem& s, double* pot, double* grad, int ni, cudaStream_t st);
// FP32 point-per-thread P2M for the mixed form (accurate semantics, p <= 12:
// its kP2MItem x K staging must fit 48 KB of shared memory); returns false
// outside that range.  work: (source leaf, first source) items of up to
// kP2MItem sources (build_p2m_work_dev); a leaf of more sources is summed by
// several items with FP64 atomics, so its rows of M must be zero beforehand.
constexpr int kP2MItem = 64;
bool launch_p2m_f32(int kernel, int nwork, const int2* work, int p, int K, const int* keys, const int2* leaf,
                    const float4* spos, const float4* snrm, const float* qs, const float* bbox, double rb, double* M,
                    cudaStream_t st);
// FP32 L2P for the mixed form (accurate semantics, p <= 16); false outside its
// range.  work: (target leaf, first target) items of up to 128 targets.
bool launch_l2p_f32(int kernel, int nwork, const int2* work, int p, int K, const int* keys, const int2* leaf,
                    const float4* tpos, const float4* tnrm, const double* fac, const float* bbox, double rb,
                    double coef, const double* L, double* pot, double* grad, int ni, cudaStream_t st);
int translate_tile_size();
// batched FP64 translation (M2L / M2M / L2L), see kernels_fp64.cu
void launch_translate_f64(int ntile, int nsplit, int K, int nslots, const int* tile_boxes, const int* tile_ops,
                          const int* list, const double* ops, const double* in, double* out, cudaStream_t st);
void launch_l2p(int kernel, int nleaf, int p, int K, const int* keys, const int2* leaf, const float4* tpos, const float4* tnrm,
                const double* fac, const Sem& s, const float* bbox, double rb, const double* L, double* pot, double* grad,
                int ni, cudaStream_t st);
void launch_finalize_f32(int n, const int* perm, const double* pn, const double* pf, const double* gn, const double* gf,
                         float* pot, float* grad, cudaStream_t st);
void launch_finalize_f64(int n, const int* perm, const double* pn, const double* pf, const double* gn, const double* gf,
                         double* pot, double* grad, cudaStream_t st);
void launch_direct_f64(int kernel, int i0, int i1, const int* inv_i, const float4* tpos, const float4* tnrm, int nj,
                       const float4* spos, const float4* snrm, const float* qs, const Sem& s, double* pot, double* grad,
                       cudaStream_t st);

}  // namespace fmmb

namespace fmmb {
// tensor-core translations (translate_tc.cu)
int tc_tile();
// p[i] *= s; out[k n + i] = w[i] * field[k n + i] (k = 0..2)
void launch_scale(float* p, size_t n, float s, cudaStream_t st);
void launch_scale(double* p, size_t n, double s, cudaStream_t st);
void launch_weight_field(int n, const float* w, const double* field, double* out, cudaStream_t st);
// FP64 box-pair translations (M2M, L2L): tiles of tp pairs of one operator
struct PairArgs {
  int ntile, tp, K, atomic;
  const int *tile_op, *tile_src, *tile_dst;  // [ntile], [ntile][tp], [ntile][tp]
  const double* opT;                         // operators transposed, [op][column][row], row stride K rounded up to even
  size_t ostride;                            // doubles per operator: K * (K rounded up to even)
  const double* xin;                         // input expansions [rows][K]
  double* out;                               // output expansions [rows][K]
};
// pairs per tile (the FP64 tensor-core kernel's 32)
int pairs_f64_tile(int K, int npair, int nsm);
// once per device, before any launch (and outside stream capture)
void prepare_translate_pairs_f64();
void launch_translate_pairs_f64(const PairArgs& a, cudaStream_t st);
// constant table of the FP32 P2M, once per device (outside stream capture)
void init_fac32();
void launch_split_tf32(int nbox, int K, int kpad, const double* M, float* Mtf, cudaStream_t st);
struct TcJobArgs {
  int ntile, K;                 // work items, real coefficients per expansion (<= tc_max_k())
  const int* tile_op;           // [ntile] operator image per work item
  const int* tile_src;          // [ntile][128] input rows
  const int2* tile_y;           // [ntile] (first pair row of y, coefficient offset)
  const float* opimg;           // operator images, see translate_tc.cu
  const float* xin;             // TF32 split of the inputs [rows][2][tc_kpad(K)]
  float* y;                     // pair rows [pairs][ys]
  int ys;                       // floats per pair row
  int* err;
};
// once per device, before any launch (and outside stream capture)
void prepare_translate_tc();
void launch_translate_tc(const TcJobArgs& a, int nsm, cudaStream_t st);
// out[rows[w]] += sum of the pair rows y[idx[ptr[w]..ptr[w+1])] (rows of ys floats; FP64, list order)
void launch_reduce_pairs(int nrow, const int* rows, const int* ptr, const int* idx, const float* y, int ys, int K,
                         double* out, cudaStream_t st);
// FP16x3 tensor-core M2L (translate_h16.cu), K <= h16_max_k(): operators of
// h16_n(K) output rows (K rounded up to 16), inputs split as [rows][2][h16_kpad(K)]
// FP16 (hi, lo) with a power-of-two exponent per row, pair rows of ys floats
struct H16JobArgs {
  int ntile, K, ys;
  const int* tile_op;           // [ntile] operator per tile (sorted)
  const int* tile_src;          // [ntile][128] input rows (-1 = empty)
  const int2* tile_y;           // [ntile] (first pair row of y, 0)
  const void* opimg;            // operator images of h16_img_bytes(K) each
  const void* xin;              // FP16 split of the inputs
  const int* xexp;              // per input row: its scaling exponent
  float* y;
  int* err;
};
int h16_max_k();
int h16_n(int K);
int h16_kpad(int K);
size_t h16_img_bytes(int K);
// once per device, before any launch (and outside stream capture)
void prepare_translate_h16();
void launch_translate_h16(const H16JobArgs& a, int nsm, cudaStream_t st);
void launch_split_h16(int nbox, int K, const double* M, void* xh, int* xexp, cudaStream_t st);
// K padded for the tensor-core operands (128, or a multiple of 32 up to tc_max_k())
int tc_kpad(int K);
int tc_max_k();

// complex Helmholtz kernel (helmholtz.cu); complex values interleaved (re, im),
// expansions [re(K) | im(K)] per box, K = (p+1)^2
struct HelmOp {          // one translation operator to build
  double dx, dy, dz;     // target centre - source centre
  double rad;            // radius of the projection sphere around the target centre
  int src_out, tgt_out;  // 1: outgoing (h_n) basis, 0: regular (j_n) basis
};
void launch_helm_gather(int n, int nrhs, const int* perm, const float* q, float* qs, cudaStream_t st);
// work: (target leaf, first target) per item of up to 256 targets; yuk: the
// Yukawa kernel (real e^{-k r}/(4 pi r), complex charges with zero imaginary parts)
// leaf_side: side of a leaf box (decides whether the FP32 phase needs its
// range reduction)
void launch_helm_p2p(bool f32, bool yuk, float k, float eps2, bool excl, float leaf_side, int nwork,
                     const int2* work, const int2* leaf_i, const int2* leaf_j, const int* list, const float4* tpos,
                     const float4* spos, const float* qs, double* pot, cudaStream_t st);
void launch_helm_gather_real(int n, int nrhs, const int* perm, const float* q, float* qs, cudaStream_t st);
template <typename T>
void launch_helm_finalize_real(int n, const int* perm, const double* near, const double* far, double scale, T* out,
                               cudaStream_t st);
// bbox: the plan's host copy {xmin, ymin, zmin, rd}
void launch_helm_p2m(int nleaf, int p, double k, bool yuk, const int* keys, const int2* leaf, const float4* spos,
                     const float* qs, const float* bbox, double w, double* M, cudaStream_t st);
void launch_helm_l2p(int nleaf, int p, double k, bool yuk, const int* keys, const int2* leaf, const float4* tpos,
                     const float* bbox, double w, const double* L, double* pot, cudaStream_t st);
void launch_helm_direct(int i0, int i1, const int* inv_i, const float4* tpos, int nj, const float4* spos,
                        const float* qs, double k, bool yuk, double eps2, bool excl, double* out, cudaStream_t st);
template <typename T>
void launch_helm_finalize(int n, const int* perm, const double* near, const double* far, T* out, cudaStream_t st);
// operators in the real 2K x 2K form, transposed ([op][column][row], row stride 2K)
void launch_helm_build_ops(int p, double k, bool yuk, int nops, const HelmOp* ops, const double* gl_x,
                           const double* gl_w, const double* ybar_q, double* opT, cudaStream_t st);
}  // namespace fmmb

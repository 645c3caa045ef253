// Internal declarations of libfmmb (not part of the C ABI).
#pragma once

#include <cuda_runtime.h>

#include <complex>
#include <cstdint>
#include <memory>
#include <string>
#include <vector>

#include "../../include/fmmb.h"

namespace fmmb {

// ---- error handling: every entry point returns a status, nothing aborts ----
void set_error(const std::string& msg);
struct Error {
  int code;
  std::string msg;
};
#define FMMB_CUDA(call)                                                                      \
  do {                                                                                       \
    cudaError_t e_ = (call);                                                                 \
    if (e_ != cudaSuccess)                                                                   \
      throw ::fmmb::Error{FMMB_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)}; \
  } while (0)
#define FMMB_CHECK_LAUNCH() FMMB_CUDA(cudaGetLastError())
#define FMMB_REQUIRE(cond, code, msg) \
  do {                                \
    if (!(cond)) throw ::fmmb::Error{code, msg}; \
  } while (0)

// Owning device buffer (allocated at plan/geometry time only).
template <typename T>
struct DevBuf {
  T* ptr = nullptr;
  size_t n = 0;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() { release(); }
  void release() {
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    n = 0;
  }
  void alloc(size_t count) {
    if (count <= n && ptr) return;
    release();
    size_t bytes = (count ? count : 1) * sizeof(T);
    cudaError_t e = cudaMalloc(&ptr, bytes);
    if (e != cudaSuccess) {
      ptr = nullptr;
      throw Error{FMMB_ERR_NOMEM, std::string("cudaMalloc ") + std::to_string(bytes) + " B: " + cudaGetErrorString(e)};
    }
    n = count;
  }
  T* get() const { return ptr; }
};

// Per-device memory pool of the set-up scratch (tree build, work lists):
// stream-ordered, keeping up to kScratchPoolKeep bytes between calls so that
// repeated geometries of similar size reuse its memory.
constexpr uint64_t kScratchPoolKeep = 512ull << 20;
cudaMemPool_t scratch_pool();

// Scratch buffer of one set-up call: allocated from scratch_pool() in the
// order of stream `s` and freed in that order on destruction, so freeing it
// waits for nothing (cudaFree synchronises the device).
template <typename T>
struct TmpBuf {
  T* ptr = nullptr;
  size_t n = 0;
  cudaStream_t s = nullptr;
  explicit TmpBuf(cudaStream_t st) : s(st) {}
  TmpBuf(const TmpBuf&) = delete;
  TmpBuf& operator=(const TmpBuf&) = delete;
  TmpBuf(TmpBuf&& o) noexcept : ptr(o.ptr), n(o.n), s(o.s) {
    o.ptr = nullptr;
    o.n = 0;
  }
  ~TmpBuf() { release(); }
  void release() {
    if (ptr) cudaFreeAsync(ptr, s);
    ptr = nullptr;
    n = 0;
  }
  void alloc(size_t count) {
    if (count <= n && ptr) return;
    release();
    const size_t bytes = (count ? count : 1) * sizeof(T);
    cudaError_t e = cudaMallocFromPoolAsync(reinterpret_cast<void**>(&ptr), bytes, scratch_pool(), s);
    if (e != cudaSuccess) {
      ptr = nullptr;
      throw Error{FMMB_ERR_NOMEM, std::string("cudaMallocFromPoolAsync ") + std::to_string(bytes) + " B: " +
                                      cudaGetErrorString(e)};
    }
    n = count;
  }
  T* get() const { return ptr; }
};

inline int isym(int n, int m) { return n * (n + 1) / 2 + m; }
inline int ifull(int n, int m) { return n * n + n + m; }

// Number of M2L slots per target box: children of the parent's 27 neighbours
// that are not adjacent (fmm/ijbox.cxx:74-109).
constexpr int kM2LSlots = 189;
constexpr int kP2PSlots = 27;
constexpr int kRelCodes = 343;  // (dx+3)*49 + (dy+3)*7 + (dz+3)

// Host-side operator tables (operators.cpp).
struct Operators {
  int p = 0, K = 0;
  bool ref = true;
  std::vector<double> fac;   // ifull(n,m), n <= p (P2M/L2P normalisation)
  // Scaled, real-packed operators, K x K row-major (out row, in col).
  std::vector<double> m2m;   // [8][K][K]   child octant -> parent
  std::vector<double> l2l;   // [8][K][K]   parent -> child octant
  std::vector<double> m2l;   // [nsets][316][K][K]
  int m2l_sets = 0;          // 1 (accurate) or one per level 2..lmax (reference)
  int m2l_lmax = 0;
  float m2l_rd = 0;
  std::vector<int> rel_to_op;  // [343] -> operator slot (0..315) or -1
  std::vector<int> op_rel;     // [316] rel code of each operator slot
  std::vector<int> slot_rel;   // [8][189] rel code of each M2L slot per octant
  // Wigner rotation tables per relative position (forward, inverse)
  std::vector<std::vector<std::vector<std::complex<double>>>> Wf, Wb;
};
// fac, M2M, L2L, slot maps and rotation tables (independent of the geometry)
void build_static_operators(Operators& ops, int p, bool ref_semantics);
// M2L sets: one in accurate semantics; one per level 2..lmax in reference
// semantics, where the distance carries an absolute eps (needs the root size).
void build_m2l_operators(Operators& ops, int lmax, float rd);
// TF32 hi/lo images of nmat K x K operators in the tensor-core operand layout
void build_tc_images(const std::vector<double>& mats, int nmat, int K, int kpad, std::vector<float>& img);
// FP16 hi/lo images (row-scaled) for the FP16x3 M2L, img_bytes each
void build_h16_images(const std::vector<double>& mats, int nmat, int K, int n, int kpad, size_t img_bytes,
                      std::vector<unsigned char>& img);

struct Stream2 {
  cudaStream_t main = nullptr, side = nullptr;
  cudaStream_t cap = nullptr;  // private stream the evaluate graphs are captured on
  cudaEvent_t fork = nullptr, join = nullptr;
  cudaEvent_t near_done = nullptr;  // the all-right-hand-side near field finished
  // host copies that overlap the main stream's work (fmmb_adjoint_f64):
  // a stream made on first use, and its two ordering events
  cudaStream_t copy = nullptr;
  cudaEvent_t copy_ev[2] = {nullptr, nullptr};
};

}  // namespace fmmb

struct fmmb_plan {
  fmmb_config cfg{};
  int p = 0, K = 0, P = 0;
  int device = 0;
  fmmb::Stream2 st;
  bool own_stream = true;
  cudaEvent_t ev[8] = {};
  // per-launch timing: event pairs recorded around each phase launch and
  // summed per phase when fmmb_get_timings is called
  static constexpr int kEvPool = 96;
  cudaEvent_t evp[kEvPool] = {};
  int ev_used = 0;
  std::vector<std::pair<int, int>> ev_phase;  // (phase, first event index of the pair)
  int launches = 0;                           // kernel launches of the last evaluate

  // host copies of the configuration-dependent constants
  double eps2 = 0, coef = 0, rho_eps = 0, ang_eps = 0, pi_ang = 0;
  bool ref = true;
  fmmb::Operators ops;

  // ---- geometry (set_geometry) ----
  bool have_geometry = false;
  bool have_expansions = false;
  int ni = 0, nj = 0, lmax = 0;
  float bbox[4] = {0, 0, 0, 1};
  std::vector<int> nbox_i, nbox_j;  // boxes per level [lmax+1]
  std::vector<int> off_i, off_j;    // offsets of each level in all-level arrays (lmax first)
  int tot_i = 0, tot_j = 0;
  long long p2p_pairs = 0, m2l_pairs = 0;
  double tree_ms = 0, setup_ms = 0;  // wall time of the octree build and of the whole fmmb_set_geometry

  // sorted particles
  fmmb::DevBuf<int> perm_i, perm_j;          // sorted position -> caller index
  fmmb::DevBuf<float4> tpos, tnrm;           // targets (x,y,z,0), normals
  fmmb::DevBuf<float4> spos, snrm;           // sources
  // boxes (all levels concatenated, lmax first)
  fmmb::DevBuf<int> key_i, key_j;            // Morton keys at their level
  fmmb::DevBuf<int> parent_i, parent_j;      // index (within level l-1) of the parent, -1 at level 2
  fmmb::DevBuf<int2> leaf_i, leaf_j;         // leaf (first, count) in sorted order
  fmmb::DevBuf<int> p2p_list;                // [nleaf_i][27] source leaf or -1
  fmmb::DevBuf<int> m2l_list;                // [tot_i][189] source box (within level) or -1
  fmmb::DevBuf<int> leafkey_i, leafkey_j;    // leaf keys without the problem bits (box centres)
  // independent problems in one plan (fmmb_set_geometry_batch): problem b owns
  // targets [prob_toff[b], prob_toff[b+1]) and sources [prob_soff[b], ..),
  // in caller and in sorted order alike; on the device [toff | soff]
  int nprob = 1;
  std::vector<int> prob_toff, prob_soff;
  fmmb::DevBuf<int> d_prob_off;
  fmmb::DevBuf<int> child_start_j;           // for M2M: per source box at level l (<lmax): first child index, count
  fmmb::DevBuf<int> child_count_j;

  // operators on the device
  fmmb::DevBuf<double> d_fac, d_m2l;
  fmmb::DevBuf<double> d_m2m_t, d_l2l_t;    // [8][column][row] (transposed for the FP64 pair kernel)
  fmmb::DevBuf<int> d_slot_rel, d_rel_to_op;
  fmmb::DevBuf<float> d_img_m2l;             // [sets*316][4 K-blocks][2][128*32] TF32 images (mixed)

  // evaluation buffers
  fmmb::DevBuf<float> qs;                    // sorted charges [nrhs][nj]
  fmmb::DevBuf<double> M, L;                 // [tot][K] scaled real-packed
  fmmb::DevBuf<float> Mtf;                   // [tot_j][2][tc_kpad(K)] TF32 hi/lo split of M (mixed, M2L input)
  fmmb::DevBuf<int> d_err;                   // device error code of the tensor-core kernels
  int* h_err = nullptr;                      // pinned copy, checked by the next call
  bool use_tc = false;                       // M2L on the tensor cores in TF32x3 (mixed, h16_max_k() < K <= 256)
  bool use_h16 = false;                      // M2L on the tensor cores in FP16x3 (mixed, K <= h16_max_k())
  fmmb::DevBuf<unsigned char> d_img_h16;     // [sets*316] FP16 operator images
  fmmb::DevBuf<unsigned short> Xh;           // [tot_j][2][h16_kpad(K)] scaled FP16 hi/lo split of M
  fmmb::DevBuf<int> xexp;                    // [tot_j] its exponents
  // The plan-internal part of a one-right-hand-side evaluate (sorted charges ->
  // sorted outputs, plan-owned buffers only) captured once per geometry as a
  // CUDA graph, without / with gradient, with the phase-timer records and the
  // launch count of the capturing call.
  bool use_graph = true;
  bool capturing = false;
  // transposed FMM (fmmb_evaluate_transpose, fmmb_position_grad): caller-order
  // copies of the geometry [tx ty tz tnx tny tnz | sx sy sz snx sny snz] and the
  // plan with targets and sources swapped, built on first use
  fmmb::DevBuf<float> geo;
  bool geo_tn = false, geo_sn = false;
  bool same_sets = false;  // targets and sources given as the same arrays (one problem)
  fmmb_plan* tplan = nullptr;  // == this plan for a symmetric kernel on one point set
  fmmb::DevBuf<double> pg_tmp;                 // position-gradient work space
  fmmb::DevBuf<double> adj_tmp;                // fmmb_adjoint_f64 work space
  fmmb::DevBuf<float> adj_qs, adj_ws;          // its staged charges and weights
  // graphs [without / with gradient] x [whole evaluate / far field only]
  cudaGraphExec_t gexec[4] = {nullptr, nullptr, nullptr, nullptr};
  std::vector<std::pair<int, int>> gphase[4];
  int glaunches[4] = {0, 0, 0, 0};
  // many right-hand sides (mixed form): the near field of all of them in one
  // pass (p2p_multi.cu) into near_all ([nrhs][ni] potentials, then
  // [nrhs][3][ni] gradients), the far field per right-hand side through the
  // far-field-only graph, whose charges are qs_far
  bool far_only = false;
  bool serial = false;  // near field on the main stream (fmmb_set_overlap(0))
  // fmmb_gmres workspaces (Krylov vectors, per-system state, chunk tables)
  fmmb::DevBuf<int> gm_ci, gm_si;
  fmmb::DevBuf<double> gm_vec, gm_sd;
  fmmb::DevBuf<float> gm_q, gm_w;
  fmmb::DevBuf<double> near_all;
  fmmb::DevBuf<float> qs_far;
  fmmb::DevBuf<int2> m_p2p_work;  // (target leaf, first target), up to 128 targets each
  int m_p2p_nwork = 0;
  // P2M work items of the mixed form: (source leaf, first source), up to
  // kP2MItem sources each, in leaf order
  fmmb::DevBuf<int2> p2m_work;
  int p2m_nwork = 0;
  // the same items for the one-right-hand-side near field, heaviest first in
  // each of its two launches: [0, p2p_nwork0) and [p2p_nwork0, p2p_nwork)
  fmmb::DevBuf<int2> p2p_work;
  int p2p_nwork = 0, p2p_nwork0 = 0;
  int opimg_sets = 0;
  float opimg_rd = 0;
  // tensor-core translation jobs: work items of 64 output boxes with their slots
  struct TcJob {  // work items of the tensor-core M2L (translate_tc.cu)
    int ntile = 0;                               // work items (pair tile x block of 128 output rows)
    fmmb::DevBuf<int> tile_op, tile_src, tile_y; // operator image, input rows, (pair row, row offset)
    // the launch stores pair rows of ys floats to tc_y and reduce_pairs sums
    // them per output row: rows, CSR offsets, pair rows (tile*128 + column)
    int nred = 0, ys = 128;
    fmmb::DevBuf<int> red_rows, red_ptr, red_idx;
  };
  fmmb::DevBuf<float> tc_y;                                  // pair rows of the M2L launch
  TcJob tc_m2l;                                              // all levels
  int nsm = 148;                                             // SMs of the plan's device
  // FP64 pair tiles of M2M (into parents at a level) and L2L (into children
  // at a level), index = level
  struct PairJob {
    int ntile = 0, tp = 0;
    fmmb::DevBuf<int> tile_op, tile_src, tile_dst;
  };
  std::vector<std::unique_ptr<PairJob>> m2m_pairs, l2l_pairs;
  // complex Helmholtz: dense operators in the real 2K x 2K form (transposed),
  // [M2M child levels 3..lmax x 8 | L2L likewise | M2L levels 2..lmax x 316],
  // and the M2L pairs of all levels
  fmmb::DevBuf<double> d_hops;
  int hop_m2m0 = 0, hop_l2l0 = 0, hop_m2l0 = 0;
  fmmb::DevBuf<int2> h_p2p_work;  // P2P work items: (target leaf, first target), up to 256 targets each
  int h_p2p_nwork = 0;
  std::unique_ptr<PairJob> h_m2l;
  fmmb::DevBuf<double> pot_s, grad_s;        // sorted outputs [ni], [3][ni]
  fmmb::DevBuf<float> stage_f;               // host<->device staging
  fmmb::DevBuf<double> stage_d;
  fmmb::DevBuf<int> inv_i;                   // caller index -> sorted target position
  fmmb::DevBuf<char> stage_out;              // device staging of host outputs
  bool timings_valid = false;
  // FP64 translation tiles per level (kernels_fp64.cu translate_f64): output
  // boxes [ntile][32] and per-tile operator index per slot [ntile][nslots]
  struct TileSet {
    int ntile = 0;
    fmmb::DevBuf<int> boxes, ops;
  };
  std::vector<std::unique_ptr<TileSet>> m2l_tiles;  // index = level
  fmmb::DevBuf<int> m2m_list;                                            // [tot_j][8] child (within level) or -1
};

namespace fmmb {
// work lists built on the device from the tree (setup.cu): the FP16 M2L's pair
// tiles and reduction CSR (false: too large for the int enumeration, build on
// the host), the near-field work items, the inverse target permutation
bool build_m2l_job_dev(fmmb_plan* pl, fmmb_plan::TcJob& job, int ys, cudaStream_t s);
void build_p2p_work_dev(fmmb_plan* pl, cudaStream_t s);
void build_p2m_work_dev(fmmb_plan* pl, cudaStream_t s);
void build_inverse_perm_dev(fmmb_plan* pl, cudaStream_t s);
// complex Helmholtz and Yukawa operators, pair jobs and buffers (helmholtz_host.cpp)
void helm_setup(fmmb_plan* pl);
// the kernels of the Helmholtz machinery (complex expansions, dense operators)
inline bool helm_family(int kernel) { return kernel == FMMB_HELMHOLTZ_G || kernel == FMMB_YUKAWA; }
void build_tree(fmmb_plan* pl, int ni, const float* tx, const float* ty, const float* tz, const float* tnx,
                const float* tny, const float* tnz, int nj, const float* sx, const float* sy, const float* sz,
                const float* snx, const float* sny, const float* snz, const float* bbox_in);
}

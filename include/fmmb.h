/*
 * fmmb.h -- C ABI of libfmmb.so, a B200-native fast multipole matvec for the
 * Laplace kernels of exafmm/old_fmm_bem.
 *
 * The reference exposes its FMM as `void fmm(int mi, int mj, int neq)`
 * (fmm/fmm.cxx:29) over global, pre-sorted particle arrays, with the GPU work
 * behind the batch ABI p2pgpu_/p2mgpu_/m2lgpu_/l2pgpu_ (libgpu/gpufmm.cu:57,
 * 200, 336, 481).  This ABI replaces both with a handle: a plan owns the tree,
 * the translation operators and all device buffers; fmmb_set_geometry builds
 * the octree on the GPU; fmmb_evaluate runs P2P, P2M, M2M, M2L, L2L and L2P on
 * the GPU.  Kernel numbering follows the reference's `neq` (fmm/fmm.cxx:47-65).
 *
 * Conventions
 *  - Arrays are structure-of-arrays float32, like the reference's xi/yi/zi...
 *    (include/arrays.h:5-12).  Pointers may be host or device memory; host
 *    inputs are copied to the device and host outputs copied back inside the
 *    call (cudaPointerGetAttributes decides).
 *  - Every call returns FMMB_OK (0) or a negative error code; the message of
 *    the last error on the calling thread is fmmb_last_error().  Nothing
 *    aborts the process (the reference exits through CUDA_SAFE_CALL).
 *  - A plan is used by one host thread at a time; different plans are
 *    independent.  Work is queued on the plan's stream (fmmb_set_stream).
 */
#ifndef FMMB_H
#define FMMB_H

#if defined(__GNUC__)
#define FMMB_API __attribute__((visibility("default")))
#else
#define FMMB_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define FMMB_OK 0
#define FMMB_ERR_ARG (-1)       /* invalid argument or configuration */
#define FMMB_ERR_CUDA (-2)      /* a CUDA call failed */
#define FMMB_ERR_STATE (-3)     /* call out of order (e.g. evaluate before geometry) */
#define FMMB_ERR_CAPACITY (-4)  /* a size exceeds what the plan supports */
#define FMMB_ERR_NOMEM (-5)     /* device allocation failed */

/* Kernels, numbered like the reference's neq (fmm/fmm.cxx:47-65). */
#define FMMB_LAPLACE_G 0    /* potential sum q/(4 pi r) and its gradient */
#define FMMB_LAPLACE_GNI 1  /* target-normal derivative: sum q (r.n_i)/(4 pi r^3) */
#define FMMB_LAPLACE_GNJ 2  /* source-normal (double layer): sum q (r.n_j)/(4 pi r^3) */
#define FMMB_YUKAWA 10      /* the reference's neq 10 (kernel/Helmholtz_G_p2p.cxx:18-23): sum q
                               (pi/2) e^{-l r}/(l r), l = cfg.wavenumber; real charges and
                               potentials; no gradient; FMMB_SEM_ACCURATE only (no eps in r) */
#define FMMB_HELMHOLTZ_G 20 /* complex sum q e^{ikr}/(4 pi r), k = cfg.wavenumber: charges and
                               potentials are complex, interleaved (re, im) floats; no gradient;
                               FMMB_SEM_ACCURATE only. */

/* Precision of the evaluation. */
#define FMMB_FP64 0   /* every phase in FP64 on the CUDA cores */
#define FMMB_MIXED 1  /* FP32 P2P with compensated sums, M2L as TF32x3 tensor-core GEMMs */

/* Arithmetic semantics. */
#define FMMB_SEM_REFERENCE 0 /* the reference's conventions: eps=1e-6f added to r^2 and to
                                expansion radii, single-precision pi, fac/anm/sr tables
                                rounded to float, self pairs included */
#define FMMB_SEM_ACCURATE 1  /* exact angles and constants; eps2 as given; exclude_self honoured */

typedef struct {
  int kernel;       /* FMMB_LAPLACE_* */
  int p;            /* expansion order, 1..20 (the reference's mp = p+1) */
  int lmax;         /* octree depth of the leaves, 2..10 */
  int precision;    /* FMMB_FP64 or FMMB_MIXED */
  int semantics;    /* FMMB_SEM_REFERENCE or FMMB_SEM_ACCURATE */
  double eps2;      /* P2P softening added to r^2 (FMMB_SEM_ACCURATE only) */
  int exclude_self; /* skip pairs at zero distance (FMMB_SEM_ACCURATE only) */
  int nrhs;         /* right-hand sides per evaluate, >= 1 */
  double wavenumber; /* k of FMMB_HELMHOLTZ_G, lambda of FMMB_YUKAWA (> 0); unused otherwise */
} fmmb_config;

typedef struct fmmb_plan fmmb_plan;

/* Fills cfg with defaults: Laplace G, p=8, lmax=3, FP64, reference semantics, nrhs=1. */
FMMB_API int fmmb_config_init(fmmb_config* cfg);

/* Replaces the reference's compile-time setup (include/constants.h:11-35,
 * fmm/alloc.cxx:32-84, kernel/precalc.cxx:10-213): validates cfg, selects the
 * current CUDA device, builds the rotation/translation operators. */
FMMB_API int fmmb_plan_create(const fmmb_config* cfg, fmmb_plan** plan);
FMMB_API int fmmb_plan_destroy(fmmb_plan* plan);

/* Work of this plan is queued on `stream` (a cudaStream_t; NULL = the plan's own;
 * cudaStreamLegacy for the legacy default stream). */
FMMB_API int fmmb_set_stream(fmmb_plan* plan, void* stream);

/* Builds the octree on the GPU (replaces fmm/boxn.cxx, sort/csort.cxx,
 * sort/sorti.cxx, sort/sortj.cxx, fmm/boxdata{i,j}.cxx, fmm/boxm2m{i,j}.cxx,
 * fmm/ijbox.cxx).  Targets (tx,ty,tz) with normals (tnx..; used by
 * FMMB_LAPLACE_GNI, may be NULL otherwise); sources (sx,sy,sz) with normals
 * (snx..; used by FMMB_LAPLACE_GNJ).  bbox = {xmin, ymin, zmin, rd} is the
 * root cube, like the reference's xmin/ymin/zmin/rd globals; NULL computes a
 * cube enclosing all points.  Points are given in caller order: the
 * permutation into Morton order is internal. */
FMMB_API int fmmb_set_geometry(fmmb_plan* plan, int ni, const float* tx, const float* ty, const float* tz,
                      const float* tnx, const float* tny, const float* tnz, int nj,
                      const float* sx, const float* sy, const float* sz, const float* snx,
                      const float* sny, const float* snz, const float* bbox);

/* Many independent problems in one plan (a forest of octrees): problem b owns
 * targets [t_off[b], t_off[b+1]) and sources [s_off[b], s_off[b+1]) of the
 * concatenated arrays (t_off[0] = s_off[0] = 0; t_off[nprob] = ni and
 * s_off[nprob] = nj are the totals).  Points of different problems never
 * interact: the problem index sits above the Morton bits of every box key, so
 * neighbour and interaction lists stay inside a problem, and each problem's
 * result equals that of its own plan over the same root cube.  All problems
 * share bbox (NULL: a cube enclosing all points) and lmax; 3*lmax +
 * ceil(log2(nprob)) <= 30.  fmmb_evaluate then runs every problem in the
 * same launches; q / pot keep the concatenated order (nrhs blocks of nj / ni).
 * Offsets may be host or device arrays.  The reference runs one problem per
 * fmm() call (bio/main.cxx:377-413); no counterpart. */
FMMB_API int fmmb_set_geometry_batch(fmmb_plan* plan, int nprob, const int* t_off, const float* tx,
                                     const float* ty, const float* tz, const float* tnx, const float* tny,
                                     const float* tnz, const int* s_off, const float* sx, const float* sy,
                                     const float* sz, const float* snx, const float* sny, const float* snz,
                                     const float* bbox);

/* One FMM matvec (replaces fmm(mi, mj, neq), fmm/fmm.cxx:29-152).
 * q: nrhs x nj charges (caller order).  pot: nrhs x ni potentials (overwritten,
 * unlike the reference's += into vi).  grad (may be NULL): nrhs x 3 x ni
 * gradient of the potential w.r.t. the target position -- the field for
 * FMMB_LAPLACE_G; for FMMB_LAPLACE_GNI / FMMB_LAPLACE_GNJ the normals are held
 * fixed (accurate semantics only, FMMB_ERR_ARG otherwise); ignored for the
 * complex kernels. */
FMMB_API int fmmb_evaluate(fmmb_plan* plan, const float* q, float* pot, float* grad);
/* Same with FP64 outputs. */
FMMB_API int fmmb_evaluate_f64(fmmb_plan* plan, const float* q, double* pot, double* grad);

/* Transposed matvec (the charge adjoint): out[nj] = A^T w for w[ni] (nrhs
 * blocks), A being this plan's FMM.  G is symmetric, so A^T is the G-FMM from
 * the targets to the sources; for the normal-derivative kernels
 * d/dx_j G = -d/dx_i G gives Gni^T = -Gnj and Gnj^T = -Gni with the point
 * sets swapped.  grad[3 nj] (Laplace kernels, may be NULL) receives the
 * gradient of A^T w w.r.t. the source position (normals fixed).  For G on
 * one point set given as the same arrays the transposed plan is this plan;
 * otherwise the transposed plan (same root cube,
 * same settings) is built on the first call after fmmb_set_geometry.  No
 * counterpart in the reference (its fmm() has no adjoint). */
FMMB_API int fmmb_evaluate_transpose(fmmb_plan* plan, const float* w, float* out, float* grad);
FMMB_API int fmmb_evaluate_transpose_f64(fmmb_plan* plan, const float* w, double* out, double* grad);

/* Position gradients of L = sum_i w_i pot_i for the Laplace kernels (normals
 * held fixed; Gni / Gnj in accurate semantics), one right-hand side:
 * dxt[3 ni] = w * grad_t(pot) and dxs[3 nj] = q * grad_s(psi), psi = A^T w
 * (either output may be NULL; when targets and sources are the same points
 * the caller adds the two).  Costs one matvec and one transposed matvec, both
 * with gradient.  No reference counterpart. */
FMMB_API int fmmb_position_grad(fmmb_plan* plan, const float* q, const float* w, double* dxt, double* dxs);

/* The backward pass of one matvec pot = A q for L = sum_i w_i pot_i, given
 * the forward's field: dq[nj] = A^T w (the transposed matvec, as
 * fmmb_evaluate_transpose_f64), dxs[3 nj] = q * grad(psi)(x_s) with
 * psi = A^T w, and dxt[3 ni] = w * field_t, field_t[3 ni] being the gradient
 * output of the forward fmmb_evaluate_f64 with the same q.  Any of dq, dxs,
 * dxt may be NULL (dxt needs field_t); position gradients of Gni / Gnj need
 * accurate semantics.  Costs one transposed matvec (with gradient when dxs is
 * asked for); host or device pointers.  With host pointers, q's copy to the
 * device and dxt's copy to the host run on a second stream of the plan (made
 * on first use) while the transposed matvec runs; host outputs are complete
 * on return.  When the targets and sources were given as the same arrays the
 * transposed matvec runs on this plan.  No reference counterpart (the
 * reference has no adjoint). */
FMMB_API int fmmb_adjoint_f64(fmmb_plan* plan, const float* q, const float* w, const double* field_t, double* dq,
                              double* dxt, double* dxs);

/* Direct O(ni*nj) sum on the GPU with the plan's kernel and semantics
 * (replaces G_dir/Gni_dir/Gnj_dir, kernel/G_dir.cxx:6-30,
 * kernel/Gni_dir.cxx:6-21, kernel/Gnj_dir.cxx:6-21), FP64 arithmetic.  Uses
 * the geometry and the first right-hand side of q; targets [i0, i1).  grad
 * (may be NULL): 3 x (i1 - i0), the gradient w.r.t. the target position
 * (normals fixed), for every Laplace kernel. */
FMMB_API int fmmb_direct_f64(fmmb_plan* plan, const float* q, int i0, int i1, double* pot, double* grad);

/* The reference's batch near-field call p2pgpu_ (libgpu/gpufmm.cu:57-61) with
 * its exact arguments and record format (host arrays; the GPU work is
 * synchronous): targets xi..gzi in blocks of 128 (nvecd[1] blocks, gx.. the
 * target normals), sources xj..vj (nvecd[3] of them, gx.. the source normals),
 * nvecd[4] = neq 0/1/2, per block b: nvecd[b*nvecd[2] + 10] source ranges,
 * range r = (first nvecd[b*nvecd[2] + 2r + 11], count nvecd[b*nvecd[2] + 2r + 12]).
 * Overwrites vi, gxi, gyi, gzi of every packed target (gradient for neq 0,
 * zeros otherwise) with the reference's arithmetic (eps = 1e-6 on r^2).
 * compat/gpufmm_compat.cpp defines p2pgpu_ over it. */
FMMB_API int fmmb_gpu_p2p(const int* nvecd, float* xi, float* yi, float* zi, float* gxi, float* gyi, float* gzi,
                          float* vi, const float* xj, const float* yj, const float* zj, const float* gxj,
                          const float* gyj, const float* gzj, const float* vj);

/* The reference's batch P2M call p2mgpu_ (libgpu/gpufmm.cu:200-205): per
 * block b (nvecd[1] blocks, stride nvecd[2]) the source leaf's Morton key
 * nvecd[b*stride + 10] and its sources [nvecd[..+11], +nvecd[..+12]) of xj..vj
 * (nvecd[3] in all), nvecd[4] = 0 (G) or 1 (Gn, source normals gxj..),
 * nvecd[6] = mp (mp (mp+1) / 2 <= 64); rb the leaf side, xmin.. the root
 * corner.  Writes the multipole coefficients M_n^m of block b, in the
 * reference's normalisation, to brex/bimx[b*64 + n(n+1)/2 + m] (the other
 * slots of the block zeroed).  The reference's float fac table is not read:
 * the same table is built here.  compat/gpufmm_compat.cpp defines p2mgpu_. */
FMMB_API int fmmb_gpu_p2m(const int* nvecd, const double* rb, const double* xmin, const double* ymin,
                          const double* zmin, const float* xj, const float* yj, const float* zj, const float* gxj,
                          const float* gyj, const float* gzj, const float* vj, float* brex, float* bimx);

/* The reference's batch translation call m2lgpu_ (libgpu/gpufmm.cu:336-338):
 * nvecd[4] = 0 (M2M), 1 (M2L), 2 (L2L), nvecd[6] = mp (mp (mp+1) / 2 <= 64);
 * per block b (nvecd[1] blocks, stride nvecd[2]) nvecd[b*stride + 10] inputs,
 * input r = (offset of its coefficients in brex/bimx nvecd[..+2r+11],
 * relative-position code + 1 nvecd[..+2r+12]) with the codes of
 * kernel/m2m_gpu.cxx, m2l_gpu.cxx, l2l_gpu.cxx; rb the side of the output
 * boxes (parents for M2M, children for L2L).  Writes the sum over the block's
 * inputs of the translated coefficients (reference normalisation) to
 * arex/aimx[b*64 + n(n+1)/2 + m].  Reference semantics, every order (the
 * reference's own kernel is valid for mp <= 5 only). */
FMMB_API int fmmb_gpu_m2l(const int* nvecd, const double* rb, float* arex, float* aimx, const float* brex,
                          const float* bimx);

/* The reference's batch L2P call l2pgpu_ (libgpu/gpufmm.cu:481-486): blocks of
 * 64 targets xi.. (gxi.. their normals for nvecd[4] = 1), per block the leaf
 * key nvecd[b*stride + 10] and the offset nvecd[..+11] of its local
 * coefficients in arex/aimx (mp (mp+1) / 2 of them, nvecd[3] in all).
 * Overwrites vi (potential; for Gn -n.grad, the target-normal derivative) and
 * gxi.. (the gradient for G, zeros for Gn) of every packed target.  The
 * reference's Gn kernel stores its results at scrambled positions
 * (libgpu/Gn_l2p.cu writes veck[tx], libgpu/kernel.cu reads veck[4*tx+i]);
 * here every target gets its own value, as the reference's CPU Gn_l2p does.
 * compat/gpufmm_compat.cpp defines l2pgpu_. */
FMMB_API int fmmb_gpu_l2p(const int* nvecd, const double* rb, const double* xmin, const double* ymin,
                          const double* zmin, const float* xi, const float* yi, const float* zi, float* gxi,
                          float* gyi, float* gzi, float* vi, const float* arex, const float* aimx);

/* GMRES for the boundary-integral systems of a plan whose targets are its
 * sources (problem by problem):  A x = diag * x + K (weight .* x),  left
 * preconditioned by y = precond * x.  This is the reference's PETSc shell
 * solve (bio/main.cxx:27-53 mymatmult: weight = are/e1, diag =
 * (e1+e2)/(2 e1 (e1-e2)); :55-70 mypcshell: precond = 1/diag; :377-413
 * KSPSolve with KSPGMRES) moved onto the GPU, for nrhs x nprob independent
 * systems at once: each iteration is one fmmb_evaluate of all of them. */
typedef struct fmmb_gmres_config {
  int restart;    /* Krylov vectors per cycle, 1..64 (PETSc's default 30) */
  int max_iter;   /* iterations (matvecs after the initial residual) in all */
  double rtol;    /* a system stops when its preconditioned residual norm falls to
                     rtol times its initial one; 0 runs max_iter iterations */
  double diag;    /* identity term of A */
  double precond; /* scale of the preconditioner */
} fmmb_gmres_config;

/* Defaults: restart 30, max_iter 20, rtol 0, diag 0, precond 1. */
FMMB_API int fmmb_gmres_config_init(fmmb_gmres_config* cfg);

/* b: nrhs x n right-hand sides; x: nrhs x n initial guess, overwritten by the
 * solution (FP64, host or device; n = the plan's point count).  weight: n
 * floats or NULL (= 1).  iters: iterations done (may be NULL).  resid (may be
 * NULL): nrhs x nprob relative preconditioned residuals of the returned x per
 * system, ||precond (b - A x)|| / ||precond (b - A x0)||, computed with one
 * more matvec at exit (A being this plan's FMM; the rtol test during the
 * iterations uses the Givens estimate). */
FMMB_API int fmmb_gmres(fmmb_plan* plan, const fmmb_gmres_config* cfg, const float* weight, const double* b,
                        double* x, int* iters, double* resid);

/* Direct sum without a plan that allocates nothing (no cudaMalloc/cudaFree,
 * no allocating library routine).  It has no counterpart in the reference:
 * it serves callers that must not allocate device memory -- a host framework
 * that reserves the whole device memory up front for its own allocator, or a
 * loop that cannot take the implicit device synchronisation and the possible
 * failure of an allocation.  Same arithmetic as fmmb_direct_f64 (FP64, the
 * kernel, semantics, eps2 and exclude_self of cfg; the other fields are
 * ignored), float outputs pot[ni] and, for FMMB_LAPLACE_G, grad[3*ni] (may be
 * NULL).  Every pointer must be device memory of the current device (or
 * managed memory), else FMMB_ERR_ARG; work is queued on `stream` (a
 * cudaStream_t, NULL = the legacy default stream).
 * The FP64 partial sums of its source split live in one static device array of
 * FMMB_STATIC_SCRATCH_BYTES per device, reserved on every device that loads
 * this library's device code (at module load, whether or not this entry point
 * is called): ncomp * ni must not exceed
 * FMMB_STATIC_SCRATCH_BYTES / 8 (ncomp = 4 for G with grad, else 1), larger
 * sizes return FMMB_ERR_CAPACITY.  All calls on a device share that array:
 * calls that overlap on the GPU race and must be ordered by the caller.  The
 * first call on a device (that device current) looks the array up with
 * cudaGetSymbolAddress and keeps its address for the life of the process;
 * make it before any stream capture, and do not reset the device
 * (cudaDeviceReset) after it. */
#define FMMB_STATIC_SCRATCH_BYTES (16u << 20)
FMMB_API int fmmb_direct_static(const fmmb_config* cfg, int ni, const float* tx, const float* ty, const float* tz,
                                const float* tnx, const float* tny, const float* tnz, int nj, const float* sx,
                                const float* sy, const float* sz, const float* snx, const float* sny,
                                const float* snz, const float* q, float* pot, float* grad, void* stream);

/* Chooses the octree depth for a geometry: for each lmax in [lmin, lmax_hi]
 * (0, 0 = a range around 64 points per leaf) builds the tree of the given
 * targets / sources (arguments as for fmmb_set_geometry) with the settings of
 * cfg, times `reps` evaluates of fixed pseudo-random charges with CUDA events
 * and returns the fastest depth in *best; ms_out (may be NULL) receives the
 * milliseconds per evaluate of each candidate (-1 for a depth that did not fit
 * in device memory).  The reference fixes lmax from a table of N
 * (fmm/nlevel.cxx:5-31); this is the tuned replacement. */
FMMB_API int fmmb_autotune_lmax(const fmmb_config* cfg, int ni, const float* tx, const float* ty, const float* tz,
                                const float* tnx, const float* tny, const float* tnz, int nj, const float* sx,
                                const float* sy, const float* sz, const float* snx, const float* sny,
                                const float* snz, const float* bbox, int lmin, int lmax_hi, int reps, int* best,
                                float* ms_out);

/* Chooses the expansion order and octree depth for an accuracy target.  For
 * p = p_lo, p_lo + 1, ... p_hi: the depth from fmmb_autotune_lmax (reps timed
 * evaluates per candidate depth), then one FP64-output evaluate at that
 * (p, depth) of fixed pseudo-random charges, compared with the FP64 direct
 * sum (fmmb_direct_f64) on nsample targets (0: 1024) taken as 16 runs of
 * consecutive targets spread over the set.  Stops at the first order whose
 * relative error (2-norm over the sample) is at most tol: *p_out, *lmax_out,
 * *err_out (may be NULL) and *ms_out (may be NULL, ms per evaluate at that
 * depth) describe it; when no order in the range reaches tol they describe
 * p_hi and *err_out > tol tells.  Laplace kernels; the other cfg fields
 * (precision, semantics, ...) as given.  The reference fixes the order at
 * compile time (include/constants.h:15, mp); this chooses it per geometry and
 * tolerance, the depth as fmmb_autotune_lmax (fmm/nlevel.cxx:5-31). */
FMMB_API int fmmb_autotune_order(const fmmb_config* cfg, int ni, const float* tx, const float* ty, const float* tz,
                                 const float* tnx, const float* tny, const float* tnz, int nj, const float* sx,
                                 const float* sy, const float* sz, const float* snx, const float* sny,
                                 const float* snz, const float* bbox, double tol, int p_lo, int p_hi, int nsample,
                                 int reps, int* p_out, int* lmax_out, double* err_out, float* ms_out);

/* fmmb_autotune_lmax for a batch of independent problems
 * (fmmb_set_geometry_batch's arguments): the one depth of the forest. */
FMMB_API int fmmb_autotune_lmax_batch(const fmmb_config* cfg, int nprob, const int* t_off, const float* tx,
                                      const float* ty, const float* tz, const float* tnx, const float* tny,
                                      const float* tnz, const int* s_off, const float* sx, const float* sy,
                                      const float* sz, const float* snx, const float* sny, const float* snz,
                                      const float* bbox, int lmin, int lmax_hi, int reps, int* best, float* ms_out);

/* ---- inspection (tests, tooling) ---- */

/* Tree of the current geometry.  kind: 0 target permutation (sorted position
 * -> caller index, like the reference's nbi), 1 source permutation (nbj),
 * 2 target box keys of all levels lmax..2 concatenated (nfi), 3 source box
 * keys (nfj), 4/5 boxes per level [lmax+1], 6/7 leaf ranges (first, last)
 * pairs (ndi/ndj), 8 interaction lists as a stream
 * [lev, mode, nbox_i, nbox_j, counts..., entries...] per list in the order
 * fmm() builds them (mode 0 near field at lmax, 1 level 2, 2 levels 3..lmax).
 * fmmb_get_tree_size returns the element count (or an error). */
FMMB_API long fmmb_get_tree_size(fmmb_plan* plan, int kind);
FMMB_API int fmmb_get_tree(fmmb_plan* plan, int kind, int* out);

/* Expansions after the last evaluate (first right-hand side), in the
 * reference's unscaled normalisation: which 0 = multipoles of all source boxes,
 * 1 = locals of all target boxes, levels lmax..2 concatenated; per box
 * (p+1)(p+2)/2 complex coefficients (n, m>=0 at n(n+1)/2+m) as (re, im). */
FMMB_API long fmmb_get_expansion_size(fmmb_plan* plan, int which);
FMMB_API int fmmb_get_expansions(fmmb_plan* plan, int which, double* out);

/* Device time in ms of the phases of the last evaluate, summed over the
 * launches of each phase (all right-hand sides): [0] P2P, [1] P2M, [2] M2M,
 * [3] M2L, [4] L2L, [5] L2P, [6] whole evaluate (P2P overlaps the far field). */
FMMB_API int fmmb_get_timings(fmmb_plan* plan, float* ms7);

/* Overlap of the near field with the far field (default on).  With on = 0
 * the near field runs on the plan's stream between the far-field phases, so
 * that fmmb_get_timings gives each phase's time with the GPU to itself, as the
 * reference's per-routine timers do for its serial phases (tfmm[],
 * fmm/alloc.cxx:121); the results are the same.  Captured evaluates are
 * rebuilt. */
FMMB_API int fmmb_set_overlap(fmmb_plan* plan, int on);

/* Counts of the current geometry: [0] ni, [1] nj, [2] target leaves,
 * [3] source leaves, [4] P2P pairs (sum over near-field leaf pairs of
 * ni*nj), [5] M2L box pairs, [6] lmax, [7] kernel launches of the last
 * evaluate. */
FMMB_API int fmmb_get_stats(fmmb_plan* plan, long long* out8);

/* Wall times (ms) of the last fmmb_set_geometry: [0] the octree build on the
 * GPU (keys, radix sort, levels, lists; it synchronises between levels),
 * [1] the whole call (tree, interaction tiles and work lists built on the
 * host, operator images, buffers). */
FMMB_API int fmmb_get_setup_times(fmmb_plan* plan, double* ms2);

FMMB_API const char* fmmb_last_error(void);

#ifdef __cplusplus
}
#endif
#endif /* FMMB_H */

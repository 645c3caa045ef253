// CPU restatement of the reference FMM (test infrastructure only).
//
// This is the oracle the GPU library is checked against.  It follows the
// reference's algorithm step by step (each function in fmm_oracle.cpp cites the
// reference file:line it restates) but takes the expansion order at run time
// and keeps every level's expansions so that each phase can be compared.
// Only tests/, __graft_entry__.smoke() and bench.py's CPU baseline load it.
#ifndef FMM_ORACLE_H
#define FMM_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  int p;              // expansion order (the reference's mp = p+1)
  int lmax;           // octree depth (leaf level)
  int neq;            // 0 Laplace G, 1 Gni, 2 Gnj (reference fmm/fmm.cxx:29 numbering)
  int ref_semantics;  // 1: reference arithmetic (float tables, float pi, eps in rho,
                      //    float output accumulation); 0: accurate FP64 semantics
  double eps2;        // P2P/direct softening added to r^2 (reference: 1e-6f)
  int exclude_self;   // skip pairs with r^2 == 0 (accurate mode)
  float xmin, ymin, zmin, rd;  // root box
} oracle_config;

// Full FMM.  Inputs unsorted (caller order); outputs in caller order, FP64.
// Target normals (tn*) are used by neq 1, source normals (sn*) by neq 2.
// grad (3 arrays) is filled for neq 0 only; pass NULLs otherwise.
int oracle_fmm(const oracle_config* cfg, int ni, int nj,
               const float* tx, const float* ty, const float* tz,
               const float* tnx, const float* tny, const float* tnz,
               const float* sx, const float* sy, const float* sz,
               const float* snx, const float* sny, const float* snz, const float* q,
               double* pot, double* gx, double* gy, double* gz);

// Records of the last oracle_fmm call (sizes first, then copies).
//   kind 0 perm_i, 1 perm_j (sorted position -> caller index)
//   kind 2 target box keys, all levels lmax..2 concatenated (reference nfi)
//   kind 3 source box keys (reference nfj); kind 4/5 level counts [lmax+1]
//   kind 6/7 leaf ranges (first,last) pairs for targets/sources
//   kind 8 list stream [lev, mode, nbox_i, nbox_j, counts..., entries...] per list
long oracle_record_size(int kind);
int oracle_record_copy(int kind, int* dst);
// Expansions of the last call: which 0 = multipoles (source boxes, all levels,
// reference order), 1 = locals (target boxes, all levels).  Each box holds
// (p+1)(p+2)/2 complex coefficients (n, m>=0 at n(n+1)/2+m) as (re, im).
long oracle_expansion_size(int which);
int oracle_expansion_copy(int which, double* dst);

// FP64 direct sum over all pairs (restates kernel/G_dir.cxx:6-30,
// kernel/Gni_dir.cxx:6-21, kernel/Gnj_dir.cxx:6-21), with explicit softening
// and self-exclusion.  coef_ref_pi: 1 uses the reference's single-precision pi
// in 1/(4 pi), 0 uses the exact value.  Targets [i0, i1) only.
int oracle_direct(int neq, double eps2, int exclude_self, int coef_ref_pi,
                  int ni, int nj, int i0, int i1,
                  const float* tx, const float* ty, const float* tz,
                  const float* tnx, const float* tny, const float* tnz,
                  const float* sx, const float* sy, const float* sz,
                  const float* snx, const float* sny, const float* snz, const float* q,
                  double* pot, double* gx, double* gy, double* gz);

#ifdef __cplusplus
}
#endif
#endif

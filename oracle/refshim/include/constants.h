// Build shim for compiling the reference's own CPU sources (test infrastructure).
//
// The reference's hot-path translation units (fmm/*.cxx, kernel/*.cxx, sort/*.cxx)
// all begin with `#include "../include/constants.h"`.  oracle/Makefile compiles
// each of those files from standard input with the working directory set to
// oracle/refshim/src, so that this header is the one they see.  It declares the
// same configuration names and global scalars as the reference's
// include/constants.h:11-101 (an interface the reference's sources need,
// restated here), with two differences:
//   * the expansion order `mp` comes from -DREF_MP=<p+1> so one build recipe
//     produces a library per order (the reference fixes mp=9 at compile time);
//   * ngpu comes from -DREF_NGPU (default 0: the CPU path, alloc() skips the
//     GPU staging buffers of fmm/alloc.cxx:85-118; 1 for the build whose
//     near field goes through the reference's p2pgpu_ callers).
// Nothing here computes anything on the FMM path.
#ifndef ORACLE_REFSHIM_CONSTANTS_H
#define ORACLE_REFSHIM_CONSTANTS_H

#include <cassert>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <sys/time.h>

#ifndef REF_MP
#error "compile with -DREF_MP=<expansion order + 1>"
#endif

const int mp      = REF_MP;      // degrees n = 0..mp-1 (order p = mp-1)
#ifndef REF_NGPU
#define REF_NGPU 0
#endif
const int ngpu    = REF_NGPU;    // 0: CPU-only build
const int mprint  = 0;
const int nwmax   = 50000;
const int npmax   = 4194304;     // only sizes host staging; raised for 1M-point runs
const int mpmax   = mp*mp;
const int mpsym   = mp*(mp+1)/2;
const int mpcmp   = mp;
const int nebm    = 189;         // max boxes in one interaction list
const int nrbm    = 512;         // relative-position table size (8^3)
const int nmpi    = 2;
const int nsplit  = 4;
const int mpim    = 500000;
const int nimax   = 300000;
const int njmax   = 200000;
const int nblok0  = 128;
const int nblok1  = 64;
const int nblok2  = 4;
const int ins     = 50;
#ifdef REF_NGL
const int ngl     = REF_NGL;     // Gauss points per triangle (the biobem geometry build sets it)
#else
const int ngl     = 3;
#endif
const float eps   = 1e-6;        // softening / angle guard, single precision like the reference
const float pi    = M_PI;        // single-precision pi, as the reference uses it

#ifdef MAIN
int ncheck, nbmax, nbne, nbnet, nbned, lmax, m2lrp2p, nsub, nwn, nwe, nch;
int nprocs, myrank, maxfour, maxwave, maxexp, nmax;
float mem, umem, xmin, ymin, zmin, rd;
double lambda, scale, tic, toc;
double get_time(void) {
  struct timeval tv;
  gettimeofday(&tv, 0);
  return (double)tv.tv_sec + tv.tv_usec * 1.0e-6;
}
#else
extern int ncheck, nbmax, nbne, nbnet, nbned, lmax, m2lrp2p, nsub, nwn, nwe, nch;
extern int nprocs, myrank, maxfour, maxwave, maxexp, nmax;
extern float mem, umem, xmin, ymin, zmin, rd;
extern double lambda, scale, tic, toc;
extern double get_time(void);
#endif

#endif

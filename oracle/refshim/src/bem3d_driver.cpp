// Driver of the reference's 6-node boundary-element geometry, built from the
// reference's sources by oracle/Makefile into oracle/_ref/bem3d_ref_ngl<n>
// (test infrastructure: its outputs are the golden fixtures of the mesh6
// tests, made by tests/golden/make_mesh6_golden.py).
//
// It runs the start of the reference's biobem driver (biobem/main.cxx:97-99:
// geometry(), gauss_trgl(), elm_geom()) and writes every array those build:
// the 6-node mesh (biobem/geometry.cxx:86-162: ptr, ntr, nne), the triangle
// quadrature (biobem/bem3d.cxx:9-246: xiq, etq, wq) and the element geometry
// (biobem/bem3d.cxx:325-542: are, hsg, p1..p6, vna, vta, vsa), plus the
// charges read with the mesh.  geometry() reads ../bio/data/sphere.* relative
// to the working directory, so the binary runs in the reference's biobem/.
//
//   bem3d_ref_ngl<n> <output file>
//
// Output: int32 nwe, nwn, nch, ngl; then float32 ptr[nwn][3], int32
// ntr[nwe][6], int32 nne[nwn][0..8], float32 xiq, etq, wq [ngl], are[nwe],
// hsg[nwe][ngl], p1..p6[nwe][ngl], vna, vta, vsa [nwn][3], xq, yq, zq, vq [nch].
#define MAIN
#include "../include/constants.h"
#include <arrays.h>
#undef MAIN

#include <cstdio>
#include <vector>

extern void geometry();
extern void gauss_trgl();
extern void elm_geom();

namespace {
template <typename T>
void put(FILE* f, const T* p, size_t n) {
  fwrite(p, sizeof(T), n, f);
}
}  // namespace

int main(int argc, char** argv) {
  if (argc < 2) {
    fprintf(stderr, "usage: %s <output file>\n", argv[0]);
    return 2;
  }
  const int n = 100000;  // capacity of every per-node / per-element array
  xq = new float[n];
  yq = new float[n];
  zq = new float[n];
  vq = new float[n];
  face = new int[3 * n];
  vert = new float[3 * n];
  xvert = new float[n][6];
  yvert = new float[n][6];
  zvert = new float[n][6];
  ptr = new float[n][3];
  ntr = new int[n][6];
  nne = new int[n][20];
  vna = new float[n][3];
  vta = new float[n][3];
  vsa = new float[n][3];
  p1 = new float[n][13];
  p2 = new float[n][13];
  p3 = new float[n][13];
  p4 = new float[n][13];
  p5 = new float[n][13];
  p6 = new float[n][13];
  hsg = new float[n][13];
  are = new float[n];
  crv = new float[n];
  xiq = new float[20];
  etq = new float[20];
  wq = new float[20];

  geometry();
  gauss_trgl();
  elm_geom();

  FILE* f = fopen(argv[1], "wb");
  if (!f) return 1;
  const int hdr[4] = {nwe, nwn, nch, ngl};
  put(f, hdr, 4);
  put(f, &ptr[0][0], (size_t)nwn * 3);
  put(f, &ntr[0][0], (size_t)nwe * 6);
  for (int i = 0; i < nwn; i++) put(f, &nne[i][0], 9);
  put(f, xiq, ngl);
  put(f, etq, ngl);
  put(f, wq, ngl);
  put(f, are, nwe);
  float(*tabs[7])[13] = {hsg, p1, p2, p3, p4, p5, p6};
  for (auto* t : tabs)
    for (int i = 0; i < nwe; i++) put(f, &t[i][0], ngl);
  put(f, &vna[0][0], (size_t)nwn * 3);
  put(f, &vta[0][0], (size_t)nwn * 3);
  put(f, &vsa[0][0], (size_t)nwn * 3);
  put(f, xq, nch);
  put(f, yq, nch);
  put(f, zq, nch);
  put(f, vq, nch);
  fclose(f);
  return 0;
}

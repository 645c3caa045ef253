// Test driver for old_fmm_bem_b200/compat/fmm_compat.cpp, shaped like the
// reference's test/test.cxx: it owns the global particle arrays, calls the
// reference entry points fmm(ni, nj, neq) and G_dir/Gni_dir/Gnj_dir, and
// writes the outputs.  Usage: compat_driver <dir> <n> <lmax> <p> [lambda]
//   reads  <dir>/in.bin  = t(3n) tn(3n) s(3n) sn(3n) q(n) float32
//   writes <dir>/out.bin = v0(n) g0(3n) v1(n) v2(n) d0(n) d1(n) d2(n)
//                          [v10(n) d10(n) with lambda: fmm(n, n, 10), Helmholtz_G_dir] float32
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

float *xi, *yi, *zi, *gxi, *gyi, *gzi, *vi;
float *xj, *yj, *zj, *gxj, *gyj, *gzj, *vj;
int lmax;
float xmin, ymin, zmin, rd;
double lambda;

void fmm(int, int, int);
void G_dir(int, int, int, int);
void Gni_dir(int, int, int, int);
void Gnj_dir(int, int, int, int);
void Helmholtz_G_dir(int, int, int, int);
extern "C" void fmmb_compat_set_order(int);

int main(int argc, char** argv) {
  if (argc < 5) return 2;
  const std::string dir = argv[1];
  const int n = std::atoi(argv[2]);
  lmax = std::atoi(argv[3]);
  fmmb_compat_set_order(std::atoi(argv[4]));
  std::vector<float> in((size_t)13 * n);
  FILE* f = std::fopen((dir + "/in.bin").c_str(), "rb");
  if (!f || std::fread(in.data(), sizeof(float), in.size(), f) != in.size()) return 3;
  std::fclose(f);
  std::vector<float> T(in.begin(), in.begin() + 3 * n), TN(in.begin() + 3 * n, in.begin() + 6 * n),
      S(in.begin() + 6 * n, in.begin() + 9 * n), SN(in.begin() + 9 * n, in.begin() + 12 * n),
      Q(in.begin() + 12 * n, in.end());
  std::vector<float> a(7 * (size_t)n), b(7 * (size_t)n);
  xi = a.data(); yi = xi + n; zi = yi + n; gxi = zi + n; gyi = gxi + n; gzi = gyi + n; vi = gzi + n;
  xj = b.data(); yj = xj + n; zj = yj + n; gxj = zj + n; gyj = gxj + n; gzj = gyj + n; vj = gzj + n;
  auto load = [&](bool normals_i) {
    for (int k = 0; k < n; k++) {
      xi[k] = T[k]; yi[k] = T[n + k]; zi[k] = T[2 * n + k];
      gxi[k] = normals_i ? TN[k] : 0.f; gyi[k] = normals_i ? TN[n + k] : 0.f; gzi[k] = normals_i ? TN[2 * n + k] : 0.f;
      xj[k] = S[k]; yj[k] = S[n + k]; zj[k] = S[2 * n + k];
      gxj[k] = SN[k]; gyj[k] = SN[n + k]; gzj[k] = SN[2 * n + k];
      vj[k] = Q[k];
      vi[k] = 0.f;
    }
  };
  xmin = ymin = zmin = 0.f;
  rd = 1.f;
  std::vector<float> out;
  load(false);
  fmm(n, n, 0);
  out.insert(out.end(), vi, vi + n);
  out.insert(out.end(), gxi, gxi + n);
  out.insert(out.end(), gyi, gyi + n);
  out.insert(out.end(), gzi, gzi + n);
  load(true);
  fmm(n, n, 1);
  out.insert(out.end(), vi, vi + n);
  load(false);
  fmm(n, n, 2);
  out.insert(out.end(), vi, vi + n);
  load(false);
  G_dir(0, n - 1, 0, n - 1);
  out.insert(out.end(), vi, vi + n);
  load(true);
  Gni_dir(0, n - 1, 0, n - 1);
  out.insert(out.end(), vi, vi + n);
  load(false);
  Gnj_dir(0, n - 1, 0, n - 1);
  out.insert(out.end(), vi, vi + n);
  if (argc > 5) {  // Yukawa
    lambda = std::atof(argv[5]);
    load(false);
    fmm(n, n, 10);
    out.insert(out.end(), vi, vi + n);
    load(false);
    Helmholtz_G_dir(0, n - 1, 0, n - 1);
    out.insert(out.end(), vi, vi + n);
  }
  f = std::fopen((dir + "/out.bin").c_str(), "wb");
  if (!f) return 4;
  std::fwrite(out.data(), sizeof(float), out.size(), f);
  std::fclose(f);
  return 0;
}

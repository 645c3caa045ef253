// fmmb_direct_static: the direct O(ni*nj) sum of include/fmmb.h with float
// outputs, run without a plan and without allocating anything.
//
// The sum is split over sources so that small target sets still fill the
// GPU: block (bx, by) sums the 128 targets bx*128.. over the source chunk by
// in FP64 and writes its partial sums to a scratch array; a second kernel adds
// the nsplit partials of each target in split order (deterministic) and rounds
// to float.  The scratch is the file-scope device array g_direct_scratch
// (FMMB_STATIC_SCRATCH_BYTES), so the entry point calls no cudaMalloc or
// cudaFree and no allocating library routine.
//
// * Set-up: the first call on each device (with that device current) looks
//   the array's address up with cudaGetSymbolAddress, which may load the
//   module; make that first call before any stream capture.  Later calls
//   reuse the address.
// * Every call on a device shares the one array and it keeps the last call's
//   contents.  Each partial is written before it is read, so nothing needs
//   clearing; calls that overlap on the GPU (two streams, two threads) race on
//   the array and must be ordered by the caller.
// * Limit: nsplit * ncomp * ni doubles must fit, ncomp = 4 for Laplace G with
//   a gradient and 1 otherwise; ncomp * ni above the array's capacity is
//   rejected with FMMB_ERR_CAPACITY before any GPU work.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <mutex>
#include <string>

#include "internal.h"
#include "kernels.h"

namespace fmmb {
namespace {

constexpr size_t kScratchDoubles = FMMB_STATIC_SCRATCH_BYTES / sizeof(double);
constexpr int kMaxDevices = 64;
constexpr int kBlock = 128;

static __device__ __align__(256) double g_direct_scratch[kScratchDoubles];

std::mutex g_mu;
double* g_scratch_ptr[kMaxDevices] = {};

double* scratch_for_current_device() {
  int dev = 0;
  FMMB_CUDA(cudaGetDevice(&dev));
  FMMB_REQUIRE(dev >= 0 && dev < kMaxDevices, FMMB_ERR_ARG, "device ordinal out of range");
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_scratch_ptr[dev]) {
    void* p = nullptr;
    FMMB_CUDA(cudaGetSymbolAddress(&p, g_direct_scratch));
    g_scratch_ptr[dev] = static_cast<double*>(p);
  }
  return g_scratch_ptr[dev];
}

// Device memory of the current device, or managed memory: the only memory
// the kernels here may touch (another GPU's allocation would be a peer access
// the caller never enabled, a fault instead of an argument error).
bool on_device(const void* p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  if (a.type == cudaMemoryTypeManaged) return true;
  if (a.type != cudaMemoryTypeDevice) return false;
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.device == dev;
}

struct Soa {
  const float *x, *y, *z, *nx, *ny, *nz;
};

// Partial sums of targets [bx*128, +128) over sources [by*chunk, +chunk):
// part[(by*ncomp + c)*ni + i], c = 0 potential, 1..3 gradient.
template <int KER>
__global__ void __launch_bounds__(kBlock) direct_partial(int ni, int nj, int chunk, int ncomp, Soa t, Soa s,
                                                         const float* __restrict__ q, Sem sem,
                                                         double* __restrict__ part) {
  __shared__ float px[kBlock], py[kBlock], pz[kBlock], pq[kBlock], pn[3][kBlock];
  const int i = blockIdx.x * kBlock + threadIdx.x;
  const bool act = i < ni;
  const float xi = act ? t.x[i] : 0.f, yi = act ? t.y[i] : 0.f, zi = act ? t.z[i] : 0.f;
  float nxi = 0.f, nyi = 0.f, nzi = 0.f;
  if (KER == FMMB_LAPLACE_GNI && act) {
    nxi = t.nx[i];
    nyi = t.ny[i];
    nzi = t.nz[i];
  }
  const int j_begin = blockIdx.y * chunk;
  const int j_end = min(nj, j_begin + chunk);
  double p = 0, fx = 0, fy = 0, fz = 0;
  for (int j0 = j_begin; j0 < j_end; j0 += kBlock) {
    __syncthreads();
    const int j = j0 + threadIdx.x;
    if (j < j_end) {
      px[threadIdx.x] = s.x[j];
      py[threadIdx.x] = s.y[j];
      pz[threadIdx.x] = s.z[j];
      pq[threadIdx.x] = q[j];
      if (KER == FMMB_LAPLACE_GNJ) {
        pn[0][threadIdx.x] = s.nx[j];
        pn[1][threadIdx.x] = s.ny[j];
        pn[2][threadIdx.x] = s.nz[j];
      }
    }
    __syncthreads();
    const int nl = min(kBlock, j_end - j0);
    for (int jj = 0; jj < nl; jj++) {
      double dx, dy, dz;
      if (sem.ref) {  // the reference subtracts in float (kernel/G_dir.cxx:13-15)
        dx = (double)__fsub_rn(xi, px[jj]);
        dy = (double)__fsub_rn(yi, py[jj]);
        dz = (double)__fsub_rn(zi, pz[jj]);
      } else {
        dx = (double)xi - (double)px[jj];
        dy = (double)yi - (double)py[jj];
        dz = (double)zi - (double)pz[jj];
      }
      if (sem.excl_self && dx == 0.0 && dy == 0.0 && dz == 0.0) continue;
      const double r2 = dx * dx + dy * dy + dz * dz + sem.eps2;
      const double rinv = 1.0 / sqrt(r2);
      const double qr = sem.coef * (double)pq[jj] * rinv;
      if (KER == FMMB_LAPLACE_G) {
        p += qr;
        const double qr3 = qr * rinv * rinv;
        fx -= dx * qr3;
        fy -= dy * qr3;
        fz -= dz * qr3;
      } else if (KER == FMMB_LAPLACE_GNI) {
        p += (dx * nxi + dy * nyi + dz * nzi) * qr * rinv * rinv;
      } else {
        p += (dx * pn[0][jj] + dy * pn[1][jj] + dz * pn[2][jj]) * qr * rinv * rinv;
      }
    }
  }
  if (act) {
    double* out = part + (size_t)blockIdx.y * ncomp * ni;
    out[i] = p;
    if (ncomp == 4) {
      out[ni + i] = fx;
      out[2 * (size_t)ni + i] = fy;
      out[3 * (size_t)ni + i] = fz;
    }
  }
}

// pot[i] (and grad[c*ni + i]) = float(sum over splits in order).
__global__ void direct_finish(int ni, int nsplit, int ncomp, const double* __restrict__ part, float* __restrict__ pot,
                              float* __restrict__ grad) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ni) return;
  for (int c = 0; c < ncomp; c++) {
    double a = 0;
    for (int y = 0; y < nsplit; y++) a += part[((size_t)y * ncomp + c) * ni + i];
    if (c == 0)
      pot[i] = (float)a;
    else
      grad[(size_t)(c - 1) * ni + i] = (float)a;
  }
}

}  // namespace
}  // namespace fmmb

using namespace fmmb;

extern "C" FMMB_API int fmmb_direct_static(const fmmb_config* cfg, int ni, const float* tx, const float* ty,
                                           const float* tz, const float* tnx, const float* tny, const float* tnz,
                                           int nj, const float* sx, const float* sy, const float* sz,
                                           const float* snx, const float* sny, const float* snz, const float* q,
                                           float* pot, float* grad, void* stream) {
  try {
    FMMB_REQUIRE(cfg, FMMB_ERR_ARG, "null config");
    const int ker = cfg->kernel;
    FMMB_REQUIRE(ker == FMMB_LAPLACE_G || ker == FMMB_LAPLACE_GNI || ker == FMMB_LAPLACE_GNJ, FMMB_ERR_ARG,
                 "kernel must be FMMB_LAPLACE_G, _GNI or _GNJ");
    FMMB_REQUIRE(cfg->semantics == FMMB_SEM_REFERENCE || cfg->semantics == FMMB_SEM_ACCURATE, FMMB_ERR_ARG,
                 "unknown semantics");
    FMMB_REQUIRE(cfg->eps2 >= 0.0, FMMB_ERR_ARG, "eps2 must be >= 0");
    FMMB_REQUIRE(ni >= 0 && nj >= 0, FMMB_ERR_ARG, "negative size");
    const int ncomp = (ker == FMMB_LAPLACE_G && grad) ? 4 : 1;
    FMMB_REQUIRE((size_t)ncomp * (size_t)ni <= kScratchDoubles, FMMB_ERR_CAPACITY,
                 "fmmb_direct_static: " + std::to_string(ncomp) + " x ni = " + std::to_string((size_t)ncomp * ni) +
                     " partial sums exceed the static scratch of " + std::to_string(kScratchDoubles) +
                     " doubles (FMMB_STATIC_SCRATCH_BYTES)");
    if (ni == 0) return FMMB_OK;
    FMMB_REQUIRE(tx && ty && tz && pot, FMMB_ERR_ARG, "null target coordinates or output");
    FMMB_REQUIRE(nj == 0 || (sx && sy && sz && q), FMMB_ERR_ARG, "null source coordinates or charges");
    FMMB_REQUIRE(ker != FMMB_LAPLACE_GNI || (tnx && tny && tnz), FMMB_ERR_ARG, "Gni needs target normals");
    FMMB_REQUIRE(ker != FMMB_LAPLACE_GNJ || nj == 0 || (snx && sny && snz), FMMB_ERR_ARG,
                 "Gnj needs source normals");
    const void* dev_ptrs[] = {tx, ty, tz, pot, q, grad, tnx, tny, tnz, sx, sy, sz, snx, sny, snz};
    for (const void* p : dev_ptrs)
      FMMB_REQUIRE(!p || on_device(p), FMMB_ERR_ARG, "fmmb_direct_static takes device memory of the current device (or managed memory) only");

    double* part = scratch_for_current_device();
    const bool ref = cfg->semantics == FMMB_SEM_REFERENCE;
    Sem sem{};
    sem.eps2 = ref ? (double)1e-6f : cfg->eps2;
    sem.coef = ref ? 0.25 / (double)(float)M_PI : 0.25 / M_PI;
    sem.ref = ref ? 1 : 0;
    sem.excl_self = (!ref && cfg->exclude_self) ? 1 : 0;

    // Split the sources until about four blocks per SM are busy, within the
    // scratch capacity and the grid's y limit.
    int sms = 148;
    {
      int dev = 0;
      FMMB_CUDA(cudaGetDevice(&dev));
      FMMB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    }
    const int tblocks = (ni + kBlock - 1) / kBlock;
    long long nsplit = (4LL * sms + tblocks - 1) / tblocks;
    nsplit = std::min<long long>(nsplit, std::max(1, (nj + kBlock - 1) / kBlock));
    nsplit = std::min<long long>(nsplit, (long long)(kScratchDoubles / ((size_t)ncomp * ni)));
    nsplit = std::max<long long>(1, std::min<long long>(nsplit, 65535));
    const int chunk = std::max(1, (int)((nj + nsplit - 1) / nsplit));
    nsplit = std::max(1, (nj + chunk - 1) / chunk);

    cudaStream_t st = (cudaStream_t)stream;
    const Soa t{tx, ty, tz, tnx, tny, tnz}, s{sx, sy, sz, snx, sny, snz};
    const dim3 grid(tblocks, (unsigned)nsplit);
    if (ker == FMMB_LAPLACE_G)
      direct_partial<FMMB_LAPLACE_G><<<grid, kBlock, 0, st>>>(ni, nj, chunk, ncomp, t, s, q, sem, part);
    else if (ker == FMMB_LAPLACE_GNI)
      direct_partial<FMMB_LAPLACE_GNI><<<grid, kBlock, 0, st>>>(ni, nj, chunk, ncomp, t, s, q, sem, part);
    else
      direct_partial<FMMB_LAPLACE_GNJ><<<grid, kBlock, 0, st>>>(ni, nj, chunk, ncomp, t, s, q, sem, part);
    FMMB_CHECK_LAUNCH();
    direct_finish<<<(ni + 255) / 256, 256, 0, st>>>(ni, (int)nsplit, ncomp, part, pot, grad);
    FMMB_CHECK_LAUNCH();
    return FMMB_OK;
  } catch (const Error& e) {
    set_error(e.msg);
    return e.code;
  } catch (const std::exception& e) {
    set_error(e.what());
    return FMMB_ERR_ARG;
  }
}

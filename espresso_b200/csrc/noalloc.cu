// Allocation-free variant of the k-space error estimate.
//
// Who needs it: host programs that must not allocate device memory once
// they are running.  Examples are simulation engines that hand all GPU memory
// to their own pool at start-up and forbid later cudaMalloc/cudaFree, and
// latency-critical loops that cannot afford the implicit device-wide
// synchronisation cudaMalloc/cudaFree may perform.  p3mx_error_estimate
// creates a temporary engine (stream and device buffers) per call;
// p3mx_error_estimate_noalloc computes the same two numbers without any
// allocation: the per-block partial sums of the k-space error live in the
// fixed file-scope array below.
//
// Costs and rules of the shared array:
//  * it is 4097 doubles (about 32 KiB) and every GPU that loads libp3mx.so
//    holds it until the process exits;
//  * a mesh may have at most kNoAllocMaxPoints = 4096 * 16384 points
//    (e.g. 406^3); larger meshes are rejected with P3MX_EDOMAIN;
//  * every call reuses the same array and leaves its contents behind; each
//    call overwrites every slot it reads, so nothing has to start at zero;
//  * calls whose kernels overlap on the GPU (different streams or threads
//    at the same time) race on the array: serialise them;
//  * every call looks up the array's device address on the current device
//    (cudaGetSymbolAddress: no allocation), so the address cannot go stale
//    after a cudaDeviceReset; the first call on a device may load the
//    library's device code, so make that first call before any stream
//    capture on the device;
//  * each call waits for its result (device-to-host copy of one double and a
//    stream synchronisation).
#include "../../include/p3mx.h"
#include "p3m_kernels.cuh"

#include <cmath>
#include <cstdio>

namespace p3mx {
namespace {

constexpr int kNoAllocPartials = 4096;                    // one partial sum per CTA
constexpr long long kNoAllocPointsPerBlock = 256LL * 64;  // k-points per CTA
constexpr long long kNoAllocMaxPoints = kNoAllocPartials * kNoAllocPointsPerBlock;

// slots [0, nblk): partial sums of the current call; slot kNoAllocPartials:
// the total
static __device__ __align__(256) double g_noalloc_scratch[kNoAllocPartials + 1];

// Fixed-order sum of the first nblk partials into the last slot
// (deterministic: strided per-thread sums, then a fixed tree).
__global__ void k_noalloc_sum_partials(int nblk) {
  __shared__ double red[256];
  double s = 0.0;
  for (int b = threadIdx.x; b < nblk; b += blockDim.x)
    s += g_noalloc_scratch[b];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w)
      red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0)
    g_noalloc_scratch[kNoAllocPartials] = red[0];
}

// Device address of the array on the current device, looked up on every
// call.
cudaError_t noalloc_scratch(double **out) {
  double *ptr = nullptr;
  cudaError_t const e = cudaGetSymbolAddress(reinterpret_cast<void **>(&ptr), g_noalloc_scratch);
  if (e != cudaSuccess)
    return e;
  *out = ptr;
  return cudaSuccess;
}

void noalloc_msg(char *buf, size_t len, const char *text) {
  if (buf && len)
    std::snprintf(buf, len, "%s", text);
}

} // namespace
} // namespace p3mx

extern "C" int p3mx_error_estimate_noalloc(const int *mesh, int cao, int n_c_part,
                                           double sum_q2, double alpha_L, double r_cut_iL,
                                           const double *box, double prefactor,
                                           double *rs_err, double *ks_err, void *stream,
                                           char *errbuf, size_t errbuf_len) {
  using namespace p3mx;
  noalloc_msg(errbuf, errbuf_len, "");
  if (!mesh || !box) {
    noalloc_msg(errbuf, errbuf_len, "mesh and box must not be NULL");
    return P3MX_EHANDLE;
  }
  if (mesh[0] < 1 || mesh[1] < 1 || mesh[2] < 1) {
    noalloc_msg(errbuf, errbuf_len, "Parameter 'mesh' must be > 0");
    return P3MX_EDOMAIN;
  }
  if (cao < 1 || cao > 7) {
    noalloc_msg(errbuf, errbuf_len, "Parameter 'cao' must be >= 1 and <= 7");
    return P3MX_EDOMAIN;
  }
  if (n_c_part < 1 || !(alpha_L > 0.0) || !(r_cut_iL > 0.0)) {
    noalloc_msg(errbuf, errbuf_len, "n_c_part, alpha_L and r_cut_iL must be > 0");
    return P3MX_EDOMAIN;
  }
  long long const points = static_cast<long long>(mesh[0]) * mesh[1] * mesh[2];
  if (points > kNoAllocMaxPoints) {
    char text[200];
    std::snprintf(text, sizeof(text),
                  "mesh of %lld points exceeds the allocation-free maximum of %lld points "
                  "(fixed scratch of %d partial sums); use p3mx_error_estimate",
                  points, kNoAllocMaxPoints, kNoAllocPartials);
    noalloc_msg(errbuf, errbuf_len, text);
    return P3MX_EDOMAIN;
  }
  double *scratch = nullptr;
  cudaError_t e = noalloc_scratch(&scratch);
  if (e != cudaSuccess) {
    noalloc_msg(errbuf, errbuf_len, cudaGetErrorString(e));
    return P3MX_ECUDA;
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  int const nblk = static_cast<int>((points + kNoAllocPointsPerBlock - 1) / kNoAllocPointsPerBlock);
  k_ks_error<<<nblk, 256, 0, st>>>(mesh[0], mesh[1], mesh[2], cao, alpha_L, scratch);
  k_noalloc_sum_partials<<<1, 256, 0, st>>>(nblk);
  double he_q = 0.0;
  e = cudaGetLastError();
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(&he_q, scratch + kNoAllocPartials, sizeof(double), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess)
    e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    noalloc_msg(errbuf, errbuf_len, cudaGetErrorString(e));
    return P3MX_ECUDA;
  }
  // p3m_k_space_error and p3m_real_space_error (p3m.cpp:187-243)
  if (ks_err)
    *ks_err = 2. * prefactor * sum_q2 * std::sqrt(he_q / static_cast<double>(n_c_part)) /
              (box[1] * box[2]);
  if (rs_err) {
    double const V = box[0] * box[1] * box[2];
    *rs_err = (2. * prefactor * sum_q2 * std::exp(-(r_cut_iL * alpha_L) * (r_cut_iL * alpha_L))) /
              std::sqrt(static_cast<double>(n_c_part) * r_cut_iL * box[0] * V);
  }
  return P3MX_OK;
}

// Shared definitions of the p3mx CUDA engine (sm_100a).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <stdexcept>
#include <string>

namespace p3mx {

constexpr double kPi = 3.14159265358979323846;

// Status exception used inside the library; the C ABI converts it to a
// return code plus message (no exception crosses the ABI).
struct Error : std::runtime_error {
  int code;
  Error(int c, std::string const &m) : std::runtime_error(m), code(c) {}
};

#define P3MX_CUDA(call)                                                       \
  do {                                                                        \
    cudaError_t err_ = (call);                                                \
    if (err_ != cudaSuccess)                                                  \
      throw ::p3mx::Error(3, std::string("CUDA error: ") +                    \
                                 cudaGetErrorString(err_) + " at " +          \
                                 __FILE__ + ":" + std::to_string(__LINE__));  \
  } while (0)

template <typename Real> struct CplxOf;
template <> struct CplxOf<float> { using type = float2; };
template <> struct CplxOf<double> { using type = double2; };

template <typename Real> struct Real4Of;
template <> struct Real4Of<float> { using type = float4; };
// 32-byte aligned four-double record
struct __align__(32) double4a {
  double x, y, z, w;
};
template <> struct Real4Of<double> { using type = double4a; };

template <typename C> __host__ __device__ inline C cmul(C a, C b) {
  return C{a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x};
}
template <typename C> __host__ __device__ inline C cadd(C a, C b) {
  return C{a.x + b.x, a.y + b.y};
}
template <typename C> __host__ __device__ inline C csub(C a, C b) {
  return C{a.x - b.x, a.y - b.y};
}
template <typename C> __host__ __device__ inline C cconj(C a) {
  return C{a.x, -a.y};
}

// Maximum number of radix stages of one FFT length.
constexpr int kMaxStages = 12;

// FFT plan of one axis length, stored in the replica descriptor.
struct AxisPlan {
  int n;
  int nstages;
  int radix[kMaxStages];
  int tw_off; // offset of exp(-2 pi i k / n), k < n, in the twiddle table
};

// Per-replica device descriptor (one system of the batch).
struct RepGeom {
  double box[3], box_i[3];
  double ai[3], ld_pos[3];
  double pos_shift;
  double alpha, r_cut, prefactor, epsilon, V;
  double sum_q2, sum_q; // set by the charge census
  int ld_ind[3];
  int mesh[3];
  int hp;  // padded length of the r2c axis (>= mesh[2]/2+1, multiple of 4)
  int cao;
  long long p0, np;  // particle range
  long long rm_off;  // real mesh offset (elements)
  long long bin_off; // corner key offset: bricks of brick^3 corners
  long long brk_off; // brick (sort key) offset
  int brick;         // brick edge (corner units) of the charge assignment
  int nbx, nby, nbz; // bricks per dimension
  long long km_off;  // complex half mesh offset (elements)
  AxisPlan plan[3];
  // short-range cell system
  int cg[3];
  double inv_cs[3];
  long long cell_off;
  double max_cut, skin, coulomb_cut;
  // Verlet list of this replica: neighbour k of particle p0+i at
  // nb[nb_off + k*np + i], capacity max_nb per particle
  long long nb_off;
  int max_nb;
};

// Batched global -> shared copy: each thread issues U loads before its
// stores, so U loads are in flight per thread.
template <int U, typename L, typename S>
__device__ inline void staged_copy(int total, L const &load, S const &store) {
  for (int e0 = threadIdx.x; e0 < total; e0 += U * blockDim.x) {
    decltype(load(0)) v[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      int const e = e0 + u * blockDim.x;
      if (e < total)
        v[u] = load(e);
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      int const e = e0 + u * blockDim.x;
      if (e < total)
        store(e, v[u]);
    }
  }
}

inline int ceil_div(long long a, long long b) {
  return static_cast<int>((a + b - 1) / b);
}

} // namespace p3mx

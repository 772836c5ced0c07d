// Shared definitions of the p3mx CUDA engine (sm_100a).
#pragma once

#include <cuda.h>
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
  long long re_off;  // field mesh offset (records of 4 values)
  int epad[3];       // field mesh extent: mesh plus high-side ghost layers
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
  int oct_on;   // cells sorted by octant (list build skips far octants)
  int oct_mult; // sort keys per cell: 8 when any replica sorts by octant, else 1
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

// ---- bulk-copy engine (TMA) helpers: cp.async.bulk global -> shared with
// completion on an mbarrier (transaction bytes); waits are bounded.
__device__ inline unsigned smem_u32(const void *p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}
__device__ inline void mbar_init(unsigned long long *bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
               : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
// Arrive (one of the barrier's expected arrivals) and add `bytes` to the
// transaction count of the current phase.
__device__ inline void mbar_arrive_expect_tx(unsigned long long *bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}
// Bulk copy of `bytes` (multiple of 16, both addresses 16-byte aligned).
__device__ inline void bulk_g2s(void *dst, const void *src, unsigned bytes,
                                unsigned long long *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
          "r"(smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}
// Tiled 3-d tensor copy global -> shared (TMA engine) of the box at
// coordinates (c0 innermost, c1, c2) of the tensor map, completing on the
// mbarrier; the shared destination is 128-byte aligned and c0 times the
// element size a multiple of 16 bytes.
__device__ inline void tma_load_3d(void *dst, const CUtensorMap *map, int c0, int c1, int c2,
                                   unsigned long long *bar) {
  asm volatile("cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
               " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_u32(dst)),
               "l"(reinterpret_cast<unsigned long long>(map)), "r"(c0), "r"(c1), "r"(c2),
               "r"(smem_u32(bar))
               : "memory");
}
// Acquire a tensor map that lives in global memory for the tensor proxy.
__device__ inline void tensormap_acquire(const CUtensorMap *map) {
  asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(
                   reinterpret_cast<unsigned long long>(map))
               : "memory");
}
// Wait until the phase with the given parity completes; false when the
// iteration limit ran out (the caller reports it and bails out).
__device__ inline bool mbar_wait(unsigned long long *bar, unsigned parity) {
  for (int it = 0; it < (1 << 22); ++it) {
    unsigned done = 0;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    if (done)
      return true;
  }
  return false;
}

inline int ceil_div(long long a, long long b) {
  return static_cast<int>((a + b - 1) / b);
}

} // namespace p3mx

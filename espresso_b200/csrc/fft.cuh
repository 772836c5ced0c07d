// Hand-written mixed-radix 3D FFT for the P3M mesh (sm_100a).
//
// Real mesh [M0][M1][M2] (z fastest) <-> complex half mesh [M0][M1][hp]
// (kz < M2/2+1 used, hp = padded row length).  Forward = exp(-i k x),
// backward = exp(+i k x), both unnormalised, as the reference's FFTW
// plans (fft/fft.cpp:682-696).  Each pass stages a tile of lines in shared
// memory and runs Stockham autosort stages of radix 4, 2 or a generic
// prime radix (Govindaraju et al. 2008 formulation); twiddles come from an
// FP64-computed table rounded to the working precision.
//
// The x pass is fused with the P3M k-space work that follows the forward
// transform: optimal influence function, ik-differentiation (three field
// components), k-space energy and pressure-tensor sums, and the three
// backward x transforms -- one HBM round trip instead of five.
#pragma once

#include "common.cuh"

namespace p3mx {

// Block work item of an FFT pass: replica, first item, item count.
struct Blk {
  int rep;
  int a;   // first line / x / y index
  int b;   // second index (kz tile start) or unused
  int pad;
};

// Shared-memory position of element i of a staged line: one pad slot per 16
// elements, so the stride-R accesses of the early Stockham stages (and the
// stride-16 transposed loads) fall into distinct banks.
__host__ __device__ inline int pix(int i) { return i + (i >> 4); }
// Line stride (elements) of staged lines of length n: padded length, odd so
// that consecutive lines start in different banks.
__host__ __device__ inline int line_ld(int n) { return (n + ((n - 1) >> 4)) | 1; }

// body(l, k) for l < nl, k < n over the block: lines shorter than the block
// run several at a time (one division per thread, not per element).
template <typename F> __device__ inline void for_lines(int nl, int n, F const &body) {
  int const per = blockDim.x / n;
  if (per > 0) {
    int const lq = threadIdx.x / n, k = threadIdx.x - lq * n;
    if (lq < per)
      for (int l = lq; l < nl; l += per)
        body(l, k);
  } else {
    for (int l = 0; l < nl; ++l)
      for (int k = threadIdx.x; k < n; k += blockDim.x)
        body(l, k);
  }
}

// Copy the twiddle table exp(-2 pi i k / n), k < n, of one axis to shared
// memory (caller synchronises).
template <typename C>
__device__ inline void load_twiddles(C *dst, const C *__restrict__ twtab, AxisPlan const &pl) {
  const C *src = twtab + pl.tw_off;
  for (int k = threadIdx.x; k < pl.n; k += blockDim.x)
    dst[k] = src[k];
}

template <typename C> __device__ inline C ld_tw(const C *__restrict__ tw, int k, bool inv) {
  C w = tw[k];
  if (inv)
    w.y = -w.y;
  return w;
}

// cos(2 pi k / 16) and sin(2 pi k / 16), k = 0..15 (exact constants of the
// sixteenth roots of unity: 1, cos(pi/8), sqrt(1/2), sin(pi/8), 0).
__host__ __device__ constexpr double cos16(int k) {
  constexpr double c1 = 0.92387953251128675613, c2 = 0.70710678118654752440,
                   c3 = 0.38268343236508977173;
  switch (k & 15) {
  case 0: return 1.0;
  case 1: return c1;
  case 2: return c2;
  case 3: return c3;
  case 4: return 0.0;
  case 5: return -c3;
  case 6: return -c2;
  case 7: return -c1;
  case 8: return -1.0;
  case 9: return -c1;
  case 10: return -c2;
  case 11: return -c3;
  case 12: return 0.0;
  case 13: return c3;
  case 14: return c2;
  default: return c1;
  }
}
__host__ __device__ constexpr double sin16(int k) { return cos16(k - 4); }

// In-register DFT of a power-of-two length R <= 16 (radix-2 decimation in
// time on top of the radix-4 kernel), constant twiddles.
template <typename C, int R> __device__ __forceinline__ void dft_pow2(C *v, bool inv) {
  using Real = decltype(v[0].x);
  if constexpr (R == 2) {
    C const a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
  } else if constexpr (R == 4) {
    C const s0 = cadd(v[0], v[2]), s1 = csub(v[0], v[2]);
    C const s2 = cadd(v[1], v[3]), s3 = csub(v[1], v[3]);
    C const s3r = inv ? C{-s3.y, s3.x} : C{s3.y, -s3.x};
    v[0] = cadd(s0, s2);
    v[2] = csub(s0, s2);
    v[1] = cadd(s1, s3r);
    v[3] = csub(s1, s3r);
  } else {
    constexpr int H = R / 2;
    C e[H], o[H];
#pragma unroll
    for (int i = 0; i < H; ++i) {
      e[i] = v[2 * i];
      o[i] = v[2 * i + 1];
    }
    dft_pow2<C, H>(e, inv);
    dft_pow2<C, H>(o, inv);
#pragma unroll
    for (int k = 0; k < H; ++k) {
      C t;
      if (k == 0) {
        t = o[0];
      } else if (2 * k == H) {
        // exp(-+ i pi/2) = -+i
        t = inv ? C{-o[k].y, o[k].x} : C{o[k].y, -o[k].x};
      } else {
        Real const wr = static_cast<Real>(cos16(k * (16 / R)));
        Real const ws = static_cast<Real>(sin16(k * (16 / R)));
        Real const wi = inv ? ws : -ws;
        t = C{o[k].x * wr - o[k].y * wi, o[k].x * wi + o[k].y * wr};
      }
      v[k] = cadd(e[k], t);
      v[k + H] = csub(e[k], t);
    }
  }
}

template <typename C, int R>
__device__ inline void dft_small(C *v, const C *__restrict__ tw, int n, bool inv) {
  if constexpr (R == 8 || R == 16) {
    dft_pow2<C, R>(v, inv);
  } else if constexpr (R == 2) {
    C const a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
  } else if constexpr (R == 4) {
    C const s0 = cadd(v[0], v[2]), s1 = csub(v[0], v[2]);
    C const s2 = cadd(v[1], v[3]), s3 = csub(v[1], v[3]);
    // forward: multiply s3 by -i; backward: by +i
    C const s3r = inv ? C{-s3.y, s3.x} : C{s3.y, -s3.x};
    v[0] = cadd(s0, s2);
    v[2] = csub(s0, s2);
    v[1] = cadd(s1, s3r);
    v[3] = csub(s1, s3r);
  } else {
    C out[R];
    int const step = n / R;
#pragma unroll
    for (int m = 0; m < R; ++m) {
      C acc = v[0];
#pragma unroll
      for (int r = 1; r < R; ++r) {
        int const e = (r * m) % R;
        acc = cadd(acc, cmul(v[r], ld_tw(tw, e * step, inv)));
      }
      out[m] = acc;
    }
#pragma unroll
    for (int m = 0; m < R; ++m)
      v[m] = out[m];
  }
}

// Generic (runtime) radix for primes beyond the templated set.
template <typename C>
__device__ inline void dft_dyn(C *v, int R, const C *__restrict__ tw, int n, bool inv) {
  C out[32];
  int const step = n / R;
  for (int m = 0; m < R; ++m) {
    C acc = v[0];
    for (int r = 1; r < R; ++r) {
      int const e = (r * m) % R;
      acc = cadd(acc, cmul(v[r], ld_tw(tw, e * step, inv)));
    }
    out[m] = acc;
  }
  for (int m = 0; m < R; ++m)
    v[m] = out[m];
}

// Quotient of small non-negative ints (< 2^24) by a runtime divisor via the
// FP32 reciprocal plus one correction step (replaces the ~20-instruction
// integer division in the FFT index maps).
__device__ inline int qdiv(int a, int b, float rb) {
  int q = __float2int_rz(__int2float_rn(a) * rb);
  int const r = a - q * b;
  q += (r >= b) - (r < 0);
  return q;
}

// One Stockham stage over `nlines` lines of length n held in shared memory
// with line stride ld (ld > n pads the lines against bank conflicts).
// Twiddle index r*jm*tstride < n, so no modulo is needed.
template <typename C, int R>
__device__ inline void fft_stage_t(const C *src, C *dst, int n, int ld, int nlines, int Ns,
                                   const C *__restrict__ tw, bool inv) {
  int const nb = n / R;
  int const total = nb * nlines;
  int const tstride = n / (Ns * R);
  float const rnb = 1.0f / static_cast<float>(nb);
  float const rNs = 1.0f / static_cast<float>(Ns);
  for (int t = threadIdx.x; t < total; t += blockDim.x) {
    int const line = qdiv(t, nb, rnb);
    int const j = t - line * nb;
    C const *s = src + line * ld;
    C *d = dst + line * ld;
    int const jq = qdiv(j, Ns, rNs);
    int const jm = j - jq * Ns;
    C v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      v[r] = s[pix(j + r * nb)];
      if (r > 0 && jm != 0)
        v[r] = cmul(v[r], ld_tw(tw, r * jm * tstride, inv));
    }
    dft_small<C, R>(v, tw, n, inv);
    int const base = jq * Ns * R + jm;
#pragma unroll
    for (int r = 0; r < R; ++r)
      d[pix(base + r * Ns)] = v[r];
  }
}

template <typename C>
__device__ inline void fft_stage_dyn(const C *src, C *dst, int n, int ld, int nlines, int Ns,
                                     int R, const C *__restrict__ tw, bool inv) {
  int const nb = n / R;
  int const total = nb * nlines;
  int const tstride = n / (Ns * R);
  for (int t = threadIdx.x; t < total; t += blockDim.x) {
    int const line = t / nb;
    int const j = t - line * nb;
    C const *s = src + line * ld;
    C *d = dst + line * ld;
    int const jm = j % Ns;
    C v[32];
    for (int r = 0; r < R; ++r) {
      v[r] = s[pix(j + r * nb)];
      if (r > 0 && jm != 0)
        v[r] = cmul(v[r], ld_tw(tw, r * jm * tstride, inv));
    }
    dft_dyn(v, R, tw, n, inv);
    int const base = (j / Ns) * Ns * R + jm;
    for (int r = 0; r < R; ++r)
      d[pix(base + r * Ns)] = v[r];
  }
}

// Power-of-two line length N = N1 * N2 (N1, N2 <= 16) in two register
// steps (n = t + N2 m, k = k1 + N1 k2):
//   step 1, item (line, t): Y[t][k1] = w_N^(t k1) * DFT_N1 over m of x[t + N2 m],
//           written in place at t + N2 k1;
//   step 2, item (line, k1): X[k1 + N1 k2] = DFT_N2 over t of Y[t][k1],
//           written to `b` in natural order.
// Strides are compile-time constants; the padded layout (pix) keeps both
// steps free of bank conflicts.  Returns b.
template <typename C, int N1, int N2>
__device__ C *fft_2step(C *a, C *b, int nlines, int ld, const C *__restrict__ tw, bool inv) {
  for (int it = threadIdx.x; it < nlines * N2; it += blockDim.x) {
    int const l = it / N2, t = it - l * N2;
    C *s = a + l * ld;
    C v[N1];
#pragma unroll
    for (int m = 0; m < N1; ++m)
      v[m] = s[pix(t + N2 * m)];
    dft_pow2<C, N1>(v, inv);
#pragma unroll
    for (int k1 = 1; k1 < N1; ++k1)
      v[k1] = cmul(v[k1], ld_tw(tw, t * k1, inv));
#pragma unroll
    for (int k1 = 0; k1 < N1; ++k1)
      s[pix(t + N2 * k1)] = v[k1];
  }
  __syncthreads();
  for (int it = threadIdx.x; it < nlines * N1; it += blockDim.x) {
    int const l = it / N1, k1 = it - l * N1;
    const C *s = a + l * ld;
    C *d = b + l * ld;
    C v[N2];
#pragma unroll
    for (int t = 0; t < N2; ++t)
      v[t] = s[pix(t + N2 * k1)];
    dft_pow2<C, N2>(v, inv);
#pragma unroll
    for (int k2 = 0; k2 < N2; ++k2)
      d[pix(k1 + N1 * k2)] = v[k2];
  }
  __syncthreads();
  return b;
}

// In-place form of fft_2step for nlines * 16 <= blockDim.x (one item per
// thread and step): step 2 reads its column into registers, the block
// synchronises, then every thread writes its outputs back to `a`.
template <typename C, int N1, int N2>
__device__ C *fft_2step_inplace(C *a, int nlines, int ld, const C *__restrict__ tw, bool inv) {
  int const it = threadIdx.x;
  if (it < nlines * N2) {
    int const l = it / N2, t = it - l * N2;
    C *s = a + l * ld;
    C v[N1];
#pragma unroll
    for (int m = 0; m < N1; ++m)
      v[m] = s[pix(t + N2 * m)];
    dft_pow2<C, N1>(v, inv);
#pragma unroll
    for (int k1 = 1; k1 < N1; ++k1)
      v[k1] = cmul(v[k1], ld_tw(tw, t * k1, inv));
#pragma unroll
    for (int k1 = 0; k1 < N1; ++k1)
      s[pix(t + N2 * k1)] = v[k1];
  }
  __syncthreads();
  bool const act = it < nlines * N1;
  int const l = it / N1, k1 = it - l * N1;
  C v[N2];
  if (act) {
    const C *s = a + l * ld;
#pragma unroll
    for (int t = 0; t < N2; ++t)
      v[t] = s[pix(t + N2 * k1)];
    dft_pow2<C, N2>(v, inv);
  }
  __syncthreads();
  if (act) {
    C *d = a + l * ld;
#pragma unroll
    for (int k2 = 0; k2 < N2; ++k2)
      d[pix(k1 + N1 * k2)] = v[k2];
  }
  __syncthreads();
  return a;
}

// True when lines of length n transform in place (fft_lines_inplace): n a
// power of two in 32..256 and nlines * 16 <= threads.
__host__ __device__ inline bool fft_inplace_ok(int n, int nlines, int threads) {
  return (n == 32 || n == 64 || n == 128 || n == 256) && nlines * 16 <= threads;
}

// In-place transform of nlines lines in `a` (requires fft_inplace_ok);
// returns a.  A separate function from fft_lines, so that kernels that never
// transform in place do not carry its code (and registers).
template <typename C>
__device__ C *fft_lines_inplace(C *a, int nlines, int ld, AxisPlan const &pl,
                                const C *__restrict__ tw, bool inv) {
  switch (pl.n) {
  case 32: return fft_2step_inplace<C, 16, 2>(a, nlines, ld, tw, inv);
  case 64: return fft_2step_inplace<C, 16, 4>(a, nlines, ld, tw, inv);
  case 128: return fft_2step_inplace<C, 16, 8>(a, nlines, ld, tw, inv);
  default: return fft_2step_inplace<C, 16, 16>(a, nlines, ld, tw, inv);
  }
}

// Full transform of nlines lines in `a` (scratch `b`; element i of line l at
// l*ld + pix(i)); tw = the axis twiddle table (shared memory).  Returns the
// buffer holding the result.  All threads of the block must call it.
template <typename C>
__device__ C *fft_lines(C *a, C *b, int nlines, int ld, AxisPlan const &pl,
                        const C *__restrict__ tw, bool inv) {
  int const n = pl.n;
  switch (n) {
  case 32: return fft_2step<C, 16, 2>(a, b, nlines, ld, tw, inv);
  case 64: return fft_2step<C, 16, 4>(a, b, nlines, ld, tw, inv);
  case 128: return fft_2step<C, 16, 8>(a, b, nlines, ld, tw, inv);
  case 256: return fft_2step<C, 16, 16>(a, b, nlines, ld, tw, inv);
  default: break;
  }
  int Ns = 1;
  C *src = a, *dst = b;
  for (int s = 0; s < pl.nstages; ++s) {
    int const R = pl.radix[s];
    switch (R) {
    case 2: fft_stage_t<C, 2>(src, dst, n, ld, nlines, Ns, tw, inv); break;
    case 3: fft_stage_t<C, 3>(src, dst, n, ld, nlines, Ns, tw, inv); break;
    case 4: fft_stage_t<C, 4>(src, dst, n, ld, nlines, Ns, tw, inv); break;
    case 8: fft_stage_t<C, 8>(src, dst, n, ld, nlines, Ns, tw, inv); break;
    case 16: fft_stage_t<C, 16>(src, dst, n, ld, nlines, Ns, tw, inv); break;
    case 5: fft_stage_t<C, 5>(src, dst, n, ld, nlines, Ns, tw, inv); break;
    case 7: fft_stage_t<C, 7>(src, dst, n, ld, nlines, Ns, tw, inv); break;
    default: fft_stage_dyn<C>(src, dst, n, ld, nlines, Ns, R, tw, inv); break;
    }
    __syncthreads();
    Ns *= R;
    C *t = src;
    src = dst;
    dst = t;
  }
  return src;
}

// Copy the contiguous global range [src, src + count) to shared memory with
// one bulk copy (TMA engine) when its 16-byte aligned superset fits in the
// `room` bytes at `area`.  Returns the shared-memory copy of src, or nullptr
// when the range does not fit (nothing copied; the decision is uniform over
// the block).  Called by all threads of the block; the copy has landed when
// it returns.  A wait that runs out sets *err and `failed` (the caller
// returns).  The aligned superset may reach up to 15 bytes past the range:
// the buffer behind src is allocated with that slack.
template <typename T>
__device__ inline const T *bulk_stage(const T *src, long long count, unsigned char *area,
                                      size_t room, unsigned long long *bar, int *err,
                                      bool &failed) {
  uintptr_t const g0 = reinterpret_cast<uintptr_t>(src) & ~uintptr_t(15);
  uintptr_t const g1 = (reinterpret_cast<uintptr_t>(src + count) + 15) & ~uintptr_t(15);
  unsigned const pad = (16u - (smem_u32(area) & 15u)) & 15u;
  size_t const bytes = g1 - g0;
  if (pad + bytes > room || bytes >= (1u << 20))
    return nullptr;
  unsigned char *dst = area + pad;
  if (threadIdx.x == 0) {
    mbar_init(bar, 1);
    mbar_arrive_expect_tx(bar, static_cast<unsigned>(bytes));
    bulk_g2s(dst, reinterpret_cast<const void *>(g0), static_cast<unsigned>(bytes), bar);
  }
  __syncthreads(); // barrier initialised before anyone waits on it
  bool const ok = mbar_wait(bar, 0);
  if (__syncthreads_or(!ok)) {
    if (threadIdx.x == 0) {
      atomicExch(err, 1);
      mbar_wait(bar, 0); // second bounded wait for the copy in flight
    }
    failed = true;
    return nullptr;
  }
  return reinterpret_cast<const T *>(dst + (reinterpret_cast<uintptr_t>(src) - g0));
}

// ---- pass z, forward: real lines -> complex half lines -----------------
// Two real lines per complex transform: Z = x0 + i x1, then
// X0[k] = (Z[k] + conj Z[n-k]) / 2 and X1[k] = -i (Z[k] - conj Z[n-k]) / 2.
// bk.b real lines per block (an odd last line is paired with zeros).
// Shared memory: 2 x ceil(bk.b/2) staged lines of line_ld(n), twiddles (n).
template <typename Real>
__global__ void __launch_bounds__(256, sizeof(Real) == 4 ? 4 : 2)
k_fft_z_fwd(const RepGeom *__restrict__ reps, const Blk *__restrict__ blks,
            const Real *__restrict__ rmesh, typename CplxOf<Real>::type *__restrict__ cmesh,
            const typename CplxOf<Real>::type *__restrict__ twtab, int *__restrict__ err) {
  using C = typename CplxOf<Real>::type;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Blk const bk = blks[blockIdx.x];
  RepGeom const &G = reps[bk.rep];
  int const n = G.mesh[2];
  int const ld = line_ld(n);
  int const nl = bk.b;          // real lines in this block
  int const np = (nl + 1) >> 1; // complex lines
  C *a = reinterpret_cast<C *>(smem_raw);
  C *b = a + np * ld;
  C *tw = b + np * ld;
  load_twiddles(tw, twtab, G.plan[2]);
  long long const line0 = bk.a;
  const Real *src = rmesh + G.rm_off + line0 * n;
  // the block's nl real lines are one contiguous range of the mesh: stage it
  // in b (the FFT scratch) with one bulk copy when it fits there
  __shared__ __align__(8) unsigned long long bar;
  bool failed = false;
  const Real *sv = bulk_stage(src, static_cast<long long>(nl) * n,
                              reinterpret_cast<unsigned char *>(b), np * ld * sizeof(C), &bar,
                              err, failed);
  if (failed)
    return;
  if (sv == nullptr)
    sv = src;
  // real line l, element k -> real or imaginary part of slot l/2
  Real *ar = reinterpret_cast<Real *>(a);
  // odd count: the last slot's imaginary part is line nl, all zeros
  for_lines(nl + (nl & 1), n, [&](int l, int k) {
    ar[2 * ((l >> 1) * ld + pix(k)) + (l & 1)] = (l < nl) ? sv[l * n + k] : Real(0);
  });
  __syncthreads();
  C *res = fft_lines<C>(a, b, np, ld, G.plan[2], tw, false);
  int const H = n / 2 + 1;
  int const hp = G.hp;
  for_lines(nl, hp, [&](int l, int k) {
    C v{Real(0), Real(0)};
    if (k < H) {
      C const z = res[(l >> 1) * ld + pix(k)];
      C const zc = res[(l >> 1) * ld + pix(k == 0 ? 0 : n - k)];
      if ((l & 1) == 0)
        v = C{Real(0.5) * (z.x + zc.x), Real(0.5) * (z.y - zc.y)};
      else
        v = C{Real(0.5) * (z.y + zc.y), Real(0.5) * (zc.x - z.x)};
    }
    cmesh[G.km_off + (line0 + l) * hp + k] = v;
  });
}

// ---- pass y (either direction, nf field arrays via blockIdx.y) ---------
// Shared memory: tile staged lines of line_ld(M1) (two sets unless the
// lines transform in place), twiddles (M1).
// INPL: every replica's lines transform in place (the host checks), so the
// instance carries none of the out-of-place transform's code or registers.
template <typename Real, bool INPL>
__global__ void __launch_bounds__(256, sizeof(Real) == 4 ? 4 : 2)
k_fft_y(const RepGeom *__restrict__ reps, const Blk *__restrict__ blks,
        typename CplxOf<Real>::type *__restrict__ c0, long long field_stride, int tile,
        bool inv, const typename CplxOf<Real>::type *__restrict__ twtab) {
  using C = typename CplxOf<Real>::type;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Blk const bk = blks[blockIdx.x];
  RepGeom const &G = reps[bk.rep];
  C *cm = c0 + field_stride * blockIdx.y;
  int const M1 = G.mesh[1];
  int const H = G.mesh[2] / 2 + 1;
  int const x = bk.a, kz0 = bk.b;
  int const T = min(tile, H - kz0);
  int const ld = line_ld(M1);
  bool const inplace = INPL || fft_inplace_ok(M1, tile, blockDim.x);
  C *a = reinterpret_cast<C *>(smem_raw);
  C *b = inplace ? nullptr : a + tile * ld;
  C *tw = a + (inplace ? 1 : 2) * tile * ld;
  load_twiddles(tw, twtab, G.plan[1]);
  long long const rowbase = G.km_off + static_cast<long long>(x) * M1 * G.hp + kz0;
  long long const hp = G.hp;
  // 16 x 16 thread mapping (tile <= 16 columns): column tq, rows yq + 16 i
  int const tq = threadIdx.x & 15, yq = threadIdx.x >> 4;
  bool const col = tq < T;
  // all of a thread's rows in flight at once (up to 16: M1 <= 256 in one
  // round)
  for (int y0 = yq; y0 < M1; y0 += 256) {
    C v[16];
#pragma unroll
    for (int u = 0; u < 16; ++u) {
      int const y = y0 + 16 * u;
      if (col && y < M1)
        v[u] = cm[rowbase + y * hp + tq];
    }
#pragma unroll
    for (int u = 0; u < 16; ++u) {
      int const y = y0 + 16 * u;
      if (col && y < M1)
        a[tq * ld + pix(y)] = v[u];
    }
  }
  __syncthreads();
  C *res;
  if constexpr (INPL)
    res = fft_lines_inplace<C>(a, T, ld, G.plan[1], tw, inv);
  else
    res = inplace ? fft_lines_inplace<C>(a, T, ld, G.plan[1], tw, inv)
                  : fft_lines<C>(a, b, T, ld, G.plan[1], tw, inv);
  if (col)
    for (int y = yq; y < M1; y += 16)
      cm[rowbase + y * hp + tq] = res[tq * ld + pix(y)];
}

// ---- pass x fused with the k-space operator -----------------------------
// Per block: one ky, a tile of kz; partials[blk*8 + {E, Pxx, Pxy, Pxz, Pyy,
// Pyz, Pzz, diag}] in FP64 (Hermitian weights 1 for kz = 0, M2/2, else 2).
// Shared memory: 3 x tile staged lines of line_ld(M0) (phi, field lines,
// scratch), twiddles (M0).
// EV: energy / virial partials (a template parameter, so that the
// forces-only instance carries none of their registers).  MINB: blocks per
// SM the registers are sized for -- 3 pays where the shared memory of a
// launch (small meshes) leaves room for a third block.
template <typename Real, bool EV, int MINB = 2>
__global__ void __launch_bounds__(256, MINB)
k_fft_x_kspace(const RepGeom *__restrict__ reps, const Blk *__restrict__ blks,
               const typename CplxOf<Real>::type *__restrict__ rho_hat,
               const Real *__restrict__ ginf, typename CplxOf<Real>::type *__restrict__ field0,
               long long field_stride, int tile, int want_fields,
               double *__restrict__ partials,
               const typename CplxOf<Real>::type *__restrict__ twtab) {
  using C = typename CplxOf<Real>::type;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Blk const bk = blks[blockIdx.x];
  RepGeom const &G = reps[bk.rep];
  int const M0 = G.mesh[0], M1 = G.mesh[1], M2 = G.mesh[2];
  int const H = M2 / 2 + 1;
  int const y = bk.a, kz0 = bk.b;
  int const T = min(tile, H - kz0);
  int const ld = line_ld(M0);
  int const L = tile * ld;
  C *a = reinterpret_cast<C *>(smem_raw);
  C *b = a + L;
  C *c = b + L; // three line buffers: phi, field lines, FFT scratch
  C *tw = c + L;
  load_twiddles(tw, twtab, G.plan[0]);
  long long const stride_x = static_cast<long long>(M1) * G.hp;
  long long const base = G.km_off + static_cast<long long>(y) * G.hp + kz0;
  // 16 x 16 thread mapping (tile <= 16 columns): column tq, rows xq + 16 i
  int const tq = threadIdx.x & 15, xq = threadIdx.x >> 4;
  bool const col = tq < T;
  for (int x0 = xq; x0 < M0; x0 += 64) {
    C v[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      int const x = x0 + 16 * u;
      if (col && x < M0)
        v[u] = rho_hat[base + x * stride_x + tq];
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      int const x = x0 + 16 * u;
      if (col && x < M0)
        a[tq * ld + pix(x)] = v[u];
    }
  }
  __syncthreads();
  C *res = fft_lines<C>(a, b, T, ld, G.plan[0], tw, false);
  C *fb = (res == a) ? b : a; // field lines go to the free buffer
  // k-space operator
  double const wv[3] = {2.0 * kPi * G.box_i[0], 2.0 * kPi * G.box_i[1],
                        2.0 * kPi * G.box_i[2]};
  double const hai2 = (1.0 / 2.0 / G.alpha) * (1.0 / 2.0 / G.alpha);
  double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  // d_op (Nyquist zeroed) integer shift of index i in a mesh of size m
  auto dop = [](int i, int m) { return (i == m / 2) ? 0 : (i < m / 2 ? i : i - m); };
  int const kyd = dop(y, M1);
  for (int x = xq; col && x < M0; x += 16) {
    // t fastest across lanes: the influence-function reads are T-contiguous
    int const t = tq;
    int const kz = kz0 + t;
    C const rh = res[t * ld + pix(x)];
    Real const g = ginf[base + x * stride_x + t];
    int const kxd = dop(x, M0), kzd = dop(kz, M2);
    if constexpr (EV) {
      double const wgt = (kz == 0 || kz == M2 / 2) ? 1.0 : 2.0;
      double const ek = wgt * static_cast<double>(g) *
                        (static_cast<double>(rh.x) * rh.x + static_cast<double>(rh.y) * rh.y);
      acc[0] += ek;
      double const kx = kxd * wv[0], ky = kyd * wv[1], kzv = kzd * wv[2];
      double const nsq = kx * kx + ky * ky + kzv * kzv;
      if (nsq != 0.0) {
        double const pr = ek * (-2.0 * (1.0 / nsq + hai2));
        acc[1] += pr * kx * kx;
        acc[2] += pr * kx * ky;
        acc[3] += pr * kx * kzv;
        acc[4] += pr * ky * ky;
        acc[5] += pr * ky * kzv;
        acc[6] += pr * kzv * kzv;
        acc[7] += ek;
      }
    }
    // phi = G rho_hat replaces rho_hat in place (same thread, same point)
    res[t * ld + pix(x)] = C{g * rh.x, g * rh.y};
  }
  if constexpr (EV) {
    // block reduction of the 8 partial sums (fixed order -> deterministic)
    __shared__ double red[8][32];
    int const lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      double v = acc[k];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1)
        v += __shfl_down_sync(0xffffffffu, v, o);
      if (lane == 0)
        red[k][wid] = v;
    }
    __syncthreads();
    if (threadIdx.x < 8) {
      double s = 0.0;
      int const nw = (blockDim.x + 31) >> 5;
      for (int w = 0; w < nw; ++w)
        s += red[threadIdx.x][w];
      partials[static_cast<long long>(blockIdx.x) * 8 + threadIdx.x] = s;
    }
  }
  if (!want_fields)
    return;
  // the three field components, one after another: E_d = i k_d phi, then
  // the backward x transform of its T lines
  int const kvec_y = kyd;
  for (int d = 0; d < 3; ++d) {
    __syncthreads(); // phi complete / previous component stored
    Real const wd = static_cast<Real>(wv[d]);
    for (int x = xq; col && x < M0; x += 16) {
      int const t = tq;
      int const kd = (d == 0) ? dop(x, M0) : (d == 1 ? kvec_y : dop(kz0 + t, M2));
      Real const k = static_cast<Real>(kd) * wd;
      C const phi = res[t * ld + pix(x)];
      fb[t * ld + pix(x)] = C{-k * phi.y, k * phi.x};
    }
    __syncthreads();
    C *fres = fft_lines<C>(fb, c, T, ld, G.plan[0], tw, true);
    if (col)
      for (int x = xq; x < M0; x += 16)
        field0[field_stride * d + base + x * stride_x + tq] = fres[tq * ld + pix(x)];
  }
}

// ---- pass z, backward for the 3 field components -> real fields --------
// Stride of a staged half row and size (elements) of the second buffer,
// which holds either the FFT scratch lines or the 3 nl staged half rows.
__host__ __device__ inline int z_inv_half_ld(int n) { return (n / 2 + 2) | 1; }
__host__ __device__ inline int z_inv_b_size(int nl, int n) {
  int const nc = nl + (nl + 1) / 2;
  int const s1 = nc * line_ld(n), s2 = 3 * nl * z_inv_half_ld(n);
  return s1 > s2 ? s1 : s2;
}

// Two real outputs per complex transform: slot l < nl carries Ex + i Ey of
// line l, slot nl + j carries Ez of lines 2j and 2j+1.  Each half row is
// extended by Hermitian symmetry with the imaginary parts of the k = 0 and
// k = n/2 entries dropped (c2r semantics), so both packed outputs are real.
// Shared memory: 2 x (nl + ceil(nl/2)) staged lines of line_ld(n),
// twiddles (n).  FP32: four blocks per SM -- the block's load, transform and
// store phases do not overlap, so the fourth resident block pays for the
// spills of the 64-register bound.
template <typename Real>
__global__ void __launch_bounds__(256, sizeof(Real) == 4 ? 4 : 2)
k_fft_z_inv3(const RepGeom *__restrict__ reps, const Blk *__restrict__ blks,
             const typename CplxOf<Real>::type *__restrict__ field0, long long field_stride,
             Real *__restrict__ efield, const typename CplxOf<Real>::type *__restrict__ twtab,
             int *__restrict__ err) {
  using C = typename CplxOf<Real>::type;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Blk const bk = blks[blockIdx.x];
  RepGeom const &G = reps[bk.rep];
  int const n = G.mesh[2];
  int const H = n / 2 + 1;
  int const ld = line_ld(n);
  int const nl = bk.b;
  int const nz = (nl + 1) >> 1;
  int const nc = nl + nz;
  long long const line0 = bk.a;
  // b doubles as the staging area of the 3 nl half rows (stride hl)
  int const hl = z_inv_half_ld(n);
  C *a = reinterpret_cast<C *>(smem_raw);
  C *b = a + nc * ld;
  C *tw = b + z_inv_b_size(nl, n);
  load_twiddles(tw, twtab, G.plan[2]);
  // stage the half rows of the 3 fields (field d, line l at
  // sb[(d * nl + l) * hs]), then build the packed lines in a.  A field's nl
  // rows are one contiguous range (row stride hp): one bulk copy (TMA
  // engine) per field when the three fit in b, else plain loads (stride hl)
  const C *fsrc = field0 + G.km_off + line0 * G.hp;
  __shared__ __align__(8) unsigned long long bar;
  size_t const rb = static_cast<size_t>(nl) * G.hp * sizeof(C);
  unsigned char *const bb = reinterpret_cast<unsigned char *>(b);
  unsigned const pad = (16u - (smem_u32(bb) & 15u)) & 15u;
  bool const bulk =
      ((reinterpret_cast<uintptr_t>(fsrc) | static_cast<uintptr_t>(field_stride * sizeof(C))) &
       15u) == 0 &&
      rb % 16 == 0 && pad + 3 * rb <= z_inv_b_size(nl, n) * sizeof(C) && 3 * rb < (1u << 20);
  C *sb = b;
  int hs = hl;
  if (bulk) {
    sb = reinterpret_cast<C *>(bb + pad);
    hs = G.hp;
    if (threadIdx.x == 0) {
      mbar_init(&bar, 1);
      mbar_arrive_expect_tx(&bar, static_cast<unsigned>(3 * rb));
      for (int d = 0; d < 3; ++d)
        bulk_g2s(bb + pad + d * rb, fsrc + field_stride * d, static_cast<unsigned>(rb), &bar);
    }
    __syncthreads(); // barrier initialised before anyone waits on it
    bool const ok = mbar_wait(&bar, 0);
    if (__syncthreads_or(!ok)) {
      if (threadIdx.x == 0) {
        atomicExch(err, 1);
        mbar_wait(&bar, 0); // second bounded wait for the copies in flight
      }
      return;
    }
  } else {
    // row dl = d * nl + l of the three fields
    for_lines(3 * nl, H, [&](int dl, int k) {
      int const d = (dl >= 2 * nl) ? 2 : (dl >= nl ? 1 : 0), l = dl - d * nl;
      b[dl * hl + k] = fsrc[field_stride * d + static_cast<long long>(l) * G.hp + k];
    });
    __syncthreads();
  }
  auto herm = [&](int d, int l, int k) -> C {
    const C *row = sb + (d * nl + l) * hs;
    if (k < H) {
      C v = row[k];
      if (k == 0 || 2 * k == n)
        v.y = Real(0);
      return v;
    }
    return cconj(row[n - k]);
  };
  for_lines(nc, n, [&](int j, int k) {
    C X, Y;
    if (j < nl) {
      X = herm(0, j, k);
      Y = herm(1, j, k);
    } else {
      int const l0 = 2 * (j - nl);
      X = herm(2, l0, k);
      Y = (l0 + 1 < nl) ? herm(2, l0 + 1, k) : C{Real(0), Real(0)};
    }
    a[j * ld + pix(k)] = C{X.x - Y.y, X.y + Y.x};
  });
  __syncthreads();
  C *res = fft_lines<C>(a, b, nc, ld, G.plan[2], tw, true);
  // packed field mesh: one (Ex, Ey, Ez, 0) record per mesh point, so the
  // interpolation gathers one 16-byte (FP32) record per stencil point
  // (ghost-padded: every record also goes to its periodic images in the
  // high-side ghost layers of extent epad)
  using R4 = typename Real4Of<Real>::type;
  R4 *out = reinterpret_cast<R4 *>(efield) + G.re_off;
  int const M1 = G.mesh[1], M0 = G.mesh[0];
  int const P0 = G.epad[0], P1 = G.epad[1], P2 = G.epad[2];
  int const x0 = static_cast<int>(line0 / M1), y0 = static_cast<int>(line0 - static_cast<long long>(x0) * M1);
  for_lines(nl, n, [&](int l, int k) {
    C const xy = res[l * ld + pix(k)];
    C const zz = res[(nl + (l >> 1)) * ld + pix(k)];
    R4 v;
    v.x = xy.x;
    v.y = xy.y;
    v.z = (l & 1) ? zz.y : zz.x;
    v.w = Real(0);
    int x = x0, y = y0 + l;
    while (y >= M1) {
      y -= M1;
      ++x;
    }
    for (int xg = x; xg < P0; xg += M0)
      for (int yg = y; yg < P1; yg += M1) {
        R4 *row = out + (static_cast<long long>(xg) * P1 + yg) * P2;
        for (int zg = k; zg < P2; zg += n)
          row[zg] = v;
      }
  });
}

} // namespace p3mx

// P3M particle <-> mesh kernels (sm_100a): corner binning, B-spline weights,
// gather-based deterministic charge assignment, force back-interpolation,
// influence function, charge census and the k-space error sum.
#pragma once

#include "common.cuh"

namespace p3mx {

// Fold into [0, L) like algorithm/periodic_fold.hpp:72-89 (repeated shifts);
// far-away coordinates are first brought close by whole periods.
__device__ inline double fold_coord(double x, double L) {
  if (x < -2.0 * L || x >= 3.0 * L)
    x -= floor(x / L) * L;
  int guard = 0;
  while (x < 0.0 && guard++ < 8)
    x += L;
  while (x >= L && guard++ < 16)
    x -= L;
  return x;
}

// Cardinal B-spline weights of order P at the P points around a particle
// (x = distance to the nearest mesh point, [-0.5, 0.5]) by the Cox-de Boor
// recursion; w[i] = M_P(x + 1/2 + P-1-i), the values tabulated in
// utils/math/bspline.hpp:30-177.
template <int P, typename Real>
__device__ inline void bspline_weights(Real x, Real *w) {
  Real c[P];
  Real const u = x + Real(0.5);
  c[0] = Real(1);
#pragma unroll
  for (int n = 1; n < P; ++n) {
    Real const inv_n = Real(1) / Real(n);
    c[n] = Real(0);
#pragma unroll
    for (int k = n; k >= 0; --k) {
      Real const left = (k > 0) ? c[k - 1] : Real(0);
      c[k] = ((u + Real(k)) * c[k] + (Real(n + 1) - u - Real(k)) * left) * inv_n;
    }
  }
#pragma unroll
  for (int i = 0; i < P; ++i)
    w[i] = c[P - 1 - i];
}

// Per particle: nearest-mesh-point corner and the distance to it, following
// p3m_calculate_interpolation_weights (p3m/interpolation.hpp:138-178) with
// the single-rank CA-mesh origin of P3MLocalMesh (p3m/common.cpp:34-106).
// key = corner, brick-major: bin_off + brick*B^3 + (lx*B + ly)*B + lz with
// brick = (bx*nby + by)*nbz + bz and (lx, ly, lz) the corner inside it; the
// sort key bkey = brk_off + brick, so the particles of one brick form one
// contiguous range of the sorted order (particle index order inside it).
template <typename Real>
__global__ void k_p3m_bin(const RepGeom *__restrict__ reps, const int *__restrict__ rep_of,
                          const double *__restrict__ pos, long long n,
                          int *__restrict__ key, int *__restrict__ bkey, int *__restrict__ slot,
                          int *__restrict__ cnt, Real *__restrict__ dist) {
  long long const i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n)
    return;
  RepGeom const &G = reps[rep_of[i]];
  int g[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    double const xf = fold_coord(pos[3 * i + d], G.box[d]);
    double const p = ((xf - G.ld_pos[d]) * G.ai[d]) - G.pos_shift;
    int const nmp = static_cast<int>(p);
    double const ds = (p - nmp) - 0.5;
    int c = (G.ld_ind[d] + nmp) % G.mesh[d];
    if (c < 0)
      c += G.mesh[d];
    g[d] = c;
    dist[3 * i + d] = static_cast<Real>(ds);
  }
  int const B = G.brick;
  int const brick = ((g[0] / B) * G.nby + g[1] / B) * G.nbz + g[2] / B;
  int const k = static_cast<int>(G.bin_off) + brick * B * B * B +
                ((g[0] % B) * B + g[1] % B) * B + g[2] % B;
  key[i] = k;
  int const b = static_cast<int>(G.brk_off) + brick;
  bkey[i] = b;
  slot[i] = atomicAdd(&cnt[b], 1);
}

// Per-particle weight record for order P (R = 4):
// {q*wx[0..P), wy[0..P), 0[R-1], wz[0..P), 0[R-1]}, zero-padded; the stride
// is a multiple of 4 elements (16 bytes in FP32, 32 in FP64) so that records
// are stored as vectors and runs of records are legal 16-byte asynchronous
// copies.
template <int P, int R> __host__ __device__ constexpr int wstride() {
  return (3 * P + 2 * (R - 1) + 3) / 4 * 4;
}
template <int P, int R> __host__ __device__ constexpr int wz_off() { return 2 * P + (R - 1); }
// Record stride of every order (that of order 7), so that replicas of one
// batch may use different orders: a sorted particle's record starts at
// s * kRecStride whatever its replica's order.
constexpr int kRecStride = wstride<7, 4>();

// Weight record of one sorted particle for order P (R = 4):
// {q*wx[0..P), wy[0..P), 0[R-1], wz[0..P), 0[R-1]}, zero-padded to the
// common stride kRecStride, stored as 16- or 32-byte vectors.
template <typename Real, int P>
__device__ inline void weights_record(const Real *dist3, double q, Real *__restrict__ out) {
  constexpr int R = 4;
  Real w[3][P];
  bspline_weights<P>(dist3[0], w[0]);
  bspline_weights<P>(dist3[1], w[1]);
  bspline_weights<P>(dist3[2], w[2]);
  Real const qi = static_cast<Real>(q);
  constexpr int WS = kRecStride;
  Real rec[WS];
#pragma unroll
  for (int k = 0; k < WS; ++k)
    rec[k] = Real(0);
#pragma unroll
  for (int k = 0; k < P; ++k) {
    rec[k] = qi * w[0][k];
    rec[P + k] = w[1][k];
    rec[wz_off<P, R>() + k] = w[2][k];
  }
  using R4 = typename Real4Of<Real>::type;
  R4 *o = reinterpret_cast<R4 *>(out);
#pragma unroll
  for (int k = 0; k < WS / 4; ++k) {
    R4 v;
    v.x = rec[4 * k];
    v.y = rec[4 * k + 1];
    v.z = rec[4 * k + 2];
    v.w = rec[4 * k + 3];
    o[k] = v;
  }
}

// Weights in brick-sorted order (each replica's order), the corner key
// (relative to the replica's corner range) of every sorted particle, and
// each replica's largest |q| (FP32 bits rounded up, atomic maximum:
// order-independent) for the fixed-point scale of the charge assignment.
template <typename Real>
__global__ void __launch_bounds__(256)
k_p3m_weights(const RepGeom *__restrict__ reps, const int *__restrict__ perm,
              const int *__restrict__ key, const Real *__restrict__ dist,
              const double *__restrict__ q, const int *__restrict__ rep_of,
              long long n, Real *__restrict__ W, int *__restrict__ s_key,
              unsigned *__restrict__ qmax_bits) {
  // FP32 records are built in shared memory and each warp's 32 records
  // (contiguous in W) leave with 16-byte lane stores of consecutive
  // addresses; a thread's own record would be 7 stores 112 bytes apart
  constexpr bool kStage = sizeof(Real) == 4;
  __shared__ __align__(16) Real s_rec[kStage ? 256 * kRecStride : 1];
  long long const s = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  int const lane = threadIdx.x & 31;
  if (s < n) {
    int const i = perm[s];
    int const rep = rep_of[i];
    RepGeom const &G = reps[rep];
    {
      // one atomic per group of lanes of the same replica
      unsigned const qb = __float_as_uint(__double2float_ru(fabs(q[i])));
      unsigned const act = __activemask();
      unsigned const grp = __match_any_sync(act, rep);
      unsigned const mx = __reduce_max_sync(grp, qb);
      if (lane == __ffs(grp) - 1)
        atomicMax(&qmax_bits[rep], mx);
    }
    Real *out = kStage ? s_rec + threadIdx.x * kRecStride : W + s * kRecStride;
    const Real *d3 = dist + 3 * i;
    switch (G.cao) {
    case 1: weights_record<Real, 1>(d3, q[i], out); break;
    case 2: weights_record<Real, 2>(d3, q[i], out); break;
    case 3: weights_record<Real, 3>(d3, q[i], out); break;
    case 4: weights_record<Real, 4>(d3, q[i], out); break;
    case 5: weights_record<Real, 5>(d3, q[i], out); break;
    case 6: weights_record<Real, 6>(d3, q[i], out); break;
    default: weights_record<Real, 7>(d3, q[i], out); break;
    }
    s_key[s] = key[i] - static_cast<int>(G.bin_off);
  }
  if constexpr (kStage) {
    __syncwarp();
    long long const s0 = s - lane;
    if (s0 >= n)
      return;
    int const nv = static_cast<int>(min(32LL, n - s0));
    const float4 *src = reinterpret_cast<const float4 *>(s_rec + (threadIdx.x - lane) * kRecStride);
    float4 *dst = reinterpret_cast<float4 *>(W + s0 * kRecStride);
    for (int k = lane; k < nv * (kRecStride / 4); k += 32)
      dst[k] = src[k];
  }
}

// Edge (mesh points) of the sort bricks that bin the particles by stencil
// corner for order P (the interpolation stages one brick's field tile of
// (B + P - 1)^3 points; owner blocks of the assignment are whole numbers
// of bricks).
template <int P> __host__ __device__ constexpr int brick_edge() { return (P <= 5) ? 4 : 8; }

struct TileStrides {
  int sy, sx;
};

// ---------------------------------------------------------------------------
// Charge assignment by super-bricks (AssignCharges, p3m.cpp:225-265;
// charge_assign, p3m.cpp:283-330).  One CTA takes the particles whose
// stencil corners lie in a super-brick of E^3 corner positions (whole
// sort bricks: a few contiguous ranges of the brick-major order), so every
// particle is visited once.  For each particle one warp covers its P^2
// (x, y) stencil rows (one row per lane, the P z points of a row unrolled)
// and adds q wx wy wz into a shared-memory tile of (E + P - 1)^3
// points, in fixed point; the tile is then added to the mesh.  E = 16, or 8
// when the 16^3 super-bricks of one colour would not give every SM a block
// (small meshes: more, smaller tiles with a larger halo share).  Tiles of
// neighbouring super-bricks overlap by P - 1 points, so super-bricks are
// coloured (greedy interval colouring per dimension: tiles of one colour
// never overlap, modulo the mesh) and launched colour by colour: the plain
// read-add-write of a tile is race-free and the colour order fixes the
// order of the FP adds, so the mesh is bitwise reproducible.  The colour
// launches are chained by programmatic dependent launch: a colour fills its
// tiles while the previous one drains, and waits (griddepcontrol.wait) only
// before its read-add-write of the mesh.
//
// Fixed point: a term v = q wx wy wz becomes t = rint(v S) by one FP64 FMA
// with the magic constant 1.5 * 2^52 (the bits of the sum are those of the
// constant plus t while |t| < 2^51) and is added with one integer atomic:
// FP32-mixed path, the low 32 bits (the constant's low word is zero, so the
// word is t modulo 2^32, and a tile point's sum is exact modulo 2^32); FP64
// path, the 64-bit t.  S is a power of two with n qmax wmax^3 S < 2^31
// (FP32-mixed) or < 2^62 and qmax wmax^3 S < 2^51 (FP64), n the particles of
// the super-brick, qmax the replica's largest |q|, wmax the largest B-spline
// weight of order P: no term leaves the exact range and no tile point's
// final sum overflows (wrap-around of intermediate two's complement sums
// cancels).  Integer sums do not depend on the order of the atomics; the
// quantum 1/S is about 2^-25 of a charge at 2^20 ions on a 256^3 mesh
// (FP32-mixed) and 2^-56 in FP64, and each tile point is rounded once to
// the working precision before it is added to the mesh.
constexpr int kSbEdge = 16;   // corner positions per dimension of a super-brick (multiple of 4 and 8)
constexpr int kSbEdgeSmall = 8; // the edge for meshes with too few 16^3 super-bricks to fill the GPU
constexpr int kSbWarps = 8;   // warps per super-brick block
constexpr int kSbChunk = 64;  // particles whose records are staged at a time

// Largest cardinal B-spline weight of order P over dist in [-1/2, 1/2],
// rounded up (1, 1, 3/4, 2/3, 115/192, 11/20, 0.51102...).
template <int P> __host__ __device__ constexpr double bspline_wmax() {
  return P <= 2 ? 1.0 : P == 3 ? 0.7501 : P == 4 ? 0.6668 : P == 5 ? 0.5991 : P == 6 ? 0.5501 : 0.5112;
}

template <typename Real> struct SbWord;
template <> struct SbWord<float> {
  using type = unsigned;
  static constexpr int sum_bits = 31;
};
template <> struct SbWord<double> {
  using type = unsigned long long;
  static constexpr int sum_bits = 62;
};
constexpr int kSbTermBits = 51;
// t = rint(a b) for |a b| < 2^51, added modulo 2^32 (low word of the FMA
// with the magic constant) or as a 64-bit integer
__device__ inline void sb_add(unsigned *p, double a, double b) {
  double const r = fma(a, b, 6755399441055744.0); // 1.5 * 2^52
  atomicAdd(p, static_cast<unsigned>(__double2loint(r)));
}
// FP64 path: the 64-bit t added as two 32-bit words (the low word's atomic
// returns its old value, whose wrap-around gives the carry into the high
// word), so the sum is exact modulo 2^64 with native 32-bit shared-memory
// atomics only
__device__ inline void sb_add(unsigned long long *p, double a, double b) {
  double const r = fma(a, b, 6755399441055744.0);
  unsigned long long const t =
      static_cast<unsigned long long>(__double_as_longlong(r)) - 0x4338000000000000ull;
  unsigned *w = reinterpret_cast<unsigned *>(p); // little endian: w[0] low, w[1] high
  unsigned const lo = static_cast<unsigned>(t);
  unsigned const old = atomicAdd(w, lo);
  unsigned const hi = static_cast<unsigned>(t >> 32) + ((old + lo < old) ? 1u : 0u);
  if (hi != 0u)
    atomicAdd(w + 1, hi);
}
__device__ inline float sb_value(unsigned v, float inv_s) {
  return static_cast<float>(static_cast<int>(v)) * inv_s;
}
__device__ inline double sb_value(unsigned long long v, double inv_s) {
  return static_cast<double>(static_cast<long long>(v)) * inv_s;
}

// Tile edge of a super-brick of edge E for order P.
template <int P, int E> __host__ __device__ constexpr int sb_tile_edge() { return E + P - 1; }
// Strides of the tile [x][y][z] (z contiguous, words of WB bytes): the
// smallest y stride >= the tile edge and x stride >= edge * (y stride) for
// which the lanes of one shared-memory wavefront (128 bytes: 32 lanes of
// 4-byte words, 16 of 8-byte words), one (x, y) stencil row each (row
// r = lane + 32 q, x = r / P, y = r % P), hit distinct banks.
template <int P, int WB, int E> __host__ __device__ constexpr TileStrides sb_strides() {
  constexpr int TE = sb_tile_edge<P, E>();
  constexpr int L = 128 / WB;
  for (int sy = TE; sy < TE + L; ++sy)
    for (int sx = TE * sy; sx < TE * sy + 2 * L; ++sx) {
      bool ok = true;
      for (int r0 = 0; r0 < P * P && ok; r0 += L) {
        unsigned long long used = 0;
        for (int r = r0; r < r0 + L && r < P * P; ++r) {
          unsigned long long const bit = 1ull << (((r / P) * sx + (r % P) * sy) % L);
          if (used & bit) {
            ok = false;
            break;
          }
          used |= bit;
        }
      }
      if (ok)
        return TileStrides{sy, sx};
    }
  return TileStrides{TE, TE * TE};
}
template <typename Real, int P, int E> __host__ __device__ constexpr size_t sb_tile_bytes() {
  using W = typename SbWord<Real>::type;
  return (sizeof(W) * sb_tile_edge<P, E>() * static_cast<size_t>(sb_strides<P, sizeof(W), E>().sx) +
          15) / 16 * 16;
}
// shared memory: tile, staged weight records, per staged particle its z
// weights times S in FP64 (8 slots) and its tile offset
template <typename Real, int P, int E> __host__ __device__ constexpr size_t sb_smem() {
  return sb_tile_bytes<Real, P, E>() + sizeof(Real) * kSbChunk * kRecStride +
         sizeof(double) * 8 * kSbChunk + sizeof(int) * kSbChunk;
}
// sort-brick runs of a super-brick: (kSbEdge / B)^2 brick columns, one
// contiguous z run each
constexpr int kSbMaxRuns = (kSbEdge / 4) * (kSbEdge / 4);

template <typename Real, int P, int E, bool MC>
__global__ void __launch_bounds__(32 * kSbWarps, sizeof(Real) == 4 ? 4 : 1)
k_p3m_assign_sb(const RepGeom *__restrict__ reps, const int2 *__restrict__ sbs, int nsb,
                const int *__restrict__ start, const Real *__restrict__ W,
                const int *__restrict__ s_key, const unsigned *__restrict__ qmax_bits,
                Real *__restrict__ rho, int *__restrict__ err, long long comp_w,
                long long comp_rho, int comp_q) {
  // MC: blockIdx.y picks one of several charge sets assigned by one launch
  // (the dipole components): its weight records, mesh and |q| maxima lie
  // comp_w / comp_rho / comp_q elements after the previous set's. The
  // single-set instance leaves the three pointers as kernel parameters: the
  // offset copies cost six registers, which spill the FP32 order-7 16^3
  // instance at its 64-register bound (0.239 -> 0.307 ms at 2^20 ions).
  if constexpr (MC) {
    W += blockIdx.y * comp_w;
    rho += blockIdx.y * comp_rho;
    qmax_bits += blockIdx.y * comp_q;
  }
  using Word = typename SbWord<Real>::type;
  constexpr int R = 4;
  constexpr int WS = kRecStride;
  constexpr int WZ = wz_off<P, R>();
  constexpr int P2 = P * P;
  constexpr int NQ = (P2 + 31) / 32;
  constexpr int NT = 32 * kSbWarps;
  constexpr int TE = sb_tile_edge<P, E>();
  constexpr int B = brick_edge<P>(), B3 = B * B * B, NBS = E / B;
  constexpr int LB = (B == 4) ? 2 : 3;
  constexpr TileStrides TS = sb_strides<P, sizeof(Word), E>();
  constexpr int SY = TS.sy, SX = TS.sx;
  constexpr int TW = static_cast<int>(sb_tile_bytes<Real, P, E>() / sizeof(Word));
  static_assert(E % B == 0 && E <= kSbEdge, "super-brick edge: a multiple of the sort brick");
  constexpr int CH = kSbChunk;
  static_assert(NBS * NBS <= kSbMaxRuns, "run table too small");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ __align__(8) unsigned long long bar;
  __shared__ int s_r0[kSbMaxRuns], s_r1[kSbMaxRuns];
  __shared__ int s_count;
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  if (static_cast<int>(blockIdx.x) >= nsb)
    return; // whole block
  Word *tile = reinterpret_cast<Word *>(smem_raw);
  Real *rec = reinterpret_cast<Real *>(smem_raw + sb_tile_bytes<Real, P, E>());
  double *wzd = reinterpret_cast<double *>(rec + CH * WS);
  int *toff = reinterpret_cast<int *>(wzd + 8 * CH);
  int const tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

  int2 const sb = sbs[blockIdx.x];
  RepGeom const &G = reps[sb.x];
  int const M0 = G.mesh[0], M1 = G.mesh[1], M2 = G.mesh[2];
  int const no1 = (M1 + E - 1) / E, no2 = (M2 + E - 1) / E;
  int const o0 = (sb.y / (no1 * no2)) * E, o1 = ((sb.y / no2) % no1) * E, o2 = (sb.y % no2) * E;
  // the super-brick's sort bricks (fewer at the high end of a mesh that is
  // not a multiple of E)
  int const bx0 = o0 / B, by0 = o1 / B, bz0 = o2 / B;
  int const nbx = min(NBS, G.nbx - bx0), nby = min(NBS, G.nby - by0), nbz = min(NBS, G.nbz - bz0);
  int const ncol = nbx * nby;
  if (tid < ncol) {
    const int *st = start + G.brk_off;
    int const col = ((bx0 + tid / nby) * G.nby + (by0 + tid % nby)) * G.nbz + bz0;
    s_r0[tid] = st[col];
    s_r1[tid] = st[col + nbz];
  }
  // zero the tile; initialise the staging barrier
  for (int t = tid; t < TW; t += NT)
    tile[t] = Word(0);
  if (tid == 0)
    mbar_init(&bar, 1);
  __syncthreads();
  if (warp == 0) {
    int c = (lane < ncol) ? s_r1[lane] - s_r0[lane] : 0;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1)
      c += __shfl_xor_sync(0xffffffffu, c, off);
    if (lane == 0)
      s_count = c;
  }
  __syncthreads();
  int const count = s_count;
  float const qmax = __uint_as_float(qmax_bits[sb.x]);
  if (count == 0 || !(qmax > 0.0f))
    return; // nothing to add to the mesh
  int es;
  {
    double const unit = static_cast<double>(qmax) * bspline_wmax<P>() * bspline_wmax<P>() *
                        bspline_wmax<P>();
    int ea, eb;
    frexp(unit, &ea);
    frexp(unit * static_cast<double>(count), &eb);
    es = min(kSbTermBits - ea, SbWord<Real>::sum_bits - eb);
    es = max(min(es, 1000), -1000);
  }
  double const S = ldexp(1.0, es);
  // per-lane (x, y) stencil row of each round and its tile offset
  int qx[NQ], qy[NQ], qoff[NQ];
#pragma unroll
  for (int q = 0; q < NQ; ++q) {
    int const r = lane + 32 * q;
    int const rr = (r < P2) ? r : 0;
    qx[q] = rr / P;
    qy[q] = rr % P;
    qoff[q] = qx[q] * SX + qy[q] * SY;
  }
  unsigned parity = 0;
  for (int run = 0; run < ncol; ++run) {
    int const s0 = s_r0[run], s1 = s_r1[run];
    int const bx = bx0 + run / nby, by = by0 + run % nby;
    int const b0 = (bx * G.nby + by) * G.nbz + bz0;
    for (int c0 = s0; c0 < s1; c0 += CH) {
      int const cn = min(CH, s1 - c0);
      __syncthreads(); // the previous chunk is consumed
      if (tid == 0) {
        unsigned const nbytes = static_cast<unsigned>(cn * WS * sizeof(Real));
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        mbar_arrive_expect_tx(&bar, nbytes);
        bulk_g2s(rec, W + static_cast<long long>(c0) * WS, nbytes, &bar);
      }
      for (int j = tid; j < cn; j += NT) {
        // corner offset inside the super-brick, [0, E)^3
        int const sk = s_key[c0 + j];
        int const bz = bz0 + ((sk >> (3 * LB)) - b0);
        int const l = sk & (B3 - 1);
        int const dx = bx * B + (l >> (2 * LB)) - o0, dy = by * B + ((l >> LB) & (B - 1)) - o1,
                  dz = bz * B + (l & (B - 1)) - o2;
        toff[j] = dx * SX + dy * SY + dz;
      }
      bool const got = mbar_wait(&bar, parity);
      parity ^= 1u;
      if (__syncthreads_or(!got)) {
        if (tid == 0) {
          atomicExch(err, 1);
          mbar_wait(&bar, parity ^ 1u); // bounded wait for the copy in flight
        }
        return;
      }
      // z weights of the staged records in FP64, times S
      for (int t = tid; t < cn * P; t += NT) {
        int const j = t / P, k = t - j * P;
        wzd[8 * j + k] = static_cast<double>(rec[j * WS + WZ + k]) * S;
      }
      __syncthreads();
      for (int j = warp; j < cn; j += kSbWarps) {
        int const base = toff[j];
        const Real *w = rec + j * WS;
        double wz[P];
#pragma unroll
        for (int k = 0; k < P; ++k)
          wz[k] = wzd[8 * j + k];
#pragma unroll
        for (int q = 0; q < NQ; ++q) {
          if (lane + 32 * q < P2) {
            double const wxy = static_cast<double>(w[qx[q]] * w[P + qy[q]]);
            Word *pt = tile + base + qoff[q];
#pragma unroll
            for (int k = 0; k < P; ++k)
              sb_add(pt + k, wxy, wz[k]);
          }
        }
      }
    }
  }
  __syncthreads();
  Real const inv_S = static_cast<Real>(ldexp(1.0, -es));
  // the previous colour's read-add-write has completed and is visible
  asm volatile("griddepcontrol.wait;" ::: "memory");
  // add the tile to the mesh: real extent of the super-brick plus the stencil
  int const ex0 = min(E, M0 - o0) + P - 1, ey = min(E, M1 - o1) + P - 1,
            ez = min(E, M2 - o2) + P - 1;
  Real *mesh = rho + G.rm_off;
  // a tile wider than the mesh maps two tile points onto one mesh point:
  // add such points in separate passes (one per wrap class)
  bool const self_wrap = (ex0 > M0) || (ey > M1) || (ez > M2);
  int const passes = self_wrap ? 8 : 1;
  // each thread owns fixed (y, z) slots of the tile's yz plane; loop over x
  constexpr int NS = (TE * TE + NT - 1) / NT;
  int yzt[NS], yzg[NS], ycls[NS];
  int const nyz = ey * ez;
#pragma unroll
  for (int k2 = 0; k2 < NS; ++k2) {
    int const t = tid + NT * k2;
    int const y = (t < nyz) ? t / ez : 0, z = (t < nyz) ? t - (t / ez) * ez : 0;
    int gy = o1 + y, gz = o2 + z, cls = 0;
    if (gy >= M1) { gy -= M1; cls |= 2; }
    if (gy >= M1) gy -= M1;
    if (gz >= M2) { gz -= M2; cls |= 4; }
    if (gz >= M2) gz -= M2;
    yzt[k2] = (t < nyz) ? y * SY + z : -1;
    yzg[k2] = gy * M2 + gz;
    ycls[k2] = cls;
  }
  if (!self_wrap) {
    // every tile point maps to its own mesh point: issue the thread's mesh
    // loads of XG x planes first, then the adds and stores
    constexpr int XG = 8;
#pragma unroll 1
    for (int xg = 0; xg < ex0; xg += XG) {
      Real old[XG][NS];
#pragma unroll
      for (int xx = 0; xx < XG; ++xx) {
        int const x = xg + xx;
        int gx = o0 + x;
        gx -= (gx >= M0) ? M0 : 0;
        long long const gbase = static_cast<long long>(gx) * M1 * M2;
#pragma unroll
        for (int k2 = 0; k2 < NS; ++k2)
          if (x < ex0 && yzt[k2] >= 0)
            old[xx][k2] = mesh[gbase + yzg[k2]];
      }
#pragma unroll
      for (int xx = 0; xx < XG; ++xx) {
        int const x = xg + xx;
        int gx = o0 + x;
        gx -= (gx >= M0) ? M0 : 0;
        long long const gbase = static_cast<long long>(gx) * M1 * M2;
#pragma unroll
        for (int k2 = 0; k2 < NS; ++k2)
          if (x < ex0 && yzt[k2] >= 0)
            mesh[gbase + yzg[k2]] = old[xx][k2] + sb_value(tile[x * SX + yzt[k2]], inv_S);
      }
    }
    return;
  }
  for (int pass = 0; pass < passes; ++pass) {
    for (int x = 0; x < ex0; ++x) {
      int gx = o0 + x, xcls = 0;
      if (gx >= M0) { gx -= M0; xcls = 1; }
      if (gx >= M0) gx -= M0;
      long long const gbase = static_cast<long long>(gx) * M1 * M2;
#pragma unroll
      for (int k2 = 0; k2 < NS; ++k2) {
        if (yzt[k2] < 0 || (xcls | ycls[k2]) != pass)
          continue;
        mesh[gbase + yzg[k2]] += sb_value(tile[x * SX + yzt[k2]], inv_S);
      }
    }
    __syncthreads();
  }
}

// Force back-interpolation (AssignForces, electrostatics/p3m.cpp:344-373) as
// a warp-specialised pipeline over bricks.  Each block takes the bricks
// blockIdx.x, blockIdx.x + gridDim.x, ... (a persistent grid); its warp 0
// (the producer) fills kInterpStages shared-memory stages ahead of the
// kInterpWarps consumer warps.  A stage holds one brick's field tile --
// (B+P-1)^3 packed (Ex, Ey, Ez, 0) records from the brick origin, one 3-d
// tensor copy (TMA engine) from the replica's ghost-padded field mesh, whose
// high-side ghost layers hold the periodic images -- and the weight records,
// sort keys and source indices of up to kInterpCap of the brick's particles
// (contiguous in the brick-major order: one bulk copy each).  A full barrier
// per stage counts the producer lanes' arrivals and the copied bytes; an
// empty barrier per stage counts the consumer warps that finished with it.
// Consumers read shared memory only (particles past the cap of a dense brick
// read their records from global memory) and store the forces.
//
// Eight lanes serve one particle: lane kz owns the stencil z offset kz and
// walks the P^2 (x, y) rows; lane sums are FP32 (FP64 for the FP64 path),
// the group reduction is FP64 in a fixed shuffle order (deterministic).
// F -= prefactor/V * sum (q wx wy wz) E, plus the dipole term for
// epsilon != 0 (p3m.cpp:540-547).  Writes (or adds) f[3*i] of the original
// particle index.  Every barrier wait is bounded: on a timeout the kernel
// sets *err, the producer waits (bounded) for its copies in flight, and the
// block returns.
constexpr int kInterpStages = 2;
constexpr int kInterpWarps = 8; // consumer warps
constexpr int kInterpCap = 64;  // particles per stage with staged records

template <typename Real, int P> struct InterpStage {
  using R4 = typename Real4Of<Real>::type;
  static constexpr int Ed = brick_edge<P>() + P - 1;
  static constexpr size_t tile = sizeof(R4) * Ed * Ed * Ed;
  static constexpr size_t rec = sizeof(Real) * kInterpCap * kRecStride;
  // key / index window: the 16-byte aligned superset of the staged range
  static constexpr size_t ids = sizeof(int) * (kInterpCap + 8);
  // stages start on 128-byte boundaries (tensor copy destinations)
  static constexpr size_t bytes = (tile + rec + 2 * ids + 127) / 128 * 128;
  static_assert(tile % 16 == 0 && rec % 16 == 0 && ids % 16 == 0, "bulk copy alignment");
};
// (+ 128: the kernel rounds the dynamic shared-memory base up to 128 bytes)
template <typename Real, int P> __host__ __device__ constexpr size_t interp_smem() {
  return kInterpStages * InterpStage<Real, P>::bytes + 128;
}

struct InterpInfo {
  int rep, brick, s0, s1; // rep < 0: no more bricks
  double pref, cdip;
};

__device__ inline void mbar_arrive(unsigned long long *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

template <typename Real, int P>
__global__ void __launch_bounds__(32 * (1 + kInterpWarps), sizeof(Real) == 4 ? 2 : 1)
k_p3m_interp(const RepGeom *__restrict__ reps, const int2 *__restrict__ bricks, int nbricks,
             const int *__restrict__ start, const int *__restrict__ perm,
             const int *__restrict__ s_key, const Real *__restrict__ W,
             const Real *__restrict__ E, const CUtensorMap *__restrict__ tmaps,
             const double *__restrict__ q, const double *__restrict__ dipole,
             double *__restrict__ f, int overwrite, int *__restrict__ err) {
  static_assert(P <= 8, "one lane per stencil z offset");
  constexpr int R = 4;
  constexpr int WS = kRecStride;
  constexpr int WZ = wz_off<P, R>();
  constexpr int S = kInterpStages, CW = kInterpWarps, CAP = kInterpCap;
  using L = InterpStage<Real, P>;
  using R4 = typename L::R4;
  constexpr int B = brick_edge<P>(), B3 = B * B * B, Ed = L::Ed, E2 = Ed * Ed;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ __align__(8) unsigned long long full[S], empty[S];
  __shared__ InterpInfo s_info[S];
  int const tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (tid == 0) {
#pragma unroll
    for (int k = 0; k < S; ++k) {
      mbar_init(&full[k], 32);  // the producer's lanes
      mbar_init(&empty[k], CW); // one arrival per consumer warp
    }
  }
  __syncthreads();
  unsigned char *const smem_base = smem_raw + ((128u - (smem_u32(smem_raw) & 127u)) & 127u);
  auto stage_ptr = [&](int k) { return smem_base + static_cast<size_t>(k) * L::bytes; };

  if (warp == 0) {
    // ---------------- producer ----------------
    // the next brick's table entry and particle range are fetched one brick
    // ahead, so their load latency overlaps the copies of the current one
    int it = 0, last_rep = -1;
    bool ok = true;
    int n = blockIdx.x;
    int2 bk = make_int2(0, 0);
    int s0 = 0, s1 = 0;
    if (n < nbricks) {
      bk = bricks[n];
      const int *st = start + reps[bk.x].brk_off;
      s0 = st[bk.y];
      s1 = st[bk.y + 1];
    }
    for (; n < nbricks; n += gridDim.x) {
      int const nn = n + gridDim.x;
      int2 const bkn = (nn < nbricks) ? bricks[nn] : make_int2(0, 0);
      if (s0 != s1) {
        RepGeom const &G = reps[bk.x];
        int const k = it % S;
        bool const got = mbar_wait(&empty[k], ((it / S) & 1) ^ 1u);
        if (!__all_sync(0xffffffffu, got)) {
          ok = false;
          break;
        }
        unsigned char *sp = stage_ptr(k);
        R4 *tile = reinterpret_cast<R4 *>(sp);
        Real *rec = reinterpret_cast<Real *>(sp + L::tile);
        int *keys = reinterpret_cast<int *>(sp + L::tile + L::rec);
        int *pm = reinterpret_cast<int *>(sp + L::tile + L::rec + L::ids);
        int const cn = min(s1 - s0, CAP);
        int const a0 = s0 & ~3, a1 = (s0 + cn + 3) & ~3;
        if (lane == 0) {
          InterpInfo inf;
          inf.rep = bk.x;
          inf.brick = bk.y;
          inf.s0 = s0;
          inf.s1 = s1;
          inf.pref = G.prefactor / G.V;
          inf.cdip = (G.epsilon != 0.0)
                         ? G.prefactor * 4.0 * kPi / G.V / (2.0 * G.epsilon + 1.0)
                         : 0.0;
          s_info[k] = inf;
        }
        // the consumers' reads of the stage were generic-proxy accesses:
        // order them before the asynchronous-proxy writes that refill it
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        int const bz = bk.y % G.nbz, by = (bk.y / G.nbz) % G.nby, bx = bk.y / (G.nbz * G.nby);
        // lane 0: the tile; lanes 1..3: one particle array each
        unsigned bytes = 0;
        if (lane == 0)
          bytes = static_cast<unsigned>(E2 * Ed * sizeof(R4));
        else if (lane == 1)
          bytes = static_cast<unsigned>(cn * WS * sizeof(Real));
        else if (lane == 2 || lane == 3)
          bytes = static_cast<unsigned>((a1 - a0) * sizeof(int));
        mbar_arrive_expect_tx(&full[k], bytes);
        if (lane == 0) {
          if (bk.x != last_rep) {
            tensormap_acquire(&tmaps[bk.x]);
            last_rep = bk.x;
          }
          tma_load_3d(tile, &tmaps[bk.x], 4 * bz * B, by * B, bx * B, &full[k]);
        } else if (lane == 1) {
          bulk_g2s(rec, W + static_cast<long long>(s0) * WS,
                   static_cast<unsigned>(cn * WS * sizeof(Real)), &full[k]);
        } else if (lane == 2) {
          bulk_g2s(keys, s_key + a0, static_cast<unsigned>((a1 - a0) * sizeof(int)), &full[k]);
        } else if (lane == 3) {
          bulk_g2s(pm, perm + a0, static_cast<unsigned>((a1 - a0) * sizeof(int)), &full[k]);
        }
        ++it;
      }
      int s0n = 0, s1n = 0;
      if (nn < nbricks) {
        const int *st = start + reps[bkn.x].brk_off;
        s0n = st[bkn.y];
        s1n = st[bkn.y + 1];
      }
      bk = bkn;
      s0 = s0n;
      s1 = s1n;
    }
    // end marker for the consumers
    if (ok) {
      int const k = it % S;
      bool const got = mbar_wait(&empty[k], ((it / S) & 1) ^ 1u);
      if (__all_sync(0xffffffffu, got)) {
        if (lane == 0)
          s_info[k].rep = -1;
        mbar_arrive(&full[k]);
      } else {
        ok = false;
      }
    }
    if (!ok) {
      if (lane == 0)
        atomicExch(err, 1);
      // bounded wait for the fills that may still be in flight
      for (int j = max(0, it - S); j < it; ++j)
        mbar_wait(&full[j % S], (j / S) & 1);
    }
    return;
  }

  // ---------------- consumers ----------------
  int const cw = warp - 1, g = lane >> 3, kz = lane & 7;
  for (int it = 0;; ++it) {
    int const k = it % S;
    bool const got = mbar_wait(&full[k], (it / S) & 1);
    if (!__all_sync(0xffffffffu, got)) {
      if (lane == 0)
        atomicExch(err, 1);
      return;
    }
    InterpInfo const inf = s_info[k];
    if (inf.rep < 0)
      return;
    unsigned char *sp = stage_ptr(k);
    const R4 *tile = reinterpret_cast<const R4 *>(sp);
    const Real *rec = reinterpret_cast<const Real *>(sp + L::tile);
    const int *keys = reinterpret_cast<const int *>(sp + L::tile + L::rec);
    const int *pm = reinterpret_cast<const int *>(sp + L::tile + L::rec + L::ids);
    int const s0 = inf.s0, s1 = inf.s1, a0 = s0 & ~3;
    // four particles per warp (one per 8-lane group), warps interleaved
    for (int sb = s0 + 4 * cw; sb < s1; sb += 4 * CW) {
      int const s = sb + g, j = s - s0;
      bool const live = s < s1;
      Real ax = Real(0), ay = Real(0), az = Real(0);
      if (live && kz < P) {
        bool const staged = j < CAP;
        int const l = (staged ? keys[s - a0] : s_key[s]) - inf.brick * B3;
        int const lb = __ffs(B) - 1; // B is a power of two
        int const lx = l >> (2 * lb), ly = (l >> lb) & (B - 1), lz = l & (B - 1);
        const Real *w = staged ? rec + j * WS : W + static_cast<long long>(s) * WS;
        Real wx[P], wy[P];
#pragma unroll
        for (int kk = 0; kk < P; ++kk) {
          wx[kk] = w[kk];
          wy[kk] = w[P + kk];
        }
        Real const wzk = w[WZ + kz];
        const R4 *tp = tile + (lx * Ed + ly) * Ed + lz + kz;
#pragma unroll
        for (int kx = 0; kx < P; ++kx) {
          Real const wxz = wx[kx] * wzk;
#pragma unroll
          for (int ky = 0; ky < P; ++ky) {
            R4 const e = tp[(kx * Ed + ky) * Ed];
            Real const wt = wxz * wy[ky];
            ax += wt * e.x;
            ay += wt * e.y;
            az += wt * e.z;
          }
        }
      }
      double fx = static_cast<double>(ax), fy = static_cast<double>(ay),
             fz = static_cast<double>(az);
#pragma unroll
      for (int o = 1; o < 8; o <<= 1) {
        fx += __shfl_xor_sync(0xffffffffu, fx, o);
        fy += __shfl_xor_sync(0xffffffffu, fy, o);
        fz += __shfl_xor_sync(0xffffffffu, fz, o);
      }
      if (live && kz == 0) {
        int const i = (j < CAP) ? pm[s - a0] : perm[s];
        double ox = -inf.pref * fx, oy = -inf.pref * fy, oz = -inf.pref * fz;
        if (inf.cdip != 0.0) {
          double const qi = q[i];
          ox -= qi * inf.cdip * dipole[3 * inf.rep + 0];
          oy -= qi * inf.cdip * dipole[3 * inf.rep + 1];
          oz -= qi * inf.cdip * dipole[3 * inf.rep + 2];
        }
        if (overwrite) {
          f[3 * i + 0] = ox;
          f[3 * i + 1] = oy;
          f[3 * i + 2] = oz;
        } else {
          f[3 * i + 0] += ox;
          f[3 * i + 1] += oy;
          f[3 * i + 2] += oz;
        }
      }
    }
    __syncwarp();
    if (lane == 0)
      mbar_arrive(&empty[k]);
  }
}

// sinc with the Taylor branch of p3m/math.hpp:53-81.
__device__ inline double sinc_d(double x) {
  double const pix = kPi * x;
  if (fabs(x) > 0.1)
    return sin(pix) / pix;
  double const p2 = pix * pix;
  return 1.0 + p2 * (-1.0 / 6.0 + p2 * (1.0 / 120.0 + p2 * (-1.0 / 5040.0 + p2 * (1.0 / 362880.0))));
}

// Optimal influence function on the r2c half mesh for m = 0 aliasing
// (G_opt<S,0>, p3m/influence_function.hpp:53-150): computed in FP64,
// stored in the working precision.  With m = 0 the force (S=1) and energy
// (S=0) functions are identical, so one array serves both.
template <typename Real>
__global__ void k_influence(const RepGeom *__restrict__ reps, const int2 *__restrict__ blk,
                            Real *__restrict__ ginf) {
  int2 const bk = blk[blockIdx.x];
  RepGeom const &G = reps[bk.x];
  int const M0 = G.mesh[0], M1 = G.mesh[1], M2 = G.mesh[2];
  long long const local = static_cast<long long>(bk.y) * blockDim.x + threadIdx.x;
  long long const csize = static_cast<long long>(M0) * M1 * G.hp;
  if (local >= csize)
    return;
  int const kz = static_cast<int>(local % G.hp);
  int const y = static_cast<int>((local / G.hp) % M1);
  int const x = static_cast<int>(local / (static_cast<long long>(M1) * G.hp));
  double val = 0.0;
  if (kz <= M2 / 2) {
    bool const all_half = (x % (M0 / 2) == 0) && (y % (M1 / 2) == 0) && (kz % (M2 / 2) == 0);
    if (!all_half) {
      auto shift = [](int i, int m) { return (i < m / 2) ? i : i - m; }; // M/2 -> -M/2
      int const sh[3] = {shift(x, M0), shift(y, M1), shift(kz, M2)};
      double k[3], fnm[3];
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        k[d] = sh[d] * ((2.0 * kPi) * G.box_i[d]);
        double const h = G.box[d] / G.mesh[d];
        double const wvi = 1.0 / ((2.0 * kPi) / h);
        fnm[d] = sinc_d(k[d] * wvi);
      }
      double const k2 = k[0] * k[0] + k[1] * k[1] + k[2] * k[2];
      if (k2 != 0.0) {
        double const U2 = pow(fnm[0] * fnm[1] * fnm[2], 2.0 * G.cao);
        double const ex = (1.0 / (2.0 * G.alpha)) * (1.0 / (2.0 * G.alpha)) * k2;
        double num = 0.0;
        if (ex < 30.0)
          num = U2 * (exp(-ex) * (4.0 * kPi / k2));
        val = num / (U2 * U2);
      }
    }
  }
  ginf[G.km_off + local] = static_cast<Real>(val);
}

// Per-block FP64 partial sums over particles of one replica:
// {n_charged, sum q, sum q^2, Mx, My, Mz} (p3m.cpp:98-115, 376-386).
__global__ void k_census(const int2 *__restrict__ blk, const RepGeom *__restrict__ reps,
                         const double *__restrict__ pos, const double *__restrict__ q,
                         double *__restrict__ partials) {
  int2 const bk = blk[blockIdx.x];
  RepGeom const &G = reps[bk.x];
  long long const i0 = G.p0 + static_cast<long long>(bk.y) * 2048;
  long long const i1 = min(G.p0 + G.np, i0 + 2048);
  double acc[6] = {0, 0, 0, 0, 0, 0};
  for (long long i = i0 + threadIdx.x; i < i1; i += blockDim.x) {
    double const qi = q[i];
    if (qi != 0.0) {
      acc[0] += 1.0;
      acc[1] += qi;
      acc[2] += qi * qi;
      acc[3] += qi * pos[3 * i + 0];
      acc[4] += qi * pos[3 * i + 1];
      acc[5] += qi * pos[3 * i + 2];
    }
  }
  __shared__ double red[6][32];
  int const lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < 6; ++k) {
    double v = acc[k];
    for (int o = 16; o > 0; o >>= 1)
      v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0)
      red[k][wid] = v;
  }
  __syncthreads();
  if (threadIdx.x < 6) {
    double s = 0.0;
    for (int w = 0; w < (blockDim.x >> 5); ++w)
      s += red[threadIdx.x][w];
    partials[static_cast<long long>(blockIdx.x) * 6 + threadIdx.x] = s;
  }
}

// Sum per-block partials of each replica in block order (deterministic).
__global__ void k_reduce_partials(const double *__restrict__ partials, int width,
                                  const int *__restrict__ blk_start, int n_rep,
                                  double *__restrict__ out) {
  int const r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n_rep)
    return;
  for (int k = 0; k < width; ++k) {
    double s = 0.0;
    for (int b = blk_start[r]; b < blk_start[r + 1]; ++b)
      s += partials[static_cast<long long>(b) * width + k];
    out[static_cast<long long>(r) * width + k] = s;
  }
}

// Closed-form aliasing sum sum_m sinc^(2P)(n/M + m) (Hockney & Eastwood
// eq. 7-66, p3m/math.hpp:92-149).
__device__ inline double cot_sum(int cao, int n, double mesh_i) {
  double const th = static_cast<double>(n) * mesh_i * kPi;
  double const c = cos(th) * cos(th);
  switch (cao) {
  case 1: return 1.0;
  case 2: return (1. + c * 2.) / 3.;
  case 3: return (2. + c * (11. + c * 2.)) / 15.;
  case 4: return (17. + c * (180. + c * (114. + c * 4.))) / 315.;
  case 5: return (62. + c * (1072. + c * (1452. + c * (247. + c * 2.)))) / 2835.;
  case 6:
    return (1382. + c * (35396. + c * (83021. + c * (34096. + c * (2026. + c * 4.))))) / 155925.;
  default:
    return (21844. + c * (776661. + c * (2801040. + c * (2123860. + c * (349500. + c * (8166. + c * 4.)))))) /
           6081075.;
  }
}

// Hockney-Eastwood k-space error sum in FP64 (p3m_k_space_error with
// p3m_tune_aliasing_sums, p3m.cpp:146-243; the GPU version of
// p3m_gpu_error_cuda.cu:47-143), per-block partials, fixed-order reduce.
__global__ void k_ks_error(int M0, int M1, int M2, int cao, double alpha_L,
                           double *__restrict__ partials) {
  long long const total = static_cast<long long>(M0) * M1 * M2;
  double const mi0 = 1.0 / M0, mi1 = 1.0 / M1, mi2 = 1.0 / M2;
  double const f1 = (kPi / alpha_L) * (kPi / alpha_L);
  double acc = 0.0;
  for (long long t = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; t < total;
       t += static_cast<long long>(gridDim.x) * blockDim.x) {
    int const nz = static_cast<int>(t % M2) - M2 / 2;
    int const ny = static_cast<int>((t / M2) % M1) - M1 / 2;
    int const nx = static_cast<int>(t / (static_cast<long long>(M1) * M2)) - M0 / 2;
    if (nx == 0 && ny == 0 && nz == 0)
      continue;
    double const n2 = double(nx) * nx + double(ny) * ny + double(nz) * nz;
    double const cs = cot_sum(cao, nx, mi0) * cot_sum(cao, ny, mi1) * cot_sum(cao, nz, mi2);
    double const ex = exp(-f1 * n2);
    double const en = pow(sinc_d(nx * mi0) * sinc_d(ny * mi1) * sinc_d(nz * mi2), 2.0 * cao);
    double const a1 = ex * ex / n2;
    double const a2 = en * ex * n2 / n2;
    double const d = a1 - (a2 / cs) * (a2 / cs) / n2;
    if (d > 0.0 && fabs(d / a1) > 1e-14)
      acc += d;
  }
  __shared__ double red[32];
  for (int o = 16; o > 0; o >>= 1)
    acc += __shfl_down_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0)
    red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < (blockDim.x >> 5); ++w)
      s += red[w];
    partials[blockIdx.x] = s;
  }
}

} // namespace p3mx

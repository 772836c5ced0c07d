// Short-range path (sm_100a): regular-decomposition cell binning, Verlet
// list build, and the real-space erfc-Coulomb + LJ/WCA pair kernel.
#pragma once

#include "common.cuh"
#include "p3m_kernels.cuh"

#include <type_traits>

namespace p3mx {

// LJ/WCA parameters of a type pair, device copy (lj.hpp, wca.hpp).
struct PairIA {
  double lj_eps, lj_sig, lj_cut, lj_shift, lj_offset, lj_min;
  double wca_eps, wca_sig, wca_cut;
  double ia_cut; // max of active cutoffs, -1 when inactive
};

// FP32 offset of a particle from the corner of cell `loc` (cell index inside
// the replica) that it was binned into at the last list build: the folded
// build-time position minus the corner, plus the minimum-image displacement
// since the build (below skin/2 by the Verlet rebuild rule), so the offset
// stays continuous when the particle leaves its cell or crosses the box
// boundary, for any cell grid.  At build time xref = x.
__device__ inline float4 cell_offset(RepGeom const &G, int loc, const double *xref,
                                     const double *x, double q) {
  int const c[3] = {loc % G.cg[0], (loc / G.cg[0]) % G.cg[1], loc / (G.cg[0] * G.cg[1])};
  float o[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    double const cs = G.box[d] / G.cg[d];
    double const v = fold_coord(xref[d], G.box[d]) - c[d] * cs;
    double dd = x[d] - xref[d];
    dd -= G.box[d] * rint(dd * G.box_i[d]);
    o[d] = static_cast<float>(v + dd);
  }
  return make_float4(o[0], o[1], o[2], static_cast<float>(q));
}

// Cell of a folded position, position_to_cell_index
// (RegularDecomposition.cpp:51-80) on a single rank: floor(x/cell)+1,
// clamped to the grid for x < L.  Returns interior coordinates 0..cg-1.
__device__ inline void cell_coords(RepGeom const &G, const double *xf, int *c) {
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    int cp = static_cast<int>(floor(xf[d] * G.inv_cs[d])) + 1;
    if (cp < 1)
      cp = 1;
    else if (cp > G.cg[d])
      cp = G.cg[d];
    c[d] = cp - 1;
  }
}

// Cell key (column-major over the interior grid, x fastest, as the
// reference orders cells) and counting-sort slot of every particle; also
// the folded position (double4 with charge in w) for the pair kernels.  The
// sort runs on G.oct_mult keys per cell (8 when any replica sorts by
// octant, else 1): cell * oct_mult + the octant of the cell the particle
// lies in (each axis halved) where the replica sorts by octant (G.oct_on:
// crowded cells, whose far octants the list build skips), else
// cell * oct_mult; bkey keeps the sort key.
__global__ void k_cell_bin(const RepGeom *__restrict__ reps, const int *__restrict__ rep_of,
                           const double *__restrict__ pos, const double *__restrict__ q,
                           long long n, int *__restrict__ key, int *__restrict__ bkey,
                           int *__restrict__ slot, int *__restrict__ cnt,
                           double4 *__restrict__ pq, int *__restrict__ ghost_index,
                           const int *__restrict__ cond, const int *__restrict__ rflag) {
  if (cond && !*cond)
    return;
  long long const i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n)
    return;
  RepGeom const &G = reps[rep_of[i]];
  double xf[3];
#pragma unroll
  for (int d = 0; d < 3; ++d)
    xf[d] = fold_coord(pos[3 * i + d], G.box[d]);
  int c[3];
  cell_coords(G, xf, c);
  int kb;
  if (rflag && !rflag[rep_of[i]]) {
    // replica keeps its lists: same cells, hence the same sorted order
    kb = bkey[i];
  } else {
    int const k = static_cast<int>(G.cell_off) + c[0] + G.cg[0] * (c[1] + G.cg[1] * c[2]);
    int oct = 0;
    if (G.oct_on) {
#pragma unroll
      for (int d = 0; d < 3; ++d)
        oct |= (xf[d] * G.inv_cs[d] - c[d] >= 0.5) ? (1 << d) : 0;
    }
    kb = G.oct_mult * k + oct;
    key[i] = k;
    bkey[i] = kb;
  }
  slot[i] = atomicAdd(&cnt[kb], 1);
  pq[i] = make_double4(xf[0], xf[1], xf[2], q[i]);
  if (ghost_index) {
    int const g0 = G.cg[0] + 2, g1 = G.cg[1] + 2;
    ghost_index[i] = (c[0] + 1) + g0 * ((c[1] + 1) + g1 * (c[2] + 1));
  }
}

// Gather particle data into cell-sorted order (and the inverse permutation).
__global__ void k_cell_gather(const RepGeom *__restrict__ reps, const int *__restrict__ rep_of,
                              const int *__restrict__ perm, const double4 *__restrict__ pq,
                              const int *__restrict__ type, const int *__restrict__ key,
                              long long n, double4 *__restrict__ spq, float4 *__restrict__ spf,
                              int *__restrict__ stype, int *__restrict__ scell,
                              int *__restrict__ inv, const int *__restrict__ cond) {
  if (cond && !*cond)
    return;
  long long const s = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (s >= n)
    return;
  int const i = perm[s];
  inv[i] = static_cast<int>(s); // sorted slot of particle i
  double4 const v = pq[i];
  spq[s] = v;
  stype[s] = type ? type[i] : 0;
  scell[s] = key[i];
  RepGeom const &G = reps[rep_of[i]];
  double const xv[3] = {v.x, v.y, v.z};
  spf[s] = cell_offset(G, key[i] - static_cast<int>(G.cell_off), xv, xv, v.w);
}

__device__ inline double mi_d(double dx, double L, double Li) {
  // get_mi_coord (BoxGeometry.hpp:47-60)
  if (fabs(dx) > 0.5 * L)
    return dx - rint(dx * Li) * L;
  return dx;
}

// Verlet list layout: per warp tile of 32 consecutive particles of a replica,
// each particle's entries in groups of 8 (one 32-byte sector), the groups of
// the 32 particles interleaved: entry k of local particle la at
//   nb_off + ((la/32) * (cap/8) + k/8) * 256 + (la%32) * 8 + k%8
// (cap, the per-replica capacity, a multiple of 8).  The build writes whole
// groups with vector stores and the pair kernels read whole groups with
// vector loads.  An entry packs the partner's index inside the replica
// (26 bits) and its cell offset code (cell_offset_code, 6 bits).
constexpr int kNbIndexBits = 26;
constexpr unsigned kNbIndexMask = (1u << kNbIndexBits) - 1u;
// Cell offset code of an entry: the partner image's cell offset dc (each
// axis -1, 0 or +1) as three 2-bit fields dc + 1 (x lowest), in the 6 bits
// above the index.
__host__ __device__ constexpr int cell_offset_code(int dx, int dy, int dz) {
  return (dx + 1) | ((dy + 1) << 2) | ((dz + 1) << 4);
}
// dc of axis d from a code, as an FP32 value (exact: 2^23 + field, minus
// 2^23 + 1)
__device__ inline float code_axis(unsigned code, int d) {
  return __uint_as_float(0x4B000000u | ((code >> (2 * d)) & 3u)) - 8388609.0f;
}
// First entry (group 0) of local particle la; group g at + g * 256.
__host__ __device__ inline long long nb_base(long long nb_off, int cap, long long la) {
  return nb_off + (((la >> 5) * (cap >> 3)) << 8) + ((la & 31) << 3);
}
__host__ __device__ inline long long nb_entry(long long base, int k) {
  return base + (static_cast<long long>(k >> 3) << 8) + (k & 7);
}
// Two classes of entries share a particle's capacity: class A (the pair's
// LJ / WCA range plus the skin at build time: all terms) fills groups from
// the first one up, class B (beyond it: the pair stays outside the LJ / WCA
// cutoff until the next rebuild, as no particle moves more than skin/2, so
// only Coulomb can act) fills groups from the last one down.  nb_cnt packs
// nA (low 16 bits) and nB (high 16 bits).
__host__ __device__ inline int nb_count_a(int c) { return c & 0xFFFF; }
__host__ __device__ inline int nb_count_b(int c) { return static_cast<int>(static_cast<unsigned>(c) >> 16); }
__host__ __device__ inline int nb_count(int c) { return nb_count_a(c) + nb_count_b(c); }
// Group g of class B (g = 0 the first).
__host__ __device__ inline long long nb_group_b(long long base, int cap, int g) {
  return base + (static_cast<long long>((cap >> 3) - 1 - g) << 8);
}
// Entry k of the logical list [class A entries, class B entries].
__host__ __device__ inline long long nb_logical(long long base, int cap, int na, int k) {
  if (k < na)
    return nb_entry(base, k);
  int const kk = k - na;
  return nb_group_b(base, cap, kk >> 3) + (kk & 7);
}

// Copy one group of 8 entries (32 bytes, 16-byte aligned on both sides).
__device__ inline void store_group(int *p, const int *g) {
  reinterpret_cast<int4 *>(p)[0] = reinterpret_cast<const int4 *>(g)[0];
  reinterpret_cast<int4 *>(p)[1] = reinterpret_cast<const int4 *>(g)[1];
}

// Verlet list (full, both directions) of every cell-sorted particle a:
// partners b != a in the 27 (unique) neighbour cells with the
// VerletCriterion (VerletCriterion.hpp:68-97): d^2 <= (max_cut+skin)^2 and
// (both charged and d^2 <= (r_cut+skin)^2, or the type pair is active and
// d^2 <= (ia_cut+skin)^2).  Stored in the warp-tiled layout above
// (per-replica capacity G.max_nb), class A entries (type pair active and
// d^2 <= (ia_cut+skin)^2) from the first group up, class B from the last
// group down; a replica whose capacity is exceeded reports the capacity it
// needs in overflow[replica] (nothing more is stored for that particle and
// its counts are those of the entries stored).
// Verlet list of one cell-sorted particle a (k_verlet_build); gbuf / gbuf_b
// are the lane's shared-memory buffers of the class A / B group being
// filled, s_icut the ia_cut table of the type pairs in shared memory.
template <bool OCT>
__device__ inline void verlet_build_one(long long a, const RepGeom *__restrict__ reps,
                                        const int *__restrict__ rep_of_sorted,
                                        const double4 *__restrict__ spq,
                                        const float4 *__restrict__ spf,
                                        const int *__restrict__ stype,
                                        const int *__restrict__ scell,
                                        const int *__restrict__ cstart,
                                        const PairIA *__restrict__ ia, int ntypes,
                                        int *__restrict__ nb, int *__restrict__ nb_cnt,
                                        int *__restrict__ overflow,
                                        const int *__restrict__ rflag, const float *s_icut,
                                        int *gbuf, int *gbuf_b) {
  int const rep = rep_of_sorted[a];
  if (rflag && !rflag[rep])
    return; // this replica keeps its list
  RepGeom const &G = reps[rep];
  int const max_nb = G.max_nb;
  int *nbp = nb + nb_base(G.nb_off, max_nb, a - G.p0);
  int const ngroups = max_nb >> 3;
  double4 const pa = spq[a];
  double const cs[3] = {G.box[0] / G.cg[0], G.box[1] / G.cg[1], G.box[2] / G.cg[2]};
  double const ics[3] = {G.cg[0] * G.box_i[0], G.cg[1] * G.box_i[1], G.cg[2] * G.box_i[2]};
  bool const small_grid = (G.cg[0] < 3) || (G.cg[1] < 3) || (G.cg[2] < 3);
  // FP32 geometry on the cell-relative offsets (error ~1e-6 of the cell
  // size): a candidate whose FP32 distance lies within a relative band of
  // 1e-4 around one of its thresholds is decided by the FP64 minimum-image
  // test (the reference's criterion); all others are decided in FP32, which
  // cannot differ from FP64 outside the band, so the pair set is the FP64 one
  float4 const pfa = spf[a];
  float const csf[3] = {static_cast<float>(cs[0]), static_cast<float>(cs[1]),
                        static_cast<float>(cs[2])};
  int const ta = stype[a];
  int const loc = scell[a] - static_cast<int>(G.cell_off);
  int const c0 = loc % G.cg[0];
  int const c1 = (loc / G.cg[0]) % G.cg[1];
  int const c2 = loc / (G.cg[0] * G.cg[1]);
  double const emax2 = (G.max_cut + G.skin) * (G.max_cut + G.skin);
  float const emax2_pre = static_cast<float>(emax2 * (1.0 + 1e-4));
  double const ecoul2 = (G.coulomb_cut > 0.0) ? (G.coulomb_cut + G.skin) * (G.coulomb_cut + G.skin) : -1.0;
  // Coulomb threshold band in FP32 (no Coulomb pairs when a is uncharged)
  bool const coul_a = ecoul2 >= 0.0 && pa.w != 0.0;
  float const ec_lo = static_cast<float>(ecoul2 * (1.0 - 1e-4));
  float const ec_hi = static_cast<float>(ecoul2 * (1.0 + 1e-4));
  float const skin_f = static_cast<float>(G.skin);
  double const Li[3] = {G.box_i[0], G.box_i[1], G.box_i[2]};
  int na = 0, nb_b = 0; // entries stored per class
  int need_a = 0, need_b = 0; // entries found per class
  // store one taken entry of class A (LJ / WCA range) or B
  auto put = [&](int b, bool cls_a, int code) {
    // room for the entry: class A groups [0, ceil(na'/8)) and class B
    // groups [ngroups - ceil(nb'/8), ngroups) disjoint
    bool const room = (need_a == na) && (need_b == nb_b) &&
                      ((cls_a ? (na & 7) : (nb_b & 7)) != 0 ||
                       ((na + 7) >> 3) + ((nb_b + 7) >> 3) + 1 <= ngroups);
    if (room) {
      int const ent = static_cast<int>(static_cast<unsigned>(b - G.p0) |
                                       (static_cast<unsigned>(code) << kNbIndexBits));
      if (cls_a) {
        int const slot = na & 7;
        gbuf[slot] = ent;
        if (slot == 7)
          store_group(nbp + (static_cast<long long>(na >> 3) << 8), gbuf);
        ++na;
      } else {
        int const slot = nb_b & 7;
        gbuf_b[slot] = ent;
        if (slot == 7)
          store_group(nbp + (static_cast<long long>(ngroups - 1 - (nb_b >> 3)) << 8), gbuf_b);
        ++nb_b;
      }
    }
    if (cls_a)
      ++need_a;
    else
      ++need_b;
  };
  // offsets per axis without duplicates for grids of size 1 or 2
  int lo[3], hi[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    lo[d] = (G.cg[d] >= 3) ? -1 : 0;
    hi[d] = (G.cg[d] >= 2) ? 1 : 0;
  }
  for (int dz = lo[2]; dz <= hi[2]; ++dz) {
    int z = c2 + dz;
    z = (z < 0) ? z + G.cg[2] : (z >= G.cg[2] ? z - G.cg[2] : z);
    for (int dy = lo[1]; dy <= hi[1]; ++dy) {
      int y = c1 + dy;
      y = (y < 0) ? y + G.cg[1] : (y >= G.cg[1] ? y - G.cg[1] : y);
      for (int dx = lo[0]; dx <= hi[0]; ++dx) {
        int x = c0 + dx;
        x = (x < 0) ? x + G.cg[0] : (x >= G.cg[0] ? x - G.cg[0] : x);
        int const cell = static_cast<int>(G.cell_off) + x + G.cg[0] * (y + G.cg[1] * z);
        if (!small_grid) {
          // skip a neighbour cell lying wholly beyond the list range: distance
          // from the particle (cell-relative offset) to the cell's box
          float const ax = (dx == 0) ? 0.f : (dx > 0 ? csf[0] - pfa.x : pfa.x);
          float const ay = (dy == 0) ? 0.f : (dy > 0 ? csf[1] - pfa.y : pfa.y);
          float const az = (dz == 0) ? 0.f : (dz > 0 ? csf[2] - pfa.z : pfa.z);
          float const bx = fmaxf(ax, 0.f), by = fmaxf(ay, 0.f), bz = fmaxf(az, 0.f);
          if (bx * bx + by * by + bz * bz > emax2_pre)
            continue;
        }
        float const shx = -dx * csf[0], shy = -dy * csf[1], shz = -dz * csf[2];
        // exact (FP64 minimum-image) test and store of one candidate
        auto consider = [&](int b) {
            double4 const pb = spq[b];
            double const d0 = mi_d(pa.x - pb.x, G.box[0], Li[0]);
            double const d1 = mi_d(pa.y - pb.y, G.box[1], Li[1]);
            double const d2v = mi_d(pa.z - pb.z, G.box[2], Li[2]);
            double const d2 = d0 * d0 + d1 * d1 + d2v * d2v;
            if (d2 > emax2)
              return;
            double const ic = ia[ta * ntypes + stype[b]].ia_cut;
            bool const cls_a = (ic != -1.0) && d2 <= (ic + G.skin) * (ic + G.skin);
            bool const take =
                cls_a || (ecoul2 >= 0.0 && d2 <= ecoul2 && pa.w != 0.0 && pb.w != 0.0);
            if (take) {
              // cell offset dc of the partner's image: x_b' - x_a = dc cs +
              // (off_b - off_a), an exact multiple of the cell size; with
              // cells >= the list range, dc is -1, 0 or +1 per axis.  With
              // 3 or more cells along an axis the minimum image is the image
              // in the visited neighbour cell, so dc is the loop offset;
              // with 1 or 2 cells it follows from the minimum-image vector.
              int dcv[3] = {dx, dy, dz};
              if (small_grid) {
                int const lb = scell[b] - static_cast<int>(G.cell_off);
                int const cb[3] = {lb % G.cg[0], (lb / G.cg[0]) % G.cg[1],
                                   lb / (G.cg[0] * G.cg[1])};
                int const ca[3] = {c0, c1, c2};
                double const xa[3] = {pa.x, pa.y, pa.z}, xb[3] = {pb.x, pb.y, pb.z};
                double const dmi[3] = {-d0, -d1, -d2v};
#pragma unroll
                for (int d = 0; d < 3; ++d)
                  if (G.cg[d] < 3) {
                    double const oa = xa[d] - ca[d] * cs[d], ob = xb[d] - cb[d] * cs[d];
                    dcv[d] = static_cast<int>(rint((dmi[d] - (ob - oa)) * ics[d]));
                  }
              }
              put(b, cls_a, cell_offset_code(dcv[0], dcv[1], dcv[2]));
            }
        };
        if (small_grid) {
          int const om = G.oct_mult;
          int const b_lo = cstart[om * cell], b_hi = cstart[om * cell + om];
          for (int b = b_lo; b < b_hi; ++b)
            if (b != a)
              consider(b);
        } else {
          int const code = cell_offset_code(dx, dy, dz);
          // with octant-sorted cells, the octants of the neighbour cell
          // wholly beyond the list range are skipped (the particle relative
          // to the neighbour cell's corner against each half-cell box)
          float const qx = pfa.x + shx, qy = pfa.y + shy, qz = pfa.z + shz;
          float const hx = 0.5f * csf[0], hy = 0.5f * csf[1], hz = 0.5f * csf[2];
          int const noct = (OCT && G.oct_on) ? 8 : 1;
          for (int oct = 0; oct < noct; ++oct) {
          int b_lo = cstart[G.oct_mult * cell], b_hi = cstart[G.oct_mult * (cell + 1)];
          if (OCT && G.oct_on) {
            float const lx = (oct & 1) ? hx : 0.f, ly = (oct & 2) ? hy : 0.f,
                        lz = (oct & 4) ? hz : 0.f;
            float const ex = fmaxf(fmaxf(lx - qx, qx - (lx + hx)), 0.f);
            float const ey = fmaxf(fmaxf(ly - qy, qy - (ly + hy)), 0.f);
            float const ez = fmaxf(fmaxf(lz - qz, qz - (lz + hz)), 0.f);
            if (ex * ex + ey * ey + ez * ez > emax2_pre)
              continue;
            b_lo = cstart[G.oct_mult * cell + oct];
            b_hi = cstart[G.oct_mult * cell + oct + 1];
          }
          // kPre candidates per round (loads issued together): an FP32
          // pre-check, then for the candidates near or inside the list
          // range the FP32 decision, or the FP64 test inside the bands
          constexpr int kPre = 8;
          for (int b0 = b_lo; b0 < b_hi; b0 += kPre) {
            float4 pf[kPre];
#pragma unroll
            for (int u = 0; u < kPre; ++u)
              pf[u] = (b0 + u < b_hi) ? spf[b0 + u] : pfa;
            unsigned keep = 0;
            float r2v[kPre];
#pragma unroll
            for (int u = 0; u < kPre; ++u) {
              float const e0 = (pfa.x - pf[u].x) + shx, e1 = (pfa.y - pf[u].y) + shy,
                          e2 = (pfa.z - pf[u].z) + shz;
              r2v[u] = e0 * e0 + e1 * e1 + e2 * e2;
              bool const in = (b0 + u < b_hi) && (b0 + u != a) && (r2v[u] <= emax2_pre);
              keep |= (in ? 1u : 0u) << u;
            }
            while (keep) {
              int const u = __ffs(keep) - 1;
              keep &= keep - 1;
              int const b = b0 + u;
              float r2 = r2v[0];
              float qb = pf[0].w;
#pragma unroll
              for (int w = 1; w < kPre; ++w) {
                r2 = (u == w) ? r2v[w] : r2;
                qb = (u == w) ? pf[w].w : qb;
              }
              float const icf = (ntypes == 1) ? s_icut[0] : s_icut[ta * ntypes + stype[b]];
              float const it = icf + skin_f;
              float const it2 = it * it;
              bool const ia_on = icf != -1.f;
              bool const a_lo = ia_on && r2 < it2 * (1.f - 1e-4f);
              bool const a_band = ia_on && !a_lo && r2 <= it2 * (1.f + 1e-4f);
              // Coulomb: both charged (an FP32 zero charge is checked in FP64)
              bool const c_lo = coul_a && qb != 0.f && r2 < ec_lo;
              bool const c_band = coul_a && r2 <= ec_hi && !c_lo;
              if (a_band || c_band)
                consider(b);
              else if (a_lo || c_lo)
                put(b, a_lo, code);
            }
          }
          }
        }
      }
    }
  }
  // last partial groups (entries beyond the counts are never read)
  if (na & 7)
    store_group(nbp + (static_cast<long long>(na >> 3) << 8), gbuf);
  if (nb_b & 7)
    store_group(nbp + (static_cast<long long>(ngroups - 1 - (nb_b >> 3)) << 8), gbuf_b);
  nb_cnt[a] = na | (nb_b << 16);
  int const need = 8 * (((need_a + 7) >> 3) + ((need_b + 7) >> 3));
  if (need > max_nb)
    atomicMax(&overflow[rep], need);
}

// Verlet lists, one thread per cell-sorted particle (the 32 lanes of a warp
// are consecutive particles: the same or adjacent cells).
template <bool OCT>
__global__ void __launch_bounds__(256, 2)
k_verlet_build(const RepGeom *__restrict__ reps, const int *__restrict__ rep_of_sorted,
               const double4 *__restrict__ spq, const float4 *__restrict__ spf,
               const int *__restrict__ stype, const int *__restrict__ scell,
               const int *__restrict__ cstart, const PairIA *__restrict__ ia, int ntypes,
               long long n, int *__restrict__ nb, int *__restrict__ nb_cnt,
               int *__restrict__ overflow, const int *__restrict__ cond,
               const int *__restrict__ rflag) {
  if (cond && !*cond)
    return;
  __shared__ __align__(16) int s_group[256 * 8], s_group_b[256 * 8];
  // ia_cut of every type pair (-1: inactive) in shared memory (the skin,
  // per replica, is added per candidate)
  extern __shared__ float s_icut[];
  for (int k = threadIdx.x; k < ntypes * ntypes; k += blockDim.x)
    s_icut[k] = static_cast<float>(ia[k].ia_cut);
  __syncthreads();
  long long const a = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (a >= n)
    return;
  verlet_build_one<OCT>(a, reps, rep_of_sorted, spq, spf, stype, scell, cstart, ia, ntypes, nb,
                   nb_cnt, overflow, rflag, s_icut, s_group + threadIdx.x * 8,
                   s_group_b + threadIdx.x * 8);
}

// A&S 7.1.26 approximation of exp(d^2) erfc(d), as the reference's real-
// space kernel uses it (utils/math/AS_erfc_part.hpp:29-40).
template <typename Real> __device__ inline Real as_erfc_part(Real d) {
  Real const a1 = Real(0.254829592), a2 = Real(-0.284496736), a3 = Real(1.421413741),
             a4 = Real(-1.453152027), a5 = Real(1.061405429), p = Real(0.3275911);
  Real const t = Real(1) / (Real(1) + p * d);
  return t * (a1 + t * (a2 + t * (a3 + t * (a4 + t * a5))));
}

// FP32 exp(x) for the real-space kernel (x = -(alpha r)^2 in [-88, 0]):
// e^x = 2^y with y = x log2(e) split error-free into y_hi + y_lo (the FMA
// residual of the product, Dekker's TwoProduct, plus the low part of the
// constant), then 2^y = 2^y_hi (hardware ex2.approx, ~2 ulp) * (1 + y_lo ln 2).
// Relative error ~2^-21 over the range, against ~2^-24 * |y| for a plain
// ex2(x * log2 e).
__device__ inline float exp_fast(float x) {
  float const l2e_hi = 1.44269502162933349609375f;    // log2(e) rounded to FP32
  float const l2e_lo = 1.9259629911266175e-8f;        // log2(e) - l2e_hi
  float const y_hi = x * l2e_hi;
  float const y_lo = fmaf(x, l2e_hi, -y_hi) + x * l2e_lo;
  float e;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(e) : "f"(y_hi));
  return fmaf(e, y_lo * 0.693147180559945309f, e);
}
template <typename Real> __device__ inline Real exp_r(Real x);
template <> __device__ inline float exp_r<float>(float x) { return exp_fast(x); }
template <> __device__ inline double exp_r<double>(double x) { return exp(x); }
template <typename Real> __device__ inline Real sqrt_r(Real x);
template <> __device__ inline float sqrt_r<float>(float x) { return sqrtf(x); }
template <> __device__ inline double sqrt_r<double>(double x) { return sqrt(x); }

// Reciprocal / reciprocal square root in the working precision: FP32 uses
// the hardware approximations (~1 ulp; the FP32-mixed path tolerates
// ulp-level differences); FP64 keeps IEEE division and sqrt.
template <typename Real> __device__ inline Real rcp_r(Real x);
template <> __device__ inline float rcp_r<float>(float x) {
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}
template <> __device__ inline double rcp_r<double>(double x) { return 1.0 / x; }
template <typename Real> __device__ inline Real rsqrt_r(Real x);
template <> __device__ inline float rsqrt_r<float>(float x) { return rsqrtf(x); }
template <> __device__ inline double rsqrt_r<double>(double x) { return 1.0 / sqrt(x); }

// LJ/WCA parameters of one type pair in the working precision.
template <typename Real> struct PairR {
  Real lcut, lmin, loff, lsig, leps, lshift, wcut, wsig, weps;
  bool active;
  __device__ explicit PairR(PairIA const &p)
      : lcut(static_cast<Real>(p.lj_cut + p.lj_offset)),
        lmin(static_cast<Real>(p.lj_min + p.lj_offset)), loff(static_cast<Real>(p.lj_offset)),
        lsig(static_cast<Real>(p.lj_sig)), leps(static_cast<Real>(p.lj_eps)),
        lshift(static_cast<Real>(p.lj_shift)), wcut(static_cast<Real>(p.wca_cut)),
        wsig(static_cast<Real>(p.wca_sig)), weps(static_cast<Real>(p.wca_eps)),
        active(p.ia_cut != -1.0) {}
};

// LJ + WCA force factor and energy of one pair (lj.hpp:41-60, wca.hpp:39-55).
template <typename Real>
__device__ inline void lj_wca(PairR<Real> const &p, Real dist, Real inv_d, Real &fn, Real &en) {
  if (dist < p.lcut && dist > p.lmin) {
    Real const r_off = dist - p.loff;
    Real const inv_off = rcp_r(r_off);
    Real const s = p.lsig * inv_off;
    Real const s2 = s * s;
    Real const f6 = s2 * s2 * s2;
    fn += Real(48) * p.leps * f6 * (f6 - Real(0.5)) * (inv_off * inv_d);
    en += Real(4) * p.leps * (f6 * f6 - f6 + p.lshift);
  }
  if (dist < p.wcut) {
    Real const s = p.wsig * inv_d;
    Real const s2 = s * s;
    Real const f6 = s2 * s2 * s2;
    fn += Real(48) * p.weps * f6 * (f6 - Real(0.5)) * (inv_d * inv_d);
    en += Real(4) * p.weps * (f6 * f6 - f6 + Real(0.25));
  }
}

// Branch-free form of lj_wca for the FP32 kernel: every term is evaluated
// and selected by its range test (the lanes of a warp, different particles,
// would otherwise diverge on the tests); WCA only when the pair has it.
__device__ inline void lj_wca_sel(PairR<float> const &p, float dist, float inv_d, float &fn,
                                  float &en) {
  {
    float const r_off = dist - p.loff;
    float const inv_off = rcp_r(r_off);
    float const s = p.lsig * inv_off;
    float const s2 = s * s;
    float const f6 = s2 * s2 * s2;
    bool const in = dist < p.lcut && dist > p.lmin;
    fn += in ? 48.f * p.leps * f6 * (f6 - 0.5f) * (inv_off * inv_d) : 0.f;
    en += in ? 4.f * p.leps * (f6 * f6 - f6 + p.lshift) : 0.f;
  }
  if (p.wcut > 0.f) {
    float const s = p.wsig * inv_d;
    float const s2 = s * s;
    float const f6 = s2 * s2 * s2;
    bool const in = dist < p.wcut;
    fn += in ? 48.f * p.weps * f6 * (f6 - 0.5f) * (inv_d * inv_d) : 0.f;
    en += in ? 4.f * p.weps * (f6 * f6 - f6 + 0.25f) : 0.f;
  }
}

// Branch-free LJ + WCA for pairs without an LJ offset (r_off = r, so the
// LJ powers come from the same 1/r^2 as WCA's): one reciprocal square root
// serves every term.  in_lj / in_wca select the terms by range.
__device__ inline void lj_wca_sel_nooff(PairR<float> const &p, float dist, float inv_d2,
                                        float &fn) {
  {
    float const s2 = (p.lsig * p.lsig) * inv_d2;
    float const f6 = s2 * s2 * s2;
    bool const in = dist < p.lcut && dist > p.lmin;
    fn += in ? 48.f * p.leps * f6 * (f6 - 0.5f) * inv_d2 : 0.f;
  }
  if (p.wcut > 0.f) {
    float const s2 = (p.wsig * p.wsig) * inv_d2;
    float const f6 = s2 * s2 * s2;
    bool const in = dist < p.wcut;
    fn += in ? 48.f * p.weps * f6 * (f6 - 0.5f) * inv_d2 : 0.f;
  }
}

// 2^x, hardware approximation (ex2.approx, relative error ~2^-22).
__device__ inline float ex2_approx(float x) {
  float e;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(e) : "f"(x));
  return e;
}

// The FP32 exponentials of the real-space kernels on n values, for their
// accuracy test: out[k] = exp_fast(x), out[n + k] = one ex2.approx of
// x log2(e) rounded to FP32 (the form of the force-only kernel, which folds
// log2(e) into its coefficient), out[2n + k] = CUDA's expf(x).
__global__ void k_exp_check(long long n, const float *__restrict__ x, float *__restrict__ out) {
  long long const k = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (k >= n)
    return;
  float const v = x[k];
  out[k] = exp_fast(v);
  out[n + k] = ex2_approx(v * 1.44269504088896341f);
  out[2 * n + k] = expf(v);
}

__device__ inline float rsqrt_approx(float x) {
  float r;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

// Pair kernel over the Verlet list: real-space Coulomb
// (CoulombP3M::pair_force / pair_energy, p3m.hpp:146-180) plus LJ and WCA
// (lj.hpp:41-60, wca.hpp:39-55).  Minimum-image difference in FP64, pair
// arithmetic in Real, per-particle accumulation in FP64 (no atomics: each
// particle owns its force, full list).  EV adds energies and virials: each
// pair is seen from both ends, so per-particle sums are halved; per-block
// FP64 partials {E_coul, E_nb, Vc[9], Vn[9]} (width 20).  Blocks map to
// replicas through the block table so partials never straddle replicas.
// Neighbour loads are issued two entries ahead of their use.
// FP32-mixed real-space kernel over the same Verlet lists: positions are
// FP32 offsets from each particle's build-time cell corner (cell_offset), the
// list stores every partner's cell offset code, so
//   d = x_a - x_b' = (off_a - off_b) - dc * cs
// is formed in FP32 from small numbers (no minimum-image arithmetic, 16-byte
// gathers); the geometry error is about one ulp of the cell size.  Pair
// physics as k_pair_forces; per-particle force sums are FP32 over runs of 8
// partners and FP64 across runs.
// NOOFF: one particle type whose LJ has no offset (the host checks), so the
// LJ and WCA powers use the Coulomb term's 1/r^2 (lj_wca_sel_nooff).
template <bool EV, bool NOOFF = false>
__global__ void __launch_bounds__(256, EV ? 1 : 4)
k_pair_forces_rel(const RepGeom *__restrict__ reps, const int2 *__restrict__ blk,
                  const float4 *__restrict__ spf, const int *__restrict__ stype,
                  const int *__restrict__ perm, const PairIA *__restrict__ ia_g, int ntypes,
                  const int *__restrict__ nb, const int *__restrict__ nb_cnt,
                  double *__restrict__ f, int overwrite,
                  double *__restrict__ partials) {
  using Real = float;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  PairIA *ia = reinterpret_cast<PairIA *>(smem_raw);
  for (int k = threadIdx.x; k < ntypes * ntypes; k += blockDim.x)
    ia[k] = ia_g[k];
  int2 const bk = blk[blockIdx.x];
  RepGeom const &G = reps[bk.x];
  // cell sizes: the image shift of an entry is -dc cs per axis, dc from
  // its offset code (registers, no table lookup per entry)
  float const cs_x = static_cast<float>(G.box[0] / G.cg[0]);
  float const cs_y = static_cast<float>(G.box[1] / G.cg[1]);
  float const cs_z = static_cast<float>(G.box[2] / G.cg[2]);
  __syncthreads();
  long long const a = G.p0 + static_cast<long long>(bk.y) * blockDim.x + threadIdx.x;
  double ev[EV ? 20 : 1];
#pragma unroll
  for (int k = 0; k < (EV ? 20 : 1); ++k)
    ev[k] = 0.0;
  bool const active = a < G.p0 + G.np;
  // groups of 8 entries: class A first (all terms), then class B
  // (Coulomb only); the loop runs to the warp's largest group count so that
  // the vote on LJ stays warp-wide
  int na = 0, nbb = 0;
  if (active) {
    int const c = nb_cnt[a];
    na = nb_count_a(c);
    nbb = nb_count_b(c);
  }
  int const ga = (na + 7) >> 3, gt = ga + ((nbb + 7) >> 3);
  int const gmax = __reduce_max_sync(0xffffffffu, gt);
  float4 const pa = active ? spf[a] : make_float4(0.f, 0.f, 0.f, 0.f);
  int const ta = active ? stype[a] : 0;
  Real const rc2 = static_cast<Real>(G.r_cut * G.r_cut);
  Real const two_a_sqrt_pi_i = static_cast<Real>(2.0 * G.alpha / sqrt(kPi));
  Real const pref_qa = static_cast<Real>(G.prefactor) * pa.w;
  // exp(-(alpha r)^2) = 2^(c_exp r^2); A&S t = 1 / (1 + p alpha r)
  Real const c_exp = static_cast<Real>(-G.alpha * G.alpha * 1.4426950408889634);
  Real const p_alpha = static_cast<Real>(0.3275911 * G.alpha);
  bool const one_type = (ntypes == 1);
  PairR<Real> const p0(ia[0]);
  double fx = 0.0, fy = 0.0, fz = 0.0;
  const int *nbp = nb + nb_base(G.nb_off, G.max_nb, active ? a - G.p0 : 0);
  int const ngroups = G.max_nb >> 3;
  long long const base0 = G.p0;
  // the particle itself with the zero cell offset (code 13: dc = 0)
  unsigned const self_ent = static_cast<unsigned>(active ? a - G.p0 : 0) |
                            (static_cast<unsigned>(cell_offset_code(0, 0, 0)) << kNbIndexBits);
  // one entry: Coulomb always, LJ / WCA when the group may hold class A
  auto entry = [&](auto lj, unsigned e, float4 pb, float &sx, float &sy, float &sz) {
    // d = (x_a - x_b) - dc cs (dc in {-1, 0, 1}: the FMA's product is
    // exact, so this rounds as the sum with a stored shift would)
    unsigned const code = e >> kNbIndexBits;
    Real const d0 = fmaf(code_axis(code, 0), -cs_x, pa.x - pb.x);
    Real const d1 = fmaf(code_axis(code, 1), -cs_y, pa.y - pb.y);
    Real const d2v = fmaf(code_axis(code, 2), -cs_z, pa.z - pb.z);
    Real const dist2 = d0 * d0 + d1 * d1 + d2v * d2v;
    Real const inv_d = rsqrt_approx(dist2);
    Real const dist = dist2 * inv_d;
    bool const pos = dist2 > Real(0);
    Real const ex = ex2_approx(c_exp * dist2);
    Real const t = rcp_r(fmaf(p_alpha, dist, Real(1)));
    Real const asp =
        t * (Real(0.254829592) +
             t * (Real(-0.284496736) +
                  t * (Real(1.421413741) + t * (Real(-1.453152027) + t * Real(1.061405429)))));
    Real const erfc_part_ri = asp * inv_d;
    Real const pq = pref_qa * pb.w;
    bool const in_c = pos && dist2 < rc2;
    Real const fc =
        in_c ? (pq * ex) * (erfc_part_ri + two_a_sqrt_pi_i) * (inv_d * inv_d) : Real(0);
    Real fn = Real(0), en = Real(0);
    if constexpr (decltype(lj)::value) {
      if constexpr (NOOFF) {
        lj_wca_sel_nooff(p0, dist, inv_d * inv_d, fn);
      } else if (one_type) {
        if (p0.active)
          lj_wca_sel(p0, dist, inv_d, fn, en);
      } else {
        int const b = static_cast<int>(base0 + (e & kNbIndexMask));
        PairR<Real> const p(ia[ta * ntypes + stype[b]]);
        if (p.active)
          lj_wca_sel(p, dist, inv_d, fn, en);
      }
      fn = pos ? fn : Real(0);
      en = pos ? en : Real(0);
    }
    Real const ft = fc + fn;
    sx += ft * d0;
    sy += ft * d1;
    sz += ft * d2v;
    if constexpr (EV) {
      Real const ec = in_c ? pq * erfc_part_ri * ex : Real(0);
      double const dd[3] = {d0, d1, d2v};
      ev[0] += 0.5 * double(ec);
      ev[1] += 0.5 * double(en);
#pragma unroll
      for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          ev[2 + 3 * r + c] += 0.5 * double(fc) * dd[r] * dd[c];
          ev[11 + 3 * r + c] += 0.5 * double(fn) * dd[r] * dd[c];
        }
    }
  };
  auto group = [&](auto lj, int v) {
    // the lane's group v: class A group v, or class B group v - ga
    bool const in_a = v < ga;
    int const grp = in_a ? v : ngroups - 1 - (v - ga);
    int const kn = in_a ? min(8, na - 8 * v) : min(8, nbb - 8 * (v - ga));
    const int4 *gp = reinterpret_cast<const int4 *>(nbp + (static_cast<long long>(grp) << 8));
    int4 const g0 = gp[0], g1 = gp[1];
    unsigned const ent[8] = {static_cast<unsigned>(g0.x), static_cast<unsigned>(g0.y),
                             static_cast<unsigned>(g0.z), static_cast<unsigned>(g0.w),
                             static_cast<unsigned>(g1.x), static_cast<unsigned>(g1.y),
                             static_cast<unsigned>(g1.z), static_cast<unsigned>(g1.w)};
    float sx = 0.f, sy = 0.f, sz = 0.f;
#pragma unroll
    for (int h = 0; h < 8; h += 4) {
      // entries past the count stand for the particle itself (zero
      // distance: no term passes its range test), so no lane branches on
      // the count; the partners' positions, four gathers in flight
      unsigned eu[4];
      float4 pbv[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        eu[u] = (h + u < kn) ? ent[h + u] : self_ent;
        pbv[u] = spf[base0 + (eu[u] & kNbIndexMask)];
      }
#pragma unroll
      for (int u = 0; u < 4; ++u)
        entry(lj, eu[u], pbv[u], sx, sy, sz);
    }
    // FP32 sums of this group into the FP64 accumulators
    fx += static_cast<double>(sx);
    fy += static_cast<double>(sy);
    fz += static_cast<double>(sz);
  };
  for (int v = 0; v < gmax; ++v) {
    bool const any_a = __any_sync(0xffffffffu, active && v < ga);
    if (active && v < gt) {
      if (any_a)
        group(std::true_type{}, v);
      else
        group(std::false_type{}, v);
    }
  }
  if (active) {
    int const i = perm[a];
    if (overwrite) {
      f[3 * i + 0] = fx;
      f[3 * i + 1] = fy;
      f[3 * i + 2] = fz;
    } else {
      f[3 * i + 0] += fx;
      f[3 * i + 1] += fy;
      f[3 * i + 2] += fz;
    }
  }
  if constexpr (EV) {
    __shared__ double red[20][8];
    int const lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < 20; ++k) {
      double v = ev[k];
      for (int o = 16; o > 0; o >>= 1)
        v += __shfl_down_sync(0xffffffffu, v, o);
      if (lane == 0)
        red[k][wid] = v;
    }
    __syncthreads();
    if (threadIdx.x < 20) {
      double s = 0.0;
      for (int w = 0; w < (blockDim.x >> 5); ++w)
        s += red[threadIdx.x][w];
      partials[static_cast<long long>(blockIdx.x) * 20 + threadIdx.x] = s;
    }
  }
}

template <typename Real, bool EV>
__global__ void __launch_bounds__(256, (sizeof(Real) == 4 && !EV) ? 4 : 1)
k_pair_forces(const RepGeom *__restrict__ reps, const int2 *__restrict__ blk,
              const double4 *__restrict__ spq, const int *__restrict__ stype,
              const int *__restrict__ perm, const PairIA *__restrict__ ia_g, int ntypes,
              long long n, const int *__restrict__ nb, const int *__restrict__ nb_cnt,
              double *__restrict__ f, int overwrite, double *__restrict__ partials) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  PairIA *ia = reinterpret_cast<PairIA *>(smem_raw);
  for (int k = threadIdx.x; k < ntypes * ntypes; k += blockDim.x)
    ia[k] = ia_g[k];
  __syncthreads();
  int2 const bk = blk[blockIdx.x];
  RepGeom const &G = reps[bk.x];
  long long const a = G.p0 + static_cast<long long>(bk.y) * blockDim.x + threadIdx.x;
  double ev[EV ? 20 : 1];
#pragma unroll
  for (int k = 0; k < (EV ? 20 : 1); ++k)
    ev[k] = 0.0;
  if (a < G.p0 + G.np) {
    double4 const pa = spq[a];
    int const ta = stype[a];
    double const L0 = G.box[0], L1 = G.box[1], L2 = G.box[2];
    double const Li0 = G.box_i[0], Li1 = G.box_i[1], Li2 = G.box_i[2];
    Real const alpha = static_cast<Real>(G.alpha);
    Real const r_cut = static_cast<Real>(G.r_cut);
    Real const two_a_sqrt_pi_i = static_cast<Real>(2.0 * G.alpha / sqrt(kPi));
    Real const pref_qa = static_cast<Real>(G.prefactor * pa.w);
    bool const one_type = (ntypes == 1);
    PairR<Real> const p0(ia[0]);
    double fx = 0.0, fy = 0.0, fz = 0.0;
    int const cw = nb_cnt[a];
    int const cnt = nb_count(cw), cna = nb_count_a(cw);
    const int *nbp = nb + nb_base(G.nb_off, G.max_nb, a - G.p0);
    int const base0 = static_cast<int>(G.p0);
    int b_next =
        (cnt > 0) ? base0 + static_cast<int>(static_cast<unsigned>(nbp[nb_logical(0, G.max_nb, cna, 0)]) &
                                             kNbIndexMask)
                  : 0;
    double4 p_next = (cnt > 0) ? spq[b_next] : pa;
    for (int k = 0; k < cnt; ++k) {
      int const b = b_next;
      double4 const pb = p_next;
      if (k + 1 < cnt) {
        b_next = base0 + static_cast<int>(static_cast<unsigned>(nbp[nb_logical(0, G.max_nb, cna, k + 1)]) &
                                          kNbIndexMask);
        p_next = spq[b_next];
      }
      // geometry in FP64 (two conversions per pair instead of four)
      double const d0 = mi_d(pa.x - pb.x, L0, Li0);
      double const d1 = mi_d(pa.y - pb.y, L1, Li1);
      double const d2v = mi_d(pa.z - pb.z, L2, Li2);
      Real const dist2 = static_cast<Real>(d0 * d0 + d1 * d1 + d2v * d2v);
      Real const inv_d = rsqrt_r(dist2);
      Real const dist = dist2 * inv_d;
      Real fc = Real(0), ec = Real(0);
      Real const qb = static_cast<Real>(pb.w);
      if (qb != Real(0) && pref_qa != Real(0) && dist < r_cut && dist > Real(0)) {
        Real const adist = alpha * dist;
        Real const ex = exp_r(-adist * adist);
        Real const t = rcp_r(Real(1) + Real(0.3275911) * adist);
        Real const asp = t * (Real(0.254829592) +
                              t * (Real(-0.284496736) +
                                   t * (Real(1.421413741) + t * (Real(-1.453152027) + t * Real(1.061405429)))));
        Real const erfc_part_ri = asp * inv_d;
        Real const pq = pref_qa * qb;
        fc = pq * (ex * (erfc_part_ri + two_a_sqrt_pi_i) * (inv_d * inv_d));
        if constexpr (EV)
          ec = pq * erfc_part_ri * ex;
      }
      Real fn = Real(0), en = Real(0);
      if (one_type) {
        if (p0.active)
          lj_wca(p0, dist, inv_d, fn, en);
      } else {
        PairR<Real> const p(ia[ta * ntypes + stype[b]]);
        if (p.active)
          lj_wca(p, dist, inv_d, fn, en);
      }
      double const ft = static_cast<double>(fc + fn);
      fx += ft * d0;
      fy += ft * d1;
      fz += ft * d2v;
      if constexpr (EV) {
        double const dd[3] = {d0, d1, d2v};
        ev[0] += 0.5 * double(ec);
        ev[1] += 0.5 * double(en);
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            ev[2 + 3 * r + c] += 0.5 * double(fc) * dd[r] * dd[c];
            ev[11 + 3 * r + c] += 0.5 * double(fn) * dd[r] * dd[c];
          }
      }
    }
    int const i = perm[a];
    if (overwrite) {
      f[3 * i + 0] = fx;
      f[3 * i + 1] = fy;
      f[3 * i + 2] = fz;
    } else {
      f[3 * i + 0] += fx;
      f[3 * i + 1] += fy;
      f[3 * i + 2] += fz;
    }
  }
  if constexpr (EV) {
    __shared__ double red[20][8];
    int const lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < 20; ++k) {
      double v = ev[k];
      for (int o = 16; o > 0; o >>= 1)
        v += __shfl_down_sync(0xffffffffu, v, o);
      if (lane == 0)
        red[k][wid] = v;
    }
    __syncthreads();
    if (threadIdx.x < 20) {
      double s = 0.0;
      for (int w = 0; w < (blockDim.x >> 5); ++w)
        s += red[threadIdx.x][w];
      partials[static_cast<long long>(blockIdx.x) * 20 + threadIdx.x] = s;
    }
  }
}

// Largest squared displacement since the last list build, as a flag:
// set when any particle moved more than skin/2 (check_resort_required,
// CellStructure.hpp:393-401).
// A particle whose type differs from its type at the last build also
// triggers the rebuild: the lists hold per-type-pair cutoffs and the sorted
// types (as the reference resorts on a particle type change).
__global__ void k_displacement_check(const RepGeom *__restrict__ reps, const int *__restrict__ rep_of,
                                     const double *__restrict__ pos, const double *__restrict__ pos_ref,
                                     const int *__restrict__ type,
                                     const int *__restrict__ type_ref, long long n,
                                     int *__restrict__ flag, int *__restrict__ rflag) {
  long long const i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n)
    return;
  int const r = rep_of[i];
  RepGeom const &G = reps[r];
  double d2 = 0.0;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    double const dx = pos[3 * i + d] - pos_ref[3 * i + d];
    d2 += dx * dx;
  }
  double const lim = 0.5 * G.skin;
  if (d2 > lim * lim || type[i] != type_ref[i]) {
    atomicOr(flag, 1);
    if (rflag) // per-replica decision: only this replica rebuilds
      atomicOr(&rflag[r], 1);
  }
}

// Reference positions and types of the replicas that rebuilt (all when
// rflag is null).
__global__ void k_copy_pos_ref(double *__restrict__ pos_ref, const double *__restrict__ pos,
                               int *__restrict__ type_ref, const int *__restrict__ type,
                               const int *__restrict__ rep_of, const int *__restrict__ rflag,
                               long long n, const int *__restrict__ cond) {
  if (cond && !*cond)
    return;
  long long const i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n || (rflag && !rflag[rep_of[i]]))
    return;
#pragma unroll
  for (int d = 0; d < 3; ++d)
    pos_ref[3 * i + d] = pos[3 * i + d];
  type_ref[i] = type[i];
}

} // namespace p3mx

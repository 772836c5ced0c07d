// Exclusive scan and deterministic counting sort (device primitives).
//
// The counting sort orders items by an integer key (assignment brick or link
// cell) and then restores, inside every key bucket, ascending item order, so
// the permutation is a pure function of the keys: the same input gives the
// same bitwise output on every run, whatever the atomic order was.
#pragma once

#include "common.cuh"

#include <climits>

namespace p3mx {

constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;

__device__ inline int warp_incl_scan(int v) {
  unsigned const lane = threadIdx.x & 31u;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int const t = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= static_cast<unsigned>(o))
      v += t;
  }
  return v;
}

// Block-wide exclusive scan of one int per thread; returns the block total.
__device__ inline int block_excl_scan(int v, int &total) {
  __shared__ int warp_sums[32];
  int const incl = warp_incl_scan(v);
  int const lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 31)
    warp_sums[wid] = incl;
  __syncthreads();
  if (wid == 0) {
    int const nw = (blockDim.x + 31) >> 5;
    int s = (lane < nw) ? warp_sums[lane] : 0;
    s = warp_incl_scan(s);
    warp_sums[lane] = s;
  }
  __syncthreads();
  int const warp_off = (wid > 0) ? warp_sums[wid - 1] : 0;
  total = warp_sums[((blockDim.x + 31) >> 5) - 1];
  __syncthreads();
  return warp_off + incl - v;
}

// Pass 1: tile-local exclusive scan, tile totals to tile_sums.
__global__ void k_scan_tiles(const int *__restrict__ in, int *__restrict__ out,
                             int *__restrict__ tile_sums, long long n,
                             const int *__restrict__ cond) {
  if (cond && !*cond)
    return;
  long long const base = static_cast<long long>(blockIdx.x) * kScanTile +
                         static_cast<long long>(threadIdx.x) * kScanItems;
  int v[kScanItems];
  int s = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    v[k] = (base + k < n) ? in[base + k] : 0;
    s += v[k];
  }
  int total;
  int run = block_excl_scan(s, total);
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    if (base + k < n)
      out[base + k] = run;
    run += v[k];
  }
  if (threadIdx.x == 0)
    tile_sums[blockIdx.x] = total;
}

// Pass 2: exclusive scan of the tile totals by one block; writes the grand
// total to out[n].
__global__ void k_scan_tile_sums(int *__restrict__ tile_sums, int ntiles,
                                 int *__restrict__ out, long long n,
                                 const int *__restrict__ cond) {
  if (cond && !*cond)
    return;
  int const per = (ntiles + blockDim.x - 1) / blockDim.x;
  int const b0 = threadIdx.x * per;
  int s = 0;
  for (int k = 0; k < per; ++k)
    if (b0 + k < ntiles)
      s += tile_sums[b0 + k];
  int total;
  int run = block_excl_scan(s, total);
  for (int k = 0; k < per; ++k) {
    if (b0 + k < ntiles) {
      int const t = tile_sums[b0 + k];
      tile_sums[b0 + k] = run;
      run += t;
    }
  }
  if (threadIdx.x == 0)
    out[n] = total;
}

// Pass 3: add tile offsets.
__global__ void k_scan_add(int *__restrict__ out, const int *__restrict__ tile_sums,
                           long long n, const int *__restrict__ cond) {
  if (cond && !*cond)
    return;
  long long const i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i < n)
    out[i] += tile_sums[i / kScanTile];
}

// Place every item at start[key] + slot (slot from the counting atomics).
__global__ void k_place(const int *__restrict__ key, const int *__restrict__ slot,
                        const int *__restrict__ start, int *__restrict__ perm,
                        long long n, const int *__restrict__ cond) {
  if (cond && !*cond)
    return;
  long long const i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i < n)
    perm[start[key[i]] + slot[i]] = static_cast<int>(i);
}

// Restore particle-index order inside every bucket (the atomic slots of the
// binning pass arrive in any order): one warp per bucket.  Buckets of up to
// 128 entries are held in registers (4 per lane) and every entry's rank is
// counted by shuffle comparisons against all others (entries are distinct
// particle indices, so ranks are unique); larger buckets are left to
// k_fix_big_buckets.
__global__ void k_fix_buckets(const int *__restrict__ start, int *__restrict__ perm,
                              long long nbuckets, const int *__restrict__ cond) {
  if (cond && !*cond)
    return;
  constexpr int NV = 4;
  long long const b = (static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  int const lane = threadIdx.x & 31;
  if (b >= nbuckets)
    return; // whole warp
  int const s0 = start[b], s1 = start[b + 1];
  int const n = s1 - s0;
  if (n < 2)
    return;
  if (n > 32 * NV)
    return; // large bucket: k_fix_big_buckets
  int v[NV], rank[NV];
#pragma unroll
  for (int u = 0; u < NV; ++u) {
    int const idx = u * 32 + lane;
    v[u] = (idx < n) ? perm[s0 + idx] : INT_MAX;
    rank[u] = 0;
  }
#pragma unroll
  for (int u2 = 0; u2 < NV; ++u2) {
    if (u2 * 32 >= n)
      break; // warp-uniform
    for (int k = 0; k < 32; ++k) {
      int const o = __shfl_sync(0xffffffffu, v[u2], k);
#pragma unroll
      for (int u = 0; u < NV; ++u)
        rank[u] += (o < v[u]) ? 1 : 0;
    }
  }
  __syncwarp();
#pragma unroll
  for (int u = 0; u < NV; ++u)
    if (u * 32 + lane < n)
      perm[s0 + rank[u]] = v[u];
}

// Large buckets (> 128 entries): each thread checks one bucket, the block
// collects the large ones and sorts them one after another: the bucket is
// copied to shared memory and every thread counts the rank of its entries
// against the whole bucket (O(n^2 / threads)); buckets beyond kBigBucket
// entries fall back to an insertion sort by thread 0.
constexpr int kBigBucket = 8192;
__global__ void __launch_bounds__(256)
k_fix_big_buckets(const int *__restrict__ start, int *__restrict__ perm, long long nbuckets,
                  const int *__restrict__ cond) {
  if (cond && !*cond)
    return;
  __shared__ int sv[kBigBucket];
  __shared__ long long list[256];
  __shared__ int nlist;
  for (long long base = static_cast<long long>(blockIdx.x) * blockDim.x; base < nbuckets;
       base += static_cast<long long>(gridDim.x) * blockDim.x) {
    // every thread checks one bucket; the large ones are handled by the block
    if (threadIdx.x == 0)
      nlist = 0;
    __syncthreads();
    long long const bt = base + threadIdx.x;
    if (bt < nbuckets && start[bt + 1] - start[bt] > 128)
      list[atomicAdd(&nlist, 1)] = bt;
    __syncthreads();
    int const nl = nlist;
    for (int li = 0; li < nl; ++li) {
      long long const b = list[li];
      int const s0 = start[b], s1 = start[b + 1];
      int const n = s1 - s0;
      if (n > kBigBucket) {
        if (threadIdx.x == 0)
          for (int i = s0 + 1; i < s1; ++i) {
            int const v = perm[i];
            int j = i - 1;
            while (j >= s0 && perm[j] > v) {
              perm[j + 1] = perm[j];
              --j;
            }
            perm[j + 1] = v;
          }
        __syncthreads();
        continue;
      }
      for (int k = threadIdx.x; k < n; k += blockDim.x)
        sv[k] = perm[s0 + k];
      __syncthreads();
      for (int k = threadIdx.x; k < n; k += blockDim.x) {
        int const v = sv[k];
        int r = 0;
        for (int m = 0; m < n; ++m)
          r += (sv[m] < v) ? 1 : 0;
        perm[s0 + r] = v;
      }
      __syncthreads();
    }
  }
}

// Conditional fill for graph-captured paths (no-op when *cond is zero).
__global__ void k_fill_int(int *__restrict__ p, int v, long long n, const int *__restrict__ cond) {
  if (cond && !*cond)
    return;
  for (long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<long long>(gridDim.x) * blockDim.x)
    p[i] = v;
}

// Exclusive scan of up to kScanOneMax items by one block of 32 warps: warp
// w scans the segment [w L, (w+1) L) (L = 32 R) in R rounds of 32
// consecutive items (coalesced), the warp totals are scanned across the
// block; writes the total to out[n].
constexpr int kScanOneRounds = 32;
constexpr long long kScanOneMax = 32LL * 32 * kScanOneRounds;
__global__ void __launch_bounds__(1024) k_scan_one(const int *__restrict__ in,
                                                   int *__restrict__ out, long long n,
                                                   const int *__restrict__ cond) {
  if (cond && !*cond)
    return;
  int const lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  int const R = static_cast<int>((n + 1023) / 1024);
  long long const seg = static_cast<long long>(w) * 32 * R;
  int v[kScanOneRounds];
  int s = 0;
#pragma unroll
  for (int r = 0; r < kScanOneRounds; ++r) {
    long long const i = seg + 32 * r + lane;
    v[r] = (r < R && i < n) ? in[i] : 0;
    s += v[r];
  }
  // warp total, then the exclusive scan of the 32 warp totals
  for (int o = 16; o > 0; o >>= 1)
    s += __shfl_xor_sync(0xffffffffu, s, o);
  int total;
  int carry = block_excl_scan(lane == 0 ? s : 0, total);
  carry = __shfl_sync(0xffffffffu, carry, 0);
#pragma unroll
  for (int r = 0; r < kScanOneRounds; ++r) {
    if (r < R) {
      int const incl = warp_incl_scan(v[r]);
      long long const i = seg + 32 * r + lane;
      if (i < n)
        out[i] = carry + incl - v[r];
      carry += __shfl_sync(0xffffffffu, incl, 31);
    }
  }
  if (threadIdx.x == 0)
    out[n] = total;
}

// Host driver of the exclusive scan (out has n+1 entries): one block for up
// to kScanOneMax items, else three passes; returns the kernels launched.
// `cond` (device int, may be NULL) skips the whole scan when zero, so the
// scan can sit inside a captured CUDA graph behind a device-side decision.
inline int exclusive_scan(const int *in, int *out, int *tile_buf, long long n,
                          cudaStream_t st, const int *cond = nullptr) {
  if (n <= kScanOneMax) {
    k_scan_one<<<1, 1024, 0, st>>>(in, out, n, cond);
    return 1;
  }
  int const ntiles = ceil_div(n, kScanTile);
  k_scan_tiles<<<ntiles, kScanThreads, 0, st>>>(in, out, tile_buf, n, cond);
  k_scan_tile_sums<<<1, 1024, 0, st>>>(tile_buf, ntiles, out, n, cond);
  k_scan_add<<<ceil_div(n, 256), 256, 0, st>>>(out, tile_buf, n, cond);
  return 3;
}

} // namespace p3mx

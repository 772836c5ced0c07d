// Engine implementation: geometry, FFT plans, block tables and the two
// force pipelines (see engine.cuh).
#include "engine.cuh"
#include "p3m_kernels.cuh"
#include "sort.cuh"

#include <cudaTypedefs.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <complex>
#include <map>
#include <utility>

namespace p3mx {

namespace {

// Dynamic shared-memory opt-in of every charge-assignment instance of one
// precision: orders 1..7, both super-brick edges, single- and multi-set.
template <typename K> void set_smem_limit(K kern, size_t limit) {
  P3MX_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(limit)));
}
template <typename Real, bool MC, int... P>
void assign_smem_attrs_mc(size_t limit, std::integer_sequence<int, P...>) {
  (set_smem_limit(k_p3m_assign_sb<Real, P + 1, kSbEdge, MC>, limit), ...);
  (set_smem_limit(k_p3m_assign_sb<Real, P + 1, kSbEdgeSmall, MC>, limit), ...);
}
template <typename Real> void assign_smem_attrs(size_t limit) {
  assign_smem_attrs_mc<Real, false>(limit, std::make_integer_sequence<int, 7>{});
  assign_smem_attrs_mc<Real, true>(limit, std::make_integer_sequence<int, 7>{});
}

// Radix factorisation of an FFT length: the power of two as radix-16 stages
// (then one 8, 4 or 2), then 3, 5, 7 and any remaining prime (handled by the
// generic radix, up to 31).
AxisPlan make_plan(int n, int tw_off) {
  AxisPlan pl{};
  pl.n = n;
  pl.tw_off = tw_off;
  int m = n;
  std::vector<int> f;
  while (m % 16 == 0) {
    f.push_back(16);
    m /= 16;
  }
  for (int r : {8, 4, 2})
    if (m % r == 0) {
      f.push_back(r);
      m /= r;
    }
  for (int p = 3; m > 1; p += 2) {
    while (m % p == 0) {
      f.push_back(p);
      m /= p;
    }
  }
  if (f.empty())
    f.push_back(1);
  if (static_cast<int>(f.size()) > kMaxStages)
    throw Error(1, "FFT length " + std::to_string(n) + " has too many factors");
  for (int p : f)
    if (p > 31)
      throw Error(1, "mesh size " + std::to_string(n) +
                         " has a prime factor > 31; choose a mesh with factors <= 31");
  pl.nstages = (n == 1) ? 0 : static_cast<int>(f.size());
  for (int s = 0; s < pl.nstages; ++s)
    pl.radix[s] = f[s];
  return pl;
}

int cell_grid_host(const double *box, double range, int *cg, double *cs) {
  // RegularDecomposition::create_cell_grid on one rank
  // (RegularDecomposition.cpp:289-385, max_num_cells 32768).
  int const max_num_cells = 32768, min_num_cells = 8;
  double cell_range[3] = {range, range, range};
  if (range <= 0.0) {
    for (int i = 0; i < 3; ++i)
      cg[i] = 2;
  } else {
    double const volume = box[0] * box[1] * box[2];
    double const scale = std::cbrt(max_num_cells / volume);
    for (int i = 0; i < 3; ++i) {
      cg[i] = static_cast<int>(std::ceil(box[i] * scale));
      cell_range[i] = box[i] / static_cast<double>(cg[i]);
      if (cell_range[i] < range) {
        cg[i] = static_cast<int>(std::floor(box[i] / range));
        if (cg[i] < 1)
          return 2;
        cell_range[i] = box[i] / static_cast<double>(cg[i]);
      }
    }
    for (;;) {
      long const nc = long(cg[0]) * cg[1] * cg[2];
      if (nc <= max_num_cells)
        break;
      int mi = 0;
      double ms = cell_range[0];
      for (int i = 1; i < 3; ++i)
        if (cg[i] > 1 && cell_range[i] < ms) {
          mi = i;
          ms = cell_range[i];
        }
      cg[mi]--;
      cell_range[mi] = box[mi] / cg[mi];
    }
    if (long(cg[0]) * cg[1] * cg[2] < min_num_cells)
      return 3;
  }
  for (int i = 0; i < 3; ++i)
    cs[i] = box[i] / static_cast<double>(cg[i]);
  return 0;
}

template <typename T> void upload_vec(DevBuf &b, std::vector<T> const &v, cudaStream_t st) {
  b.ensure(std::max<size_t>(1, v.size()) * sizeof(T));
  if (!v.empty())
    P3MX_CUDA(cudaMemcpyAsync(b.p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, st));
}

} // namespace

Engine::Engine(bool fp32) : m_fp32(fp32) {
  P3MX_CUDA(cudaStreamCreateWithFlags(&m_stream, cudaStreamNonBlocking));
  m_ia.assign(1, PairIA{0, 0, 0, 0, 0, 0, 0, 0, 0, -1.0});
}

Engine::~Engine() {
  if (m_check_ev)
    cudaEventDestroy(m_check_ev);
  if (m_flag_host)
    cudaFreeHost(m_flag_host);
  if (m_stream)
    cudaStreamDestroy(m_stream);
}

void Engine::set_pair_table(int ntypes, std::vector<PairIA> const &tab) {
  if (ntypes < 1 || static_cast<int>(tab.size()) != ntypes * ntypes)
    throw Error(1, "pair table must hold ntypes^2 entries");
  m_ntypes = ntypes;
  m_ia = tab;
  upload_vec(m_ia_d, m_ia, m_stream);
  m_lists_valid = false;
  if (!m_conf.empty())
    configure(std::vector<ReplicaConf>(m_conf), m_n);
}

void Engine::configure(std::vector<ReplicaConf> const &conf, long long n_total) {
  m_conf = conf;
  m_n = n_total;
  int const R = static_cast<int>(conf.size());
  m_geom.assign(R, RepGeom{});
  m_cap.clear();
  // twiddle tables for every distinct axis length
  std::map<int, int> tw_off;
  std::vector<std::complex<double>> tw;
  auto twoff = [&](int n) {
    auto it = tw_off.find(n);
    if (it != tw_off.end())
      return it->second;
    int const off = static_cast<int>(tw.size());
    for (int k = 0; k < n; ++k)
      tw.push_back(std::polar(1.0, -2.0 * kPi * k / n));
    tw_off[n] = off;
    return off;
  };
  double max_ia = -1.0;
  for (auto const &e : m_ia)
    max_ia = std::max(max_ia, e.ia_cut);
  m_bins = m_cplx = m_cells = m_nkeys = m_ncorner = m_ebins = 0;
  for (int r = 0; r < R; ++r) {
    auto const &c = conf[r];
    auto &G = m_geom[r];
    G.cao = c.cao;
    G.alpha = c.alpha;
    G.r_cut = c.r_cut;
    G.prefactor = c.prefactor;
    G.epsilon = c.epsilon;
    G.V = c.box[0] * c.box[1] * c.box[2];
    G.p0 = c.p0;
    G.np = c.np;
    // pos_shift, interpolation.hpp:142
    G.pos_shift = std::floor((c.cao - 1) / 2.0) - (c.cao % 2) / 2.0;
    for (int d = 0; d < 3; ++d) {
      if (c.mesh[d] < 2 || c.mesh[d] % 2)
        throw Error(1, "P3M requires an even number of mesh points in all directions");
      G.box[d] = c.box[d];
      G.box_i[d] = 1.0 / c.box[d];
      G.mesh[d] = c.mesh[d];
      G.ai[d] = c.mesh[d] / c.box[d];
      double const a = 1.0 / G.ai[d];
      double const cao_cut = (static_cast<double>(c.cao) / 2.0) * a;
      double const outer_ld_grid = (0.0 - (cao_cut + c.skin)) * G.ai[d] - c.mesh_off[d];
      G.ld_ind[d] = static_cast<int>(std::ceil(outer_ld_grid));
      G.ld_pos[d] = (G.ld_ind[d] + c.mesh_off[d]) * a;
      G.plan[d] = make_plan(c.mesh[d], twoff(c.mesh[d]));
    }
    G.hp = ((c.mesh[2] / 2 + 1) + 3) / 4 * 4;
    // sort bricks (stencil corners binned by brick; interpolation tiles)
    G.brick = (c.cao <= 5) ? 4 : 8; // brick_edge<cao>() of the kernels
    G.nbx = (c.mesh[0] + G.brick - 1) / G.brick;
    G.nby = (c.mesh[1] + G.brick - 1) / G.brick;
    G.nbz = (c.mesh[2] + G.brick - 1) / G.brick;
    G.bin_off = m_ncorner;
    m_ncorner += static_cast<long long>(G.nbx) * G.nby * G.nbz * G.brick * G.brick * G.brick;
    G.brk_off = m_nkeys;
    m_nkeys += static_cast<long long>(G.nbx) * G.nby * G.nbz;
    G.rm_off = m_bins;
    G.km_off = m_cplx;
    // field mesh: ghost layers (periodic images) on the high side, so that
    // the interpolation tile of every brick (brick + cao - 1 points from the
    // brick origin) is one box of the padded mesh
    {
      int const nb[3] = {G.nbx, G.nby, G.nbz};
      for (int d = 0; d < 3; ++d)
        G.epad[d] = std::max(c.mesh[d], (nb[d] - 1) * G.brick + G.brick + c.cao - 1);
      G.re_off = m_ebins;
      m_ebins += static_cast<long long>(G.epad[0]) * G.epad[1] * G.epad[2];
    }
    m_bins += static_cast<long long>(c.mesh[0]) * c.mesh[1] * c.mesh[2];
    m_cplx += static_cast<long long>(c.mesh[0]) * c.mesh[1] * G.hp;
    // short-range cell system
    G.skin = c.skin;
    G.coulomb_cut = (c.prefactor != 0.0) ? c.r_cut : 0.0;
    G.max_cut = std::max(G.coulomb_cut, max_ia);
    double cs[3];
    if (cell_grid_host(c.box, G.max_cut + c.skin, G.cg, cs))
      throw Error(2, "interaction range " + std::to_string(G.max_cut + c.skin) +
                         " is larger than the box allows");
    for (int d = 0; d < 3; ++d)
      G.inv_cs[d] = 1.0 / cs[d];
    G.cell_off = m_cells;
    long long const ncell = static_cast<long long>(G.cg[0]) * G.cg[1] * G.cg[2];
    m_cells += ncell;
    // octant sort where a cell holds >= 64 particles on average (octants of
    // >= 8: the build's 8-wide candidate rounds stay full); 3 cells per axis
    // at least (the small-grid build visits whole cells)
    G.oct_on = (c.np >= 64 * ncell && G.cg[0] >= 3 && G.cg[1] >= 3 && G.cg[2] >= 3) ? 1 : 0;
  }
  // sort keys per cell: octants (8) as soon as one replica uses them
  m_oct_mult = 1;
  for (auto const &G : m_geom)
    if (G.oct_on)
      m_oct_mult = 8;
  for (auto &G : m_geom)
    G.oct_mult = m_oct_mult;
  if (m_ncorner >= (1LL << 31) || m_bins >= (1LL << 31) || m_n >= (1LL << 31))
    throw Error(1, "batch too large for 32-bit bin/particle indices");
  for (auto const &G : m_geom)
    if (G.np >= (1LL << kNbIndexBits))
      throw Error(1, "a replica holds more than 2^26 particles (Verlet list index limit)");
  cudaStream_t st = m_stream;
  upload_vec(m_geom_d, m_geom, st);
  {
    std::vector<typename CplxOf<double>::type> t64(tw.size());
    for (size_t k = 0; k < tw.size(); ++k)
      t64[k] = double2{tw[k].real(), tw[k].imag()};
    if (m_fp32) {
      std::vector<float2> t32(tw.size());
      for (size_t k = 0; k < tw.size(); ++k)
        t32[k] = float2{static_cast<float>(tw[k].real()), static_cast<float>(tw[k].imag())};
      upload_vec(m_tw, t32, st);
    } else {
      upload_vec(m_tw, t64, st);
    }
  }
  // replica id of every particle
  {
    std::vector<int> rep_of(std::max<long long>(1, m_n), 0);
    for (int r = 0; r < R; ++r)
      for (long long i = conf[r].p0; i < conf[r].p0 + conf[r].np; ++i)
        rep_of[i] = r;
    upload_vec(m_rep_of, rep_of, st);
  }
  // block tables
  size_t const csz = m_fp32 ? sizeof(float2) : sizeof(double2);
  size_t const cap = m_fp32 ? 4096 : 2048; // complex elements per smem buffer
  {
    std::vector<int2> bm, bc, bcen, bp, nat;
    m_blk_census_start.assign(1, 0);
    m_blk_pair_start.assign(1, 0);
    for (int r = 0; r < R; ++r) {
      long long const ms = static_cast<long long>(m_geom[r].mesh[0]) * m_geom[r].mesh[1] * m_geom[r].mesh[2];
      long long const cs2 = static_cast<long long>(m_geom[r].mesh[0]) * m_geom[r].mesh[1] * m_geom[r].hp;
      (void)ms;
      for (int b = 0; b < ceil_div(cs2, 256); ++b)
        bc.push_back(int2{r, b});
      for (int b = 0; b < std::max(1, ceil_div(conf[r].np, 2048)); ++b)
        bcen.push_back(int2{r, b});
      m_blk_census_start.push_back(static_cast<int>(bcen.size()));
      for (int b = 0; b < std::max(1, ceil_div(conf[r].np, 256)); ++b)
        bp.push_back(int2{r, b});
      m_blk_pair_start.push_back(static_cast<int>(bp.size()));
    }
    // super-bricks of the charge assignment grouped by colour: per
    // dimension, the tile intervals [bE, bE + min(E, M - bE) + cao - 1) of
    // the super-bricks (E = kSbEdge) on the periodic axis are coloured
    // greedily so that intervals of one colour never intersect (modulo M);
    // super-bricks sharing the colour triple then have disjoint tiles.  All
    // sort bricks in spatial order feed the interpolation.
    {
      // super-brick edge: 16, unless one colour's 16^3 super-bricks (about
      // an eighth of them) would leave SMs without a block
      {
        long long n16 = 0;
        for (auto const &G : m_geom)
          n16 += static_cast<long long>(ceil_div(G.mesh[0], kSbEdge)) * ceil_div(G.mesh[1], kSbEdge) *
                 ceil_div(G.mesh[2], kSbEdge);
        int dev = 0, sms = 148;
        if (cudaGetDevice(&dev) == cudaSuccess)
          cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        m_sb_edge = (n16 / 8 < sms) ? kSbEdgeSmall : kSbEdge;
      }
      auto colours = [](int M, int B, int P) {
        int const nb = (M + B - 1) / B;
        std::vector<int> s(nb), e(nb), col(nb, -1);
        for (int b = 0; b < nb; ++b) {
          s[b] = b * B;
          e[b] = s[b] + std::min(B, M - s[b]) + P - 1;
        }
        auto hit = [&](int a, int b) {
          if (e[a] - s[a] >= M || e[b] - s[b] >= M)
            return true;
          for (int k = -1; k <= 1; ++k)
            if (s[a] < e[b] + k * M && s[b] + k * M < e[a])
              return true;
          return false;
        };
        for (int b = 0; b < nb; ++b) {
          std::vector<char> used(nb + 1, 0);
          for (int a = 0; a < nb; ++a)
            if (a != b && col[a] >= 0 && hit(a, b))
              used[col[a]] = 1;
          int c = 0;
          while (used[c])
            ++c;
          col[b] = c;
        }
        return col;
      };
      // replicas may differ in cao: one phase per (cao, colour), and the
      // sort bricks grouped by cao (one interpolation launch per order)
      std::vector<std::vector<int2>> phase;
      std::vector<std::vector<int2>> bricks_of(8);
      nat.clear();
      for (int r = 0; r < R; ++r) {
        auto const &G = m_geom[r];
        auto const cxv = colours(G.mesh[0], m_sb_edge, G.cao);
        auto const cyv = colours(G.mesh[1], m_sb_edge, G.cao);
        auto const czv = colours(G.mesh[2], m_sb_edge, G.cao);
        int const n0 = static_cast<int>(cxv.size()), n1 = static_cast<int>(cyv.size()),
                  n2 = static_cast<int>(czv.size());
        for (int bx = 0; bx < n0; ++bx)
          for (int by = 0; by < n1; ++by)
            for (int bz = 0; bz < n2; ++bz) {
              int const p = (G.cao - 1) * 512 + cxv[bx] + 8 * (cyv[by] + 8 * czv[bz]);
              if (static_cast<int>(phase.size()) <= p)
                phase.resize(p + 1);
              phase[p].push_back(int2{r, (bx * n1 + by) * n2 + bz});
            }
        for (int b = 0; b < G.nbx * G.nby * G.nbz; ++b)
          bricks_of[G.cao].push_back(int2{r, b});
      }
      m_phase_off.assign(1, 0);
      m_phase_cao.clear();
      for (size_t p = 0; p < phase.size(); ++p) {
        if (phase[p].empty())
          continue;
        bm.insert(bm.end(), phase[p].begin(), phase[p].end());
        m_phase_off.push_back(static_cast<int>(bm.size()));
        m_phase_cao.push_back(static_cast<int>(p / 512) + 1);
      }
      m_brick_off.assign(9, 0);
      for (int c = 1; c <= 7; ++c) {
        nat.insert(nat.end(), bricks_of[c].begin(), bricks_of[c].end());
        m_brick_off[c + 1] = static_cast<int>(nat.size());
      }
      m_brick_off[1] = 0;
    }
    m_n_blk_mesh = static_cast<int>(bm.size());
    m_n_bricks = static_cast<int>(nat.size());
    m_n_blk_cplx = static_cast<int>(bc.size());
    m_n_blk_census = static_cast<int>(bcen.size());
    m_n_blk_pair = static_cast<int>(bp.size());
    upload_vec(m_blk_mesh, bm, st);
    upload_vec(m_blk_brick, nat, st);
    upload_vec(m_blk_cplx, bc, st);
    upload_vec(m_blk_census, bcen, st);
    upload_vec(m_blk_pair, bp, st);
    upload_vec(m_blk_census_start_d, m_blk_census_start, st);
    upload_vec(m_blk_pair_start_d, m_blk_pair_start, st);
  }
  {
    std::vector<Blk> zf, y, x, zi;
    m_blk_x_start.assign(1, 0);
    int maxM0 = 1, maxM1 = 1, maxM2 = 1;
    for (auto const &G : m_geom) {
      maxM0 = std::max(maxM0, G.mesh[0]);
      maxM1 = std::max(maxM1, G.mesh[1]);
      maxM2 = std::max(maxM2, G.mesh[2]);
    }
    // staged lines are padded (line_ld); every pass also holds its axis
    // twiddle table (n complex) in shared memory
    size_t const ldy = line_ld(maxM1), ldx = line_ld(maxM0);
    // y pass: power-of-two lines of 32..256 transform in place (no scratch
    // buffer)
    bool yin = true;
    for (auto const &G : m_geom)
      yin = yin && fft_inplace_ok(G.mesh[1], 16, 256);
    m_yin = yin;
    m_tile_y = static_cast<int>(std::max<size_t>(1, std::min<size_t>(16, cap / ldy)));
    // x pass: three line buffers (phi, field lines, scratch) of T kz columns
    size_t const x_budget = 96 * 1024;
    m_tile_x = static_cast<int>(
        std::max<size_t>(1, std::min<size_t>(16, x_budget / (3 * ldx * csz))));
    size_t smem_zf = 0, smem_zi = 0;
    for (int r = 0; r < R; ++r) {
      auto const &G = m_geom[r];
      int const M0 = G.mesh[0], M1 = G.mesh[1], M2 = G.mesh[2];
      int const H = M2 / 2 + 1;
      int const lines = M0 * M1;
      int const ldz = line_ld(M2);
      // forward z: two real lines per complex transform; FP32: as many line
      // pairs as keep four blocks within the SM's shared memory (24 lines at
      // 256^3: forward z+y 0.102 -> 0.098 ms against 30 at three blocks)
      int lz = static_cast<int>(std::max<size_t>(1, cap / ldz)) * 2;
      if (m_fp32) {
        int q = 1;
        while ((2 * static_cast<size_t>(q + 1) * ldz + M2) * csz <= 54 * 1024)
          ++q;
        lz = 2 * q;
      }
      for (int l = 0; l < lines; l += lz)
        zf.push_back(Blk{r, l, std::min(lz, lines - l), 0});
      smem_zf = std::max(smem_zf,
                         (2 * static_cast<size_t>((std::min(lz, lines) + 1) / 2) * ldz + M2) * csz);
      // backward z: nl lines -> nl (Ex, Ey) + ceil(nl/2) (Ez pairs) transforms.
      // FP32: as many lines as keep a block within a quarter of the SM's
      // shared memory, so that four blocks are resident (8 lines at 256^3:
      // 0.287 -> 0.271 ms for the backward y+z stage against 10 lines at
      // three blocks per SM)
      auto const zi_smem = [&](int nl) {
        size_t const nc = nl + (nl + 1) / 2;
        return (nc * ldz + z_inv_b_size(nl, M2) + M2) * csz;
      };
      int lzi = static_cast<int>(std::max<size_t>(1, 2 * (cap / ldz) / 3));
      if (m_fp32) {
        lzi = 1;
        while (lzi < lines && zi_smem(lzi + 1) <= 54 * 1024)
          ++lzi;
      }
      for (int l = 0; l < lines; l += lzi)
        zi.push_back(Blk{r, l, std::min(lzi, lines - l), 0});
      int const nzi = std::min(lzi, lines);
      size_t const nci = nzi + (nzi + 1) / 2;
      smem_zi = std::max(smem_zi, (nci * ldz + z_inv_b_size(nzi, M2) + M2) * csz);
      for (int xx = 0; xx < M0; ++xx)
        for (int k0 = 0; k0 < H; k0 += m_tile_y)
          y.push_back(Blk{r, xx, k0, 0});
      for (int yy = 0; yy < M1; ++yy)
        for (int k0 = 0; k0 < H; k0 += m_tile_x)
          x.push_back(Blk{r, yy, k0, 0});
      m_blk_x_start.push_back(static_cast<int>(x.size()));
    }
    m_smem_zf = smem_zf;
    m_smem_zi = smem_zi;
    m_smem_y = ((yin ? 1 : 2) * static_cast<size_t>(m_tile_y) * ldy + maxM1) * csz;
    m_smem_x = (3 * static_cast<size_t>(m_tile_x) * ldx + maxM0) * csz;
    m_n_blk_zf = static_cast<int>(zf.size());
    m_n_blk_y = static_cast<int>(y.size());
    m_n_blk_x = static_cast<int>(x.size());
    m_n_blk_zi = static_cast<int>(zi.size());
    upload_vec(m_blk_zf, zf, st);
    upload_vec(m_blk_y, y, st);
    upload_vec(m_blk_x, x, st);
    upload_vec(m_blk_zi, zi, st);
    upload_vec(m_blk_x_start_d, m_blk_x_start, st);
    // opt-in dynamic shared memory; static arrays of the kernels (<= 2 KB)
    // stay inside the 227 KB per-block limit
    size_t const limit = 220 * 1024;
    if (std::max({m_smem_zf, m_smem_zi, m_smem_y, m_smem_x}) > limit)
      throw Error(1, "mesh too large for the shared-memory FFT tiles");
    // one process-wide opt-in value, so engines of different sizes coexist
    auto attr = [limit](auto kern, size_t) {
      P3MX_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     static_cast<int>(limit)));
    };
    {
      // assignment: super-brick tile plus staged records (above 48 KB)
      auto aset = [&](auto kern) {
        P3MX_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       static_cast<int>(limit)));
      };
      if (m_fp32) {
        assign_smem_attrs<float>(limit);
        aset(k_p3m_interp<float, 1>); aset(k_p3m_interp<float, 2>); aset(k_p3m_interp<float, 3>);
        aset(k_p3m_interp<float, 4>); aset(k_p3m_interp<float, 5>); aset(k_p3m_interp<float, 6>);
        aset(k_p3m_interp<float, 7>);
      } else {
        assign_smem_attrs<double>(limit);
        aset(k_p3m_interp<double, 1>); aset(k_p3m_interp<double, 2>); aset(k_p3m_interp<double, 3>);
        aset(k_p3m_interp<double, 4>); aset(k_p3m_interp<double, 5>); aset(k_p3m_interp<double, 6>);
        aset(k_p3m_interp<double, 7>);
      }
    }
    if (m_fp32) {
      attr(k_fft_z_fwd<float>, m_smem_zf);
      attr(k_fft_y<float, true>, m_smem_y);
      attr(k_fft_y<float, false>, m_smem_y);
      attr(k_fft_x_kspace<float, true>, m_smem_x);
      attr(k_fft_x_kspace<float, false>, m_smem_x);
      attr(k_fft_x_kspace<float, false, 3>, m_smem_x);
      attr(k_fft_z_inv3<float>, m_smem_zi);
    } else {
      attr(k_fft_z_fwd<double>, m_smem_zf);
      attr(k_fft_y<double, true>, m_smem_y);
      attr(k_fft_y<double, false>, m_smem_y);
      attr(k_fft_x_kspace<double, true>, m_smem_x);
      attr(k_fft_x_kspace<double, false>, m_smem_x);
      attr(k_fft_z_inv3<double>, m_smem_zi);
    }
  }
  // buffers
  size_t const rsz = m_fp32 ? sizeof(float) : sizeof(double);
  long long const n = std::max<long long>(1, m_n);
  m_pos.ensure(3 * n * sizeof(double));
  m_q.ensure(n * sizeof(double));
  m_type.ensure(n * sizeof(int));
  m_force.ensure(3 * n * sizeof(double));
  m_key.ensure(n * sizeof(int));
  m_bkey.ensure(n * sizeof(int));
  m_slot.ensure(n * sizeof(int));
  // + 8: the back-interpolation copies 16-byte aligned windows of these
  m_perm.ensure((n + 8) * sizeof(int));
  // sort-brick counts, then one word per replica: the bits of its largest
  // |q| (FP32, rounded up), which the assignment's fixed-point scale needs
  m_cnt.ensure((m_nkeys + 1 + R) * sizeof(int));
  m_start.ensure((m_nkeys + 1) * sizeof(int));
  m_scan_tiles.ensure((ceil_div(std::max(m_nkeys, m_oct_mult * m_cells) + 1, kScanTile) + 1) * sizeof(int));
  m_dist.ensure(3 * n * rsz);
  m_W.ensure(static_cast<size_t>(wstride<7, 4>()) * n * rsz);
  m_skey.ensure((n + 8) * sizeof(int));
  m_rho.ensure(m_bins * rsz + 64); // + slack: bulk copies of 16-byte aligned supersets
  m_E.ensure(4 * m_ebins * rsz);
  encode_field_maps(st);
  m_ck.ensure(m_cplx * csz);
  m_field.ensure(3 * m_cplx * csz);
  m_ginf.ensure(m_cplx * rsz);
  m_part_x.ensure(static_cast<size_t>(m_n_blk_x) * 8 * sizeof(double));
  m_sums_x.ensure(static_cast<size_t>(R) * 8 * sizeof(double));
  m_part_census.ensure(static_cast<size_t>(m_n_blk_census) * 6 * sizeof(double));
  m_sums_census.ensure(static_cast<size_t>(R) * 6 * sizeof(double));
  m_dipole.ensure(static_cast<size_t>(R) * 3 * sizeof(double));
  m_ckey.ensure(n * sizeof(int));
  m_cslot.ensure(n * sizeof(int));
  // counting sort of the particles by cell octant (8 keys per cell)
  m_ccnt.ensure((m_oct_mult * m_cells + 1) * sizeof(int));
  m_cstart.ensure((m_oct_mult * m_cells + 1) * sizeof(int));
  m_cbkey.ensure(n * sizeof(int));
  m_cperm.ensure(n * sizeof(int));
  m_cinv.ensure(n * sizeof(int));
  m_pq.ensure(n * sizeof(double4));
  m_spq.ensure(n * sizeof(double4));
  m_spf.ensure(n * sizeof(float4));
  m_stype.ensure(n * sizeof(int));
  m_scell.ensure(n * sizeof(int));
  m_nb_cnt.ensure(n * sizeof(int));
  m_overflow.ensure(static_cast<size_t>(std::max(R, 1)) * sizeof(int));
  m_rflag.ensure(static_cast<size_t>(std::max(R, 1)) * sizeof(int));
  m_flag.ensure(sizeof(int));
  // the list check's two alternating flag words, both zero
  m_chk.ensure(2 * sizeof(int));
  P3MX_CUDA(cudaMemsetAsync(m_chk.p, 0, 2 * sizeof(int), st));
  m_chk_slot = 0;
  if (m_kerr.p == nullptr) {
    m_kerr.ensure(4 * sizeof(int));
    P3MX_CUDA(cudaMemsetAsync(m_kerr.p, 0, 4 * sizeof(int), st));
  }
  m_pos_ref.ensure(3 * n * sizeof(double));
  m_type_ref.ensure(n * sizeof(int));
  m_part_pair.ensure(static_cast<size_t>(m_n_blk_pair) * 20 * sizeof(double));
  m_sums_pair.ensure(static_cast<size_t>(R) * 20 * sizeof(double));
  if (m_ia_d.p == nullptr)
    upload_vec(m_ia_d, m_ia, st);
  m_ginf_valid = false;
  m_lists_valid = false;
  P3MX_CUDA(cudaStreamSynchronize(st));
}

void Engine::upload(const double *pos, const double *q, const int *type, bool device_ptrs,
                    cudaStream_t st) {
  cudaMemcpyKind const k = device_ptrs ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
  if (m_n == 0)
    return;
  P3MX_CUDA(cudaMemcpyAsync(m_pos.p, pos, 3 * m_n * sizeof(double), k, st));
  P3MX_CUDA(cudaMemcpyAsync(m_q.p, q, m_n * sizeof(double), k, st));
  if (type)
    P3MX_CUDA(cudaMemcpyAsync(m_type.p, type, m_n * sizeof(int), k, st));
  else
    P3MX_CUDA(cudaMemsetAsync(m_type.p, 0, m_n * sizeof(int), st));
}

void Engine::upload_positions(const double *pos, bool device_ptrs, cudaStream_t st) {
  if (m_n == 0)
    return;
  P3MX_CUDA(cudaMemcpyAsync(m_pos.p, pos, 3 * m_n * sizeof(double),
                            device_ptrs ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, st));
}

void Engine::census(cudaStream_t st) {
  int const R = n_rep();
  k_census<<<m_n_blk_census, 256, 0, st>>>(m_blk_census.as<int2>(), m_geom_d.as<RepGeom>(),
                                           d_pos(), d_q(), m_part_census.as<double>()); ++m_launches;
  k_reduce_partials<<<ceil_div(R, 128), 128, 0, st>>>(m_part_census.as<double>(), 6,
                                                      m_blk_census_start_d.as<int>(), R,
                                                      m_sums_census.as<double>()); ++m_launches;
  m_census_h.assign(static_cast<size_t>(R) * 6, 0.0);
  P3MX_CUDA(cudaMemcpyAsync(m_census_h.data(), m_sums_census.p, R * 6 * sizeof(double),
                            cudaMemcpyDeviceToHost, st));
  P3MX_CUDA(cudaStreamSynchronize(st));
  std::vector<double> dip(3 * R);
  for (int r = 0; r < R; ++r) {
    m_geom[r].sum_q = m_census_h[6 * r + 1];
    m_geom[r].sum_q2 = m_census_h[6 * r + 2];
    for (int d = 0; d < 3; ++d)
      dip[3 * r + d] = m_census_h[6 * r + 3 + d];
  }
  upload_vec(m_geom_d, m_geom, st);
  upload_vec(m_dipole, dip, st);
}

void Engine::sort_keys(int *key, int *slot, int *cnt, int *start, int *perm, long long nkeys,
                       cudaStream_t st, const int *cond, bool index_order) {
  m_launches += exclusive_scan(cnt, start, m_scan_tiles.as<int>(), nkeys, st, cond);
  k_place<<<ceil_div(m_n, 256), 256, 0, st>>>(key, slot, start, perm, m_n, cond); ++m_launches;
  if (!index_order)
    return;
  k_fix_buckets<<<ceil_div(nkeys * 32, 256), 256, 0, st>>>(start, perm, nkeys, cond); ++m_launches;
  k_fix_big_buckets<<<static_cast<int>(std::min<long long>(ceil_div(nkeys, 256), 296)), 256, 0,
                      st>>>(
      start, perm, nkeys, cond); ++m_launches;
}

namespace {
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 const fn = [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult res = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &res) !=
            cudaSuccess ||
        res != cudaDriverEntryPointSuccess || p == nullptr) {
      cudaGetLastError();
      throw Error(4, "cuTensorMapEncodeTiled is not available from the CUDA driver");
    }
    return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }();
  return fn;
}
} // namespace

// One tensor map per replica over its packed, ghost-padded field mesh E (4
// values per point): dims (4 E2, E1, E0) with E = epad, box (4 Ed, Ed, Ed)
// with Ed = brick + cao - 1 (<= epad by construction).
void Engine::encode_field_maps(cudaStream_t st) {
  auto enc = tensor_map_encoder();
  size_t const es = m_fp32 ? sizeof(float) : sizeof(double);
  std::vector<CUtensorMap> maps(m_geom.size());
  for (size_t r = 0; r < m_geom.size(); ++r) {
    RepGeom const &G = m_geom[r];
    cuuint32_t const Ed = static_cast<cuuint32_t>(G.brick + G.cao - 1);
    cuuint64_t const E0 = G.epad[0], E1 = G.epad[1], E2 = G.epad[2];
    if (Ed > E0 || Ed > E1 || Ed > E2 || 4 * Ed > 256)
      throw Error(1, "interpolation tile larger than the field mesh box limits");
    cuuint64_t dims[3] = {4 * E2, E1, E0};
    cuuint64_t strides[2] = {4 * E2 * es, 4 * E2 * E1 * es};
    cuuint32_t box[3] = {4 * Ed, Ed, Ed};
    cuuint32_t estr[3] = {1, 1, 1};
    void *base = static_cast<char *>(m_E.p) + 4 * static_cast<size_t>(G.re_off) * es;
    CUresult const rc =
        enc(&maps[r], m_fp32 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64,
            3, base, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
            CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (rc != CUDA_SUCCESS)
      throw Error(4, "tensor map encoding of the field mesh failed (" + std::to_string(rc) + ")");
  }
  upload_vec(m_tmap, maps, st);
}

namespace {
// One colour launch of the charge assignment; `chained` launches it as a
// programmatic dependent of the previous colour (see k_p3m_assign_sb).
template <typename Real, int P, int E>
void launch_assign_e(bool chained, int cnt, cudaStream_t st, RepGeom const *geom, int2 const *tab,
                     int const *start, Real const *W, int const *s_key, unsigned const *qmax_bits,
                     Real *rho, int *err, int ncomp, long long comp_w, long long comp_rho,
                     int comp_q) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(static_cast<unsigned>(cnt), static_cast<unsigned>(ncomp));
  cfg.blockDim = dim3(32 * kSbWarps);
  cfg.dynamicSmemBytes = sb_smem<Real, P, E>();
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = chained ? 1 : 0;
  auto const kern = ncomp > 1 ? k_p3m_assign_sb<Real, P, E, true> : k_p3m_assign_sb<Real, P, E, false>;
  P3MX_CUDA(cudaLaunchKernelEx(&cfg, kern, geom, tab, cnt, start, W, s_key, qmax_bits, rho, err,
                               comp_w, comp_rho, comp_q));
}
// ... with the engine's super-brick edge (16 or 8); ncomp charge sets
// (records, meshes and |q| maxima comp_w / comp_rho / comp_q apart)
template <typename Real, int P>
void launch_assign(int edge, bool chained, int cnt, cudaStream_t st, RepGeom const *geom,
                   int2 const *tab, int const *start, Real const *W, int const *s_key,
                   unsigned const *qmax_bits, Real *rho, int *err, int ncomp = 1,
                   long long comp_w = 0, long long comp_rho = 0, int comp_q = 0) {
  if (edge == kSbEdgeSmall)
    launch_assign_e<Real, P, kSbEdgeSmall>(chained, cnt, st, geom, tab, start, W, s_key, qmax_bits,
                                           rho, err, ncomp, comp_w, comp_rho, comp_q);
  else
    launch_assign_e<Real, P, kSbEdge>(chained, cnt, st, geom, tab, start, W, s_key, qmax_bits, rho,
                                      err, ncomp, comp_w, comp_rho, comp_q);
}

// Persistent grid of the back-interpolation pipeline: resident blocks per
// SM times the SM count (computed once per kernel instance and process),
// at most one block per brick.
template <typename Real, int P> int interp_grid(int nbricks) {
  static std::atomic<int> blocks{0};
  int b = blocks.load(std::memory_order_relaxed);
  if (b == 0) {
    int dev = 0, sms = 0, per_sm = 0;
    P3MX_CUDA(cudaGetDevice(&dev));
    P3MX_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    P3MX_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
        &per_sm, k_p3m_interp<Real, P>, 32 * (1 + kInterpWarps), interp_smem<Real, P>()));
    b = std::max(1, per_sm) * std::max(1, sms);
    blocks.store(b, std::memory_order_relaxed);
  }
  return std::max(1, std::min(nbricks, b));
}
} // namespace

#define P3MX_CAO_DISPATCH_R(cao, KERNEL_CALL)                                  \
  switch (cao) {                                                               \
  case 1: { constexpr int P = 1; KERNEL_CALL; } break;                         \
  case 2: { constexpr int P = 2; KERNEL_CALL; } break;                         \
  case 3: { constexpr int P = 3; KERNEL_CALL; } break;                         \
  case 4: { constexpr int P = 4; KERNEL_CALL; } break;                         \
  case 5: { constexpr int P = 5; KERNEL_CALL; } break;                         \
  case 6: { constexpr int P = 6; KERNEL_CALL; } break;                         \
  default: { constexpr int P = 7; KERNEL_CALL; } break;                        \
  }
template <typename Real>
void Engine::long_range_t(double *f, bool overwrite, bool want_e, bool want_v,
                          cudaStream_t st) {
  using C = typename CplxOf<Real>::type;
  int const R = n_rep();
  // replicas may differ in mesh and cao: the order-templated kernels run
  // once per order present
  RepGeom const *geom = m_geom_d.as<RepGeom>();
  if (!m_ginf_valid) {
    k_influence<Real><<<m_n_blk_cplx, 256, 0, st>>>(geom, m_blk_cplx.as<int2>(), m_ginf.as<Real>()); ++m_launches;
    m_ginf_valid = true;
  }
  mark("start", st);
  // 1. corner binning + deterministic counting sort
  P3MX_CUDA(cudaMemsetAsync(m_cnt.p, 0, (m_nkeys + 1 + R) * sizeof(int), st));
  unsigned *qmax_bits = reinterpret_cast<unsigned *>(m_cnt.as<int>() + m_nkeys + 1);
  int const nb = ceil_div(m_n, 256);
  if (m_n > 0) {
    k_p3m_bin<Real><<<nb, 256, 0, st>>>(geom, m_rep_of.as<int>(), d_pos(), m_n, m_key.as<int>(),
                                        m_bkey.as<int>(),
                                        m_slot.as<int>(), m_cnt.as<int>(), m_dist.as<Real>()); ++m_launches;
    // the order inside a brick is left as the atomic slots made it: the
    // fixed-point assignment sums integers and the interpolation treats
    // every particle on its own, so the results do not depend on it
    sort_keys(m_bkey.as<int>(), m_slot.as<int>(), m_cnt.as<int>(), m_start.as<int>(),
              m_perm.as<int>(), m_nkeys, st, nullptr, false);
    mark("p3m_sort", st);
    k_p3m_weights<Real><<<nb, 256, 0, st>>>(geom, m_perm.as<int>(), m_key.as<int>(),
                                            m_dist.as<Real>(), d_q(), m_rep_of.as<int>(), m_n,
                                            m_W.as<Real>(), m_skey.as<int>(), qmax_bits);
    ++m_launches;
    mark("p3m_weights", st);
  } else {
    P3MX_CUDA(cudaMemsetAsync(m_start.p, 0, (m_nkeys + 1) * sizeof(int), st));
  }
  // 2. charge assignment: one block per super-brick, colour by colour
  P3MX_CUDA(cudaMemsetAsync(m_rho.p, 0, m_bins * sizeof(Real), st));
  {
    bool chained = false; // the first colour waits for the mesh memset normally
    for (size_t p = 0; p + 1 < m_phase_off.size(); ++p) {
      int const cnt = m_phase_off[p + 1] - m_phase_off[p];
      if (cnt == 0)
        continue;
      int2 const *tab = m_blk_mesh.as<int2>() + m_phase_off[p];
      P3MX_CAO_DISPATCH_R(m_phase_cao[p], (launch_assign<Real, P>(m_sb_edge, chained, cnt, st, geom, tab,
                                                       m_start.as<int>(), m_W.as<Real>(),
                                                       m_skey.as<int>(), qmax_bits,
                                                       m_rho.as<Real>(), m_kerr.as<int>())));
      chained = true;
      ++m_launches;
    }
  }
  mark("p3m_assign", st);
  // 3. forward FFT z (r2c) and y
  C const *tw = m_tw.as<C>();
  k_fft_z_fwd<Real><<<m_n_blk_zf, 256, m_smem_zf, st>>>(geom, m_blk_zf.as<Blk>(), m_rho.as<Real>(),
                                                        m_ck.as<C>(), tw, m_kerr.as<int>());
  ++m_launches;
  launch_fft_y<Real>(m_ck.p, 0, 1, false, st);
  mark("fft_fwd_zy", st);
  // 4. x pass fused with the k-space operator (+ energy/virial partials)
  bool const want_f = (f != nullptr);
  bool const want_ev = want_e || want_v;
  if (want_ev)
    k_fft_x_kspace<Real, true><<<m_n_blk_x, 256, m_smem_x, st>>>(
        geom, m_blk_x.as<Blk>(), m_ck.as<C>(), m_ginf.as<Real>(), m_field.as<C>(), m_cplx,
        m_tile_x, want_f ? 1 : 0, m_part_x.as<double>(), tw);
  else if (sizeof(Real) == 4 && 3 * (m_smem_x + 1024) <= 228 * 1024)
    // the shared memory leaves room for three blocks per SM: the instance
    // whose registers allow them
    k_fft_x_kspace<Real, false, 3><<<m_n_blk_x, 256, m_smem_x, st>>>(
        geom, m_blk_x.as<Blk>(), m_ck.as<C>(), m_ginf.as<Real>(), m_field.as<C>(), m_cplx,
        m_tile_x, want_f ? 1 : 0, m_part_x.as<double>(), tw);
  else
    k_fft_x_kspace<Real, false><<<m_n_blk_x, 256, m_smem_x, st>>>(
        geom, m_blk_x.as<Blk>(), m_ck.as<C>(), m_ginf.as<Real>(), m_field.as<C>(), m_cplx,
        m_tile_x, want_f ? 1 : 0, m_part_x.as<double>(), tw);
  ++m_launches;
  if (want_ev) {
    k_reduce_partials<<<ceil_div(R, 128), 128, 0, st>>>(m_part_x.as<double>(), 8,
                                                        m_blk_x_start_d.as<int>(), R,
                                                        m_sums_x.as<double>());
    ++m_launches;
  }
  mark("fft_x_kspace", st);
  if (!want_f)
    return;
  // 5. backward FFT y (3 fields), z (c2r, 3 fields)
  launch_fft_y<Real>(m_field.p, m_cplx, 3, true, st);
  k_fft_z_inv3<Real><<<m_n_blk_zi, 256, m_smem_zi, st>>>(geom, m_blk_zi.as<Blk>(), m_field.as<C>(),
                                                         m_cplx, m_E.as<Real>(), tw, m_kerr.as<int>());
  ++m_launches;
  mark("fft_inv_yz", st);
  // 6. force back-interpolation
  for (int c = 1; m_n > 0 && c <= 7; ++c) {
    int const nbr = m_brick_off[c + 1] - m_brick_off[c];
    if (nbr == 0)
      continue;
    int2 const *tab = m_blk_brick.as<int2>() + m_brick_off[c];
    P3MX_CAO_DISPATCH_R(c, (k_p3m_interp<Real, P><<<interp_grid<Real, P>(nbr),
                               32 * (1 + kInterpWarps), interp_smem<Real, P>(), st>>>(
                               geom, tab, nbr, m_start.as<int>(), m_perm.as<int>(),
                               m_skey.as<int>(), m_W.as<Real>(), m_E.as<Real>(),
                               m_tmap.as<CUtensorMap>(), d_q(), m_dipole.as<double>(), f,
                               overwrite ? 1 : 0, m_kerr.as<int>())));
    ++m_launches;
  }
  mark("p3m_interp", st);
}

void Engine::long_range(double *f, bool overwrite, bool want_energy, bool want_virial,
                        cudaStream_t st, std::vector<double> *energies,
                        std::vector<double> *virials) {
  if (m_fp32)
    long_range_t<float>(f, overwrite, want_energy, want_virial, st);
  else
    long_range_t<double>(f, overwrite, want_energy, want_virial, st);
  P3MX_CUDA(cudaGetLastError());
  if (want_energy || want_virial) {
    int const R = n_rep();
    std::vector<double> sums(static_cast<size_t>(R) * 8);
    P3MX_CUDA(cudaMemcpyAsync(sums.data(), m_sums_x.p, sums.size() * sizeof(double),
                              cudaMemcpyDeviceToHost, st));
    P3MX_CUDA(cudaStreamSynchronize(st));
    if (energies)
      energies->assign(R, 0.0);
    if (virials)
      virials->assign(static_cast<size_t>(R) * 9, 0.0);
    for (int r = 0; r < R; ++r) {
      auto const &G = m_geom[r];
      double const *s = &sums[8 * r];
      if (energies) {
        // p3m.cpp:551-589: mesh sum / 2V, self energy, net charge, dipole
        double e = s[0] / (2.0 * G.V);
        e -= G.sum_q2 * G.alpha / std::sqrt(kPi);
        e -= G.sum_q * G.sum_q * kPi / (2.0 * G.V * G.alpha * G.alpha);
        if (G.epsilon != 0.0) {
          double const *m = &m_census_h[6 * r + 3];
          e += 4.0 * kPi / G.V / (2.0 * G.epsilon + 1.0) * (m[0] * m[0] + m[1] * m[1] + m[2] * m[2]);
        }
        (*energies)[r] = e * G.prefactor;
      }
      if (virials) {
        // long_range_pressure, p3m.cpp:394-449
        double t[9];
        t[0] = s[1] + s[7];
        t[1] = s[2];
        t[2] = s[3];
        t[4] = s[4] + s[7];
        t[5] = s[5];
        t[8] = s[6] + s[7];
        t[3] = t[1];
        t[6] = t[2];
        t[7] = t[5];
        for (int k = 0; k < 9; ++k)
          (*virials)[9 * r + k] = t[k] * G.prefactor / (2.0 * G.V);
      }
    }
  }
}

void Engine::build_lists(cudaStream_t st) {
  RepGeom const *geom = m_geom_d.as<RepGeom>();
  int const nb = ceil_div(m_n, 256);
  P3MX_CUDA(cudaMemsetAsync(m_ccnt.p, 0, (m_oct_mult * m_cells + 1) * sizeof(int), st));
  k_cell_bin<<<nb, 256, 0, st>>>(geom, m_rep_of.as<int>(), d_pos(), d_q(), m_n, m_ckey.as<int>(),
                                 m_cbkey.as<int>(), m_cslot.as<int>(), m_ccnt.as<int>(), m_pq.as<double4>(), nullptr, nullptr,
                                 nullptr); ++m_launches;
  sort_keys(m_cbkey.as<int>(), m_cslot.as<int>(), m_ccnt.as<int>(), m_cstart.as<int>(),
            m_cperm.as<int>(), m_oct_mult * m_cells, st);
  k_cell_gather<<<nb, 256, 0, st>>>(geom, m_rep_of.as<int>(), m_cperm.as<int>(), m_pq.as<double4>(), d_type(), m_ckey.as<int>(),
                                    m_n, m_spq.as<double4>(), m_spf.as<float4>(), m_stype.as<int>(), m_scell.as<int>(), m_cinv.as<int>(), nullptr); ++m_launches;
  if (m_cap.size() != m_geom.size())
    set_list_capacity(1.5);
  int const R = n_rep();
  for (int attempt = 0; attempt < 4; ++attempt) {
    P3MX_CUDA(cudaMemsetAsync(m_overflow.p, 0, R * sizeof(int), st));
    (m_oct_mult == 8 ? k_verlet_build<true> : k_verlet_build<false>)<<<nb, 256, m_ntypes * m_ntypes * sizeof(float), st>>>(geom, m_rep_of.as<int>(), m_spq.as<double4>(),
                                       m_spf.as<float4>(), m_stype.as<int>(),
                                       m_scell.as<int>(), m_cstart.as<int>(), m_ia_d.as<PairIA>(),
                                       m_ntypes, m_n, m_nb.as<int>(), m_nb_cnt.as<int>(),
                                       m_overflow.as<int>(), nullptr, nullptr); ++m_launches;
    std::vector<int> ov(R);
    P3MX_CUDA(cudaMemcpyAsync(ov.data(), m_overflow.p, R * sizeof(int), cudaMemcpyDeviceToHost, st));
    P3MX_CUDA(cudaStreamSynchronize(st));
    bool grown = false;
    for (int r = 0; r < R; ++r)
      if (ov[r] > 0) {
        m_cap[r] = (ov[r] + ov[r] / 4 + 16 + 7) / 8 * 8; // whole groups of 8
        grown = true;
      }
    if (!grown)
      break;
    if (attempt == 3)
      throw Error(2, "Verlet list overflow");
    layout_lists(st);
  }
  P3MX_CUDA(cudaMemcpyAsync(m_pos_ref.p, d_pos(), 3 * m_n * sizeof(double), cudaMemcpyDeviceToDevice, st));
  P3MX_CUDA(cudaMemcpyAsync(m_type_ref.p, d_type(), m_n * sizeof(int), cudaMemcpyDeviceToDevice, st));
  m_lists_valid = true;
}

__global__ void k_refresh_spq(const RepGeom *__restrict__ reps, const int *__restrict__ rep_of,
                              const int *__restrict__ perm, const double *__restrict__ pos,
                              const double *__restrict__ q, const int *__restrict__ scell,
                              const double *__restrict__ pos_ref, long long n,
                              double4 *__restrict__ spq, float4 *__restrict__ spf) {
  long long const s = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (s >= n)
    return;
  int const i = perm[s];
  RepGeom const &G = reps[rep_of[i]];
  double const qi = q[i];
  if (spq) // FP64 pair kernel positions, only when that kernel runs next
    spq[s] = make_double4(fold_coord(pos[3 * i], G.box[0]), fold_coord(pos[3 * i + 1], G.box[1]),
                          fold_coord(pos[3 * i + 2], G.box[2]), qi);
  spf[s] = cell_offset(G, scell[s] - static_cast<int>(G.cell_off), pos_ref + 3 * i, pos + 3 * i,
                       qi);
}

// Displacement check fused with the sorted-position refresh: sets *flag
// when a particle moved more than skin/2 or changed type since the last
// build (k_displacement_check's test) and writes the pair kernel's sorted
// records as k_refresh_spq does (a rebuild that follows rewrites them).
// One thread per particle in index order (coalesced reads of positions,
// reference positions, types and build-time cells), each writing its
// records to its sorted slot inv[i].
__global__ void k_check_refresh(const RepGeom *__restrict__ reps, const int *__restrict__ rep_of,
                                const int *__restrict__ inv, const double *__restrict__ pos,
                                const double *__restrict__ q, const int *__restrict__ ckey,
                                const double *__restrict__ pos_ref, const int *__restrict__ type,
                                const int *__restrict__ type_ref, long long n,
                                double4 *__restrict__ spq, float4 *__restrict__ spf,
                                int *__restrict__ flag, int *__restrict__ flag_next) {
  // the flag word of the next check starts at zero (no memset between checks)
  if (blockIdx.x == 0 && threadIdx.x == 0)
    *flag_next = 0;
  long long const i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n)
    return;
  int const s = inv[i];
  RepGeom const &G = reps[rep_of[i]];
  double d2 = 0.0;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    double const dx = pos[3 * i + d] - pos_ref[3 * i + d];
    d2 += dx * dx;
  }
  double const lim = 0.5 * G.skin;
  if (d2 > lim * lim || type[i] != type_ref[i])
    atomicOr(flag, 1);
  double const qi = q[i];
  if (spq)
    spq[s] = make_double4(fold_coord(pos[3 * i], G.box[0]), fold_coord(pos[3 * i + 1], G.box[1]),
                          fold_coord(pos[3 * i + 2], G.box[2]), qi);
  spf[s] = cell_offset(G, ckey[i] - static_cast<int>(G.cell_off), pos_ref + 3 * i, pos + 3 * i,
                       qi);
}

void Engine::refresh_sorted_positions(cudaStream_t st, bool want_spq) {
  k_refresh_spq<<<ceil_div(m_n, 256), 256, 0, st>>>(m_geom_d.as<RepGeom>(), m_rep_of.as<int>(),
                                                    m_cperm.as<int>(), d_pos(), d_q(),
                                                    m_scell.as<int>(), m_pos_ref.as<double>(),
                                                    m_n, want_spq ? m_spq.as<double4>() : nullptr,
                                                    m_spf.as<float4>()); ++m_launches;
}

// Displacement check (host decision) and list rebuild or sorted-position
// refresh: after it the pair kernel can run.
void Engine::check_lists(cudaStream_t st, bool need_spq) {
  m_check_pending = true;
  m_check_rebuild = !m_lists_valid;
  if (m_check_rebuild)
    return;
  if (!m_flag_host) {
    P3MX_CUDA(cudaMallocHost(&m_flag_host, sizeof(int)));
    P3MX_CUDA(cudaEventCreateWithFlags(&m_check_ev, cudaEventDisableTiming));
  }
  // check and refresh in one pass; the records it writes stand unless a
  // rebuild follows
  RepGeom const *geom = m_geom_d.as<RepGeom>();
  int const nb = ceil_div(m_n, 256);
  int *const flag = m_chk.as<int>() + m_chk_slot;
  m_chk_slot ^= 1;
  k_check_refresh<<<nb, 256, 0, st>>>(geom, m_rep_of.as<int>(), m_cinv.as<int>(), d_pos(), d_q(),
                                      m_ckey.as<int>(), m_pos_ref.as<double>(), d_type(),
                                      m_type_ref.as<int>(), m_n,
                                      need_spq ? m_spq.as<double4>() : nullptr,
                                      m_spf.as<float4>(), flag, m_chk.as<int>() + m_chk_slot);
  ++m_launches;
  P3MX_CUDA(cudaMemcpyAsync(m_flag_host, flag, sizeof(int), cudaMemcpyDeviceToHost, st));
  P3MX_CUDA(cudaEventRecord(m_check_ev, st));
}

void Engine::prepare_short_range(cudaStream_t st, bool need_spq) {
  if (!m_check_pending)
    check_lists(st, need_spq);
  m_check_pending = false;
  bool rebuild = m_check_rebuild;
  if (!rebuild) {
    P3MX_CUDA(cudaEventSynchronize(m_check_ev));
    rebuild = (*m_flag_host != 0);
  }
  mark("sr_check", st);
  if (rebuild) {
    build_lists(st);
    mark("sr_rebuild", st);
  }
}

// The y pass over nf field arrays field_stride complex elements apart, with
// the in-place instance when every replica's y lines allow it.
template <typename Real>
void Engine::launch_fft_y(void *c0, long long field_stride, int nf, bool inv, cudaStream_t st) {
  using C = typename CplxOf<Real>::type;
  auto const kern = m_yin ? k_fft_y<Real, true> : k_fft_y<Real, false>;
  kern<<<dim3(m_n_blk_y, nf), 256, m_smem_y, st>>>(m_geom_d.as<RepGeom>(), m_blk_y.as<Blk>(),
                                                   static_cast<C *>(c0), field_stride, m_tile_y,
                                                   inv, m_tw.as<C>());
  ++m_launches;
}

template <typename Real>
void Engine::launch_pair(double *f, bool overwrite, bool want_ev, cudaStream_t st) {
  RepGeom const *geom = m_geom_d.as<RepGeom>();
  size_t const smem = static_cast<size_t>(m_ntypes) * m_ntypes * sizeof(PairIA);
  if constexpr (sizeof(Real) == 4) {
    // FP32-mixed: cell-relative FP32 geometry
    if (want_ev)
      k_pair_forces_rel<true><<<m_n_blk_pair, 256, smem, st>>>(
          geom, m_blk_pair.as<int2>(), m_spf.as<float4>(), m_stype.as<int>(), m_cperm.as<int>(),
          m_ia_d.as<PairIA>(), m_ntypes, m_nb.as<int>(), m_nb_cnt.as<int>(), f,
          overwrite ? 1 : 0, m_part_pair.as<double>());
    else if (m_ntypes == 1 && m_ia[0].ia_cut != -1.0 && m_ia[0].lj_offset == 0.0)
      k_pair_forces_rel<false, true><<<m_n_blk_pair, 256, smem, st>>>(
          geom, m_blk_pair.as<int2>(), m_spf.as<float4>(), m_stype.as<int>(), m_cperm.as<int>(),
          m_ia_d.as<PairIA>(), m_ntypes, m_nb.as<int>(), m_nb_cnt.as<int>(), f,
          overwrite ? 1 : 0, m_part_pair.as<double>());
    else
      k_pair_forces_rel<false><<<m_n_blk_pair, 256, smem, st>>>(
          geom, m_blk_pair.as<int2>(), m_spf.as<float4>(), m_stype.as<int>(), m_cperm.as<int>(),
          m_ia_d.as<PairIA>(), m_ntypes, m_nb.as<int>(), m_nb_cnt.as<int>(), f,
          overwrite ? 1 : 0, m_part_pair.as<double>());
    ++m_launches;
  } else {
    // FP64: FP64 geometry (minimum image on absolute positions)
    if (want_ev)
      k_pair_forces<Real, true><<<m_n_blk_pair, 256, smem, st>>>(
          geom, m_blk_pair.as<int2>(), m_spq.as<double4>(), m_stype.as<int>(), m_cperm.as<int>(),
          m_ia_d.as<PairIA>(), m_ntypes, m_n, m_nb.as<int>(), m_nb_cnt.as<int>(), f,
          overwrite ? 1 : 0, m_part_pair.as<double>());
    else
      k_pair_forces<Real, false><<<m_n_blk_pair, 256, smem, st>>>(
          geom, m_blk_pair.as<int2>(), m_spq.as<double4>(), m_stype.as<int>(), m_cperm.as<int>(),
          m_ia_d.as<PairIA>(), m_ntypes, m_n, m_nb.as<int>(), m_nb_cnt.as<int>(), f,
          overwrite ? 1 : 0, m_part_pair.as<double>());
    ++m_launches;
  }
}

template <typename Real>
void Engine::short_range_t(double *f, bool overwrite, bool want_ev, cudaStream_t st) {
  if (m_n == 0)
    return;
  prepare_short_range(st, sizeof(Real) == 8);
  launch_pair<Real>(f, overwrite, want_ev, st);
  mark("pair_forces", st);
}

// Forces only (no energies or virials): the pair kernel runs on a side
// stream, concurrently with the k-space chain (sort, assignment, FFTs); the
// interpolation waits for it and adds the k-space forces on top.
void Engine::forces_all(double *f, bool overwrite, cudaStream_t st) {
  if (m_n == 0 || m_profiling) {
    long_range(f, overwrite, false, false, st, nullptr, nullptr);
    short_range(f, false, false, st, nullptr, nullptr);
    bond_forces(f, st);
    return;
  }
  // one stream: the list check, the k-space chain, then the pair kernel.
  // The host waits for the check's flag (an event behind it) while the GPU
  // runs the k-space chain, so the pair kernel (or the list rebuild) is
  // queued before the GPU gets to it.  The stage kernels each fill the GPU;
  // this measured faster than the pair kernel on a second stream beside the
  // k-space chain (1.58 vs 1.62 ms at 2^20 ions)
  check_lists(st, !m_fp32);
  try {
    long_range(f, overwrite, false, false, st, nullptr, nullptr);
  } catch (...) {
    m_check_pending = false;
    throw;
  }
  prepare_short_range(st, !m_fp32);
  if (m_fp32)
    launch_pair<float>(f, false, false, st);
  else
    launch_pair<double>(f, false, false, st);
  bond_forces(f, st);
}

void Engine::short_range(double *f, bool overwrite, bool want_ev, cudaStream_t st,
                         std::vector<double> *energies, std::vector<double> *virials,
                         bool fp64_math) {
  if (m_fp32 && !fp64_math)
    short_range_t<float>(f, overwrite, want_ev, st);
  else
    short_range_t<double>(f, overwrite, want_ev, st);
  P3MX_CUDA(cudaGetLastError());
  if (want_ev && m_n > 0) {
    int const R = n_rep();
    k_reduce_partials<<<ceil_div(R, 128), 128, 0, st>>>(m_part_pair.as<double>(), 20,
                                                        m_blk_pair_start_d.as<int>(), R,
                                                        m_sums_pair.as<double>()); ++m_launches;
    std::vector<double> sums(static_cast<size_t>(R) * 20);
    P3MX_CUDA(cudaMemcpyAsync(sums.data(), m_sums_pair.p, sums.size() * sizeof(double),
                              cudaMemcpyDeviceToHost, st));
    P3MX_CUDA(cudaStreamSynchronize(st));
    if (energies)
      energies->assign(static_cast<size_t>(R) * 2, 0.0);
    if (virials)
      virials->assign(static_cast<size_t>(R) * 18, 0.0);
    for (int r = 0; r < R; ++r) {
      if (energies) {
        (*energies)[2 * r] = sums[20 * r];
        (*energies)[2 * r + 1] = sums[20 * r + 1];
      }
      if (virials)
        for (int k = 0; k < 18; ++k)
          (*virials)[18 * r + k] = sums[20 * r + 2 + k];
    }
  }
}

// Graph-capturable short-range step: the displacement check raises a device
// flag (and one per replica), and the rebuild chain (cell binning, counting
// sort, gather, Verlet build, reference positions) runs only when it is set,
// so no host decision is needed between steps.  Only the replicas whose
// particles moved more than skin/2 rebuild: the others keep their cell keys,
// hence their sorted order, lists and reference positions.
void Engine::short_range_graph(double *f, bool overwrite, cudaStream_t st) {
  if (m_n == 0)
    return;
  RepGeom const *geom = m_geom_d.as<RepGeom>();
  int const nb = ceil_div(m_n, 256);
  int const R = n_rep();
  int *flag = m_flag.as<int>();
  int *rflag = m_rflag.as<int>();
  k_fill_int<<<1, 32, 0, st>>>(flag, 0, 1, nullptr); ++m_launches;
  k_fill_int<<<ceil_div(R, 256), 256, 0, st>>>(rflag, 0, R, nullptr); ++m_launches;
  k_displacement_check<<<nb, 256, 0, st>>>(geom, m_rep_of.as<int>(), d_pos(), m_pos_ref.as<double>(),
                                           d_type(), m_type_ref.as<int>(), m_n, flag, rflag);
  ++m_launches;
  k_fill_int<<<ceil_div(m_oct_mult * m_cells + 1, 256), 256, 0, st>>>(m_ccnt.as<int>(), 0, m_oct_mult * m_cells + 1, flag); ++m_launches;
  k_cell_bin<<<nb, 256, 0, st>>>(geom, m_rep_of.as<int>(), d_pos(), d_q(), m_n, m_ckey.as<int>(),
                                 m_cbkey.as<int>(), m_cslot.as<int>(), m_ccnt.as<int>(), m_pq.as<double4>(), nullptr, flag,
                                 rflag); ++m_launches;
  sort_keys(m_cbkey.as<int>(), m_cslot.as<int>(), m_ccnt.as<int>(), m_cstart.as<int>(),
            m_cperm.as<int>(), m_oct_mult * m_cells, st, flag);
  k_cell_gather<<<nb, 256, 0, st>>>(geom, m_rep_of.as<int>(), m_cperm.as<int>(), m_pq.as<double4>(), d_type(), m_ckey.as<int>(),
                                    m_n, m_spq.as<double4>(), m_spf.as<float4>(), m_stype.as<int>(), m_scell.as<int>(), m_cinv.as<int>(), flag); ++m_launches;
  (m_oct_mult == 8 ? k_verlet_build<true> : k_verlet_build<false>)<<<nb, 256, m_ntypes * m_ntypes * sizeof(float), st>>>(geom, m_rep_of.as<int>(), m_spq.as<double4>(),
                                       m_spf.as<float4>(), m_stype.as<int>(),
                                     m_scell.as<int>(), m_cstart.as<int>(), m_ia_d.as<PairIA>(),
                                     m_ntypes, m_n, m_nb.as<int>(), m_nb_cnt.as<int>(),
                                     m_overflow.as<int>(), flag, rflag); ++m_launches;
  k_copy_pos_ref<<<nb, 256, 0, st>>>(m_pos_ref.as<double>(), d_pos(), m_type_ref.as<int>(),
                                     d_type(), m_rep_of.as<int>(), rflag, m_n,
                                     flag); ++m_launches;
  refresh_sorted_positions(st, !m_fp32);
  if (m_fp32)
    launch_pair<float>(f, overwrite, false, st);
  else
    launch_pair<double>(f, overwrite, false, st);
}

int Engine::list_overflow(cudaStream_t st) {
  std::vector<int> ov(std::max(1, n_rep()));
  P3MX_CUDA(cudaMemcpyAsync(ov.data(), m_overflow.p, ov.size() * sizeof(int), cudaMemcpyDeviceToHost, st));
  P3MX_CUDA(cudaStreamSynchronize(st));
  return *std::max_element(ov.begin(), ov.end());
}

// Per-replica neighbour capacity from the densest local estimate
// margin * 4/3 pi (max_cut + skin)^3 rho + 48, never shrinking an existing one.
void Engine::set_list_capacity(double margin) {
  int const R = n_rep();
  bool changed = (static_cast<int>(m_cap.size()) != R) || m_nb.p == nullptr;
  m_cap.resize(R, 0);
  for (int r = 0; r < R; ++r) {
    auto const &G = m_geom[r];
    double const rc = G.max_cut + G.skin;
    double const est = margin * 4.18879 * rc * rc * rc * (G.np / G.V) + 48.0;
    int const cap = std::max(
        m_cap[r],
        (static_cast<int>(std::min(est, double(std::max<long long>(G.np, 1)))) + 1 + 7) / 8 * 8);
    changed = changed || (cap != m_cap[r]);
    m_cap[r] = cap;
  }
  // a new layout invalidates the lists; an unchanged one keeps them
  if (changed)
    layout_lists(m_stream);
}

void Engine::layout_lists(cudaStream_t st) {
  long long off = 0;
  for (int r = 0; r < n_rep(); ++r) {
    m_geom[r].nb_off = off;
    m_geom[r].max_nb = m_cap[r];
    // warp tiles of 32 particles, capacity in groups of 8 (nb_base)
    off += static_cast<long long>(m_cap[r]) * ((m_geom[r].np + 31) / 32 * 32);
  }
  m_nb.ensure(static_cast<size_t>(std::max<long long>(off, 1)) * sizeof(int));
  upload_vec(m_geom_d, m_geom, st);
  m_lists_valid = false;
}

void Engine::ensure_lists(cudaStream_t st, double nb_margin) {
  std::vector<int> before = m_cap;
  if (m_cap.size() != m_geom.size() || nb_margin > 1.0)
    set_list_capacity(std::max(nb_margin, 1.5));
  if (m_cap != before)
    m_lists_valid = false;
  if (!m_lists_valid)
    build_lists(st);
}

std::vector<int> Engine::cell_index_ghost(cudaStream_t st) {
  std::vector<int> out(m_n);
  if (m_n == 0)
    return out;
  DevBuf gi;
  gi.ensure(m_n * sizeof(int));
  P3MX_CUDA(cudaMemsetAsync(m_ccnt.p, 0, (m_oct_mult * m_cells + 1) * sizeof(int), st));
  k_cell_bin<<<ceil_div(m_n, 256), 256, 0, st>>>(m_geom_d.as<RepGeom>(), m_rep_of.as<int>(), d_pos(),
                                                 d_q(), m_n, m_ckey.as<int>(), m_cbkey.as<int>(),
                                                 m_cslot.as<int>(), m_ccnt.as<int>(),
                                                 m_pq.as<double4>(), gi.as<int>(),
                                                 nullptr, nullptr); ++m_launches;
  P3MX_CUDA(cudaMemcpyAsync(out.data(), gi.p, m_n * sizeof(int), cudaMemcpyDeviceToHost, st));
  P3MX_CUDA(cudaStreamSynchronize(st));
  m_lists_valid = false;
  return out;
}

std::vector<int> Engine::verlet_pairs(cudaStream_t st) {
  build_lists(st);
  std::vector<int> cnt(m_n), perm(m_n);
  long long total = 0;
  for (auto const &G : m_geom)
    total += static_cast<long long>(G.max_nb) * ((G.np + 31) / 32 * 32);
  std::vector<int> nbh(total);
  P3MX_CUDA(cudaMemcpyAsync(cnt.data(), m_nb_cnt.p, m_n * sizeof(int), cudaMemcpyDeviceToHost, st));
  P3MX_CUDA(cudaMemcpyAsync(perm.data(), m_cperm.p, m_n * sizeof(int), cudaMemcpyDeviceToHost, st));
  P3MX_CUDA(cudaMemcpyAsync(nbh.data(), m_nb.p, nbh.size() * sizeof(int), cudaMemcpyDeviceToHost, st));
  P3MX_CUDA(cudaStreamSynchronize(st));
  std::vector<int> pairs;
  for (auto const &G : m_geom)
    for (long long a = G.p0; a < G.p0 + G.np; ++a)
      for (int k = 0; k < nb_count(cnt[a]); ++k) {
        unsigned const ent = static_cast<unsigned>(
            nbh[nb_logical(nb_base(G.nb_off, G.max_nb, a - G.p0), G.max_nb, nb_count_a(cnt[a]), k)]);
        int const b = static_cast<int>(G.p0 + (ent & kNbIndexMask));
        int const i = perm[a], j = perm[b];
        if (i < j) {
          pairs.push_back(i);
          pairs.push_back(j);
        }
      }
  return pairs;
}

std::vector<double> Engine::mesh_copy(int r, cudaStream_t st) {
  auto const &G = m_geom[r];
  long long const ms = static_cast<long long>(G.mesh[0]) * G.mesh[1] * G.mesh[2];
  std::vector<double> out(ms);
  if (m_fp32) {
    std::vector<float> t(ms);
    P3MX_CUDA(cudaMemcpyAsync(t.data(), m_rho.as<float>() + G.rm_off, ms * sizeof(float),
                              cudaMemcpyDeviceToHost, st));
    P3MX_CUDA(cudaStreamSynchronize(st));
    for (long long k = 0; k < ms; ++k)
      out[k] = t[k];
  } else {
    P3MX_CUDA(cudaMemcpyAsync(out.data(), m_rho.as<double>() + G.rm_off, ms * sizeof(double),
                              cudaMemcpyDeviceToHost, st));
    P3MX_CUDA(cudaStreamSynchronize(st));
  }
  return out;
}

void Engine::cell_grid(int r, int *cg, double *cs) const {
  for (int d = 0; d < 3; ++d) {
    cg[d] = m_geom[r].cg[d];
    cs[d] = 1.0 / m_geom[r].inv_cs[d];
  }
}

double Engine::ks_error(const int *mesh, int cao, int n_c_part, double sum_q2, double alpha_L,
                        const double *box, double prefactor) {
  int const nblk = 296;
  m_ks_part.ensure(nblk * sizeof(double));
  k_ks_error<<<nblk, 256, 0, m_stream>>>(mesh[0], mesh[1], mesh[2], cao, alpha_L,
                                         m_ks_part.as<double>()); ++m_launches;
  std::vector<double> part(nblk);
  P3MX_CUDA(cudaMemcpyAsync(part.data(), m_ks_part.p, nblk * sizeof(double), cudaMemcpyDeviceToHost,
                            m_stream));
  P3MX_CUDA(cudaStreamSynchronize(m_stream));
  double he_q = 0.0;
  for (double v : part)
    he_q += v;
  return 2. * prefactor * sum_q2 * std::sqrt(he_q / static_cast<double>(n_c_part)) / (box[1] * box[2]);
}

void Engine::check_kernel_error(cudaStream_t st) {
  if (m_kerr.p == nullptr)
    return;
  int w[4] = {0, 0, 0, 0};
  P3MX_CUDA(cudaMemcpyAsync(w, m_kerr.p, sizeof(w), cudaMemcpyDeviceToHost, st));
  P3MX_CUDA(cudaStreamSynchronize(st));
  if (w[0] || w[1]) {
    P3MX_CUDA(cudaMemsetAsync(m_kerr.p, 0, sizeof(w), st));
    if (w[0])
      throw Error(3, "a bulk copy into shared memory did not complete within the wait limit");
    // bond_error.cpp:28-35 and the zero-distance messages of fene.hpp /
    // harmonic.hpp (runtime errors in the reference)
    if (w[1] == 1)
      throw Error(2, "bond broken between particles " + std::to_string(w[2]) + ", " +
                         std::to_string(w[3]));
    throw Error(2, "Bond: Particles " + std::to_string(w[2]) + " and " + std::to_string(w[3]) +
                       " have zero distance. This is most likely an error in the system "
                       "setup.");
  }
}

void Engine::set_bonds(std::vector<BondParam> const &types, std::vector<int> const &bonds,
                       cudaStream_t st) {
  long long const nb = static_cast<long long>(bonds.size() / 3);
  m_nbonds = 0;
  if (nb == 0)
    return;
  // CSR over particles, both ends of every bond, entries in bond order
  std::vector<int> cnt(static_cast<size_t>(m_n) + 1, 0);
  for (long long b = 0; b < nb; ++b) {
    int const t = bonds[3 * b], i = bonds[3 * b + 1], j = bonds[3 * b + 2];
    if (t < 0 || t >= static_cast<int>(types.size()))
      throw Error(1, "bond type " + std::to_string(t) + " is not defined");
    if (i < 0 || j < 0 || i >= m_n || j >= m_n || i == j)
      throw Error(1, "bond between invalid particles " + std::to_string(i) + ", " +
                         std::to_string(j));
    ++cnt[i + 1];
    ++cnt[j + 1];
  }
  for (long long i = 0; i < m_n; ++i)
    cnt[i + 1] += cnt[i];
  std::vector<int2> ent(static_cast<size_t>(2 * nb));
  std::vector<int> fill(cnt.begin(), cnt.end() - 1);
  for (long long b = 0; b < nb; ++b) {
    int const t = bonds[3 * b], i = bonds[3 * b + 1], j = bonds[3 * b + 2];
    ent[fill[i]++] = make_int2(j, t);
    ent[fill[j]++] = make_int2(i, t);
  }
  upload_vec(m_bstart, cnt, st);
  upload_vec(m_bent, ent, st);
  upload_vec(m_bparam, types, st);
  m_bpart.ensure(static_cast<size_t>(ceil_div(m_n, 256)) * 10 * sizeof(double));
  m_nbonds = nb;
  m_bond_n = m_n;
}

// CoulombP3M::pair_force / pair_energy (electrostatics/p3m.hpp:146-180) in
// FP64 for the ELC image terms.
__device__ inline void elc_p3m_pair(RepGeom const &G, double q1q2, double const d[3],
                                    double F[3], double &E) {
  double const r = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
  if (q1q2 == 0.0 || r >= G.r_cut || r <= 0.0)
    return;
  double const ad = G.alpha * r;
  double const t = 1.0 / (1.0 + 0.3275911 * ad);
  double const asp =
      t * (0.254829592 + t * (-0.284496736 + t * (1.421413741 + t * (-1.453152027 +
                                                                       t * 1.061405429))));
  double const ex = exp(-ad * ad);
  double const eri = asp / r;
  double const fac = ex * (eri + 2.0 * G.alpha / sqrt(kPi)) / (r * r) * G.prefactor * q1q2;
  F[0] += fac * d[0];
  F[1] += fac * d[1];
  F[2] += fac * d[2];
  E += G.prefactor * q1q2 * eri * ex;
}

// ELC dielectric-layer corrections (elc.hpp dielectric_layers_contribution,
// dielectric_layers_self_forces / _self_energy, add_pair_force_corrections,
// pair_energy_correction): particle a within sl of the bottom (top) wall,
// image x' = (x, y, -z) ((x, y, 2h - z)), q_eff = delta q_a q_b: a gets
// pair_force(q_eff, mi(x_b - x')) for each Verlet partner b and for itself
// (b = a); energy: half of each term.  Positions and charges are read in
// the original order through the sort permutation (always current).
template <bool EV>
__global__ void __launch_bounds__(256)
k_elc_image_pairs(const RepGeom *__restrict__ reps, const int2 *__restrict__ blk,
                  const int *__restrict__ perm, const double *__restrict__ pos,
                  const double *__restrict__ qv, const int *__restrict__ nb,
                  const int *__restrict__ nb_cnt, double sl, double h, double db, double dt,
                  double *__restrict__ f, double *__restrict__ epart) {
  int2 const bk = blk[blockIdx.x];
  RepGeom const &G = reps[bk.x];
  long long const a = G.p0 + static_cast<long long>(bk.y) * blockDim.x + threadIdx.x;
  double en = 0.0;
  if (a < G.p0 + G.np) {
    int const i = perm[a];
    double const qa = qv[i];
    double xa[3];
    for (int d = 0; d < 3; ++d)
      xa[d] = pos[3 * i + d] - floor(pos[3 * i + d] * G.box_i[d]) * G.box[d];
    bool const mb = qa != 0.0 && xa[2] < sl;
    bool const mt = qa != 0.0 && xa[2] > h - sl;
    if (mb || mt) {
      double F[3] = {0.0, 0.0, 0.0};
      int const cnt = nb_count(nb_cnt[a]), cna = nb_count_a(nb_cnt[a]);
      const int *nbp = nb + nb_base(G.nb_off, G.max_nb, a - G.p0);
      for (int side = 0; side < 2; ++side) {
        if (!(side == 0 ? mb : mt))
          continue;
        double const dl = side == 0 ? db : dt;
        double const img[3] = {xa[0], xa[1], side == 0 ? -xa[2] : 2.0 * h - xa[2]};
        double d[3];
        for (int c = 0; c < 3; ++c)
          d[c] = mi_d(xa[c] - img[c], G.box[c], G.box_i[c]);
        double E = 0.0;
        elc_p3m_pair(G, dl * qa * qa, d, F, E);
        for (int k = 0; k < cnt; ++k) {
          long long const b =
              G.p0 + static_cast<long long>(static_cast<unsigned>(nbp[nb_logical(0, G.max_nb, cna, k)]) &
                                            kNbIndexMask);
          int const j = perm[b];
          double const qb = qv[j];
          if (qb == 0.0)
            continue;
          for (int c = 0; c < 3; ++c) {
            double const xb = pos[3 * j + c] - floor(pos[3 * j + c] * G.box_i[c]) * G.box[c];
            d[c] = mi_d(xb - img[c], G.box[c], G.box_i[c]);
          }
          elc_p3m_pair(G, dl * qa * qb, d, F, E);
        }
        en += 0.5 * E;
      }
      f[3 * i + 0] += F[0];
      f[3 * i + 1] += F[1];
      f[3 * i + 2] += F[2];
    }
  }
  if constexpr (EV) {
    __shared__ double red[8];
    for (int o = 16; o > 0; o >>= 1)
      en += __shfl_down_sync(0xffffffffu, en, o);
    if ((threadIdx.x & 31) == 0)
      red[threadIdx.x >> 5] = en;
    __syncthreads();
    if (threadIdx.x == 0) {
      double s = 0.0;
      for (int w = 0; w < 8; ++w)
        s += red[w];
      epart[blockIdx.x] = s;
    }
  }
}

void Engine::elc_image_pairs(double sl, double h, double db, double dt, double *f,
                             double *energy, cudaStream_t st) {
  if (energy)
    *energy = 0.0;
  if (m_n == 0)
    return;
  RepGeom const *geom = m_geom_d.as<RepGeom>();
  if (energy) {
    m_elc_epart.ensure(static_cast<size_t>(m_n_blk_pair) * sizeof(double));
    k_elc_image_pairs<true><<<m_n_blk_pair, 256, 0, st>>>(
        geom, m_blk_pair.as<int2>(), m_cperm.as<int>(), d_pos(), d_q(), m_nb.as<int>(),
        m_nb_cnt.as<int>(), sl, h, db, dt, f, m_elc_epart.as<double>());
    ++m_launches;
    std::vector<double> ep(m_n_blk_pair);
    P3MX_CUDA(cudaMemcpyAsync(ep.data(), m_elc_epart.p, ep.size() * sizeof(double),
                              cudaMemcpyDeviceToHost, st));
    P3MX_CUDA(cudaStreamSynchronize(st));
    for (double v : ep)
      *energy += v;
  } else {
    k_elc_image_pairs<false><<<m_n_blk_pair, 256, 0, st>>>(
        geom, m_blk_pair.as<int2>(), m_cperm.as<int>(), d_pos(), d_q(), m_nb.as<int>(),
        m_nb_cnt.as<int>(), sl, h, db, dt, f, nullptr);
    ++m_launches;
  }
  P3MX_CUDA(cudaGetLastError());
}

void Engine::bond_forces(double *f, cudaStream_t st) {
  if (m_nbonds == 0)
    return;
  if (m_bond_n != m_n)
    throw Error(2, "bonds were set for a different particle count");
  k_bond_forces<<<ceil_div(m_n, 256), 256, 0, st>>>(
      m_geom_d.as<RepGeom>(), m_rep_of.as<int>(), d_pos(), m_bstart.as<int>(), m_bent.as<int2>(),
      m_bparam.as<BondParam>(), m_n, f, m_kerr.as<int>());
  ++m_launches;
}

std::vector<double> Engine::bond_energies(cudaStream_t st) {
  std::vector<double> out(m_geom.size(), 0.0);
  if (m_nbonds == 0)
    return out;
  if (m_bond_n != m_n)
    throw Error(2, "bonds were set for a different particle count");
  DevBuf e_pp;
  e_pp.ensure(static_cast<size_t>(m_n) * sizeof(double));
  k_bond_energy_pp<<<ceil_div(m_n, 256), 256, 0, st>>>(
      m_geom_d.as<RepGeom>(), m_rep_of.as<int>(), d_pos(), m_bstart.as<int>(), m_bent.as<int2>(),
      m_bparam.as<BondParam>(), m_n, e_pp.as<double>(), m_kerr.as<int>());
  ++m_launches;
  std::vector<double> h(static_cast<size_t>(m_n));
  P3MX_CUDA(cudaMemcpyAsync(h.data(), e_pp.p, h.size() * sizeof(double), cudaMemcpyDeviceToHost,
                            st));
  check_kernel_error(st); // synchronises
  for (size_t r = 0; r < m_geom.size(); ++r)
    for (long long i = m_geom[r].p0; i < m_geom[r].p0 + m_geom[r].np; ++i)
      out[r] += h[static_cast<size_t>(i)];
  return out;
}

void Engine::bond_observables(cudaStream_t st, double *energy, double *virial9) {
  for (int k = 0; k < 9; ++k)
    virial9[k] = 0.0;
  *energy = 0.0;
  if (m_nbonds == 0)
    return;
  if (m_bond_n != m_n)
    throw Error(2, "bonds were set for a different particle count");
  int const nblk = static_cast<int>(ceil_div(m_n, 256));
  k_bond_observables<<<nblk, 256, 0, st>>>(m_geom_d.as<RepGeom>(), m_rep_of.as<int>(), d_pos(),
                                           m_bstart.as<int>(), m_bent.as<int2>(),
                                           m_bparam.as<BondParam>(), m_n, m_bpart.as<double>(),
                                           m_kerr.as<int>());
  ++m_launches;
  std::vector<double> part(static_cast<size_t>(nblk) * 10);
  P3MX_CUDA(cudaMemcpyAsync(part.data(), m_bpart.p, part.size() * sizeof(double),
                            cudaMemcpyDeviceToHost, st));
  check_kernel_error(st); // synchronises
  for (int b = 0; b < nblk; ++b) {
    *energy += part[10 * b];
    for (int k = 0; k < 9; ++k)
      virial9[k] += part[10 * b + 1 + k];
  }
}

void Engine::mark(const char *name, cudaStream_t st) {
  if (!m_profiling)
    return;
  cudaEvent_t e;
  P3MX_CUDA(cudaEventCreate(&e));
  P3MX_CUDA(cudaEventRecord(e, st));
  m_marks.emplace_back(name, e);
}

std::vector<std::pair<std::string, double>> Engine::profile(int reps, cudaStream_t st) {
  std::vector<std::pair<std::string, double>> acc;
  for (int r = 0; r < reps; ++r) {
    m_marks.clear();
    m_profiling = true;
    long_range(d_force(), true, false, false, st, nullptr, nullptr);
    short_range(d_force(), false, false, st, nullptr, nullptr);
    m_profiling = false;
    P3MX_CUDA(cudaStreamSynchronize(st));
    for (size_t k = 1; k < m_marks.size(); ++k) {
      float ms = 0.f;
      P3MX_CUDA(cudaEventElapsedTime(&ms, m_marks[k - 1].second, m_marks[k].second));
      std::string const &name = m_marks[k].first;
      auto it = std::find_if(acc.begin(), acc.end(), [&](auto const &p) { return p.first == name; });
      if (it == acc.end())
        acc.emplace_back(name, ms / reps);
      else
        it->second += ms / reps;
    }
    for (auto &m : m_marks)
      cudaEventDestroy(m.second);
    m_marks.clear();
  }
  return acc;
}

} // namespace p3mx

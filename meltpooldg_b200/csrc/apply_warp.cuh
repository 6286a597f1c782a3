// Warp-per-cell operator apply (the hot path of vmult), included by
// operator_kernels.cu after the shared tables and kernel parameters.
//
// Layout and schedule:
//  * the operator's coefficients are merged per quadrature point before the
//    apply (merge_kernel): c_mass JxW and c_diff k(T_q) JxW J^-1 J^-T, so that
//    k(T) costs nothing per apply (T is fixed during a linear solve, as in the
//    reference's Newton step);
//  * a warp owns CPW = 32 / n^2 cells (n = degree + 1; one cell for Q4, two
//    for Q3, three for Q2, eight for Q1); lane (i, j) of a cell keeps the DoF
//    column (i, j, 0..n-1) in registers, so z-contractions are register FMAs
//    and x/y contractions go through a per-cell shared tile with __syncwarp
//    only -- no block-wide barrier anywhere in the cell pipeline;
//  * warps are persistent over the cells of one parity colour and software
//    pipelined: the coefficient block of the warp's next cells (padded to 16
//    bytes per cell) is brought into shared memory by one TMA bulk copy
//    (cp.async.bulk + mbarrier complete_tx) issued as soon as the stage is
//    read, and the next cells' src columns are loaded into registers while the
//    current cells are computed;
//  * scatter is atomic-free: the colours run in order 0..7 and, for every DoF,
//    the cell whose parity bits are zero in all directions in which the DoF is
//    shared with a neighbour is the first to touch it; that cell stores, later
//    colours add.  dst needs no clearing pass.
#pragma once

constexpr int kWarpsPerCTA = 4;
constexpr long kMbarSpinLimit = 1L << 26;  // bounded wait on a bulk copy

template <int n>
struct WCfg {
  static constexpr int cpw = (n == 2) ? 8 : (n == 3) ? 3 : (n == 4) ? 2 : 1;
};

__device__ __forceinline__ unsigned smem_u32(const void *p)
{
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count)
{
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, unsigned bytes)
{
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}

__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, unsigned bytes, uint64_t *bar)
{
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

// the same copy with an L2 eviction-priority hint: the coefficient stream is
// read once per apply, so it is marked evict-first and leaves the L2 to the
// DoF vectors, which the colour launches read again
__device__ __forceinline__ uint64_t l2_policy_evict_first()
{
  uint64_t pol;
  asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
  return pol;
}

__device__ __forceinline__ void bulk_g2s_hint(void *dst, const void *src, unsigned bytes, uint64_t *bar,
                                              uint64_t pol)
{
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], "
      "%4;" ::"r"(smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar)), "l"(pol)
      : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, unsigned phase)
{
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(phase)
      : "memory");
  return ok != 0;
}

// programmatic dependent launch: a colour launch may start while the previous
// colour's last cells finish; it reads src and its coefficients (which the
// previous colour does not write) at once and waits for the previous grid only
// before its first read of dst
__device__ __forceinline__ void grid_dep_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void grid_dep_launch_dependents() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

// polls of the first phase of a bounded wait before it reports expiry
// (mpdg_debug_set_wait_polls lowers it to exercise the expiry path; the retry
// phase always has the full limit, so results do not change)
__constant__ long long c_wait_first_polls = kMbarSpinLimit;

// bounded wait: on expiry the error word is set and the wait is retried once
// with the full limit, so that no copy is left targeting this CTA's shared
// memory when the kernel goes on
__device__ __forceinline__ void mbar_wait_bounded(uint64_t *bar, unsigned phase, int *err)
{
  const long long first = c_wait_first_polls;
  for (long long polls = 0;; ++polls) {
    if (polls >= first) {
      if (err) atomicExch(err, 1);
      long again = 0;
      while (!mbar_try_wait(bar, phase) && ++again < kMbarSpinLimit) {
      }
      return;
    }
    if (mbar_try_wait(bar, phase)) return;
  }
}

// ---- warp-synchronous sum factorisation with line ownership.
// The n^2 lanes of a cell own one 1D line of the n^3 tensor at a time, in one
// of three layouts (lane l = a + n b):
//   Z: lane (a, b) = (i, j) holds v[k], k = 0..n-1
//   X: lane (a, b) = (j, k) holds v[i]
//   Y: lane (a, b) = (i, k) holds v[j]
// Every 1D contraction runs in registers on the owned line (tables in
// constant memory, compile-time indices); the layout changes go through the
// cell's shared tile t[k S2 + j n + i] with n stores and n loads per lane.
// The former scheme read n^2 tile values per lane for each x or y pass.
//
// Tile layout: z-plane stride S2 and offset SC between the cells of a warp,
// the layouts with the fewest shared-memory wavefronts over the Z, X and Y
// accesses of a search over all linear layouts (64-bit accesses in two
// half-warps, 32-bit in one pass; per set of 3n accesses):
//   Q1 (8 cells per warp): S2 = 5,  SC = 12:  64-bit 24 -> 16, 32-bit 12 -> 8
//   Q2 (3 cells):          S2 = 34, SC = 9:   27 -> 24, 15 -> 12
//   Q3 (2 cells):          S2 = 19, SC = 80:  72 -> 32, 40 -> 16
//   Q4 (1 cell):           S2 = 25 (the plain layout is already the best)
// (TUNED = false: the plain layout)
template <int n, bool TUNED = true>
__host__ __device__ constexpr int tile_s2()
{
  return !TUNED ? n * n : n == 2 ? 5 : n == 3 ? 34 : n == 4 ? 19 : n * n;
}
template <int n, bool TUNED = true>
__host__ __device__ constexpr int tile_sc()
{
  return !TUNED ? n * n * n : n == 2 ? 12 : n == 3 ? 9 : n == 4 ? 80 : n * n * n;
}
// elements of one tile of a warp with plane stride S2
template <int n, int S2, bool TUNED = true>
__host__ __device__ constexpr int tile_elems()
{
  return (WCfg<n>::cpw - 1) * tile_sc<n, TUNED>() + (n - 1) * S2 + n * n;
}

template <int n, int S2 = tile_s2<n>(), typename Real>
__device__ __forceinline__ void putZ(Real *t, int a, int b, const Real (&v)[n])
{
#pragma unroll
  for (int k = 0; k < n; ++k) t[k * S2 + b * n + a] = v[k];
}
template <int n, int S2 = tile_s2<n>(), typename Real>
__device__ __forceinline__ void getZ(const Real *t, int a, int b, Real (&v)[n])
{
#pragma unroll
  for (int k = 0; k < n; ++k) v[k] = t[k * S2 + b * n + a];
}
template <int n, int S2 = tile_s2<n>(), typename Real>
__device__ __forceinline__ void putX(Real *t, int a, int b, const Real (&v)[n])
{
#pragma unroll
  for (int i = 0; i < n; ++i) t[b * S2 + a * n + i] = v[i];
}
template <int n, int S2 = tile_s2<n>(), typename Real>
__device__ __forceinline__ void getX(const Real *t, int a, int b, Real (&v)[n])
{
#pragma unroll
  for (int i = 0; i < n; ++i) v[i] = t[b * S2 + a * n + i];
}
template <int n, int S2 = tile_s2<n>(), typename Real>
__device__ __forceinline__ void putY(Real *t, int a, int b, const Real (&v)[n])
{
#pragma unroll
  for (int j = 0; j < n; ++j) t[b * S2 + j * n + a] = v[j];
}
template <int n, int S2 = tile_s2<n>(), typename Real>
__device__ __forceinline__ void getY(const Real *t, int a, int b, Real (&v)[n])
{
#pragma unroll
  for (int j = 0; j < n; ++j) v[j] = t[b * S2 + j * n + a];
}

// z-plane stride of the second tile t1.  t1 is only accessed in the Z and Y
// layouts; for Q4 in FP32 a plane stride of 37 makes both conflict-free (the
// 25-stride of t0 costs Y accesses a second wavefront).  FP64 keeps 25: its
// shared-memory traffic was measured slower with the wider tile.
template <int n, typename Real, bool TUNED = true>
__host__ __device__ constexpr int t1s2() { return (n == 5 && sizeof(Real) == 4) ? 37 : tile_s2<n, TUNED>(); }
// both tiles of a warp
template <int n, typename Real, bool TUNED = true>
__host__ __device__ constexpr int warp_tile_elems()
{
  return tile_elems<n, tile_s2<n, TUNED>(), TUNED>() + tile_elems<n, t1s2<n, Real, TUNED>(), TUNED>();
}

// Tiles of one cell group of GROUP threads: plane strides s0, s1 and cell
// offsets sc0, sc1 of t0 and t1.  GROUP = 32 is the warp-per-group apply (the
// layouts above).  GROUP = 128 lets the CTA's four warps share the cells: a
// Q4 cell has 25 lines and a Q2 cell 9, so a warp leaves 7 (Q4) or 5 (Q2) lanes
// idle, a CTA only 3 or 2 (5 Q4 cells, or 14 Q2 cells, per 128 threads).
// Their layouts come from the same wavefront search over the CTA's four
// warps (32-bit accesses in one pass, 64-bit in two half-warps): t0 over the Z,
// X and Y accesses, t1 (only Z and Y) on its own --
//   Q4 FP32: t0 25 / 125, t1 25 / 153: 100 + 60 wavefronts per 5 cells
//   Q4 FP64: t0 25 / 125, t1 27 / 137: 180 + 115
//   Q2 FP32: t0 9 / 27,   t1 11 / 41:  60 + 36 per 14 cells
//   Q2 FP64: t0 9 / 27,   t1 19 / 57:  117 + 48
// per cell the same as the warp layouts; Q1 and Q3 fill a warp exactly and
// keep their warp layouts (cell c at c sc).
template <int n, typename Real, int GROUP>
struct TileLayout {
  static constexpr bool cta = GROUP == 128 && (n == 5 || n == 3);
  static constexpr bool f64 = sizeof(Real) == 8;
  static constexpr int cells = GROUP / (n * n);
  static constexpr int s0 = cta ? n * n : tile_s2<n>();
  static constexpr int sc0 = cta ? n * n * n : tile_sc<n>();
  static constexpr int s1 = cta ? (n == 5 ? (f64 ? 27 : 25) : (f64 ? 19 : 11)) : t1s2<n, Real>();
  static constexpr int sc1 = cta ? (n == 5 ? (f64 ? 137 : 153) : (f64 ? 57 : 41)) : tile_sc<n>();
  static constexpr int t0_elems = (cells - 1) * sc0 + (n - 1) * s0 + n * n;
  static constexpr int t1_elems = (cells - 1) * sc1 + (n - 1) * s1 + n * n;
  static constexpr int elems = t0_elems + t1_elems;
};

// the plain tile layout of a warp group (z-plane stride n^2, cell offset n^3):
// one of the layouts the batched apply's autotuner tries
template <int n, typename Real>
struct PlainTileLayout {
  static constexpr int cells = 32 / (n * n);
  static constexpr int s0 = n * n, sc0 = n * n * n, s1 = n * n, sc1 = n * n * n;
  static constexpr int t0_elems = (cells - 1) * sc0 + (n - 1) * s0 + n * n;
  static constexpr int t1_elems = t0_elems;
  static constexpr int elems = t0_elems + t1_elems;
};

// the tiles of a cell group are shared by a warp (GROUP 32) or the whole CTA
template <bool CTA>
__device__ __forceinline__ void group_sync()
{
  if constexpr (CTA) __syncthreads();
  else __syncwarp();
}

// nodal values u (Z layout) -> values uq and collocation gradients gx, gy, gz
// at the Gauss points, all in Z layout.  S, Dc: tables in constant memory.
template <int n, typename Real, class L = TileLayout<n, Real, 32>, bool CTA = false>
__device__ __forceinline__ void l_forward(const Tables<Real> &T, Real *t0, Real *t1, bool wr, int a, int b,
                                          const Real (&u)[n], Real (&uq)[n], Real (&gx)[n], Real (&gy)[n],
                                          Real (&gz)[n])
{
  Real v[n], w[n];
  c1<n, Real, false, false>(T.S, T.eS, u, v);  // z: nodes -> Gauss points
  if (wr) putZ<n, L::s0>(t0, a, b, v);
  group_sync<CTA>();
  getX<n, L::s0>(t0, a, b, w);
  group_sync<CTA>();
  c1<n, Real, false, false>(T.S, T.eS, w, v);  // x
  if (wr) putX<n, L::s0>(t0, a, b, v);
  group_sync<CTA>();
  getY<n, L::s0>(t0, a, b, w);
  group_sync<CTA>();
  c1<n, Real, false, false>(T.S, T.eS, w, v);    // y: v = values at the Gauss points (Y layout)
  c1<n, Real, false, true>(T.Dc, T.eDc, v, w);   // d/dy (Y layout)
  if (wr) {
    putY<n, L::s0>(t0, a, b, v);
    putY<n, L::s1>(t1, a, b, w);
  }
  group_sync<CTA>();
  getZ<n, L::s0>(t0, a, b, uq);
  getX<n, L::s0>(t0, a, b, w);
  getZ<n, L::s1>(t1, a, b, gy);
  group_sync<CTA>();
  c1<n, Real, false, true>(T.Dc, T.eDc, uq, gz);  // d/dz (Z layout)
  c1<n, Real, false, true>(T.Dc, T.eDc, w, v);    // d/dx (X layout)
  if (wr) putX<n, L::s0>(t0, a, b, v);
  group_sync<CTA>();
  getZ<n, L::s0>(t0, a, b, gx);
  group_sync<CTA>();
}

// test functions: out = S^T (val + Dc_x^T fx + Dc_y^T fy + Dc_z^T fz) in all
// three directions; inputs at the Gauss points and output at the nodes, Z layout
template <int n, typename Real, class L = TileLayout<n, Real, 32>, bool CTA = false>
__device__ __forceinline__ void l_backward(const Tables<Real> &T, Real *t0, Real *t1, bool wr, int a, int b,
                                           const Real (&val)[n], const Real (&fx)[n], const Real (&fy)[n],
                                           const Real (&fz)[n], Real (&out)[n])
{
  Real A[n], B[n], C[n], w[n];
  c1<n, Real, true, true>(T.Dc, T.eDct, fz, A);
#pragma unroll
  for (int k = 0; k < n; ++k) A[k] += val[k];  // Z layout
  if (wr) {
    putZ<n, L::s0>(t0, a, b, fx);
    putZ<n, L::s1>(t1, a, b, fy);
  }
  group_sync<CTA>();
  getX<n, L::s0>(t0, a, b, w);
  getY<n, L::s1>(t1, a, b, C);
  group_sync<CTA>();
  c1<n, Real, true, true>(T.Dc, T.eDct, w, B);  // x part (X layout)
  c1<n, Real, true, true>(T.Dc, T.eDct, C, w);  // y part (Y layout)
  if (wr) {
    putZ<n, L::s1>(t1, a, b, A);
    putX<n, L::s0>(t0, a, b, B);
  }
  group_sync<CTA>();
  getY<n, L::s1>(t1, a, b, A);
  getY<n, L::s0>(t0, a, b, B);
  group_sync<CTA>();
#pragma unroll
  for (int q = 0; q < n; ++q) C[q] = w[q] + A[q] + B[q];  // sum in Y layout
  c1<n, Real, true, false>(T.S, T.eSt, C, w);  // y: Gauss points -> nodes
  if (wr) putY<n, L::s0>(t0, a, b, w);
  group_sync<CTA>();
  getX<n, L::s0>(t0, a, b, C);
  group_sync<CTA>();
  c1<n, Real, true, false>(T.S, T.eSt, C, w);  // x
  if (wr) putX<n, L::s0>(t0, a, b, w);
  group_sync<CTA>();
  getZ<n, L::s0>(t0, a, b, C);
  group_sync<CTA>();
  c1<n, Real, true, false>(T.S, T.eSt, C, out);  // z
}

// dynamic shared memory per cell group, in units of Real, rounded up to a
// multiple of 8 elements so that every group's stage starts on a 32-byte
// boundary (bulk copies need 16-byte aligned shared-memory destinations)
template <int P, typename Real, int GEOM, int GROUP = 32>
__host__ __device__ constexpr int warp_smem_elems(bool vel)
{
  constexpr int n = P + 1, CPW = GROUP / (n * n);
  return (((GEOM == GEOM_GENERAL ? CPW * (metric_stride(n) + (vel ? velb_stride(n) : 0)) : 0) +
           TileLayout<n, Real, GROUP>::elems) + 7) / 8 * 8;
}
constexpr int kSmemAlign = 128;  // the dynamic shared-memory base is aligned by hand

// cell (ix, iy, iz) of colour-local index cidx, by multiply-shift division
template <typename KPT>
__device__ __forceinline__ void colour_cell(int cidx, const KPT &p, int &ix, int &iy, int &iz)
{
  const unsigned x = (unsigned)cidx;
  const unsigned q0 = (unsigned)(((unsigned long long)x * p.div0_magic) >> 40);   // x / cn0
  const unsigned q01 = (unsigned)(((unsigned long long)x * p.div01_magic) >> 40); // x / (cn0 cn1)
  ix = 2 * (int)(x - q0 * (unsigned)p.cn[0]) + p.par[0];
  iy = 2 * (int)(q0 - q01 * (unsigned)p.cn[1]) + p.par[1];
  iz = 2 * (int)q01 + p.par[2];
}

template <int P, typename Real>
struct WOcc {
  static constexpr int min_blocks = (sizeof(Real) == 8) ? (P == 4 ? 3 : P == 3 ? 4 : P == 2 ? 5 : 6)
                                                       : (P == 4 ? 5 : P == 3 ? 6 : P == 2 ? 7 : 8);
};

// MULTI: applies the operator to p.nvec (<= kMaxMultiVec) vectors msrc[v] ->
// mdst[v] (msrc[0] = src, mdst[0] = dst) in one pass: each group's coefficient
// block is staged once and serves every vector
// MAPPED: a mapped mesh's cells, gathered and scattered through the
// cell->DoF map p.cmap; the mesh's greedy colouring keeps the cells of a
// launch apart, and the per-cell mask p.cell_first names the DoFs a cell
// touches first in colour order: it stores them, later colours add
// GROUP: threads that share a group of cells -- 32 (a warp per group, four
// groups per CTA) or 128 (the whole CTA per group, fewer idle lanes for Q2/Q4;
// every tile exchange is then a CTA barrier)
template <int P, typename Real, int GEOM, bool HANG = false, bool MULTI = false, bool MAPPED = false,
          int GROUP = 32>
__global__ void __launch_bounds__(kWarpsPerCTA * 32, WOcc<P, Real>::min_blocks)
    warp_apply_kernel(const KP<Real> p, int *err)
{
  static_assert(!(HANG && MULTI), "the multi-vector apply has no hanging-node path");
  static_assert(!(MAPPED && (HANG || MULTI || GEOM != GEOM_GENERAL)), "mapped meshes: general geometry, one vector");
  static_assert(GROUP == 32 || (GROUP == kWarpsPerCTA * 32 && !HANG && !MULTI && !MAPPED),
                "CTA-wide cell groups: plain applies only");
  constexpr bool CTA = GROUP != 32;
  using L = TileLayout<P + 1, Real, GROUP>;
  constexpr int n = P + 1, n2 = n * n, n3 = n2 * n, CPW = GROUP / n2;
  constexpr int GPC = kWarpsPerCTA * 32 / GROUP;  // cell groups per CTA
  constexpr int MS = metric_stride(n), VS = velb_stride(n);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ __align__(8) uint64_t bars[GPC];
  const Tables<Real> &T = tab<Real>(P);
  const int warp = CTA ? 0 : threadIdx.x >> 5, lane = CTA ? threadIdx.x : threadIdx.x & 31;
  const bool has_vel = p.vel_kind != MPDG_VEL_NONE;
  const bool gvel = GEOM == GEOM_GENERAL && has_vel;

  if (lane == 0) mbar_init(&bars[warp], 1);
  fence_mbar_init();
  __syncthreads();
  // the next colour's CTAs may be scheduled as this grid's CTAs retire
  if (p.pdl) grid_dep_launch_dependents();
  // launched as a dependent of the previous colour: dst is read only after
  // grid_dep_wait, which the first group of each warp does after its compute
  bool dep_pending = p.pdl != 0;

  unsigned char *base = smem_raw + ((kSmemAlign - (smem_u32(smem_raw) & (kSmemAlign - 1))) & (kSmemAlign - 1));
  Real *wsm = reinterpret_cast<Real *>(base) + warp * warp_smem_elems<P, Real, GEOM, GROUP>(gvel);
  Real *stage = wsm;
  Real *vstage = wsm + (GEOM == GEOM_GENERAL ? CPW * MS : 0);
  Real *tiles = wsm + (GEOM == GEOM_GENERAL ? CPW * (MS + (gvel ? VS : 0)) : 0);

  // lanes past the last cell (warp groups: Q2 5, Q4 7; CTA groups: Q2 2, Q4
  // 3) copy the position of the lane GROUP - CPW n^2 below them: their unused
  // shared-memory loads then read the same addresses as active lanes of their
  // own half-warp (a broadcast), which keeps 64-bit loads at two wavefronts
  const bool lane_ok = lane < CPW * n2;
  const int mlane = lane_ok ? lane : lane - (GROUP - CPW * n2);
  const int sub = mlane / n2, l = mlane % n2, i = l % n, j = l / n;
  const int s_sub = sub;
  Real *t0 = tiles + s_sub * L::sc0;
  Real *t1 = tiles + L::t0_elems + s_sub * L::sc1;
  // DoF offsets are 32-bit: the launcher checks that the lattice has < 2^32 DoFs
  const unsigned NXu = (unsigned)p.NX, NYu = (unsigned)p.NY, zs = NXu * NYu;
  const int count = (int)p.ccount;
  const int gstride = gridDim.x * GPC;
  unsigned phase = 0;

  auto issue_stage = [&](int grp) {
    const int c0 = grp * CPW;
    const int ncell = min(CPW, count - c0);
    const unsigned mb = ncell * MS * sizeof(Real), vb = gvel ? ncell * VS * sizeof(Real) : 0;
    fence_proxy_async();
    mbar_expect_tx(&bars[warp], mb + vb);
    if (p.stream_evict_first) {
      const uint64_t pol = l2_policy_evict_first();
      bulk_g2s_hint(stage, p.metric + (p.cfirst + c0) * (long)MS, mb, &bars[warp], pol);
      if (gvel) bulk_g2s_hint(vstage, p.velb + (p.cfirst + c0) * (long)VS, vb, &bars[warp], pol);
    } else {
      bulk_g2s(stage, p.metric + (p.cfirst + c0) * (long)MS, mb, &bars[warp]);
      if (gvel) bulk_g2s(vstage, p.velb + (p.cfirst + c0) * (long)VS, vb, &bars[warp]);
    }
  };
  // raw src column and constrained-DoF mask of the lane's cell in group grp;
  // nothing here consumes a load, so the loads stay in flight while the
  // current group is computed
  const bool use_mask = p.cell_mask != nullptr && (p.masked_read || p.masked_write);
  // the lane's cell (ix, iy, iz) in group grp and the lattice offset g0 of its
  // DoF (i, j, 0), carried from the gather to the group's compute
  // idle lanes gather their mirror lane's column too: they then compute the
  // same values and their shared-memory stores repeat the mirror's, so no
  // store needs a lane predicate (only the global scatter is restricted to
  // lane_ok lanes)
  auto gather = [&](int grp, Real (&A)[n], uint4 &cm, int &ix, int &iy, int &iz, unsigned &g0) {
    const int cidx = grp * CPW + sub;
    const bool act = grp * CPW < count && cidx < count;
    ix = 0, iy = 0, iz = 0;
    if (act) colour_cell(cidx, p, ix, iy, iz);
    g0 = ((unsigned)(iz * P) * NYu + (unsigned)(iy * P + j)) * NXu + (unsigned)(ix * P + i);
    if (HANG && act && ix == 0 && i == 0) {
      // hanging DoF (0, j, k): the coarse face's interpolant at the fine node,
      // H along y then along z (subface iy % 2, iz % 2 of coarse face (iy/2, iz/2))
      const int cy = iy >> 1, sy = iy & 1, cz = iz >> 1, sz = iz & 1;
      Real sk[n];
#pragma unroll
      for (int kp = 0; kp < n; ++kp) {
        Real sacc = 0;
#pragma unroll
        for (int jp = 0; jp < n; ++jp) {
          const long gc = ((long)(cz * P + kp) * p.hNYc + (cy * P + jp)) * p.hNXc + (p.hNXc - 1);
          const Real c = (p.masked_read && p.hmask && p.hmask[gc]) ? Real(0) : p.hsrc[gc];
          sacc += T.H[(sy * n + j) * n + jp] * c;
        }
        sk[kp] = sacc;
      }
#pragma unroll
      for (int k = 0; k < n; ++k) {
        Real sacc = 0;
#pragma unroll
        for (int kp = 0; kp < n; ++kp) sacc += T.H[(sz * n + k) * n + kp] * sk[kp];
        A[k] = sacc;
      }
    } else if (MAPPED) {
      const int *cmap = p.cmap + (p.cfirst + (long)(act ? cidx : 0)) * n3 + l;
#pragma unroll
      for (int k = 0; k < n; ++k) A[k] = act ? p.src[cmap[k * n2]] : Real(0);
    } else {
#pragma unroll
      for (int k = 0; k < n; ++k) A[k] = act ? p.src[g0 + k * zs] : Real(0);
    }
    cm = (act && use_mask) ? p.cell_mask[p.cfirst + cidx] : make_uint4(0u, 0u, 0u, 0u);
  };
  auto mask_bit = [&](const uint4 &cm, int k) -> bool {
    const int b = k * n2 + l;
    const unsigned w = (b < 32) ? cm.x : (b < 64) ? cm.y : (b < 96) ? cm.z : cm.w;
    return (w >> (b & 31)) & 1u;
  };

  int group = blockIdx.x * GPC + warp;
  if (GEOM == GEOM_GENERAL && lane == 0 && group * CPW < count) issue_stage(group);
  Real A[n];
  uint4 cmA;
  int nix, niy, niz;
  unsigned ng0;
  gather(group, A, cmA, nix, niy, niz, ng0);

  for (; group * CPW < count; group += gstride) {
    const int gnext = group + gstride;
    const bool has_next = gnext * CPW < count;
    const int cidx = group * CPW + sub;
    const bool active = lane_ok && cidx < count;
    const int ix = nix, iy = niy, iz = niz;
    const unsigned g0 = ng0;
    // constrained DoFs of the lane's column (bit k: DoF (i, j, k)); skipped as a
    // whole when no lane's cell has one (the interior of the mesh)
    unsigned lmask = 0;
    const bool cell_has_mask = (cmA.x | cmA.y | cmA.z | cmA.w) != 0u;
    bool any_mask;
    if constexpr (CTA) any_mask = __syncthreads_or(cell_has_mask) != 0;
    else any_mask = __any_sync(0xffffffffu, cell_has_mask);
    if (any_mask) {
#pragma unroll
      for (int k = 0; k < n; ++k) lmask |= (unsigned)mask_bit(cmA, k) << k;
    }
    const unsigned rmask = p.masked_read ? lmask : 0u;
    // global DoFs of the lane's column
    unsigned gk[n];
#pragma unroll
    for (int k = 0; k < n; ++k)
      gk[k] = MAPPED ? (active ? (unsigned)p.cmap[(p.cfirst + cidx) * (long)n3 + k * n2 + l] : 0u) : g0 + k * zs;

    // hanging lane of the fine block: its column is the coarse face's interpolant,
    // its slots are never written (stored 0 by the first cell), its result is staged
    const bool hl = HANG && active && ix == 0 && i == 0;
    // store-or-add decision and the early loads of the values to add to
    const bool sx = (i == 0 && ix > 0) || (i == P && ix < p.nc[0] - 1);
    const bool sy = (j == 0 && iy > 0) || (j == P && iy < p.nc[1] - 1);
    const bool later_xy = (sx && (ix & 1)) || (sy && (iy & 1));
    unsigned first_bits = 0, mask_bits = 0;
    // mapped meshes: the cell's first-touch DoFs (lowest colour among their
    // cells) from the per-cell mask; none when the mesh has no masks (dst cleared)
    uint4 cfm = make_uint4(0u, 0u, 0u, 0u);
    if constexpr (MAPPED) {
      if (p.cell_first && active) cfm = p.cell_first[p.cfirst + cidx];
    }
#pragma unroll
    for (int k = 0; k < n; ++k) {
      const bool sz = (k == 0 && iz > 0) || (k == P && iz < p.nc[2] - 1);
      const bool first = MAPPED ? mask_bit(cfm, k) : !(later_xy || (sz && (iz & 1)));
      first_bits |= (unsigned)first << k;
    }
    mask_bits = p.masked_write ? lmask : 0u;
    const int nv = MULTI ? p.nvec : 1;
    for (int v = 0; v < nv; ++v) {
    Real *dst_v = (MULTI && v > 0) ? p.mdst[v] : p.dst;
    Real dpre[n];
    const bool late_dst = dep_pending;
    auto load_dpre = [&]() {
#pragma unroll
      for (int k = 0; k < n; ++k) {
        const bool first = (first_bits >> k) & 1, masked = (mask_bits >> k) & 1;
        dpre[k] = (active && !first && !masked && !hl) ? dst_v[gk[k]] : Real(0);
      }
    };
    if (!late_dst) load_dpre();

    Real u[n];
    if (!MULTI || v == 0) {
#pragma unroll
      for (int k = 0; k < n; ++k) u[k] = A[k];
      if (has_next) gather(gnext, A, cmA, nix, niy, niz, ng0);
    } else {
      const Real *src_v = p.msrc[v];
#pragma unroll
      for (int k = 0; k < n; ++k) u[k] = (cidx < count) ? src_v[g0 + k * zs] : Real(0);
    }
    if (any_mask) {
#pragma unroll
      for (int k = 0; k < n; ++k) u[k] = ((rmask >> k) & 1u) ? Real(0) : u[k];
    }

    Real uq[n], gx[n], gy[n], gz[n];
    l_forward<n, Real, L, CTA>(T, t0, t1, true, i, j, u, uq, gx, gy, gz);

    if (GEOM == GEOM_GENERAL && v == 0) {
      mbar_wait_bounded(&bars[warp], phase, err);
      phase ^= 1;
    }

    // velocity parts that do not vary along the lane's z column (uniform mesh)
    Real uv0[3] = {0, 0, 0};
    const bool nodal_vel = GEOM != GEOM_GENERAL && p.vel_kind == MPDG_VEL_NODAL;
    if (GEOM != GEOM_GENERAL && has_vel && p.vel_kind != MPDG_VEL_ROTATION && !nodal_vel)
      uniform_velocity<Real, n>(p, T, ix, iy, iz, i, j, 0, uv0);
    // velocity given as a DoF vector on a uniform mesh: the stream JxW J^-1 u,
    // read from global memory (lanes of a cell read consecutive values)
    const Real *vq = nodal_vel ? p.velb + (p.cfirst + (cidx < count ? cidx : 0)) * (long)VS + j * n + i : nullptr;

    Real val[n], fx[n], fy[n], fz[n];
    const Real *ms = stage + s_sub * MS + j * n + i;
    const Real *vs = vstage + s_sub * VS + j * n + i;
#pragma unroll
    for (int k = 0; k < n; ++k) {
      Real b0 = 0, b1 = 0, b2 = 0;
      if (GEOM == GEOM_GENERAL) {
        const Real *m = ms + k * n2;
        const Real cm = m[0], G00 = m[n3], G01 = m[2 * n3], G02 = m[3 * n3], G11 = m[4 * n3],
                   G12 = m[5 * n3], G22 = m[6 * n3];
        if (gvel) {
          b0 = p.c_vel * vs[k * n2];
          b1 = p.c_vel * vs[k * n2 + n3];
          b2 = p.c_vel * vs[k * n2 + 2 * n3];
        }
        val[k] = cm * uq[k] + (b0 * gx[k] + b1 * gy[k] + b2 * gz[k]);
        fx[k] = G00 * gx[k] + G01 * gy[k] + G02 * gz[k];
        fy[k] = G01 * gx[k] + G11 * gy[k] + G12 * gz[k];
        fz[k] = G02 * gx[k] + G12 * gy[k] + G22 * gz[k];
      } else {
        const Real JxW = p.hvol * T.w[i] * T.w[j] * T.w[k];
        if (nodal_vel) {
          b0 = p.c_vel * vq[k * n2];
          b1 = p.c_vel * vq[k * n2 + n3];
          b2 = p.c_vel * vq[k * n2 + 2 * n3];
        } else if (has_vel) {
          Real uv[3] = {uv0[0], uv0[1], uv0[2]};
          if (p.vel_kind == MPDG_VEL_ROTATION) uniform_velocity<Real, n>(p, T, ix, iy, iz, i, j, k, uv);
          const Real cj = p.c_vel * JxW;
          b0 = cj * uv[0] * p.ih[0];
          b1 = cj * uv[1] * p.ih[1];
          b2 = cj * uv[2] * p.ih[2];
        }
        val[k] = p.c_mass * JxW * uq[k] + (b0 * gx[k] + b1 * gy[k] + b2 * gz[k]);
        const Real kd = p.c_diff * JxW;
        fx[k] = kd * p.ih2[0] * gx[k];
        fy[k] = kd * p.ih2[1] * gy[k];
        fz[k] = kd * p.ih2[2] * gz[k];
      }
    }
    if (GEOM == GEOM_GENERAL && v == nv - 1) {
      // the stage is consumed by every vector: start the next group's copy now
      group_sync<CTA>();
      if (lane == 0 && has_next) issue_stage(gnext);
    }

    Real out[n];
    l_backward<n, Real, L, CTA>(T, t0, t1, true, i, j, val, fx, fy, fz, out);

    if (HANG && __any_sync(0xffffffffu, hl)) {
      // transposed interpolation of the hanging results onto the coarse face:
      // H^T along z in registers, then along y across the cell's i = 0 lanes
      Real w[n];
#pragma unroll
      for (int kp = 0; kp < n; ++kp) {
        Real sacc = 0;
#pragma unroll
        for (int k = 0; k < n; ++k) sacc += T.H[((iz & 1) * n + k) * n + kp] * out[k];
        w[kp] = sacc;
      }
      if (hl) {
#pragma unroll
        for (int kp = 0; kp < n; ++kp) t0[j * n + kp] = w[kp];
      }
      __syncwarp();
      if (hl) {
        Real *st = p.hstage + ((long)iz * p.hnc1 + iy) * n * n;
#pragma unroll
        for (int kp = 0; kp < n; ++kp) {
          Real sacc = 0;
#pragma unroll
          for (int jj = 0; jj < n; ++jj) sacc += T.H[((iy & 1) * n + jj) * n + j] * t0[jj * n + kp];
          st[kp * n + j] = sacc;
        }
      }
      __syncwarp();
    }

    if (late_dst) {
      grid_dep_wait();
      dep_pending = false;
      load_dpre();
    }

    if (!HANG && !any_mask) {
      // no constrained DoF in the warp's cells: dpre is 0 where the cell stores first
      if (active) {
#pragma unroll
        for (int k = 0; k < n; ++k) dst_v[gk[k]] = dpre[k] + out[k];
      }
    } else if (active) {
#pragma unroll
      for (int k = 0; k < n; ++k) {
        const unsigned g = gk[k];
        if (hl) {
          if ((first_bits >> k) & 1) dst_v[g] = Real(0);
        } else if ((first_bits >> k) & 1) {
          dst_v[g] = ((mask_bits >> k) & 1) ? Real(0) : out[k];
        } else if (!((mask_bits >> k) & 1)) {
          dst_v[g] = dpre[k] + out[k];
        }
      }
    }
    }  // vectors
  }
}

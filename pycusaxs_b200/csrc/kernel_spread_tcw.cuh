// Part of the translation unit of plan.cu, which includes it inside its
// anonymous namespace; not a standalone header.
// k_spread_zdft_tcw: the default wide-tile (128-column) tensor-core spreading +
// z-DFT kernel.

// ---------------------------------------------------------------------------
// Wide-tile tensor-core spreading + z-axis DFT (k_spread_zdft_tcw)
// ---------------------------------------------------------------------------
// The same GEMM as k_spread_zdft_tc with M = 128 columns per work item (a tile
// of 8 x-columns by 16 y-rows, column m = 16*lx + ly in TMEM lane m): twice the
// columns per item halve the per-item fixed work and the halo share of the
// atoms, and M = 128 runs the tensor core at its full rate.  The tile is
// accumulated in shared memory in 32-bit fixed point (integer atomics; see
// tw_scale) as [m][z] rows of twRS words (twRS = tcR + 4, so that 8 consecutive
// rows of 16-byte loads and the 16 taps of one atom fall in distinct banks),
// then split into an f16 head and remainder straight into tensor memory, where
// the kind::f16 MMAs (K = 16) read A.
// An MMA costs about the same up to N = 192 (it is bound by its issue and
// accumulator latency, not by its N), so B holds the twiddle head and
// remainder side by side, B' = [Bh | Bl] (N' = 2*twN), and one k step is two
// MMAs, D += Ah * B' and D += Al * B', where three were needed with separate
// operands; the epilogue adds the two halves of D:
// D[:, n] + D[:, twN + n] = (Ah + Al)(Bh + Bl), all four products, and scales
// the sum back by 2^17 / scale.
// Tensor memory (512 columns):
//   [0, 256)    A ring: kTwRing = 8 slots of kTwChunk z (f16 pairs), head in
//               the first 16 columns of a slot, remainder in the next 16
//   [256, 512)  two accumulator stages of 2*twN <= 128 columns
constexpr int kTwX = 8, kTwY = 16;  // wide tile: x-columns, y-rows (M = 128)
// 20 producer warps: 864 threads leave 72 registers a thread, which the taps'
// 32-bit shared addressing needs without spills (24 warps: 64 registers)
constexpr int kTwProducerWarps = 20;
constexpr int kTwMmaWarp = kTwProducerWarps;
constexpr int kTwLoaderWarp = kTwProducerWarps + 1;
constexpr int kTwReleaseWarp = kTwProducerWarps + 6;
constexpr int kTwThreads = 32 * (kTwProducerWarps + 7);  // producers, MMA, loader, 4 epilogue, release
constexpr int kTwChunk = 32; // z per A ring slot
constexpr int kTwSlotCols = 32;  // tensor-memory columns of an A ring slot: 16 head + 16 remainder (f16 pairs)
constexpr int kTwRing = 8;   // A ring slots (two items of 128 z in flight)
static_assert(kTwRing * kTwSlotCols <= 256, "A ring and accumulator stages share 512 TMEM columns");

// Record ranges of an item's home bins (up to 4 along x times 8 along y).
struct TileAtomsW {
  int start[32];
  int cum[33];
  int nb;
};

struct TwSlot {
  TileAtomsW ta;
  int f, t, x0, y0, cw, ch;
  float mean;
  float scale;    // fixed-point scale of the item's tile (see tw_scale)
  float mean_fx;  // mean * scale
};

// The wide kernel accumulates its tile in 32-bit fixed point: shared-memory
// integer atomics issue about three times faster than FP32 ones on sm_100
// (1.97 against 6.6 cycles per warp-wide add per SM, measured).  A voxel of
// column (x, y) receives taps only from atoms whose home columns lie within
// four columns of it in x and in y: at most 3 x 3 home bins (2 x 2 unless a
// partial bin at the periodic edge is crossed), and each tap is a product of
// three B-spline weights: at most (2/3)^3 with two or more taps per axis, and
// (1/6)^3 with one (only the first cubic weight is used).  With `most` the
// largest home-bin count of the item, no voxel exceeds
// min(nvis, 9 * most) * tapmax and each rounded tap adds at most 1/2, so the
// scale 2^e with 2^e * (tapmax * bound + |mean|) <= 2e9 keeps every sum, and
// every sum minus mean * 2^e, below 2^31 in magnitude.  The scale is also kept
// at or below 2^22 / tapmax, so that a tap (below 2^22 units) can be rounded to
// an integer by adding 1.5 * 2^23 in FP32 (tap_fixed).  Each tap is rounded to
// 1/scale; at the 100k-atom workload (bound ~700, scale 2^23) that is an
// absolute error of at most 6e-8 per tap.
__device__ __forceinline__ float tw_scale(int nvis, int most, float mean, int ntaps) {
  const float tapmax = ntaps >= 2 ? 0.2964f : 0.00464f;
  const float bound = static_cast<float>(max(1, min(nvis, 9 * most)));
  const float e = floorf(log2f(2.0e9f / (tapmax * bound + fabsf(mean))));
  const float cap = floorf(log2f(4194304.0f / tapmax));
  return exp2f(fminf(e, cap));
}

// round(a * b) for 0 <= a * b < 2^22: one FMA with 1.5 * 2^23 leaves the rounded
// integer in the low mantissa bits (round to nearest even, as __float2int_rn).
__device__ __forceinline__ int tap_fixed(float a, float b) {
  return __float_as_int(fmaf(a, b, 12582912.0f)) - 0x4B400000;
}

// Padding mean of the item's type and frame, and the item's fixed-point scale:
// the loader and the epilogue evaluate the same expressions (one full warp).
__device__ __forceinline__ float tw_item_mean(const DevArgs &a, int f, int t) {
  return a.pad_val ? a.pad_val[t] : static_cast<float>(a.border[static_cast<int64_t>(f) * a.T + t] / a.border_count);
}

// Loader, first half, for wide tiles: lane 4*iy + ix loads the record range of
// home bin (hx[ix], hy[iy]); home_y holds eight bins per wide y tile.
__device__ __forceinline__ void home_ranges_load_w(const DevArgs &a, const int4 *home_x, const int4 *home_y,
                                                   int f, int t, int tx, int ty, int &s0, int &cnt,
                                                   bool &valid) {
  const int lane = threadIdx.x & 31;
  const int ix = lane & 3, iy = lane >> 2;
  const int4 hxv = home_x[tx], hyv = home_y[2 * ty + (iy >> 2)];
  const int hx = ix == 0 ? hxv.x : ix == 1 ? hxv.y : ix == 2 ? hxv.z : hxv.w;
  const int jy = iy & 3;
  const int hy = jy == 0 ? hyv.x : jy == 1 ? hyv.y : jy == 2 ? hyv.z : hyv.w;
  valid = hx >= 0 && hy >= 0;
  s0 = 0;
  cnt = 0;
  if (valid) {
    const int *off = a.offsets + static_cast<int64_t>(f) * (a.nbins + 1);
    const int bin = (t * a.tiles[1] + hy) * a.tiles[0] + hx;
    s0 = off[bin];
    cnt = off[bin + 1] - s0;
  }
}

__device__ __forceinline__ void home_ranges_publish_w(TileAtomsW &ta, int s0, int cnt, bool valid) {
  const int lane = threadIdx.x & 31;
  const unsigned bal = __ballot_sync(0xffffffffu, valid);
  const int pos = __popc(bal & ((1u << lane) - 1u));
  int inc = cnt;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const int v = __shfl_up_sync(0xffffffffu, inc, d);
    if (lane >= d) inc += v;
  }
  if (valid) {
    ta.start[pos] = s0;
    ta.cum[pos + 1] = inc;
  }
  if (lane == 0) {
    ta.cum[0] = 0;
    ta.nb = __popc(bal);
  }
}

// Pre-pass for wide tiles: as spread_prepass, with z offsets that are plain z
// rows of the [m][z] tile, and only the atoms whose stencil reaches the tile
// kept: each warp appends its reaching atoms to the table at *count (a
// shared-memory counter that starts at 0).
__device__ __forceinline__ void spread_prepass_w(const DevArgs &a, const TileAtomsW &ta, const float4 *srec,
                                                 int nrec_smem, int f, int v0, int nv, const AtomTabW &tab,
                                                 int x0, int y0, int cw, int ch, int rs, float scale, int tid,
                                                 int nthreads, int *count) {
  const int P = a.order, nt = a.ntaps, nz = a.n[2];
  const int lane = tid & 31;
  for (int i0 = tid - lane; i0 < nv; i0 += nthreads) {
    const int i = i0 + lane;
    const int v = v0 + min(i, nv - 1);
    float4 q;
    if (v < nrec_smem) {
      q = srec[v];
    } else {
      int j = 0;
      while (v >= ta.cum[j + 1]) ++j;
      q = a.rec[static_cast<int64_t>(f) * a.M + ta.start[j] + (v - ta.cum[j])];
    }
    const int m0 = static_cast<int>(q.x), m1 = static_cast<int>(q.y), m2 = static_cast<int>(q.z);
    float wx[4], wy[4], wz[4];
    cubic_weights(q.x - static_cast<float>(m0), wx);
    cubic_weights(q.y - static_cast<float>(m1), wy);
    cubic_weights(q.z - static_cast<float>(m2), wz);
    int xo[4], lyp = 0, zo[4];
    bool anyx = false;
#pragma unroll
    for (int o = 0; o < 4; ++o) {
      int by = 0xFF, zz = 0;
      xo[o] = -1;
      if (o < nt) {
        int x = m0 - P + o;
        if (x < 0) x += a.n[0];
        if (static_cast<unsigned>(x - x0) < static_cast<unsigned>(cw)) {
          xo[o] = (x - x0) * kTwY * rs;
          anyx = true;
        }
        int y = m1 - P + o;
        if (y < 0) y += a.n[1];
        if (static_cast<unsigned>(y - y0) < static_cast<unsigned>(ch)) by = y - y0;
        int z = m2 - P + o;
        if (z < 0) z += nz;
        zz = z;
      } else {
        wz[o] = 0.0f;  // a missing z tap adds 0 at row 0; a missing y tap is outside
      }
      lyp |= by << (8 * o);
      zo[o] = zz;
    }
    const bool reach = i < nv && anyx && lyp != -1;
    const unsigned m = __ballot_sync(0xffffffffu, reach);
    int base = 0;
    if (lane == 0 && m) base = atomicAdd(count, __popc(m));
    base = __shfl_sync(0xffffffffu, base, 0);
    if (reach) {
      const int e = base + __popc(m & ((1u << lane) - 1u));
      tab.wxs[e] = make_float4(wx[0] * scale, wx[1] * scale, wx[2] * scale, wx[3] * scale);
      tab.wy[e] = make_float4(wy[0], wy[1], wy[2], wy[3]);
      tab.wz[e] = make_float4(wz[0], wz[1], wz[2], wz[3]);
      tab.zo[e] = make_int4(zo[0], zo[1], zo[2], zo[3]);
      tab.xo[e] = make_int4(xo[0], xo[1], xo[2], xo[3]);
      tab.ly[e] = lyp;
    }
  }
}

// Taps for wide tiles: one lane per (atom, y tap, z tap), four x taps each, into
// the [m][z] tile (row stride rs, m = 16*lx + ly).  With rs = 4 (mod 32) the 16
// lanes of an atom write banks 4*ly + z (mod 32), all distinct.  Each thread
// takes two units per round and reads both units' table entries before either
// unit's atomics, so the shared-memory loads of one overlap the other.
struct TapUnit {
  uint32_t col;  // shared-window byte address of the unit's (y tap, z tap) row start
  int i;         // the atom's table entry, or -1 when the unit is outside
  float w;       // wy * wz
};

__device__ __forceinline__ TapUnit tap_unit(const AtomTabW &tab, int u, int nu, uint32_t A, int rs) {
  TapUnit t;
  t.i = -1;
  if (u >= nu) return t;
  const int i = u >> 4, p = (u >> 2) & 3, r = u & 3;
  const int ly = reinterpret_cast<const unsigned char *>(&tab.ly[i])[p];  // byte p
  if (ly == 0xFF) return t;
  const float wy = reinterpret_cast<const float *>(&tab.wy[i])[p];
  const float wz = reinterpret_cast<const float *>(&tab.wz[i])[r];
  const int zo = reinterpret_cast<const int *>(&tab.zo[i])[r];
  t.i = i;
  t.w = wy * wz;
  t.col = A + 4u * static_cast<uint32_t>(zo + ly * rs);
  return t;
}

__device__ __forceinline__ void tap_apply(const AtomTabW &tab, const TapUnit &t) {
  if (t.i < 0) return;
  const float4 w4 = tab.wxs[t.i];
  const int4 x4 = tab.xo[t.i];
  const float wx[4] = {w4.x, w4.y, w4.z, w4.w};
  const int xo[4] = {x4.x, x4.y, x4.z, x4.w};
#pragma unroll
  for (int o = 0; o < 4; ++o)
    if (xo[o] >= 0)
      asm volatile("red.shared.add.u32 [%0], %1;" ::"r"(t.col + 4u * static_cast<uint32_t>(xo[o])),
                   "r"(tap_fixed(wx[o], t.w))
                   : "memory");
}

__device__ __forceinline__ void spread_taps_w(const AtomTabW &tab, int nv, int *A, int rs, int tid,
                                              int nthreads) {
  const int nu = nv * 16;
  const uint32_t a32 = smem_addr(A);
  for (int u = tid; u < nu; u += 2 * nthreads) {
    const TapUnit t0 = tap_unit(tab, u, nu, a32, rs);
    const TapUnit t1 = tap_unit(tab, u + nthreads, nu, a32, rs);
    tap_apply(tab, t0);
    tap_apply(tab, t1);
  }
}

// Persistent, warp-specialized like k_spread_zdft_tc; grid = min(work items,
// SMs), block kTwThreads.  Work items w = ((f*tw_nd + i)*stw + ty)*stiles[0] + tx
// over the dense element types t = tw_types[i] (all types unless the plan sends
// the sparse ones to k_spread_zdft_sparse).
//   producer warps: twG groups on alternate items, each with its own fixed-point
//               tile and atom table: pre-pass and shared-memory taps into the
//               tile, then the split, chunk by chunk of kTwChunk z: chunk q
//               (q = j*CH + c over the CTA's items j) goes to ring slot
//               q % kTwRing once the MMAs of chunk q - kTwRing are complete;
//               warp q (mod 4) with rank h < 2 among the group's warps of that
//               lane quarter converts rows 32q..32q+31, z in [32c + 16h, +16)
//               ((tile - mean) * 2^-17 -> f16 head and remainder) with
//               tcgen05.st and zeroes what it read
//   MMA warp    one lane issues per chunk 2 x (kTwChunk/16) kind::f16 MMAs with A
//               from tensor memory (M = 128, N = 2*twN, K = 16) into the item's
//               accumulator stage, chunk by chunk as the split delivers them
//   loader warp home-bin record ranges (up to 32 bins), item data, bulk copies
//   4 epilogue  accumulator halves summed -> Z (lane m = column 16*lx + ly)
//   release     one lane waits for the MMA completion of every chunk in order
//               and publishes the count of completed chunks (`released`)
// Hand-offs (mbarriers, every wait bounded):
//   rec_full[b] / rec_empty[b]   loader <-> producers, record slot b
//   a_full[s]                    8 split units (4 lane quarters x 2) -> MMA
//   a_empty[s]                   MMA commit -> release lane
//   released                     release lane -> split warps (a counter)
//   acc_full[d] / acc_empty[d]   MMA commit -> epilogue -> MMA, stage d
// Each mbarrier has waiters that observe every one of its phases in order and
// can neither fall two phases behind nor run two ahead (parity waits cannot
// tell those apart); the ring slots, filled by both groups, are handed back
// through the monotonic counter instead.
// Dynamic shared memory: B' (tcK x 2*twN halves), twG tiles of 128 x twRS
// words, two record buffers of twRB float4, the home-bin tables (stiles[0] +
// 2*stw int4) and twG atom tables of twCap entries (kTwAtomBytes each).
__global__ void __launch_bounds__(kTwThreads, 1) k_spread_zdft_tcw(DevArgs a, int items) {
  pdl_release();
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ TwSlot slot[2];
  __shared__ __align__(8) uint64_t bars[4 + 2 * kTwRing + 4];
  __shared__ uint32_t tmem_slot;
  __shared__ volatile int abort_flag;
  __shared__ volatile int released;
  __shared__ int tab_count[2][2][2];  // reaching atoms in the table: [group][item parity][chunk parity]
  const int NB = a.twN, N = 2 * a.twN, KT = a.tcK, R = a.tcR, RB = a.twRB, RS = a.twRS, G = a.twG;
  // split warps per lane quarter: the item's 16-z units u = 2c + h (chunk c,
  // half h) go to rank u mod SR, and the other ranks pre-pass the next item
  // meanwhile (SR = 4 split faster but left the dense types' pre-pass too few
  // warps: 2.42 against 2.32 ms per 100 frames of the 100k-atom workload)
  constexpr int SR = 2;
  const int CH = (KT + kTwChunk - 1) / kTwChunk;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  float *bh = reinterpret_cast<float *>(smem);  // B' = [Bh | Bl], f16, K-major, N columns
  float *tiles = bh + KT * N / 2;
  float4 *recs = reinterpret_cast<float4 *>(tiles + static_cast<size_t>(G) * 128 * RS);
  int4 *home_x = reinterpret_cast<int4 *>(recs + 2 * RB);
  int4 *home_y = home_x + a.stiles[0];
  const int gwarps = kTwProducerWarps / G;
  const int group = warp < kTwProducerWarps ? warp / gwarps : 0;
  const int gthreads = 32 * gwarps, gtid = tid - group * gthreads;
  const int cap = a.twCap;
  AtomTabW tab;
  tab.wxs = reinterpret_cast<float4 *>(reinterpret_cast<unsigned char *>(home_y + 2 * a.stw) +
                                       static_cast<size_t>(group) * cap * kTwAtomBytes);
  tab.wy = tab.wxs + cap;
  tab.wz = tab.wy + cap;
  tab.zo = reinterpret_cast<int4 *>(tab.wz + cap);
  tab.xo = tab.zo + cap;
  tab.ly = reinterpret_cast<int *>(tab.xo + cap);
  uint64_t *rec_full = bars, *rec_empty = bars + 2, *a_full = bars + 4, *a_empty = bars + 4 + kTwRing,
           *acc_full = bars + 4 + 2 * kTwRing, *acc_empty = acc_full + 2;
  {
    const float4 *src = reinterpret_cast<const float4 *>(a.twz_tcw);
    float4 *dst = reinterpret_cast<float4 *>(bh);
    for (int i = tid; i < KT * N / 8; i += blockDim.x) dst[i] = src[i];
    float4 *t4 = reinterpret_cast<float4 *>(tiles);
    for (int i = tid; i < G * 32 * RS; i += blockDim.x) t4[i] = make_float4(0.f, 0.f, 0.f, 0.f);
    for (int i = tid; i < a.stiles[0]; i += blockDim.x) home_x[i] = a.home_x[i];
    for (int i = tid; i < 2 * a.stw; i += blockDim.x) home_y[i] = a.home_yw[i];
  }
  if (warp == kTwMmaWarp) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_addr(&tmem_slot)),
                 "r"(512));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
  }
  if (tid == 0) {
    for (int i = 0; i < 4 + 2 * kTwRing + 4; ++i) {
      int cnt = 1;
      if (i >= 4 && i < 4 + kTwRing) cnt = 8;  // a_full: 4 lane quarters x 2 units of 16 z
      if (i >= 4 + 2 * kTwRing + 2) cnt = 4;   // acc_empty: 4 epilogue warps
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(&bars[i])), "r"(cnt));
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    abort_flag = 0;
    released = 0;
    for (int i = 0; i < 8; ++i) (&tab_count[0][0][0])[i] = 0;
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_slot;
  pdl_wait();  // set-up above touched only plan constants, shared and tensor memory

  auto wait = [&](uint64_t *bar, int parity) {
    if (abort_flag) return;
    if (!mbar_wait(smem_addr(bar), static_cast<uint32_t>(parity & 1))) {
      abort_flag = 1;
      atomicOr(a.status, kStatusZ);
    }
  };
  // bounded wait until the MMAs of the first `n` chunks are complete: an acquire
  // load of the counter the release lane publishes with a release store (a
  // fence here would also wait for this warp's outstanding tap reductions)
  const uint32_t released_addr = smem_addr(const_cast<const int *>(&released));
  auto released_acquire = [&]() {
    int v;
    asm volatile("ld.acquire.cta.shared::cta.b32 %0, [%1];" : "=r"(v) : "r"(released_addr) : "memory");
    return v;
  };
  auto wait_released = [&](int n) {
    if (released_acquire() >= n || abort_flag) return;
    const uint64_t t0 = global_ns();
    while (released_acquire() < n && !abort_flag) {
      if (global_ns() - t0 > 2000000000ull) {
        abort_flag = 1;
        atomicOr(a.status, kStatusZ);
      }
      __nanosleep(64);
    }
  };

  if (warp < kTwProducerWarps) {
    const int bar_id = 1 + group;
    float *A = tiles + static_cast<size_t>(group) * 128 * RS;
    const int gw = warp - group * gwarps;          // warp within the group (groups start at multiples of 4)
    const int quarter = warp & 3, rq = gw >> 2;
    const int m = 32 * quarter + lane;             // the tile row this lane splits
    float *row = A + static_cast<size_t>(m) * RS;
    // split warps: rank < SR in their lane quarter (group threads 0..128*SR-1);
    // the group's other warps pre-pass the next item's first table chunk while
    // the split warps split the current item
    const bool splitter = rq < SR;
    const int ns_tid = gtid - 128 * SR, ns_threads = gthreads - 128 * SR;
    for (int j = group, w = blockIdx.x + group * gridDim.x; w < items; j += G, w += G * gridDim.x) {
      const int b = j & 1, ip = (j / G) & 1;
      wait(&rec_full[b], j >> 1);
      const TwSlot &sl = slot[b];
      // chunk k of an item's visible atoms counts its reaching atoms in
      // tab_count[group][item parity][k & 1]
      if (!splitter && !__any_sync(0xffffffffu, abort_flag != 0)) {
        const int nvis = sl.ta.cum[sl.ta.nb];
        spread_prepass_w(a, sl.ta, recs + static_cast<size_t>(b) * RB, min(nvis, RB), sl.f, 0, min(cap, nvis),
                         tab, sl.x0, sl.y0, sl.cw, sl.ch, RS, sl.scale, ns_tid, ns_threads, &tab_count[group][ip][0]);
      }
      // the first chunk's table is complete and the previous item's split done
      const bool skip = producers_sync_or(abort_flag != 0, bar_id, gthreads);
      if (gtid == 0) tab_count[group][ip ^ 1][0] = tab_count[group][ip ^ 1][1] = 0;  // the next item's
      const float mean_fx = sl.mean_fx;
      if (!skip) {
        const int nvis = sl.ta.cum[sl.ta.nb];
        const int nrec = min(nvis, RB);
        for (int v0 = 0, k = 0; v0 < nvis; v0 += cap, ++k) {
          if (k > 0) {
            // further chunks: all producer warps; the counter of chunk k - 1's
            // predecessor is free (its readers passed the barrier above)
            producers_sync(bar_id, gthreads);
            if (gtid == 0) tab_count[group][ip][(k + 1) & 1] = 0;
            spread_prepass_w(a, sl.ta, recs + static_cast<size_t>(b) * RB, nrec, sl.f, v0, min(cap, nvis - v0),
                             tab, sl.x0, sl.y0, sl.cw, sl.ch, RS, sl.scale, gtid, gthreads,
                             &tab_count[group][ip][k & 1]);
            producers_sync(bar_id, gthreads);
          }
          spread_taps_w(tab, tab_count[group][ip][k & 1], reinterpret_cast<int *>(A), RS, gtid, gthreads);
        }
        // diagnostic: the most table chunks an item needed
        if (gtid == 0 && nvis > cap) atomicMax(a.status + 1, (nvis + cap - 1) / cap);
      }
      producers_sync(bar_id, gthreads);
      if (gtid == 0) mbar_arrive(smem_addr(&rec_empty[b]));
      if (!splitter) continue;
      // rows z in [tcK, tcR) meet no twiddle: cleared for the next item
      for (int i = gtid; i < 128 * ((R - KT) / 4); i += 128 * SR) {
        const int mm = i / ((R - KT) / 4), zq = i % ((R - KT) / 4);
        reinterpret_cast<float4 *>(A + static_cast<size_t>(mm) * RS + KT)[zq] = make_float4(0.f, 0.f, 0.f, 0.f);
      }
      // split, in batches of up to kTwRing chunks through the A ring: one bounded
      // wait until the batch's ring slots are free (the release counter is
      // monotonic), the tensor-memory stores of this warp's units of the batch,
      // one wait for their completion, then the units' chunks handed to the MMA
      // warp (a_full counts the 8 units of a chunk, 2 per lane quarter)
      const float mz0 = -mean_fx * 0x1p-17f;
      for (int cb = 0; cb < CH; cb += kTwRing) {
        const int ce = min(CH, cb + kTwRing);
        const int q_last = j * CH + ce - 1;
        if (q_last >= kTwRing) wait_released(q_last - kTwRing + 1);
        __syncwarp();  // converged for the .sync.aligned tensor-memory stores
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        for (int u = 2 * cb + rq; u < 2 * ce; u += SR) {
          const int c = u >> 1, h = u & 1;
          const int s = (j * CH + c) % kTwRing;
          // 16 z: (tile - mean) * 2^-17 in fixed-point units, split into an f16
          // head and remainder; two halves per tensor-memory column, head to the
          // slot's columns 8h.., remainder to 16 + 8h..
          const int z0 = kTwChunk * c + 16 * h;
          uint32_t hi[8], lo[8];
          // all four loads, then the zeroing stores, then the arithmetic
          int4 iv[4];
          int4 *p = reinterpret_cast<int4 *>(row + z0);
          const int nq = z0 < KT ? 4 : 0;  // KT is a multiple of 16: all or none of the 16 z
#pragma unroll
          for (int k4 = 0; k4 < 4; ++k4) iv[k4] = k4 < nq ? p[k4] : make_int4(0, 0, 0, 0);
#pragma unroll
          for (int k4 = 0; k4 < 4; ++k4)
            if (k4 < nq) p[k4] = make_int4(0, 0, 0, 0);
          // (v - mean) * 2^-17 as one FMA: scaling by a power of two is exact, so
          // v * 2^-17 - mean * 2^-17 rounds to the same value
          const float mz = z0 < KT ? mz0 : 0.0f;
#pragma unroll
          for (int k4 = 0; k4 < 4; ++k4) {
            const float v[4] = {fmaf(__int2float_rn(iv[k4].x), 0x1p-17f, mz), fmaf(__int2float_rn(iv[k4].y), 0x1p-17f, mz),
                                fmaf(__int2float_rn(iv[k4].z), 0x1p-17f, mz), fmaf(__int2float_rn(iv[k4].w), 0x1p-17f, mz)};
#pragma unroll
            for (int e = 0; e < 4; e += 2) {
              const __half2 hh = __floats2half2_rn(v[e], v[e + 1]);
              const float2 hf = __half22float2(hh);
              const __half2 ll = __floats2half2_rn(v[e] - hf.x, v[e + 1] - hf.y);
              hi[2 * k4 + e / 2] = *reinterpret_cast<const uint32_t *>(&hh);
              lo[2 * k4 + e / 2] = *reinterpret_cast<const uint32_t *>(&ll);
            }
          }
          const uint32_t dst = tmem + (static_cast<uint32_t>(32 * quarter) << 16) +
                               static_cast<uint32_t>(kTwSlotCols * s + 8 * h);
          asm volatile("tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8};" ::"r"(dst),
                       "r"(hi[0]), "r"(hi[1]), "r"(hi[2]), "r"(hi[3]), "r"(hi[4]), "r"(hi[5]), "r"(hi[6]),
                       "r"(hi[7])
                       : "memory");
          asm volatile("tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8};" ::"r"(dst + 16),
                       "r"(lo[0]), "r"(lo[1]), "r"(lo[2]), "r"(lo[3]), "r"(lo[4]), "r"(lo[5]), "r"(lo[6]),
                       "r"(lo[7])
                       : "memory");
        }
        asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncwarp();
        if (lane == 0)
          for (int u = 2 * cb + rq; u < 2 * ce; u += SR) mbar_arrive(smem_addr(&a_full[(j * CH + (u >> 1)) % kTwRing]));
      }
    }
  } else if (warp == kTwMmaWarp) {
    if (lane == 0) {
      // kind::f16 (f16 A and B), D f32, A from tensor memory, B' K-major, N >> 3 at bit 17, M = 128
      const uint32_t idesc = (1u << 4) | (static_cast<uint32_t>(N >> 3) << 17) |
                             (static_cast<uint32_t>(128 >> 4) << 24);
      const uint64_t db0 = umma_desc(smem_addr(bh), N * 16, 128);
      const uint64_t bstep = static_cast<uint64_t>(N) * 2;  // 16 z of f16 B' in 16-byte units
      int j = 0;
      uint32_t last_bar = 0;
      int last_parity = 0;
      for (int w = blockIdx.x; w < items && !abort_flag; w += gridDim.x, ++j) {
        const int d = j & 1;
        const uint32_t dcol = tmem + 256u + static_cast<uint32_t>(128 * d);
        for (int c = 0; c < CH; ++c) {
          const int q = j * CH + c, s = q % kTwRing;
          wait(&a_full[s], q / kTwRing);
          if (c == 0 && j >= 2) wait(&acc_empty[d], (j - 2) >> 1);
          if (abort_flag) break;
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
          const int ks = min(kTwChunk, KT - kTwChunk * c) / 16;
          for (int kk = 0; kk < ks; ++kk) {
            const uint32_t ahi = tmem + static_cast<uint32_t>(kTwSlotCols * s + 8 * kk);
            const uint64_t db = db0 + static_cast<uint64_t>(kTwChunk / 16 * c + kk) * bstep;
            umma_f16_ts(dcol, ahi + 16, db, idesc, (c | kk) ? 1u : 0u);
            umma_f16_ts(dcol, ahi, db, idesc, 1u);
          }
          asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                           smem_addr(&a_empty[s]))
                       : "memory");
        }
        if (abort_flag) break;
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                         smem_addr(&acc_full[d]))
                     : "memory");
        last_bar = smem_addr(&acc_full[d]);
        last_parity = j >> 1;
      }
      if (abort_flag && last_bar) mbar_wait(last_bar, static_cast<uint32_t>(last_parity & 1));
    }
  } else if (warp == kTwLoaderWarp) {
    ItemIter it;
    it.init_dims(blockIdx.x, gridDim.x, a.stiles[0], a.stw, a.tw_nd);  // it.t: index into tw_types
    int j = 0;
    for (int w = blockIdx.x; w < items; w += gridDim.x, ++j, it.next()) {
      const int b = j & 1;
      const int x0 = it.tx * kTwX, y0 = it.ty * kTwY;
      int s0, cnt;
      bool valid;
      const int tt = a.tw_types[it.t];
      home_ranges_load_w(a, home_x, home_y, it.f, tt, it.tx, it.ty, s0, cnt, valid);
      const int most = __reduce_max_sync(0xffffffffu, static_cast<unsigned>(valid ? cnt : 0));
      const int nall = __reduce_add_sync(0xffffffffu, static_cast<unsigned>(valid ? cnt : 0));
      const float mean = tw_item_mean(a, it.f, tt);
      if (j >= 2) wait(&rec_empty[b], (j - 2) >> 1);
      if (__any_sync(0xffffffffu, abort_flag != 0)) break;
      TwSlot &sl = slot[b];
      home_ranges_publish_w(sl.ta, s0, cnt, valid);
      if (lane == 0) {
        sl.f = it.f;
        sl.t = tt;
        sl.x0 = x0;
        sl.y0 = y0;
        sl.cw = min(kTwX, a.ext[0] - x0);
        sl.ch = min(kTwY, a.ext[1] - y0);
        sl.mean = mean;
        sl.scale = tw_scale(nall, most, mean, a.ntaps);
        sl.mean_fx = mean * sl.scale;
      }
      __syncwarp();
      if (lane == 0) {
        const TileAtomsW &tb = sl.ta;
        const int nrec = min(tb.cum[tb.nb], RB);
        const uint32_t bar = smem_addr(&rec_full[b]);
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(nrec * 16)
                     : "memory");
        const float4 *src = a.rec + static_cast<int64_t>(it.f) * a.M;
        const uint32_t dst = smem_addr(recs + static_cast<size_t>(b) * RB);
        int r = 0;
        while (r < tb.nb && tb.cum[r] < nrec) {
          int e = r;
          while (e + 1 < tb.nb && tb.start[e + 1] == tb.start[e] + (tb.cum[e + 1] - tb.cum[e])) ++e;
          const int lo = tb.cum[r], hi = min(tb.cum[e + 1], nrec);
          if (hi > lo)
            asm volatile(
                "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                    dst + static_cast<uint32_t>(lo) * 16),
                "l"(src + tb.start[r]), "r"((hi - lo) * 16), "r"(bar)
                : "memory");
          r = e + 1;
        }
      }
    }
  } else if (warp == kTwReleaseWarp) {
    if (lane == 0) {
      const int mine = items > static_cast<int>(blockIdx.x)
                           ? (items - 1 - static_cast<int>(blockIdx.x)) / static_cast<int>(gridDim.x) + 1
                           : 0;
      for (int q = 0; q < mine * CH && !abort_flag; ++q) {
        wait(&a_empty[q % kTwRing], q / kTwRing);
        if (abort_flag) break;
        asm volatile("st.release.cta.shared::cta.b32 [%0], %1;" ::"r"(released_addr), "r"(q + 1) : "memory");
      }
    }
  } else {
    const int quarter = warp & 3;
    ItemIter it;
    it.init_dims(blockIdx.x, gridDim.x, a.stiles[0], a.stw, a.tw_nd);  // it.t: index into tw_types
    const int64_t zplane = static_cast<int64_t>(a.ext[0]) * a.ext[1];
    int j = 0;
    for (int w = blockIdx.x; w < items; w += gridDim.x, ++j, it.next()) {
      const int d = j & 1;
      const int tt = a.tw_types[it.t];
      // the item's fixed-point scale, as the loader computed it (before the wait,
      // so that its loads overlap it): Z = D * 2^17 / scale
      float unscale;
      {
        int s0, cnt;
        bool valid;
        home_ranges_load_w(a, home_x, home_y, it.f, tt, it.tx, it.ty, s0, cnt, valid);
        const int most = __reduce_max_sync(0xffffffffu, static_cast<unsigned>(valid ? cnt : 0));
        const int nall = __reduce_add_sync(0xffffffffu, static_cast<unsigned>(valid ? cnt : 0));
        unscale = 131072.0f / tw_scale(nall, most, tw_item_mean(a, it.f, tt), a.ntaps);
      }
      wait(&acc_full[d], j >> 1);
      if (__any_sync(0xffffffffu, abort_flag != 0)) break;
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const int x0 = it.tx * kTwX, y0 = it.ty * kTwY;
      float2 *Zft = a.Z + (static_cast<int64_t>(it.f) * a.T + tt) * a.nkz * zplane;
      const int m = 32 * quarter + lane, lx = m >> 4, ly = m & 15;
      const bool valid = lx < min(kTwX, a.ext[0] - x0) && ly < min(kTwY, a.ext[1] - y0);
      // offsets within the (frame, type) block of nkz planes fit in 32 bits
      const int zp32 = static_cast<int>(zplane);
      int off = (x0 + lx) * a.ext[1] + (y0 + ly);
      const uint32_t lane_base = tmem + (static_cast<uint32_t>(32 * quarter) << 16) + 256u +
                                 static_cast<uint32_t>(128 * d);
      for (int c0 = 0; c0 < NB; c0 += 8, off += 4 * zp32) {
        uint32_t r[8], t[8];
        asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                     : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
                       "=r"(r[7])
                     : "r"(lane_base + c0));
        asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                     : "=r"(t[0]), "=r"(t[1]), "=r"(t[2]), "=r"(t[3]), "=r"(t[4]), "=r"(t[5]), "=r"(t[6]),
                       "=r"(t[7])
                     : "r"(lane_base + NB + c0));
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        if (valid) {
          // columns past 2*nkz (NB pads it to 16) only in the last groups
          const int nk = min(4, a.nkz - c0 / 2);
#pragma unroll
          for (int jj = 0; jj < 4; ++jj)
            if (jj < nk)
              Zft[off + jj * zp32] =
                  make_float2((__uint_as_float(r[2 * jj]) + __uint_as_float(t[2 * jj])) * unscale,
                              (__uint_as_float(r[2 * jj + 1]) + __uint_as_float(t[2 * jj + 1])) * unscale);
        }
      }
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      __syncwarp();
      if (lane == 0) mbar_arrive(smem_addr(&acc_empty[d]));
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (warp == kTwMmaWarp)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512));
}


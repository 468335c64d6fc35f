// Part of the translation unit of plan.cu, which includes it inside its
// anonymous namespace; not a standalone header.
// Shared tcgen05 helpers and k_spread_zdft_tc: the 64-column tensor-core
// spreading + z-DFT kernel.

// ---------------------------------------------------------------------------
// Tensor-core z-axis DFT (tcgen05, 3xTF32)
// ---------------------------------------------------------------------------
//
// The column DFT of one 8x8 column tile is the GEMM D[c][n] = sum_z g[z][c] B[z][n]
// with M = 64 columns, N = 2*nkz (re, im interleaved, padded to a multiple of 8)
// and K = the z extent.  Both operands sit in shared memory in the K-major
// no-swizzle canonical layout of tcgen05 (core matrices of 8 rows x 16 bytes):
//   A (64 x K):  float offset (z/4)*256 + (c/8)*32 + (c%8)*4 + z%4
//                 (LBO = 1024 B between z quads, SBO = 128 B between 8-column groups)
//   B (N x K):   float offset (z/4)*(N/8)*32 + (n/8)*32 + (n%8)*4 + z%4
//                 (LBO = N*16 B, SBO = 128 B)
// Column c of the tile is (lx, ly) = (c/8, c%8).  FP32 accuracy comes from
// splitting each operand into a TF32 head (low 13 mantissa bits cleared) and the
// exact FP32 remainder: A*B ~ Ah*Bh + Ah*Bl + Al*Bh, accumulated in FP32 in
// tensor memory.  The dropped Al*Bl term and the TF32 rounding of the remainders
// are below 2^-19 of each product.
constexpr int kTcProducerWarps = 24;
constexpr int kTcProducers = 32 * kTcProducerWarps;
constexpr int kTcMmaWarp = kTcProducerWarps;
constexpr int kTcLoaderWarp = kTcProducerWarps + 1;
constexpr int kTcThreads = 32 * (kTcProducerWarps + 6);  // producers, MMA, loader, 4 epilogue warps

__device__ __forceinline__ uint32_t smem_addr(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory matrix descriptor: start, leading/stride byte offsets (>> 4),
// descriptor version 1 at bit 46, base offset 0, no swizzle.
__device__ __forceinline__ uint64_t umma_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return static_cast<uint64_t>((addr >> 4) & 0x3FFFu) |
         (static_cast<uint64_t>((lbo >> 4) & 0x3FFFu) << 16) |
         (static_cast<uint64_t>((sbo >> 4) & 0x3FFFu) << 32) | (static_cast<uint64_t>(1) << 46);
}

__device__ __forceinline__ void umma_tf32(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc,
                                          uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(idesc), "r"(accumulate), "r"(0), "r"(0), "r"(0), "r"(0));
}

// The same with A read from tensor memory (row m of A in lane m, K along columns).
__device__ __forceinline__ void umma_tf32_ts(uint32_t tmem_d, uint32_t tmem_a, uint64_t db, uint32_t idesc,
                                             uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], [%1], %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem_d),
      "r"(tmem_a), "l"(db), "r"(idesc), "r"(accumulate), "r"(0), "r"(0), "r"(0), "r"(0));
}

// The same with kind::f16 (f16 A and B, FP32 D, K = 16): A in tensor memory
// holds two K-consecutive halves per 32-bit column, the even one in the low half.
__device__ __forceinline__ void umma_f16_ts(uint32_t tmem_d, uint32_t tmem_a, uint64_t db, uint32_t idesc,
                                            uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], [%1], %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem_d),
      "r"(tmem_a), "l"(db), "r"(idesc), "r"(accumulate), "r"(0), "r"(0), "r"(0), "r"(0));
}

__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Bounded wait for the given phase parity of an mbarrier: each try suspends the
// thread until the phase completes or 0.1 ms pass (so waiting warps do not take
// issue slots from working ones); gives up after 2^16 tries or 2 s, whichever
// comes first, and returns false.
__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{\n\t.reg .pred P1;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2, %3;\n\t"
      "selp.b32 %0, 1, 0, P1;\n\t}\n"
      : "=r"(done)
      : "r"(bar), "r"(parity), "r"(100000)
      : "memory");
  return done != 0;
}

// Bounded wait: at most 2^16 + 1 tries and `limit_ns`.  The global timer is
// read only once the first try has failed (a read of it costs hundreds of
// cycles, and most waits in the pipelines below find their phase already
// complete).
__device__ __forceinline__ bool mbar_wait_for(uint32_t bar, uint32_t parity, unsigned long long limit_ns) {
  if (mbar_try(bar, parity)) return true;
  const uint64_t t0 = global_ns();
  for (int it = 0; it < (1 << 16); ++it) {
    if (mbar_try(bar, parity)) return true;
    if (global_ns() - t0 > limit_ns) return false;
  }
  return false;
}

// The pipelines' waits: 2 s.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
  return mbar_wait_for(bar, parity, 2000000000ull);
}

__device__ __forceinline__ float tf32_head(float v) {
  return __uint_as_float(__float_as_uint(v) & 0xFFFFE000u);
}

// Shared-memory bytes per entry of the spreading pre-pass atom table (the plan
// sizes the table, DevArgs::tcCap entries).
constexpr int kTcAtomBytes = 3 * 16 + 16 + 2 * 4;  // wx, wy, wz (float4), z offsets (int4), lx, ly

// What the loader publishes with an item's records: the home-bin record ranges,
// the item's frame, type and tile, and its padding mean.
struct TcSlot {
  TileAtoms ta;
  int f, t, x0, y0, cw, ch;
  float mean;
};

// Grid-stride walk over work items w = ((f*T + t)*sy + ty)*sx + tx without
// divisions after the first item: each step adds the grid size digit by digit.
struct ItemIter {
  int tx, ty, t, f;
  int dtx, dty, dt, df;
  int sx, sy, T;
  __device__ __forceinline__ void init(const DevArgs &a, int w0, int g) {
    init_dims(w0, g, a.stiles[0], a.stiles[1], a.T);
  }
  __device__ __forceinline__ void init_dims(int w0, int g, int sx_, int sy_, int T_) {
    sx = sx_;
    sy = sy_;
    T = T_;
    const int st = sx * sy;
    tx = (w0 % st) % sx;
    ty = (w0 % st) / sx;
    t = (w0 / st) % T;
    f = (w0 / st) / T;
    dtx = (g % st) % sx;
    dty = (g % st) / sx;
    dt = (g / st) % T;
    df = (g / st) / T;
  }
  __device__ __forceinline__ void next() {
    tx += dtx;
    int c = tx >= sx;
    if (c) tx -= sx;
    ty += dty + c;
    c = ty >= sy;
    if (c) ty -= sy;
    t += dt + c;
    c = t >= T;
    if (c) t -= T;
    f += df + c;
  }
};

// Loader, first half: lane 4*iy + ix of the calling warp loads the record range
// of home bin (hx[ix], hy[iy]) (bins adjacent in x are adjacent in memory).
__device__ __forceinline__ void home_ranges_load(const DevArgs &a, const int4 *home_x,
                                                 const int4 *home_y, int f, int t, int x0, int y0,
                                                 int &s0, int &cnt, bool &valid) {
  const int lane = threadIdx.x & 31;
  const int4 hxv = home_x[x0 / kTile], hyv = home_y[y0 / kTile];
  const int iy = (lane >> 2) & 3, ix = lane & 3;
  const int hx = ix == 0 ? hxv.x : ix == 1 ? hxv.y : ix == 2 ? hxv.z : hxv.w;
  const int hy = iy == 0 ? hyv.x : iy == 1 ? hyv.y : iy == 2 ? hyv.z : hyv.w;
  valid = lane < 16 && hx >= 0 && hy >= 0;
  s0 = 0;
  cnt = 0;
  if (valid) {
    const int *off = a.offsets + static_cast<int64_t>(f) * (a.nbins + 1);
    const int bin = (t * a.tiles[1] + hy) * a.tiles[0] + hx;
    s0 = off[bin];
    cnt = off[bin + 1] - s0;
  }
}

// Loader, second half: compaction and prefix sum of the ranges into `ta`.
__device__ __forceinline__ void home_ranges_publish(TileAtoms &ta, int s0, int cnt, bool valid) {
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

// Shared-memory atom table of the spreading pre-pass (struct of arrays).
struct AtomTab {
  float4 *wx, *wy, *wz;  // B-spline weights of the four taps per axis
  int4 *zo;              // A-tile offsets (z/4)*256 + z%4 of the four z taps
  int *lx, *ly;          // tile column of each x / y tap, one byte each, 0xFF outside
};

// Atom table of the wide kernel: x weights pre-multiplied by the item's
// fixed-point scale, and the four x taps' tile offsets (lx * 16 * row stride,
// -1 outside) precomputed, so that a tap costs no byte extraction or multiply.
struct AtomTabW {
  float4 *wxs, *wy, *wz;  // scale * x weights, y and z weights
  int4 *zo;               // z row of each z tap
  int4 *xo;               // tile offset of each x tap's column, -1 outside
  int *ly;                // tile row (16 * lx + ly) y part of each y tap, one byte each, 0xFF outside
};
constexpr int kTwAtomBytes = 5 * 16 + 4;

// Spreading pre-pass: atom v0 + i (i < nv) -> weights, z offsets and in-tile tap
// columns.  Records [0, nrec_smem) come from the staged copy, the rest from
// global memory.
__device__ __forceinline__ void spread_prepass(const DevArgs &a, const TileAtoms &ta,
                                               const float4 *srec, int nrec_smem, int f, int v0,
                                               int nv, const AtomTab &tab, int x0, int y0, int cw,
                                               int ch, int tid, int nthreads) {
  const int P = a.order, nt = a.ntaps, nz = a.n[2];
  for (int i = tid; i < nv; i += nthreads) {
    const int v = v0 + i;
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
    int lxp = 0, lyp = 0, zo[4];
#pragma unroll
    for (int o = 0; o < 4; ++o) {
      int bx = 0xFF, by = 0xFF, zz = 0;
      if (o < nt) {
        int x = m0 - P + o;
        if (x < 0) x += a.n[0];
        if (static_cast<unsigned>(x - x0) < static_cast<unsigned>(cw)) bx = x - x0;
        int y = m1 - P + o;
        if (y < 0) y += a.n[1];
        if (static_cast<unsigned>(y - y0) < static_cast<unsigned>(ch)) by = y - y0;
        int z = m2 - P + o;
        if (z < 0) z += nz;
        zz = (z >> 2) * 256 + (z & 3);
      }
      lxp |= bx << (8 * o);
      lyp |= by << (8 * o);
      zo[o] = zz;
    }
    tab.wx[i] = make_float4(wx[0], wx[1], wx[2], wx[3]);
    tab.wy[i] = make_float4(wy[0], wy[1], wy[2], wy[3]);
    tab.wz[i] = make_float4(wz[0], wz[1], wz[2], wz[3]);
    tab.zo[i] = make_int4(zo[0], zo[1], zo[2], zo[3]);
    tab.lx[i] = lxp;
    tab.ly[i] = lyp;
  }
}

// Spreading taps: one lane per (atom, y tap, z tap), four x taps each.  The 16
// lanes of an atom write 16 different banks (bank = 4*ly + z%4).
__device__ __forceinline__ void spread_taps(const AtomTab &tab, int nv, int nt, float *A, int tid,
                                            int nthreads) {
  for (int u = tid; u < nv * 16; u += nthreads) {
    const int i = u >> 4, p = (u >> 2) & 3, r = u & 3;
    if (p >= nt || r >= nt) continue;
    const int ly = (tab.ly[i] >> (8 * p)) & 0xFF;
    const int lxp = tab.lx[i];
    if (ly == 0xFF || lxp == -1) continue;
    const float wy = reinterpret_cast<const float *>(&tab.wy[i])[p];
    const float wz = reinterpret_cast<const float *>(&tab.wz[i])[r];
    const int zo = reinterpret_cast<const int *>(&tab.zo[i])[r];
    const float4 wx4 = tab.wx[i];
    const float wx[4] = {wx4.x, wx4.y, wx4.z, wx4.w};
    float *col = A + zo + ly * 4;
#pragma unroll
    for (int o = 0; o < 4; ++o) {
      const int lx = (lxp >> (8 * o)) & 0xFF;
      if (lx != 0xFF) atomicAdd(col + lx * 32, (wx[o] * wy) * wz);
    }
  }
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

// Named barrier `id` over `count` producer threads.
__device__ __forceinline__ void producers_sync(int id, int count) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(count) : "memory");
}

// The same barrier, also returning the OR of `v` over its threads.
__device__ __forceinline__ bool producers_sync_or(bool v, int id, int count) {
  uint32_t out;
  asm volatile(
      "{\n\t.reg .pred pi, po;\n\t"
      "setp.ne.u32 pi, %1, 0;\n\t"
      "bar.red.or.pred po, %2, %3, pi;\n\t"
      "selp.u32 %0, 1, 0, po;\n\t}\n"
      : "=r"(out)
      : "r"(static_cast<uint32_t>(v)), "r"(id), "r"(count)
      : "memory");
  return out != 0;
}

// Persistent, warp-specialized: grid = min(work items, resident CTAs), block
// kTcThreads.  Work items as in k_spread_zdft, in the same order in every role:
//   producer warps (kTcProducerWarps): zero the stage's A tile, spread the
//               item's atoms into it (a per-atom pre-pass, then shared-memory
//               atomics per tap), subtract the padding mean and split it into
//               the TF32 head (in place) and remainder.  With two operand
//               stages they form two groups that take alternate items (group g:
//               items j = g mod 2, stage and record slot g, named barrier 1 + g,
//               its own atom table), so one group's barriers and waits overlap
//               the other group's work
//   next warp   one lane issues the 3xTF32 MMAs of an item into its TMEM stage
//   next warp   loader: home-bin record ranges, frame/type/tile and padding mean
//               of an item, and bulk copies (cp.async.bulk) of its atom records
//               into a staging buffer
//   last 4      epilogue: TMEM accumulator -> Z (warp w reads lane quarter w%4)
// Hand-offs are mbarriers, every wait bounded:
//   rec_full[b]   loader -> producers (records + item data of slot b landed)
//   rec_empty[b]  producers -> loader (slot b spread)
//   full[s]       producers -> MMA (stage s operands written)
//   done[s]       MMA commit -> epilogue (accumulator ready) and producers
//                 (stage s operands free again)
//   tmem_empty[s] epilogue -> MMA (TMEM stage s read out)
// Dynamic shared memory: Bh, Bl (tcK x tcN floats each), tcS stages of
// A32 (tcR x 64) + Al (tcK x 64), two record buffers of tcRB float4, the
// home-bin tables (stiles[0] + stiles[1] int4) and one atom table per producer
// group.
__global__ void __launch_bounds__(kTcThreads, 1) k_spread_zdft_tc(DevArgs a, int items) {
  pdl_release();
  extern __shared__ __align__(16) unsigned char smem[];  // no-swizzle operands need 16 B
  __shared__ TcSlot slot[2];
  __shared__ __align__(8) uint64_t bars[10];
  __shared__ uint32_t tmem_slot;
  __shared__ volatile int abort_flag;
  const int N = a.tcN, KT = a.tcK, R = a.tcR, S = a.tcS, RB = a.tcRB;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  float *bh = reinterpret_cast<float *>(smem);
  float *bl = bh + KT * N;
  float *stages = bl + KT * N;
  float4 *recs = reinterpret_cast<float4 *>(stages + static_cast<size_t>(S) * (R + KT) * 64);
  int4 *home_x = reinterpret_cast<int4 *>(recs + 2 * RB);
  int4 *home_y = home_x + a.stiles[0];
  // producer groups: two when there are two operand stages
  const int G = (S == 2 && a.tcG == 2) ? 2 : 1;
  const int group = warp < kTcProducerWarps ? warp / (kTcProducerWarps / G) : 0;
  const int gthreads = kTcProducers / G, gtid = tid - group * gthreads;
  const int cap = a.tcCap;
  AtomTab tab;
  tab.wx = reinterpret_cast<float4 *>(reinterpret_cast<unsigned char *>(home_y + a.stiles[1]) +
                                      static_cast<size_t>(group) * cap * kTcAtomBytes);
  tab.wy = tab.wx + cap;
  tab.wz = tab.wy + cap;
  tab.zo = reinterpret_cast<int4 *>(tab.wz + cap);
  tab.lx = reinterpret_cast<int *>(tab.zo + cap);
  tab.ly = tab.lx + cap;
  uint64_t *rec_full = bars, *rec_empty = bars + 2, *full = bars + 4, *done = bars + 6,
           *tmem_empty = bars + 8;
  {
    const float4 *src = reinterpret_cast<const float4 *>(a.twz_tc);
    float4 *dst = reinterpret_cast<float4 *>(bh);
    for (int i = tid; i < KT * N / 2; i += blockDim.x) dst[i] = src[i];
    for (int i = tid; i < a.stiles[0]; i += blockDim.x) home_x[i] = a.home_x[i];
    for (int i = tid; i < a.stiles[1]; i += blockDim.x) home_y[i] = a.home_y[i];
  }
  if (warp == kTcMmaWarp) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_addr(&tmem_slot)),
                 "r"(a.tcCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
  }
  if (tid == 0) {
    const int counts[10] = {1, 1, 1, 1, kTcProducerWarps / G, kTcProducerWarps / G, 1, 1, 4, 4};
    for (int i = 0; i < 10; ++i)
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(&bars[i])), "r"(counts[i]));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    abort_flag = 0;
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_slot;
  pdl_wait();  // set-up above touched only plan constants, shared and tensor memory

  // bounded wait; on a timeout the whole block switches to skipping its work
  auto wait = [&](uint64_t *bar, int parity) {
    if (abort_flag) return;
    if (!mbar_wait(smem_addr(bar), static_cast<uint32_t>(parity & 1))) {
      abort_flag = 1;
      atomicOr(a.status, kStatusZ);
    }
  };

  if (warp < kTcProducerWarps) {
    const int bar_id = 1 + group;
    for (int j = group, w = blockIdx.x + group * gridDim.x; w < items; j += G, w += G * gridDim.x) {
      const int b = j & 1, s = S == 2 ? (j & 1) : 0;
      float *A32 = stages + static_cast<size_t>(s) * (R + KT) * 64;
      float *Al = A32 + static_cast<size_t>(R) * 64;
      if (j >= S) wait(&done[s], (j - S) / S);  // the stage's previous MMAs are finished
      {
        float4 *t4 = reinterpret_cast<float4 *>(A32);
        for (int i = gtid; i < R * 16; i += gthreads) t4[i] = make_float4(0.f, 0.f, 0.f, 0.f);
      }
      wait(&rec_full[b], j >> 1);
      // one decision for all producers: the spreading below has barriers inside
      const bool skip = producers_sync_or(abort_flag != 0, bar_id, gthreads);
      const TcSlot &sl = slot[b];
      const float mean = sl.mean;
      if (!skip) {
        const int nvis = sl.ta.cum[sl.ta.nb];
        const int nrec = min(nvis, RB);
        for (int v0 = 0; v0 < nvis; v0 += cap) {
          const int nv = min(cap, nvis - v0);
          if (v0 > 0) producers_sync(bar_id, gthreads);  // the previous chunk's taps have read the table
          spread_prepass(a, sl.ta, recs + static_cast<size_t>(b) * RB, nrec, sl.f, v0, nv, tab, sl.x0,
                         sl.y0, sl.cw, sl.ch, gtid, gthreads);
          producers_sync(bar_id, gthreads);
          spread_taps(tab, nv, a.ntaps, A32, gtid, gthreads);
        }
      }
      producers_sync(bar_id, gthreads);
      if (gtid == 0) mbar_arrive(smem_addr(&rec_empty[b]));
      {
        // padding mean applied before the TF32 split: the tensor cores see
        // g - mean (rows z >= ez meet zero twiddles)
        float4 *h4 = reinterpret_cast<float4 *>(A32);
        float4 *l4 = reinterpret_cast<float4 *>(Al);
        for (int i = gtid; i < KT * 16; i += gthreads) {
          float4 v = h4[i];
          v.x -= mean;
          v.y -= mean;
          v.z -= mean;
          v.w -= mean;
          const float4 h = make_float4(tf32_head(v.x), tf32_head(v.y), tf32_head(v.z), tf32_head(v.w));
          h4[i] = h;
          l4[i] = make_float4(v.x - h.x, v.y - h.y, v.z - h.z, v.w - h.w);
        }
      }
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      __syncwarp();
      if (lane == 0) mbar_arrive(smem_addr(&full[s]));
    }
  } else if (warp == kTcMmaWarp) {
    if (lane == 0) {
      // kind::tf32 instruction descriptor: D f32 (bits 4-5 = 1), A and B tf32 (2),
      // both K-major, N >> 3 at bit 17, M >> 4 at bit 24 (M = 64).
      const uint32_t idesc = (1u << 4) | (2u << 7) | (2u << 10) |
                             (static_cast<uint32_t>(N >> 3) << 17) | (static_cast<uint32_t>(64 >> 4) << 24);
      const uint32_t bstep = static_cast<uint32_t>(N) * 32;  // bytes per 8 z of B
      const uint64_t dbh0 = umma_desc(smem_addr(bh), N * 16, 128);
      const uint64_t dbl0 = umma_desc(smem_addr(bl), N * 16, 128);
      int j = 0;
      uint32_t last_bar = 0;
      int last_parity = 0;
      for (int w = blockIdx.x; w < items && !abort_flag; w += gridDim.x, ++j) {
        const int s = S == 2 ? (j & 1) : 0;
        const float *A32 = stages + static_cast<size_t>(s) * (R + KT) * 64;
        const float *Al = A32 + static_cast<size_t>(R) * 64;
        wait(&full[s], j / S);
        if (j >= S) wait(&tmem_empty[s], (j - S) / S);
        if (abort_flag) break;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t d = tmem + static_cast<uint32_t>(s * N);
        const uint64_t dah0 = umma_desc(smem_addr(A32), 1024, 128);
        const uint64_t dal0 = umma_desc(smem_addr(Al), 1024, 128);
        // descriptor start addresses are in 16-byte units: one k step of A is
        // 2048 B (+128), of B N*32 B (+N*2)
        for (int kk = 0; kk < KT / 8; ++kk) {
          const uint64_t dah = dah0 + static_cast<uint64_t>(kk * 128);
          const uint64_t dal = dal0 + static_cast<uint64_t>(kk * 128);
          const uint64_t dbh = dbh0 + static_cast<uint64_t>(kk * (bstep >> 4));
          const uint64_t dbl = dbl0 + static_cast<uint64_t>(kk * (bstep >> 4));
          umma_tf32(d, dal, dbh, idesc, kk > 0 ? 1u : 0u);
          umma_tf32(d, dah, dbl, idesc, 1u);
          umma_tf32(d, dah, dbh, idesc, 1u);
        }
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                         smem_addr(&done[s]))
                     : "memory");
        last_bar = smem_addr(&done[s]);
        last_parity = j / S;
      }
      // a wait ran out somewhere: let the newest MMAs finish (bounded) before the
      // tensor memory is released
      if (abort_flag && last_bar) mbar_wait(last_bar, static_cast<uint32_t>(last_parity & 1));
    }
  } else if (warp == kTcLoaderWarp) {
    ItemIter it;
    it.init(a, blockIdx.x, gridDim.x);
    int j = 0;
    for (int w = blockIdx.x; w < items; w += gridDim.x, ++j, it.next()) {
      const int b = j & 1;
      const int x0 = it.tx * kTile, y0 = it.ty * kTile;
      int s0, cnt;
      bool valid;
      // the range and mean loads are issued before the wait for the slot
      home_ranges_load(a, home_x, home_y, it.f, it.t, x0, y0, s0, cnt, valid);
      const float pmean = a.pad_val ? a.pad_val[it.t] : 0.0f;
      const double bsum = a.pad_val ? 0.0 : a.border[static_cast<int64_t>(it.f) * a.T + it.t];
      if (j >= 2) wait(&rec_empty[b], (j - 2) >> 1);
      if (__any_sync(0xffffffffu, abort_flag != 0)) break;
      TcSlot &sl = slot[b];
      home_ranges_publish(sl.ta, s0, cnt, valid);
      if (lane == 0) {
        sl.f = it.f;
        sl.t = it.t;
        sl.x0 = x0;
        sl.y0 = y0;
        sl.cw = min(kTile, a.ext[0] - x0);
        sl.ch = min(kTile, a.ext[1] - y0);
        sl.mean = a.pad_val ? pmean : static_cast<float>(bsum / a.border_count);
      }
      __syncwarp();
      if (lane == 0) {
        const TileAtoms &tb = sl.ta;
        const int nrec = min(tb.cum[tb.nb], RB);
        const uint32_t bar = smem_addr(&rec_full[b]);
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar),
                     "r"(nrec * 16)
                     : "memory");
        const float4 *src = a.rec + static_cast<int64_t>(it.f) * a.M;
        const uint32_t dst = smem_addr(recs + static_cast<size_t>(b) * RB);
        // one bulk copy per run of ranges that are contiguous in global memory
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
  } else {
    // epilogue warps
    const int quarter = warp & 3;
    ItemIter it;
    it.init(a, blockIdx.x, gridDim.x);
    const int64_t zplane = static_cast<int64_t>(a.ext[0]) * a.ext[1];
    int j = 0;
    for (int w = blockIdx.x; w < items; w += gridDim.x, ++j, it.next()) {
      const int s = S == 2 ? (j & 1) : 0;
      wait(&done[s], j / S);
      if (__any_sync(0xffffffffu, abort_flag != 0)) break;
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const int x0 = it.tx * kTile, y0 = it.ty * kTile;
      float2 *Zft = a.Z + (static_cast<int64_t>(it.f) * a.T + it.t) * a.nkz * zplane;
      // with M = 64, row c of D sits in TMEM lane (c % 16) + 32 * (c / 16)
      const int c = 16 * quarter + lane, lx = c >> 3, ly = c & 7;
      const bool valid = lane < 16 && lx < min(kTile, a.ext[0] - x0) && ly < min(kTile, a.ext[1] - y0);
      const int64_t cell = static_cast<int64_t>(x0 + lx) * a.ext[1] + (y0 + ly);
      const uint32_t lane_base = tmem + (static_cast<uint32_t>(32 * quarter) << 16) + static_cast<uint32_t>(s * N);
      for (int c0 = 0; c0 < N; c0 += 8) {
        uint32_t r[8];
        asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                     : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]),
                       "=r"(r[6]), "=r"(r[7])
                     : "r"(lane_base + c0));
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        if (valid) {
#pragma unroll
          for (int jj = 0; jj < 4; ++jj) {
            const int kz = c0 / 2 + jj;
            if (kz < a.nkz)
              Zft[kz * zplane + cell] = make_float2(__uint_as_float(r[2 * jj]), __uint_as_float(r[2 * jj + 1]));
          }
        }
      }
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      __syncwarp();
      if (lane == 0) mbar_arrive(smem_addr(&tmem_empty[s]));
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (warp == kTcMmaWarp)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(a.tcCols));
}



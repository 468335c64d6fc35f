// Part of the translation unit of plan.cu, which includes it inside its
// anonymous namespace; not a standalone header.
// k_spread_zdft_ag: spreading + z-axis DFT as one tensor-core GEMM over atoms.

// ---------------------------------------------------------------------------
// Atom-GEMM spreading + z-axis DFT (k_spread_zdft_ag)
// ---------------------------------------------------------------------------
// For a tile of 8 x-columns by 16 y-rows (column m = 16 lx + ly, M = 128, the
// tiles of k_spread_zdft_tcw) the z-transformed columns are
//   Z[m][kz] = sum_a W[m][a] S[a][kz] - mean * sum_{z < ez} tw[z][kz],
// the sum over the atoms a whose stencil reaches the tile, with W[m][a] =
// wx(lx) * wy(ly) the atom's weight on column m (16 non-zeros per atom) and
// S[a][kz] = sum_o wz(o) tw[z_o][kz] the transform of its z taps.  That is a
// GEMM whose K runs over atoms: the spreading itself runs on the tensor cores,
// with no shared-memory atomics and no per-voxel tile to convert.  Per chunk of
// kAgK atoms the producer warps write W - f16 head and rounded remainder, each
// 128 x kAgK K-major in shared memory, zeroed first - and S, whose head and
// remainder sit side by side (B' = [Sh | Sl], kAgK x N2 with N2 = 2 * NB), and
// one thread issues per 16 atoms two kind::f16 MMAs, D += Wh B' and D += Wl B'
// (M = 128, N = N2, K = 16).  The epilogue adds the two halves of D (all four
// products, 22 bits of each operand, as k_spread_zdft_tcw), subtracts the
// transform of the padding mean and writes Z.  An item's cost grows with its
// atoms only: an element type with few atoms per tile costs one chunk, where
// the dense-tile kernels pay a fixed per-item conversion of 128 x 128 voxels.
//
// Shared-memory operands, K-major without swizzle (core matrices of 8 rows x 16
// bytes):  W half (m, k) at ((k / 8) * 128 + m) * 8 + k % 8   (LBO 2048 B, SBO 128 B)
//          B' half (k, n) at ((k / 8) * N2 + n) * 8 + k % 8   (LBO N2 * 16 B, SBO 128 B)
constexpr int kAgK = 64;                 // atoms per chunk
constexpr int kAgSlots = 2;              // chunk slots (W head, W remainder, B')
constexpr int kAgProducerWarps = 24;
constexpr int kAgProducers = 32 * kAgProducerWarps;
constexpr int kAgMmaWarp = kAgProducerWarps;
constexpr int kAgLoaderWarp = kAgProducerWarps + 1;
constexpr int kAgThreads = 32 * (kAgProducerWarps + 6);  // producers, MMA, loader, 4 epilogue
constexpr int kAgBar = 1;                // named barrier of the producer warps
constexpr int kAgAtomBytes = 4 * 16 + 8; // atom table entry (see AgTab)
constexpr size_t kAgWBytes = static_cast<size_t>(128) * kAgK * 2;  // one W operand (f16)

// Reaching atoms of the current table chunk.
struct AgTab {
  float4 *wx, *wy, *wz;  // B-spline weights of the four taps per axis (0 for missing z taps)
  int4 *zo;              // z row of each z tap
  int2 *lxy;             // in-tile column of each x tap and row of each y tap, one byte each, 0xFF outside
};

struct AgSlot {
  TileAtomsW ta;
  int f, t, x0, y0, cw, ch;
};

struct AgChunk {
  int kc;     // atoms in the chunk (0: an empty chunk that only zeroes or closes the item)
  int first;  // the item's first chunk: the MMAs start a fresh accumulator
  int last;   // the item's last chunk: the accumulator goes to the epilogue
};

__device__ __forceinline__ void umma_f16_ss(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc,
                                            uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(idesc), "r"(accumulate), "r"(0), "r"(0), "r"(0), "r"(0));
}

__device__ __forceinline__ void st_half(uint16_t *p, float v) {
  *p = __half_as_ushort(__float2half_rn(v));
}

// Pre-pass: visible atom v0 + i (i < nv) -> weights, z rows and in-tile tap
// columns; the atoms whose stencil reaches the tile are appended to the table
// at *count (a shared counter that starts at 0).  Records [0, nrec_smem) come
// from the staged copy, the rest from global memory.
__device__ __forceinline__ void ag_prepass(const DevArgs &a, const TileAtomsW &ta, const float4 *srec,
                                           int nrec_smem, int f, int v0, int nv, const AgTab &tab, int x0,
                                           int y0, int cw, int ch, int tid, int nthreads, int *count) {
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
    int lxp = 0, lyp = 0, zo[4];
    bool anyx = false, anyy = false;
#pragma unroll
    for (int o = 0; o < 4; ++o) {
      int bx = 0xFF, by = 0xFF, zz = 0;
      if (o < nt) {
        int x = m0 - P + o;
        if (x < 0) x += a.n[0];
        if (static_cast<unsigned>(x - x0) < static_cast<unsigned>(cw)) {
          bx = x - x0;
          anyx = true;
        }
        int y = m1 - P + o;
        if (y < 0) y += a.n[1];
        if (static_cast<unsigned>(y - y0) < static_cast<unsigned>(ch)) {
          by = y - y0;
          anyy = true;
        }
        int z = m2 - P + o;
        if (z < 0) z += nz;
        zz = z;
      } else {
        wz[o] = 0.0f;  // a missing tap: no z weight and no column
      }
      lxp |= bx << (8 * o);
      lyp |= by << (8 * o);
      zo[o] = zz;
    }
    const bool reach = i < nv && anyx && anyy;
    const unsigned msk = __ballot_sync(0xffffffffu, reach);
    int base = 0;
    if (lane == 0 && msk) base = atomicAdd(count, __popc(msk));
    base = __shfl_sync(0xffffffffu, base, 0);
    if (reach) {
      const int e = base + __popc(msk & ((1u << lane) - 1u));
      tab.wx[e] = make_float4(wx[0], wx[1], wx[2], wx[3]);
      tab.wy[e] = make_float4(wy[0], wy[1], wy[2], wy[3]);
      tab.wz[e] = make_float4(wz[0], wz[1], wz[2], wz[3]);
      tab.zo[e] = make_int4(zo[0], zo[1], zo[2], zo[3]);
      tab.lxy[e] = make_int2(lxp, lyp);
    }
  }
}

// The operands of table atoms [k0, k0 + kc) in one chunk slot: W (head, Wh, and
// remainder, Wl; zeroed beforehand) and B' = [Sh | Sl].  W: two atoms per warp
// pass, a lane per (x tap, y tap).  S: a warp per atom, a lane per kz (and
// kz + 32), reading the z twiddles tws[z][kz] from shared memory (the kernel's
// shared memory leaves too little L1 to keep them cached).
__device__ __forceinline__ void ag_operands(const DevArgs &a, const AgTab &tab, const float2 *tws, int k0, int kc,
                                            uint16_t *Wh, uint16_t *Wl, uint16_t *Bp, int NB, int tid,
                                            int nthreads) {
  const int N2 = 2 * NB;
  const int lane = tid & 31, warp = tid >> 5, nwarps = nthreads >> 5;
  for (int p = warp; 2 * p < kc; p += nwarps) {
    const int kk = 2 * p + (lane >> 4);
    if (kk < kc) {
      const int ox = (lane >> 2) & 3, oy = lane & 3;
      const int2 lxy = tab.lxy[k0 + kk];
      const int lx = (lxy.x >> (8 * ox)) & 0xFF, ly = (lxy.y >> (8 * oy)) & 0xFF;
      if (lx != 0xFF && ly != 0xFF) {
        const float w = reinterpret_cast<const float *>(&tab.wx[k0 + kk])[ox] *
                        reinterpret_cast<const float *>(&tab.wy[k0 + kk])[oy];
        const __half h = __float2half_rn(w);
        const int idx = ((kk >> 3) * 128 + 16 * lx + ly) * 8 + (kk & 7);
        Wh[idx] = __half_as_ushort(h);
        st_half(Wl + idx, w - __half2float(h));
      }
    }
  }
  // taps on rows z >= ez meet no twiddle
  const int nkz = a.nkz, ez = a.ext[2];
  for (int kk = warp; kk < kc; kk += nwarps) {
    const float4 wz4 = tab.wz[k0 + kk];
    const int4 zo4 = tab.zo[k0 + kk];
    const float wz[4] = {wz4.x, wz4.y, wz4.z, wz4.w};
    const int zo[4] = {zo4.x, zo4.y, zo4.z, zo4.w};
    const int base = (kk >> 3) * N2 * 8 + (kk & 7);
    for (int kz = lane; kz < nkz; kz += 32) {
      float sr = 0.0f, si = 0.0f;
#pragma unroll
      for (int o = 0; o < 4; ++o) {
        if (zo[o] < ez && wz[o] != 0.0f) {
          const float2 tw = tws[zo[o] * nkz + kz];
          sr = fmaf(wz[o], tw.x, sr);
          si = fmaf(wz[o], tw.y, si);
        }
      }
      const __half hr = __float2half_rn(sr), hi = __float2half_rn(si);
      Bp[base + (2 * kz) * 8] = __half_as_ushort(hr);
      Bp[base + (2 * kz + 1) * 8] = __half_as_ushort(hi);
      st_half(Bp + base + (NB + 2 * kz) * 8, sr - __half2float(hr));
      st_half(Bp + base + (NB + 2 * kz + 1) * 8, si - __half2float(hi));
    }
  }
}

// Persistent, warp-specialized; grid = min(work items, SMs), block kAgThreads.
// Work items w = ((f*T + t)*stw + ty)*stiles[0] + tx, as k_spread_zdft_tcw.
//   loader warp   home-bin record ranges (up to 32 bins), item data, bulk copies
//                 of the records (2 record slots)
//   producers     per item: the pre-pass of the visible atoms in table chunks of
//                 agCap, and for each kAgK reaching atoms of a table chunk the
//                 chunk's W and B' into chunk slot q % kAgSlots (q counts the
//                 CTA's chunks), once the MMAs of chunk q - kAgSlots are done;
//                 every item has at least one chunk (an atom-less item has one
//                 empty chunk, whose zeroed W gives D = 0)
//   MMA warp      one lane: per chunk, ceil(kc / 16) k steps of two MMAs into the
//                 item's accumulator stage (at least one k step for a first
//                 chunk, so that D starts from zero), then a commit that frees
//                 the slot; after the item's last chunk a commit to the epilogue
//   4 epilogue    accumulator halves summed, the padding mean's transform
//                 subtracted -> Z (lane m = column 16*lx + ly)
// Hand-offs (mbarriers, every wait bounded; the producers decide together at
// named barriers whether to go on):
//   rec_full[b] / rec_empty[b]   loader <-> producers, record slot b
//   a_full[s] / a_empty[s]       producers <-> MMA, chunk slot s
//   acc_full[d] / acc_empty[d]   MMA -> epilogue -> MMA, accumulator stage d
// Dynamic shared memory (128-byte aligned): kAgSlots chunk slots {Wh, Wl, B'},
// two record buffers of agRB float4, the home-bin tables (stiles[0] + 2*stw
// int4), the z twiddles (ez x nkz float2) and an atom table of agCap entries.
// Tensor memory: two accumulator stages of N2 columns.
__global__ void __launch_bounds__(kAgThreads, 1) k_spread_zdft_ag(DevArgs a, int items) {
  pdl_release();
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ AgSlot slot[2];
  __shared__ AgChunk meta[kAgSlots];
  __shared__ __align__(8) uint64_t bars[4 + 2 * kAgSlots + 4];
  __shared__ uint32_t tmem_slot;
  __shared__ volatile int abort_flag;
  __shared__ int tab_count;
  const int NB = a.agNB, N2 = 2 * a.agNB, RB = a.agRB, cap = a.agCap;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  unsigned char *base = smem + ((128u - (smem_addr(smem) & 127u)) & 127u);
  const size_t slot_bytes = 2 * kAgWBytes + static_cast<size_t>(kAgK) * N2 * 2;
  auto wh_of = [&](int s) { return reinterpret_cast<uint16_t *>(base + s * slot_bytes); };
  auto wl_of = [&](int s) { return reinterpret_cast<uint16_t *>(base + s * slot_bytes + kAgWBytes); };
  auto bp_of = [&](int s) { return reinterpret_cast<uint16_t *>(base + s * slot_bytes + 2 * kAgWBytes); };
  float4 *recs = reinterpret_cast<float4 *>(base + kAgSlots * slot_bytes);
  int4 *home_x = reinterpret_cast<int4 *>(recs + 2 * RB);
  int4 *home_y = home_x + a.stiles[0];
  float2 *tws = reinterpret_cast<float2 *>(home_y + 2 * a.stw);
  AgTab tab;
  tab.wx = reinterpret_cast<float4 *>(tws + ((a.ext[2] * a.nkz + 1) & ~1));  // 16-byte aligned
  tab.wy = tab.wx + cap;
  tab.wz = tab.wy + cap;
  tab.zo = reinterpret_cast<int4 *>(tab.wz + cap);
  tab.lxy = reinterpret_cast<int2 *>(tab.zo + cap);
  uint64_t *rec_full = bars, *rec_empty = bars + 2, *a_full = bars + 4, *a_empty = bars + 4 + kAgSlots,
           *acc_full = bars + 4 + 2 * kAgSlots, *acc_empty = acc_full + 2;
  {
    // B' rows past a chunk's atoms and its padding columns are read as they are
    // (the zeroed W columns meet them): start from zero
    int4 *z = reinterpret_cast<int4 *>(base);
    const int n16 = static_cast<int>(kAgSlots * slot_bytes / 16);
    for (int i = tid; i < n16; i += blockDim.x) z[i] = make_int4(0, 0, 0, 0);
    for (int i = tid; i < a.stiles[0]; i += blockDim.x) home_x[i] = a.home_x[i];
    for (int i = tid; i < 2 * a.stw; i += blockDim.x) home_y[i] = a.home_yw[i];
    for (int i = tid; i < a.ext[2] * a.nkz; i += blockDim.x) tws[i] = a.twz[(i / a.nkz) * a.nkzp + i % a.nkz];
  }
  const uint32_t tcols = 2 * N2 <= 32 ? 32 : 2 * N2 <= 64 ? 64 : 2 * N2 <= 128 ? 128 : 2 * N2 <= 256 ? 256 : 512;
  if (warp == kAgMmaWarp) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_addr(&tmem_slot)),
                 "r"(tcols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
  }
  if (tid == 0) {
    for (int i = 0; i < 4 + 2 * kAgSlots + 4; ++i) {
      const int cnt = (i >= 4 + 2 * kAgSlots + 2) ? 4 : 1;  // acc_empty: 4 epilogue warps
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(&bars[i])), "r"(cnt));
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    abort_flag = 0;
    tab_count = 0;
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

  if (warp < kAgProducerWarps) {
    const int ptid = tid;  // producers are threads 0 .. kAgProducers - 1
    int q = 0;             // chunks of this CTA so far
    for (int j = 0, w = blockIdx.x; w < items; ++j, w += gridDim.x) {
      const int b = j & 1;
      wait(&rec_full[b], j >> 1);
      bool skip = producers_sync_or(abort_flag != 0, kAgBar, kAgProducers);
      const AgSlot &sl = slot[b];
      const int nvis = skip ? 0 : sl.ta.cum[sl.ta.nb];
      const int nrec = min(nvis, RB);
      // diagnostic: the most table chunks an item needed
      if (ptid == 0 && nvis > cap) atomicMax(a.status + 1, (nvis + cap - 1) / cap);
      bool emitted = false;
      for (int v0 = 0; !skip && (v0 < nvis || !emitted); v0 += cap) {
        const int nv = max(0, min(cap, nvis - v0));
        if (ptid == 0) tab_count = 0;
        producers_sync(kAgBar, kAgProducers);  // the table is free and its counter zero
        ag_prepass(a, sl.ta, recs + static_cast<size_t>(b) * RB, nrec, sl.f, v0, nv, tab, sl.x0, sl.y0, sl.cw,
                   sl.ch, ptid, kAgProducers, &tab_count);
        producers_sync(kAgBar, kAgProducers);
        const int n = tab_count;
        const bool last_table = v0 + cap >= nvis;
        const int nk = (n + kAgK - 1) / kAgK;
        const int nch = (last_table && nk == 0) ? 1 : nk;
        for (int c = 0; c < nch; ++c, ++q) {
          const int s = q % kAgSlots;
          if (q >= kAgSlots) wait(&a_empty[s], q / kAgSlots - 1);  // the slot's MMAs are done
          skip = producers_sync_or(abort_flag != 0, kAgBar, kAgProducers);
          if (skip) break;
          const int k0 = c * kAgK, kc = max(0, min(kAgK, n - k0));
          {
            // the K columns the chunk's MMAs read (whole 16-atom k steps, at least
            // one): (zk / 8) core-matrix groups of 128 rows x 16 bytes per operand
            const int zk = max(16, (kc + 15) & ~15), n16 = zk * 16;
            int4 *zh = reinterpret_cast<int4 *>(wh_of(s)), *zl = reinterpret_cast<int4 *>(wl_of(s));
            for (int i = ptid; i < 2 * n16; i += kAgProducers)
              (i < n16 ? zh : zl)[i < n16 ? i : i - n16] = make_int4(0, 0, 0, 0);
          }
          producers_sync(kAgBar, kAgProducers);
          ag_operands(a, tab, tws, k0, kc, wh_of(s), wl_of(s), bp_of(s), NB, ptid, kAgProducers);
          asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // generic writes -> tensor core reads
          producers_sync(kAgBar, kAgProducers);
          if (ptid == 0) {
            meta[s].kc = kc;
            meta[s].first = emitted ? 0 : 1;
            meta[s].last = (last_table && c == nch - 1) ? 1 : 0;
            mbar_arrive(smem_addr(&a_full[s]));
          }
          emitted = true;
        }
      }
      producers_sync(kAgBar, kAgProducers);  // every read of record slot b is done
      if (ptid == 0) mbar_arrive(smem_addr(&rec_empty[b]));
    }
  } else if (warp == kAgMmaWarp) {
    if (lane == 0) {
      // kind::f16 (f16 A and B), D f32, both K-major, N >> 3 at bit 17, M = 128
      const uint32_t idesc = (1u << 4) | (static_cast<uint32_t>(N2 >> 3) << 17) |
                             (static_cast<uint32_t>(128 >> 4) << 24);
      int q = 0, j = 0;
      uint32_t last_bar = 0;
      int last_parity = 0;
      for (int w = blockIdx.x; w < items && !abort_flag; w += gridDim.x, ++j) {
        const int d = j & 1;
        const uint32_t dcol = tmem + static_cast<uint32_t>(d * N2);
        for (;;) {
          const int s = q % kAgSlots;
          wait(&a_full[s], q / kAgSlots);
          if (abort_flag) break;
          const int kc = meta[s].kc, first = meta[s].first, last = meta[s].last;
          if (first && j >= 2) wait(&acc_empty[d], (j - 2) >> 1);
          if (abort_flag) break;
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
          int steps = (kc + 15) / 16;
          if (first && steps == 0) steps = 1;
          const uint64_t dwh = umma_desc(smem_addr(wh_of(s)), 2048, 128);
          const uint64_t dwl = umma_desc(smem_addr(wl_of(s)), 2048, 128);
          const uint64_t db = umma_desc(smem_addr(bp_of(s)), N2 * 16, 128);
          for (int k = 0; k < steps; ++k) {
            // 16 atoms: two 8-atom core-matrix groups of W (4096 B) and of B' (2 * N2 * 16 B)
            const uint64_t wstep = static_cast<uint64_t>(k) * 256, bstep = static_cast<uint64_t>(k) * 2 * N2;
            umma_f16_ss(dcol, dwl + wstep, db + bstep, idesc, (first && k == 0) ? 0u : 1u);
            umma_f16_ss(dcol, dwh + wstep, db + bstep, idesc, 1u);
          }
          asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                           smem_addr(&a_empty[s]))
                       : "memory");
          ++q;
          if (last) {
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                             smem_addr(&acc_full[d]))
                         : "memory");
            last_bar = smem_addr(&acc_full[d]);
            last_parity = j >> 1;
            break;
          }
        }
        if (abort_flag) break;
      }
      if (abort_flag && last_bar) mbar_wait(last_bar, static_cast<uint32_t>(last_parity & 1));
    }
  } else if (warp == kAgLoaderWarp) {
    ItemIter it;
    it.init_dims(blockIdx.x, gridDim.x, a.stiles[0], a.stw, a.T);
    int j = 0;
    for (int w = blockIdx.x; w < items; w += gridDim.x, ++j, it.next()) {
      const int b = j & 1;
      int s0, cnt;
      bool valid;
      home_ranges_load_w(a, home_x, home_y, it.f, it.t, it.tx, it.ty, s0, cnt, valid);
      if (j >= 2) wait(&rec_empty[b], (j - 2) >> 1);
      if (__any_sync(0xffffffffu, abort_flag != 0)) break;
      AgSlot &sl = slot[b];
      home_ranges_publish_w(sl.ta, s0, cnt, valid);
      if (lane == 0) {
        sl.f = it.f;
        sl.t = it.t;
        sl.x0 = it.tx * kTwX;
        sl.y0 = it.ty * kTwY;
        sl.cw = min(kTwX, a.ext[0] - sl.x0);
        sl.ch = min(kTwY, a.ext[1] - sl.y0);
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
  } else {
    const int quarter = warp & 3;
    ItemIter it;
    it.init_dims(blockIdx.x, gridDim.x, a.stiles[0], a.stw, a.T);
    const int64_t zplane = static_cast<int64_t>(a.ext[0]) * a.ext[1];
    int j = 0;
    for (int w = blockIdx.x; w < items; w += gridDim.x, ++j, it.next()) {
      const int d = j & 1;
      const float mean = tw_item_mean(a, it.f, it.t);
      wait(&acc_full[d], j >> 1);
      if (__any_sync(0xffffffffu, abort_flag != 0)) break;
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const int x0 = it.tx * kTwX, y0 = it.ty * kTwY;
      float2 *Zft = a.Z + (static_cast<int64_t>(it.f) * a.T + it.t) * a.nkz * zplane;
      const int m = 32 * quarter + lane, lx = m >> 4, ly = m & 15;
      const bool valid = lx < min(kTwX, a.ext[0] - x0) && ly < min(kTwY, a.ext[1] - y0);
      const int64_t cell = static_cast<int64_t>(x0 + lx) * a.ext[1] + (y0 + ly);
      const uint32_t lane_base = tmem + (static_cast<uint32_t>(32 * quarter) << 16) + static_cast<uint32_t>(d * N2);
      for (int c0 = 0; c0 < NB; c0 += 8) {
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
#pragma unroll
          for (int jj = 0; jj < 4; ++jj) {
            const int kz = c0 / 2 + jj;
            if (kz < a.nkz)
              Zft[kz * zplane + cell] =
                  make_float2(__uint_as_float(r[2 * jj]) + __uint_as_float(t[2 * jj]) - mean * a.twz_sum[2 * kz],
                              __uint_as_float(r[2 * jj + 1]) + __uint_as_float(t[2 * jj + 1]) -
                                  mean * a.twz_sum[2 * kz + 1]);
          }
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
  if (warp == kAgMmaWarp)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(tcols));
}

// Part of the translation unit of plan.cu, which includes it inside its
// anonymous namespace after kernel_spread_tcw.cuh; not a standalone header.
// k_spread_zdft_sparse: spreading + z DFT of the element types too sparse for a
// dense tile.

// ---------------------------------------------------------------------------
// Direct spreading + z-axis DFT for sparse element types
// ---------------------------------------------------------------------------
// The wide kernel's cost per work item hardly depends on its atoms: the split of
// the 128 x 128 fixed-point tile, its MMAs and hand-offs take ~6k cycles whether
// 13 or 300 atoms reach the tile.  For an element type whose items see only a few
// atoms this kernel computes the same Z directly: per reaching atom the z
// spectrum of its z taps, T(kz) = sum_r wz[r] * tw[z_r][kz] (the plan's FP32
// twiddles, z_r < ez), then for each of its x/y taps inside the tile
// acc[column][kz] += wx * wy * T(kz) (shared-memory integer atomics in fixed
// point, one lane per kz), and at the end Z = acc - mean * sum_{z < ez} tw[z][kz] (the padding mean
// over the data rows, as the wide kernel subtracts it inside its tile).
// Work items are those of the wide kernel (frame, type, 8 x 16 column tile) for
// the types tw_types[tw_nd + i]: w = ((f*tw_ns + i)*stw + ty)*stiles[0] + tx.
// One CTA per item, 128 threads, eight per SM (26 KB of shared memory and 63
// registers each; six per SM with 35 KB were 0.15 ms per 100 frames slower on the
// 100k-atom workload).  Dynamic shared memory: acc[128 columns][2][nkz] ints (real
// parts, then imaginary parts, of a column).
constexpr int kSpThreads = 128;
// Fixed-point scale of an item's accumulator (integer shared-memory atomics
// issue about three times faster than FP32 ones).  A term wx*wy*T, T = sum_r
// wz[r]*tw, has |term| <= max wx * max wy * sum wz: (2/3)^2 with two or more taps
// per axis, (1/6)^3 with one (only the first cubic weight).  The scale 2^e is at
// most 2^22 / that bound, so a scaled term rounds with one FMA (tap_fixed), and
// small enough that nvis terms per column (each atom adds at most one term to a
// column) stay below 2^31.
__device__ __forceinline__ float sp_scale(int nvis, int ntaps) {
  const float tmax = ntaps >= 2 ? 0.4445f : 0.00464f;
  const float e = floorf(log2f(2.0e9f / (tmax * static_cast<float>(max(nvis, 1)))));
  const float cap = floorf(log2f(4194304.0f / tmax));
  return exp2f(fminf(e, cap));
}

// One reaching atom, staged by its thread for the warps' broadcast reads.
struct SpAtom {
  float4 wx, wy, wz;
  uint32_t z01, z23;  // z tap rows, 16 bits each (0xFFFF for none)
  uint32_t lx, ly;    // in-tile x and y tap positions, one byte each, 0xFF outside
};
constexpr int kSpRound = 64;  // atoms staged per round

__global__ void __launch_bounds__(kSpThreads, 8) k_spread_zdft_sparse(DevArgs a) {
  pdl_release();
  extern __shared__ int acc[];  // fixed point, sp_scale units
  __shared__ TileAtomsW ta;
  __shared__ SpAtom sp_stage[kSpRound];  // a round's reaching atoms
  __shared__ int sp_count[2];
  const int nkz = a.nkz, nkzp = a.nkzp;
  const int w = blockIdx.x;
  const int tx = w % a.stiles[0], ty = (w / a.stiles[0]) % a.stw;
  const int rest = w / (a.stiles[0] * a.stw);
  const int f = rest / a.tw_ns;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int i = tid; i < 128 * 2 * nkz; i += kSpThreads) acc[i] = 0;
  if (tid == 0) sp_count[0] = sp_count[1] = 0;
  // plan constants before the wait for the sort: the type, and per lane of warp 0
  // one home bin (lane 4*iy + ix: home_x[tx] entry ix, home_yw entry iy) or -1
  const int t = a.tw_types[a.tw_nd + rest % a.tw_ns];
  const int x0 = tx * kTwX, y0 = ty * kTwY;
  const int cw = min(kTwX, a.ext[0] - x0), ch = min(kTwY, a.ext[1] - y0);
  int hbin = -1;
  if (warp == 0) {
    const int ix = lane & 3, iy = lane >> 2, jy = iy & 3;
    const int4 hxv = a.home_x[tx], hyv = a.home_yw[2 * ty + (iy >> 2)];
    const int hx = ix == 0 ? hxv.x : ix == 1 ? hxv.y : ix == 2 ? hxv.z : hxv.w;
    const int hy = jy == 0 ? hyv.x : jy == 1 ? hyv.y : jy == 2 ? hyv.z : hyv.w;
    if (hx >= 0 && hy >= 0) hbin = (t * a.tiles[1] + hy) * a.tiles[0] + hx;
  }
  pdl_wait();  // the sort's records, offsets and border sums
  const float mean = tw_item_mean(a, f, t);  // loaded now, used at the end
  if (warp == 0) {
    int s0 = 0, cnt = 0;
    if (hbin >= 0) {
      const int *off = a.offsets + static_cast<int64_t>(f) * (a.nbins + 1);
      s0 = off[hbin];
      cnt = off[hbin + 1] - s0;
    }
    home_ranges_publish_w(ta, s0, cnt, hbin >= 0);
  }
  __syncthreads();
  const int nvis = ta.cum[ta.nb];
  const float scale = sp_scale(nvis, a.ntaps);
  const float inv_scale = 1.0f / scale;  // exact: scale is a power of two
  const float4 *rec = a.rec + static_cast<int64_t>(f) * a.M;
  const int P = a.order, nt = a.ntaps, ez = a.ext[2];
  for (int base = 0, round = 0; base < nvis; base += kSpRound, ++round) {
    // thread i stages atom base + i if it reaches the tile: its weights, in-tile
    // x/y tap positions (bytes, 0xFF outside) and z tap rows (-1 for a missing
    // tap or a row outside the data), compacted to sp_stage[0, count); rounds
    // alternate between two counters, each reset one round after its use
    int *count = &sp_count[round & 1];
    const int v = base + tid;
    float4 q = make_float4(0.f, 0.f, 0.f, 0.f);
    uint32_t lxb = 0xFFFFFFFFu, lyb = 0xFFFFFFFFu;
    if (tid < kSpRound && v < nvis) {
      int j = 0;
      while (v >= ta.cum[j + 1]) ++j;
      q = rec[ta.start[j] + (v - ta.cum[j])];
      const int m0 = static_cast<int>(q.x), m1 = static_cast<int>(q.y);
#pragma unroll
      for (int o = 0; o < 4; ++o) {
        if (o < nt) {
          int x = m0 - P + o;
          if (x < 0) x += a.n[0];
          if (static_cast<unsigned>(x - x0) < static_cast<unsigned>(cw))
            lxb = (lxb & ~(0xFFu << (8 * o))) | (static_cast<uint32_t>(x - x0) << (8 * o));
          int y = m1 - P + o;
          if (y < 0) y += a.n[1];
          if (static_cast<unsigned>(y - y0) < static_cast<unsigned>(ch))
            lyb = (lyb & ~(0xFFu << (8 * o))) | (static_cast<uint32_t>(y - y0) << (8 * o));
        }
      }
    }
    const bool reach = lxb != 0xFFFFFFFFu && lyb != 0xFFFFFFFFu;
    const unsigned bal = __ballot_sync(0xffffffffu, reach);
    int pos = 0;
    if (lane == 0 && bal) pos = atomicAdd(count, __popc(bal));
    pos = __shfl_sync(0xffffffffu, pos, 0) + __popc(bal & ((1u << lane) - 1u));
    if (reach) {
      const int m0 = static_cast<int>(q.x), m1 = static_cast<int>(q.y), m2 = static_cast<int>(q.z);
      float wx[4], wy[4], wz[4];
      cubic_weights(q.x - static_cast<float>(m0), wx);
      cubic_weights(q.y - static_cast<float>(m1), wy);
      cubic_weights(q.z - static_cast<float>(m2), wz);
      uint32_t zr[4];
#pragma unroll
      for (int o = 0; o < 4; ++o) {
        int z = m2 - P + o;
        if (z < 0) z += a.n[2];
        zr[o] = o < nt && z < ez ? static_cast<uint32_t>(z) : 0xFFFFu;
      }
      SpAtom &e = sp_stage[pos];
      e.wx = make_float4(wx[0], wx[1], wx[2], wx[3]);
      e.wy = make_float4(wy[0], wy[1], wy[2], wy[3]);
      e.wz = make_float4(wz[0], wz[1], wz[2], wz[3]);
      e.z01 = zr[0] | (zr[1] << 16);
      e.z23 = zr[2] | (zr[3] << 16);
      e.lx = lxb;
      e.ly = lyb;
    }
    if (tid == 0) sp_count[(round & 1) ^ 1] = 0;  // the next round's counter
    __syncthreads();
    const int nr = *count;
    // the reaching atoms, every 8th to each warp, all lanes of a warp over kz
    for (int k = warp; k < nr; k += kSpThreads / 32) {
      const SpAtom &b = sp_stage[k];
      const float4 bz = b.wz;
      const uint32_t z01 = b.z01, z23 = b.z23;
      const uint32_t lxb = b.lx, lyb = b.ly;
      for (int k0 = 0; k0 < nkz; k0 += 32) {
        const int kz = k0 + lane;
        if (kz >= nkz) continue;
        float tr = 0.f, ti = 0.f;
        const float wzv[4] = {bz.x, bz.y, bz.z, bz.w};
        const uint32_t zrv[4] = {z01 & 0xFFFFu, z01 >> 16, z23 & 0xFFFFu, z23 >> 16};
#pragma unroll
        for (int r = 0; r < 4; ++r)
          if (zrv[r] != 0xFFFFu) {
            const float2 c = a.twz[static_cast<size_t>(zrv[r]) * nkzp + kz];
            tr = fmaf(wzv[r], c.x, tr);
            ti = fmaf(wzv[r], c.y, ti);
          }
        const float4 bx = b.wx, by = b.wy;
        const float wxv[4] = {bx.x, bx.y, bx.z, bx.w}, wyv[4] = {by.x, by.y, by.z, by.w};
#pragma unroll
        for (int o = 0; o < 4; ++o) {
          const uint32_t cx = (lxb >> (8 * o)) & 0xFFu;
          if (cx == 0xFFu) continue;
#pragma unroll
          for (int p = 0; p < 4; ++p) {
            const uint32_t cy = (lyb >> (8 * p)) & 0xFFu;
            if (cy == 0xFFu) continue;
            const float wxy = wxv[o] * wyv[p] * scale;
            int *col = acc + (16 * cx + cy) * 2 * nkz;
            atomicAdd(col + kz, tap_fixed(wxy, tr));
            atomicAdd(col + nkz + kz, tap_fixed(wxy, ti));
          }
        }
      }
    }
    __syncthreads();  // the stage is reused by the next round
  }
  __syncthreads();
  // Z = acc - mean * sum_{z < ez} tw[z][kz], the tile's valid columns, y fastest
  const int64_t zplane = static_cast<int64_t>(a.ext[0]) * a.ext[1];
  float2 *Zft = a.Z + (static_cast<int64_t>(f) * a.T + t) * nkz * zplane;
  for (int i = tid; i < nkz * 128; i += kSpThreads) {
    const int kz = i >> 7, c = i & 127, cx = c >> 4, cy = c & 15;
    if (cx < cw && cy < ch) {
      const int *col = acc + c * 2 * nkz;
      Zft[kz * zplane + static_cast<int64_t>(x0 + cx) * a.ext[1] + (y0 + cy)] =
          make_float2(fmaf(-mean, a.twz_sum[2 * kz], static_cast<float>(col[kz]) * inv_scale), fmaf(-mean, a.twz_sum[2 * kz + 1], static_cast<float>(col[nkz + kz]) * inv_scale));
    }
  }
}

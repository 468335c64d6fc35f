// Part of the translation unit of plan.cu, which includes it inside its
// anonymous namespace; not a standalone header.
// The y and x DFT passes (SIMT and tcgen05), the histogram and the nvt
// accumulation.

// grid (ceil(ex/64), nkz, frames*T), block 256: y-axis DFT.
// Y[f,t,kz][ky][x] = sum_y Z[f,t,kz][x][y] * exp(-2 pi i ja y / nny).
__global__ void __launch_bounds__(kThreads) k_ydft(DevArgs a) {
  pdl_release();
  pdl_wait();
  extern __shared__ __align__(16) unsigned char smem[];
  float2 *zs = reinterpret_cast<float2 *>(smem);        // [kYChunk][kYStride]
  float2 *tys = zs + kYChunk * kYStride;                // [kYChunk][nkyp]
  const int ft = blockIdx.z, kz = blockIdx.y;
  const int xb = blockIdx.x * kYRows;
  const int ex = a.ext[0], ey = a.ext[1];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const float2 *Zp = a.Z + (static_cast<int64_t>(ft) * a.nkz + kz) * ex * ey;
  float2 *Yp = a.Y + (static_cast<int64_t>(ft) * a.nkz + kz) * a.nky * ex;
  const int xr0 = xb + 2 * lane;
  for (int kp = 0; kp * kKyPass < a.nky; ++kp) {
    const int kbase = kp * kKyPass + warp * kKyGroup;
    float2 acc0[kKyGroup], acc1[kKyGroup];
#pragma unroll
    for (int j = 0; j < kKyGroup; ++j) acc0[j] = acc1[j] = make_float2(0.f, 0.f);
    for (int y0 = 0; y0 < ey; y0 += kYChunk) {
      const int yn = min(kYChunk, ey - y0);
      for (int i = tid; i < kYRows * kYChunk; i += blockDim.x) {
        const int row = i / kYChunk, yy = i % kYChunk;
        const int x = xb + row, y = y0 + yy;
        zs[yy * kYStride + row] =
            (x < ex && yy < yn) ? Zp[static_cast<int64_t>(x) * ey + y] : make_float2(0.f, 0.f);
      }
      {
        const float4 *src = reinterpret_cast<const float4 *>(a.twy + static_cast<size_t>(y0) * a.nkyp);
        float4 *dst = reinterpret_cast<float4 *>(tys);
        const int n4 = yn * a.nkyp / 2;
        for (int i = tid; i < n4; i += blockDim.x) dst[i] = src[i];
      }
      __syncthreads();
      if (kbase < a.nky) {
        for (int yy = 0; yy < yn; ++yy) {
          const float4 z2 = *reinterpret_cast<const float4 *>(zs + yy * kYStride + 2 * lane);
          const float4 *w4 = reinterpret_cast<const float4 *>(tys + yy * a.nkyp + kbase);
#pragma unroll
          for (int j = 0; j < kKyGroup / 2; ++j) {
            const float4 w = w4[j];
            // (z.x + i z.y)(w.x + i w.y)
            acc0[2 * j].x = fmaf(z2.x, w.x, fmaf(-z2.y, w.y, acc0[2 * j].x));
            acc0[2 * j].y = fmaf(z2.x, w.y, fmaf(z2.y, w.x, acc0[2 * j].y));
            acc1[2 * j].x = fmaf(z2.z, w.x, fmaf(-z2.w, w.y, acc1[2 * j].x));
            acc1[2 * j].y = fmaf(z2.z, w.y, fmaf(z2.w, w.x, acc1[2 * j].y));
            acc0[2 * j + 1].x = fmaf(z2.x, w.z, fmaf(-z2.y, w.w, acc0[2 * j + 1].x));
            acc0[2 * j + 1].y = fmaf(z2.x, w.w, fmaf(z2.y, w.z, acc0[2 * j + 1].y));
            acc1[2 * j + 1].x = fmaf(z2.z, w.z, fmaf(-z2.w, w.w, acc1[2 * j + 1].x));
            acc1[2 * j + 1].y = fmaf(z2.z, w.w, fmaf(z2.w, w.z, acc1[2 * j + 1].y));
          }
        }
      }
      __syncthreads();
    }
    if (kbase < a.nky) {
#pragma unroll
      for (int j = 0; j < kKyGroup; ++j) {
        const int ky = kbase + j;
        if (ky < a.nky) {
          if (xr0 < ex) Yp[static_cast<int64_t>(ky) * ex + xr0] = acc0[j];
          if (xr0 + 1 < ex) Yp[static_cast<int64_t>(ky) * ex + xr0 + 1] = acc1[j];
        }
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Tensor-core y- and x-axis DFTs (tcgen05, 3xTF32)
// ---------------------------------------------------------------------------
//
// Both passes are real GEMMs  D[r][n'] = sum_k' A[r][k'] B'[k'][n']  over blocks
// of 128 rows, with complex data read as real:
//   A[r][2u + c] = component c (0 re, 1 im) of the row's complex values at u
//                  (each row is contiguous in memory, so A is that memory read
//                  as floats), K' = 2 * (extent of u),
//   B'[2u + c][2k + d] = { Wr, Wi ; -Wi, Wr }[c][d] of the twiddle W[u][k],
//   D[r][2k + d] = component d of the transformed row at k,  N' = 2 * (number
//                  of k) padded to 16.
// y pass: rows are the x rows of one z-transformed plane Z[x][y] (u = y, k =
//   ky), 128 per item; the epilogue writes Y[ky][x].
// x pass: rows are (ky, type) pairs of one (frame, kz), row = (ky - ky0) * T +
//   type, kyb = 128 / T ky per item (rows beyond T*kyb unused), u = x, k = kx;
//   the epilogue applies the form factors, then the four warps of an epilogue
//   slot sum the types of each ky through shared memory, square and multiply by
//   the B-spline moduli (the SIMT kernel's k_xdft_post), writing
//   ibox[kz][ky][kx].
// K is streamed in chunks of kDtcChunk values of u: per chunk the loader warp
// issues one tensor copy (cp.async.bulk.tensor into this CTA only, 128-byte swizzle)
// of the 128 rows x 32 floats into a raw staging tile (rows outside the data
// zero-filled by the tensor map) and one bulk copy of the B' chunk.  The
// producers split the raw rows into a TF32 head and remainder and store them to
// tensor memory, where the MMA reads A: row r of A is TMEM lane r, element k'
// column a0 + k'.  B' stays in shared memory, K-major no-swizzle (core matrices
// of 8 rows x 16 B): element (n', k') at (k'/4)*(N'/8)*32 + (n'/8)*32 + (n'%8)*4
// + k'%4 floats (LBO N'*16 B, SBO 128 B), split on the host.
constexpr int kDtcChunk = 16;                  // u values per K chunk (K' = 32)
constexpr int kDtcProducerWarps = 8;
constexpr int kDtcMmaWarp = kDtcProducerWarps;
constexpr int kDtcLoaderWarp = kDtcProducerWarps + 1;
// epilogue warps: 4 for the y pass (stores only), 12 for the x pass (form factors
// per element), a multiple of 4 so each TMEM lane quarter has the same number
template <bool kX>
__host__ __device__ constexpr int dtc_epi_warps() { return kX ? 12 : 4; }
template <bool kX>
__host__ __device__ constexpr int dtc_threads() { return 32 * (kDtcProducerWarps + 2 + dtc_epi_warps<kX>()); }
constexpr int kDtcMaxStages = 8;

// One pass's GEMM shape: N', K chunks, stages, TMEM columns, B' table.
// With `lo_smem` (when 2N' <= 256): only A's TF32 head goes to tensor memory (32
// columns per stage); the producers write A's remainder back in place into the
// 128-byte-swizzled tensor-copy tile, which the MMA reads as a K-major SWIZZLE_128B
// shared-memory operand, and B' holds head and remainder side by side (2N'
// columns).  A k step is then two MMAs, D += Ah [Bh|Bl] and D += Al [Bh|Bl] (a
// tf32 MMA costs about the same up to N = 192), instead of three; the epilogue
// adds the two halves of D.
//
// With `f16` the pass runs in f16 instead of 3xTF32: the producers scale A by
// a power of two per type (dtc_f16_scale), split it into an f16 head and the
// rounded f16 remainder (both in tensor memory, two K values per column, the
// even one in the low half: 16 columns each per chunk), B' holds the twiddles'
// f16 head and remainder, and the MMAs are kind::f16 with K = 16, so a chunk
// (K' = 32) takes two k steps instead of four.  With `side` the two halves of B'
// sit side by side ([Bh | Bl], N = 2N') and a k step is two MMAs, D += Ah B' and
// D += Al B', whose halves the epilogue adds; otherwise three, D += Al Bh + Ah Bl
// + Ah Bh.  Head and remainder keep 22 bits of each operand, the precision of
// 3xTF32, and an MMA costs about the same either way, so f16 halves the y and x
// passes' MMA issue (which bounds them).
struct DtcShape {
  int N, chunks, S, cols;
  int lo_smem;
  int f16, side;
  const float *B;  // [chunk]: head block then remainder block (N' x 2*kDtcChunk
                   // each), or one block of 2N' x 2*kDtcChunk with lo_smem or
                   // side (f16: the same blocks in halves, packed two per float)
};

// Power-of-two scale of type t's rows in an f16 pass, from bounds that need no
// look at the data: a z-transformed column |Z| <= M_t + ez * mean_t (the type's
// M_t atoms carry weight 1 each; the average padding mean is at most M_t over
// the nx * ny voxels of a border plane), a y-transformed row |Y| <= ey * max|Z|.
// The scaled values stay below 2^14, well inside f16's range.
__device__ __forceinline__ float dtc_f16_scale(const DevArgs &a, int t, bool x_pass) {
  const float m = static_cast<float>(a.type_start[t + 1] - a.type_start[t]);
  const float pad = a.pad_val ? a.pad_val[t] * static_cast<float>(a.ext[2])
                              : m * static_cast<float>(a.ext[2]) / (static_cast<float>(a.n[0]) * a.n[1]);
  float bound = m + pad + 1.0f;
  if (x_pass) bound *= static_cast<float>(a.ext[1]);
  return exp2f(14.0f - ceilf(log2f(bound)));
}

// Tensor copy of chunk c of item w's 128 rows into `dst`, 1024-byte aligned
// (128-byte swizzle: the 16-byte piece j of row r lands at piece j ^ (r % 8) of
// the row) (y pass: 3-D map
// {2*ey floats, ex rows, planes}; x pass: 5-D map {2*ex floats, type, ky, kz,
// frame} whose box {32, T, kyb, 1, 1} lands rows in (ky, type) order).
template <bool kX>
__device__ __forceinline__ void dtc_tensor_copy(const DevArgs &a, const CUtensorMap *map, int w, int c,
                                                uint32_t dst, uint32_t bar) {
  const uint64_t m = reinterpret_cast<uint64_t>(map);
  const int u0 = c * 2 * kDtcChunk;
  if (!kX) {
    const int xblocks = (a.ext[0] + 127) / 128;
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, "
        "%4}], [%5];" ::"r"(dst),
        "l"(m), "r"(u0), "r"((w % xblocks) * 128), "r"(w / xblocks), "r"(bar)
        : "memory");
  } else {
    const int kyb = a.xtcKyb;
    const int nblk = (a.nky + kyb - 1) / kyb;
    const int f = w / (a.nkz * nblk), kz = (w / nblk) % a.nkz;
    asm volatile(
        "cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, "
        "%4, %5, %6}], [%7];" ::"r"(dst),
        "l"(m), "r"(u0), "r"(0), "r"((w % nblk) * kyb), "r"(kz), "r"(f), "r"(bar)
        : "memory");
  }
}

// Persistent, warp-specialized: grid = min(items, resident CTAs), block
// dtc_threads<kX>() (producers, MMA warp, loader warp, epilogue warps).  Items: y pass (plane, block of 128 x rows), planes ordered
// (frame, type, kz) like Z and Y; x pass (frame, kz, block of 128/TP ky).
// Barriers (all waits bounded):
//   bfull[st] loader copies -> producers and MMA (raw A rows and B' landed)
//   afull[st] producers -> MMA (A chunk of stage st split and written)
//   empty[st] MMA commit -> loader (stage st read)
//   dfull[d]  MMA commit -> epilogue (accumulator d complete)
//   dempty[d] epilogue -> MMA (accumulator d read out)
// Dynamic shared memory: S stages of { raw A rows (128 x K'), B' head, B'
// remainder (N' x K') } floats, 1024-byte aligned.  Tensor memory (512
// columns): accumulators d at columns d*N', A stage st at 2N' + 64*st (head) and
// + 32 (remainder).
template <bool kX>
__global__ void __launch_bounds__(dtc_threads<kX>(), 1)
    k_dft_tc(DevArgs a, DtcShape sh, const __grid_constant__ CUtensorMap amap, int items) {
  pdl_release();
  extern __shared__ __align__(16) unsigned char smem[];
  // x pass: per epilogue slot, the 128 rows x 8 kx of f_t * F summed over types
  __shared__ float2 xsum[kX ? 3 * 128 * 8 : 1];
  __shared__ __align__(8) uint64_t bars[3 * kDtcMaxStages + 4];
  __shared__ uint32_t tmem_slot;
  __shared__ volatile int abort_flag;
  const int N = sh.N, NS = sh.S, NC = sh.chunks;
  const bool F16 = sh.f16 != 0;
  const bool halves = F16 ? sh.side != 0 : sh.lo_smem != 0;  // B' = [Bh | Bl]: D in two halves
  const int NM = halves ? 2 * N : N;                 // MMA N, accumulator stage width
  const int AW = (F16 || sh.lo_smem) ? 32 : 64;      // tensor-memory columns of an A stage
  const int KP = 2 * kDtcChunk;                      // K' per chunk
  const int a_floats = 128 * KP;                     // raw A tile
  const int b_floats = F16 ? N * KP / 2 : N * KP;    // B' head or remainder (f16: halves)
  const int stage_floats = a_floats + 2 * b_floats;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  // swizzled tensor copies need a 1024-byte aligned destination: the stages
  // start at the first 1024-byte boundary of the dynamic shared memory
  float *stages = reinterpret_cast<float *>(smem + ((1024u - (smem_addr(smem) & 1023u)) & 1023u));
  uint64_t *afull = bars, *bfull = bars + kDtcMaxStages, *empty = bars + 2 * kDtcMaxStages,
           *dfull = bars + 3 * kDtcMaxStages, *dempty = dfull + 2;
  if (warp == kDtcMmaWarp) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_addr(&tmem_slot)),
                 "r"(sh.cols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
  }
  if (tid == 0) {
    for (int i = 0; i < NS; ++i) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(&afull[i])), "r"(kDtcProducerWarps));
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(&bfull[i])), "r"(1));
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(&empty[i])), "r"(1));
    }
    for (int d = 0; d < 2; ++d) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(&dfull[d])), "r"(1));
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(&dempty[d])), "r"(dtc_epi_warps<kX>()));
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    abort_flag = 0;
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_slot;
  pdl_wait();  // set-up above touched only plan constants, shared and tensor memory

  auto wait = [&](uint64_t *bar, int parity) {
    if (abort_flag) return;
    if (!mbar_wait(smem_addr(bar), static_cast<uint32_t>(parity & 1))) {
      abort_flag = 1;
      atomicOr(a.status, kX ? kStatusX : kStatusY);
    }
  };

  if (warp < kDtcProducerWarps) {
    // warp w owns TMEM lane quarter w % 4 (rows 32*(w%4) + lane) and K' columns
    // 16*(w/4) .. +15 of each chunk: four 16-byte reads of its row (swizzled
    // pieces, conflict-free across the 8 rows of a 1024-byte block), split, two
    // 16-column stores to tensor memory
    static_assert(kDtcProducerWarps == 8 && kDtcChunk == 16, "8 producer warps cover 128 rows x 32 columns");
    const int quarter = warp & 3, half = warp >> 2;
    const int r = 32 * quarter + lane;
    const uint32_t lane_off = static_cast<uint32_t>(32 * quarter) << 16;
    int g = 0;
    for (int w = blockIdx.x; w < items; w += gridDim.x) {
      // f16: this row's scale (y pass: the item's type; x pass: row r's type)
      float rs = 1.0f;
      if (F16) {
        const int xblocks = (a.ext[0] + 127) / 128;
        const int t = kX ? r % a.T : (w / xblocks / a.nkz) % a.T;
        rs = dtc_f16_scale(a, t, kX);
      }
      for (int c = 0; c < NC; ++c, ++g) {
        const int st = g % NS;
        if (g >= NS) wait(&empty[st], g / NS - 1);  // the stage's MMAs have read its TMEM columns
        wait(&bfull[st], g / NS);
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        float *raw = stages + static_cast<size_t>(st) * stage_floats;
        if (F16) {
          // K' 16*half .. +15 of row r: scaled, f16 head and rounded remainder,
          // two K values per column (the even one low), head then remainder
          uint32_t hi[8], lo[8];
#pragma unroll
          for (int jj = 0; jj < 4; ++jj) {
            const int j = 4 * half + jj;
            const float4 v = *reinterpret_cast<const float4 *>(raw + r * KP + 4 * (j ^ (r & 7)));
            const float vv[4] = {v.x * rs, v.y * rs, v.z * rs, v.w * rs};
#pragma unroll
            for (int e = 0; e < 4; e += 2) {
              const __half2 hh = __floats2half2_rn(vv[e], vv[e + 1]);
              const float2 hf = __half22float2(hh);
              const __half2 ll = __floats2half2_rn(vv[e] - hf.x, vv[e + 1] - hf.y);
              hi[2 * jj + e / 2] = *reinterpret_cast<const uint32_t *>(&hh);
              lo[2 * jj + e / 2] = *reinterpret_cast<const uint32_t *>(&ll);
            }
          }
          const uint32_t col = tmem + lane_off + static_cast<uint32_t>(2 * NM + AW * st + 8 * half);
          asm volatile("tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8};" ::"r"(col),
                       "r"(hi[0]), "r"(hi[1]), "r"(hi[2]), "r"(hi[3]), "r"(hi[4]), "r"(hi[5]), "r"(hi[6]),
                       "r"(hi[7])
                       : "memory");
          asm volatile("tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8};" ::"r"(col + 16),
                       "r"(lo[0]), "r"(lo[1]), "r"(lo[2]), "r"(lo[3]), "r"(lo[4]), "r"(lo[5]), "r"(lo[6]),
                       "r"(lo[7])
                       : "memory");
          asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
          asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
          __syncwarp();
          if (lane == 0) mbar_arrive(smem_addr(&afull[st]));
          continue;
        }
        uint32_t hi[16], lo[16];
#pragma unroll
        for (int jj = 0; jj < 4; ++jj) {
          const int j = 4 * half + jj;
          float4 *p = reinterpret_cast<float4 *>(raw + r * KP + 4 * (j ^ (r & 7)));
          const float4 v = *p;
          const float vv[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            const float h = tf32_head(vv[e]);
            hi[4 * jj + e] = __float_as_uint(h);
            lo[4 * jj + e] = __float_as_uint(vv[e] - h);
          }
          if (sh.lo_smem)  // the remainder replaces the raw values in the swizzled tile
            *p = make_float4(__uint_as_float(lo[4 * jj]), __uint_as_float(lo[4 * jj + 1]),
                             __uint_as_float(lo[4 * jj + 2]), __uint_as_float(lo[4 * jj + 3]));
        }
        const uint32_t col = tmem + lane_off + static_cast<uint32_t>(2 * NM + AW * st + 16 * half);
        if (sh.lo_smem) asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        asm volatile(
            "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], "
            "{%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16};" ::"r"(col),
            "r"(hi[0]), "r"(hi[1]), "r"(hi[2]), "r"(hi[3]), "r"(hi[4]), "r"(hi[5]), "r"(hi[6]), "r"(hi[7]),
            "r"(hi[8]), "r"(hi[9]), "r"(hi[10]), "r"(hi[11]), "r"(hi[12]), "r"(hi[13]), "r"(hi[14]), "r"(hi[15]));
        if (!sh.lo_smem)
          asm volatile(
              "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], "
              "{%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16};" ::"r"(col + 32),
              "r"(lo[0]), "r"(lo[1]), "r"(lo[2]), "r"(lo[3]), "r"(lo[4]), "r"(lo[5]), "r"(lo[6]), "r"(lo[7]),
              "r"(lo[8]), "r"(lo[9]), "r"(lo[10]), "r"(lo[11]), "r"(lo[12]), "r"(lo[13]), "r"(lo[14]), "r"(lo[15]));
        asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncwarp();
        if (lane == 0) mbar_arrive(smem_addr(&afull[st]));
      }
    }
  } else if (warp == kDtcLoaderWarp) {
    if (lane == 0) {
      const uint32_t bbytes = static_cast<uint32_t>(2 * b_floats * sizeof(float));
      // the tensor copy lands T*kyb rows in the x pass (128 in the y pass)
      const int arows = kX ? a.T * a.xtcKyb : 128;
      const uint32_t abytes = static_cast<uint32_t>(arows * KP * sizeof(float));
      int g = 0;
      for (int w = blockIdx.x; w < items && !abort_flag; w += gridDim.x) {
        for (int c = 0; c < NC; ++c, ++g) {
          const int st = g % NS;
          if (g >= NS) wait(&empty[st], g / NS - 1);
          if (abort_flag) break;
          const uint32_t bar = smem_addr(&bfull[st]);
          float *sb = stages + static_cast<size_t>(st) * stage_floats;
          asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bbytes + abytes)
                       : "memory");
          asm volatile(
              "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                  smem_addr(sb + a_floats)),
              "l"(sh.B + static_cast<size_t>(c) * 2 * b_floats), "r"(bbytes), "r"(bar)
              : "memory");
          dtc_tensor_copy<kX>(a, &amap, w, c, smem_addr(sb), bar);
        }
      }
    }
  } else if (warp == kDtcMmaWarp) {
    if (lane == 0) {
      // kind::tf32: D f32, A and B tf32, both K-major, N >> 3 at bit 17, M = 128
      const uint32_t idesc = (1u << 4) | (2u << 7) | (2u << 10) |
                             (static_cast<uint32_t>(NM >> 3) << 17) | (static_cast<uint32_t>(128 >> 4) << 24);
      int g = 0, i = 0;
      uint32_t last_bar = 0;
      int last_parity = 0;
      for (int w = blockIdx.x; w < items && !abort_flag; w += gridDim.x, ++i) {
        const int d = i & 1;
        if (i >= 2) wait(&dempty[d], (i - 2) >> 1);
        const uint32_t dcol = tmem + static_cast<uint32_t>(d * NM);
        for (int c = 0; c < NC; ++c, ++g) {
          const int st = g % NS;
          wait(&bfull[st], g / NS);
          wait(&afull[st], g / NS);
          if (abort_flag) break;
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
          const float *sb = stages + static_cast<size_t>(st) * stage_floats;
          const uint32_t ah0 = tmem + static_cast<uint32_t>(2 * NM + AW * st);
          if (F16) {
            // kind::f16 (f16 A and B), D f32, N = NM, M = 128; B' K-major, 16-byte
            // K blocks of N2 rows; a k step of 16 K advances two blocks
            const uint32_t idesc16 = (1u << 4) | (static_cast<uint32_t>(NM >> 3) << 17) |
                                     (static_cast<uint32_t>(128 >> 4) << 24);
            const int N2 = sh.side ? 2 * N : N;
            const uint64_t dbh0 = umma_desc(smem_addr(sb + a_floats), N2 * 16, 128);
            const uint64_t dbl0 = umma_desc(smem_addr(sb + a_floats + b_floats), N * 16, 128);
            for (int kk = 0; kk < KP / 16; ++kk) {
              const uint32_t ah = ah0 + 8 * kk, al = ah + 16;
              const uint64_t dbh = dbh0 + static_cast<uint64_t>(kk * 2 * N2);
              umma_f16_ts(dcol, al, dbh, idesc16, (c > 0 || kk > 0) ? 1u : 0u);
              if (!sh.side) umma_f16_ts(dcol, ah, dbl0 + static_cast<uint64_t>(kk * 2 * N), idesc16, 1u);
              umma_f16_ts(dcol, ah, dbh, idesc16, 1u);
            }
          } else if (sh.lo_smem) {
            // B' = [Bh | Bl] (2N' columns); Al is the swizzled tile itself: a K-major
            // SWIZZLE_128B descriptor (layout type 2, 8-row groups 1024 B apart) whose
            // start advances 32 B per k step of 8 floats within the 128-byte rows
            const uint64_t db0 = umma_desc(smem_addr(sb + a_floats), NM * 16, 128);
            const uint64_t dal0 = umma_desc(smem_addr(sb), 16, 1024) | (static_cast<uint64_t>(2) << 61);
            for (int kk = 0; kk < KP / 8; ++kk) {
              const uint64_t db = db0 + static_cast<uint64_t>(kk * 2 * NM);
              umma_tf32_ts(dcol, ah0 + 8 * kk, db, idesc, (c > 0 || kk > 0) ? 1u : 0u);
              umma_tf32(dcol, dal0 + static_cast<uint64_t>(2 * kk), db, idesc, 1u);
            }
          } else {
            const uint64_t dbh0 = umma_desc(smem_addr(sb + a_floats), N * 16, 128);
            const uint64_t dbl0 = umma_desc(smem_addr(sb + a_floats + b_floats), N * 16, 128);
            // one k step (8 of K'): A advances 8 TMEM columns, B' N*32 B (+N*2)
            for (int kk = 0; kk < KP / 8; ++kk) {
              const uint32_t ah = ah0 + 8 * kk, al = ah + 32;
              const uint64_t dbh = dbh0 + static_cast<uint64_t>(kk * 2 * N);
              const uint64_t dbl = dbl0 + static_cast<uint64_t>(kk * 2 * N);
              umma_tf32_ts(dcol, al, dbh, idesc, (c > 0 || kk > 0) ? 1u : 0u);
              umma_tf32_ts(dcol, ah, dbl, idesc, 1u);
              umma_tf32_ts(dcol, ah, dbh, idesc, 1u);
            }
          }
          asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                           smem_addr(&empty[st]))
                       : "memory");
          last_bar = smem_addr(&empty[st]);
          last_parity = g / NS;
        }
        if (abort_flag) break;
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                         smem_addr(&dfull[d]))
                     : "memory");
      }
      if (abort_flag && last_bar) mbar_wait(last_bar, static_cast<uint32_t>(last_parity & 1));
    }
  } else {
    // epilogue: warp w reads TMEM lanes 32*(w%4).. = rows of the block; the
    // epilogue warps of one lane quarter take every EQ-th 16-column group
    constexpr int EQ = dtc_epi_warps<kX>() / 4;
    const int quarter = warp & 3;
    const int eslot = (warp - (kDtcLoaderWarp + 1)) / 4;
    const int r = 32 * quarter + lane;
    int i = 0;
    for (int w = blockIdx.x; w < items; w += gridDim.x, ++i) {
      const int d = i & 1;
      // x pass: the item's geometry, form factors and padding mean, loaded before
      // the wait so that their latency overlaps it
      float ocs[9], ff[9], mean = 0.0f;
      if (kX) {
        const int T = a.T, kyb = a.xtcKyb;
        const int nblk = (a.nky + kyb - 1) / kyb;
        const int f = w / (a.nkz * nblk);
        const int kyl = r / T, t = r % T, ky = (w % nblk) * kyb + kyl;
#pragma unroll
        for (int q = 0; q < 9; ++q) ocs[q] = a.geom[f * kGeom + 9 + q];
#pragma unroll
        for (int q = 0; q < 9; ++q) ff[q] = a.ff[9 * t + q];
        if (r < T * kyb && ky < a.nky) mean = padding_mean(a, f, t);
      }
      wait(&dfull[d], i >> 1);
      // x pass: the four warps of a slot meet at named barriers, so they decide together
      if (kX ? producers_sync_or(abort_flag != 0, 1 + eslot, 128) : __any_sync(0xffffffffu, abort_flag != 0))
        break;
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t lane_base = tmem + (static_cast<uint32_t>(32 * quarter) << 16) + static_cast<uint32_t>(d * NM);
      // 16 accumulator columns from c0 (with lo_smem: the sum of the two halves)
      // f16: the row's scale is undone here (y pass: the item's type; x pass: row r's)
      float unscale = 1.0f;
      if (F16) {
        const int xblocks = (a.ext[0] + 127) / 128;
        const int t = kX ? r % a.T : (w / xblocks / a.nkz) % a.T;
        unscale = 1.0f / dtc_f16_scale(a, t, kX);
      }
      auto load16 = [&](int c0, uint32_t v[16]) {
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
            "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
            : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
              "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
            : "r"(lane_base + c0));
        if (halves) {
          uint32_t u[16];
          asm volatile(
              "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
              "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
              : "=r"(u[0]), "=r"(u[1]), "=r"(u[2]), "=r"(u[3]), "=r"(u[4]), "=r"(u[5]), "=r"(u[6]), "=r"(u[7]),
                "=r"(u[8]), "=r"(u[9]), "=r"(u[10]), "=r"(u[11]), "=r"(u[12]), "=r"(u[13]), "=r"(u[14]), "=r"(u[15])
              : "r"(lane_base + N + c0));
          asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
          for (int q = 0; q < 16; ++q) v[q] = __float_as_uint(__uint_as_float(v[q]) + __uint_as_float(u[q]));
        } else {
          asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        }
        if (F16) {
#pragma unroll
          for (int q = 0; q < 16; ++q) v[q] = __float_as_uint(__uint_as_float(v[q]) * unscale);
        }
      };
      if (!kX) {
        const int ex = a.ext[0];
        const int xblocks = (ex + 127) / 128;
        const int64_t plane = w / xblocks;
        const int x = (w % xblocks) * 128 + r;
        float2 *Yp = a.Y + plane * a.nky * ex;
        for (int c0 = 16 * eslot; c0 < N; c0 += 16 * EQ) {
          uint32_t v[16];
          load16(c0, v);
          if (x < ex) {
#pragma unroll
            for (int jj = 0; jj < 8; ++jj) {
              const int ky = c0 / 2 + jj;
              if (ky < a.nky)
                Yp[static_cast<int64_t>(ky) * ex + x] =
                    make_float2(__uint_as_float(v[2 * jj]), __uint_as_float(v[2 * jj + 1]));
            }
          }
        }
      } else {
        // rows r = kyl * T + t (kyl < kyb); each lane finishes f_t * F for its row,
        // the four warps of this epilogue slot (one per lane quarter) meet in
        // shared memory to sum the types of each ky, square and scale
        const int T = a.T, kyb = a.xtcKyb;
        const int nblk = (a.nky + kyb - 1) / kyb;
        const int f = w / (a.nkz * nblk), kz = (w / nblk) % a.nkz;
        const int ky0 = (w % nblk) * kyb;
        const int kyl = r / T, ky = ky0 + kyl;
        const bool row_ok = r < T * kyb && ky < a.nky;
        const int ka = signed_k(kz, a.nn[2], a.nf[2]);
        const int ja = a.ky_lo + min(ky, a.nky - 1);
        // the per-row form factors use the float |q|; their cut-off test is made
        // inclusive by 1e-6 relative (kpoint_q_f32 is within a few ulp of the
        // reference's expression), and the reference's expression itself decides
        // below which outputs are kept
        const float qcut_incl = a.qcut * (1.0f + 1e-6f);
        const float inv4pi = static_cast<float>(1.0 / (4.0 * M_PI));
        float2 *red = xsum + eslot * 128 * 8;  // [row][8 kx]
        const int rid = 32 * quarter + lane;    // 0..127 over the slot's four warps
        const uint32_t bar_id = 1 + eslot;
        for (int c0 = 16 * eslot; c0 < N; c0 += 16 * EQ) {
          uint32_t v[16];
          load16(c0, v);
#pragma unroll
          for (int jj = 0; jj < 8; ++jj) {
            const int kx = c0 / 2 + jj;
            const int ia = a.kx_lo + min(kx, a.nkx - 1);
            const float mw = kpoint_q_f32(ocs, ia, ja, ka);
            const bool inside = row_ok && kx < a.nkx && !(mw > qcut_incl);
            float2 F = make_float2(__uint_as_float(v[2 * jj]), __uint_as_float(v[2 * jj + 1]));
            // the padding mean's constant over the whole supercell lands at k = 0
            if (ka == 0 && ja == 0 && ia == 0)
              F.x += static_cast<float>(static_cast<double>(mean) * a.nn3);
            float2 A = make_float2(0.f, 0.f);
            if (inside) {
              const float q = mw * inv4pi;
              const float ft = form_factor(ff, q * q);
              A.x = ft * F.x;
              A.y = ft * F.y;
            }
            red[r * 8 + jj] = A;
          }
          asm volatile("bar.sync %0, 128;" ::"r"(bar_id) : "memory");
          for (int p = rid; p < kyb * 8; p += 128) {
            const int kl = p >> 3, jj = p & 7;
            const int kyy = ky0 + kl, kx = c0 / 2 + jj;
            if (kyy < a.nky && kx < a.nkx) {
              float2 A = make_float2(0.f, 0.f);
              for (int tt = 0; tt < T; ++tt) {
                const float2 e = red[(kl * T + tt) * 8 + jj];
                A.x += e.x;
                A.y += e.y;
              }
              const int ia = a.kx_lo + kx, jb = a.ky_lo + kyy;
              const float mw = kpoint_q(ocs, ia, jb, ka);
              const int iw = ia < 0 ? ia + a.nn[0] : ia, jw = jb < 0 ? jb + a.nn[1] : jb;
              a.ibox[((static_cast<int64_t>(f) * a.nkz + kz) * a.nky + kyy) * a.nkx + kx] =
                  !(mw > a.qcut) ? (A.x * A.x + A.y * A.y) * (a.modx[iw] * (a.mody[jw] * a.modz[kz])) : 0.0f;
            }
          }
          asm volatile("bar.sync %0, 128;" ::"r"(bar_id) : "memory");  // before the next group's writes
        }
      }
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      __syncwarp();
      if (lane == 0) mbar_arrive(smem_addr(&dempty[d]));
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (warp == kDtcMmaWarp)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(sh.cols));
}

// grid (ceil(nky/4), nkz, frames), block 256: x-axis DFT, form factors, type
// sum, modulus.  Dynamic shared memory, for an x chunk of `xc` values:
// twx xc*nkxp | Y rows T*xc | F T*nkxp (all float2).
__global__ void __launch_bounds__(kThreads) k_xdft_post(DevArgs a, int xc) {
  pdl_release();
  pdl_wait();
  extern __shared__ __align__(16) unsigned char smem[];
  const int ex = a.ext[0];
  float2 *txs = reinterpret_cast<float2 *>(smem);
  float2 *ys = txs + static_cast<size_t>(xc) * a.nkxp;
  float2 *fs = ys + static_cast<size_t>(a.T) * xc;
  __shared__ float ocs[9];
  __shared__ float means[64];
  const int f = blockIdx.z, kz = blockIdx.y;
  const int tid = threadIdx.x;
  if (tid < 9) ocs[tid] = a.geom[f * kGeom + 9 + tid];
  for (int t = tid; t < a.T && t < 64; t += blockDim.x)
    means[t] = padding_mean(a, f, t);
  const bool one_chunk = xc >= ex;
  if (one_chunk) {
    const float4 *src = reinterpret_cast<const float4 *>(a.twx);
    float4 *dst = reinterpret_cast<float4 *>(txs);
    const int n4 = ex * a.nkxp / 2;
    for (int i = tid; i < n4; i += blockDim.x) dst[i] = src[i];
  }
  const int ka = signed_k(kz, a.nn[2], a.nf[2]);
  const int npairs = a.T * a.nkx;
  for (int r = 0; r < kXRows; ++r) {
    const int ky = blockIdx.x * kXRows + r;
    if (ky >= a.nky) break;
    const int ja = a.ky_lo + ky;
    for (int p0 = 0; p0 < npairs; p0 += blockDim.x) {
      const int i = p0 + tid;
      const int t = i / a.nkx, kx = i % a.nkx;
      float2 acc = make_float2(0.f, 0.f);
      for (int x0 = 0; x0 < ex; x0 += xc) {
        const int xn = min(xc, ex - x0);
        __syncthreads();
        for (int j = tid; j < a.T * xn; j += blockDim.x) {
          const int tt = j / xn, x = j % xn;
          ys[tt * xc + x] = a.Y[((static_cast<int64_t>(f) * a.T + tt) * a.nkz + kz) * a.nky * ex +
                                static_cast<int64_t>(ky) * ex + x0 + x];
        }
        if (!one_chunk) {
          const float4 *src = reinterpret_cast<const float4 *>(a.twx + static_cast<size_t>(x0) * a.nkxp);
          float4 *dst = reinterpret_cast<float4 *>(txs);
          const int n4 = xn * a.nkxp / 2;
          for (int j = tid; j < n4; j += blockDim.x) dst[j] = src[j];
        }
        __syncthreads();
        if (i < npairs) {
          const float2 *yr = ys + t * xc;
          for (int x = 0; x < xn; ++x) {
            const float2 v = yr[x];
            const float2 w = txs[x * a.nkxp + kx];
            acc.x = fmaf(v.x, w.x, fmaf(-v.y, w.y, acc.x));
            acc.y = fmaf(v.x, w.y, fmaf(v.y, w.x, acc.y));
          }
        }
      }
      if (i < npairs) {
        if (ka == 0 && ja == 0 && a.kx_lo + kx == 0)
          acc.x += static_cast<float>(static_cast<double>(means[t < 64 ? t : 63]) * a.nn3);
        fs[t * a.nkxp + kx] = acc;
      }
    }
    __syncthreads();
    for (int kx = tid; kx < a.nkx; kx += blockDim.x) {
      const int ia = a.kx_lo + kx;
      const float mw = kpoint_q(ocs, ia, ja, ka);
      float I = 0.0f;
      if (!(mw > a.qcut)) {
        const float q = mw / (4.0 * M_PI);
        const float q2 = q * q;
        float2 A = make_float2(0.f, 0.f);
        for (int t = 0; t < a.T; ++t) {
          const float ft = form_factor(a.ff + 9 * t, q2);
          const float2 F = fs[t * a.nkxp + kx];
          A.x = fmaf(ft, F.x, A.x);
          A.y = fmaf(ft, F.y, A.y);
        }
        const int i = ia < 0 ? ia + a.nn[0] : ia;
        const int j = ja < 0 ? ja + a.nn[1] : ja;
        const float bsp = a.modx[i] * a.mody[j] * a.modz[kz];
        I = (A.x * A.x + A.y * A.y) * bsp;
      }
      a.ibox[((static_cast<int64_t>(f) * a.nkz + kz) * a.nky + ky) * a.nkx + kx] = I;
    }
  }
}

// grid (nkz, planes), block 256: mirror-weighted histogram of one kz plane.
// `vals` holds nkz*nky*nkx values per plane; `geom` the frame geometry.
template <typename V>
__global__ void __launch_bounds__(kThreads)
    k_hist(DevArgs a, const V *vals, const float *geom, int geom_stride, double fact,
           double *hist, double *nhist) {
  pdl_release();
  pdl_wait();
  extern __shared__ __align__(16) unsigned char smem[];
  const int npts = a.nky * a.nkx;
  const bool in_smem = a.num_bins <= kHistSmemBins;
  double *sh = reinterpret_cast<double *>(smem);
  double *sn = sh + (in_smem ? a.num_bins : 0);
  __shared__ float ocs[9];
  const int kz = blockIdx.x, f = blockIdx.y;
  const int tid = threadIdx.x;
  if (tid < 9) ocs[tid] = geom[f * geom_stride + 9 + tid];
  if (in_smem)
    for (int b = tid; b < 2 * a.num_bins; b += blockDim.x) sh[b] = 0.0;
  const V *pl = vals + (static_cast<int64_t>(f) * a.nkz + kz) * npts;
  __syncthreads();
  const int ka = signed_k(kz, a.nn[2], a.nf[2]);
  const int kx_hi = a.kx_lo + a.nkx - 1, ky_hi = a.ky_lo + a.nky - 1;
  double *dh = in_smem ? sh : hist;
  double *dn = in_smem ? sn : nhist;
  // Neighbouring k-points (consecutive lanes) mostly fall in the same bin: each
  // warp sums runs of equal bins in lane order (a segmented shuffle scan) and
  // the last lane of a run adds the run's sums, so the FP64 atomics contend
  // far less.
  const int lane = tid & 31;
  for (int p0 = tid - lane; p0 < npts; p0 += blockDim.x) {
    const int p = p0 + lane;
    int h0 = -1;
    double v = 0.0, c = 0.0;
    if (p < npts && a.dq > 0.0f) {
      const int ky = p / a.nkx, kx = p % a.nkx;
      const int ia = a.kx_lo + kx, ja = a.ky_lo + ky;
      const float mw = kpoint_q(ocs, ia, ja, ka);
      const int hb = static_cast<int>(mw / a.dq);
      if (!(mw > a.qcut) && hb >= 0 && hb < a.num_bins) {
        h0 = hb;
        if (ia == 0 && ja == 0 && ka == 0) {
          v = static_cast<double>(pl[p]) * fact;
          c = 1.0;
        } else {
          int ib = -ia, jb = -ja;
          if (ib > kx_hi) ib = ia;
          if (jb > ky_hi) jb = ja;
          const int pm = (jb - a.ky_lo) * a.nkx + (ib - a.kx_lo);
          if (sizeof(V) == 4)
            v = static_cast<double>(static_cast<float>(pl[p]) + static_cast<float>(pl[pm])) * fact;
          else
            v = (static_cast<double>(pl[p]) + static_cast<double>(pl[pm])) * fact;
          c = 2.0;
        }
      }
    }
    // first lane of this lane's run of equal bins
    const int hprev = __shfl_up_sync(0xffffffffu, h0, 1);
    int start = (lane == 0 || hprev != h0) ? lane : 0;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) start = max(start, __shfl_up_sync(0xffffffffu, start, d));
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const double vo = __shfl_up_sync(0xffffffffu, v, d);
      const double co = __shfl_up_sync(0xffffffffu, c, d);
      if (lane - d >= start) {
        v += vo;
        c += co;
      }
    }
    const int hnext = __shfl_down_sync(0xffffffffu, h0, 1);
    if (h0 >= 0 && (lane == 31 || hnext != h0)) {
      atomicAdd(dh + h0, v);
      atomicAdd(dn + h0, c);
    }
  }
  if (in_smem) {
    __syncthreads();
    for (int b = tid; b < a.num_bins; b += blockDim.x) {
      if (sn[b] != 0.0) {
        atomicAdd(hist + b, sh[b]);
        atomicAdd(nhist + b, sn[b]);
      }
    }
  }
}

// grid (ceil(points/256)), block 256: nvt intensity sum over the batch's frames.
__global__ void k_accumulate(DevArgs a, int nframes) {
  const int64_t npl = static_cast<int64_t>(a.nkz) * a.nky * a.nkx;
  const int64_t p = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (p >= npl) return;
  double s = a.iacc[p];
  for (int f = 0; f < nframes; ++f) s += static_cast<double>(a.ibox[f * npl + p]);
  a.iacc[p] = s;
}

// grid 1, block 256: the last launch of the allocation-free single-frame
// forward.  When a kernel of the frame reported an error through the status
// word, the frame's histogram is overwritten with NaN: the caller of that
// asynchronous call receives no status code for it, so the error travels in
// the output itself.
__global__ void k_flag_invalid(const int *status, double *hist, double *nhist, int nb) {
  if (status[0] == 0) return;
  const double nan = __longlong_as_double(0x7ff8000000000000ll);
  for (int b = threadIdx.x; b < nb; b += blockDim.x) {
    hist[b] = nan;
    nhist[b] = nan;
  }
}

// grid 1, block 32: the bounded mbarrier wait of the pipelined kernels
// (mbar_wait_for) on a barrier that no thread arrives at, so that it gives up
// after `limit_ns` and sets kStatusProbe in the status word, as those kernels
// set their bits.  Nothing else is in flight in this kernel, so giving up
// leaves no copy or tensor-core operation behind.
__global__ void k_wait_probe(int *status, unsigned long long limit_ns) {
  __shared__ __align__(8) uint64_t bar;
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(&bar)), "r"(1));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  if (threadIdx.x == 0 && !mbar_wait_for(smem_addr(&bar), 0u, limit_ns)) atomicOr(status, kStatusProbe);
  __syncthreads();
  if (threadIdx.x == 0) asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_addr(&bar)) : "memory");
}

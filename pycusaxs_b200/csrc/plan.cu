// pycusaxs_b200: B200-native per-frame SAXS path: the plan, its buffers and the
// launch sequence.  The kernels live in the kernel_*.cuh files, included below
// into this translation unit.
//
// Pipeline of one batch of frames (all kernels hand-written for sm_100a):
//
//   k_sort_atoms    one thread-block cluster per (type, frame): atoms ->
//                   float32 grid coordinates (the reference's float steps,
//                   saxsDeviceKernels.cu:355-368), counting sort into
//                   (type, home tile) order with shared-memory counters shared
//                   across the cluster, per-type FP64 z-border sums for the
//                   padding mean (saxsDeviceKernels.cu:446-465 evaluated per
//                   atom instead of per voxel).
//   k_spread_zdft   one CTA per (frame, type, 8x8 column tile): B-spline
//                   spreading into a shared-memory column tile (no global
//                   atomics), mean padding folded in as "subtract the mean",
//                   then the z-axis DFT of every column restricted to the
//                   kz values the q-cut can reach.
//   k_ydft          y-axis DFT restricted to the ky range (complex GEMM-shaped
//                   tiles in shared memory, FP32 FMA).
//   k_xdft_post     x-axis DFT restricted to the kx range, then per k-point:
//                   form factor f_t(|q|), complex sum over types, |F|^2 times
//                   the B-spline moduli (saxsDeviceKernels.cu:142-216).
//   k_hist          mirror-weighted radial histogram with the reference's
//                   float32 bin rule (saxsDeviceKernels.cu:67-125), FP64
//                   shared-memory bins, one global flush per CTA.
//
// Why no full FFT: the reference zero-pads (mean-pads) the nx^3 grid into an
// nn^3 supercell and runs a full R2C FFT, but only k-points with |q| <= qcut
// ever reach the histogram, and qcut is clamped so that these form a small
// ellipsoid around the origin (|m| <= ~20 of 256 at 100k atoms / 256^3).  The
// padded transform is F = DFT(g - mean over the corner block) + mean*nn^3 at
// k = 0, evaluated exactly by three pruned DFT passes that never touch the
// zero region.
#include <cuda.h>  // CUtensorMap and its enums (the encoder is fetched at run time)
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "pycusaxs_b200.h"
#include "scratch_forward.h"
#include "setup.h"

namespace {

#include "kernels_common.cuh"
#include "kernel_sort.cuh"
#include "kernel_spread_simt.cuh"
#include "kernel_spread_tc.cuh"
#include "kernel_spread_tcw.cuh"
#include "kernel_spread_sparse.cuh"
#include "kernel_spread_ag.cuh"
#include "kernel_dft.cuh"
#include "kernel_adjoint.cuh"

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
struct Ring {
  float *host = nullptr;
  cudaEvent_t ev[kRing] = {};
  int next = 0;
};

// Timed stages of saxs_forward, in launch order.
enum Stage { kStSort, kStSpread, kStYdft, kStXdft, kStHist, kStages };
const char *kStageNames[kStages] = {"k_sort_atoms", "k_spread_zdft", "k_ydft", "k_xdft_post", "k_hist"};

struct StageRecord {
  cudaEvent_t start[kStages] = {};
  cudaEvent_t stop[kStages] = {};
  bool used[kStages] = {};
};

}  // namespace

struct SaxsPlan {
  int device = 0;
  SaxsParams p{};
  std::vector<float> ff;
  std::vector<float> pad;  // given padding densities per type (empty: z-border mean)
  std::vector<int32_t> ea_host, et_host;  // the caller's atom lists, kept to re-plan a wider k-box
  int graph_refs = 0;      // graphs (saxs_graph_create) holding this plan's buffers
  DevArgs a{};
  int ensemble = SAXS_NPT;
  long long half[3] = {0, 0, 0};
  bool full_axis[3] = {false, false, false};
  float sigma_scale = 1.0f;  // nx / nnx
  int frames = 0;            // frames accumulated
  int last_frame_batch = 0;  // frames in the last forward batch
  size_t bytes = 0;
  size_t smem_spread = 0, smem_ydft = 0, smem_xdft = 0, smem_hist = 0;
  std::vector<void *> allocations;
  Ring ring;
  float *d_geom0 = nullptr;
  double *d_tmp_hist = nullptr;
  // adjoint buffers, allocated by the first saxs_backward
  double *d_adj_dl = nullptr, *d_adj_S = nullptr;
  float2 *d_adj_G = nullptr, *d_adj_twyT = nullptr, *d_adj_twzT = nullptr;
  float *d_adj_dg = nullptr, *d_adj_dcg = nullptr;
  int adj_eyp = 0, adj_ezp = 0, zadj_ctas = 1;
  bool adj_tiled_y = false, adj_tiled_z = false;
  size_t smem_yadj = 0, smem_zadj = 0;
  int spread_ctas = 1;  // resident CTAs of the persistent spreading kernel
  int sort_slots = 1;    // resident k_sort_atoms CTAs on the device
  int sort_cluster = 1;  // largest k_sort_atoms cluster size the device can schedule (<= kSortMaxCluster)
  int sort_max_type = 0; // entries of the largest type
  bool use_tc = false;   // z-axis DFT on the tensor cores
  bool use_tcw = false;  // ... with the wide-tile kernel (k_spread_zdft_tcw), else k_spread_zdft_tc
  size_t smem_spread_tc = 0, smem_spread_tcw = 0;
  size_t smem_sparse = 0;  // k_spread_zdft_sparse's accumulator (0: no sparse types)
  int tc_ctas = 1, tcw_ctas = 1;
  bool tcn_ok = false, tcw_ok = false;  // z kernels the plan can run: 64- and 128-column tiles
  int twG_max = 1;                      // producer groups the wide kernel's shared memory allows
  int tw_cap[2] = {0, 0}, tw_rb[2] = {0, 0};  // wide kernel atom table / record buffer, 1 or 2 groups
  size_t tw_smem[2] = {0, 0};
  bool tc_ok = false, ytc_ok = false, xtc_ok = false;  // tensor-core kernels the plan can run
  bool ag_ok = false, use_ag = false;  // atom-GEMM spreading (k_spread_zdft_ag): runnable, in use
  size_t smem_spread_ag = 0;
  int ag_ctas = 1;
  bool use_ytc = false;  // y-axis DFT on the tensor cores (k_dft_tc<false>)
  bool use_xtc = false;  // x-axis DFT + post on the tensor cores (k_dft_tc<true>)
  DtcShape yshape{}, xshape{};
  size_t smem_ydft_tc = 0, smem_xdft_tc = 0;
  int ytc_ctas = 1, xtc_ctas = 1;
  int xc = 1;           // x values per shared-memory chunk in k_xdft_post
  bool profiling = false;
  std::vector<StageRecord> prof_pending;
  std::vector<cudaEvent_t> event_pool;
};

namespace {

// The wide kernel's producer groups with the table sizes planned for them.
void set_wide_groups(SaxsPlan *pl, int g) {
  pl->a.twG = g;
  pl->a.twCap = pl->tw_cap[g - 1];
  pl->a.twRB = pl->tw_rb[g - 1];
  pl->smem_spread_tcw = pl->tw_smem[g - 1];
}

int optin_smem() {
  int dev = 0, v = 0;
  cudaGetDevice(&dev);
  if (cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess) {
    cudaGetLastError();
    return 48 * 1024;
  }
  return v;
}

template <typename K>
size_t static_smem(K kernel) {
  cudaFuncAttributes fa{};
  if (cudaFuncGetAttributes(&fa, kernel) != cudaSuccess) {
    cudaGetLastError();
    return 1024;
  }
  return fa.sharedSizeBytes;
}

template <typename K>
cudaError_t raise_smem_limit(K kernel) {
  const int lim = optin_smem() - static_cast<int>(static_smem(kernel));
  return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
}

template <typename T>
int dalloc(SaxsPlan *pl, T **ptr, size_t count) {
  const size_t bytes = std::max<size_t>(count, 1) * sizeof(T);
  cudaError_t e = cudaMalloc(reinterpret_cast<void **>(ptr), bytes);
  if (e != cudaSuccess) {
    cudaGetLastError();
    size_t fr = 0, tot = 0;
    cudaMemGetInfo(&fr, &tot);
    return fail(SAXS_E_NOMEM, "device allocation of " + std::to_string(bytes) +
                                  " bytes failed (" + cudaGetErrorString(e) + "; free " +
                                  std::to_string(fr) + " of " + std::to_string(tot) + ")");
  }
  pl->allocations.push_back(*ptr);
  pl->bytes += bytes;
  return SAXS_OK;
}

// Distinct home bins (width bin_w) whose atoms can reach the columns
// [c0, c0+cw) of each spread tile along an axis of length n, for stencils of
// `order` taps that start at an atom's home column.  Returns false when a tile
// would need more than four bins.
bool home_tile_table(int ext, int n, int order, int bin_w, std::vector<int4> *out) {
  out->clear();
  for (int c0 = 0; c0 < ext; c0 += kTile) {
    const int cw = std::min(kTile, ext - c0);
    int h[4] = {-1, -1, -1, -1}, cnt = 0;
    for (int d = 0; d < cw + order - 1; ++d) {
      int x = (c0 - order + 1 + d) % n;
      if (x < 0) x += n;
      const int t = x / bin_w;
      bool seen = false;
      for (int k = 0; k < cnt; ++k) seen |= (h[k] == t);
      if (!seen) {
        if (cnt == 4) return false;
        h[cnt++] = t;
      }
    }
    out->push_back(make_int4(h[0], h[1], h[2], h[3]));
  }
  return true;
}

// The same for the 16-row y tiles of k_spread_zdft_tcw: up to eight bins per
// tile, two int4 each.  Returns false when a tile would need more.
bool home_tile_table_w(int ext, int n, int order, int bin_w, std::vector<int4> *out) {
  out->clear();
  for (int c0 = 0; c0 < ext; c0 += kTwY) {
    const int cw = std::min(kTwY, ext - c0);
    int h[8] = {-1, -1, -1, -1, -1, -1, -1, -1}, cnt = 0;
    for (int d = 0; d < cw + order - 1; ++d) {
      int x = (c0 - order + 1 + d) % n;
      if (x < 0) x += n;
      const int t = x / bin_w;
      bool seen = false;
      for (int k = 0; k < cnt; ++k) seen |= (h[k] == t);
      if (!seen) {
        if (cnt == 8) return false;
        h[cnt++] = t;
      }
    }
    out->push_back(make_int4(h[0], h[1], h[2], h[3]));
    out->push_back(make_int4(h[4], h[5], h[6], h[7]));
  }
  return true;
}

// Per-frame geometry: g[0..9) = oc, the map from Cartesian to fractional
// coordinates (rows); g[9..18) = the map from k indices to q / 2pi used by the
// k-point code (rows).  Reference parity: oc from the box's upper triangle and
// q rows = sigma' oc.  Triclinic mode: oc = H^-T and q = 2 pi (sigma' oc)^T m,
// so the q rows are the transpose.
void frame_geometry(const SaxsPlan *pl, const float box[9], float g[kGeom]) {
  float oc[9];
  if (pl->p.box_mode == SAXS_BOX_TRICLINIC)
    saxs::cell_oc_triclinic(box, oc);
  else
    saxs::cell_oc(box, oc);
  const bool tr = pl->p.box_mode == SAXS_BOX_TRICLINIC;
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) {
      g[3 * r + c] = oc[3 * r + c];
      g[9 + 3 * r + c] = pl->sigma_scale * (tr ? oc[3 * c + r] : oc[3 * r + c]);
    }
  for (int i = 18; i < kGeom; ++i) g[i] = 0.0f;
}

int check_box(const float box[9]) {
  for (int i = 0; i < 9; ++i)
    if (!std::isfinite(box[i])) return fail(SAXS_E_INVALID, "box contains a non-finite value");
  if (!(box[0] > 0.f) || !(box[4] > 0.f) || !(box[8] > 0.f))
    return fail(SAXS_E_INVALID, "box diagonal must be positive");
  return SAXS_OK;
}

void destroy(SaxsPlan *pl) {
  if (!pl) return;
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(pl->device);
  for (void *p : pl->allocations) cudaFree(p);
  for (int i = 0; i < kRing; ++i)
    if (pl->ring.ev[i]) cudaEventDestroy(pl->ring.ev[i]);
  for (auto &r : pl->prof_pending)
    for (int k = 0; k < kStages; ++k) {
      if (r.start[k]) cudaEventDestroy(r.start[k]);
      if (r.stop[k]) cudaEventDestroy(r.stop[k]);
    }
  for (cudaEvent_t e : pl->event_pool) cudaEventDestroy(e);
  if (pl->ring.host) cudaFreeHost(pl->ring.host);
  cudaSetDevice(prev);
  delete pl;
}

// GEMM shape of a tensor-core DFT pass over `extent` values of u to `nk` values
// of k: N' = 2*nk padded to 16 (at most 256), two to four K-chunk stages in
// `avail` bytes of shared memory.  Returns false when the pass does not fit.
bool dtc_shape(int nk, int extent, size_t avail, DtcShape *sh, size_t *smem, bool allow_lo_smem) {
  const int N = round_up(2 * nk, 16);
  const size_t stage_bytes = (128 + 2 * static_cast<size_t>(N)) * 2 * kDtcChunk * sizeof(float);
  const int S_smem = static_cast<int>((avail - 1024) / stage_bytes);
  // tensor memory: two accumulators of N' columns and 64 columns of A per stage;
  // with the A remainder in shared memory (2N' <= 256): two accumulators of 2N'
  // columns and 32 columns per stage.  PYCUSAXS_DTC=split keeps the first form.
  // Measured on the 100k-atom workload: the y pass 0.60 ms per 100 frames with
  // the remainder in shared memory against 0.65 ms; the x pass, whose epilogue
  // then reads twice the accumulator columns, 0.34 against 0.33 ms, so it keeps
  // the first form.
  const char *mode = std::getenv("PYCUSAXS_DTC");
  sh->f16 = sh->side = 0;
  // f16 (the default; PYCUSAXS_DTC=tf32 or =split keep 3xTF32): per stage the
  // raw A tile and B' in halves; tensor memory: two accumulators of 2N' columns
  // ([Bh | Bl] side by side) or of N' columns, and 32 columns per stage
  if (!(mode && (std::strcmp(mode, "tf32") == 0 || std::strcmp(mode, "split") == 0))) {
    const size_t stage16 = (128 * sizeof(float) + 2 * static_cast<size_t>(N) * sizeof(uint16_t)) * 2 * kDtcChunk;
    const int S16 = static_cast<int>((avail - 1024) / stage16);
    // [Bh | Bl] side by side (two MMAs per k step) needs accumulators of 2N'
    // columns; the three-MMA form leaves tensor memory for more A stages, and is
    // taken when it gets more: at N' = 96 seven stages against four, y pass 0.574
    // -> 0.567 and x pass 0.249 -> 0.245 ms per 100 frames of the 100k-atom workload
    const int S_side = 2 * N <= 256 ? std::min({kDtcMaxStages, S16, (512 - 4 * N) / 32}) : 0;
    const int S_three = std::min({kDtcMaxStages, S16, (512 - 2 * N) / 32});
    int S = S_side, side = 1;
    if (S_three > S_side) {
      S = S_three;
      side = 0;
    }
    if (S >= 2 && N <= 256) {
      sh->f16 = 1;
      sh->side = side;
      sh->lo_smem = 0;
      sh->N = N;
      sh->chunks = (extent + kDtcChunk - 1) / kDtcChunk;
      sh->S = S;
      sh->cols = 512;
      *smem = S * stage16 + 1024;
      return true;
    }
  }
  int S = std::min({kDtcMaxStages, S_smem, (512 - 2 * N) / 64});
  sh->lo_smem = 0;
  if (allow_lo_smem && !(mode && std::strcmp(mode, "split") == 0) && 2 * N <= 256) {
    const int Sl = std::min({kDtcMaxStages, S_smem, (512 - 4 * N) / 32});
    if (Sl >= 2) {
      sh->lo_smem = 1;
      S = Sl;
    }
  }
  if (N > 256 || S < 2) return false;
  sh->N = N;
  sh->chunks = (extent + kDtcChunk - 1) / kDtcChunk;
  sh->S = S;
  sh->cols = 512;
  *smem = S * stage_bytes + 1024;  // + alignment slack of the stage base
  return true;
}

// B' operand of a tensor-core DFT pass from twiddles tw[u * stride + k] (u <
// extent, k < nk): per K chunk a head block then a remainder block, each N' x
// 2*kDtcChunk K-major, B'[2u + c][2k + d] = {Wr, Wi ; -Wi, Wr}[c][d].
std::vector<float> dtc_bprime(const std::vector<float2> &tw, int stride, int extent, int nk,
                              const DtcShape &sh) {
  const int KP = 2 * kDtcChunk, Np = sh.N;
  const size_t blk = static_cast<size_t>(Np) * KP;
  std::vector<float> out(static_cast<size_t>(sh.chunks) * 2 * blk, 0.0f);
  // element (n', k') of the head (part 0) or remainder (part 1) of chunk c: two
  // N'-column blocks, or one 2N'-column block with the parts side by side
  auto at = [&](int c, int part, int np, int kp) {
    const int n2 = sh.lo_smem ? np + part * Np : np, N2 = sh.lo_smem ? 2 * Np : Np;
    const size_t off = static_cast<size_t>(c) * 2 * blk + (sh.lo_smem ? 0 : part * blk);
    return off + static_cast<size_t>(kp / 4) * (N2 / 8) * 32 + (n2 / 8) * 32 + (n2 % 8) * 4 + kp % 4;
  };
  for (int c = 0; c < sh.chunks; ++c)
    for (int uu = 0; uu < kDtcChunk; ++uu) {
      const int u = c * kDtcChunk + uu;
      if (u >= extent) continue;
      for (int k = 0; k < nk; ++k) {
        const float2 w = tw[static_cast<size_t>(u) * stride + k];
        const float vals[2][2] = {{w.x, w.y}, {-w.y, w.x}};
        for (int cz = 0; cz < 2; ++cz)
          for (int d = 0; d < 2; ++d) {
            const int kp = 2 * uu + cz, np = 2 * k + d;
            const float v = vals[cz][d];
            uint32_t bits;
            std::memcpy(&bits, &v, sizeof(bits));
            bits &= 0xFFFFE000u;
            float head;
            std::memcpy(&head, &bits, sizeof(head));
            out[at(c, 0, np, kp)] = head;
            out[at(c, 1, np, kp)] = v - head;
          }
      }
    }
  return out;
}

// The same B' for an f16 pass: head = the twiddle rounded to f16, remainder =
// the rounded difference, in K-major blocks of 16-byte K groups (element (n',
// k') at half ((k' / 8) * N2 + n') * 8 + k' % 8, N2 the block's columns), head
// and remainder side by side (one block of 2N' columns) or one after the other;
// packed two halves per float.
std::vector<float> dtc_bprime16(const std::vector<float2> &tw, int stride, int extent, int nk,
                                const DtcShape &sh) {
  const int KP = 2 * kDtcChunk, Np = sh.N, N2 = sh.side ? 2 * Np : Np;
  const size_t blk = static_cast<size_t>(Np) * KP;  // halves of a head or remainder block
  std::vector<__half> out(static_cast<size_t>(sh.chunks) * 2 * blk, __float2half_rn(0.0f));
  auto at = [&](int c, int part, int np, int kp) {
    const int n2 = sh.side ? np + part * Np : np;
    const size_t off = static_cast<size_t>(c) * 2 * blk + (sh.side ? 0 : part * blk);
    return off + (static_cast<size_t>(kp / 8) * N2 + n2) * 8 + kp % 8;
  };
  for (int c = 0; c < sh.chunks; ++c)
    for (int uu = 0; uu < kDtcChunk; ++uu) {
      const int u = c * kDtcChunk + uu;
      if (u >= extent) continue;
      for (int k = 0; k < nk; ++k) {
        const float2 w = tw[static_cast<size_t>(u) * stride + k];
        const float vals[2][2] = {{w.x, w.y}, {-w.y, w.x}};
        for (int cz = 0; cz < 2; ++cz)
          for (int d = 0; d < 2; ++d) {
            const int kp = 2 * uu + cz, np = 2 * k + d;
            const float v = vals[cz][d];
            const __half h = __float2half_rn(v);
            out[at(c, 0, np, kp)] = h;
            out[at(c, 1, np, kp)] = __float2half_rn(v - __half2float(h));
          }
      }
    }
  std::vector<float> packed(out.size() / 2);
  std::memcpy(packed.data(), out.data(), packed.size() * sizeof(float));
  return packed;
}

// `min_half`, when given, is the smallest k-box half-width per axis the plan
// must have (a re-plan for a frame whose box grew past the margin).
int create(const SaxsParams *prm, SaxsPlan **out, const long long *min_half = nullptr) {
  if (!prm || !out) return fail(SAXS_E_INVALID, "null argument");
  *out = nullptr;
  const SaxsParams &p = *prm;
  for (int d = 0; d < 3; ++d)
    if (p.grid[d] <= 0) return fail(SAXS_E_INVALID, "Grid dimensions must be positive");
  if (p.order < 1 || p.order > 8)
    return fail(SAXS_E_INVALID, "Spline order must be between 1 and 8");
  if (p.ntypes < 1 || !p.form_factors) return fail(SAXS_E_INVALID, "at least one atom type is required");
  if (p.natoms < 0 || p.nentries < 0) return fail(SAXS_E_INVALID, "negative atom count");
  if (p.nentries > 0 && (!p.entry_atom || !p.entry_type))
    return fail(SAXS_E_INVALID, "atom lists missing");
  if (p.max_frames < 1) return fail(SAXS_E_INVALID, "max_frames must be >= 1");
  if (p.ensemble != SAXS_NPT && p.ensemble != SAXS_NVT)
    return fail(SAXS_E_INVALID, "ensemble must be npt or nvt");
  if (int rc = check_box(p.box0)) return rc;
  if (p.box_mode != SAXS_BOX_PARITY && p.box_mode != SAXS_BOX_TRICLINIC)
    return fail(SAXS_E_INVALID, "box_mode must be parity (0) or triclinic (1)");
  if (p.padding_mode != SAXS_PAD_AVERAGE && p.padding_mode != SAXS_PAD_GIVEN)
    return fail(SAXS_E_INVALID, "padding_mode must be average (0) or given (1)");
  if (p.padding_mode == SAXS_PAD_GIVEN) {
    if (!p.padding_values) return fail(SAXS_E_INVALID, "given padding needs padding_values");
    for (int t = 0; t < p.ntypes; ++t)
      if (!std::isfinite(p.padding_values[t]) || p.padding_values[t] < 0.0f)
        return fail(SAXS_E_INVALID, "padding values must be finite and non-negative");
  }
  for (int i = 0; i < p.nentries; ++i) {
    if (p.entry_atom[i] < 0 || p.entry_atom[i] >= p.natoms)
      return fail(SAXS_E_INVALID, "atom index " + std::to_string(p.entry_atom[i]) +
                                      " out of range [0, " + std::to_string(p.natoms) + ")");
    if (p.entry_type[i] < 0 || p.entry_type[i] >= p.ntypes)
      return fail(SAXS_E_INVALID, "type index out of range");
  }
  const bool scaled = p.scaled_grid[0] > 0 || p.scaled_grid[1] > 0 || p.scaled_grid[2] > 0;
  int nn[3];
  for (int d = 0; d < 3; ++d) {
    if (scaled) {
      if (p.scaled_grid[d] <= 0) return fail(SAXS_E_INVALID, "Scaled grid dimensions must be positive");
      nn[d] = p.scaled_grid[d];
    } else {
      if (!(p.scale_factor > 0.0f))
        return fail(SAXS_E_INVALID, "Scale factor must be positive when scaled grid is not provided");
      const long long v = saxs::closest_product(p.grid[d], p.scale_factor);
      if (v < 1 || v > (1 << 20)) return fail(SAXS_E_INVALID, "scaled grid out of range");
      nn[d] = static_cast<int>(v);
    }
  }
  const int ntaps = std::min(p.order, 4);
  for (int d = 0; d < 3; ++d) {
    if (p.grid[d] < p.order)
      return fail(SAXS_E_INVALID, "grid dimension smaller than the spline order");
    if (nn[d] < 2) return fail(SAXS_E_INVALID, "scaled grid dimension must be >= 2");
  }

  SaxsPlan *pl = new SaxsPlan();
  cudaGetDevice(&pl->device);
  pl->p = p;
  if (p.padding_mode == SAXS_PAD_GIVEN) pl->pad.assign(p.padding_values, p.padding_values + p.ntypes);
  pl->p.padding_values = nullptr;  // the caller's array is not kept
  pl->ensemble = p.ensemble;
  pl->ff.assign(p.form_factors, p.form_factors + 9 * p.ntypes);
  pl->ea_host.assign(p.entry_atom, p.entry_atom + p.nentries);
  pl->et_host.assign(p.entry_type, p.entry_type + p.nentries);
  pl->p.form_factors = nullptr;  // nor are the caller's arrays
  pl->p.entry_atom = pl->p.entry_type = nullptr;
  DevArgs &a = pl->a;
  for (int d = 0; d < 3; ++d) {
    a.n[d] = p.grid[d];
    a.nn[d] = nn[d];
    a.ext[d] = std::min(p.grid[d], nn[d]);
    a.nf[d] = saxs::nf_of(nn[d]);
  }
  a.order = p.order;
  a.ntaps = ntaps;
  a.T = p.ntypes;
  a.M = p.nentries;
  // home bins 4 columns wide cut the atoms an item visits without reaching its
  // tile (about half with 8-wide bins, a sixth with 4-wide ones)
  std::vector<int4> hxt, hyt;
  a.bin_w = 4;
  if (!home_tile_table(a.ext[0], a.n[0], a.order, 4, &hxt) ||
      !home_tile_table(a.ext[1], a.n[1], a.order, 4, &hyt)) {
    a.bin_w = 8;
    if (!home_tile_table(a.ext[0], a.n[0], a.order, 8, &hxt) ||
        !home_tile_table(a.ext[1], a.n[1], a.order, 8, &hyt)) {
      destroy(pl);
      return fail(SAXS_E_INVALID, "spline order too large for the spread tiles");
    }
  }
  a.tiles[0] = (a.n[0] + a.bin_w - 1) / a.bin_w;
  a.tiles[1] = (a.n[1] + a.bin_w - 1) / a.bin_w;
  a.stiles[0] = (a.ext[0] + kTile - 1) / kTile;
  a.stiles[1] = (a.ext[1] + kTile - 1) / kTile;
  std::vector<int4> hywt;
  a.stw = home_tile_table_w(a.ext[1], a.n[1], a.order, a.bin_w, &hywt) ? (a.ext[1] + kTwY - 1) / kTwY : 0;
  a.nbins = a.T * a.tiles[0] * a.tiles[1];
  a.dz = static_cast<int>(0.07f * a.n[2] / 2);  // borderBins (saxsKernel.h:107-110)
  {
    int planes = 0;
    for (int z = 0; z < a.n[2]; ++z)
      if (!(z > a.dz && z < a.n[2] - a.dz)) ++planes;
    a.border_count = static_cast<double>(a.n[0]) * a.n[1] * planes;
  }
  a.nn3 = static_cast<double>(nn[0]) * nn[1] * nn[2];

  pl->sigma_scale = static_cast<float>(a.n[0]) / static_cast<float>(nn[0]);
  float geo0[kGeom];
  frame_geometry(pl, p.box0, geo0);
  float oc0[9], ocs0[9];
  for (int i = 0; i < 9; ++i) {
    oc0[i] = geo0[i];
    ocs0[i] = geo0[9 + i];
  }
  saxs::histogram_parameters(nn, oc0, p.scale_factor, p.bin_size, p.qcut, &a.dq, &a.qcut,
                             &a.num_bins);
  if (a.num_bins < 1) a.num_bins = 1;

  // k-box: every integer k with |2 pi ocs k| <= qcut for the first frame and
  // for boxes up to `box_margin` smaller.
  const double margin = std::max(0.0f, p.box_margin) + 1e-5;
  saxs::kbox_halfwidths(ocs0, a.qcut, margin, pl->half);
  if (min_half)
    for (int d = 0; d < 3; ++d) pl->half[d] = std::max(pl->half[d], min_half[d]);
  for (int d = 0; d < 2; ++d) {
    const long long hmax = a.nf[d] - 1;
    if (pl->half[d] >= hmax) {
      pl->full_axis[d] = true;
      pl->half[d] = hmax;
    }
  }
  a.kx_lo = pl->full_axis[0] ? a.nf[0] - nn[0] : -static_cast<int>(pl->half[0]);
  a.nkx = pl->full_axis[0] ? nn[0] : 2 * static_cast<int>(pl->half[0]) + 1;
  a.ky_lo = pl->full_axis[1] ? a.nf[1] - nn[1] : -static_cast<int>(pl->half[1]);
  a.nky = pl->full_axis[1] ? nn[1] : 2 * static_cast<int>(pl->half[1]) + 1;
  if (pl->half[2] >= nn[2] / 2) {
    pl->full_axis[2] = true;
    pl->half[2] = nn[2] / 2;
  }
  a.nkz = static_cast<int>(pl->half[2]) + 1;
  a.nkzp = round_up(a.nkz, kKzThread);
  a.nkxp = round_up(a.nkx, 2);
  a.nkyp = round_up(a.nky, kKyGroup);

  // shared-memory budgets (rows of twiddles / x chunks shrink to fit)
  const size_t optin = static_cast<size_t>(optin_smem());
  {
    const size_t NP = 2 * static_cast<size_t>(a.nkzp);
    const size_t tile = std::max<size_t>(static_cast<size_t>(a.n[2]) * kCols, kCols * NP) * sizeof(float);
    const size_t avail = optin - static_smem(k_spread_zdft);
    size_t zc = a.ext[2];
    while (zc > 8 && zc * NP * sizeof(float) + tile > avail) zc = (zc > 16) ? zc / 2 : 8;
    a.zc = static_cast<int>(zc);
    pl->smem_spread = zc * NP * sizeof(float) + tile;
  }
  pl->smem_ydft = static_cast<size_t>(kYChunk) * kYStride * sizeof(float2) +
                  static_cast<size_t>(kYChunk) * a.nkyp * sizeof(float2);
  {
    const size_t avail = optin - static_smem(k_xdft_post);
    const size_t fixed = static_cast<size_t>(a.T) * a.nkxp * sizeof(float2);
    const size_t per_x = (static_cast<size_t>(a.nkxp) + a.T) * sizeof(float2);
    size_t xc = a.ext[0];
    if (fixed + xc * per_x > avail) xc = avail > fixed + 2 * per_x ? (avail - fixed) / per_x : 2;
    xc = std::max<size_t>(2, xc & ~static_cast<size_t>(1));
    pl->xc = static_cast<int>(std::min<size_t>(xc, a.ext[0]));
    pl->smem_xdft = fixed + static_cast<size_t>(pl->xc) * per_x;
  }
  {
    // tensor-core z-DFT: N = 2*nkz padded to 8 (<= 256; to 16 and <= 128 for wide tiles),
    // K = ez padded to 8, two operand stages when they fit, else one.
    // PYCUSAXS_ZDFT=simt keeps the FP32 SIMT kernel, PYCUSAXS_ZDFT=narrow the
    // 64-column tensor-core kernel.
    const char *mode = std::getenv("PYCUSAXS_ZDFT");
    const bool simt_only = mode && std::strcmp(mode, "simt") == 0;
    const bool narrow_only = mode && std::strcmp(mode, "narrow") == 0;
    const int N = round_up(2 * a.nkz, 8);
    const int NW = round_up(2 * a.nkz, 16);  // M = 128 needs N a multiple of 16
    const int KT = round_up(a.ext[2], 16);  // K = 16 per f16 MMA of the wide kernel
    const int R = std::max(KT, round_up(a.n[2], 8));
    const size_t avail = optin - static_smem(k_spread_zdft_tc);
    const size_t b_bytes = 2 * static_cast<size_t>(KT) * N * sizeof(float);
    const size_t stage_bytes = static_cast<size_t>(R + KT) * 64 * sizeof(float);
    const size_t home_bytes = static_cast<size_t>(a.stiles[0] + a.stiles[1]) * sizeof(int4);
    // two operand stages before larger record buffers before a larger atom
    // table; records beyond the staging buffer are read from global memory,
    // atoms beyond the table are spread in further chunks
    // (one atom table per producer group: two groups with two stages)
    int S = 0, RB = 0, CAP = 0;
    for (int s_try = 2; s_try >= 1 && S == 0; --s_try)
      for (int cap = 256; cap >= 64 && S == 0; cap /= 2)
        for (int rb = 1024; rb >= 128 && S == 0; rb /= 2)
          if (b_bytes + s_try * stage_bytes + 2 * static_cast<size_t>(rb) * 16 + home_bytes +
                  static_cast<size_t>(s_try) * cap * kTcAtomBytes <= avail) {
            S = s_try;
            RB = rb;
            CAP = cap;
          }
    // wide tiles, for one and for two producer groups: twG fixed-point tiles of
    // 128 x (R + 4) words, then the largest atom table (each table chunk costs a
    // latency-bound pre-pass and two barriers), then the largest record buffer
    // that fit beside them
    const int RSW = R + 4;
    const size_t home_w = static_cast<size_t>(a.stiles[0] + 2 * a.stw) * sizeof(int4);
    const size_t bw_bytes = 2 * static_cast<size_t>(KT) * NW * sizeof(uint16_t);  // f16 B''
    auto wide_bytes = [&](int g, int rb, int cap) {
      return bw_bytes + static_cast<size_t>(g) * 128 * RSW * sizeof(float) + 2 * static_cast<size_t>(rb) * 16 +
             home_w + static_cast<size_t>(g) * cap * kTwAtomBytes;
    };
    int GW = 0;
    if (a.stw > 0 && NW <= 64) {  // two accumulator stages of 2*NW columns
      const size_t avail_w = optin - static_smem(k_spread_zdft_tcw);
      static const int cand[][2] = {{1024, 1024}, {1024, 512}, {512, 1024}, {512, 512}, {1024, 256},
                                    {512, 256},   {256, 1024}, {256, 512},  {256, 256}, {128, 512},
                                    {128, 256},   {128, 128},  {64, 128}};  // {cap, records}
      for (int g = 1; g <= 2; ++g)
        for (const auto &c : cand)
          if (pl->tw_cap[g - 1] == 0 && wide_bytes(g, c[1], c[0]) <= avail_w) {
            pl->tw_cap[g - 1] = c[0];
            pl->tw_rb[g - 1] = c[1];
            GW = g;
          }
    }
    // atom-GEMM tiles: B' = [Sh | Sl] of 2 * NB columns (NB = 2 * nkz padded to
    // 16, N2 <= 256 and two accumulator stages in 512 columns), kAgSlots chunk
    // slots, then the largest atom table and record buffer beside them
    {
      const int NB = round_up(2 * a.nkz, 16);
      const char *agm = std::getenv("PYCUSAXS_ZAG");  // PYCUSAXS_ZAG=0: not available
      if (a.stw > 0 && 2 * NB <= 256 && !simt_only && !(agm && std::strcmp(agm, "0") == 0)) {
        const size_t avail_ag = optin - static_smem(k_spread_zdft_ag);
        const size_t fixed = 128 + kAgSlots * (2 * kAgWBytes + static_cast<size_t>(kAgK) * 2 * NB * 2) +
                             static_cast<size_t>(a.stiles[0] + 2 * a.stw) * sizeof(int4) +
                             static_cast<size_t>(round_up(a.ext[2] * a.nkz, 2)) * sizeof(float2);
        static const int cand[][2] = {{1024, 1024}, {1024, 512}, {512, 1024}, {512, 512}, {1024, 256},
                                      {512, 256},   {256, 512},  {256, 256},  {128, 256}, {128, 128}};
        for (const auto &c : cand)
          if (!pl->ag_ok && fixed + 2 * static_cast<size_t>(c[1]) * 16 + static_cast<size_t>(c[0]) * kAgAtomBytes <=
                                avail_ag) {
            pl->ag_ok = true;
            a.agNB = NB;
            a.agCap = c[0];
            a.agRB = c[1];
            pl->smem_spread_ag = fixed + 2 * static_cast<size_t>(c[1]) * 16 + static_cast<size_t>(c[0]) * kAgAtomBytes;
          }
      }
    }
    pl->tcn_ok = !simt_only && N <= 256 && S > 0;
    // (the wide kernel's epilogue indexes a (frame, type) block of Z in 32 bits)
    pl->tcw_ok = !simt_only && !narrow_only && GW > 0 &&
                 static_cast<int64_t>(a.nkz) * a.ext[0] * a.ext[1] < (int64_t{1} << 31);
    if (pl->ag_ok) pl->use_ag = mode && std::strcmp(mode, "atoms") == 0;  // PYCUSAXS_ZDFT=atoms
    if (pl->tcn_ok || pl->tcw_ok || pl->ag_ok) {
      pl->use_tc = true;
      pl->use_tcw = pl->tcw_ok;
      a.tcN = N;
      a.tcK = KT;
      a.tcR = R;
    }
    if (pl->tcw_ok) {
      a.twN = NW;
      a.twRS = RSW;
      pl->twG_max = GW;
      for (int g = 1; g <= GW; ++g) pl->tw_smem[g - 1] = wide_bytes(g, pl->tw_rb[g - 1], pl->tw_cap[g - 1]);
      // one group by default: its larger atom table measured faster than two
      // groups on the 100k-atom trajectory workload (2.95 vs 3.42 ms per 100 frames)
      set_wide_groups(pl, 1);
    }
    if (pl->tcn_ok) {
      a.tcS = S;
      a.tcRB = RB;
      a.tcCap = CAP;
      a.tcG = S == 2 ? 2 : 1;
      int cols = 32;
      while (cols < S * N) cols *= 2;
      a.tcCols = cols;
      pl->smem_spread_tc = b_bytes + S * stage_bytes + 2 * static_cast<size_t>(RB) * 16 + home_bytes +
                           static_cast<size_t>(S) * CAP * kTcAtomBytes;
    }
  }
  {
    // tensor-core y- and x-axis DFTs when their shapes fit; the x pass needs at
    // most 16 types.  PYCUSAXS_YDFT=simt / PYCUSAXS_XDFT=simt keep the FP32
    // SIMT kernels.
    const char *ym = std::getenv("PYCUSAXS_YDFT");
    const char *xm = std::getenv("PYCUSAXS_XDFT");
    // the tensor maps need row strides that are multiples of 16 bytes: even extents
    if (!(ym && std::strcmp(ym, "simt") == 0) && a.ext[1] % 2 == 0)
      pl->use_ytc = dtc_shape(a.nky, a.ext[1], optin - static_smem(k_dft_tc<false>), &pl->yshape,
                              &pl->smem_ydft_tc, true);
    a.xtcKyb = 128 / a.T;
    if (!(xm && std::strcmp(xm, "simt") == 0) && a.T <= 16 && a.ext[0] % 2 == 0)
      pl->use_xtc = dtc_shape(a.nkx, a.ext[0], optin - static_smem(k_dft_tc<true>), &pl->xshape,
                              &pl->smem_xdft_tc, false);
  }
  pl->tc_ok = pl->use_tc;
  pl->ytc_ok = pl->use_ytc;
  pl->xtc_ok = pl->use_xtc;
  pl->smem_hist = a.num_bins <= kHistSmemBins ? 2 * sizeof(double) * a.num_bins : 0;
  const size_t smem_sort = 2 * sizeof(int) * static_cast<size_t>(a.tiles[0]) * a.tiles[1];
  if (pl->smem_spread + static_smem(k_spread_zdft) > optin ||
      pl->smem_ydft + static_smem(k_ydft) > optin ||
      pl->smem_xdft + static_smem(k_xdft_post) > optin ||
      pl->smem_hist + static_smem(k_hist<double>) > optin || smem_sort + static_smem(k_sort_atoms) > optin) {
    destroy(pl);
    return fail(SAXS_E_INVALID,
                "grid / q-cut combination exceeds the shared-memory budget (z extent " +
                    std::to_string(a.n[2]) + ", k-box " + std::to_string(a.nkx) + "x" +
                    std::to_string(a.nky) + "x" + std::to_string(a.nkz) + ")");
  }
  if (a.T > 64) {
    destroy(pl);
    return fail(SAXS_E_INVALID, "at most 64 element types are supported");
  }

  const int B = p.max_frames;
  const int ex = a.ext[0], ey = a.ext[1], ez = a.ext[2];
  {
    // free-memory check before allocating, as the reference does
    // (saxsKernel.cu:284-314), over the buffers that grow with the frames per call
    const size_t per_frame = (sizeof(int2) + sizeof(float4)) * static_cast<size_t>(a.M) +
                             sizeof(int) * (static_cast<size_t>(a.nbins) + 1) + sizeof(double) * a.T +
                             sizeof(float2) * static_cast<size_t>(a.T) * a.nkz * ex * ey +
                             sizeof(float2) * static_cast<size_t>(a.T) * a.nkz * a.nky * ex +
                             sizeof(float) * static_cast<size_t>(a.nkz) * a.nky * a.nkx;
    const double need = static_cast<double>(per_frame) * B;
    size_t fr = 0, tot = 0;
    if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) {
      cudaGetLastError();
    } else if (need > static_cast<double>(fr)) {
      destroy(pl);
      char msg[256];
      std::snprintf(msg, sizeof(msg),
                    "not enough device memory: %d frames per call need %.3g GB of frame buffers, "
                    "%.3g GB of %.3g GB are free (lower max_frames)",
                    B, need / 1e9, fr / 1e9, tot / 1e9);
      return fail(SAXS_E_NOMEM, msg);
    }
  }
  int rc = SAXS_OK;
  int32_t *d_ea = nullptr, *d_et = nullptr;
  float2 *d_twz = nullptr, *d_twy = nullptr, *d_twx = nullptr;
  float *d_modx = nullptr, *d_mody = nullptr, *d_modz = nullptr, *d_ff = nullptr, *d_geom = nullptr;
  int *d_status = nullptr;
#define ALLOC(ptr, cnt)                       \
  do {                                        \
    if ((rc = dalloc(pl, &(ptr), (cnt)))) {   \
      destroy(pl);                            \
      return rc;                              \
    }                                         \
  } while (0)
  ALLOC(d_ea, a.M);
  ALLOC(d_et, a.M);
  int *d_ts = nullptr;
  ALLOC(d_ts, a.T + 1);
  // entries grouped by type (stable), the sort kernel's per-type ranges
  std::vector<int32_t> ea_sorted(a.M), et_sorted(a.M);
  std::vector<int> type_start(a.T + 1, 0);
  for (int i = 0; i < a.M; ++i) ++type_start[p.entry_type[i] + 1];
  for (int t = 0; t < a.T; ++t) {
    pl->sort_max_type = std::max(pl->sort_max_type, type_start[t + 1]);
    type_start[t + 1] += type_start[t];
  }
  {
    std::vector<int> fill(type_start.begin(), type_start.end() - 1);
    for (int i = 0; i < a.M; ++i) {
      const int k = fill[p.entry_type[i]]++;
      ea_sorted[k] = p.entry_atom[i];
      et_sorted[k] = p.entry_type[i];
    }
  }
  ALLOC(d_twz, static_cast<size_t>(ez) * a.nkzp);
  ALLOC(d_twy, static_cast<size_t>(ey) * a.nkyp);
  ALLOC(d_twx, static_cast<size_t>(ex) * a.nkxp);
  ALLOC(d_modx, nn[0]);
  ALLOC(d_mody, nn[1]);
  ALLOC(d_modz, nn[2]);
  ALLOC(d_ff, 9 * a.T);
  float *d_pad = nullptr;
  if (!pl->pad.empty()) ALLOC(d_pad, a.T);
  int4 *d_hx = nullptr, *d_hy = nullptr;
  float *d_twzs = nullptr, *d_twztc = nullptr, *d_twytc = nullptr, *d_twxtc = nullptr;
  ALLOC(d_twzs, 2 * a.nkzp);
  int4 *d_hyw = nullptr;
  float *d_twztcw = nullptr;
  if (pl->tcn_ok) ALLOC(d_twztc, 2 * static_cast<size_t>(a.tcK) * a.tcN);
  if (pl->tcw_ok) ALLOC(d_twztcw, 2 * static_cast<size_t>(a.tcK) * a.twN);
  if (pl->tcw_ok) ALLOC(d_hyw, 2 * static_cast<size_t>(a.stw));
  // Element types whose wide items would see fewer than r atoms on average
  // (expected atoms reaching an 8 x 16 column tile; r = PYCUSAXS_SPARSE_REACH,
  // default 24, 0 turns it off) go to k_spread_zdft_sparse, whose cost grows with
  // the atoms where the wide kernel's hardly does (~6k cycles per item + ~14 per
  // atom).  On the 100k-atom workload r = 24 sends its two 1% types (~13 atoms per
  // tile): 2.30 -> 2.06 ms per 100 frames; adding the 5% type (~64) was slower
  // (2.15 ms).  The order of tw_types is the wide kernel's types, then the sparse
  // ones.
  std::vector<int> tw_types;
  {
    const char *sr = std::getenv("PYCUSAXS_SPARSE_REACH");
    const double lim = sr ? std::atof(sr) : 24.0;
    const size_t sp_smem = 2 * 128 * static_cast<size_t>(a.nkz) * sizeof(int);
    const bool can = pl->tcw_ok && lim > 0.0 && sp_smem + static_smem(k_spread_zdft_sparse) <= optin_smem();
    const double cols = static_cast<double>(kTwX + a.ntaps - 1) * (kTwY + a.ntaps - 1) /
                        (static_cast<double>(a.n[0]) * a.n[1]);
    std::vector<int> sparse;
    for (int t = 0; t < a.T; ++t) {
      const double reach = (type_start[t + 1] - type_start[t]) * cols;
      if (can && reach < lim) sparse.push_back(t);
      else tw_types.push_back(t);
    }
    a.tw_nd = static_cast<int>(tw_types.size());
    a.tw_ns = static_cast<int>(sparse.size());
    tw_types.insert(tw_types.end(), sparse.begin(), sparse.end());
    pl->smem_sparse = a.tw_ns > 0 ? sp_smem : 0;
  }
  int *d_twt = nullptr;
  ALLOC(d_twt, a.T);
  if (pl->use_ytc) ALLOC(d_twytc, static_cast<size_t>(pl->yshape.chunks) * 4 * pl->yshape.N * kDtcChunk);
  if (pl->use_xtc) ALLOC(d_twxtc, static_cast<size_t>(pl->xshape.chunks) * 4 * pl->xshape.N * kDtcChunk);
  ALLOC(d_hx, a.stiles[0]);
  ALLOC(d_hy, a.stiles[1]);
  ALLOC(d_geom, static_cast<size_t>(B) * kGeom);
  ALLOC(pl->d_geom0, kGeom);
  ALLOC(d_status, 4);
  ALLOC(a.key, static_cast<size_t>(B) * a.M);
  ALLOC(a.offsets, static_cast<size_t>(B) * (a.nbins + 1));
  ALLOC(a.rec, static_cast<size_t>(B) * a.M);
  ALLOC(a.border, static_cast<size_t>(B) * a.T);
  ALLOC(a.Z, static_cast<size_t>(B) * a.T * a.nkz * ex * ey);
  ALLOC(a.Y, static_cast<size_t>(B) * a.T * a.nkz * a.nky * ex);
  ALLOC(a.ibox, static_cast<size_t>(B) * a.nkz * a.nky * a.nkx);
  ALLOC(a.hist, a.num_bins);
  ALLOC(a.nhist, a.num_bins);
  ALLOC(pl->d_tmp_hist, 2 * a.num_bins);
  if (pl->ensemble == SAXS_NVT) ALLOC(a.iacc, static_cast<size_t>(a.nkz) * a.nky * a.nkx);
#undef ALLOC
  a.entry_atom = d_ea;
  a.type_start = d_ts;
  a.entry_type = d_et;
  a.twz = d_twz;
  a.twy = d_twy;
  a.twx = d_twx;
  a.modx = d_modx;
  a.mody = d_mody;
  a.modz = d_modz;
  a.ff = d_ff;
  a.pad_val = d_pad;
  a.twz_sum = d_twzs;
  a.twz_tc = d_twztc;
  a.twz_tcw = d_twztcw;
  pl->yshape.B = d_twytc;
  pl->xshape.B = d_twxtc;
  a.home_x = d_hx;
  a.home_y = d_hy;
  a.home_yw = d_hyw;
  a.tw_types = d_twt;
  a.geom = d_geom;
  a.status = d_status;

  // host tables
  std::vector<float2> twz(static_cast<size_t>(ez) * a.nkzp, make_float2(0.f, 0.f));
  for (int z = 0; z < ez; ++z)
    for (int k = 0; k < a.nkz; ++k) saxs::twiddle(k, z, nn[2], &twz[z * a.nkzp + k].x, &twz[z * a.nkzp + k].y);
  std::vector<float> twzs(2 * a.nkzp, 0.0f);
  for (int k = 0; k < a.nkz; ++k) {
    double re = 0.0, im = 0.0;
    for (int z = 0; z < ez; ++z) {
      long long r = (static_cast<long long>(k) * z) % nn[2];
      const double ang = -2.0 * M_PI * static_cast<double>(r) / nn[2];
      re += std::cos(ang);
      im += std::sin(ang);
    }
    twzs[2 * k] = static_cast<float>(re);
    twzs[2 * k + 1] = static_cast<float>(im);
  }
  // the same z twiddles in the tensor-core B layout, split into a TF32 head and
  // the exact remainder
  // B operand of the tensor-core z passes, N columns: the z twiddles split into a
  // TF32 head and remainder, K-major canonical layout
  auto z_operand = [&](int N) {
    std::vector<float> out(2 * static_cast<size_t>(a.tcK) * N, 0.0f);
    const size_t half = static_cast<size_t>(a.tcK) * N;
    for (int z = 0; z < ez; ++z)
      for (int n = 0; n < 2 * a.nkz; ++n) {
        const float2 w = twz[z * a.nkzp + n / 2];
        const float v = (n & 1) ? w.y : w.x;
        uint32_t bits;
        std::memcpy(&bits, &v, sizeof(bits));
        bits &= 0xFFFFE000u;
        float head;
        std::memcpy(&head, &bits, sizeof(head));
        const size_t o = static_cast<size_t>(z / 4) * (N / 8) * 32 + (n / 8) * 32 + (n % 8) * 4 + z % 4;
        out[o] = head;
        out[half + o] = v - head;
      }
    return out;
  };
  const std::vector<float> twtc = pl->tcn_ok ? z_operand(a.tcN) : std::vector<float>();
  // wide tiles: B' = [Bh | Bl] as one K-major operand of 2*twN columns
  // wide kernel: B' = [Bh | Bl] in f16, Bh the twiddle rounded to f16 and Bl the
  // rounded remainder; element (z, n) at half ((z / 8) * 2twN + n) * 8 + z % 8
  // (K-major, 16-byte K blocks of 2twN rows)
  std::vector<__half> twtcw;
  if (pl->tcw_ok) {
    const int NB = a.twN, N2 = 2 * a.twN;
    twtcw.assign(static_cast<size_t>(a.tcK) * N2, __float2half_rn(0.0f));
    for (int z = 0; z < ez; ++z)
      for (int n = 0; n < 2 * a.nkz; ++n) {
        const float2 w = twz[z * a.nkzp + n / 2];
        const float v = (n & 1) ? w.y : w.x;
        const __half h = __float2half_rn(v);
        const __half l = __float2half_rn(v - __half2float(h));
        twtcw[(static_cast<size_t>(z / 8) * N2 + n) * 8 + z % 8] = h;
        twtcw[(static_cast<size_t>(z / 8) * N2 + n + NB) * 8 + z % 8] = l;
      }
  }
  std::vector<float2> twy(static_cast<size_t>(ey) * a.nkyp, make_float2(0.f, 0.f));
  for (int y = 0; y < ey; ++y)
    for (int k = 0; k < a.nky; ++k)
      saxs::twiddle(a.ky_lo + k, y, nn[1], &twy[y * a.nkyp + k].x, &twy[y * a.nkyp + k].y);
  std::vector<float2> twx(static_cast<size_t>(ex) * a.nkxp, make_float2(0.f, 0.f));
  for (int x = 0; x < ex; ++x)
    for (int k = 0; k < a.nkx; ++k)
      saxs::twiddle(a.kx_lo + k, x, nn[0], &twx[x * a.nkxp + k].x, &twx[x * a.nkxp + k].y);
  auto bprime = [&](const std::vector<float2> &tw, int stride, int extent, int nk, const DtcShape &sh) {
    return sh.f16 ? dtc_bprime16(tw, stride, extent, nk, sh) : dtc_bprime(tw, stride, extent, nk, sh);
  };
  const std::vector<float> twytc = pl->use_ytc ? bprime(twy, a.nkyp, ey, a.nky, pl->yshape) : std::vector<float>();
  const std::vector<float> twxtc = pl->use_xtc ? bprime(twx, a.nkxp, ex, a.nkx, pl->xshape) : std::vector<float>();
  const int ndim = std::max(nn[0], std::max(nn[1], nn[2]));
  std::vector<float> mx(nn[0]), my(nn[1]), mz(nn[2]);
  saxs::bspline_moduli(nn[0], ndim, mx.data());
  saxs::bspline_moduli(nn[1], ndim, my.data());
  saxs::bspline_moduli(nn[2], ndim, mz.data());
  float g0[kGeom];
  frame_geometry(pl, p.box0, g0);

  auto up = [&](void *dst, const void *src, size_t bytes) -> int {
    if (bytes == 0) return SAXS_OK;
    cudaError_t e = cudaMemcpy(dst, src, bytes, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return fail(SAXS_E_CUDA, std::string("upload: ") + cudaGetErrorString(e));
    return SAXS_OK;
  };
  if ((rc = up(d_ea, ea_sorted.data(), sizeof(int32_t) * a.M)) ||
      (rc = up(d_et, et_sorted.data(), sizeof(int32_t) * a.M)) ||
      (rc = up(d_ts, type_start.data(), sizeof(int) * (a.T + 1))) ||
      (rc = up(d_twz, twz.data(), sizeof(float2) * twz.size())) ||
      (rc = up(d_twy, twy.data(), sizeof(float2) * twy.size())) ||
      (rc = up(d_twx, twx.data(), sizeof(float2) * twx.size())) ||
      (rc = up(d_modx, mx.data(), sizeof(float) * nn[0])) ||
      (rc = up(d_mody, my.data(), sizeof(float) * nn[1])) ||
      (rc = up(d_modz, mz.data(), sizeof(float) * nn[2])) ||
      (rc = up(d_ff, pl->ff.data(), sizeof(float) * pl->ff.size())) ||
      (rc = up(d_pad, pl->pad.data(), sizeof(float) * pl->pad.size())) ||
      (rc = up(d_hx, hxt.data(), sizeof(int4) * hxt.size())) ||
      (rc = up(d_twzs, twzs.data(), sizeof(float) * twzs.size())) ||
      (rc = up(d_twztc, twtc.data(), sizeof(float) * twtc.size())) ||
      (rc = up(d_twztcw, twtcw.data(), sizeof(__half) * twtcw.size())) ||
      (rc = up(d_twytc, twytc.data(), sizeof(float) * twytc.size())) ||
      (rc = up(d_twxtc, twxtc.data(), sizeof(float) * twxtc.size())) ||
      (rc = up(d_hy, hyt.data(), sizeof(int4) * hyt.size())) ||
      (rc = up(d_hyw, hywt.data(), pl->tcw_ok ? sizeof(int4) * hywt.size() : 0)) ||
      (rc = up(d_twt, tw_types.data(), sizeof(int) * tw_types.size())) ||
      (rc = up(pl->d_geom0, g0, sizeof(g0)))) {
    destroy(pl);
    return rc;
  }
  cudaError_t e = cudaMemset(a.hist, 0, sizeof(double) * a.num_bins);
  if (e == cudaSuccess) e = cudaMemset(a.nhist, 0, sizeof(double) * a.num_bins);
  if (e == cudaSuccess && a.iacc)
    e = cudaMemset(a.iacc, 0, sizeof(double) * a.nkz * a.nky * a.nkx);
  if (e == cudaSuccess) e = cudaMemset(d_status, 0, 4 * sizeof(int));
  if (e == cudaSuccess) e = cudaMallocHost(reinterpret_cast<void **>(&pl->ring.host),
                                           sizeof(float) * kRing * B * kGeom);
  for (int i = 0; e == cudaSuccess && i < kRing; ++i)
    e = cudaEventCreateWithFlags(&pl->ring.ev[i], cudaEventDisableTiming);
  // The dynamic shared-memory limit is per kernel function, not per plan, so
  // it is raised once to the largest value each kernel allows (the opt-in
  // per-block limit minus the kernel's static shared memory).
  if (e == cudaSuccess) e = raise_smem_limit(k_spread_zdft);
  if (e == cudaSuccess) e = raise_smem_limit(k_sort_atoms);
  if (e == cudaSuccess) e = raise_smem_limit(k_ydft);
  if (e == cudaSuccess) e = raise_smem_limit(k_xdft_post);
  if (e == cudaSuccess) e = raise_smem_limit(k_hist<float>);
  if (e == cudaSuccess) e = raise_smem_limit(k_hist<double>);
  if (e == cudaSuccess) e = raise_smem_limit(k_spread_zdft_tc);
  if (e == cudaSuccess) e = raise_smem_limit(k_spread_zdft_tcw);
  if (e == cudaSuccess) e = raise_smem_limit(k_spread_zdft_sparse);
  if (e == cudaSuccess) e = raise_smem_limit(k_spread_zdft_ag);
  if (e == cudaSuccess) e = raise_smem_limit(k_dft_tc<false>);
  if (e == cudaSuccess) e = raise_smem_limit(k_dft_tc<true>);
  // load the allocation-free forward's last kernel now (under lazy module
  // loading a kernel's code is loaded at its first use), so that call loads nothing
  if (e == cudaSuccess) {
    cudaFuncAttributes fa{};
    e = cudaFuncGetAttributes(&fa, k_flag_invalid);
  }
  if (e == cudaSuccess) {
    int per_sm = 0, sms = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_spread_zdft, kThreads,
                                                      pl->smem_spread);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, pl->device);
    pl->spread_ctas = std::max(1, per_sm) * std::max(1, sms);
    int sort_per_sm = 0;
    if (e == cudaSuccess)
      e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&sort_per_sm, k_sort_atoms, kSortThreads,
                                                        2 * sizeof(int) * a.tiles[0] * a.tiles[1]);
    pl->sort_slots = std::max(1, sort_per_sm) * std::max(1, sms);
    // the largest cluster size with at least one schedulable cluster at this
    // plan's shared-memory size
    for (int c = kSortMaxCluster; e == cudaSuccess && c >= 1; c /= 2) {
      cudaLaunchConfig_t occ = {};
      occ.gridDim = dim3(c);
      occ.blockDim = dim3(kSortThreads);
      occ.dynamicSmemBytes = 2 * sizeof(int) * a.tiles[0] * a.tiles[1];
      cudaLaunchAttribute cat[1];
      cat[0].id = cudaLaunchAttributeClusterDimension;
      cat[0].val.clusterDim.x = c;
      cat[0].val.clusterDim.y = 1;
      cat[0].val.clusterDim.z = 1;
      occ.attrs = cat;
      occ.numAttrs = 1;
      int nclusters = 0;
      if (cudaOccupancyMaxActiveClusters(&nclusters, k_sort_atoms, &occ) == cudaSuccess && nclusters > 0) {
        pl->sort_cluster = c;
        break;
      }
      cudaGetLastError();  // a size the device cannot schedule is not an error of the plan
    }
    if (e == cudaSuccess && pl->tcw_ok) pl->tcw_ctas = std::max(1, sms);  // 512 TMEM columns: one per SM
    if (e == cudaSuccess && pl->ag_ok) pl->ag_ctas = std::max(1, sms);    // its shared memory: one per SM
    if (e == cudaSuccess && pl->tcn_ok) {
      // resident CTAs whose tensor-memory allocations fit the SM's 512 columns together
      int tc_per_sm = 0;
      e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&tc_per_sm, k_spread_zdft_tc, kTcThreads,
                                                        pl->smem_spread_tc);
      tc_per_sm = std::min(std::max(1, tc_per_sm), 512 / a.tcCols);
      pl->tc_ctas = tc_per_sm * std::max(1, sms);
    }
    if (e == cudaSuccess && pl->use_ytc) {
      int per = 0;
      e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_dft_tc<false>, dtc_threads<false>(),
                                                        pl->smem_ydft_tc);
      per = std::min(std::max(1, per), 512 / pl->yshape.cols);
      pl->ytc_ctas = per * std::max(1, sms);
    }
    if (e == cudaSuccess && pl->use_xtc) {
      int per = 0;
      e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_dft_tc<true>, dtc_threads<true>(),
                                                        pl->smem_xdft_tc);
      per = std::min(std::max(1, per), 512 / pl->xshape.cols);
      pl->xtc_ctas = per * std::max(1, sms);
    }
  }
  if (e != cudaSuccess) {
    destroy(pl);
    return fail(SAXS_E_CUDA, std::string("plan setup: ") + cudaGetErrorString(e));
  }
  *out = pl;
  return SAXS_OK;
}

int launch_check(const char *what) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(SAXS_E_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
  return SAXS_OK;
}

cudaEvent_t pooled_event(SaxsPlan *pl) {
  if (!pl->event_pool.empty()) {
    cudaEvent_t e = pl->event_pool.back();
    pl->event_pool.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  cudaEventCreate(&e);
  return e;
}

// Records CUDA events around one stage when profiling is on.
struct StageTimer {
  SaxsPlan *pl;
  StageRecord *rec;
  cudaStream_t st;
  void begin(int k) {
    if (!rec) return;
    rec->start[k] = pooled_event(pl);
    rec->stop[k] = pooled_event(pl);
    rec->used[k] = true;
    cudaEventRecord(rec->start[k], st);
  }
  void end(int k) {
    if (rec) cudaEventRecord(rec->stop[k], st);
  }
};

// Launch with programmatic stream serialization (see pdl_wait).
template <typename... KArgs, typename... Args>
int launch_pdl(const char *name, void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st,
               Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  static const bool off = [] {
    const char *v = std::getenv("PYCUSAXS_PDL");  // PYCUSAXS_PDL=0: plain launches
    return v && std::strcmp(v, "0") == 0;
  }();
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = off ? 0 : 1;
  const cudaError_t e = cudaLaunchKernelEx(&cfg, kernel, static_cast<KArgs>(args)...);
  if (e != cudaSuccess) return fail(SAXS_E_CUDA, std::string(name) + ": " + cudaGetErrorString(e));
  return launch_check(name);
}

// Counting sort of `nframes` frames' atoms into home-bin order (the first kernel
// of a batch: launched without programmatic serialization).  The cluster size C
// is the smallest power of two, at least 4, for which the largest type's slice
// (max_type / C entries) is no more than an even share of the launch's entries
// over the device's resident CTAs, capped at kSortMaxCluster.
int launch_sort(const SaxsPlan *pl, const DevArgs &a, int nframes, cudaStream_t st,
                const float *host_geom = nullptr) {
  static_assert(sizeof(DevArgs) + sizeof(SortGeom) + 2 * sizeof(int) <= 32764, "kernel parameter space");
  SortGeom gp{};
  const int step = host_geom ? kSortParamFrames : nframes;
  for (int f0 = 0; f0 < nframes; f0 += step) {
    const int n = std::min(step, nframes - f0);
    if (host_geom) std::memcpy(gp.g, host_geom + static_cast<size_t>(f0) * kGeom, sizeof(float) * n * kGeom);
    // at least 4 (measured slightly faster than 2 at 100 frames of 100k atoms),
    // at most what the device can schedule at this shared-memory size
    int C = std::min(4, pl->sort_cluster);
    const long long total = static_cast<long long>(a.M) * n;
    while (C < pl->sort_cluster &&
           static_cast<long long>(pl->sort_max_type) * pl->sort_slots > static_cast<long long>(C) * total)
      C *= 2;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(a.T * C, n);
    cfg.blockDim = dim3(kSortThreads);
    cfg.dynamicSmemBytes = 2 * sizeof(int) * a.tiles[0] * a.tiles[1];
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = C;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    const cudaError_t e = cudaLaunchKernelEx(&cfg, k_sort_atoms, a, gp, host_geom ? 1 : 0, f0);
    if (e != cudaSuccess) return fail(SAXS_E_CUDA, std::string("k_sort_atoms: ") + cudaGetErrorString(e));
    if (int rc = launch_check("k_sort_atoms")) return rc;
  }
  return SAXS_OK;
}

// Spreading + z-axis DFT of `nframes` frames: the wide-tile or 64-column
// tensor-core kernel the plan is configured for, else the FP32 SIMT kernel.
int launch_spread(const SaxsPlan *pl, const DevArgs &a, int nframes, cudaStream_t st) {
  if (pl->use_tc && pl->use_ag) {
    const int items = a.stiles[0] * a.stw * a.T * nframes;
    return launch_pdl("k_spread_zdft_ag", k_spread_zdft_ag, dim3(std::max(1, std::min(items, pl->ag_ctas))),
                      dim3(kAgThreads), pl->smem_spread_ag, st, a, items);
  }
  if (pl->use_tc && pl->use_tcw) {
    // the dense types' items on the wide kernel, the sparse types' on the direct one
    const int items = a.stiles[0] * a.stw * a.tw_nd * nframes;
    if (items > 0)
      if (int rc = launch_pdl("k_spread_zdft_tcw", k_spread_zdft_tcw,
                              dim3(std::max(1, std::min(items, pl->tcw_ctas))), dim3(kTwThreads),
                              pl->smem_spread_tcw, st, a, items))
        return rc;
    const int sitems = a.stiles[0] * a.stw * a.tw_ns * nframes;
    if (sitems > 0)
      return launch_pdl("k_spread_zdft_sparse", k_spread_zdft_sparse, dim3(sitems), dim3(kSpThreads),
                        pl->smem_sparse, st, a);
    return SAXS_OK;
  }
  const int items = a.stiles[0] * a.stiles[1] * a.T * nframes;
  if (pl->use_tc) {
    return launch_pdl("k_spread_zdft_tc", k_spread_zdft_tc, dim3(std::max(1, std::min(items, pl->tc_ctas))),
                      dim3(kTcThreads), pl->smem_spread_tc, st, a, items);
  }
  return launch_pdl("k_spread_zdft", k_spread_zdft, dim3(std::max(1, std::min(items, pl->spread_ctas))),
                    dim3(kThreads), pl->smem_spread, st, a, items);
}

// cuTensorMapEncodeTiled, fetched from the driver once (no link to libcuda).
using EncodeTiledFn = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                   const cuuint64_t *, const cuuint32_t *, const cuuint32_t *,
                                   CUtensorMapInterleave, CUtensorMapSwizzle, CUtensorMapL2promotion,
                                   CUtensorMapFloatOOBfill);

EncodeTiledFn encode_tiled() {
  static EncodeTiledFn fn = [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess) {
      cudaGetLastError();
      p = nullptr;
    }
    return reinterpret_cast<EncodeTiledFn>(p);
  }();
  return fn;
}

// Float32 tiled tensor map over `base` (128-byte swizzle, zero fill outside).
int encode_map(CUtensorMap *m, const void *base, int rank, const cuuint64_t *dims, const cuuint64_t *strides,
               const cuuint32_t *box) {
  EncodeTiledFn fn = encode_tiled();
  if (!fn) return fail(SAXS_E_CUDA, "cuTensorMapEncodeTiled is not available from the driver");
  const cuuint32_t estr[5] = {1, 1, 1, 1, 1};
  const CUresult r = fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, static_cast<cuuint32_t>(rank), const_cast<void *>(base),
                        dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                        CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return fail(SAXS_E_CUDA, "tensor map encoding failed (" + std::to_string(r) + ")");
  return SAXS_OK;
}

// y-axis DFT of `planes` z-transformed planes: the tensor-core kernel when the
// plan has it, else the FP32 SIMT kernel.
int launch_ydft(const SaxsPlan *pl, const DevArgs &a, int planes, cudaStream_t st) {
  if (pl->use_ytc) {
    const int items = planes * ((a.ext[0] + 127) / 128);
    // Z[plane][x][y] as {2*ey floats, x, plane}
    const cuuint64_t ex = a.ext[0], ey = a.ext[1];
    const cuuint64_t dims[3] = {2 * ey, ex, static_cast<cuuint64_t>(planes)};
    const cuuint64_t strides[2] = {8 * ey, 8 * ey * ex};
    const cuuint32_t box[3] = {2 * kDtcChunk, 128, 1};
    CUtensorMap map;
    if (int rc = encode_map(&map, a.Z, 3, dims, strides, box)) return rc;
    return launch_pdl("k_dft_tc<y>", k_dft_tc<false>, dim3(std::max(1, std::min(items, pl->ytc_ctas))),
                      dim3(dtc_threads<false>()), pl->smem_ydft_tc, st, a, pl->yshape, map, items);
  }
  dim3 gy((a.ext[0] + kYRows - 1) / kYRows, a.nkz, planes / a.nkz);
  return launch_pdl("k_ydft", k_ydft, gy, dim3(kThreads), pl->smem_ydft, st, a);
}

// x-axis DFT, form factors, type sum and moduli of `nframes` frames into ibox:
// the tensor-core kernel when the plan has it, else the FP32 SIMT kernel.
int launch_xdft(const SaxsPlan *pl, const DevArgs &a, int nframes, cudaStream_t st) {
  if (pl->use_xtc) {
    const int kyb = a.xtcKyb;
    const int items = nframes * a.nkz * ((a.nky + kyb - 1) / kyb);
    // Y[f][t][kz][ky][x] as {2*ex floats, t, ky, kz, f}
    const cuuint64_t ex = a.ext[0];
    const cuuint64_t dims[5] = {2 * ex, static_cast<cuuint64_t>(a.T), static_cast<cuuint64_t>(a.nky),
                                static_cast<cuuint64_t>(a.nkz), static_cast<cuuint64_t>(nframes)};
    const cuuint64_t row = 8 * ex;
    const cuuint64_t strides[4] = {row * a.nky * a.nkz, row, row * a.nky, row * a.nky * a.nkz * a.T};
    const cuuint32_t box[5] = {2 * kDtcChunk, static_cast<cuuint32_t>(a.T), static_cast<cuuint32_t>(kyb), 1, 1};
    CUtensorMap map;
    if (int rc = encode_map(&map, a.Y, 5, dims, strides, box)) return rc;
    return launch_pdl("k_dft_tc<x>", k_dft_tc<true>, dim3(std::max(1, std::min(items, pl->xtc_ctas))),
                      dim3(dtc_threads<true>()), pl->smem_xdft_tc, st, a, pl->xshape, map, items);
  }
  dim3 gx((a.nky + kXRows - 1) / kXRows, a.nkz, nframes);
  return launch_pdl("k_xdft_post", k_xdft_post, gx, dim3(kThreads), pl->smem_xdft, st, a, pl->xc);
}

// Enqueue the memsets and kernels of one batch of `nframes` frames whose
// geometry is already in (or queued for) a.geom.  Host work free, so that it can
// be captured in a CUDA graph.
int enqueue_batch(SaxsPlan *pl, const DevArgs &a, int nframes, cudaStream_t st, bool timed,
                  const float *host_geom = nullptr) {
  StageTimer tm{pl, nullptr, st};
  if (timed && pl->profiling) {
    pl->prof_pending.emplace_back();
    tm.rec = &pl->prof_pending.back();
  }
  {
    tm.begin(kStSort);
    const int rc = launch_sort(pl, a, nframes, st, host_geom);
    tm.end(kStSort);
    if (rc) return rc;
  }
  {
    tm.begin(kStSpread);
    const int rc = launch_spread(pl, a, nframes, st);
    tm.end(kStSpread);
    if (rc) return rc;
  }
  {
    tm.begin(kStYdft);
    const int rc = launch_ydft(pl, a, nframes * a.T * a.nkz, st);
    tm.end(kStYdft);
    if (rc) return rc;
  }
  {
    tm.begin(kStXdft);
    const int rc = launch_xdft(pl, a, nframes, st);
    tm.end(kStXdft);
    if (rc) return rc;
  }
  tm.begin(kStHist);
  if (pl->ensemble == SAXS_NPT) {
    dim3 gh(a.nkz, nframes);
    if (int rc = launch_pdl("k_hist", k_hist<float>, gh, dim3(kThreads), pl->smem_hist, st, a, a.ibox, a.geom,
                            kGeom, 1.0, a.hist, a.nhist))
      return rc;
  } else {
    const int64_t npl = static_cast<int64_t>(a.nkz) * a.nky * a.nkx;
    k_accumulate<<<static_cast<unsigned>((npl + kThreads - 1) / kThreads), kThreads, 0, st>>>(a, nframes);
  }
  tm.end(kStHist);
  if (int rc = launch_check("k_hist")) return rc;
  return SAXS_OK;
}

// Widen the plan's k-box in place to half-widths of at least `need` (plus 5%
// headroom): a new plan with the same parameters and atoms, the kernel
// configuration kept where the new plan can run it, the accumulators, status
// words, frame count and pending profile records carried over; the caller's
// SaxsPlan pointer stays valid.  Waits for `st`.  Refused for plans whose
// buffers a graph holds.
int regrow(SaxsPlan *pl, const long long need[3], cudaStream_t st) {
  if (pl->graph_refs > 0)
    return fail(SAXS_E_RANGE, "a frame's box grew beyond the planned k-box margin and the plan is "
                              "captured in a graph, whose buffers cannot move; create the plan with a "
                              "larger box_margin");
  CUDA_TRY(cudaStreamSynchronize(st));
  SaxsParams p = pl->p;
  p.form_factors = pl->ff.data();
  p.entry_atom = pl->ea_host.data();
  p.entry_type = pl->et_host.data();
  p.padding_values = pl->pad.empty() ? nullptr : pl->pad.data();
  long long minh[3];
  for (int d = 0; d < 3; ++d) minh[d] = std::max(pl->half[d], need[d] + need[d] / 20 + 1);
  SaxsPlan *np = nullptr;
  if (int rc = create(&p, &np, minh)) return rc;
  const DevArgs &o = pl->a;
  DevArgs &n = np->a;
  int rc = SAXS_OK;
  auto cuda = [&](cudaError_t e, const char *what) {
    if (e != cudaSuccess && rc == SAXS_OK) rc = fail(SAXS_E_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
  };
  // accumulators: Delta-q, q-cut and the bins depend on the first box only, so
  // the histograms carry over as they are; an nvt intensity sum moves into the
  // matching k-points of the wider box
  cuda(cudaMemcpyAsync(n.hist, o.hist, sizeof(double) * o.num_bins, cudaMemcpyDeviceToDevice, st), "regrow");
  cuda(cudaMemcpyAsync(n.nhist, o.nhist, sizeof(double) * o.num_bins, cudaMemcpyDeviceToDevice, st), "regrow");
  cuda(cudaMemcpyAsync(n.status, o.status, sizeof(int) * kStatusWords, cudaMemcpyDeviceToDevice, st), "regrow");
  if (o.iacc && rc == SAXS_OK) {
    std::vector<double> src(static_cast<size_t>(o.nkz) * o.nky * o.nkx);
    std::vector<double> dst(static_cast<size_t>(n.nkz) * n.nky * n.nkx, 0.0);
    cuda(cudaMemcpy(src.data(), o.iacc, sizeof(double) * src.size(), cudaMemcpyDeviceToHost), "regrow");
    const int dx = o.kx_lo - n.kx_lo, dy = o.ky_lo - n.ky_lo;
    for (int kz = 0; kz < o.nkz; ++kz)
      for (int ky = 0; ky < o.nky; ++ky)
        for (int kx = 0; kx < o.nkx; ++kx)
          dst[(static_cast<size_t>(kz) * n.nky + ky + dy) * n.nkx + kx + dx] =
              src[(static_cast<size_t>(kz) * o.nky + ky) * o.nkx + kx];
    cuda(cudaMemcpy(n.iacc, dst.data(), sizeof(double) * dst.size(), cudaMemcpyHostToDevice), "regrow");
  }
  cuda(cudaStreamSynchronize(st), "regrow");
  if (rc != SAXS_OK) {
    destroy(np);
    return rc;
  }
  // the kernel configuration in use (an autotuned choice), where it still fits
  if ((!pl->use_tc || (pl->use_ag ? np->ag_ok : pl->use_tcw ? np->tcw_ok : np->tcn_ok)) &&
      (!pl->use_ytc || np->ytc_ok) && (!pl->use_xtc || np->xtc_ok)) {
    np->use_tc = pl->use_tc;
    np->use_ag = pl->use_ag;
    np->use_tcw = pl->use_tcw;
    np->use_ytc = pl->use_ytc;
    np->use_xtc = pl->use_xtc;
    if (np->use_tc && np->use_tcw && pl->a.twG <= np->twG_max) set_wide_groups(np, pl->a.twG);
    if (np->use_tc && !np->use_tcw && np->a.tcS == 2) np->a.tcG = pl->a.tcG;
  }
  np->frames = pl->frames;
  np->profiling = pl->profiling;
  np->prof_pending.swap(pl->prof_pending);
  np->event_pool.swap(pl->event_pool);
  std::swap(*pl, *np);
  destroy(np);  // the old buffers
  return SAXS_OK;
}

// Check the boxes of `nframes` frames against the plan's k-box; when one needs
// a larger k-box, widen the plan (`grow`) or return SAXS_E_RANGE.
int fit_kbox(SaxsPlan *pl, const float *boxes, int nframes, cudaStream_t st, bool grow) {
  long long need[3] = {0, 0, 0};
  bool over = false;
  for (int f = 0; f < nframes; ++f) {
    const float *box = boxes + 9 * f;
    if (int rc = check_box(box)) return rc;
    float g[kGeom];
    frame_geometry(pl, box, g);
    long long h[3];
    saxs::kbox_halfwidths(g + 9, pl->a.qcut, 1e-5, h);
    for (int d = 0; d < 3; ++d) {
      need[d] = std::max(need[d], h[d]);
      over |= !pl->full_axis[d] && h[d] > pl->half[d];
    }
  }
  if (!over) return SAXS_OK;
  if (!grow)
    return fail(SAXS_E_RANGE, "a frame's box grew beyond the planned k-box margin; create the plan "
                              "with a larger box_margin, or use saxs_forward, which widens the plan");
  return regrow(pl, need, st);
}

int forward(SaxsPlan *pl, const float *xyz, int64_t stride, int nframes, const float *boxes,
            cudaStream_t st) {
  if (!pl) return fail(SAXS_E_INVALID, "null plan");
  if (nframes < 1 || nframes > pl->p.max_frames)
    return fail(SAXS_E_INVALID, "nframes must be in [1, max_frames]");
  if (!boxes || (!xyz && pl->a.M > 0)) return fail(SAXS_E_INVALID, "null positions or boxes");
  if (stride < 3ll * pl->p.natoms) return fail(SAXS_E_INVALID, "frame stride smaller than 3*natoms");
  if (int rc = fit_kbox(pl, boxes, nframes, st, true)) return rc;
  DevArgs a = pl->a;
  a.xyz = xyz;
  a.frame_stride = stride;
  // geometry of each frame, checked against the planned k-box
  Ring &ring = pl->ring;
  const int slot = ring.next;
  ring.next = (ring.next + 1) % kRing;
  CUDA_TRY(cudaEventSynchronize(ring.ev[slot]));
  float *g = ring.host + static_cast<size_t>(slot) * pl->p.max_frames * kGeom;
  for (int f = 0; f < nframes; ++f) frame_geometry(pl, boxes + 9 * f, g + f * kGeom);
  // the geometry travels as k_sort_atoms' kernel parameters
  if (int rc = enqueue_batch(pl, a, nframes, st, true, g)) return rc;
  pl->frames += nframes;
  pl->last_frame_batch = nframes;
  return SAXS_OK;
}

}  // namespace

struct SaxsGraph {
  std::vector<SaxsPlan *> plans;
  std::vector<DevArgs> args;
  std::vector<int> nframes;
  std::vector<int> offset;  // first frame of each plan in the geometry slots
  int total = 0;
  int device = 0;
  float *pinned[2] = {nullptr, nullptr};
  cudaGraphExec_t exec[2] = {nullptr, nullptr};
  cudaEvent_t done[2] = {nullptr, nullptr};
  int next = 0;
  bool holds_plans = false;  // the plans' graph_refs count this graph
};

namespace {

void graph_destroy(SaxsGraph *g) {
  if (!g) return;
  if (g->holds_plans)
    for (SaxsPlan *pl : g->plans) --pl->graph_refs;
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(g->device);
  for (int k = 0; k < 2; ++k) {
    if (g->done[k]) {
      cudaEventSynchronize(g->done[k]);
      cudaEventDestroy(g->done[k]);
    }
    if (g->exec[k]) cudaGraphExecDestroy(g->exec[k]);
    if (g->pinned[k]) cudaFreeHost(g->pinned[k]);
  }
  cudaSetDevice(prev);
  delete g;
}

int graph_create(SaxsPlan *const *plans, const float *const *xyz, const int64_t *stride,
                 const int *nframes, int count, SaxsGraph **out) {
  if (!plans || !xyz || !stride || !nframes || !out || count < 1)
    return fail(SAXS_E_INVALID, "null argument or empty plan list");
  *out = nullptr;
  SaxsGraph *g = new SaxsGraph();
  g->device = plans[0] ? plans[0]->device : 0;
  for (int i = 0; i < count; ++i) {
    SaxsPlan *pl = plans[i];
    if (!pl) {
      graph_destroy(g);
      return fail(SAXS_E_INVALID, "null plan in the list");
    }
    for (int k = 0; k < i; ++k)
      if (plans[k] == pl) {
        graph_destroy(g);
        return fail(SAXS_E_INVALID, "a plan appears twice in one graph");
      }
    if (pl->device != g->device) {
      graph_destroy(g);
      return fail(SAXS_E_INVALID, "all plans of a graph must be on one device");
    }
    if (nframes[i] < 1 || nframes[i] > pl->p.max_frames || stride[i] < 3ll * pl->p.natoms ||
        (!xyz[i] && pl->a.M > 0)) {
      graph_destroy(g);
      return fail(SAXS_E_INVALID, "bad frame count, stride or positions for plan " + std::to_string(i));
    }
    DevArgs a = pl->a;
    a.xyz = xyz[i];
    a.frame_stride = stride[i];
    g->plans.push_back(pl);
    g->args.push_back(a);
    g->nframes.push_back(nframes[i]);
    g->offset.push_back(g->total);
    g->total += nframes[i];
  }
  cudaStream_t origin = nullptr;
  std::vector<cudaStream_t> br(count, nullptr);
  std::vector<cudaEvent_t> fork(count, nullptr), join(count, nullptr);
  cudaError_t e = cudaStreamCreateWithFlags(&origin, cudaStreamNonBlocking);
  for (int i = 0; e == cudaSuccess && i < count; ++i) {
    e = cudaStreamCreateWithFlags(&br[i], cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&fork[i], cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&join[i], cudaEventDisableTiming);
  }
  int rc = SAXS_OK;
  for (int k = 0; e == cudaSuccess && rc == SAXS_OK && k < 2; ++k) {
    e = cudaMallocHost(reinterpret_cast<void **>(&g->pinned[k]), sizeof(float) * g->total * kGeom);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&g->done[k], cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaStreamBeginCapture(origin, cudaStreamCaptureModeThreadLocal);
    for (int i = 0; e == cudaSuccess && rc == SAXS_OK && i < count; ++i) {
      const DevArgs &a = g->args[i];
      e = cudaEventRecord(fork[i], origin);
      if (e == cudaSuccess) e = cudaStreamWaitEvent(br[i], fork[i], 0);
      if (e == cudaSuccess)
        e = cudaMemcpyAsync(const_cast<float *>(a.geom), g->pinned[k] + g->offset[i] * kGeom,
                            sizeof(float) * g->nframes[i] * kGeom, cudaMemcpyHostToDevice, br[i]);
      if (e == cudaSuccess) rc = enqueue_batch(g->plans[i], a, g->nframes[i], br[i], false);
      if (e == cudaSuccess && rc == SAXS_OK) e = cudaEventRecord(join[i], br[i]);
      if (e == cudaSuccess && rc == SAXS_OK) e = cudaStreamWaitEvent(origin, join[i], 0);
    }
    cudaGraph_t graph = nullptr;
    const cudaError_t ee = cudaStreamEndCapture(origin, &graph);
    if (e == cudaSuccess) e = ee;
    if (e == cudaSuccess && rc == SAXS_OK) e = cudaGraphInstantiate(&g->exec[k], graph, 0);
    if (graph) cudaGraphDestroy(graph);
  }
  for (int i = 0; i < count; ++i) {
    if (br[i]) cudaStreamDestroy(br[i]);
    if (fork[i]) cudaEventDestroy(fork[i]);
    if (join[i]) cudaEventDestroy(join[i]);
  }
  if (origin) cudaStreamDestroy(origin);
  if (e != cudaSuccess || rc != SAXS_OK) {
    graph_destroy(g);
    if (rc != SAXS_OK) return rc;
    cudaGetLastError();
    return fail(SAXS_E_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
  }
  for (SaxsPlan *pl : g->plans) ++pl->graph_refs;  // their buffers may no longer move
  g->holds_plans = true;
  *out = g;
  return SAXS_OK;
}

int graph_launch(SaxsGraph *g, const float *boxes, cudaStream_t st) {
  if (!g || !boxes) return fail(SAXS_E_INVALID, "null argument");
  const int slot = g->next;
  g->next ^= 1;
  CUDA_TRY(cudaEventSynchronize(g->done[slot]));
  for (size_t i = 0; i < g->plans.size(); ++i) {
    SaxsPlan *pl = g->plans[i];
    for (int f = 0; f < g->nframes[i]; ++f) {
      const int k = g->offset[i] + f;
      const float *box = boxes + 9 * k;
      if (int rc = check_box(box)) return rc;
      float *geo = g->pinned[slot] + static_cast<size_t>(k) * kGeom;
      frame_geometry(pl, box, geo);
      long long h[3];
      saxs::kbox_halfwidths(geo + 9, pl->a.qcut, 1e-5, h);
      for (int d = 0; d < 3; ++d)
        if (!pl->full_axis[d] && h[d] > pl->half[d])
          return fail(SAXS_E_RANGE, "a frame's box grew beyond the planned k-box margin of plan " +
                                        std::to_string(i) + "; a graph's buffers cannot move: create "
                                        "the plan with a larger box_margin");
    }
  }
  CUDA_TRY(cudaGraphLaunch(g->exec[slot], st));
  CUDA_TRY(cudaEventRecord(g->done[slot], st));
  for (size_t i = 0; i < g->plans.size(); ++i) {
    g->plans[i]->frames += g->nframes[i];
    g->plans[i]->last_frame_batch = g->nframes[i];
  }
  return SAXS_OK;
}

// The message of a non-zero status word (kStatus* bits).
std::string status_message(int bits) {
  std::string who;
  auto add = [&](const char *name) {
    if (!who.empty()) who += "; ";
    who += name;
  };
  if (bits & kStatusInput) add("k_sort_atoms: a position was NaN or infinite (placed at the cell origin)");
  if (bits & kStatusZ) add("the spreading + z-axis DFT kernel (k_spread_zdft_tcw / k_spread_zdft_tc): a bounded wait gave up");
  if (bits & kStatusY) add("the y-axis DFT kernel (k_dft_tc<y>): a bounded wait gave up");
  if (bits & kStatusX) add("the x-axis DFT kernel (k_dft_tc<x>): a bounded wait gave up");
  if (bits & kStatusProbe) add("the bounded-wait probe (k_wait_probe) gave up, as asked");
  return who + "; the frames processed since then are invalid (saxs_reset clears this error)";
}

int histogram(SaxsPlan *pl, double *hist, double *nhist, cudaStream_t st) {
  if (!pl || !hist || !nhist) return fail(SAXS_E_INVALID, "null argument");
  const DevArgs &a = pl->a;
  const size_t nb = static_cast<size_t>(a.num_bins);
  if (pl->ensemble == SAXS_NVT) {
    double *th = pl->d_tmp_hist, *tn = pl->d_tmp_hist + nb;
    CUDA_TRY(cudaMemsetAsync(th, 0, 2 * nb * sizeof(double), st));
    if (pl->frames > 0) {
      const float fact = static_cast<float>(1.0 / static_cast<float>(pl->frames));
      dim3 gh(a.nkz, 1);
      k_hist<double><<<gh, kThreads, pl->smem_hist, st>>>(a, a.iacc, pl->d_geom0, kGeom,
                                                          static_cast<double>(fact), th, tn);
      if (int rc = launch_check("k_hist(nvt)")) return rc;
    }
    CUDA_TRY(cudaMemcpyAsync(hist, th, nb * sizeof(double), cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaMemcpyAsync(nhist, tn, nb * sizeof(double), cudaMemcpyDeviceToHost, st));
  } else {
    CUDA_TRY(cudaMemcpyAsync(hist, a.hist, nb * sizeof(double), cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaMemcpyAsync(nhist, a.nhist, nb * sizeof(double), cudaMemcpyDeviceToHost, st));
  }
  int status = 0;
  CUDA_TRY(cudaMemcpyAsync(&status, a.status, sizeof(int), cudaMemcpyDeviceToHost, st));
  CUDA_TRY(cudaStreamSynchronize(st));
  if (status != 0) return fail(SAXS_E_DEVICE, status_message(status));
  return SAXS_OK;
}


// The accumulated histogram into device buffers, enqueued on `st` without a
// wait: npt copies the FP64 accumulators, nvt bins the intensity sum with the
// first frame's box.  The status word is left for saxs_histogram /
// saxs_debug_counters to report.
int histogram_device(SaxsPlan *pl, double *hist, double *nhist, cudaStream_t st) {
  if (!pl || !hist || !nhist) return fail(SAXS_E_INVALID, "null argument");
  const DevArgs &a = pl->a;
  const size_t nb = static_cast<size_t>(a.num_bins);
  if (pl->ensemble == SAXS_NVT) {
    CUDA_TRY(cudaMemsetAsync(hist, 0, nb * sizeof(double), st));
    CUDA_TRY(cudaMemsetAsync(nhist, 0, nb * sizeof(double), st));
    if (pl->frames > 0) {
      const float fact = static_cast<float>(1.0 / static_cast<float>(pl->frames));
      k_hist<double><<<dim3(a.nkz, 1), kThreads, pl->smem_hist, st>>>(a, a.iacc, pl->d_geom0, kGeom,
                                                                     static_cast<double>(fact), hist, nhist);
      if (int rc = launch_check("k_hist(nvt)")) return rc;
    }
  } else {
    CUDA_TRY(cudaMemcpyAsync(hist, a.hist, nb * sizeof(double), cudaMemcpyDeviceToDevice, st));
    CUDA_TRY(cudaMemcpyAsync(nhist, a.nhist, nb * sizeof(double), cudaMemcpyDeviceToDevice, st));
  }
  return SAXS_OK;
}

int ensure_adjoint(SaxsPlan *pl) {
  if (pl->d_adj_G) return SAXS_OK;
  const DevArgs &a = pl->a;
  const int ex = a.ext[0], ey = a.ext[1], ez = a.ext[2];
  pl->adj_eyp = round_up(ey, 16);
  pl->adj_ezp = round_up(ez, 8);
  int rc;
  if ((rc = dalloc(pl, &pl->d_adj_dl, a.num_bins)) ||
      (rc = dalloc(pl, &pl->d_adj_S, a.T)) ||
      (rc = dalloc(pl, &pl->d_adj_dcg, a.T)) ||
      (rc = dalloc(pl, &pl->d_adj_G, static_cast<size_t>(a.T) * a.nkz * a.nky * a.nkx)) ||
      (rc = dalloc(pl, &pl->d_adj_twyT, static_cast<size_t>(a.nky) * pl->adj_eyp)) ||
      (rc = dalloc(pl, &pl->d_adj_twzT, static_cast<size_t>(a.nkz) * pl->adj_ezp)))
    return rc;
  std::vector<float2> ty(static_cast<size_t>(a.nky) * pl->adj_eyp, make_float2(0.f, 0.f));
  for (int k = 0; k < a.nky; ++k)
    for (int y = 0; y < ey; ++y)
      saxs::twiddle(a.ky_lo + k, y, a.nn[1], &ty[k * pl->adj_eyp + y].x, &ty[k * pl->adj_eyp + y].y);
  std::vector<float2> tz(static_cast<size_t>(a.nkz) * pl->adj_ezp, make_float2(0.f, 0.f));
  for (int k = 0; k < a.nkz; ++k)
    for (int z = 0; z < ez; ++z)
      saxs::twiddle(k, z, a.nn[2], &tz[k * pl->adj_ezp + z].x, &tz[k * pl->adj_ezp + z].y);
  CUDA_TRY(cudaMemcpy(pl->d_adj_twyT, ty.data(), sizeof(float2) * ty.size(), cudaMemcpyHostToDevice));
  CUDA_TRY(cudaMemcpy(pl->d_adj_twzT, tz.data(), sizeof(float2) * tz.size(), cudaMemcpyHostToDevice));
  const size_t optin = static_cast<size_t>(optin_smem());
  pl->smem_yadj = (static_cast<size_t>(a.nky) * 64 + static_cast<size_t>(a.nky) * pl->adj_eyp) *
                  sizeof(float2);
  pl->smem_zadj = (static_cast<size_t>(a.nkz) * pl->adj_ezp + static_cast<size_t>(a.nkz) * kCols) *
                      sizeof(float2) + static_cast<size_t>(ez) * kCols * sizeof(float);
  pl->adj_tiled_y = pl->smem_yadj + static_smem(k_yadj_tile) <= optin;
  pl->adj_tiled_z = pl->smem_zadj + static_smem(k_zadj_gather) <= optin;
  CUDA_TRY(raise_smem_limit(k_xdft_grad));
  if (pl->adj_tiled_y) CUDA_TRY(raise_smem_limit(k_yadj_tile));
  if (pl->adj_tiled_z) {
    CUDA_TRY(raise_smem_limit(k_zadj_gather));
    int per_sm = 0, sms = 0;
    CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_zadj_gather, kThreads,
                                                           pl->smem_zadj));
    CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, pl->device));
    pl->zadj_ctas = std::max(1, per_sm) * std::max(1, sms);
  } else {
    if ((rc = dalloc(pl, &pl->d_adj_dg, static_cast<size_t>(a.T) * ex * ey * ez))) return rc;
  }
  return SAXS_OK;
}

int backward(SaxsPlan *pl, const float *xyz, const float *box, const double *dl, float *grad,
             cudaStream_t st, bool dl_on_device) {
  if (!pl || !box || !dl || !grad || (!xyz && pl->a.M > 0)) return fail(SAXS_E_INVALID, "null argument");
  if (int rc = fit_kbox(pl, box, 1, st, true)) return rc;
  if (int rc = ensure_adjoint(pl)) return rc;
  DevArgs a = pl->a;
  a.xyz = xyz;
  a.frame_stride = 3ll * pl->p.natoms;
  AdjArgs j{};
  j.dl = pl->d_adj_dl;
  j.G = pl->d_adj_G;
  j.H1 = a.Y;  // Y is consumed by k_xdft_grad before k_xadj overwrites it
  j.H2 = a.Z;  // Z is consumed by k_ydft before the y adjoint overwrites it
  j.twyT = pl->d_adj_twyT;
  j.twzT = pl->d_adj_twzT;
  j.eyp = pl->adj_eyp;
  j.ezp = pl->adj_ezp;
  j.dg = pl->d_adj_dg;
  j.S = pl->d_adj_S;
  j.dcg = pl->d_adj_dcg;
  j.grad = grad;
  // geometry of the frame through the pinned ring, checked against the k-box
  Ring &ring = pl->ring;
  const int slot = ring.next;
  ring.next = (ring.next + 1) % kRing;
  CUDA_TRY(cudaEventSynchronize(ring.ev[slot]));
  float *g = ring.host + static_cast<size_t>(slot) * pl->p.max_frames * kGeom;
  frame_geometry(pl, box, g);
  CUDA_TRY(cudaMemcpyAsync(const_cast<float *>(a.geom), g, sizeof(float) * kGeom,
                           cudaMemcpyHostToDevice, st));
  CUDA_TRY(cudaEventRecord(ring.ev[slot], st));
  CUDA_TRY(cudaMemcpyAsync(pl->d_adj_dl, dl, sizeof(double) * a.num_bins,
                           dl_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, st));
  CUDA_TRY(cudaMemsetAsync(pl->d_adj_S, 0, sizeof(double) * a.T, st));
  CUDA_TRY(cudaMemsetAsync(grad, 0, sizeof(float) * 3 * static_cast<size_t>(pl->p.natoms), st));
  // recompute the frame's y-transformed planes (nothing is kept from the forward)
  if (int rc = launch_sort(pl, a, 1, st)) return rc;
  if (int rc = launch_spread(pl, a, 1, st)) return rc;
  if (int rc = launch_ydft(pl, a, a.T * a.nkz, st)) return rc;
  const int items = a.stiles[0] * a.stiles[1] * a.T;  // 8 x 8 column tiles of the z adjoint
  // adjoint passes
  dim3 gx((a.nky + kXRows - 1) / kXRows, a.nkz, 1);
  k_xdft_grad<<<gx, kThreads, pl->smem_xdft, st>>>(a, j, pl->xc);
  const int64_t n1 = static_cast<int64_t>(a.T) * a.nkz * a.nky * a.ext[0];
  k_xadj<<<static_cast<unsigned>((n1 + kThreads - 1) / kThreads), kThreads, 0, st>>>(a, j);
  if (pl->adj_tiled_y) {
    dim3 gya((a.ext[0] + 63) / 64, a.nkz, a.T);
    k_yadj_tile<<<gya, kThreads, pl->smem_yadj, st>>>(a, j);
  } else {
    const int64_t n2 = static_cast<int64_t>(a.T) * a.nkz * a.ext[0] * a.ext[1];
    k_yadj<<<static_cast<unsigned>((n2 + kThreads - 1) / kThreads), kThreads, 0, st>>>(a, j);
  }
  if (pl->adj_tiled_z) {
    k_zadj_gather<<<std::max(1, std::min(items, pl->zadj_ctas)), kThreads, pl->smem_zadj, st>>>(
        a, j, items);
  } else {
    const int64_t n3 = static_cast<int64_t>(a.T) * a.ext[0] * a.ext[1] * a.ext[2];
    k_zadj<<<static_cast<unsigned>((n3 + kThreads - 1) / kThreads), kThreads, 0, st>>>(a, j);
    k_sum_dg<<<dim3(64, a.T), kThreads, 0, st>>>(a, j);
    if (a.M > 0) k_gather<<<(a.M + kThreads - 1) / kThreads, kThreads, 0, st>>>(a, j);
  }
  if (pl->adj_tiled_z && a.M > 0)
    k_mean_grad<<<(a.M + kThreads - 1) / kThreads, kThreads, 0, st>>>(a, j);
  return launch_check("backward");
}

}  // namespace

// ---------------------------------------------------------------------------
// single frame into caller scratch (used by the allocation-free entry point)
// ---------------------------------------------------------------------------
namespace saxs {

namespace {

// Byte offsets of the per-frame buffers inside one scratch block.
struct ScratchLayout {
  size_t status, geom, key, offsets, rec, border, Z, Y, ibox, total;
};

ScratchLayout scratch_layout(const DevArgs &a) {
  auto up = [](size_t v) { return (v + 255) / 256 * 256; };
  ScratchLayout L{};
  size_t o = 0;
  L.status = o;
  o = up(o + sizeof(int) * kStatusWords);
  L.geom = o;
  o = up(o + sizeof(float) * kGeom);
  L.key = o;
  o = up(o + sizeof(int2) * static_cast<size_t>(a.M));
  L.offsets = o;
  o = up(o + sizeof(int) * (static_cast<size_t>(a.nbins) + 1));
  L.rec = o;
  o = up(o + sizeof(float4) * static_cast<size_t>(a.M));
  L.border = o;
  o = up(o + sizeof(double) * static_cast<size_t>(a.T));
  L.Z = o;
  o = up(o + sizeof(float2) * static_cast<size_t>(a.T) * a.nkz * a.ext[0] * a.ext[1]);
  L.Y = o;
  o = up(o + sizeof(float2) * static_cast<size_t>(a.T) * a.nkz * a.nky * a.ext[0]);
  L.ibox = o;
  o = up(o + sizeof(float) * static_cast<size_t>(a.nkz) * a.nky * a.nkx);
  L.total = o;
  return L;
}

}  // namespace

int plan_device(const SaxsPlan *plan) { return plan->device; }

size_t single_frame_scratch_bytes(const SaxsPlan *plan) { return scratch_layout(plan->a).total; }

int record_error(int code, const char *msg) { return fail(code, msg); }

void clear_error() { g_err.clear(); }

int forward_into_scratch(SaxsPlan *pl, const float *xyz, const float *box, unsigned char *scratch,
                         size_t scratch_bytes, double *hist, double *nhist, cudaStream_t st) {
  if (!pl || !box || !scratch || !hist || !nhist || (!xyz && pl->a.M > 0))
    return fail(SAXS_E_INVALID, "null argument");
  // widening the k-box would allocate: a box beyond the margin is refused
  if (int rc = fit_kbox(pl, box, 1, st, false)) return rc;
  DevArgs a = pl->a;
  const ScratchLayout L = scratch_layout(a);
  if (L.total > scratch_bytes) return fail(SAXS_E_RANGE, "scratch too small for this plan");
  a.xyz = xyz;
  a.frame_stride = 3ll * pl->p.natoms;
  a.geom = reinterpret_cast<const float *>(scratch + L.geom);
  a.key = reinterpret_cast<int2 *>(scratch + L.key);
  a.offsets = reinterpret_cast<int *>(scratch + L.offsets);
  a.rec = reinterpret_cast<float4 *>(scratch + L.rec);
  a.border = reinterpret_cast<double *>(scratch + L.border);
  a.Z = reinterpret_cast<float2 *>(scratch + L.Z);
  a.Y = reinterpret_cast<float2 *>(scratch + L.Y);
  a.ibox = reinterpret_cast<float *>(scratch + L.ibox);
  a.hist = hist;
  a.nhist = nhist;
  // the frame's own status words: the plan's are left alone, and a frame whose
  // kernels report an error gets a NaN histogram (k_flag_invalid)
  a.status = reinterpret_cast<int *>(scratch + L.status);
  // frame geometry, checked against the k-box, staged through the plan's pinned ring
  Ring &ring = pl->ring;
  const int slot = ring.next;
  ring.next = (ring.next + 1) % kRing;
  CUDA_TRY(cudaEventSynchronize(ring.ev[slot]));
  float *g = ring.host + static_cast<size_t>(slot) * pl->p.max_frames * kGeom;
  frame_geometry(pl, box, g);
  CUDA_TRY(cudaMemcpyAsync(const_cast<float *>(a.geom), g, sizeof(float) * kGeom,
                           cudaMemcpyHostToDevice, st));
  CUDA_TRY(cudaEventRecord(ring.ev[slot], st));
  // the block keeps the previous call's contents: clear what accumulates
  CUDA_TRY(cudaMemsetAsync(hist, 0, sizeof(double) * a.num_bins, st));
  CUDA_TRY(cudaMemsetAsync(nhist, 0, sizeof(double) * a.num_bins, st));
  CUDA_TRY(cudaMemsetAsync(a.status, 0, sizeof(int) * kStatusWords, st));
  if (int rc = launch_sort(pl, a, 1, st)) return rc;
  if (int rc = launch_spread(pl, a, 1, st)) return rc;
  if (int rc = launch_ydft(pl, a, a.T * a.nkz, st)) return rc;
  if (int rc = launch_xdft(pl, a, 1, st)) return rc;
  dim3 gh(a.nkz, 1);
  k_hist<float><<<gh, kThreads, pl->smem_hist, st>>>(a, a.ibox, a.geom, kGeom, 1.0, hist, nhist);
  if (int rc = launch_check("k_hist")) return rc;
  k_flag_invalid<<<1, kThreads, 0, st>>>(a.status, hist, nhist, a.num_bins);
  return launch_check("k_flag_invalid");
}

}  // namespace saxs

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
extern "C" {

int saxs_plan_create(const SaxsParams *params, SaxsPlan **plan) {
  g_err.clear();
  const int rc = create(params, plan);
  // look up the allocation-free entry point's scratch array now, while the
  // caller can afford a load of it onto the device (a failure is not the
  // plan's: that entry point tries again and reports it)
  if (rc == SAXS_OK && saxs::noalloc_attach((*plan)->device) != SAXS_OK) g_err.clear();
  return rc;
}

void saxs_plan_destroy(SaxsPlan *plan) { destroy(plan); }

int saxs_plan_info(const SaxsPlan *pl, SaxsPlanInfo *info) {
  if (!pl || !info) return fail(SAXS_E_INVALID, "null argument");
  const DevArgs &a = pl->a;
  for (int d = 0; d < 3; ++d) {
    info->grid[d] = a.n[d];
    info->scaled_grid[d] = a.nn[d];
  }
  info->bin_size = a.dq;
  info->qcut = a.qcut;
  info->num_bins = a.num_bins;
  info->kbox[0] = a.nkx;
  info->kbox[1] = a.nky;
  info->kbox[2] = a.nkz;
  info->kz_count = a.nkz;
  info->path = (pl->use_tc ? 1 : 0) | (pl->use_ytc ? 2 : 0) | (pl->use_xtc ? 4 : 0) |
               (pl->use_tc && !pl->use_ag && pl->use_tcw ? 8 : 0) | (pl->use_tc && pl->use_ag ? 16 : 0) |
               (pl->use_tc && !pl->use_ag && pl->use_tcw && pl->a.tw_ns > 0 ? 32 : 0);
  info->device_bytes = pl->bytes;
  info->frames_accumulated = pl->frames;
  return SAXS_OK;
}

int saxs_plan_config(const SaxsPlan *pl, SaxsPlanConfig *cfg) {
  if (!pl || !cfg) return fail(SAXS_E_INVALID, "null argument");
  cfg->z_tensor_cores = pl->use_tc ? 1 : 0;
  cfg->y_tensor_cores = pl->use_ytc ? 1 : 0;
  cfg->x_tensor_cores = pl->use_xtc ? 1 : 0;
  cfg->z_wide_tiles = pl->use_tc && pl->use_tcw ? 1 : 0;
  cfg->z_producer_groups = !pl->use_tc ? 1 : pl->use_tcw ? pl->a.twG : pl->a.tcG;
  cfg->z_tensor_cores_available = pl->tc_ok ? 1 : 0;
  cfg->y_tensor_cores_available = pl->ytc_ok ? 1 : 0;
  cfg->x_tensor_cores_available = pl->xtc_ok ? 1 : 0;
  cfg->z_narrow_tiles_available = pl->tcn_ok ? 1 : 0;
  cfg->z_wide_tiles_available = pl->tcw_ok ? 1 : 0;
  cfg->z_producer_groups_max = (pl->tcn_ok && pl->a.tcS == 2) ? 2 : 1;
  cfg->z_wide_producer_groups_max = pl->tcw_ok ? pl->twG_max : 1;
  cfg->z_atom_gemm = pl->use_tc && pl->use_ag ? 1 : 0;
  cfg->z_atom_gemm_available = pl->ag_ok ? 1 : 0;
  if (cfg->z_atom_gemm) {  // its tiles are the wide ones; it has no producer groups
    cfg->z_wide_tiles = 1;
    cfg->z_producer_groups = 1;
  }
  return SAXS_OK;
}

int saxs_plan_set_config(SaxsPlan *pl, const SaxsPlanConfig *cfg) {
  if (!pl || !cfg) return fail(SAXS_E_INVALID, "null argument");
  if (cfg->z_atom_gemm) {
    if (!pl->ag_ok || !cfg->z_tensor_cores)
      return fail(SAXS_E_INVALID, "the atom-GEMM spreading was requested but the plan cannot run it");
    if ((cfg->y_tensor_cores && !pl->ytc_ok) || (cfg->x_tensor_cores && !pl->xtc_ok))
      return fail(SAXS_E_INVALID, "a tensor-core pass the plan cannot run was requested");
    pl->use_tc = true;
    pl->use_ag = true;
    pl->use_ytc = cfg->y_tensor_cores != 0;
    pl->use_xtc = cfg->x_tensor_cores != 0;
    return SAXS_OK;
  }
  const bool z = cfg->z_tensor_cores != 0, wide = z && cfg->z_wide_tiles != 0;
  if ((z && !(wide ? pl->tcw_ok : pl->tcn_ok)) || (cfg->y_tensor_cores && !pl->ytc_ok) ||
      (cfg->x_tensor_cores && !pl->xtc_ok))
    return fail(SAXS_E_INVALID, "a tensor-core pass the plan cannot run was requested");
  const int gmax = !z ? 1 : wide ? pl->twG_max : (pl->a.tcS == 2 ? 2 : 1);
  if (cfg->z_producer_groups < 1 || cfg->z_producer_groups > gmax)
    return fail(SAXS_E_INVALID, "z_producer_groups must be 1.." + std::to_string(gmax));
  pl->use_tc = z;
  pl->use_tcw = wide;
  pl->use_ag = false;
  pl->use_ytc = cfg->y_tensor_cores != 0;
  pl->use_xtc = cfg->x_tensor_cores != 0;
  if (wide)
    set_wide_groups(pl, cfg->z_producer_groups);
  else if (z)
    pl->a.tcG = cfg->z_producer_groups;
  return SAXS_OK;
}

int saxs_forward(SaxsPlan *plan, const float *xyz_dev, int64_t frame_stride, int nframes,
                 const float *boxes_host, void *stream) {
  g_err.clear();
  int prev = 0;
  cudaGetDevice(&prev);
  if (plan && prev != plan->device) cudaSetDevice(plan->device);
  const int rc = forward(plan, xyz_dev, frame_stride, nframes, boxes_host,
                         static_cast<cudaStream_t>(stream));
  if (plan && prev != plan->device) cudaSetDevice(prev);
  return rc;
}

int saxs_histogram(SaxsPlan *plan, double *hist_host, double *nhist_host, void *stream) {
  g_err.clear();
  return histogram(plan, hist_host, nhist_host, static_cast<cudaStream_t>(stream));
}

int saxs_reset(SaxsPlan *pl, void *stream) {
  if (!pl) return fail(SAXS_E_INVALID, "null plan");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const DevArgs &a = pl->a;
  CUDA_TRY(cudaMemsetAsync(a.hist, 0, sizeof(double) * a.num_bins, st));
  CUDA_TRY(cudaMemsetAsync(a.nhist, 0, sizeof(double) * a.num_bins, st));
  if (a.iacc) CUDA_TRY(cudaMemsetAsync(a.iacc, 0, sizeof(double) * a.nkz * a.nky * a.nkx, st));
  CUDA_TRY(cudaMemsetAsync(a.status, 0, sizeof(int) * kStatusWords, st));
  pl->frames = 0;
  return SAXS_OK;
}

int saxs_debug_counters(SaxsPlan *pl, int *out, void *stream) {
  if (!pl || !out) return fail(SAXS_E_INVALID, "null argument");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  CUDA_TRY(cudaMemcpyAsync(out, pl->a.status, sizeof(int) * kStatusWords, cudaMemcpyDeviceToHost, st));
  CUDA_TRY(cudaStreamSynchronize(st));
  return SAXS_OK;
}

int saxs_debug_wait_probe(SaxsPlan *pl, double limit_seconds, void *stream) {
  g_err.clear();
  if (!pl) return fail(SAXS_E_INVALID, "null plan");
  if (!(limit_seconds > 0.0) || limit_seconds > 2.0)
    return fail(SAXS_E_INVALID, "the probe's wait limit must be in (0, 2] seconds");
  int prev = 0;
  cudaGetDevice(&prev);
  if (prev != pl->device) cudaSetDevice(pl->device);
  k_wait_probe<<<1, 32, 0, static_cast<cudaStream_t>(stream)>>>(
      pl->a.status, static_cast<unsigned long long>(limit_seconds * 1e9));
  const int rc = launch_check("k_wait_probe");
  if (prev != pl->device) cudaSetDevice(prev);
  return rc;
}

int saxs_debug_kbox_intensity(SaxsPlan *pl, float *out, void *stream) {
  if (!pl || !out) return fail(SAXS_E_INVALID, "null argument");
  if (pl->last_frame_batch < 1) return fail(SAXS_E_INVALID, "no frame processed yet");
  const DevArgs &a = pl->a;
  const size_t npl = static_cast<size_t>(a.nkz) * a.nky * a.nkx;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  CUDA_TRY(cudaMemcpyAsync(out, a.ibox + (pl->last_frame_batch - 1) * npl, npl * sizeof(float),
                           cudaMemcpyDeviceToHost, st));
  CUDA_TRY(cudaStreamSynchronize(st));
  return SAXS_OK;
}

int saxs_debug_border_sums(SaxsPlan *pl, double *out, void *stream) {
  if (!pl || !out) return fail(SAXS_E_INVALID, "null argument");
  if (pl->last_frame_batch < 1) return fail(SAXS_E_INVALID, "no frame processed yet");
  const DevArgs &a = pl->a;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  CUDA_TRY(cudaMemcpyAsync(out, a.border + static_cast<size_t>(pl->last_frame_batch - 1) * a.T,
                           a.T * sizeof(double), cudaMemcpyDeviceToHost, st));
  CUDA_TRY(cudaStreamSynchronize(st));
  return SAXS_OK;
}

int saxs_backward(SaxsPlan *plan, const float *xyz_dev, const float *box_host,
                  const double *dl_dprofile_host, float *grad_xyz_dev, void *stream) {
  g_err.clear();
  int prev = 0;
  cudaGetDevice(&prev);
  if (plan && prev != plan->device) cudaSetDevice(plan->device);
  const int rc = backward(plan, xyz_dev, box_host, dl_dprofile_host, grad_xyz_dev,
                          static_cast<cudaStream_t>(stream), false);
  if (plan && prev != plan->device) cudaSetDevice(prev);
  return rc;
}

int saxs_histogram_device(SaxsPlan *plan, double *hist_dev, double *nhist_dev, void *stream) {
  g_err.clear();
  int prev = 0;
  cudaGetDevice(&prev);
  if (plan && prev != plan->device) cudaSetDevice(plan->device);
  const int rc = histogram_device(plan, hist_dev, nhist_dev, static_cast<cudaStream_t>(stream));
  if (plan && prev != plan->device) cudaSetDevice(prev);
  return rc;
}

int saxs_backward_device(SaxsPlan *plan, const float *xyz_dev, const float *box_host,
                         const double *dl_dhist_dev, float *grad_xyz_dev, void *stream) {
  g_err.clear();
  int prev = 0;
  cudaGetDevice(&prev);
  if (plan && prev != plan->device) cudaSetDevice(plan->device);
  const int rc = backward(plan, xyz_dev, box_host, dl_dhist_dev, grad_xyz_dev,
                          static_cast<cudaStream_t>(stream), true);
  if (plan && prev != plan->device) cudaSetDevice(prev);
  return rc;
}

int saxs_graph_create(SaxsPlan *const *plans, const float *const *xyz_dev,
                      const int64_t *frame_stride, const int *nframes, int count, SaxsGraph **graph) {
  g_err.clear();
  int prev = 0;
  cudaGetDevice(&prev);
  const int dev = (plans && count > 0 && plans[0]) ? plans[0]->device : prev;
  if (prev != dev) cudaSetDevice(dev);
  const int rc = graph_create(plans, xyz_dev, frame_stride, nframes, count, graph);
  if (prev != dev) cudaSetDevice(prev);
  return rc;
}

int saxs_graph_launch(SaxsGraph *graph, const float *boxes_host, void *stream) {
  g_err.clear();
  int prev = 0;
  cudaGetDevice(&prev);
  if (graph && prev != graph->device) cudaSetDevice(graph->device);
  const int rc = graph_launch(graph, boxes_host, static_cast<cudaStream_t>(stream));
  if (graph && prev != graph->device) cudaSetDevice(prev);
  return rc;
}

void saxs_graph_destroy(SaxsGraph *graph) { graph_destroy(graph); }

int saxs_profile_stages(void) { return kStages; }

const char *saxs_profile_stage_name(int i) {
  return (i >= 0 && i < kStages) ? kStageNames[i] : "";
}

int saxs_profile_enable(SaxsPlan *pl, int enable) {
  if (!pl) return fail(SAXS_E_INVALID, "null plan");
  pl->profiling = enable != 0;
  return SAXS_OK;
}

int saxs_profile_read(SaxsPlan *pl, double *ms_out, int *launches_out) {
  if (!pl || !ms_out) return fail(SAXS_E_INVALID, "null argument");
  for (auto &r : pl->prof_pending) {
    for (int k = 0; k < kStages; ++k) {
      if (!r.used[k]) continue;
      CUDA_TRY(cudaEventSynchronize(r.stop[k]));
      float ms = 0.f;
      CUDA_TRY(cudaEventElapsedTime(&ms, r.start[k], r.stop[k]));
      ms_out[k] += ms;
      if (launches_out) launches_out[k] += 1;
      pl->event_pool.push_back(r.start[k]);
      pl->event_pool.push_back(r.stop[k]);
      r.start[k] = r.stop[k] = nullptr;
    }
  }
  pl->prof_pending.clear();
  return SAXS_OK;
}

int64_t saxs_closest_product(int n, float sigma) { return saxs::closest_product(n, sigma); }

int saxs_cell_oc(const float box[9], float oc_out[9]) {
  if (!box || !oc_out) return fail(SAXS_E_INVALID, "null argument");
  saxs::cell_oc(box, oc_out);
  return SAXS_OK;
}

int saxs_histogram_parameters(const int nn[3], const float oc[9], float sigma, float bin_size,
                              float qcut, float *bin_out, float *qcut_out, int *num_bins_out) {
  if (!nn || !oc || !bin_out || !qcut_out || !num_bins_out) return fail(SAXS_E_INVALID, "null argument");
  saxs::histogram_parameters(nn, oc, sigma, bin_size, qcut, bin_out, qcut_out, num_bins_out);
  return SAXS_OK;
}

int saxs_bspline_moduli(int n, int ndim, float *out) {
  if (n < 1 || !out) return fail(SAXS_E_INVALID, "bad argument");
  saxs::bspline_moduli(n, ndim, out);
  return SAXS_OK;
}

const char *saxs_last_error(void) { return g_err.c_str(); }

const char *saxs_version(void) { return "pycusaxs_b200 0.1 (sm_100a)"; }

}  // extern "C"

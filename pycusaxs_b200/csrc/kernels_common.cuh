// Part of the translation unit of plan.cu, which includes it inside its
// anonymous namespace; not a standalone header.
// Constants, the device argument block and device helpers of the forward and
// adjoint kernels.

constexpr int kTile = 8;                  // spread tile edge (columns per axis)
constexpr int kCols = kTile * kTile;      // columns per tile
constexpr int kThreads = 256;
constexpr int kGeom = 24;                 // floats of per-frame geometry: oc[9], ocs[9]
constexpr int kRing = 4;                  // pinned geometry slots in flight
constexpr int kKzThread = 6;              // kz outputs (complex) per thread in k_spread_zdft
constexpr int kKyGroup = 10;              // ky outputs per warp in k_ydft
constexpr int kKyPass = 8 * kKyGroup;     // ky outputs per pass (eight warps)
constexpr int kYChunk = 32;               // y values staged per step in k_ydft
constexpr int kYRows = 64;                // x rows per CTA in k_ydft
constexpr int kYStride = kYRows + 2;      // padded shared row (float2), 16-byte aligned
constexpr int kXRows = 4;                 // ky rows per CTA in k_xdft_post
constexpr int kHistSmemBins = 2048;       // bins held in shared memory by k_hist

// Bits of the status word (DevArgs::status[0]) a kernel sets when one of its
// bounded waits gives up; the work of that launch, and every result that
// depends on it, is then invalid.  status[1] holds the most atom-table chunks
// one item of the wide spreading kernel needed (a diagnostic, not an error).
constexpr int kStatusZ = 1;      // spreading + z-axis DFT (tensor-core kernels)
constexpr int kStatusY = 2;      // y-axis DFT (tensor-core kernel)
constexpr int kStatusX = 4;      // x-axis DFT + post (tensor-core kernel)
constexpr int kStatusProbe = 8;  // the bounded-wait probe (saxs_debug_wait_probe)
constexpr int kStatusInput = 16; // a position was NaN or infinite (k_sort_atoms)
constexpr int kStatusWords = 4;

thread_local std::string g_err;

int fail(int code, const std::string &msg) {
  g_err = msg;
  return code;
}

#define CUDA_TRY(x)                                                                   \
  do {                                                                                \
    cudaError_t e_ = (x);                                                             \
    if (e_ != cudaSuccess)                                                            \
      return fail(SAXS_E_CUDA, std::string(#x) + ": " + cudaGetErrorString(e_));      \
  } while (0)

inline int round_up(int v, int m) { return (v + m - 1) / m * m; }

// Everything a kernel needs, passed by value.
struct DevArgs {
  int n[3], nn[3], ext[3];
  int order, ntaps;
  int T, M;
  int tiles[2], stiles[2], nbins;
  int bin_w;  // home-bin width (columns) of the atom counting sort: 4, or 8 when 4 would
              // need more than four bins per spread tile and axis
  int kx_lo, nkx, ky_lo, nky, nkz, nkzp, nkxp, nkyp;
  int zc;  // z rows of twiddles k_spread_zdft holds in shared memory at once
  // tensor-core z-DFT (k_spread_zdft_tc): GEMM N, K, spread rows, stages, TMEM columns
  int tcN, tcK, tcR, tcS, tcCols, tcRB, tcCap;
  int tcG;  // producer groups of k_spread_zdft_tc (1, or 2 with two operand stages)
  // wide-tile variant (k_spread_zdft_tcw): tile row stride (floats), record buffer,
  // atom table entries, producer groups; y tiles of 16 rows
  int twN, twRS, twRB, twCap, twG, stw;
  // atom-GEMM variant (k_spread_zdft_ag): B' half width (N2 = 2 * agNB), atom
  // table entries, record buffer
  int agNB, agCap, agRB;
  int xtcKyb;  // tensor-core x-axis DFT: ky values per item (rows (ky, type), T per ky)
  int nf[3];
  int dz;
  float dq, qcut;
  int num_bins;
  double border_count;
  double nn3;
  int64_t frame_stride;
  const float *xyz;
  const int32_t *entry_atom;
  const int32_t *entry_type;
  const int *type_start;  // [T + 1]: entries are grouped by type, type t owns [type_start[t], type_start[t+1])
  const float *geom;
  const float2 *twz;  // [ez][nkzp], nkzp a multiple of kKzThread
  const float2 *twy;  // [ey][nkyp]
  const float2 *twx;  // [ex][nkxp]
  const float *modx, *mody, *modz;
  const float *ff;    // [T][9]
  const float *twz_sum; // [2*nkzp]: sum over z < ez of the z twiddles (re, im)
  const float *twz_tc;  // [2][tcK x tcN]: z twiddles as TF32 head / remainder, K-major
  const float *twz_tcw; // [tcK x 2*twN] f16 (wide tiles): head and remainder side by side
  const int4 *home_x; // per spread tile along x: home tiles whose atoms reach it (-1 padded)
  const int4 *home_y;
  const int4 *home_yw; // per 16-row y tile: up to eight home tiles (two int4, -1 padded)
  int2 *key;
  int *offsets;
  float4 *rec;
  double *border;
  const float *pad_val;  // [T] given padding densities (atoms per grid point); null: z-border mean
  float2 *Z;
  float2 *Y;
  float *ibox;
  double *hist, *nhist;
  double *iacc;
  int *status;
  // element types of the wide z kernel (tw_types[0, tw_nd)) and of the direct
  // kernel for types too sparse for a dense tile (tw_types[tw_nd, tw_nd + tw_ns));
  // tw_ns = 0: every type in the wide kernel, in order
  const int *tw_types;
  int tw_nd, tw_ns;
};

// ---------------------------------------------------------------------------
// device helpers
// ---------------------------------------------------------------------------

// Grid coordinate r = n * frac(oc_row . x), written as the reference writes it
// (saxsDeviceKernels.cu:355-361) so that nvcc evaluates it the same way.
__device__ __forceinline__ float grid_coord(const float *oc, float x0, float y0, float z0, int n) {
  float x1 = oc[0] * x0 + oc[1] * y0 + oc[2] * z0;
  return static_cast<float>(n * (x1 - rint(x1 - 0.5)));
}

// The same, with a result outside [0, n] - only a NaN or infinite position
// gives one - replaced by 0 and reported in `bad`.  Stencil indices are derived
// from these values by truncation, so they must stay inside the cell.
__device__ __forceinline__ float grid_coord_checked(const float *oc, float x0, float y0, float z0, int n,
                                                   bool &bad) {
  const float r = grid_coord(oc, x0, y0, z0, n);
  if (r >= 0.0f && r <= static_cast<float>(n)) return r;
  bad = true;
  return 0.0f;
}

// |q| of the k-point with signed indices (ia, ja, ka), in the reference's
// float32 form (saxsDeviceKernels.cu:85-92): the dot products in float, the
// 2*pi factor applied in double, then sqrtf of the sum of squares.
__device__ __forceinline__ float kpoint_q(const float *oc, int ia, int ja, int ka) {
  float mw1, mw2, mw3, mw;
  mw1 = oc[0] * ia + oc[1] * ja + oc[2] * ka;
  mw1 = 2.0 * M_PI * mw1;
  mw2 = oc[3] * ia + oc[4] * ja + oc[5] * ka;
  mw2 = 2.0 * M_PI * mw2;
  mw3 = oc[6] * ia + oc[7] * ja + oc[8] * ka;
  mw3 = 2.0 * M_PI * mw3;
  mw = sqrtf(mw1 * mw1 + mw2 * mw2 + mw3 * mw3);
  return mw;
}

// |q| of the same k-point in float arithmetic only (the 2*pi factor in float):
// within a few ulp of kpoint_q, for uses that tolerate that - the form factor's
// argument, and a cut-off test made slightly inclusive - where kpoint_q's three
// double-precision multiplies per point would dominate.
__device__ __forceinline__ float kpoint_q_f32(const float *oc, int ia, int ja, int ka) {
  const float tp = 6.28318530717958647692f;
  const float fa = static_cast<float>(ia), fb = static_cast<float>(ja), fc = static_cast<float>(ka);
  const float m1 = tp * (oc[0] * fa + oc[1] * fb + oc[2] * fc);
  const float m2 = tp * (oc[3] * fa + oc[4] * fb + oc[5] * fc);
  const float m3 = tp * (oc[6] * fa + oc[7] * fb + oc[8] * fc);
  return sqrtf(m1 * m1 + m2 * m2 + m3 * m3);
}

// Cubic (order-4) cardinal B-spline weights of the four taps at fractional
// offset u in [0, 1]: tap 0 is the farthest-left grid point.
__device__ __forceinline__ void cubic_weights(float u, float w[4]) {
  const float v = 1.0f - u;
  const float u2 = u * u, u3 = u2 * u;
  const float s = 1.0f / 6.0f;
  w[0] = v * v * v * s;
  w[1] = (3.0f * u3 - 6.0f * u2 + 4.0f) * s;
  w[2] = (-3.0f * u3 + 3.0f * u2 + 3.0f * u + 1.0f) * s;
  w[3] = u3 * s;
}

// Form factor sum_i a_i exp(-b_i s2) + c at s2 = (q/4pi)^2 (opsfact.cu:30-35).
__device__ __forceinline__ float form_factor(const float *c, float q2) {
  return c[0] * expf(-c[4] * q2) + c[1] * expf(-c[5] * q2) + c[2] * expf(-c[6] * q2) +
         c[3] * expf(-c[7] * q2) + c[8];
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ int signed_k(int k, int nn, int nf) { return k < nf ? k : k - nn; }

// Padding density of type t in frame f: the plan's given value, or the mean of
// the type's z-border planes (saxsKernel.cu:150-162).
__device__ __forceinline__ float padding_mean(const DevArgs &a, int f, int t) {
  return a.pad_val ? a.pad_val[t]
                   : static_cast<float>(a.border[static_cast<int64_t>(f) * a.T + t] / a.border_count);
}

// Programmatic dependent launch: the forward's kernels after the first are
// launched with programmatic stream serialization, so a kernel's grid may start
// while the previous one drains.  Each such kernel lets its own successor launch
// at once (every CTA is then resident, so the successor cannot starve it of
// SMs) and waits for its predecessor's completion and memory before it reads
// anything the predecessor wrote; only set-up that touches plan constants,
// shared and tensor memory runs before the wait.  Both are no-ops for kernels
// launched without the attribute.
__device__ __forceinline__ void pdl_release() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }


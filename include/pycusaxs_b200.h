/*
 * pycusaxs_b200 — C ABI of the B200-native per-frame SAXS path.
 *
 * The reference exposes this path only through its pybind11 module
 * (`pycusaxs_cuda.run`, cpp-src/pybind/cuda_bindings.cpp:172-196) which drives
 * RunSaxs::Run (cpp-src/Exec/RunSaxs.cu:94-271) and saxsKernel
 * (cpp-src/Saxs/saxsKernel.h:30-114).  This header is the plain-C boundary
 * underneath the new drop-in: plain pointers and sizes, status codes instead of
 * exceptions, caller-owned device buffers for per-frame data, an explicit CUDA
 * stream.  Each entry point names the reference code it replaces.
 *
 * Units follow the reference: positions and boxes in Angstrom, q in 1/Angstrom.
 * Arrays are row-major; boxes are 3x3 with the cell vectors as rows (the
 * MDAnalysis `triclinic_dimensions` layout, pycusaxs/topology.py:565-577).
 *
 * Every function returns SAXS_OK (0) or a negative SAXS_E* code; the message of
 * the last failure on the calling thread is available from saxs_last_error().
 */
#ifndef PYCUSAXS_B200_H
#define PYCUSAXS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define SAXS_OK 0
#define SAXS_E_INVALID (-1)   /* bad argument (the reference raises ValueError) */
#define SAXS_E_CUDA (-2)      /* CUDA runtime or driver failure */
#define SAXS_E_NOMEM (-3)     /* device allocation refused (saxsKernel.cu:301-314) */
#define SAXS_E_RANGE (-4)     /* a frame left the planned k-box or capacity */
#define SAXS_E_DEVICE (-5)    /* a kernel reported an error through the plan's status word:
                                 a bounded wait gave up, or a position was NaN/infinite;
                                 saxs_last_error() names the kernel, saxs_reset clears it */

/* ensembles (cpp-src/Exec/Options.cpp:16, cudaSAXS.cu:84-87) */
#define SAXS_NPT 0 /* one histogram per frame, summed over frames (saxsKernel.cu:190-196) */
#define SAXS_NVT 1 /* intensities summed over frames, binned once (saxsKernel.cu:184-189, 17-39) */

typedef struct SaxsPlan SaxsPlan;

/* Run parameters: the fields of CudaSaxsConfig (cpp-src/include/CudaSaxsInterface.h:10-28)
 * that reach the numerics, plus the topology's per-type atom lists. */
typedef struct SaxsParams {
  int grid[3];          /* nx, ny, nz                                              */
  int scaled_grid[3];   /* nnx, nny, nnz; all 0 = derive from scale_factor          */
  int order;            /* B-spline order 1..8 (only 4 is meaningful, as upstream)  */
  float scale_factor;   /* sigma                                                   */
  float bin_size;       /* requested Delta-q (1/A), reset upward (saxsKernel.cu:489-526) */
  float qcut;           /* requested q cut-off (1/A), reset downward                */
  int ensemble;         /* SAXS_NPT or SAXS_NVT                                    */
  int ntypes;           /* number of element types                                 */
  const float *form_factors; /* ntypes x 9 (a1..a4, b1..b4, c), host memory         */
  int natoms;           /* rows of the per-frame position array                    */
  int nentries;         /* length of entry_atom / entry_type (sum of type lists)   */
  const int32_t *entry_atom; /* host: position row spread by each entry            */
  const int32_t *entry_type; /* host: type index 0..ntypes-1 of each entry         */
  float box0[9];        /* first-frame box: fixes Delta-q, q-cut and the k-box     */
  int max_frames;       /* frames per saxs_forward call (batch capacity)           */
  float box_margin;     /* relative box growth the k-box covers (e.g. 0.05); a frame */
                        /* beyond it makes saxs_forward / saxs_backward widen the   */
                        /* plan (new buffers, same accumulators; waits for the      */
                        /* stream), saxs_graph_launch and saxs_forward_noalloc      */
                        /* return SAXS_E_RANGE                                      */
  /* Opt-in physics extensions (no counterpart in the reference's output; 0 keeps
   * the reference's behaviour):                                                  */
  int box_mode;         /* SAXS_BOX_PARITY: oc from the box's upper triangle       */
                        /* (Cell.cpp:111-126); SAXS_BOX_TRICLINIC: full H^-T, and   */
                        /* q from its transpose                                    */
  int padding_mode;     /* SAXS_PAD_AVERAGE: z-border mean per type per frame      */
                        /* (saxsKernel.cu:150-162); SAXS_PAD_GIVEN: padding_values  */
  const float *padding_values; /* [ntypes] atoms per grid point (given mode)      */
} SaxsParams;

#define SAXS_BOX_PARITY 0
#define SAXS_BOX_TRICLINIC 1
#define SAXS_PAD_AVERAGE 0
#define SAXS_PAD_GIVEN 1

/* Sizes derived at plan creation. */
typedef struct SaxsPlanInfo {
  int grid[3];
  int scaled_grid[3];   /* the supercell actually used                             */
  float bin_size;       /* effective Delta-q                                       */
  float qcut;           /* effective q cut-off                                     */
  int num_bins;         /* int(qcut/bin_size)+1 (saxsKernel.cu:247)                */
  int kbox[3];          /* k-points evaluated per axis (x, y: signed range; z: 0..)*/
  int kz_count;
  int path;             /* pruned separable DFT; bits 0, 1, 2: z-, y-, x-axis DFT   */
                        /* on tcgen05; a clear bit: that pass in FP32 SIMT; bit 3:  */
                        /* 128-column z tiles, bit 4: the atom-GEMM z pass, bit 5:  */
                        /* sparse element types on the direct SIMT z kernel         */
  size_t device_bytes;  /* device memory held by the plan                          */
  int frames_accumulated;
} SaxsPlanInfo;

/* Create a plan: grid sizing, Delta-q/q-cut reset, B-spline moduli, twiddle
 * tables, device buffers.  Replaces saxsKernel::{scaledCell,
 * resetHistogramParameters, createMemory, setcufftPlan}
 * (saxsKernel.cu:470-488, 489-526, 240-366; saxsKernel.h:55-58) and the setup
 * half of RunSaxs::Run (RunSaxs.cu:107-133).  The current CUDA device is used. */
int saxs_plan_create(const SaxsParams *params, SaxsPlan **plan);

/* Release every resource of the plan (saxsKernel::~saxsKernel, saxsKernel.cu:546-553). */
void saxs_plan_destroy(SaxsPlan *plan);

int saxs_plan_info(const SaxsPlan *plan, SaxsPlanInfo *info);

/* Kernel configuration of a plan, for tuning (no counterpart in the reference,
 * which has one fixed kernel sequence).  The plan picks the tensor-core passes
 * whose operands fit; an autotuner may time the alternatives on real frames and
 * set the fastest.  Graphs built by saxs_graph_create keep the configuration
 * they were captured with. */
typedef struct SaxsPlanConfig {
  int z_tensor_cores;     /* 1: spreading + z-axis DFT on tcgen05, 0: FP32 SIMT      */
  int y_tensor_cores;     /* 1: y-axis DFT on tcgen05, 0: FP32 SIMT                   */
  int x_tensor_cores;     /* 1: x-axis DFT + post on tcgen05, 0: FP32 SIMT            */
  int z_wide_tiles;       /* with z_tensor_cores: 1 = 128-column tiles (A in tensor
                             memory), 0 = 64-column tiles                            */
  int z_producer_groups;  /* producer warp groups of the tensor-core spreading: 1|2  */
  /* read by saxs_plan_config only: what the plan can run */
  int z_tensor_cores_available, y_tensor_cores_available, x_tensor_cores_available;
  int z_narrow_tiles_available, z_wide_tiles_available;
  int z_producer_groups_max;       /* 64-column tiles  */
  int z_wide_producer_groups_max;  /* 128-column tiles */
  int z_atom_gemm;        /* 1: spreading + z-axis DFT as one tensor-core GEMM over the
                             atoms (128-column tiles, k_spread_zdft_ag); with it the
                             z_wide_tiles and z_producer_groups fields are not used   */
  int z_atom_gemm_available;  /* read by saxs_plan_config only                          */
} SaxsPlanConfig;

int saxs_plan_config(const SaxsPlan *plan, SaxsPlanConfig *cfg);
/* Select a configuration among those saxs_plan_config reports as available. */
int saxs_plan_set_config(SaxsPlan *plan, const SaxsPlanConfig *cfg);

/* Process `nframes` frames (<= max_frames).  Frame f's positions are
 * xyz_dev[f*frame_stride .. +3*natoms) (float32, device memory); its box is
 * boxes_host[9*f .. +9] (host memory).  npt: the frames' histograms are added
 * to the plan's FP64 accumulators; nvt: their intensities are added to the
 * plan's FP64 intensity sum.  Enqueued on `stream`; returns without waiting.
 * Replaces saxsKernel::runPKernel (saxsKernel.cu:59-209) and the per-frame body
 * of RunSaxs::Run (RunSaxs.cu:171-203). */
int saxs_forward(SaxsPlan *plan, const float *xyz_dev, int64_t frame_stride, int nframes,
                 const float *boxes_host, void *stream);

/* Finish the run: for nvt bin the summed intensities with the first-frame box
 * (saxsKernel::getHistogram, saxsKernel.cu:17-39); then copy the FP64
 * histogram and counts (num_bins each) to host memory and wait for them
 * (saxsKernel::getSaxs, saxsKernel.cu:210-225).  The accumulators are kept.
 * Returns SAXS_E_DEVICE when a kernel of a processed frame reported an error
 * (the histogram is then invalid; saxs_last_error() names the kernel). */
int saxs_histogram(SaxsPlan *plan, double *hist_host, double *nhist_host, void *stream);

/* Zero the accumulators and the status word so the plan can serve another run. */
int saxs_reset(SaxsPlan *plan, void *stream);

/* Intensities |sum_t f_t F_t|^2 * M of the last frame processed by
 * saxs_forward, over the plan's k-box (kz, ky, kx order, float32), for tests
 * and diagnostics.  `out_host` holds kbox[0]*kbox[1]*kz_count floats. */
int saxs_debug_kbox_intensity(SaxsPlan *plan, float *out_host, void *stream);

/* Per-type FP64 z-border sums of the last frame (saxsDeviceKernels.cu:446-465). */
int saxs_debug_border_sums(SaxsPlan *plan, double *out_host, void *stream);

/* Kernel diagnostics since plan creation or the last saxs_reset (no reference
 * counterpart; waits for `stream`): out_host[0] = the status word (0: no error;
 * bit 1: spreading/z pass, 2: y pass, 4: x pass gave up on a bounded wait,
 * 8: the wait probe below, 16: a NaN or infinite position), out_host[1] = the
 * most atom-table chunks one item of the wide spreading kernel needed (0: every
 * item's atoms fit its table at once), out_host[2..3] reserved (0). */
int saxs_debug_counters(SaxsPlan *plan, int *out_host, void *stream);

/* Run the bounded mbarrier wait that the pipelined kernels use, on a barrier
 * nothing arrives at, for `limit_seconds` (0 < limit <= 2): it gives up and sets
 * bit 8 of the plan's status word, so that the next saxs_histogram reports
 * SAXS_E_DEVICE; saxs_reset clears it.  Tests the device-side failure path
 * without faulting or hanging the GPU (no reference counterpart). */
int saxs_debug_wait_probe(SaxsPlan *plan, double limit_seconds, void *stream);

/* Reverse-mode derivative with respect to the positions of one frame.  Given
 * dL/dhist for each histogram bin of that frame (num_bins doubles, host memory;
 * the reported profile is hist/nhist, so dL/dhist = dL/dI(q) / nhist and 0 for
 * bins that are not reported), recompute the frame's transforms and write dL/dxyz
 * (3*natoms float32, device, overwritten) for positions xyz_dev with box
 * box_host.  The plan's accumulators are not touched; its intermediate buffers
 * are.  No reference counterpart: the reference has no derivative. */
int saxs_backward(SaxsPlan *plan, const float *xyz_dev, const float *box_host,
                  const double *dl_dhist_host, float *grad_xyz_dev, void *stream);

/* Device-resident forms for optimisation loops that must not wait for the host
 * (no reference counterpart).  saxs_histogram_device enqueues on `stream` the
 * accumulated FP64 histogram and counts into device buffers (num_bins each; nvt
 * bins the intensity sum first) and returns without waiting; a kernel error is
 * left in the status word for saxs_histogram / saxs_debug_counters to report.
 * saxs_backward_device is saxs_backward with dL/dhist read from device memory. */
int saxs_histogram_device(SaxsPlan *plan, double *hist_dev, double *nhist_dev, void *stream);
int saxs_backward_device(SaxsPlan *plan, const float *xyz_dev, const float *box_host,
                         const double *dl_dhist_dev, float *grad_xyz_dev, void *stream);

/* ---- batched form: many systems and frames per CUDA graph launch (no counterpart
 * in the reference, which processes one frame of one system per call) ---- */

typedef struct SaxsGraph SaxsGraph;

/* Capture the forwards of `count` distinct plans into one CUDA graph: plan i
 * processes nframes[i] (<= its max_frames) frames from xyz_dev[i] (device,
 * frame_stride[i] floats apart; the buffers are read at every launch), each
 * plan's kernels on its own graph branch so that small systems run side by
 * side.  Two executable copies alternate so the host can stage the next
 * launch's geometry while the previous one runs. */
int saxs_graph_create(SaxsPlan *const *plans, const float *const *xyz_dev,
                      const int64_t *frame_stride, const int *nframes, int count,
                      SaxsGraph **graph);

/* One launch: boxes_host holds one 3x3 box per frame, plans in order and frames
 * within a plan in order (sum of nframes boxes).  Each plan's accumulators grow
 * as with saxs_forward.  Enqueued on `stream`. */
int saxs_graph_launch(SaxsGraph *graph, const float *boxes_host, void *stream);

void saxs_graph_destroy(SaxsGraph *graph);

/* ---- allocation-free single frame (no counterpart in the reference) ----
 *
 * For hosts that cannot let the library allocate device memory while they run
 * (an MD engine or application that owns all device memory through its own
 * pool, or a per-step loop that must not stall on, or fail in, the allocator).
 * Runs one frame of `plan` - positions xyz_dev (natoms x 3 float32, device),
 * box box_host (3x3, host) - and writes that frame's histogram to hist_dev and
 * nhist_dev (num_bins doubles each, device; overwritten).  The plan's own
 * accumulators are left alone.  Every temporary comes from one fixed device
 * array of SAXS_NOALLOC_SCRATCH_BYTES held by every GPU that loads the library
 * until exit; plans needing more per frame get SAXS_E_RANGE.  Calls share that
 * array, so calls that overlap on the GPU must be serialised by the caller.
 * saxs_plan_create looks the array up (cudaGetSymbolAddress), which loads it
 * onto the plan's device; only if that failed does the first call look it up
 * (that call should then come before any stream capture).  cudaDeviceReset
 * invalidates plans and the cached address; plans created afterwards refresh
 * it.  The call is asynchronous: a kernel error of the frame (a bounded wait
 * that gave up, or NaN/infinite positions) makes hist_dev and nhist_dev NaN.
 * Allocates nothing; the plan is created, with allocation, beforehand by
 * saxs_plan_create. */
#define SAXS_NOALLOC_SCRATCH_BYTES ((size_t)32 << 20)
int saxs_forward_noalloc(SaxsPlan *plan, const float *xyz_dev, const float *box_host,
                         double *hist_dev, double *nhist_dev, void *stream);

/* ---- per-kernel timing (diagnostics; no reference counterpart: the reference
 * times only whole frames with one event pair, saxsKernel.cu:64-67,197-208) ---- */

/* Number of timed kernel stages and the name of stage i. */
int saxs_profile_stages(void);
const char *saxs_profile_stage_name(int i);

/* Enable (1) or disable (0) CUDA-event timing around every kernel that
 * saxs_forward launches, on the stream it launches on. */
int saxs_profile_enable(SaxsPlan *plan, int enable);

/* Wait for the timed work, then add each stage's milliseconds since the last
 * read into ms_out[0..saxs_profile_stages()), and its launch count into
 * launches_out (may be NULL).  Clears the pending records. */
int saxs_profile_read(SaxsPlan *plan, double *ms_out, int *launches_out);

/* ---- trajectory readers without MDAnalysis ----
 * The reference reads every frame through MDAnalysis (pycusaxs/topology.py:52-75
 * Universe(tpr, xtc), 536-577 read_frame/get_box, 621-737 iter_frames_stream),
 * converting GROMACS nanometres to Angstrom.  These read GROMACS TRR and XTC
 * and CHARMM/NAMD DCD files natively into caller buffers: positions (natoms x 3,
 * Angstrom) and the box as three row vectors (Angstrom; zeros when the file has
 * no box).  Errors go to saxs_last_error(). */
#define SAXS_TRAJ_AUTO 0 /* by file extension (.trr / .dcd / .xtc) */
#define SAXS_TRAJ_TRR 1
#define SAXS_TRAJ_DCD 2
#define SAXS_TRAJ_XTC 3 /* GROMACS compressed coordinates (xdr3dfcoord) */
typedef struct SaxsTraj SaxsTraj;

/* Open and index a trajectory (frame byte offsets, atom count). */
int saxs_traj_open(const char *path, int format, SaxsTraj **out);
int saxs_traj_info(const SaxsTraj *traj, int *natoms, long long *nframes);
/* Frame `frame` (0-based) into xyz[3*natoms], box[9]; time_ps may be NULL.
 * Reads use pread: concurrent calls on one handle (other frames) are safe. */
int saxs_traj_read(SaxsTraj *traj, long long frame, float *xyz, float *box, double *time_ps);
void saxs_traj_close(SaxsTraj *traj);

/* ---- setup numerics, exposed so that tests can pin them against the reference ---- */

/* Nearest 2^a 3^b 5^c 7^d to round(n*sigma), ties to the smaller
 * (saxsKernel::findClosestProduct, saxsKernel.cu:449-469). */
int64_t saxs_closest_product(int n, float sigma);

/* oc from the upper triangle of a 3x3 box (Cell::calculateMatrices, Cell.cpp:111-126). */
int saxs_cell_oc(const float box[9], float oc_out[9]);

/* Effective Delta-q, q-cut and bin count (saxsKernel.cu:489-526, :247). */
int saxs_histogram_parameters(const int nn[3], const float oc[9], float sigma, float bin_size,
                              float qcut, float *bin_out, float *qcut_out, int *num_bins_out);

/* Inverse B-spline moduli of one axis of length n (BSpmod, BSpmod.cpp:45-129). */
int saxs_bspline_moduli(int n, int ndim, float *out);

/* Message of the last failure on the calling thread ("" if none). */
const char *saxs_last_error(void);

/* Library version string. */
const char *saxs_version(void);

#ifdef __cplusplus
}
#endif

#endif /* PYCUSAXS_B200_H */

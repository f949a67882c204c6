/*
 * yrt_b200.h -- C ABI of the B200 (sm_100a) projection library libyrtb.so.
 *
 * Drop-in boundary for YRT-PET's projection hot path: list-mode and
 * histogram forward/back projectors (Siddon, multi-ray Siddon, distance-driven
 * with TOF and projection-space PSF), the sensitivity image and the OSEM
 * multiplicative update.  Plain pointers and sizes only; no C++ or torch types
 * cross this boundary and no exception escapes it.
 *
 * Conventions
 *  - Pointers named d_* are device pointers owned by the caller (ImageDevice
 *    buffers, torch tensors, cudaMalloc'd arrays).  Handles own only their
 *    internal tables (detector LUT, PSF taps, histogram maps).
 *  - Images are float32, frame-major [t][z][y][x] (the reference Image
 *    layout, include/yrt-pet/datastruct/image/Image.hpp).
 *  - Every call enqueues work on the given stream and returns without
 *    synchronising, except where stated.
 *  - Return value: YRTB_OK or an error code; yrtb_last_error() gives the
 *    message of the last failing call on the calling thread.
 *
 * Each entry point names the reference interface it replaces (paths inside
 * the yrt-pet project).
 */
#ifndef YRT_B200_H
#define YRT_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int yrtb_status;
#define YRTB_OK 0
#define YRTB_ERR_ARGUMENT 1     /* invalid argument (reference: ASSERT_MSG -> std::runtime_error) */
#define YRTB_ERR_CUDA 2         /* CUDA runtime error */
#define YRTB_ERR_RANGE 3        /* detector pair outside the histogram (reference: std::range_error) */
#define YRTB_ERR_EVENT 4        /* events with detector ids >= number of detectors were skipped */

typedef struct CUstream_st* yrtb_stream; /* cudaStream_t; NULL = legacy default stream */

/* Scanner description: the arguments of the reference Scanner constructor
 * (src/datastruct/scanner/Scanner.cpp:102-127). */
typedef struct
{
	float axial_fov, crystal_size_z, crystal_size_trans, crystal_depth,
	    scanner_radius;
	uint64_t dets_per_ring, num_rings, num_doi, max_ring_diff, min_ang_diff,
	    dets_per_block;
} yrtb_scanner;

/* Image grid: the reference ImageParams(nx, ny, nz, length_x, length_y,
 * length_z, off_x, off_y, off_z, nt) (src/datastruct/image/ImageParams.cpp:136-218).
 * Voxel size = length / n; FOV radius = max(lx, ly)/2 - max(vx, vy)/1000. */
typedef struct
{
	int64_t nx, ny, nz, nt;
	float length_x, length_y, length_z, off_x, off_y, off_z;
} yrtb_image_params;

#define YRTB_SIDDON 0
#define YRTB_DD 1

/* Arithmetic of the traversal. */
#define YRTB_MIRROR 0       /* FP32 in the reference's operation order (bit-exact voxel sequence) */
#define YRTB_COMPENSATED 1  /* FP64 entry-voxel placement, Kahan-compensated FP32 forward sums,
                               TOF Gaussian as a multiply by 1/sigma and the fast exponential */

/* Projector options: the reference ProjectorParams
 * (include/yrt-pet/operators/ProjectorParams.hpp:27-71) plus the PSF table
 * that ProjectionPsfManager reads from its CSV
 * (src/operators/ProjectionPsfManager.cpp:27-50). */
typedef struct
{
	int projector;          /* YRTB_SIDDON or YRTB_DD */
	int num_rays;           /* Siddon multi-ray count (>= 1) */
	float tof_fwhm_ps;      /* <= 0: no TOF */
	int tof_n_std;          /* truncation in sigmas (<= 0: none) */
	int psf_num_s;          /* projection-space PSF kernels (DD only); 0: no PSF */
	int psf_size;           /* taps per kernel (odd) */
	float psf_s_step, psf_k_spacing;
	const float* psf_taps;  /* host, psf_num_s * psf_size */
	int precision;          /* YRTB_MIRROR or YRTB_COMPENSATED */
	int deterministic;      /* 1: back projections (yrtb_backward, yrtb_em_step, the histogram
	                           kernels and everything built on them) run in two passes and
	                           accumulate in 64-bit fixed point, so their images are bit-identical
	                           whatever the order of events and atomics (the exact sum to within
	                           n * 2^-61 of n * max|v w| for n events); the projector then holds
	                           an 8-byte-per-voxel image (nx*ny*nz*nt).  No reference counterpart:
	                           the reference accumulates with float atomics (CPU atomic_ref,
	                           GPU atomicAdd) and is order dependent. */
} yrtb_projector_params;

/* Events (list-mode) in structure-of-arrays form, device pointers.  Either
 * (d1, d2) detector ids or lor (6 floats per event: p1 xyz, p2 xyz) must be
 * given; with lor, distance-driven and multi-ray projection also need orient
 * (6 floats per event: the two crystals' orientations n1 xyz, n2 xyz; the
 * reference's DET_ORIENT property).  All other arrays are optional (NULL):
 *   tof_ps        TOF value in ps (needs a TOF projector)
 *   frame         dynamic frame; events with frame < 0 are skipped, frames
 *                 >= nt are counted as invalid and skipped
 *   motion_frame  rigid-motion frame per event; motion: 12 floats per motion
 *                 frame in the reference's transform_t order (r00 r01 r02 tx
 *                 r10 r11 r12 ty r20 r21 r22 tz, include/yrt-pet/utils/Types.hpp:57),
 *                 applied
 *                 to both endpoints as in ProjectionData::getLOR
 *                 (src/datastruct/projection/ProjectionData.cpp:275-321);
 *                 a negative motion frame leaves the LOR unmoved;
 *                 num_motion_frames bounds the motion-frame index
 *   measurement   per-event measurement (histogram bins); 1 when NULL
 *   sens, att     multiplicative correction factors per event
 *   additive      randoms + scatter estimate per event */
typedef struct
{
	const uint32_t* d1;
	const uint32_t* d2;
	const float* lor;
	const float* tof_ps;
	const int32_t* frame;
	const int32_t* motion_frame;
	const float* motion;
	uint64_t num_motion_frames;
	const float* measurement;
	const float* sens;
	const float* att;
	const float* additive;
	uint64_t count;
	const float* orient;
} yrtb_events;

/* Events start + k*stride for k < count: one OSEM subset of the reference
 * BinIteratorChronologicalInterleaved (BinIterator.cpp:261-265) when
 * start = subset, stride = numSubsets.  count = 0 selects every event of the
 * subset. */
typedef struct
{
	uint64_t start, stride, count;
} yrtb_range;

typedef struct yrtb_projector yrtb_projector;

/* ---------------------------------------------------------------- misc --- */
const char* yrtb_last_error(void);
int yrtb_version(void);
/* Number of events skipped because of invalid detector ids since the last
 * call (synchronises the handle's error counter). */
yrtb_status yrtb_projector_take_event_errors(yrtb_projector* h,
                                             uint64_t* count);

/* ---------------------------------------------------- scanner geometry --- */
/* Regular detector LUT, out[d*6 + 0..5] = x, y, z, orient x, y, z.
 * Replaces DetRegular::generateLUT (src/datastruct/scanner/DetRegular.cpp:113-183);
 * host call, bit-identical to the reference. */
yrtb_status yrtb_scanner_regular_lut(const yrtb_scanner* scanner,
                                     float* out_host);

/* Histogram3D dimensions {numZBin, numPhi, numR}
 * (src/datastruct/projection/Histogram3D.cpp:165-203). */
yrtb_status yrtb_histo3d_dims(const yrtb_scanner* scanner, uint64_t* dims3);

/* ---------------------------------------------------------- projector --- */
/* Creates a projector for one scanner and image grid.  det_lut_host:
 * numDets*6 floats (positions, orientations) or NULL for the regular LUT.
 * Replaces OperatorProjectorDevice::create / util::createOperatorProjectorDevice
 * (include/yrt-pet/operators/OperatorProjectorDevice.cuh:27-31,
 * src/utils/ReconstructionUtilsDevice.cu:313). */
yrtb_status yrtb_projector_create(const yrtb_scanner* scanner,
                                  const float* det_lut_host,
                                  const yrtb_image_params* image,
                                  const yrtb_projector_params* params,
                                  yrtb_projector** out);
void yrtb_projector_destroy(yrtb_projector* h);

/* Launch configuration of the single-ray Siddon event kernels (yrtb_forward,
 * yrtb_backward, yrtb_em_step and the OSEM driver) and of the event ordering.
 * No reference counterpart: the reference launches one thread per event in
 * 256-thread blocks (GPUBatchSetup, include/yrt-pet/utils/GPUTypes.cuh:17-55)
 * on events in file order.  Default: {256, 1, 3, YRTB_ORDER_LOR, 1, 2}. */
#define YRTB_ORDER_LOR 0      /* inside a ray-length bucket: by LOR (Histogram3D bin), then TOF */
#define YRTB_ORDER_SPATIAL 1  /* inside a ray-length bucket: by direction sector (16 azimuthal x
                                 2 axial), then the Morton code of the TOF kernel centre (the
                                 LOR midpoint without TOF) on cells of tile_shift */
#define YRTB_ORDER_SPATIAL_FINE 2  /* as YRTB_ORDER_SPATIAL with 64 azimuthal sectors (and 128
                                      centre cells per axis instead of 256) */
typedef struct
{
	int block;            /* threads per block: 128 or 256 */
	int threads_per_lor;  /* single-ray Siddon: 1, 2 or 4 threads walk one LOR,
	                         each a piece cut at voxel planes, the forward sum
	                         reduced over the group; > 1 needs YRTB_COMPENSATED
	                         precision (the pieces' sums round differently from
	                         one walk).  Multi-ray Siddon: 1 (one thread walks
	                         the rays in turn) or the number of rays rounded up
	                         to a power of two, at most 8 (one lane per ray, the
	                         rays' forward sums added in ray order: the same
	                         bits as one thread; the default up to 8 rays).  Not
	                         used by deterministic back projections */
	int bucket_shift;     /* yrtb_events_subset_order groups rays by
	                         (voxel crossings >> bucket_shift), 0..7 */
	int order;            /* YRTB_ORDER_LOR, YRTB_ORDER_SPATIAL or YRTB_ORDER_SPATIAL_FINE */
	int tile_shift;       /* YRTB_ORDER_SPATIAL: cells of (voxel size * 2^tile_shift), 0..4 */
	int vector_groups;    /* bit 0: one-thread-per-LOR walks read the image as aligned
	                         float4 groups (consecutive x steps reuse the group held in
	                         registers); bit 1: they send the contributions to one group as a
	                         single red.global.add.v4.f32, summed in registers; bit 2: the
	                         same with the group staged in shared memory (wins over bit 1);
	                         bit 3: pairs of voxels sent as one red.global.add.v2.f32 (bits 1
	                         and 2 win over it).  Multi-ray walks use bits 1 and 3 (each ray's
	                         group or pair sent at the end of the ray; default 8 with one
	                         lane per ray, else 2).  Images must be
	                         16-byte aligned with a multiple of 4 voxels per frame, else
	                         scalar accesses are used */
} yrtb_launch_config;

yrtb_status yrtb_projector_set_launch(yrtb_projector* h,
                                      const yrtb_launch_config* cfg);
yrtb_status yrtb_projector_get_launch(const yrtb_projector* h,
                                      yrtb_launch_config* cfg);

/* Image layouts.  ROW_MAJOR is the reference's (x fastest, then y, z, frame).
 * TILE_4X2 stores each z plane as tiles of 4 x 2 voxels (x, y), 8 floats per
 * tile (one 32-byte sector: voxel (x, y) of a tile at (x & 1) + 2 (y & 1) +
 * 4 ((x >> 1) & 1)), tiles in row-major order inside the plane, planes and
 * frames as in ROW_MAJOR; it needs nx % 4 == 0 and ny % 2 == 0.  An aligned
 * group of 4 floats is then a 2 x 2 square, which a ray crosses in more
 * steps than 4 voxels of a row, so the walks send fewer L2 requests.  No
 * reference counterpart. */
#define YRTB_LAYOUT_ROW_MAJOR 0
#define YRTB_LAYOUT_TILE_4X2 1

/* Layout of the images given to this projector's list-mode projections
 * (yrtb_forward, yrtb_backward, yrtb_em_step, yrtb_em_step_model).  TILE_4X2
 * needs a single-ray Siddon projector without deterministic back projection
 * and image dimensions as above, and its walks run one thread per LOR
 * whatever threads_per_lor says; yrtb_osem_listmode then also walks tiles
 * internally (without an image-space PSF).  Every other call (histogram
 * mode, sensitivity images, attenuation images, the image-space PSF, the
 * OSEM drivers' arguments) takes ROW_MAJOR images whatever this setting.
 * On the C2 TOF workload TILE_4X2 sends 22 % fewer L2 requests but runs
 * 5 % slower (the parity bookkeeping adds instructions to an issue-bound
 * walk), so ROW_MAJOR is the default.  No reference counterpart. */
yrtb_status yrtb_projector_set_image_layout(yrtb_projector* h, int layout);
yrtb_status yrtb_projector_get_image_layout(const yrtb_projector* h, int* layout);

/* Converts nt frames of an image between layouts (d_src and d_dst distinct
 * device buffers of ip->nx * ny * nz * nt floats).  to_layout: the layout of
 * d_dst; d_src is in the other one.  No reference counterpart. */
yrtb_status yrtb_image_convert_layout(const float* d_src, float* d_dst,
                                      const yrtb_image_params* ip, int to_layout,
                                      yrtb_stream stream);

/* Temporaries of yrtb_events_subset_order, yrtb_attenuation_factors and
 * yrtb_autotune come from a stream-ordered memory pool per device that keeps
 * freed blocks for later calls (ordering 50M events holds about 3.6 GB).
 * This returns them to the CUDA driver (synchronises every device that has a
 * pool).  No reference counterpart. */
yrtb_status yrtb_release_cached_memory(void);

#define YRTB_TUNE_MAX 64

typedef struct
{
	yrtb_launch_config best;
	int num_tried;
	uint64_t sample_events;
	yrtb_launch_config tried[YRTB_TUNE_MAX];
	float ms[YRTB_TUNE_MAX];  /* best of 3 timed EM steps over the sample */
} yrtb_tune_report;

/* Autotuner (no reference counterpart).  Times the fused EM step of this
 * projector over a sample of the events -- subset 0 of num_subsets
 * interleaved subsets, at most max_sample events -- in two stages: first
 * 9 event orders (bucket_shift x order x tile_shift, the sample ordered
 * with each) x 5 vector_groups modes (2, 8, 4, 1, 0) with the current block
 * size and one thread per LOR (a multi-ray projector: modes 2, 8 and 0 with
 * its lanes per event), then every block size x threads per LOR the
 * projector admits on the fastest of those.
 * Keeps the fastest (yrtb_projector_set_launch) and reports all timings.  d_image: the image
 * the EM steps read (nx*ny*nz*nt floats; its values do not change the work).
 * Setup-time call: allocates temporaries and synchronises the stream, so it
 * must not run under stream capture.  Projectors other than Siddon
 * (single or multi-ray) keep the default configuration (num_tried = 0). */
yrtb_status yrtb_autotune(yrtb_projector* h, const float* d_image,
                          const yrtb_events* ev, int num_subsets,
                          uint64_t max_sample, yrtb_tune_report* report,
                          yrtb_stream stream);

/* Offsets drawn by the multi-ray Siddon projector for events k = 0..count-1
 * of a range: d_out[k*4*(num_rays-1) + 4*(ray-1) + {0..3}] = (i1, j1, i2, j2),
 * uniforms in [-0.5, 0.5) along z and across the crystal at each endpoint.
 * Same stream as the reference device path (curand XORWOW, seed 13,
 * subsequence = index in the batch; SiddonKernels.cuh:27-84).  For
 * validation against CPU re-computations of the same rays. */
yrtb_status yrtb_multiray_offsets(yrtb_projector* h, uint64_t count,
                                  float* d_out, yrtb_stream stream);

/* Builds (or grows to count item indices) a table of those offsets that the
 * projector keeps: multi-ray projections of a range then read item k's
 * offsets from it when k < count, instead of deriving the generator state
 * for subsequence k per event and per walk (the reference device path calls
 * curand_init per event, SiddonKernels.cuh:27-84).  Same values, so the same
 * projections.  Allocates count * 16 * (num_rays - 1) bytes and synchronises
 * the device when it grows; no-op for single-ray projectors or when the
 * table already covers count.  Without a table the generator is used. */
yrtb_status yrtb_multiray_table(yrtb_projector* h, uint64_t count,
                                yrtb_stream stream);

/* d_out[e] = (A x)_e for every event e of the range (entries of other events
 * untouched).  Replaces OperatorProjectorDevice::applyA
 * (src/operators/OperatorProjectorDevice.cu:442-544) with the kernels of
 * OperatorProjectorSiddon_GPU / _DD_GPU. */
yrtb_status yrtb_forward(yrtb_projector* h, const float* d_image,
                         const yrtb_events* ev, yrtb_range range,
                         float* d_out, yrtb_stream stream);

/* d_image += A^T v over the range (v = d_values[e]).  Replaces
 * OperatorProjectorDevice::applyAH (src/operators/OperatorProjectorDevice.cu:546-706). */
yrtb_status yrtb_backward(yrtb_projector* h, const float* d_values,
                          const yrtb_events* ev, yrtb_range range,
                          float* d_image, yrtb_stream stream);

/* One fused EM pass over the range: per event u = A x, corrections, ratio,
 * d_em += A^T u.  Replaces computeEMUpdateImage_kernel
 * (src/recon/OSEM_GPU.cu:1159-1341) and OSEM_CPU::computeEMUpdateImage
 * (src/recon/OSEM_CPU.cpp:284-393); corrections are applied in the CPU
 * order: *sens, *att, *global, +additive, |u| > denom_threshold. */
yrtb_status yrtb_em_step(yrtb_projector* h, const float* d_image,
                         float* d_em, const yrtb_events* ev,
                         yrtb_range range, float global_scale,
                         float denom_threshold, yrtb_stream stream);

/* yrtb_em_step that also writes each event's model value u (the corrected
 * forward projection, the EM ratio's denominator; 0 for a skipped event)
 * to d_model[e].  With unit measurements and no corrections the pass yields
 * the list-mode Poisson log-likelihood's terms log u_e and the back
 * projection A^T (1/u) of its gradient in one traversal per event, which the
 * reference computes as separate forward and back projections
 * (util::forwProject / util::backProject, src/utils/ReconstructionUtils.cpp:
 * 1005-1061). */
yrtb_status yrtb_em_step_model(yrtb_projector* h, const float* d_image,
                               float* d_em, const yrtb_events* ev,
                               yrtb_range range, float global_scale,
                               float denom_threshold, float* d_model,
                               yrtb_stream stream);

/* Number of voxel crossings (Siddon) or footprint voxels (DD) of every event
 * of the range, summed over rays: d_out[e] (uint32).  Used to count the
 * algorithmic traffic of a projection; no counterpart in the reference. */
yrtb_status yrtb_count_crossings(yrtb_projector* h, const yrtb_events* ev,
                                 yrtb_range range, uint32_t* d_out,
                                 yrtb_stream stream);

/* Diagnostics: the walk of every event of the range as the projector's
 * forward projection visits it, in visit order: for item k (k = 0 ..
 * count-1 of the range) at most cap (voxel offset within the event's
 * frame, weight) pairs at d_offsets / d_weights[k * cap ...], and the number
 * of visits (which may exceed cap) in d_counts[k].  Multi-ray walks list
 * their rays one after the other.  Offsets are row-major whatever the
 * projector's image layout.  Pins the voxel index sequence of the walks
 * against a CPU restatement; no counterpart in the reference. */
yrtb_status yrtb_trace_walks(yrtb_projector* h, const yrtb_events* ev,
                             yrtb_range range, uint32_t cap, int32_t* d_offsets,
                             float* d_weights, uint32_t* d_counts,
                             yrtb_stream stream);

/* Per-event attenuation factors exp(-0.1 * Siddon(mu-image)).  Replaces the
 * Corrector's ACF precompute (src/recon/Corrector.cpp:601-612,
 * include/yrt-pet/utils/Tools.hpp:98-102). */
yrtb_status yrtb_attenuation_factors(yrtb_projector* h, const float* d_mu,
                                     const yrtb_image_params* mu_params,
                                     const yrtb_events* ev, yrtb_range range,
                                     float* d_out, yrtb_stream stream);

/* Per-event gather of a Histogram3D through the detector pair (sensitivity,
 * randoms, scatter histograms).  invert != 0 replaces nonzero v by 1/v
 * (Corrector::getSensitivity, src/recon/Corrector.cpp:294-306).  Pairs that
 * map to no bin give 0 and are counted in the error counter. */
yrtb_status yrtb_gather_histo3d(yrtb_projector* h, const float* d_histo,
                                const yrtb_events* ev, yrtb_range range,
                                int invert, float* d_out, yrtb_stream stream);

/* Per-event LOR sensitivity from per-crystal factors: d_out[e] =
 * eff[d1] * eff[d2] (FP32), the value a sensitivity Histogram3D filled with
 * eff[d1] * eff[d2] gives through yrtb_gather_histo3d, without building the
 * histogram (1.44e9 bins, 5.8 GB on an 80-ring x 672-crystal scanner).  The
 * reference reads it per bin from its sensitivity histogram
 * (Corrector::getMultiplicativeCorrectionFactor,
 * src/recon/Corrector_CPU.cpp:17-45; Corrector.cpp:294-306).  Detector ids
 * outside the scanner give 0 and are counted in the error counter. */
yrtb_status yrtb_gather_crystal_product(yrtb_projector* h,
                                        const float* d_crystal_eff,
                                        const yrtb_events* ev, yrtb_range range,
                                        float* d_out, yrtb_stream stream);

/* ------------------------------------------------------- event ordering --- */
/* Permutation that groups events by OSEM subset (event index mod
 * num_subsets, the reference's chronological interleaving) and, inside a
 * subset, by dynamic frame (when given), ray length (voxel crossings of the
 * single-ray Siddon projector, in steps of 2^bucket_shift of the projector's
 * launch configuration), then LOR (Histogram3D bin or
 * detector pair) and TOF, so that neighbouring GPU threads trace
 * neighbouring rays of similar length in one frame's image.  num_subsets <=
 * 65535 (4095 with dynamic frames).
 * d_perm[i] = source index of output position i (n uint64); subset_offsets
 * (host, num_subsets+1) delimits the subsets in the reordered arrays.  The
 * result of an OSEM subset does not depend on the order of its events
 * beyond floating-point summation order.  No counterpart in the reference
 * (its batches keep file order). */
yrtb_status yrtb_events_subset_order(yrtb_projector* h, const yrtb_events* ev,
                                     int num_subsets, uint64_t* d_perm,
                                     uint64_t* subset_offsets,
                                     yrtb_stream stream);

/* The same for one shard of a longer event stream: local event e is the
 * stream's event first_global_index + e, and belongs to subset
 * (first_global_index + e) mod num_subsets, so that shards cut anywhere keep
 * the reference's subsets of the whole stream (BinIteratorChronological
 * Interleaved, src/datastruct/projection/BinIterator.cpp:261-265).
 * yrtb_events_subset_order is this with first_global_index = 0. */
yrtb_status yrtb_events_subset_order_from(yrtb_projector* h, const yrtb_events* ev,
                                          int num_subsets,
                                          uint64_t first_global_index,
                                          uint64_t* d_perm, uint64_t* subset_offsets,
                                          yrtb_stream stream);

/* Byte layout of one event row of the reference's device batches: the
 * projection-property rows of PropStructManager<ProjectionPropertyType>
 * (include/yrt-pet/datastruct/projection/ProjectionProperties.hpp:59-140,
 * src/datastruct/projection/ProjectionProperties.cpp:40-81), which
 * ProjectionListDevice / LORsDevice and OSEM_GPU keep on the device (one row
 * per event, the properties packed in enum order).  Each field is the
 * property's byte offset in the row (PropStructManager::getOffset), -1 when
 * the row does not hold it. */
typedef struct
{
	uint32_t row_bytes;   /* PropStructManager::getElementSize */
	int32_t lor;          /* LOR: 6 floats */
	int32_t det_orient;   /* DET_ORIENT: 6 floats */
	int32_t tof;          /* TOF: float, ps */
	int32_t dynamic_frame;/* DYNAMIC_FRAME: int32 */
	int32_t measurement;  /* MEASUREMENT: float */
	int32_t sensitivity;  /* SENSITIVITY: float */
	int32_t attenuation;  /* ATTENUATION: float */
	int32_t randoms;      /* RANDOMS_ESTIMATE: float */
	int32_t scatter;      /* SCATTER_ESTIMATE: float */
} yrtb_row_layout;

/* Unpacks count rows (device memory, 4-byte aligned, layout->row_bytes
 * apart) into the structure of arrays of `out`: out->lor (6 floats per
 * event) must be given, and every other array of `out` that is not NULL
 * receives its property (orient, tof_ps, frame, measurement, sens, att;
 * additive = randoms + scatter, either may be absent); an array whose
 * property the row does not hold is an error.  This is how the reference's
 * own batches (OperatorProjectorDevice::applyAOnLoadedBatch,
 * OSEM_GPU::computeEMUpdateImageForLoadedBatch,
 * src/recon/OSEM_GPU.cu:877-982) reach the projection kernels, which read
 * each field per event from the rows instead
 * (OSEM_GPU.cu:1172-1265, SiddonKernels.cuh:502-574). */
yrtb_status yrtb_events_from_rows(const void* d_rows, uint64_t count,
                                  const yrtb_row_layout* layout,
                                  const yrtb_events* out, yrtb_stream stream);

/* out->X[i] = in->X[d_perm[i]] for every array present in `in` (output
 * buffers allocated by the caller; out->count == in->count).  d_perm must be
 * a permutation of 0..count-1, as yrtb_events_subset_order produces. */
yrtb_status yrtb_events_gather(const yrtb_events* in, const uint64_t* d_perm,
                               const yrtb_events* out, yrtb_stream stream);

/* ----------------------------------------------------- histogram mode --- */
/* Sensitivity image over one subset of Histogram3D bins (phi = subset mod
 * num_subsets), non-TOF: d_sens += A^T (sens_bin * acf_bin).  d_sens_histo /
 * d_acf_histo may be NULL (1); d_mu (with mu_params) gives ACFs from an
 * attenuation image when d_acf_histo is NULL.  Replaces
 * generateSensImage_kernel (src/recon/OSEM_GPU.cu:1048-1157) and
 * OSEM_CPU::generateSensitivityImageForCurrentSubset (src/recon/OSEM_CPU.cpp:127-188)
 * without the final threshold (see yrtb_apply_threshold). */
yrtb_status yrtb_sensitivity_histo3d(yrtb_projector* h, float* d_sens,
                                     const float* d_sens_histo,
                                     const float* d_acf_histo,
                                     const float* d_mu,
                                     const yrtb_image_params* mu_params,
                                     int num_subsets, int subset,
                                     yrtb_stream stream);

/* The same sensitivity image with each bin's LOR sensitivity formed in the
 * kernel as d_crystal_eff[d1] * d_crystal_eff[d2] (FP32, bit-identical to a
 * sensitivity histogram holding those products): the reference's
 * generateSensImage_kernel over a Histogram3D sensitivity
 * (src/recon/OSEM_GPU.cu:1048-1157, Corrector_CPU.cpp:17-45) without the
 * histogram in memory. */
yrtb_status yrtb_sensitivity_histo3d_crystal(yrtb_projector* h, float* d_sens,
                                             const float* d_crystal_eff,
                                             const float* d_acf_histo,
                                             const float* d_mu,
                                             const yrtb_image_params* mu_params,
                                             int num_subsets, int subset,
                                             yrtb_stream stream);

/* Histogram-mode EM pass over one subset of bins: bins with zero measurement
 * are skipped (OSEM_GPU.cu:1224-1225).  Optional per-bin histograms: sens,
 * acf (multiplicative), additive. */
yrtb_status yrtb_em_step_histo3d(yrtb_projector* h, const float* d_image,
                                 float* d_em, const float* d_measurements,
                                 const float* d_sens_histo,
                                 const float* d_acf_histo,
                                 const float* d_additive_histo,
                                 int num_subsets, int subset,
                                 float global_scale, float denom_threshold,
                                 yrtb_stream stream);

/* The bins of one subset that the histogram EM pass does work for (valid
 * detector pair, measurement != 0), as subset-local indices in increasing
 * order: d_k (device, capacity >= the subset's bin count) receives them and
 * *n_out their number (synchronises the stream).  Replaces the skip of
 * zero-measurement bins inside the bin loop of computeEMUpdateImage_kernel
 * (OSEM_GPU.cu:1224-1225) by selecting them once per reconstruction. */
yrtb_status yrtb_histo3d_subset_nonzero(yrtb_projector* h,
                                        const float* d_measurements,
                                        int num_subsets, int subset,
                                        uint64_t* d_k, uint64_t capacity,
                                        uint64_t* n_out, yrtb_stream stream);

/* yrtb_em_step_histo3d over the n listed bins of the subset only (the list of
 * yrtb_histo3d_subset_nonzero): the same per-bin work, with warps that hold
 * only bins that do work.  Same image as the full-subset pass (bit-identical
 * in deterministic mode). */
yrtb_status yrtb_em_step_histo3d_list(yrtb_projector* h, const float* d_image,
                                      float* d_em, const float* d_measurements,
                                      const float* d_sens_histo,
                                      const float* d_acf_histo,
                                      const float* d_additive_histo,
                                      int num_subsets, int subset,
                                      const uint64_t* d_k, uint64_t n,
                                      float global_scale, float denom_threshold,
                                      yrtb_stream stream);

/* List-mode -> Histogram3D: d_histo[bin(d1,d2)] += value for value > 0 and
 * d1 != d2 (values NULL: 1).  Pairs outside the histogram (ring difference,
 * minimum angle) are skipped and counted in *n_invalid (the reference
 * throws; this call returns YRTB_ERR_RANGE when any are found).  Synchronises
 * the stream.  Replaces util::convertToHistogram3D
 * (src/utils/ReconstructionUtils.cpp:659-800). */
yrtb_status yrtb_listmode_to_histo3d(yrtb_projector* h, const uint32_t* d_d1,
                                     const uint32_t* d_d2,
                                     const float* d_values, uint64_t n,
                                     float* d_histo, uint64_t* n_invalid,
                                     yrtb_stream stream);

/* List-mode file records on the device (after one H2D copy of the raw file
 * bytes) -> structure of arrays.  Record layout of ListModeLUT files
 * (src/datastruct/projection/ListModeLUT.cpp:224-307): u32 timestamp, u32 d1,
 * u32 d2, then f32 TOF if has_tof, then f32 randoms if has_randoms.  d_ts,
 * d_tof, d_randoms may be NULL to drop a field.  Records with a detector id
 * >= num_dets make the call return YRTB_ERR_EVENT naming the first such
 * event (the reference throws "Detectors invalid in list-mode event N").
 * Synchronises the stream.  Replaces the host-side ListModeLUTOwned::
 * readFromFile unpacking and the per-batch host gather of
 * OSEM_GPU::precomputeBatchPropsForRecon (src/recon/OSEM_GPU.cu:698-805). */
yrtb_status yrtb_unpack_listmode(const void* d_raw, uint64_t n, int has_tof,
                                 int has_randoms, uint32_t num_dets,
                                 uint32_t* d_ts, uint32_t* d_d1, uint32_t* d_d2,
                                 float* d_tof, float* d_randoms,
                                 yrtb_stream stream);

/* Histogram3D maps on the device: bin ids of detector pairs (UINT64_MAX for
 * pairs outside the histogram) and detector pairs of bin ids.  Replace
 * Histogram3D::getBinIdFromDetPair / getDetPairFromBinId
 * (src/datastruct/projection/Histogram3D.cpp:366-426). */
yrtb_status yrtb_histo3d_bins(yrtb_projector* h, const uint32_t* d_d1,
                              const uint32_t* d_d2, uint64_t n,
                              uint64_t* d_bins, yrtb_stream stream);
yrtb_status yrtb_histo3d_detpairs(yrtb_projector* h, const uint64_t* d_bins,
                                  uint64_t n, uint32_t* d_d1, uint32_t* d_d2,
                                  yrtb_stream stream);

/* -------------------------------------------------------- image space --- */
/* x *= u / s where s > threshold.  sens_nt == 1 broadcasts one sensitivity
 * image over nt frames; d_frame_scale (nullable, nt floats) divides u and
 * the threshold per frame and, as updateEMThresholdDynamic with sensScaling,
 * always reads the first sensitivity frame.  Replaces Image::updateEMThreshold{Static,
 * DynamicWithScaling,DynamicWith4DSens} (src/datastruct/image/Image.cpp:651-833)
 * and updateEM_kernel / updateEMDynamic_kernel
 * (src/datastruct/image/ImageSpaceKernels.cu:13-76). */
yrtb_status yrtb_em_update(float* d_image, const float* d_em,
                           const float* d_sens, uint64_t voxels_per_frame,
                           int64_t nt, int64_t sens_nt, float threshold,
                           const float* d_frame_scale, yrtb_stream stream);

/* x = x*le_scale + le_off where mask <= threshold, else x*gt_scale + gt_off.
 * broadcast != 0 applies a one-frame mask to every frame.  Replaces
 * Image::applyThreshold / applyThresholdBroadcast
 * (src/datastruct/image/Image.cpp:594-649). */
yrtb_status yrtb_apply_threshold(float* d_image, const float* d_mask,
                                 uint64_t voxels_per_frame, int64_t nt,
                                 int broadcast, float threshold,
                                 float le_scale, float le_off, float gt_scale,
                                 float gt_off, yrtb_stream stream);

/* d_x[i] = value (ImageDevice::fill). */
yrtb_status yrtb_fill(float* d_x, uint64_t n, float value, yrtb_stream stream);

/* d_x[i] *= scale (ImageDevice::multWithScalar). */
yrtb_status yrtb_scale(float* d_x, uint64_t n, float scale,
                       yrtb_stream stream);

/* ---------------------------------------------------- image-space PSF --- */
/* Spatially invariant, separable image-space PSF: OperatorPsf /
 * OperatorPsfDevice (include/yrt-pet/operators/OperatorPsf.hpp:19-70,
 * src/operators/OperatorPsf.cpp:288-375, src/operators/OperatorPsfDevice.cu).
 * Three 1-D kernels of odd length (x, y, z); applyA convolves with them,
 * applyAH with the flipped kernels. */
typedef struct yrtb_psf yrtb_psf;

yrtb_status yrtb_psf_create(const float* kernel_x, int size_x,
                            const float* kernel_y, int size_y,
                            const float* kernel_z, int size_z, yrtb_psf** out);
void yrtb_psf_destroy(yrtb_psf* psf);

/* d_out = PSF d_in (adjoint = 0) or PSF^H d_in (adjoint = 1), every frame:
 * passes along x, y, z, each out[i] = sum_kk k[kk + c] in[circ(i - kk)],
 * kk = -c..c, with circular borders and FP32 sums in tap order (bit-identical
 * to the reference CPU operator).  d_in != d_out; d_tmp: nx*ny*nz*nt floats
 * of scratch, or NULL (taken from the library's pool).  A kernel half-width
 * must be smaller than the image along its axis. */
yrtb_status yrtb_psf_apply(const yrtb_psf* psf, const float* d_in, float* d_out,
                           const yrtb_image_params* image, int adjoint,
                           float* d_tmp, yrtb_stream stream);

/* -------------------------------------- spatially variant image PSF --- */
/* OperatorVarPsf / OperatorVarPsfDevice
 * (include/yrt-pet/operators/OperatorVarPsf.hpp:66-100,
 * src/operators/OperatorVarPsf.cpp:290-455): voxel (i, j, k) is blurred by
 * its own 3-D kernel, the LUT entry nearest to the voxel centre's distance
 * from the image centre: index (a, b, c) = round(|d| / gap) per axis, clamped
 * to floor(range / gap), LUT index a + A (b + B c). */
typedef struct yrtb_varpsf yrtb_varpsf;

/* One Gaussian (columns = 3: sigma x, y, z) or two-Gaussian mixture
 * (columns = 7: sigma1 x y z, sigma2 x y z, weight2) kernel of the LUT
 * (ConvolutionKernelGaussian / ConvolutionKernelGaussianMixture): half sizes
 * max(1, floor(sigma_max nstd / v) - 1), weights z-major, then y, then x.
 * Writes the half sizes (x, y, z) and the weight count; weights only when
 * out != NULL (cap floats). Host-side, no device work. */
yrtb_status yrtb_varpsf_gaussian_kernel(const float* sigmas, int columns, const float* nstd,
                                        const yrtb_image_params* image, float* out,
                                        uint64_t cap, int32_t* half_sizes, uint64_t* size);

/* Kernel LUT: num_kernels kernels back to back in weights (kernel i:
 * (2hz+1)(2hy+1)(2hx+1) floats, z-major), half_sizes 3 per kernel (x, y, z);
 * range / gap: 3 floats (x, y, z) as OperatorVarPsf::setRangeAndGap. */
yrtb_status yrtb_varpsf_create(const float* weights, const int32_t* half_sizes,
                               int num_kernels, const float* range, const float* gap,
                               yrtb_varpsf** out);
void yrtb_varpsf_destroy(yrtb_varpsf* psf);

/* d_out = A d_in (adjoint = 0: each output voxel sums its own kernel over
 * the input, FP32 in the reference's z, y, x tap order, bit-identical) or
 * A^H d_in (adjoint = 1: each input voxel's kernel spread to its
 * neighbours, gathered per output voxel without atomics), circular borders,
 * every frame.  d_out is overwritten (the reference accumulates into an
 * output it zeroes first).  d_in != d_out. */
yrtb_status yrtb_varpsf_apply(const yrtb_varpsf* psf, const float* d_in, float* d_out,
                              const yrtb_image_params* image, int adjoint,
                              yrtb_stream stream);

/* ------------------------------------------- low-rank dynamic images --- */
/* Low-rank image model of the LR updater (ProjectorUpdaterLR,
 * src/operators/ProjectorUpdater.cpp:228-280; ProjectorUpdaterDeviceLR,
 * include/yrt-pet/operators/ProjectorUpdaterDevice.cuh:53-225; LREM,
 * src/recon/LREM.cpp:175-260): frame t of the image is
 * x_t = sum_l H[l][t] W_l, with W = rank images of voxels_per_frame floats
 * (rank-major) and H = rank x frames floats (row-major, HBasis[r][t]).
 * Instead of the rank sum at every voxel crossing, a projection of the
 * low-rank image projects the expanded frames (yrtb_lr_expand, then any
 * frame-indexed projector call with nt = frames), and a back projection is
 * contracted onto the basis afterwards (yrtb_lr_contract_w for W,
 * yrtb_lr_contract_h for H).  rank <= 32. */

/* X[t][j] = sum_l W[l][j] H[l][t], l ascending, FP32 products and sums in the
 * reference updater's order (X: frames x voxels_per_frame floats). */
yrtb_status yrtb_lr_expand(const float* d_W, const float* d_H, int rank, int frames,
                           uint64_t voxels_per_frame, float* d_X, yrtb_stream stream);

/* Wn[l][j] = sum_t E[t][j] H[l][t] (E: frames x voxels_per_frame, e.g. the
 * EM image of an EM step over the expanded frames; Wn: rank images). */
yrtb_status yrtb_lr_contract_w(const float* d_E, const float* d_H, int rank, int frames,
                               uint64_t voxels_per_frame, float* d_Wn, yrtb_stream stream);

/* Hn[l][t] = sum_j W[l][j] E[t][j] (FP32 products, FP64 sums in a fixed order:
 * deterministic).  rank x frames <= 2048 and rank + frames <= 440.  With
 * frames = 1 and E = a sensitivity image it gives LREM's H-update scaling
 * c_r = sum_j W[r][j] s[j] (LREM::generateHUpdateSensScaling). */
yrtb_status yrtb_lr_contract_h(const float* d_W, const float* d_E, int rank, int frames,
                               uint64_t voxels_per_frame, double* d_Hn, yrtb_stream stream);

/* H[r][t] *= float(Hn[r][t]) * (1 / max(c[r], eps))  (LREM::applyHUpdate,
 * src/recon/LREM.cpp:175-199).  d_c: rank floats. */
yrtb_status yrtb_lr_update_h(float* d_H, const double* d_Hn, const float* d_c, int rank,
                             int frames, float eps, yrtb_stream stream);

/* ------------------------------------------------------ OSEM (driver) --- */
/* List-mode OSEM over device-resident events.  Mirrors OSEM::reconstruct
 * (src/recon/OSEM.cpp:315-365) with the GPU hooks of OSEM_GPU
 * (src/recon/OSEM_GPU.cu:311-537): x0 = 0.125 (or the given estimate),
 * masked by sens > 0, sensitivity divided by the number of subsets,
 * subsets = chronologically interleaved events.  d_image holds nt frames and
 * is both the initial estimate (when init_from_image != 0) and the result.
 * d_sens: one image (voxels_per_frame floats).  d_work: scratch of
 * nt*voxels_per_frame floats + voxels_per_frame floats, plus
 * 2*nt*voxels_per_frame floats with an image-space PSF.  use_graph != 0
 * captures each subset (reset, EM pass, update) into a CUDA graph and
 * replays it. */
typedef struct
{
	int iterations, subsets;
	float global_scale, denom_threshold, em_threshold;
	int init_from_image;
	int use_graph;
	const float* d_frame_scale; /* nullable, nt floats */
	const uint64_t* subset_offsets; /* host, subsets+1; NULL: interleaved
	                                   events (stride = subsets); else subset s
	                                   = events [off[s], off[s+1]) as produced
	                                   by yrtb_events_subset_order */
	const yrtb_psf* psf;  /* image-space PSF or NULL: each subset projects PSF x and
	                         applies PSF^H to the EM image before the update
	                         (OSEM_GPU::computeEMUpdateImage, src/recon/OSEM_GPU.cu:456-509);
	                         d_sens must already include PSF^H, as
	                         OSEM::generateSensitivityImages makes it */
	const yrtb_varpsf* varpsf; /* spatially variant image-space PSF or NULL (used
	                              like psf; at most one of the two) */
} yrtb_osem_params;

yrtb_status yrtb_osem_listmode(yrtb_projector* h, const yrtb_events* ev,
                               const float* d_sens, float* d_image,
                               float* d_work, const yrtb_osem_params* p,
                               yrtb_stream stream);

/* Same as yrtb_osem_listmode, for callers that cannot allocate device
 * memory: it takes no work buffer and calls no allocating routine.  Some
 * hosts own every byte of device memory through their own pool, or run
 * inside a real-time loop where cudaMalloc / cudaFree (which synchronise the
 * device) are not allowed after start-up; they still have to reconstruct.
 * The scratch (EM image and scaled sensitivity: (nt + 1) x voxels floats;
 * with an image-space PSF also the blurred image and the PSF's temporary:
 * (3 nt + 1) x voxels floats) lives in one static device array of
 * YRTB_OSEM_STATIC_MAX_FLOATS floats (16 MiB) that every GPU loading the
 * library holds until exit; larger images are rejected with
 * YRTB_ERR_ARGUMENT.  use_graph must be 0.  Every call looks up the array's
 * device address with the projector's device current; the first call on a
 * device may load the library's device code, which is when the array is
 * allocated, so make it during start-up, before any stream capture.  All
 * calls share the one array: calls that overlap on the GPU (other streams,
 * other host threads, same device) race and must be serialised by the
 * caller.  No counterpart in the reference. */
#define YRTB_OSEM_STATIC_MAX_FLOATS (4u * 1024u * 1024u)
yrtb_status yrtb_osem_listmode_static(yrtb_projector* h, const yrtb_events* ev,
                                      const float* d_sens, float* d_image,
                                      const yrtb_osem_params* p,
                                      yrtb_stream stream);

#ifdef __cplusplus
}
#endif

#endif /* YRT_B200_H */

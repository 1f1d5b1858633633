/*
 * xrecon_b200.h -- C ABI of the B200 distance-driven (DD) projector library
 * (libxrecon_b200.so).  Plain pointers, sizes and a CUDA stream; no torch
 * types.  Every call is asynchronous on `stream`, allocates nothing (the
 * caller passes a device workspace sized by the matching *_workspace_size
 * call), never exits the process, and returns an xr_status.
 *
 * Reference interface being replaced: the pybind module `xrecon_C` of XRecon
 * (src/api/torch_binding.cpp:615-638), whose functions all take
 * (Tensor input, Tensor options float32, Tensor angles float32 [V]) and
 * return a new tensor.  The geometry structs below carry exactly the fields
 * the reference unpacks from `options` (torch_binding.cpp:62-124), in the same
 * packed units (3D flat: raw du and the raw shift in mm, the kernels apply
 * SOD/SDD; 3D arc: du/SDD in radians; 2D: the "effective" spacing of
 * xrecon/projector/geometry.py:105-113).
 */
#ifndef XRECON_B200_H
#define XRECON_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    XR_OK = 0,
    XR_ERR_INVALID_ARGUMENT = 1,  /* bad geometry, shape, op or dtype      */
    XR_ERR_WORKSPACE = 2,         /* workspace missing or too small         */
    XR_ERR_CUDA = 3,              /* a CUDA launch or runtime call failed   */
    XR_ERR_UNSUPPORTED = 4        /* valid request the library cannot serve */
} xr_status;

/* Operators, numbered as the six per-dimension bindings of the reference. */
typedef enum {
    XR_PROJECTION = 0,                 /* forward_projection{2,3}d                    */
    XR_PROJECTION_T = 1,               /* projection_transpose{2,3}d                  */
    XR_BACKPROJECTION = 2,             /* backward_projection{2,3}d                   */
    XR_BACKPROJECTION_T = 3,           /* backward_projection_transpose{2,3}d         */
    XR_WEIGHTED_BACKPROJECTION = 4,    /* weighted_backward_projection{2,3}d          */
    XR_WEIGHTED_BACKPROJECTION_T = 5   /* weighted_backward_projection_transpose{2,3}d*/
} xr_op;

/* Scan geometry, values of the reference's scan_id (geometry.py:63-103). */
typedef enum { XR_PARALLEL = 0, XR_FAN_FLAT = 1, XR_FAN_ARC = 2 } xr_geometry_type;

/* Storage dtype of image / sinogram buffers.  Accumulation is FP32 always. */
typedef enum { XR_FLOAT32 = 0, XR_BFLOAT16 = 1, XR_FLOAT16 = 2 } xr_dtype;

/* 2D geometry: the 12 packed options of Projector2d (projector.py:106-110),
 * unpacked as torch_binding.cpp:62-79. */
typedef struct {
    int W, H, Nu, type;
    float dx, dy, du, sod, sdd, shift_x, shift_y, shift_u;
} xr_geom2d;

/* 3D geometry: the 18 packed options of Projector3d (projector3d.py:98-107),
 * unpacked as torch_binding.cpp:82-124 (the helical fields travel in
 * xr_helical_opts). */
typedef struct {
    int W, H, D, Nu, Nv, type;
    float dx, dy, dz, du, dv, sod, sdd;
    float shift_x, shift_y, shift_z, shift_u, shift_v;
} xr_geom3d;

/* Device workspace (bytes) that xr_dd2d / xr_dd3d need for these arguments,
 * for any storage dtype. */
size_t xr_dd2d_workspace_size(int op, const xr_geom2d* geom, int nbatch, int nview);
size_t xr_dd3d_workspace_size(int op, const xr_geom3d* geom, int nbatch, int nview);

/*
 * Apply one 2D DD operator (replaces the six *2d bindings,
 * torch_binding.cpp:140-351).
 *   in / out : device buffers; image layout [nbatch, H, W], sinogram layout
 *              [nbatch, nview, Nu] (nbatch = B*C of the reference).  `out` is
 *              fully overwritten (no zero-fill needed).
 *   angles   : device float32 [nview], radians.
 *   dtype_in / dtype_out : xr_dtype of `in` / `out`.
 */
int xr_dd2d(int op, const xr_geom2d* geom, const void* in, int dtype_in, void* out, int dtype_out,
            const float* angles, int nbatch, int nview, void* workspace, size_t workspace_bytes,
            void* stream);

/*
 * Apply one 3D DD operator (replaces forward_projection3d,
 * projection_transpose3d, backward_projection3d,
 * weighted_backward_projection3d, backward_projection_transpose3d and
 * weighted_backward_projection_transpose3d, torch_binding.cpp:407-523).
 *   image layout [nbatch, D, H, W], sinogram layout [nbatch, nview, Nv, Nu].
 */
int xr_dd3d(int op, const xr_geom3d* geom, const void* in, int dtype_in, void* out, int dtype_out,
            const float* angles, int nbatch, int nview, void* workspace, size_t workspace_bytes,
            void* stream);

/*
 * Helical cone-beam scans with an arc detector (replaces the six *_helical3d
 * bindings, torch_binding.cpp:525-612, over src/kernels/helical_arc3d.cu).
 * Options: entries 18..23 of HelicalProjector3d's packed options
 * (projector3d.py:375-400), with the binding's defaults
 * (torch_binding.cpp:103-108): view_mode 2, weight_mode 0, view_turns 0,
 * halfscan_coef 1, tang_k 5, tang_blend 0.
 */
typedef struct {
    int view_mode;      /* 0 auto (from the pitch), 1 half scan, 2 one turn, 3 view_turns turns */
    int weight_mode;    /* 0 conjugate-ray redundancy ("2d"), 1 tangential ("tang3d") */
    float view_turns, halfscan_coef, tang_k, tang_blend;
} xr_helical_opts;

size_t xr_helical3d_workspace_size(int op, const xr_geom3d* geom, int nbatch, int nview);

/*
 * Apply one helical operator (op as xr_op; geom->type must be XR_FAN_ARC).
 *   in / out   : device float32, image [nbatch, D, H, W], sinogram
 *                [nbatch, nview, Nv, Nu]; `out` is fully overwritten.
 *   angles     : device float32 [nview].
 *   source_pos : device float32 [4, nview], rows source_z, shift_radius,
 *                shift_angle, shift_z (the reference's source_pos,
 *                torch_binding.cpp:128-138).
 * The reference supports float32 only; so does this entry.
 */
int xr_helical3d(int op, const xr_geom3d* geom, const xr_helical_opts* opts, const float* in, float* out,
                 const float* angles, const float* source_pos, int nbatch, int nview, void* workspace,
                 size_t workspace_bytes, void* stream);

/*
 * Fused FBP/FDK pre-filter (replaces the `sino * weight` and
 * conv2d/conv3d(padding Nu-1) steps of filtered_backprojection,
 * projector.py:200-201 and projector3d.py:189-190):
 *   out[row, i] = sum_j in[row, j] * pw[row_view, j] * cosw[j] * filt[j - i + Nu - 1]
 * for every detector row (nrows = nbatch*nview*Nv rows of Nu samples).
 *   cosw   : device float32 [Nu] cosine weight (may be NULL = ones)
 *   filt   : device float32 [2*Nu-1] spatial filter
 *   parker : device float32 [nview, Nu] short-scan weight or NULL
 *   rows_per_view : Nv (3D) or 1 (2D), to index `parker` by view.
 * Rows of up to 2048 cells are filtered by FFT (a circular convolution of
 * length 2^ceil(log2(2 Nu - 1)), FP32 rows, the filter's spectrum in FP64):
 * within a few 1e-6 of the exact correlation, relative L2, on projection
 * rows with the ramp filter.  Wider rows, and every row while
 * xr_set_plain_kernels is on, take the direct correlation (FP32 sums).
 */
int xr_fbp_filter(const void* in, int dtype_in, float* out, int nrows, int Nu, int nview, int rows_per_view,
                  const float* cosw, const float* filt, const float* parker, void* stream);

/*
 * Read (and optionally clear) the device-wide error word of the current
 * device: 0 when no kernel has reported a problem.  Bit 0 = a bounded wait
 * for a TMA transfer gave up (the projection kernel's CTA then left its
 * line loop and stored nothing); bit 1 = a grid barrier of the ragged batch
 * kernel gave up (the kernel returned).  The outputs of the launch that set a
 * bit are not valid.  Synchronous (reads device memory); the operators never
 * read it themselves, so callers that want the check poll it, for example
 * after each batch of work.  Replaces the reference's exit() on a CUDA error
 * (include/utils.h:7-11): the process and its context stay usable.
 */
int xr_device_error(unsigned int* code, int clear);

/*
 * Poll limits of the bounded waits on the current device: tma_polls for an
 * mbarrier wait of the projection kernel (each poll suspends at most about
 * 1 us; default 2^20), barrier_polls for a grid barrier of the ragged kernel
 * (polls of about 128 ns; default 2^22).  Values <= 0 restore the defaults.
 * Synchronous.  No reference counterpart.
 */
int xr_set_wait_limits(long long tma_polls, long long barrier_polls);

/*
 * Testing aid, no reference counterpart: failure injection for the bounded
 * waits, on the current device (0 = off, the default).  Bit 0: the
 * projection kernel's producer arms each barrier for a box but issues no
 * copy, so every consumer wait runs out with nothing in flight.  Bit 1: the
 * ragged kernel's grid barriers expect one block more than the grid, so every
 * barrier wait runs out.  Nothing faults; the waits end at their limits
 * (xr_set_wait_limits) and set the device error word.  Bit 2: the staged
 * prefix backprojection treats every odd view as not fitting its box, so its
 * fallback launch adds those views.  Bit 3 (read on the host): the prefix
 * backprojection is not staged.  Synchronous.
 */
int xr_test_hooks(unsigned int hooks);

/* Staging plan of the 3D projection kernel for this geometry: whether the
 * TMA line windows are used, their box size (pixels x z voxels), and whether
 * the fine-row kernel (detector rows shorter than a voxel) is chosen. */
int xr_cell_plan(const xr_geom3d* geom, int* ok, int* box_pixels, int* box_z, int* rows_per_thread, int* fine);

/* Staging plan of the 3D prefix backprojection (B, Bw, A^T) for this
 * geometry: whether each view's table footprint is staged into shared memory
 * (flat, parallel and arc detectors with an even column count), and the box
 * size in table columns x rows.  Host-only; no device is touched. */
int xr_pfx_stage_plan(const xr_geom3d* geom, int* ok, int* box_cols, int* box_rows);

/* Testing aid: nonzero routes every operator through the plain (non-TMA)
 * kernels, so both paths can be compared. */
int xr_set_plain_kernels(int on);

/*
 * Allocation-free variant of xr_dd2d.  It has no counterpart in the
 * reference, which allocates its outputs and scratch on every call.
 *
 * Who needs it: a caller that cannot allocate device memory while it runs,
 * such as a reconstruction service that reserves its whole device-memory
 * budget at start-up, or code running inside a host framework that owns the
 * device allocator.  For such callers a cudaMalloc in mid-run can fail, or
 * stall the device while it waits for free memory.
 *
 * Same operators, layouts and results as xr_dd2d.  The caller still passes
 * its inputs and outputs; the scratch (per-view tables and the flipped image
 * transpose) lives in a fixed static device array of
 * XR_NOALLOC_SCRATCH_BYTES inside the library, held by every GPU that loads
 * the library until the process exits.  No call allocates or frees device
 * memory.  Requests that need more scratch than that (see
 * xr_dd2d_workspace_size) fail with XR_ERR_WORKSPACE.  Every scratch byte a
 * call reads is first written by the same call, so nothing needs clearing.
 * The first call on a device looks up the array's device address
 * (cudaGetSymbolAddress) and caches it per device and CUDA context (after a
 * device reset the next call looks it up again); make that first call before
 * any stream capture.  There is one array per device: calls whose executions
 * overlap on the GPU (different streams, or threads) race on it and must be
 * serialised by the caller.
 */
#define XR_NOALLOC_SCRATCH_BYTES (32u << 20)
int xr_dd2d_noalloc(int op, const xr_geom2d* geom, const void* in, int dtype_in, void* out, int dtype_out,
                    const float* angles, int nbatch, int nview, void* stream);

/*
 * Fan/cone -> parallel rebinning along the detector columns (replaces the
 * grid_sample step of fan_to_parallel_rebin, xrecon/utils/rebin.py:10-95).
 *   in   : [nbatch][nview][Nv][Nu] fan sinogram (xr_dtype dtype_in)
 *   grid : device float [nview_out][Nt][2], the reference's normalized
 *          sampling grid (x: detector column, y: view), align_corners=True
 *   out  : float [nbatch][nview_out][Nv][Nt]; bilinear samples with zero
 *          padding (grid_sample semantics)
 *   filt : NULL, or [2 Nt - 1] filter taps: the rebinned rows are then
 *          filtered in the same pass (as xr_fbp_filter, no weights).
 */
int xr_rebin_parallel(const void* in, int dtype_in, float* out, int nbatch, int nview, int Nv, int Nu,
                      const float* grid, int nview_out, int Nt, const float* filt, void* stream);

/*
 * Sparse export of the projection matrix A (replaces system_matrix2d /
 * system_matrix3d, torch_binding.cpp:353-405, which build it on the CPU with
 * src/cpu/system_matrix2d.cpp and src/cpu/system_matrix3d.cpp).  Two passes
 * over the cells, numbered c = (view * Nv + det_row) * Nu + k with k the
 * traversal-order column (2D: Nv = 1):
 *   offsets == NULL : counts[c] = number of nonzero weights of cell c;
 *   offsets != NULL : the weights of cell c are written at rows/cols/vals
 *                     [offsets[c], offsets[c] + counts[c]) (offsets is the
 *                     exclusive scan of counts).
 * Entries: row = (view * Nv + det_row) * Nu + physical column, col = voxel
 * index (iz * H + iy) * W + ix, value = the projection's weight (FP32), so
 * that the matrix times the flattened image equals xr_dd*d(XR_PROJECTION).
 * Zero weights are skipped, as in the reference.  angles: device [nview].
 */
size_t xr_sysmat2d_workspace_size(const xr_geom2d* geom, int nview);
size_t xr_sysmat3d_workspace_size(const xr_geom3d* geom, int nview);
int xr_sysmat2d(const xr_geom2d* geom, const float* angles, int nview, const long long* offsets, long long* counts,
                long long* rows, long long* cols, float* vals, void* workspace, size_t workspace_bytes, void* stream);
int xr_sysmat3d(const xr_geom3d* geom, const float* angles, int nview, const long long* offsets, long long* counts,
                long long* rows, long long* cols, float* vals, void* workspace, size_t workspace_bytes, void* stream);

/*
 * Ragged batch of 2D reconstructions: projection then FBP for many
 * instances with different geometries, image sizes, view counts and
 * detectors, in one persistent cooperative kernel launch (no reference
 * counterpart: the reference runs each instance through Projector2d,
 * projector.py:176-206, with one launch per operator).  Buffers hold the
 * instances back to back; offsets are in elements:
 *   images / recon : [H][W] at img_offset         (recon: the FBP output)
 *   sino           : [nview][Nu] at sino_offset   (the projection output)
 *   angles         : [nview] at ang_offset
 *   filt           : [2 Nu - 1] filter taps at filt_offset (as xr_fbp_filter)
 *   cosw           : [Nu] cosine weight at cosw_offset
 * recon = scale * Bw(corr_u(sino * cosw, filt)) per instance.
 */
typedef struct {
    xr_geom2d geom;
    int nview;
    long long img_offset, sino_offset, ang_offset, filt_offset, cosw_offset;
    float scale;
} xr_ragged2d_instance;

typedef struct xr_ragged2d_plan xr_ragged2d_plan;

/* Validate the instances and lay out the device workspace (host only). */
int xr_ragged2d_plan_create(const xr_ragged2d_instance* inst, int ninst, xr_ragged2d_plan** plan,
                            size_t* workspace_bytes);
/* Bind buffers and workspace: uploads the per-instance descriptors
 * (synchronous; call before any stream capture). */
int xr_ragged2d_plan_bind(xr_ragged2d_plan* plan, const float* images, float* sino, float* recon,
                          const float* angles, const float* filt, const float* cosw, void* workspace,
                          size_t workspace_bytes);
/* One persistent launch over the whole batch (capturable in a CUDA graph).
 * project = 0 skips the projection (sino is then an input).  Tile shape:
 * 32 << a_cols_log2 detector columns per projection tile, 1 << view_split_log2
 * threads per pixel in the backprojection (both 0..3).  Calls on one plan
 * must not overlap (they share the workspace's tile counters). */
int xr_ragged2d_run(const xr_ragged2d_plan* plan, int project, int a_cols_log2, int view_split_log2, void* stream);
/* Grid size of the persistent launch and the tile counts of its ten tile
 * lists (tables, filter rows, projection per a_cols, backprojection per
 * view split). */
int xr_ragged2d_plan_info(const xr_ragged2d_plan* plan, int* grid, int* tiles10);
void xr_ragged2d_plan_destroy(xr_ragged2d_plan* plan);

/*
 * DICOM-CT-PD projection series reader (host code; no GPU, no stream).
 * Replaces the per-file loop of load_projection_stack
 * (xrecon/utils/mayo.py:145-170, pydicom.dcmread per view): reads the
 * `nfiles` files, spread over `nthreads` threads (<= 0: one per core), and
 * writes
 *   sino  [nfiles, ceil(cols / row_stride), ceil(rows / col_stride)] float32:
 *         stored pixel [c * col_stride, r * row_stride] rescaled as
 *         float32(raw) * float32(RescaleSlope) + float32(RescaleIntercept)
 *         (two float32 roundings), at [view, r, c];
 *   views [nfiles, 5] float32: angle (7031,1001), source z (7031,1002),
 *         shift z (7033,100B), shift angle (7033,100C), shift radius
 *         (7033,100D); absent shifts are 0.
 * `rows` x `cols` is the stored pixel matrix (Rows = detector columns,
 * Columns = detector rows) every file must have.  Files in implicit or
 * explicit VR little endian with native single-frame 8/16/32-bit pixels and
 * single-valued tags are read; any other file (deflated or compressed
 * encodings, multi-valued or oddly typed tags, a different matrix, an
 * unreadable or malformed file) stops the call with XR_ERR_UNSUPPORTED and
 * its index in *failed_file, for a general reader to handle or reject.
 */
int xr_ctpd_load(const char* const* paths, int nfiles, int rows, int cols, int col_stride, int row_stride,
                 int nthreads, float* sino, float* views, int* failed_file);

/* Number of CUDA kernels this library has launched in this process (all
 * devices and threads). */
unsigned long long xr_launch_count(void);

/* Human-readable message for the last non-OK status returned on this thread. */
const char* xr_last_error(void);

/* Library version string. */
const char* xr_version(void);

#ifdef __cplusplus
}
#endif

#endif /* XRECON_B200_H */

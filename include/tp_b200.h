/*
 * tp_b200.h - C ABI of the B200-native (sm_100a) tile processor.
 *
 * Drop-in host entry points for the frequency-domain tile processor of
 * mfkiwl/tile_processor_gpu.  Each tp_* call replaces one `extern "C"
 * __global__` kernel of the reference (launched there with <<<>>> by
 * src/dtt8x8.cu or by name through JCuda) and takes the same arguments, in the
 * same order and with the same meaning, plus:
 *   - a tp_geometry block that replaces the reference's compile-time
 *     IMG_WIDTH / IMG_HEIGHT / KERNELS_* / TILES* defines
 *     (src/TileProcessor.cuh:43-73,145-175), so one library serves every frame
 *     size;
 *   - the CUDA stream to launch on (NULL = legacy default stream).
 *
 * Buffers are caller-owned device memory, exactly as in the reference
 * (src/dtt8x8.cu:53-142): pitched float images, per-camera pointer arrays that
 * live in device memory (float ** on the device), pitched outputs.  Strides are
 * in floats.  Outputs that the reference accumulates into (imclt_rbg, the RGBA
 * texture image) are accumulated here too.
 *
 * Every call validates its host-visible arguments and returns TP_OK or a
 * negative TP_ERR_* code (the reference kernels return void and silently skip
 * bad input); tp_last_error() gives a one-line reason.  No call allocates
 * device memory, and none synchronises the device or reads device data on the
 * host, except the first tensor-core call on a device (it copies the
 * transform tables) and tp_tc_status, which say so.
 * Device-side inputs that the host cannot see (task records, index lists) are
 * range-checked in the kernels: an out-of-range entry is skipped instead of
 * being read or written out of bounds.
 */
#ifndef TP_B200_H
#define TP_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st *tp_stream_t; /* same object as cudaStream_t */

/* ---- fixed sizes (the reference hard-codes the same values) ---------------- */
#define TP_DTT_SIZE        8   /* DTT_SIZE            src/dtt8x8.cuh:52        */
#define TP_NUM_CAMS        4   /* NUM_CAMS            src/TileProcessor.cuh:44 */
#define TP_NUM_PAIRS       6   /* NUM_PAIRS           src/TileProcessor.cuh:45 */
#define TP_NUM_COLORS      3   /* NUM_COLORS          src/TileProcessor.cuh:46 */
#define TP_CORR_NTILE_SHIFT 8  /* CORR_NTILE_SHIFT    src/TileProcessor.cuh:60 */
#define TP_TASK_CORR_BITS  4   /* TASK_CORR_BITS      src/TileProcessor.cuh:63 */
#define TP_LIST_TEXTURE_BIT 7  /* LIST_TEXTURE_BIT    src/TileProcessor.cuh:69 */
#define TP_TASK_TEXTURE_BITS 0xf /* N/E/S/W bits 0..3 src/TileProcessor.cuh:64-67,96 */
#define TP_MAX_CORR_RADIUS 7   /* (2r+1)^2 <= 15x15   src/TileProcessor.cuh:2950-3008 */

/* Per-tile task record, byte-identical to `struct tp_task`
 * (src/TileProcessor.cuh:179-186) with NUM_CAMS = 4: 40 bytes.
 *   task : bits 0..3 texture N/E/S/W, bits 4..9 correlation pair mask;
 *   txy  : tile x in bits 0..15, tile y in bits 16..31;
 *   xy   : tile centre in each camera's pixel coordinates. */
typedef struct tp_task {
    int   task;
    int   txy;
    float xy[TP_NUM_CAMS][2];
} tp_task;

/* Kernel-tile offsets, byte-identical to `struct CltExtra`
 * (src/TileProcessor.cuh:187-196): 8 floats per kernel tile. */
typedef struct tp_clt_extra {
    float data_x, data_y, center_x, center_y;
    float dxc_dx, dxc_dy, dyc_dx, dyc_dy;
} tp_clt_extra;

/* How the Bayer fetch treats tiles whose 16x16 window leaves the image. */
enum {
    /* The reference's addressing (src/TileProcessor.cuh:3183-3193,3328-3361):
     * right-edge corner clamp `itlx & 1 + (W-10)` (C precedence: itlx & (W-9)),
     * columns clamped with IMG_HEIGHT/2 and rows with IMG_WIDTH/2.  Reads that
     * the reference makes past the end of the caller's image allocation
     * (tp_geometry.image_rows rows of dstride floats) read the allocation's last
     * float instead; every other read is at the reference's address. */
    TP_BORDER_REFERENCE = 0,
    /* Same corner logic with the precedence fixed, and every pixel clamped
     * into the image by Bayer pairs (columns to W, rows to H). */
    TP_BORDER_CLAMP = 1
};

/* Runtime geometry (the reference's compile-time defines). */
typedef struct tp_geometry {
    int img_width;      /* IMG_WIDTH, multiple of 8, >= 32                     */
    int img_height;     /* IMG_HEIGHT, multiple of 8, >= 32                    */
    int kernels_hor;    /* KERNELS_HOR   (kernel-table columns)                */
    int kernels_vert;   /* KERNELS_VERT  (kernel-table rows)                   */
    int kernels_lstep;  /* KERNELS_LSTEP (kernel grid step = 1 << lstep px)    */
    int image_rows;     /* rows allocated per source image, >= img_height      */
    int border_mode;    /* TP_BORDER_REFERENCE or TP_BORDER_CLAMP              */
    int debug_marks;    /* 1: imclt_rbg also makes the reference's debug writes
                           (tile (0,0) := 100, tile (161,111) doubled,
                           src/TileProcessor.cuh:2687-2700); 0: plain output */
} tp_geometry;

/* Status codes. */
enum {
    TP_OK            = 0,
    TP_ERR_ARG       = -1, /* NULL pointer, negative count, bad stride/radius  */
    TP_ERR_GEOMETRY  = -2, /* inconsistent tp_geometry                         */
    TP_ERR_CUDA      = -3, /* a CUDA runtime call or launch failed             */
    TP_ERR_UNSUPPORTED = -4, /* valid in the reference, not in this build      */
    TP_ERR_NO_DEVICE = -5  /* no CUDA device visible                           */
};

/* One-line description of the last error on the calling thread. */
const char *tp_last_error(void);
/* Library version string. */
const char *tp_version(void);

/* Tiles per row / column (TILESX, TILESY, TILESYA of src/TileProcessor.cuh:146-149). */
int tp_tiles_x(const tp_geometry *g);
int tp_tiles_y(const tp_geometry *g);
int tp_tiles_ya(const tp_geometry *g);

/* ---- constant tables --------------------------------------------------------
 * The reference keeps its low-pass filters in __constant__ memory and lets the
 * caller overwrite them with cudaMemcpyToSymbol (src/TileProcessor.cuh:421-481).
 * which: 0..3 = lpf_data[0..3] (R, B, G, mono), 4 = lpf_rb_corr, 5 = lpf_corr.
 * values: 64 floats, row-major 8x8.  Applies to the current CUDA device. */
int tp_set_lpf(int which, const float *values);
int tp_get_lpf(int which, float *values);
/* Restore the built-in tables on the current device. */
int tp_reset_lpf(void);

/* ---- launch shapes ----------------------------------------------------------
 * No counterpart in the reference (its launches are fixed).  The stage kernels
 * walk their work items with grid-stride loops over a grid capped at
 * ctas_per_sm x the SM count; the cap sets how many tiles each CTA takes in
 * turn.  0 restores the built-in value (convert 8, correlate 8, textures 7).
 * Process-wide, read at every launch (a CUDA graph keeps the shape it was
 * captured with).  tile_processor_gpu_b200.autotune picks the value by timing
 * the caller's workload. */
enum {
    TP_SHAPE_CONVERT = 0,   /* k_convert_correct_tiles (tp_convert_correct_tiles) */
    TP_SHAPE_CORRELATE = 1, /* k_correlate2D (tp_correlate2D)                     */
    TP_SHAPE_TEXTURES = 2,  /* k_textures (tp_textures_accumulate, generate_RBGA) */
    TP_SHAPE_COUNT = 3
};
#define TP_MAX_CTAS_PER_SM 32
/* TP_ERR_ARG for an unknown kernel or a value outside 0..TP_MAX_CTAS_PER_SM */
int tp_set_launch_shape(int kernel, int ctas_per_sm);
/* the value in use (the built-in one when unset), TP_ERR_ARG for an unknown kernel */
int tp_get_launch_shape(int kernel);
/* how many CTAs of the stage kernel fit on one SM at once (its registers,
 * block size and shared memory); caps above it only add waves */
int tp_resident_ctas(int kernel);

/* ---- forward CLT with aberration correction ---------------------------------
 * Replaces convert_correct_tiles (src/TileProcessor.cuh:1859-1937).
 * kernel_offsets : device array [4] of device tp_clt_extra[kv*kh*3]
 * kernels        : device array [4] of device float[kv*kh*3*4*64]
 * images         : device array [4] of device float[image_rows][dstride]
 * tasks          : device tp_task[num_tiles]; tasks with task == 0 are skipped
 * clt            : device array [4] of device float[tilesy*tilesx*3*4*64]
 * lpf_mask       : bit c applies lpf_data[c] to color c */
int tp_convert_correct_tiles(const tp_geometry *g,
                             float *const *kernel_offsets,
                             float *const *kernels,
                             float *const *images,
                             const tp_task *tasks,
                             float *const *clt,
                             size_t dstride,
                             int num_tiles,
                             int lpf_mask,
                             tp_stream_t stream);
/* The same operation with the Bayer windows staged in shared memory by the
 * TMA unit (one producer warp computes each job's geometry and bulk-copies
 * the 16 x 20 window at the 16-byte boundary left of its corner; consumer
 * warps fold from shared memory and finish the jobs; windows that reach the
 * image border, or images not on 16-byte boundaries or with dstride not a
 * multiple of 4, take the global-memory path).  The CLT is bit-identical to
 * tp_convert_correct_tiles'.  A bounded wait that runs out leaves the CLT
 * incomplete and is reported by tp_tc_status. */
int tp_convert_correct_tiles_tma(const tp_geometry *g, float *const *kernel_offsets, float *const *kernels,
                                 float *const *images, const tp_task *tasks, float *const *clt, size_t dstride,
                                 int num_tiles, int lpf_mask, tp_stream_t stream);

/* ---- pairwise phase correlation ---------------------------------------------
 * Replaces correlate2D (src/TileProcessor.cuh:1176-1443).
 * corr_indices : device int[num_corr_tiles], (tile << 8) | pair, pair 0..5
 * corrs        : device float, tile i's (2r+1)^2 floats at corrs + i*corr_stride */
int tp_correlate2D(const tp_geometry *g,
                   float *const *clt,
                   int colors,
                   float scale0, float scale1, float scale2,
                   float fat_zero,
                   size_t num_corr_tiles,
                   const int *corr_indices,
                   size_t corr_stride,
                   int corr_radius,
                   float *corrs,
                   tp_stream_t stream);

/* ---- texture tiles -----------------------------------------------------------
 * Replaces textures_accumulate (src/TileProcessor.cuh:2207-2579).
 * texture_indices : device int[num_texture_tiles], (tile << 8) | (1 << 7) | nbr
 * woi             : device int[4] {x, y, width, height} in tiles (read only
 *                   when texture_rbg is used)
 * port_offsets    : device float[4][2]
 * texture_rbg     : overlapped RGBA image, += (NULL or stride 0 = skip)
 * texture_tiles   : non-overlapped 16x16 tiles, tile i at i*texture_stride
 *                   (NULL or stride 0 = skip) */
int tp_textures_accumulate(const tp_geometry *g,
                           const int *woi,
                           float *const *clt,
                           size_t num_texture_tiles,
                           const int *texture_indices,
                           const float *port_offsets,
                           int colors, int is_lwir,
                           float min_shot, float scale_shot,
                           float diff_sigma, float diff_threshold,
                           float min_agree,
                           float weight0, float weight1, float weight2,
                           int dust_remove, int keep_weights,
                           size_t texture_rbg_stride, float *texture_rbg,
                           size_t texture_stride, float *texture_tiles,
                           tp_stream_t stream);

/* ---- inverse CLT into an image -----------------------------------------------
 * Replaces imclt_rbg (src/TileProcessor.cuh:2588-2710): one of the 4 parity
 * passes of one color plane.  rbg: device float[3*(H+8)][dstride], dstride >=
 * W + 8.  Pass (0,0) overwrites, the others accumulate. */
int tp_imclt_rbg(const tp_geometry *g,
                 const float *clt_one_cam,
                 float *rbg,
                 int color, int v_offset, int h_offset,
                 size_t dstride,
                 tp_stream_t stream);
/* All 3 colors x 4 passes of one camera in the order the reference's driver
 * issues them (src/dtt8x8.cu:624-662), in one call. */
int tp_imclt_rbg_all(const tp_geometry *g,
                     const float *clt_one_cam,
                     float *rbg,
                     size_t dstride,
                     tp_stream_t stream);

/* ---- texture list and RGBA driver --------------------------------------------
 * Replace the dynamic-parallelism drivers prepare_texture_list
 * (src/TileProcessor.cuh:1643-1713) and generate_RBGA (:1446-1615) with
 * host-launched kernels on one stream (no device-side launches, no host sync).
 * texture_indices   : device int[tilesx * tilesya]
 * num_texture_tiles : device int[8] (inner/border count per 2x2 parity)
 * woi               : device int[4] -> {x, y, width, height} in tiles
 * Within a sub-list, entries claimed by one warp are in task order; across
 * warps the order is the order in which their atomicAdds land (the reference's
 * order depends on atomicAdd order too).  Tiles of one sub-list never overlap,
 * so no output depends on the order.
 * tasks' bits 0..3 are rewritten with the N/E/S/W neighbour mask, as in the
 * reference. */
int tp_prepare_texture_list(const tp_geometry *g,
                            tp_task *tasks, int num_tiles,
                            int *texture_indices, int *num_texture_tiles,
                            int *woi, int width, int height,
                            tp_stream_t stream);

int tp_clear_texture_rbga(const tp_geometry *g,
                          int texture_width, int texture_slice_height,
                          size_t texture_rbga_stride, float *texture_tiles,
                          tp_stream_t stream);

int tp_generate_RBGA(const tp_geometry *g,
                     tp_task *tasks, int num_tiles,
                     int *texture_indices, int *num_texture_tiles,
                     int *woi, int width, int height,
                     float *const *clt,
                     const float *port_offsets,
                     int colors, int is_lwir,
                     float min_shot, float scale_shot,
                     float diff_sigma, float diff_threshold,
                     float min_agree,
                     float weight0, float weight1, float weight2,
                     int dust_remove, int keep_weights,
                     size_t texture_rbga_stride, float *texture_tiles,
                     tp_stream_t stream);

/* ---- generate_RBGA with library-owned list scratch ------------------------------
 * No counterpart in the reference: the same work as tp_generate_RBGA, but the
 * texture list, its eight sub-list counts and the window of interest live in
 * a fixed device array inside the library instead of caller buffers, so a
 * caller that cannot allocate device memory can still run the call: a
 * real-time frame loop that must not call cudaMalloc (it synchronises the
 * whole device and stalls the other streams), or a host binding such as the
 * reference's Java plugin that reaches the GPU only through buffers it was
 * handed and has no device allocator of its own.  Limits and rules:
 *   - scratch: TP_NOALLOC_SCRATCH_INTS ints (1 MiB); frames whose list needs
 *     more (tilesx * tilesy rounded up to 4 rows, + 16) are rejected with
 *     TP_ERR_ARG before any device work;
 *   - the first call on a device, with that device current, looks the
 *     array up (cudaGetSymbolAddress) once; make that first call before any
 *     stream capture;
 *   - the address is kept with the id of the context it was found in; after
 *     a device reset the next call looks it up again;
 *   - every call shares the array and leaves its contents behind; nothing in
 *     it needs to start at zero: each call clears the tile-marker grid over
 *     the whole frame (not only the width x height extent, which is checked
 *     but otherwise unused), so a call whose tasks lie inside the frame gets
 *     the result of tp_generate_RBGA on freshly zeroed buffers, and it resets
 *     the counts and the window; calls that overlap on the GPU race:
 *     serialise them (one stream, or events);
 *   - tasks' bits 0..3 are rewritten with the neighbour mask, as in
 *     tp_generate_RBGA; the window of interest is not returned. */
#define TP_NOALLOC_SCRATCH_INTS (1 << 18)
int tp_generate_RBGA_noalloc(const tp_geometry *g,
                             tp_task *tasks, int num_tiles,
                             int width, int height,
                             float *const *clt,
                             const float *port_offsets,
                             int colors, int is_lwir,
                             float min_shot, float scale_shot,
                             float diff_sigma, float diff_threshold,
                             float min_agree,
                             float weight0, float weight1, float weight2,
                             int dust_remove, int keep_weights,
                             size_t texture_rbga_stride, float *texture_tiles,
                             tp_stream_t stream);

/* generate_RBGA for one band of tile rows of a frame split across GPUs.  No
 * counterpart in the reference (one GPU per frame there).  Every task passed
 * in is marked as a texture tile, so it sets its neighbours' bits and the
 * window of interest, but only tiles of rows [row_first, row_last) are listed
 * and accumulated; passing the band's rows plus one tile row above and below
 * gives the band's tiles the neighbour bits, border classes and alpha fade they
 * have in the whole frame.  The RGBA image is relative to the band's window of
 * interest (woi[1] = row_first - 1 unless row_first is the frame's first row);
 * the 8 pixel rows the band's last tile row adds below row_last * 8 belong to
 * the next band, which adds them to its own (one strip exchange).  The
 * parameters the reference passes through unused (is_lwir, diff_threshold,
 * min_agree, keep_weights) are left out. */
int tp_generate_RBGA_rows(const tp_geometry *g, tp_task *tasks, int num_tiles, int *texture_indices,
                          int *num_texture_tiles, int *woi, int width, int height, float *const *clt,
                          const float *port_offsets, int colors, float min_shot, float scale_shot,
                          float diff_sigma, float weight0, float weight1, float weight2, int dust_remove,
                          size_t texture_rbga_stride, float *texture_tiles, int row_first, int row_last,
                          tp_stream_t stream);

/* ---- the whole hot path for one frame ------------------------------------------
 * No single counterpart in the reference: it runs convert_correct_tiles,
 * correlate2D and generate_RBGA (src/TileProcessor.cuh:1859-1937, :1176-1443,
 * :1446-1615) through a device CLT buffer.  Here every tile is converted,
 * correlated and textured by one block with its CLT in shared memory, in four
 * launches by 2x2 tile parity.  Same inputs as tp_convert_correct_tiles, then:
 *   corrs   : device float[num_tiles][6][corr_stride]; slot (n, pair) holds
 *             the (2r+1)^2 correlation of task n's pair when bit 4+pair of
 *             its task is set (other slots untouched)
 *   texture : the texture list and window of interest of tp_generate_RBGA
 *             (texture_indices, num_texture_tiles, woi; tasks' bits 0..3
 *             rewritten with the neighbour mask) and its overlapped RGBA
 *             image, 3 colours + alpha (keep_weights = 0)
 *   clt     : optional (NULL = not written) CLT output, layout of
 *             tp_convert_correct_tiles */
int tp_process_frame(const tp_geometry *g,
                     float *const *kernel_offsets, float *const *kernels, float *const *images,
                     size_t dstride, tp_task *tasks, int num_tiles, int lpf_mask,
                     int corr_colors, float corr_scale0, float corr_scale1, float corr_scale2,
                     float fat_zero, int corr_radius, size_t corr_stride, float *corrs,
                     const float *port_offsets, float min_shot, float scale_shot, float diff_sigma,
                     float weight0, float weight1, float weight2, int dust_remove,
                     int *texture_indices, int *num_texture_tiles, int *woi,
                     size_t texture_rbga_stride, float *texture_rbga,
                     float *const *clt,
                     tp_stream_t stream);

/* ---- disparity from the pair correlations ---------------------------------------
 * No counterpart in the reference, which hands its correlation tiles to the
 * Java caller (src/TileProcessor.cuh:1176-1443 is where it stops).  For each
 * tile with listed pairs (entries of one tile adjacent in corr_indices, as
 * the correlation lists are built), the profile
 *   S(k) = sum over its pairs p in pair_mask of C_p(k * b_p),  k = -r..r,
 * b_p = port_offsets[j] - port_offsets[i] for pair p = (i, j), C_p sampled
 * bilinearly in the centred (2r+1)^2 tile, is maximised to sub-pixel precision
 * (double precision) around its first integer maximum:
 *   mode 0: 3-point parabola; 1: 5-point least-squares parabola; 2: 3-point
 *   centroid; the sub-pixel step stays within +-1.
 * disparity[tile] = the residual disparity rho (true minus task disparity, in
 * pixels per unit of port offset: pair p peaks at rho * b_p); strength[tile]
 * = the fitted peak per pair.  Both are device float[tilesx * tilesy], written
 * only for fitted tiles.  corrs / corr_stride / corr_radius / corr_indices
 * as tp_correlate2D's output. */
int tp_disparity_fit(const tp_geometry *g,
                     const float *corrs, size_t corr_stride, int corr_radius,
                     size_t num_corr_tiles, const int *corr_indices,
                     const float *port_offsets, int pair_mask, int mode,
                     float *disparity, float *strength,
                     tp_stream_t stream);

/* ---- CLT kernel tables from spatial kernels ------------------------------------
 * No counterpart in the reference, which reads its tables from files its Java
 * caller writes (src/dtt8x8.cu:228-238).  psf: device float[n][15][15],
 * kernel taps -7..7 (rows vertical); clt_kernels: device float[n][4][8][8],
 * the entry layout of the tables tp_convert_correct_tiles reads (n =
 * kernels_vert * kernels_hor * 3 for one camera's table).  K_q[u][v] =
 * sum_mn h[m][n] A(u, m) B(v, n) with A/B = cos or sin(pi tap (2k+1) / 16)
 * (cosine vertical for CC/SC, horizontal for CC/CS), accumulated in double.
 * The CLT-domain product approximates the spatial convolution (exact for a
 * single centre tap; 1.5e-4 relative for a sigma-0.3 px Gaussian, 4% at
 * 1 px). */
int tp_psf_to_clt(const float *psf, size_t n, float *clt_kernels, tp_stream_t stream);

/* ---- host helpers for the reference harness's files and lists ------------------
 * Raw native-endian float32 files without headers (src/dtt8x8.cu:144-165):
 * returns the number of floats read / written, or TP_ERR_ARG. */
long long tp_read_floats(const char *path, float *dst, size_t count);
long long tp_write_floats(const char *path, const float *src, size_t count);
/* The harness's task list (src/dtt8x8.cu:415-428): one task per tile in
 * linescan order, bits task_bits, xy[cam] from portsxy[cam] (host
 * float[tilesy * tilesx][2], the *.portsxy files).  tasks: host array of
 * tilesx * tilesy.  Returns the number of tasks. */
int tp_tasks_from_portsxy(const float *const *portsxy, int tilesx, int tilesy, int task_bits, tp_task *tasks);
/* The harness's correlation list (src/dtt8x8.cu:432-446): (tile << 8) | pair
 * for every pair bit of every task, in task order (host arrays; NULL
 * corr_indices only counts).  Returns the number of entries. */
int tp_corr_indices_from_tasks(const tp_task *tasks, int num_tiles, int tilesx, int *corr_indices);

/* ---- learned disparity residual -------------------------------------------------
 * No counterpart in the reference (its Java caller, absent, fits disparity).
 * A small MLP refines tp_disparity_fit: features = a tile's six (2r+1)^2
 * correlation planes scaled by their largest magnitude; network 6(2r+1)^2 ->
 * 256 -> 128 -> 2 with GELU; outputs a correction to the plain fit and a
 * log-variance.  These are its building blocks (device pointers, row-major
 * float32, rows = samples); tile_processor_gpu_b200.disparity_net drives
 * them for inference and training. */
/* features[tile][p * (2r+1)^2 + k]: the tile's run of correlation entries
 * (adjacent in corr_indices), pair p in slot p, unlisted pairs zero; rows of
 * tiles without entries are not written.  feature_stride >= 6 (2r+1)^2. */
int tp_mlp_features(const tp_geometry *g, const float *corrs, size_t corr_stride, int corr_radius,
                    size_t num_corr_tiles, const int *corr_indices, float *features, size_t feature_stride,
                    tp_stream_t stream);
/* C = beta C + op(A) op(B) (+ bias), op(A) M x K (A[m][k], or A[k][m] when
 * trans_a), op(B) K x N; with z non-NULL, z = that pre-activation and
 * C = gelu(z) (exact, erf form). */
int tp_mlp_gemm(int M, int N, int K, const float *A, int lda, int trans_a, const float *B, int ldb, int trans_b,
                float beta, float *C, int ldc, const float *bias, float *z, int ldz, tp_stream_t stream);
/* The same operation on the tensor cores: each FP32 operand split into two
 * TF32 parts (hi = tf32(x), lo = tf32(x - hi)), each product as three tcgen05
 * TF32 MMAs (hi hi + hi lo + lo hi) accumulated in FP32 (about 21 significant
 * bits per operand), tiles of 128 x 64 of C.  err (device int, may be NULL) is
 * set to 1 if a wait for the tensor cores ran out (C is then not written). */
int tp_mlp_gemm_tc(int M, int N, int K, const float *A, int lda, int trans_a, const float *B, int ldb, int trans_b,
                   float beta, float *C, int ldc, const float *bias, float *z, int ldz, int *err,
                   tp_stream_t stream);
/* dz = dh * gelu'(z), rows x cols, leading dimension ld */
int tp_mlp_gelu_backward(int rows, int cols, int ld, const float *z, const float *dh, float *dz,
                         tp_stream_t stream);
/* out[c] = scale * sum over rows of x[r][c] */
int tp_mlp_colsum(int rows, int cols, int ld, const float *x, float scale, float *out, tp_stream_t stream);
/* Gaussian negative log-likelihood of out[r] = {d, s} against target[r]:
 * loss_rows[r] = w[r] (0.5 exp(-s) (d - target)^2 + 0.5 s), s clamped to
 * [-12, 12]; dout = the gradient of inv_count * sum loss_rows.  w may be NULL
 * (all ones). */
int tp_mlp_nll(int rows, const float *out, const float *target, const float *w, float inv_count, float *dout,
               float *loss_rows, tp_stream_t stream);
/* Inference on the tensor cores: the weights packed once per update
 * (w1t: device float [43 * 256 * 32], W1^T rounded to TF32 in 43 blocks of
 * 32 rows of K, each block the shared-memory image of a tcgen05 B operand;
 * w2t: device uint16 [128 * 256], W2^T in BF16, the same kind of image;
 * both 16-byte aligned), then out[r] = {d, s} for feature rows x (rows x
 * 1350, leading dimension ldx), layer 1 as TF32 and layer 2 as BF16 tcgen05
 * MMAs with FP32 accumulation, the features fetched by TMA.  Rows of x must
 * start on 16-byte boundaries (x 16-byte aligned, ldx a multiple of 4), else
 * TP_ERR_ARG.  err (device int, may be NULL) is set to 1 if a wait for the
 * copies or the tensor cores ran out (no result then). */
int tp_mlp_pack(const float *W1, const float *W2, void *w1t, void *w2t, tp_stream_t stream);
int tp_mlp_infer_tc(int rows, const float *x, int ldx, const void *w1t, const float *b1, const void *w2t,
                    const float *b2, const float *W3, const float *b3, float *out, int *err, tp_stream_t stream);
/* The learned estimate with the plain fit as its fallback: rho[i] = plain[i]
 * + out[i].d where out[i].s (the log-variance) < gate, else plain[i]; out is
 * the {d, s} pairs of tp_mlp_infer_tc (8-byte aligned).  gate = +inf keeps
 * every correction. */
int tp_mlp_combine(size_t n, const float *plain, const float *out, float gate, float *rho, tp_stream_t stream);
/* Adam step `step` (1, 2, ...) on n parameters */
int tp_mlp_adam(size_t n, float *param, const float *grad, float *m, float *v, float lr, float beta1, float beta2,
                float eps, int step, tp_stream_t stream);

/* ---- tensor-core precision forms of the stages ----------------------------------
 * The same calls as above, with each stage's batched 8x8 transforms (the
 * DCT-IV / DST-IV / DCT-II / DST-II pairs of src/dtt8x8.cuh:382-463,
 * :621-745 on every quadrant) run as tcgen05 GEMMs: 64 x 64 matrices per
 * quadrant, operands split into two 16-bit halves (hi + lo), three MMAs per
 * product, FP32 accumulation in tensor memory.  The element-wise steps (CLT
 * products, normalisation, LPFs, unfolds) are the plain path's.  `format`:
 *   TP_TC_FP16X2  FP16 halves (22 significant bits; rows scaled by a power of
 *                 two to stay in FP16 range)
 *   TP_TC_BF16X2  BF16 halves (16 significant bits, no scaling)
 * The first call on a device copies the transform tables to it (synchronous;
 * make it before any stream capture).  A bounded wait inside a kernel that
 * runs out leaves that kernel's outputs incomplete and is reported by
 * tp_tc_status. */
#define TP_TC_FP16X2 0
#define TP_TC_BF16X2 1
/* convert_correct_tiles (src/TileProcessor.cuh:1859-1937), same arguments:
 * the 2-D DCT-IV (and for green the DST-IV x DCT-IV) of each folded tile on
 * the tensor cores; fold, kernel convolution, shifts and LPF as the plain
 * path */
int tp_convert_correct_tiles_tc(const tp_geometry *g,
                                float *const *kernel_offsets,
                                float *const *kernels,
                                float *const *images,
                                const tp_task *tasks,
                                float *const *clt,
                                size_t dstride,
                                int num_tiles,
                                int lpf_mask,
                                int format,
                                tp_stream_t stream);
/* correlate2D (src/TileProcessor.cuh:1176-1443), same arguments */
int tp_correlate2D_tc(const tp_geometry *g,
                      float *const *clt,
                      int colors,
                      float scale0, float scale1, float scale2,
                      float fat_zero,
                      size_t num_corr_tiles,
                      const int *corr_indices,
                      size_t corr_stride,
                      int corr_radius,
                      float *corrs,
                      int format,
                      tp_stream_t stream);
/* textures_accumulate (src/TileProcessor.cuh:2207-2579) and generate_RBGA
 * (:1446-1615), same arguments, plus tile_scratch: a device array [4] of
 * per-camera buffers of the CLT's size and layout ([tilesy * tilesx][3][256]
 * floats) that receive each listed job's inverse CLT, computed on the tensor
 * cores, before the debayer and camera fusion read it. */
int tp_textures_accumulate_tc(const tp_geometry *g,
                              const int *woi,
                              float *const *clt,
                              size_t num_texture_tiles,
                              const int *texture_indices,
                              const float *port_offsets,
                              int colors, int is_lwir,
                              float min_shot, float scale_shot,
                              float diff_sigma, float diff_threshold,
                              float min_agree,
                              float weight0, float weight1, float weight2,
                              int dust_remove, int keep_weights,
                              size_t texture_rbg_stride, float *texture_rbg,
                              size_t texture_stride, float *texture_tiles,
                              float *const *tile_scratch,
                              int format,
                              tp_stream_t stream);
int tp_generate_RBGA_tc(const tp_geometry *g,
                        tp_task *tasks, int num_tiles,
                        int *texture_indices, int *num_texture_tiles,
                        int *woi, int width, int height,
                        float *const *clt,
                        const float *port_offsets,
                        int colors, int is_lwir,
                        float min_shot, float scale_shot,
                        float diff_sigma, float diff_threshold,
                        float min_agree,
                        float weight0, float weight1, float weight2,
                        int dust_remove, int keep_weights,
                        size_t texture_rbga_stride, float *texture_tiles,
                        float *const *tile_scratch,
                        int format,
                        tp_stream_t stream);
/* *timed_out = 1 when a tensor-core stage kernel's (or the TMA-fed convert
 * kernel's) wait ran out since the last clear (synchronous); clear != 0
 * resets it.  No counterpart in the reference. */
int tp_tc_status(int *timed_out, int clear);
/* The 64 KB shared-memory image of a stage's split transform matrices
 * (stage 0 correlation, 1 inverse CLT, 2 forward CLT): uint16 halves, the
 * four hi quadrants then the four lo, each 64 rows x 64 K, 128-byte
 * swizzled.  Host only (no device needed); for checking and inspection.  No
 * counterpart in the reference. */
int tp_tc_table_image(int format, int stage, void *out);

#ifdef __cplusplus
}
#endif
#endif /* TP_B200_H */

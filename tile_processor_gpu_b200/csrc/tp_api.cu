/*
 * tp_api.cu - C ABI of the B200 tile processor (declared in include/tp_b200.h).
 *
 * Each entry point checks its host-visible arguments, converts the geometry,
 * sizes the grid from the device's SM count and launches on the caller's
 * stream.  Nothing here allocates, synchronises or copies device data to the
 * host.
 */
#include <utility>
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>
#include <float.h>
#include <limits.h>
#include <math.h>
#include <atomic>
#include <mutex>
#include <stdarg.h>
#include <stdio.h>
#include <string.h>

#include "tp_common.cuh"
#include "tp_convert.cuh"
#include "tp_correlate.cuh"
#include "tp_texture.cuh"
#include "tp_imclt.cuh"
#include "tp_list.cuh"
#include "tp_frame.cuh"
#include "tp_disparity.cuh"
#include "tp_kernels_gen.cuh"
#include "tp_corr_tc.cuh"
#include "tp_inv_tc.cuh"
#include "tp_fwd_tc.cuh"
#include "tp_mlp.cuh"
#include "tp_gemm_tc.cuh"
#include "tp_convert_tma.cuh"

#define TP_VERSION "tile_processor_gpu_b200 0.1 (sm_100a)"

namespace {

thread_local char g_err[512] = "no error";

int fail(int code, const char *fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
    return code;
}

int cuda_status(cudaError_t e, const char *what)
{
    if (e != cudaSuccess) return fail(TP_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
    return TP_OK;
}

int check_geometry(const tp_geometry *g, tp::Geom *out)
{
    if (!g) return fail(TP_ERR_ARG, "geometry is NULL");
    if (g->img_width < 32 || g->img_height < 32 || (g->img_width & 7) || (g->img_height & 7))
        return fail(TP_ERR_GEOMETRY, "image %dx%d: width and height must be multiples of 8, >= 32",
                    g->img_width, g->img_height);
    if (g->img_width > (1 << 15) || g->img_height > (1 << 15))
        return fail(TP_ERR_GEOMETRY, "image %dx%d exceeds 32768", g->img_width, g->img_height);
    if (g->kernels_lstep < 1 || g->kernels_lstep > 8)
        return fail(TP_ERR_GEOMETRY, "kernels_lstep %d outside 1..8", g->kernels_lstep);
    if (g->kernels_hor < 1 || g->kernels_vert < 1)
        return fail(TP_ERR_GEOMETRY, "kernel grid %dx%d", g->kernels_hor, g->kernels_vert);
    if (g->image_rows < g->img_height)
        return fail(TP_ERR_GEOMETRY, "image_rows %d < img_height %d", g->image_rows, g->img_height);
    if (g->border_mode != TP_BORDER_REFERENCE && g->border_mode != TP_BORDER_CLAMP)
        return fail(TP_ERR_GEOMETRY, "border_mode %d", g->border_mode);
    out->W = g->img_width;
    out->H = g->img_height;
    out->TX = g->img_width / 8;
    out->TY = g->img_height / 8;
    out->TYA = (out->TY + 3) & ~3;
    out->KH = g->kernels_hor;
    out->KV = g->kernels_vert;
    out->ls = g->kernels_lstep;
    out->image_rows = g->image_rows;
    out->border_mode = g->border_mode;
    out->debug_marks = g->debug_marks ? 1 : 0;
    return TP_OK;
}

int sm_count(int *n)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return fail(TP_ERR_NO_DEVICE, "cudaGetDevice: %s", cudaGetErrorString(e));
    e = cudaDeviceGetAttribute(n, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return fail(TP_ERR_NO_DEVICE, "SM count: %s", cudaGetErrorString(e));
    return TP_OK;
}

/* blocks for a grid-stride kernel: enough to fill every SM `per_sm` times */
unsigned grid_for(long long items, int items_per_block, int sms, int per_sm)
{
    long long need = (items + items_per_block - 1) / items_per_block;
    long long cap = (long long)sms * per_sm;
    if (need > cap) need = cap;
    if (need < 1) need = 1;
    return (unsigned)need;
}

/* grid caps of the stage kernels in CTAs per SM (0 = the built-in value) */
std::atomic<int> g_shape[TP_SHAPE_COUNT];
const int g_shape_default[TP_SHAPE_COUNT] = {8, 8, 7};

int shape_per_sm(int which)
{
    const int v = g_shape[which].load(std::memory_order_relaxed);
    return v > 0 ? v : g_shape_default[which];
}

/* Kernels taking more shared memory than the 48 KB granted by default get
 * their attribute once per device (the first call; make it before capturing
 * a stream into a graph). */
std::mutex g_attr_mutex;
bool g_tex_attr[8][128], g_frame_attr[128], g_tc_attr[128], g_gemm_tc_attr[128], g_cv_attr[128];

int set_smem_once(bool *done, const void *func, size_t bytes, const char *what)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return fail(TP_ERR_NO_DEVICE, "cudaGetDevice: %s", cudaGetErrorString(e));
    if (dev < 0 || dev >= 128) return fail(TP_ERR_NO_DEVICE, "device %d", dev);
    std::lock_guard<std::mutex> lock(g_attr_mutex);
    if (done[dev]) return TP_OK;
    const int rc = cuda_status(cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes),
                               what);
    if (!rc) done[dev] = true;
    return rc;
}

/* the texture kernel for a colour count (1 or 3, checked by the caller) */
template <bool FROM_T, bool ALL>
static auto tex_kernel(int colors)
{
    return colors == 3 ? tp::k_textures<FROM_T, ALL, 3> : tp::k_textures<FROM_T, ALL, 1>;
}

int texture_smem_setup()
{
    const void *const kernels[8] = {
        (const void *)tp::k_textures<false, true, 1>,  (const void *)tp::k_textures<false, true, 3>,
        (const void *)tp::k_textures<true, true, 1>,   (const void *)tp::k_textures<true, true, 3>,
        (const void *)tp::k_textures<false, false, 1>, (const void *)tp::k_textures<false, false, 3>,
        (const void *)tp::k_textures<true, false, 1>,  (const void *)tp::k_textures<true, false, 3>};
    int rc = TP_OK;
    for (int i = 0; i < 8 && !rc; i++)
        rc = set_smem_once(g_tex_attr[i], kernels[i], tp::kTexSmemBytes, "cudaFuncSetAttribute(k_textures)");
    return rc;
}

/* Scratch of tp_generate_RBGA_noalloc: [0, 8) sub-list counts, [8, 12) window
 * of interest, [16, ...) the texture list and its tile-marker grid.  Needs no
 * initial contents: every call clears the whole marker grid it reads. */
static __device__ __align__(256) int g_rbga_scratch[TP_NOALLOC_SCRATCH_INTS];

/* Per-device address of g_rbga_scratch, looked up on the first call on that
 * device, together with the unique id of the context it belongs to.  A
 * device reset destroys the primary context and the module with it; the next
 * call then sees a new context id and looks the array up again instead of
 * handing the kernels an address of the old context. */
std::mutex g_scratch_mutex;
int *g_scratch_ptr[128];
unsigned long long g_scratch_ctx[128];
typedef CUresult (*PFN_ctx_get_current)(CUcontext *);
typedef CUresult (*PFN_ctx_get_id)(CUcontext, unsigned long long *);

/* unique id of the calling thread's current context (0 when unavailable) */
unsigned long long current_context_id()
{
    static PFN_ctx_get_current get_current = nullptr;
    static PFN_ctx_get_id get_id = nullptr;
    static bool looked_up = false;
    if (!looked_up) {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_current = reinterpret_cast<PFN_ctx_get_current>(p);
        p = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_id = reinterpret_cast<PFN_ctx_get_id>(p);
        looked_up = true;
    }
    CUcontext ctx = nullptr;
    unsigned long long id = 0;
    if (!get_current || !get_id || get_current(&ctx) != CUDA_SUCCESS || !ctx || get_id(ctx, &id) != CUDA_SUCCESS)
        return 0;
    return id;
}

int noalloc_scratch(int **out)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return fail(TP_ERR_NO_DEVICE, "cudaGetDevice: %s", cudaGetErrorString(e));
    if (dev < 0 || dev >= 128) return fail(TP_ERR_NO_DEVICE, "device %d", dev);
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    /* 0 when this thread has no current context yet: the lookup below makes
     * the device's primary context current, and its id is read after it */
    const unsigned long long ctx = current_context_id();
    if (!g_scratch_ptr[dev] || ctx == 0 || ctx != g_scratch_ctx[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_rbga_scratch);
        if (e != cudaSuccess) return fail(TP_ERR_CUDA, "cudaGetSymbolAddress(scratch): %s", cudaGetErrorString(e));
        g_scratch_ptr[dev] = static_cast<int *>(p);
        g_scratch_ctx[dev] = current_context_id();
    }
    *out = g_scratch_ptr[dev];
    return TP_OK;
}

/* host copy of the low-pass tables (last values set by tp_set_lpf) */
float g_lpf_host[6][64] = TP_LPF_DEFAULT_INIT;
const float g_lpf_default[6][64] = TP_LPF_DEFAULT_INIT;

/* cuTensorMapEncodeTiled from the driver, looked up once */
std::mutex g_tmap_mutex;
PFN_cuTensorMapEncodeTiled_v12000 g_encode_tiled = nullptr;

int tensor_map_encoder(PFN_cuTensorMapEncodeTiled_v12000 *fn)
{
    std::lock_guard<std::mutex> lock(g_tmap_mutex);
    if (!g_encode_tiled) {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        const cudaError_t e = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q);
        if (e != cudaSuccess || q != cudaDriverEntryPointSuccess || !p)
            return fail(TP_ERR_CUDA, "cuTensorMapEncodeTiled not available (%s)", cudaGetErrorString(e));
        g_encode_tiled = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }
    *fn = g_encode_tiled;
    return TP_OK;
}

} /* namespace */

extern "C" {

const char *tp_last_error(void) { return g_err; }

int tp_set_launch_shape(int kernel, int ctas_per_sm)
{
    if (kernel < 0 || kernel >= TP_SHAPE_COUNT) return fail(TP_ERR_ARG, "launch shape kernel %d", kernel);
    if (ctas_per_sm < 0 || ctas_per_sm > TP_MAX_CTAS_PER_SM)
        return fail(TP_ERR_ARG, "ctas_per_sm %d outside 0..%d", ctas_per_sm, TP_MAX_CTAS_PER_SM);
    g_shape[kernel].store(ctas_per_sm, std::memory_order_relaxed);
    return TP_OK;
}

int tp_get_launch_shape(int kernel)
{
    if (kernel < 0 || kernel >= TP_SHAPE_COUNT) return fail(TP_ERR_ARG, "launch shape kernel %d", kernel);
    return shape_per_sm(kernel);
}

int tp_resident_ctas(int kernel)
{
    if (kernel < 0 || kernel >= TP_SHAPE_COUNT) return fail(TP_ERR_ARG, "launch shape kernel %d", kernel);
    int n = 0, rc;
    cudaError_t e;
    if (kernel == TP_SHAPE_CONVERT) {
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, tp::k_convert_correct_tiles, 256, 0);
    } else if (kernel == TP_SHAPE_CORRELATE) {
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, tp::k_correlate2D, 128, 0);
    } else {
        if ((rc = texture_smem_setup())) return rc;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, tp::k_textures<false, false, 3>, tp::kTexThreads,
                                                          tp::kTexSmemBytes);
    }
    if (e != cudaSuccess) return cuda_status(e, "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
    return n;
}
const char *tp_version(void) { return TP_VERSION; }

int tp_tiles_x(const tp_geometry *g) { return g ? g->img_width / 8 : 0; }
int tp_tiles_y(const tp_geometry *g) { return g ? g->img_height / 8 : 0; }
int tp_tiles_ya(const tp_geometry *g) { return g ? ((g->img_height / 8 + 3) & ~3) : 0; }

int tp_set_lpf(int which, const float *values)
{
    if (which < 0 || which > 5 || !values) return fail(TP_ERR_ARG, "tp_set_lpf(%d, %p)", which, values);
    int rc = cuda_status(cudaMemcpyToSymbol(tp::d_lpf, values, 64 * sizeof(float), which * 64 * sizeof(float)),
                         "cudaMemcpyToSymbol(lpf)");
    if (rc) return rc;
    memcpy(g_lpf_host[which], values, 64 * sizeof(float));
    return TP_OK;
}

int tp_get_lpf(int which, float *values)
{
    if (which < 0 || which > 5 || !values) return fail(TP_ERR_ARG, "tp_get_lpf(%d, %p)", which, values);
    memcpy(values, g_lpf_host[which], 64 * sizeof(float));
    return TP_OK;
}

int tp_reset_lpf(void)
{
    for (int w = 0; w < 6; w++) {
        int rc = tp_set_lpf(w, g_lpf_default[w]);
        if (rc) return rc;
    }
    return TP_OK;
}

int tp_convert_correct_tiles(const tp_geometry *g, float *const *kernel_offsets, float *const *kernels,
                             float *const *images, const tp_task *tasks, float *const *clt, size_t dstride,
                             int num_tiles, int lpf_mask, tp_stream_t stream)
{
    tp::Geom gd;
    int rc = check_geometry(g, &gd);
    if (rc) return rc;
    if (!kernel_offsets || !kernels || !images || !clt) return fail(TP_ERR_ARG, "NULL pointer array");
    if (num_tiles < 0) return fail(TP_ERR_ARG, "num_tiles %d < 0", num_tiles);
    if (num_tiles > 0 && !tasks) return fail(TP_ERR_ARG, "tasks is NULL");
    if (dstride < (size_t)g->img_width) return fail(TP_ERR_ARG, "dstride %zu < width %d", dstride, g->img_width);
    if (num_tiles == 0) return TP_OK;
    int sms;
    if ((rc = sm_count(&sms))) return rc;
    const long long warps = (long long)((num_tiles + 3) / 4) * 12;
    unsigned grid = grid_for(warps, 8, sms, shape_per_sm(TP_SHAPE_CONVERT));
    tp::k_convert_correct_tiles<<<grid, 256, 0, (cudaStream_t)stream>>>(
        gd, dstride, kernel_offsets, kernels, images, tasks, clt, num_tiles, lpf_mask);
    return cuda_status(cudaGetLastError(), "convert_correct_tiles launch");
}

int tp_correlate2D(const tp_geometry *g, float *const *clt, int colors, float scale0, float scale1,
                   float scale2, float fat_zero, size_t num_corr_tiles, const int *corr_indices,
                   size_t corr_stride, int corr_radius, float *corrs, tp_stream_t stream)
{
    tp::Geom gd;
    int rc = check_geometry(g, &gd);
    if (rc) return rc;
    if (!clt) return fail(TP_ERR_ARG, "clt is NULL");
    if (colors != 1 && colors != 3) return fail(TP_ERR_ARG, "colors %d (1 or 3)", colors);
    if (corr_radius < 0 || corr_radius > TP_MAX_CORR_RADIUS)
        return fail(TP_ERR_ARG, "corr_radius %d outside 0..%d", corr_radius, TP_MAX_CORR_RADIUS);
    const size_t sz = (size_t)(2 * corr_radius + 1) * (2 * corr_radius + 1);
    if (num_corr_tiles == 0) return TP_OK;
    if (!corr_indices || !corrs) return fail(TP_ERR_ARG, "NULL corr_indices / corrs");
    if (corr_stride < sz) return fail(TP_ERR_ARG, "corr_stride %zu < (2r+1)^2 = %zu", corr_stride, sz);
    int sms;
    if ((rc = sm_count(&sms))) return rc;
    unsigned grid = grid_for((long long)num_corr_tiles, 16, sms, shape_per_sm(TP_SHAPE_CORRELATE));
    tp::k_correlate2D<<<grid, 128, 0, (cudaStream_t)stream>>>(gd, clt, colors, scale0, scale1, scale2, fat_zero,
                                                              (long long)num_corr_tiles, corr_indices,
                                                              corr_stride, corr_radius, corrs);
    return cuda_status(cudaGetLastError(), "correlate2D launch");
}

static int texture_params(int colors, float min_shot, float scale_shot, float diff_sigma, float w0, float w1,
                          float w2, int dust_remove, int keep_weights, tp::TextureParams *p)
{
    if (colors != 1 && colors != 3) return fail(TP_ERR_ARG, "colors %d (1 or 3)", colors);
    if (!(diff_sigma > 0.0f)) return fail(TP_ERR_ARG, "diff_sigma %g must be > 0", (double)diff_sigma);
    if (scale_shot > 0.0f && !(min_shot > 0.0f))
        return fail(TP_ERR_ARG, "min_shot %g must be > 0 when scale_shot > 0", (double)min_shot);
    p->colors = colors;
    /* the debayer's reciprocal square root takes max(v, min_shot) as a
     * normal float: a positive min_shot below FLT_MIN acts as FLT_MIN */
    p->min_shot = (min_shot > 0.0f && min_shot < FLT_MIN) ? FLT_MIN : min_shot;
    p->scale_shot = scale_shot;
    p->diff_sigma = diff_sigma;
    p->w0 = w0;
    p->w1 = w1;
    p->w2 = w2;
    p->dust_remove = dust_remove;
    p->keep_weights = keep_weights;
    return TP_OK;
}

int tp_textures_accumulate(const tp_geometry *g, const int *woi, float *const *clt, size_t num_texture_tiles,
                           const int *texture_indices, const float *port_offsets, int colors, int is_lwir,
                           float min_shot, float scale_shot, float diff_sigma, float diff_threshold,
                           float min_agree, float weight0, float weight1, float weight2, int dust_remove,
                           int keep_weights, size_t texture_rbg_stride, float *texture_rbg,
                           size_t texture_stride, float *texture_tiles, tp_stream_t stream)
{
    (void)is_lwir; (void)diff_threshold; (void)min_agree; /* accepted, unused (as in the reference) */
    tp::Geom gd;
    int rc = check_geometry(g, &gd);
    if (rc) return rc;
    tp::TextureParams p;
    if ((rc = texture_params(colors, min_shot, scale_shot, diff_sigma, weight0, weight1, weight2, dust_remove,
                             keep_weights, &p)))
        return rc;
    if (num_texture_tiles == 0) return TP_OK;
    if (!clt || !texture_indices || !port_offsets) return fail(TP_ERR_ARG, "NULL clt / indices / port_offsets");
    const bool want_rbg = texture_rbg && texture_rbg_stride;
    const bool want_tiles = texture_tiles && texture_stride;
    if (want_rbg && !woi) return fail(TP_ERR_ARG, "woi is NULL with an RGBA image output");
    const int ns = (colors == 3) ? (keep_weights ? 12 : 4) : (keep_weights ? 8 : 2);
    if (want_tiles && texture_stride < (size_t)ns * 256)
        return fail(TP_ERR_ARG, "texture_stride %zu < %d slices x 256", texture_stride, ns);
    int sms;
    if ((rc = sm_count(&sms))) return rc;
    if ((rc = texture_smem_setup())) return rc;
    unsigned grid = grid_for((long long)num_texture_tiles, 1, sms, shape_per_sm(TP_SHAPE_TEXTURES));
    tex_kernel<false, true>(colors)<<<grid, tp::kTexThreads, tp::kTexSmemBytes, (cudaStream_t)stream>>>(
        gd, woi, clt, (long long)num_texture_tiles, texture_indices, nullptr, 0, 0, 0, port_offsets, p,
        want_rbg ? texture_rbg_stride : 0, want_rbg ? texture_rbg : nullptr, want_tiles ? texture_stride : 0,
        want_tiles ? texture_tiles : nullptr);
    return cuda_status(cudaGetLastError(), "textures_accumulate launch");
}

int tp_imclt_rbg(const tp_geometry *g, const float *clt_one_cam, float *rbg, int color, int v_offset,
                 int h_offset, size_t dstride, tp_stream_t stream)
{
    tp::Geom gd;
    int rc = check_geometry(g, &gd);
    if (rc) return rc;
    if (!clt_one_cam || !rbg) return fail(TP_ERR_ARG, "NULL clt / rbg");
    if (color < 0 || color > 2) return fail(TP_ERR_ARG, "color %d outside 0..2", color);
    if ((v_offset & ~1) || (h_offset & ~1)) return fail(TP_ERR_ARG, "offsets must be 0 or 1");
    if (dstride < (size_t)g->img_width + 8) return fail(TP_ERR_ARG, "dstride %zu < width + 8", dstride);
    int sms;
    if ((rc = sm_count(&sms))) return rc;
    const long long ntl = (long long)((gd.TX + (h_offset ^ 1)) >> 1) * ((gd.TY + (v_offset ^ 1)) >> 1);
    unsigned grid = grid_for(ntl, 32, sms, 8);
    tp::k_imclt_rbg<<<grid, 256, 0, (cudaStream_t)stream>>>(gd, clt_one_cam, rbg, color, v_offset, h_offset,
                                                            dstride);
    return cuda_status(cudaGetLastError(), "imclt_rbg launch");
}

int tp_imclt_rbg_all(const tp_geometry *g, const float *clt_one_cam, float *rbg, size_t dstride,
                     tp_stream_t stream)
{
    for (int color = 0; color < 3; color++)
        for (int v = 0; v < 2; v++)
            for (int h = 0; h < 2; h++) {
                int rc = tp_imclt_rbg(g, clt_one_cam, rbg, color, v, h, dstride, stream);
                if (rc) return rc;
            }
    return TP_OK;
}

/* Launch kern on stream s; with `dependent` as a programmatic dependent of
 * the launch before it on s (programmatic stream serialisation): the kernel
 * may be scheduled before that launch has finished and must wait for it
 * (grid_dependency_wait) before reading anything it writes. */
extern "C++" {
template <typename... Params, typename... Args>
static cudaError_t launch_chained(bool dependent, dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                                  void (*kern)(Params...), Args &&...args)
{
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cfg.attrs = attr;
    cfg.numAttrs = dependent ? 1 : 0;
    return cudaLaunchKernelEx(&cfg, kern, std::forward<Args>(args)...);
}
} /* extern "C++" */

/* prepare_texture_list listing only tiles of rows [row_first, row_last) */
static int prepare_list(const tp_geometry *g, tp_task *tasks, int num_tiles, int *texture_indices,
                        int *num_texture_tiles, int *woi, int width, int height, int row_first, int row_last,
                        tp_stream_t stream)
{
    tp::Geom gd;
    int rc = check_geometry(g, &gd);
    if (rc) return rc;
    if (num_tiles < 0) return fail(TP_ERR_ARG, "num_tiles %d < 0", num_tiles);
    if ((num_tiles > 0 && !tasks) || !texture_indices || !num_texture_tiles || !woi)
        return fail(TP_ERR_ARG, "NULL tasks / texture_indices / num_texture_tiles / woi");
    if (width < 0 || height < 0 || width > gd.TX || height > gd.TY)
        return fail(TP_ERR_ARG, "list extent %dx%d outside %dx%d tiles", width, height, gd.TX, gd.TY);
    cudaStream_t s = (cudaStream_t)stream;
    const long long cap = (long long)gd.TX * gd.TYA;
    /* the first kernel is an ordinary launch (it follows the caller's work);
     * each later one is a programmatic dependent of the one before, which it
     * waits for on entry (chain_entry) */
    bool dep = false;
    cudaError_t err = cudaSuccess;
    if (height > 0) {
        dim3 b0((width + 1 + 255) / 256, height, 1);
        err = launch_chained(dep, b0, 256, 0, s, tp::k_clear_texture_list, texture_indices, width, height, gd.TX,
                             cap);
        dep = true;
    }
    const unsigned bt = (unsigned)((num_tiles + 255) / 256);
    if (bt && err == cudaSuccess) {
        err = launch_chained(dep, bt, 256, 0, s, tp::k_mark_texture_tiles, (const tp_task *)tasks, num_tiles,
                             texture_indices, gd.TX, cap);
        dep = true;
    }
    if (err == cudaSuccess)
        err = launch_chained(dep, 1, 32, 0, s, tp::k_woi_init, woi, num_texture_tiles, gd.TX, gd.TY);
    if (bt && err == cudaSuccess)
        err = launch_chained(true, bt, 256, 0, s, tp::k_mark_neighbor_tiles, tasks, num_tiles,
                             (const int *)texture_indices, woi, gd.TX, gd.TY, cap);
    if (bt && err == cudaSuccess)
        err = launch_chained(true, bt, 256, 0, s, tp::k_gen_texture_list, (const tp_task *)tasks, num_tiles,
                             texture_indices, num_texture_tiles, (const int *)woi, gd.TX, gd.TX * (gd.TYA >> 2),
                             cap, row_first, row_last);
    if (err == cudaSuccess) err = launch_chained(true, 1, 32, 0, s, tp::k_woi_finalize, woi);
    if (err != cudaSuccess) return cuda_status(err, "prepare_texture_list launch");
    return cuda_status(cudaGetLastError(), "prepare_texture_list launch");
}

int tp_prepare_texture_list(const tp_geometry *g, tp_task *tasks, int num_tiles, int *texture_indices,
                            int *num_texture_tiles, int *woi, int width, int height, tp_stream_t stream)
{
    return prepare_list(g, tasks, num_tiles, texture_indices, num_texture_tiles, woi, width, height, 0, INT_MAX,
                        stream);
}

int tp_clear_texture_rbga(const tp_geometry *g, int texture_width, int texture_slice_height,
                          size_t texture_rbga_stride, float *texture_tiles, tp_stream_t stream)
{
    tp::Geom gd;
    int rc = check_geometry(g, &gd);
    if (rc) return rc;
    if (!texture_tiles) return fail(TP_ERR_ARG, "texture_tiles is NULL");
    if (texture_width < 0 || texture_slice_height < 0) return fail(TP_ERR_ARG, "negative extent");
    if (texture_rbga_stride < (size_t)texture_width) return fail(TP_ERR_ARG, "stride < width");
    if (texture_width == 0 || texture_slice_height == 0) return TP_OK;
    int sms;
    if ((rc = sm_count(&sms))) return rc;
    tp::k_clear_rbga<<<grid_for(texture_slice_height, 1, sms, 16), 256, 0, (cudaStream_t)stream>>>(
        nullptr, 0, texture_width, texture_slice_height, texture_rbga_stride, texture_tiles);
    return cuda_status(cudaGetLastError(), "clear_texture_rbga launch");
}

static int inv_tc_launch(const tp::InvTcStage &st, int format, tp_stream_t stream);

/* tile_scratch / format: when format >= 0, the inverse CLT of every listed
 * tile runs first on the tensor cores (InvTcStage) into tile_scratch, and
 * the passes read those tiles (k_textures<true>) */
static int generate_rbga(const tp_geometry *g, tp_task *tasks, int num_tiles, int *texture_indices,
                         int *num_texture_tiles, int *woi, int width, int height, float *const *clt,
                         const float *port_offsets, int colors, float min_shot, float scale_shot, float diff_sigma,
                         float weight0, float weight1, float weight2, int dust_remove, size_t texture_rbga_stride,
                         float *texture_tiles, int row_first, int row_last, float *const *tile_scratch, int format,
                         tp_stream_t stream)
{
    tp::Geom gd;
    int rc = check_geometry(g, &gd);
    if (rc) return rc;
    tp::TextureParams p;
    if ((rc = texture_params(colors, min_shot, scale_shot, diff_sigma, weight0, weight1, weight2, dust_remove, 0,
                             &p)))
        return rc;
    if (!clt || !port_offsets || !texture_tiles) return fail(TP_ERR_ARG, "NULL clt / port_offsets / output");
    if (texture_rbga_stride < (size_t)(gd.TX + 1) * 8)
        return fail(TP_ERR_ARG, "texture_rbga_stride %zu < (tilesx + 1) * 8", texture_rbga_stride);
    if ((rc = prepare_list(g, tasks, num_tiles, texture_indices, num_texture_tiles, woi, width, height, row_first,
                           row_last, stream)))
        return rc;
    cudaStream_t s = (cudaStream_t)stream;
    int sms;
    if ((rc = sm_count(&sms))) return rc;
    if ((rc = texture_smem_setup())) return rc;
    /* The RGBA clear and the four passes continue prepare_list's chain of
     * programmatic dependents.  The clear waits on entry for the list's last
     * kernel and releases its dependent only after that wait.  A pass releases
     * its own dependent on entry, then prefetches its first tile's CLT and
     * reads the list, and only then waits for the launch before it (the
     * clear, or the previous pass, which read-modify-writes the RGBA image).
     * So a pass can start only after every earlier pass has started, and the
     * first pass only after the clear released it, which the clear did once
     * the list was complete: every pass reads a finished list. */
    {
        const int max_rows = (gd.TY + 1) * 8 * (colors + 1);
        const cudaError_t err = launch_chained(true, grid_for(max_rows, 1, sms, 16), 256, 0, s, tp::k_clear_rbga,
                                               (const int *)woi, colors, 0, 0, texture_rbga_stride, texture_tiles);
        if (err != cudaSuccess) return cuda_status(err, "generate_RBGA clear launch");
    }
    float *const *src = clt;
    if (format >= 0) {
        /* an ordinary launch: it reads the tasks the list kernels rewrote */
        tp::InvTcStage st{gd, clt, tile_scratch, tasks, (long long)num_tiles, nullptr, colors};
        if ((rc = inv_tc_launch(st, format, stream))) return rc;
        src = tile_scratch;
    }
    const int quarter = gd.TX * (gd.TYA >> 2);
    const unsigned grid = grid_for(quarter, 1, sms, shape_per_sm(TP_SHAPE_TEXTURES));
    /* one pass per tile parity: its inner sub-list, then its border one (the
     * reference runs the four inner passes, then the four border passes;
     * tiles of one parity never overlap, so a pass needs no ordering) */
    const auto tex = format >= 0 ? tex_kernel<true, false>(colors) : tex_kernel<false, false>(colors);
    for (int parity = 0; parity < 4; parity++) {
        const int *base = texture_indices + parity * quarter;
        const cudaError_t err =
            launch_chained(true, grid, tp::kTexThreads, tp::kTexSmemBytes, s, tex, gd, (const int *)woi, src, 0LL,
                           (const int *)base, (const int *)num_texture_tiles, parity << 1, quarter, -quarter,
                           port_offsets, p, texture_rbga_stride, texture_tiles, (size_t)0, (float *)nullptr);
        if (err != cudaSuccess) return cuda_status(err, "generate_RBGA texture pass launch");
    }
    return cuda_status(cudaGetLastError(), "generate_RBGA launch");
}

int tp_generate_RBGA(const tp_geometry *g, tp_task *tasks, int num_tiles, int *texture_indices,
                     int *num_texture_tiles, int *woi, int width, int height, float *const *clt,
                     const float *port_offsets, int colors, int is_lwir, float min_shot, float scale_shot,
                     float diff_sigma, float diff_threshold, float min_agree, float weight0, float weight1,
                     float weight2, int dust_remove, int keep_weights, size_t texture_rbga_stride,
                     float *texture_tiles, tp_stream_t stream)
{
    (void)is_lwir; (void)diff_threshold; (void)min_agree; (void)keep_weights;
    return generate_rbga(g, tasks, num_tiles, texture_indices, num_texture_tiles, woi, width, height, clt,
                         port_offsets, colors, min_shot, scale_shot, diff_sigma, weight0, weight1, weight2,
                         dust_remove, texture_rbga_stride, texture_tiles, 0, INT_MAX, nullptr, -1, stream);
}

int tp_generate_RBGA_rows(const tp_geometry *g, tp_task *tasks, int num_tiles, int *texture_indices,
                          int *num_texture_tiles, int *woi, int width, int height, float *const *clt,
                          const float *port_offsets, int colors, float min_shot, float scale_shot,
                          float diff_sigma, float weight0, float weight1, float weight2, int dust_remove,
                          size_t texture_rbga_stride, float *texture_tiles, int row_first, int row_last,
                          tp_stream_t stream)
{
    if (row_first < 0 || row_last < row_first)
        return fail(TP_ERR_ARG, "tile rows [%d, %d)", row_first, row_last);
    return generate_rbga(g, tasks, num_tiles, texture_indices, num_texture_tiles, woi, width, height, clt,
                         port_offsets, colors, min_shot, scale_shot, diff_sigma, weight0, weight1, weight2,
                         dust_remove, texture_rbga_stride, texture_tiles, row_first, row_last, nullptr, -1,
                         stream);
}

int tp_process_frame(const tp_geometry *g, float *const *kernel_offsets, float *const *kernels, float *const *images,
                     size_t dstride, tp_task *tasks, int num_tiles, int lpf_mask, int corr_colors, float corr_scale0,
                     float corr_scale1, float corr_scale2, float fat_zero, int corr_radius, size_t corr_stride,
                     float *corrs, const float *port_offsets, float min_shot, float scale_shot, float diff_sigma,
                     float weight0, float weight1, float weight2, int dust_remove, int *texture_indices,
                     int *num_texture_tiles, int *woi, size_t texture_rbga_stride, float *texture_rbga,
                     float *const *clt, tp_stream_t stream)
{
    tp::Geom gd;
    int rc = check_geometry(g, &gd);
    if (rc) return rc;
    if (!kernel_offsets || !kernels || !images) return fail(TP_ERR_ARG, "NULL pointer array");
    if (num_tiles < 0) return fail(TP_ERR_ARG, "num_tiles %d < 0", num_tiles);
    if (dstride < (size_t)g->img_width) return fail(TP_ERR_ARG, "dstride %zu < width %d", dstride, g->img_width);
    if (corr_colors != 1 && corr_colors != 3) return fail(TP_ERR_ARG, "corr_colors %d (1 or 3)", corr_colors);
    if (corr_radius < 0 || corr_radius > TP_MAX_CORR_RADIUS)
        return fail(TP_ERR_ARG, "corr_radius %d outside 0..%d", corr_radius, TP_MAX_CORR_RADIUS);
    const size_t sz = (size_t)(2 * corr_radius + 1) * (2 * corr_radius + 1);
    if (corr_stride < sz) return fail(TP_ERR_ARG, "corr_stride %zu < (2r+1)^2 = %zu", corr_stride, sz);
    tp::TextureParams tex;
    if ((rc = texture_params(3, min_shot, scale_shot, diff_sigma, weight0, weight1, weight2, dust_remove, 0, &tex)))
        return rc;
    if (texture_rbga_stride < (size_t)(gd.TX + 1) * 8)
        return fail(TP_ERR_ARG, "texture_rbga_stride %zu < (tilesx + 1) * 8", texture_rbga_stride);
    if (!corrs || !port_offsets || !texture_rbga) return fail(TP_ERR_ARG, "NULL corrs / port_offsets / texture_rbga");
    if (num_tiles == 0) return TP_OK;
    if ((rc = tp_prepare_texture_list(g, tasks, num_tiles, texture_indices, num_texture_tiles, woi, gd.TX, gd.TY,
                                      stream)))
        return rc;
    cudaStream_t s = (cudaStream_t)stream;
    int sms;
    if ((rc = sm_count(&sms))) return rc;
    {
        /* a programmatic dependent of the list's last kernel, as in generate_rbga */
        const int max_rows = (gd.TY + 1) * 8 * 4;
        const cudaError_t err = launch_chained(true, grid_for(max_rows, 1, sms, 16), 256, 0, s, tp::k_clear_rbga,
                                               (const int *)woi, 3, 0, 0, texture_rbga_stride, texture_rbga);
        if (err != cudaSuccess) return cuda_status(err, "process_frame clear launch");
    }
    tp::FrameParams fp;
    fp.lpf_mask = lpf_mask;
    fp.corr_colors = corr_colors;
    fp.s0 = corr_scale0;
    fp.s1 = corr_scale1;
    fp.s2 = corr_scale2;
    fp.fat_zero = fat_zero;
    fp.corr_radius = corr_radius;
    fp.corr_stride = corr_stride;
    fp.tex = tex;
    if ((rc = set_smem_once(g_frame_attr, (const void *)tp::k_frame, tp::kFrameSmemBytes,
                            "cudaFuncSetAttribute(k_frame)")))
        return rc;
    /* one resident wave, odd: a grid-stride walk over a raster task list then
     * visits both column parities in every block.  Each parity launch is a
     * programmatic dependent of the launch before it (the clear, or the
     * previous parity), which it waits for before its first RGBA update; it
     * releases its own dependent on entry, so a launch starts only after every
     * earlier one has started and the first only after the clear released it,
     * which the clear did once the list (and the tasks' neighbour bits it
     * rewrites) was complete. */
    const unsigned grid = grid_for(((long long)num_tiles + 3) / 4, 1, sms, tp::kFrameBlocksPerSm) | 1u;
    for (int parity = 0; parity < 4; parity++) {
        const cudaError_t err = launch_chained(true, grid, tp::kFrameThreads, tp::kFrameSmemBytes, s, tp::k_frame,
                                               gd, dstride, kernel_offsets, kernels, images, (const tp_task *)tasks,
                                               num_tiles, parity, fp, corrs, port_offsets, (const int *)woi,
                                               texture_rbga_stride, texture_rbga, clt);
        if (err != cudaSuccess) return cuda_status(err, "process_frame launch");
    }
    return cuda_status(cudaGetLastError(), "process_frame launch");
}

int tp_generate_RBGA_noalloc(const tp_geometry *g, tp_task *tasks, int num_tiles, int width, int height,
                             float *const *clt, const float *port_offsets, int colors, int is_lwir, float min_shot,
                             float scale_shot, float diff_sigma, float diff_threshold, float min_agree,
                             float weight0, float weight1, float weight2, int dust_remove, int keep_weights,
                             size_t texture_rbga_stride, float *texture_tiles, tp_stream_t stream)
{
    tp::Geom gd;
    int rc = check_geometry(g, &gd);
    if (rc) return rc;
    const long long need = (long long)gd.TX * gd.TYA + 16;
    if (need > TP_NOALLOC_SCRATCH_INTS)
        return fail(TP_ERR_ARG, "frame needs %lld scratch ints, the library holds %d (%d tiles across: at most %d "
                    "tile rows)", need, TP_NOALLOC_SCRATCH_INTS, gd.TX,
                    ((TP_NOALLOC_SCRATCH_INTS - 16) / (gd.TX > 0 ? gd.TX : 1)) & ~3);
    if (width < 0 || height < 0 || width > gd.TX || height > gd.TY)
        return fail(TP_ERR_ARG, "list extent %dx%d outside %dx%d tiles", width, height, gd.TX, gd.TY);
    int *scratch = nullptr;
    if ((rc = noalloc_scratch(&scratch))) return rc;
    /* The list kernels read the marker of every neighbour of every texture
     * tile, wherever it lies; caller buffers hold zeros there where the
     * caller's width x height extent leaves them uncleared, but the shared
     * array holds whatever an earlier call left.  So the marker grid is
     * cleared over the whole frame (tilesx + 1 columns, tilesy rows), which
     * gives the result of tp_generate_RBGA on freshly zeroed buffers for any
     * extent the caller passes. */
    (void)width;
    (void)height;
    return tp_generate_RBGA(g, tasks, num_tiles, scratch + 16, scratch, scratch + 8, gd.TX, gd.TY, clt,
                            port_offsets, colors, is_lwir, min_shot, scale_shot, diff_sigma, diff_threshold,
                            min_agree, weight0, weight1, weight2, dust_remove, keep_weights, texture_rbga_stride,
                            texture_tiles, stream);
}

int tp_mlp_features(const tp_geometry *g, const float *corrs, size_t corr_stride, int corr_radius,
                    size_t num_corr_tiles, const int *corr_indices, float *features, size_t feature_stride,
                    tp_stream_t stream)
{
    tp::Geom gd;
    int rc = check_geometry(g, &gd);
    if (rc) return rc;
    if (corr_radius < 0 || corr_radius > TP_MAX_CORR_RADIUS)
        return fail(TP_ERR_ARG, "corr_radius %d outside 0..%d", corr_radius, TP_MAX_CORR_RADIUS);
    const int n2 = (2 * corr_radius + 1) * (2 * corr_radius + 1);
    if (num_corr_tiles == 0) return TP_OK;
    if (!corrs || !corr_indices || !features) return fail(TP_ERR_ARG, "NULL corrs / corr_indices / features");
    if (corr_stride < (size_t)n2) return fail(TP_ERR_ARG, "corr_stride %zu < %d", corr_stride, n2);
    if (feature_stride < (size_t)(6 * n2)) return fail(TP_ERR_ARG, "feature_stride %zu < %d", feature_stride, 6 * n2);
    int sms;
    if ((rc = sm_count(&sms))) return rc;
    tp::k_mlp_features<<<grid_for((long long)num_corr_tiles, 8, sms, 8), 256, 0, (cudaStream_t)stream>>>(
        gd.TX * gd.TY, corrs, corr_stride, n2, (long long)num_corr_tiles, corr_indices, features, feature_stride);
    return cuda_status(cudaGetLastError(), "mlp_features launch");
}

int tp_mlp_gemm(int M, int N, int K, const float *A, int lda, int trans_a, const float *B, int ldb, int trans_b,
                float beta, float *C, int ldc, const float *bias, float *z, int ldz, tp_stream_t stream)
{
    if (M < 0 || N < 0 || K < 0) return fail(TP_ERR_ARG, "gemm %d x %d x %d", M, N, K);
    if (M == 0 || N == 0) return TP_OK;
    if (!C || (K > 0 && (!A || !B))) return fail(TP_ERR_ARG, "NULL gemm operand");
    if (lda < (trans_a ? M : K) || ldb < (trans_b ? K : N) || ldc < N || (z && ldz < N))
        return fail(TP_ERR_ARG, "gemm leading dimension too small");
    if ((M + tp::kGB - 1) / tp::kGB > 65535) return fail(TP_ERR_ARG, "gemm M %d too large", M);
    dim3 grid((unsigned)((N + tp::kGB - 1) / tp::kGB), (unsigned)((M + tp::kGB - 1) / tp::kGB), 1);
    tp::k_gemm<<<grid, 256, 0, (cudaStream_t)stream>>>(M, N, K, A, lda, trans_a, B, ldb, trans_b, beta, C, ldc, bias,
                                                       z, ldz);
    return cuda_status(cudaGetLastError(), "mlp_gemm launch");
}

int tp_mlp_gemm_tc(int M, int N, int K, const float *A, int lda, int trans_a, const float *B, int ldb, int trans_b,
                   float beta, float *C, int ldc, const float *bias, float *z, int ldz, int *err, tp_stream_t stream)
{
    if (M < 0 || N < 0 || K < 0) return fail(TP_ERR_ARG, "gemm %d x %d x %d", M, N, K);
    if (M == 0 || N == 0) return TP_OK;
    if (!C || (K > 0 && (!A || !B))) return fail(TP_ERR_ARG, "NULL gemm operand");
    if (lda < (trans_a ? M : K) || ldb < (trans_b ? K : N) || ldc < N || (z && ldz < N))
        return fail(TP_ERR_ARG, "gemm leading dimension too small");
    if ((M + tp::kGtM - 1) / tp::kGtM > 65535) return fail(TP_ERR_ARG, "gemm M %d too large", M);
    int rc;
    if ((rc = set_smem_once(g_gemm_tc_attr, (const void *)tp::k_gemm_tc, tp::kGtSmemBytes,
                            "cudaFuncSetAttribute(k_gemm_tc)")))
        return rc;
    int sms;
    if ((rc = sm_count(&sms))) return rc;
    dim3 grid((unsigned)((N + tp::kGtN - 1) / tp::kGtN), (unsigned)((M + tp::kGtM - 1) / tp::kGtM), 1);
    /* A plain product (no bias, beta 0, no GELU) with fewer tiles than SMs and
     * a long K (the weight gradients: K = the batch) splits K over up to
     * 2 x SMs CTAs, each adding its partial sums into C, zeroed first (the
     * order of those few additions per element is not fixed). */
    const long long tiles = (long long)grid.x * grid.y;
    const int chunks = (K + tp::kGtK - 1) / tp::kGtK;
    if (!bias && !z && beta == 0.0f && tiles < sms && chunks >= 8) {
        long long splits = (2LL * sms + tiles - 1) / tiles;
        if (splits > chunks / 4) splits = chunks / 4;
        if (splits > 1) {
            grid.z = (unsigned)splits;
            const cudaError_t e = cudaMemset2DAsync(C, (size_t)ldc * sizeof(float), 0, (size_t)N * sizeof(float),
                                                    (size_t)M, (cudaStream_t)stream);
            if (e != cudaSuccess) return cuda_status(e, "mlp_gemm_tc clear");
        }
    }
    tp::k_gemm_tc<<<grid, 128, tp::kGtSmemBytes, (cudaStream_t)stream>>>(M, N, K, A, lda, trans_a, B, ldb, trans_b,
                                                                       beta, C, ldc, bias, z, ldz, err);
    return cuda_status(cudaGetLastError(), "mlp_gemm_tc launch");
}

int tp_mlp_gelu_backward(int rows, int cols, int ld, const float *z, const float *dh, float *dz, tp_stream_t stream)
{
    if (rows < 0 || cols < 0 || ld < cols) return fail(TP_ERR_ARG, "gelu_backward %d x %d ld %d", rows, cols, ld);
    if (!rows || !cols) return TP_OK;
    if (!z || !dh || !dz) return fail(TP_ERR_ARG, "NULL gelu_backward operand");
    int sms, rc;
    if ((rc = sm_count(&sms))) return rc;
    const long long n = (long long)rows * cols;
    tp::k_gelu_backward<<<grid_for(n, 256, sms, 8), 256, 0, (cudaStream_t)stream>>>(n, cols, ld, z, dh, dz);
    return cuda_status(cudaGetLastError(), "mlp_gelu_backward launch");
}

int tp_mlp_colsum(int rows, int cols, int ld, const float *x, float scale, float *out, tp_stream_t stream)
{
    if (rows < 0 || cols < 0 || ld < cols) return fail(TP_ERR_ARG, "colsum %d x %d ld %d", rows, cols, ld);
    if (!cols) return TP_OK;
    if ((rows && !x) || !out) return fail(TP_ERR_ARG, "NULL colsum operand");
    tp::k_colsum<<<(cols + 31) / 32, dim3(32, tp::kColLanes), 0, (cudaStream_t)stream>>>(rows, cols, ld, x, scale,
                                                                                        out);
    return cuda_status(cudaGetLastError(), "mlp_colsum launch");
}

int tp_mlp_nll(int rows, const float *out, const float *target, const float *w, float inv_count, float *dout,
               float *loss_rows, tp_stream_t stream)
{
    if (rows < 0) return fail(TP_ERR_ARG, "nll rows %d", rows);
    if (!rows) return TP_OK;
    if (!out || !target || !dout || !loss_rows) return fail(TP_ERR_ARG, "NULL nll operand");
    tp::k_nll<<<(rows + 255) / 256, 256, 0, (cudaStream_t)stream>>>(rows, out, target, w, inv_count, dout,
                                                                    loss_rows);
    return cuda_status(cudaGetLastError(), "mlp_nll launch");
}

int tp_mlp_pack(const float *W1, const float *W2, void *w1t, void *w2t, tp_stream_t stream)
{
    if (!W1 || !W2 || !w1t || !w2t) return fail(TP_ERR_ARG, "NULL mlp_pack operand");
    if ((reinterpret_cast<uintptr_t>(w1t) | reinterpret_cast<uintptr_t>(w2t)) & 15)
        return fail(TP_ERR_ARG, "packed weights must be 16-byte aligned");
    int sms, rc;
    if ((rc = sm_count(&sms))) return rc;
    tp::k_mlp_pack<<<sms * 4, 256, 0, (cudaStream_t)stream>>>(W1, W2, static_cast<float *>(w1t),
                                                            static_cast<__nv_bfloat16 *>(w2t));
    return cuda_status(cudaGetLastError(), "mlp_pack launch");
}

int tp_mlp_infer_tc(int rows, const float *x, int ldx, const void *w1t, const float *b1, const void *w2t,
                    const float *b2, const float *W3, const float *b3, float *out, int *err, tp_stream_t stream)
{
    if (rows < 0 || ldx < 1350) return fail(TP_ERR_ARG, "mlp_infer rows %d ldx %d", rows, ldx);
    if (!rows) return TP_OK;
    if (!x || !w1t || !b1 || !w2t || !b2 || !W3 || !b3 || !out) return fail(TP_ERR_ARG, "NULL mlp_infer operand");
    if ((reinterpret_cast<uintptr_t>(w1t) | reinterpret_cast<uintptr_t>(w2t)) & 15)
        return fail(TP_ERR_ARG, "w1t / w2t must be 16-byte aligned");
    if ((reinterpret_cast<uintptr_t>(x) & 15) || (ldx & 3))
        return fail(TP_ERR_ARG, "feature rows must start on 16-byte boundaries (x aligned, ldx %d a multiple of 4)",
                    ldx);
    int sms, rc;
    if ((rc = sm_count(&sms))) return rc;
    PFN_cuTensorMapEncodeTiled_v12000 encode;
    if ((rc = tensor_map_encoder(&encode))) return rc;
    /* the features as a 2-D FP32 tensor of 1350 x rows, boxes of 32 x 128 with 128-byte swizzle */
    CUtensorMap tmap;
    const cuuint64_t dims[2] = {1350, (cuuint64_t)rows};
    const cuuint64_t strides[1] = {(cuuint64_t)ldx * sizeof(float)};
    const cuuint32_t box[2] = {(cuuint32_t)tp::kTcKB, (cuuint32_t)tp::kTcM};
    const cuuint32_t estr[2] = {1, 1};
    const CUresult cr = encode(&tmap, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float *>(x), dims, strides, box,
                               estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                               CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (cr != CUDA_SUCCESS) return fail(TP_ERR_ARG, "cuTensorMapEncodeTiled failed (%d)", (int)cr);
    if ((rc = set_smem_once(g_tc_attr, (const void *)tp::k_mlp_infer_tc, tp::kTcSmemBytes,
                            "cudaFuncSetAttribute(k_mlp_infer_tc)")))
        return rc;
    const int tiles = (rows + tp::kTcM - 1) / tp::kTcM;
    tp::k_mlp_infer_tc<<<tiles < sms ? tiles : sms, 128, tp::kTcSmemBytes, (cudaStream_t)stream>>>(
        tmap, rows, static_cast<const float *>(w1t), b1, static_cast<const __nv_bfloat16 *>(w2t), b2, W3, b3, out,
        err);
    return cuda_status(cudaGetLastError(), "mlp_infer_tc launch");
}

int tp_mlp_combine(size_t n, const float *plain, const float *out, float gate, float *rho, tp_stream_t stream)
{
    if (!n) return TP_OK;
    if (!plain || !out || !rho) return fail(TP_ERR_ARG, "NULL mlp_combine operand");
    if (reinterpret_cast<uintptr_t>(out) & 7) return fail(TP_ERR_ARG, "out must be 8-byte aligned");
    int sms, rc;
    if ((rc = sm_count(&sms))) return rc;
    tp::k_mlp_combine<<<grid_for((long long)n, 256, sms, 8), 256, 0, (cudaStream_t)stream>>>((long long)n, plain, out,
                                                                                          gate, rho);
    return cuda_status(cudaGetLastError(), "mlp_combine launch");
}

int tp_mlp_adam(size_t n, float *param, const float *grad, float *m, float *v, float lr, float beta1, float beta2,
                float eps, int step, tp_stream_t stream)
{
    if (step < 1) return fail(TP_ERR_ARG, "adam step %d < 1", step);
    if (!n) return TP_OK;
    if (!param || !grad || !m || !v) return fail(TP_ERR_ARG, "NULL adam operand");
    int sms, rc;
    if ((rc = sm_count(&sms))) return rc;
    const float c1 = (float)(1.0 / (1.0 - pow((double)beta1, step)));
    const float c2 = (float)(1.0 / (1.0 - pow((double)beta2, step)));
    tp::k_adam<<<grid_for((long long)n, 256, sms, 8), 256, 0, (cudaStream_t)stream>>>((long long)n, param, grad, m, v,
                                                                                   lr, beta1, beta2, eps, c1, c2);
    return cuda_status(cudaGetLastError(), "mlp_adam launch");
}

int tp_psf_to_clt(const float *psf, size_t n, float *clt_kernels, tp_stream_t stream)
{
    if (n == 0) return TP_OK;
    if (!psf || !clt_kernels) return fail(TP_ERR_ARG, "NULL psf / clt_kernels");
    int sms;
    int rc = sm_count(&sms);
    if (rc) return rc;
    tp::k_psf_to_clt<<<grid_for((long long)n, 1, sms, 8), 256, 0, (cudaStream_t)stream>>>(psf, (long long)n,
                                                                                         clt_kernels);
    return cuda_status(cudaGetLastError(), "psf_to_clt launch");
}

int tp_disparity_fit(const tp_geometry *g, const float *corrs, size_t corr_stride, int corr_radius,
                     size_t num_corr_tiles, const int *corr_indices, const float *port_offsets, int pair_mask,
                     int mode, float *disparity, float *strength, tp_stream_t stream)
{
    tp::Geom gd;
    int rc = check_geometry(g, &gd);
    if (rc) return rc;
    if (corr_radius < 0 || corr_radius > TP_MAX_CORR_RADIUS)
        return fail(TP_ERR_ARG, "corr_radius %d outside 0..%d", corr_radius, TP_MAX_CORR_RADIUS);
    const size_t sz = (size_t)(2 * corr_radius + 1) * (2 * corr_radius + 1);
    if (mode < 0 || mode > 2) return fail(TP_ERR_ARG, "mode %d (0, 1 or 2)", mode);
    if (num_corr_tiles == 0) return TP_OK;
    if (!corrs || !corr_indices || !port_offsets || !disparity || !strength)
        return fail(TP_ERR_ARG, "NULL corrs / corr_indices / port_offsets / disparity / strength");
    if (corr_stride < sz) return fail(TP_ERR_ARG, "corr_stride %zu < (2r+1)^2 = %zu", corr_stride, sz);
    int sms;
    if ((rc = sm_count(&sms))) return rc;
    const unsigned grid = grid_for((long long)num_corr_tiles, 8, sms, 8);
    tp::k_disparity_fit<<<grid, 256, 0, (cudaStream_t)stream>>>(gd.TX * gd.TY, corrs, corr_stride, corr_radius,
                                                               (long long)num_corr_tiles, corr_indices,
                                                               port_offsets, pair_mask, mode, disparity, strength);
    return cuda_status(cudaGetLastError(), "disparity_fit launch");
}

} /* extern "C" */

/* ---- tensor-core (hi + lo split) forms of the CLT stages -------------------
 *
 * The 64 x 64 matrices K_q = V_q (x) H_q of each stage's four quadrant
 * transforms, split into two 16-bit halves (hi = K rounded to the format,
 * lo = (K - hi) rounded) and stored as the 128-byte-swizzled B images the
 * kernels copy into shared memory (tp_tc_engine.cuh): per format and stage
 * 64 KB, the four hi quadrants then the four lo.  Built on the host in
 * double from the closed forms of the 8-point transforms, copied once per
 * device (and again after a device reset) on the first tensor-core call;
 * make that first call before any stream capture. */
enum { kTcStageCorr = 0, kTcStageInv = 1, kTcStageFwd = 2, kTcStagesN = 3 };
static __device__ __align__(1024) unsigned char g_tc_btab[2][kTcStagesN][tp::kTcBBytes];
/* set by a tensor-core kernel whose bounded wait ran out (tp_tc_status) */
static __device__ int g_tc_err;

namespace {

/* M[k][n] of the four 8-point transforms (DCT-IV, DST-IV, DCT-II, DST-II) */
double tc_dtt(int kind, int k, int n)
{
    const double pi = 3.14159265358979323846;
    switch (kind) {
    case 0: return 0.5 * cos(pi * (2 * k + 1) * (2 * n + 1) / 32.0);
    case 1: return 0.5 * sin(pi * (2 * k + 1) * (2 * n + 1) / 32.0);
    case 2: return 0.5 * cos(pi * (2 * n + 1) * k / 16.0);
    default: return 0.5 * sin(pi * (2 * n + 1) * (k + 1) / 16.0);
    }
}

/* vertical / horizontal transform kinds of quadrant q of a stage (-1: unused) */
void tc_kinds(int stage, int q, int *v, int *h)
{
    if (stage == kTcStageCorr) { /* correlate2D: DCT-II / DST-II, q1 and q3 sine horizontally, q2 and q3 vertically */
        *v = 2 + (q >> 1);
        *h = 2 + (q & 1);
    } else if (stage == kTcStageInv) { /* inverse CLT: DCT-IV / DST-IV in the same pattern */
        *v = q >> 1;
        *h = q & 1;
    } else { /* forward CLT: slot 0 CC (DCT-IV both ways), slot 1 SC (DST-IV horizontally) */
        *v = q < 2 ? 0 : -1;
        *h = q < 2 ? q : -1;
    }
}

uint16_t tc_half_bits(double x, int fmt)
{
    if (fmt == TP_TC_BF16X2) return __bfloat16_as_ushort(__double2bfloat16(x));
    return __half_as_ushort(__double2half(x));
}

double tc_half_value(uint16_t b, int fmt)
{
    if (fmt == TP_TC_BF16X2) return (double)__bfloat162float(__ushort_as_bfloat16(b));
    return (double)__half2float(__ushort_as_half(b));
}

void tc_build_table(int fmt, int stage, uint16_t *img)
{
    memset(img, 0, tp::kTcBBytes);
    for (int q = 0; q < 4; q++) {
        int kv, kh;
        tc_kinds(stage, q, &kv, &kh);
        if (kv < 0) continue;
        for (int i = 0; i < 8; i++)
            for (int j = 0; j < 8; j++)
                for (int m = 0; m < 8; m++)
                    for (int n = 0; n < 8; n++) {
                        const double x = tc_dtt(kv, i, m) * tc_dtt(kh, j, n);
                        const uint16_t hi = tc_half_bits(x, fmt);
                        const uint16_t lo = tc_half_bits(x - tc_half_value(hi, fmt), fmt);
                        const uint32_t off = tp::tc_sw_off(i * 8 + j, m * 8 + n);
                        img[(q * tp::kTcBQuadBytes + off) / 2] = hi;
                        img[((4 + q) * tp::kTcBQuadBytes + off) / 2] = lo;
                    }
    }
}

std::mutex g_tcb_mutex;
unsigned long long g_tcb_ctx[128];
bool g_tcb_ready[128];

/* the B tables on the current device (built and copied on first use) and the
 * device address of the table of (fmt, stage) */
int tc_tables(int fmt, int stage, const unsigned char **out)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return fail(TP_ERR_NO_DEVICE, "cudaGetDevice: %s", cudaGetErrorString(e));
    if (dev < 0 || dev >= 128) return fail(TP_ERR_NO_DEVICE, "device %d", dev);
    std::lock_guard<std::mutex> lock(g_tcb_mutex);
    const unsigned long long ctx = current_context_id();
    if (!g_tcb_ready[dev] || ctx == 0 || ctx != g_tcb_ctx[dev]) {
        static uint16_t img[2][kTcStagesN][tp::kTcBTableHalves];
        for (int f = 0; f < 2; f++)
            for (int st = 0; st < kTcStagesN; st++) tc_build_table(f, st, img[f][st]);
        e = cudaMemcpyToSymbol(g_tc_btab, img, sizeof(img));
        if (e != cudaSuccess) return fail(TP_ERR_CUDA, "tensor-core tables: %s", cudaGetErrorString(e));
        const int zero = 0;
        e = cudaMemcpyToSymbol(g_tc_err, &zero, sizeof(zero));
        if (e != cudaSuccess) return fail(TP_ERR_CUDA, "tensor-core status: %s", cudaGetErrorString(e));
        g_tcb_ready[dev] = true;
        g_tcb_ctx[dev] = current_context_id();
    }
    void *p = nullptr;
    e = cudaGetSymbolAddress(&p, g_tc_btab);
    if (e != cudaSuccess) return fail(TP_ERR_CUDA, "cudaGetSymbolAddress(tables): %s", cudaGetErrorString(e));
    *out = static_cast<const unsigned char *>(p) + ((size_t)fmt * kTcStagesN + stage) * tp::kTcBBytes;
    return TP_OK;
}

int tc_err_ptr(int **out)
{
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_tc_err);
    if (e != cudaSuccess) return fail(TP_ERR_CUDA, "cudaGetSymbolAddress(status): %s", cudaGetErrorString(e));
    *out = static_cast<int *>(p);
    return TP_OK;
}

/* the power of two that keeps |x| * scale below 2^15 for |x| <= bound */
float tc_fp16_scale(double bound)
{
    if (!(bound > 0.0)) return 1.0f;
    int e = 0;
    (void)frexp(bound, &e); /* bound < 2^e */
    return ldexpf(1.0f, 15 - e);
}

bool g_corr_tc_attr[2][128], g_inv_tc_attr[2][128], g_fwd_tc_attr[2][128];

/* one persistent CTA per SM (at most one per 128-row block) of the shared
 * tensor-core pipeline for stage S */
template <class S>
int tc_launch(const S &st, int format, int stage, bool (*attr)[128], tp_stream_t stream, const char *what)
{
    const unsigned char *btab = nullptr;
    int *err = nullptr;
    int rc;
    if ((rc = tc_tables(format, stage, &btab)) || (rc = tc_err_ptr(&err))) return rc;
    constexpr int smem = tp::tc_stage_smem(S::kQuads, S::kMeta, S::kAStages);
    const void *kern = format == TP_TC_BF16X2 ? (const void *)tp::k_tc_stage<S, TP_TC_BF16X2>
                                              : (const void *)tp::k_tc_stage<S, TP_TC_FP16X2>;
    if ((rc = set_smem_once(attr[format], kern, smem, what))) return rc;
    const long long blocks = (st.rows() + tp::kTcRows - 1) / tp::kTcRows;
    if (blocks <= 0) return TP_OK;
    int sms;
    if ((rc = sm_count(&sms))) return rc;
    const unsigned grid = (unsigned)(blocks < sms ? blocks : sms);
    if (format == TP_TC_BF16X2)
        tp::k_tc_stage<S, TP_TC_BF16X2><<<grid, S::kThreads, smem, (cudaStream_t)stream>>>(st, btab, err);
    else
        tp::k_tc_stage<S, TP_TC_FP16X2><<<grid, S::kThreads, smem, (cudaStream_t)stream>>>(st, btab, err);
    return cuda_status(cudaGetLastError(), what);
}

} /* namespace */

static int inv_tc_launch(const tp::InvTcStage &st, int format, tp_stream_t stream)
{
    return tc_launch(st, format, kTcStageInv, g_inv_tc_attr, stream, "inverse CLT (tensor cores)");
}

extern "C" {

int tp_tc_status(int *timed_out, int clear)
{
    if (!timed_out) return fail(TP_ERR_ARG, "timed_out is NULL");
    const unsigned char *unused;
    int rc = tc_tables(0, 0, &unused);
    if (rc) return rc;
    cudaError_t e = cudaMemcpyFromSymbol(timed_out, g_tc_err, sizeof(int));
    if (e != cudaSuccess) return fail(TP_ERR_CUDA, "tensor-core status: %s", cudaGetErrorString(e));
    if (clear) {
        const int zero = 0;
        e = cudaMemcpyToSymbol(g_tc_err, &zero, sizeof(zero));
        if (e != cudaSuccess) return fail(TP_ERR_CUDA, "tensor-core status: %s", cudaGetErrorString(e));
    }
    return TP_OK;
}

int tp_convert_correct_tiles_tma(const tp_geometry *g, float *const *kernel_offsets, float *const *kernels,
                                 float *const *images, const tp_task *tasks, float *const *clt, size_t dstride,
                                 int num_tiles, int lpf_mask, tp_stream_t stream)
{
    tp::Geom gd;
    int rc = check_geometry(g, &gd);
    if (rc) return rc;
    if (!kernel_offsets || !kernels || !images || !clt) return fail(TP_ERR_ARG, "NULL pointer array");
    if (num_tiles < 0) return fail(TP_ERR_ARG, "num_tiles %d < 0", num_tiles);
    if (num_tiles > 0 && !tasks) return fail(TP_ERR_ARG, "tasks is NULL");
    if (dstride < (size_t)g->img_width) return fail(TP_ERR_ARG, "dstride %zu < width %d", dstride, g->img_width);
    if (num_tiles == 0) return TP_OK;
    int sms, *err;
    if ((rc = sm_count(&sms)) || (rc = tc_err_ptr(&err))) return rc;
    if ((rc = set_smem_once(g_cv_attr, (const void *)tp::k_convert_tma, tp::kCvSmemBytes,
                            "cudaFuncSetAttribute(k_convert_tma)")))
        return rc;
    const long long items = (long long)((num_tiles + 3) / 4) * 12;
    const unsigned grid = grid_for(items, 1, sms, 2);
    tp::k_convert_tma<<<grid, tp::kCvThreads, tp::kCvSmemBytes, (cudaStream_t)stream>>>(
        gd, dstride, kernel_offsets, kernels, images, tasks, clt, num_tiles, lpf_mask, err);
    return cuda_status(cudaGetLastError(), "convert_correct_tiles_tma launch");
}

int tp_tc_table_image(int format, int stage, void *out)
{
    if (format != TP_TC_FP16X2 && format != TP_TC_BF16X2) return fail(TP_ERR_ARG, "format %d", format);
    if (stage < 0 || stage >= kTcStagesN) return fail(TP_ERR_ARG, "stage %d", stage);
    if (!out) return fail(TP_ERR_ARG, "out is NULL");
    tc_build_table(format, stage, static_cast<uint16_t *>(out));
    return TP_OK;
}

int tp_convert_correct_tiles_tc(const tp_geometry *g, float *const *kernel_offsets, float *const *kernels,
                                float *const *images, const tp_task *tasks, float *const *clt, size_t dstride,
                                int num_tiles, int lpf_mask, int format, tp_stream_t stream)
{
    tp::Geom gd;
    int rc = check_geometry(g, &gd);
    if (rc) return rc;
    if (format != TP_TC_FP16X2 && format != TP_TC_BF16X2) return fail(TP_ERR_ARG, "format %d", format);
    if (!kernel_offsets || !kernels || !images || !clt) return fail(TP_ERR_ARG, "NULL pointer array");
    if (num_tiles < 0) return fail(TP_ERR_ARG, "num_tiles %d < 0", num_tiles);
    if (num_tiles > 0 && !tasks) return fail(TP_ERR_ARG, "tasks is NULL");
    if (dstride < (size_t)g->img_width) return fail(TP_ERR_ARG, "dstride %zu < width %d", dstride, g->img_width);
    if (num_tiles == 0) return TP_OK;
    const tp::FwdTcStage st{gd, dstride, kernel_offsets, kernels, images, tasks, clt, num_tiles, lpf_mask};
    return tc_launch(st, format, kTcStageFwd, g_fwd_tc_attr, stream, "convert_correct_tiles_tc");
}

int tp_correlate2D_tc(const tp_geometry *g, float *const *clt, int colors, float scale0, float scale1,
                      float scale2, float fat_zero, size_t num_corr_tiles, const int *corr_indices,
                      size_t corr_stride, int corr_radius, float *corrs, int format, tp_stream_t stream)
{
    tp::Geom gd;
    int rc = check_geometry(g, &gd);
    if (rc) return rc;
    if (format != TP_TC_FP16X2 && format != TP_TC_BF16X2) return fail(TP_ERR_ARG, "format %d", format);
    if (!clt) return fail(TP_ERR_ARG, "clt is NULL");
    if (colors != 1 && colors != 3) return fail(TP_ERR_ARG, "colors %d (1 or 3)", colors);
    if (corr_radius < 0 || corr_radius > TP_MAX_CORR_RADIUS)
        return fail(TP_ERR_ARG, "corr_radius %d outside 0..%d", corr_radius, TP_MAX_CORR_RADIUS);
    const size_t sz = (size_t)(2 * corr_radius + 1) * (2 * corr_radius + 1);
    if (num_corr_tiles == 0) return TP_OK;
    if (!corr_indices || !corrs) return fail(TP_ERR_ARG, "NULL corr_indices / corrs");
    if (corr_stride < sz) return fail(TP_ERR_ARG, "corr_stride %zu < (2r+1)^2 = %zu", corr_stride, sz);
    /* the final LPF bounds the normalised product */
    double bound = 0.0;
    for (int i = 0; i < 64; i++) bound = fmax(bound, fabs((double)g_lpf_host[5][i]));
    const float up = format == TP_TC_FP16X2 ? tc_fp16_scale(bound) : 1.0f;
    const tp::CorrTcStage st{gd, clt, colors, scale0, scale1, scale2, fat_zero, (long long)num_corr_tiles,
                             corr_indices, corr_stride, corr_radius, corrs, up};
    return tc_launch(st, format, kTcStageCorr, g_corr_tc_attr, stream, "correlate2D_tc");
}

int tp_textures_accumulate_tc(const tp_geometry *g, const int *woi, float *const *clt, size_t num_texture_tiles,
                              const int *texture_indices, const float *port_offsets, int colors, int is_lwir,
                              float min_shot, float scale_shot, float diff_sigma, float diff_threshold,
                              float min_agree, float weight0, float weight1, float weight2, int dust_remove,
                              int keep_weights, size_t texture_rbg_stride, float *texture_rbg, size_t texture_stride,
                              float *texture_tiles, float *const *tile_scratch, int format, tp_stream_t stream)
{
    (void)is_lwir; (void)diff_threshold; (void)min_agree; /* accepted, unused (as in the reference) */
    tp::Geom gd;
    int rc = check_geometry(g, &gd);
    if (rc) return rc;
    if (format != TP_TC_FP16X2 && format != TP_TC_BF16X2) return fail(TP_ERR_ARG, "format %d", format);
    tp::TextureParams p;
    if ((rc = texture_params(colors, min_shot, scale_shot, diff_sigma, weight0, weight1, weight2, dust_remove,
                             keep_weights, &p)))
        return rc;
    if (num_texture_tiles == 0) return TP_OK;
    if (!clt || !texture_indices || !port_offsets || !tile_scratch)
        return fail(TP_ERR_ARG, "NULL clt / indices / port_offsets / tile_scratch");
    const bool want_rbg = texture_rbg && texture_rbg_stride;
    const bool want_tiles = texture_tiles && texture_stride;
    if (want_rbg && !woi) return fail(TP_ERR_ARG, "woi is NULL with an RGBA image output");
    const int ns = (colors == 3) ? (keep_weights ? 12 : 4) : (keep_weights ? 8 : 2);
    if (want_tiles && texture_stride < (size_t)ns * 256)
        return fail(TP_ERR_ARG, "texture_stride %zu < %d slices x 256", texture_stride, ns);
    const tp::InvTcStage st{gd, clt, tile_scratch, nullptr, (long long)num_texture_tiles, texture_indices, colors};
    if ((rc = inv_tc_launch(st, format, stream))) return rc;
    int sms;
    if ((rc = sm_count(&sms))) return rc;
    if ((rc = texture_smem_setup())) return rc;
    unsigned grid = grid_for((long long)num_texture_tiles, 1, sms, shape_per_sm(TP_SHAPE_TEXTURES));
    tex_kernel<true, true>(colors)<<<grid, tp::kTexThreads, tp::kTexSmemBytes, (cudaStream_t)stream>>>(
        gd, woi, tile_scratch, (long long)num_texture_tiles, texture_indices, nullptr, 0, 0, 0, port_offsets, p,
        want_rbg ? texture_rbg_stride : 0, want_rbg ? texture_rbg : nullptr, want_tiles ? texture_stride : 0,
        want_tiles ? texture_tiles : nullptr);
    return cuda_status(cudaGetLastError(), "textures_accumulate_tc launch");
}

int tp_generate_RBGA_tc(const tp_geometry *g, tp_task *tasks, int num_tiles, int *texture_indices,
                        int *num_texture_tiles, int *woi, int width, int height, float *const *clt,
                        const float *port_offsets, int colors, int is_lwir, float min_shot, float scale_shot,
                        float diff_sigma, float diff_threshold, float min_agree, float weight0, float weight1,
                        float weight2, int dust_remove, int keep_weights, size_t texture_rbga_stride,
                        float *texture_tiles, float *const *tile_scratch, int format, tp_stream_t stream)
{
    (void)is_lwir; (void)diff_threshold; (void)min_agree; (void)keep_weights;
    if (format != TP_TC_FP16X2 && format != TP_TC_BF16X2) return fail(TP_ERR_ARG, "format %d", format);
    if (!tile_scratch) return fail(TP_ERR_ARG, "tile_scratch is NULL");
    return generate_rbga(g, tasks, num_tiles, texture_indices, num_texture_tiles, woi, width, height, clt,
                         port_offsets, colors, min_shot, scale_shot, diff_sigma, weight0, weight1, weight2,
                         dust_remove, texture_rbga_stride, texture_tiles, 0, INT_MAX, tile_scratch, format, stream);
}

} /* extern "C" */

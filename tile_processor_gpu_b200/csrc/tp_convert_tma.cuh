/*
 * tp_convert_tma.cuh - convert_correct_tiles with the Bayer windows staged in
 * shared memory by TMA (the drop-in for the reference's convert_correct_tiles,
 * src/TileProcessor.cuh:1859-1937 with convertCorrectTile :3106-3635; the
 * same per-job arithmetic as k_convert_correct_tiles, so the CLT is
 * bit-identical to it).
 *
 * Work item: one (camera, colour) of four consecutive tasks, as the plain
 * kernel's warps take them.  Per block one producer warp and kCvConsumers
 * consumer warps around a ring of kCvSlots items:
 *   producer: eight items per pass, lane = (item, task): reads the task,
 *     computes the job's geometry (kernel tile, corner, shifts), writes it to
 *     the slot's metadata, prefetches the kernel tile into L2 and, for a
 *     window inside the image, loads the 16 x 20 box at the 16-byte boundary
 *     at or left of the corner into the slot with the TMA unit's bulk
 *     copies (one 80-byte copy per row: the images arrive as a device
 *     array of pointers, so no tensor map can be encoded for them on the
 *     host);
 *     one lane per item arms the slot's `full` mbarrier with the item's bytes;
 *   consumer warp c: items c, c + kCvConsumers, ...; waits for the slot,
 *     folds the four jobs (one 8-lane group each) from the staged windows
 *     (border windows: the global-memory path with the reference's clamps),
 *     releases the slot (its `empty` mbarrier) and finishes the jobs
 *     (transforms, convolution, shifts, store) while the producer refills it.
 * Every wait is bounded; one that runs out sets *err and stops the block's
 * work (the CLT is then incomplete); the producer waits (bounded) for its
 * last loads before it exits.
 */
#pragma once
#include "tp_convert.cuh"
#include "tp_tcgen05.cuh"

namespace tp {

constexpr int kCvConsumers = 8;
constexpr int kCvThreads = 32 * (kCvConsumers + 1);
constexpr int kCvSlots = 2 * kCvConsumers;
constexpr int kCvBatch = 8; /* items per producer pass: 32 lanes = 8 items x 4 tasks */
constexpr int kCvWinBytes = kCvWinW * kCvWinH * 4;
static_assert(kCvWinBytes % 128 == 0, "windows start on 128-byte boundaries");
static_assert(kCvSlots % kCvConsumers == 0 && kCvSlots >= kCvBatch, "ring");

/* one job's metadata in a slot */
struct __align__(16) CvMeta {
    JobGeometry jg;
    int task;     /* 0: no job (empty task, out of range, past the list) */
    int txy;
    int fast;     /* the window was staged by TMA */
    int dx;       /* corner - staged box's first column (0..3) */
};

constexpr size_t kCvSmemBytes = (size_t)kCvSlots * 4 * (kCvWinBytes + sizeof(CvMeta)) + 128;

__device__ __forceinline__ void cv_arrive(uint32_t mbar)
{
    asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.shared::cta.b64 st, [%0];\n\t}\n" ::"r"(mbar) : "memory");
}

__global__ void __launch_bounds__(kCvThreads, 2) k_convert_tma(
    Geom g, size_t dstride, float *const *kernel_offsets, float *const *kernels, float *const *images,
    const tp_task *__restrict__ tasks, float *const *clt, int num_tiles, int lpf_mask, int *__restrict__ err)
{
    extern __shared__ __align__(128) unsigned char cv_smem[];
    __shared__ __align__(8) uint64_t bars[2 * kCvSlots]; /* full[slot], then empty[slot] */
    __shared__ float tbuf[kCvConsumers * 4][8][9];
    const uint32_t base_s = (uint32_t)__cvta_generic_to_shared(cv_smem);
    const uint32_t pad = (128 - (base_s & 127)) & 127;
    unsigned char *sm = cv_smem + pad;
    const uint32_t a_win = base_s + pad;
    CvMeta *meta = reinterpret_cast<CvMeta *>(sm + (size_t)kCvSlots * 4 * kCvWinBytes);
    const uint32_t a_bar = (uint32_t)__cvta_generic_to_shared(bars);
    auto full = [&](int s) { return a_bar + 8u * (uint32_t)s; };
    auto empty = [&](int s) { return a_bar + 8u * (uint32_t)(kCvSlots + s); };
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    if (tid == 0) {
        for (int b = 0; b < 2 * kCvSlots; b++)
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(a_bar + 8 * b) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    const int chunks = (num_tiles + 3) >> 2;
    const long long total = (long long)chunks * 12;
    /* this block's items: blockIdx.x + k gridDim.x, k < nitems */
    const long long nitems = blockIdx.x < total ? (total - blockIdx.x + gridDim.x - 1) / gridDim.x : 0;
    bool ok = true;

    if (warp == kCvConsumers) {
        /* ---- producer: eight items per pass, lane = (item, task) ---- */
        long long filled = 0; /* items whose slots have been armed */
        for (long long k0 = 0; k0 < nitems && ok; k0 += kCvBatch) {
            const int ib = lane >> 2, j = lane & 3;
            const long long k = k0 + ib;
            const bool item = k < nitems;
            const int slot = (int)(k % kCvSlots);
            /* the item kCvSlots before has been folded by its consumer */
            if (item && k >= kCvSlots) ok = tc_wait(empty(slot), (uint32_t)((k / kCvSlots - 1) & 1));
            if (!__all_sync(0xffffffffu, ok)) {
                ok = false;
                break;
            }
            CvMeta m;
            m.jg = JobGeometry{};
            m.task = 0;
            m.txy = 0;
            m.fast = 0;
            m.dx = 0;
            int cam = 0;
            if (item) {
                const long long w = blockIdx.x + k * gridDim.x;
                const int chunk = (int)(w / 12), r = (int)(w - (long long)chunk * 12);
                const int color = r >> 2, n = chunk * 4 + j;
                cam = r & 3;
                if (n < num_tiles) {
                    const tp_task *t = tasks + n;
                    const int task = __ldg(&t->task), txy = __ldg(&t->txy);
                    const int tx = txy & 0xfff, ty = txy >> 16;
                    if (task && tx < g.TX && ty >= 0 && ty < g.TY) {
                        m.task = task;
                        m.txy = txy;
                        m.jg = job_geometry(g, kernel_offsets[cam], __ldg(&t->xy[cam][0]), __ldg(&t->xy[cam][1]),
                                            color, nullptr);
                        /* the in-image condition of fold_rows, and rows that start on
                         * 16-byte boundaries for the bulk copies */
                        m.fast = (m.jg.itlx >= 0) && (m.jg.itlx < g.W - 16) && (m.jg.itly >= 0) &&
                                 (m.jg.itly < g.H - 16) && !(dstride & 3) &&
                                 !(reinterpret_cast<uintptr_t>(images[cam]) & 15);
                        m.dx = m.jg.itlx & 3;
                        const float *kt = kernels[cam] + m.jg.kidx * 256;
#pragma unroll
                        for (int q = 0; q < 8; q++) asm volatile("prefetch.global.L2 [%0];" ::"l"(kt + q * 32));
                    }
                }
                meta[slot * 4 + j] = m;
            }
            const unsigned fm = __ballot_sync(0xffffffffu, item && m.fast);
            __syncwarp();
            /* one lane per item arms its slot with the bytes its loads bring */
            if (item && j == 0)
                tc_expect(full(slot), (uint32_t)(__popc((fm >> (4 * ib)) & 0xFu) * kCvWinBytes));
            __syncwarp();
            if (item && m.fast) {
                /* the window's 16 rows of 20 floats, one bulk copy each */
                const float *src = images[cam] + (size_t)m.jg.itly * dstride + (m.jg.itlx & ~3);
                const uint32_t dst = a_win + (uint32_t)((slot * 4 + j) * kCvWinBytes);
#pragma unroll 4
                for (int rr = 0; rr < kCvWinH; rr++)
                    tc_bulk_load(dst + (uint32_t)(rr * kCvWinW * 4), src + (size_t)rr * dstride,
                                 (uint32_t)(kCvWinW * 4), full(slot));
            }
            filled = k0 + kCvBatch < nitems ? k0 + kCvBatch : nitems;
        }
        /* the last fill of every slot has landed before this warp exits */
        if (lane < kCvSlots && lane < filled) {
            const long long last = lane + ((filled - 1 - lane) / kCvSlots) * kCvSlots;
            (void)tc_wait(full(lane), (uint32_t)((last / kCvSlots) & 1));
        }
    } else {
        /* ---- consumers: warp c takes items c, c + kCvConsumers, ... ---- */
        const int grp = lane >> 3, l = lane & 7;
        const unsigned gm = group_mask();
        for (long long k = warp; k < nitems; k += kCvConsumers) {
            const int slot = (int)(k % kCvSlots);
            if (ok) ok = tc_wait(full(slot), (uint32_t)((k / kCvSlots) & 1));
            if (!__all_sync(0xffffffffu, ok)) {
                ok = false;
                break;
            }
            const CvMeta m = meta[slot * 4 + grp];
            const long long w = blockIdx.x + k * gridDim.x;
            const int chunk = (int)(w / 12), r = (int)(w - (long long)chunk * 12);
            const int color = r >> 2, cam = r & 3;
            float P[8], Q[8];
            if (m.task) {
                const float *win =
                    m.fast ? reinterpret_cast<const float *>(sm + (size_t)(slot * 4 + grp) * kCvWinBytes) : nullptr;
                fold_rows(g, dstride, images[cam], m.jg, color, l, P, Q, win, m.dx);
            }
            /* the window and the metadata read: the slot may be refilled */
            __syncwarp();
            if (lane == 0) cv_arrive(empty(slot));
            if (m.task) {
                const int tx = m.txy & 0xfff, ty = m.txy >> 16;
                float *out = clt[cam] + (((size_t)ty * g.TX + tx) * 3 + color) * 256;
                convert_finish<true>(kernels[cam], m.jg, color, lpf_mask, out, tbuf[warp * 4 + grp], l, gm, P, Q);
            }
        }
    }
    if (!ok && err) atomicExch(err, 1);
}

} /* namespace tp */

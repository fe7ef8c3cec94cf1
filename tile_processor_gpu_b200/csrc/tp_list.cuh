/*
 * tp_list.cuh - texture tile list, window of interest and RGBA clear (the
 * drop-ins for the reference's clear_texture_list, mark_texture_tiles,
 * mark_texture_neighbor_tiles, gen_texture_list and clear_texture_rbga,
 * src/TileProcessor.cuh:1618-1853).
 *
 * The reference launches these from a one-thread dynamic-parallelism driver
 * and synchronises on the device; here they are ordinary kernels issued back
 * to back on one stream, and every value the reference computed on the driver
 * thread (initial window, cleared counters, final width/height, clear extent)
 * is produced by a one-thread kernel or read from device memory by the next
 * kernel, so a whole generate_RBGA sequence needs no host round trip and can
 * be captured in a CUDA graph.
 */
#pragma once
#include "tp_common.cuh"

namespace tp {

/* First statements of every kernel of the list / RGBA-clear sequence, which
 * the host launches as a chain of programmatic dependents: wait for the
 * launch before (everything it wrote is then visible), and only then let the
 * next one be scheduled.  A kernel that starts early therefore only ever runs
 * ahead of its own predecessor, never of the kernels before that. */
__device__ __forceinline__ void chain_entry()
{
    grid_dependency_wait();
    grid_dependents_launch();
}

/* marker grid: cols 0..width (inclusive, as the reference), rows 0..height-1 */
__global__ void k_clear_texture_list(int *idx, int width, int height, int TX, long long cap)
{
    chain_entry();
    const int col = blockIdx.x * blockDim.x + threadIdx.x;
    const int row = blockIdx.y;
    if (col > width || row >= height) return;
    const long long i = (long long)col + (long long)row * TX;
    if (i >= 0 && i < cap) idx[i] = 0;
}

__global__ void k_mark_texture_tiles(const tp_task *__restrict__ tasks, int num_tiles, int *idx, int TX,
                                     long long cap)
{
    chain_entry();
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= num_tiles) return;
    if (!(tasks[n].task & TP_TASK_TEXTURE_BITS)) return;
    const int cxy = tasks[n].txy;
    const long long i = (long long)(cxy & 0xffff) + (long long)(cxy >> 16) * TX;
    if (i >= 0 && i < cap) idx[i] = 1;
}

__global__ void k_woi_init(int *woi, int *counts, int TX, int TY)
{
    chain_entry();
    if (threadIdx.x == 0) {
        woi[0] = TX; woi[1] = TY; woi[2] = 0; woi[3] = 0;
    }
    if (threadIdx.x < 8) counts[threadIdx.x] = 0;
}

__device__ __forceinline__ int marker_at(const int *idx, long long i, long long cap)
{
    return (i >= 0 && i < cap) ? idx[i] : 0;
}

__global__ void k_mark_neighbor_tiles(tp_task *tasks, int num_tiles, const int *idx, int *woi, int TX,
                                      int TY, long long cap)
{
    chain_entry();
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= num_tiles) return;
    const int task = tasks[n].task;
    if (!(task & TP_TASK_TEXTURE_BITS)) return;
    const int cxy = tasks[n].txy;
    const int x = cxy & 0xffff, y = cxy >> 16;
    atomicMin(woi + 0, x);
    atomicMin(woi + 1, y);
    atomicMax(woi + 2, x);
    atomicMax(woi + 3, y);
    int d = 0;
    if (y > 0 && marker_at(idx, x + (long long)(y - 1) * TX, cap)) d |= 1;
    if (x < TX - 1 && marker_at(idx, (x + 1) + (long long)y * TX, cap)) d |= 2;
    if (y < TY - 1 && marker_at(idx, x + (long long)(y + 1) * TX, cap)) d |= 4;
    if (x > 0 && marker_at(idx, (x - 1) + (long long)y * TX, cap)) d |= 8;
    tasks[n].task = ((task ^ d) & TP_TASK_TEXTURE_BITS) ^ task;
}

/* Eight sub-lists: 2x2 tile parity x {inner, border}; inner lists grow up from
 * the start of their quarter of the buffer, border lists down from its end.
 * Slots are claimed with one atomic per (warp, sub-list). */
__global__ void k_gen_texture_list(const tp_task *__restrict__ tasks, int num_tiles, int *idx,
                                   int *counts, const int *woi, int TX, int quarter, long long cap,
                                   int row_first, int row_last)
{
    chain_entry();
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    const int lane = threadIdx.x & 31;
    int slot = -1, entry = 0, head = 0;
    if (n < num_tiles) {
        const int task = tasks[n].task & TP_TASK_TEXTURE_BITS;
        const int cxy = tasks[n].txy;
        const int x = cxy & 0xffff, y = cxy >> 16;
        /* tiles outside [row_first, row_last) stay marked (they set their
         * neighbours' bits and the window) but are not listed */
        if (task && y >= row_first && y < row_last) {
            const int border = (x == woi[0]) || (y == woi[1]) || (x == TX - 1) || (y == woi[3]);
            slot = 0;
            if (x & 1) { head += quarter; slot += 2; }
            if (y & 1) { head += 2 * quarter; slot += 4; }
            if (border) { head += quarter - 1; slot += 1; }
            entry = task | ((x + y * TX) << 8) | (1 << 7);
        }
    }
    const unsigned same = __match_any_sync(0xffffffffu, slot);
    if (slot < 0) return;
    const int leader = __ffs(same) - 1;
    int base = 0;
    if (lane == leader) base = atomicAdd(counts + slot, __popc(same));
    base = __shfl_sync(same, base, leader);
    const int k = base + __popc(same & ((1u << lane) - 1u));
    const long long pos = (slot & 1) ? (long long)head - k : (long long)head + k;
    if (pos >= 0 && pos < cap) idx[pos] = entry;
}

__global__ void k_woi_finalize(int *woi)
{
    chain_entry();
    if (threadIdx.x == 0) {
        woi[2] += 1 - woi[0];
        woi[3] += 1 - woi[1];
    }
}

/* Zero the RGBA slices: the reference clears (woi_w + 1) * 8 columns plus the
 * 8 floats a thread writes past them when the grid reaches that far, over
 * (woi_h + 1) * 8 * (colors + 1) rows.  woi == NULL: explicit extent. */
__global__ void k_clear_rbga(const int *woi, int colors, int texture_width, int slice_height,
                             size_t stride, float *buf)
{
    chain_entry();
    int tw = texture_width, rows = slice_height;
    if (woi) {
        tw = (woi[2] + 1) * 8;
        rows = (woi[3] + 1) * 8 * (colors + 1);
    }
    if (tw <= 0 || rows <= 0) return;
    const long long reach = ((long long)(tw + 255) / 256) * 256;
    long long cols = (long long)tw + 8;
    if (cols > reach) cols = reach;
    if (cols > (long long)stride) cols = (long long)stride;
    /* one block per row (grid-stride); 16-byte stores when every row starts
     * on a 16-byte boundary, the last cols % 4 floats one by one */
    const bool vec = !(reinterpret_cast<uintptr_t>(buf) & 15) && !(stride & 3);
    const long long quads = vec ? cols >> 2 : 0;
    for (long long row = blockIdx.x; row < rows; row += gridDim.x) {
        float *p = buf + (size_t)row * stride;
        float4 *p4 = reinterpret_cast<float4 *>(p);
        for (long long q = threadIdx.x; q < quads; q += blockDim.x) p4[q] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        for (long long c = quads * 4 + threadIdx.x; c < cols; c += blockDim.x) p[c] = 0.0f;
    }
}

} /* namespace tp */

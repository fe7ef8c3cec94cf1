/*
 * tp_io.cpp - host-side helpers for the reference harness's data files and
 * lists (src/dtt8x8.cu:144-165 readFloatsFromFile / writeFloatsToFile,
 * :383-446 task and correlation lists).  No CUDA: plain files and host arrays.
 *
 * The harness's files are raw native-endian float32 arrays without headers:
 *   *.kernel          [kernels_vert][kernels_hor][3][4][8][8]
 *   *.kernel_offsets  [kernels_vert][kernels_hor][3][8]   (struct CltExtra)
 *   *.bayer           [img_height][img_width]              (unpitched)
 *   *.portsxy         [tilesy * tilesx][2]                 (tile centre per camera)
 *   *.clt             [tilesy][tilesx][3][4][8][8]
 *   *.rbg             [3][img_height + 8][img_width + 8]
 *   *.corr            [num_corr][(2r+1)^2]
 *   texture *.rgba    [num_texture_tiles][slices * 256], or the overlapped
 *                     window [slices][(woi_h+1)*8][(woi_w+1)*8]
 */
#include <stdio.h>
#include <string.h>

#include "../../include/tp_b200.h"

extern "C" {

long long tp_read_floats(const char *path, float *dst, size_t count)
{
    if (!path || (!dst && count)) return TP_ERR_ARG;
    FILE *f = fopen(path, "rb");
    if (!f) return TP_ERR_ARG;
    const size_t got = count ? fread(dst, sizeof(float), count, f) : 0;
    fclose(f);
    return (long long)got;
}

long long tp_write_floats(const char *path, const float *src, size_t count)
{
    if (!path || (!src && count)) return TP_ERR_ARG;
    FILE *f = fopen(path, "wb");
    if (!f) return TP_ERR_ARG;
    const size_t put = count ? fwrite(src, sizeof(float), count, f) : 0;
    const int rc = fclose(f);
    if (put != count || rc != 0) return TP_ERR_ARG;
    return (long long)put;
}

int tp_tasks_from_portsxy(const float *const *portsxy, int tilesx, int tilesy, int task_bits, tp_task *tasks)
{
    if (!portsxy || !tasks || tilesx <= 0 || tilesy <= 0 || tilesx > 0xffff || tilesy > 0x7fff) return TP_ERR_ARG;
    for (int c = 0; c < TP_NUM_CAMS; c++)
        if (!portsxy[c]) return TP_ERR_ARG;
    for (int ty = 0; ty < tilesy; ty++)
        for (int tx = 0; tx < tilesx; tx++) {
            const int nt = ty * tilesx + tx;
            tasks[nt].task = task_bits;
            tasks[nt].txy = tx + (ty << 16);
            for (int c = 0; c < TP_NUM_CAMS; c++) {
                tasks[nt].xy[c][0] = portsxy[c][2 * nt];
                tasks[nt].xy[c][1] = portsxy[c][2 * nt + 1];
            }
        }
    return tilesx * tilesy;
}

int tp_corr_indices_from_tasks(const tp_task *tasks, int num_tiles, int tilesx, int *corr_indices)
{
    if ((!tasks && num_tiles) || num_tiles < 0 || tilesx <= 0) return TP_ERR_ARG;
    int n = 0;
    for (int k = 0; k < num_tiles; k++) {
        const int pairs = (tasks[k].task >> TP_TASK_CORR_BITS) & ((1 << TP_NUM_PAIRS) - 1);
        if (!pairs) continue;
        const int txy = tasks[k].txy;
        const int tile = (txy & 0xffff) + (txy >> 16) * tilesx;
        for (int p = 0; p < TP_NUM_PAIRS; p++)
            if ((pairs >> p) & 1) {
                if (corr_indices) corr_indices[n] = (tile << TP_CORR_NTILE_SHIFT) | p;
                n++;
            }
    }
    return n;
}

} /* extern "C" */

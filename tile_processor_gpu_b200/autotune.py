"""Launch-shape tuner for the stage kernels.

The stage kernels walk their tiles with grid-stride loops over a grid capped
at `ctas_per_sm` x the SM count (tp_set_launch_shape); the cap decides how
many tiles each CTA takes in turn and how many CTAs share an SM.  The tuner
times the caller's own workload on the GPU under each candidate cap (CUDA
events on the current stream, after warm-up runs) and keeps the fastest.
The number of CTAs that fit on an SM at once (tp_resident_ctas) is reported
beside the timings: caps above it run the extra blocks as they free up, which
for the forward transform still helps (its blocks' work is uneven) and for
the texture kernel changes nothing.  Shapes are process-wide; a CUDA graph
keeps the shapes it was captured with.
"""
from . import _native

KERNELS = {"convert": 0, "correlate": 1, "textures": 2}
CANDIDATES = {"convert": (2, 3, 4, 6, 8, 12, 16),
              "correlate": (4, 6, 8, 12, 16),
              "textures": (5, 6, 7, 14, 21)}


def resident(kernel):
    """CTAs of the stage kernel that fit on one SM at once"""
    return _native.call("tp_resident_ctas", KERNELS[kernel])


def set_shape(kernel, ctas_per_sm):
    _native.call("tp_set_launch_shape", KERNELS[kernel], int(ctas_per_sm))


def get_shape(kernel):
    return _native.call("tp_get_launch_shape", KERNELS[kernel])


def time_ms(run, repeats, warmup):
    """Mean device time of run() over `repeats` calls after `warmup` calls."""
    import torch
    for _ in range(warmup):
        run()
    stream = torch.cuda.current_stream()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for _ in range(repeats):
        run()
    b.record(stream)
    torch.cuda.synchronize()
    return a.elapsed_time(b) / repeats


def tune(kernel, run, candidates=None, repeats=10, warmup=2):
    """Time run() (a workload that launches `kernel`) under each candidate
    cap; leave the fastest set.  Returns (best, {cap: ms})."""
    cands = tuple(candidates if candidates is not None else CANDIDATES[kernel])
    times = {}
    for c in cands:
        set_shape(kernel, c)
        times[c] = time_ms(run, repeats, warmup)
    best = min(times, key=times.get)
    set_shape(kernel, best)
    return best, times


def tune_stages(stages, repeats=10, warmup=2):
    """stages: {kernel name: run callable}, tuned one after another (each run
    needs its inputs in place, e.g. the CLT before correlate).  Returns
    {kernel: {"ctas_per_sm": best, "ms": {cap: ms}}}."""
    out = {}
    for kernel, run in stages.items():
        best, times = tune(kernel, run, repeats=repeats, warmup=warmup)
        out[kernel] = {"ctas_per_sm": best, "resident": resident(kernel),
                       "ms": {str(k): round(v, 4) for k, v in times.items()}}
    return out


def reset():
    for k in KERNELS:
        set_shape(k, 0)

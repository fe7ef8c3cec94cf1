"""CPU tests of the harness file and list helpers (tp_read_floats,
tp_write_floats, tp_tasks_from_portsxy, tp_corr_indices_from_tasks)."""
import numpy as np

from tile_processor_gpu_b200 import files, synth


def test_raw_float_round_trip(native, tmp_path):
    g = synth.geometry(256, 128)
    rng = np.random.default_rng(1)
    ker, ext = synth.kernel_tables(rng, g, pool=8)
    files.write_floats(tmp_path / "c0.kernel", ker[0])
    files.write_floats(tmp_path / "c0.kernel_offsets", ext[0])
    assert np.array_equal(files.read_kernels(tmp_path / "c0.kernel", g), ker[0])
    assert np.array_equal(files.read_kernel_offsets(tmp_path / "c0.kernel_offsets", g), ext[0])
    img = rng.random((128, 256), dtype=np.float32)
    files.write_floats(tmp_path / "c0.bayer", img)
    assert np.array_equal(files.read_bayer(tmp_path / "c0.bayer", g), img)
    assert (tmp_path / "c0.bayer").stat().st_size == 256 * 128 * 4


def test_full_frame_file_sizes():
    g = synth.geometry(2592, 1936)
    assert files.kernel_floats(g) == 164 * 123 * 3 * 4 * 64          # 62.0 MB per camera


def test_short_file_is_an_error(native, tmp_path):
    files.write_floats(tmp_path / "short.bayer", np.zeros(10, np.float32))
    g = synth.geometry(32, 32)
    try:
        files.read_bayer(tmp_path / "short.bayer", g)
    except OSError as e:
        assert "10 of 1024" in str(e)
    else:
        raise AssertionError("short file accepted")


def test_tasks_from_portsxy_and_corr_list(native, tmp_path):
    """Linescan tasks from the four *.portsxy files, as the harness builds
    them, and its correlation list."""
    g = synth.geometry(128, 64)
    tx, ty = 16, 8
    rng = np.random.default_rng(2)
    ports = [rng.uniform(0, 128, (tx * ty, 2)).astype(np.float32) for _ in range(4)]
    for c in range(4):
        files.write_floats(tmp_path / ("c%d.portsxy" % c), ports[c])
    got = files.tasks_from_portsxy([files.read_portsxy(tmp_path / ("c%d.portsxy" % c), g) for c in range(4)], g)
    assert got.size == tx * ty
    n = np.arange(tx * ty)
    assert np.array_equal(got["txy"], (n % tx) + ((n // tx) << 16))
    assert np.all(got["task"] == synth.ALL_TASK_BITS)
    for c in range(4):
        assert np.array_equal(got["xy"][:, c], ports[c])
    got["task"][3] = 0xF | (0b100101 << 4)
    got["task"][5] = 0xF
    idx = files.corr_indices(got, g)
    assert np.array_equal(idx, synth.corr_indices(got, g))
    assert idx.size == 6 * tx * ty - 3 - 6

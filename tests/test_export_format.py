"""File formats of the section-cut and history exports, read back the way the reference's
plotters read them (include/plotter/plotter.py:9-14; exportSectionCutPlot.h:994-1001).
Host only."""
import numpy as np

from periodicshiftlbm_b200.grid import exportHistoryData, write_section_cut


def test_section_file_reads_like_the_reference_plotter(tmp_path):
    sec = np.random.default_rng(0).normal(size=(7, 11, 5)).astype(np.float32)
    path = str(tmp_path / "sim_data.bin")
    write_section_cut(path, 42, sec)
    with open(path, "rb") as f:
        plot_number = np.fromfile(f, dtype=np.int32, count=1)[0]
        n_vertical, n_horizontal, n_vars = np.fromfile(f, dtype=np.int32, count=3)
        data = np.fromfile(f, dtype=np.float32).reshape((n_vertical, n_horizontal, n_vars))
    assert plot_number == 42 and (n_vertical, n_horizontal, n_vars) == (7, 11, 5)
    assert np.array_equal(data, sec)


def test_history_file_layout(tmp_path):
    path = str(tmp_path / "historyData.bin")
    exportHistoryData(np.arange(10, dtype=np.float32) * 0.5, 6, path)
    raw = open(path, "rb").read()
    assert np.frombuffer(raw[:4], dtype=np.int32)[0] == 7
    assert np.array_equal(np.frombuffer(raw[4:], dtype=np.float32), np.arange(7, dtype=np.float32) * 0.5)


def test_history_file_bytes_equal_reference_export(ref, tmp_path):
    """The library's exportHistoryData writes the bytes of the reference's own
    exportHistoryData (include/plotter/exportSectionCutPlot.h:994-1001, compiled into the
    reference build)."""
    hist = np.random.default_rng(3).normal(size=40).astype(np.float32)
    mine, theirs = str(tmp_path / "mine.bin"), str(tmp_path / "theirs.bin")
    exportHistoryData(hist, 17, mine)
    ref.export_history(hist, 17, theirs)
    assert open(mine, "rb").read() == open(theirs, "rb").read()

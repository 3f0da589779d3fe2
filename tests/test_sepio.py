"""The .H reader/writer: round trips, the reference's header conventions and,
when the reference tree is mounted, its own Python reader (seppy)."""
import os
import sys

import numpy as np
import pytest

from fwi3d_b200 import sepio


def test_round_trip_model_cube(tmp_path, monkeypatch):
    monkeypatch.chdir(tmp_path)
    rng = np.random.default_rng(0)
    m = rng.standard_normal((3, 5, 4, 6)).astype(np.float32)  # [param][y][x][z]
    axes = [sepio.Axis(6, 0.0, 0.01), sepio.Axis(4, 0.1, 0.02), sepio.Axis(5, 0.0, 0.03), sepio.Axis(3)]
    binp = sepio.write("model.H", m, axes, datapath=str(tmp_path))
    assert binp == str(tmp_path) + "/model.H@"
    a, ax = sepio.read("model.H")
    assert np.array_equal(a, m)
    assert [x.n for x in ax] == [6, 4, 5, 3]
    assert ax[1].o == pytest.approx(0.1) and ax[2].d == pytest.approx(0.03)


def test_reads_reference_style_header(tmp_path):
    """Header as binWrite writes it (IO.hpp:181-222), comments, quoted in=,
    trailing unit axes dropped down to ndim0."""
    data = np.arange(24, dtype=np.float32).reshape(2, 3, 4)
    data.tofile(tmp_path / "d.H@")
    (tmp_path / "d.H").write_text(
        "# written by hand\nn1=4\no1=0\nd1=0.004\nn2=3\no2=0\nd2=1\nn3=2\no3=0\nd3=1\n"
        "n4=1\no4=0\nd4=1\nesize=4\n" + f'in="{tmp_path}/d.H@"\n')
    a, ax = sepio.read(str(tmp_path / "d.H"))
    assert a.shape == (2, 3, 4) and np.array_equal(a, data)
    a4, ax4 = sepio.read(str(tmp_path / "d.H"), ndim0=4)
    assert a4.shape == (1, 2, 3, 4) and len(ax4) == 4


def test_size_mismatch_is_an_error(tmp_path):
    np.zeros(5, np.float32).tofile(tmp_path / "x.H@")
    (tmp_path / "x.H").write_text(f"n1=6\nesize=4\nin={tmp_path}/x.H@\n")
    with pytest.raises(ValueError, match="bytes"):
        sepio.read(str(tmp_path / "x.H"))


def _reference_tree() -> str:
    """The reference tree: FWI3D_REFERENCE, else the one the oracle recipe
    compiled from (oracle/_ref/REF_PATH); empty where neither exists."""
    if os.environ.get("FWI3D_REFERENCE"):
        return os.environ["FWI3D_REFERENCE"]
    rec = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref", "REF_PATH")
    try:
        with open(rec) as f:
            return f.read().strip()
    except OSError:
        return ""


REF_PY = os.path.join(_reference_tree(), "src", "python")


@pytest.mark.skipif(not os.path.exists(os.path.join(REF_PY, "seppy.py")), reason="reference tree not mounted")
def test_reference_reader_reads_our_files(tmp_path, monkeypatch):
    monkeypatch.syspath_prepend(REF_PY)
    import seppy

    monkeypatch.chdir(tmp_path)
    rng = np.random.default_rng(1)
    m = rng.standard_normal((2, 3, 7)).astype(np.float32)
    sepio.write("w.H", m, [sepio.Axis(7, 0, 0.5), sepio.Axis(3, 1, 2), sepio.Axis(2, 0, 1)], datapath=str(tmp_path))
    ax, dat = seppy.sep().read_file("w.H", form="native")
    assert list(ax.n) == [7, 3, 2]
    assert np.array_equal(dat.reshape(m.shape), m)

"""Writers (src/Writers.jl): the Xdmf 3 metadata against the reference's own
golden document (test/test_writers.jl, extracted by tests/golden/make_golden_writers.py),
Julia float printing, raw dumps, and write_h5's error without an HDF5 library."""
import os

import numpy as np
import pytest

from conftest import load_fastice

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "xdmf3_writers_ref.xml")


def test_xdmf3_matches_the_reference_golden_document(tmp_path):
    fi = load_fastice()
    grid = fi.UniformGrid(origin=(-0.4, -0.5, 0.0), extent=(1.0, 1.1, 1.2), dims=(4, 5, 6))
    path = tmp_path / "test.xdmf3"
    fields = {"Fa": np.ones((6, 5, 4)), "Fb": 2.0 * np.ones((6, 5, 4))}
    fi.write_xdmf(grid, str(path), fields, ("test.h5",))
    assert path.read_text(encoding="utf-8") == open(GOLDEN, encoding="utf-8").read()


def test_julia_float_printing():
    fi = load_fastice()
    jf = fi.writers.julia_float
    assert [jf(v) for v in (0.0, 0.25, -0.39, 1e-5, 2.5e20, 0.09999999999999999, -1e-7)] == \
        ["0.0", "0.25", "-0.39", "1.0e-5", "2.5e20", "0.09999999999999999", "-1.0e-7"]


def test_xdmf_time_series_and_binary_attributes(tmp_path):
    fi = load_fastice()
    grid = fi.UniformGrid(origin=(0.0, 0.0, 0.0), extent=(1.0, 1.0, 0.5), dims=(8, 4, 2))
    txt = fi.writers.xdmf_text(grid, ["P"], ("a.h5", "b.h5"), timesteps=[0.0, 0.5])
    assert txt.count('<Grid GridType="Uniform">') == 2 and 'Value="0.5"' in txt and "b.h5:/P" in txt
    with pytest.raises(ValueError):
        fi.writers.xdmf_text(grid, ["P"], ("a.raw",))
    data = np.arange(64, dtype=np.float64).reshape(2, 4, 8)
    files = fi.writers.write_raw(str(tmp_path / "step0"), {"P": data})
    np.testing.assert_array_equal(np.fromfile(files["P"], dtype="<f8").reshape(2, 4, 8), data)
    txt = fi.writers.xdmf_text(grid, ["P"], ("-",), data_format="binary", raw_names=[[files["P"]]])
    assert 'Format="Binary"' in txt and 'Endian="Little"' in txt and 'Dimensions="2 4 8"' in txt


def test_write_h5_without_hdf5_raises(tmp_path):
    fi = load_fastice()
    try:
        import h5py  # noqa: F401
        pytest.skip("h5py is installed")
    except ImportError:
        pass
    grid = fi.UniformGrid(origin=(0.0, 0.0, 0.0), extent=(1.0, 1.0, 1.0), dims=(2, 2, 2))
    with pytest.raises(fi.FastIceError):
        fi.write_h5(grid, str(tmp_path / "x.h5"), {"P": np.zeros((2, 2, 2))})

"""VTI output (glide/io.py:20-202): the reference's own writer's file (golden,
made by tests/golden/make_vti_golden.py) reads back to its inputs, and this
package's writer produces the same fields, time value and layout."""
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE / "golden"))


def test_reference_file_reads_back():
    from make_vti_golden import vti_fields
    from glide_b200.io import read_vti
    ref = read_vti(HERE / "golden" / "reference_write_vti.vti")
    f = vti_fields()
    assert ref["TimeValue"] == 3.5
    assert np.array_equal(ref["H"], np.flip(f["H"], 0))
    assert np.array_equal(ref["vel"], np.stack([np.flip(c, 0) for c in f["vel"]], axis=-1))


def test_write_vti_matches_reference_writer(tmp_path):
    from make_vti_golden import vti_fields
    from glide_b200.io import read_vti, write_vti
    mine = read_vti(write_vti(tmp_path / "mine.vti", vti_fields(), 1500.0, time_value=3.5))
    ref = read_vti(HERE / "golden" / "reference_write_vti.vti")
    assert set(mine) == set(ref)
    for k in ref:
        assert np.array_equal(np.asarray(mine[k]), np.asarray(ref[k]))


def test_writer_series_and_collection(tmp_path):
    from glide_b200.io import VTIWriter, read_vti
    rng = np.random.default_rng(2)
    with VTIWriter(tmp_path, base="run", dx=1000.0) as w:
        for k in range(3):
            w.write_step(k, 10.0 * k, {"H": rng.random((4, 6)), "vel": [rng.random((4, 6)), rng.random((4, 6))]})
        pvd = w.write_pvd()
    text = pvd.read_text()
    assert text.count("<DataSet") == 3 and 'file="run_0002.vti"' in text and 'timestep="20.0"' in text
    assert read_vti(tmp_path / "run_0001.vti")["TimeValue"] == 10.0

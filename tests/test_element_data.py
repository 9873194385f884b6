"""The $ElementData reader (mhdarcy.read_element_data, the library's mh_gmsh_element_data) against the rules of the reference's
GmshMeshReader::read_element_data (src/mesh/msh_gmshreader.cc:251-396), on a file written here:
sections taken in file order up to the requested time, ids matched in ascending order, rows of
unknown elements skipped, elements without a row keeping an earlier section's value, the
requested number of components read per row."""
import numpy as np
import pytest

import mhdarcy

FILE = """$MeshFormat
2.2 0 8
$EndMeshFormat
$ElementData
1
"conductivity"
1
0.0
3
0
1
4
1 1.0
3\t 3.0
4 4.0
9 9.0
$EndElementData
$ElementData
1
"other"
0
3
0
1
2
1 -1
2 -2
$EndElementData
$ElementData
1
"conductivity"
1
1.0
3
1
1
3
0 -7.0
2 20.0
4 40.0
$EndElementData
$ElementData
1
"conductivity"
1
2.0
3
2
1
1
1 100.0
$EndElementData
$ElementData
1
"anisotropy"
1
0.0
3
0
3
2
2 1.5 2.5 3.5
3 4.5 5.5 6.5
$EndElementData
"""

IDS = [1, 2, 3, 4]


@pytest.fixture
def path(tmp_path):
    p = tmp_path / "fields.msh"
    p.write_text(FILE)
    return p


def test_time_selection(path):
    nan = np.nan
    at = lambda t: mhdarcy.read_element_data(path, "conductivity", IDS, time=t)[:, 0]
    np.testing.assert_array_equal(at(0.0), [1.0, nan, 3.0, 4.0])  # id 9 is not an element
    np.testing.assert_array_equal(at(1.0), [1.0, 20.0, 3.0, 40.0])  # id 0 skipped, 1 and 3 kept
    np.testing.assert_array_equal(at(1.5), at(1.0))
    # a time a rounding step below a section's time still reaches it (the 2 eps margin)
    np.testing.assert_array_equal(at(np.nextafter(1.0, 0.0)), at(1.0))
    np.testing.assert_array_equal(at(10.0), [100.0, 20.0, 3.0, 40.0])


def test_other_fields_and_components(path):
    o = mhdarcy.read_element_data(path, "other", IDS)
    np.testing.assert_array_equal(o[:, 0], [-1.0, -2.0, np.nan, np.nan])  # no real tag: time 0
    a = mhdarcy.read_element_data(path, "anisotropy", IDS, n_components=2)
    assert a.shape == (4, 2)
    np.testing.assert_array_equal(a[1:3], [[1.5, 2.5], [4.5, 5.5]])
    a3 = mhdarcy.read_element_data(path, "anisotropy", IDS, n_components=3)
    np.testing.assert_array_equal(a3[2], [4.5, 5.5, 6.5])


def test_errors(path):
    with pytest.raises(ValueError, match="no \\$ElementData section"):
        mhdarcy.read_element_data(path, "storativity", IDS)
    with pytest.raises(ValueError, match="at or before"):
        mhdarcy.read_element_data(path, "conductivity", IDS, time=-1.0)
    with pytest.raises(ValueError, match="ascending"):
        mhdarcy.read_element_data(path, "conductivity", [2, 1])
    with pytest.raises(ValueError, match="fewer than 4 values"):
        mhdarcy.read_element_data(path, "anisotropy", IDS, n_components=4)

"""MatrixMarket vector loader (gr_host_matrix_load_vector_mm), the mirror of
DistributedTileLayout::loadVectorFromFile (DistributedTileLayout.cpp:185-206)
and loadDoubletVectorFromFile (matrix/host/details/MatrixMarket.cpp:66-102):
a "vector" object in coordinate or array format, or the first column of a
"matrix" object; unlisted entries are 0; the result is in tile order. Host
only, so these run without a GPU."""
import numpy as np
import pytest

import graphene_b200 as gb


@pytest.fixture(scope="module")
def host():
    return gb.generate3DPoissonMatrix(gb.FLOAT32, 5, 4, 3, 4, gb.PART_RCB)


def write(tmp_path, name, text):
    p = tmp_path / name
    p.write_text(text)
    return p


def natural(h, seed=3):
    return np.random.default_rng(seed).uniform(-1, 1, h.numRows)


@pytest.mark.parametrize("t", [gb.FLOAT32, gb.FLOAT64])
def test_vector_coordinate(tmp_path, host, t):
    v = natural(host)
    keep = np.arange(host.numRows) % 3 != 1  # some entries left out: they read as 0
    lines = [f"{i + 1} {float(v[i])!r}" for i in range(host.numRows) if keep[i]][::-1]  # any order
    text = "%%MatrixMarket vector coordinate real general\n% comment\n" + \
        f"{host.numRows} {len(lines)}\n" + "\n".join(lines) + "\n"
    got = host.loadVectorFromFile(t, write(tmp_path, "v.mtx", text))
    dt = np.float32 if t == gb.FLOAT32 else np.float64
    want = np.where(keep, v, 0.0).astype(dt)
    np.testing.assert_array_equal(got, host.decomposeVector(want, t))


def test_vector_array(tmp_path, host):
    v = natural(host, 4)
    text = "%%MatrixMarket vector array real general\n" + f"{host.numRows}\n" + \
        "\n".join(repr(float(x)) for x in v) + "\n"
    got = host.loadVectorFromFile(gb.FLOAT64, write(tmp_path, "v.mtx", text))
    np.testing.assert_array_equal(got, host.decomposeVector(v, gb.FLOAT64))


def test_matrix_coordinate_first_column(tmp_path, host):
    n = host.numRows
    v = natural(host, 5)
    entries = [f"{i + 1} 1 {float(v[i])!r}" for i in range(n)] + [f"{i + 1} 2 7.5" for i in range(0, n, 2)]
    text = "%%MatrixMarket matrix coordinate real general\n" + f"{n} 2 {len(entries)}\n" + \
        "\n".join(entries) + "\n"
    got = host.loadVectorFromFile("float32", write(tmp_path, "m.mtx", text))
    np.testing.assert_array_equal(got, host.decomposeVector(v.astype(np.float32)))


def test_matrix_array_first_column(tmp_path, host):
    n = host.numRows
    v = natural(host, 6)
    col2 = np.full(n, 9.0)
    text = "%%MatrixMarket matrix array real general\n" + f"{n} 2\n" + \
        "\n".join(repr(float(x)) for x in np.concatenate([v, col2])) + "\n"  # column-major
    got = host.loadVectorFromFile(gb.FLOAT64, write(tmp_path, "m.mtx", text))
    np.testing.assert_array_equal(got, host.decomposeVector(v, gb.FLOAT64))


def test_float32_values_rounded_once(tmp_path, host):
    """Decimal strings are parsed straight to float32 (one rounding), as the
    reference's reader templated on float does: a value just above the
    midpoint of two float32 neighbours rounds up, where a detour through
    float64 would land on the midpoint and round to even (down)."""
    from decimal import Decimal, getcontext
    getcontext().prec = 60
    a = np.float32(1.0)  # even mantissa: a tie goes to a
    b = np.nextafter(a, np.float32(2.0))
    mid = (Decimal(float(a)) + Decimal(float(b))) / 2
    s = str(mid + Decimal("1e-40"))
    assert np.float32(float(s)) == a  # the double detour rounds down
    text = "%%MatrixMarket vector coordinate real general\n" + f"{host.numRows} 1\n1 {s}\n"
    got = host.composeVector(host.loadVectorFromFile(gb.FLOAT32, write(tmp_path, "v.mtx", text)))
    assert got[0] == b


@pytest.mark.parametrize("text,code", [
    ("%%MatrixMarket vector coordinate real general\n60 1\n61 1.0\n", gb._lib.GR_EPARSE),  # index out of range
    ("%%MatrixMarket vector coordinate real general\n60 2\n1 1.0\n", gb._lib.GR_EPARSE),   # entries missing
    ("%%MatrixMarket vector coordinate complex general\n60 1\n1 1.0 0.0\n", gb._lib.GR_EPARSE),
    ("%%MatrixMarket vector array real general\n59\n" + "1.0\n" * 59, gb._lib.GR_EINVAL),  # wrong size
    ("not a matrix market file\n", gb._lib.GR_EPARSE),
])
def test_errors(tmp_path, host, text, code):
    with pytest.raises(gb.GrapheneError) as e:
        host.loadVectorFromFile(gb.FLOAT32, write(tmp_path, "bad.mtx", text))
    assert e.value.code == code


def test_missing_file(tmp_path, host):
    with pytest.raises(gb.GrapheneError) as e:
        host.loadVectorFromFile(gb.FLOAT32, tmp_path / "nope.mtx")
    assert e.value.code == gb._lib.GR_EIO

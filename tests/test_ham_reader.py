"""CPU tests of the Wannier Hamiltonian reader (rgf_read_ham_dat,
w90_load_from_file, src/wannierHam.f90:68-130) against the oracle's
restatement, on generated files: commas and blanks as separators, D
exponents, a record continued over two lines, and the axis reordering."""
import numpy as np
import pytest

from oracle import ham_reader as HO


def _write(path, rng, nb=3, xs=(-1, 0, 1), ys=(0, 1)):
    lines = ["4 2\n", "lattice vectors\n", "2.5, 0.0, 0.0\n", "0.3 3.1 0.0\n", "0.0 0.0 12.0\n", "entries\n"]
    rows = []
    for x in xs:
        for y in ys:
            for m in range(1, nb + 1):
                for n in range(1, nb + 1):
                    rows.append((x, y, 0, m, n, rng.normal(), rng.normal()))
    lines.append(f"{len(rows)}\n")
    for k, r in enumerate(rows):
        if k == 3:   # one record continued over two lines
            lines.append(f"{r[0]} {r[1]} {r[2]} {r[3]}\n{r[4]} {r[5]!r} {r[6]!r}\n")
        elif k % 5 == 0:
            lines.append(f"{r[0]}, {r[1]}, {r[2]}, {r[3]}, {r[4]}, {r[5]:.15E}, {r[6]:.15E}\n".replace("E", "D"))
        else:
            lines.append(" ".join(repr(v) if isinstance(v, float) else str(v) for v in r) + "\n")
    path.write_text("".join(lines))


@pytest.mark.parametrize("axis", [None, (2, 1, 3)])
def test_ham_reader_matches_oracle(tmp_path, axis):
    from liteqt_b200 import writers as W
    f = tmp_path / "ham_dat"
    _write(f, np.random.default_rng(0))
    info, Hr = W.read_ham_dat(str(f), axis=axis)
    ref, Hr_ref = HO.read(str(f), axis=axis)
    for k in ("nvb", "spin_deg", "nb", "nx", "ny", "xmin", "xmax", "ymin", "ymax", "n_entries"):
        assert info[k] == ref[k], k
    for k in ("Lx", "Ly", "Lz", "b1", "b2", "cell"):
        assert np.allclose(info[k], ref[k], rtol=1e-14, atol=1e-14), k
    assert np.array_equal(Hr, Hr_ref)


def test_ham_reader_rejects_bad_files(tmp_path):
    from liteqt_b200 import rgf as R, writers as W
    f = tmp_path / "bad"
    f.write_text("4 2\ncomment\n1 0 0\n")
    with pytest.raises(R.RgfError, match="malformed"):
        W.read_ham_dat(str(f))

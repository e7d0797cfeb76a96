"""The reference's backup text files (all_variables_NNNN.dat), read and
written by the library's host code (no GPU): exact round trips, the
list-directed input forms a Fortran writer may produce, and errors.

Layout (22_writer.f95:1134-1150, 03_restart_primitive.f95:51-57): one
record per point, i = -6..imax+6 outer, j = -6..jmax+6 inner, columns
psi phi Bx By Bz Vx Vy Vz Ex Ey Ez q rho p, ghost points included."""
import numpy as np
import pytest

COLS = ["psi", "phi", "Bx", "By", "Bz", "vx", "vy", "vz", "Ex", "Ey", "Ez", "q", "rho", "p"]


def _random_fields(imax, jmax, seed=0):
    from cueva import PRIM_FIELDS
    rng = np.random.default_rng(seed)
    out = {}
    for k, n in enumerate(PRIM_FIELDS):
        a = rng.standard_normal((jmax + 13, imax + 13)) * 10.0 ** rng.integers(-300, 300, (jmax + 13, imax + 13))
        out[n] = a
    return out


def _records(fields, imax, jmax):
    for i in range(-6, imax + 7):
        for j in range(-6, jmax + 7):
            yield [fields[c][j + 6, i + 6] for c in COLS]


def test_round_trip_exact_with_specials(tmp_path):
    from cueva import read_all_variables, write_all_variables
    imax, jmax = 9, 7
    f = _random_fields(imax, jmax)
    f["rho"][0, 0] = np.nan
    f["p"][1, 2] = np.inf
    f["p"][2, 1] = -np.inf
    f["q"][3, 3] = -0.0
    f["psi"][4, 4] = 5e-324          # smallest subnormal
    f["phi"][5, 5] = np.finfo(float).max
    path = tmp_path / "all_variables_0001.dat"
    write_all_variables(path, imax, jmax, f, nthreads=3)
    lines = path.read_text().splitlines()
    assert len(lines) == (imax + 13) * (jmax + 13)
    assert all(len(l.split()) == 14 for l in lines)
    g = read_all_variables(path, imax, jmax, nthreads=4)
    for n in f:
        a, b = f[n], g[n]
        same = (a == b) | (np.isnan(a) & np.isnan(b))
        assert same.all(), n
        assert np.array_equal(np.signbit(a), np.signbit(b)) or n == "rho", n


def test_writer_refuses_existing_file(tmp_path):
    from cueva import CuevaError, read_all_variables, write_all_variables
    imax, jmax = 6, 6
    f = _random_fields(imax, jmax, 1)
    path = tmp_path / "b.dat"
    write_all_variables(path, imax, jmax, f)
    with pytest.raises(CuevaError, match="exists"):
        write_all_variables(path, imax, jmax, f)
    f2 = _random_fields(imax, jmax, 2)
    write_all_variables(path, imax, jmax, f2, overwrite=True)
    g = read_all_variables(path, imax, jmax)
    assert all(np.array_equal(g[n], f2[n]) for n in f2)


def _fortran_style(x):
    """A list-directed real as a Fortran compiler may print it: F form for
    moderate magnitudes, E form otherwise, the exponent letter dropped for
    three-digit exponents (1.0000000000000000-100)."""
    if x == 0.0 or 0.1 <= abs(x) < 1e15:
        return f"{x:.17g}" if "." in f"{x:.17g}" or "e" in f"{x:.17g}" else f"{x:.17g}.0"
    m, e = f"{x:.16E}".split("E")
    ei = int(e)
    if abs(ei) >= 100:
        return f"{m}{ei:+04d}"
    return f"{m}E{ei:+03d}"


def test_reader_accepts_fortran_list_directed_forms(tmp_path):
    """Letter-less exponents, D exponents, repeat counts, commas, records
    wrapped over lines, and trailing text after the 14th value."""
    from cueva import read_all_variables
    imax, jmax = 6, 6
    f = _random_fields(imax, jmax, 3)
    recs = list(_records(f, imax, jmax))
    out = []
    for k, r in enumerate(recs):
        toks = [_fortran_style(x) for x in r]
        if k % 5 == 1:
            toks = [t.replace("E", "D") for t in toks]
        if k % 5 == 2:     # wrapped after 8 values, comma separators
            out.append(", ".join(toks[:8]) + ",")
            out.append(", ".join(toks[8:]))
            continue
        if k % 5 == 3:     # repeat count for two equal values, extra values ignored
            r2 = list(r)
            r2[1] = r2[0]
            toks[0:2] = ["2*" + _fortran_style(r2[0])]
            recs[k] = r2
            out.append("  ".join(toks) + "   99.0 98.0")
            continue
        out.append("   ".join(toks))
    path = tmp_path / "fortran.dat"
    path.write_text("\n".join(out) + "\n")
    g = read_all_variables(path, imax, jmax)
    k = 0
    for i in range(-6, imax + 7):
        for j in range(-6, jmax + 7):
            for c, n in enumerate(COLS):
                assert g[n][j + 6, i + 6] == recs[k][c], (i, j, n)
            k += 1


def test_reader_null_values_and_slash_keep_previous_values(tmp_path):
    from cueva import read_all_variables
    imax, jmax = 6, 6
    base = _random_fields(imax, jmax, 4)
    arrays = {n: a.copy() for n, a in base.items()}
    recs = list(_records(base, imax, jmax))
    lines = []
    for k, r in enumerate(recs):
        toks = [repr(float(x)) for x in r]
        if k == 0:
            lines.append("1.5, , " + ", ".join(toks[2:]))      # phi null
        elif k == 1:
            lines.append(" ".join(toks[:3]) + " /")              # the rest unchanged
        elif k == 2:
            lines.append("3* " + " ".join(toks[3:]))              # three nulls
        else:
            lines.append(" ".join(toks))
    path = tmp_path / "nulls.dat"
    path.write_text("\n".join(lines) + "\n")
    for n in arrays:
        arrays[n][:] = -7.0
    from cueva import read_all_variables as rd
    g = rd(path, imax, jmax, arrays=arrays)
    # record 0 is point (i, j) = (-6, -6)
    assert g["psi"][0, 0] == 1.5 and g["phi"][0, 0] == -7.0 and g["Bx"][0, 0] == recs[0][2]
    assert g["Bx"][1, 0] == recs[1][2] and g["By"][1, 0] == -7.0 and g["p"][1, 0] == -7.0
    assert g["psi"][2, 0] == -7.0 and g["Bx"][2, 0] == -7.0 and g["By"][2, 0] == recs[2][3]


@pytest.mark.parametrize("bad,frag", [("short", "end of file"), ("word", "not a real"), ("star", "repeat")])
def test_reader_errors(tmp_path, bad, frag):
    from cueva import CuevaError, read_all_variables, write_all_variables
    imax, jmax = 6, 6
    f = _random_fields(imax, jmax, 5)
    path = tmp_path / "x.dat"
    write_all_variables(path, imax, jmax, f)
    lines = path.read_text().splitlines()
    if bad == "short":
        lines = lines[:-1]
    elif bad == "word":
        lines[10] = lines[10].replace(lines[10].split()[3], "abc", 1)
    else:
        lines[10] = "0*1.0 " + lines[10]
    path.write_text("\n".join(lines) + "\n")
    with pytest.raises(CuevaError, match=frag):
        read_all_variables(path, imax, jmax)

"""MPS reader (src/mps.cpp semantics) and the PDHG input gate (gpu/pdhg_input.hpp), on CPU through the C ABI.

The 13 gate models are the reference's own CLI test cases (gpu/pdhg_input_tests.py:57-71): 3 continuous LPs
accepted, 10 integer/quadratic models rejected with "status unsupported_model", exit 2, a reason on stderr and
no output file created or modified, on both --device values and both precisions."""
import itertools
import subprocess

import numpy as np
import pytest

import lpgen
import pdhg

INF = float("inf")


def gate_mps(name, bounds=" UP B X 2\n", quadratic="", marker=False, maximize=False):
    sense = "OBJSENSE\n MAX\n" if maximize else ""
    start = " M0 'MARKER' 'INTORG'\n" if marker else ""
    end = " M1 'MARKER' 'INTEND'\n" if marker else ""
    return (f"NAME {name}\n{sense}ROWS\n N OBJ\n G R\nCOLUMNS\n{start} X OBJ 1 R 1\n{end}RHS\n RHS R 0.5\n"
            f"BOUNDS\n{bounds}{quadratic}ENDATA\n")


GATE = [
    ("continuous_lp", gate_mps("LP"), ()),
    ("maximize_lp", gate_mps("MAXLP", maximize=True), ()),
    ("zero_quadratic", gate_mps("ZERO", quadratic="QUADOBJ\n X X 0\n"), ()),
    ("quadobj", gate_mps("QP", quadratic="QUADOBJ\n X X 2\n"), ("quadratic",)),
    ("qmatrix", gate_mps("QM", quadratic="QMATRIX\n X X 2\n"), ("quadratic",)),
    ("qsection", gate_mps("QS", quadratic="QSECTION OBJ\n X X 2\n"), ("quadratic",)),
    ("maximize_qp", gate_mps("MAXQP", quadratic="QUADOBJ\n X X -2\n", maximize=True), ("quadratic",)),
    ("intorg", gate_mps("MILP", marker=True), ("integer",)),
    ("binary_bound", gate_mps("BV", bounds=" BV B X\n"), ("integer",)),
    ("integer_lower", gate_mps("LI", bounds=" LI B X 0\n UP B X 2\n"), ("integer",)),
    ("integer_upper", gate_mps("UI", bounds=" UI B X 2\n"), ("integer",)),
    ("fixed_integer", gate_mps("FIX", bounds=" FX B X 1\n", marker=True), ("integer",)),
    ("miqp", gate_mps("MIQP", marker=True, quadratic="QUADOBJ\n X X 2\n"), ("quadratic", "integer")),
]


def write(tmp_path, text, name="m.mps"):
    p = tmp_path / name
    p.write_text(text)
    return p


@pytest.mark.parametrize("name,text,expected", GATE, ids=[g[0] for g in GATE])
def test_gate_via_reader(engine_lib, tmp_path, name, text, expected):
    m = pdhg.read_mps(write(tmp_path, text))
    err = pdhg.input_error(m)
    if expected:
        assert err is not None and "continuous LPs only" in err and all(s in err for s in expected)
    else:
        assert err is None


@pytest.mark.parametrize("name,text,expected", [g for g in GATE if g[2]], ids=[g[0] for g in GATE if g[2]])
def test_gate_via_cli(engine_lib, tmp_path, name, text, expected):
    path = write(tmp_path, text)
    outs = [tmp_path / "a.json", tmp_path / "a.sol", tmp_path / "a.dual"]
    for device, fp32, existing in itertools.product(("gpu", "cpu"), (False, True), (False, True)):
        for o in outs:
            if existing:
                o.write_text("sentinel\n")
            elif o.exists():
                o.unlink()
        cmd = [str(pdhg.CLI_PATH), str(path), "--device", device, "--json", str(outs[0]), "--sol", str(outs[1]),
               "--dual", str(outs[2])] + (["--fp32"] if fp32 else [])
        r = subprocess.run(cmd, capture_output=True, text=True, timeout=60)
        assert r.returncode == 2, r
        assert r.stdout.strip() == "status unsupported_model"
        assert "continuous LPs only" in r.stderr and all(s in r.stderr for s in expected)
        assert not any((o.read_text() != "sentinel\n") if existing else o.exists() for o in outs)


def test_cli_usage_and_parse_errors(engine_lib, tmp_path):
    r = subprocess.run([str(pdhg.CLI_PATH)], capture_output=True, text=True)
    assert r.returncode == 2 and "usage" in r.stderr
    r = subprocess.run([str(pdhg.CLI_PATH), "x.mps", "--device", "tpu"], capture_output=True, text=True)
    assert r.returncode == 2
    r = subprocess.run([str(pdhg.CLI_PATH), "x.mps", "--tol"], capture_output=True, text=True)
    assert r.returncode == 2 and "--tol" in r.stderr and "usage" not in r.stderr  # a flag without its value
    bad = write(tmp_path, "NAME B\nROWS\n N OBJ\nCOLUMNS\n X OBJ 1\n")
    r = subprocess.run([str(pdhg.CLI_PATH), str(bad)], capture_output=True, text=True)
    assert r.returncode == 1 and r.stdout.startswith("status parse_error: ") and "missing ENDATA" in r.stdout


def test_cli_refuses_cpu_device_for_lp(engine_lib, tmp_path):
    path = write(tmp_path, GATE[0][1])
    r = subprocess.run([str(pdhg.CLI_PATH), str(path), "--device", "cpu"], capture_output=True, text=True)
    assert r.returncode == 2 and "GPU only" in r.stderr


SEMANTICS = """NAME SEM
OBJSENSE
    MAX
ROWS
 N  COST
 N  FREE2
 E  EQ1
 L  LE1
 G  GE1
 E  EQR
 E  EQN
COLUMNS
    X1  COST  1.5  EQ1  2
    X1  LE1   1
    X1  FREE2 7
    X2  COST  -2d0 GE1  3
    X2  EQ1   1    EQ1  -1
    X3  EQR   1    LE1  0.5
    X4  EQN   1
RHS
    RHS  COST  10   EQ1  4
    RHS  LE1   8    GE1  1
    RHS  EQR   2    EQN  3
    OTHER LE1  99
RANGES
    RNG  LE1  3    GE1  -2
    RNG  EQR  -1   EQN  2.5
BOUNDS
 UP BND X1  -1
 MI BND X2
 UP BND X2  1e25
 LO BND X3  -1e30
 FX BND X4  2
 UP OTHER X3  5
ENDATA
"""


def test_reader_semantics(engine_lib, tmp_path):
    m = pdhg.read_mps(write(tmp_path, SEMANTICS))
    assert m.maximize and m.obj_const == -10.0 and m.name == "SEM"
    assert m.col_names == ["X1", "X2", "X3", "X4"] and m.row_names == ["EQ1", "LE1", "GE1", "EQR", "EQN"]
    assert np.array_equal(m.cost, [1.5, -2.0, 0.0, 0.0])
    # X1: EQ1 2, LE1 1 (FREE2 is a second N row: dropped); X2: EQ1 1 - 1 = 0 dropped, GE1 3
    assert list(m.col_ptr) == [0, 2, 3, 5, 6]
    assert list(m.row_idx) == [0, 1, 2, 1, 3, 4]  # X2: EQ1 1 + EQ1 -1 = 0 dropped; X3 rows sorted
    assert np.array_equal(m.val, [2, 1, 3, 0.5, 1, 1])
    assert np.array_equal(m.row_lo, [4, 5, 1, 1, 3]) and np.array_equal(m.row_up, [4, 8, 3, 2, 5.5])
    assert m.col_lo[0] == -INF and m.col_up[0] == -1  # UP < 0 with lower 0 -> lower -inf
    assert m.col_lo[1] == -INF and m.col_up[1] == INF  # MI, and 1e25 is an infinite sentinel
    assert m.col_lo[2] == -INF and m.col_up[2] == INF  # -1e30 sentinel; 'UP OTHER' set ignored
    assert m.col_lo[3] == m.col_up[3] == 2


@pytest.mark.parametrize("text,msg", [
    ("NAME A\nROWS\n N OBJ\n L R\nCOLUMNS\n X OBJ 0x10 R 1\nENDATA\n", "bad number"),
    ("NAME A\nROWS\n N OBJ\n L R\nCOLUMNS\n X OBJ nan R 1\nENDATA\n", "bad number"),
    ("NAME A\nROWS\n N OBJ\n L R\nCOLUMNS\n X OBJ 1e999 R 1\nENDATA\n", "not finite"),
    ("NAME A\nROWS\n N OBJ\n L R\nCOLUMNS\n X OBJ 1 Q 1\nENDATA\n", "unknown row"),
    ("NAME A\nROWS\n N OBJ\n L R\n L R\nCOLUMNS\nENDATA\n", "duplicate row"),
    ("NAME A\nROWS\n N OBJ\n L R\nCOLUMNS\n X R 1\n Y R 1\n X R 2\nENDATA\n", "two separate blocks"),
    ("NAME A\nROWS\n N OBJ\n L R\nCOLUMNS\n X R 1\nBOUNDS\n UP B Z 1\nENDATA\n", "unknown column"),
    ("NAME A\nROWS\n N OBJ\n L R\nCOLUMNS\n X R 1\nBOUNDS\n XX B X 1\nENDATA\n", "unsupported bound type"),
    ("NAME A\nROWS\n N OBJ\n L R\nCOLUMNS\n X R 1\nFOO\nENDATA\n", "unsupported section"),
    ("NAME A\nROWS\n N OBJ\nROWS\nENDATA\n", "appears twice"),
    ("NAME A\nROWS\n L R\nCOLUMNS\n X R 1\nENDATA\n", "no objective row"),
    ("NAME A\nROWS\n N OBJ\n L R\nCOLUMNS\n X R 1\n", "missing ENDATA"),
    ("NAME A\nROWS\n N OBJ\n K R\nENDATA\n", "bad row type"),
    ("NAME A\nOBJSENSE\n UP\nROWS\n N OBJ\nENDATA\n", "bad OBJSENSE"),
])
def test_reader_errors(engine_lib, tmp_path, text, msg):
    with pytest.raises(pdhg.TaralError) as e:
        pdhg.read_mps(write(tmp_path, text))
    assert e.value.code == pdhg.ERR_PARSE and msg in str(e.value)


def test_reader_fixed_format_fallback(engine_lib, tmp_path):
    """Names with spaces only parse in fixed columns (fields at 2-3, 5-12, 15-22, 25-36, 40-47, 50-61)."""
    def line(*f):  # fixed layout: 4 spaces, name(8), 2, name(8), 2, number(12), 3, name(8), 2, number(12)
        return "    " + f"{f[0]:<8}" + "  " + f"{f[1]:<8}" + "  " + f"{f[2]:<12}" + (
            "   " + f"{f[3]:<8}" + "  " + f"{f[4]:<12}" if len(f) > 3 else "") + "\n"
    text = ("NAME          FIX\nROWS\n N  COST\n L  LIM 1\nCOLUMNS\n" + line("MY VAR", "COST", "1.0", "LIM 1", "2.0")
            + "RHS\n" + line("RHS", "LIM 1", "4.0") + "BOUNDS\n UP BND       MY VAR    3.0\nENDATA\n")
    m = pdhg.read_mps(write(tmp_path, text))
    assert m.col_names == ["MY VAR"] and m.row_names == ["LIM 1"]
    assert m.cost[0] == 1.0 and m.val[0] == 2.0 and m.row_up[0] == 4.0 and m.col_up[0] == 3.0


def test_reader_matches_generator_roundtrip(engine_lib, tmp_path):
    for lp in (lpgen.packing(3000, seed=2), lpgen.transport(20, 30, seed=4), lpgen.general(100, 250, seed=9),
               lpgen.general(100, 250, seed=9, maximize=True)):
        m = pdhg.read_mps(write(tmp_path, lp.mps_text()))
        for k in ("col_ptr", "row_idx", "val", "cost", "col_lo", "col_up", "row_lo", "row_up"):
            assert np.array_equal(getattr(m, k), getattr(lp, k)), (lp.name, k)
        assert m.obj_const == lp.obj_const and m.maximize == lp.maximize


def _big_columns_text(lp, crlf=False):
    """lp's MPS text with a COLUMNS section of several MB (parsed by the multi-threaded tokeniser) rewritten to
    exercise every rule there: two entries per line, comments and blank lines, an integer MARKER block, a second N
    row whose entries are dropped, and a duplicate (row, +v) (row, -v) pair that sums to zero and is dropped."""
    head, rest = lp.mps_text().split("COLUMNS\n", 1)
    cols, tail = rest.split("RHS\n", 1)
    head = head.replace(" N OBJ\n", " N OBJ\n N FREE2\n", 1)
    by_col = {}
    for ln in cols.splitlines():
        c, r, v = ln.split()
        by_col.setdefault(c, []).append((r, v))
    out, is_int = [], np.zeros(lp.n, np.uint8)
    for j, (c, ents) in enumerate(by_col.items()):
        if j == 100:
            out.append("    MARKER                 'MARKER'                 'INTORG'")
        if j == 200:
            out.append("    MARKER                 'MARKER'                 'INTEND'")
        if 100 <= j < 200:
            is_int[j] = 1
        if j % 997 == 0:
            out += ["* a comment line", "   "]
        if j % 5 == 1:
            ents = ents + [("FREE2", "3.5")]
        if j % 7 == 3:  # a row outside the column's own rows, +v then -v: the zero sum is dropped
            rows = {r for r, _ in ents}
            extra = next(f"R{i}" for i in range(lp.m) if f"R{i}" not in rows)
            ents = [(extra, "1.25")] + ents + [(extra, "-1.25")]
        for k in range(0, len(ents), 2):
            pair = ents[k:k + 2]
            out.append("    " + c + "".join(f"  {r}  {v}" for r, v in pair))
    text = head + "COLUMNS\n" + "\n".join(out) + "\nRHS\n" + tail
    return (text.replace("\n", "\r\n") if crlf else text), is_int


@pytest.mark.parametrize("crlf", [False, True])
def test_reader_parallel_columns_roundtrip(engine_lib, tmp_path, crlf):
    """A COLUMNS section of several MB is tokenised on several threads and merged in file order: the model read
    equals the generator's arrays exactly, integer markers included."""
    lp = lpgen.general(8000, 24000, seed=5)
    text, is_int = _big_columns_text(lp, crlf)
    assert len(text) > 3 << 20
    m = pdhg.read_mps(write(tmp_path, text))
    for k in ("col_ptr", "row_idx", "val", "cost", "col_lo", "col_up", "row_lo", "row_up"):
        assert np.array_equal(getattr(m, k), getattr(lp, k)), k
    assert m.col_names == [f"X{j}" for j in range(lp.n)]
    assert np.array_equal(m.is_int, is_int)


@pytest.mark.parametrize("edit,msg", [
    ("dup_late", "two separate blocks"),              # a closed column reopened near the end
    ("dup_then_unknown_row", "two separate blocks"),  # the earlier error is the one reported
    ("unknown_row_then_dup", "unknown row"),
    ("bad_number_late", "bad number"),
    ("bad_marker", "bad MARKER line"),
])
def test_reader_parallel_columns_errors(engine_lib, tmp_path, edit, msg):
    """Errors in a multi-MB COLUMNS section are reported as the sequential reader reports them: the first one in
    file order."""
    lp = lpgen.general(8000, 24000, seed=5)
    text, _ = _big_columns_text(lp)
    lines = text.split("\n")
    c0 = lines.index("COLUMNS")
    c1 = lines.index("RHS")
    late, early = c1 - 10, c0 + 50
    if edit == "dup_late":
        lines.insert(late, "    X5  R0  1")
    elif edit == "dup_then_unknown_row":
        lines.insert(late, "    X5  R0  1")
        lines.insert(late + 5, "    " + lines[late + 5].split()[0] + "  NOSUCHROW  1")
    elif edit == "unknown_row_then_dup":
        lines.insert(late, "    X5  R0  1")
        lines.insert(early, "    " + lines[early].split()[0] + "  NOSUCHROW  1")
    elif edit == "bad_number_late":
        lines.insert(late, "    " + lines[late].split()[0] + "  R0  1.2.3")
    elif edit == "bad_marker":
        lines.insert(late, "    MARKER  'MARKER'")
    with pytest.raises(pdhg.TaralError) as e:
        pdhg.read_mps(write(tmp_path, "\n".join(lines)))
    free_msg = str(e.value).split(" (free format)")[0]
    assert e.value.code == pdhg.ERR_PARSE and msg in free_msg, str(e.value)


def _big_bounds_text(n=120_000, extra=""):
    """A model whose BOUNDS section is several MB (tokenised on several threads): every bound type, a second bound
    set (ignored), columns bounded twice, UP < 0 on a zero lower bound. Returns (text, expected lo, up, is_int)."""
    types = ["LO", "UP", "FX", "FR", "MI", "PL", "BV", "LI", "UI"]
    inf = float("inf")
    lo, up, isint = np.zeros(n), np.full(n, inf), np.zeros(n, np.uint8)
    cols = "\n".join(f"    X{j}  R0  1" for j in range(n))
    bl = []

    def add(t, j, v=None, bset="BND"):
        bl.append(f" {t} {bset} X{j}" + ("" if v is None else f" {v}"))
        if bset != "BND":
            return
        if t in ("BV", "LI", "UI"):
            isint[j] = 1
        if t in ("LO", "LI"):
            lo[j] = v
        elif t in ("UP", "UI"):
            up[j] = v
            if v < 0 and lo[j] == 0:
                lo[j] = -inf
        elif t == "FX":
            lo[j] = up[j] = v
        elif t == "FR":
            lo[j], up[j] = -inf, inf
        elif t == "MI":
            lo[j] = -inf
        elif t == "PL":
            up[j] = inf
        elif t == "BV":
            lo[j], up[j] = 0, 1
    for j in range(n):
        t = types[j % 9]
        v = None if t in ("FR", "MI", "PL", "BV") else (-2.5 if j % 18 == 1 else float(j % 97) + 0.5)
        add(t, j, v)
        if j % 7 == 3:
            add("UP", j, 99.0, bset="OTHER")  # a second bound set: ignored
        if j % 11 == 5:
            add("UP", j, float(j % 13) + 100.0)  # bounded twice: applied in file order
    text = ("NAME BIGB\nROWS\n N OBJ\n L R0\nCOLUMNS\n" + cols + "\nRHS\n    RHS R0 1\nBOUNDS\n" + "\n".join(bl)
            + "\n" + extra + "ENDATA\n")
    return text, lo, up, isint


def test_reader_parallel_bounds(engine_lib, tmp_path):
    text, lo, up, isint = _big_bounds_text()
    assert len(text.split("BOUNDS\n")[1]) > 2 << 20
    m = pdhg.read_mps(write(tmp_path, text))
    assert np.array_equal(m.col_lo, lo) and np.array_equal(m.col_up, up) and np.array_equal(m.is_int, isint)


@pytest.mark.parametrize("extra,msg", [
    (" UP BND NOSUCH 1\n", "unknown column 'NOSUCH' in BOUNDS"),
    (" UP OTHER NOSUCH 1\n UP OTHER X1 1.2.3\n", None),  # lines of another bound set are skipped unchecked
    (" UP\n", "bad BOUNDS line"),
    (" XX BND X1 1\n", "unsupported bound type XX"),
    (" UP BND X1 1.2.3\n", "bad number"),
    (" UP BND NOSUCH 1.2.3\n UP\n", "unknown column 'NOSUCH'"),  # the first error in file order
])
def test_reader_parallel_bounds_errors(engine_lib, tmp_path, extra, msg):
    text, lo, up, isint = _big_bounds_text(extra=extra)
    if msg is None:
        m = pdhg.read_mps(write(tmp_path, text))
        assert np.array_equal(m.col_up, up)
        return
    with pytest.raises(pdhg.TaralError) as e:
        pdhg.read_mps(write(tmp_path, text))
    assert e.value.code == pdhg.ERR_PARSE and msg in str(e.value).split(" (free format)")[0], str(e.value)

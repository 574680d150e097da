"""The grammar the GPU tokeniser implements, restated position by position in Python
and checked against the host reader (fscanf) on the edge cases and on mutated files:
every maximal run of digits is one literal, negative when the byte before it is '-';
reading fails at the first byte that is neither white space, a digit nor a sign, at
a sign not followed by a digit, at a literal beyond +-(2^31 - 1), or at the end of
the body; the file is read when the M-th zero comes before the first failure.  The
device reader is compared with the host reader on the same inputs in
test_gpu_ingest.py; this test pins the rule it implements on the CPU.
"""
import numpy as np

from cnf_cases import CASES, formatted_cnf

WS = set(b" \t\n\v\f\r")
DIG = set(b"0123456789")


def tokenise(body: bytes, m: int):
    """(literals, lengths) or the failure message, by the position-wise rule."""
    L = len(body)
    fail, fail_range = None, False
    tokens = []  # (position, value, zero)
    for q in range(L):
        c = body[q]
        if c in DIG:
            if q > 0 and body[q - 1] in DIG:
                continue
            r = q
            while r < L and body[r] in DIG:
                r += 1
            digits = body[q:r].lstrip(b"0") or b"0"
            v = int(digits) if len(digits) <= 11 else 1 << 40  # anything past 11 digits is out of range
            if v > 2147483647:
                if fail is None or q < fail:
                    fail, fail_range = q, True
            neg = q > 0 and body[q - 1] == ord("-")
            tokens.append((q, -v if neg else v, v == 0))
        elif c in b"+-":
            if q + 1 >= L or body[q + 1] not in DIG:
                if fail is None or q < fail:
                    fail, fail_range = q, False
        elif c not in WS:
            if fail is None or q < fail:
                fail, fail_range = q, False
    lits, lens, cur, zeros = [], [], 0, 0
    for q, v, zero in tokens:
        if fail is not None and q >= fail:
            break
        if zero:
            lens.append(cur)
            cur = 0
            zeros += 1
            if zeros == m:
                return lits, lens
        else:
            lits.append(v)
            cur += 1
    return "literal out of range" if (fail is not None and fail_range) else "expected more literals in file"


def parse_file(data: bytes):
    """The host reader's header scan (lines skipped until "p cnf N M"), then the body
    by `tokenise`, kept as SatProblem::AddClauses keeps it (empty clauses dropped)."""
    i, n, m, body = 0, -1, -1, None
    while i < len(data):
        if data[i] == ord("p"):
            j = i + 1
            while j < len(data) and data[j] in WS:
                j += 1
            if data[j:j + 3] != b"cnf":
                return "expected: p cnf <variables> <clauses>"
            j += 3
            vals = []
            for _ in range(2):
                while j < len(data) and data[j] in WS:
                    j += 1
                k = j + (1 if j < len(data) and data[j] in b"+-" else 0)
                e = k
                while e < len(data) and data[e] in DIG:
                    e += 1
                if e == k:
                    return "expected: p cnf <variables> <clauses>"
                vals.append(int(data[j:e]))
                j = e
            n, m = vals
            body = data[j:]
            break
        if data[i] != ord("\n"):  # the rest of the line is skipped (lines here are short)
            nl = data.find(b"\n", i)
            i = len(data) if nl < 0 else nl + 1
        else:
            i += 1
    if body is None or n < 0 or m < 0:
        return "could not find a SAT declaration"
    if n == 0 or m == 0:
        return [], []
    r = tokenise(body, m)
    if isinstance(r, str):
        return r
    lits, lens = r
    return lits, [l for l in lens if l > 0]


def host(path):
    from analogsat_b200 import SatProblem, AnalogSatError
    try:
        p = SatProblem.read_cnf(path)
    except AnalogSatError as e:
        return str(e)
    lits, lens = p.GetAllClauses()
    return list(lits), list(lens)


def _check(tmp_path, data, name):
    f = tmp_path / name
    f.write_bytes(data)
    want = host(str(f))
    got = parse_file(data)
    if isinstance(want, str) or isinstance(got, str):
        assert isinstance(got, str) and isinstance(want, str) and want.endswith(got), (name, got, want)
    else:
        assert list(got[0]) == want[0] and list(got[1]) == want[1], name


def test_rule_matches_host_reader_on_edge_cases(tmp_path):
    for name, data, expected, _ in CASES:
        if name in ("long_comment_line",):  # the header scan above does not model fgets' 1023-byte lines
            continue
        _check(tmp_path, data, name + ".cnf")


def test_rule_matches_host_reader_on_mutations(tmp_path):
    from analogsat_b200.instances import make_instance
    lits, lens, _ = make_instance("random", 60, 250, 3, seed=12)
    base = formatted_cnf(lits, lens, seed=4)
    body0 = base.index(b"\n", base.index(b"p cnf")) + 1
    alphabet = b"0123456789-+ \n\t\rx\x00"
    rng = np.random.default_rng(21)
    for i in range(400):
        data = bytearray(base)
        for _ in range(int(rng.integers(1, 4))):
            pos = int(rng.integers(body0, len(data)))
            op = rng.integers(3)
            ch = alphabet[int(rng.integers(len(alphabet)))]
            if op == 0:
                data[pos] = ch
            elif op == 1:
                data.insert(pos, ch)
            else:
                del data[pos:pos + int(rng.integers(1, 6))]
        if i % 40 == 39:
            data = data[: int(rng.integers(body0, len(data)))]
        _check(tmp_path, bytes(data), f"m{i}.cnf")


def test_rule_matches_host_reader_on_the_device_test_mutations(tmp_path):
    """The 300 mutated files of test_gpu_ingest.py's device-reader test (same
    generator and seed), so that the device reader, the host reader and the rule are
    compared on one set."""
    from analogsat_b200.instances import make_instance
    lits, lens, _ = make_instance("random", 800, 3000, 3, seed=6)
    base = formatted_cnf(lits, lens, seed=2)
    start = base.index(b"\n", base.index(b"p cnf"))
    body0 = start + 1
    alphabet = b"0123456789-+ \n\t\r\x0bx%c\x00"
    rng = np.random.default_rng(11)
    for i in range(300):
        data = bytearray(base)
        for _ in range(int(rng.integers(1, 4))):
            if i % 3 == 0:
                pos = start + 4096 * int(rng.integers(1, (len(data) - start) // 4096 + 1)) + int(rng.integers(-2, 2))
            else:
                pos = int(rng.integers(body0, len(data)))
            pos = min(max(pos, body0), len(data) - 1)
            op = rng.integers(3)
            ch = alphabet[int(rng.integers(len(alphabet)))]
            if op == 0:
                data[pos] = ch
            elif op == 1:
                data.insert(pos, ch)
            else:
                del data[pos:pos + int(rng.integers(1, 6))]
        if i % 50 == 49:
            data = data[: int(rng.integers(body0, len(data)))]
        _check(tmp_path, bytes(data), f"d{i}.cnf")

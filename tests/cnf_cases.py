"""DIMACS inputs for the CNF readers: (name, bytes, expected, reference_agrees).

expected is "ok" or the reader's message on failure.  reference_agrees is False where
the reference's CnfReader (AnalogSAT/io/CnfReader.cpp:48-141) deliberately differs:
a literal beyond +-(2^31 - 1), which its "%d" leaves undefined (glibc truncates it),
and a blank line in the preamble, after which the reference skips the next line too.
"""
from __future__ import annotations

import numpy as np

MORE = "expected more literals in file"
RANGE = "literal out of range"

CASES = [
    ("basic", b"p cnf 3 2\n1 -2 0\n2 3 0\n", "ok", True),
    ("comments", b"c hello\nc another line\np cnf 3 2\n1 -2 0\n2 3 0\n", "ok", True),
    ("several_clauses_per_line", b"p cnf 4 3\n1 -2 0 2 3 0 -4 1 0\n", "ok", True),
    ("clause_across_lines", b"p cnf 4 2\n1\n-2\n3 0\n4\n0\n", "ok", True),
    ("tabs_and_crlf", b"p cnf 3 2\r\n1\t-2 0\r\n\t2  3 0\r\n", "ok", True),
    ("vertical_tab_form_feed", b"p cnf 3 1\n1\x0b2\x0c0\n", "ok", True),
    ("plus_sign_leading_zeros", b"p cnf 3 2\n+1 -002 0\n0003 2 00\n", "ok", True),
    ("minus_zero_ends_clause", b"p cnf 3 2\n1 2 -0\n3 0\n", "ok", True),
    ("adjacent_signed_literals", b"p cnf 3 2\n1-2 0\n3+1 0\n", "ok", True),
    ("satlib_percent_trailer", b"p cnf 3 2\n1 -2 0\n2 3 0\n%\n0\n\n", "ok", True),
    ("junk_after_last_clause", b"p cnf 3 1\n1 2 0 garbage\n", "ok", True),
    ("empty_clause_dropped", b"p cnf 3 3\n1 2 0\n0\n3 0\n", "ok", True),
    ("header_n_ignored", b"p cnf 10 1\n1 2 0\n", "ok", True),
    ("no_final_newline", b"p cnf 3 1\n1 2 0", "ok", True),
    ("range_after_last_clause", b"p cnf 3 1\n1 0 99999999999\n", "ok", True),
    ("largest_literal", b"p cnf 3 1\n2147483647 -2147483647 0\n", "ok", True),
    ("long_comment_line", b"c " + b"x" * 3000 + b"\np cnf 3 1\n1 0\n", "ok", True),
    ("digits_across_tiles", b"p cnf 5 2\n" + b"0" * 5000 + b"5 -3 0\n1 0\n", "ok", True),
    ("empty_problem", b"p cnf 0 0\n", "ok", True),
    ("missing_clauses", b"p cnf 3 3\n1 -2 0\n2 3 0\n", MORE, True),
    ("junk_inside", b"p cnf 3 2\n1 x 0\n2 0\n", MORE, True),
    ("comment_inside_body", b"p cnf 3 2\n1 2 0\nc late comment\n3 0\n", MORE, True),
    ("lonely_sign", b"p cnf 3 2\n1 - 2 0\n3 0\n", MORE, True),
    ("double_sign", b"p cnf 3 1\n--1 0\n", MORE, True),
    ("sign_at_end_of_file", b"p cnf 3 1\n1 2 -", MORE, True),
    ("nul_byte", b"p cnf 3 1\n1 \x00 2 0\n", MORE, True),
    ("empty_body", b"p cnf 3 1\n", MORE, True),
    ("far_too_many_clauses", b"p cnf 3 100000\n1 0\n", MORE, True),
    ("no_declaration", b"c nothing\n1 2 0\n", "could not find a SAT declaration", True),
    ("bad_declaration", b"p dnf 3 1\n1 0\n", "expected: p cnf <variables> <clauses>", True),
    ("literal_out_of_range", b"p cnf 3 1\n1 2147483648 0\n", RANGE, False),
    ("range_before_junk", b"p cnf 3 2\n1 -99999999999999999999999 x 0\n", RANGE, False),
    ("blank_line_in_preamble", b"c a\n\np cnf 3 1\n1 0\n", "ok", False),
]


def formatted_cnf(lits, lens, seed: int) -> bytes:
    """A DIMACS body with varied formatting (white-space runs of spaces, tabs, CR LF
    and line breaks, several clauses per line, '+' signs and leading zeros) for the
    clauses (lits, lens): readers must return exactly these clauses."""
    rng = np.random.default_rng(seed)
    ws = [b" ", b"  ", b"\t", b"\n", b"\r\n", b" \n "]
    out = [b"c formatted\n", b"p cnf %d %d\n" % (int(np.abs(lits).max()), len(lens))]
    o = 0
    for ln in lens:
        for v in lits[o:o + ln]:
            v = int(v)
            r = rng.random()
            if v > 0 and r < 0.1:
                tok = b"+%d" % v
            elif r < 0.2:
                tok = (b"-" if v < 0 else b"") + b"0" * int(rng.integers(1, 4)) + b"%d" % abs(v)
            else:
                tok = b"%d" % v
            out.append(tok + ws[int(rng.integers(len(ws)))])
        o += ln
        out.append(b"0" + ws[int(rng.integers(len(ws)))])
    return b"".join(out)

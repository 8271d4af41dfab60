"""Every file:line citation of hom3 in this repository names lines that exist.

Docstrings and comments cite the hom3 code they restate as `path:a-b`
(paths relative to hom3's src/ or to a subdirectory of it, e.g.
`euler/physics.hpp:276-293`), sometimes followed by bare continuations
(`:297-310`) that refer to the last file named.  This test finds them all
and checks each range against the line counts of hom3's sources recorded in
tests/golden/reference_files.json (written by tests/golden/make_golden.py
from a hom3 checkout): the cited file must be identified unambiguously and
1 <= a <= b <= its length.  A range that points past the end of its file
cannot name the code it claims to restate.
"""
import json
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
FIXTURE = os.path.join(ROOT, "tests", "golden", "reference_files.json")

# what is scanned: the product, the oracle, the tests and the documents this
# repository writes (not the survey, review or driver records)
SCAN_DIRS = ("hom3_b200", "include", "oracle", "tests")
SCAN_FILES = ("bench.py", "__graft_entry__.py", "DESIGN.md", "INTEGRATION.md", "README.md", "BASELINE.md")
SCAN_EXT = (".py", ".cu", ".cuh", ".cpp", ".hpp", ".h", ".md", ".txt")

_PATH = r"([A-Za-z0-9_./-]+\.(?:hpp|cpp|h)|CMakeLists\.txt)"
_RANGE = r"\d+(?:\s*[-–]\s*\d+)?"
CITE = re.compile(_PATH + r"((?::\s*|\s+)" + _RANGE + r"(?:\s*,\s*" + _RANGE + r")*)")
BARE = re.compile(r"(?:(?<=\()|(?<=\s)|(?<=^)):(" + _RANGE + r"(?:\s*,\s*" + _RANGE + r")*)")
ONE = re.compile(r"(\d+)(?:\s*[-–]\s*(\d+))?")
# a bare continuation refers to a file named at most this many lines above
CONT_LINES = 12


def reference_files():
    with open(FIXTURE) as f:
        return json.load(f)["files"]


def scanned_files():
    out = [os.path.join(ROOT, f) for f in SCAN_FILES if os.path.exists(os.path.join(ROOT, f))]
    for d in SCAN_DIRS:
        for dp, dn, fn in os.walk(os.path.join(ROOT, d)):
            dn[:] = [x for x in dn if not x.startswith((".", "_")) and x != "__pycache__"]
            out += [os.path.join(dp, f) for f in fn if f.endswith(SCAN_EXT)]
    return sorted(out)


def resolve(path, files):
    """hom3 files a cited path names: itself when it is a full path from the
    checkout's root, else every file it is a suffix of."""
    if path in files:
        return [path]
    return [p for p in files if p.endswith("/" + path)]


def citations(text, files):
    """(line number, cited text, candidate files, first, last) of every
    citation in `text` whose path names a hom3 source file."""
    found = []
    last, last_ln = None, -10 ** 9
    for ln, line in enumerate(text.splitlines(), 1):
        events = []
        for m in CITE.finditer(line):
            events.append((m.start(), "cite", m))
        for m in BARE.finditer(line):
            events.append((m.start(), "bare", m))
        for _, kind, m in sorted(events, key=lambda e: e[0]):
            if kind == "cite":
                cands = resolve(m.group(1), files)
                if not cands:
                    continue
                last, last_ln = (m.group(1), cands), ln
                for r in ONE.finditer(m.group(2)):
                    a, b = int(r.group(1)), int(r.group(2) or r.group(1))
                    found.append((ln, m.group(0), cands, a, b))
            elif last is not None and ln - last_ln <= CONT_LINES:
                for r in ONE.finditer(m.group(1)):
                    a, b = int(r.group(1)), int(r.group(2) or r.group(1))
                    found.append((ln, f"{last[0]} {m.group(0)}", last[1], a, b))
    return found


def test_fixture_lists_hom3_sources():
    files = reference_files()
    assert "src/solver/fv/solver.hpp" in files and files["src/solver/fv/solver.hpp"] > 900
    assert "src/solver/fv/euler/physics.hpp" in files


def test_citations_name_existing_lines():
    files = reference_files()
    bad, ambiguous, n = [], [], 0
    for path in scanned_files():
        if os.path.abspath(path) == os.path.abspath(__file__):
            continue
        with open(path, errors="replace") as f:
            text = f.read()
        rel = os.path.relpath(path, ROOT)
        for ln, what, cands, a, b in citations(text, files):
            n += 1
            if len(cands) > 1:
                ambiguous.append(f"{rel}:{ln}: {what!r} matches {cands}")
                continue
            if not (1 <= a <= b <= files[cands[0]]):
                bad.append(f"{rel}:{ln}: {what!r} -> {cands[0]} has {files[cands[0]]} lines")
    assert n > 300, f"only {n} citations found: the scanner no longer recognises them"
    assert not ambiguous, "citations naming more than one hom3 file:\n" + "\n".join(ambiguous)
    assert not bad, "citations past the end of the cited file:\n" + "\n".join(bad)


def test_scanner_catches_a_bad_range():
    files = {"src/solver/fv/coupling.hpp": 84, "src/solver/fv/euler/physics.hpp": 330}
    text = "// coupling::apply: coupling.hpp:167-183\n// AUSM (euler/physics.hpp:276-293, theta_ :315-325)\n"
    got = [(c[3], c[4], c[2][0]) for c in citations(text, files)]
    assert (167, 183, "src/solver/fv/coupling.hpp") in got
    assert (315, 325, "src/solver/fv/euler/physics.hpp") in got
    assert any(b > files[p] for a, b, p in got)

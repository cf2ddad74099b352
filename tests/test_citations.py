"""Every reference citation in the repository's sources points inside the file it names.

Citations have the form `dir/File.jl:N` or `dir/File.jl:N-M` (dir one of the reference's src,
test, ext, gpu, docs, benchmark, examples). With the reference tree present (PFSHT_REFERENCE, by
default the checkout beside this build), each cited line must exist in that file; without it the
test is skipped."""
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.environ.get("PFSHT_REFERENCE", "/root/reference")

CITE = re.compile(r"\b((?:src|test|ext|gpu|docs|benchmark|examples)/[A-Za-z0-9_./-]+?\.(?:jl|md|toml))"
                  r":(\d+)(?:-(\d+))?")
SCAN_DIRS = ("oracle", "partialfsht.jl_b200", "include", "tests")
SCAN_FILES = ("DESIGN.md", "INTEGRATION.md", "bench.py", "__graft_entry__.py", "README.md")
EXTS = (".c", ".h", ".cu", ".cuh", ".cpp", ".hpp", ".py", ".md")


def _sources():
    for d in SCAN_DIRS:
        for base, dirs, files in os.walk(os.path.join(ROOT, d)):
            dirs[:] = [x for x in dirs if not x.startswith(("_build", "__pycache__", "golden"))]
            for f in files:
                if f.endswith(EXTS):
                    yield os.path.join(base, f)
    for f in SCAN_FILES:
        p = os.path.join(ROOT, f)
        if os.path.exists(p):
            yield p


def citations():
    out = []
    for path in _sources():
        with open(path, encoding="utf-8", errors="replace") as fh:
            for ln, line in enumerate(fh, 1):
                for m in CITE.finditer(line):
                    hi = int(m.group(3)) if m.group(3) else int(m.group(2))
                    out.append((os.path.relpath(path, ROOT), ln, m.group(1), int(m.group(2)), hi))
    return out


def test_citation_pattern_finds_citations():
    # runs without the reference tree: the scan itself works
    cs = citations()
    assert len(cs) > 100
    assert any(c[2] == "src/Legendre.jl" for c in cs)


@pytest.mark.skipif(not os.path.isdir(os.path.join(REF, "src")), reason="reference tree absent")
def test_every_citation_is_inside_its_file():
    lengths = {}
    bad = []
    for where, ln, f, lo, hi in citations():
        p = os.path.join(REF, f)
        if f not in lengths:
            lengths[f] = sum(1 for _ in open(p, encoding="utf-8", errors="replace")) if os.path.exists(p) else -1
        n = lengths[f]
        if n < 0 or lo < 1 or hi < lo or hi > n:
            bad.append(f"{where}:{ln}: {f}:{lo}-{hi} (file has {n} lines)")
    assert not bad, "\n".join(bad)

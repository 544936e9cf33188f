"""Audit of the reference citations in the sources (host only).

The reference cannot be compiled here, so the oracle's parity with it rests on a
line-by-line reading of the Fortran against the restatement; the file:line
pointers in the sources are what make that reading possible.  This test checks
every ``<file>.F90:a-b`` pointer in the oracle, the C header, the Fortran
interface module, the CUDA sources and the Python package against the reference
tree named by the ``LBM_REFERENCE`` environment variable (the project root that
holds ``src/``); it is skipped when the variable is unset.

* every cited file exists and every cited line or range lies inside it;
* every per-call entry point of ``include/lbm_b200.h`` whose comment names a
  reference subroutine (``name(args)  m_file.F90:N``) points at the line that
  opens ``subroutine name`` (and its ``kernel m_file_kernel.F90:N`` at the kernel's);
* every cited range holds at least one line of code (not only blanks and comments).
"""
import os
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
REF = os.environ.get("LBM_REFERENCE")
pytestmark = pytest.mark.skipif(not REF, reason="LBM_REFERENCE (the reference project root) is not set")

SOURCES = ["oracle", "include", "lbm_b200", "tests/golden", "bench.py", "__graft_entry__.py"]
EXTS = {".py", ".cpp", ".h", ".cu", ".cuh", ".F90"}
CITE = re.compile(r"\b([A-Za-z][A-Za-z0-9_]*\.F90)((?::\d+(?:-\d+)?)(?:,\d+(?:-\d+)?)*)")


def ref_files():
    out = {}
    for p in Path(REF).rglob("*.F90"):
        out.setdefault(p.name, p)
    return out


def source_files():
    for s in SOURCES:
        p = ROOT / s
        if p.is_file():
            yield p
        elif p.is_dir():
            for q in sorted(p.rglob("*")):
                if q.suffix in EXTS and "_build" not in q.parts:
                    yield q


def citations():
    for src in source_files():
        for ln, line in enumerate(src.read_text(errors="replace").splitlines(), 1):
            for m in CITE.finditer(line):
                for part in m.group(2).lstrip(":").split(","):
                    a, _, b = part.partition("-")
                    yield src, ln, m.group(1), int(a), int(b) if b else int(a), line


def is_code(line):
    s = line.strip()
    return bool(s) and not s.startswith("!")


def test_every_citation_lies_inside_its_file():
    files = ref_files()
    bad, n = [], 0
    for src, ln, name, a, b, _ in citations():
        if name == os.path.basename(str(src)):
            continue                     # the Fortran interface module naming itself
        n += 1
        if name not in files:
            bad.append("%s:%d: %s does not exist in the reference" % (src.relative_to(ROOT), ln, name))
            continue
        lines = files[name].read_text(errors="replace").splitlines()
        if not (1 <= a <= b <= len(lines)):
            bad.append("%s:%d: %s:%d-%d outside its %d lines" % (src.relative_to(ROOT), ln, name, a, b, len(lines)))
        elif not any(is_code(x) for x in lines[a - 1:b]):
            bad.append("%s:%d: %s:%d-%d holds no code" % (src.relative_to(ROOT), ln, name, a, b))
    assert n > 100, "expected the sources to cite the reference throughout (found %d)" % n
    assert not bad, "\n".join(bad)


HEADER_ENTRY = re.compile(r"/\*\s*(?:call\s+)?([a-z_0-9]+)\(.*?\b(m_[a-z_0-9]+\.F90):(\d+)(?:.*?kernel\s+(m_[a-z_0-9]+\.F90):(\d+))?")


def test_header_entry_points_point_at_their_subroutines():
    files = ref_files()
    bad, n = [], 0
    for ln, line in enumerate((ROOT / "include" / "lbm_b200.h").read_text().splitlines(), 1):
        m = HEADER_ENTRY.search(line)
        if not m:
            continue
        name = m.group(1)
        for fname, at, routine in ((m.group(2), m.group(3), name), (m.group(4), m.group(5), name + "_kernel")):
            if not fname:
                continue
            n += 1
            text = files[fname].read_text(errors="replace").splitlines()
            first = text[int(at) - 1].lower()
            if not re.search(r"\bsubroutine\s+%s\b" % re.escape(routine), first):
                bad.append("lbm_b200.h:%d: %s:%s is %r, not 'subroutine %s'" % (ln, fname, at, first.strip(), routine))
    assert n >= 12, n
    assert not bad, "\n".join(bad)

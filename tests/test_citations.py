"""Every reference citation in this tree's sources (file:line or file:first-last) names a file of
the reference and lines it has: full paths directly, bare file names by their unique name in the reference
tree. Skipped where the reference sources are absent."""
import collections
import os
import re
import subprocess

import pytest

from conftest import ROOT

SOURCES = ("qed_spin_b200", "include", "oracle", "tests", "bench.py", "__graft_entry__.py")
FULL = re.compile(r"\b((?:include|src|python|tests|docs|cmake)/[\w/.\-]+\.(?:h|hpp|cpp|cu|cuh|py)):(\d+)(?:-(\d+))?")
BARE = re.compile(r"(?<![\w/])([\w\-]+\.(?:h|hpp|cpp|cu|cuh|py)):(\d+)(?:-(\d+))?")


def _reference_root():
    r = subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "print-ref"], capture_output=True,
                       text=True)
    ref = r.stdout.strip()
    if r.returncode != 0 or not os.path.isdir(os.path.join(ref, "include", "ed")):
        pytest.skip("the reference sources are not in this tree's environment")
    return ref


def _files():
    for root in SOURCES:
        p = os.path.join(ROOT, root)
        if os.path.isfile(p):
            yield p
            continue
        for d, _, fs in os.walk(p):
            if "_ref" in d or "__pycache__" in d:
                continue
            for f in fs:
                if f.endswith((".cu", ".cuh", ".h", ".hpp", ".cpp", ".py")):
                    yield os.path.join(d, f)


def test_reference_citations_resolve():
    ref = _reference_root()
    by_name = collections.defaultdict(list)
    for d, _, fs in os.walk(ref):
        if "/.git" not in d:
            for f in fs:
                by_name[f].append(os.path.join(d, f))
    n_lines = {}

    def length(path):
        if path not in n_lines:
            with open(path, errors="ignore") as fh:
                n_lines[path] = sum(1 for _ in fh)
        return n_lines[path]

    bad, checked = [], 0
    for path in _files():
        for ln, line in enumerate(open(path, errors="ignore"), 1):
            for m in FULL.finditer(line):
                f, a, b = m.group(1), int(m.group(2)), int(m.group(3) or m.group(2))
                full = os.path.join(ref, f)
                checked += 1
                if not os.path.exists(full) or a > b or b > length(full):
                    bad.append(f"{os.path.relpath(path, ROOT)}:{ln}: {m.group(0)}")
            for m in BARE.finditer(line):
                f, a, b = m.group(1), int(m.group(2)), int(m.group(3) or m.group(2))
                cands = by_name.get(f, [])
                if not cands:
                    continue   # a file of this tree, or no reference file
                checked += 1
                if all(a > b or b > length(c) for c in cands):
                    bad.append(f"{os.path.relpath(path, ROOT)}:{ln}: {m.group(0)}")
    assert checked > 100
    assert not bad, "\n".join(bad)

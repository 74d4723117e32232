"""Two standing rules of the sources, checked without a GPU: every entry
point of the C ABI says which reference interface it replaces (a file:line
citation of rpba.cpp, rbacore.cpp, rpbacore.cpp or rpba.h in its comment)
or that the reference has no counterpart; and the CUDA sources name none of
the batched-copy calls that are not used on this hardware."""
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_every_entry_point_cites_the_reference():
    txt = open(os.path.join(ROOT, "include", "rpba_b200.h")).read()
    decl = re.compile(r"(/\*(?:(?!\*/).)*\*/\s*)((?:int32_t|void|const char|double|float)\s*\*?\s*(rpba_[a-z_0-9]+)\s*\()",
                      re.S)
    found = {}
    for m in decl.finditer(txt):
        com = m.group(1)
        found[m.group(3)] = bool(re.search(r"(rpba|rbacore|rpbacore)\.(cpp|h):\d+", com)) or \
            "counterpart" in com.lower()
    names = set(re.findall(r"\b(rpba_[a-z_0-9]+)\s*\(", txt))
    missing = sorted(n for n in names if not found.get(n, False))
    assert not missing, missing


def test_no_batched_copy_calls_in_device_sources():
    bad = re.compile("cu(da)?" + "Memcpy" + "(3D)?" + "Batch" + "Async")  # assembled: the names stay unwritten
    for d in ("rpba_b200/csrc", "include"):
        for f in os.listdir(os.path.join(ROOT, d)):
            if f.endswith((".cu", ".cuh", ".h", ".cpp")):
                assert not bad.search(open(os.path.join(ROOT, d, f)).read()), f

"""The C-ABI library loads without a GPU and exports every entry point include/*.h declares."""

import re

from conftest import ROOT


def _declared():
    names = set()
    for header in (ROOT / "include").glob("*.h"):
        text = header.read_text()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"\b(spx_[a-z0-9_]+)\s*\(", text):
            names.add(m.group(1))
    return names


def test_header_declares_entry_points():
    names = _declared()
    assert {"spx_otsu", "spx_ccl_label", "spx_ccl_finish", "spx_refine_centers", "spx_voronoi_labels"} <= names


def test_library_exports_every_declared_symbol():
    from imageprocessor_new_b200 import build
    from imageprocessor_new_b200._lib import SIGNATURES, load_library

    build.build()
    lib = load_library()
    declared = _declared()
    missing = [n for n in declared if not hasattr(lib, n)]
    assert not missing, missing
    # The Python binding declares exactly what the header declares.
    assert set(SIGNATURES) == declared


def test_build_targets_sm100a_only():
    from imageprocessor_new_b200 import build

    assert build.ARCH == ["-gencode", "arch=compute_100a,code=sm_100a"]

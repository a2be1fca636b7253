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


def test_fit_options_are_checked_before_any_device_work():
    """An unknown LM arithmetic or a cost tolerance outside (0, 1) is an argument error, reported
    before the entry point touches the device (so it runs without a GPU)."""
    import pytest

    from imageprocessor_new_b200 import _lib, deblend

    with pytest.raises(ValueError, match="fit_precision"):
        deblend.fit_options("fp16")
    assert deblend.fit_options("fp64").cost_tol == 1e-12
    assert deblend.fit_options("fp32").precision == _lib.FIT_F32
    lib = _lib.load_library()
    bg = _lib.BgMap()
    for opts in (_lib.FitOptions(7, 1e-6), _lib.FitOptions(_lib.FIT_F32, 0.0), _lib.FitOptions(_lib.FIT_F64, 1.5)):
        rc = lib.spx_deblend_iteration(None, 1, 1.0, 8, 8, None, None, None, 0, 4, 4, 16, bg, None, 2, None, 0.6, 30,
                                       None, None, None, None, opts, None, 0, None)
        assert rc != 0
        assert b"fit" in lib.spx_last_error()
    # A stack's rows per image must divide the image height.
    for opts in (_lib.FitOptions(_lib.FIT_F64, 1e-12, 3), _lib.FitOptions(_lib.FIT_F64, 1e-12, -8)):
        rc = lib.spx_deblend_iteration(None, 1, 1.0, 8, 8, None, None, None, 0, 4, 4, 16, bg, None, 2, None, 0.6, 30,
                                       None, None, None, None, opts, None, 0, None)
        assert rc != 0
        assert b"rows_per_image" in lib.spx_last_error()
    # Patches of a stack need the cell boxes (they say which image a cell is in).
    rc = lib.spx_extract_patches_stack(None, 1, 1.0, 2, 8, 8, None, None, 1, None, None, None)
    assert rc != 0 and b"boxes" in lib.spx_last_error()


def test_status_names_match_the_binding():
    """The library's status names (also written as UCS-4 text on the device) are the binding's."""
    from imageprocessor_new_b200 import _lib

    lib = _lib.load_library()
    assert [lib.spx_status_name(i).decode() for i in range(len(_lib.STATUS_NAMES))] == list(_lib.STATUS_NAMES)
    assert lib.spx_status_name(len(_lib.STATUS_NAMES)) is None
    assert max(len(n) for n in _lib.STATUS_NAMES) < 32

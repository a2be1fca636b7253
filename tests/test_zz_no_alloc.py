"""spx_otsu_static, the allocation-free Otsu entry point, against spx_otsu.

spx_otsu_static serves callers that cannot allocate device memory (stream capture, real-time loops,
hosts whose allocator owns all device memory): its scratch is a file-scope device array shared by
every call. This file is collected last so that a failure here comes after every other test.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _otsu_reference(lib, img_d, code, step):
    import torch

    out = torch.empty(1, dtype=torch.float64, device="cuda")
    ws = torch.empty(int(lib.spx_otsu_workspace_bytes(code)), dtype=torch.uint8, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    assert lib.spx_otsu(img_d.data_ptr(), code, img_d.shape[0], img_d.shape[1], step, out.data_ptr(),
                        ws.data_ptr(), ws.numel(), stream) == 0, lib.spx_last_error()
    return float(out.item())


def test_otsu_static_matches_allocating_entry_point_twice():
    import torch

    from imageprocessor_new_b200 import _lib, synthetic

    lib = _lib.lib()
    page = synthetic.page_square(0).image                       # uint16, Otsu ~2.2k
    rng = np.random.default_rng(7)
    noise = rng.integers(0, 65536, (300, 517)).astype(np.uint16)  # full 16-bit range
    small = (page[:200, :300] >> 4).astype(np.uint8)
    stream = torch.cuda.current_stream().cuda_stream
    for img, code, step in ((page, 1, 1), (page, 1, 4), (noise, 1, 1), (small, 0, 1)):
        img_d = torch.from_numpy(np.ascontiguousarray(img)).cuda()
        want = _otsu_reference(lib, img_d, code, step)
        for _ in range(2):  # the shared array keeps the last call's contents; each call must clear it
            out = torch.full((1,), -1.0, dtype=torch.float64, device="cuda")
            status = lib.spx_otsu_static(img_d.data_ptr(), code, img_d.shape[0], img_d.shape[1], step,
                                         out.data_ptr(), stream)
            assert status == 0, lib.spx_last_error()
            assert float(out.item()) == want  # bit-exact: both compute OpenCV's Otsu bin


def test_otsu_static_rejects_oversized_images():
    import torch

    from imageprocessor_new_b200 import _lib

    lib = _lib.lib()
    tiny = torch.zeros((4, 4), dtype=torch.uint16, device="cuda")
    out = torch.empty(1, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    # 65536 x 65537 sampled pixels exceed the 32-bit histogram counts: rejected on the host before
    # any launch (the pointer is never read).
    status = lib.spx_otsu_static(tiny.data_ptr(), 1, 65536, 65537, 1, out.data_ptr(), stream)
    assert status == -1
    assert b"exceed the maximum" in lib.spx_last_error()

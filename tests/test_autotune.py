"""The autotuner's output and the checked-in tables (no GPU): the header it
writes compiles and holds the given rows; the library's size queries answer
with the rows of the committed tables (csrc/plain_tuning.h,
csrc/batch_tuning.h); and every committed choice is among the widths the
tuner sweeps for its size, so a re-run can reproduce it."""
import ctypes
import os
import re
import subprocess

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(REPO, "era-bellman-cuda_b200", "csrc")


def table_rows(header: str):
    text = open(os.path.join(CSRC, header)).read()
    body = text[text.index("constexpr tuning_row"):]
    return [(int(a), int(b)) for a, b in re.findall(r"\{(\d+),\s*(\d+)\}", body)]


def test_written_header_compiles_with_its_rows(tmp_path):
    import autotune
    rows = [(0, 3), (5, 4), (12, 9), (22, 20)]
    path = tmp_path / "t.h"
    autotune.write_header(str(path), rows, "unit test", ["2^5: c=4 1.0 ms -> c=4"], name="TEST_TUNING", what="a test")
    prog = tmp_path / "p.cpp"
    prog.write_text('#include "t.h"\n#include <cstdio>\nint main() { for (const auto &r : msm_b200::TEST_TUNING) '
                    'std::printf("%u %u\\n", r.max_log_n, r.window_bits); }\n')
    exe = tmp_path / "p"
    subprocess.run(["g++", "-std=c++17", "-I", str(tmp_path), str(prog), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()
    assert [(int(out[i]), int(out[i + 1])) for i in range(0, len(out), 2)] == rows


@pytest.mark.parametrize("header,query", [("plain_tuning.h", "msm_b200_default_window_bits"),
                                          ("batch_tuning.h", "msm_b200_batch_window_bits")])
def test_library_answers_with_the_committed_rows(product_lib_path, header, query):
    lib = ctypes.CDLL(product_lib_path)
    fn = getattr(lib, query)
    fn.argtypes = [ctypes.c_uint, ctypes.POINTER(ctypes.c_uint)]
    fn.restype = ctypes.c_int
    rows = table_rows(header)
    assert rows and [lg for lg, _ in rows] == sorted(lg for lg, _ in rows)
    c = ctypes.c_uint()
    for lg, width in rows:
        if lg > 31:
            continue
        assert fn(1 << lg, ctypes.byref(c)) == 0 and c.value == width, (header, lg)
        if lg >= 2:  # a count just above the previous size class takes this row too
            assert fn((1 << (lg - 1)) + 1, ctypes.byref(c)) == 0 and c.value == width, (header, lg)


def test_committed_choices_are_among_the_swept_widths():
    import autotune
    for lg, width in table_rows("plain_tuning.h"):
        if lg >= 4:  # the smallest sizes are written as copies of the 2^4 row
            assert width in autotune.plain_candidates(lg), ("plain", lg, width)
    for lg, width in table_rows("batch_tuning.h"):
        if 10 <= lg <= 23:
            assert width in autotune.candidates(lg), ("batch", lg, width)

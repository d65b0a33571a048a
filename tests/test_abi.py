"""The C-ABI library: loads without a GPU, exports every function the headers
in include/ declare, and its ctypes mirror matches the C struct layout (and the
reference header's layout when the reference tree is present)."""
import ctypes
import os
import re
import subprocess

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INCLUDE = os.path.join(REPO, "include")
# the reference source tree: the REF environment variable, else a `reference`
# directory beside this repository (absent on machines without it: skipped)
REF_HEADER = os.path.join(os.environ.get("REF") or os.path.join(os.path.dirname(REPO), "reference"), "src", "bellman-cuda.h")


def declared_functions():
    names = set()
    for h in ("bellman-cuda.h", "bellman-cuda-b200.h"):
        text = open(os.path.join(INCLUDE, h)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names |= set(re.findall(r"^bc_error\s+(\w+)\s*\(", text, flags=re.M))
    return sorted(names)


def test_library_exports_every_declared_symbol(product_lib_path):
    lib = ctypes.CDLL(product_lib_path)
    names = declared_functions()
    assert len(names) >= 40
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_reference_msm_surface_is_declared():
    """Every MSM-path function of the reference ABI appears in include/bellman-cuda.h."""
    names = set(declared_functions())
    required = """bc_get_device_count bc_get_device bc_set_device bc_stream_create bc_stream_wait_event
    bc_stream_synchronize bc_stream_query bc_stream_destroy bc_launch_host_fn bc_event_create bc_event_record
    bc_event_synchronize bc_event_query bc_event_destroy bc_event_elapsed_time bc_mem_get_info bc_malloc
    bc_malloc_host bc_free bc_free_host bc_host_register bc_host_unregister bc_device_disable_peer_access
    bc_device_enable_peer_access bc_memcpy bc_memcpy_async bc_memset bc_memset_async bc_mem_pool_create
    bc_mem_pool_destroy bc_mem_pool_disable_peer_access bc_mem_pool_enable_peer_access bc_malloc_from_pool_async
    bc_free_async ff_set_up msm_set_up msm_execute_async msm_tear_down""".split()
    assert not [n for n in required if n not in names]


LAYOUT_PROGRAM = r"""
#include <stdio.h>
#include <stddef.h>
#include "bellman-cuda.h"
int main(void) {
  printf("%zu %zu %zu %zu %zu %zu %zu %zu %d %d %d %d\n", sizeof(msm_configuration),
         offsetof(msm_configuration, bases), offsetof(msm_configuration, scalars),
         offsetof(msm_configuration, results), offsetof(msm_configuration, log_scalars_count),
         offsetof(msm_configuration, h2d_copy_finished), offsetof(msm_configuration, d2h_copy_finished),
         offsetof(msm_configuration, d2h_copy_finished_callback_data),
         (int)bc_success, (int)bc_error_invalid_value, (int)bc_error_memory_allocation, (int)bc_error_not_ready);
  return 0;
}
"""


def c_layout(include_dir, tmp_path, tag):
    src = tmp_path / f"layout_{tag}.c"
    exe = tmp_path / f"layout_{tag}"
    src.write_text(LAYOUT_PROGRAM)
    subprocess.run(["gcc", "-std=c11", "-I", include_dir, str(src), "-o", str(exe)], check=True)
    return subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()


def test_struct_layout_matches_ctypes(tmp_path):
    import bellman_cuda as bc
    got = c_layout(INCLUDE, tmp_path, "b200")
    M = bc.MsmConfiguration
    mine = [ctypes.sizeof(M), M.bases.offset, M.scalars.offset, M.results.offset, M.log_scalars_count.offset,
            M.h2d_copy_finished.offset, M.d2h_copy_finished.offset, M.d2h_copy_finished_callback_data.offset, 0, 1, 2, 600]
    assert [int(v) for v in got] == mine


@pytest.mark.skipif(not os.path.exists(REF_HEADER), reason="reference tree absent")
def test_struct_layout_matches_reference_header(tmp_path):
    ref = c_layout(os.path.dirname(REF_HEADER), tmp_path, "ref")
    mine = c_layout(INCLUDE, tmp_path, "b200")
    assert ref == mine


def test_reference_build_exports_same_msm_surface():
    path = os.path.join(REPO, "oracle", "_ref", "libbellman-cuda-ref.so")
    if not os.path.exists(path):
        pytest.skip("reference GPU build absent")
    out = subprocess.run(["nm", "-D", "--defined-only", path], check=True, capture_output=True, text=True).stdout
    ref_syms = set(line.split()[-1] for line in out.splitlines())
    mine = set(declared_functions())
    assert {n for n in mine if not n.startswith("msm_b200_") and n != "ff_tear_down"} <= ref_syms


POINT_PROGRAM = r"""
#include <stdio.h>
#include <stddef.h>
#include "bellman-cuda-b200.h"
int main(void) {
  printf("%zu %zu %zu %zu\n", sizeof(msm_b200_affine_point), offsetof(msm_b200_affine_point, y),
         offsetof(msm_b200_affine_point, infinity), offsetof(msm_b200_affine_point, reserved));
  return 0;
}
"""


def test_affine_point_layout_matches_ctypes(tmp_path):
    """msm_b200_affine_point, the final sum's output, as C lays it out."""
    import bellman_cuda as bc
    src = tmp_path / "point.c"
    exe = tmp_path / "point"
    src.write_text(POINT_PROGRAM)
    subprocess.run(["gcc", "-std=c11", "-I", INCLUDE, str(src), "-o", str(exe)], check=True)
    got = [int(v) for v in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()]
    A = bc.AffinePoint
    assert got == [ctypes.sizeof(A), A.y.offset, A.infinity.offset, A.reserved.offset] == [80, 32, 64, 68]


def test_argument_checks_without_a_gpu(product_lib_path):
    """The checks that come before any CUDA call (null, misaligned or
    out-of-range arguments) return bc_error_invalid_value on a machine
    without a GPU too; the size queries answer from the tuning tables."""
    import bellman_cuda as bc
    lib = bc.BellmanCuda(product_lib_path).lib
    null_stream = bc.Handle()
    invalid = bc.BC_ERROR_INVALID_VALUE
    assert lib.msm_b200_final_sum_async(None, None, null_stream) == invalid
    assert lib.msm_b200_final_sum_async(0x1008, 0x2000, null_stream) == invalid  # results not 16-byte aligned
    assert lib.msm_b200_final_sum_async(0x1000, 0x2002, null_stream) == invalid  # point not 4-byte aligned
    assert lib.msm_b200_execute_no_alloc_async(null_stream, None, 0x1000, 0x2000, 16) == invalid
    assert lib.msm_b200_execute_no_alloc_async(null_stream, 0x1000, 0x2000, 0x3000, 0) == invalid
    assert lib.msm_b200_execute_no_alloc_async(null_stream, 0x1000, 0x2000, 0x3000, bc.NO_ALLOC_MAX_COUNT + 1) == invalid
    assert lib.msm_b200_execute_no_alloc_async(null_stream, 0x1008, 0x2000, 0x3000, 16) == invalid
    assert lib.msm_b200_execute_async(None) == invalid
    cfg = bc.MsmConfiguration()
    cfg.log_scalars_count = 32
    assert lib.msm_execute_async(cfg) == invalid
    assert lib.msm_b200_batch_create(None, None, None, 0, None) == invalid
    c = ctypes.c_uint()
    assert lib.msm_b200_default_window_bits(0, ctypes.byref(c)) == invalid
    assert lib.msm_b200_default_window_bits(1 << 22, ctypes.byref(c)) == 0 and c.value == 17
    assert lib.msm_b200_batch_window_bits(1 << 22, ctypes.byref(c)) == 0 and c.value == 20


LINK_PROGRAM = r"""
#include <stdio.h>
#include "bellman-cuda.h"
#include "bellman-cuda-b200.h"
/* A C caller of the drop-in: the reference's msm_configuration by value, and
   the extensions; run with no GPU it only exercises the argument checks. */
int main(void) {
  msm_configuration cfg = {0};
  cfg.log_scalars_count = 40;
  bc_stream stream = {0};
  int a = msm_execute_async(cfg);
  int b = msm_b200_final_sum_async(NULL, NULL, stream);
  int c = msm_b200_execute_no_alloc_async(stream, NULL, NULL, NULL, 0);
  unsigned bits = 0;
  int d = msm_b200_default_window_bits(1u << 20, &bits);
  printf("%d %d %d %d %u\n", a, b, c, d, bits);
  return 0;
}
"""


def test_c_caller_links_and_runs_without_a_gpu(product_lib_path, tmp_path):
    """A C program includes both headers, links the shared library by name
    (-lbellman_cuda_b200) and runs its argument checks on a machine without a GPU."""
    src = tmp_path / "caller.c"
    exe = tmp_path / "caller"
    src.write_text(LINK_PROGRAM)
    libdir = os.path.dirname(product_lib_path)
    subprocess.run(["gcc", "-std=c11", "-I", INCLUDE, str(src), "-L", libdir, "-lbellman_cuda_b200", "-Wl,-rpath," + libdir, "-o", str(exe)],
                   check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()
    table = open(os.path.join(os.path.dirname(INCLUDE), "era-bellman-cuda_b200", "csrc", "plain_tuning.h")).read()
    width_2_20 = re.search(r"\{20, (\d+)\}", table).group(1)  # the measured width at 2^20 points
    assert out == ["1", "1", "1", "0", width_2_20]

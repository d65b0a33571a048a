// Host build of the server's device-arena allocator (era-bellman-cuda_b200/csrc/device_arena.h)
// for tests/test_arena.py: a C interface over one arena.
#include "device_arena.h"

static msm_b200::device_arena g_arena;

extern "C" {
void arena_reset(size_t bytes) { g_arena.reset(bytes); }
int arena_allocate(size_t bytes, size_t *offset) { return g_arena.allocate(bytes, *offset) ? 1 : 0; }
void arena_release(size_t offset, size_t bytes) { g_arena.release(offset, bytes); }
size_t arena_largest_free() { return g_arena.largest_free(); }
size_t arena_used() { return g_arena.used(); }
size_t arena_free_blocks() { return g_arena.free_blocks(); }
}

"""Host-side checks that need no GPU: argument validation that must refuse a
call before anything is launched, and the per-context cache of the fixed
scratch array's device address."""
import ctypes as C
import os
import subprocess
import tempfile

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "taichi_b200", "csrc")

TC_ERR_INVALID = 1


def test_thumbnail_entries_check_params_first(tc):
    """An opening length of 2^20 or an eye element of 0 would make the
    single-CTA morphology kernel run for hours; both thumbnail entry points
    refuse them before any CUDA call (the fake device pointers are never
    touched)."""
    fake = C.c_void_p(256)
    for over in ({"open_len": 1 << 20}, {"eye_size": 0}, {"thumb_height": 1 << 16}):
        p = tc.params(**over)
        W = C.c_int(-1)
        st = tc.lib().tc_thumbnail_noalloc(1 << 20, 1 << 20, fake, fake, C.byref(p), fake,
                                           C.byref(W), None)
        assert st == TC_ERR_INVALID, (over, st)
        mF, Wv, nc = C.c_int(), C.c_int(), C.c_int()
        st = tc.lib().tc_getsdf(1 << 20, 1 << 20, fake, fake, C.byref(p), C.byref(mF), C.byref(Wv),
                                None, 0, C.byref(nc), None, None)
        assert st == TC_ERR_INVALID, (over, st)


def test_plan_params_refused_before_cuda(tc):
    """tc_params the multiply cannot honour are refused by the plan entry
    points before any CUDA call: a rows-kernel word count outside {0, 4, 6,
    8}, tile_mode 3, max_lanes 3."""
    f = tc.Format()
    out = C.c_void_p()
    for over in ({"rows_w": 5}, {"rows_w": 16}, {"tile_mode": 3}, {"max_lanes": 3}):
        p = tc.params(**over)
        st = tc.lib().tc_plan_from_format(10, 10, C.byref(f), C.byref(p), None, C.byref(out))
        assert st == TC_ERR_INVALID, (over, st)
        assert "rows_w" in tc.lib().tc_last_error().decode() or "rows_w" not in over


CACHE_TEST = r'''
#include <cstdio>
#include "tc_ctxcache.h"
static int fails = 0;
#define CHECK(c) do { if (!(c)) { std::printf("FAIL line %d: %s\n", __LINE__, #c); ++fails; } } while (0)
int main() {
    tc::ContextAddressCache<4> cache;
    int next = 100, broken = 0;
    auto resolve = [&](void **a) { if (broken) return 7; *a = (void *)(long)(next++); return 0; };
    void *p = nullptr;
    CHECK(cache.get(0, 11, resolve, &p) == 0 && p == (void *)100L);       // first lookup
    CHECK(cache.get(0, 11, resolve, &p) == 0 && p == (void *)100L);       // same context: cached
    CHECK(cache.lookups() == 1);
    CHECK(cache.get(0, 12, resolve, &p) == 0 && p == (void *)101L);       // context recreated
    CHECK(cache.get(0, 12, resolve, &p) == 0 && p == (void *)101L);
    CHECK(cache.get(1, 12, resolve, &p) == 0 && p == (void *)102L);       // another device
    CHECK(cache.get(0, 0, resolve, &p) == 0 && p == (void *)103L);        // unknown context:
    CHECK(cache.get(0, 0, resolve, &p) == 0 && p == (void *)104L);        // never cached
    CHECK(cache.get(0, 12, resolve, &p) == 0 && p == (void *)105L);       // id 0 dropped the entry
    broken = 1;
    CHECK(cache.get(2, 13, resolve, &p) == 7);                            // failure passed through
    broken = 0;
    CHECK(cache.get(2, 13, resolve, &p) == 0 && p == (void *)106L);       // and not cached
    CHECK(cache.get(4, 13, resolve, &p) == -1 && cache.get(-1, 13, resolve, &p) == -1);
    CHECK(cache.lookups() == 7);
    std::printf("%s\n", fails ? "failed" : "ok");
    return fails != 0;
}
'''


def test_context_address_cache():
    """The scratch address is reused only within the context that looked it
    up; a new context id (after cudaDeviceReset) triggers a new lookup."""
    d = tempfile.mkdtemp()
    src = os.path.join(d, "cache_test.cpp")
    exe = os.path.join(d, "cache_test")
    with open(src, "w") as f:
        f.write(CACHE_TEST)
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", CSRC, src, "-o", exe, "-lpthread"], check=True)
    r = subprocess.run([exe], stdout=subprocess.PIPE, text=True)
    assert r.returncode == 0 and r.stdout.strip() == "ok", r.stdout

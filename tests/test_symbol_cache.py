"""CPU test of the per-context symbol-address cache behind hpb_dot2_f64_noalloc
(csrc/hpb_symbol_cache.h): one lookup per context id, separate entries for
separate contexts (a context recreated after cudaDeviceReset has a new id),
a failed lookup is not cached, and the oldest entry is replaced when full.
The header is plain C++; it is compiled here with g++ and a fake lookup."""
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent

DRIVER = r'''
#include "hpb_symbol_cache.h"
#include <cstdio>
static int calls = 0;
static int fail_next = 0;
static int resolve_for(unsigned long long id, void** out) {
    ++calls;
    if (fail_next) { fail_next = 0; return 7; }
    *out = reinterpret_cast<void*>(0x1000 + id * 16);
    return 0;
}
#define CHECK(c) do { if (!(c)) { std::printf("FAIL line %d\n", __LINE__); return 1; } } while (0)
int main() {
    hpb::SymbolAddressCache<3> c;
    void* p = nullptr;
    auto get = [&](unsigned long long id) { return c.get(id, &p, [id](void** o) { return resolve_for(id, o); }); };
    CHECK(get(5) == 0 && p == reinterpret_cast<void*>(0x1000 + 5 * 16) && calls == 1);
    CHECK(get(5) == 0 && calls == 1);                 // cached: no second lookup
    CHECK(get(6) == 0 && p == reinterpret_cast<void*>(0x1000 + 6 * 16) && calls == 2);  // another context
    CHECK(get(5) == 0 && p == reinterpret_cast<void*>(0x1000 + 5 * 16) && calls == 2);
    fail_next = 1;
    CHECK(get(9) == 7 && calls == 3 && c.size() == 2);  // failure reported, not cached
    CHECK(get(9) == 0 && calls == 4 && c.size() == 3);
    CHECK(get(10) == 0 && calls == 5 && c.size() == 3); // full: oldest (5) replaced
    CHECK(get(6) == 0 && calls == 5);
    CHECK(get(5) == 0 && calls == 6);                   // 5 was evicted: looked up again
    std::printf("ok\n");
    return 0;
}
'''


@pytest.mark.skipif(shutil.which("g++") is None, reason="g++ not present")
def test_symbol_cache_logic(tmp_path):
    src = tmp_path / "cache_test.cpp"
    src.write_text(DRIVER)
    exe = tmp_path / "cache_test"
    r = subprocess.run(["g++", "-std=c++17", "-O1", "-I", str(ROOT / "high_precision_blas1_b200" / "csrc"),
                        str(src), "-o", str(exe), "-pthread"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-2000:]
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    assert r.returncode == 0 and r.stdout.strip() == "ok", r.stdout + r.stderr

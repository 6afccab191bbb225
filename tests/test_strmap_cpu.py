"""The table dictionaries' string -> id map (StrIdMap, runtime.h) against
std::unordered_map on the host: random strings of every length (the empty
one, ones sharing long prefixes, ones past the 8-byte hash step), repeated
inserts, lookups after growth, and a clear that keeps the table for reuse.
Compiled with g++ from the header alone; no GPU."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

PROGRAM = r'''
#include <cstdio>
#include <random>
#include <unordered_map>
#include "runtime.h"

int main() {
    std::mt19937_64 rng(42);
    vr::StrIdMap m;
    int bad = 0;
    for (int round = 0; round < 3; ++round) {
        std::unordered_map<std::string, int32_t> ref;
        m.clear();
        for (int i = 0; i < 200000; ++i) {
            const int len = (int)(rng() % 40);
            std::string s = (rng() % 4 == 0) ? std::string("shared-prefix-of-some-length-") : std::string();
            for (int k = 0; k < len; ++k) s.push_back((char)(rng() % 7 == 0 ? 0 : 'a' + rng() % 26));
            auto it = m.find(s);
            auto rt = ref.find(s);
            if ((it == m.end()) != (rt == ref.end())) ++bad;
            if (it == m.end()) {
                const int32_t id = (int32_t)m.size();
                auto e = m.emplace(s, id);
                if (!e.second || e.first->second != id) ++bad;
                ref.emplace(s, id);
            } else if (it->second != rt->second) {
                ++bad;
            }
            auto again = m.emplace(s, -7);  // present: no insert, the old id
            if (again.second || again.first->second != ref[s]) ++bad;
        }
        if (m.size() != ref.size()) ++bad;
        for (const auto& kv : ref) {
            auto it = m.find(kv.first);
            if (it == m.end() || it->second != kv.second) ++bad;
        }
    }
    std::printf("%d\n", bad);
    return 0;
}
'''


def test_string_id_map_matches_unordered_map(tmp_path):
    if not shutil.which("g++"):
        pytest.skip("no C++ compiler")
    src = tmp_path / "strmap.cpp"
    src.write_text(PROGRAM)
    exe = tmp_path / "strmap"
    cuda = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    inc = [os.path.join(ROOT, "include"), os.path.join(ROOT, "vecruntime_b200", "csrc"), os.path.join(cuda, "include"),
           os.path.join(ROOT, "_build", "vrgpu")]
    cmd = ["g++", "-std=c++17", "-O2", str(src), "-o", str(exe)] + [f"-I{p}" for p in inc]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0 and "cuda_runtime.h" in r.stderr:
        pytest.skip("no CUDA headers")
    assert r.returncode == 0, r.stderr[-2000:]
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.strip()
    assert out == "0"

"""Division by multiplication (fast_divisor, raytracing_b200/csrc/device_types.h): the kernels turn sample and
work-item numbers into passes, pixels and strata with n / d = high 64 bits of n * magic, magic = floor((2^64 - 1) / d)
+ 1, for n < 2^32. The host's make_fast_divisor is compiled here with g++ and the quotient checked against the plain
division for every divisor the kernels use (a round's strata a side and its passes, the tiles a row, the padded
pixels of image sizes from 1 x 1 up to 46340 x 46340) and the dividends that decide exactness (0, 1, multiples of d
and their neighbours, 2^32 - 1, random numbers)."""
import shutil
import subprocess
from pathlib import Path

import pytest

REPO = Path(__file__).resolve().parent.parent

CHECK = r"""
#include <cstdint>
#include <cstdio>
#include <random>
#include "device_types.h"

static uint32_t quotient(uint32_t n, const rtb::fast_divisor& v)
{
    return v.magic != 0 ? static_cast<uint32_t>((static_cast<unsigned __int128>(n) * v.magic) >> 64) : n;
}

int main()
{
    std::mt19937_64 gen(7);
    long long checked = 0, wrong = 0;
    auto check_divisor = [&](uint32_t d) {
        const rtb::fast_divisor v = rtb::make_fast_divisor(d);
        if (v.d != d) { ++wrong; return; }
        auto one = [&](uint32_t n) {
            ++checked;
            if (quotient(n, v) != n / d) { ++wrong; if (wrong < 5) std::printf("wrong: %u / %u\n", n, d); }
        };
        one(0); one(1); one(UINT32_MAX); one(UINT32_MAX - 1);
        for (uint64_t k : {uint64_t{1}, uint64_t{2}, uint64_t{3}, uint64_t{UINT32_MAX} / d, uint64_t{UINT32_MAX} / d - 1})
        {
            const uint64_t m = k * d;
            if (m <= UINT32_MAX) { one(static_cast<uint32_t>(m)); }
            if (m >= 1 && m - 1 <= UINT32_MAX) { one(static_cast<uint32_t>(m - 1)); }
            if (m + 1 <= UINT32_MAX) { one(static_cast<uint32_t>(m + 1)); }
        }
        for (int i = 0; i < 200; ++i) { one(static_cast<uint32_t>(gen())); }
    };
    for (uint32_t d = 1; d <= 70000; ++d) { check_divisor(d); }
    for (uint32_t s = 1; s <= 46340; s += 37) { check_divisor(s * s); }
    for (uint32_t w = 1; w <= 46340; w += 61)
    {
        for (uint32_t h : {1u, 3u, 4u, 225u, 1080u, 2160u, 46340u})
        {
            const uint64_t tiles = uint64_t{(w + 7) / 8} * ((h + 3) / 4) * 32;
            if (tiles < (uint64_t{1} << 32)) { check_divisor(static_cast<uint32_t>(tiles)); }
        }
    }
    for (int i = 0; i < 20000; ++i) { check_divisor(static_cast<uint32_t>(gen() | 1u)); }
    check_divisor(UINT32_MAX);
    std::printf("%lld %lld\n", checked, wrong);
    return wrong == 0 ? 0 : 1;
}
"""


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_division_by_multiplication_is_exact(tmp_path):
    src = tmp_path / "check.cpp"
    src.write_text(CHECK)
    exe = tmp_path / "check"
    cuda_include = Path("/usr/local/cuda/include")
    cmd = ["g++", "-O2", "-std=c++20", "-I", str(REPO / "raytracing_b200" / "csrc"), "-I", str(cuda_include),
           str(src), "-o", str(exe)]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout
    checked, wrong = map(int, r.stdout.split()[-2:])
    assert wrong == 0 and checked > 10_000_000

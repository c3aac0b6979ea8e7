"""The random stream of the reference's beam-grid reduction (Beams/Grid.hxx:558-598: Rng over
std::mt19937_64 and std::uniform_real_distribution<float>, Misc/Rng.hxx:51-62), as the GPU grid
build restates it (k_mt64_floats in smallupbp_b200/csrc/upbp_grid.cu): the 64-bit Mersenne Twister,
each output x mapped to float(x) / 2^64 and clamped below 1, which is how libstdc++ computes
uniform_real_distribution<float> from one 64-bit output.  Checked here against the C++ standard's
known answer and against the C++ library itself, compiled with g++ as the reference is.
"""
import shutil
import subprocess

import numpy as np
import pytest

MASK = (1 << 64) - 1


def mt19937_64(seed: int):
    """The 64-bit Mersenne Twister (n 312, m 156, r 31), seeded as std::mt19937_64(seed)."""
    n, m = 312, 156
    upper, lower, a = 0xFFFFFFFF80000000, 0x7FFFFFFF, 0xB5026F5AA96619E9
    mt = [seed & MASK]
    for i in range(1, n):
        mt.append((6364136223846793005 * (mt[-1] ^ (mt[-1] >> 62)) + i) & MASK)
    while True:
        for i in range(n):
            x = (mt[i] & upper) | (mt[(i + 1) % n] & lower)
            mt[i] = mt[(i + m) % n] ^ (x >> 1) ^ (a if x & 1 else 0)
        for y in mt:
            y ^= (y >> 29) & 0x5555555555555555
            y ^= (y << 17) & 0x71D67FFFEDA60000 & MASK
            y ^= (y << 37) & 0xFFF7EEE000000000 & MASK
            y ^= y >> 43
            yield y


def canonical_float(x: int) -> np.float32:
    f = np.float32(np.uint64(x)) * np.float32(2.0 ** -64)
    return f if f < np.float32(1) else np.nextafter(np.float32(1), np.float32(0))


def test_mt19937_64_known_answer():
    # [rand.predef]: the 10000th consecutive output of a default-constructed mt19937_64 (seed 5489)
    g = mt19937_64(5489)
    for _ in range(9999):
        next(g)
    assert next(g) == 9981545732273789042


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_stream_matches_the_cpp_library(tmp_path):
    src = tmp_path / "rng.cpp"
    src.write_text(
        "#include <cstdio>\n#include <cstdlib>\n#include <cstring>\n#include <random>\n"
        "int main(int argc, char** argv) {\n"
        "  std::mt19937_64 r(std::atoi(argv[1]));\n"
        "  std::uniform_real_distribution<float> d;\n"
        "  for (int i = 0; i < std::atoi(argv[2]); ++i) {\n"
        "    float f = d(r); unsigned u; std::memcpy(&u, &f, 4); std::printf(\"%u\\n\", u);\n"
        "  }\n}\n")
    exe = tmp_path / "rng"
    subprocess.check_call(["g++", "-O2", "-msse4.2", str(src), "-o", str(exe)])
    for seed in (1234, 77, -5, 2 ** 31 - 1):
        want = np.array(subprocess.check_output([str(exe), str(seed), "3000"]).split(), np.uint32)
        g = mt19937_64(seed)
        got = np.array([canonical_float(next(g)) for _ in range(3000)], np.float32).view(np.uint32)
        np.testing.assert_array_equal(got, want, err_msg="seed %d" % seed)

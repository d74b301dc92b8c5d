"""div_rn (aero_device.cuh), the exact division the LU-SGS sweeps use, checked
bit for bit against IEEE division on the host: the same source compiled as
plain C++ (fma and fabs from <cmath>), on random operands over the whole
exponent range it accepts and on quotients next to rounding midpoints."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SRC = r"""
#include <cmath>
#include <cstdio>
#include <cstdint>
#include <cstring>
#include <random>
using std::fabs; using std::fma;
#define __host__
#define __device__
#define __forceinline__ inline
#include "aero_device.cuh"
int main() {
  std::mt19937_64 g(3);
  std::uniform_real_distribution<double> u(1.0, 2.0);
  long bad = 0, n = 0;
  auto check = [&](double a, double b) {
    double q = aero::div_rn(a, b, 1.0 / b), t = a / b;
    ++n;
    if (std::memcmp(&q, &t, 8) && !(std::isnan(q) && std::isnan(t))) {
      if (bad < 5) std::printf("a=%a b=%a got=%a want=%a\n", a, b, q, t);
      ++bad;
    }
  };
  for (int e1 = -1000; e1 <= 1000; e1 += 13)
    for (int e2 = -1000; e2 <= 1000; e2 += 17)
      for (int s = 0; s < 40; ++s) check(std::ldexp(u(g), e1) * ((g() & 1) ? -1 : 1), std::ldexp(u(g), e2));
  for (long s = 0; s < 3000000; ++s) {
    double q = u(g), b = std::ldexp(u(g), (int)(g() % 60) - 30);
    double a = (double)((long double)(q + std::ldexp(1.0, -53)) * (long double)b);
    int k = (int)(g() % 5) - 2;
    for (int i = 0; i < (k < 0 ? -k : k); ++i) a = std::nextafter(a, k > 0 ? INFINITY : -INFINITY);
    check(a, b);
  }
  check(0.0, 3.0); check(-0.0, 3.0); check(1.0, 0.0); check(NAN, 2.0); check(INFINITY, 2.0);
  std::printf("n=%ld bad=%ld\n", n, bad);
  return bad != 0;
}
"""


def test_div_rn_matches_ieee_division(tmp_path):
    cxx = shutil.which("g++")
    if cxx is None:
        pytest.skip("g++ not available")
    src = tmp_path / "t.cpp"
    src.write_text(SRC)
    exe = tmp_path / "t"
    subprocess.run([cxx, "-O2", "-std=c++17", "-ffp-contract=off", "-I", os.path.join(ROOT, "aerocfd_b200", "csrc"),
                    str(src), "-o", str(exe)], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr

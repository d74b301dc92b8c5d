"""div_rn and div2_rn (aero_device.cuh), the exact divisions the LU-SGS sweeps
use, checked bit for bit against IEEE division on the host: the same source
compiled as plain C++ (fma and fabs from <cmath>), on random operands over the
whole exponent range, across the bounds of the fast paths, and on quotients
next to rounding midpoints."""
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
#define __noinline__
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
  // (a / b1) / b2 as the sweeps form it
  auto check2 = [&](double a, double b1, double b2) {
    double q = aero::div2_rn(a, b1, 1.0 / b1, b2, 1.0 / b2, aero::divisors_ok(b1, b2)), t = a / b1 / b2;
    ++n;
    if (std::memcmp(&q, &t, 8) && !(std::isnan(q) && std::isnan(t))) {
      if (bad < 5) std::printf("a=%a b1=%a b2=%a got=%a want=%a\n", a, b1, b2, q, t);
      ++bad;
    }
  };
  for (int ea = -1000; ea <= 1000; ea += 37)
    for (int e1 = -260; e1 <= 260; e1 += 20)
      for (int e2 = -260; e2 <= 260; e2 += 20)
        for (int s = 0; s < 4; ++s)
          check2(std::ldexp(u(g), ea) * ((g() & 1) ? -1 : 1), std::ldexp(u(g), e1) * ((g() & 1) ? -1 : 1),
                 std::ldexp(u(g), e2));
  for (int ea : {-501, -500, -499, 499, 500, 501})
    for (int e1 : {-201, -200, -199, 199, 200, 201})
      for (int s = 0; s < 50; ++s) check2(std::ldexp(u(g), ea), std::ldexp(u(g), e1), std::ldexp(u(g), -e1));
  for (long s = 0; s < 1000000; ++s)
    check2(std::ldexp(u(g), (int)(g() % 80) - 40), std::ldexp(u(g), (int)(g() % 60) - 30),
           std::ldexp(u(g), (int)(g() % 60) - 30));
  check2(0.0, 3.0, 5.0); check2(-0.0, 3.0, -5.0); check2(1.0, 0.0, 2.0); check2(NAN, 2.0, 3.0);
  check2(INFINITY, 2.0, 3.0); check2(1.0, 1e-300, 1e-300); check2(1e300, 1e-10, 1e-10);
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

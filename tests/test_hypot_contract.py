"""The probability p = cabs(a)^2 that drives the reference's sampling is
computed with glibc's hypot.  The engine reproduces glibc 2.39's published
algorithm (Borges 2019, corrected variant without fused multiply-add) on
the device (moonlab_b200/csrc/hypot_glibc.cuh).  This test pins that
algorithm against the host glibc on random inputs over a wide range of
scales; the GPU tests then check the device's p values bit for bit."""
from __future__ import annotations

import subprocess
import tempfile
from pathlib import Path

SRC = r"""
#include <complex.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>
static uint64_t s = 0x1234567;
static uint64_t sm(void) { uint64_t z = (s += 0x9e3779b97f4a7c15ULL);
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL; z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
  return z ^ (z >> 31); }
static double U(void) { return (sm() >> 11) * 0x1p-53; }
static double kern(double ax, double ay) {
  double h = sqrt(ax * ax + ay * ay), t1, t2;
  if (h <= 2.0 * ay) { double d = h - ay; t1 = ax * (2.0 * d - ax); t2 = (d - 2.0 * (ax - ay)) * d; }
  else { double d = h - ax; t1 = 2.0 * d * (ax - 2.0 * ay); t2 = (4.0 * d - ay) * ay + d * d; }
  return h - (t1 + t2) / (2.0 * h);
}
static double hyp(double x, double y) {
  x = fabs(x); y = fabs(y);
  double ax = x < y ? y : x, ay = x < y ? x : y;
  if (ax > 0x1p511) { if (ay <= ax * 0x1p-54) return ax + ay; return kern(ax * 0x1p-600, ay * 0x1p-600) / 0x1p-600; }
  if (ay < 0x1p-511) { if (ax >= ay / 0x1p-54) return ax + ay; return kern(ax / 0x1p-600, ay / 0x1p-600) * 0x1p-600; }
  if (ay <= ax * 0x1p-54) return ax + ay;
  return kern(ax, ay);
}
int main(void) {
  long bad = 0, N = 3000000;
  for (long k = 0; k < N; k++) {
    double sc = ldexp(1.0, -(int)(sm() % 80));
    double x = (U() * 2 - 1) * sc, y = (U() * 2 - 1) * sc * ((k & 3) ? 1 : ldexp(1.0, -(int)(sm() % 60)));
    if (k % 1000 == 0) x = ldexp(x, -600);
    double g = cabs(CMPLX(x, y));
    if (hyp(x, y) != g || g * g != hyp(x, y) * hyp(x, y)) bad++;
  }
  printf("%ld\n", bad);
  return 0;
}
"""


def test_borges_hypot_matches_glibc():
    with tempfile.TemporaryDirectory() as d:
        src = Path(d) / "h.c"
        exe = Path(d) / "h"
        src.write_text(SRC)
        subprocess.run(["gcc", "-O2", "-ffp-contract=off", str(src), "-o", str(exe), "-lm"], check=True)
        out = subprocess.run([str(exe)], check=True, capture_output=True, text=True, timeout=120)
        assert int(out.stdout.strip()) == 0

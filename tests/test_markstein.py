"""The fast path divides by dx with Markstein's method (rh::divDx in
rhybrid_b200/csrc/k_fast.cuh): q = RN(x * r), r = RN(1/dx), then
RN(q + fma(-q, dx, x) * r). This checks, on the CPU with the same IEEE
fused multiply-add, that it returns the correctly rounded x / dx bit for bit
on random and adversarial inputs for several cell sizes; the GPU parity tests
check the kernels' results against the oracle's IEEE divisions."""
import os
import shutil
import subprocess

import pytest

SRC = r"""
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>
static uint64_t s = 88172645463325252ull;
static uint64_t rnd(void) { s ^= s << 13; s ^= s >> 7; s ^= s << 17; return s; }
static double u01(void) { return (rnd() >> 11) * 0x1.0p-53; }
static double divdx(double x, double dx, double r) {
   const double q = x * r;
   const double aq = fabs(q);
   if (!(aq >= 0x1p-500 && aq <= 0x1p+500)) return x / dx;
   const double e = fma(-q, dx, x);
   return fma(e, r, q);
}
int main(void) {
   const double dxs[] = {100e3, 300e3, 1.0, 3.0, 0.1, 7.3e5, 123456.789, 1e-3, 2440e3 / 17.0};
   long bad = 0, tot = 0;
   for (int d = 0; d < 9; ++d) {
      const double dx = dxs[d], r = 1.0 / dx;
      for (long n = 0; n < 4000000; ++n) {
         double x;
         const int m = n % 5;
         if (m == 0) x = u01() * dx;
         else if (m == 1) x = (u01() * 3 - 1) * dx;
         else if (m == 2) { uint64_t b = rnd(); memcpy(&x, &b, 8); }
         else if (m == 3) x = nextafter(dx * (double)(rnd() % 4), (rnd() & 1) ? 0.0 : 1e300);
         else x = (rnd() & 1) ? 0.0 : -0.0;
         const double a = x / dx, b = divdx(x, dx, r);
         ++tot;
         if (memcmp(&a, &b, 8) && !(isnan(a) && isnan(b))) { if (bad < 5) printf("dx %.17g x %.17g: %.17g vs %.17g\n", dx, x, a, b); ++bad; }
      }
   }
   printf("%ld %ld\n", tot, bad);
   return bad != 0;
}
"""


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs gcc")
def test_markstein_division_is_correctly_rounded(tmp_path):
    src = tmp_path / "mk.c"
    src.write_text(SRC)
    exe = tmp_path / "mk"
    subprocess.run(["gcc", "-O2", "-ffp-contract=off", "-o", str(exe), str(src), "-lm"], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True)
    assert out.returncode == 0, out.stdout
    tot, bad = map(int, out.stdout.split()[-2:])
    assert tot > 30_000_000 and bad == 0

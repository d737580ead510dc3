"""Generate ``dark_pow_table.h``: the inputs on which the host C library's
``powf(x, 1.2f)`` is not the correctly rounded binary32 power.

The dark-protection weight of the adaptive quantiser is
``powf(72 / (16 + mean), 1.2f)`` clamped to [1, 4.5] (src/aq_common.rs:312-345,
DarkAq::on constants at :177-214).  The reference calls the C library's
``powf`` (glibc on x86-64 Linux), which is accurate to < 1 ulp but not
correctly rounded.  The device evaluates the power in binary64 and rounds it
once to binary32; that equals glibc's ``powf`` except on the inputs listed here,
for which the table carries glibc's result.

An input is listed when (a) glibc's ``powf`` differs from the binary64 power
rounded to binary32, or (b) the binary64 power lies within 2^-44 (relative) of
a binary32 rounding boundary, where a few-ulp binary64 error could round either
way.  Every binary32 x in (1, 4.5] is checked; below 1 the weight clamps to 1
and 4.5 is the largest reachable base (mean >= 0).

Usage (from the repository root; needs gcc and the same C library as the
oracle)::

    python maroontree_b200/csrc/gen_dark_pow_table.py
"""
import os
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "dark_pow_table.h")

PROGRAM = r"""
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>
static float f_of(uint32_t u) { float f; memcpy(&f, &u, 4); return f; }
static uint32_t u_of(float f) { uint32_t u; memcpy(&u, &f, 4); return u; }
int main(void) {
  const float g = 1.2f;
  const uint32_t lo = u_of(1.0f) + 1, hi = u_of(4.5f);
  long n = 0;
  for (uint32_t u = lo; u <= hi; u++) {
    const float x = f_of(u);
    const float r = powf(x, g);
    const double p = pow((double)x, (double)g);
    const float c = (float)p;
    const float nb = (p >= (double)c) ? nextafterf(c, INFINITY) : nextafterf(c, -INFINITY);
    const double mid = ((double)c + (double)nb) * 0.5;
    const int near = fabs(p - mid) < ldexp(p, -44);
    if (r != c || near) {
      printf("%u %u\n", u, u_of(r));
      n++;
    }
  }
  fprintf(stderr, "%ld entries\n", n);
  return 0;
}
"""


def generate():
    with tempfile.TemporaryDirectory() as d:
        src = os.path.join(d, "gen.c")
        exe = os.path.join(d, "gen")
        with open(src, "w") as f:
            f.write(PROGRAM)
        subprocess.run(["gcc", "-O2", "-ffp-contract=off", "-fno-fast-math", src, "-o", exe, "-lm"], check=True)
        out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout
    rows = [tuple(int(v) for v in line.split()) for line in out.splitlines() if line.strip()]
    lines = [
        "/* Generated by gen_dark_pow_table.py: binary32 inputs x in (1, 4.5] on which",
        " * the C library's powf(x, 1.2f) differs from (or may round differently than)",
        " * the binary64 power rounded once to binary32, with the library's result.",
        " * Sorted by the bit pattern of x.  Device arrays: include from one .cu file.",
        " * Do not edit. */",
        "#pragma once",
        "#include <stdint.h>",
        "",
        f"#define MT_DARK_POW_N {len(rows)}",
        f"__device__ const uint32_t kDarkPowX[{len(rows)}] = {{",
    ]
    for i in range(0, len(rows), 8):
        lines.append("  " + ",".join(f"0x{x:08x}" for x, _ in rows[i:i + 8]) + ",")
    lines.append("};")
    lines.append(f"__device__ const uint32_t kDarkPowR[{len(rows)}] = {{")
    for i in range(0, len(rows), 8):
        lines.append("  " + ",".join(f"0x{r:08x}" for _, r in rows[i:i + 8]) + ",")
    lines.append("};")
    # Bucket index: entries of bucket b (x bits in [BASE + b * 4096, BASE + (b+1) * 4096))
    # are kDarkPowX[kDarkPowB[b] .. kDarkPowB[b + 1]).
    base, shift = 0x3F800000, 12
    nb = ((0x40900000 - base) >> shift) + 1
    starts, k = [], 0
    for b_ in range(nb + 1):
        while k < len(rows) and ((rows[k][0] - base) >> shift) < b_:
            k += 1
        starts.append(k)
    lines.append(f"#define MT_DARK_POW_BASE 0x{base:08x}u")
    lines.append(f"#define MT_DARK_POW_SHIFT {shift}")
    lines.append(f"#define MT_DARK_POW_NB {nb}")
    lines.append(f"__device__ const uint16_t kDarkPowB[{nb + 1}] = {{")
    for i in range(0, len(starts), 16):
        lines.append("  " + ",".join(str(v) for v in starts[i:i + 16]) + ",")
    lines.append("};")
    with open(OUT, "w") as f:
        f.write("\n".join(lines) + "\n")
    return len(rows)


if __name__ == "__main__":
    n = generate()
    print(f"{OUT}: {n} entries", file=sys.stderr)

"""Host checks of the step's fast variants of stream functions (pliscuda_b200/csrc/plis_stream.h).

The kernels use plis_exp_normal / plis_expf_normal for the leap's e^-lambda and Philox blocks computed
from precomputed round keys (plis_round_keys, plis_philox4x32_10_rk, plis_group_uniforms_rk_d/_f); the
oracle uses plis_exp / plis_expf and plis_philox4x32_10.  The header is the same source on both sides,
so these bit-for-bit equalities on the host pin the claim the device parity tests rely on.
"""
import os
import subprocess
import tempfile

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

PROGRAM = r"""
#include <cstdio>
#include <cstring>
#include "plis_stream.h"

static uint64_t s = 0x9E3779B97F4A7C15ull;
static uint64_t next() { s ^= s << 13; s ^= s >> 7; s ^= s << 17; return s; }

int main() {
  long bad = 0;
  // e^-lambda for 0 <= lambda < 20: the normal-range variants equal the full functions bit for bit
  for (long i = 0; i < 2000000; ++i) {
    const double lam = (double)(next() >> 11) * (20.0 / 9007199254740992.0);
    const double a = plis_exp(-lam), b = plis_exp_normal(-lam);
    if (memcmp(&a, &b, 8) != 0) ++bad;
    const float lf = (float)lam;
    const float c = plis_expf(-lf), d = plis_expf_normal(-lf);
    if (memcmp(&c, &d, 4) != 0) ++bad;
  }
  const double edges[] = {0.0, 1e-300, 5e-324, 1e-17, 0.5, 1.0, 10.0, 19.999999999999996};
  for (double lam : edges) {
    const double a = plis_exp(-lam), b = plis_exp_normal(-lam);
    if (memcmp(&a, &b, 8) != 0) ++bad;
  }
  // Philox blocks from precomputed round keys equal plis_philox4x32_10 / plis_group_block
  for (long i = 0; i < 200000; ++i) {
    const uint64_t seed = next();
    const uint32_t replica = (uint32_t)next();
    uint32_t rk0[10], rk1[10];
    plis_round_keys(seed, replica, rk0, rk1);
    const plis_stream g = plis_stream_make(seed, replica, (uint32_t)next(), 2u, next(), (uint32_t)next() & 0xFFFu,
                                           (uint32_t)next() & 0xFFFFFu);
    for (uint32_t blk = 0; blk < 2; ++blk) {
      const plis_u32x4 a = plis_group_block(&g, blk), b = plis_group_block_rk(&g, blk, rk0, rk1);
      if (a.x != b.x || a.y != b.y || a.z != b.z || a.w != b.w) ++bad;
    }
    double ud[6], vd[6];
    float uf[6], vf[6];
    plis_group_uniforms_d(&g, 0x3Fu, ud, 6);
    plis_group_uniforms_rk_d(&g, 0x3Fu, vd, 6, rk0, rk1);
    plis_group_uniforms_f(&g, 0x3Fu, uf, 6);
    plis_group_uniforms_rk_f(&g, 0x3Fu, vf, 6, rk0, rk1);
    if (memcmp(ud, vd, sizeof ud) != 0 || memcmp(uf, vf, sizeof uf) != 0) ++bad;
  }
  printf("%ld\n", bad);
  return bad != 0;
}
"""


def test_fast_stream_variants_are_bit_identical():
    with tempfile.TemporaryDirectory() as d:
        src, exe = os.path.join(d, "variants.cpp"), os.path.join(d, "variants")
        with open(src, "w") as f:
            f.write(PROGRAM)
        # the oracle's flags: no contraction, so the host evaluates the header's operations as written
        subprocess.run(["g++", "-std=c++17", "-O2", "-mfma", "-ffp-contract=off",
                        "-I" + os.path.join(ROOT, "pliscuda_b200", "csrc"), src, "-o", exe], check=True)
        r = subprocess.run([exe], capture_output=True, text=True)
        assert r.returncode == 0, f"{r.stdout.strip()} mismatches"

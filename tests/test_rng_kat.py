"""Philox4x32-10 against the published known-answer vectors (Salmon et al.,
SC'11; the Random123 distribution's kat_vectors file), for both copies of
the generator: the oracle's (oracle/irbc_rng.h) and the library's
(csrc/common.cuh, its __host__ __device__ function compiled for the host by
nvcc).  The draw stream of every phase is built on this function, so a
wrong round or key schedule would move every random number on both sides
alike; only these vectors catch that."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

# (counter, key) -> output, 32-bit words
KAT = [
    ((0x00000000, 0x00000000, 0x00000000, 0x00000000), (0x00000000, 0x00000000),
     (0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8)),
    ((0xffffffff, 0xffffffff, 0xffffffff, 0xffffffff), (0xffffffff, 0xffffffff),
     (0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd)),
    ((0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344), (0xa4093822, 0x299f31d0),
     (0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1)),
]

_ORACLE_MAIN = r"""
#include <stdio.h>
#include "irbc_rng.h"
int main(void) {
  unsigned c[4], k[2];
  while (scanf("%x %x %x %x %x %x", &c[0], &c[1], &c[2], &c[3], &k[0], &k[1]) == 6) {
    uint32_t ci[4] = {c[0], c[1], c[2], c[3]}, ki[2] = {k[0], k[1]}, o[4];
    orc_philox4x32_10(ci, ki, o);
    printf("%08x %08x %08x %08x\n", o[0], o[1], o[2], o[3]);
  }
  return 0;
}
"""

_LIBRARY_MAIN = r"""
#include <cstdio>
#include "common.cuh"
int main() {
  unsigned c[4], k[2];
  while (std::scanf("%x %x %x %x %x %x", &c[0], &c[1], &c[2], &c[3], &k[0], &k[1]) == 6) {
    uint32_t o[4];
    irbc::philox4x32_10(c[0], c[1], c[2], c[3], k[0], k[1], o);
    std::printf("%08x %08x %08x %08x\n", o[0], o[1], o[2], o[3]);
  }
  return 0;
}
"""


def _run(exe):
    inp = "".join(" ".join("%08x" % w for w in c + k) + "\n" for c, k, _ in KAT)
    out = subprocess.run([exe], input=inp, capture_output=True, text=True, check=True).stdout.split("\n")
    return [tuple(int(w, 16) for w in line.split()) for line in out if line.strip()]


def test_oracle_philox_known_answers(tmp_path):
    src = tmp_path / "kat.c"
    src.write_text(_ORACLE_MAIN)
    exe = tmp_path / "kat_oracle"
    subprocess.run(["gcc", "-O2", "-I", os.path.join(ROOT, "oracle"), str(src), "-o", str(exe), "-lm"], check=True)
    assert _run(str(exe)) == [o for _, _, o in KAT]


def test_library_philox_known_answers(tmp_path):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(nvcc):
        pytest.skip("nvcc not found")
    src = tmp_path / "kat.cu"
    src.write_text(_LIBRARY_MAIN)
    exe = tmp_path / "kat_library"
    subprocess.run([nvcc, "-O2", "-std=c++17", "-I", os.path.join(ROOT, "irbc-code_b200", "csrc"), str(src),
                    "-o", str(exe)], check=True)
    assert _run(str(exe)) == [o for _, _, o in KAT]

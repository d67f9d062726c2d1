"""CPU: the space bookkeeping of the pinned upload ring (thx_ring.h).

The ring stages host->device uploads; a span is reused only after its copy
has completed, so a placement that overlaps a live span would corrupt an
upload still queued on the stream.  A small C++ driver (compiled here with
g++) places and retires spans in seeded random order and checks every
placement against the live spans, including the wrap that fills the ring
exactly."""
import os
import shutil
import subprocess
import tempfile

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "..", "theseus_b200", "csrc")

DRIVER = r"""
#include "thx_ring.h"
#include <cstdio>
#include <deque>
#include <random>
#include <utility>

static int check(thx::RingSpace &r, std::deque<std::pair<size_t, size_t>> &live, size_t need,
                 size_t cap) {
  size_t off;
  while (!r.place(need, &off)) {
    if (live.empty()) { std::printf("no placement in an empty ring\n"); return 1; }
    live.pop_front();
    r.pop();
  }
  if (off + need > cap) { std::printf("span past the end: %zu+%zu\n", off, need); return 1; }
  for (auto &s : live)
    if (off < s.first + s.second && s.first < off + need) {
      std::printf("overlap: [%zu,%zu) with live [%zu,%zu)\n", off, off + need, s.first,
                  s.first + s.second);
      return 1;
    }
  live.push_back({off, need});
  r.push(off, need);
  return 0;
}

int main() {
  // the exact-fill wrap: A[0,10) B[10,20) C[20,28), retire A, D[0,5), E[5,10)
  // fills [0,10) up to the tail B: the next span must wait for B and C
  {
    thx::RingSpace r(30);
    std::deque<std::pair<size_t, size_t>> live;
    for (size_t n : {10, 10, 8}) if (check(r, live, n, 30)) return 1;
    live.pop_front(); r.pop();
    for (size_t n : {5, 5, 10}) if (check(r, live, n, 30)) return 1;
  }
  std::mt19937_64 g(7);
  for (int trial = 0; trial < 200; ++trial) {
    const size_t cap = 64 + g() % 4096;
    thx::RingSpace r(cap);
    std::deque<std::pair<size_t, size_t>> live;
    for (int it = 0; it < 4000; ++it) {
      if (!live.empty() && g() % 3 == 0) {  // a copy completes
        live.pop_front();
        r.pop();
        continue;
      }
      const size_t need = 1 + g() % (cap / 2);
      if (check(r, live, need, cap)) return 1;
    }
  }
  std::printf("ok\n");
  return 0;
}
"""


@pytest.mark.skipif(shutil.which("g++") is None, reason="g++ not found")
def test_ring_space_never_overlaps_live_spans():
    with tempfile.TemporaryDirectory() as d:
        src = os.path.join(d, "ring.cpp")
        exe = os.path.join(d, "ring")
        with open(src, "w") as f:
            f.write(DRIVER)
        subprocess.run(["g++", "-std=c++17", "-O1", "-I", CSRC, src, "-o", exe], check=True)
        out = subprocess.run([exe], capture_output=True, text=True, timeout=60)
        assert out.returncode == 0 and out.stdout.strip() == "ok", out.stdout + out.stderr

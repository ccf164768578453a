"""The physics Verlet list's layout (`nl_word`, quantom_b200/csrc/physkern.cuh),
checked on the host against the invariants the step kernel's loads rely on:

* every (slot i < n_pad, entry k < cap) has its own word, inside the
  cap * n_pad words allocated;
* lane g of a particle finds its entries g + 8 (4q + u), u = 0..3, in four
  consecutive words starting on a multiple of 4 words, so one 8-byte (16-bit
  ids) or 16-byte (32-bit ids) vector load reads them aligned; chunk 0's
  vector is the (8 i + g)-th vector of the list and chunk q's lies q n_pad 8
  vectors further;
* the 4 particles of one warp own 128 contiguous words of every chunk, the
  range one bulk L2 prefetch per chunk covers;
* the capacity rounds up to whole 32-entry chunks.

The check is a host program compiled from the header with nvcc (no GPU).
"""
import shutil
import subprocess

import pytest

from conftest import ROOT

CHECK = r"""
#include <cstdio>
#include <vector>
#include "physkern.cuh"
using lima::nl_word;
int main() {
    const unsigned pads[] = {32u, 64u, 96u, 32032u};
    const int wants[] = {1, 31, 32, 33, 295, 576};
    for (int want : wants) {
        const int cap = lima::nl_round_cap(want);
        if (cap % lima::kListChunk || cap < want || cap - want >= lima::kListChunk) { puts("cap"); return 1; }
        for (unsigned n_pad : pads) {
            const size_t words = (size_t)cap * n_pad;
            std::vector<unsigned char> seen(words, 0);
            for (unsigned i = 0; i < n_pad; i++)
                for (unsigned k = 0; k < (unsigned)cap; k++) {
                    const size_t w = nl_word(n_pad, i, k);
                    if (w >= words || seen[w]) { printf("bijection %u %u %u\n", n_pad, i, k); return 1; }
                    seen[w] = 1;
                }
            for (unsigned i = 0; i < n_pad; i++)
                for (unsigned g = 0; g < 8; g++) {
                    if (nl_word(n_pad, i, g) != (8 * i + g) * 4) { puts("column base"); return 1; }
                    for (unsigned q = 0; q < (unsigned)cap / 32; q++) {
                        const size_t w0 = nl_word(n_pad, i, g + 32 * q);
                        if (w0 % 4 || w0 != ((size_t)q * n_pad * 8 + 8 * i + g) * 4) { puts("vector"); return 1; }
                        for (unsigned u = 1; u < 4; u++)
                            if (nl_word(n_pad, i, g + 8 * (4 * q + u)) != w0 + u) { puts("run"); return 1; }
                    }
                }
            for (unsigned i0 = 0; i0 < n_pad; i0 += 4)
                for (unsigned q = 0; q < (unsigned)cap / 32; q++) {
                    const size_t lo = ((size_t)q * n_pad + i0) * 32;
                    for (unsigned p = 0; p < 4; p++)
                        for (unsigned k = 32 * q; k < 32 * q + 32; k++) {
                            const size_t w = nl_word(n_pad, i0 + p, k);
                            if (w < lo || w >= lo + 128) { puts("warp span"); return 1; }
                        }
                }
        }
    }
    puts("ok");
    return 0;
}
"""


def test_list_layout_invariants(tmp_path):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not shutil.which(nvcc) and not (ROOT / nvcc).exists():
        pytest.skip("nvcc not found")
    src = tmp_path / "check.cu"
    src.write_text(CHECK)
    exe = tmp_path / "check"
    cmd = [nvcc, "-std=c++17", "-O2", f"-I{ROOT / 'include'}", f"-I{ROOT / 'quantom_b200' / 'csrc'}", str(src), "-o",
           str(exe), "-Wno-deprecated-gpu-targets"]
    subprocess.run(cmd, check=True, capture_output=True, timeout=600)
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=600)
    assert out.returncode == 0 and out.stdout.strip() == "ok", out.stdout

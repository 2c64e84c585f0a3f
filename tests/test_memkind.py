"""The rule that decides how the library treats an array argument
(clgpu_b200/csrc/memkind.h), checked on the CPU: pinned host memory is
staged by direct DMA, ordinary (pageable) host memory through the handle's
pinned bounce buffers, memory of the handle's GPU (or managed memory) is used
in place, and device memory of any other GPU is rejected before a copy or a
kernel could touch it.  The header has no CUDA dependency, so it compiles
here with g++ alone; no kernel is launched."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

PROGRAM = r"""
#include <cstdio>
#include "memkind.h"
using iclb::MemKind;
using iclb::classify_memory;
int main() {
    int bad = 0;
    // cudaMemoryType: 0 unregistered, 1 host (pinned), 2 device, 3 managed
    struct { int type, ptr_dev, handle_dev; MemKind want; } cases[] = {
        {0, -2, 0, MemKind::Pageable},      // malloc'd memory: through the pinned bounce buffers
        {1, 0, 0, MemKind::Host},           // pinned host memory is staged too
        {1, 3, 0, MemKind::Host},
        {2, 0, 0, MemKind::Device},         // the handle's GPU
        {2, 5, 5, MemKind::Device},
        {2, 1, 0, MemKind::OtherDevice},    // another GPU: rejected
        {2, 0, 7, MemKind::OtherDevice},
        {3, 1, 0, MemKind::Device},         // managed memory: any GPU reaches it
    };
    for (auto& c : cases) {
        MemKind got = classify_memory(c.type, c.ptr_dev, c.handle_dev);
        if (got != c.want) {
            std::printf("type %d ptr_dev %d handle_dev %d: got %d want %d\n", c.type, c.ptr_dev, c.handle_dev,
                        (int)got, (int)c.want);
            ++bad;
        }
    }
    std::printf("%d bad\n", bad);
    return bad;
}
"""


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_other_gpu_memory_is_rejected_not_used(tmp_path):
    src = tmp_path / "memkind_check.cpp"
    src.write_text(PROGRAM)
    exe = tmp_path / "memkind_check"
    r = subprocess.run(["g++", "-std=c++17", "-I", os.path.join(ROOT, "clgpu_b200", "csrc"), str(src), "-o",
                        str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout
    assert "0 bad" in r.stdout

"""Builds tests/_native/libmqp_emu.so, the host emulation of the 2D kernel,
of the 2D block kernel for large windows, of the 3D kernels and of the
post-processing kernels, of the direct small-window kernels and of the 2D
kernel for search windows above 128 used by the CPU tests (see mqp_emu.cu,
mqp_emu_big.cu, mqp_emu3d.cu, mqp_emu_post.cu, mqp_emu_direct.cu,
mqp_emu_huge.cu)."""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
CSRC = os.path.join(ROOT, "multi_quickpiv_b200", "csrc")
OUT = os.path.join(os.path.dirname(HERE), "_native", "libmqp_emu.so")


def build(force=False):
    srcs = [os.path.join(HERE, f) for f in ("mqp_emu.cu", "mqp_emu3d.cu", "mqp_emu_post.cu", "mqp_emu_big.cu", "mqp_emu_direct.cu", "mqp_emu_huge.cu")]
    deps = srcs + [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".inc"))]
    if not force and os.path.exists(OUT) and all(os.path.getmtime(d) <= os.path.getmtime(OUT) for d in deps):
        return OUT
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    cmd = ["nvcc", "-std=c++17", "-O2", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC,-fvisibility=hidden",
           "-shared", "-I", CSRC] + srcs + ["-o", OUT]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(r.stdout + r.stderr)
    return OUT


if __name__ == "__main__":
    print(build("--force" in sys.argv))

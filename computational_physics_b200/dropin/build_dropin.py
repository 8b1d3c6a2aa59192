"""Builds the reference's own Ising2D program with the nvidia_gpu target plugged in.

The reference (flwende/computational_physics) selects its target device through a few seams:
the DeviceName enum and Device<> map (utility/device/device.hpp), GetDevice / DispatchCall
(utility/device/helper.{hpp,cpp}), the Lattice<2> GPU hooks (ising/include/lattice.hpp) and a
SwendsenWang_2D / LCG32 per target.  This recipe

  1. copies the reference sources it needs (utility/, ising/, random/) into a scratch
     directory (never into this repository),
  2. adds the files under dropin/src/ (this project's own code: the NVIDIA_GPU device and
     CudaContext, LCG32<NVIDIA_GPU>, SwendsenWang_2D<LCG32, NVIDIA_GPU> over libswb200.so,
     the Lattice<2> hooks),
  3. inserts the lines that register the target at those seams (the INSERTS table below:
     each anchor must occur exactly once, else the build stops), all behind CP_NVIDIA_GPU,
  4. compiles the reference's Ising2D (ising/src/ising_2d.cpp and the sources it links, the
     CPU target included) with the reference's own compiler flags plus -DCP_NVIDIA_GPU, linked
     against libswb200.so,

and writes only computational_physics_b200/lib/dropin/Ising2D.  `--target=cpu` of that binary
is the reference's unchanged CPU path, `--target=nvidia_gpu` the B200 engine.

    python -m computational_physics_b200.dropin.build_dropin [--ref DIR]

DIR defaults to $SWB_REFERENCE_DIR, else /root/reference.  The lcg32 lane count of the CPU path
is the compiler's SIMD width: -march=x86-64-v4 (AVX-512) gives 16, the nvidia_gpu target's.
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)
ROOT = os.path.dirname(PKG)
OUT_DIR = os.path.join(PKG, "lib", "dropin")

# (file, anchor, text, where): `text` goes right after / right before the anchor, or replaces it.
INSERTS = [
    ("utility/device/device.hpp", "AMD_GPU = 2", """,
#if defined CP_NVIDIA_GPU
        NVIDIA_GPU = 3
#endif""", "after"),
    ("utility/device/device.hpp", '#include "device_amd_gpu.hpp"', """
#include "device_nvidia_gpu.hpp\"""", "after"),
    ("utility/device/helper.hpp", """        else
            throw std::runtime_error("Unknown device name.");""", """    #if defined CP_NVIDIA_GPU
        else if (device_name == "nvidia_gpu")
            return func(static_cast<NVIDIA_GPU&>(device), std::forward<Args>(args)...);
    #endif
""", "before"),
    ("utility/device/helper.cpp", """        else
            throw std::runtime_error("Unknown target device.");""", """#if defined CP_NVIDIA_GPU
        else if (device_name == "nvidia_gpu")
            return std::make_unique<NVIDIA_GPU>();
#endif
""", "before"),
    ("random/include/random/lcg32.hpp", "#undef XXX_NAMESPACE", """

#include "lcg32_nvidia_gpu.hpp\"""", "after_last"),
    ("ising/include/lattice.hpp", """            GpuPointer<Spin> gpu_spins {};
#endif""", """
#if defined CP_NVIDIA_GPU
            NvGpuPointer<Spin> nv_gpu_spins {};
#endif""", "after"),
    ("ising/include/lattice.hpp", """                    InitializeGpuSpins(target);
""", """#if defined CP_NVIDIA_GPU
                if constexpr (Target::Name() == DeviceName::NVIDIA_GPU)
                    InitializeGpuSpins(target);
#endif
""", "after"),
    ("ising/include/lattice.hpp", """            auto RawGpuPointer() const noexcept { return gpu_spins.get(); }
#endif""", """
#if defined CP_NVIDIA_GPU
            auto RawGpuPointer() noexcept { return nv_gpu_spins.get(); }
            auto RawGpuPointer() const noexcept { return nv_gpu_spins.get(); }
#endif""", "after"),
    ("ising/include/lattice.hpp", """            void InitializeGpuSpins(AMD_GPU& gpu);
#endif""", """
#if defined CP_NVIDIA_GPU
            void InitializeGpuSpins(NVIDIA_GPU& gpu);
#endif""", "after"),
    ("ising/include/swendsen_wang.hpp", '#include "swendsen_wang_selflabeling.hpp"', """
#include "swendsen_wang_nvidia_gpu.hpp\"""", "after"),
    ("ising/src/ising_2d.cpp", """                  << "  --temperature""", """#if defined CP_NVIDIA_GPU
                  << "  --target=<name>    Set target device (default: cpu)" << std::endl
                  << "      Supported target devices: cpu, nvidia_gpu" << std::endl
#endif
""", "before"),
    ("ising/src/ising_2d.cpp", '(target->Name() == DeviceName::CPU ? "CPU" : "AMD GPU")',
     '(target->Name() == DeviceName::CPU ? "CPU" : TargetName(target->Name()))', "replace"),
    ("ising/src/ising_2d.cpp", "using namespace XXX_NAMESPACE;", """

// Printed name of a GPU target (the nvidia_gpu target added to the reference's CPU / AMD GPU).
static const char* TargetName(const DeviceName name)
{
#if defined CP_NVIDIA_GPU
    if (name == DeviceName::NVIDIA_GPU)
        return "NVIDIA GPU";
#endif
    return "AMD GPU";
}""", "after"),
]

REF_SOURCES = ["ising/src/ising_2d.cpp", "ising/src/swendsen_wang.cpp", "ising/src/swendsen_wang_cpu.cpp",
               "ising/src/lattice.cpp", "random/src/lcg32.cpp", "utility/device/helper.cpp"]
OWN_SOURCES = ["ising/src/swendsen_wang_nvidia_gpu.cpp", "ising/src/lattice_nvidia_gpu.cpp"]
# The reference's flags (CMakeLists.txt:8-12, ising/src/CMakeLists.txt:1-15) with a fixed ISA
# level in place of -march=native, so that the CPU path's lane count is 16.
FLAGS = ["-std=c++20", "-O3", "-fopenmp-simd", "-ftree-vectorize", "-ffast-math", "-DRANDOM_SHUFFLE_STATE",
         "-Wno-ignored-attributes", "-march=x86-64-v4", "-DCP_NVIDIA_GPU"]


def apply_inserts(tree: str) -> None:
    for rel, anchor, text, where in INSERTS:
        path = os.path.join(tree, rel)
        src = open(path).read()
        n = src.count(anchor)
        if n == 0 or (n > 1 and where != "after_last"):
            raise SystemExit(f"{rel}: anchor found {n} times: {anchor!r}")
        if where == "after":
            src = src.replace(anchor, anchor + text, 1)
        elif where == "after_last":
            i = src.rindex(anchor) + len(anchor)
            src = src[:i] + text + src[i:]
        elif where == "before":
            src = src.replace(anchor, text + anchor, 1)
        else:
            src = src.replace(anchor, text, 1)
        with open(path, "w") as f:
            f.write(src)


def build(ref: str, verbose: bool = True) -> str:
    if not os.path.isdir(os.path.join(ref, "ising")):
        raise SystemExit(f"reference sources not found under {ref}")
    lib = os.path.join(PKG, "lib", "libswb200.so")
    if not os.path.exists(lib):
        raise SystemExit("build libswb200.so first: python -m computational_physics_b200.build")
    os.makedirs(OUT_DIR, exist_ok=True)
    exe = os.path.join(OUT_DIR, "Ising2D")
    with tempfile.TemporaryDirectory(prefix="swb_dropin_") as tree:
        for d in ("utility", "ising", "random"):
            shutil.copytree(os.path.join(ref, d), os.path.join(tree, d))
        shutil.copytree(os.path.join(HERE, "src"), tree, dirs_exist_ok=True)
        apply_inserts(tree)
        inc = ["-I", os.path.join(tree, "utility"), "-I", os.path.join(tree, "ising", "include"),
               "-I", os.path.join(tree, "random", "include"), "-I", os.path.join(ROOT, "include")]
        srcs = [os.path.join(tree, s) for s in REF_SOURCES + OWN_SOURCES]
        cmd = ["/usr/bin/g++", *FLAGS, *inc, "-o", exe, *srcs, "-L", os.path.dirname(lib), "-lswb200",
               f"-Wl,-rpath,{os.path.dirname(lib)}", "-Wl,-rpath,$ORIGIN/..", "-lpthread", "-lm"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return exe


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("SWB_REFERENCE_DIR", "/root/reference"))
    args = ap.parse_args()
    print(build(args.ref))


if __name__ == "__main__":
    sys.exit(main())

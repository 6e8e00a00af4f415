"""Build recipe for the test oracle (TEST INFRASTRUCTURE ONLY).

Two things are built here, both as checkers, never as the product:

1. ``oracle/_build/libbp_oracle.so`` -- the FP64 C restatement in ``bp_oracle.c``.
2. ``oracle/_ref/`` -- the reference's own code, compiled from its sources where they
   lie in the mmNorm checkout (only when that checkout is present):
     * ``imaging<ext>``: the reference C++ OpenMP imager
       (src/data_processing/cpp/imaging.cpp, imaging.h, utils/include/mmwave_common.h),
       with the flags of its Makefile (src/data_processing/cpp/Makefile:7) except that
       ``-march=native`` becomes ``-march=x86-64-v3`` so the library runs on any
       x86-64-v3 host, and the unused boost libraries are not linked;
     * ``imaging_gpu.cubin`` / ``surface_normal_est.cubin``: the reference CUDA kernels
       (src/data_processing/cuda/imaging_gpu.cu, surface_normal_est.cu) compiled
       unmodified for sm_100a, to be launched by ``oracle/ref_cuda.py``;
     * ``raytrace/ray_tracing_ref.so``: the reference's ray-marching extension
       (src/data_processing/cpp/ray_tracing.cpp + src/data_processing/cuda/
       ray_tracing_kernel.cu, the two sources its setup.py lists) compiled unmodified for
       sm_100a with torch's extension builder, imported by ``oracle/iso_oracle.py``.

Outputs under ``oracle/_ref`` and ``oracle/_build`` are git-ignored build products.
Usage: ``python oracle/build.py [--ref-root PATH]``; the mmNorm checkout comes from
``--ref-root`` or the ``MMNORM_REF_ROOT`` environment variable, and without either only
the C oracle is built.
"""
from __future__ import annotations

import os
import subprocess
import sys
import sysconfig

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "_build")
REF_OUT = os.path.join(HERE, "_ref")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")


def _run(cmd: list[str]) -> None:
    proc = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if proc.returncode != 0:
        raise RuntimeError("command failed: %s\n%s" % (" ".join(cmd), proc.stdout))


def _stale(out: str, srcs: list[str]) -> bool:
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(s) > t for s in srcs)


def build_oracle(force: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    src = os.path.join(HERE, "bp_oracle.c")
    out = os.path.join(BUILD, "libbp_oracle.so")
    if force or _stale(out, [src]):
        _run(["gcc", "-O2", "-fopenmp", "-fPIC", "-shared", "-ffp-contract=off",
              "-march=x86-64-v2", src, "-o", out, "-lm"])
    return out


def build_ref(ref_root: str | None = None, force: bool = False) -> dict:
    """Compile the reference's imager and kernels from the checkout at `ref_root` (default:
    $MMNORM_REF_ROOT); returns {name: path} of what exists.  Without a checkout nothing is
    built."""
    built = {}
    ref_root = ref_root or os.environ.get("MMNORM_REF_ROOT")
    if not ref_root or not os.path.isdir(ref_root):
        return built
    os.makedirs(REF_OUT, exist_ok=True)
    cpp_dir = os.path.join(ref_root, "src", "data_processing", "cpp")
    cu_dir = os.path.join(ref_root, "src", "data_processing", "cuda")
    inc = os.path.join(ref_root, "src", "utils", "include")

    ext = sysconfig.get_config_var("EXT_SUFFIX") or ".so"
    imaging_src = os.path.join(cpp_dir, "imaging.cpp")
    imaging_out = os.path.join(REF_OUT, "imaging" + ext)
    if os.path.exists(imaging_src):
        if force or _stale(imaging_out, [imaging_src]):
            import pybind11  # noqa: WPS433 (build-time dependency)
            py_inc = sysconfig.get_paths()["include"]
            _run(["g++", "-Wall", "-Ofast", "-std=c++14", "-fPIC", "-shared",
                  "-march=x86-64-v3", "-frename-registers", "-fopenmp", imaging_src,
                  "-o", imaging_out, "-I" + py_inc, "-I" + pybind11.get_include(),
                  "-I" + cpp_dir, "-I" + inc])
        built["imaging"] = imaging_out

    for name in ("imaging_gpu", "surface_normal_est"):
        src = os.path.join(cu_dir, name + ".cu")
        out = os.path.join(REF_OUT, name + ".cubin")
        if not os.path.exists(src):
            continue
        if force or _stale(out, [src]):
            _run([NVCC, "-cubin", "-gencode", "arch=compute_100a,code=sm_100a",
                  "-o", out, src])
        built[name] = out

    rt_cpp = os.path.join(cpp_dir, "ray_tracing.cpp")
    rt_cu = os.path.join(cu_dir, "ray_tracing_kernel.cu")
    if os.path.exists(rt_cpp) and os.path.exists(rt_cu):
        out_dir = os.path.join(REF_OUT, "raytrace")
        so = os.path.join(out_dir, "ray_tracing_ref.so")
        if force or _stale(so, [rt_cpp, rt_cu]):
            os.makedirs(out_dir, exist_ok=True)
            os.environ["TORCH_CUDA_ARCH_LIST"] = ""   # the -gencode below decides the arch
            try:
                from torch.utils import cpp_extension
                cpp_extension.load(name="ray_tracing_ref", sources=[rt_cpp, rt_cu],
                                   extra_cuda_cflags=["-gencode",
                                                      "arch=compute_100a,code=sm_100a", "-O3"],
                                   extra_cflags=["-O2"], build_directory=out_dir, verbose=False)
            except Exception as e:  # the checker is optional: its tests skip without it
                print("reference ray-marching extension not built: %s" % str(e)[:300])
        if os.path.exists(so):
            built["ray_tracing"] = so
    return built


def main(argv: list[str]) -> int:
    ref_root = None
    if "--ref-root" in argv:
        ref_root = argv[argv.index("--ref-root") + 1]
    force = "--force" in argv
    print("oracle:", build_oracle(force))
    for k, v in build_ref(ref_root, force).items():
        print("reference %s: %s" % (k, v))
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv[1:]))

"""Recipe that compiles the UNMODIFIED reference CUDA sources into oracle/_ref/.

Test infrastructure only.  The reference is read where it lies (never copied
into this repository); the outputs are torch extension modules placed under
oracle/_ref/ (git-ignored, but shipped with the working tree to the GPU host):

  ref_rasterizer_C.so   antialias/cuda_rasterizer/{rasterizer_impl,forward,backward}.cu
                        + antialias/rasterize_points.cu + antialias/ext.cpp
                        (the diff_gaussian_rasterization_wodilate._C module)
  ref_compute_radius_v2.so  FilterGS/cuda/compute_radius_kernel_v2.cu
  ref_gather_attributes.so  FilterGS/cuda/gather_attributes_kernel.cu

The reference's own build system (setup.py / CMake) is not run.  Its sources
carry no architecture flags; the arch here is sm_100 (what
TORCH_CUDA_ARCH_LIST=10.0 produces), the include path is the vendored glm, and
the FilterGS kernels get the -O2 their JIT loaders pass.
"""
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
# The reference checkout: FGS_REFERENCE_ROOT, else a `reference` directory beside this repository.
REF_ROOT = os.environ.get("FGS_REFERENCE_ROOT",
                          os.path.join(os.path.dirname(os.path.dirname(HERE)), "reference"))
OUT = os.path.join(HERE, "_ref")

MODULES = {
    "ref_rasterizer_C": dict(
        sources=["antialias/cuda_rasterizer/rasterizer_impl.cu", "antialias/cuda_rasterizer/forward.cu",
                 "antialias/cuda_rasterizer/backward.cu", "antialias/rasterize_points.cu", "antialias/ext.cpp"],
        cflags=[]),
    "ref_compute_radius_v2": dict(sources=["FilterGS/cuda/compute_radius_kernel_v2.cu"], cflags=["-O2"]),
    "ref_gather_attributes": dict(sources=["FilterGS/cuda/gather_attributes_kernel.cu"], cflags=["-O2"]),
}


def available():
    return os.path.isdir(os.path.join(REF_ROOT, "antialias", "cuda_rasterizer"))


def built(name):
    return os.path.exists(os.path.join(OUT, name + ".so"))


def build(verbose=False, force=False):
    """Compile every reference module that is not built yet.  No-op without the reference tree."""
    if not available():
        return False
    from torch.utils import cpp_extension
    os.makedirs(OUT, exist_ok=True)
    glm = os.path.join(REF_ROOT, "antialias", "third_party", "glm")
    for name, spec in MODULES.items():
        if built(name) and not force:
            continue
        bdir = os.path.join(OUT, "build_" + name)
        os.makedirs(bdir, exist_ok=True)
        srcs = [os.path.join(REF_ROOT, s) for s in spec["sources"]]
        cpp_extension.load(
            name=name, sources=srcs, build_directory=bdir, verbose=verbose,
            extra_include_paths=[glm],
            extra_cuda_cflags=["-gencode=arch=compute_100,code=sm_100"] + spec["cflags"],
            is_python_module=True, with_cuda=True)
        os.replace(os.path.join(bdir, name + ".so"), os.path.join(OUT, name + ".so"))
    return True


def load(name):
    """Import a built reference module from oracle/_ref (None when it is not built)."""
    import importlib.util
    path = os.path.join(OUT, name + ".so")
    if not os.path.exists(path):
        return None
    if name in sys.modules:
        return sys.modules[name]
    import torch  # noqa: F401  (the modules link against torch)
    spec = importlib.util.spec_from_file_location(name, path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    sys.modules[name] = mod
    return mod


if __name__ == "__main__":
    ok = build(verbose="-v" in sys.argv, force="--force" in sys.argv)
    print("reference build:", "done" if ok else "reference tree not present")

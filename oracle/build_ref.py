"""Build recipe for the reference extensions, compiled from their own sources
as checkers (TEST INFRASTRUCTURE ONLY).

Compiles, from the sources of the reference checkout (GSPARC_REFERENCE_ROOT,
default /root/reference; read in place, never copied), with this repository's recipe rather than the reference's setup.py:
  * cuda_kernel_rasterize/{rasterize_points.cu, ext.cpp,
    cuda_wireless_rasterizer/{rasterizer_impl,forward,backward}.cu}
    -> oracle/_ref/raster/gsparc_ref_rasterizer*.so
  * fused-ssim/{ssim.cu, ext.cpp} -> oracle/_ref/ssim/gsparc_ref_fused_ssim*.so

GLM 0.9.9.8, which the rasterizer includes, is not available; the project's
stand-in header oracle/glm_subset/glm/glm.hpp supplies the subset it uses.
oracle/ref_build_prelude.h is force-included to turn glibc's _Float32
constants into plain float literals (nvcc rejects the former in device
code).  Outputs go to oracle/_ref/ only (git-ignored; travels to the GPU box).

Run:  python oracle/build_ref.py     (needs the reference checkout; no GPU needed)
Load: oracle.build_ref.load_ref()    (on a GPU box, from the prebuilt .so)
"""
from __future__ import annotations

import glob
import importlib.util
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
# where the reference checkout lives (read only, never copied)
REF_ROOT = os.environ.get("GSPARC_REFERENCE_ROOT", "/root/reference")
OUT = os.path.join(HERE, "_ref")
ARCH = ["-gencode=arch=compute_100a,code=sm_100a"]


def _sources():
    r = os.path.join(REF_ROOT, "cuda_kernel_rasterize")
    raster = [os.path.join(r, "rasterize_points.cu"), os.path.join(r, "ext.cpp")] + [
        os.path.join(r, "cuda_wireless_rasterizer", f) for f in ("rasterizer_impl.cu", "forward.cu", "backward.cu")]
    s = os.path.join(REF_ROOT, "fused-ssim")
    ssim = [os.path.join(s, "ssim.cu"), os.path.join(s, "ext.cpp")]
    return raster, ssim


def build(verbose: bool = False) -> bool:
    """Compile both reference extensions into oracle/_ref.  Returns False (and
    builds nothing) when the reference sources are absent."""
    raster, ssim = _sources()
    if not all(os.path.exists(p) for p in raster + ssim):
        return False
    from torch.utils.cpp_extension import load
    prelude = os.path.join(HERE, "ref_build_prelude.h")
    glm = os.path.join(HERE, "glm_subset")
    for name, srcs, sub in (("gsparc_ref_rasterizer", raster, "raster"), ("gsparc_ref_fused_ssim", ssim, "ssim")):
        bdir = os.path.join(OUT, sub)
        os.makedirs(bdir, exist_ok=True)
        load(name=name, sources=srcs, build_directory=bdir, verbose=verbose,
             extra_include_paths=[glm, os.path.join(REF_ROOT, "cuda_kernel_rasterize")],
             extra_cflags=["-O3"],
             extra_cuda_cflags=ARCH + ["-O3", "-include", prelude],
             is_python_module=True)
    return True


def _load_so(name, sub):
    cands = glob.glob(os.path.join(OUT, sub, name + "*.so"))
    if not cands:
        return None
    spec = importlib.util.spec_from_file_location(name, cands[0])
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def reference_present() -> bool:
    """Whether the reference checkout's sources are here (only in the build container)."""
    raster, ssim = _sources()
    return all(os.path.exists(p) for p in raster + ssim)


def load_ref():
    """(rasterizer module, fused-ssim module) from the prebuilt .so files, or
    (None, None) if they were not built.  Requires torch to be imported."""
    import torch  # noqa: F401  (the extensions link against libtorch)
    return _load_so("gsparc_ref_rasterizer", "raster"), _load_so("gsparc_ref_fused_ssim", "ssim")


if __name__ == "__main__":
    ok = build(verbose="-v" in sys.argv)
    print("reference extensions built" if ok else "reference sources absent; nothing built")

"""Build libgci.so (CUDA sm_100a kernels + C ABI) in-tree with nvcc.

Run as a script or call ``build()``; objects go to ``_lib/obj``, the shared
library to ``_lib/libgci.so`` and the same objects as a static archive to
``_lib/libgci.a`` next to this file.  Recompiles only sources
newer than their object.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
OUT = HERE / "_lib"
OBJ = OUT / "obj"
LIB = OUT / "libgci.so"
ARCHIVE = OUT / "libgci.a"
CUDA_HOME = Path(os.environ.get("CUDA_HOME", "/usr/local/cuda"))
NVCC = str(CUDA_HOME / "bin" / "nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
          "-I", str(HERE.parent / "include"), "-I", str(CSRC)]
SOURCES = ["eri_kernels.cu", "eri_classes_a.cu", "eri_kf_a.cu", "eri_kf_b.cu", "eri_kf_c.cu", "eri_kf_d.cu",
           "grad_kernels.cu", "grad_pot_a.cu", "grad_pot_b.cu", "grad_pot_c.cu",
           "eri_hm_vectors.cu", "eri_hm_0.cu", "eri_hm_1.cu", "eri_hm_2.cu", "eri_hm_3.cu",
           "eri_hm_4.cu", "eri_hm_5.cu", "eri_hm_6.cu", "chol_kernels.cu", "ozaki_gemm.cu", "dense_fp64.cu", "gci_api.cu", "host_math.cpp"]
# ptxas at -O3 keeps the largest unrolled potential kernels (level sums >= 8)
# entirely in local memory; -O1 allocates registers for them
EXTRA = {"grad_pot_b.cu": ["-Xptxas", "-O1"], "grad_pot_c.cu": ["-Xptxas", "-O1"]}
HEADERS = sorted(CSRC.glob("*.h")) + sorted(CSRC.glob("*.cuh")) + [HERE.parent / "include" / "gci.h"]


def _deps(src: Path, seen=None) -> set:
    """Local headers a source includes, transitively (#include "...")."""
    seen = set() if seen is None else seen
    for line in src.read_text().splitlines():
        line = line.strip()
        if line.startswith("#include \""):
            name = line.split('"')[1]
            for d in (src.parent, CSRC, HERE.parent / "include"):
                h = (d / name).resolve()
                if h.exists():
                    if h not in seen:
                        seen.add(h)
                        _deps(h, seen)
                    break
    return seen


def _stale(src: Path, obj: Path) -> bool:
    if not obj.exists():
        return True
    t = obj.stat().st_mtime
    return src.stat().st_mtime > t or any(h.stat().st_mtime > t for h in _deps(src))


def _compile(src: Path, obj: Path, verbose: bool) -> None:
    cmd = [NVCC, *ARCH, *COMMON, *EXTRA.get(src.name, []), "-c", str(src), "-o", str(obj)]
    if src.suffix == ".cpp":
        cmd = [NVCC, *COMMON, "-x", "c++", "-c", str(src), "-o", str(obj)]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src.name}:\n{r.stdout}\n{r.stderr}")
    if verbose:
        sys.stderr.write(r.stderr)


def build(verbose: bool = False, jobs: int | None = None) -> Path:
    OBJ.mkdir(parents=True, exist_ok=True)
    todo = []
    objs = []
    for s in SOURCES:
        src = CSRC / s
        obj = OBJ / (src.stem + ".o")
        objs.append(obj)
        if _stale(src, obj):
            todo.append((src, obj))
    with cf.ThreadPoolExecutor(max_workers=jobs or os.cpu_count() or 4) as ex:
        for f in [ex.submit(_compile, s, o, verbose) for s, o in todo]:
            f.result()
    if todo or not LIB.exists():
        cmd = [NVCC, *ARCH, "-shared", "-o", str(LIB), *map(str, objs), "-Xlinker", f"-rpath={CUDA_HOME / 'lib64'}"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    if todo or not ARCHIVE.exists():
        # the same objects as a static archive, for a Fortran build that links the
        # library into its own cholesky.a-based executable (the caller adds
        # -lcudart -lstdc++)
        if ARCHIVE.exists():
            ARCHIVE.unlink()
        r = subprocess.run(["ar", "rcs", str(ARCHIVE), *map(str, objs)], capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"ar failed:\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))

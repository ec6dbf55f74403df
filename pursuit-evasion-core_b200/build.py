"""Build libpe_b200.so in-tree for B200 (sm_100a).

    python pursuit-evasion-core_b200/build.py [--verbose-ptxas]

Every csrc/*.cu is compiled by nvcc for `-gencode arch=compute_100a,code=sm_100a`
with -lineinfo and linked into pursuit_evasion_b200/libpe_b200.so next to the
Python package that loads it.  Exact-arithmetic translation units
(*_exact.cu) are compiled with -fmad=false so that no multiply-add is fused:
their results are compared bit for bit with the reference CPU executables.
"""

from __future__ import annotations

import argparse
import concurrent.futures
import hashlib
import os
from pathlib import Path
import shutil
import subprocess
import sys

HERE = Path(__file__).resolve().parent
REPO = HERE.parent
CSRC = HERE / "csrc"
INCLUDE = REPO / "include"
OUT_DIR = HERE / "pursuit_evasion_b200"
LIBRARY = OUT_DIR / "libpe_b200.so"
OBJ_DIR = HERE / "_build"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for candidate in (
        shutil.which("nvcc"),
        "/usr/local/cuda/bin/nvcc",
    ):
        if candidate and Path(candidate).exists():
            return candidate
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build")


def host_compiler() -> str:
    # The system g++ (an environment CXX may point at a reduced toolchain).
    return "/usr/bin/g++" if Path("/usr/bin/g++").exists() else "g++"


def flags_for(source: Path, verbose: bool) -> list[str]:
    flags = [
        "-O3",
        "-std=c++17",
        *ARCH,
        "-lineinfo",
        "-Xcompiler",
        "-fPIC",
        "-ccbin",
        host_compiler(),
        f"-I{INCLUDE}",
        f"-I{CSRC}",
    ]
    if source.name.endswith("_exact.cu"):
        flags.append("-fmad=false")
    if verbose:
        flags += ["-Xptxas", "-v"]
    return flags


def compile_one(source: Path, verbose: bool) -> Path:
    obj = OBJ_DIR / (source.stem + ".o")
    headers = sorted(CSRC.glob("*.cuh")) + sorted(CSRC.glob("*.h"))
    headers += sorted(INCLUDE.glob("*.h"))
    flags = flags_for(source, verbose)
    stamp_text = " ".join(flags) + "".join(
        hashlib.sha256(p.read_bytes()).hexdigest() for p in [source, *headers]
    )
    stamp = OBJ_DIR / (source.stem + ".stamp")
    if (
        not verbose
        and obj.exists()
        and stamp.exists()
        and stamp.read_text() == stamp_text
    ):
        return obj
    cmd = [nvcc(), *flags, "-c", str(source), "-o", str(obj)]
    result = subprocess.run(cmd, capture_output=True, text=True)
    if result.returncode != 0:
        raise RuntimeError(f"nvcc failed for {source.name}:\n{result.stderr}")
    if verbose and result.stderr:
        sys.stderr.write(result.stderr)
    stamp.write_text(stamp_text)
    return obj


def build(verbose: bool = False) -> Path:
    OBJ_DIR.mkdir(exist_ok=True)
    sources = sorted(CSRC.glob("*.cu"))
    workers = min(len(sources), os.cpu_count() or 4)
    with concurrent.futures.ThreadPoolExecutor(workers) as pool:
        objects = list(pool.map(lambda s: compile_one(s, verbose), sources))
    tmp = LIBRARY.with_suffix(".so.tmp")
    cmd = [
        nvcc(),
        *ARCH,
        "-shared",
        "-ccbin",
        host_compiler(),
        "-o",
        str(tmp),
        *map(str, objects),
    ]
    result = subprocess.run(cmd, capture_output=True, text=True)
    if result.returncode != 0:
        raise RuntimeError(f"link failed:\n{result.stderr}")
    os.replace(tmp, LIBRARY)
    return LIBRARY


def main() -> None:
    parser = argparse.ArgumentParser(description=__doc__)
    parser.add_argument("--verbose-ptxas", action="store_true")
    args = parser.parse_args()
    print(build(args.verbose_ptxas))


if __name__ == "__main__":
    main()

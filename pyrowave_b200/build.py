"""Build libpyrowave-shared.so.0 (the C-ABI library) in-tree with nvcc for sm_100a,
and the command-line tools pyrowave-encode / pyrowave-decode against it.

    python -m pyrowave_b200.build [--force]

Objects go to pyrowave_b200/_build/; the library to pyrowave_b200/ with a
libpyrowave-shared.so symlink; the tools to pyrowave_b200/bin/ (they find the
library through their run path). Only pyrowave_* symbols are exported (the
reference's link.T does the same).
"""
from __future__ import annotations

import concurrent.futures
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")
BUILD = os.path.join(HERE, "_build")
SONAME = "libpyrowave-shared.so.0"
LIB = os.path.join(HERE, SONAME)
LINK = os.path.join(HERE, "libpyrowave-shared.so")

SOURCES = ["pw_encode.cu", "pw_decode.cu", "pw_packets.cu", "pw_quality.cu", "pw_analysis.cu", "pw_host.cpp", "pw_server.cpp"]
HEADERS = ["pw_internal.h", "pw_device.cuh", "pw_decode_body.cuh"]
PUBLIC_HEADERS = ["pyrowave.h", "pyrowave_cuda.h", "pyrowave_vk_types.h"]

CLI = os.path.join(HERE, "cli")
BIN = os.path.join(HERE, "bin")
# Tool name -> its main source; every tool also compiles CLI_COMMON.
CLI_TOOLS = {"pyrowave-encode": "pyrowave_encode.cpp", "pyrowave-decode": "pyrowave_decode.cpp"}
CLI_COMMON = ["y4m.cpp", "wave_container.cpp"]
CLI_HEADERS = ["y4m.hpp", "wave_container.hpp"]

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "--fmad=false", "-DPYROWAVE_EXPORT_SYMBOLS",
          "-Xcompiler", "-fPIC,-fvisibility=hidden", "-I", INCLUDE, "-I", CSRC]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _newest(paths):
    return max(os.path.getmtime(p) for p in paths)


def _compile(src: str, verbose: bool) -> str:
    obj = os.path.join(BUILD, src + ".o")
    cmd = [nvcc()] + ARCH + COMMON + ["-c", os.path.join(CSRC, src), "-o", obj]
    if verbose and src.endswith(".cu"):
        cmd += ["-Xptxas", "-v"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    if verbose:
        sys.stderr.write(r.stderr)
    return obj


def cli_sources(tool: str):
    """Source files of one command-line tool (tests build them against other libraries)."""
    return [os.path.join(CLI, f) for f in [CLI_TOOLS[tool]] + CLI_COMMON]


def build_tools(force: bool = False) -> list:
    """Links pyrowave-encode and pyrowave-decode against the in-tree library."""
    cxx = os.environ.get("CXX") or shutil.which("g++") or "g++"
    os.makedirs(BIN, exist_ok=True)
    out = []
    for tool in CLI_TOOLS:
        exe = os.path.join(BIN, tool)
        deps = cli_sources(tool) + [os.path.join(CLI, h) for h in CLI_HEADERS] + [LIB, __file__]
        if force or not os.path.exists(exe) or os.path.getmtime(exe) < _newest(deps):
            cmd = [cxx, "-O2", "-std=c++17", "-Wall", "-I", INCLUDE, "-I", CLI] + cli_sources(tool) + [
                "-o", exe, "-L", HERE, f"-l:{SONAME}", "-Wl,-rpath,$ORIGIN/.."]
            r = subprocess.run(cmd, capture_output=True, text=True)
            if r.returncode != 0:
                raise RuntimeError(f"building {tool} failed:\n{r.stdout}\n{r.stderr}")
        out.append(exe)
    return out


def build(force: bool = False, verbose: bool = False) -> str:
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS] + [os.path.join(INCLUDE, f) for f in PUBLIC_HEADERS]
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= _newest(deps + [__file__]):
        build_tools(force)
        return LIB
    os.makedirs(BUILD, exist_ok=True)
    with concurrent.futures.ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose), SOURCES))
    cmd = [nvcc()] + ARCH + ["-shared", "-o", LIB] + objs + [
        "-cudart", "static",
        "-Xlinker", f"--version-script={os.path.join(CSRC, 'libpyrowave.map')}",
        "-Xlinker", f"-soname={SONAME}",
    ]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    if os.path.lexists(LINK):
        os.remove(LINK)
    os.symlink(SONAME, LINK)
    build_tools(force=True)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))

"""Build the CUDA extension in-tree: ``python -m torchls_b200.build``.

Compiles every ``csrc/*.cu`` for sm_100a with nvcc into
``torchls_b200/libtorchls_b200.so`` (a plain C-ABI shared library; no torch
headers). Objects are cached under ``torchls_b200/_build/`` by source hash.
"""

from __future__ import annotations

import hashlib
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")
OUT = os.path.join(HERE, "libtorchls_b200.so")
BUILD = os.path.join(HERE, "_build")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC",
         "-Xcompiler", "-fvisibility=hidden", "--expt-relaxed-constexpr"]


def _headers_digest():
    h = hashlib.sha256()
    for root in (CSRC, INCLUDE):
        for name in sorted(os.listdir(root)):
            if name.endswith((".cuh", ".h")):
                with open(os.path.join(root, name), "rb") as fh:
                    h.update(name.encode() + fh.read())
    return h.hexdigest()


def build(verbose: bool = False, jobs: int | None = None) -> str:
    os.makedirs(BUILD, exist_ok=True)
    sources = sorted(f for f in os.listdir(CSRC) if f.endswith(".cu"))
    hdr = _headers_digest()
    objs, cmds = [], []
    for src in sources:
        path = os.path.join(CSRC, src)
        with open(path, "rb") as fh:
            digest = hashlib.sha256(fh.read() + hdr.encode() + " ".join(FLAGS + ARCH).encode()).hexdigest()[:16]
        obj = os.path.join(BUILD, f"{src[:-3]}-{digest}.o")
        objs.append(obj)
        if not os.path.exists(obj):
            cmds.append([NVCC, *ARCH, *FLAGS, "-I", INCLUDE, "-I", CSRC, "-c", path, "-o", obj])
    procs = []
    limit = jobs or os.cpu_count() or 4
    for cmd in cmds:
        while len(procs) >= limit:
            _wait(procs.pop(0), verbose)
        if verbose:
            print(" ".join(cmd), flush=True)
        procs.append((cmd, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
    while procs:
        _wait(procs.pop(0), verbose)
    newest = max(os.path.getmtime(o) for o in objs)
    if not os.path.exists(OUT) or os.path.getmtime(OUT) < newest or cmds:
        link = [NVCC, *ARCH, "-shared", "-o", OUT + ".tmp", *objs, "-lcudart"]
        subprocess.run(link, check=True)
        os.replace(OUT + ".tmp", OUT)
    return OUT


def _wait(item, verbose):
    cmd, proc = item
    out, _ = proc.communicate()
    if proc.returncode != 0:
        sys.stderr.write(out.decode())
        raise RuntimeError(f"nvcc failed: {' '.join(cmd)}")
    if verbose and out:
        sys.stderr.write(out.decode())


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))

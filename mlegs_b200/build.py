"""Build libmlegs_b200.so in-tree with nvcc for sm_100a (no JIT, no torch).

Usage: python -m mlegs_b200.build [--verbose]
"""

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libmlegs_b200.so")
SOURCES = ["tables.cu", "kernels.cu", "fft.cu", "gemm.cu", "gemm_dmma.cu", "solve.cu", "phys.cu", "ctx.cu", "solve_static.cu", "split_gemm.cu", "hyperadj.cu", "ensemble.cu", "adjoint.cu", "gemm_bulk.cu"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
FLAGS = ["-std=c++17", "-O3", "-lineinfo", "-gencode", "arch=compute_100a,code=sm_100a",
         "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr"]


def _digest():
    import hashlib
    h = hashlib.sha256()
    for f in sorted(os.listdir(CSRC)):
        h.update(f.encode())
        h.update(open(os.path.join(CSRC, f), "rb").read())
    h.update(open(os.path.join(HERE, "..", "include", "mlegs_b200.h"), "rb").read())
    h.update(" ".join(FLAGS).encode())
    return h.hexdigest()


def _stale():
    """Rebuild only when the sources or flags changed (content hash, not mtimes,
    so a copied tree with a prebuilt library does not recompile)."""
    if not os.path.exists(OUT) or not os.path.exists(OUT + ".sha256"):
        return True
    return open(OUT + ".sha256").read().strip() != _digest()


def build(force=False, verbose=False):
    """Compile every CUDA source and link the shared library; returns its path."""
    if not force and not _stale():
        return OUT
    build_dir = os.path.join(HERE, "_build")
    os.makedirs(build_dir, exist_ok=True)
    jobs = []
    for src in SOURCES:
        path = os.path.join(CSRC, src)
        if not os.path.exists(path):
            continue
        obj = os.path.join(build_dir, src.replace(".cu", ".o"))
        cmd = [NVCC] + FLAGS + (["-Xptxas", "-v"] if verbose else []) + ["-c", path, "-o", obj]
        jobs.append((src, obj, cmd))

    def compile_one(job):
        src, obj, cmd = job
        return src, subprocess.run(cmd, capture_output=True, text=True)

    # one nvcc per source, several at a time (each is single-threaded)
    from concurrent.futures import ThreadPoolExecutor
    with ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as ex:
        results = list(ex.map(compile_one, jobs))
    objs = []
    for (src, r), (_, obj, _) in zip(results, jobs):
        if r.returncode != 0:
            raise RuntimeError("nvcc failed for %s:\n%s" % (src, r.stderr))
        if verbose:
            sys.stderr.write(r.stderr)
        objs.append(obj)
    cmd = [NVCC, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-o", OUT] + objs + ["-lcudart"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("link failed:\n%s" % r.stderr)
    with open(OUT + ".sha256", "w") as fh:
        fh.write(_digest())
    return OUT


if __name__ == "__main__":
    print(build(force=True, verbose="--verbose" in sys.argv))

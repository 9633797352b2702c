"""Build the rs_b200 CUDA library in-tree: reed-solomon_b200/librsb200.so.

nvcc cross-compiles for sm_100a (B200) only; no GPU is needed to build.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "librsb200.so")
SOURCES = ["rs_abi.cu", "rs16_abi.cu", "rs_batch.cu", "mlp.cu", "rs_noalloc.cu", "rs_frame.cu", "rs_queue.cu", "rs_server.cu", "fft16.cu", "fft_k_small.cu", "fft_k16.cu", "fft_k32.cu",
           "fft_k64.cu", "fft_k128.cu", "gen_k.cu", "gen_k_more.cu"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
    "--expt-relaxed-constexpr",
    "-I", os.path.join(ROOT, "include"), "-I", CSRC,
]


def stale():
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    deps.append(os.path.join(ROOT, "include", "rs_b200.h"))
    deps.append(os.path.abspath(__file__))
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=False):
    if not force and not stale():
        return OUT
    from concurrent.futures import ThreadPoolExecutor

    build_dir = os.path.join(HERE, "_build")
    os.makedirs(build_dir, exist_ok=True)
    extra = ["-Xptxas", "-v"] if verbose else []
    objs = [os.path.join(build_dir, src.replace(".cu", ".o")) for src in SOURCES]

    def compile_one(i):
        cmd = [NVCC, *FLAGS, *extra, "-c", os.path.join(CSRC, SOURCES[i]), "-o", objs[i]]
        return subprocess.run(cmd, capture_output=True, text=True)

    # Largest translation units first; one nvcc per core.
    order = sorted(range(len(SOURCES)), key=lambda i: -os.path.getsize(os.path.join(CSRC, SOURCES[i])))
    with ThreadPoolExecutor(max_workers=max(1, min(len(SOURCES), os.cpu_count() or 1))) as ex:
        results = dict(zip(order, ex.map(compile_one, order)))
    for i in range(len(SOURCES)):
        r = results[i]
        if verbose or r.returncode:
            sys.stderr.write(r.stdout + r.stderr)
        if r.returncode:
            raise subprocess.CalledProcessError(r.returncode, "nvcc " + SOURCES[i])
    tmp = OUT + ".tmp"
    subprocess.run([NVCC, "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", tmp, *objs,
                    "-Xcompiler", "-fPIC"], check=True)
    os.replace(tmp, OUT)
    return OUT


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(OUT)

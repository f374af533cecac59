"""Build the B200 backend library in-tree: fainttrail_b200/libft_b200.so.

Every CUDA source is compiled for sm_100a only
(-gencode arch=compute_100a,code=sm_100a) with --fmad=false, so no multiply-add
is ever contracted (the results must round exactly as the reference CPU code,
which is built with -ffp-contract=off). Host C++ goes through the same nvcc
driver. Run: python -m fainttrail_b200.build  (or __graft_entry__.build()).
"""
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libft_b200.so")
ADAPTER_SRC = os.path.join(HERE, "adapter", "b200_backend.cpp")
ADAPTER_LIB = os.path.join(HERE, "adapter", "libft_b200_adapter.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "--fmad=false", "-lineinfo", "-Xcompiler", "-fPIC,-ffp-contract=off",
          "-I" + os.path.join(ROOT, "include"), "-I" + CSRC]


def nvcc():
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cu", ".cpp")))


def _newer(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    return hs + [os.path.join(ROOT, "include", "ft_b200.h")]


def build(verbose=False, ptxas_info=False):
    os.makedirs(OBJ, exist_ok=True)
    cc = nvcc()
    hdrs = _headers()
    jobs = []
    objs = []
    for src in _sources():
        obj = os.path.join(OBJ, os.path.basename(src) + ".o")
        objs.append(obj)
        if _newer(obj, [src] + hdrs) or ptxas_info:
            cmd = [cc] + ARCH + COMMON + ["-c", src, "-o", obj]
            if ptxas_info and src.endswith(".cu"):
                cmd += ["-Xptxas", "-v"]
            jobs.append(cmd)
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        for cmd, res in zip(jobs, ex.map(lambda c: subprocess.run(c, capture_output=True, text=True), jobs)):
            if verbose or ptxas_info:
                sys.stdout.write(res.stdout + res.stderr)
            if res.returncode != 0:
                raise RuntimeError("compile failed: " + " ".join(cmd) + "\n" + res.stdout + res.stderr)
    if _newer(LIB, objs):
        cmd = [cc] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart", "-Xlinker", "-rpath,$ORIGIN"]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError("link failed: " + " ".join(cmd) + "\n" + res.stdout + res.stderr)
    return LIB


def reference_root():
    """The FaintTrail source tree the checkers are built from: $FAINTTRAIL_REF, or
    a `reference` directory beside the repository."""
    return os.environ.get("FAINTTRAIL_REF") or os.path.join(os.path.dirname(ROOT), "reference")


def build_adapter(ref_root=None, ref_lib_dir=None):
    """SearchBackend adapter ("b200") for the reference library. Needs the
    reference headers (only where the reference tree is present) and links
    libft_b200.so; the reference library itself is resolved at load time."""
    ref_root = ref_root or reference_root()
    inc = os.path.join(ref_root, "include")
    if not os.path.isdir(inc) or not os.path.exists(ADAPTER_SRC):
        return None
    deps = [ADAPTER_SRC, LIB, os.path.join(ROOT, "include", "ft_b200.h")]
    if not _newer(ADAPTER_LIB, deps):
        return ADAPTER_LIB
    cmd = ["/usr/bin/g++", "-std=c++17", "-O2", "-fPIC", "-shared", "-ffp-contract=off", "-I" + inc,
           "-I" + os.path.join(ROOT, "include"), ADAPTER_SRC, "-o", ADAPTER_LIB, "-L" + HERE, "-lft_b200",
           "-Wl,-rpath,$ORIGIN/..", "-Wl,--allow-shlib-undefined"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError("adapter build failed:\n" + res.stdout + res.stderr)
    return ADAPTER_LIB


if __name__ == "__main__":
    print(build(verbose=True, ptxas_info="--ptxas" in sys.argv))

"""Build libneat_b200.so (sm_100a) in-tree with nvcc, and the libtorch shim
libneat_torch.so on top of it with g++.

Usage: python -m neat_b200.csrc.build [--verbose-ptxas]

Every .cu file is compiled separately for sm_100a (compute_100a PTX is not
embedded), then linked into neat_b200/libneat_b200.so next to the package.
neat_synth.cu is compiled with --fmad=false so the f64 projector rounds
every operation as written.  neat_b200/shim/neat_torch.cpp (the reference's
libtorch module API in C++) is compiled against the installed torch's
headers and libraries into neat_b200/libneat_torch.so, which finds
libneat_b200.so beside it ($ORIGIN).
"""
import concurrent.futures
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)
ROOT = os.path.dirname(PKG)
OUT = os.path.join(PKG, "libneat_b200.so")
SHIM_OUT = os.path.join(PKG, "libneat_torch.so")
SHIM_DIR = os.path.join(PKG, "shim")
BUILD = os.path.join(ROOT, "_build", "neat_b200")

SOURCES = ["neat_rays.cu", "neat_step.cu", "neat_tc.cu", "neat_image.cu", "neat_igs.cu", "neat_api.cu", "neat_synth.cu",
           "neat_volume.cu", "neat_proposal.cu", "neat_regularizers.cu",
           "neat_structure.cu", "neat_pose.cu", "neat_bwd_rec.cu"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-I" + os.path.join(ROOT, "include"),
          "--expt-relaxed-constexpr"]
PER_FILE = {"neat_synth.cu": ["--fmad=false"]}


def _compile(src, verbose):
    obj = os.path.join(BUILD, src.replace(".cu", ".o"))
    cmd = [NVCC, *ARCH, *COMMON, *PER_FILE.get(src, []), "-c", os.path.join(HERE, src), "-o", obj]
    if verbose:
        cmd += ["-Xptxas", "-v"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    return src, obj, r.returncode, r.stdout + r.stderr


def build(verbose=False):
    out = build_cuda(verbose)
    build_shim()
    return out


def build_cuda(verbose=False):
    os.makedirs(BUILD, exist_ok=True)
    srcs = [os.path.join(HERE, s) for s in SOURCES]
    deps = srcs + [os.path.join(HERE, f) for f in os.listdir(HERE) if f.endswith((".cuh", ".h"))]
    deps.append(os.path.join(ROOT, "include", "neat_b200.h"))
    if os.path.exists(OUT) and not verbose:
        newest = max(os.path.getmtime(p) for p in deps)
        if os.path.getmtime(OUT) >= newest:
            return OUT
    objs, logs, failed = [], [], False
    with concurrent.futures.ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        for src, obj, rc, log in ex.map(lambda s: _compile(s, verbose), SOURCES):
            objs.append(obj)
            if log.strip():
                logs.append(f"--- {src}\n{log}")
            if rc != 0:
                failed = True
    if logs and (failed or verbose):
        sys.stderr.write("\n".join(logs) + "\n")
    if failed:
        raise RuntimeError("nvcc failed")
    tmp = OUT + ".tmp"
    cmd = [NVCC, *ARCH, "-shared", "-o", tmp, *objs, "-lcudart"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("link failed:\n" + r.stdout + r.stderr)
    os.replace(tmp, OUT)
    return OUT


def build_shim():
    """g++ the libtorch shim against the installed torch (its headers, its C++
    ABI flag and its libraries) and libneat_b200.so."""
    import torch
    srcs = [os.path.join(SHIM_DIR, f) for f in ("neat_torch.cpp", "neat_torch.h")]
    deps = srcs + [os.path.join(ROOT, "include", "neat_b200.h"), OUT]
    if os.path.exists(SHIM_OUT) and os.path.getmtime(SHIM_OUT) >= max(os.path.getmtime(p) for p in deps):
        return SHIM_OUT
    tdir = os.path.dirname(torch.__file__)
    cuda_home = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    abi = int(torch._C._GLIBCXX_USE_CXX11_ABI)
    tmp = SHIM_OUT + ".tmp"
    cmd = [os.environ.get("CXX", "g++"), "-O2", "-std=c++17", "-shared", "-fPIC", f"-D_GLIBCXX_USE_CXX11_ABI={abi}",
           "-I" + os.path.join(tdir, "include"), "-I" + os.path.join(tdir, "include", "torch", "csrc", "api", "include"),
           "-I" + os.path.join(cuda_home, "include"), "-I" + os.path.join(ROOT, "include"), "-I" + SHIM_DIR,
           srcs[0], "-o", tmp, "-L" + os.path.join(tdir, "lib"), "-ltorch", "-ltorch_cpu", "-ltorch_cuda", "-lc10",
           "-lc10_cuda", "-L" + PKG, "-lneat_b200", "-Wl,-rpath,$ORIGIN", "-Wl,-rpath," + os.path.join(tdir, "lib")]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("libneat_torch.so build failed:\n" + r.stdout + r.stderr)
    os.replace(tmp, SHIM_OUT)
    return SHIM_OUT


if __name__ == "__main__":
    print(build(verbose="--verbose-ptxas" in sys.argv))

"""In-tree build of the native libraries (no JIT cache, so the .so files travel with the tree).

  libccnn.so        the detection path: CUDA kernels for sm_100a + host runtime + C ABI
  libccnn_synth.so  the seeded synthetic-frame generator used by the benchmark and tests
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

CU_SOURCES = ["capi.cu", "detector.cu", "k_image.cu", "k_stage1.cu", "k_candidates.cu", "k_window.cu", "k_replay.cu", "noalloc.cu", "server.cu", "k_facial.cu", "gate.cu", "synth_device.cu", "k_legacy.cu", "k_peak.cu"]
CPP_SOURCES = ["model.cpp", "convert.cpp"]

# -fmad=false: the kernels must reproduce the reference's uncontracted IEEE single arithmetic.
NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-fmad=false", "-std=c++17",
              "-Xcompiler", "-fPIC,-fvisibility=hidden", "-shared"]


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.check_call(cmd, cwd=HERE)


def build(verbose=False, force=False):
    out = os.path.join(HERE, "libccnn.so")
    srcs = [os.path.join(CSRC, s) for s in CU_SOURCES + CPP_SOURCES]
    deps = srcs + [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh", ".c"))]
    deps += [os.path.join(HERE, "..", "include", f) for f in ("ccnn.h", "ccnn_inspect.h", "ccnn_server.h", "ccnn_gate.h", "ccnn_cnn.h")]
    if force or _stale(out, deps):
        tmp = out + ".tmp"
        if os.path.exists(out):
            os.remove(out)  # a failed build must not leave a stale library behind
        _run([NVCC] + NVCC_FLAGS + ["-o", tmp] + srcs + ["-ldl"], verbose)
        os.replace(tmp, out)
    synth = os.path.join(HERE, "libccnn_synth.so")
    ssrc = [os.path.join(CSRC, f) for f in ("synth_frame.c", "synth_frame.h", "synth_common.h")]
    if force or _stale(synth, ssrc):
        _run(["gcc", "-std=c11", "-O2", "-ffp-contract=off", "-fno-fast-math", "-fPIC", "-shared", "-o", synth, ssrc[0]], verbose)
    return out


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv)

"""Build recipe of the engine's shared library (libctprj.so), in-tree.

Compiles every CUDA source in csrc/ for sm_100a only and links them into
``imgrecsrc_b200/libctprj.so`` (CUDA runtime linked statically), which the
package loads with ctypes.  Run ``python -m imgrecsrc_b200.build``.

Build-time variants (launch shapes and staging choices that were measured
against the default) go to a library of their own, which the package loads
when CTPRJ_LIB names it:

    python -m imgrecsrc_b200.build -D CTPRJ_FWD_STAGE=1 -o imgrecsrc_b200/libctprj_fwdstage.so
"""
import concurrent.futures
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(PKG, "csrc")
OBJ = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libctprj.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O2", "--expt-relaxed-constexpr"]


def nvcc():
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cu"))


def _compile(src, verbose, defines=(), objdir=OBJ, extra=()):
    obj = os.path.join(objdir, os.path.basename(src)[:-3] + ".o")
    deps = [src] + [os.path.join(CSRC, h) for h in os.listdir(CSRC) if h.endswith((".h", ".cuh"))]
    inc = os.path.join(os.path.dirname(PKG), "include")
    deps += [os.path.join(inc, h) for h in os.listdir(inc) if h.endswith(".h")]
    if os.path.exists(obj) and all(os.path.getmtime(obj) >= os.path.getmtime(d) for d in deps):
        return obj, ""
    cmd = [nvcc()] + ARCH + FLAGS + list(extra) + ["-D" + d for d in defines] + \
        (["-Xptxas", "-v"] if verbose else []) + ["-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed for %s:\n%s\n%s" % (src, " ".join(cmd), r.stderr))
    return obj, r.stderr


def build(verbose=False, defines=(), out=LIB, extra=()):
    tag = "_".join([d.replace("=", "") for d in defines] + [f.strip("-").replace("=", "") for f in extra])
    objdir = OBJ if not tag else OBJ + "_" + tag
    os.makedirs(objdir, exist_ok=True)
    with concurrent.futures.ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as ex:
        results = list(ex.map(lambda s: _compile(s, verbose, defines, objdir, extra), sources()))
    objs = [o for o, _ in results]
    if verbose:
        for _, log in results:
            if log:
                sys.stderr.write(log)
    if not os.path.exists(out) or any(os.path.getmtime(o) > os.path.getmtime(out) for o in objs):
        tmp = out + ".tmp"
        cmd = [nvcc()] + ARCH + ["-shared", "-Xcompiler", "-fPIC", "-o", tmp] + objs
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n%s\n%s" % (" ".join(cmd), r.stderr))
        os.replace(tmp, out)
    return out


if __name__ == "__main__":
    import argparse
    ap = argparse.ArgumentParser()
    ap.add_argument("-v", action="store_true", help="ptxas register and spill report")
    ap.add_argument("-D", action="append", default=[], help="preprocessor definition of a variant")
    ap.add_argument("-o", default=LIB, help="output library")
    ap.add_argument("-X", action="append", default=[], help="extra nvcc flag of a variant (e.g. -X=-fmad=false)")
    a = ap.parse_args()
    print(build(verbose=a.v, defines=tuple(a.D), out=os.path.abspath(a.o), extra=tuple(a.X)))

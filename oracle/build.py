"""Build recipe for the oracle (test infrastructure only).

* ``oracle/liboracle.so``: the C restatement in taichi_oracle.c (gcc, OpenMP).
* ``oracle/_ref/libtaichi_ref.so``: the reference's own TaiChi.cu and mmio.cpp,
  compiled unmodified from their sources under the reference checkout named by
  the caller (argument, or $TAICHI_REFERENCE) with the shim headers in
  oracle/ref_shims and the bridge in oracle/ref_bridge.cpp.  Built only where
  the reference sources exist; the built library then travels with the tree.

Run: ``python oracle/build.py [--ref CHECKOUT]`` (TAICHI_REFERENCE=CHECKOUT
works too; with neither, only the C restatement is built).
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
REF_DIR = os.path.join(HERE, "_ref")
REF_LIB = os.path.join(REF_DIR, "libtaichi_ref.so")


def _run(cmd):
    r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if r.returncode != 0:
        raise RuntimeError("command failed: %s\n%s" % (" ".join(cmd), r.stdout))


def _stale(out, deps):
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps)


def build_oracle(force=False):
    src = os.path.join(HERE, "taichi_oracle.c")
    hdr = os.path.join(HERE, "taichi_oracle.h")
    if force or _stale(LIB, [src, hdr, __file__]):
        _run(["gcc", "-O2", "-std=c11", "-fPIC", "-shared", "-fopenmp", "-fno-fast-math",
              "-o", LIB, src, "-lm"])
    return LIB


def build_ref(ref_src=None, force=False):
    """Compile the reference's sources from the checkout `ref_src` (default:
    $TAICHI_REFERENCE); returns the library path, or the one built earlier,
    or None when no checkout is named or it lacks the sources."""
    ref_src = ref_src or os.environ.get("TAICHI_REFERENCE")
    if not ref_src:
        return REF_LIB if os.path.exists(REF_LIB) else None
    taichi_cu = os.path.join(ref_src, "TaiChi.cu")
    mmio = os.path.join(ref_src, "mmio.cpp")
    if not (os.path.exists(taichi_cu) and os.path.exists(mmio)):
        return REF_LIB if os.path.exists(REF_LIB) else None
    bridge = os.path.join(HERE, "ref_bridge.cpp")
    orc = os.path.join(HERE, "taichi_oracle.c")
    deps = [taichi_cu, mmio, bridge, orc, __file__]
    if not (force or _stale(REF_LIB, deps)):
        return REF_LIB
    os.makedirs(REF_DIR, exist_ok=True)
    objd = os.path.join(REF_DIR, "obj")
    os.makedirs(objd, exist_ok=True)
    inc = ["-I", os.path.join(HERE, "ref_shims"), "-I", ref_src, "-I", HERE]
    # No -fopenmp: the shape loop's pragma is ignored, giving the sequential
    # (race-free) order of the reference's partition.
    nv = ["nvcc", "-O2", "-w", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a",
          "-Xcompiler", "-fPIC"]
    objs = []
    for src in (taichi_cu, mmio, bridge):
        obj = os.path.join(objd, os.path.basename(src) + ".o")
        _run(nv + inc + ["-c", src, "-o", obj])
        objs.append(obj)
    oobj = os.path.join(objd, "taichi_oracle.o")
    _run(["gcc", "-O2", "-std=c11", "-fPIC", "-fno-fast-math", "-c", orc, "-o", oobj])
    objs.append(oobj)
    _run(nv + ["-shared", "-o", REF_LIB] + objs + ["-lcudart"])
    return REF_LIB


if __name__ == "__main__":
    print(build_oracle(force=True))
    src = sys.argv[sys.argv.index("--ref") + 1] if "--ref" in sys.argv[:-1] else None
    r = build_ref(src, force=True)
    if r is None and src:
        sys.exit("reference sources (TaiChi.cu, mmio.cpp) not found under %s" % src)
    print(r)

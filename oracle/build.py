#!/usr/bin/env python3
"""oracle/build.py -- TEST INFRASTRUCTURE build recipe.

Builds
  oracle/liboracle.so                  the CPU oracle restatement (always)
  oracle/_ref/<variant>/libref.so      the reference compiled from its own
                                       sources where they lie (only when the
                                       reference tree is present)

Reference variants.  The reference fixes its parameters at compile time in
define.h.  `cfg1*` variants compile every source file in place, unmodified.
The other variants need other values (a smaller solvent count for fast tests,
the 128x64x64 box of the large workload): for them a define.h with those
values substituted is written into oracle/_ref/<variant>/tree/, next to
symbolic links to the reference's own source files (tree/maincode.cpp,
tree/Src/*.cpp, tree/Include).  The compiler resolves `#include "define.h"`
and `#include "../define.h"` against the folder of the link, so the unchanged
sources see the substituted values; nothing is copied.

  replay variants link oracle/ref_replay_rng.cpp (the counter draw stream in
  place of the Mersenne Twister) -> bit-comparable with the oracle;
  timing variants link the reference's own Src/mersenne.cpp, Src/stoc1.cpp
  and Src/userintf.cpp -> the reference's CPU baseline.

Every variant also links oracle/ref_hooks.cpp, which receives main()'s calls
to TotalVA / CollisionStep / llistupdate / sortsolvent_initial1 (renamed with
-D) to snapshot, time and stop the run.  Outputs go only to oracle/_ref/.
"""
import math
import os
import re
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.environ.get("IRBC_REFERENCE_DIR", "/root/reference")
OUT = os.path.join(HERE, "_ref")

CXX = os.environ.get("IRBC_CXX", "g++")  # the system g++ (has libgomp)
REF_FLAGS = ["-c", "-g", "-O3", "-fopenmp", "-fPIC", "-w"]  # makefile:4 plus -fPIC
HOOK_RENAMES = [
    "-Dmain=irbc_ref_main",
    "-DTotalVA=irbc_hook_TotalVA",
    "-DCollisionStep=irbc_hook_CollisionStep",
    "-Dllistupdate=irbc_hook_llistupdate",
    "-Dsortsolvent_initial1=irbc_hook_sortsolvent_initial1",
]


def _alpha(deg):
    r = deg * math.pi / 180.0
    return {"cosalpha": repr(math.cos(r)), "sinalpha": repr(math.sin(r))}


# values substituted into define.h for the generated variants
VARIANTS = {
    "cfg1": dict(replay=True, defines=None),
    "cfg1_timing": dict(replay=False, defines=None),
    "small": dict(replay=True, defines={"Ns": "40000"}),
    # the large workload's membrane (2562-vertex discocyte), angle, dtcd and
    # wall speed in a 32^3 box with a thin solvent, for bit-exact tests
    "disc_small": dict(replay=True, defines=dict(
        Lx="32.0", Ly="32.0", Lz="32.0", Ns="40000", Nt="2562", dtcd="0.025", walls="0.32",
        **_alpha(130.0))),
    "large_timing": dict(replay=False, defines=dict(
        Lx="128.0", Ly="64.0", Lz="64.0", Ns="5242880", Nt="2562", dtcd="0.025",
        walls="0.64", **_alpha(130.0))),
}


def run(cmd, **kw):
    r = subprocess.run(cmd, capture_output=True, text=True, **kw)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise RuntimeError("build step failed: " + cmd[0])
    return r


def newer(target, sources):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources if os.path.exists(s))


def build_oracle():
    src = os.path.join(HERE, "irbc_oracle.cpp")
    out = os.path.join(HERE, "liboracle.so")
    deps = [src, os.path.join(HERE, "irbc_oracle.h"), os.path.join(HERE, "irbc_rng.h")]
    if newer(out, deps):
        run([CXX, "-O2", "-fPIC", "-shared", "-ffp-contract=off", "-std=c++17", src, "-o", out])
    return out


def write_tree(dst_dir, values):
    """define.h with `values` substituted, plus links to the sources."""
    text = open(os.path.join(REF, "define.h")).read()
    for name, val in values.items():
        pat = re.compile(r"^(#define\s+%s\s+)(\S+)" % re.escape(name), re.M)
        text, n = pat.subn(lambda m: m.group(1) + val, text)
        if n != 1:
            raise RuntimeError("define %s not found exactly once" % name)
    tree = os.path.join(dst_dir, "tree")
    os.makedirs(os.path.join(tree, "Src"), exist_ok=True)
    p = os.path.join(tree, "define.h")
    old = open(p).read() if os.path.exists(p) else None
    if old != text:
        with open(p, "w") as f:
            f.write(text)

    def link(src, dst):
        if os.path.islink(dst) and os.readlink(dst) == src:
            return
        if os.path.lexists(dst):
            os.remove(dst)
        os.symlink(src, dst)

    link(os.path.join(REF, "maincode.cpp"), os.path.join(tree, "maincode.cpp"))
    link(os.path.join(REF, "Include"), os.path.join(tree, "Include"))
    for f in os.listdir(os.path.join(REF, "Src")):
        link(os.path.join(REF, "Src", f), os.path.join(tree, "Src", f))
    return tree


def build_variant(name):
    spec = VARIANTS[name]
    d = os.path.join(OUT, name)
    os.makedirs(d, exist_ok=True)
    if spec["defines"] is None:
        root = REF
    else:
        root = write_tree(d, spec["defines"])
    inc = ["-I" + root, "-I" + os.path.join(root, "Include"), "-I" + HERE]
    define_h = os.path.join(root, "define.h")
    srcs = [("maincode", os.path.join(root, "maincode.cpp"), HOOK_RENAMES)]
    for s in ("solfuncs", "memfuncs", "poly34"):
        srcs.append((s, os.path.join(root, "Src", s + ".cpp"), []))
    if not spec["replay"]:
        for s in ("mersenne", "stoc1", "userintf"):
            srcs.append((s, os.path.join(root, "Src", s + ".cpp"), []))
    objs = []
    for stem, path, extra in srcs:
        o = os.path.join(d, stem + ".o")
        if newer(o, [path, define_h, __file__]):
            run([CXX] + REF_FLAGS + extra + inc + [path, "-o", o])
        objs.append(o)
    mine = [os.path.join(HERE, "ref_hooks.cpp")]
    if spec["replay"]:
        mine.append(os.path.join(HERE, "ref_replay_rng.cpp"))
    hdrs = [os.path.join(HERE, h) for h in ("irbc_oracle.h", "irbc_rng.h")]
    for path in mine:
        o = os.path.join(d, os.path.basename(path)[:-4] + ".o")
        if newer(o, [path, define_h] + hdrs):
            run([CXX, "-c", "-O3", "-fopenmp", "-fPIC", "-std=c++17"] + inc + [path, "-o", o])
        objs.append(o)
    lib = os.path.join(d, "libref.so")
    if newer(lib, objs):
        run([CXX, "-shared", "-fopenmp", "-o", lib] + objs)
    return lib


def reference_present():
    return os.path.exists(os.path.join(REF, "maincode.cpp"))


def build_all(variants=None, quiet=False):
    out = {"oracle": build_oracle()}
    if reference_present():
        for v in variants or VARIANTS:
            out[v] = build_variant(v)
    elif not quiet:
        print("reference tree not present: oracle/_ref not rebuilt (prebuilt files are used)")
    return out


if __name__ == "__main__":
    names = sys.argv[1:] or None
    for k, v in build_all(names).items():
        print(k, v)

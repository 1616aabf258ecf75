"""Builds the reference's seven application mains, unchanged, against the
drop-in header gswitch_b200/compat/gswitch.h (the reference sources are
compiled where they lie; nothing of them is copied).  Output:
gswitch_b200/compat/_bin/<app>.

    python -m gswitch_b200.compat.build_apps [reference_root]

(reference_root defaults to $GSW_REFERENCE_TREE).
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
APPS = ("bfs", "cc", "sssp", "pagerank", "bc", "gc", "mbfs")
NVCC = os.environ.get("NVCC", "nvcc")
FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-std=c++17", "--expt-relaxed-constexpr", "-w",
         "-lineinfo", "-I", HERE]


# The reference's applications keep their training hook commented out
# (application/bfs.cu:95: "// fets.record(); // for training"); a user who
# collects training records enables that line.  bfs_record is the reference's
# bfs.cu built that way: the line is enabled in a temporary copy outside the
# repository, which is deleted once compiled.
RECORD_HOOK = "// fets.record(); // for training"


def build_record_variant(ref_root: str, out_dir: str, newest: float, verbose: bool = False) -> str:
    import tempfile

    src = os.path.join(ref_root, "application", "bfs.cu")
    exe = os.path.join(out_dir, "bfs_record")
    if os.path.exists(exe) and os.path.getmtime(exe) >= max(newest, os.path.getmtime(src)):
        return exe
    text = open(src).read()
    if RECORD_HOOK not in text:
        raise RuntimeError("training hook not found in application/bfs.cu")
    with tempfile.TemporaryDirectory() as d:
        tmp = os.path.join(d, "bfs_record.cu")
        with open(tmp, "w") as f:
            f.write(text.replace(RECORD_HOOK, "fets.record();"))
        cmd = [NVCC, *FLAGS, "-o", exe + ".tmp", tmp]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.check_call(cmd)
    os.replace(exe + ".tmp", exe)
    return exe


def build(ref_root: str, verbose: bool = False) -> list[str]:
    out_dir = os.path.join(HERE, "_bin")
    os.makedirs(out_dir, exist_ok=True)
    deps = [os.path.join(HERE, "gswitch.h")]
    for root, _, files in os.walk(os.path.join(os.path.dirname(HERE), "csrc")):
        deps += [os.path.join(root, f) for f in files if f.endswith((".cuh", ".h"))]
    newest = max(os.path.getmtime(d) for d in deps)
    built = []
    for app in APPS:
        src = os.path.join(ref_root, "application", app + ".cu")
        exe = os.path.join(out_dir, app)
        if os.path.exists(exe) and os.path.getmtime(exe) >= max(newest, os.path.getmtime(src)):
            built.append(exe)
            continue
        cmd = [NVCC, *FLAGS, "-o", exe + ".tmp", src]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.check_call(cmd)
        os.replace(exe + ".tmp", exe)
        built.append(exe)
    built.append(build_record_variant(ref_root, out_dir, newest, verbose))
    return built


if __name__ == "__main__":
    from gswitch_b200.compat import reference_tree

    print("\n".join(build(sys.argv[1] if len(sys.argv) > 1 else reference_tree(), verbose=True)))

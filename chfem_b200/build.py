"""Build the chfem_b200 native libraries in-tree for sm_100a (python -m chfem_b200.build)."""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def build(jobs=None, verbose=False):
    cmd = ["make", "-C", os.path.join(HERE, "csrc"), f"-j{jobs or os.cpu_count() or 4}"]
    out = subprocess.run(cmd, capture_output=not verbose, text=True)
    if out.returncode != 0:
        raise RuntimeError("native build failed:\n" + (out.stdout or "") + (out.stderr or ""))


if __name__ == "__main__":
    build(verbose="-v" in sys.argv)
    print("built", os.listdir(os.path.join(HERE, "lib")))

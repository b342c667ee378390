"""Build oracle/_ref/libref_cpu.so from the reference's own CPU sources.

Test infrastructure.  Needs the reference checkout: REFERENCE_DIR, else the
location it has in the build container (/root/reference); where neither is
present it does nothing (a GPU host uses the built file).  Tests locate the
checkout through reference_dir()."""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.environ.get("REFERENCE_DIR", "/root/reference")


def reference_dir():
    """The reference checkout, or None where it is absent."""
    return REF if os.path.isdir(os.path.join(REF, "source")) else None

if __name__ == "__main__":
    if reference_dir() is None:
        print("reference sources not present; skipping", file=sys.stderr)
        sys.exit(0)
    sys.exit(subprocess.call(["make", "-C", HERE, f"REF={REF}"]))

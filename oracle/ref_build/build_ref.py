"""Build oracle/_ref/libref_cpu.so from the reference's own CPU sources
(needs the reference checkout; the GPU box only uses the built file)."""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.environ.get("DNS_REFERENCE_DIR", "/root/reference")

if __name__ == "__main__":
    if not os.path.isdir(REF):
        print("reference sources not present; skipping", file=sys.stderr)
        sys.exit(0)
    sys.exit(subprocess.call(["make", "-C", HERE, f"REF={REF}"]))

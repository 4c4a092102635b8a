"""Regenerate the golden fixtures of tests/golden/ from the reference.

Compiles the reference's hand-written known-answer programs
(tests/system_tests/test_cases/test_<name>.manual.ref.c, where they lie in
the reference tree) with oracle/Makefile's `manual` target, runs each one and
stores its stdout xz-compressed as <name>.txt.xz, plus a manifest of SHA-256
digests. Run it where the reference is present:

    python tests/golden/make_golden.py [--ref /path/to/reference]
"""
import argparse
import hashlib
import json
import lzma
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.abspath(os.path.join(HERE, "..", ".."))
NAMES = ["7-pt", "7-pt-multi-iterations", "7-pt-neumann-cond", "7-pt-periodic",
         "7-pt-double-type", "7-pt-type-mix", "7-pt-int-type", "27-pt", "27-pt-periodic",
         "asymmetric", "asymmetric-periodic", "stencil-hole", "16", "3-pt-1d", "3-pt-periodic",
         "9-pt-2d", "mixed-dim", "mixed-dim2", "mixed-dim3", "redblack", "redblack-periodic",
         "15", "user-defined-type1", "user-defined-type3", "user-defined-type5",
         "user-defined-type-multi-members", "user-defined-type-multi-dim-member"]


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("PHYSIS_REFERENCE", "/root/reference"))
    args = ap.parse_args()
    oracle_dir = os.path.join(ROOT, "oracle")
    targets = ["_ref/manual/%s.exe" % n for n in NAMES]
    subprocess.run(["make", "-s", "-C", oracle_dir, "REF=" + args.ref] + targets, check=True)
    manifest = {}
    for n in NAMES:
        exe = os.path.join(oracle_dir, "_ref", "manual", n + ".exe")
        out = subprocess.run([exe], check=True, capture_output=True).stdout
        with lzma.open(os.path.join(HERE, n + ".txt.xz"), "wb", preset=9) as f:
            f.write(out)
        manifest[n] = {"sha256": hashlib.sha256(out).hexdigest(), "bytes": len(out),
                       "source": "tests/system_tests/test_cases/test_%s.manual.ref.c" % n}
    with open(os.path.join(HERE, "manifest.json"), "w") as f:
        json.dump(manifest, f, indent=1, sort_keys=True)
    print("wrote %d fixtures" % len(NAMES))


if __name__ == "__main__":
    main()

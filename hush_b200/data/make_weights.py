"""Copies the reference's built-in MLP weight blob into the package, byte for byte.

The blob is data (812 little-endian f16 values, layout W1 b1 W2 b2 W3 b3, row-major (out, in)), shipped by the
reference under the MIT licence at src/denoise/hush-weights.bin (also base64 in src/denoise/hush-weights.js:2-23).
It is the only trained artefact of the reference and the default weights of the drop-in ``Hush`` class, so it is
kept bit-identical; the SHA-256 below pins it.

Usage: python hush_b200/data/make_weights.py <path to the reference checkout>
"""
import hashlib
import os
import sys

SHA256 = "728d4cb712ee4bedbf87b12b263de19a0c6318e41b27d57dfbbc6b68388bd0b5"


def main(ref_root: str) -> None:
    src = os.path.join(ref_root, "src", "denoise", "hush-weights.bin")
    blob = open(src, "rb").read()
    if hashlib.sha256(blob).hexdigest() != SHA256:
        raise SystemExit(f"unexpected weight blob at {src}")
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "hush-weights.bin")
    with open(dst, "wb") as f:
        f.write(blob)
    print(f"wrote {dst} ({len(blob)} bytes)")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        raise SystemExit("usage: python hush_b200/data/make_weights.py <path to the reference checkout>")
    main(sys.argv[1])

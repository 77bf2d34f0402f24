"""Regenerates ffbf_b200/csrc/ffbf_sbox.h, the 256-entry S-box table of the rolling hash.

The table is the hash's definition (src/hashes/hash_rot_sbox_pre_2.h:59-124 in efficient/ffbf), so the
device kernels and the oracle must use the same 256 words. This script reads them from a checkout of the
reference and writes them, one word per line with its index, into a header of this project. It is run by
hand when the header needs to be rebuilt; tests compare the committed header with the reference when the
reference is present and with a fixed digest always.

Usage: python oracle/extract_sbox.py /path/to/reference > ffbf_b200/csrc/ffbf_sbox.h
"""
import hashlib
import re
import sys


def read_reference_sbox(ref_root):
    src = open(f"{ref_root}/src/hashes/hash_rot_sbox_pre_2.h").read()
    body = src.split("sbox[] = {", 1)[1].split("};", 1)[0]
    words = [int(x, 16) for x in re.findall(r"0x[0-9a-fA-F]+", body)]
    if len(words) != 256:
        raise SystemExit(f"expected 256 S-box words, found {len(words)}")
    return words


def digest(words):
    return hashlib.sha256(b"".join(w.to_bytes(8, "little") for w in words)).hexdigest()


def main():
    words = read_reference_sbox(sys.argv[1])
    out = [
        "// Generated by oracle/extract_sbox.py. S-box of the 64-bit rotate+S-box rolling hash",
        "// (efficient/ffbf src/hashes/hash_rot_sbox_pre_2.h:59-124). Index = input byte after the",
        "// high-bit mapping of src/rabin-karp/ffbf.cpp:127-130.",
        f"// sha256 of the 256 little-endian words: {digest(words)}",
        "#pragma once",
        "#define FFBF_SBOX_WORDS \\",
    ]
    for i, w in enumerate(words):
        sep = "," if i < 255 else ""
        out.append(f"    0x{w:016x}ull{sep} /* {i:3d} */ \\")
    out.append("")
    print("\n".join(out))


if __name__ == "__main__":
    main()

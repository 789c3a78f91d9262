"""Embed the device headers into the library for runtime kernel compilation.

Writes a C++ fragment with each header's text as a raw string literal and the name
the NVRTC program includes it by.
"""
import re
import sys

HEADERS = [
    ("ml_internal.hpp", "ml_internal.hpp"),
    ("ml_args.hpp", "ml_args.hpp"),
    ("ml_device.cuh", "ml_device.cuh"),
    ("ml_agg.cuh", "ml_agg.cuh"),
    ("../../include/minilake_gpu.h", "../../include/minilake_gpu.h"),
]
# Device code needs only the public header's constants: its host function declarations
# are not valid in an NVRTC program, so that header contributes its enums alone.
ENUMS_ONLY = {"../../include/minilake_gpu.h"}
DELIM = "MLJIT"


def main(out_path):
    parts = []
    for path, name in HEADERS:
        text = open(path).read()
        if path in ENUMS_ONLY:
            text = "#pragma once\n" + "\n".join(re.findall(r"enum\s*\{.*?\};", text, re.S)) + "\n"
        if ")" + DELIM + '"' in text:
            raise SystemExit(f"{path} contains the raw-string delimiter")
        parts.append((name, text))
    with open(out_path, "w") as f:
        f.write("// Generated by embed_headers.py: device headers for runtime compilation.\n")
        f.write(f"static const int kJitHeaderCount = {len(parts)};\n")
        f.write("static const char* const kJitHeaderName[] = {\n")
        for name, _ in parts:
            f.write(f'    "{name}",\n')
        f.write("};\nstatic const char* const kJitHeaderText[] = {\n")
        for _, text in parts:
            f.write(f'    R"{DELIM}({text}){DELIM}",\n')
        f.write("};\n")


if __name__ == "__main__":
    main(sys.argv[1])

"""Run the pipe-rate probe (``csrc/pipe_probe.cu``) on the current CUDA device.

Prints one line per probe: name, operations per SM clock, SM clock in MHz.
The rates size the fold (FP64 multiply/add, 32-bit multiply-high, shared
atomics) and the box sweep (FP32) against the B200's pipes.
"""

from __future__ import annotations

import ctypes
import os
import sys


def main() -> int:
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libbls_probe.so")
    lib = ctypes.CDLL(path)
    lib.bls_probe_pipes.argtypes = [ctypes.c_char_p, ctypes.c_int]
    lib.bls_probe_pipes.restype = ctypes.c_int
    buf = ctypes.create_string_buffer(8192)
    rc = lib.bls_probe_pipes(buf, len(buf))
    sys.stdout.write(buf.value.decode())
    if rc != 0:
        print(f"probe failed: CUDA error {rc}", file=sys.stderr)
    return rc


if __name__ == "__main__":
    raise SystemExit(main())

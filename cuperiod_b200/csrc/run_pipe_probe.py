"""Run the pipe-rate probe (libbls_probe.so, built from pipe_probe.cu by
`make -C cuperiod_b200/csrc probe`) on the current CUDA device and print one line per probe: name,
operations per SM clock for a whole SM, and the SM clock in MHz seen during it.
With ``--fold``: the search kernel's fast fold path alone in three variants
(milliseconds and point-folds per second each).

These rates are the denominators of the engine's SM-pipe roofline (shared-memory
atomics for the fold, FP64 for the phase, FP32 for the box screen)."""

import ctypes
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def main() -> int:
    lib = ctypes.CDLL(os.path.join(HERE, "..", "libbls_probe.so"))
    buf = ctypes.create_string_buffer(16384)
    if "--fold" in sys.argv[1:]:
        # the fold's fast path alone, three variants (bls_probe_fold)
        lib.bls_probe_fold.argtypes = [ctypes.c_char_p, ctypes.c_int]
        lib.bls_probe_fold.restype = ctypes.c_int
        rc = lib.bls_probe_fold(buf, len(buf))
        header = "probe ms point_folds_per_s_1e9"
    else:
        lib.bls_probe_pipes.argtypes = [ctypes.c_char_p, ctypes.c_int]
        lib.bls_probe_pipes.restype = ctypes.c_int
        rc = lib.bls_probe_pipes(buf, len(buf))
        header = "probe ops_per_sm_clock sm_mhz"
    if rc:
        print(f"probe failed: CUDA error {rc}", file=sys.stderr)
        return 1
    print(header)
    print(buf.value.decode(), end="")
    return 0


if __name__ == "__main__":
    sys.exit(main())

"""Measures the LDG.128 L1 hit bandwidth of GPU 0 with liblctprobe.so (the peak the benchmark
quotes the backprojector's on-chip roofline against) and prints it.

    python -m listctrecons_b200.probe.l1_peak
"""
import ctypes as C
import sys


def main() -> int:
    import torch

    from listctrecons_b200 import capi

    torch.cuda.set_device(0)
    gbs, ms = C.c_double(), C.c_double()
    rc = capi.load_probe().lctp_l1_load_gbs(8192, 1, 2, C.byref(gbs), C.byref(ms))
    print(f"rc {rc}  L1 LDG.128 hit bandwidth {gbs.value:.1f} GB/s  ({ms.value:.3f} ms per launch)")
    return rc


if __name__ == "__main__":
    sys.exit(main())

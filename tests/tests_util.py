import ctypes


def cuda_count():
    try:
        lib = ctypes.CDLL("libcudart.so")
    except OSError:
        try:
            import glob
            import os
            cands = glob.glob("/usr/local/cuda/lib64/libcudart.so*")
            lib = ctypes.CDLL(cands[0])
        except Exception:
            return 0
    n = ctypes.c_int(0)
    if lib.cudaGetDeviceCount(ctypes.byref(n)) != 0:
        return 0
    return n.value

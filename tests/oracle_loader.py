"""Loads the oracle (test infrastructure): oracle/liboracle.so, built from oracle/rans_oracle.c
by oracle/Makefile (gcc).  Built on first use if missing or older than its source."""
import ctypes
import os
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_SO = os.path.join(ROOT, "oracle", "liboracle.so")
_lib = None


def oracle_lib():
    global _lib
    if _lib is None:
        src = os.path.join(ROOT, "oracle", "rans_oracle.c")
        if not os.path.exists(ORACLE_SO) or os.path.getmtime(ORACLE_SO) < os.path.getmtime(src):
            subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), ORACLE_SO], check=True,
                           capture_output=True)
        _lib = ctypes.CDLL(ORACLE_SO)
    return _lib

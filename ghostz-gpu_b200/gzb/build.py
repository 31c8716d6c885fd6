"""Compiles libghostz_b200.so (sm_100a) in place with the package Makefile."""
import os
import subprocess

PKG = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(PKG, "libghostz_b200.so")


def build(jobs: int = 8) -> str:
    subprocess.check_call(["make", "-s", "-j", str(jobs), "-C", PKG])
    return LIB

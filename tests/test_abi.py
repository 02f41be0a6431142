"""The C-ABI library loads and exports every function include/mpcd_gpu.h
declares; its ctypes mirror matches the header; no compute call needs a GPU
for these checks."""
import os
import re
import subprocess

import pytest

from mpcd_b200 import abi, gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "mpcd_gpu.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"^\s*int\s+(mpcd_\w+)\s*\(", src, flags=re.M)))


def test_header_declares_the_binding_list():
    assert declared_functions() == sorted(gpu.EXPORTS)


def test_library_exports_every_declared_symbol():
    lib = gpu.load()
    out = subprocess.run(["nm", "-D", "--defined-only", gpu.LIB_PATH],
                         capture_output=True, text=True, check=True).stdout
    exported = set(l.split()[-1] for l in out.splitlines() if " T " in l)
    for name in declared_functions():
        assert name in exported, name
        assert hasattr(lib, name)
    assert lib.mpcd_abi_version() == abi.ABI_VERSION


def test_struct_layout_matches_header():
    # offsets the C compiler gives the header's structs, checked with gcc
    prog = r'''
#include <stdio.h>
#include <stddef.h>
#include "mpcd_gpu.h"
int main(void){
 printf("%zu %zu %zu %zu %zu %zu %zu %zu\n", sizeof(mpcd_config), sizeof(mpcd_wall),
   sizeof(mpcd_species), sizeof(mpcd_status), offsetof(mpcd_config, walls),
   offsetof(mpcd_config, capacity), offsetof(mpcd_wall, inter), offsetof(mpcd_config, seed));
 return 0;}
'''
    tmp = os.path.join(ROOT, "_build")
    os.makedirs(tmp, exist_ok=True)
    src = os.path.join(tmp, "layout.c")
    exe = os.path.join(tmp, "layout")
    open(src, "w").write(prog)
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), src, "-o", exe], check=True)
    got = [int(x) for x in subprocess.run([exe], capture_output=True, text=True,
                                          check=True).stdout.split()]
    import ctypes as C
    want = [C.sizeof(abi.Config), C.sizeof(abi.Wall), C.sizeof(abi.Species),
            C.sizeof(abi.Status), abi.Config.walls.offset, abi.Config.capacity.offset,
            abi.Wall.inter.offset, abi.Config.seed.offset]
    assert got == want


def test_invalid_arguments_are_rejected_without_a_device():
    lib = gpu.load()
    import ctypes as C
    assert lib.mpcd_create(None, None) == abi.ERR_ARG
    assert lib.mpcd_destroy(None) == abi.ERR_ARG
    assert lib.mpcd_step(None, 1, 0) == abi.ERR_ARG
    cfg = abi.Config()
    cfg.dim = 4
    h = C.c_void_p()
    assert lib.mpcd_create(C.byref(cfg), C.byref(h)) == abi.ERR_UNSUPPORTED
